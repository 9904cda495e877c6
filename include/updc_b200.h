/* updc_b200 — B200-native (sm_100a) UPDC iteration engine, C ABI.
 *
 * Drop-in boundary for the reference engine handoff: updc/_engine.py execs
 * the frozen core with 18 positional arguments (updc/_engine.py:1381-1390),
 * whose entry point is UPDC_ALL (updc/c_core/updc_core.c:1289-1293).  This
 * library exports that entry point unchanged plus a handle API with status
 * returns, so Python (ctypes) and C callers can drive the same solver without
 * a process boundary.  All functions returning int give 0 on success and a
 * non-zero status on failure; updc_last_error() then holds the message the
 * reference core would have printed after "UPDC_ALL: ".  No function of this
 * library calls exit(), except UPDC_ALL, which keeps the reference's
 * behaviour (message on stderr, exit status 1).
 */
#ifndef UPDC_B200_H
#define UPDC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Precision forms.  FP32: FP32 FFTs, gathers and ratios with FP64 PSF
 * normalisation sum, FP64 one-time denominator and FP64 cross-exposure
 * frequency-domain accumulation.  FP64: everything in double.  FP32_KAHAN:
 * FP32 with Kahan-compensated cross-exposure sums.  FP32_REFERENCE: the
 * reference core's precision choices (all FP32, plain sums, Neumaier FP32
 * PSF sum, plain fmaf raw_mu). */
enum { UPDC_FORM_FP32 = 0, UPDC_FORM_FP64 = 1, UPDC_FORM_FP32_KAHAN = 2, UPDC_FORM_FP32_REFERENCE = 3 };

/* Planes readable with updc_read_plane / writable with updc_write_plane. */
enum {
    UPDC_PLANE_ESTIMATE = 0, UPDC_PLANE_COVERAGE = 1, UPDC_PLANE_DENOMINATOR = 2, UPDC_PLANE_CORRECTION = 3,
    UPDC_PLANE_BLUR = 4, UPDC_PLANE_SCATTER = 5, UPDC_PLANE_SCIENCE = 6, UPDC_PLANE_WEIGHT = 7,
    UPDC_PLANE_WR = 8, UPDC_PLANE_FROZEN = 9
};

typedef struct updc_engine updc_engine;

typedef struct {
    int form;            /* UPDC_FORM_* */
    int compensated_mu;  /* -1: form default (on for FP32/FP32_KAHAN) */
    int use_graph;       /* capture each iteration as one CUDA graph */
    int device;          /* CUDA device ordinal */
    int reuse_links;     /* reuse a valid <vertices>.links file instead of rebuilding */
    int verbose;
    int fft_width;       /* 0: smallest even 7-smooth >= the minimum width (see fft_linear) */
    int fft_height;      /* 0: smallest 7-smooth >= the minimum height (see fft_linear) */
    int stage_timing;    /* per-stage CUDA-event timing (disables the graph) */
    int autotune;        /* time candidate FFT shapes and radix splits on the device at setup
                            (select_fft_shape, updc_core.c:242-291) */
    int retune;          /* ignore a cached autotune choice */
    const char *tune_cache_dir; /* directory of the autotune cache; NULL or "" = none */
    int fft_linear;      /* minimum FFT lengths: 1 = W + pw - 1, H + ph - 1, the full linear
                            convolution (updc_core.c:1335-1341); 0 (default) = W + pw/2, H + ph/2:
                            only the W x H window of each circular convolution is kept, and with
                            the PSF centred at offset -pw/2 (updc_core.c:814-819) that window is
                            already exactly the linear convolution's at this length */
} updc_options;

typedef struct {
    double seconds;          /* device time of the iteration */
    double signed_sum;       /* sum of the updated estimate */
    uint64_t negative;       /* negative pixels of the updated estimate */
    double stage_seconds[8]; /* with stage_timing: estimate x-pass, forward y-passes, forward x-pass,
                                detector, adjoint gather, scatter x-pass, adjoint y/x-passes, update */
} updc_iter_stats;

const char *updc_version(void);
/* Message of the last failure in this thread ("" when none). */
const char *updc_last_error(void);
void updc_default_options(updc_options *opt);

/* Handle lifecycle. Replaces the file-scope state of updc_core.c:91-107. */
int updc_create(const updc_options *opt, updc_engine **out);
int updc_destroy(updc_engine *h);

/* Manifest parse, updc_core.c:426-461 (same 8-field TSV and checks). */
int updc_load_manifest(updc_engine *h, const char *manifest, int width, int height, int input_width,
                       int input_height, int exposures, int psf_transposed);
/* Everything before the iteration loop, updc_core.c:1330-1398: FFT shape,
 * LinkMaps (read, or built on the GPU), SCI/WHT planes and weight
 * normalisation, PSF spectra, initial drizzle estimate, denominator. */
int updc_setup(updc_engine *h);
/* n iterations of updc_core.c:1410-1456.  stats (n entries) and the
 * per-exposure FreezeMu arrays (n * exposures entries) may be NULL.
 * check_each = 1 synchronises after every iteration (errors stop there). */
int updc_iterate(updc_engine *h, int n, int check_each, updc_iter_stats *stats, uint64_t *new_frozen,
                 uint64_t *total_frozen, double *min_raw_mu);
/* Copy a plane to host memory (float32, or float64 when as_double) / from host memory. */
int updc_read_plane(updc_engine *h, int which, int exposure, void *host, int as_double);
int updc_write_plane(updc_engine *h, int which, int exposure, const void *host, int as_double);
/* Scalars: 0 weight_scale, 1 max_sensitivity, 2 FFT width, 3 FFT height, 4 masked pixels,
 * 5 working precision bits, 6 compensated raw_mu flag, 7 FFT autotune seconds,
 * 8 FFT plans timed by the autotuner, 9 autotune cache hit, 10 modelled spectral
 * ms per iteration of the tuned choice, 11 kernel variants of the iteration as
 * bits (1: row transforms compiled for their radix sequence, 2: column
 * transforms likewise, 4: adjoint gather fused into the scatter row transform,
 * 8: rows longer than one block, four-step, 16: columns likewise, 32: FP32
 * rows of more than half a block in two-row tiles of 1024 threads). */
double updc_scalar(updc_engine *h, int which);
/* Radix split of an FFT axis (0: the row transform of FW/2 points, 1: the
 * column transform of FH points) in stage order; *count receives the number
 * of stages (at most `capacity` are written). */
int updc_fft_radices(updc_engine *h, int axis, int *radices, int capacity, int *count);
/* Per-stage CUDA-event timing of the following iterations (on: eager launches, no graph). */
int updc_set_stage_timing(updc_engine *h, int on);
size_t updc_device_bytes(updc_engine *h);

/* Stage hooks (parity checks of single kernels):
 *   forward:    blur_k = crop(C2R(R2C(pad(x)) * K_k))/nf for every exposure (updc_core.c:745-776)
 *   detector:   the fused detector loop + transposed adjoint gather on the current blur planes
 *               (updc_core.c:1152-1177), FreezeMu counters per exposure
 *   correction: C = crop(C2R(sum_k conj(K_k) R2C(pad(scatter_k))))/nf (updc_core.c:1181-1183, 1280-1287)
 *   update:     x *= C/D with the reference's guards (updc_core.c:1437-1456) */
int updc_stage_forward(updc_engine *h);
int updc_stage_detector(updc_engine *h, uint64_t *new_frozen, uint64_t *total_frozen, double *min_raw_mu);
int updc_stage_correction(updc_engine *h);
int updc_stage_update(updc_engine *h, double *signed_sum, uint64_t *negative);

/* The update x *= C/D (updc_stage_update's kernels and grid) on caller-owned
 * FP32 device planes of n pixels, for callers that may not allocate device
 * memory at this point: an allocator-managed pool, a real-time or
 * memory-capped host process, a caller holding its own memory pool.  No
 * counterpart in the reference, whose update is a host loop on its own
 * buffers (updc_core.c:1437-1456).
 *   - allocates nothing: no cudaMalloc/cudaFree, no allocating library call;
 *     its scratch is one file-scope __device__ array of
 *     UPDC_UPDATE_NOALLOC_SCRATCH_BYTES bytes per device;
 *   - the first call on each device looks the scratch up with
 *     cudaGetSymbolAddress, and so does the first call after the device's
 *     context changed (cudaDeviceReset); make those calls before any stream
 *     capture begins on the device;
 *   - nothing in the scratch has to start at zero: each call first sets the
 *     error record to "none", and every partial slot is written before it is
 *     read;
 *   - the scratch is shared by every call on a device, so calls that overlap
 *     in time (other streams or threads) race; order them on one stream or
 *     serialise them on the host;
 *   - n must be 1 .. UPDC_UPDATE_NOALLOC_MAX_PIXELS (the width of the device
 *     error record's pixel index); other sizes return status 1 with a message;
 *   - runs on the current device and on `stream` (a cudaStream_t; NULL for the
 *     legacy default stream), waits for it, and returns the signed sum and the
 *     negative count of the updated estimate, or the reference's failure
 *     message through updc_last_error(). */
#define UPDC_UPDATE_NOALLOC_SCRATCH_BYTES ((size_t)(16 * 148 * 16 + 24))
#define UPDC_UPDATE_NOALLOC_MAX_PIXELS ((uint64_t)1 << 40)
int updc_update_noalloc(const float *correction, const float *denominator, float *estimate, uint64_t n,
                        float max_sensitivity, void *stream, double *signed_sum, uint64_t *negative);

/* Differentiable model (no reference counterpart; the gradient of the
 * weighted Poisson negative log-likelihood whose multiplicative update the
 * reference runs, updc_core.c:1140-1183, 1437-1456):
 *   mu_k = S_k P_k x + background_k + pedestal_k,  y_k = SCI_k + pedestal_k,
 *   L = sum_k sum_p W_kp (mu_kp - y_kp log mu_kp)  over pixels with W > 0, mu > 0.
 * updc_set_exposure_offsets / updc_set_psf replace one exposure's background
 * and pedestal, or its PSF (FP32, or FP64 with as_double, manifest layout, no
 * larger than the PSF the FFT shape was chosen for; normalised by its sum
 * like core:777-843).
 * updc_nll runs the forward model of the current estimate and writes per
 * exposure 4 doubles {L_k, sum r, sum W log mu, pixels left out} with
 * r = W (1 - y/mu) kept in the WR planes; updc_nll_adjoint then leaves
 * dL/dx = sum_k H_k^T r_k in the CORRECTION plane; updc_psf_gradient gives
 * dL/dpsi for the normalised PSF of one exposure (psf_width x psf_height
 * doubles, PSF layout).  updc_copy_plane_device copies a plane to or from
 * caller device memory (to_engine = 1 writes the plane) after `stream`. */
int updc_set_exposure_offsets(updc_engine *h, int exposure, double background, double pedestal);
int updc_set_psf(updc_engine *h, int exposure, const void *psf, int psf_width, int psf_height, int as_double);
int updc_nll(updc_engine *h, double *terms);
/* The FP64 per-block partial sums behind the last updc_nll (exposures x
 * blocks x 4, the terms' order); *count receives their number.  Differences
 * of two evaluations taken partial by partial are exact where nothing
 * changed (finite differences of single pixels). */
int updc_nll_partials(updc_engine *h, double *out, size_t capacity, size_t *count);
int updc_nll_adjoint(updc_engine *h);
int updc_psf_gradient(updc_engine *h, int exposure, double *out);
int updc_copy_plane_device(updc_engine *h, int which, int exposure, void *device_ptr, int to_engine, int as_double,
                           void *stream);

/* Exposure shards (multi-GPU solve of one field; no reference counterpart,
 * the reference runs one process): after updc_setup on the whole field,
 * iterate only exposures [first, first + count).  A rank then runs
 * updc_stage_forward / _detector / _correction for its shard, sums the
 * CORRECTION plane over ranks (the one exchange of the iteration,
 * updc_core.c:1280-1287 split by exposure), writes it back and runs
 * updc_stage_update.  updc_refresh_sensitivity recomputes max_sensitivity
 * after the DENOMINATOR plane was replaced. */
int updc_set_active_exposures(updc_engine *h, int first, int count);
int updc_refresh_sensitivity(updc_engine *h);
/* Shard setup (no reference counterpart): updc_set_active_exposures called
 * between updc_load_manifest and updc_setup sets the shard up alone — only
 * its exposures' LinkMaps and PSF spectra are built — and updc_setup leaves
 * partial planes: COVERAGE, ESTIMATE (the drizzle's data sum), CORRECTION
 * (its background sum) and DENOMINATOR, each over the shard's exposures.  The
 * caller sums each of the four over the shards in place (e.g. NCCL
 * all-reduce through updc_plane_device_pointer) and calls
 * updc_finish_shard_setup, which forms the drizzle estimate and the maximum
 * sensitivity; iterations are refused until then.  Results equal the whole
 * field's up to the order of the cross-shard sums. */
int updc_finish_shard_setup(updc_engine *h);
/* The same exchange without host round trips (no reference counterpart):
 * updc_plane_device_pointer gives the engine's own device address of a
 * target plane (ESTIMATE, COVERAGE, DENOMINATOR or CORRECTION: W x H
 * elements of the form's precision, row-major; valid until updc_destroy) and
 * updc_engine_stream the CUDA stream every launch of the engine is issued on
 * (a cudaStream_t).  updc_enqueue_partial enqueues, without waiting, the
 * partial correction of the active exposures into the CORRECTION plane;
 * updc_enqueue_update enqueues the update from the CORRECTION plane as it
 * stands.  A rank sums the CORRECTION plane over ranks in place on the
 * engine's stream between the two (e.g. an NCCL all-reduce), so the three
 * steps can also be captured in one CUDA graph.  updc_finish_iteration waits
 * for the stream, reports a device error recorded by either half like
 * updc_iterate, and returns the update's signed sum and negative count and
 * the per-exposure FreezeMu counters (arrays of `exposures` entries; NULL
 * skips). */
int updc_plane_device_pointer(updc_engine *h, int which, void **device_ptr);
int updc_engine_stream(updc_engine *h, void **stream);
int updc_enqueue_partial(updc_engine *h);
int updc_enqueue_update(updc_engine *h);
int updc_finish_iteration(updc_engine *h, double *signed_sum, uint64_t *negative, uint64_t *new_frozen,
                          uint64_t *total_frozen, double *min_raw_mu);

/* Checkpoint / resume (no reference counterpart: the reference writes the
 * estimate only, core:1460-1470).  updc_save_state writes the estimate and the
 * persistent FreezeMu masks with an iteration count; updc_load_state, on an
 * engine set up from the same manifest and form, restores them, so the next
 * iterations continue the saved run exactly. */
int updc_save_state(updc_engine *h, const char *path, uint64_t iteration);
int updc_load_state(updc_engine *h, const char *path, uint64_t *iteration);

/* LinkMap v2 (updc_core.c:40-79, 463-496, 530-609, 645-662). */
uint64_t updc_link_count(updc_engine *h, int exposure);
int updc_link_encoding(updc_engine *h, int exposure);
/* Absolute target of every link of an exposure, decoded on the GPU (link_target_at, updc_core.c:76-78). */
int updc_decode_links(updc_engine *h, int exposure, uint32_t *targets);
/* Build a LinkMap file from a vertex map on the GPU (AreaLinkList_O2TAD_stream, updc_core.c:530-609). */
int updc_build_linkmap(const char *vertices_path, const char *links_path, int input_width, int input_height,
                       int width, int height, uint64_t *nlinks, int *encoding);

/* Batched fields (no reference counterpart: the reference solves one field
 * per process).  Many independent fields of uneven grid size and exposure
 * count, each with its own manifest, FFT shape (autotuned when opt->autotune)
 * and LinkMaps, iterate together: every stage of an iteration is one
 * persistent launch over the work units of all fields, and n iterations
 * without per-iteration checks run as one CUDA graph.  Each field computes
 * exactly what its own engine computes (updc_core.c:1410-1456 per field).
 * updc_batch_iterate fills, per iteration i, seconds[i] (device time of the
 * whole batch), signed_sum/negative[i * fields + f] and
 * total_frozen[i * E + e] (E = all exposures, fields in order); any may be
 * NULL.  updc_batch_field returns a handle owned by the batch for the plane
 * and scalar queries of one field (do not destroy it). */
typedef struct updc_batch updc_batch;
int updc_batch_create(const updc_options *opt, updc_batch **out);
int updc_batch_destroy(updc_batch *b);
int updc_batch_add_field(updc_batch *b, const char *manifest, int width, int height, int input_width,
                         int input_height, int exposures, int psf_transposed);
int updc_batch_setup(updc_batch *b);
int updc_batch_fields(updc_batch *b);
updc_engine *updc_batch_field(updc_batch *b, int field);
/* Work units of a stage (0 estimate rows, 1 columns, 2 forward rows, 3 detector,
 * 4 adjoint gather, 5 scatter rows, 6 update, 7 adjoint rows). */
size_t updc_batch_units(updc_batch *b, int stage);
int updc_batch_iterate(updc_batch *b, int n, int check_each, double *seconds, double *signed_sum, uint64_t *negative,
                       uint64_t *total_frozen);

/* PSF projection (psf_projector.c:82-172) on the GPU: input PSF (raw f32,
 * width x height) and its (width+1) x (height+1) mapped corner offsets (raw
 * f64 x,y pairs) -> projected PSF (raw f32, out_width x out_height, the
 * symmetric extent of the mapped corners), bit-identical to the reference
 * projector.  Returns 0, 1 with the reference's message, or 2 when the
 * projection is not flux-conserving (|rel| > 5e-5; the sums are filled). */
int updc_psf_project_file(const char *input, int width, int height, const char *vertices, const char *output,
                          int *out_width, int *out_height, double *input_sum, double *output_sum, uint64_t *overlaps,
                          char *message, size_t capacity);

/* Per-exposure weight preprocessing on the GPU: the numeric part of the
 * reference's Level-2 preparation, prepare_weighted_inputs.prepare_one
 * (updc/_engine.py:349-397) with robust_background_mask (_engine.py:287-310)
 * and build_weight (_engine.py:313-333), results identical to the reference's
 * NumPy code.  Reading the FITS planes stays with the caller (the reference
 * reads SCI, DQ, VAR_POISSON, VAR_RNOISE, VAR_FLAT with astropy).
 *
 * Status: 0; 1 with the reference's ValueError message in updc_last_error()
 * ("Too few valid pixels for robust background estimation", "Cannot estimate
 * a positive background RMS", "Cannot estimate sky VAR_POISSON", "No usable
 * pixels remain in <source>", "Automatic pedestal failed to make y_eff
 * positive in <source>"); 3 for an unknown weight mode, raised where the
 * reference raises ValueError(mode), after the sky VAR_POISSON median; -2
 * CUDA failure.  With device_pointers = 0 the planes are host arrays
 * (copied in and out on `stream`); with 1 they are device pointers used on
 * `stream` (a cudaStream_t; NULL = the legacy default stream). */
enum { UPDC_WEIGHT_MASK = 0, UPDC_WEIGHT_RNOISE_SKY = 1, UPDC_WEIGHT_TOTALVAR = 2 };

typedef struct updc_preprocess_metrics {
    /* the metric record of _engine.py:387-398 */
    double background;               /* sigma-clipped median of SCI */
    double background_sigma;         /* 1.4826 x MAD of the clipped SCI */
    double poisson_pedestal;         /* max(auto, requested) */
    double auto_positivity_pedestal;
    double requested_pedestal;
    double min_valid_science;
    double sky_var_poisson;          /* median VAR_POISSON over the sky mask */
    double wht_valid_median;         /* median of the positive WHT values */
    int64_t base_invalid;
    int64_t nonpositive_valid_before_pedestal;
    int64_t nonpositive_after_pedestal;
    int64_t wht_zero;
    /* diagnostics with no reference counterpart */
    int32_t clip_passes;             /* clipping passes run (at most 6) */
    int32_t std_fallbacks;           /* passes whose MAD was zero (standard deviation used) */
} updc_preprocess_metrics;

/* prepare_one's numeric steps for one exposure of npix pixels: WHT (float32,
 * zero where unusable) to `wht`, the final sky mask (0/1) to `sky_mask` when
 * not NULL, and the metrics.  `source` names the exposure in the messages. */
int updc_preprocess_exposure(const float *science, const uint32_t *dq, const double *var_poisson,
                             const double *var_rnoise, const double *var_flat, int64_t npix, int weight_mode,
                             uint32_t bad_dq_mask, double pedestal_sigma, const char *source, float *wht,
                             uint8_t *sky_mask, updc_preprocess_metrics *metrics, int device_pointers, void *stream);

/* robust_background_mask (_engine.py:287-310): asymmetric sigma clipping of
 * SCI over base_valid (0/1 bytes), at most max_iter passes; the final mask
 * (0/1) to `mask`, the background and sigma of its last step. */
int updc_robust_background(const float *science, const uint8_t *base_valid, int64_t npix, int max_iter,
                           uint8_t *mask, double *background, double *sigma, int *passes, int device_pointers,
                           void *stream);

/* Geometry (overlap.c:72-116) and the known-answer self-test (updc_core.c:1545-1564). */
float updc_polygon_area(const double *xy, int count);
float updc_overlap_area(const double *quad8, int x, int y);
int updc_self_test(char *message, size_t capacity);
/* Device-side failure detection check (no reference counterpart): runs, on
 * the current device, a bounded mbarrier wait that nothing completes (no copy
 * is issued), polled at most `polls` times per thread.  It returns status 1
 * with updc_last_error() = "device wait timed out" once the wait ran out and
 * the kernel returned (the path a stuck TMA tile of the row transforms
 * takes); the context stays usable. */
int updc_device_wait_check(uint32_t polls);

/* The 18-argument solve with status return (no exit): writes <prefix>_NN.bin,
 * <prefix>_mufreeze.csv, <prefix>_timing.csv and the WHT file exactly where the
 * reference core does.  Honours UPDC_PERSIST_CACHE like updc_core.c:1319. */
int updc_all(const char *manifest, int width, int height, int input_width, int input_height, int exposures,
             int transpose_psf, int iterations, const char *iter_prefix, const char *weight_output,
             int fft_worker_count, int exposure_worker_count, int preprocess_worker_count, int plan_measure,
             int autotune, int retune_fft, const char *wisdom_path, int save_every);

/* Reference-compatible entry point, updc_core.c:1289-1293: on failure prints
 * "UPDC_ALL: <message>" to stderr and exits with status 1. */
void UPDC_ALL(const char *manifest, int width, int height, int input_width, int input_height, int exposures,
              int transpose_psf, int iterations, const char *iter_prefix, const char *weight_output,
              int fft_worker_count, int exposure_worker_count, int preprocess_worker_count, int plan_measure,
              int autotune, int retune_fft, const char *wisdom_path, int save_every_arg);

#ifdef __cplusplus
}
#endif

#endif
