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
    int fft_width;       /* 0: smallest even 7-smooth >= W + pw - 1 */
    int fft_height;      /* 0: smallest 7-smooth >= H + ph - 1 */
    int stage_timing;    /* per-stage CUDA-event timing (disables the graph) */
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
 * 5 working precision bits, 6 compensated raw_mu flag. */
double updc_scalar(updc_engine *h, int which);
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
 *     cudaGetSymbolAddress; make that first call before any stream capture
 *     begins on the device;
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

/* LinkMap v2 (updc_core.c:40-79, 463-496, 530-609, 645-662). */
uint64_t updc_link_count(updc_engine *h, int exposure);
int updc_link_encoding(updc_engine *h, int exposure);
/* Absolute target of every link of an exposure, decoded on the GPU (link_target_at, updc_core.c:76-78). */
int updc_decode_links(updc_engine *h, int exposure, uint32_t *targets);
/* Build a LinkMap file from a vertex map on the GPU (AreaLinkList_O2TAD_stream, updc_core.c:530-609). */
int updc_build_linkmap(const char *vertices_path, const char *links_path, int input_width, int input_height,
                       int width, int height, uint64_t *nlinks, int *encoding);

/* Geometry (overlap.c:72-116) and the known-answer self-test (updc_core.c:1545-1564). */
float updc_polygon_area(const double *xy, int count);
float updc_overlap_area(const double *quad8, int x, int y);
int updc_self_test(char *message, size_t capacity);

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
