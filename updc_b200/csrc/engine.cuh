// Host orchestration of the UPDC solver on one B200: the B200-native
// replacement for UPDC_ALL (updc/c_core/updc_core.c:1289-1543).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "fft.cuh"

namespace updc {

enum Form { FORM_FP32 = 0, FORM_FP64 = 1, FORM_FP32_KAHAN = 2, FORM_FP32_REFERENCE = 3 };

struct EngineOptions {
    int form = FORM_FP32;
    int compensated_mu = -1;  // -1: the form's default
    int use_graph = 1;
    int device = 0;
    int reuse_links = 1;      // reuse a valid LinkMap file instead of rebuilding it
    int verbose = 0;
    int fft_width = 0;        // 0: smallest even 7-smooth width >= the minimum of the length rule
    int fft_height = 0;       // 0: smallest 7-smooth height >= the minimum of the length rule
    int stage_timing = 0;     // time each stage with events (no graph)
    int autotune = 0;         // time candidate FFT shapes and radix splits on the device
    int retune = 0;           // ignore a cached autotune result
    std::string tune_cache_dir;  // directory of the autotune cache ("" = no cache)
    int fft_linear = 0;       // 1: minimum lengths W + pw - 1, H + ph - 1 (the reference's rule);
                              // 0: W + pw/2, H + ph/2 (the kept window is exactly the same)
};

// Outcome of the FFT autotuner (or of the fixed choice without it).
struct FftChoice {
    int width = 0, height = 0;
    std::vector<int> row_radices, col_radices;
    double predicted_ms = 0;  // modelled spectral time per iteration
    int candidates = 0;       // plans timed (0: fixed choice or cache hit)
    bool cache_hit = false;
    double seconds = 0;       // wall time of the tuning
};

struct ExposureInput {
    std::string science, weight, psf, vertices, links;
    int psf_width = 0, psf_height = 0;
    double background = 0, pedestal = 0;      // as parsed in double
    float backgroundf = 0, pedestalf = 0;     // as parsed by strtof (updc_core.c:447-448)
};

struct IterationRecord {
    double seconds = 0;       // device time of the whole iteration
    double stage_seconds[8] = {};
    double signed_sum = 0;
    uint64_t negative = 0;
    std::vector<uint64_t> new_frozen, total_frozen;
    std::vector<double> min_raw_mu;
};

// Planes that can be read back.
enum Plane { PLANE_ESTIMATE = 0, PLANE_COVERAGE = 1, PLANE_DENOMINATOR = 2, PLANE_CORRECTION = 3, PLANE_BLUR = 4,
             PLANE_SCATTER = 5, PLANE_SCIENCE = 6, PLANE_WEIGHT = 7, PLANE_WR = 8, PLANE_FROZEN = 9 };

class Engine {
  public:
    virtual ~Engine() = default;
    // Parses the manifest (updc_core.c:426-461).
    virtual void load(const std::string &manifest, int W, int H, int iw, int ih, int nexp, int psf_transposed) = 0;
    // FFT shape, PSF spectra, LinkMaps, planes, weight scale, drizzle, denominator.
    virtual void setup() = 0;
    // Runs n iterations; records are appended (one per iteration).
    virtual void iterate(int n, bool check_each, std::vector<IterationRecord> *records) = 0;
    // Copies a plane to host memory as float (as_double=0) or double.
    virtual void read_plane(int which, int k, void *host, int as_double) = 0;
    // Writes a plane from host memory (float or double) into the engine.
    virtual void write_plane(int which, int k, const void *host, int as_double) = 0;
    // Stage hooks for kernel-level parity checks (device pointers of the
    // engine's precision): forward model of exposure k into its blur plane,
    // detector + adjoint gather of exposure k on the current blur plane,
    // update on the current correction plane.
    virtual void stage_forward(int k) = 0;
    virtual void stage_detector(int k, IterationRecord *rec) = 0;
    virtual void stage_update(IterationRecord *rec) = 0;
    virtual void stage_correction() = 0;
    virtual void decode_links(int k, uint32_t *host_targets) = 0;
    virtual uint64_t link_count(int k) const = 0;
    virtual int link_encoding(int k) const = 0;
    // Scalars: 0 weight_scale, 1 max_sensitivity, 2 FW, 3 FH, 4 masked pixels, 5 precision bits
    virtual double scalar(int which) const = 0;
    virtual size_t device_bytes() const = 0;
    virtual const std::vector<ExposureInput> &exposures() const = 0;
    virtual double setup_seconds(int stage) const = 0;
    // Per-stage event timing on the next iterations (eager launches, no graph).
    virtual void set_stage_timing(int on) = 0;
    // FFT shape and radix splits in use, and how they were chosen.
    virtual const FftChoice &fft_choice() const = 0;

    // Differentiable model (nll.cuh).  Per-exposure background and pedestal,
    // and a replacement PSF (FP32 or FP64 host array in the manifest's
    // layout, no larger than the PSF the FFT shape was chosen for).
    virtual void set_exposure_offsets(int k, double background, double pedestal) = 0;
    virtual void set_psf(int k, const void *psf, int psf_width, int psf_height, int as_double) = 0;
    // Forward model of the current estimate, then the NLL terms per exposure
    // (nexp x 4: sum W(mu - y log mu), sum r, sum W log mu, pixels left out)
    // and r = W (1 - y/mu) in the WR planes.
    virtual void nll(double *terms) = 0;
    // Per-block FP64 partial sums behind the last nll() (nexp x blocks x 4).
    virtual const std::vector<double> &nll_partials() const = 0;
    // CORRECTION <- sum_k H_k^T r_k = dL/dx (after nll).
    virtual void nll_adjoint() = 0;
    // dL/dpsi_k for the normalised PSF of exposure k, in the PSF's own layout
    // (after nll_adjoint); psf_width x psf_height doubles.
    virtual void psf_gradient(int k, double *out) = 0;
    // Plane <-> caller device memory (to_engine = 1 writes the plane), on the
    // engine's stream after `stream` (0: legacy default) has reached this call.
    virtual void copy_plane_device(int which, int k, void *dptr, int to_engine, int as_double, cudaStream_t stream) = 0;
    // Iterate only exposures [k0, k0 + n) (an exposure shard of a multi-GPU
    // solve: every other setup product stays that of the whole field).
    // Called before setup(), the shard is set up alone: LinkMaps and PSF
    // spectra of its exposures only, and the drizzle and denominator leave
    // partial planes (COVERAGE, ESTIMATE = data sum, CORRECTION = background
    // sum, DENOMINATOR) that the caller sums over the shards before
    // finish_shard_setup() forms the estimate and the maximum sensitivity.
    virtual void set_active_exposures(int k0, int n) = 0;
    virtual void finish_shard_setup() = 0;
    // Recompute max_sensitivity from the denominator plane (after it was
    // replaced, e.g. by a sum over shards).
    virtual void refresh_sensitivity() = 0;
    // Device address of a target plane (estimate, coverage, denominator or
    // correction: W x H elements of the engine's precision, row-major), valid
    // while the engine lives, and the stream every launch is issued on.
    virtual void *plane_device(int which) = 0;
    virtual cudaStream_t stream() const = 0;
    // The two halves of an iteration, enqueued on the engine's stream without
    // waiting, for a caller that puts a collective between them on the same
    // stream (an exposure shard): the partial correction of the active
    // exposures (forward model, detector loop, gather, adjoint) into the
    // correction plane, then the update from the correction plane as it
    // stands.  finish_iteration waits for the stream, raises a recorded
    // device error, and fills the FreezeMu counters of every exposure (the
    // inactive ones zero) and the update's signed sum and negative count.
    virtual void enqueue_partial() = 0;
    virtual void enqueue_update() = 0;
    virtual void finish_iteration(IterationRecord *rec) = 0;
    // Checkpoint / resume: the estimate and the FreezeMu masks with the
    // iteration count they belong to.
    virtual void save_state(const std::string &path, uint64_t iteration) = 0;
    virtual void load_state(const std::string &path, uint64_t *iteration) = 0;
    // Device-side view of the set-up field for the batched launches (batch.cu).
    virtual struct FieldView field_view() const = 0;
};

// Everything the batched launches need of one set-up field: sizes, plans
// and the device addresses of its planes, spectra and diagnostics (typed by
// the engine's precision, 4 or 8 bytes).
struct FieldView {
    int elem_bytes = 4, form = 0, comp_mu = 0;
    int W = 0, H = 0, M = 0, FH = 0, ldh = 0, row_b = 0, nexp = 0, upd_grid = 0;
    size_t nin = 0, nout = 0;
    FftPlan plan_m, plan_h;
    double scale = 0, max_sens = 0;
    const void *post = nullptr;
    void *estimate = nullptr, *den = nullptr, *correction = nullptr, *blur = nullptr, *scatter = nullptr, *wr = nullptr;
    void *rx = nullptr, *y = nullptr, *rs = nullptr, *cr = nullptr, *khat = nullptr;
    bool needs_aux = false;  // a column transform keeps its plane outside shared memory
    const void *exps = nullptr;  // ExpDesc<T>[nexp]
    void *stats = nullptr;       // ExpStats[nexp]
    unsigned long long *err = nullptr;
    double *part_sum = nullptr, *red_sum = nullptr;
    unsigned long long *part_neg = nullptr, *red_neg = nullptr;
};

std::unique_ptr<Engine> make_engine(const EngineOptions &opt);

// Many independent fields (uneven grids and exposure counts) solved
// together: every stage of an iteration is one persistent launch over the
// work units of all fields, and the whole loop can run as one CUDA graph.
struct BatchRecord {
    double seconds = 0;                    // device time of the batch iteration
    std::vector<double> signed_sum;        // per field
    std::vector<uint64_t> negative;        // per field
    std::vector<uint64_t> new_frozen, total_frozen;  // per exposure, fields in order
};
class Batch {
  public:
    virtual ~Batch() = default;
    virtual void add_field(const std::string &manifest, int W, int H, int iw, int ih, int nexp, int transposed) = 0;
    virtual void setup() = 0;
    virtual void iterate(int n, bool check_each, std::vector<BatchRecord> *records) = 0;
    virtual int fields() const = 0;
    virtual Engine &field(int i) = 0;
    virtual size_t units(int stage) const = 0;  // work units of a stage (diagnostics)
};
std::unique_ptr<Batch> make_batch(const EngineOptions &opt);

// Runs a device wait that runs out after `polls` polls of an mbarrier that
// nothing completes; throws the engine's "device wait timed out" error when
// the kernel recorded it (the bounded-wait path of the row transforms).
void device_wait_check(uint32_t polls);

// Smallest even / any 7-smooth integer >= n.
int next_smooth(int n, bool even);

// The update on caller-owned FP32 device planes with file-scope scratch
// (noalloc.cu); throws Error with the reference's message on failure.
void update_noalloc(const float *correction, const float *denominator, float *estimate, uint64_t n,
                    float max_sensitivity, cudaStream_t stream, double *signed_sum, uint64_t *negative);

}  // namespace updc
