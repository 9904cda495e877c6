// Host orchestration of the UPDC solver on one B200: the B200-native
// replacement for UPDC_ALL (updc/c_core/updc_core.c:1289-1543).
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace updc {

enum Form { FORM_FP32 = 0, FORM_FP64 = 1, FORM_FP32_KAHAN = 2, FORM_FP32_REFERENCE = 3 };

struct EngineOptions {
    int form = FORM_FP32;
    int compensated_mu = -1;  // -1: the form's default
    int use_graph = 1;
    int device = 0;
    int reuse_links = 1;      // reuse a valid LinkMap file instead of rebuilding it
    int verbose = 0;
    int fft_width = 0;        // 0: smallest even 7-smooth width >= W + pw - 1
    int fft_height = 0;       // 0: smallest 7-smooth height >= H + ph - 1
    int stage_timing = 0;     // time each stage with events (no graph)
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
};

std::unique_ptr<Engine> make_engine(const EngineOptions &opt);

// Smallest even / any 7-smooth integer >= n.
int next_smooth(int n, bool even);

// The update on caller-owned FP32 device planes with file-scope scratch
// (noalloc.cu); throws Error with the reference's message on failure.
void update_noalloc(const float *correction, const float *denominator, float *estimate, uint64_t n,
                    float max_sensitivity, cudaStream_t stream, double *signed_sum, uint64_t *negative);

}  // namespace updc
