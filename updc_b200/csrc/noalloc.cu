// The multiplicative update on caller-owned device planes with no allocation:
// its scratch (per-block partial sums, the device error record and the two
// reduced results) lives in one file-scope __device__ array.
//
// The kernels (pointwise.cuh k_update and k_reduce_partials,
// updc/c_core/updc_core.c:1437-1456) apply the engine update stage's per-pixel
// arithmetic, so the estimate and the negative count are the ones
// updc_stage_update gives for the same planes; the signed sum is the same
// double-precision sum taken over a different grouping of partial sums (it
// agrees to rounding).  Caller planes need no particular alignment.
#include <mutex>

#include "../../include/updc_b200.h"
#include "common.cuh"
#include "pointwise.cuh"

namespace updc {

// Partial-sum slots: one per block of the update grid, which never exceeds
// UPDATE_MAX_BLOCKS (the engine's 1-D grid cap, 16 blocks per SM x 148 SMs).
constexpr int UPDATE_MAX_BLOCKS = 148 * 16;
constexpr size_t SCRATCH_PARTIAL_SUM = 0;                                            // double[UPDATE_MAX_BLOCKS]
constexpr size_t SCRATCH_PARTIAL_NEG = SCRATCH_PARTIAL_SUM + 8 * UPDATE_MAX_BLOCKS;  // u64[UPDATE_MAX_BLOCKS]
constexpr size_t SCRATCH_ERROR = SCRATCH_PARTIAL_NEG + 8 * UPDATE_MAX_BLOCKS;        // u64 error key
constexpr size_t SCRATCH_SUM = SCRATCH_ERROR + 8;                                    // double
constexpr size_t SCRATCH_NEG = SCRATCH_SUM + 8;                                      // u64
constexpr size_t SCRATCH_BYTES = SCRATCH_NEG + 8;
static_assert(SCRATCH_BYTES == UPDC_UPDATE_NOALLOC_SCRATCH_BYTES, "scratch size must match the header");

static __device__ __align__(256) unsigned char g_update_scratch[SCRATCH_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
// Per device: the context the address was looked up in, and the address.
struct ScratchEntry {
    void *context = nullptr;
    unsigned char *addr = nullptr;
};
ScratchEntry g_scratch[MAX_DEVICES];

// The calling thread's current driver context (cuCtxGetCurrent, reached
// through the runtime's entry-point query so the library needs no -lcuda).
void *current_context() {
    using GetCurrent = int (*)(void **);
    static GetCurrent get = nullptr;
    if (!get) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        UPDC_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess) throw Error(-2, "cuCtxGetCurrent is unavailable");
        get = (GetCurrent)fn;
    }
    void *ctx = nullptr;
    if (get(&ctx) != 0) throw Error(-2, "cuCtxGetCurrent failed");
    return ctx;
}

// Device address of this device's scratch.  It is looked up on the first
// call on each device and again whenever the device's context changed since
// (cudaDeviceReset tears the context down and the module, with its scratch,
// is loaded anew in the next one), so a stale address is never used.
unsigned char *scratch_for(int device) {
    void *ctx = current_context();
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    ScratchEntry &e = g_scratch[device];
    if (!ctx || !e.addr || e.context != ctx) {
        void *p = nullptr;
        // also makes the device's primary context current in this thread
        UPDC_CUDA(cudaGetSymbolAddress(&p, g_update_scratch));
        e.addr = static_cast<unsigned char *>(p);
        e.context = current_context();
    }
    return e.addr;
}

}  // namespace

void update_noalloc(const float *correction, const float *denominator, float *estimate, uint64_t n,
                    float max_sensitivity, cudaStream_t stream, double *signed_sum, uint64_t *negative) {
    if (!correction || !denominator || !estimate) throw Error(1, "update_noalloc: null plane pointer");
    if (n == 0) throw Error(1, "update_noalloc: empty plane (n = 0)");
    if (n > UPDC_UPDATE_NOALLOC_MAX_PIXELS)
        throw Error(1, "update_noalloc: plane of " + std::to_string((unsigned long long)n) +
                           " pixels exceeds the maximum of " +
                           std::to_string((unsigned long long)UPDC_UPDATE_NOALLOC_MAX_PIXELS));
    int device = 0;
    UPDC_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= MAX_DEVICES) throw Error(1, "update_noalloc: device ordinal out of range");
    unsigned char *s = scratch_for(device);
    double *part_sum = reinterpret_cast<double *>(s + SCRATCH_PARTIAL_SUM);
    unsigned long long *part_neg = reinterpret_cast<unsigned long long *>(s + SCRATCH_PARTIAL_NEG);
    unsigned long long *err = reinterpret_cast<unsigned long long *>(s + SCRATCH_ERROR);
    double *sum = reinterpret_cast<double *>(s + SCRATCH_SUM);
    unsigned long long *neg = reinterpret_cast<unsigned long long *>(s + SCRATCH_NEG);

    size_t g = (n + 255) / 256;
    if (g > (size_t)UPDATE_MAX_BLOCKS) g = UPDATE_MAX_BLOCKS;
    const int grid = (int)g;
    // the error record starts at "none" on every call; partial slots and the
    // results are written before they are read, so they need no initial value
    UPDC_CUDA(cudaMemsetAsync(err, 0xFF, 8, stream));
    k_update<float><<<grid, 256, 0, stream>>>((size_t)n, correction, denominator, estimate, max_sensitivity, err,
                                              part_sum, part_neg);
    k_reduce_partials<<<1, 256, 0, stream>>>(part_sum, part_neg, grid, sum, neg);
    UPDC_CUDA(cudaGetLastError());
    unsigned long long key = ~0ull, hneg = 0;
    double hsum = 0;
    UPDC_CUDA(cudaMemcpyAsync(&key, err, 8, cudaMemcpyDeviceToHost, stream));
    UPDC_CUDA(cudaMemcpyAsync(&hsum, sum, 8, cudaMemcpyDeviceToHost, stream));
    UPDC_CUDA(cudaMemcpyAsync(&hneg, neg, 8, cudaMemcpyDeviceToHost, stream));
    UPDC_CUDA(cudaStreamSynchronize(stream));
    if (key != ~0ull) {
        const uint32_t code = (uint32_t)(key & 0xFF);
        const uint64_t index = (key >> 8) & 0xFFFFFFFFFFull;
        if (code == ERR_NEGATIVE_CORRECTION && index < n) {
            float c = 0, d = 0;
            UPDC_CUDA(cudaMemcpy(&c, correction + index, 4, cudaMemcpyDeviceToHost));
            UPDC_CUDA(cudaMemcpy(&d, denominator + index, 4, cudaMemcpyDeviceToHost));
            fprintf(stderr, "negative correction at target %llu: C=%.9g numerator=%.9g denominator=%.9g\n",
                    (unsigned long long)index, (double)(c / d), (double)c, (double)d);
        }
        throw Error(1, error_message(code));
    }
    if (signed_sum) *signed_sum = hsum;
    if (negative) *negative = hneg;
}

}  // namespace updc
