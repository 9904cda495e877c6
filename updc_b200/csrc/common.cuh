// Shared definitions for the UPDC B200 engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>

namespace updc {

// ----------------------------------------------------------------------------- errors
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define UPDC_CUDA(call)                                                                        \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw ::updc::Error(-2, std::string("CUDA error: ") + cudaGetErrorString(e_) +     \
                                           " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
    } while (0)

// Device-side error record.  Kernels never trap; they record the first
// failure in the reference's serial order with atomicMin on
//   key = (stage << 56) | (index << 8) | code
// so the host reports the same message the reference core would have printed
// first (updc/c_core/updc_core.c:109 fail()).
enum DevErrorCode : uint32_t {
    ERR_NONE = 0,
    ERR_NONFINITE_MEAN = 1,          // "non-finite forward mean"
    ERR_NONFINITE_RATIO = 2,         // "non-finite y/raw_mu ratio"
    ERR_NONFINITE_CORRECTION = 3,    // "non-finite multiplicative correction"
    ERR_NEGATIVE_CORRECTION = 4,     // "substantially negative multiplicative correction"
    ERR_NONFINITE_ESTIMATE = 5,      // "non-finite signed UPDC estimate"
    ERR_INVALID_NORM_WHT = 6,        // "invalid normalized WHT"
    ERR_NEGATIVE_YEFF = 7,           // "negative/non-finite y_eff reached solver"
    ERR_NONFINITE_INITIAL = 8,       // "non-finite signed initial estimate"
    ERR_INVALID_PSF_PIXEL = 9,       // "invalid PSF pixel"
    ERR_LINKMAP_TARGET = 10,         // LinkMap target outside the grid (defensive bounds check)
    ERR_DEVICE_TIMEOUT = 11,         // a bounded device-side wait ran out
};
enum DevErrorStage : uint64_t { STAGE_DETECTOR = 1, STAGE_UPDATE = 2, STAGE_SETUP = 3, STAGE_TRANSFORM = 4 };

__host__ __device__ inline uint64_t make_error_key(uint64_t stage, uint64_t index, uint32_t code) {
    return (stage << 56) | ((index & 0xFFFFFFFFFFull) << 8) | (uint64_t)code;
}

const char *error_message(uint32_t code);

// Raises a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device.  The attribute belongs to the function, process-wide, so
// it only ever grows: lowering it for one engine would make another engine's
// launches of the same kernel (other FFT shape) fail.
inline void raise_smem_limit(const void *func, size_t bytes) {
    static std::mutex m;
    static std::map<std::pair<int, const void *>, size_t> current;
    int dev = 0;
    UPDC_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(m);
    size_t &c = current[{dev, func}];
    if (bytes <= c) return;
    UPDC_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    c = bytes;
}

// ----------------------------------------------------------------------------- complex
template <typename T> struct cx { T x, y; };

template <typename T> __host__ __device__ __forceinline__ cx<T> cmk(T a, T b) { return cx<T>{a, b}; }
template <typename T> __host__ __device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T> __host__ __device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) { return {a.x - b.x, a.y - b.y}; }
// (a.x b.x - a.y b.y, a.x b.y + a.y b.x), evaluated without contraction so the
// FP32 products round like the reference's separate multiplies.
template <typename T> __device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b);
template <> __device__ __forceinline__ cx<float> cmul(cx<float> a, cx<float> b) {
    return {__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
template <> __device__ __forceinline__ cx<double> cmul(cx<double> a, cx<double> b) {
    return {__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x))};
}
// Fast complex multiply for FFT internals (contraction allowed).
template <typename T> __host__ __device__ __forceinline__ cx<T> fmulc(cx<T> a, cx<T> b) {
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T> __host__ __device__ __forceinline__ cx<T> fmulc_conj(cx<T> a, cx<T> b) {  // a * conj(b)
    return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename T> __host__ __device__ __forceinline__ cx<T> cscale(cx<T> a, T s) { return {a.x * s, a.y * s}; }

// ----------------------------------------------------------------------------- misc
__host__ __device__ inline size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }

// Order-preserving map of float to uint32 for atomicMin on floats.
__device__ __forceinline__ uint32_t float_to_ordered(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ inline float ordered_to_float(uint32_t u) {
    uint32_t v = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
    float f;
    memcpy(&f, &v, 4);
    return f;
}
__device__ __forceinline__ unsigned long long double_to_ordered(double d) {
    unsigned long long u = (unsigned long long)__double_as_longlong(d);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ inline double ordered_to_double(unsigned long long u) {
    unsigned long long v = (u & 0x8000000000000000ull) ? (u & 0x7FFFFFFFFFFFFFFFull) : ~u;
    double d;
    memcpy(&d, &v, 8);
    return d;
}

}  // namespace updc
