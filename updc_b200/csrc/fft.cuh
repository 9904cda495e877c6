// Shared-memory mixed-radix Stockham FFT for sm_100a.
//
// One thread block transforms a batch of `batch` contiguous complex sequences
// of length n held in shared memory, in place.  Each stage with radix R and
// Ns = product of the earlier radices does, for every butterfly j < n/R:
//     k = j mod Ns,  v[r] = buf[j + r n/R] * w^(r k / (Ns R)),  V = DFT_R(v),
//     buf[(j - k) R + k + s Ns] = V[s]
// (self-sorting Stockham).  All loads of a stage are staged in registers
// before a barrier and all stores follow it, so one buffer suffices.
// Twiddles come from a table computed in double precision on the host.
#pragma once

#include <vector>

#include "common.cuh"

namespace updc {

constexpr int FFT_MAX_STAGES = 24;

// Division by a run-time constant d for x < 2^31: q = (umulhi(x, mul) + x) >> shift
// with shift = ceil(log2 d) and mul = floor(2^32 (2^shift - d) / d) + 1
// (the round-up method for unsigned division by invariant integers).
struct FastDiv {
    uint32_t d = 1, mul = 1, shift = 0;
    FastDiv() = default;
    explicit FastDiv(uint32_t div) : d(div) {
        shift = 0;
        while ((1ull << shift) < div) ++shift;
        mul = (uint32_t)((((1ull << 32) * ((1ull << shift) - div)) / div) + 1);
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t x) const {
#ifdef __CUDA_ARCH__
        return (__umulhi(x, mul) + x) >> shift;
#else
        return (uint32_t)((((uint64_t)x * mul >> 32) + x) >> shift);
#endif
    }
};

struct FftPlan {
    int n = 0;
    int nstage = 0;
    int radix[FFT_MAX_STAGES] = {};
    int ns[FFT_MAX_STAGES] = {};
    int twoff[FFT_MAX_STAGES] = {};
    FastDiv ns_div[FFT_MAX_STAGES];   // division by Ns
    FastDiv nb_div[FFT_MAX_STAGES];   // division by n / radix
    const void *tw = nullptr;  // device table of cx<T>, forward sign
};

// Radix order: 8s first, then 4, 2, 7, 5, 3.  Returns false when n has a
// prime factor above 7.
bool fft_factor(int n, std::vector<int> &radices);

// Builds the host twiddle table for n (complex, forward sign) and fills the
// plan's stage fields.  The caller uploads the table and sets plan.tw.
template <typename T> std::vector<cx<T>> fft_make_table(int n, FftPlan &plan);

// ----------------------------------------------------------------------------- DFT kernels
template <typename T> struct DftConst;
template <> struct DftConst<float> {
    static constexpr float S3 = 0.866025403784438646763723170753f;
    static constexpr float C51 = 0.309016994374947424102293417183f, S51 = 0.951056516295153572116439333379f;
    static constexpr float C52 = -0.809016994374947424102293417183f, S52 = 0.587785252292473129168705954639f;
    static constexpr float C71 = 0.623489801858733530525004884004f, S71 = 0.781831482468029808708444526674f;
    static constexpr float C72 = -0.222520933956314404288902564497f, S72 = 0.974927912181823607018131682994f;
    static constexpr float C73 = -0.900968867902419126236102319507f, S73 = 0.433883739117558120475768332849f;
    static constexpr float R2 = 0.707106781186547524400844362105f;
};
template <> struct DftConst<double> {
    static constexpr double S3 = 0.866025403784438646763723170753;
    static constexpr double C51 = 0.309016994374947424102293417183, S51 = 0.951056516295153572116439333379;
    static constexpr double C52 = -0.809016994374947424102293417183, S52 = 0.587785252292473129168705954639;
    static constexpr double C71 = 0.623489801858733530525004884004, S71 = 0.781831482468029808708444526674;
    static constexpr double C72 = -0.222520933956314404288902564497, S72 = 0.974927912181823607018131682994;
    static constexpr double C73 = -0.900968867902419126236102319507, S73 = 0.433883739117558120475768332849;
    static constexpr double R2 = 0.707106781186547524400844362105;
};

// multiply by sign*i, sign = -1 (forward) or +1 (inverse)
template <bool INV, typename T> __device__ __forceinline__ cx<T> mul_si(cx<T> a) {
    return INV ? cx<T>{-a.y, a.x} : cx<T>{a.y, -a.x};
}

template <int R, bool INV, typename T> struct Dft;

template <bool INV, typename T> struct Dft<2, INV, T> {
    __device__ __forceinline__ static void run(cx<T> *v) {
        const cx<T> a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};
template <bool INV, typename T> struct Dft<4, INV, T> {
    __device__ __forceinline__ static void run(cx<T> *v) {
        const cx<T> t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3];
        const cx<T> t3 = mul_si<INV>(v[1] - v[3]);
        v[0] = t0 + t2;
        v[2] = t0 - t2;
        v[1] = t1 + t3;
        v[3] = t1 - t3;
    }
};
template <bool INV, typename T> struct Dft<8, INV, T> {
    __device__ __forceinline__ static void run(cx<T> *v) {
        cx<T> e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4, INV, T>::run(e);
        Dft<4, INV, T>::run(o);
        const T c = DftConst<T>::R2;
        // w8^q o[q]
        const cx<T> o1 = INV ? cx<T>{c * (o[1].x - o[1].y), c * (o[1].x + o[1].y)}
                             : cx<T>{c * (o[1].x + o[1].y), c * (o[1].y - o[1].x)};
        const cx<T> o2 = mul_si<INV>(o[2]);
        const cx<T> o3 = INV ? cx<T>{-c * (o[3].x + o[3].y), c * (o[3].x - o[3].y)}
                             : cx<T>{c * (o[3].y - o[3].x), -c * (o[3].x + o[3].y)};
        v[0] = e[0] + o[0];
        v[4] = e[0] - o[0];
        v[1] = e[1] + o1;
        v[5] = e[1] - o1;
        v[2] = e[2] + o2;
        v[6] = e[2] - o2;
        v[3] = e[3] + o3;
        v[7] = e[3] - o3;
    }
};
template <bool INV, typename T> struct Dft<3, INV, T> {
    __device__ __forceinline__ static void run(cx<T> *v) {
        const cx<T> a = v[1] + v[2], b = v[1] - v[2];
        const cx<T> A = {v[0].x - T(0.5) * a.x, v[0].y - T(0.5) * a.y};
        const cx<T> iB = mul_si<INV>(cscale(b, DftConst<T>::S3));
        v[0] = v[0] + a;
        v[1] = A + iB;
        v[2] = A - iB;
    }
};
template <bool INV, typename T> struct Dft<5, INV, T> {
    __device__ __forceinline__ static void run(cx<T> *v) {
        using K = DftConst<T>;
        const cx<T> a1 = v[1] + v[4], b1 = v[1] - v[4], a2 = v[2] + v[3], b2 = v[2] - v[3];
        const cx<T> A1 = {v[0].x + a1.x * K::C51 + a2.x * K::C52, v[0].y + a1.y * K::C51 + a2.y * K::C52};
        const cx<T> A2 = {v[0].x + a1.x * K::C52 + a2.x * K::C51, v[0].y + a1.y * K::C52 + a2.y * K::C51};
        const cx<T> B1 = {b1.x * K::S51 + b2.x * K::S52, b1.y * K::S51 + b2.y * K::S52};
        const cx<T> B2 = {b1.x * K::S52 - b2.x * K::S51, b1.y * K::S52 - b2.y * K::S51};
        const cx<T> iB1 = mul_si<INV>(B1), iB2 = mul_si<INV>(B2);
        v[0] = v[0] + a1 + a2;
        v[1] = A1 + iB1;
        v[4] = A1 - iB1;
        v[2] = A2 + iB2;
        v[3] = A2 - iB2;
    }
};
template <bool INV, typename T> struct Dft<7, INV, T> {
    __device__ __forceinline__ static void run(cx<T> *v) {
        using K = DftConst<T>;
        const cx<T> a1 = v[1] + v[6], b1 = v[1] - v[6];
        const cx<T> a2 = v[2] + v[5], b2 = v[2] - v[5];
        const cx<T> a3 = v[3] + v[4], b3 = v[3] - v[4];
        const cx<T> A1 = {v[0].x + a1.x * K::C71 + a2.x * K::C72 + a3.x * K::C73,
                          v[0].y + a1.y * K::C71 + a2.y * K::C72 + a3.y * K::C73};
        const cx<T> A2 = {v[0].x + a1.x * K::C72 + a2.x * K::C73 + a3.x * K::C71,
                          v[0].y + a1.y * K::C72 + a2.y * K::C73 + a3.y * K::C71};
        const cx<T> A3 = {v[0].x + a1.x * K::C73 + a2.x * K::C71 + a3.x * K::C72,
                          v[0].y + a1.y * K::C73 + a2.y * K::C71 + a3.y * K::C72};
        // sin(2 pi a q / 7): a=1: (S1, S2, S3); a=2: (S2, -S3, -S1); a=3: (S3, -S1, S2)
        const cx<T> B1 = {b1.x * K::S71 + b2.x * K::S72 + b3.x * K::S73, b1.y * K::S71 + b2.y * K::S72 + b3.y * K::S73};
        const cx<T> B2 = {b1.x * K::S72 - b2.x * K::S73 - b3.x * K::S71, b1.y * K::S72 - b2.y * K::S73 - b3.y * K::S71};
        const cx<T> B3 = {b1.x * K::S73 - b2.x * K::S71 + b3.x * K::S72, b1.y * K::S73 - b2.y * K::S71 + b3.y * K::S72};
        const cx<T> iB1 = mul_si<INV>(B1), iB2 = mul_si<INV>(B2), iB3 = mul_si<INV>(B3);
        v[0] = v[0] + a1 + a2 + a3;
        v[1] = A1 + iB1;
        v[6] = A1 - iB1;
        v[2] = A2 + iB2;
        v[5] = A2 - iB2;
        v[3] = A3 + iB3;
        v[4] = A3 - iB3;
    }
};

// ----------------------------------------------------------------------------- stages
template <int R, int K, bool INV, int NT, typename T>
__device__ __forceinline__ void fft_stage(cx<T> *buf, int n, int batch, int Ns, FastDiv ns_div, FastDiv nb_div,
                                          const cx<T> *__restrict__ tw) {
    const int nb = n / R;
    const int total = nb * batch;
    const int tid = threadIdx.x;
    // v is defined on every path: a conditionally defined array becomes live
    // around the back-edge of any loop that calls the FFT, which keeps every
    // stage's registers live at once and spills.
    cx<T> v[K][R];
    int ob[K];
#pragma unroll
    for (int kk = 0; kk < K; ++kk) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[kk][r] = cx<T>{T(0), T(0)};
    }
#pragma unroll
    for (int kk = 0; kk < K; ++kk) {
        const int b = tid + kk * NT;
        ob[kk] = -1;
        if (b < total) {
            const int row = batch == 1 ? 0 : (int)nb_div.div((uint32_t)b);
            const int j = b - row * nb;
            const int k = j - (int)ns_div.div((uint32_t)j) * Ns;
            const cx<T> *base = buf + row * n;
#pragma unroll
            for (int r = 0; r < R; ++r) v[kk][r] = base[j + r * nb];
            if (k) {
                const cx<T> *t = tw + k * (R - 1);
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    cx<T> w = t[r - 1];
                    if (INV) w.y = -w.y;
                    v[kk][r] = fmulc(v[kk][r], w);
                }
            }
            Dft<R, INV, T>::run(v[kk]);
            ob[kk] = row * n + (j - k) * R + k;
        }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < K; ++kk) {
        if (ob[kk] >= 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) buf[ob[kk] + r * Ns] = v[kk][r];
        }
    }
    __syncthreads();
}

template <int R, int NT, int CAP> struct StageK {
    static constexpr int value = (CAP / R + NT - 1) / NT;
};

__device__ __forceinline__ FastDiv FastDiv_v(const volatile FastDiv &v) {
    FastDiv r;
    r.d = v.d;
    r.mul = v.mul;
    r.shift = v.shift;
    return r;
}

// Copies a plan from device memory into the block's shared copy.  Kernels
// keep the plan in shared memory: indexing a kernel-parameter array
// dynamically would force a local copy of the structure, and reading the
// fields from global memory on every stage exposes a full memory latency.
__device__ __forceinline__ void load_plan(const FftPlan *__restrict__ g, FftPlan *s) {
    const int *src = reinterpret_cast<const int *>(g);
    int *dst = reinterpret_cast<int *>(s);
    for (int i = threadIdx.x; i < (int)(sizeof(FftPlan) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

// Transforms `batch` sequences of length plan.n stored back to back in buf
// (batch * n <= CAP).  Every thread of the block must call this; `plan` points
// to the block's shared copy.  Stages are ordered by radix (fft_factor), and
// each radix gets its own loop so that only one radix's registers are live at
// a time (a single switch inside one loop makes ptxas spill).
template <bool INV, int NT, int CAP, typename T>
__device__ __forceinline__ void fft_batch(cx<T> *buf, int batch, const FftPlan *plan) {
    // volatile (shared-memory) reads keep the per-stage fields from being
    // hoisted out of the callers' loops (a hoisted copy of the whole plan
    // would spill)
    const volatile FftPlan *vp = plan;
    const cx<T> *tw = reinterpret_cast<const cx<T> *>(vp->tw);
    const int n = vp->n, nstage = vp->nstage;
    int s = 0;
#define UPDC_FFT_RUN(R)                                                                                   \
    _Pragma("unroll 1") while (s < nstage && vp->radix[s] == R) {                                                           \
        fft_stage<R, StageK<R, NT, CAP>::value, INV, NT>(buf, n, batch, vp->ns[s],                       \
                                                         FastDiv_v(vp->ns_div[s]), FastDiv_v(vp->nb_div[s]), \
                                                         tw + vp->twoff[s]);                             \
        ++s;                                                                                             \
    }
    UPDC_FFT_RUN(8)
    UPDC_FFT_RUN(4)
    UPDC_FFT_RUN(2)
    UPDC_FFT_RUN(7)
    UPDC_FFT_RUN(5)
    UPDC_FFT_RUN(3)
#undef UPDC_FFT_RUN
}

}  // namespace updc
