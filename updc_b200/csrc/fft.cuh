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
//
// Radices are 2, 3, 4, 5, 7, 8 and composites R = A*B (up to 32) computed in
// registers as A-point DFTs, internal twiddles, then B-point DFTs; composites
// leave their outputs in a compile-time permuted register order that the
// stage's store phase undoes, so no extra registers are needed.  Fewer,
// larger stages mean fewer shared-memory passes and barriers.  The shared
// buffer is padded by one element every 32 (fpad) so the strided stores of
// early stages do not pile onto one bank.
#pragma once

#include <type_traits>
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
    int pad_shift = 31;               // shared-memory padding: one slot every 2^pad_shift elements
    const void *tw = nullptr;  // device table of cx<T>, forward sign
};

// Splits n into radices no larger than rmax (greedy, largest first), ordered
// as the device stage loops run them (descending).  Returns false when n has
// a prime factor above 7.
bool fft_factor(int n, int rmax, std::vector<int> &radices);

// Padded shared-memory index of logical element e: one pad slot every
// 2^shift elements (shift 31: no padding).  The plan's shift is chosen on the
// host by simulating the bank pattern of its stages (fft_choose_padding).
__host__ __device__ __forceinline__ int fpad(int e, int shift) { return e + (e >> shift); }
// Shared-memory elements for `count` logical elements.
__host__ __device__ __forceinline__ int fpad_size(int count, int shift) { return count + (count >> shift) + 1; }
// Picks the padding shift with the fewest simulated shared-memory wavefronts
// for the plan's stages (8-byte elements, NT threads, batch transforms).
int fft_choose_padding(const FftPlan &plan, int nt, int cap, int batch);

// Every split of n into radices no larger than rmax, each a non-increasing
// sequence (the device's stage order), with at most `extra_stages` stages
// more than the greedy split; the candidates the FFT autotuner times.
void fft_factorizations(int n, int rmax, int extra_stages, std::vector<std::vector<int>> &out);

// Builds the host twiddle table for n (complex, forward sign) and fills the
// plan's stage fields (greedy split, or the given radices in device order).
// The caller uploads the table and sets plan.tw.
template <typename T> std::vector<cx<T>> fft_make_table(int n, int rmax, FftPlan &plan);
template <typename T> std::vector<cx<T>> fft_make_table(int n, const std::vector<int> &radices, FftPlan &plan);

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
template <bool INV, typename T> __host__ __device__ __forceinline__ cx<T> mul_si(cx<T> a) {
    return INV ? cx<T>{-a.y, a.x} : cx<T>{a.y, -a.x};
}

template <int R, bool INV, typename T> struct Dft;

template <bool INV, typename T> struct Dft<2, INV, T> {
    static constexpr int out(int p) { return p; }  // natural output order
    __host__ __device__ __forceinline__ static void run(cx<T> *v) {
        const cx<T> a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};
template <bool INV, typename T> struct Dft<4, INV, T> {
    static constexpr int out(int p) { return p; }  // natural output order
    __host__ __device__ __forceinline__ static void run(cx<T> *v) {
        const cx<T> t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3];
        const cx<T> t3 = mul_si<INV>(v[1] - v[3]);
        v[0] = t0 + t2;
        v[2] = t0 - t2;
        v[1] = t1 + t3;
        v[3] = t1 - t3;
    }
};
template <bool INV, typename T> struct Dft<8, INV, T> {
    static constexpr int out(int p) { return p; }  // natural output order
    __host__ __device__ __forceinline__ static void run(cx<T> *v) {
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
    static constexpr int out(int p) { return p; }  // natural output order
    __host__ __device__ __forceinline__ static void run(cx<T> *v) {
        const cx<T> a = v[1] + v[2], b = v[1] - v[2];
        const cx<T> A = {v[0].x - T(0.5) * a.x, v[0].y - T(0.5) * a.y};
        const cx<T> iB = mul_si<INV>(cscale(b, DftConst<T>::S3));
        v[0] = v[0] + a;
        v[1] = A + iB;
        v[2] = A - iB;
    }
};
template <bool INV, typename T> struct Dft<5, INV, T> {
    static constexpr int out(int p) { return p; }  // natural output order
    __host__ __device__ __forceinline__ static void run(cx<T> *v) {
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
    static constexpr int out(int p) { return p; }  // natural output order
    __host__ __device__ __forceinline__ static void run(cx<T> *v) {
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

// ----------------------------------------------------------------------------- composites
// Compile-time loop and trigonometry for the composite codelets.
template <int I, int N, class F> __host__ __device__ __forceinline__ void static_for(F &&f) {
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        static_for<I + 1, N>(f);
    }
}
// cos/sin(2 pi m / R) by Taylor series after reduction to [-pi, pi] (double,
// evaluated at compile time).
constexpr double ct_pi = 3.14159265358979323846264338327950288;
constexpr double ct_series_cos(double x) {
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 24; ++k) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}
constexpr double ct_series_sin(double x) {
    double term = x, sum = x;
    for (int k = 1; k < 24; ++k) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
constexpr double ct_angle(int m, int R) {
    const int r = ((m % R) + R) % R;
    const int c = 2 * r > R ? r - R : r;  // in (-R/2, R/2]
    return 2.0 * ct_pi * (double)c / (double)R;
}
constexpr double ct_cos(int m, int R) { return ct_series_cos(ct_angle(m, R)); }
constexpr double ct_sin(int m, int R) { return ct_series_sin(ct_angle(m, R)); }

// x * exp(sign * 2 pi i m / R) with m, R compile-time (trivial angles exact).
template <int M, int R, bool INV, typename T> __host__ __device__ __forceinline__ cx<T> twiddle_ct(cx<T> x) {
    constexpr int m = ((M % R) + R) % R;
    if constexpr (m == 0) {
        return x;
    } else if constexpr (2 * m == R) {
        return cx<T>{-x.x, -x.y};
    } else if constexpr (4 * m == R) {
        return mul_si<INV>(x);
    } else if constexpr (4 * m == 3 * R) {
        return mul_si<!INV>(x);
    } else {
        constexpr double c = ct_cos(m, R);
        constexpr double sn = INV ? ct_sin(m, R) : -ct_sin(m, R);
        return cx<T>{x.x * (T)c - x.y * (T)sn, x.x * (T)sn + x.y * (T)c};
    }
}

template <int R> struct Split;  // R = A * B for the composite radices
#define UPDC_SPLIT(R_, A_, B_)                      \
    template <> struct Split<R_> {                  \
        static constexpr int A = A_, B = B_;        \
    };
UPDC_SPLIT(6, 2, 3)
UPDC_SPLIT(9, 3, 3)
UPDC_SPLIT(10, 2, 5)
UPDC_SPLIT(12, 4, 3)
UPDC_SPLIT(14, 2, 7)
UPDC_SPLIT(15, 3, 5)
UPDC_SPLIT(16, 4, 4)
UPDC_SPLIT(18, 2, 9)
UPDC_SPLIT(20, 4, 5)
UPDC_SPLIT(21, 3, 7)
UPDC_SPLIT(24, 8, 3)
UPDC_SPLIT(25, 5, 5)
UPDC_SPLIT(27, 3, 9)
UPDC_SPLIT(28, 4, 7)
UPDC_SPLIT(32, 4, 8)
#undef UPDC_SPLIT

// R = A*B point DFT in place: for each n2 < B the A-point DFT of
// x[B*n1 + n2] (written back at B*k1 + n2, times w_R^(n2*k1)), then for each
// k1 the B-point DFT of the B consecutive values v[B*k1 .. B*k1+B).  Register
// p = B*k1 + q then holds X[k1 + A*out_B(q)]; out() gives that map.
template <int R, bool INV, typename T> struct DftComposite {
    static constexpr int A = Split<R>::A, B = Split<R>::B;
    static constexpr int out(int p) { return p / B + A * Dft<B, INV, T>::out(p % B); }
    __host__ __device__ __forceinline__ static void run(cx<T> *v) {
        static_for<0, B>([&](auto n2) {
            cx<T> a[A];
            static_for<0, A>([&](auto n1) { a[n1] = v[B * n1 + n2]; });
            Dft<A, INV, T>::run(a);
            static_for<0, A>([&](auto q) {
                constexpr int k1 = Dft<A, INV, T>::out(q);
                v[B * k1 + n2] = twiddle_ct<(int)n2 * k1, R, INV>(a[q]);
            });
        });
        static_for<0, A>([&](auto k1) { Dft<B, INV, T>::run(v + B * k1); });
    }
};
#define UPDC_COMPOSITE(R_)                                                         \
    template <bool INV, typename T> struct Dft<R_, INV, T> : DftComposite<R_, INV, T> {};
UPDC_COMPOSITE(6)
UPDC_COMPOSITE(9)
UPDC_COMPOSITE(10)
UPDC_COMPOSITE(12)
UPDC_COMPOSITE(14)
UPDC_COMPOSITE(15)
UPDC_COMPOSITE(16)
UPDC_COMPOSITE(18)
UPDC_COMPOSITE(20)
UPDC_COMPOSITE(21)
UPDC_COMPOSITE(24)
UPDC_COMPOSITE(25)
UPDC_COMPOSITE(27)
UPDC_COMPOSITE(28)
UPDC_COMPOSITE(32)
#undef UPDC_COMPOSITE

// ----------------------------------------------------------------------------- stages
template <int R, int K, bool INV, int NT, typename T>
__device__ __forceinline__ void fft_stage(cx<T> *buf, int n, int batch, int Ns, FastDiv ns_div, FastDiv nb_div,
                                          const cx<T> *__restrict__ tw, int sh) {
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
            const int base = row * n + j;
#pragma unroll
            for (int r = 0; r < R; ++r) v[kk][r] = buf[fpad(base + r * nb, sh)];
            if (k) {
                const cx<T> *t = tw + k;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    cx<T> w = t[(r - 1) * Ns];
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
            static_for<0, R>([&](auto p) {
                constexpr int s = Dft<R, INV, T>::out(p);
                buf[fpad(ob[kk] + s * Ns, sh)] = v[kk][p];
            });
        }
    }
    __syncthreads();
}

template <int R, int NT, int CAP> struct StageK {
    static constexpr int value = (CAP / R + NT - 1) / NT;
};

// Transforms `batch` sequences of length plan.n stored back to back (logical
// index b*n + i, shared-memory slot fpad(., plan.pad_shift)) in buf (batch * n <= CAP).
// Every thread of the block must call this; `plan` is the kernel's
// __grid_constant__ parameter, so its per-stage fields are read from the
// constant bank with a block-uniform index (no shared or local copy, nothing
// held in registers across the callers' loops).  Radices must not exceed
// RMAX.  Stages run in descending radix order (fft_factor), one loop per
// radix, so that only one radix's registers are live at a time (a single
// switch inside one loop makes ptxas spill).
// The plan's padding shift, or PADSH when a kernel is compiled for one
// (PADSH = 31: no padding, so every fpad() folds away).
template <int PADSH> __device__ __forceinline__ int plan_shift(const FftPlan &plan) {
    if constexpr (PADSH >= 0) return PADSH;
    else return plan.pad_shift;
}

template <bool INV, int NT, int CAP, int RMAX, int PADSH = -1, typename T>
__device__ __forceinline__ void fft_batch(cx<T> *buf, int batch, const FftPlan &plan) {
    const cx<T> *tw = reinterpret_cast<const cx<T> *>(plan.tw);
    const int n = plan.n, nstage = plan.nstage, sh = plan_shift<PADSH>(plan);
    int s = 0;
#define UPDC_FFT_RUN(R)                                                                                     \
    if constexpr (R <= RMAX) {                                                                             \
        _Pragma("unroll 1") while (s < nstage && plan.radix[s] == R) {                                     \
            fft_stage<R, StageK<R, NT, CAP>::value, INV, NT>(buf, n, batch, plan.ns[s], plan.ns_div[s],         \
                                                             plan.nb_div[s], tw + plan.twoff[s], sh);           \
            ++s;                                                                                           \
        }                                                                                                  \
    }
    UPDC_FFT_RUN(32)
    UPDC_FFT_RUN(28)
    UPDC_FFT_RUN(27)
    UPDC_FFT_RUN(25)
    UPDC_FFT_RUN(24)
    UPDC_FFT_RUN(21)
    UPDC_FFT_RUN(20)
    UPDC_FFT_RUN(18)
    UPDC_FFT_RUN(16)
    UPDC_FFT_RUN(15)
    UPDC_FFT_RUN(14)
    UPDC_FFT_RUN(12)
    UPDC_FFT_RUN(10)
    UPDC_FFT_RUN(9)
    UPDC_FFT_RUN(8)
    UPDC_FFT_RUN(7)
    UPDC_FFT_RUN(6)
    UPDC_FFT_RUN(5)
    UPDC_FFT_RUN(4)
    UPDC_FFT_RUN(3)
    UPDC_FFT_RUN(2)
#undef UPDC_FFT_RUN
}

}  // namespace updc
