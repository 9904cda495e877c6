// Compile-time mixed-radix Stockham FFT stages for sm_100a.
//
// The same self-sorting transform as fft.cuh (stage with radix R and Ns =
// product of the earlier radices: v[r] = buf[j + r N/R] * w^(r k/(Ns R)),
// V = DFT_R(v), buf[(j - k) R + k + s Ns] = V[s], k = j mod Ns), but with the
// length, the radix sequence, the batch and the block size known to the
// compiler.  Every shared-memory offset r*N/R and s*Ns, every twiddle offset
// and every division by Ns or N/R is then a constant: loads and stores take
// immediate offsets from one base register, the first stage has no twiddles,
// and the rounds of butterflies a thread runs are unrolled with a
// warp-uniform test only on the last, partial one.
//
// The twiddle table is the r-major table of fft_make_table for the same
// radix sequence (stage s starts at sum over t < s of (R_t - 1) Ns_t).
#pragma once

#include "fft.cuh"

namespace updc {

template <int... R> struct CtProd;
template <> struct CtProd<> {
    static constexpr int value = 1;
};
template <int A, int... R> struct CtProd<A, R...> {
    static constexpr int value = A * CtProd<R...>::value;
};

// One stage over BATCH sequences of length N stored back to back in buf.
// Butterfly b = tid + kk*NT of round kk; rounds before the last are full for
// every thread, the last is entered only by warps that own a butterfly.
template <int R, int NS, int TWOFF, int N, int BATCH, int NT, bool INV, typename T>
__device__ __forceinline__ void ct_stage(cx<T> *buf, const cx<T> *__restrict__ tw) {
    constexpr int NB = N / R;
    constexpr int TOTAL = NB * BATCH;
    constexpr int K = (TOTAL + NT - 1) / NT;
    constexpr bool LAST_FULL = TOTAL % NT == 0;
    const int tid = threadIdx.x;
    cx<T> v[K][R];
    int ob[K];
#pragma unroll
    for (int kk = 0; kk < K; ++kk) {
        const bool full = kk < K - 1 || LAST_FULL;
        const bool warp_on = full || (tid & ~31) + kk * NT < TOTAL;
        if (warp_on) {
            int b = tid + kk * NT;
            if (!full) b = b < TOTAL ? b : TOTAL - 1;  // idle lanes of the last warp repeat a butterfly
            const int row = BATCH == 1 ? 0 : b / NB;
            const int j = b - row * NB;
            const int k = NS == 1 ? 0 : j % NS;
            const cx<T> *src = buf + row * N + j;
#pragma unroll
            for (int r = 0; r < R; ++r) v[kk][r] = src[r * NB];
            if constexpr (NS > 1) {
                const cx<T> *t = tw + TWOFF + k;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    cx<T> w = t[(r - 1) * NS];
                    if (INV) w.y = -w.y;
                    v[kk][r] = fmulc(v[kk][r], w);
                }
            }
            Dft<R, INV, T>::run(v[kk]);
            ob[kk] = (full || tid + kk * NT < TOTAL) ? row * N + (j - k) * R + k : -1;
        } else {
            ob[kk] = -1;
        }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < K; ++kk) {
        const bool full = kk < K - 1 || LAST_FULL;
        if (full || ob[kk] >= 0) {
            cx<T> *dst = buf + ob[kk];
            static_for<0, R>([&](auto p) {
                constexpr int s = Dft<R, INV, T>::out(p);
                dst[s * NS] = v[kk][p];
            });
        }
    }
    __syncthreads();
}

template <int N, int BATCH, int NT, bool INV, typename T, int NS, int TWOFF, int... R> struct CtStages;
template <int N, int BATCH, int NT, bool INV, typename T, int NS, int TWOFF>
struct CtStages<N, BATCH, NT, INV, T, NS, TWOFF> {
    __device__ __forceinline__ static void run(cx<T> *, const cx<T> *) {}
};
template <int N, int BATCH, int NT, bool INV, typename T, int NS, int TWOFF, int R0, int... R>
struct CtStages<N, BATCH, NT, INV, T, NS, TWOFF, R0, R...> {
    __device__ __forceinline__ static void run(cx<T> *buf, const cx<T> *tw) {
        ct_stage<R0, NS, TWOFF, N, BATCH, NT, INV, T>(buf, tw);
        CtStages<N, BATCH, NT, INV, T, NS * R0, TWOFF + (R0 - 1) * NS, R...>::run(buf, tw);
    }
};

// The whole transform of BATCH sequences of length N = R0*R1*... in buf
// (unpadded, back to back), every thread of the NT-thread block calling it.
// The caller synchronises before (buf written) and the last stage ends with
// a barrier.
template <int BATCH, int NT, bool INV, typename T, int... R>
__device__ __forceinline__ void ct_fft(cx<T> *buf, const cx<T> *__restrict__ tw) {
    CtStages<CtProd<R...>::value, BATCH, NT, INV, T, 1, 0, R...>::run(buf, tw);
}

}  // namespace updc
