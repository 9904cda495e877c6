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
    // v is defined on every path (the zeros of the full rounds are dead
    // stores): registers defined on only some paths stay live around the
    // back-edge of any loop that calls the transform, and spill
    cx<T> v[K][R];
    int ob[K];
#pragma unroll
    for (int kk = 0; kk < K; ++kk) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[kk][r] = cx<T>{T(0), T(0)};
        ob[kk] = -1;
    }
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

// ---------------------------------------------------------------------------- edge stages
// The first stage reads its inputs through `in(row, i)` (element i of
// sequence row, e.g. straight from global memory) and writes the shared
// buffer; the last stage reads the shared buffer and hands its outputs to
// `out(row, i, v)`.  Neither reads and writes the same memory, so each
// butterfly is loaded, transformed and stored before the next one (no
// registers held across a barrier), and a transform of S stages makes S - 1
// shared-memory round trips instead of S + 1.
//
// First stage: Ns = 1, no twiddles; butterfly j reads i = j + r N/R and
// writes j R + s.  Ends with a barrier.
template <int R, int N, int BATCH, int NT, bool INV, typename T, class In>
__device__ __forceinline__ void ct_first(const In &in, cx<T> *buf) {
    constexpr int NB = N / R;
    constexpr int TOTAL = NB * BATCH;
    constexpr int K = (TOTAL + NT - 1) / NT;
#pragma unroll
    for (int kk = 0; kk < K; ++kk) {
        const int b = threadIdx.x + kk * NT;
        if ((kk + 1) * NT <= TOTAL || b < TOTAL) {
            const int row = BATCH == 1 ? 0 : b / NB;
            const int j = b - row * NB;
            cx<T> v[R];
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = in(row, j + r * NB);
            Dft<R, INV, T>::run(v);
            cx<T> *dst = buf + row * N + j * R;
            static_for<0, R>([&](auto p) { dst[Dft<R, INV, T>::out(p)] = v[p]; });
        }
    }
    __syncthreads();
}

// Last stage: Ns = N/R, so k = j and butterfly j writes i = j + s N/R.
// Starts from a complete buffer; no barrier at its end.
template <int R, int TWOFF, int N, int BATCH, int NT, bool INV, typename T, class Out>
__device__ __forceinline__ void ct_last(const cx<T> *buf, const cx<T> *__restrict__ tw, const Out &out) {
    constexpr int NB = N / R;
    constexpr int TOTAL = NB * BATCH;
    constexpr int K = (TOTAL + NT - 1) / NT;
#pragma unroll
    for (int kk = 0; kk < K; ++kk) {
        const int b = threadIdx.x + kk * NT;
        if ((kk + 1) * NT <= TOTAL || b < TOTAL) {
            const int row = BATCH == 1 ? 0 : b / NB;
            const int j = b - row * NB;
            cx<T> v[R];
            const cx<T> *src = buf + row * N + j;
#pragma unroll
            for (int r = 0; r < R; ++r) v[r] = src[r * NB];
            const cx<T> *t = tw + TWOFF + j;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                cx<T> w = t[(r - 1) * NB];
                if (INV) w.y = -w.y;
                v[r] = fmulc(v[r], w);
            }
            Dft<R, INV, T>::run(v);
            static_for<0, R>([&](auto p) { out(row, j + Dft<R, INV, T>::out(p) * NB, v[p]); });
        }
    }
}

template <int N, int BATCH, int NT, bool INV, typename T, int NS, int TWOFF, class Out, int... R> struct CtTail;
template <int N, int BATCH, int NT, bool INV, typename T, int NS, int TWOFF, class Out, int RL>
struct CtTail<N, BATCH, NT, INV, T, NS, TWOFF, Out, RL> {
    __device__ __forceinline__ static void run(cx<T> *buf, const cx<T> *tw, const Out &out) {
        static_assert(NS * RL == N, "radices must multiply to the length");
        ct_last<RL, TWOFF, N, BATCH, NT, INV, T>(buf, tw, out);
    }
};
template <int N, int BATCH, int NT, bool INV, typename T, int NS, int TWOFF, class Out, int R0, int R1, int... R>
struct CtTail<N, BATCH, NT, INV, T, NS, TWOFF, Out, R0, R1, R...> {
    __device__ __forceinline__ static void run(cx<T> *buf, const cx<T> *tw, const Out &out) {
        ct_stage<R0, NS, TWOFF, N, BATCH, NT, INV, T>(buf, tw);
        CtTail<N, BATCH, NT, INV, T, NS * R0, TWOFF + (R0 - 1) * NS, Out, R1, R...>::run(buf, tw, out);
    }
};

// Transform of BATCH sequences with at least two stages: inputs through
// `in`, outputs through `out`, `buf` (BATCH*N complex) as the exchange.
// The caller synchronises before `buf` is written again.
template <int BATCH, int NT, bool INV, typename T, int R0, int... R, class In, class Out>
__device__ __forceinline__ void ct_fft_io(const In &in, cx<T> *buf, const cx<T> *__restrict__ tw, const Out &out) {
    static_assert(sizeof...(R) >= 1, "at least two stages");
    constexpr int N = CtProd<R0, R...>::value;
    ct_first<R0, N, BATCH, NT, INV, T>(in, buf);
    CtTail<N, BATCH, NT, INV, T, R0, R0 - 1, Out, R...>::run(buf, tw, out);
}

}  // namespace updc
