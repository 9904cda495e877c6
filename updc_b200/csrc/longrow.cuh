// Row transforms longer than one block's shared memory holds (FW/2 above the
// row capacity of 5632 complex points): the half-length complex FFT of
// z[m] = x[2m] + i x[2m+1] (m < M) split four-step as M = M1 * M2, both
// factors within a block, with m = n1 + M1 n2 and bin k = k2 + M2 k1:
//
//   X[k2 + M2 k1] = sum_n1 w_M1^(n1 k1) [ w_M^(n1 k2) sum_n2 z[n1 + M1 n2] w_M2^(n2 k2) ]
//
// R2C, pass A: for a group of LONG_G consecutive n1, the M2-point FFTs over
//   n2 (strided input from the plane), times w_M^(n1 k2), into a global
//   scratch laid out [plane][row][k2][n1];
// R2C, pass B: for k2 and its partner M2 - k2, the M1-point FFTs over n1
//   (contiguous scratch rows) give X[k2 + M2 k1] for every k1, and with it the
//   partner bins X[M - u] the split post-processing of the real transform
//   needs (for k2 = 0 they lie in the same sequence); bins go to the u-major
//   spectrum.
// C2R runs the same steps backwards: pass A forms Z[u] from the bins u and
// M - u (the real transform's pre-processing) for two k2 per block and runs
// the inverse M1-point FFTs over k1 times w_M^-(n1 k2); pass B runs the
// inverse M2-point FFTs over k2 for LONG_G consecutive n1 and writes the
// cropped, scaled real outputs.  The arithmetic of the pre- and
// post-processing is that of the single-block row kernels (kernels.cuh).
#pragma once

#include "kernels.cuh"

namespace updc {

constexpr int LONG_G = 8;  // sequences per block of the strided passes

// The split of one long row length, and its device tables.
struct LongRowPlan {
    int M = 0, M1 = 0, M2 = 0;
    FftPlan p1, p2;             // M1- and M2-point plans (no padding)
    const void *twm = nullptr;  // cx<T>[M]: w_M^e = exp(-2 pi i e / M)
};

// w_M^(a b) (conjugated for the inverse), from the table of M roots.
template <bool INV, typename T>
__device__ __forceinline__ cx<T> long_twiddle(const cx<T> *__restrict__ twm, int M, uint32_t a, uint32_t b) {
    cx<T> w = twm[(uint32_t)(((uint64_t)a * b) % (uint64_t)M)];
    if (INV) w.y = -w.y;
    return w;
}

// Bin u of the real transform from Z = X[u mod M] and Zm = X[(M - u) mod M]
// of the half-length transform (the split post-processing of r2c_bin).
template <typename T> __device__ __forceinline__ cx<T> r2c_split(cx<T> Z, cx<T> Zm, cx<T> w) {
    const T half = T(0.5);
    const cx<T> Zc = {Zm.x, -Zm.y};
    const cx<T> E = {half * (Z.x + Zc.x), half * (Z.y + Zc.y)};
    const cx<T> D = {half * (Z.x - Zc.x), half * (Z.y - Zc.y)};
    const cx<T> P = fmulc(D, w);
    return {E.x + P.y, E.y - P.x};
}

// ---------------------------------------------------------------------------- R2C
// grid (ceil(M1 / LONG_G), rows, planes); LONG_G * M2 complex of shared memory.
template <typename T, int NT, int CAP, class Loader>
__global__ void __launch_bounds__(NT) k_long_r2c_a(const __grid_constant__ LongRowPlan lp, Loader ld, int W, int rows,
                                                   cx<T> *__restrict__ scratch) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int M1 = lp.M1, M2 = lp.M2;
    const int n10 = blockIdx.x * LONG_G, y = blockIdx.y, k = blockIdx.z;
    for (int i = threadIdx.x; i < LONG_G * M2; i += NT) {
        const int g = i % LONG_G, n2 = i / LONG_G;
        cx<T> z = {T(0), T(0)};
        if (n10 + g < M1) {
            const int x = 2 * (n10 + g + M1 * n2);
            if (x < W) z.x = ld(k, y, x);
            if (x + 1 < W) z.y = ld(k, y, x + 1);
        }
        buf[g * M2 + n2] = z;
    }
    __syncthreads();
    fft_batch<false, NT, CAP, FFT_RMAX, 31>(buf, LONG_G, lp.p2);
    __syncthreads();
    const cx<T> *twm = reinterpret_cast<const cx<T> *>(lp.twm);
    cx<T> *dst = scratch + ((size_t)k * rows + y) * lp.M;
    for (int i = threadIdx.x; i < LONG_G * M2; i += NT) {
        const int g = i % LONG_G, k2 = i / LONG_G, n1 = n10 + g;
        if (n1 < M1) dst[(size_t)k2 * M1 + n1] = fmulc(buf[g * M2 + k2], long_twiddle<false>(twm, lp.M, n1, k2));
    }
}

// grid (M2 / 2 + 1, rows, planes); 2 * M1 complex of shared memory.
template <typename T, int NT, int CAP>
__global__ void __launch_bounds__(NT) k_long_r2c_b(const __grid_constant__ LongRowPlan lp, const cx<T> *__restrict__ scratch,
                                                   const cx<T> *__restrict__ post, int rows, SpecRef out) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int M = lp.M, M1 = lp.M1, M2 = lp.M2;
    const int ka = blockIdx.x, kb = (M2 - ka) % M2, y = blockIdx.y, k = blockIdx.z;
    const int ns = kb == ka ? 1 : 2;
    const cx<T> *src = scratch + ((size_t)k * rows + y) * M;
    for (int i = threadIdx.x; i < ns * M1; i += NT) {
        const int s = i / M1, n1 = i - s * M1;
        buf[i] = src[(size_t)(s ? kb : ka) * M1 + n1];
    }
    __syncthreads();
    fft_batch<false, NT, CAP, FFT_RMAX, 31>(buf, ns, lp.p1);
    __syncthreads();
    cx<T> *dst = reinterpret_cast<cx<T> *>(out.p) + k * out.batch_stride;
    for (int i = threadIdx.x; i < ns * M1; i += NT) {
        const int s = i / M1, k1 = i - s * M1;
        const int k2 = s ? kb : ka, u = k2 + M2 * k1;
        // the partner bin (M - u) mod M
        const int sp = k2 == 0 ? s : (ns == 2 ? 1 - s : s);
        const int k1p = k2 == 0 ? (M1 - k1) % M1 : M1 - 1 - k1;
        const cx<T> Z = buf[i], Zm = buf[sp * M1 + k1p];
        dst[(size_t)u * out.ld + y] = r2c_split(Z, Zm, post[u]);
        if (u == 0) dst[(size_t)M * out.ld + y] = r2c_split(Z, Z, post[M]);
    }
}

// ---------------------------------------------------------------------------- C2R
// grid (ceil(M2 / 2), rows, planes); 2 * M1 complex of shared memory.
template <typename T, int NT, int CAP>
__global__ void __launch_bounds__(NT) k_long_c2r_a(const __grid_constant__ LongRowPlan lp, const cx<T> *__restrict__ post,
                                                   SpecRef in, int rows, cx<T> *__restrict__ scratch) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int M = lp.M, M1 = lp.M1, M2 = lp.M2;
    const int k20 = 2 * blockIdx.x, y = blockIdx.y, k = blockIdx.z;
    const int ns = min(2, M2 - k20);
    const cx<T> *src = reinterpret_cast<const cx<T> *>(in.p) + k * in.batch_stride;
    for (int i = threadIdx.x; i < ns * M1; i += NT) {
        const int s = i / M1, k1 = i - s * M1;
        const int u = k20 + s + M2 * k1;
        buf[i] = c2r_input(src[(size_t)u * in.ld + y], src[(size_t)(M - u) * in.ld + y], u, post);
    }
    __syncthreads();
    fft_batch<true, NT, CAP, FFT_RMAX, 31>(buf, ns, lp.p1);
    __syncthreads();
    const cx<T> *twm = reinterpret_cast<const cx<T> *>(lp.twm);
    cx<T> *dst = scratch + ((size_t)k * rows + y) * M;
    for (int i = threadIdx.x; i < ns * M1; i += NT) {
        const int s = i / M1, n1 = i - s * M1, k2 = k20 + s;
        dst[(size_t)k2 * M1 + n1] = fmulc(buf[i], long_twiddle<true>(twm, M, n1, k2));
    }
}

// grid (ceil(M1 / LONG_G), rows, planes); LONG_G * M2 complex of shared memory.
template <typename T, int NT, int CAP, class Epi>
__global__ void __launch_bounds__(NT) k_long_c2r_b(const __grid_constant__ LongRowPlan lp, const cx<T> *__restrict__ scratch,
                                                   int rows, int W, T scale, Epi epi) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int M1 = lp.M1, M2 = lp.M2;
    const int n10 = blockIdx.x * LONG_G, y = blockIdx.y, k = blockIdx.z;
    const cx<T> *src = scratch + ((size_t)k * rows + y) * lp.M;
    for (int i = threadIdx.x; i < LONG_G * M2; i += NT) {
        const int g = i % LONG_G, k2 = i / LONG_G;
        buf[g * M2 + k2] = n10 + g < M1 ? src[(size_t)k2 * M1 + n10 + g] : cx<T>{T(0), T(0)};
    }
    __syncthreads();
    fft_batch<true, NT, CAP, FFT_RMAX, 31>(buf, LONG_G, lp.p2);
    __syncthreads();
    for (int i = threadIdx.x; i < LONG_G * M2; i += NT) {
        const int g = i % LONG_G, n2 = i / LONG_G, n1 = n10 + g;
        if (n1 >= M1) continue;
        const cx<T> z = buf[g * M2 + n2];
        const int x = 2 * (n1 + M1 * n2);
        if (x < W) epi(k, y, x, mul_scale(z.x, scale));
        if (x + 1 < W) epi(k, y, x + 1, mul_scale(z.y, scale));
    }
}

// The factor pair of a long row length: M2 the largest divisor with
// LONG_G * M2 <= cap such that M1 = M / M2 fits two to a block (2 M1 <= cap);
// false when M has none.
inline bool long_row_split(int M, int cap, int &M1, int &M2) {
    for (int d = cap / LONG_G; d >= 2; --d)
        if (M % d == 0 && 2 * (M / d) <= cap) {
            M2 = d;
            M1 = M / d;
            return true;
        }
    return false;
}

}  // namespace updc
