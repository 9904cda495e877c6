// Row and column transforms longer than one block's shared memory holds.
//
// Rows (FW/2 above the
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

// ---------------------------------------------------------------------------- long columns
// Columns longer than one block holds (FH above the column capacity): the
// complex FFT of each u-row (column) of length N = N1 * N2, four-step with
// n = n1 + N1 n2 and k = k2 + N2 k1, through a scratch [u][k2][n1]; inputs
// beyond rows_in are zero, outputs past rows_out are not stored.  Pass A
// takes LONG_G consecutive n1 of one column, pass B LONG_G consecutive k2.
struct LongColPlan {
    int N = 0, N1 = 0, N2 = 0;
    FftPlan p1, p2;             // N1- and N2-point plans (no padding)
    const void *twm = nullptr;  // cx<T>[N]: w_N^e
};

// grid (ceil(N1 / LONG_G), columns); LONG_G * N2 complex of shared memory.
template <typename T, int NT, int CAP, bool INV>
__global__ void __launch_bounds__(NT) k_long_col_a(const __grid_constant__ LongColPlan lp, const cx<T> *__restrict__ in,
                                                   int ld_in, int rows_in, cx<T> *__restrict__ scratch) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int N1 = lp.N1, N2 = lp.N2;
    const int n10 = blockIdx.x * LONG_G, u = blockIdx.y;
    const cx<T> *src = in + (size_t)u * ld_in;
    for (int i = threadIdx.x; i < LONG_G * N2; i += NT) {
        const int g = i % LONG_G, n2 = i / LONG_G, n = n10 + g + N1 * n2;
        buf[g * N2 + n2] = (n10 + g < N1 && n < rows_in) ? src[n] : cx<T>{T(0), T(0)};
    }
    __syncthreads();
    fft_batch<INV, NT, CAP, FFT_RMAX, 31>(buf, LONG_G, lp.p2);
    __syncthreads();
    const cx<T> *twm = reinterpret_cast<const cx<T> *>(lp.twm);
    cx<T> *dst = scratch + (size_t)u * lp.N;
    for (int i = threadIdx.x; i < LONG_G * N2; i += NT) {
        const int g = i % LONG_G, k2 = i / LONG_G, n1 = n10 + g;
        if (n1 < N1) dst[(size_t)k2 * N1 + n1] = fmulc(buf[g * N2 + k2], long_twiddle<INV>(twm, lp.N, n1, k2));
    }
}

// grid (ceil(N2 / LONG_G), columns); LONG_G * N1 complex of shared memory.
template <typename T, int NT, int CAP, bool INV>
__global__ void __launch_bounds__(NT) k_long_col_b(const __grid_constant__ LongColPlan lp, const cx<T> *__restrict__ scratch,
                                                   cx<T> *__restrict__ out, int ld_out, int rows_out) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int N1 = lp.N1, N2 = lp.N2;
    const int k20 = blockIdx.x * LONG_G, u = blockIdx.y;
    const cx<T> *src = scratch + (size_t)u * lp.N;
    for (int i = threadIdx.x; i < LONG_G * N1; i += NT) {
        const int g = i / N1, n1 = i - g * N1;
        buf[i] = k20 + g < N2 ? src[(size_t)(k20 + g) * N1 + n1] : cx<T>{T(0), T(0)};
    }
    __syncthreads();
    fft_batch<INV, NT, CAP, FFT_RMAX, 31>(buf, LONG_G, lp.p1);
    __syncthreads();
    cx<T> *dst = out + (size_t)u * ld_out;
    for (int i = threadIdx.x; i < LONG_G * N1; i += NT) {
        const int k1 = i / LONG_G, g = i - k1 * LONG_G, k2 = k20 + g;
        const int k = k2 + N2 * k1;
        if (k2 < N2 && k < rows_out) dst[k] = buf[g * N1 + k1];
    }
}

// Elementwise steps of the long-column forward model and adjoint over
// n = columns x FH values: p = a * b (the OTF product), and the conj-OTF
// accumulation s (+)= conj(K) * v through an accumulator policy (kernels.cuh).
template <typename T>
__global__ void k_long_mul(const cx<T> *__restrict__ a, const cx<T> *__restrict__ b, cx<T> *__restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = cmul(a[i], b[i]);
}
template <typename T, class Acc>
__global__ void k_long_acc(const cx<T> *__restrict__ v, const cx<T> *__restrict__ k, typename Acc::S *__restrict__ s,
                           size_t n, int first) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        typename Acc::S a;
        if (first) Acc::zero(a);
        else a = s[i];
        Acc::add(a, v[i], k[i]);
        s[i] = a;
    }
}
template <typename T, class Acc>
__global__ void k_long_get(const typename Acc::S *__restrict__ s, cx<T> *__restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const auto g = Acc::get(s[i]);
        out[i] = cx<T>{(T)g.x, (T)g.y};
    }
}

// The factor pair of a long column length: N1 and N2 both with
// LONG_G * N <= cap; false when there is none.
inline bool long_col_split(int N, int cap, int &N1, int &N2) {
    for (int d = cap / LONG_G; d >= 2; --d)
        if (N % d == 0 && LONG_G * (N / d) <= cap) {
            N2 = d;
            N1 = N / d;
            return true;
        }
    return false;
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
