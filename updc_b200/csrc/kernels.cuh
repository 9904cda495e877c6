// Kernels of the UPDC iteration (sm_100a).  Spectra are stored "u-major":
// for R2C along x (rows of FW reals -> M+1 = FW/2+1 bins) the bin u of every
// row y is stored at spec[u * ld + y], so each u-row is one contiguous column
// transform.  Only the first H (or rows_in) y-entries of a row-pass
// intermediate are stored: the zero padding rows are never read or written.
#pragma once

#include "common.cuh"
#include "fft.cuh"
#include "tma.cuh"

namespace updc {

// FP32 blocks of <= 512 threads over at most 5632 complex elements are
// compiled for two resident blocks per SM (64 registers a thread); FP64,
// larger transforms and larger blocks for one (their butterflies need up to
// 128 registers).
// Threads per block of the spectral kernels: 512 (two blocks per SM) except
// the FP32 adjoint column kernel, whose accumulator plane limits it to one
// block per SM and which therefore runs 1024 threads (FP64 butterflies need
// the 128-register budget of 512-thread blocks).
constexpr int SPEC_NT = 512;
template <typename T> struct SpecNtAdj {
    static constexpr int value = sizeof(T) == 4 ? 1024 : 512;
};
constexpr size_t SPEC_SMEM_LIMIT = 227 * 1024;
// Threads of the column kernels of the single-field engine: 384 for FP32
// (three blocks per SM; the block's X-hat and adjoint accumulator then live
// in a global scratch that stays in L2), 512 for FP64.  Measured on B200 for
// 5600- and 3584-point columns: 384 threads x 3 blocks is 1.2x faster than
// 512 x 2 and 1.8x faster than 1024 x 1.
template <typename T> struct SpecColNt {
    static constexpr int value = sizeof(T) == 4 ? 384 : 512;
};
// Threads of the single-field engine's row kernels: 256 for FP32 (four
// blocks per SM, which fit because the TMA tile is staged in the FFT
// buffer's memory; measured on c1 against 384 x 3 and 512 x 2: 6.44, 6.53
// and 6.69 ms per iteration), 512 for FP64.
template <typename T> struct SpecRowNt {
    static constexpr int value = sizeof(T) == 4 ? 256 : 512;
};
// Shared-memory capacity (complex elements) of the FFT instantiations.
template <typename T> struct SpecCaps {
    static constexpr int ROW = 5632;
    static constexpr int COL_S = 5632;
    static constexpr int COL_L = 11264;
};

// Blocks per SM a kernel is compiled for (its register budget is
// 65536 / (NT * value)): FP32 transforms of the small capacity run 4, 3 or 2
// blocks of 256, 384 or 512 threads; everything else one block.
template <int NT, int CAP, typename T> struct MinBlocks {
    static constexpr int value =
        (CAP <= 5632 && sizeof(T) == 4) ? (NT <= 256 ? 4 : NT <= 384 ? 3 : NT <= 512 ? 2 : 1) : 1;
};

// ---------------------------------------------------------------------------- loaders
// Real input of the row transform: value of exposure k, row y, column x.
template <typename T> struct PlaneLoader {
    const T *p;
    int pitch;
    size_t batch_stride;
    __device__ __forceinline__ T operator()(int k, int y, int x) const {
        return p[k * batch_stride + (size_t)y * pitch + x];
    }
};

// Centre-wrapped, normalised PSF on the FW x FH grid (updc_core.c:813-821):
// PSF pixel (x, y) goes to ((x - fw/2) mod FW, (y - fh/2) mod FH); with
// transposed storage the source index is x*pw + y.
template <typename T, typename P = float> struct PsfLoader {
    const P *psf;
    int pw, fwid, fhei, FW, FH, transposed;
    T inv;
    __device__ __forceinline__ T operator()(int, int yy, int xx) const {
        const int y = (yy + fhei / 2) % FH, x = (xx + fwid / 2) % FW;
        if (y >= fhei || x >= fwid) return T(0);
        const size_t src = transposed ? (size_t)x * pw + y : (size_t)y * pw + x;
        return mul_rn((T)psf[src], inv);
    }
    __device__ __forceinline__ static float mul_rn(float a, float b) { return __fmul_rn(a, b); }
    __device__ __forceinline__ static double mul_rn(double a, double b) { return __dmul_rn(a, b); }
};

// The u-major side of a row transform: either plain loads/stores at
// spec[k*batch_stride + u*ld + y] (TMA = false) or a 3-D tensor map over the
// same array (TMA = true, 8-byte elements, box {B*EW, TMA_UBOX, 1}).
constexpr int TMA_UBOX = 256;
template <typename T> struct TmaElems {
    static constexpr int value = sizeof(cx<T>) / 8;  // 8-byte tensor elements per complex value
};
struct SpecRef {
    void *p;
    int ld;
    size_t batch_stride;
};

// Shared layout of a row kernel: the FFT buffer (B*M complex) and, with TMA,
// a staging tile of nbox*ubox*B complex (ubox = min(256, M+1) u-rows a box).
// FFT radices are limited to 16 (register budget of 64 per thread).
constexpr int FFT_RMAX = 16;
__host__ __device__ inline size_t fft_buf_bytes(int count, size_t csize, int shift) {
    return ((size_t)fpad_size(count, shift) * csize + 127) / 128 * 128;
}
__host__ __device__ inline size_t row_buf_bytes(int B, int M, size_t csize, int shift) { return fft_buf_bytes(B * M, csize, shift); }
__host__ __device__ inline int row_ubox(int M) { return M + 1 < TMA_UBOX ? M + 1 : TMA_UBOX; }
__host__ __device__ inline int row_nbox(int M) { return (M + 1 + row_ubox(M) - 1) / row_ubox(M); }
__host__ __device__ inline size_t row_stage_bytes(int B, int M, size_t csize) {
    return (size_t)row_nbox(M) * row_ubox(M) * B * csize;
}

// Division by the rows of a row tile: by a compile-time B where the kernel is
// compiled for one (BR > 0), else with the runtime divisor.
template <int BR> __device__ __forceinline__ int div_rows(const FastDiv &d, int q) {
    if constexpr (BR > 0) return q / BR;
    else return (int)d.div((uint32_t)q);
}

// ---------------------------------------------------------------------------- TMA tiles in place
// With TMA the row kernels stage the block's u-major tile ({all bins} x {B
// rows}, box by box) in the same shared memory as the FFT buffer: every
// thread first reads what it needs into registers (its bin pairs u, M - u),
// the block synchronises, and only then is the region overwritten in the
// other layout.  Shared memory is the larger of the two layouts, not their
// sum, so three blocks of 384 threads fit per SM.
// Most bin pairs one thread holds: (M/2 + 1) * B <= CAP/2 + B with B <= 256.
template <int CAP, int NT> struct RowPairs {
    static constexpr int value = (CAP / 2 + 256 + NT - 1) / NT;
};
__host__ __device__ inline size_t row_tma_smem(int B, int M, size_t csize, int shift) {
    const size_t a = row_buf_bytes(B, M, csize, shift), b = row_stage_bytes(B, M, csize);
    return a > b ? a : b;
}

// Bin u of row b of the R2C output from the half-length FFT in buf.
template <typename T>
__device__ __forceinline__ cx<T> r2c_bin(const cx<T> *buf, int row0, int u, int M, int sh, const cx<T> *post) {
    const T half = T(0.5);
    const cx<T> Z = buf[fpad(row0 + (u == M ? 0 : u), sh)];
    const cx<T> Zm = buf[fpad(row0 + (u == 0 ? 0 : M - u), sh)];
    const cx<T> Zc = {Zm.x, -Zm.y};
    const cx<T> E = {half * (Z.x + Zc.x), half * (Z.y + Zc.y)};
    const cx<T> D = {half * (Z.x - Zc.x), half * (Z.y - Zc.y)};
    const cx<T> P = fmulc(D, post[u]);
    return {E.x + P.y, E.y - P.x};
}

template <typename T, int NT, int CAP, int BR = 0>
__device__ __forceinline__ void row_r2c_store_tma(cx<T> *buf, const cx<T> *__restrict__ post, int M, int sh, int B,
                                                  int nb, FastDiv bdiv, const CUtensorMap *omap, int y0, int kexp) {
    if constexpr (BR > 0) B = BR;
    constexpr int KP = RowPairs<CAP, NT>::value;
    const int npairs = (M / 2 + 1) * B;
    cx<T> xa[KP], xb[KP];
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        const int q = threadIdx.x + j * NT;
        xa[j] = xb[j] = cx<T>{T(0), T(0)};
        if (q < npairs) {
            const int u = div_rows<BR>(bdiv, q), b = q - u * B;
            if (b < nb) {
                xa[j] = r2c_bin(buf, b * M, u, M, sh, post);
                xb[j] = r2c_bin(buf, b * M, M - u, M, sh, post);
            }
        }
    }
    __syncthreads();  // the FFT buffer is read; it becomes the staging tile
    cx<T> *stage = buf;
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        const int q = threadIdx.x + j * NT;
        if (q < npairs) {
            const int u = div_rows<BR>(bdiv, q), b = q - u * B;
            stage[u * B + b] = xa[j];
            if (M - u != u) stage[(M - u) * B + b] = xb[j];
        }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
        constexpr int EW = TmaElems<T>::value;
        const int ub = row_ubox(M);
        for (int bx = 0; bx < row_nbox(M); ++bx)
            tma_store_3d(omap, stage + (size_t)bx * ub * B, y0 * EW, bx * ub, kexp);
        tma_store_commit_and_wait();
    }
}

// Inputs k and M - k of the C2R's half-length FFT from bins X[k], X[M-k].
template <typename T>
__device__ __forceinline__ cx<T> c2r_input(cx<T> X, cx<T> Xm, int k, const cx<T> *post) {
    if (k == 0) {
        X.y = 0;
        Xm.y = 0;
    }
    const cx<T> S = {X.x + Xm.x, X.y - Xm.y};
    const cx<T> D = {X.x - Xm.x, X.y + Xm.y};
    const cx<T> w = post[k];
    const cx<T> Q = fmulc_conj(D, w);
    return {S.x - Q.y, S.y + Q.x};
}

// ---------------------------------------------------------------------------- row R2C
// Rows [0, rows) of the real plane, zero-padded from W to FW = 2M columns,
// transformed along x with an M-point complex FFT of z[m] = x[2m] + i x[2m+1]
// and the split z -> X post-processing; bins are stored u-major.  Exposure =
// blockIdx.y.
// One block's tile: rows [y0, y0 + B) of plane `kexp`.  The block-level
// body shared by the single-field kernel and the batched one (batch.cuh).
template <typename T, int NT, int CAP, class Loader, bool TMA, int PADSH = -1, int BR = 0>
__device__ __forceinline__ void row_r2c_tile(const FftPlan &plan, const cx<T> *__restrict__ post, const Loader &ld,
                                             int W, int rows, int B, FastDiv bdiv, SpecRef out,
                                             const CUtensorMap *omap, int y0, int kexp, unsigned char *smem_raw) {
    if constexpr (BR > 0) B = BR;
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int M = plan.n, sh = plan_shift<PADSH>(plan);
    const int nb = min(B, rows - y0);
    for (int b = 0; b < B; ++b)
        for (int m = threadIdx.x; m < M; m += NT) {
            T a = 0, c = 0;
            if (b < nb) {
                const int x = 2 * m;
                if (x < W) a = ld(kexp, y0 + b, x);
                if (x + 1 < W) c = ld(kexp, y0 + b, x + 1);
            }
            buf[fpad(b * M + m, sh)] = {a, c};
        }
    __syncthreads();
    fft_batch<false, NT, CAP, FFT_RMAX, PADSH>(buf, B, plan);
    if constexpr (TMA) {
        row_r2c_store_tma<T, NT, CAP, BR>(buf, post, M, sh, B, nb, bdiv, omap, y0, kexp);
        return;
    }
    cx<T> *dst = reinterpret_cast<cx<T> *>(out.p) + kexp * out.batch_stride;
    const T half = T(0.5);
    for (int i = threadIdx.x; i < (M + 1) * B; i += NT) {
        const int u = div_rows<BR>(bdiv, i), b = i - u * B;
        cx<T> X = {0, 0};
        if (b < nb) {
            const cx<T> Z = buf[fpad(b * M + (u == M ? 0 : u), sh)];
            const cx<T> Zm = buf[fpad(b * M + (u == 0 ? 0 : M - u), sh)];
            const cx<T> Zc = {Zm.x, -Zm.y};
            const cx<T> E = {half * (Z.x + Zc.x), half * (Z.y + Zc.y)};
            const cx<T> D = {half * (Z.x - Zc.x), half * (Z.y - Zc.y)};
            const cx<T> P = fmulc(D, post[u]);
            X = {E.x + P.y, E.y - P.x};
        }
        if (b < nb) dst[(size_t)u * out.ld + y0 + b] = X;
    }
}

template <typename T, int NT, int CAP, class Loader, bool TMA, int PADSH = -1, int BR = 0>
__global__ void __launch_bounds__(NT, MinBlocks<NT, CAP, T>::value)
    k_row_r2c(const __grid_constant__ FftPlan plan, const cx<T> *__restrict__ post, Loader ld, int W, int rows, int B,
              FastDiv bdiv, SpecRef out, const __grid_constant__ CUtensorMap omap) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    row_r2c_tile<T, NT, CAP, Loader, TMA, PADSH, BR>(plan, post, ld, W, rows, BR > 0 ? BR : B, bdiv, out, &omap,
                                                     blockIdx.x * (BR > 0 ? BR : B), blockIdx.y, smem_raw);
}

// ---------------------------------------------------------------------------- row C2R
__device__ __forceinline__ float mul_scale(float a, float s) { return __fmul_rn(a, s); }
__device__ __forceinline__ double mul_scale(double a, double s) { return __dmul_rn(a, s); }
template <typename T> struct PlaneStore {
    T *p;
    int pitch;
    size_t batch_stride;
    __device__ __forceinline__ void operator()(int k, int y, int x, T v) const { p[k * batch_stride + (size_t)y * pitch + x] = v; }
};

// Inverse of k_row_r2c for rows [0, rows): bins u-major in `in`, output
// x in [0, W) of each row times `scale` (the crop of updc_core.c:765-766).
// The imaginary parts of the DC and Nyquist bins are ignored, as FFTW does.
// With TMA the block's {B rows} x {all u} tile arrives through the tensor map.
template <typename T, int NT, int CAP, class Epi, bool TMA, int PADSH = -1, int BR = 0>
__device__ __forceinline__ void row_c2r_tile(const FftPlan &plan, const cx<T> *__restrict__ post, SpecRef in,
                                             const CUtensorMap *imap, int rows, int W, int B, FastDiv bdiv, T scale,
                                             const Epi &epi, unsigned long long *__restrict__ err, int y0, int kexp,
                                             unsigned char *smem_raw) {
    if constexpr (BR > 0) B = BR;
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    __shared__ __align__(8) uint64_t bar;
    const int M = plan.n, sh = plan_shift<PADSH>(plan);
    const int nb = min(B, rows - y0);
    cx<T> *stage = buf;  // TMA: the tile arrives in the FFT buffer's memory
    const cx<T> *src = reinterpret_cast<const cx<T> *>(in.p) + kexp * in.batch_stride;
    if (TMA) {
        if (threadIdx.x == 0) mbar_init(&bar, 1);
        __syncthreads();
        if (threadIdx.x == 0) {
            constexpr int EW = TmaElems<T>::value;
            const int nbox = row_nbox(M), ub = row_ubox(M);
            mbar_arrive_expect_tx(&bar, (uint32_t)row_stage_bytes(B, M, sizeof(cx<T>)));
            for (int bx = 0; bx < nbox; ++bx)
                tma_load_3d(stage + (size_t)bx * ub * B, imap, &bar, y0 * EW, bx * ub, kexp);
        }
        // every thread's wait is bounded; the block then decides together
        // (one barrier vote), so either all of it goes on or all of it returns
        const bool arrived = mbar_wait_bounded(&bar, 0);
        if (__syncthreads_or(!arrived)) {
            if (threadIdx.x == 0)
                atomicMin(err, (unsigned long long)make_error_key(STAGE_TRANSFORM, blockIdx.x, ERR_DEVICE_TIMEOUT));
            return;
        }
        // pairs (k, M - k): both inputs read into registers, then the tile's
        // memory is overwritten with the FFT buffer
        constexpr int KP = RowPairs<CAP, NT>::value;
        const int npairs = (M / 2 + 1) * B;
        cx<T> za[KP], zb[KP];
#pragma unroll
        for (int j = 0; j < KP; ++j) {
            const int q = threadIdx.x + j * NT;
            za[j] = zb[j] = cx<T>{T(0), T(0)};
            if (q < npairs) {
                const int k = div_rows<BR>(bdiv, q), b = q - k * B;
                if (b < nb) {
                    const cx<T> X = stage[k * B + b], Xm = stage[(M - k) * B + b];
                    za[j] = c2r_input(X, Xm, k, post);
                    if (k > 0) zb[j] = c2r_input(Xm, X, M - k, post);
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < KP; ++j) {
            const int q = threadIdx.x + j * NT;
            if (q < npairs) {
                const int k = div_rows<BR>(bdiv, q), b = q - k * B;
                buf[fpad(b * M + k, sh)] = za[j];
                if (k > 0 && M - k != k) buf[fpad(b * M + M - k, sh)] = zb[j];
            }
        }
    } else {
        for (int i = threadIdx.x; i < M * B; i += NT) {
            const int k = div_rows<BR>(bdiv, i), b = i - k * B;
            cx<T> Zp = {0, 0};
            if (b < nb) Zp = c2r_input(src[(size_t)k * in.ld + y0 + b], src[(size_t)(M - k) * in.ld + y0 + b], k, post);
            buf[fpad(b * M + k, sh)] = Zp;
        }
    }
    __syncthreads();
    fft_batch<true, NT, CAP, FFT_RMAX, PADSH>(buf, B, plan);
    for (int b = 0; b < nb; ++b)
        for (int x = threadIdx.x; x < W; x += NT) {
            const cx<T> z = buf[fpad(b * M + (x >> 1), sh)];
            epi(kexp, y0 + b, x, mul_scale((x & 1) ? z.y : z.x, scale));
        }
}

template <typename T, int NT, int CAP, class Epi, bool TMA, int PADSH = -1, int BR = 0>
__global__ void __launch_bounds__(NT, MinBlocks<NT, CAP, T>::value)
    k_row_c2r(const __grid_constant__ FftPlan plan, const cx<T> *__restrict__ post, SpecRef in,
              const __grid_constant__ CUtensorMap imap, int rows, int W, int B, FastDiv bdiv, T scale, Epi epi,
              unsigned long long *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    row_c2r_tile<T, NT, CAP, Epi, TMA, PADSH, BR>(plan, post, in, &imap, rows, W, BR > 0 ? BR : B, bdiv, scale, epi,
                                                  err, blockIdx.x * (BR > 0 ? BR : B), blockIdx.y, smem_raw);
}


// ---------------------------------------------------------------------------- columns
// Forward model for every exposure from the estimate's row-pass intermediate:
//   Xhat[u] = FFT_y(Rx[u]);  Y_k[u] = IFFT_y(Xhat[u] * K_k[u]) for y < rows_out.
// The product is (ac - bd, ad + bc) (updc_core.c:753-759).  Xhat never leaves
// the block: it is kept in shared memory (or in `aux` when it does not fit).
// All transforms go through one forward-FFT call site; the inverse is
// conj(FFT(conj(.))), which keeps a single inlined copy of the FFT (two
// copies make ptxas spill).
// Asks L2 to fetch [p, p + bytes) of this GPU's memory ahead of its use
// (bulk prefetch, no destination; the range is rounded inwards to 16 bytes).
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
    uintptr_t a = (uintptr_t)p, e = a + bytes;
    a = (a + 15) & ~(uintptr_t)15;
    e &= ~(uintptr_t)15;
    if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(e - a)) : "memory");
}

// Evict-first (ld.global.cs / st.global.cs) accesses of complex values read
// or written once: the column kernels' input spectra, OTF columns and
// outputs, so the L2 keeps X-hat and the FP64 accumulator (forward y 0.54 ->
// 0.52 ms, adjoint 0.85 -> 0.83 ms on the 5040-point columns of the
// 8 x 2048^2 -> 4096^2 field).
__device__ __forceinline__ cx<float> ldcs_cx(const cx<float> *p) {
    const float2 v = __ldcs(reinterpret_cast<const float2 *>(p));
    return {v.x, v.y};
}
__device__ __forceinline__ void stcs_cx(cx<float> *p, cx<float> v) {
    __stcs(reinterpret_cast<float2 *>(p), make_float2(v.x, v.y));
}

// L2 evict-last accesses (createpolicy + .L2::cache_hint) of the data a
// kernel re-reads while it streams read-once inputs past it: the compiled
// column adjoint's FP64 accumulator (adjoint 0.83 -> 0.75 ms on the
// 5040-point columns of the 8 x 2048^2 -> 4096^2 field) and the weighted
// ratio plane the fused gather reads at random (1.16 -> 1.14 ms).  The
// run-time-plan column adjoint keeps plain accumulator accesses: with them
// evict-last, 16 exposures of 8960-point columns took 12.5 ms instead of
// 10.3 ms.
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
template <typename S> __device__ __forceinline__ S ld_keep(const S *p) {
    if constexpr (sizeof(S) == 16) {
        double a, b;
        asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                     : "=d"(a), "=d"(b)
                     : "l"(p), "l"(l2_evict_last_policy()));
        S r;
        memcpy(&r, &a, 8);
        memcpy(reinterpret_cast<char *>(&r) + 8, &b, 8);
        return r;
    } else if constexpr (sizeof(S) == 8) {
        float a, b;
        asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                     : "=f"(a), "=f"(b)
                     : "l"(p), "l"(l2_evict_last_policy()));
        S r;
        memcpy(&r, &a, 4);
        memcpy(reinterpret_cast<char *>(&r) + 4, &b, 4);
        return r;
    } else {
        return *p;
    }
}
template <typename S> __device__ __forceinline__ void st_keep(S *p, const S &v) {
    if constexpr (sizeof(S) == 16) {
        double a, b;
        memcpy(&a, &v, 8);
        memcpy(&b, reinterpret_cast<const char *>(&v) + 8, 8);
        asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(a), "d"(b),
                     "l"(l2_evict_last_policy())
                     : "memory");
    } else if constexpr (sizeof(S) == 8) {
        float a, b;
        memcpy(&a, &v, 4);
        memcpy(&b, reinterpret_cast<const char *>(&v) + 4, 4);
        asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(a), "f"(b),
                     "l"(l2_evict_last_policy())
                     : "memory");
    } else {
        *p = v;
    }
}
__device__ __forceinline__ float ld_keep_f(const float *p) {
    float v;
    asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(l2_evict_last_policy()));
    return v;
}
// The evict-first accesses, or plain ones when POL is false (FP64 form,
// batched fields).
template <bool POL, typename T> __device__ __forceinline__ cx<T> ld_once(const cx<T> *p) {
    if constexpr (POL && sizeof(T) == 4) return ldcs_cx(p);
    else return *p;
}
template <bool POL, typename T> __device__ __forceinline__ void st_once(cx<T> *p, cx<T> v) {
    if constexpr (POL && sizeof(T) == 4) stcs_cx(p, v);
    else *p = v;
}

// AUX = 1: the caller guarantees `aux` (global scratch) is given, so its
// accesses compile to global loads and stores; AUX = 0 decides at run time
// between `aux` and shared memory (generic accesses).
template <typename T, int NT, int CAP, int AUX = 0, int PADSH = -1>
__device__ __forceinline__ void col_forward_column(const FftPlan &plan, const cx<T> *__restrict__ rx, int ldr,
                                                   int rows_in, const cx<T> *__restrict__ khat, size_t khat_stride,
                                                   int nexp, cx<T> *__restrict__ y, int ldy, size_t y_stride,
                                                   int rows_out, cx<T> *aux, int u, unsigned char *smem_raw) {
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int n = plan.n, sh = plan_shift<PADSH>(plan);
    constexpr bool POL = AUX == 1 && sizeof(T) == 4;  // L2 policies (scratch known to be global)
    cx<T> *xh;
    if constexpr (AUX == 1) xh = aux + (size_t)u * n;
    else xh = aux ? aux + (size_t)u * n : reinterpret_cast<cx<T> *>(smem_raw + fft_buf_bytes(n, sizeof(cx<T>), sh));
    const cx<T> *src = rx + (size_t)u * ldr;
#pragma unroll 1
    for (int it = 0; it <= nexp; ++it) {
        // the OTF column of the next exposure is fetched into L2 during this FFT
        if (threadIdx.x == 0 && it < nexp) prefetch_l2(khat + it * khat_stride + (size_t)u * n, (size_t)n * sizeof(cx<T>));
        if (it == 0) {
            for (int v = threadIdx.x; v < n; v += NT) buf[fpad(v, sh)] = v < rows_in ? ld_once<POL>(src + v) : cx<T>{0, 0};
        } else {
            const cx<T> *kr = khat + (it - 1) * khat_stride + (size_t)u * n;
            for (int v = threadIdx.x; v < n; v += NT) {
                const cx<T> p = cmul(xh[v], ld_once<POL>(kr + v));
                buf[fpad(v, sh)] = {p.x, -p.y};
            }
        }
        __syncthreads();
        fft_batch<false, NT, CAP, FFT_RMAX, PADSH>(buf, 1, plan);
        if (it == 0) {
            for (int v = threadIdx.x; v < n; v += NT) st_once<POL>(xh + v, buf[fpad(v, sh)]);
        } else {
            cx<T> *dst = y + (it - 1) * y_stride + (size_t)u * ldy;
            for (int v = threadIdx.x; v < rows_out; v += NT) {
                const cx<T> q = buf[fpad(v, sh)];
                st_once<POL>(dst + v, cx<T>{q.x, -q.y});
            }
        }
        __syncthreads();
    }
}

template <typename T, int NT, int CAP, int AUX = 0, int PADSH = -1>
__global__ void __launch_bounds__(NT, (MinBlocks<NT, CAP, T>::value)) k_col_forward(const __grid_constant__ FftPlan plan, const cx<T> *__restrict__ rx, int ldr, int rows_in,
                                                    const cx<T> *__restrict__ khat, size_t khat_stride, int nexp,
                                                    cx<T> *__restrict__ y, int ldy, size_t y_stride, int rows_out,
                                                    int nu, cx<T> *aux) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    (void)nu;
    col_forward_column<T, NT, CAP, AUX, PADSH>(plan, rx, ldr, rows_in, khat, khat_stride, nexp, y, ldy, y_stride, rows_out,
                                        aux, blockIdx.x, smem_raw);
}

// Cross-exposure accumulation policies for the adjoint sum
//   acc += (a c + b d, b c - a d)   (updc_core.c:988-995)
template <typename T> struct AccPlain {  // reference order, working precision
    using S = cx<T>;
    __device__ __forceinline__ static void zero(S &s) { s = {0, 0}; }
    __device__ __forceinline__ static void add(S &s, cx<float> a, cx<float> c) {
        s.x = __fadd_rn(s.x, __fadd_rn(__fmul_rn(a.x, c.x), __fmul_rn(a.y, c.y)));
        s.y = __fadd_rn(s.y, __fsub_rn(__fmul_rn(a.y, c.x), __fmul_rn(a.x, c.y)));
    }
    __device__ __forceinline__ static void add(S &s, cx<double> a, cx<double> c) {
        s.x = __dadd_rn(s.x, __dadd_rn(__dmul_rn(a.x, c.x), __dmul_rn(a.y, c.y)));
        s.y = __dadd_rn(s.y, __dsub_rn(__dmul_rn(a.y, c.x), __dmul_rn(a.x, c.y)));
    }
    __device__ __forceinline__ static cx<T> get(const S &s) { return s; }
};
struct AccF64 {  // FP32 operands, FP64 products and sum
    using S = cx<double>;
    __device__ __forceinline__ static void zero(S &s) { s = {0, 0}; }
    __device__ __forceinline__ static void add(S &s, cx<float> a, cx<float> c) {
        const double ax = a.x, ay = a.y, cxr = c.x, cy = c.y;
        s.x += ax * cxr + ay * cy;
        s.y += ay * cxr - ax * cy;
    }
    __device__ __forceinline__ static cx<float> get(const S &s) { return {(float)s.x, (float)s.y}; }
};
struct AccKahan {  // FP32 products, Kahan-compensated FP32 sum
    struct S { float sx, cx_, sy, cy; };
    __device__ __forceinline__ static void zero(S &s) { s = {0, 0, 0, 0}; }
    __device__ __forceinline__ static void kadd(float &sum, float &c, float v) {
        const float y = __fsub_rn(v, c);
        const float t = __fadd_rn(sum, y);
        c = __fsub_rn(__fsub_rn(t, sum), y);
        sum = t;
    }
    __device__ __forceinline__ static void add(S &s, cx<float> a, cx<float> c) {
        kadd(s.sx, s.cx_, __fadd_rn(__fmul_rn(a.x, c.x), __fmul_rn(a.y, c.y)));
        kadd(s.sy, s.cy, __fsub_rn(__fmul_rn(a.y, c.x), __fmul_rn(a.x, c.y)));
    }
    __device__ __forceinline__ static cx<float> get(const S &s) { return {s.sx, s.sy}; }
};

// Adjoint for every exposure:  C[u] = IFFT_y( sum_k conj(K_k[u]) * FFT_y(Rs_k[u]) )
// for y < rows_out.  The sum over k runs in exposure order inside the block;
// the final inverse goes through the same forward-FFT call site as
// conj(FFT(conj(.))).
template <typename T, class Acc, int NT, int CAP, int AUX = 0, int PADSH = -1>
__device__ __forceinline__ void col_adjoint_column(const FftPlan &plan, const cx<T> *__restrict__ rs, int ldr,
                                                   size_t rs_stride, int rows_in, const cx<T> *__restrict__ khat,
                                                   size_t khat_stride, int nexp, cx<T> *__restrict__ c, int ldc,
                                                   int rows_out, typename Acc::S *aux, int u, unsigned char *smem_raw) {
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int n = plan.n, sh = plan_shift<PADSH>(plan);
    typename Acc::S *acc;
    if constexpr (AUX == 1) acc = aux + (size_t)u * n;
    else acc = aux ? aux + (size_t)u * n
                   : reinterpret_cast<typename Acc::S *>(smem_raw + fft_buf_bytes(n, sizeof(cx<T>), sh));
    for (int v = threadIdx.x; v < n; v += NT) Acc::zero(acc[v]);
#pragma unroll 1
    for (int it = 0; it <= nexp; ++it) {
        if (it < nexp) {
            const cx<T> *src = rs + it * rs_stride + (size_t)u * ldr;
            for (int v = threadIdx.x; v < n; v += NT) buf[fpad(v, sh)] = v < rows_in ? src[v] : cx<T>{0, 0};
        } else {
            for (int v = threadIdx.x; v < n; v += NT) {
                const cx<T> a = Acc::get(acc[v]);
                buf[fpad(v, sh)] = {a.x, -a.y};
            }
        }
        __syncthreads();
        fft_batch<false, NT, CAP, FFT_RMAX, PADSH>(buf, 1, plan);
        if (it < nexp) {
            const cx<T> *kr = khat + it * khat_stride + (size_t)u * n;
            for (int v = threadIdx.x; v < n; v += NT) Acc::add(acc[v], buf[fpad(v, sh)], kr[v]);
        } else {
            cx<T> *dst = c + (size_t)u * ldc;
            for (int v = threadIdx.x; v < rows_out; v += NT) {
                const cx<T> q = buf[fpad(v, sh)];
                dst[v] = {q.x, -q.y};
            }
        }
        __syncthreads();
    }
}

template <typename T, class Acc, int NT, int CAP, int AUX = 0, int PADSH = -1>
__global__ void __launch_bounds__(NT, (MinBlocks<NT, CAP, T>::value)) k_col_adjoint(const __grid_constant__ FftPlan plan, const cx<T> *__restrict__ rs, int ldr, size_t rs_stride,
                                                    int rows_in, const cx<T> *__restrict__ khat, size_t khat_stride, int nexp,
                                                    cx<T> *__restrict__ c, int ldc, int rows_out, typename Acc::S *aux) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    col_adjoint_column<T, Acc, NT, CAP, AUX, PADSH>(plan, rs, ldr, rs_stride, rows_in, khat, khat_stride, nexp, c, ldc,
                                             rows_out, aux, blockIdx.x, smem_raw);
}

// Plain column transform (setup: PSF spectra and generic 2-D transforms).
template <typename T, int NT, int CAP, bool INV, int PADSH = -1>
__global__ void __launch_bounds__(NT, (MinBlocks<NT, CAP, T>::value)) k_col_fft(const __grid_constant__ FftPlan plan, const cx<T> *__restrict__ in, int ldi, int rows_in,
                                                cx<T> *__restrict__ out, int ldo, int rows_out) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<T> *buf = reinterpret_cast<cx<T> *>(smem_raw);
    const int n = plan.n, sh = plan_shift<PADSH>(plan);
    const int u = blockIdx.x;
    const cx<T> *src = in + (size_t)u * ldi;
    for (int v = threadIdx.x; v < n; v += NT) buf[fpad(v, sh)] = v < rows_in ? src[v] : cx<T>{0, 0};
    __syncthreads();
    fft_batch<INV, NT, CAP, FFT_RMAX, PADSH>(buf, 1, plan);
    cx<T> *dst = out + (size_t)u * ldo;
    for (int v = threadIdx.x; v < rows_out; v += NT) dst[v] = buf[fpad(v, sh)];
}

}  // namespace updc
