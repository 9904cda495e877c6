// FP32 iteration kernels on compile-time transforms (fft_ct.cuh).
//
// Same data flow and arithmetic order as kernels.cuh (u-major spectra, crop
// and 1/nf in the C2R, the (ac - bd, ad + bc) OTF product, the conj-OTF sum
// in exposure order), but the transform length and radix sequence are
// template arguments, and the transforms read their first stage straight
// from global memory and write their last stage straight to global memory
// where the data allow it:
//   * column forward: the row-pass column (zero padded) or the product
//     X-hat * K_k in, X-hat or the cropped inverse out;
//   * column adjoint: the scatter spectrum column in, the conj-OTF product
//     accumulated straight into the column's accumulator; then the
//     accumulator in and the cropped inverse out;
//   * row R2C: the real plane in (two reals per complex point); the last
//     stage stays in shared memory for the split post-processing;
//   * row C2R: the last stage writes the cropped, scaled real row.
// Inverse transforms are conj(FFT(conj(.))), so each kernel inlines one
// forward transform.
#pragma once

#include <vector>

#include "fft_ct.cuh"
#include "kernels.cuh"

namespace updc {

// A compile-time radix list (the catalog's entries).
template <int... R> struct CtRadices {
    static constexpr int n = CtProd<R...>::value;
    static constexpr int stages = sizeof...(R);
};

// First stage, then every other stage in place (the last one included).
template <int BATCH, int NT, bool INV, typename T, int R0, int... R, class In>
__device__ __forceinline__ void ct_fft_in(const In &in, cx<T> *buf, const cx<T> *__restrict__ tw) {
    constexpr int N = CtProd<R0, R...>::value;
    ct_first<R0, N, BATCH, NT, INV, T>(in, buf);
    CtStages<N, BATCH, NT, INV, T, R0, R0 - 1, R...>::run(buf, tw);
}

// Every stage but the last in place, the last one through `out`.
template <int BATCH, int NT, bool INV, typename T, int... R, class Out>
__device__ __forceinline__ void ct_fft_out(cx<T> *buf, const cx<T> *__restrict__ tw, const Out &out) {
    CtTail<CtProd<R...>::value, BATCH, NT, INV, T, 1, 0, Out, R...>::run(buf, tw, out);
}

// ---------------------------------------------------------------------------- row R2C
// Complex point m of a row tile's row b: (x[2m], x[2m+1]) of plane row y0+b,
// zero beyond W and beyond the plane's rows.
struct RowPairIn {
    const float *plane;  // this plane's row y0
    int pitch, W, nb;
    bool even;           // W and pitch even: one 8-byte load per point
    __device__ __forceinline__ cx<float> operator()(int b, int m) const {
        const int x = 2 * m;
        if (b >= nb || x >= W) return {0.f, 0.f};
        const float *p = plane + (size_t)b * pitch + x;
        if (even) {
            const float2 v = *reinterpret_cast<const float2 *>(p);
            return {v.x, v.y};
        }
        return {p[0], x + 1 < W ? p[1] : 0.f};
    }
};

template <int NT, int BR, int... R>
__global__ void __launch_bounds__(NT, 4)
    k_row_r2c_ct(const cx<float> *__restrict__ post, const float *__restrict__ planes, int W, int rows,
                 size_t plane_stride, const cx<float> *__restrict__ tw, const __grid_constant__ CUtensorMap omap) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int M = CtProd<R...>::value;
    cx<float> *buf = reinterpret_cast<cx<float> *>(smem_raw);
    const int y0 = blockIdx.x * BR, kexp = blockIdx.y;
    const int nb = min(BR, rows - y0);
    const RowPairIn in{planes + kexp * plane_stride + (size_t)y0 * W, W, W, nb, (W & 1) == 0};
    ct_fft_in<BR, NT, false, float, R...>(in, buf, tw);
    row_r2c_store_tma<float, NT, BR * M, BR>(buf, post, M, 31, BR, nb, FastDiv(), &omap, y0, kexp);
}

// ---------------------------------------------------------------------------- row C2R
// Output point m of row b: reals 2m and 2m+1 times the scale, kept for
// x < W and rows of the plane.
struct RowPairOut {
    float *plane;  // this plane's row y0
    int pitch, W, nb;
    float scale;
    bool even;
    __device__ __forceinline__ void operator()(int b, int m, cx<float> v) const {
        const int x = 2 * m;
        if (b >= nb || x >= W) return;
        float *p = plane + (size_t)b * pitch + x;
        const float a = __fmul_rn(v.x, scale), c = __fmul_rn(v.y, scale);
        if (even) {
            *reinterpret_cast<float2 *>(p) = make_float2(a, c);
        } else {
            p[0] = a;
            if (x + 1 < W) p[1] = c;
        }
    }
};

template <int NT, int BR, int... R>
__global__ void __launch_bounds__(NT, 4)
    k_row_c2r_ct(const cx<float> *__restrict__ post, const __grid_constant__ CUtensorMap imap, int rows, int W,
                 float scale, float *__restrict__ planes, size_t plane_stride, const cx<float> *__restrict__ tw,
                 unsigned long long *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int M = CtProd<R...>::value;
    constexpr int B = BR;
    cx<float> *buf = reinterpret_cast<cx<float> *>(smem_raw);
    __shared__ __align__(8) uint64_t bar;
    const int y0 = blockIdx.x * B, kexp = blockIdx.y;
    const int nb = min(B, rows - y0);
    // the block's {B rows} x {all u} tile arrives through the tensor map into
    // the transform buffer's memory
    cx<float> *stage = buf;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nbox = row_nbox(M), ub = row_ubox(M);
        mbar_arrive_expect_tx(&bar, (uint32_t)row_stage_bytes(B, M, sizeof(cx<float>)));
        for (int bx = 0; bx < nbox; ++bx) tma_load_3d(stage + (size_t)bx * ub * B, &imap, &bar, y0, bx * ub, kexp);
    }
    const bool arrived = mbar_wait_bounded(&bar, 0);
    if (__syncthreads_or(!arrived)) {
        if (threadIdx.x == 0)
            atomicMin(err, (unsigned long long)make_error_key(STAGE_TRANSFORM, blockIdx.x, ERR_DEVICE_TIMEOUT));
        return;
    }
    // pairs (k, M - k) of the half-length transform's input, read into
    // registers before the tile's memory becomes the transform buffer
    constexpr int NPAIRS = (M / 2 + 1) * B;
    constexpr int KP = (NPAIRS + NT - 1) / NT;
    cx<float> za[KP], zb[KP];
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        const int q = threadIdx.x + j * NT;
        za[j] = zb[j] = cx<float>{0.f, 0.f};
        if (q < NPAIRS) {
            const int k = q / B, b = q - k * B;
            if (b < nb) {
                const cx<float> X = stage[k * B + b], Xm = stage[(M - k) * B + b];
                za[j] = c2r_input(X, Xm, k, post);
                if (k > 0) zb[j] = c2r_input(Xm, X, M - k, post);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < KP; ++j) {
        const int q = threadIdx.x + j * NT;
        if (q < NPAIRS) {
            const int k = q / B, b = q - k * B;
            buf[b * M + k] = za[j];
            if (k > 0 && M - k != k) buf[b * M + M - k] = zb[j];
        }
    }
    __syncthreads();
    const RowPairOut out{planes + kexp * plane_stride + (size_t)y0 * W, W, W, nb, scale, (W & 1) == 0};
    ct_fft_out<B, NT, true, float, R...>(buf, tw, out);
}

// ---------------------------------------------------------------------------- columns
constexpr int CT_COL_NT = 384;

// Column forward model: transform 0 is FFT(pad(rx[u])) -> X-hat (global
// scratch, L2-resident); transform it >= 1 is IFFT(X-hat * K_{it-1}) for
// rows < rows_out, computed as conj(FFT(conj(.))).  Every transform's input
// is staged in shared memory by all threads together (the product's two
// loads per element in flight at once), the stages run in place, and the last
// one writes X-hat or the cropped output straight to global memory.  One
// transform call site, so one inlined copy of the stages.
struct ColForwardOut {
    cx<float> *dst;
    int lim;
    float sign;
    __device__ __forceinline__ void operator()(int, int i, cx<float> v) const {
        if (i < lim) dst[i] = {v.x, sign * v.y};
    }
};

template <int NT, int... R>
__global__ void __launch_bounds__(NT, 3)
    k_col_forward_ct(const cx<float> *__restrict__ rx, int ldr, int rows_in, const cx<float> *__restrict__ khat,
                     size_t khat_stride, int nexp, cx<float> *__restrict__ y, int ldy, size_t y_stride, int rows_out,
                     cx<float> *__restrict__ aux, const cx<float> *__restrict__ tw) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int N = CtProd<R...>::value;
    cx<float> *buf = reinterpret_cast<cx<float> *>(smem_raw);
    const int u = blockIdx.x;
    cx<float> *xh = aux + (size_t)u * N;
#pragma unroll 1
    for (int it = 0; it <= nexp; ++it) {
        // the OTF column of the next exposure is fetched into L2 during this transform
        if (threadIdx.x == 0 && it < nexp) prefetch_l2(khat + it * khat_stride + (size_t)u * N, (size_t)N * sizeof(cx<float>));
        if (it == 0) {
            const cx<float> *src = rx + (size_t)u * ldr;
            for (int v = threadIdx.x; v < N; v += NT) buf[v] = v < rows_in ? src[v] : cx<float>{0.f, 0.f};
        } else {
            const cx<float> *kr = khat + (it - 1) * khat_stride + (size_t)u * N;
            for (int v = threadIdx.x; v < N; v += NT) {
                const cx<float> p = cmul(xh[v], kr[v]);
                buf[v] = {p.x, -p.y};
            }
        }
        __syncthreads();
        const ColForwardOut out{it == 0 ? xh : y + (it - 1) * y_stride + (size_t)u * ldy, it == 0 ? N : rows_out,
                                it == 0 ? 1.f : -1.f};
        ct_fft_out<1, NT, false, float, R...>(buf, tw, out);
        __syncthreads();  // buf and X-hat are read by the next transform
    }
}

// Column adjoint: C[u] = IFFT( sum_k conj(K_k[u]) * FFT(pad(Rs_k[u])) ) for
// rows < rows_out; the sum is taken in exposure order in the column's
// accumulator (global scratch of Acc::S), the first exposure's product
// written over whatever the scratch held.
template <class Acc> struct ColAdjointIO {
    const cx<float> *src;   // scatter spectrum column of the current exposure
    const cx<float> *kr;    // K column of the current exposure
    typename Acc::S *acc;
    cx<float> *dst;
    int rows_in, rows_out, phase;  // 0: first exposure, 1: later exposures, 2: the inverse of the sum
    __device__ __forceinline__ cx<float> operator()(int, int i) const {
        if (phase < 2) return i < rows_in ? src[i] : cx<float>{0.f, 0.f};
        const cx<float> a = Acc::get(acc[i]);
        return {a.x, -a.y};
    }
    __device__ __forceinline__ void operator()(int, int i, cx<float> v) const {
        if (phase < 2) {
            typename Acc::S s;
            if (phase == 0) Acc::zero(s);
            else s = acc[i];
            Acc::add(s, v, kr[i]);
            acc[i] = s;
        } else if (i < rows_out) {
            dst[i] = {v.x, -v.y};
        }
    }
};

template <class Acc, int NT, int... R>
__global__ void __launch_bounds__(NT, 3)
    k_col_adjoint_ct(const cx<float> *__restrict__ rs, int ldr, size_t rs_stride, int rows_in,
                     const cx<float> *__restrict__ khat, size_t khat_stride, int nexp, cx<float> *__restrict__ c,
                     int ldc, int rows_out, typename Acc::S *__restrict__ aux, const cx<float> *__restrict__ tw) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int N = CtProd<R...>::value;
    cx<float> *buf = reinterpret_cast<cx<float> *>(smem_raw);
    const int u = blockIdx.x;
    ColAdjointIO<Acc> io{nullptr, nullptr, aux + (size_t)u * N, c + (size_t)u * ldc, rows_in, rows_out, 0};
#pragma unroll 1
    for (int it = 0; it <= nexp; ++it) {
        if (it < nexp) {
            io.src = rs + it * rs_stride + (size_t)u * ldr;
            io.kr = khat + it * khat_stride + (size_t)u * N;
            io.phase = it == 0 ? 0 : 1;
        } else {
            io.phase = 2;
        }
        ct_fft_io<1, NT, false, float, R...>(io, buf, tw, io);
        __syncthreads();  // buf and the accumulator are read by the next transform
    }
}

// ---------------------------------------------------------------------------- catalog
// Transform lengths and radix orders with compile-time FP32 iteration
// kernels, chosen by timing every split of the candidate lengths of the
// 8 x 2048^2 -> 4096^2 field with 1431^2 PSFs (FFT 5040^2: rows of 2520
// complex points two to a block, 5040-point columns).  Other shapes use the
// run-time-plan kernels of kernels.cuh.
template <class F> bool ct_row_catalog(const std::vector<int> &rad, F &&f) {
    if (rad == std::vector<int>{14, 12, 15}) return f(CtRadices<14, 12, 15>{}), true;
    return false;
}
template <class F> bool ct_col_catalog(const std::vector<int> &rad, F &&f) {
    if (rad == std::vector<int>{21, 16, 15}) return f(CtRadices<21, 16, 15>{}), true;
    return false;
}
// Every catalog split of one length (rows: axis 0, columns: axis 1).
inline std::vector<std::vector<int>> ct_catalog_splits(int axis, int n) {
    const std::vector<std::vector<int>> rows = {{14, 12, 15}}, cols = {{21, 16, 15}};
    std::vector<std::vector<int>> out;
    for (const auto &r : axis == 0 ? rows : cols) {
        long p = 1;
        for (int v : r) p *= v;
        if (p == n) out.push_back(r);
    }
    return out;
}

}  // namespace updc
