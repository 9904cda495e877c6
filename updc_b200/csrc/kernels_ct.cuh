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
#include "pointwise.cuh"

namespace updc {

// Threads and resident blocks per SM of the compile-time row kernels, and
// resident blocks per SM of the column kernels.
#ifndef UPDC_CT_ROW_NT
#define UPDC_CT_ROW_NT 256
#endif
#ifndef UPDC_CT_ROW_MINB
#define UPDC_CT_ROW_MINB 4
#endif
#ifndef UPDC_CT_COL_MINB
#define UPDC_CT_COL_MINB 3
#endif
constexpr int CT_ROW_NT = UPDC_CT_ROW_NT;

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
__global__ void __launch_bounds__(NT, UPDC_CT_ROW_MINB)
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

// ---------------------------------------------------------------------------- adjoint gather + row R2C
// S^T(wr) of targets whose transposed entries are [a[g], b[g]): for each,
// the ordered chain acc = fmaf(frac, wr[src], acc) over its entries
// (increasing source pixel, updc_core.c:1173-1176 as seen from the target).
// The G chains run together, their loads issued in chunks of CH entries.
template <int CH, int G>
__device__ __forceinline__ void gather_chains(const ExpDesc<float> &e, const float *__restrict__ wr,
                                              const uint32_t (&a)[G], const uint32_t (&b)[G], float (&r)[G]) {
    float acc[G];
    uint32_t i0[G];
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g] = 0.f, i0[g] = a[g];
    bool more = true;
    while (more) {
        uint32_t sr[G][CH];
        float fr[G][CH], v[G][CH];
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int i = 0; i < CH; ++i) {
                const bool ok = i0[g] + i < b[g];
                const uint2 en = ok ? e.tent[i0[g] + i] : make_uint2(0u, 0u);
                sr[g][i] = en.x;
                fr[g][i] = __uint_as_float(en.y);
            }
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int i = 0; i < CH; ++i) v[g][i] = i0[g] + i < b[g] ? ld_keep_f(wr + sr[g][i]) : 0.f;
        more = false;
#pragma unroll
        for (int g = 0; g < G; ++g) {
#pragma unroll
            for (int i = 0; i < CH; ++i)
                if (i0[g] + i < b[g]) acc[g] = __fmaf_rn(fr[g][i], v[g][i], acc[g]);
            i0[g] += CH;
            more |= i0[g] < b[g];
        }
    }
#pragma unroll
    for (int g = 0; g < G; ++g) r[g] = acc[g];
}

// Targets a thread gathers together per step of the fused gather.
#ifndef UPDC_GATHER_TARGETS
#define UPDC_GATHER_TARGETS 2
#endif

// Rows [y0, y0 + 2) of exposure blockIdx.y's scatter plane S_k^T(wr_k) are
// gathered through the target-major map straight into the transform buffer
// (real row b at floats [b*2M, b*2M + W), zeros up to 2M), so the scatter
// plane never goes through HBM; then the row R2C of k_row_r2c_ct.  The
// gathered values are bit-identical to k_scatter_t's (same chain per
// target).  A thread takes G targets a step (NT apart, so a warp's loads
// stay coalesced) and loads the next step's CSR offsets before walking this
// step's entries.
template <int NT, int... R>
__global__ void __launch_bounds__(NT, UPDC_CT_ROW_MINB)
    k_gather_row_r2c_ct(const cx<float> *__restrict__ post, const ExpDesc<float> *__restrict__ exps,
                        const float *__restrict__ wr_all, size_t nin, int W, int rows,
                        const cx<float> *__restrict__ tw, const __grid_constant__ CUtensorMap omap) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int M = CtProd<R...>::value;
    constexpr int BR = 2, G = UPDC_GATHER_TARGETS;
    cx<float> *buf = reinterpret_cast<cx<float> *>(smem_raw);
    float *rowf = reinterpret_cast<float *>(smem_raw);
    const int y0 = blockIdx.x * BR, kexp = blockIdx.y;
    const int nb = min(BR, rows - y0);
    const ExpDesc<float> e = exps[kexp];
    const float *wr = wr_all + (size_t)kexp * nin;
    const int count = nb * W;
    const uint32_t *__restrict__ toff = e.toff + (size_t)y0 * (size_t)W;
    // CSR offsets of the step at q: targets q + g NT
    auto offsets = [&](int q, uint32_t (&a)[G], uint32_t (&b)[G]) {
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const bool h = q + g * NT < count;
            a[g] = h ? toff[q + g * NT] : 0u;
            b[g] = h ? toff[q + g * NT + 1] : 0u;
        }
    };
    uint32_t a[G], b[G];
    offsets(threadIdx.x, a, b);
    for (int q = threadIdx.x; q < count; q += G * NT) {
        uint32_t na[G], nb_[G];
        offsets(q + G * NT, na, nb_);  // in flight during this step's walk
        float r[G];
        gather_chains<4, G>(e, wr, a, b, r);
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int qg = q + g * NT;
            if (qg < count) {
                const int c = qg >= W ? 1 : 0;
                rowf[c * 2 * M + qg - c * W] = r[g];
            }
            a[g] = na[g];
            b[g] = nb_[g];
        }
    }
    // zero padding of the rows (and the whole of a missing second row)
    for (int rb = 0; rb < BR; ++rb) {
        const int x0 = rb < nb ? W : 0;
        for (int x = x0 + threadIdx.x; x < 2 * M; x += NT) rowf[rb * 2 * M + x] = 0.f;
    }
    __syncthreads();
    ct_fft<BR, NT, false, float, R...>(buf, tw);
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
__global__ void __launch_bounds__(NT, UPDC_CT_ROW_MINB)
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
// Threads of the compile-time column kernels (three blocks per SM).
#ifndef UPDC_CT_COL_NT
#define UPDC_CT_COL_NT 384
#endif
// Accumulator and OTF elements a thread loads together in the column adjoint.
#ifndef UPDC_COL_ADJ_B
#define UPDC_COL_ADJ_B 4
#endif
constexpr int CT_COL_NT = UPDC_CT_COL_NT;

// Element v = threadIdx.x + j*NT (j < ceil(N/NT)) of a column, visited in
// batches of B: the loads of a batch are issued before any of its results
// is used, so a thread keeps B independent global accesses in flight instead
// of one at a time.
template <int N, int NT, int B, class F> __device__ __forceinline__ void column_batches(const F &f) {
    constexpr int KE = (N + NT - 1) / NT;
#pragma unroll
    for (int j0 = 0; j0 < KE; j0 += B) f(j0);
}
template <int N, int NT> __device__ __forceinline__ bool column_has(int j) {
    constexpr int KE = (N + NT - 1) / NT;
    return j < KE && (N % NT == 0 || (int)threadIdx.x + j * NT < N);
}

// buf[v] = load(v) over the column, B loads in flight per thread.
template <int N, int NT, int B, class Load> __device__ __forceinline__ void stage_column(cx<float> *buf, const Load &load) {
    column_batches<N, NT, B>([&](int j0) {
        cx<float> t[B];
#pragma unroll
        for (int j = 0; j < B; ++j)
            if (column_has<N, NT>(j0 + j)) t[j] = load((int)threadIdx.x + (j0 + j) * NT);
#pragma unroll
        for (int j = 0; j < B; ++j)
            if (column_has<N, NT>(j0 + j)) buf[threadIdx.x + (j0 + j) * NT] = t[j];
    });
}

// Column forward model: transform 0 is FFT(pad(rx[u])) -> X-hat (global
// scratch, L2-resident); transform it >= 1 is IFFT(X-hat * K_{it-1}) for
// rows < rows_out, computed as conj(FFT(conj(.))).  Every transform's input
// is staged in shared memory by all threads together (seven elements' loads
// in flight per thread), the stages run in place, and the last one writes
// X-hat or the cropped output straight to global memory.  One transform call
// site, so one inlined copy of the stages.
// Stores are evict-first (st.global.cs): measured on the 5040-point columns
// of the 8 x 2048^2 -> 4096^2 field, the forward y passes take 0.59 ms with
// plain stores, 0.56 ms with X-hat stored plainly and the y spectra
// evict-first, and 0.54 ms with every store evict-first (X-hat is still
// found in L2 by the block's next transforms).
struct ColForwardOut {
    cx<float> *dst;
    int lim;
    float sign;
    __device__ __forceinline__ void operator()(int, int i, cx<float> v) const {
        if (i < lim) __stcs(reinterpret_cast<float2 *>(dst + i), make_float2(v.x, sign * v.y));
    }
};

template <int NT, int... R>
__global__ void __launch_bounds__(NT, UPDC_CT_COL_MINB)
    k_col_forward_ct(const cx<float> *__restrict__ rx, int ldr, int rows_in, const cx<float> *__restrict__ khat,
                     size_t khat_stride, int nexp, cx<float> *__restrict__ y, int ldy, size_t y_stride, int rows_out,
                     cx<float> *__restrict__ aux, const cx<float> *__restrict__ tw) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int N = CtProd<R...>::value;
    cx<float> *buf = reinterpret_cast<cx<float> *>(smem_raw);
    const int u = blockIdx.x;
    cx<float> *__restrict__ xh = aux + (size_t)u * N;
#pragma unroll 1
    for (int it = 0; it <= nexp; ++it) {
        // the OTF column of the next exposure is fetched into L2 during this transform
        if (threadIdx.x == 0 && it < nexp) prefetch_l2(khat + it * khat_stride + (size_t)u * N, (size_t)N * sizeof(cx<float>));
        if (it == 0) {
            const cx<float> *__restrict__ src = rx + (size_t)u * ldr;
            stage_column<N, NT, 7>(buf, [&](int v) { return v < rows_in ? ldcs_cx(src + v) : cx<float>{0.f, 0.f}; });
        } else {
            const cx<float> *__restrict__ kr = khat + (it - 1) * khat_stride + (size_t)u * N;
            stage_column<N, NT, 7>(buf, [&](int v) {
                const cx<float> p = cmul(xh[v], ldcs_cx(kr + v));
                return cx<float>{p.x, -p.y};
            });
        }
        __syncthreads();
        const ColForwardOut out{it == 0 ? xh : y + (it - 1) * y_stride + (size_t)u * ldy, it == 0 ? N : rows_out,
                                it == 0 ? 1.f : -1.f};
        ct_fft_out<1, NT, false, float, R...>(buf, tw, out);
        __syncthreads();  // buf and X-hat are read by the next transform
    }
}

// Column adjoint: C[u] = IFFT( sum_k conj(K_k[u]) * FFT(pad(Rs_k[u])) ) for
// rows < rows_out.  Each exposure's transform reads its first stage straight
// from the scatter spectrum and ends in shared memory; the conj-OTF product
// is then added into the column's accumulator (global scratch of Acc::S, in
// exposure order, the first exposure's product written over whatever the
// scratch held) with four elements' accumulator and OTF loads in flight per
// thread.  Finally the sum is staged back and inverse-transformed.
struct ColIn {
    const cx<float> *src;
    int rows_in;
    __device__ __forceinline__ cx<float> operator()(int, int i) const {
        return i < rows_in ? ldcs_cx(src + i) : cx<float>{0.f, 0.f};
    }
};

template <class Acc, int NT, int... R>
__global__ void __launch_bounds__(NT, UPDC_CT_COL_MINB)
    k_col_adjoint_ct(const cx<float> *__restrict__ rs, int ldr, size_t rs_stride, int rows_in,
                     const cx<float> *__restrict__ khat, size_t khat_stride, int nexp, cx<float> *__restrict__ c,
                     int ldc, int rows_out, typename Acc::S *__restrict__ aux, const cx<float> *__restrict__ tw) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr int N = CtProd<R...>::value;
    constexpr int B = UPDC_COL_ADJ_B;
    cx<float> *buf = reinterpret_cast<cx<float> *>(smem_raw);
    const int u = blockIdx.x;
    typename Acc::S *__restrict__ acc = aux + (size_t)u * N;
#pragma unroll 1
    for (int it = 0; it < nexp; ++it) {
        ct_fft_in<1, NT, false, float, R...>(ColIn{rs + it * rs_stride + (size_t)u * ldr, rows_in}, buf, tw);
        const cx<float> *__restrict__ kr = khat + it * khat_stride + (size_t)u * N;
        const bool first = it == 0;
        column_batches<N, NT, B>([&](int j0) {
            typename Acc::S s[B];
            cx<float> k[B];
#pragma unroll
            for (int j = 0; j < B; ++j)
                if (column_has<N, NT>(j0 + j)) {
                    const int v = threadIdx.x + (j0 + j) * NT;
                    k[j] = ldcs_cx(kr + v);
                    if (first) Acc::zero(s[j]);
                    else s[j] = ld_keep(acc + v);
                }
#pragma unroll
            for (int j = 0; j < B; ++j)
                if (column_has<N, NT>(j0 + j)) {
                    const int v = threadIdx.x + (j0 + j) * NT;
                    Acc::add(s[j], buf[v], k[j]);
                    st_keep(acc + v, s[j]);
                }
        });
        __syncthreads();  // buf is rewritten by the next transform
    }
    stage_column<N, NT, B>(buf, [&](int v) {
        const cx<float> a = Acc::get(ld_keep(acc + v));
        return cx<float>{a.x, -a.y};
    });
    __syncthreads();
    ct_fft_out<1, NT, false, float, R...>(buf, tw, ColForwardOut{c + (size_t)u * ldc, rows_out, -1.f});
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
