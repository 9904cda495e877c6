// Detector-space, target-space and setup kernels of the UPDC iteration.
#pragma once

#include "common.cuh"

namespace updc {

// Per-exposure device descriptor (one per exposure, uploaded at setup).
template <typename T> struct ExpDesc {
    const uint32_t *off, *base, *tgt;
    const uint16_t *delta;
    const float *frac;
    const uint32_t *toff;
    const uint2 *tent;  // transposed entries {source pixel, fraction bits}
    const T *sci, *wht;
    uint8_t *frozen;
    T background, pedestal, mean_offset;
    int delta16;
};

// Per-iteration, per-exposure FreezeMu counters (updc_core.c:1151-1164).
struct ExpStats {
    unsigned long long nnew, ntotal, min_ordered;  // min raw_mu as order-preserving bits of a double
    unsigned long long pad;
};

__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

__device__ __forceinline__ void record_error(unsigned long long *err, uint64_t stage, uint64_t index, uint32_t code) {
    atomicMin(err, (unsigned long long)make_error_key(stage, index, code));
}

template <typename T> __device__ __forceinline__ T block_sum_warp(T v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// ---------------------------------------------------------------------------- detector
// Warp-cooperative, software-pipelined tiles.  A warp owns 32 consecutive
// detector pixels (one pixel a lane) per tile and walks its tiles in grid
// stride.  The links of a tile occupy one contiguous range of the LinkMap,
// which the warp copies into shared memory with asynchronous 16-byte copies
// (cp.async: four fractions, eight DELTA16 offsets or four ABS32 targets per
// copy, from the range's start rounded down to a 16-byte boundary) into one
// of two buffers, so the copy of tile i+1's links is in flight while the
// lanes walk tile i's.  The per-pixel words of a tile (weight, science,
// DELTA16 base, FreezeMu mask) are loaded into registers one tile ahead and
// its CSR offsets two tiles ahead, so no load of a tile waits when the tile's
// turn comes except the blur gathers of the walk, which a lane issues four
// links at a time.  Ranges longer than DET_LCAP links are walked with direct
// loads.  The LinkMap arrays are allocated with 16 bytes of slack
// (linkmap_load), so the last vector of a range ending at the map's last link
// stays inside its allocation.
constexpr int DET_WARPS = 8;
constexpr int DET_LCAP = 384;
constexpr int DET_SLOTS = DET_LCAP + 8;  // room for the rounded-down start

template <typename T> struct LinkSum {
    // COMP: the sum runs in FP64 (products of FP32 operands are exact in
    // FP64), and raw_mu is that sum plus the offset rounded once to T.
    T s = T(0);
    double d = 0.0;
    template <bool COMP> __device__ __forceinline__ void add(float f, T bl) {
        if (!COMP) s = fma_rn((T)f, bl, s);
        else d = __fma_rn((double)f, (double)bl, d);
    }
    template <bool COMP> __device__ __forceinline__ T finish(T offset) const {
        if (!COMP) return add_rn(s, offset);
        return (T)__dadd_rn(d, (double)offset);
    }
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most one of this thread's committed copy groups is pending.
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// The fused detector loop of updc_core.c:1152-1176 for exposure blockIdx.y:
//   pred = sum_z fmaf(frac[z], blur[t(z)], pred) in link order;
//   raw_mu = pred + (background + pedestal);  FreezeMu;  ratio;  wr = W * ratio.
// Writes wr (0 for skipped pixels) for the adjoint gather.  With COMP the
// prediction is accumulated in FP64 and raw_mu is rounded once from the FP64
// sum with the offset, so the FreezeMu threshold is decided on a compensated
// raw_mu.
// Block `block` of `nblocks` over exposure k's pixels (grid-stride); the
// body of k_detector and of the batched detector (batch.cuh).
// Dynamic shared memory of a detector block (50.4 KB).
struct DetShared {
    float4 frac[DET_WARPS][2][DET_SLOTS / 4];  // staged fractions, two tiles
    uint4 idx[DET_WARPS][2][DET_SLOTS / 4];    // staged u32 targets or u16 offsets
    unsigned long long nnew[DET_WARPS], ntot[DET_WARPS], mn[DET_WARPS];
};

// Per-pixel words of one tile held by a lane.
template <typename T> struct PixelWords {
    uint32_t z0 = 0, z1 = 0, bse = 0;
    T w = T(0), sci = T(0);
    uint8_t fz = 0;
};

template <typename T, bool COMP, bool DELTA16>
__device__ __forceinline__ void detector_tiles_enc(const ExpDesc<T> &e, int k, size_t nin, const T *__restrict__ blur,
                                                   T *__restrict__ wr, ExpStats *__restrict__ stats,
                                                   unsigned long long *__restrict__ err, unsigned block,
                                                   unsigned nblocks, DetShared &sh) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr uint32_t IPV = DELTA16 ? 8u : 4u;  // index entries per 16-byte vector
    unsigned long long nnew = 0, ntot = 0, mn = ~0ull;
    const size_t step = (size_t)nblocks * DET_WARPS * 32;
    // CSR offsets of a tile, and the rest of its per-pixel words
    auto offsets = [&](size_t t0, PixelWords<T> &q) {
        const size_t p = t0 + lane;
        q.z0 = p < nin ? e.off[p] : 0u;
        q.z1 = p < nin ? e.off[p + 1] : 0u;
    };
    auto words = [&](size_t t0, PixelWords<T> &q) {
        const size_t p = t0 + lane;
        const bool v = p < nin;
        q.w = v ? e.wht[p] : T(0);
        q.bse = (v && DELTA16) ? e.base[p] : 0u;
        q.sci = v ? e.sci[p] : T(0);
        q.fz = v ? e.frozen[p] : (uint8_t)0;
    };
    // the tile's link range [zb, ze) (lanes past nin hold z0 = z1 = 0)
    auto range = [&](size_t t0, const PixelWords<T> &q, uint32_t &zb, uint32_t &ze) {
        const int last = (int)min((size_t)31, nin - 1 - t0);
        zb = __shfl_sync(0xffffffffu, q.z0, 0);
        ze = __shfl_sync(0xffffffffu, q.z1, last);
    };
    // asynchronous copy of a tile's links into buffer b (nothing when the
    // range exceeds DET_LCAP); always commits one group
    auto stage = [&](size_t t0, const PixelWords<T> &q, int b) {
        if (t0 < nin) {
            uint32_t zb, ze;
            range(t0, q, zb, ze);
            if (ze - zb <= (uint32_t)DET_LCAP) {
                const uint32_t fa = zb & ~3u, ia = zb & ~(IPV - 1u);
                const uint32_t nf = (ze - fa + 3u) >> 2, ni = (ze - ia + IPV - 1u) / IPV;
                const float4 *fsrc = reinterpret_cast<const float4 *>(e.frac) + (fa >> 2);
                const uint4 *isrc = DELTA16 ? reinterpret_cast<const uint4 *>(e.delta) + (ia >> 3)
                                            : reinterpret_cast<const uint4 *>(e.tgt) + (ia >> 2);
                for (uint32_t v = lane; v < nf; v += 32) cp_async16(&sh.frac[warp][b][v], fsrc + v);
                for (uint32_t v = lane; v < ni; v += 32) cp_async16(&sh.idx[warp][b][v], isrc + v);
            }
        }
        cp_async_commit();
    };

    size_t p0 = ((size_t)block * DET_WARPS + warp) * 32;
    PixelWords<T> cur, nxt, nn;
    offsets(p0, cur);
    words(p0, cur);
    offsets(p0 + step, nxt);
    words(p0 + step, nxt);
    offsets(p0 + 2 * step, nn);
    stage(p0, cur, 0);
    for (int it = 0; p0 < nin; ++it, p0 += step) {
        const int b = it & 1;
        stage(p0 + step, nxt, b ^ 1);  // tile i+1's links, in flight during this walk
        cp_async_wait_prior();         // tile i's links have arrived
        __syncwarp();
        uint32_t zb, ze;
        range(p0, cur, zb, ze);
        const bool staged = ze - zb <= (uint32_t)DET_LCAP;
        const uint32_t fa = zb & ~3u, ia = zb & ~(IPV - 1u);
        const float *sf = reinterpret_cast<const float *>(sh.frac[warp][b]);
        const uint16_t *si16 = reinterpret_cast<const uint16_t *>(sh.idx[warp][b]);
        const uint32_t *si32 = reinterpret_cast<const uint32_t *>(sh.idx[warp][b]);
        const size_t p = p0 + lane;
        if (p < nin) {
            const uint32_t z0 = cur.z0, z1 = cur.z1;
            const T w = cur.w;
            T out = T(0);
            if (w > T(0) && z0 != z1) {
                LinkSum<T> acc;
                if (staged) {
                    // the pixel's staged links from base pointers; the gathers
                    // of a chunk of four are issued together, then the ordered
                    // sum (whole chunks unpredicated, one predicated tail)
                    constexpr int CH = 4;
                    const uint32_t n = z1 - z0;
                    const float *fr = sf + (z0 - fa);
                    const uint16_t *dl = si16 + (z0 - ia);
                    const uint32_t *tg = si32 + (z0 - ia);
                    const T *bp = DELTA16 ? blur + cur.bse : blur;
                    uint32_t j = 0;
                    for (; j + CH <= n; j += CH) {
                        T bl[CH];
#pragma unroll
                        for (int i = 0; i < CH; ++i) bl[i] = bp[DELTA16 ? (uint32_t)dl[j + i] : tg[j + i]];
#pragma unroll
                        for (int i = 0; i < CH; ++i) acc.template add<COMP>(fr[j + i], bl[i]);
                    }
                    if (j < n) {
                        T bl[CH - 1];
#pragma unroll
                        for (int i = 0; i < CH - 1; ++i)
                            bl[i] = j + i < n ? bp[DELTA16 ? (uint32_t)dl[j + i] : tg[j + i]] : T(0);
#pragma unroll
                        for (int i = 0; i < CH - 1; ++i)
                            if (j + i < n) acc.template add<COMP>(fr[j + i], bl[i]);
                    }
                } else {
                    for (uint32_t z = z0; z < z1; ++z) {
                        const uint32_t t = DELTA16 ? cur.bse + (uint32_t)e.delta[z] : e.tgt[z];
                        acc.template add<COMP>(e.frac[z], blur[t]);
                    }
                }
                const T raw_mu = acc.template finish<COMP>(e.mean_offset);
                if (!isfinite(raw_mu)) {
                    record_error(err, STAGE_DETECTOR, (uint64_t)k * nin + p, ERR_NONFINITE_MEAN);
                } else {
                    const unsigned long long o = double_to_ordered((double)raw_mu);
                    mn = o < mn ? o : mn;
                    uint8_t fz = cur.fz;
                    if (!fz && !(raw_mu > T(0))) {
                        fz = 1;
                        e.frozen[p] = 1;
                        ++nnew;
                    }
                    T ratio;
                    if (fz) {
                        ++ntot;
                        ratio = T(1);
                    } else {
                        const T y = add_rn(cur.sci, e.pedestal);
                        ratio = div_rn(y, raw_mu);
                        if (!isfinite(ratio)) record_error(err, STAGE_DETECTOR, (uint64_t)k * nin + p, ERR_NONFINITE_RATIO);
                    }
                    out = mul_rn(w, ratio);
                }
            }
            wr[p] = out;
        }
        __syncwarp();  // buffer b is refilled by the staging of tile i+2
        cur = nxt;
        nxt.z0 = nn.z0;
        nxt.z1 = nn.z1;
        words(p0 + 2 * step, nxt);
        offsets(p0 + 3 * step, nn);
    }
    cp_async_wait_all();  // no copy of this thread outlives the kernel
    // block reduction of the counters
    auto &s_new = sh.nnew;
    auto &s_tot = sh.ntot;
    auto &s_min = sh.mn;
    nnew = block_sum_warp(nnew);
    ntot = block_sum_warp(ntot);
    mn = warp_min_u64(mn);
    if (lane == 0) {
        s_new[warp] = nnew;
        s_tot[warp] = ntot;
        s_min[warp] = mn;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long a = 0, b = 0, m = ~0ull;
        for (int i = 0; i < DET_WARPS; ++i) {
            a += s_new[i];
            b += s_tot[i];
            m = s_min[i] < m ? s_min[i] : m;
        }
        if (a) atomicAdd(&stats[k].nnew, a);
        if (b) atomicAdd(&stats[k].ntotal, b);
        if (m != ~0ull) atomicMin(&stats[k].min_ordered, m);
    }
}

// Four 256-thread blocks per SM (64 registers; measured 5% faster than three
// blocks at 80 registers on B200).
// The exposure's LinkMap encoding is fixed per exposure; each block takes
// the instantiation of its encoding (a block-uniform branch).
template <typename T, bool COMP>
__device__ __forceinline__ void detector_tiles(const ExpDesc<T> &e, int k, size_t nin, const T *__restrict__ blur,
                                               T *__restrict__ wr, ExpStats *__restrict__ stats,
                                               unsigned long long *__restrict__ err, unsigned block, unsigned nblocks,
                                               unsigned char *smem) {
    DetShared &sh = *reinterpret_cast<DetShared *>(smem);
    if (e.delta16) detector_tiles_enc<T, COMP, true>(e, k, nin, blur, wr, stats, err, block, nblocks, sh);
    else detector_tiles_enc<T, COMP, false>(e, k, nin, blur, wr, stats, err, block, nblocks, sh);
}

// Resident detector blocks per SM the kernel is compiled for (its register
// budget is 65536 / (256 * blocks) a thread).
#ifndef UPDC_DET_MIN_BLOCKS
#define UPDC_DET_MIN_BLOCKS 4
#endif
template <typename T, bool COMP>
__global__ void __launch_bounds__(DET_WARPS * 32, UPDC_DET_MIN_BLOCKS) k_detector(const ExpDesc<T> *__restrict__ exps, size_t nin, size_t nout,
                                                           const T *__restrict__ blur_all, T *__restrict__ wr_all,
                                                           ExpStats *__restrict__ stats, unsigned long long *__restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int k = blockIdx.y;
    const ExpDesc<T> e = exps[k];
    detector_tiles<T, COMP>(e, k, nin, blur_all + k * nout, wr_all + k * nin, stats, err, blockIdx.x, gridDim.x, smem_raw);
}

// ---------------------------------------------------------------------------- adjoint gather
// scatter_k[t] = sum over the transposed entries of t, in increasing source
// pixel order, of fmaf(frac, value[p], acc): the exact sequence of
// updc_core.c:1173-1176 for target t.  ACC may be wider than T.  Entries are
// read in chunks: all loads of a chunk first, then the ordered fma chain.
template <typename T, typename ACC, typename V>
__device__ __forceinline__ void scatter_targets(const ExpDesc<T> &e, size_t nout, const V *__restrict__ val,
                                                int use_weight, ACC *__restrict__ out, unsigned block, unsigned nblocks) {
    constexpr int CH = 4;
    for (size_t t = block * (size_t)blockDim.x + threadIdx.x; t < nout; t += (size_t)nblocks * blockDim.x) {
        const uint32_t a = e.toff[t], b = e.toff[t + 1];
        ACC acc = ACC(0);
        for (uint32_t ic = a; ic < b; ic += CH) {
            uint32_t src[CH];
            float fr[CH];
            ACC v[CH];
            bool use[CH];
#pragma unroll
            for (int i = 0; i < CH; ++i) {
                const bool ok = ic + i < b;
                const uint2 en = ok ? e.tent[ic + i] : make_uint2(0u, 0u);
                src[i] = en.x;
                fr[i] = __uint_as_float(en.y);
            }
#pragma unroll
            for (int i = 0; i < CH; ++i) {
                const bool ok = ic + i < b;
                if (use_weight) {
                    const T w = ok ? e.wht[src[i]] : T(0);
                    use[i] = ok && w > T(0);  // masked pixels are skipped (updc_core.c:1061)
                    v[i] = (ACC)w;
                } else {
                    use[i] = ok;
                    v[i] = ok ? (ACC)val[src[i]] : ACC(0);
                }
            }
#pragma unroll
            for (int i = 0; i < CH; ++i)
                if (use[i]) acc = fma_rn((ACC)fr[i], v[i], acc);
        }
        out[t] = acc;
    }
}

template <typename T, typename ACC, typename V>
__global__ void __launch_bounds__(256) k_scatter_t(const ExpDesc<T> *__restrict__ exps, size_t nin, size_t nout,
                                                   const V *__restrict__ val_all, int use_weight, ACC *__restrict__ out_all) {
    const int k = blockIdx.y;
    const ExpDesc<T> e = exps[k];
    scatter_targets<T, ACC, V>(e, nout, use_weight ? nullptr : val_all + k * nin, use_weight, out_all + k * nout,
                               blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------- update
// updc_core.c:1437-1456, with per-block partial sums for the diagnostics.
template <typename T>
__device__ __forceinline__ void update_block(size_t nout, const T *__restrict__ corr, const T *__restrict__ den,
                                             T *__restrict__ x, T max_sens, unsigned long long *__restrict__ err,
                                             double *__restrict__ part_sum, unsigned long long *__restrict__ part_neg,
                                             unsigned block, unsigned nblocks) {
    double sum = 0.0;
    unsigned long long neg = 0;
    const T thr = mul_rn((T)-1.0e-6f, max_sens);
    for (size_t t = block * (size_t)blockDim.x + threadIdx.x; t < nout; t += (size_t)nblocks * blockDim.x) {
        const T d = den[t];
        T v = x[t];
        if (d > (T)1e-8f) {
            T f = div_rn(corr[t], d);
            if (!isfinite(f)) record_error(err, STAGE_UPDATE, t, ERR_NONFINITE_CORRECTION);
            if (f < T(0)) {
                if (corr[t] < thr) record_error(err, STAGE_UPDATE, t, ERR_NEGATIVE_CORRECTION);
                f = T(0);
            }
            v = mul_rn(v, f);
        } else {
            v = T(0);
        }
        if (!isfinite(v)) record_error(err, STAGE_UPDATE, t, ERR_NONFINITE_ESTIMATE);
        x[t] = v;
        sum += (double)v;
        neg += v < T(0) ? 1ull : 0ull;
    }
    __shared__ double s_sum[8];
    __shared__ unsigned long long s_neg[8];
    sum = block_sum_warp(sum);
    neg = block_sum_warp(neg);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_sum[warp] = sum;
        s_neg[warp] = neg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0;
        unsigned long long b = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            a += s_sum[i];
            b += s_neg[i];
        }
        part_sum[block] = a;
        part_neg[block] = b;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_update(size_t nout, const T *__restrict__ corr, const T *__restrict__ den,
                                                T *__restrict__ x, T max_sens, unsigned long long *__restrict__ err,
                                                double *__restrict__ part_sum, unsigned long long *__restrict__ part_neg) {
    update_block<T>(nout, corr, den, x, max_sens, err, part_sum, part_neg, blockIdx.x, gridDim.x);
}

// Fixed-order final reduction of per-block partials (deterministic).  The
// partials are read through L2 (ld.global.cg): other blocks of the same
// launch may have written them.
__device__ __forceinline__ void reduce_partials_block(const double *part_sum, const unsigned long long *part_neg, int n,
                                                      double *out_sum, unsigned long long *out_neg) {
    __shared__ double s[256];
    __shared__ unsigned long long c[256];
    double a = 0;
    unsigned long long b = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a += __ldcg(part_sum + i);
        b += __ldcg(part_neg + i);
    }
    s[threadIdx.x] = a;
    c[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s[threadIdx.x] += s[threadIdx.x + o];
            c[threadIdx.x] += c[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *out_sum = s[0];
        *out_neg = c[0];
    }
}
static __global__ void k_reduce_partials(const double *part_sum, const unsigned long long *part_neg, int n, double *out_sum,
                                         unsigned long long *out_neg) {
    reduce_partials_block(part_sum, part_neg, n, out_sum, out_neg);
}

// ---------------------------------------------------------------------------- update, 16-byte accesses
// The update of updc_core.c:1437-1456 (the per-pixel arithmetic of
// update_block) with every thread moving 16 bytes of each plane per access:
// four floats or two doubles.  Pixels past the last whole vector go to the
// first threads of block 0.  Each block writes its partial sum and negative
// count to its slot, as update_block does.
template <typename T> struct Vec16;
template <> struct Vec16<float> {
    using V = float4;
    static constexpr int n = 4;
    __device__ __forceinline__ static void split(const float4 &v, float *o) { o[0] = v.x, o[1] = v.y, o[2] = v.z, o[3] = v.w; }
    __device__ __forceinline__ static float4 join(const float *o) { return make_float4(o[0], o[1], o[2], o[3]); }
};
template <> struct Vec16<double> {
    using V = double2;
    static constexpr int n = 2;
    __device__ __forceinline__ static void split(const double2 &v, double *o) { o[0] = v.x, o[1] = v.y; }
    __device__ __forceinline__ static double2 join(const double *o) { return make_double2(o[0], o[1]); }
};

template <typename T>
__device__ __forceinline__ T update_pixel(T c, T d, T v, T thr, size_t t, unsigned long long *__restrict__ err) {
    if (d > (T)1e-8f) {
        T f = div_rn(c, d);
        if (!isfinite(f)) record_error(err, STAGE_UPDATE, t, ERR_NONFINITE_CORRECTION);
        if (f < T(0)) {
            if (c < thr) record_error(err, STAGE_UPDATE, t, ERR_NEGATIVE_CORRECTION);
            f = T(0);
        }
        v = mul_rn(v, f);
    } else {
        v = T(0);
    }
    if (!isfinite(v)) record_error(err, STAGE_UPDATE, t, ERR_NONFINITE_ESTIMATE);
    return v;
}

// Planes 16-byte aligned (the engine's own allocations).
template <typename T>
__device__ __forceinline__ void update_block_vec(size_t nout, const T *__restrict__ corr, const T *__restrict__ den,
                                                 T *__restrict__ x, T max_sens, unsigned long long *__restrict__ err,
                                                 double *__restrict__ part_sum, unsigned long long *__restrict__ part_neg,
                                                 unsigned block, unsigned nblocks) {
    using VT = typename Vec16<T>::V;
    constexpr int NV = Vec16<T>::n;
    const size_t nvec = nout / NV;
    const T thr = mul_rn((T)-1.0e-6f, max_sens);
    double sum = 0.0;
    unsigned long long neg = 0;
    const VT *cv = reinterpret_cast<const VT *>(corr);
    const VT *dv = reinterpret_cast<const VT *>(den);
    VT *xv = reinterpret_cast<VT *>(x);
    for (size_t i = block * (size_t)blockDim.x + threadIdx.x; i < nvec; i += (size_t)nblocks * blockDim.x) {
        T c[NV], d[NV], v[NV];
        Vec16<T>::split(__ldcs(cv + i), c);
        Vec16<T>::split(__ldcs(dv + i), d);
        Vec16<T>::split(xv[i], v);
#pragma unroll
        for (int j = 0; j < NV; ++j) {
            v[j] = update_pixel(c[j], d[j], v[j], thr, i * NV + j, err);
            sum += (double)v[j];
            neg += v[j] < T(0) ? 1ull : 0ull;
        }
        xv[i] = Vec16<T>::join(v);
    }
    if (block == 0) {
        for (size_t t = nvec * NV + threadIdx.x; t < nout; t += blockDim.x) {
            const T v = update_pixel(corr[t], den[t], x[t], thr, t, err);
            x[t] = v;
            sum += (double)v;
            neg += v < T(0) ? 1ull : 0ull;
        }
    }
    __shared__ double s_sum[8];
    __shared__ unsigned long long s_neg[8];
    sum = block_sum_warp(sum);
    neg = block_sum_warp(neg);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_sum[warp] = sum;
        s_neg[warp] = neg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0;
        unsigned long long b = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            a += s_sum[i];
            b += s_neg[i];
        }
        part_sum[block] = a;
        part_neg[block] = b;
    }
}

// One launch: the vectorised update, then the last block to finish reduces
// the partials in block order (the order of k_reduce_partials) and re-arms
// the completion counter `done` (zero before the first launch).
template <typename T>
__global__ void __launch_bounds__(256) k_update_vec(size_t nout, const T *__restrict__ corr, const T *__restrict__ den,
                                                    T *__restrict__ x, T max_sens, unsigned long long *__restrict__ err,
                                                    double *__restrict__ part_sum, unsigned long long *__restrict__ part_neg,
                                                    unsigned *__restrict__ done, double *__restrict__ red_sum,
                                                    unsigned long long *__restrict__ red_neg) {
    update_block_vec<T>(nout, corr, den, x, max_sens, err, part_sum, part_neg, blockIdx.x, gridDim.x);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();  // this block's partials are visible before it is counted
        last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    reduce_partials_block(part_sum, part_neg, (int)gridDim.x, red_sum, red_neg);
    if (threadIdx.x == 0) *done = 0u;
}

// ---------------------------------------------------------------------------- setup
// Mask and normalise one exposure's planes (updc_core.c:407-419).
template <typename T>
__global__ void k_weight_norm(size_t nin, const float *__restrict__ sci_raw, const float *__restrict__ wht_raw,
                              T *__restrict__ sci, T *__restrict__ wht, T scale, T pedestal, int k,
                              unsigned long long *__restrict__ masked, unsigned long long *__restrict__ err) {
    unsigned long long m = 0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < nin; p += (size_t)gridDim.x * blockDim.x) {
        T s = (T)sci_raw[p], w = (T)wht_raw[p];
        if (!isfinite(s) || !isfinite(w) || !(w > T(0))) {
            sci[p] = T(0);
            wht[p] = T(0);
            ++m;
            continue;
        }
        w = div_rn(w, scale);
        if (!isfinite(w) || !(w > T(0))) record_error(err, STAGE_SETUP, (uint64_t)k * nin + p, ERR_INVALID_NORM_WHT);
        const T y = add_rn(s, pedestal);
        if (!isfinite(y) || y < T(0)) record_error(err, STAGE_SETUP, (uint64_t)k * nin + p, ERR_NEGATIVE_YEFF);
        sci[p] = s;
        wht[p] = w;
    }
    m = block_sum_warp(m);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(masked, m);
}

// Every 64th weight of one exposure, finite and > 0 (updc_core.c:380-384).
static __global__ void k_weight_sample(size_t nin, const float *__restrict__ wht_raw, float *__restrict__ out,
                                unsigned int *__restrict__ count) {
    for (size_t p = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) * 64; p < nin; p += (size_t)gridDim.x * blockDim.x * 64) {
        const float w = wht_raw[p];
        if (isfinite(w) && w > 0.0f) {
            // positions are re-sorted afterwards, so the slot order is irrelevant
            out[atomicAdd(count, 1u)] = w;
        }
    }
}

// PSF validity and FP64 sum (fixed-order block tree; deterministic).
template <typename P>
__global__ void k_psf_sum_f64(const P *__restrict__ psf, size_t n, double *__restrict__ partial,
                              unsigned long long *__restrict__ err) {
    __shared__ double s[256];
    double a = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const P v = psf[i];
        if (!isfinite(v) || v < P(0)) record_error(err, STAGE_SETUP, i, ERR_INVALID_PSF_PIXEL);
        a += (double)v;
    }
    s[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x / 2; o; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

// Neumaier float sum in the reference's serial order (updc_core.c:777-789),
// for the reference-precision form.  One thread; setup only.
static __global__ void k_psf_sum_neumaier(const float *__restrict__ psf, size_t n, float *__restrict__ out,
                                   unsigned long long *__restrict__ err) {
    if (threadIdx.x || blockIdx.x) return;
    float sum = 0.0f, comp = 0.0f;
    for (size_t p = 0; p < n; ++p) {
        const float v = psf[p];
        if (!isfinite(v) || v < 0.0f) {
            record_error(err, STAGE_SETUP, p, ERR_INVALID_PSF_PIXEL);
            return;
        }
        const float t = __fadd_rn(sum, v);
        if (fabsf(sum) >= fabsf(v)) comp = __fadd_rn(comp, __fadd_rn(__fsub_rn(sum, t), v));
        else comp = __fadd_rn(comp, __fadd_rn(__fsub_rn(v, t), sum));
        sum = t;
    }
    *out = __fadd_rn(sum, comp);
}

// Initial signed drizzle estimate and coverage (updc_core.c:947-971): for each
// target, exposures in order, transposed entries in source-pixel order.
template <typename T>
__global__ void __launch_bounds__(256) k_drizzle(const ExpDesc<T> *__restrict__ exps, int nexp, size_t nout,
                                                 T *__restrict__ estimate, T *__restrict__ coverage,
                                                 unsigned long long *__restrict__ err) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nout; t += (size_t)gridDim.x * blockDim.x) {
        T cov = 0, data = 0, bkg = 0;
        for (int k = 0; k < nexp; ++k) {
            const ExpDesc<T> &e = exps[k];
            const uint32_t a = e.toff[t], b = e.toff[t + 1];
            for (uint32_t i = a; i < b; ++i) {
                const uint2 en = e.tent[i];
                const uint32_t p = en.x;
                const T w = e.wht[p];
                if (!(w > T(0))) continue;
                const T q = mul_rn((T)__uint_as_float(en.y), w);
                cov = add_rn(cov, q);
                data = fma_rn(q, e.sci[p], data);
                bkg = fma_rn(q, e.background, bkg);
            }
        }
        coverage[t] = cov;
        T est = T(0);
        if (cov > (T)1e-12f) {
            est = sub_rn(div_rn(data, cov), div_rn(bkg, cov));
            if (!isfinite(est)) record_error(err, STAGE_SETUP, t, ERR_NONFINITE_INITIAL);
        }
        estimate[t] = est;
    }
}

// The drizzle's three per-target sums over exposures [0, nexp) of `exps`
// only (an exposure shard, set up alone): coverage, data and background, in
// the order k_drizzle forms them.  The shards' planes are summed over ranks,
// then k_drizzle_finish forms the estimate as k_drizzle does.
template <typename T>
__global__ void __launch_bounds__(256) k_drizzle_partial(const ExpDesc<T> *__restrict__ exps, int nexp, size_t nout,
                                                         T *__restrict__ coverage, T *__restrict__ data,
                                                         T *__restrict__ background) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nout; t += (size_t)gridDim.x * blockDim.x) {
        T cov = 0, dat = 0, bkg = 0;
        for (int k = 0; k < nexp; ++k) {
            const ExpDesc<T> &e = exps[k];
            const uint32_t a = e.toff[t], b = e.toff[t + 1];
            for (uint32_t i = a; i < b; ++i) {
                const uint2 en = e.tent[i];
                const uint32_t p = en.x;
                const T w = e.wht[p];
                if (!(w > T(0))) continue;
                const T q = mul_rn((T)__uint_as_float(en.y), w);
                cov = add_rn(cov, q);
                dat = fma_rn(q, e.sci[p], dat);
                bkg = fma_rn(q, e.background, bkg);
            }
        }
        coverage[t] = cov;
        data[t] = dat;
        background[t] = bkg;
    }
}
template <typename T>
__global__ void __launch_bounds__(256) k_drizzle_finish(size_t nout, const T *__restrict__ coverage,
                                                        const T *__restrict__ data, const T *__restrict__ background,
                                                        T *__restrict__ estimate, unsigned long long *__restrict__ err) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nout; t += (size_t)gridDim.x * blockDim.x) {
        const T cov = coverage[t];
        T est = T(0);
        if (cov > (T)1e-12f) {
            est = sub_rn(div_rn(data[t], cov), div_rn(background[t], cov));
            if (!isfinite(est)) record_error(err, STAGE_SETUP, t, ERR_NONFINITE_INITIAL);
        }
        estimate[t] = est;
    }
}

template <typename A, typename B>
__global__ void k_convert(const A *__restrict__ in, B *__restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) out[i] = (B)in[i];
}

// Maximum of a plane (order-independent), as an ordered double.
template <typename T>
__global__ void k_max_ordered(const T *__restrict__ in, size_t n, unsigned long long *__restrict__ out) {
    unsigned long long m = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long o = double_to_ordered((double)in[i]);
        m = o > m ? o : m;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, m, o);
        m = w > m ? w : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

template <typename T> __global__ void k_scale_plane(const T *__restrict__ in, T s, T *__restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = mul_rn(in[i], s);
}

}  // namespace updc
