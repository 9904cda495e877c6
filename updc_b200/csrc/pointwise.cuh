// Detector-space, target-space and setup kernels of the UPDC iteration.
#pragma once

#include "common.cuh"

namespace updc {

// Per-exposure device descriptor (one per exposure, uploaded at setup).
template <typename T> struct ExpDesc {
    const uint32_t *off, *base, *tgt;
    const uint16_t *delta;
    const float *frac;
    const uint32_t *toff, *tsrc;
    const float *tfrac;
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
// Warp-cooperative link staging.  A warp owns 32 consecutive detector pixels;
// their links occupy one contiguous range of the LinkMap, which the warp
// copies into shared memory with coalesced loads (one lane per link) before
// each lane walks its own pixel's links from there.  Ranges longer than
// DET_LCAP links fall back to direct loads for that tile.
constexpr int DET_WARPS = 8;
constexpr int DET_LCAP = 384;

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

// The fused detector loop of updc_core.c:1152-1176 for exposure blockIdx.y:
//   pred = sum_z fmaf(frac[z], blur[t(z)], pred) in link order;
//   raw_mu = pred + (background + pedestal);  FreezeMu;  ratio;  wr = W * ratio.
// Writes wr (0 for skipped pixels) for the adjoint gather.  With COMP the
// prediction is accumulated in FP64 and raw_mu is rounded once from the FP64
// sum with the offset, so the FreezeMu threshold is decided on a compensated
// raw_mu.
// Block `block` of `nblocks` over exposure k's pixels (grid-stride); the
// body of k_detector and of the batched detector (batch.cuh).
struct DetShared {
    uint32_t idx[DET_WARPS][DET_LCAP];
    float frac[DET_WARPS][DET_LCAP];
    unsigned long long nnew[DET_WARPS], ntot[DET_WARPS], mn[DET_WARPS];
};

template <typename T, bool COMP, bool DELTA16>
__device__ __forceinline__ void detector_tiles_enc(const ExpDesc<T> &e, int k, size_t nin, const T *__restrict__ blur,
                                                   T *__restrict__ wr, ExpStats *__restrict__ stats,
                                                   unsigned long long *__restrict__ err, unsigned block,
                                                   unsigned nblocks, DetShared &sh) {
    auto &s_idx = sh.idx;
    auto &s_frac = sh.frac;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long nnew = 0, ntot = 0, mn = ~0ull;
    const size_t step = (size_t)nblocks * DET_WARPS * 32;
    for (size_t p0 = ((size_t)block * DET_WARPS + warp) * 32; p0 < nin; p0 += step) {
        const size_t p = p0 + lane;
        const bool valid = p < nin;
        // every per-pixel load first (independent of each other)
        const uint32_t z0 = valid ? e.off[p] : 0u, z1 = valid ? e.off[p + 1] : 0u;
        const T w = valid ? e.wht[p] : T(0);
        const uint32_t bse = (valid && DELTA16) ? e.base[p] : 0u;
        const T sci = valid ? e.sci[p] : T(0);
        uint8_t fz = valid ? e.frozen[p] : (uint8_t)0;
        const int last = (int)min((size_t)31, nin - 1 - p0);
        const uint32_t zb = __shfl_sync(0xffffffffu, z0, 0);
        const uint32_t ze = __shfl_sync(0xffffffffu, z1, last);
        const uint32_t cnt = ze - zb;
        const bool staged = cnt <= (uint32_t)DET_LCAP;
        if (staged) {
            // all staging loads are issued before any store
            constexpr int NS = DET_LCAP / 32;
            float fv[NS];
            uint32_t iv[NS];
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                const uint32_t i = lane + 32u * j;
                fv[j] = i < cnt ? e.frac[zb + i] : 0.0f;
                iv[j] = i < cnt ? (DELTA16 ? (uint32_t)e.delta[zb + i] : e.tgt[zb + i]) : 0u;
            }
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                const uint32_t i = lane + 32u * j;
                if (i < cnt) {
                    s_frac[warp][i] = fv[j];
                    s_idx[warp][i] = iv[j];
                }
            }
        }
        __syncwarp();
        T out = T(0);
        if (valid) {
            if (w > T(0) && z0 != z1) {
                LinkSum<T> acc;
                if (staged) {
                    // gathers of a chunk are issued together, then the ordered sum
                    constexpr int CH = 4;
                    for (uint32_t zc = z0; zc < z1; zc += CH) {
                        T bl[CH];
                        float fr[CH];
#pragma unroll
                        for (int i = 0; i < CH; ++i) {
                            const bool ok = zc + i < z1;
                            const uint32_t j = ok ? zc + i - zb : 0u;
                            fr[i] = s_frac[warp][j];
                            bl[i] = ok ? blur[bse + s_idx[warp][j]] : T(0);
                        }
#pragma unroll
                        for (int i = 0; i < CH; ++i)
                            if (zc + i < z1) acc.template add<COMP>(fr[i], bl[i]);
                    }
                } else {
                    for (uint32_t z = z0; z < z1; ++z) {
                        const uint32_t t = DELTA16 ? bse + (uint32_t)e.delta[z] : e.tgt[z];
                        acc.template add<COMP>(e.frac[z], blur[t]);
                    }
                }
                const T raw_mu = acc.template finish<COMP>(e.mean_offset);
                if (!isfinite(raw_mu)) {
                    record_error(err, STAGE_DETECTOR, (uint64_t)k * nin + p, ERR_NONFINITE_MEAN);
                } else {
                    const unsigned long long o = double_to_ordered((double)raw_mu);
                    mn = o < mn ? o : mn;
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
                        const T y = add_rn(sci, e.pedestal);
                        ratio = div_rn(y, raw_mu);
                        if (!isfinite(ratio)) record_error(err, STAGE_DETECTOR, (uint64_t)k * nin + p, ERR_NONFINITE_RATIO);
                    }
                    out = mul_rn(w, ratio);
                }
            }
            wr[p] = out;
        }
        __syncwarp();  // the next tile reuses this warp's staging area
    }
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
                                               unsigned long long *__restrict__ err, unsigned block, unsigned nblocks) {
    __shared__ DetShared sh;
    if (e.delta16) detector_tiles_enc<T, COMP, true>(e, k, nin, blur, wr, stats, err, block, nblocks, sh);
    else detector_tiles_enc<T, COMP, false>(e, k, nin, blur, wr, stats, err, block, nblocks, sh);
}

template <typename T, bool COMP>
__global__ void __launch_bounds__(DET_WARPS * 32, 4) k_detector(const ExpDesc<T> *__restrict__ exps, size_t nin, size_t nout,
                                                           const T *__restrict__ blur_all, T *__restrict__ wr_all,
                                                           ExpStats *__restrict__ stats, unsigned long long *__restrict__ err) {
    const int k = blockIdx.y;
    const ExpDesc<T> e = exps[k];
    detector_tiles<T, COMP>(e, k, nin, blur_all + k * nout, wr_all + k * nin, stats, err, blockIdx.x, gridDim.x);
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
                src[i] = ok ? e.tsrc[ic + i] : 0u;
                fr[i] = ok ? e.tfrac[ic + i] : 0.0f;
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

// Fixed-order final reduction of per-block partials (deterministic).
__device__ __forceinline__ void reduce_partials_block(const double *part_sum, const unsigned long long *part_neg, int n,
                                                      double *out_sum, unsigned long long *out_neg) {
    __shared__ double s[256];
    __shared__ unsigned long long c[256];
    double a = 0;
    unsigned long long b = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a += part_sum[i];
        b += part_neg[i];
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
                const uint32_t p = e.tsrc[i];
                const T w = e.wht[p];
                if (!(w > T(0))) continue;
                const T q = mul_rn((T)e.tfrac[i], w);
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
