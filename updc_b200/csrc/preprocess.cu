// Per-exposure weight preprocessing on the GPU: the numeric part of the
// reference's Level-2 preparation (updc/_engine.py:287-408) — base-valid mask,
// asymmetric sigma clipping of SCI for the sky background, the sky
// VAR_POISSON median, the weight plane of the chosen mode, the pedestals and
// the metrics record — with results identical to the reference's NumPy code.
//
// Design.  Every median the reference takes is an order statistic, computed
// exactly here:
//  * SCI over the base-valid pixels is sorted once (radix sort of
//    order-preserving 32-bit keys).  Every clipping mask is base_valid ∩ an
//    open value window, i.e. one contiguous range of that sorted array, so a
//    clipping pass needs no pass over the image: the median is an index, the
//    MAD (median of |fl32(v - med)|) is the k-th smallest element of two
//    sorted runs (values below and above the median, whose deviations grow
//    away from it) found by a merge-path binary search, and the next window's
//    range is two binary searches.  Two masks are equal exactly when their
//    ranges are.
//  * VAR_POISSON over the sky mask and the positive WHT values are sorted the
//    same way (64- and 32-bit keys) for their medians.
//  * The rare standard-deviation fallback (MAD of zero) compacts the clipped
//    values in pixel order and sums them in NumPy's pairwise order (blocks of
//    at most 128 values with eight interleaved accumulators, halves split at
//    multiples of eight), so the float32 result is NumPy's.
// Thresholds follow NumPy 2's promotion rules: the float64 window bounds are
// rounded to float32 before comparing float32 SCI; a float32 median of an
// even count is the float32 mean of the middle pair; the final sigma is a
// float32 product of the float32-rounded 1.4826 and the float32 MAD.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/updc_b200.h"
#include "common.cuh"
#include "preprocess.cuh"

namespace updc {
namespace {

constexpr int PRE_NT = 256;
constexpr int PW_BLOCK = 128;  // NumPy's pairwise-summation block
constexpr double MAD_TO_SIGMA = 1.4826, CLIP_LOW = 4.5, CLIP_HIGH = 2.5;

enum WeightMode : int { WM_MASK = 0, WM_RNOISE_SKY = 1, WM_TOTALVAR = 2 };

unsigned pre_grid(size_t n) { return (unsigned)std::max<size_t>(1, std::min<size_t>(ceil_div(n, PRE_NT), 148 * 8)); }

struct PreCounters {
    unsigned long long valid, usable, nonpos_before, nonpos_after, wht_zero, wht_pos, sky;
    unsigned int min_usable_key;  // order-preserving key of the smallest usable SCI
    unsigned int pad;
};

// A thread's count, summed over its warp, added with one atomic per warp.
__device__ __forceinline__ void warp_add(unsigned count, unsigned long long *dst) {
    const unsigned sum = __reduce_add_sync(0xffffffffu, count);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(dst, (unsigned long long)sum);
}

__device__ __forceinline__ float key_value(const uint32_t *sorted, unsigned long long i) {
    return ordered_to_float(sorted[i]);
}

// base_valid (_engine.py:356-360) and the sort keys of valid SCI.  Counting
// kernels keep their counts in registers and add them once per warp; every
// thread of a warp runs the same number of loop trips (n rounded up).
__global__ void k_pre_valid(const float *__restrict__ sci, const uint32_t *__restrict__ dq,
                            const double *__restrict__ vp, const double *__restrict__ vr,
                            const double *__restrict__ vf, size_t n, uint32_t bad, int totalvar,
                            uint8_t *__restrict__ valid, uint32_t *__restrict__ keys, PreCounters *cnt) {
    unsigned c = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float s = sci[i];
        const bool ok = isfinite(s) && (dq[i] & bad) == 0 && isfinite(vp[i]) && isfinite(vr[i]) &&
                        (!totalvar || isfinite(vf[i]));
        valid[i] = ok;
        keys[i] = ok ? float_to_ordered(s) : 0xFFFFFFFFu;
        c += ok;
    }
    warp_add(c, &cnt->valid);
}

// the same keys from a caller-given base_valid mask
__global__ void k_pre_keys(const float *__restrict__ sci, const uint8_t *__restrict__ valid, size_t n,
                           uint32_t *__restrict__ keys, PreCounters *cnt) {
    unsigned c = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const bool ok = valid[i] != 0;
        keys[i] = ok ? float_to_ordered(sci[i]) : 0xFFFFFFFFu;
        c += ok;
    }
    warp_add(c, &cnt->valid);
}

// Smallest i in [lo, hi) with pred(i) true (pred goes false -> true once),
// or hi.  One warp: each round the 32 lanes test the last element of 32
// equal chunks and the search continues in the first chunk that ends true,
// so a range of 2^22 takes five rounds of loads instead of 22.
template <class Pred>
__device__ unsigned long long warp_first_true(unsigned long long lo, unsigned long long hi, Pred pred) {
    const unsigned lane = threadIdx.x & 31;
    while (hi - lo > 32) {
        const unsigned long long len = hi - lo, step = (len + 31) / 32;
        const unsigned long long end = min((unsigned long long)(lane + 1) * step, len);
        const unsigned m = __ballot_sync(0xffffffffu, pred(lo + end - 1));
        if (!m) return hi;
        const unsigned f = __ffs(m) - 1;
        hi = lo + min((unsigned long long)(f + 1) * step, len);
        lo += (unsigned long long)f * step;
    }
    const unsigned long long i = lo + lane;
    const unsigned m = __ballot_sync(0xffffffffu, i < hi && pred(i));
    return m ? lo + (__ffs(m) - 1) : hi;
}

// k-th smallest (0-based) of |fl32(v - med)| over sorted[a, b), split at p
// (values <= med before p): run A walks down from p-1, run B up from p, both
// with non-decreasing deviations; merge-path search for how many of the k+1
// smallest come from A.
__device__ float warp_kth_deviation(const uint32_t *s, unsigned long long a, unsigned long long b,
                                    unsigned long long p, float med, unsigned long long k) {
    const unsigned long long la = p - a, lb = b - p;
    auto A = [&](unsigned long long j) { return fabsf(__fsub_rn(key_value(s, p - 1 - j), med)); };
    auto B = [&](unsigned long long j) { return fabsf(__fsub_rn(key_value(s, p + j), med)); };
    const unsigned long long lo = (k + 1 > lb) ? k + 1 - lb : 0, hi = (k + 1 < la) ? k + 1 : la;
    const unsigned long long i = warp_first_true(lo, hi, [&](unsigned long long t) { return !(A(t) < B(k - t)); });
    const unsigned long long j = k + 1 - i;
    float r = -INFINITY;
    if (i > 0) r = A(i - 1);
    if (j > 0) r = fmaxf(r, B(j - 1));
    return r;
}

// median and MAD of sorted[a, b), b > a (numpy.median semantics in float32)
__device__ void warp_center(const uint32_t *s, unsigned long long a, unsigned long long b, float *med_out,
                            float *mad_out) {
    const unsigned long long m = b - a, k1 = (m - 1) / 2, k2 = m / 2;
    const float v1 = key_value(s, a + k1), v2 = key_value(s, a + k2);
    const float med = (m & 1) ? v1 : __fdiv_rn(__fadd_rn(v1, v2), 2.0f);
    const unsigned long long p = warp_first_true(a, b, [&](unsigned long long i) { return key_value(s, i) > med; });
    const float d1 = warp_kth_deviation(s, a, b, p, med, k1);
    const float d2 = (m & 1) ? d1 : warp_kth_deviation(s, a, b, p, med, k2);
    *med_out = med;
    *mad_out = (m & 1) ? d1 : __fdiv_rn(__fadd_rn(d1, d2), 2.0f);
}

enum ClipStatus : int { CLIP_RUN = 0, CLIP_DONE = 1, CLIP_TOO_FEW = 2, CLIP_NEED_STD = 3, CLIP_NO_RMS = 4 };

struct ClipState {
    unsigned long long a, b;  // current mask = sorted range [a, b) of the valid values
    int it, passes, fallbacks, status, windowed;
    float lo, hi;             // window of the current mask (windowed = 0: the mask is base_valid)
    double background, sigma;
};

// The clipping loop of _engine.py:293-310 on the sorted valid SCI, one warp.
// It stops with CLIP_NEED_STD when a pass's MAD is zero; the host then
// computes numpy.std of the current mask and relaunches with it.
__global__ void k_pre_clip(const uint32_t *__restrict__ s, unsigned long long nv, unsigned long long need,
                           int max_iter, ClipState *state, int has_std, float std_value) {
    ClipState c = *state;
    c.status = CLIP_RUN;
    for (; c.it < max_iter; ++c.it) {
        if (c.b - c.a < need) {
            c.status = CLIP_TOO_FEW;
            break;
        }
        float med, mad;
        warp_center(s, c.a, c.b, &med, &mad);
        double sig = __dmul_rn(MAD_TO_SIGMA, (double)mad);
        if (!(isfinite(sig) && sig > 0.0)) {
            if (!has_std) {
                c.status = CLIP_NEED_STD;
                break;
            }
            has_std = 0;
            sig = (double)std_value;
            ++c.fallbacks;
        }
        if (!(isfinite(sig) && sig > 0.0)) {
            c.status = CLIP_NO_RMS;
            break;
        }
        ++c.passes;
        // float64 bounds rounded to float32 for the float32 comparison
        c.lo = __double2float_rn(__dsub_rn((double)med, __dmul_rn(CLIP_LOW, sig)));
        c.hi = __double2float_rn(__dadd_rn((double)med, __dmul_rn(CLIP_HIGH, sig)));
        c.windowed = 1;
        const float lo = c.lo, hi = c.hi;
        unsigned long long a = warp_first_true(0, nv, [&](unsigned long long i) { return key_value(s, i) > lo; });
        unsigned long long b = warp_first_true(0, nv, [&](unsigned long long i) { return key_value(s, i) >= hi; });
        if (b <= a) a = b = 0;  // empty masks compare equal
        const bool same = a == c.a && b == c.b;
        c.a = a;
        c.b = b;
        if (same) break;
    }
    if (c.status == CLIP_RUN) {
        float med = NAN, mad = NAN;  // numpy.median of nothing
        if (c.b > c.a) warp_center(s, c.a, c.b, &med, &mad);
        c.background = med;
        // the final MAD stays float32, so 1.4826 is rounded to float32 too
        c.sigma = (double)__fmul_rn((float)MAD_TO_SIGMA, mad);
        c.status = CLIP_DONE;
    }
    if (threadIdx.x == 0) *state = c;
}

// flags of the pixels in the current clipping mask (pixel order)
__global__ void k_pre_mask_flags(const float *__restrict__ sci, const uint8_t *__restrict__ valid, size_t n,
                                 int windowed, float lo, float hi, uint8_t *__restrict__ flags) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float s = sci[i];
        flags[i] = valid[i] && (!windowed || (s > lo && s < hi));
    }
}

// ---- NumPy pairwise summation, float32
struct Leaf {
    unsigned long long lo;
    unsigned int n, pad;
};

__global__ void k_pw_leaves(unsigned long long n, Leaf *leaves, unsigned long long *count) {
    if (blockIdx.x || threadIdx.x) return;
    unsigned long long st_lo[128], st_n[128];
    int sp = 0;
    unsigned long long c = 0;
    st_lo[sp] = 0;
    st_n[sp++] = n;
    while (sp > 0) {
        --sp;
        const unsigned long long lo = st_lo[sp], len = st_n[sp];
        if (len <= PW_BLOCK) {
            leaves[c++] = Leaf{lo, (unsigned)len, 0};
            continue;
        }
        unsigned long long h = len / 2;
        h -= h % 8;
        st_lo[sp] = lo + h;  // right half below the left: left is taken first
        st_n[sp++] = len - h;
        st_lo[sp] = lo;
        st_n[sp++] = h;
    }
    *count = c;
}

__global__ void k_pw_leaf_sums(const float *__restrict__ v, const Leaf *__restrict__ leaves,
                               const unsigned long long *count, float *__restrict__ sums) {
    const unsigned long long nl = *count;
    for (unsigned long long l = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; l < nl;
         l += (unsigned long long)gridDim.x * blockDim.x) {
        const float *a = v + leaves[l].lo;
        const unsigned n = leaves[l].n;
        float res;
        if (n < 8) {
            res = -0.0f;
            for (unsigned i = 0; i < n; ++i) res = __fadd_rn(res, a[i]);
        } else {
            float r[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) r[j] = a[j];
            unsigned i = 8;
            for (; i < n - (n % 8); i += 8)
#pragma unroll
                for (int j = 0; j < 8; ++j) r[j] = __fadd_rn(r[j], a[i + j]);
            res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                            __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
            for (; i < n; ++i) res = __fadd_rn(res, a[i]);
        }
        sums[l] = res;
    }
}

// the recursion of the pairwise sum over the leaf sums, in its own order
__global__ void k_pw_combine(unsigned long long n, const float *__restrict__ sums, float *out) {
    if (blockIdx.x || threadIdx.x) return;
    struct Frame {
        unsigned long long n;
        int phase;
        float left;
    };
    Frame st[128];
    int sp = 0;
    unsigned long long cur = 0;
    float ret = 0.0f;
    st[sp++] = Frame{n, 0, 0.0f};
    while (sp > 0) {
        Frame &f = st[sp - 1];
        if (f.n <= PW_BLOCK) {
            ret = sums[cur++];
            --sp;
            continue;
        }
        unsigned long long h = f.n / 2;
        h -= h % 8;
        if (f.phase == 0) {
            f.phase = 1;
            st[sp++] = Frame{h, 0, 0.0f};
        } else if (f.phase == 1) {
            f.left = ret;
            f.phase = 2;
            st[sp++] = Frame{f.n - h, 0, 0.0f};
        } else {
            ret = __fadd_rn(f.left, ret);
            --sp;
        }
    }
    *out = __fadd_rn(-0.0f, ret);
}

__global__ void k_pre_sqdev(const float *__restrict__ v, unsigned long long n, float mean, float *__restrict__ out) {
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const float d = __fsub_rn(v[i], mean);
        out[i] = __fmul_rn(d, d);
    }
}

// final sky mask and the sort keys of VAR_POISSON over it (_engine.py:315)
__global__ void k_pre_sky(const float *__restrict__ sci, const uint8_t *__restrict__ valid,
                          const double *__restrict__ vp, size_t n, float lo, float hi, uint8_t *__restrict__ sky,
                          unsigned long long *__restrict__ keys, PreCounters *cnt) {
    unsigned c = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float s = sci[i];
        const bool in = valid[i] && s > lo && s < hi;
        if (sky) sky[i] = in;
        const double v = vp[i];
        const bool take = in && isfinite(v) && v >= 0.0;
        keys[i] = take ? double_to_ordered(v) : ~0ull;
        c += take;
    }
    warp_add(c, &cnt->sky);
}

// weights of the mode (_engine.py:317-332), the usable mask (in place of
// base_valid), WHT, and the counts and minimum of _engine.py:365-385
__global__ void k_pre_weight(const float *__restrict__ sci, uint8_t *__restrict__ valid_usable,
                             const double *__restrict__ vp, const double *__restrict__ vr,
                             const double *__restrict__ vf, size_t n, int mode, double sky_var_p,
                             float *__restrict__ wht, uint32_t *__restrict__ wkeys, PreCounters *cnt) {
    unsigned n_usable = 0, n_nonpos = 0, n_zero = 0, n_pos = 0, kmin = 0xFFFFFFFFu;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double w;
        if (mode == WM_MASK)
            w = 1.0;
        else if (mode == WM_RNOISE_SKY)
            w = __ddiv_rn(1.0, __dadd_rn(vr[i], sky_var_p));
        else
            w = __ddiv_rn(1.0, __dadd_rn(__dadd_rn(vp[i], vr[i]), vf[i]));
        const float s = sci[i];
        const bool usable = valid_usable[i] && isfinite(w) && w > 0.0;
        valid_usable[i] = usable;
        const float o = usable ? __double2float_rn(w) : 0.0f;
        wht[i] = o;
        wkeys[i] = o > 0.0f ? __float_as_uint(o) : 0xFFFFFFFFu;
        n_usable += usable;
        n_nonpos += usable && s <= 0.0f;
        n_zero += o == 0.0f;
        n_pos += o > 0.0f;
        if (usable) kmin = min(kmin, float_to_ordered(s));
    }
    warp_add(n_usable, &cnt->usable);
    warp_add(n_nonpos, &cnt->nonpos_before);
    warp_add(n_zero, &cnt->wht_zero);
    warp_add(n_pos, &cnt->wht_pos);
    kmin = __reduce_min_sync(0xffffffffu, kmin);
    if ((threadIdx.x & 31) == 0 && kmin != 0xFFFFFFFFu) atomicMin(&cnt->min_usable_key, kmin);
}

// ---- exact selection of the two middle order statistics of a key array
// (numpy.median's pair) without sorting: MSB-first radix select over 11-bit
// digits for both ranks at once.  Each pass histograms the keys that match
// the digits fixed so far; the last block of the pass to finish (a ticket
// counter, no waiting) fixes the next digit of each rank and clears the
// histograms for the next pass.  Keys equal to the all-ones sentinel mark
// non-participants and sort last, so they are never selected.
constexpr int SEL_BITS = 11, SEL_BINS = 1 << SEL_BITS;

template <typename K> struct SelectState {
    K prefix[2];
    unsigned long long rank[2];
    unsigned split;  // the two ranks' prefixes differ in the digits fixed so far
    unsigned ticket;
};

template <typename K>
__global__ void k_sel_init(SelectState<K> *st, const unsigned long long *count, unsigned *hist) {
    const unsigned long long m = *count;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->prefix[0] = st->prefix[1] = 0;
        st->rank[0] = m ? (m - 1) / 2 : 0;
        st->rank[1] = m / 2;
        st->split = 0;
        st->ticket = 0;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * SEL_BINS; i += gridDim.x * blockDim.x) hist[i] = 0;
}

// fix digit [shift, shift + width) of rank r from histogram h (SEL_PICK_NT threads)
constexpr int SEL_PICK_NT = 256, SEL_PER_THREAD = SEL_BINS / SEL_PICK_NT;

template <typename K>
__device__ void sel_fix_digit(SelectState<K> *st, int r, const unsigned *h, int shift, int width) {
    using Scan = cub::BlockScan<unsigned long long, SEL_PICK_NT>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int digit;
    __shared__ unsigned long long below;
    const int t = threadIdx.x, nb = 1 << width;
    unsigned c[SEL_PER_THREAD];
    unsigned long long mine = 0;
#pragma unroll
    for (int j = 0; j < SEL_PER_THREAD; ++j) {
        const int b = t * SEL_PER_THREAD + j;
        c[j] = b < nb ? __ldcg(h + b) : 0u;
        mine += c[j];
    }
    unsigned long long excl;
    Scan(tmp).ExclusiveSum(mine, excl);
    const unsigned long long rank = st->rank[r];
    if (rank >= excl && rank < excl + mine) {
        unsigned long long run = excl;
#pragma unroll
        for (int j = 0; j < SEL_PER_THREAD; ++j) {
            if (rank >= run && rank < run + c[j]) {
                digit = t * SEL_PER_THREAD + j;
                below = run;
            }
            run += c[j];
        }
    }
    __syncthreads();
    if (t == 0) {
        st->rank[r] = rank - below;
        st->prefix[r] |= (K)digit << shift;
    }
    __syncthreads();
}

template <typename K>
__global__ void __launch_bounds__(SEL_PICK_NT) k_sel_pass(const K *__restrict__ keys, size_t n, SelectState<K> *st,
                                                          int shift, int width, unsigned *hist) {
    __shared__ unsigned h[2 * SEL_BINS];
    __shared__ bool last;
    for (int i = threadIdx.x; i < 2 * SEL_BINS; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int bits = 8 * (int)sizeof(K);
    const K above = shift + width >= bits ? K(0) : (~K(0) << (shift + width));
    const K p0 = st->prefix[0] & above, p1 = st->prefix[1] & above;
    const bool split = st->split != 0;
    const unsigned dmask = (1u << width) - 1u;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const K k = keys[i];
        const unsigned d = (unsigned)(k >> shift) & dmask;
        const K hk = k & above;
        if (hk == p0) {
            const unsigned peers = __match_any_sync(__activemask(), d);
            if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&h[d], (unsigned)__popc(peers));
        }
        if (split && hk == p1) {
            const unsigned peers = __match_any_sync(__activemask(), d);
            if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&h[SEL_BINS + d], (unsigned)__popc(peers));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * SEL_BINS; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    sel_fix_digit(st, 0, hist, shift, width);
    sel_fix_digit(st, 1, hist + (split ? SEL_BINS : 0), shift, width);
    for (int i = threadIdx.x; i < 2 * SEL_BINS; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) {
        st->split = st->prefix[0] != st->prefix[1];
        st->ticket = 0;
    }
}

// ----------------------------------------------------------------------------- host side
// Scratch comes from a memory pool of its own per device that keeps what it
// has reserved (release threshold: never), so repeated calls reuse the same
// physical memory instead of mapping ~30 bytes per pixel afresh each time.
cudaMemPool_t scratch_pool() {
    static std::mutex m;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    UPDC_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(m);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    UPDC_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = UINT64_MAX;
    UPDC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[dev] = pool;
    return pool;
}

// Stream-ordered scratch, released (to the pool) in the destructor.
struct Scratch {
    cudaStream_t st;
    cudaMemPool_t pool;
    std::vector<void *> ptrs;
    explicit Scratch(cudaStream_t s) : st(s), pool(scratch_pool()) {}
    template <typename T> T *get(size_t n) {
        void *p = nullptr;
        UPDC_CUDA(cudaMallocFromPoolAsync(&p, std::max<size_t>(n, 1) * sizeof(T), pool, st));
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    ~Scratch() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
    }
};

template <typename T> void to_host(T *dst, const T *src, size_t n, cudaStream_t st) {
    UPDC_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    UPDC_CUDA(cudaStreamSynchronize(st));
}

// Python's max(a, b): the first argument unless the second is larger
double py_max(double a, double b) { return b > a ? b : a; }

// numpy.std of the values of the current mask, in pixel order (float32)
float masked_std(const float *sci, const uint8_t *valid, size_t n, bool windowed, float lo, float hi,
                 Scratch &S, cudaStream_t st) {
    uint8_t *flags = S.get<uint8_t>(n);
    float *vals = S.get<float>(n);
    unsigned long long *nsel = S.get<unsigned long long>(1);
    k_pre_mask_flags<<<pre_grid(n), PRE_NT, 0, st>>>(sci, valid, n, windowed, lo, hi, flags);
    size_t tb = 0;
    UPDC_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, sci, flags, vals, nsel, (int64_t)n, st));
    void *tmp = S.get<unsigned char>(tb);
    UPDC_CUDA(cub::DeviceSelect::Flagged(tmp, tb, sci, flags, vals, nsel, (int64_t)n, st));
    unsigned long long m = 0;
    to_host(&m, nsel, 1, st);
    const unsigned long long max_leaves = m / 64 + 2;
    Leaf *leaves = S.get<Leaf>(max_leaves);
    float *sums = S.get<float>(max_leaves);
    unsigned long long *nleaf = S.get<unsigned long long>(1);
    float *total = S.get<float>(1);
    float *sq = S.get<float>(m);
    const unsigned lg = pre_grid(max_leaves);
    k_pw_leaves<<<1, 1, 0, st>>>(m, leaves, nleaf);
    k_pw_leaf_sums<<<lg, PRE_NT, 0, st>>>(vals, leaves, nleaf, sums);
    k_pw_combine<<<1, 1, 0, st>>>(m, sums, total);
    float s1 = 0;
    to_host(&s1, total, 1, st);
    // mean: float32 sum / intp count in float64, stored back as float32
    const float mean = (float)((double)s1 / (double)m);
    k_pre_sqdev<<<pre_grid(m), PRE_NT, 0, st>>>(vals, m, mean, sq);
    k_pw_leaf_sums<<<lg, PRE_NT, 0, st>>>(sq, leaves, nleaf, sums);
    k_pw_combine<<<1, 1, 0, st>>>(m, sums, total);
    float s2 = 0;
    to_host(&s2, total, 1, st);
    const float var = (float)((double)s2 / (double)m);
    return sqrtf(var);
}

struct ClipResult {
    float lo = 0, hi = 0;  // window of the final mask (windowed = false: the mask is base_valid)
    bool windowed = false;
    double background = 0, sigma = 0;
    int passes = 0, fallbacks = 0;
};

template <typename K> void sort_keys(const K *keys, K *sorted, size_t n, Scratch &S, cudaStream_t st) {
    size_t tb = 0;
    UPDC_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys, sorted, (int)n, 0, 8 * (int)sizeof(K), st));
    void *tmp = S.get<unsigned char>(tb);
    UPDC_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tb, keys, sorted, (int)n, 0, 8 * (int)sizeof(K), st));
}

// the two middle order statistics (ranks (m-1)/2 and m/2) of the m keys that
// are not the sentinel; `count` is m on the device
template <typename K>
void middle_pair(const K *keys, size_t n, const unsigned long long *count, K *lo, K *hi, Scratch &S,
                 cudaStream_t st) {
    SelectState<K> *dst = S.get<SelectState<K>>(1);
    unsigned *hist = S.get<unsigned>(2 * SEL_BINS);
    k_sel_init<K><<<8, 256, 0, st>>>(dst, count, hist);
    const unsigned g = pre_grid(n);
    for (int top = 8 * (int)sizeof(K); top > 0;) {
        const int shift = std::max(0, top - SEL_BITS), width = top - shift;
        k_sel_pass<K><<<g, SEL_PICK_NT, 0, st>>>(keys, n, dst, shift, width, hist);
        top = shift;
    }
    UPDC_CUDA(cudaGetLastError());
    SelectState<K> h;
    to_host(&h, dst, 1, st);
    *lo = h.prefix[0];
    *hi = h.prefix[1];
}

// robust_background_mask (_engine.py:287-310) over device SCI and base_valid;
// `keys` holds the order-preserving keys of valid SCI (0xFFFFFFFF elsewhere)
ClipResult robust_clip(const float *sci, const uint8_t *valid, const uint32_t *keys, size_t n, int max_iter,
                       PreCounters *dcnt, Scratch &S, cudaStream_t st) {
    uint32_t *sorted = S.get<uint32_t>(n);
    ClipState *dstate = S.get<ClipState>(1);
    sort_keys(keys, sorted, n, S, st);
    PreCounters hc;
    to_host(&hc, dcnt, 1, st);
    const unsigned long long nv = hc.valid;
    const unsigned long long need = std::max<unsigned long long>(32, std::min<unsigned long long>(1000, n / 100));
    ClipState c = {};
    c.a = 0;
    c.b = nv;
    UPDC_CUDA(cudaMemcpyAsync(dstate, &c, sizeof(c), cudaMemcpyHostToDevice, st));
    int has_std = 0;
    float std_value = 0.0f;
    for (;;) {
        k_pre_clip<<<1, 32, 0, st>>>(sorted, nv, need, max_iter, dstate, has_std, std_value);
        UPDC_CUDA(cudaGetLastError());
        to_host(&c, dstate, 1, st);
        if (c.status == CLIP_TOO_FEW) throw Error(1, "Too few valid pixels for robust background estimation");
        if (c.status == CLIP_NO_RMS) throw Error(1, "Cannot estimate a positive background RMS");
        if (c.status != CLIP_NEED_STD) break;
        std_value = masked_std(sci, valid, n, c.windowed != 0, c.lo, c.hi, S, st);
        has_std = 1;
    }
    ClipResult r;
    r.lo = c.lo;
    r.hi = c.hi;
    r.windowed = c.windowed != 0;
    r.background = c.background;
    r.sigma = c.sigma;
    r.passes = c.passes;
    r.fallbacks = c.fallbacks;
    return r;
}

void check_size(size_t n) {
    if (n == 0 || n > (size_t)0x7FFFFFFF) throw Error(1, "invalid exposure size");
}

struct DeviceInputs {
    const float *sci;
    const uint32_t *dq;
    const double *vp, *vr, *vf;
};

}  // namespace

// ----------------------------------------------------------------------------- drivers
// prepare_one's numeric steps (_engine.py:356-397) on device planes.  WHT
// goes to `wht`, the sky mask to `sky` (both device, sky may be null).
// Throws Error(1, <the reference's ValueError message>), or Error(3, ...) for
// an unknown weight mode after the steps the reference runs before that check.
void preprocess_device(const DeviceInputs &in, size_t n, int mode, uint32_t bad, double pedestal_sigma,
                       const std::string &source, float *wht, uint8_t *sky, updc_preprocess_metrics *M,
                       cudaStream_t st) {
    check_size(n);
    Scratch S(st);
    const unsigned g = pre_grid(n);
    PreCounters *dcnt = S.get<PreCounters>(1);
    UPDC_CUDA(cudaMemsetAsync(dcnt, 0, sizeof(PreCounters), st));
    UPDC_CUDA(cudaMemsetAsync(&dcnt->min_usable_key, 0xFF, sizeof(unsigned), st));
    uint8_t *valid = S.get<uint8_t>(n);
    uint32_t *keys = S.get<uint32_t>(n);
    k_pre_valid<<<g, PRE_NT, 0, st>>>(in.sci, in.dq, in.vp, in.vr, in.vf, n, bad, mode == WM_TOTALVAR, valid, keys,
                                      dcnt);
    UPDC_CUDA(cudaGetLastError());
    const ClipResult clip = robust_clip(in.sci, valid, keys, n, 6, dcnt, S, st);

    // build_weight: sky VAR_POISSON median (_engine.py:315-317)
    unsigned long long *k64 = S.get<unsigned long long>(n);
    k_pre_sky<<<g, PRE_NT, 0, st>>>(in.sci, valid, in.vp, n, clip.lo, clip.hi, sky, k64, dcnt);
    UPDC_CUDA(cudaGetLastError());
    PreCounters hc;
    to_host(&hc, dcnt, 1, st);
    double sky_var_p = NAN;
    if (hc.sky) {
        unsigned long long lo = 0, hi = 0;
        middle_pair(k64, n, &dcnt->sky, &lo, &hi, S, st);
        const double v1 = ordered_to_double(lo), v2 = ordered_to_double(hi);
        sky_var_p = (hc.sky & 1) ? v1 : (v1 + v2) / 2.0;
    }
    if (!std::isfinite(sky_var_p) || sky_var_p < 0) throw Error(1, "Cannot estimate sky VAR_POISSON");
    if (mode != WM_MASK && mode != WM_RNOISE_SKY && mode != WM_TOTALVAR)
        throw Error(3, "unknown weight mode " + std::to_string(mode));

    // weights, usable mask, WHT and the pedestals (_engine.py:365-386)
    k_pre_weight<<<g, PRE_NT, 0, st>>>(in.sci, valid, in.vp, in.vr, in.vf, n, mode, sky_var_p, wht, keys, dcnt);
    UPDC_CUDA(cudaGetLastError());
    to_host(&hc, dcnt, 1, st);
    if (hc.usable == 0) throw Error(1, "No usable pixels remain in " + source);
    const double min_valid = (double)ordered_to_float(hc.min_usable_key);
    const double floor_ = py_max(1.0e-12, 1.0e-6 * clip.sigma);
    const double auto_ped = py_max(0.0, floor_ - min_valid);
    const double requested = py_max(0.0, pedestal_sigma * clip.sigma - clip.background);
    const double pedestal = py_max(auto_ped, requested);
    // y_eff = SCI + pedestal (float64) is monotonic in SCI, so a usable pixel
    // with y_eff <= 0 exists exactly when the smallest usable SCI gives one;
    // the reference raises before reporting how many
    if (min_valid + pedestal <= 0.0) throw Error(1, "Automatic pedestal failed to make y_eff positive in " + source);
    if (hc.wht_pos == 0) throw Error(1, "No usable pixels remain in " + source);

    // median of the positive WHT values (_engine.py:393)
    uint32_t lo = 0, hi = 0;
    middle_pair(keys, n, &dcnt->wht_pos, &lo, &hi, S, st);
    float w1, w2;
    memcpy(&w1, &lo, 4);
    memcpy(&w2, &hi, 4);
    const float wmed = (hc.wht_pos & 1) ? w1 : (w1 + w2) / 2.0f;

    M->background = clip.background;
    M->background_sigma = clip.sigma;
    M->poisson_pedestal = pedestal;
    M->auto_positivity_pedestal = auto_ped;
    M->requested_pedestal = requested;
    M->min_valid_science = min_valid;
    M->sky_var_poisson = sky_var_p;
    M->wht_valid_median = (double)wmed;
    M->base_invalid = (int64_t)(n - hc.valid);
    M->nonpositive_valid_before_pedestal = (int64_t)hc.nonpos_before;
    M->nonpositive_after_pedestal = 0;
    M->wht_zero = (int64_t)hc.wht_zero;
    M->clip_passes = clip.passes;
    M->std_fallbacks = clip.fallbacks;
}

// robust_background_mask alone: the final clipping mask to `mask` (device)
void robust_background_device(const float *sci, const uint8_t *base_valid, size_t n, int max_iter, uint8_t *mask,
                              double *background, double *sigma, int *passes, cudaStream_t st) {
    check_size(n);
    Scratch S(st);
    const unsigned g = pre_grid(n);
    PreCounters *dcnt = S.get<PreCounters>(1);
    UPDC_CUDA(cudaMemsetAsync(dcnt, 0, sizeof(PreCounters), st));
    uint32_t *keys = S.get<uint32_t>(n);
    k_pre_keys<<<g, PRE_NT, 0, st>>>(sci, base_valid, n, keys, dcnt);
    UPDC_CUDA(cudaGetLastError());
    const ClipResult clip = robust_clip(sci, base_valid, keys, n, max_iter, dcnt, S, st);
    k_pre_mask_flags<<<g, PRE_NT, 0, st>>>(sci, base_valid, n, clip.windowed, clip.lo, clip.hi, mask);
    UPDC_CUDA(cudaGetLastError());
    UPDC_CUDA(cudaStreamSynchronize(st));
    *background = clip.background;
    *sigma = clip.sigma;
    if (passes) *passes = clip.passes;
}

// Host-or-device wrapper of preprocess_device: with host pointers the planes
// are copied in and WHT / the sky mask copied out on `st`.
void preprocess_exposure(const float *sci, const uint32_t *dq, const double *vp, const double *vr,
                         const double *vf, size_t n, int mode, uint32_t bad, double pedestal_sigma,
                         const std::string &source, float *wht, uint8_t *sky, updc_preprocess_metrics *M,
                         bool device_pointers, cudaStream_t st) {
    check_size(n);
    if (!sci || !dq || !vp || !vr || !vf || !wht || !M) throw Error(1, "null preprocessing argument");
    if (device_pointers) {
        preprocess_device(DeviceInputs{sci, dq, vp, vr, vf}, n, mode, bad, pedestal_sigma, source, wht, sky, M, st);
        UPDC_CUDA(cudaStreamSynchronize(st));
        return;
    }
    Scratch S(st);
    float *dsci = S.get<float>(n), *dwht = S.get<float>(n);
    uint32_t *ddq = S.get<uint32_t>(n);
    double *dvp = S.get<double>(n), *dvr = S.get<double>(n), *dvf = S.get<double>(n);
    uint8_t *dsky = sky ? S.get<uint8_t>(n) : nullptr;
    UPDC_CUDA(cudaMemcpyAsync(dsci, sci, n * 4, cudaMemcpyHostToDevice, st));
    UPDC_CUDA(cudaMemcpyAsync(ddq, dq, n * 4, cudaMemcpyHostToDevice, st));
    UPDC_CUDA(cudaMemcpyAsync(dvp, vp, n * 8, cudaMemcpyHostToDevice, st));
    UPDC_CUDA(cudaMemcpyAsync(dvr, vr, n * 8, cudaMemcpyHostToDevice, st));
    UPDC_CUDA(cudaMemcpyAsync(dvf, vf, n * 8, cudaMemcpyHostToDevice, st));
    preprocess_device(DeviceInputs{dsci, ddq, dvp, dvr, dvf}, n, mode, bad, pedestal_sigma, source, dwht, dsky, M,
                      st);
    UPDC_CUDA(cudaMemcpyAsync(wht, dwht, n * 4, cudaMemcpyDeviceToHost, st));
    if (sky) UPDC_CUDA(cudaMemcpyAsync(sky, dsky, n, cudaMemcpyDeviceToHost, st));
    UPDC_CUDA(cudaStreamSynchronize(st));
}

void robust_background(const float *sci, const uint8_t *base_valid, size_t n, int max_iter, uint8_t *mask,
                       double *background, double *sigma, int *passes, bool device_pointers, cudaStream_t st) {
    check_size(n);
    if (!sci || !base_valid || !mask || !background || !sigma) throw Error(1, "null preprocessing argument");
    if (device_pointers) {
        robust_background_device(sci, base_valid, n, max_iter, mask, background, sigma, passes, st);
        return;
    }
    Scratch S(st);
    float *dsci = S.get<float>(n);
    uint8_t *dvalid = S.get<uint8_t>(n), *dmask = S.get<uint8_t>(n);
    UPDC_CUDA(cudaMemcpyAsync(dsci, sci, n * 4, cudaMemcpyHostToDevice, st));
    UPDC_CUDA(cudaMemcpyAsync(dvalid, base_valid, n, cudaMemcpyHostToDevice, st));
    robust_background_device(dsci, dvalid, n, max_iter, dmask, background, sigma, passes, st);
    UPDC_CUDA(cudaMemcpyAsync(mask, dmask, n, cudaMemcpyDeviceToHost, st));
    UPDC_CUDA(cudaStreamSynchronize(st));
}

}  // namespace updc
