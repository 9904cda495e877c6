// GPU PSF projector: a PSF sampled on detector pixels, each pixel's four
// corners mapped into target-pixel offsets about the PSF centre, is
// redistributed onto the target grid by exact polygon overlap
// (updc/c_core/psf_projector.c:82-172).  Output pixel q receives
//     out[q] = fmaf(value_p, area_pq / full_area_p, out[q])
// over the input pixels p in row-major order, with the overlap area of
// overlap.c (geometry.cuh, compiled without multiply-add contraction), so the
// projected PSF is bit-identical to the reference projector's.  On the GPU:
// count the overlaps of every input pixel, fill (q, p, frac) entries in p
// order, stable-sort them by q (entries of one q keep their p order), and let
// one thread per output pixel run its fmaf chain.
#include <cub/cub.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/updc_b200.h"
#include "common.cuh"
#include "geometry.cuh"

namespace updc {
namespace {

struct ProjShape {
    int iw, ih, hx, hy, ow, oh;
};

__device__ __forceinline__ bool proj_quad(const double *v, const float *in, const ProjShape &s, int p, Pt q[4],
                                          float *full, int *x0, int *x1, int *y0, int *y1) {
    const int x = p % s.iw, y = p / s.iw;
    if (in[p] == 0.0f) return false;
    const size_t a = 2 * ((size_t)y * (s.iw + 1) + x), b = a + 2 * (size_t)(s.iw + 1);
    q[0] = Pt{v[a], v[a + 1]};
    q[1] = Pt{v[b], v[b + 1]};
    q[2] = Pt{v[b + 2], v[b + 3]};
    q[3] = Pt{v[a + 2], v[a + 3]};
    *full = geo_area(q, 4);
    if (!isfinite(*full) || !(*full > 1.0e-12f)) return false;
    double mnx = q[0].x, mxx = mnx, mny = q[0].y, mxy = mny;
    for (int j = 1; j < 4; ++j) {
        if (q[j].x < mnx) mnx = q[j].x;
        if (q[j].x > mxx) mxx = q[j].x;
        if (q[j].y < mny) mny = q[j].y;
        if (q[j].y > mxy) mxy = q[j].y;
    }
    *x0 = (int)floor(mnx + 0.5);
    *x1 = (int)floor(mxx + 0.5);
    *y0 = (int)floor(mny + 0.5);
    *y1 = (int)floor(mxy + 0.5);
    if (*x0 < -s.hx) *x0 = -s.hx;
    if (*x1 > s.hx) *x1 = s.hx;
    if (*y0 < -s.hy) *y0 = -s.hy;
    if (*y1 > s.hy) *y1 = s.hy;
    return true;
}

__global__ void k_proj_count(const double *__restrict__ v, const float *__restrict__ in, ProjShape s,
                             uint32_t *__restrict__ count) {
    const int n = s.iw * s.ih;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        Pt q[4];
        float full;
        int x0, x1, y0, y1;
        uint32_t c = 0;
        if (proj_quad(v, in, s, p, q, &full, &x0, &x1, &y0, &y1))
            for (int ty = y0; ty <= y1; ++ty)
                for (int tx = x0; tx <= x1; ++tx)
                    if (geo_overlap(q, tx, ty) > 1.0e-8f) ++c;
        count[p] = c;
    }
}

__global__ void k_proj_fill(const double *__restrict__ v, const float *__restrict__ in, ProjShape s,
                            const uint32_t *__restrict__ off, uint32_t *__restrict__ key, uint32_t *__restrict__ src,
                            float *__restrict__ frac) {
    const int n = s.iw * s.ih;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        Pt q[4];
        float full;
        int x0, x1, y0, y1;
        uint32_t z = off[p];
        if (!proj_quad(v, in, s, p, q, &full, &x0, &x1, &y0, &y1)) continue;
        for (int ty = y0; ty <= y1; ++ty)
            for (int tx = x0; tx <= x1; ++tx) {
                const float area = geo_overlap(q, tx, ty);
                if (!(area > 1.0e-8f)) continue;
                key[z] = (uint32_t)((ty + s.hy) * s.ow + (tx + s.hx));
                src[z] = (uint32_t)p;
                frac[z] = __fdiv_rn(area, full);
                ++z;
            }
    }
}

// Segment starts of the q-sorted entries: first[q] = first entry of q.
__global__ void k_proj_bounds(const uint32_t *__restrict__ key, size_t n, uint32_t *__restrict__ first, size_t nout) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i <= n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t lo = i == 0 ? 0u : key[i - 1] + 1u;
        const uint32_t hi = i == n ? (uint32_t)nout : key[i];
        for (uint32_t q = lo; q <= hi && q < nout + 1; ++q) first[q] = (uint32_t)i;
    }
}

__global__ void k_proj_gather(const uint32_t *__restrict__ first, const uint32_t *__restrict__ src,
                              const float *__restrict__ frac, const float *__restrict__ in, size_t nout,
                              float *__restrict__ out) {
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nout; q += (size_t)gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (uint32_t z = first[q]; z < first[q + 1]; ++z) acc = __fmaf_rn(in[src[z]], frac[z], acc);
        out[q] = acc;
    }
}

__global__ void k_proj_iota(uint32_t *__restrict__ idx, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        idx[i] = (uint32_t)i;
}
__global__ void k_proj_permute(const uint32_t *__restrict__ idx, const uint32_t *__restrict__ src,
                               const float *__restrict__ frac, size_t n, uint32_t *__restrict__ src2,
                               float *__restrict__ frac2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        src2[i] = src[idx[i]];
        frac2[i] = frac[idx[i]];
    }
}

template <typename T> T *dev(size_t n) {
    T *p = nullptr;
    UPDC_CUDA(cudaMalloc(&p, (n ? n : 1) * sizeof(T)));
    return p;
}

// Exact-size raw read with the reference's messages (psf_projector.c:47-61).
void read_exact(const std::string &path, void *out, size_t bytes, const char *what) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) throw Error(1, std::string("cannot open ") + what);
    const bool full = fread(out, 1, bytes, f) == bytes;
    const bool trailing = full && fgetc(f) != EOF;
    fclose(f);
    if (!full) throw Error(1, std::string("short ") + what);
    if (trailing) throw Error(1, std::string(what) + " has trailing bytes");
}

double serial_sum(const float *d, size_t n, const char *what) {
    double t = 0.0;
    for (size_t i = 0; i < n; ++i) {
        if (!std::isfinite(d[i]) || d[i] < 0.0f) throw Error(1, std::string("PSF contains negative/non-finite pixels") + what);
        t += (double)d[i];
    }
    return t;
}

int half_extent(double m) {
    if (!(m >= 0.0) || !std::isfinite(m)) throw Error(1, "invalid PSF mapped extent");
    const double needed = m - 0.5 - 1.0e-7;
    if (needed <= 0.0) return 0;
    if (needed > 1000000.0) throw Error(1, "unreasonable PSF mapped extent");
    return (int)std::ceil(needed);
}

}  // namespace

// One projection (psf_projector.c:82-172): returns the projected PSF and fills
// the job record; throws Error with the reference's message on failure.
std::vector<float> psf_project(const float *input, int iw, int ih, const double *vertices, int *ow_out, int *oh_out,
                               double *input_sum, double *output_sum, uint64_t *overlaps) {
    const size_t nin = (size_t)iw * ih, nvert = (size_t)(iw + 1) * (ih + 1);
    *input_sum = serial_sum(input, nin, "");
    if (!(*input_sum > 0.0)) throw Error(1, "PSF input sum is zero");
    double mx = 0.0, my = 0.0;
    for (size_t i = 0; i < nvert; ++i) {
        const double x = vertices[2 * i], y = vertices[2 * i + 1];
        if (!std::isfinite(x) || !std::isfinite(y)) throw Error(1, "non-finite PSF mapped vertex");
        mx = std::max(mx, std::fabs(x));
        my = std::max(my, std::fabs(y));
    }
    ProjShape s{iw, ih, half_extent(mx), half_extent(my), 0, 0};
    s.ow = 2 * s.hx + 1;
    s.oh = 2 * s.hy + 1;
    const size_t nout = (size_t)s.ow * s.oh;
    if ((uint64_t)nout >= 0xFFFFFFFFull) throw Error(1, "invalid PSF output shape");
    cudaStream_t st;
    UPDC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    std::vector<void *> bufs;
    auto keep = [&](void *p) { bufs.push_back(p); return p; };
    std::vector<float> out(nout);
    try {
        double *dv = (double *)keep(dev<double>(2 * nvert));
        float *din = (float *)keep(dev<float>(nin));
        uint32_t *cnt = (uint32_t *)keep(dev<uint32_t>(nin + 1));
        uint32_t *off = (uint32_t *)keep(dev<uint32_t>(nin + 1));
        UPDC_CUDA(cudaMemcpyAsync(dv, vertices, 2 * nvert * 8, cudaMemcpyHostToDevice, st));
        UPDC_CUDA(cudaMemcpyAsync(din, input, nin * 4, cudaMemcpyHostToDevice, st));
        UPDC_CUDA(cudaMemsetAsync(cnt, 0, (nin + 1) * 4, st));
        const unsigned g = (unsigned)std::min<size_t>(ceil_div(nin, 128), 148 * 16);
        k_proj_count<<<g, 128, 0, st>>>(dv, din, s, cnt);
        size_t tmpb = 0;
        UPDC_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmpb, cnt, off, (int)(nin + 1), st));
        void *tmp = keep(dev<unsigned char>(tmpb));
        UPDC_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmpb, cnt, off, (int)(nin + 1), st));
        uint32_t total = 0;
        UPDC_CUDA(cudaMemcpyAsync(&total, off + nin, 4, cudaMemcpyDeviceToHost, st));
        UPDC_CUDA(cudaStreamSynchronize(st));
        *overlaps = total;
        uint32_t *key = (uint32_t *)keep(dev<uint32_t>(total)), *key2 = (uint32_t *)keep(dev<uint32_t>(total));
        uint32_t *src = (uint32_t *)keep(dev<uint32_t>(total)), *src2 = (uint32_t *)keep(dev<uint32_t>(total));
        float *fr = (float *)keep(dev<float>(total)), *fr2 = (float *)keep(dev<float>(total));
        uint32_t *idx = (uint32_t *)keep(dev<uint32_t>(total)), *idx2 = (uint32_t *)keep(dev<uint32_t>(total));
        k_proj_fill<<<g, 128, 0, st>>>(dv, din, s, off, key, src, fr);
        // stable sort of (key, entry index): entries of one output pixel keep
        // their input-pixel order
        k_proj_iota<<<(unsigned)std::min<size_t>(ceil_div((size_t)total, 256), 148 * 16), 256, 0, st>>>(idx, total);
        int bits = 1;
        while (bits < 32 && (1ull << bits) < nout) ++bits;
        size_t sb = 0;
        UPDC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, sb, key, key2, idx, idx2, (int)total, 0, bits, st));
        void *stmp = keep(dev<unsigned char>(sb));
        UPDC_CUDA(cub::DeviceRadixSort::SortPairs(stmp, sb, key, key2, idx, idx2, (int)total, 0, bits, st));
        k_proj_permute<<<(unsigned)std::min<size_t>(ceil_div((size_t)total, 256), 148 * 16), 256, 0, st>>>(
            idx2, src, fr, total, src2, fr2);
        uint32_t *first = (uint32_t *)keep(dev<uint32_t>(nout + 1));
        k_proj_bounds<<<(unsigned)std::min<size_t>(ceil_div((size_t)total + 1, 256), 148 * 16), 256, 0, st>>>(
            key2, total, first, nout);
        float *dout = (float *)keep(dev<float>(nout));
        k_proj_gather<<<(unsigned)std::min<size_t>(ceil_div(nout, 256), 148 * 16), 256, 0, st>>>(first, src2, fr2, din,
                                                                                                  nout, dout);
        UPDC_CUDA(cudaGetLastError());
        UPDC_CUDA(cudaMemcpyAsync(out.data(), dout, nout * 4, cudaMemcpyDeviceToHost, st));
        UPDC_CUDA(cudaStreamSynchronize(st));
    } catch (...) {
        for (void *p : bufs) cudaFree(p);
        cudaStreamDestroy(st);
        throw;
    }
    for (void *p : bufs) cudaFree(p);
    cudaStreamDestroy(st);
    *output_sum = serial_sum(out.data(), nout, "");
    *ow_out = s.ow;
    *oh_out = s.oh;
    return out;
}

}  // namespace updc

using namespace updc;

extern "C" int updc_psf_project_file(const char *input, int width, int height, const char *vertices,
                                      const char *output, int *out_width, int *out_height, double *input_sum,
                                      double *output_sum, uint64_t *overlaps, char *message, size_t capacity) {
    try {
        if (!input || !vertices || !output || width < 1 || height < 1) throw Error(1, "invalid PSF input dimensions");
        const size_t nin = (size_t)width * height, nv = 2 * (size_t)(width + 1) * (height + 1);
        std::vector<float> in(nin);
        std::vector<double> v(nv);
        read_exact(input, in.data(), nin * 4, "PSF raw input");
        read_exact(vertices, v.data(), nv * 8, "PSF vertex map");
        int ow = 0, oh = 0;
        double is = 0, os = 0;
        uint64_t ov = 0;
        std::vector<float> out = psf_project(in.data(), width, height, v.data(), &ow, &oh, &is, &os, &ov);
        if (out_width) *out_width = ow;
        if (out_height) *out_height = oh;
        if (input_sum) *input_sum = is;
        if (output_sum) *output_sum = os;
        if (overlaps) *overlaps = ov;
        if (std::fabs((os - is) / is) > 5.0e-5) {
            if (message && capacity) snprintf(message, capacity, "PSF polygon projection is not flux-conserving");
            return 2;
        }
        FILE *f = fopen(output, "wb");
        if (!f) throw Error(1, "cannot create projected PSF raw output");
        const bool ok = fwrite(out.data(), sizeof(float), out.size(), f) == out.size();
        if (!ok) {
            fclose(f);
            throw Error(1, "short PSF raw output write");
        }
        if (fclose(f)) throw Error(1, "cannot close projected PSF raw output");
        if (message && capacity) message[0] = 0;
        return 0;
    } catch (const std::exception &e) {
        if (message && capacity) snprintf(message, capacity, "%s", e.what());
        return 1;
    }
}
