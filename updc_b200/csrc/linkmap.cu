// LinkMap v2 reader, GPU builder, validation and target-major transpose.
// Compiled with -fmad=false (see geometry.cuh).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cub/cub.cuh>
#include <cstring>
#include <memory>

#include "geometry.cuh"
#include "linkmap.cuh"

namespace updc {

void DevLinkMap::release() {
    for (void *p : {(void *)off, (void *)base, (void *)tgt, (void *)delta, (void *)frac, (void *)toff, (void *)tent})
        if (p) cudaFree(p);
    off = base = tgt = toff = nullptr;
    tent = nullptr;
    delta = nullptr;
    frac = nullptr;
}

size_t linkmap_expected_bytes(const LinkMapHeader &h, size_t nin) {
    if (h.header_bytes != sizeof(LinkMapHeader)) return 0;
    if (h.nin != nin || h.nlinks > UINT32_MAX) return 0;
    size_t pos = sizeof(LinkMapHeader) + (nin + 1) * sizeof(uint32_t);
    if (h.encoding == LINKMAP_DELTA16) {
        pos += nin * sizeof(uint32_t);
        pos += (size_t)h.nlinks * sizeof(uint16_t);
        pos = (pos + 3) & ~(size_t)3;
        pos += (size_t)h.nlinks * sizeof(float);
    } else if (h.encoding == LINKMAP_ABS32) {
        pos += (size_t)h.nlinks * sizeof(uint32_t);
        pos += (size_t)h.nlinks * sizeof(float);
    } else {
        return 0;
    }
    return pos;
}

namespace {

struct PinnedBuffer {
    void *p = nullptr;
    size_t n = 0;
    ~PinnedBuffer() {
        if (p) cudaFreeHost(p);
    }
    void *get(size_t bytes) {
        if (bytes > n) {
            if (p) cudaFreeHost(p);
            p = nullptr;
            n = 0;
            UPDC_CUDA(cudaMallocHost(&p, bytes));
            n = bytes;
        }
        return p;
    }
};

template <typename T> T *dev_alloc(size_t count) {
    T *p = nullptr;
    UPDC_CUDA(cudaMalloc(&p, (count ? count : 1) * sizeof(T)));
    return p;
}

bool read_exact(int fd, void *dst, size_t bytes) {
    char *d = (char *)dst;
    while (bytes) {
        ssize_t r = ::read(fd, d, bytes > (1u << 30) ? (1u << 30) : bytes);
        if (r <= 0) return false;
        d += r;
        bytes -= (size_t)r;
    }
    return true;
}

}  // namespace

bool linkmap_load(const std::string &path, size_t nin, int W, int H, DevLinkMap &out, cudaStream_t s) {
    struct stat st;
    if (stat(path.c_str(), &st) || st.st_size < (off_t)sizeof(LinkMapHeader)) return false;
    int fd = open(path.c_str(), O_RDONLY);
    if (fd < 0) return false;
    LinkMapHeader h;
    if (!read_exact(fd, &h, sizeof(h)) || h.magic != LINKMAP_MAGIC || h.version != LINKMAP_VERSION ||
        h.target_width != (uint32_t)W || h.target_height != (uint32_t)H) {
        close(fd);
        return false;
    }
    const size_t expected = linkmap_expected_bytes(h, nin);
    if (!expected || (size_t)st.st_size != expected) {
        close(fd);
        return false;
    }
    static PinnedBuffer staging;
    const size_t body = expected - sizeof(h);
    char *host = (char *)staging.get(body);
    const bool ok = read_exact(fd, host, body);
    close(fd);
    if (!ok) return false;
    const uint32_t *hoff = (const uint32_t *)host;
    if (hoff[nin] != (uint32_t)h.nlinks) throw Error(1, "LinkMap offset/link-count mismatch");
    out.release();
    out.encoding = h.encoding;
    out.nlinks = h.nlinks;
    out.nin = nin;
    out.file_bytes = expected;
    size_t pos = 0;
    out.off = dev_alloc<uint32_t>(nin + 1);
    UPDC_CUDA(cudaMemcpyAsync(out.off, host + pos, (nin + 1) * 4, cudaMemcpyHostToDevice, s));
    pos += (nin + 1) * 4;
    if (h.encoding == LINKMAP_DELTA16) {
        out.base = dev_alloc<uint32_t>(nin);
        UPDC_CUDA(cudaMemcpyAsync(out.base, host + pos, nin * 4, cudaMemcpyHostToDevice, s));
        pos += nin * 4;
        out.delta = dev_alloc<uint16_t>(h.nlinks + 8);  // 16 bytes of slack: whole-vector loads
        UPDC_CUDA(cudaMemcpyAsync(out.delta, host + pos, h.nlinks * 2, cudaMemcpyHostToDevice, s));
        pos += h.nlinks * 2;
        pos = ((pos + sizeof(h) + 3) & ~(size_t)3) - sizeof(h);
    } else {
        out.tgt = dev_alloc<uint32_t>(h.nlinks + 4);  // 16 bytes of slack: whole-vector loads
        UPDC_CUDA(cudaMemcpyAsync(out.tgt, host + pos, h.nlinks * 4, cudaMemcpyHostToDevice, s));
        pos += h.nlinks * 4;
    }
    out.frac = dev_alloc<float>(h.nlinks + 4);  // 16 bytes of slack: whole-vector loads
    UPDC_CUDA(cudaMemcpyAsync(out.frac, host + pos, h.nlinks * 4, cudaMemcpyHostToDevice, s));
    UPDC_CUDA(cudaStreamSynchronize(s));  // the staging buffer is reused by the next call
    return true;
}

// ---------------------------------------------------------------------------- builder
namespace {

__global__ void k_lm_count(const double *__restrict__ v, int iw, int ih, int W, int H, uint32_t *__restrict__ count,
                           uint32_t *__restrict__ first, unsigned int *__restrict__ flags) {
    const size_t nin = (size_t)iw * ih;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < nin; p += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % iw), y = (int)(p / iw);
        Pt q[4];
        float full;
        int x0, x1, y0, y1;
        uint32_t c = 0, f = 0, l = 0;
        if (geo_pixel_quad(v, iw, W, H, x, y, q, &full, &x0, &x1, &y0, &y1)) {
            for (int ty = y0; ty <= y1; ++ty)
                for (int tx = x0; tx <= x1; ++tx) {
                    if (geo_overlap(q, tx, ty) <= 1.0e-5f) continue;
                    const uint32_t t = (uint32_t)((size_t)ty * W + tx);
                    if (c == 0) f = t;
                    l = t;
                    ++c;
                }
        }
        count[p] = c;
        first[p] = c ? f : 0u;
        if (c && l - f > 0xFFFFu) atomicOr(flags, 1u);
    }
}

__global__ void k_lm_fill(const double *__restrict__ v, int iw, int ih, int W, int H, const uint64_t *__restrict__ off,
                          const uint32_t *__restrict__ first, int delta16, uint16_t *__restrict__ delta,
                          uint32_t *__restrict__ tgt, float *__restrict__ frac) {
    const size_t nin = (size_t)iw * ih;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < nin; p += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % iw), y = (int)(p / iw);
        Pt q[4];
        float full;
        int x0, x1, y0, y1;
        uint64_t z = off[p];
        if (!geo_pixel_quad(v, iw, W, H, x, y, q, &full, &x0, &x1, &y0, &y1)) continue;
        for (int ty = y0; ty <= y1; ++ty)
            for (int tx = x0; tx <= x1; ++tx) {
                const float area = geo_overlap(q, tx, ty);
                if (area <= 1.0e-5f) continue;
                const uint32_t t = (uint32_t)((size_t)ty * W + tx);
                if (delta16) delta[z] = (uint16_t)(t - first[p]);
                else tgt[z] = t;
                frac[z] = area / full;
                ++z;
            }
    }
}

__global__ void k_u32_to_u64(const uint32_t *in, uint64_t *out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) out[i] = in[i];
}

int grid_for(size_t n, int threads) {
    size_t g = (n + threads - 1) / threads;
    return (int)(g > 148 * 32 ? 148 * 32 : (g ? g : 1));
}

}  // namespace

void linkmap_build(const std::string &vertices_path, const std::string &path, int iw, int ih, int W, int H,
                   cudaStream_t s, LinkBuildStats *stats) {
    const size_t nin = (size_t)iw * ih, nv = 2 * (size_t)(iw + 1) * (ih + 1);
    std::vector<double> hv(nv);
    {
        FILE *f = fopen(vertices_path.c_str(), "rb");
        if (!f) throw Error(1, "cannot open vertex map");
        const size_t got = fread(hv.data(), sizeof(double), nv, f);
        fclose(f);
        if (got != nv) throw Error(1, "short vertex map");
    }
    double *dv = dev_alloc<double>(nv);
    uint32_t *count = dev_alloc<uint32_t>(nin + 1), *first = dev_alloc<uint32_t>(nin);
    uint64_t *count64 = dev_alloc<uint64_t>(nin + 1), *off64 = dev_alloc<uint64_t>(nin + 1);
    unsigned int *flags = dev_alloc<unsigned int>(1);
    UPDC_CUDA(cudaMemcpyAsync(dv, hv.data(), nv * 8, cudaMemcpyHostToDevice, s));
    UPDC_CUDA(cudaMemsetAsync(flags, 0, 4, s));
    UPDC_CUDA(cudaMemsetAsync(count + nin, 0, 4, s));
    k_lm_count<<<grid_for(nin, 256), 256, 0, s>>>(dv, iw, ih, W, H, count, first, flags);
    UPDC_CUDA(cudaGetLastError());
    k_u32_to_u64<<<grid_for(nin + 1, 256), 256, 0, s>>>(count, count64, nin + 1);
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, count64, off64, (int)(nin + 1), s);
    void *tmp = dev_alloc<char>(tmp_bytes);
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, count64, off64, (int)(nin + 1), s);
    uint64_t nlinks = 0;
    unsigned int hflags = 0;
    UPDC_CUDA(cudaMemcpyAsync(&nlinks, off64 + nin, 8, cudaMemcpyDeviceToHost, s));
    UPDC_CUDA(cudaMemcpyAsync(&hflags, flags, 4, cudaMemcpyDeviceToHost, s));
    UPDC_CUDA(cudaStreamSynchronize(s));
    if (nlinks > UINT32_MAX) throw Error(1, "LinkMap exceeds uint32 offset capacity");
    const int delta16 = (hflags & 1u) ? 0 : 1;
    LinkMapHeader h;
    memset(&h, 0, sizeof(h));
    h.magic = LINKMAP_MAGIC;
    h.version = LINKMAP_VERSION;
    h.encoding = delta16 ? LINKMAP_DELTA16 : LINKMAP_ABS32;
    h.header_bytes = sizeof(h);
    h.nin = nin;
    h.nlinks = nlinks;
    h.target_width = (uint32_t)W;
    h.target_height = (uint32_t)H;
    const size_t bytes = linkmap_expected_bytes(h, nin);
    if (!bytes) throw Error(1, "cannot size LinkMap");
    uint16_t *ddelta = delta16 ? dev_alloc<uint16_t>(nlinks) : nullptr;
    uint32_t *dtgt = delta16 ? nullptr : dev_alloc<uint32_t>(nlinks);
    float *dfrac = dev_alloc<float>(nlinks);
    k_lm_fill<<<grid_for(nin, 256), 256, 0, s>>>(dv, iw, ih, W, H, off64, first, delta16, ddelta, dtgt, dfrac);
    UPDC_CUDA(cudaGetLastError());
    // offsets as u32 for the file
    std::vector<uint64_t> hoff64(nin + 1);
    std::vector<char> file(bytes, 0);
    UPDC_CUDA(cudaMemcpyAsync(hoff64.data(), off64, (nin + 1) * 8, cudaMemcpyDeviceToHost, s));
    size_t pos = sizeof(h);
    memcpy(file.data(), &h, sizeof(h));
    char *off_dst = file.data() + pos;
    pos += (nin + 1) * 4;
    if (delta16) {
        UPDC_CUDA(cudaMemcpyAsync(file.data() + pos, first, nin * 4, cudaMemcpyDeviceToHost, s));
        pos += nin * 4;
        UPDC_CUDA(cudaMemcpyAsync(file.data() + pos, ddelta, nlinks * 2, cudaMemcpyDeviceToHost, s));
        pos += nlinks * 2;
        pos = (pos + 3) & ~(size_t)3;
    } else {
        UPDC_CUDA(cudaMemcpyAsync(file.data() + pos, dtgt, nlinks * 4, cudaMemcpyDeviceToHost, s));
        pos += nlinks * 4;
    }
    UPDC_CUDA(cudaMemcpyAsync(file.data() + pos, dfrac, nlinks * 4, cudaMemcpyDeviceToHost, s));
    UPDC_CUDA(cudaStreamSynchronize(s));
    for (size_t p = 0; p <= nin; ++p) {
        const uint32_t o = (uint32_t)hoff64[p];
        memcpy(off_dst + 4 * p, &o, 4);
    }
    uint32_t maxl = 0;
    uint64_t active = 0;
    for (size_t p = 0; p < nin; ++p) {
        const uint32_t c = (uint32_t)(hoff64[p + 1] - hoff64[p]);
        if (c) ++active;
        if (c > maxl) maxl = c;
    }
    const std::string tmp_path = path + ".build." + std::to_string((long)getpid());
    FILE *f = fopen(tmp_path.c_str(), "wb");
    if (!f) throw Error(1, "cannot create LinkMap");
    const bool wrote = fwrite(file.data(), 1, bytes, f) == bytes;
    const bool synced = fflush(f) == 0 && fsync(fileno(f)) == 0;
    if (fclose(f) || !wrote || !synced) throw Error(1, "LinkMap close failed");
    if (rename(tmp_path.c_str(), path.c_str())) throw Error(1, "LinkMap rename failed");
    for (void *p : {(void *)dv, (void *)count, (void *)first, (void *)count64, (void *)off64, (void *)flags, tmp,
                    (void *)ddelta, (void *)dtgt, (void *)dfrac})
        if (p) cudaFree(p);
    if (stats) {
        stats->nlinks = nlinks;
        stats->encoding = h.encoding;
        stats->active = active;
        stats->max_links = maxl;
    }
}

// ---------------------------------------------------------------------------- transpose
namespace {

// owner pixel and absolute target of every link; validates offsets/targets
__global__ void k_lm_expand(const uint32_t *__restrict__ off, const uint32_t *__restrict__ base,
                            const uint16_t *__restrict__ delta, const uint32_t *__restrict__ tgt, size_t nin,
                            uint64_t nlinks, size_t nout, uint32_t *__restrict__ owner, uint32_t *__restrict__ target,
                            uint32_t *__restrict__ cnt, unsigned int *__restrict__ bad) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < nin; p += (size_t)gridDim.x * blockDim.x) {
        const uint32_t z0 = off[p], z1 = off[p + 1];
        if (z0 > z1 || z1 > nlinks) {
            atomicOr(bad, 1u);
            continue;
        }
        for (uint32_t z = z0; z < z1; ++z) {
            const uint32_t t = base ? base[p] + (uint32_t)delta[z] : tgt[z];
            if ((size_t)t >= nout) {
                atomicOr(bad, 2u);
                target[z] = 0xFFFFFFFFu;
                owner[z] = (uint32_t)p;
                continue;
            }
            owner[z] = (uint32_t)p;
            target[z] = t;
            atomicAdd(&cnt[t], 1u);
        }
    }
}

// links never referenced by an offset range keep owner = target = ~0
__global__ void k_fill_u32(uint32_t *p, uint32_t v, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_lm_scatter_entries(const uint32_t *__restrict__ owner, const uint32_t *__restrict__ target,
                                     const float *__restrict__ frac, uint64_t nlinks, const uint32_t *__restrict__ toff,
                                     uint32_t *__restrict__ cursor, uint2 *__restrict__ tent) {
    for (size_t z = blockIdx.x * (size_t)blockDim.x + threadIdx.x; z < nlinks; z += (size_t)gridDim.x * blockDim.x) {
        const uint32_t t = target[z];
        if (t == 0xFFFFFFFFu) continue;
        const uint32_t pos = toff[t] + atomicAdd(&cursor[t], 1u);
        tent[pos] = make_uint2(owner[z], __float_as_uint(frac[z]));
    }
}

// insertion sort of each target's short segment by source pixel
__global__ void k_lm_sort_segments(const uint32_t *__restrict__ toff, size_t nout, uint2 *__restrict__ tent) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nout; t += (size_t)gridDim.x * blockDim.x) {
        const uint32_t a = toff[t], b = toff[t + 1];
        for (uint32_t i = a + 1; i < b; ++i) {
            const uint2 k = tent[i];
            uint32_t j = i;
            while (j > a && tent[j - 1].x > k.x) {
                tent[j] = tent[j - 1];
                --j;
            }
            tent[j] = k;
        }
    }
}

__global__ void k_lm_decode(const uint32_t *__restrict__ off, const uint32_t *__restrict__ base,
                            const uint16_t *__restrict__ delta, const uint32_t *__restrict__ tgt, size_t nin,
                            uint32_t *__restrict__ out) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < nin; p += (size_t)gridDim.x * blockDim.x) {
        for (uint32_t z = off[p]; z < off[p + 1]; ++z) out[z] = base ? base[p] + (uint32_t)delta[z] : tgt[z];
    }
}

}  // namespace

void linkmap_transpose(DevLinkMap &m, size_t nout, cudaStream_t s) {
    const size_t nin = m.nin;
    const uint64_t nl = m.nlinks;
    uint32_t *owner = dev_alloc<uint32_t>(nl), *target = dev_alloc<uint32_t>(nl);
    uint32_t *cnt = dev_alloc<uint32_t>(nout + 1);
    unsigned int *bad = dev_alloc<unsigned int>(1);
    UPDC_CUDA(cudaMemsetAsync(cnt, 0, (nout + 1) * 4, s));
    UPDC_CUDA(cudaMemsetAsync(bad, 0, 4, s));
    k_fill_u32<<<grid_for(nl, 256), 256, 0, s>>>(target, 0xFFFFFFFFu, nl);
    k_lm_expand<<<grid_for(nin, 256), 256, 0, s>>>(m.off, m.encoding == LINKMAP_DELTA16 ? m.base : nullptr, m.delta,
                                                  m.tgt, nin, nl, nout, owner, target, cnt, bad);
    UPDC_CUDA(cudaGetLastError());
    unsigned int hbad = 0;
    UPDC_CUDA(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, s));
    UPDC_CUDA(cudaStreamSynchronize(s));
    if (hbad) {
        cudaFree(owner);
        cudaFree(target);
        cudaFree(cnt);
        cudaFree(bad);
        throw Error(1, (hbad & 2u) ? "LinkMap target outside the target grid" : "invalid or obsolete LinkMap cache");
    }
    m.toff = dev_alloc<uint32_t>(nout + 1);
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cnt, m.toff, (int)(nout + 1), s);
    void *tmp = dev_alloc<char>(tmp_bytes);
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cnt, m.toff, (int)(nout + 1), s);
    UPDC_CUDA(cudaMemsetAsync(cnt, 0, (nout + 1) * 4, s));
    m.tent = dev_alloc<uint2>(nl);
    k_lm_scatter_entries<<<grid_for(nl, 256), 256, 0, s>>>(owner, target, m.frac, nl, m.toff, cnt, m.tent);
    k_lm_sort_segments<<<grid_for(nout, 256), 256, 0, s>>>(m.toff, nout, m.tent);
    UPDC_CUDA(cudaGetLastError());
    UPDC_CUDA(cudaStreamSynchronize(s));
    cudaFree(owner);
    cudaFree(target);
    cudaFree(cnt);
    cudaFree(bad);
    cudaFree(tmp);
}

void linkmap_decode(const DevLinkMap &m, uint32_t *targets, cudaStream_t s) {
    k_lm_decode<<<grid_for(m.nin, 256), 256, 0, s>>>(m.off, m.encoding == LINKMAP_DELTA16 ? m.base : nullptr,
                                                      m.delta, m.tgt, m.nin, targets);
    UPDC_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------- self-test
namespace {
__global__ void k_geo_selftest(float *out) {
    const Pt unit[4] = {{1000.0, 2000.0}, {1000.0, 2001.0}, {1001.0, 2001.0}, {1001.0, 2000.0}};
    const Pt half[4] = {{-0.5, -0.5}, {-0.5, 0.5}, {0.0, 0.5}, {0.0, -0.5}};
    out[0] = geo_area(unit, 4);
    out[1] = geo_overlap(half, 0, 0);
}
}  // namespace

int geometry_self_test(char *msg, size_t cap) {
    const Pt unit[4] = {{1000.0, 2000.0}, {1000.0, 2001.0}, {1001.0, 2001.0}, {1001.0, 2000.0}};
    const Pt half[4] = {{-0.5, -0.5}, {-0.5, 0.5}, {0.0, 0.5}, {0.0, -0.5}};
    float host[2] = {geo_area(unit, 4), geo_overlap(half, 0, 0)};
    float dev[2] = {host[0], host[1]};
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0) {
        float *d = nullptr;
        if (cudaMalloc(&d, 8) == cudaSuccess) {
            k_geo_selftest<<<1, 1>>>(d);
            cudaMemcpy(dev, d, 8, cudaMemcpyDeviceToHost);
            cudaFree(d);
        }
    }
    for (int i = 0; i < 2; ++i) {
        const float want = i == 0 ? 1.0f : 0.5f;
        const float got[2] = {host[i], dev[i]};
        for (float g : got)
            if (fabsf(g - want) > 2.0e-6f) {
                snprintf(msg, cap, "self-test %s failed: %.9g", i == 0 ? "polygon area" : "overlap", (double)g);
                return 1;
            }
    }
    if (sizeof(LinkMapHeader) != 64) {
        snprintf(msg, cap, "self-test LinkMap ABI failed: header=%zu", sizeof(LinkMapHeader));
        return 1;
    }
    return 0;
}

float geometry_polygon_area_host(const double *xy, int count) {
    Pt p[64];
    if (count > 64 || count < 0) return -1.0f;
    for (int i = 0; i < count; ++i) p[i] = Pt{xy[2 * i], xy[2 * i + 1]};
    return geo_area(p, count);
}
float geometry_overlap_area_host(const double *quad8, int x, int y) {
    Pt q[4];
    for (int i = 0; i < 4; ++i) q[i] = Pt{quad8[2 * i], quad8[2 * i + 1]};
    return geo_overlap(q, x, y);
}

}  // namespace updc
