// LinkMap v2 (updc/c_core/updc_core.c:40-79, 463-496, 530-609, 645-662) on the GPU.
#pragma once

#include <string>
#include <vector>

#include "common.cuh"

namespace updc {

constexpr uint32_t LINKMAP_MAGIC = 0x324d4c55u;  // "ULM2"
constexpr uint32_t LINKMAP_VERSION = 2u;
constexpr uint32_t LINKMAP_ABS32 = 1u;
constexpr uint32_t LINKMAP_DELTA16 = 2u;

struct LinkMapHeader {
    uint32_t magic, version, encoding, header_bytes;
    uint64_t nin, nlinks;
    uint32_t target_width, target_height;
    uint32_t reserved[6];
};
static_assert(sizeof(LinkMapHeader) == 64, "LinkMap v2 header is 64 bytes");

// Byte size of a LinkMap file with this header, or 0 when the header is not
// a valid v2 header for nin detector pixels (updc_core.c:469-483).
size_t linkmap_expected_bytes(const LinkMapHeader &h, size_t nin);

// Device copy of one exposure's LinkMap: the file's sections as they are
// (CSR offsets, DELTA16 base+delta or ABS32 targets, f32 fractions) plus the
// target-major transpose used by every adjoint (S^T) product.
struct DevLinkMap {
    uint32_t encoding = 0;
    uint64_t nlinks = 0;
    size_t nin = 0;
    size_t file_bytes = 0;
    uint32_t *off = nullptr, *base = nullptr, *tgt = nullptr;
    uint16_t *delta = nullptr;
    float *frac = nullptr;
    // transpose: for target t, entries [toff[t], toff[t+1]) hold {source
    // pixel, fraction bits} (one 8-byte entry each) in increasing
    // source-pixel order, the order in which the reference's serial scatter
    // loop visits them.
    uint32_t *toff = nullptr;
    uint2 *tent = nullptr;
    void release();
};

struct LinkBuildStats {
    uint64_t nlinks = 0;
    uint32_t encoding = 0;
    uint64_t active = 0;
    uint32_t max_links = 0;
};

// Reads and validates a LinkMap file as read_linkmap_header + open_links do;
// returns false (leaving `out` empty) when the file is absent or invalid.
bool linkmap_load(const std::string &path, size_t nin, int W, int H, DevLinkMap &out, cudaStream_t s);

// Polygon-overlap LinkMap construction on the GPU, written to `path` through a
// temporary file and rename (updc_core.c:530-609).  Byte-identical to the
// reference's file for the same vertices.
void linkmap_build(const std::string &vertices_path, const std::string &path, int iw, int ih, int W, int H,
                   cudaStream_t s, LinkBuildStats *stats);

// Validates CSR offsets and target indices on the device and builds the
// target-major transpose.  Throws Error on an invalid map.
void linkmap_transpose(DevLinkMap &m, size_t nout, cudaStream_t s);

// Absolute target of every link (link_target_at, updc_core.c:76-78).
void linkmap_decode(const DevLinkMap &m, uint32_t *targets, cudaStream_t s);

// Known-answer geometry checks of the reference self-test (updc_core.c:1545-1564)
// evaluated on the device (and on the host).  Returns 0 on success.
int geometry_self_test(char *msg, size_t cap);

// Geometry entry points for tests: polygon area and unit-pixel overlap.
float geometry_polygon_area_host(const double *xy, int count);
float geometry_overlap_area_host(const double *quad8, int x, int y);

}  // namespace updc
