/* TEST INFRASTRUCTURE ONLY — the parity oracle.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg load this library; the product never does.
 *
 * A plain-C restatement of the reference core's numerical path
 * (updc/c_core/updc_core.c and overlap.c), exported for ctypes:
 *   - polygon geometry (overlap.c:14-116) and the LinkMap v2 builder
 *     (updc_core.c:503-609), which must write byte-identical files;
 *   - LinkMap v2 header validation and decode (updc_core.c:463-496, 645-662);
 *   - the solver stages in FP32 (the reference's operation order) and FP64,
 *     instantiated from oracle_solver.h.
 * Parity is pinned by tests that compare this library with the reference
 * core compiled from its own sources (oracle/_ref/updc_jwst_c).
 */
#define _POSIX_C_SOURCE 200809L
#include <errno.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

static int orc_cmp_float(const void *a, const void *b) {
    float x = *(const float *)a, y = *(const float *)b;
    return (x > y) - (x < y);
}

#define FE_REAL float
#define FE_NS(name) orcf_##name
#include "fft_engine.h"
#define OR_REAL float
#define OR_NS(name) orcf_##name
#define OR_FMA fmaf
#include "oracle_solver.h"
#undef FE_REAL
#undef FE_NS
#undef OR_REAL
#undef OR_NS
#undef OR_FMA

#define FE_REAL double
#define FE_NS(name) orcd_##name
#include "fft_engine.h"
#define OR_REAL double
#define OR_NS(name) orcd_##name
#define OR_FMA fma
#include "oracle_solver.h"
#undef FE_REAL
#undef FE_NS
#undef OR_REAL
#undef OR_NS
#undef OR_FMA

/* ------------------------------------------------------------------ geometry
 * Restates overlap.c:14-116: Sutherland-Hodgman clipping of a quadrilateral
 * against the unit target pixel [x-.5,x+.5] x [y-.5,y+.5] in the order left,
 * right, bottom, top, with f64 coordinates, and a shoelace area taken in f32
 * about the polygon's first vertex with fmaf. */
typedef struct { double x, y; } OPoint;

static int o_inside(OPoint p, int side, double v) {
    switch (side) {
        case 0: return p.x >= v;
        case 1: return p.x <= v;
        case 2: return p.y >= v;
        default: return p.y <= v;
    }
}
static OPoint o_cross(OPoint a, OPoint b, int side, double v) {
    OPoint r = a;
    if (side < 2) {
        const double d = b.x - a.x;
        if (fabs(d) > 1.0e-15) { const double t = (v - a.x) / d; r.x = v; r.y = a.y + t * (b.y - a.y); }
    } else {
        const double d = b.y - a.y;
        if (fabs(d) > 1.0e-15) { const double t = (v - a.y) / d; r.x = a.x + t * (b.x - a.x); r.y = v; }
    }
    return r;
}
static int o_clip(const OPoint *in, int n, OPoint *out, int side, double v) {
    int m = 0;
    OPoint prev = in[n - 1];
    int pin = o_inside(prev, side, v);
    for (int i = 0; i < n; ++i) {
        const OPoint cur = in[i];
        const int cin = o_inside(cur, side, v);
        if (cin) {
            if (!pin) out[m++] = o_cross(prev, cur, side, v);
            out[m++] = cur;
        } else if (pin) out[m++] = o_cross(prev, cur, side, v);
        prev = cur; pin = cin;
    }
    return m;
}
static float o_area(const OPoint *p, int n) {
    if (n < 3) return 0.0f;
    const double ox = p[0].x, oy = p[0].y;
    float twice = 0.0f;
    for (int i = 0; i < n; ++i) {
        const int j = (i + 1) % n;
        const float xi = (float)(p[i].x - ox), yi = (float)(p[i].y - oy);
        const float xj = (float)(p[j].x - ox), yj = (float)(p[j].y - oy);
        twice += fmaf(xi, yj, -(xj * yi));
    }
    return 0.5f * fabsf(twice);
}
static float o_overlap(const OPoint q[4], int x, int y) {
    OPoint a[16], b[16], *in = a, *out = b;
    int n = 4;
    const double v[4] = {(double)x - 0.5, (double)x + 0.5, (double)y - 0.5, (double)y + 0.5};
    for (int j = 0; j < 4; ++j) in[j] = q[j];
    for (int side = 0; side < 4; ++side) {
        n = o_clip(in, n, out, side, v[side]);
        if (n < 3) return 0.0f;
        OPoint *t = in; in = out; out = t;
    }
    return o_area(in, n);
}

float orc_polygon_area(const double *xy, int count) {
    OPoint p[64];
    if (count > 64) return -1.0f;
    for (int i = 0; i < count; ++i) { p[i].x = xy[2 * i]; p[i].y = xy[2 * i + 1]; }
    return o_area(p, count);
}
float orc_overlap_area(const double *quad8, int x, int y) {
    OPoint q[4];
    for (int i = 0; i < 4; ++i) { q[i].x = quad8[2 * i]; q[i].y = quad8[2 * i + 1]; }
    return o_overlap(q, x, y);
}

/* core:512-528 mapped detector pixel quad, its area and target bounding box */
static int o_pixel_quad(const double *v, int iw, int W, int H, int x, int y, OPoint q[4], float *full,
                        int *x0, int *x1, int *y0, int *y1) {
    const size_t a = 2 * ((size_t)y * (iw + 1) + x), b = a + 2 * (size_t)(iw + 1);
    q[0].x = v[a]; q[0].y = v[a + 1];
    q[1].x = v[b]; q[1].y = v[b + 1];
    q[2].x = v[b + 2]; q[2].y = v[b + 3];
    q[3].x = v[a + 2]; q[3].y = v[a + 3];
    *full = o_area(q, 4);
    if (!isfinite(*full) || *full <= 1.0e-12f) return 0;
    double mnx = q[0].x, mxx = mnx, mny = q[0].y, mxy = mny;
    for (int j = 1; j < 4; ++j) {
        if (q[j].x < mnx) mnx = q[j].x;
        if (q[j].x > mxx) mxx = q[j].x;
        if (q[j].y < mny) mny = q[j].y;
        if (q[j].y > mxy) mxy = q[j].y;
    }
    if (!isfinite(mnx) || !isfinite(mxx) || !isfinite(mny) || !isfinite(mxy) ||
        mxx < -.5 || mxy < -.5 || mnx > W - .5 || mny > H - .5) return 0;
    *x0 = (int)floor(mnx + .5); *x1 = (int)floor(mxx + .5);
    *y0 = (int)floor(mny + .5); *y1 = (int)floor(mxy + .5);
    if (*x0 < 0) *x0 = 0;
    if (*y0 < 0) *y0 = 0;
    if (*x1 >= W) *x1 = W - 1;
    if (*y1 >= H) *y1 = H - 1;
    return *x0 <= *x1 && *y0 <= *y1;
}

/* ------------------------------------------------------------------ LinkMap v2 */
typedef struct {
    uint32_t magic, version, encoding, header_bytes;
    uint64_t nin, nlinks;
    uint32_t target_width, target_height;
    uint32_t reserved[6];
} OHeader;

static size_t o_linkmap_bytes(const OHeader *h, size_t nin) {
    if (h->header_bytes != sizeof(OHeader)) return 0;
    if (h->nin != nin || h->nlinks > UINT32_MAX) return 0;
    size_t pos = sizeof(OHeader) + (nin + 1) * 4;
    if (h->encoding == 2) {
        pos += nin * 4;
        pos += (size_t)h->nlinks * 2;
        pos = (pos + 3) & ~(size_t)3;
        pos += (size_t)h->nlinks * 4;
    } else if (h->encoding == 1) {
        pos += (size_t)h->nlinks * 8;
    } else return 0;
    return pos;
}

/* Builds the LinkMap of one exposure from its vertex file and writes it to
 * out_path (core:530-609).  Returns 0, or -1 on error. */
int orc_linkmap_build(const char *vertices_path, int iw, int ih, int W, int H, const char *out_path,
                      uint64_t *nlinks_out, int *encoding_out) {
    const size_t nin = (size_t)iw * ih, nv = 2 * (size_t)(iw + 1) * (ih + 1);
    double *v = (double *)malloc(nv * sizeof(double));
    FILE *vf = fopen(vertices_path, "rb");
    if (!v || !vf || fread(v, sizeof(double), nv, vf) != nv) { if (vf) fclose(vf); free(v); return -1; }
    fclose(vf);
    uint32_t *offset = (uint32_t *)malloc((nin + 1) * 4);
    uint32_t *base = (uint32_t *)calloc(nin, 4);
    uint64_t count = 0;
    int all16 = 1;
    OPoint q[4];
    for (int y = 0; y < ih; ++y)
        for (int x = 0; x < iw; ++x) {
            const size_t p = (size_t)y * iw + x;
            offset[p] = (uint32_t)count;
            float full; int x0, x1, y0, y1;
            if (!o_pixel_quad(v, iw, W, H, x, y, q, &full, &x0, &x1, &y0, &y1)) continue;
            const uint64_t before = count;
            uint32_t first = 0, last = 0;
            for (int ty = y0; ty <= y1; ++ty)
                for (int tx = x0; tx <= x1; ++tx) {
                    if (o_overlap(q, tx, ty) <= 1.0e-5f) continue;
                    const uint32_t t = (uint32_t)((size_t)ty * W + tx);
                    if (count == before) first = t;
                    last = t;
                    ++count;
                }
            if (count > before) {
                base[p] = first;
                if (last - first > 0xFFFFu) all16 = 0;
            }
        }
    offset[nin] = (uint32_t)count;
    OHeader h;
    memset(&h, 0, sizeof(h));
    h.magic = 0x324d4c55u; h.version = 2; h.encoding = all16 ? 2 : 1; h.header_bytes = sizeof(h);
    h.nin = nin; h.nlinks = count; h.target_width = (uint32_t)W; h.target_height = (uint32_t)H;
    const size_t bytes = o_linkmap_bytes(&h, nin);
    char *buf = (char *)calloc(1, bytes);
    memcpy(buf, &h, sizeof(h));
    size_t pos = sizeof(h);
    memcpy(buf + pos, offset, (nin + 1) * 4); pos += (nin + 1) * 4;
    uint16_t *delta = NULL; uint32_t *tgt = NULL;
    if (all16) {
        memcpy(buf + pos, base, nin * 4); pos += nin * 4;
        delta = (uint16_t *)(buf + pos); pos += (size_t)count * 2; pos = (pos + 3) & ~(size_t)3;
    } else {
        tgt = (uint32_t *)(buf + pos); pos += (size_t)count * 4;
    }
    float *frac = (float *)(buf + pos);
    for (int y = 0; y < ih; ++y)
        for (int x = 0; x < iw; ++x) {
            const size_t p = (size_t)y * iw + x;
            float full; int x0, x1, y0, y1;
            uint32_t z = offset[p];
            if (!o_pixel_quad(v, iw, W, H, x, y, q, &full, &x0, &x1, &y0, &y1)) continue;
            for (int ty = y0; ty <= y1; ++ty)
                for (int tx = x0; tx <= x1; ++tx) {
                    const float area = o_overlap(q, tx, ty);
                    if (area <= 1.0e-5f) continue;
                    const uint32_t t = (uint32_t)((size_t)ty * W + tx);
                    if (all16) delta[z] = (uint16_t)(t - base[p]); else tgt[z] = t;
                    frac[z] = area / full;
                    ++z;
                }
        }
    FILE *f = fopen(out_path, "wb");
    int rc = (f && fwrite(buf, 1, bytes, f) == bytes) ? 0 : -1;
    if (f && fclose(f)) rc = -1;
    if (nlinks_out) *nlinks_out = count;
    if (encoding_out) *encoding_out = (int)h.encoding;
    free(buf); free(offset); free(base); free(v);
    return rc;
}

/* Validates a LinkMap file like read_linkmap_header (core:485-496).
 * Returns 0 and the link count / encoding, or -1 when invalid. */
int orc_linkmap_info(const char *path, int iw, int ih, int W, int H, uint64_t *nlinks, int *encoding) {
    struct stat st;
    OHeader h;
    if (stat(path, &st) || st.st_size < (off_t)sizeof(h)) return -1;
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    const int ok = fread(&h, sizeof(h), 1, f) == 1;
    fclose(f);
    if (!ok || h.magic != 0x324d4c55u || h.version != 2 || h.target_width != (uint32_t)W ||
        h.target_height != (uint32_t)H) return -1;
    const size_t expect = o_linkmap_bytes(&h, (size_t)iw * ih);
    if (!expect || (size_t)st.st_size != expect) return -1;
    if (nlinks) *nlinks = h.nlinks;
    if (encoding) *encoding = (int)h.encoding;
    return 0;
}

/* Decodes a LinkMap into CSR offsets, absolute targets and fractions
 * (core:645-662 layout, link_target_at core:76-78). */
int orc_linkmap_decode(const char *path, int iw, int ih, int W, int H, uint32_t *offset, uint32_t *target, float *frac) {
    uint64_t nl; int enc;
    if (orc_linkmap_info(path, iw, ih, W, H, &nl, &enc)) return -1;
    const size_t nin = (size_t)iw * ih;
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    OHeader h;
    if (fread(&h, sizeof(h), 1, f) != 1 || fread(offset, 4, nin + 1, f) != nin + 1) { fclose(f); return -1; }
    if (offset[nin] != (uint32_t)nl) { fclose(f); return -1; }
    int rc = 0;
    if (enc == 2) {
        uint32_t *base = (uint32_t *)malloc(nin * 4);
        uint16_t *delta = (uint16_t *)malloc(nl * 2 + 2);
        if (fread(base, 4, nin, f) != nin || fread(delta, 2, nl, f) != nl) rc = -1;
        if (!rc && (nl * 2) % 4) { char pad[2]; if (fread(pad, 1, 2, f) != 2) rc = -1; }
        if (!rc && fread(frac, 4, nl, f) != nl) rc = -1;
        for (size_t p = 0; !rc && p < nin; ++p)
            for (uint32_t z = offset[p]; z < offset[p + 1]; ++z) target[z] = base[p] + (uint32_t)delta[z];
        free(base); free(delta);
    } else {
        if (fread(target, 4, nl, f) != nl || fread(frac, 4, nl, f) != nl) rc = -1;
    }
    fclose(f);
    return rc;
}

/* core:117-126 */
int orc_next_fast_size(int n) {
    for (;; ++n) {
        int q = n;
        while (q % 2 == 0) q /= 2;
        while (q % 3 == 0) q /= 3;
        while (q % 5 == 0) q /= 5;
        while (q % 7 == 0) q /= 7;
        if (q == 1) return n;
    }
}

/* ------------------------------------------------------------------ solver API */
typedef struct {
    char science[1024], weight[1024], psf[1024], vertices[1024];
    int pw, ph;
    double background, pedestal;
    float backgroundf, pedestalf;
} ORow;

static int o_parse_manifest(const char *path, int nexp, ORow *rows, char *err, int errcap) {
    FILE *f = fopen(path, "r");
    if (!f) { snprintf(err, errcap, "cannot open manifest"); return -1; }
    for (int k = 0; k < nexp; ++k) {
        char line[8192];
        char *save = NULL, *fld[8];
        if (!fgets(line, sizeof(line), f)) { fclose(f); snprintf(err, errcap, "manifest has fewer rows than expected"); return -1; }
        for (int j = 0; j < 8; ++j) fld[j] = strtok_r(j ? NULL : line, "\t\r\n", &save);
        for (int j = 0; j < 8; ++j) if (!fld[j]) { fclose(f); snprintf(err, errcap, "manifest requires 8 fields"); return -1; }
        snprintf(rows[k].science, 1024, "%s", fld[0]);
        snprintf(rows[k].weight, 1024, "%s", fld[1]);
        snprintf(rows[k].psf, 1024, "%s", fld[2]);
        rows[k].pw = (int)strtol(fld[3], NULL, 10);
        rows[k].ph = (int)strtol(fld[4], NULL, 10);
        snprintf(rows[k].vertices, 1024, "%s", fld[5]);
        rows[k].background = strtod(fld[6], NULL);
        rows[k].pedestal = strtod(fld[7], NULL);
        rows[k].backgroundf = strtof(fld[6], NULL);
        rows[k].pedestalf = strtof(fld[7], NULL);
    }
    fclose(f);
    return 0;
}

static int o_read_f32(const char *path, float *out, size_t count) {
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    int ok = fread(out, 4, count, f) == count && fgetc(f) == EOF;
    fclose(f);
    return ok ? 0 : -1;
}

typedef struct {
    int precision; /* 32 or 64 */
    void *s;       /* orcf_solver or orcd_solver */
    uint32_t **offset, **target;
    float **frac;
    int nexp;
} OHandle;

#define O_SETUP_BODY(NS, REAL, PARSE_BG, PARSE_PED)                                                  \
    NS##solver *s = (NS##solver *)calloc(1, sizeof(NS##solver));                                     \
    hd->s = s;                                                                                       \
    s->W = W; s->H = H; s->iw = iw; s->ih = ih; s->nexp = nexp; s->FW = FW; s->FH = FH;              \
    s->transposed = transposed;                                                                      \
    s->nout = (size_t)W * H; s->nin = (size_t)iw * ih; s->nf = (size_t)FW * FH;                      \
    s->nc = (size_t)FH * (FW / 2 + 1);                                                               \
    s->background = (REAL *)calloc(nexp, sizeof(REAL));                                              \
    s->pedestal = (REAL *)calloc(nexp, sizeof(REAL));                                                \
    s->mean_offset = (REAL *)calloc(nexp, sizeof(REAL));                                             \
    s->psf_w = (int *)calloc(nexp, sizeof(int)); s->psf_h = (int *)calloc(nexp, sizeof(int));        \
    s->spectrum = (REAL **)calloc(nexp, sizeof(REAL *));                                             \
    s->offset = (const uint32_t **)hd->offset; s->target = (const uint32_t **)hd->target;            \
    s->frac = (const float **)hd->frac;                                                              \
    s->sci = (REAL *)malloc(nexp * s->nin * sizeof(REAL));                                           \
    s->wht = (REAL *)malloc(nexp * s->nin * sizeof(REAL));                                           \
    s->frozen = (uint8_t *)calloc(nexp * s->nin, 1);                                                 \
    s->estimate = (REAL *)calloc(s->nout, sizeof(REAL)); s->coverage = (REAL *)calloc(s->nout, sizeof(REAL)); \
    s->denominator = (REAL *)calloc(s->nout, sizeof(REAL)); s->correction = (REAL *)calloc(s->nout, sizeof(REAL)); \
    s->blur = (REAL *)calloc(s->nout, sizeof(REAL)); s->scatter = (REAL *)calloc(s->nout, sizeof(REAL)); \
    s->fft_image = (REAL *)calloc(s->nf, sizeof(REAL));                                              \
    s->fft_freq = (REAL *)calloc(2 * s->nc, sizeof(REAL));                                           \
    s->estimate_freq = (REAL *)calloc(2 * s->nc, sizeof(REAL));                                      \
    s->partial = (REAL *)calloc(2 * s->nc, sizeof(REAL));                                            \
    s->new_frozen = (uint64_t *)calloc(nexp, 8); s->total_frozen = (uint64_t *)calloc(nexp, 8);      \
    s->min_raw_mu = (REAL *)calloc(nexp, sizeof(REAL));                                              \
    s->plan = NS##plan2d_create(FH, FW, nthreads);                                                   \
    float *tmp = (float *)malloc(s->nin * sizeof(float));                                            \
    for (int k = 0; k < nexp; ++k) {                                                                 \
        s->background[k] = (REAL)rows[k].PARSE_BG; s->pedestal[k] = (REAL)rows[k].PARSE_PED;         \
        s->mean_offset[k] = s->background[k] + s->pedestal[k];                                       \
        s->psf_w[k] = rows[k].pw; s->psf_h[k] = rows[k].ph;                                          \
        s->spectrum[k] = (REAL *)malloc(2 * s->nc * sizeof(REAL));                                   \
        float *psf = (float *)malloc((size_t)rows[k].pw * rows[k].ph * sizeof(float));               \
        if (o_read_f32(rows[k].psf, psf, (size_t)rows[k].pw * rows[k].ph)) { free(psf); snprintf(err, errcap, "PSF raw read failed"); return -1; } \
        if (NS##prepare_psf(s, k, psf)) { free(psf); snprintf(err, errcap, "%s", s->error); return -1; } \
        free(psf);                                                                                   \
        if (o_read_f32(rows[k].science, tmp, s->nin)) { snprintf(err, errcap, "SCI raw read failed"); return -1; } \
        for (size_t p = 0; p < s->nin; ++p) s->sci[k * s->nin + p] = (REAL)tmp[p];                   \
        if (o_read_f32(rows[k].weight, tmp, s->nin)) { snprintf(err, errcap, "WHT raw read failed"); return -1; } \
        for (size_t p = 0; p < s->nin; ++p) s->wht[k * s->nin + p] = (REAL)tmp[p];                   \
    }                                                                                                \
    free(tmp);                                                                                       \
    if (NS##weight_scale(s) || NS##drizzle(s) || NS##denominator_stage(s)) {                         \
        snprintf(err, errcap, "%s", s->error); return -1; }                                          \
    return 0;

static int o_setup32(OHandle *hd, ORow *rows, int W, int H, int iw, int ih, int nexp, int transposed, int FW, int FH,
                     int nthreads, char *err, int errcap) {
    O_SETUP_BODY(orcf_, float, backgroundf, pedestalf)
}
static int o_setup64(OHandle *hd, ORow *rows, int W, int H, int iw, int ih, int nexp, int transposed, int FW, int FH,
                     int nthreads, char *err, int errcap) {
    O_SETUP_BODY(orcd_, double, background, pedestal)
}

/* Creates a solver: parses the manifest, builds (or, with reuse_links, reuses
 * valid) LinkMaps, prepares PSF spectra, weight normalisation, the initial
 * drizzle estimate and the sensitivity denominator (core:1322-1392). */
void *orc_create(int precision, const char *manifest, int W, int H, int iw, int ih, int nexp, int transposed,
                 int FW, int FH, int nthreads, int reuse_links, char *err, int errcap) {
    OHandle *hd = (OHandle *)calloc(1, sizeof(OHandle));
    hd->precision = precision;
    hd->nexp = nexp;
    ORow *rows = (ORow *)calloc(nexp, sizeof(ORow));
    if (o_parse_manifest(manifest, nexp, rows, err, errcap)) { free(rows); free(hd); return NULL; }
    hd->offset = (uint32_t **)calloc(nexp, sizeof(uint32_t *));
    hd->target = (uint32_t **)calloc(nexp, sizeof(uint32_t *));
    hd->frac = (float **)calloc(nexp, sizeof(float *));
    for (int k = 0; k < nexp; ++k) {
        char links[1100];
        snprintf(links, sizeof(links), "%s.links", rows[k].vertices);
        uint64_t nl; int enc;
        if (!reuse_links || orc_linkmap_info(links, iw, ih, W, H, &nl, &enc))
            if (orc_linkmap_build(rows[k].vertices, iw, ih, W, H, links, &nl, &enc)) {
                snprintf(err, errcap, "LinkMap build failed"); free(rows); return NULL;
            }
        hd->offset[k] = (uint32_t *)malloc(((size_t)iw * ih + 1) * 4);
        hd->target[k] = (uint32_t *)malloc(nl * 4 + 4);
        hd->frac[k] = (float *)malloc(nl * 4 + 4);
        if (orc_linkmap_decode(links, iw, ih, W, H, hd->offset[k], hd->target[k], hd->frac[k])) {
            snprintf(err, errcap, "invalid or obsolete LinkMap cache"); free(rows); return NULL;
        }
    }
    int rc = precision == 64 ? o_setup64(hd, rows, W, H, iw, ih, nexp, transposed, FW, FH, nthreads, err, errcap)
                             : o_setup32(hd, rows, W, H, iw, ih, nexp, transposed, FW, FH, nthreads, err, errcap);
    free(rows);
    return rc ? NULL : hd;
}

/* Runs n iterations; stats receives per exposure (new, total) of the last
 * iteration and min_raw_mu as double. Returns 0, or -1 with the message in err. */
int orc_iterate(void *h, int n, uint64_t *new_frozen, uint64_t *total_frozen, double *min_raw_mu,
                char *err, int errcap) {
    OHandle *hd = (OHandle *)h;
    for (int i = 0; i < n; ++i) {
        if (hd->precision == 64) {
            orcd_solver *s = (orcd_solver *)hd->s;
            if (orcd_iterate(s)) { snprintf(err, errcap, "%s", s->error); return -1; }
            for (int k = 0; k < hd->nexp; ++k) {
                if (new_frozen) new_frozen[(size_t)i * hd->nexp + k] = s->new_frozen[k];
                if (total_frozen) total_frozen[(size_t)i * hd->nexp + k] = s->total_frozen[k];
                if (min_raw_mu) min_raw_mu[(size_t)i * hd->nexp + k] = s->min_raw_mu[k];
            }
        } else {
            orcf_solver *s = (orcf_solver *)hd->s;
            if (orcf_iterate(s)) { snprintf(err, errcap, "%s", s->error); return -1; }
            for (int k = 0; k < hd->nexp; ++k) {
                if (new_frozen) new_frozen[(size_t)i * hd->nexp + k] = s->new_frozen[k];
                if (total_frozen) total_frozen[(size_t)i * hd->nexp + k] = s->total_frozen[k];
                if (min_raw_mu) min_raw_mu[(size_t)i * hd->nexp + k] = s->min_raw_mu[k];
            }
        }
    }
    return 0;
}

/* Plane access: 0 estimate, 1 coverage, 2 denominator, 3 correction, 4 blur,
 * 5 scatter, 6 sci (nexp*nin), 7 wht (nexp*nin).  Returns a pointer to REAL
 * data of the solver's precision. */
void *orc_plane(void *h, int which) {
    OHandle *hd = (OHandle *)h;
#define O_PLANE(S) switch (which) { case 0: return S->estimate; case 1: return S->coverage; \
        case 2: return S->denominator; case 3: return S->correction; case 4: return S->blur; \
        case 5: return S->scatter; case 6: return S->sci; case 7: return S->wht; default: return NULL; }
    if (hd->precision == 64) { orcd_solver *s = (orcd_solver *)hd->s; O_PLANE(s) }
    else { orcf_solver *s = (orcf_solver *)hd->s; O_PLANE(s) }
#undef O_PLANE
}
uint8_t *orc_frozen(void *h) {
    OHandle *hd = (OHandle *)h;
    return hd->precision == 64 ? ((orcd_solver *)hd->s)->frozen : ((orcf_solver *)hd->s)->frozen;
}
double orc_scalar(void *h, int which) {
    OHandle *hd = (OHandle *)h;
    if (hd->precision == 64) {
        orcd_solver *s = (orcd_solver *)hd->s;
        return which == 0 ? s->weight_scale : which == 1 ? s->max_sensitivity : which == 2 ? s->last_sum : (double)s->last_negative;
    }
    orcf_solver *s = (orcf_solver *)hd->s;
    return which == 0 ? s->weight_scale : which == 1 ? s->max_sensitivity : which == 2 ? s->last_sum : (double)s->last_negative;
}
/* Spectrum of exposure k (FFTW layout, FH x (FW/2+1) interleaved complex). */
void *orc_spectrum(void *h, int k) {
    OHandle *hd = (OHandle *)h;
    return hd->precision == 64 ? (void *)((orcd_solver *)hd->s)->spectrum[k] : (void *)((orcf_solver *)hd->s)->spectrum[k];
}

/* Forward model of exposure k from the current estimate into the blur plane
 * (core:745-747 + 773-776). */
void orc_forward_blur(void *h, int k) {
    OHandle *hd = (OHandle *)h;
    if (hd->precision == 64) {
        orcd_solver *s = (orcd_solver *)hd->s;
        orcd_forward_target(s, s->estimate, s->estimate_freq);
        for (size_t p = 0; p < s->nc; ++p) {
            const double a = s->estimate_freq[2 * p], b = s->estimate_freq[2 * p + 1];
            const double c = s->spectrum[k][2 * p], d = s->spectrum[k][2 * p + 1];
            s->fft_freq[2 * p] = a * c - b * d; s->fft_freq[2 * p + 1] = a * d + b * c;
        }
        orcd_inverse_crop(s, s->blur);
    } else {
        orcf_solver *s = (orcf_solver *)hd->s;
        orcf_forward_target(s, s->estimate, s->estimate_freq);
        for (size_t p = 0; p < s->nc; ++p) {
            const float a = s->estimate_freq[2 * p], b = s->estimate_freq[2 * p + 1];
            const float c = s->spectrum[k][2 * p], d = s->spectrum[k][2 * p + 1];
            s->fft_freq[2 * p] = a * c - b * d; s->fft_freq[2 * p + 1] = a * d + b * c;
        }
        orcf_inverse_crop(s, s->blur);
    }
}

/* Detector loop of exposure k on a caller-supplied blur plane, writing the
 * scatter plane and updating the solver's freeze mask (core:1152-1177). */
int orc_detector(void *h, int k, const void *blur, void *scatter, uint64_t *nnew, uint64_t *ntotal, double *minmu,
                 char *err, int errcap) {
    OHandle *hd = (OHandle *)h;
    if (hd->precision == 64) {
        double m;
        int rc = orcd_detector((orcd_solver *)hd->s, k, (const double *)blur, (double *)scatter, nnew, ntotal, &m, err, errcap);
        *minmu = m;
        return rc;
    }
    float m;
    int rc = orcf_detector((orcf_solver *)hd->s, k, (const float *)blur, (float *)scatter, nnew, ntotal, &m, err, errcap);
    *minmu = m;
    return rc;
}

/* H^T of detector planes v (nexp x nin, the solver's precision) into out
 * (nout), with the reference's scatter and frequency-domain adjoint. */
void orc_adjoint(void *h, const void *v, void *out) {
    OHandle *hd = (OHandle *)h;
    if (hd->precision == 64) orcd_adjoint((orcd_solver *)hd->s, (const double *)v, (double *)out);
    else orcf_adjoint((orcf_solver *)hd->s, (const float *)v, (float *)out);
}

/* Update stage on the solver's correction plane (core:1437-1456). */
int orc_update(void *h, char *err, int errcap) {
    OHandle *hd = (OHandle *)h;
    int rc;
    if (hd->precision == 64) { orcd_solver *s = (orcd_solver *)hd->s; rc = orcd_update(s); if (rc) snprintf(err, errcap, "%s", s->error); }
    else { orcf_solver *s = (orcf_solver *)hd->s; rc = orcf_update(s); if (rc) snprintf(err, errcap, "%s", s->error); }
    return rc;
}

/* Plain 2-D transforms in the oracle's precision, FFTW layout. */
void orc_fft_r2c(int precision, int n0, int n1, int nthreads, const void *in, void *out) {
    if (precision == 64) { orcd_plan2d *p = orcd_plan2d_create(n0, n1, nthreads); orcd_exec_r2c(p, (const double *)in, (double *)out); orcd_plan2d_free(p); }
    else { orcf_plan2d *p = orcf_plan2d_create(n0, n1, nthreads); orcf_exec_r2c(p, (const float *)in, (float *)out); orcf_plan2d_free(p); }
}
void orc_fft_c2r(int precision, int n0, int n1, int nthreads, void *in, void *out) {
    if (precision == 64) { orcd_plan2d *p = orcd_plan2d_create(n0, n1, nthreads); orcd_exec_c2r(p, (double *)in, (double *)out); orcd_plan2d_free(p); }
    else { orcf_plan2d *p = orcf_plan2d_create(n0, n1, nthreads); orcf_exec_c2r(p, (float *)in, (float *)out); orcf_plan2d_free(p); }
}

void orc_destroy(void *h) {
    /* Test processes are short-lived; the solver's buffers are released at exit. */
    (void)h;
}
