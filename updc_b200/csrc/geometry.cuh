// Exact detector-pixel / target-pixel overlap geometry.
//
// Restates updc/c_core/overlap.c:14-116 and updc_core.c:512-528: a detector
// pixel is the quadrilateral of its four mapped corners (f64); it is clipped
// against the unit target pixel [x-.5,x+.5] x [y-.5,y+.5] with
// Sutherland-Hodgman in the order left, right, bottom, top; the area is a
// shoelace sum taken in f32 about the polygon's first vertex with fmaf.  The
// translation unit that includes this header is compiled with -fmad=false so
// that no multiply-add is contracted, which keeps every f64 intermediate and
// therefore every LinkMap byte identical to the reference's.
#pragma once

#include <math.h>

namespace updc {

struct Pt { double x, y; };

__host__ __device__ inline int geo_inside(Pt p, int side, double v) {
    switch (side) {
        case 0: return p.x >= v;
        case 1: return p.x <= v;
        case 2: return p.y >= v;
        default: return p.y <= v;
    }
}

__host__ __device__ inline Pt geo_cross(Pt a, Pt b, int side, double v) {
    Pt r = a;
    if (side < 2) {
        const double d = b.x - a.x;
        if (fabs(d) > 1.0e-15) {
            const double t = (v - a.x) / d;
            r.x = v;
            r.y = a.y + t * (b.y - a.y);
        }
    } else {
        const double d = b.y - a.y;
        if (fabs(d) > 1.0e-15) {
            const double t = (v - a.y) / d;
            r.x = a.x + t * (b.x - a.x);
            r.y = v;
        }
    }
    return r;
}

__host__ __device__ inline int geo_clip(const Pt *in, int n, Pt *out, int side, double v) {
    int m = 0;
    Pt prev = in[n - 1];
    int pin = geo_inside(prev, side, v);
    for (int i = 0; i < n; ++i) {
        const Pt cur = in[i];
        const int cin = geo_inside(cur, side, v);
        if (cin) {
            if (!pin) out[m++] = geo_cross(prev, cur, side, v);
            out[m++] = cur;
        } else if (pin) {
            out[m++] = geo_cross(prev, cur, side, v);
        }
        prev = cur;
        pin = cin;
    }
    return m;
}

__host__ __device__ inline float geo_area(const Pt *p, int n) {
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

__host__ __device__ inline float geo_overlap(const Pt q[4], int x, int y) {
    Pt a[16], b[16];
    Pt *in = a, *out = b;
    int n = 4;
    const double v[4] = {(double)x - 0.5, (double)x + 0.5, (double)y - 0.5, (double)y + 0.5};
    for (int j = 0; j < 4; ++j) in[j] = q[j];
    for (int side = 0; side < 4; ++side) {
        n = geo_clip(in, n, out, side, v[side]);
        if (n < 3) return 0.0f;
        Pt *t = in;
        in = out;
        out = t;
    }
    return geo_area(in, n);
}

// Mapped quad of detector pixel (x, y), its area and the clamped target
// bounding box; returns 0 when the pixel maps to nothing (updc_core.c:512-528).
__host__ __device__ inline int geo_pixel_quad(const double *v, int iw, int W, int H, int x, int y, Pt q[4], float *full,
                                              int *x0, int *x1, int *y0, int *y1) {
    const size_t a = 2 * ((size_t)y * (iw + 1) + x), b = a + 2 * (size_t)(iw + 1);
    q[0] = Pt{v[a], v[a + 1]};
    q[1] = Pt{v[b], v[b + 1]};
    q[2] = Pt{v[b + 2], v[b + 3]};
    q[3] = Pt{v[a + 2], v[a + 3]};
    *full = geo_area(q, 4);
    if (!isfinite(*full) || *full <= 1.0e-12f) return 0;
    double mnx = q[0].x, mxx = mnx, mny = q[0].y, mxy = mny;
    for (int j = 1; j < 4; ++j) {
        if (q[j].x < mnx) mnx = q[j].x;
        if (q[j].x > mxx) mxx = q[j].x;
        if (q[j].y < mny) mny = q[j].y;
        if (q[j].y > mxy) mxy = q[j].y;
    }
    if (!isfinite(mnx) || !isfinite(mxx) || !isfinite(mny) || !isfinite(mxy) || mxx < -.5 || mxy < -.5 ||
        mnx > W - .5 || mny > H - .5)
        return 0;
    *x0 = (int)floor(mnx + .5);
    *x1 = (int)floor(mxx + .5);
    *y0 = (int)floor(mny + .5);
    *y1 = (int)floor(mxy + .5);
    if (*x0 < 0) *x0 = 0;
    if (*y0 < 0) *y0 = 0;
    if (*x1 >= W) *x1 = W - 1;
    if (*y1 >= H) *y1 = H - 1;
    return *x0 <= *x1 && *y0 <= *y1;
}

}  // namespace updc
