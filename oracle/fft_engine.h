/* TEST INFRASTRUCTURE ONLY — part of the parity oracle, never linked by the product.
 *
 * Portable mixed-radix Stockham FFT used by the FFTW-API shim (fftw_shim.c) and
 * by the C restatement of the solver (updc_oracle.c).  This file is a macro
 * template: define FE_REAL (float or double) and FE_NS(name) (a name prefix)
 * before including it.  It restates the discrete Fourier transform with FFTW's
 * conventions (unnormalised, forward sign -1, real-to-complex output of n/2+1
 * bins per row, complex-to-real ignoring the imaginary parts of the DC and
 * Nyquist bins), which is all the reference core relies on
 * (updc/c_core/updc_core.c:733-772).
 *
 * Stage formula (self-sorting Stockham, any radix R, Ns = product of earlier
 * radices):  for j in [0, n/R):  k = j mod Ns;
 *   v[r] = in[j + r n/R] * w^(r k/(Ns R));  V = DFT_R(v);
 *   out[(j/Ns) Ns R + k + s Ns] = V[s].
 * Odd radices use the symmetric-pair form of the length-R DFT.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#ifndef FE_REAL
#error "define FE_REAL before including fft_engine.h"
#endif

#define FE_MAX_STAGES 48
#define FE_MAX_ODD 64

typedef struct {
    int n;
    int nstage;
    int radix[FE_MAX_STAGES];
    int ns[FE_MAX_STAGES];
    FE_REAL *tw[FE_MAX_STAGES];  /* stage twiddles: Ns*(R-1) complex, forward sign */
    FE_REAL *odd_cos[FE_MAX_STAGES];
    FE_REAL *odd_sin[FE_MAX_STAGES];
} FE_NS(plan1d);

static void FE_NS(plan1d_free)(FE_NS(plan1d) *p) {
    if (!p) return;
    for (int s = 0; s < p->nstage; ++s) {
        free(p->tw[s]);
        free(p->odd_cos[s]);
        free(p->odd_sin[s]);
    }
    free(p);
}

static FE_NS(plan1d) *FE_NS(plan1d_create)(int n) {
    FE_NS(plan1d) *p = (FE_NS(plan1d) *)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->n = n;
    int m = n, ns = 1;
    int radices[FE_MAX_STAGES], nr = 0;
    while (m % 8 == 0) { radices[nr++] = 8; m /= 8; }
    while (m % 4 == 0) { radices[nr++] = 4; m /= 4; }
    while (m % 2 == 0) { radices[nr++] = 2; m /= 2; }
    for (int q = 3; m > 1; q += 2) {
        while (m % q == 0) {
            if (nr >= FE_MAX_STAGES || q > FE_MAX_ODD) { FE_NS(plan1d_free)(p); return NULL; }
            radices[nr++] = q; m /= q;
        }
    }
    const double two_pi = 6.283185307179586476925286766559;
    for (int s = 0; s < nr; ++s) {
        const int R = radices[s];
        p->radix[s] = R;
        p->ns[s] = ns;
        p->tw[s] = (FE_REAL *)malloc(sizeof(FE_REAL) * 2 * (size_t)ns * (size_t)(R > 1 ? R - 1 : 1));
        if (!p->tw[s]) { p->nstage = s; FE_NS(plan1d_free)(p); return NULL; }
        for (int k = 0; k < ns; ++k)
            for (int r = 1; r < R; ++r) {
                const double a = -two_pi * (double)r * (double)k / ((double)ns * (double)R);
                FE_REAL *t = p->tw[s] + 2 * ((size_t)k * (R - 1) + (r - 1));
                t[0] = (FE_REAL)cos(a);
                t[1] = (FE_REAL)sin(a);
            }
        if (R % 2 == 1) {
            const int h = (R - 1) / 2;
            p->odd_cos[s] = (FE_REAL *)malloc(sizeof(FE_REAL) * (size_t)(h * h + 1));
            p->odd_sin[s] = (FE_REAL *)malloc(sizeof(FE_REAL) * (size_t)(h * h + 1));
            for (int a = 1; a <= h; ++a)
                for (int q = 1; q <= h; ++q) {
                    const double ang = two_pi * (double)((long)a * q % R) / (double)R;
                    p->odd_cos[s][(a - 1) * h + (q - 1)] = (FE_REAL)cos(ang);
                    p->odd_sin[s][(a - 1) * h + (q - 1)] = (FE_REAL)sin(ang);
                }
        }
        ns *= R;
    }
    p->nstage = nr;
    return p;
}

/* One length-R DFT on v (interleaved complex), in place, with sign -1 (forward)
 * or +1 (inverse). */
static void FE_NS(small_dft)(const FE_NS(plan1d) *p, int s, FE_REAL *v, int sign) {
    const int R = p->radix[s];
    if (R == 2) {
        FE_REAL ar = v[0], ai = v[1], br = v[2], bi = v[3];
        v[0] = ar + br; v[1] = ai + bi; v[2] = ar - br; v[3] = ai - bi;
        return;
    }
    if (R == 4 || R == 8) {
        /* radix-4 kernel on (v0, v[st], v[2st], v[3st]) */
        FE_REAL out[16];
        if (R == 4) {
            FE_REAL t0r = v[0] + v[4], t0i = v[1] + v[5];
            FE_REAL t1r = v[0] - v[4], t1i = v[1] - v[5];
            FE_REAL t2r = v[2] + v[6], t2i = v[3] + v[7];
            FE_REAL dr = v[2] - v[6], di = v[3] - v[7];
            /* t3 = sign * i * (v1 - v3) */
            FE_REAL t3r = sign < 0 ? di : -di, t3i = sign < 0 ? -dr : dr;
            v[0] = t0r + t2r; v[1] = t0i + t2i;
            v[4] = t0r - t2r; v[5] = t0i - t2i;
            v[2] = t1r + t3r; v[3] = t1i + t3i;
            v[6] = t1r - t3r; v[7] = t1i - t3i;
            return;
        }
        /* R == 8: two radix-4 DFTs on even and odd samples, then combine */
        FE_REAL e[8], o[8];
        for (int q = 0; q < 4; ++q) {
            e[2 * q] = v[4 * q]; e[2 * q + 1] = v[4 * q + 1];
            o[2 * q] = v[4 * q + 2]; o[2 * q + 1] = v[4 * q + 3];
        }
        FE_REAL *arr[2] = {e, o};
        for (int h = 0; h < 2; ++h) {
            FE_REAL *x = arr[h];
            FE_REAL t0r = x[0] + x[4], t0i = x[1] + x[5];
            FE_REAL t1r = x[0] - x[4], t1i = x[1] - x[5];
            FE_REAL t2r = x[2] + x[6], t2i = x[3] + x[7];
            FE_REAL dr = x[2] - x[6], di = x[3] - x[7];
            FE_REAL t3r = sign < 0 ? di : -di, t3i = sign < 0 ? -dr : dr;
            x[0] = t0r + t2r; x[1] = t0i + t2i;
            x[4] = t0r - t2r; x[5] = t0i - t2i;
            x[2] = t1r + t3r; x[3] = t1i + t3i;
            x[6] = t1r - t3r; x[7] = t1i - t3i;
        }
        const FE_REAL c = (FE_REAL)0.70710678118654752440084436210485;
        for (int q = 0; q < 4; ++q) {
            FE_REAL orr = o[2 * q], oi = o[2 * q + 1], wr, wi;
            /* w8^q with the transform sign */
            switch (q) {
                case 0: wr = 1; wi = 0; break;
                case 1: wr = c; wi = sign < 0 ? -c : c; break;
                case 2: wr = 0; wi = sign < 0 ? -1 : 1; break;
                default: wr = -c; wi = sign < 0 ? -c : c; break;
            }
            FE_REAL pr = orr * wr - oi * wi, pi = orr * wi + oi * wr;
            out[2 * q] = e[2 * q] + pr; out[2 * q + 1] = e[2 * q + 1] + pi;
            out[2 * (q + 4)] = e[2 * q] - pr; out[2 * (q + 4) + 1] = e[2 * q + 1] - pi;
        }
        memcpy(v, out, sizeof(out));
        return;
    }
    /* odd radix, symmetric-pair form */
    const int h = (R - 1) / 2;
    FE_REAL ar[FE_MAX_ODD], ai[FE_MAX_ODD], br[FE_MAX_ODD], bi[FE_MAX_ODD];
    FE_REAL s0r = v[0], s0i = v[1];
    for (int q = 1; q <= h; ++q) {
        ar[q] = v[2 * q] + v[2 * (R - q)];
        ai[q] = v[2 * q + 1] + v[2 * (R - q) + 1];
        br[q] = v[2 * q] - v[2 * (R - q)];
        bi[q] = v[2 * q + 1] - v[2 * (R - q) + 1];
        s0r += ar[q]; s0i += ai[q];
    }
    FE_REAL outv[2 * FE_MAX_ODD];
    outv[0] = s0r; outv[1] = s0i;
    for (int a = 1; a <= h; ++a) {
        FE_REAL Ar = v[0], Ai = v[1], Br = 0, Bi = 0;
        for (int q = 1; q <= h; ++q) {
            const FE_REAL cs = p->odd_cos[s][(a - 1) * h + (q - 1)];
            const FE_REAL sn = p->odd_sin[s][(a - 1) * h + (q - 1)];
            Ar += ar[q] * cs; Ai += ai[q] * cs;
            Br += br[q] * sn; Bi += bi[q] * sn;
        }
        /* V[a] = A + sign*i*B ; V[R-a] = A - sign*i*B */
        FE_REAL iBr = -Bi, iBi = Br;
        if (sign < 0) { iBr = -iBr; iBi = -iBi; }
        outv[2 * a] = Ar + iBr; outv[2 * a + 1] = Ai + iBi;
        outv[2 * (R - a)] = Ar - iBr; outv[2 * (R - a) + 1] = Ai - iBi;
    }
    memcpy(v, outv, sizeof(FE_REAL) * 2 * (size_t)R);
}

/* Complex FFT of p->n points. data and work each hold n complex values; the
 * result ends in data. */
static void FE_NS(fft1d)(const FE_NS(plan1d) *p, FE_REAL *data, FE_REAL *work, int sign) {
    const int n = p->n;
    FE_REAL *in = data, *out = work;
    for (int s = 0; s < p->nstage; ++s) {
        const int R = p->radix[s], Ns = p->ns[s], stride = n / R;
        const FE_REAL *tw = p->tw[s];
        FE_REAL v[2 * FE_MAX_ODD];
        memset(v, 0, sizeof(v));
        for (int j = 0; j < stride; ++j) {
            const int k = j % Ns;
            for (int r = 0; r < R; ++r) {
                FE_REAL xr = in[2 * (j + r * stride)], xi = in[2 * (j + r * stride) + 1];
                if (r > 0 && k > 0) {
                    const FE_REAL wr = tw[2 * (k * (R - 1) + r - 1)];
                    const FE_REAL wi = sign < 0 ? tw[2 * (k * (R - 1) + r - 1) + 1] : -tw[2 * (k * (R - 1) + r - 1) + 1];
                    const FE_REAL tr = xr * wr - xi * wi;
                    xi = xr * wi + xi * wr;
                    xr = tr;
                }
                v[2 * r] = xr; v[2 * r + 1] = xi;
            }
            FE_NS(small_dft)(p, s, v, sign);
            const int base = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; ++r) {
                out[2 * (base + r * Ns)] = v[2 * r];
                out[2 * (base + r * Ns) + 1] = v[2 * r + 1];
            }
        }
        FE_REAL *t = in; in = out; out = t;
    }
    if (in != data) memcpy(data, in, sizeof(FE_REAL) * 2 * (size_t)n);
}

/* 2-D real<->complex transform plan with FFTW's layout. */
typedef struct {
    int n0, n1, m;           /* rows, columns, m = n1/2+1 */
    int half;                /* 1 when n1 is even: rows use an n1/2-point complex FFT */
    int nthreads;
    FE_NS(plan1d) *row;      /* n1/2 (half) or n1 points */
    FE_NS(plan1d) *col;      /* n0 points */
    FE_REAL *post;           /* exp(-2 pi i k / n1), k = 0..n1/2 (half only) */
} FE_NS(plan2d);

static void FE_NS(plan2d_free)(FE_NS(plan2d) *p) {
    if (!p) return;
    FE_NS(plan1d_free)(p->row);
    FE_NS(plan1d_free)(p->col);
    free(p->post);
    free(p);
}

static FE_NS(plan2d) *FE_NS(plan2d_create)(int n0, int n1, int nthreads) {
    if (n0 < 1 || n1 < 1) return NULL;
    FE_NS(plan2d) *p = (FE_NS(plan2d) *)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->n0 = n0; p->n1 = n1; p->m = n1 / 2 + 1;
    p->half = (n1 % 2 == 0) && n1 >= 2;
    p->nthreads = nthreads < 1 ? 1 : nthreads;
    p->row = FE_NS(plan1d_create)(p->half ? n1 / 2 : n1);
    p->col = FE_NS(plan1d_create)(n0);
    if (!p->row || !p->col) { FE_NS(plan2d_free)(p); return NULL; }
    if (p->half) {
        p->post = (FE_REAL *)malloc(sizeof(FE_REAL) * 2 * (size_t)(n1 / 2 + 1));
        const double two_pi = 6.283185307179586476925286766559;
        for (int k = 0; k <= n1 / 2; ++k) {
            p->post[2 * k] = (FE_REAL)cos(-two_pi * k / n1);
            p->post[2 * k + 1] = (FE_REAL)sin(-two_pi * k / n1);
        }
    }
    return p;
}

/* real row (n1 values) -> n1/2+1 complex bins */
static void FE_NS(row_r2c)(const FE_NS(plan2d) *p, const FE_REAL *x, FE_REAL *X, FE_REAL *buf, FE_REAL *work) {
    const int n1 = p->n1;
    if (!p->half) {
        for (int i = 0; i < n1; ++i) { buf[2 * i] = x[i]; buf[2 * i + 1] = 0; }
        FE_NS(fft1d)(p->row, buf, work, -1);
        memcpy(X, buf, sizeof(FE_REAL) * 2 * (size_t)p->m);
        return;
    }
    const int M = n1 / 2;
    memcpy(buf, x, sizeof(FE_REAL) * (size_t)n1); /* z[m] = x[2m] + i x[2m+1] */
    FE_NS(fft1d)(p->row, buf, work, -1);
    for (int k = 0; k <= M; ++k) {
        const int a = k % M, b = (M - k) % M;
        const FE_REAL zr = buf[2 * a], zi = buf[2 * a + 1];
        const FE_REAL cr = buf[2 * b], ci = -buf[2 * b + 1];  /* conj(Z[M-k]) */
        const FE_REAL er = (FE_REAL)0.5 * (zr + cr), ei = (FE_REAL)0.5 * (zi + ci);
        const FE_REAL dr = (FE_REAL)0.5 * (zr - cr), di = (FE_REAL)0.5 * (zi - ci);
        /* X = E - i w^k D */
        const FE_REAL wr = p->post[2 * k], wi = p->post[2 * k + 1];
        const FE_REAL pr = dr * wr - di * wi, pi = dr * wi + di * wr;
        X[2 * k] = er + pi;
        X[2 * k + 1] = ei - pr;
    }
}

/* n1/2+1 complex bins -> n1 real values (unnormalised inverse) */
static void FE_NS(row_c2r)(const FE_NS(plan2d) *p, const FE_REAL *X, FE_REAL *x, FE_REAL *buf, FE_REAL *work) {
    const int n1 = p->n1;
    if (!p->half) {
        for (int k = 0; k < p->m; ++k) { buf[2 * k] = X[2 * k]; buf[2 * k + 1] = X[2 * k + 1]; }
        buf[1] = 0;
        for (int k = p->m; k < n1; ++k) { buf[2 * k] = X[2 * (n1 - k)]; buf[2 * k + 1] = -X[2 * (n1 - k) + 1]; }
        FE_NS(fft1d)(p->row, buf, work, +1);
        for (int i = 0; i < n1; ++i) x[i] = buf[2 * i];
        return;
    }
    const int M = n1 / 2;
    for (int k = 0; k < M; ++k) {
        FE_REAL ar = X[2 * k], ai = X[2 * k + 1];
        FE_REAL br = X[2 * (M - k)], bi = -X[2 * (M - k) + 1];  /* conj(X[M-k]) */
        if (k == 0) { ai = 0; bi = 0; }
        const FE_REAL sr = ar + br, si = ai + bi;
        const FE_REAL dr = ar - br, di = ai - bi;
        /* Z' = S + i conj(w^k) D */
        const FE_REAL wr = p->post[2 * k], wi = -p->post[2 * k + 1];
        const FE_REAL qr = dr * wr - di * wi, qi = dr * wi + di * wr;
        buf[2 * k] = sr - qi;
        buf[2 * k + 1] = si + qr;
    }
    FE_NS(fft1d)(p->row, buf, work, +1);
    memcpy(x, buf, sizeof(FE_REAL) * (size_t)n1);
}

typedef struct {
    const FE_NS(plan2d) *p;
    const FE_REAL *rin;
    FE_REAL *cdata;    /* n0 x m complex */
    FE_REAL *rout;
    int tid, nt, phase;
} FE_NS(job);

#define FE_COL_BATCH 8

static void *FE_NS(job_run)(void *opaque) {
    FE_NS(job) *jb = (FE_NS(job) *)opaque;
    const FE_NS(plan2d) *p = jb->p;
    const int n0 = p->n0, n1 = p->n1, m = p->m;
    const size_t rowlen = (size_t)(n1 > n0 ? n1 : n0);
    FE_REAL *buf = (FE_REAL *)malloc(sizeof(FE_REAL) * 2 * rowlen * (FE_COL_BATCH + 1));
    FE_REAL *work = (FE_REAL *)malloc(sizeof(FE_REAL) * 2 * rowlen);
    if (!buf || !work) abort();
    if (jb->phase == 0 || jb->phase == 3) {   /* r2c rows / c2r rows */
        const int y0 = (int)((long)n0 * jb->tid / jb->nt), y1 = (int)((long)n0 * (jb->tid + 1) / jb->nt);
        for (int y = y0; y < y1; ++y) {
            if (jb->phase == 0) FE_NS(row_r2c)(p, jb->rin + (size_t)y * n1, jb->cdata + 2 * (size_t)y * m, buf, work);
            else FE_NS(row_c2r)(p, jb->cdata + 2 * (size_t)y * m, jb->rout + (size_t)y * n1, buf, work);
        }
    } else {                                   /* columns, forward (1) or inverse (2) */
        const int sign = jb->phase == 1 ? -1 : +1;
        const int nbatch = (m + FE_COL_BATCH - 1) / FE_COL_BATCH;
        FE_REAL *colbuf = buf + 2 * rowlen;
        for (int bidx = jb->tid; bidx < nbatch; bidx += jb->nt) {
            const int c0 = bidx * FE_COL_BATCH;
            const int nb = (m - c0) < FE_COL_BATCH ? (m - c0) : FE_COL_BATCH;
            for (int y = 0; y < n0; ++y) {
                const FE_REAL *src = jb->cdata + 2 * ((size_t)y * m + c0);
                for (int c = 0; c < nb; ++c) {
                    colbuf[2 * ((size_t)c * n0 + y)] = src[2 * c];
                    colbuf[2 * ((size_t)c * n0 + y) + 1] = src[2 * c + 1];
                }
            }
            for (int c = 0; c < nb; ++c) FE_NS(fft1d)(p->col, colbuf + 2 * (size_t)c * n0, work, sign);
            for (int y = 0; y < n0; ++y) {
                FE_REAL *dst = jb->cdata + 2 * ((size_t)y * m + c0);
                for (int c = 0; c < nb; ++c) {
                    dst[2 * c] = colbuf[2 * ((size_t)c * n0 + y)];
                    dst[2 * c + 1] = colbuf[2 * ((size_t)c * n0 + y) + 1];
                }
            }
        }
    }
    free(buf); free(work);
    return NULL;
}

static void FE_NS(run_phase)(const FE_NS(plan2d) *p, const FE_REAL *rin, FE_REAL *cdata, FE_REAL *rout, int phase) {
    int nt = p->nthreads;
    if (nt > 256) nt = 256;
    FE_NS(job) jobs[256];
    pthread_t th[256];
    for (int t = 0; t < nt; ++t) {
        jobs[t].p = p; jobs[t].rin = rin; jobs[t].cdata = cdata; jobs[t].rout = rout;
        jobs[t].tid = t; jobs[t].nt = nt; jobs[t].phase = phase;
    }
    if (nt == 1) { FE_NS(job_run)(&jobs[0]); return; }
    for (int t = 0; t < nt; ++t)
        if (pthread_create(&th[t], NULL, FE_NS(job_run), &jobs[t])) abort();
    for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
}

/* out (n0 x m complex) = R2C(in (n0 x n1 real)) */
static void FE_NS(exec_r2c)(const FE_NS(plan2d) *p, const FE_REAL *in, FE_REAL *out) {
    FE_NS(run_phase)(p, in, out, NULL, 0);
    FE_NS(run_phase)(p, NULL, out, NULL, 1);
}

/* out (n0 x n1 real) = unnormalised C2R(in); in is overwritten, as FFTW's
 * complex-to-real transforms are allowed to do. */
static void FE_NS(exec_c2r)(const FE_NS(plan2d) *p, FE_REAL *in, FE_REAL *out) {
    FE_NS(run_phase)(p, NULL, in, NULL, 2);
    FE_NS(run_phase)(p, NULL, in, out, 3);
}
