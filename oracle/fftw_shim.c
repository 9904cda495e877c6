#define _POSIX_C_SOURCE 200809L
/* TEST INFRASTRUCTURE ONLY — part of the parity oracle, never linked by the product.
 *
 * FFTW3f-API shim: lets the unmodified reference core (updc/c_core/updc_core.c)
 * compile and run here, where FFTW3f is absent.  Only the API subset in
 * fftw3.h is provided.  Transforms are computed by fft_engine.h in single
 * precision with double-precision twiddle tables.  Plans are immutable after
 * creation and every execute call allocates its own scratch, so concurrent
 * new-array execution from several threads is safe (the reference relies on
 * this at updc_core.c:853-854 and 1216-1217).
 */
#include "fftw3.h"

#include <stdio.h>

#define FE_REAL float
#define FE_NS(name) shimf_##name
#include "fft_engine.h"

const char fftwf_version[] = "updc-oracle-fftw-shim-1";

struct fftwf_plan_s {
    int kind; /* 0 r2c, 1 c2r */
    shimf_plan2d *p;
    float *rbuf;
    fftwf_complex *cbuf;
};

static int g_nthreads = 1;

float *fftwf_alloc_real(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, (n ? n : 1) * sizeof(float))) return NULL;
    return (float *)p;
}
fftwf_complex *fftwf_alloc_complex(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, (n ? n : 1) * sizeof(fftwf_complex))) return NULL;
    return (fftwf_complex *)p;
}
void fftwf_free(void *p) { free(p); }

int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int nthreads) { g_nthreads = nthreads < 1 ? 1 : nthreads; }
void fftwf_cleanup_threads(void) { g_nthreads = 1; }

int fftwf_import_wisdom_from_filename(const char *filename) { (void)filename; return 0; }
int fftwf_export_wisdom_to_filename(const char *filename) {
    FILE *f = fopen(filename, "w");
    if (!f) return 0;
    fprintf(f, "(%s no-wisdom)\n", fftwf_version);
    return fclose(f) == 0;
}

static fftwf_plan make_plan(int kind, int n0, int n1, float *r, fftwf_complex *c) {
    struct fftwf_plan_s *pl = (struct fftwf_plan_s *)calloc(1, sizeof(*pl));
    if (!pl) return NULL;
    pl->kind = kind;
    pl->p = shimf_plan2d_create(n0, n1, g_nthreads);
    if (!pl->p) { free(pl); return NULL; }
    pl->rbuf = r; pl->cbuf = c;
    return pl;
}

fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *in, fftwf_complex *out, unsigned flags) {
    (void)flags;
    return make_plan(0, n0, n1, in, out);
}
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *in, float *out, unsigned flags) {
    (void)flags;
    return make_plan(1, n0, n1, out, in);
}

void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out) {
    shimf_exec_r2c(p->p, in, (float *)out);
}
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out) {
    shimf_exec_c2r(p->p, (float *)in, out);
}
void fftwf_execute(const fftwf_plan p) {
    if (p->kind == 0) fftwf_execute_dft_r2c(p, p->rbuf, p->cbuf);
    else fftwf_execute_dft_c2r(p, p->cbuf, p->rbuf);
}
void fftwf_destroy_plan(fftwf_plan p) {
    if (!p) return;
    shimf_plan2d_free(p->p);
    free(p);
}
