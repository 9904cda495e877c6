/* TEST INFRASTRUCTURE ONLY — part of the parity oracle, never linked by the product.
 *
 * A minimal FFTW3 single-precision API shim.  The reference core
 * (updc/c_core/updc_core.c:18, call sites 159-168, 225-240, 733-743, 761-772,
 * 822, 1324-1328, 1358-1365, 1534-1537) includes <fftw3.h> and links FFTW3f,
 * which is not installed in this environment.  This header declares exactly the
 * subset of FFTW's public API that the core uses, with FFTW's documented
 * semantics (unnormalised transforms, row-major arrays, the last axis stored
 * half-complex as n1/2+1 values, new-array execute functions safe to call
 * concurrently).  The arithmetic behind it is this project's own mixed-radix
 * FFT in fftw_shim.c; nothing of FFTW's source is used.
 */
#ifndef UPDC_ORACLE_FFTW3_SHIM_H
#define UPDC_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

extern const char fftwf_version[];

fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *in, float *out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out);
void fftwf_destroy_plan(fftwf_plan p);

float *fftwf_alloc_real(size_t n);
fftwf_complex *fftwf_alloc_complex(size_t n);
void fftwf_free(void *p);

int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
void fftwf_cleanup_threads(void);

int fftwf_import_wisdom_from_filename(const char *filename);
int fftwf_export_wisdom_to_filename(const char *filename);

#ifdef __cplusplus
}
#endif

#endif
