/*
 * fftw3.h -- project-written FFTW-API subset (TEST INFRASTRUCTURE, oracle only).
 *
 * FFTW3 is not installed on this machine.  The reference solver calls a small
 * part of the FFTW3 double-precision API (src/fft/fft.h:66-140,
 * src/field.cxx:37-39,58-66).  This header declares exactly that part so the
 * reference's own translation units compile unmodified; fftw_shim.c implements
 * it with a project-written mixed-radix Stockham FFT (twiddles in long double).
 * The numerical results are FFTW's mathematical definitions (unnormalised DFTs,
 * FFTW_FORWARD = exp(-i...), r2c/c2r on the last dimension halved), not FFTW's
 * operation order, so round-off differs from a real FFTW build at the 1e-16 level.
 *
 * Only tests/, the oracle build and bench.py's reference arm use this.
 */
#ifndef QX_ORACLE_FFTW3_SHIM_H
#define QX_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct qx_shim_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

/* planner flags: accepted and ignored (there is only one algorithm) */
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_complex *fftw_alloc_complex(size_t n);
double *fftw_alloc_real(size_t n);

int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in,
                           fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in,
                               fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in,
                               double *out, unsigned flags);

void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
