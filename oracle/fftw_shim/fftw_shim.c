/*
 * fftw_shim.c -- project-written implementation of the FFTW-API subset declared
 * in fftw3.h (TEST INFRASTRUCTURE: used only to build the reference solver as a
 * CPU oracle and as the timed CPU baseline; never linked into the product).
 *
 * Algorithm: iterative mixed-radix Stockham autosort FFT (Cooley-Tukey
 * decomposition, radices 4, 2, 3, 5 and a direct DFT for any remaining prime),
 * written from the textbook method.  Twiddles are evaluated in long double and
 * rounded once to double.  Multi-dimensional transforms apply the 1D transform
 * along every axis; strided axes are gathered in blocks of pencils into a
 * contiguous buffer for cache locality.  OpenMP parallelises over pencils.
 *
 * Semantics follow FFTW's documented definitions, as used by the reference
 * (src/fft/fft.h:91-140): unnormalised; FFTW_FORWARD uses exp(-2 pi i jk/n);
 * r2c/c2r halve the LAST (fastest) dimension to n/2+1; c2r treats its input as
 * Hermitian (imaginary parts of the self-conjugate modes are ignored) and here
 * leaves the input array unchanged.
 */
#define _POSIX_C_SOURCE 200112L
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    double re, im;
} cplx;

enum { K_C2C = 0, K_R2C = 1, K_C2R = 2 };

typedef struct {
    int n;          /* length */
    int nrad;       /* number of stages */
    int rad[64];    /* radices in order */
    cplx *tw;       /* tw[t] = exp(-2 pi i t / n), t in [0, n) */
} plan1d;

struct qx_shim_plan_s {
    int kind;
    int rank;
    int dims[3];
    int sign;
    plan1d p[3];  /* 1D plans per axis (last axis: n/2+1 not needed; full n) */
    void *in, *out;
};

static int g_nthreads = 1;

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
    return p;
}
void fftw_free(void *p) { free(p); }
fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)fftw_malloc(n * sizeof(fftw_complex)); }
double *fftw_alloc_real(size_t n) { return (double *)fftw_malloc(n * sizeof(double)); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads > 0 ? nthreads : 1; }
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}

static void plan1d_init(plan1d *p, int n) {
    p->n = n;
    p->nrad = 0;
    int m = n;
    while (m % 4 == 0) { p->rad[p->nrad++] = 4; m /= 4; }
    while (m % 2 == 0) { p->rad[p->nrad++] = 2; m /= 2; }
    while (m % 3 == 0) { p->rad[p->nrad++] = 3; m /= 3; }
    while (m % 5 == 0) { p->rad[p->nrad++] = 5; m /= 5; }
    for (int f = 7; m > 1; f += 2) {
        while (m % f == 0) { p->rad[p->nrad++] = f; m /= f; }
    }
    p->tw = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int t = 0; t < n; ++t) {
        long double a = -twopi * (long double)t / (long double)n;
        p->tw[t].re = (double)cosl(a);
        p->tw[t].im = (double)sinl(a);
    }
}

static inline cplx cmul(cplx a, cplx b) {
    cplx c = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return c;
}

/* twiddle exp(sign * 2 pi i * t / n) for t taken mod n */
static inline cplx twid(const plan1d *p, long t, int sign) {
    cplx w = p->tw[t % p->n];
    if (sign > 0) w.im = -w.im;
    return w;
}

/* One 1D transform of length p->n on contiguous data a (result back in a).
 * b is scratch of the same length. */
static void fft1d(const plan1d *p, cplx *a, cplx *b, int sign) {
    const int n = p->n;
    if (n == 1) return;
    cplx *src = a, *dst = b;
    long Ns = 1;
    cplx v[64], V[64];
    for (int s = 0; s < p->nrad; ++s) {
        const int r = p->rad[s];
        const int nr = n / r;
        const long stride_tw = n / (Ns * r);  /* exp(i 2pi km/(Ns r)) = W_n^{k m n/(Ns r)} */
        for (int j = 0; j < nr; ++j) {
            const long k = j % Ns;
            for (int m = 0; m < r; ++m) {
                cplx x = src[j + m * nr];
                v[m] = (k == 0 || m == 0) ? x : cmul(x, twid(p, k * m * stride_tw, sign));
            }
            if (r == 2) {
                V[0].re = v[0].re + v[1].re; V[0].im = v[0].im + v[1].im;
                V[1].re = v[0].re - v[1].re; V[1].im = v[0].im - v[1].im;
            } else if (r == 4) {
                cplx t0 = {v[0].re + v[2].re, v[0].im + v[2].im};
                cplx t1 = {v[0].re - v[2].re, v[0].im - v[2].im};
                cplx t2 = {v[1].re + v[3].re, v[1].im + v[3].im};
                cplx t3 = {v[1].re - v[3].re, v[1].im - v[3].im};
                /* multiply t3 by sign*i : forward (sign=-1) -> -i */
                cplx t3r = sign < 0 ? (cplx){t3.im, -t3.re} : (cplx){-t3.im, t3.re};
                V[0].re = t0.re + t2.re; V[0].im = t0.im + t2.im;
                V[2].re = t0.re - t2.re; V[2].im = t0.im - t2.im;
                V[1].re = t1.re + t3r.re; V[1].im = t1.im + t3r.im;
                V[3].re = t1.re - t3r.re; V[3].im = t1.im - t3r.im;
            } else {
                /* direct r-point DFT with exact-rounded roots of unity */
                const long step = n / r;
                for (int q = 0; q < r; ++q) {
                    double sr = 0.0, si = 0.0;
                    for (int m = 0; m < r; ++m) {
                        cplx w = twid(p, (long)((q * m) % r) * step, sign);
                        sr += v[m].re * w.re - v[m].im * w.im;
                        si += v[m].re * w.im + v[m].im * w.re;
                    }
                    V[q].re = sr; V[q].im = si;
                }
            }
            const long idxD = (j / Ns) * Ns * r + k;
            for (int m = 0; m < r; ++m) dst[idxD + m * Ns] = V[m];
        }
        cplx *t = src; src = dst; dst = t;
        Ns *= r;
    }
    if (src != a) memcpy(a, src, sizeof(cplx) * (size_t)n);
}

#define QX_BLK 16

/* Transform axis `ax` of a complex array with logical dims d[0..rank-1]
 * (last fastest). */
static void c2c_axis(const plan1d *p, cplx *data, int rank, const int *d, int ax, int sign) {
    const int n = d[ax];
    long inner = 1, outer = 1;
    for (int i = ax + 1; i < rank; ++i) inner *= d[i];
    for (int i = 0; i < ax; ++i) outer *= d[i];
    if (n == 1) return;
    if (inner == 1) {
        #pragma omp parallel num_threads(g_nthreads)
        {
            cplx *scr = (cplx *)malloc(sizeof(cplx) * (size_t)n);
            #pragma omp for schedule(static)
            for (long o = 0; o < outer; ++o) fft1d(p, data + o * n, scr, sign);
            free(scr);
        }
        return;
    }
    const long nblk = (inner + QX_BLK - 1) / QX_BLK;
    #pragma omp parallel num_threads(g_nthreads)
    {
        cplx *buf = (cplx *)malloc(sizeof(cplx) * (size_t)n * QX_BLK);
        cplx *scr = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        #pragma omp for schedule(static) collapse(2)
        for (long o = 0; o < outer; ++o) {
            for (long bk = 0; bk < nblk; ++bk) {
                const long c0 = bk * QX_BLK;
                const int w = (int)((inner - c0) < QX_BLK ? (inner - c0) : QX_BLK);
                cplx *base = data + o * n * inner + c0;
                for (int i = 0; i < n; ++i)
                    for (int c = 0; c < w; ++c) buf[(long)c * n + i] = base[(long)i * inner + c];
                for (int c = 0; c < w; ++c) fft1d(p, buf + (long)c * n, scr, sign);
                for (int i = 0; i < n; ++i)
                    for (int c = 0; c < w; ++c) base[(long)i * inner + c] = buf[(long)c * n + i];
            }
        }
        free(scr);
        free(buf);
    }
}

static fftw_plan mkplan(int kind, int rank, const int *dims, int sign, void *in, void *out) {
    fftw_plan pl = (fftw_plan)calloc(1, sizeof(*pl));
    if (!pl) return NULL;
    pl->kind = kind;
    pl->rank = rank;
    pl->sign = sign;
    pl->in = in;
    pl->out = out;
    for (int i = 0; i < rank; ++i) {
        if (dims[i] < 1) { free(pl); return NULL; }
        pl->dims[i] = dims[i];
        plan1d_init(&pl->p[i], dims[i]);
    }
    return pl;
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags; int d[2] = {n0, n1}; return mkplan(K_C2C, 2, d, sign, in, out);
}
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags; int d[3] = {n0, n1, n2}; return mkplan(K_C2C, 3, d, sign, in, out);
}
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags) {
    (void)flags; int d[2] = {n0, n1}; return mkplan(K_R2C, 2, d, FFTW_FORWARD, in, out);
}
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags) {
    (void)flags; int d[3] = {n0, n1, n2}; return mkplan(K_R2C, 3, d, FFTW_FORWARD, in, out);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags) {
    (void)flags; int d[2] = {n0, n1}; return mkplan(K_C2R, 2, d, FFTW_BACKWARD, in, out);
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags) {
    (void)flags; int d[3] = {n0, n1, n2}; return mkplan(K_C2R, 3, d, FFTW_BACKWARD, in, out);
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    for (int i = 0; i < p->rank; ++i) free(p->p[i].tw);
    free(p);
}

static void exec_c2c(const fftw_plan p, fftw_complex *in, fftw_complex *out) {
    long total = 1;
    for (int i = 0; i < p->rank; ++i) total *= p->dims[i];
    if (out != in) memcpy(out, in, sizeof(fftw_complex) * (size_t)total);
    for (int ax = p->rank - 1; ax >= 0; --ax)
        c2c_axis(&p->p[ax], (cplx *)out, p->rank, p->dims, ax, p->sign);
}

static void exec_r2c(const fftw_plan p, double *in, fftw_complex *out) {
    const int rank = p->rank;
    const int n = p->dims[rank - 1];
    const int nh = n / 2 + 1;
    long rows = 1;
    for (int i = 0; i < rank - 1; ++i) rows *= p->dims[i];
    cplx *o = (cplx *)out;
    #pragma omp parallel num_threads(g_nthreads)
    {
        cplx *row = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        cplx *scr = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        #pragma omp for schedule(static)
        for (long r = 0; r < rows; ++r) {
            for (int i = 0; i < n; ++i) { row[i].re = in[r * n + i]; row[i].im = 0.0; }
            fft1d(&p->p[rank - 1], row, scr, FFTW_FORWARD);
            for (int i = 0; i < nh; ++i) o[r * nh + i] = row[i];
        }
        free(scr);
        free(row);
    }
    int hd[3];
    for (int i = 0; i < rank; ++i) hd[i] = p->dims[i];
    hd[rank - 1] = nh;
    for (int ax = rank - 2; ax >= 0; --ax) c2c_axis(&p->p[ax], o, rank, hd, ax, FFTW_FORWARD);
}

static void exec_c2r(const fftw_plan p, fftw_complex *in, double *out) {
    const int rank = p->rank;
    const int n = p->dims[rank - 1];
    const int nh = n / 2 + 1;
    long rows = 1;
    for (int i = 0; i < rank - 1; ++i) rows *= p->dims[i];
    cplx *tmp = (cplx *)fftw_malloc(sizeof(cplx) * (size_t)(rows * nh));
    memcpy(tmp, in, sizeof(cplx) * (size_t)(rows * nh));
    int hd[3];
    for (int i = 0; i < rank; ++i) hd[i] = p->dims[i];
    hd[rank - 1] = nh;
    for (int ax = rank - 2; ax >= 0; --ax) c2c_axis(&p->p[ax], tmp, rank, hd, ax, FFTW_BACKWARD);
    #pragma omp parallel num_threads(g_nthreads)
    {
        cplx *row = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        cplx *scr = (cplx *)malloc(sizeof(cplx) * (size_t)n);
        #pragma omp for schedule(static)
        for (long r = 0; r < rows; ++r) {
            const cplx *h = tmp + r * nh;
            for (int i = 0; i < nh; ++i) row[i] = h[i];
            for (int i = nh; i < n; ++i) { row[i].re = h[n - i].re; row[i].im = -h[n - i].im; }
            fft1d(&p->p[rank - 1], row, scr, FFTW_BACKWARD);
            for (int i = 0; i < n; ++i) out[r * n + i] = row[i].re;
        }
        free(scr);
        free(row);
    }
    fftw_free(tmp);
}

void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) { exec_c2c(p, in, out); }
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) { exec_r2c(p, in, out); }
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) { exec_c2r(p, in, out); }
void fftw_execute(const fftw_plan p) {
    if (p->kind == K_C2C) exec_c2c(p, (fftw_complex *)p->in, (fftw_complex *)p->out);
    else if (p->kind == K_R2C) exec_r2c(p, (double *)p->in, (fftw_complex *)p->out);
    else exec_c2r(p, (fftw_complex *)p->in, (double *)p->out);
}
