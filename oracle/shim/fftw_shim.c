/*
 * FFTW 3 API subset -- TEST INFRASTRUCTURE ONLY (oracle build).
 * See fftw3.h for scope.  Transforms are computed by a recursive mixed-radix
 * decimation-in-time DFT (any length; radices are the prime factors of n)
 * with twiddles exp(-2 pi i j / n) taken from a per-length cos/sin table.
 *
 * shim_set_exact_dft(1) switches every later fftw_execute to a direct DFT
 * summed in long double (x87 80-bit, 64-bit mantissa) and rounded to double
 * once: a second, differently rounded and more accurate DFT, used to measure
 * how much the reference's results depend on which correct FFT it links
 * (FFTW's own output bits are unpinned).
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cplx;

enum kind { K_R2C, K_C2R, K_C2C };

struct shim_fftw_plan {
    enum kind kind;
    int n, sign;
    int nloop;                 /* number of howmany loops (1 or 2) */
    int hn[2], his[2], hos[2]; /* loop counts and strides (elements) */
    int is, os;                /* element strides inside one transform */
    void *in, *out;
    cplx *tw;                  /* tw[j] = exp(-2 pi i j / n), j < n */
};

void *fftw_malloc(size_t n) { return aligned_alloc(64, (n + 63) / 64 * 64); }
void fftw_free(void *p) { free(p); }

static cplx *make_twiddles(int n)
{
    cplx *tw = (cplx *) malloc(sizeof(cplx) * (size_t) (n > 0 ? n : 1));
    for (int j = 0; j < n; j++) {
        double a = 2.0 * M_PI * (double) j / (double) n;
        tw[j].re = cos(a);
        tw[j].im = -sin(a);
    }
    return tw;
}

static int smallest_factor(int n)
{
    if (n % 4 == 0) return 4;
    for (int p = 2; p * p <= n; p++)
        if (n % p == 0) return p;
    return n;
}

/* out[k] = sum_t x[t*stride] exp(sign 2 pi i t k / n), for a sub-transform of
 * length n of a top-level transform of length N (twiddle table tw of length N). */
static void dft_rec(const cplx *x, size_t stride, int n, int N, int sign,
                    const cplx *tw, cplx *out)
{
    if (n == 1) {
        out[0] = x[0];
        return;
    }
    int p = smallest_factor(n);
    int m = n / p;
    cplx *sub = (cplx *) malloc(sizeof(cplx) * (size_t) n);
    for (int r = 0; r < p; r++) dft_rec(x + (size_t) r * stride, stride * (size_t) p, m, N, sign, tw, sub + (size_t) r * m);
    int step = N / n;
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < p; q++) {
            int kk = k + q * m;
            double sr = 0.0, si = 0.0;
            for (int r = 0; r < p; r++) {
                long j = ((long) r * kk) % n;
                cplx w = tw[j * step];
                if (sign > 0) w.im = -w.im;
                cplx y = sub[(size_t) r * m + k];
                sr += w.re * y.re - w.im * y.im;
                si += w.re * y.im + w.im * y.re;
            }
            out[kk].re = sr;
            out[kk].im = si;
        }
    }
    free(sub);
}

static int exact_dft = 0;
void shim_set_exact_dft(int on) { exact_dft = on; }

/* out[k] = sum_t x[t] exp(sign 2 pi i t k / n), summed in long double. */
static void dft_exact(const cplx *x, int n, int sign, cplx *out)
{
    long double *c = (long double *) malloc(sizeof(long double) * 2 * (size_t) n);
    long double *s = c + n;
    for (int j = 0; j < n; j++) {
        long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double) j / (long double) n;
        c[j] = cosl(a);
        s[j] = (long double) sign * sinl(a);
    }
    for (int k = 0; k < n; k++) {
        long double sr = 0.0L, si = 0.0L;
        for (int t = 0; t < n; t++) {
            const int j = (int) (((long) t * k) % n);
            sr += c[j] * (long double) x[t].re - s[j] * (long double) x[t].im;
            si += c[j] * (long double) x[t].im + s[j] * (long double) x[t].re;
        }
        out[k].re = (double) sr;
        out[k].im = (double) si;
    }
    free(c);
}

static void dft(const cplx *x, int n, int sign, const cplx *tw, cplx *out)
{
    if (exact_dft) dft_exact(x, n, sign, out);
    else dft_rec(x, 1, n, n, sign, tw, out);
}

void shim_fft_c2c(int n, int sign, const fftw_complex *in, fftw_complex *out)
{
    cplx *tw = make_twiddles(n);
    cplx *x = (cplx *) malloc(sizeof(cplx) * (size_t) n);
    cplx *y = (cplx *) malloc(sizeof(cplx) * (size_t) n);
    memcpy(x, in, sizeof(cplx) * (size_t) n);
    dft_rec(x, 1, n, n, sign, tw, y);
    memcpy(out, y, sizeof(cplx) * (size_t) n);
    free(x); free(y); free(tw);
}

static fftw_plan new_plan(enum kind kind, int n, int sign)
{
    fftw_plan p = (fftw_plan) calloc(1, sizeof(*p));
    p->kind = kind;
    p->n = n;
    p->sign = sign;
    p->tw = make_twiddles(n);
    return p;
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags)
{
    (void) inembed; (void) onembed; (void) flags;
    if (rank != 1) return NULL;
    fftw_plan p = new_plan(K_R2C, n[0], FFTW_FORWARD);
    p->nloop = 1;
    p->hn[0] = howmany; p->his[0] = idist; p->hos[0] = odist;
    p->is = istride; p->os = ostride;
    p->in = in; p->out = out;
    return p;
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist,
                                 unsigned flags)
{
    (void) inembed; (void) onembed; (void) flags;
    if (rank != 1) return NULL;
    fftw_plan p = new_plan(K_C2R, n[0], FFTW_BACKWARD);
    p->nloop = 1;
    p->hn[0] = howmany; p->his[0] = idist; p->hos[0] = odist;
    p->is = istride; p->os = ostride;
    p->in = in; p->out = out;
    return p;
}

fftw_plan fftw_plan_guru_dft(int rank, const fftw_iodim *dims,
                             int howmany_rank, const fftw_iodim *howmany_dims,
                             fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{
    (void) flags;
    if (rank != 1 || howmany_rank < 0 || howmany_rank > 2) return NULL;
    fftw_plan p = new_plan(K_C2C, dims[0].n, sign);
    p->nloop = 2;
    p->hn[0] = p->hn[1] = 1;
    p->his[0] = p->his[1] = p->hos[0] = p->hos[1] = 0;
    for (int d = 0; d < howmany_rank; d++) {
        p->hn[d] = howmany_dims[d].n;
        p->his[d] = howmany_dims[d].is;
        p->hos[d] = howmany_dims[d].os;
    }
    p->is = dims[0].is; p->os = dims[0].os;
    p->in = in; p->out = out;
    return p;
}

static void run_one(const struct shim_fftw_plan *p, size_t ioff, size_t ooff, cplx *x, cplx *y)
{
    int n = p->n;
    if (p->kind == K_R2C) {
        const double *in = (const double *) p->in + ioff;
        for (int j = 0; j < n; j++) { x[j].re = in[(size_t) j * p->is]; x[j].im = 0.0; }
        dft(x, n, -1, p->tw, y);
        cplx *out = (cplx *) p->out + ooff;
        for (int k = 0; k <= n / 2; k++) out[(size_t) k * p->os] = y[k];
    } else if (p->kind == K_C2R) {
        const cplx *in = (const cplx *) p->in + ioff;
        for (int k = 0; k <= n / 2; k++) x[k] = in[(size_t) k * p->is];
        x[0].im = 0.0;
        if (n % 2 == 0) x[n / 2].im = 0.0;
        for (int k = n / 2 + 1; k < n; k++) { x[k].re = x[n - k].re; x[k].im = -x[n - k].im; }
        dft(x, n, +1, p->tw, y);
        double *out = (double *) p->out + ooff;
        for (int j = 0; j < n; j++) out[(size_t) j * p->os] = y[j].re;
    } else {
        const cplx *in = (const cplx *) p->in + ioff;
        for (int j = 0; j < n; j++) x[j] = in[(size_t) j * p->is];
        dft(x, n, p->sign, p->tw, y);
        cplx *out = (cplx *) p->out + ooff;
        for (int k = 0; k < n; k++) out[(size_t) k * p->os] = y[k];
    }
}

void fftw_execute(const fftw_plan p)
{
    cplx *x = (cplx *) malloc(sizeof(cplx) * (size_t) p->n);
    cplx *y = (cplx *) malloc(sizeof(cplx) * (size_t) p->n);
    int n1 = p->nloop == 2 ? p->hn[1] : 1;
    for (int a = 0; a < p->hn[0]; a++)
        for (int b = 0; b < n1; b++) {
            size_t ioff = (size_t) a * (size_t) p->his[0] + (p->nloop == 2 ? (size_t) b * (size_t) p->his[1] : 0);
            size_t ooff = (size_t) a * (size_t) p->hos[0] + (p->nloop == 2 ? (size_t) b * (size_t) p->hos[1] : 0);
            run_one(p, ioff, ooff, x, y);
        }
    free(x);
    free(y);
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    free(p->tw);
    free(p);
}
