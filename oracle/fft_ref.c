/*
 * fft_ref.c -- FP64 mixed-radix FFT for the CPU oracle (TEST INFRASTRUCTURE).
 *
 * The reference delegates every FFT to Intel MKL DFTI, a third-party library
 * that is not in the reference tree (Makefile:1-2,19 link MKL; call sites
 * parallel_filter_subsampling.cpp:224-228,308,432,517 and pfft.c:224-228,642).
 * MKL's arithmetic is not pinned by any reference test -- only the SNR of the
 * whole transform against a direct DFT is (test.c:283-293, input.c:292-425) --
 * so this restatement implements the same mathematical transform (forward,
 * unnormalised, exp(-2*pi*i*j*k/n)) and is itself pinned against a long-double
 * naive DFT in tests/.
 *
 * Algorithm: Stockham autosort, mixed radix (8, 4, 2, 3, 5, 7 and a generic
 * O(p^2) butterfly for other primes).  Twiddles are computed in long double and
 * rounded once to double.  Lengths >= 2^15 with a balanced split use a
 * four-step decomposition parallelised with OpenMP.
 */
#include "fft_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cplx;

#define MAX_STAGES 64
#define FOURSTEP_MIN 32768

struct fftr_plan {
    size_t n;
    int nstages;
    int radix[MAX_STAGES];
    cplx *tw;           /* tw[k] = exp(-2 pi i k / n), k < n            */
    /* four-step: n = n1 * n2 */
    int fourstep;
    size_t n1, n2;
    struct fftr_plan *p1, *p2;
};

static inline cplx cmul(cplx a, cplx b)
{
    cplx r = { a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re };
    return r;
}

static const long double PI_L = 3.141592653589793238462643383279502884L;

static cplx *make_twiddles(size_t n)
{
    cplx *tw = (cplx *)malloc(sizeof(cplx) * (n ? n : 1));
    for (size_t k = 0; k < n; ++k) {
        /* reduce to the first octant-free form: angle = 2 pi k / n */
        long double a = 2.0L * PI_L * (long double)k / (long double)n;
        tw[k].re = (double)cosl(a);
        tw[k].im = (double)-sinl(a);
    }
    return tw;
}

static int factorize(size_t n, int *rad)
{
    int t = 0;
    while (n % 8 == 0 && n > 8) { rad[t++] = 8; n /= 8; }
    while (n % 4 == 0) { rad[t++] = 4; n /= 4; }
    while (n % 2 == 0) { rad[t++] = 2; n /= 2; }
    for (size_t p = 3; n > 1; p += 2) {
        while (n % p == 0) { rad[t++] = (int)p; n /= p; }
        if (p * p > n && n > 1) { rad[t++] = (int)n; n = 1; }
    }
    if (t == 0) rad[t++] = 1;
    return t;
}

fftr_plan *fftr_create(size_t n)
{
    fftr_plan *p = (fftr_plan *)calloc(1, sizeof(fftr_plan));
    p->n = n;
    p->tw = make_twiddles(n);
    if (n >= FOURSTEP_MIN) {
        /* balanced split n = n1*n2 with n1 <= n2 */
        size_t best = 0;
        for (size_t a = 2; a * a <= n; ++a)
            if (n % a == 0) best = a;
        if (best >= 32) {
            p->fourstep = 1;
            p->n1 = best;
            p->n2 = n / best;
            p->p1 = fftr_create(p->n1);
            p->p2 = fftr_create(p->n2);
            return p;
        }
    }
    p->nstages = factorize(n, p->radix);
    return p;
}

void fftr_destroy(fftr_plan *p)
{
    if (!p) return;
    if (p->fourstep) { fftr_destroy(p->p1); fftr_destroy(p->p2); }
    free(p->tw);
    free(p);
}

size_t fftr_size(const fftr_plan *p) { return p->n; }

/* small DFT kernels, in place on v[0..R) */
static void dft2(cplx *v)
{
    cplx a = v[0], b = v[1];
    v[0].re = a.re + b.re; v[0].im = a.im + b.im;
    v[1].re = a.re - b.re; v[1].im = a.im - b.im;
}

static void dft4(cplx *v)
{
    cplx a0 = { v[0].re + v[2].re, v[0].im + v[2].im };
    cplx a1 = { v[0].re - v[2].re, v[0].im - v[2].im };
    cplx a2 = { v[1].re + v[3].re, v[1].im + v[3].im };
    cplx a3 = { v[1].re - v[3].re, v[1].im - v[3].im };
    /* -i * a3 */
    cplx m3 = { a3.im, -a3.re };
    v[0].re = a0.re + a2.re; v[0].im = a0.im + a2.im;
    v[2].re = a0.re - a2.re; v[2].im = a0.im - a2.im;
    v[1].re = a1.re + m3.re; v[1].im = a1.im + m3.im;
    v[3].re = a1.re - m3.re; v[3].im = a1.im - m3.im;
}

static void dft8(cplx *v)
{
    const double h = 0.70710678118654752440084436210484903928;
    cplx e[4] = { v[0], v[2], v[4], v[6] };
    cplx o[4] = { v[1], v[3], v[5], v[7] };
    dft4(e);
    dft4(o);
    /* twiddles exp(-2 pi i k / 8), k = 0..3 */
    cplx t1 = { h * (o[1].re + o[1].im), h * (o[1].im - o[1].re) };
    cplx t2 = { o[2].im, -o[2].re };
    cplx t3 = { h * (o[3].im - o[3].re), -h * (o[3].re + o[3].im) };
    cplx t[4] = { o[0], t1, t2, t3 };
    for (int k = 0; k < 4; ++k) {
        v[k].re = e[k].re + t[k].re; v[k].im = e[k].im + t[k].im;
        v[k + 4].re = e[k].re - t[k].re; v[k + 4].im = e[k].im - t[k].im;
    }
}

static void dft_generic(cplx *v, int R, const cplx *tw, size_t twstride)
{
    /* tw[k*twstride] = exp(-2 pi i k / R) */
    cplx out[64];
    cplx *o = out;
    cplx *heap = NULL;
    if (R > 64) { heap = (cplx *)malloc(sizeof(cplx) * R); o = heap; }
    for (int k = 0; k < R; ++k) {
        double sr = 0, si = 0;
        for (int r = 0; r < R; ++r) {
            cplx w = tw[(size_t)((r * (size_t)k) % R) * twstride];
            sr += v[r].re * w.re - v[r].im * w.im;
            si += v[r].re * w.im + v[r].im * w.re;
        }
        o[k].re = sr; o[k].im = si;
    }
    memcpy(v, o, sizeof(cplx) * R);
    free(heap);
}

static void dft_small(cplx *v, int R, const cplx *tw, size_t n)
{
    switch (R) {
    case 1: return;
    case 2: dft2(v); return;
    case 4: dft4(v); return;
    case 8: dft8(v); return;
    default: dft_generic(v, R, tw, n / R); return;
    }
}

/* Stockham autosort: src -> dst per stage, ping-pong; result returned */
static cplx *stockham(const fftr_plan *p, cplx *a, cplx *b)
{
    size_t n = p->n;
    size_t Ns = 1;
    cplx v[64];
    for (int s = 0; s < p->nstages; ++s) {
        int R = p->radix[s];
        cplx *vv = v;
        cplx *heap = NULL;
        if (R > 64) { heap = (cplx *)malloc(sizeof(cplx) * R); vv = heap; }
        size_t stride = n / R;
        size_t twstep = n / (Ns * R);
        for (size_t j = 0; j < n / R; ++j) {
            size_t jm = j % Ns;
            for (int r = 0; r < R; ++r) {
                cplx x = a[j + r * stride];
                if (r && jm) x = cmul(x, p->tw[(jm * r * twstep) % n]);
                vv[r] = x;
            }
            dft_small(vv, R, p->tw, n);
            size_t idxD = (j / Ns) * Ns * R + jm;
            for (int r = 0; r < R; ++r) b[idxD + r * Ns] = vv[r];
        }
        free(heap);
        cplx *t = a; a = b; b = t;
        Ns *= R;
    }
    return a;
}

static void exec_direct(const fftr_plan *p, cplx *x)
{
    size_t n = p->n;
    if (n <= 1) return;
    cplx stackbuf[4096];
    cplx *scratch = n <= 4096 ? stackbuf : (cplx *)malloc(sizeof(cplx) * n);
    cplx *res = stockham(p, x, scratch);
    if (res != x) memcpy(x, res, sizeof(cplx) * n);
    if (scratch != stackbuf) free(scratch);
}

static void exec_fourstep(const fftr_plan *p, cplx *x)
{
    /* x[j1*n2 + j2], j1 < n1, j2 < n2.
     * step 1: for each j2, FFT over j1 -> Y[k1][j2]; twiddle w^(j2*k1)
     * step 2: for each k1, FFT over j2 -> X[k1 + n1*k2]
     */
    size_t n1 = p->n1, n2 = p->n2, n = p->n;
    cplx *tmp = (cplx *)malloc(sizeof(cplx) * n);
#pragma omp parallel
    {
        cplx *col = (cplx *)malloc(sizeof(cplx) * n1);
#pragma omp for schedule(static)
        for (size_t j2 = 0; j2 < n2; ++j2) {
            for (size_t j1 = 0; j1 < n1; ++j1) col[j1] = x[j1 * n2 + j2];
            if (p->p1->fourstep) exec_fourstep(p->p1, col); else exec_direct(p->p1, col);
            for (size_t k1 = 0; k1 < n1; ++k1) {
                cplx w = p->tw[(j2 * k1) % n];
                tmp[k1 * n2 + j2] = cmul(col[k1], w);
            }
        }
        free(col);
#pragma omp barrier
#pragma omp for schedule(static)
        for (size_t k1 = 0; k1 < n1; ++k1) {
            cplx *row = tmp + k1 * n2;
            if (p->p2->fourstep) exec_fourstep(p->p2, row); else exec_direct(p->p2, row);
        }
#pragma omp barrier
#pragma omp for schedule(static)
        for (size_t k2 = 0; k2 < n2; ++k2)
            for (size_t k1 = 0; k1 < n1; ++k1) x[k1 + n1 * k2] = tmp[k1 * n2 + k2];
    }
    free(tmp);
}

void fftr_execute(const fftr_plan *p, double *x)
{
    if (p->fourstep) exec_fourstep(p, (cplx *)x);
    else exec_direct(p, (cplx *)x);
}

void fftr_forward(double *x, size_t n)
{
    fftr_plan *p = fftr_create(n);
    fftr_execute(p, x);
    fftr_destroy(p);
}

void fftr_naive_dft(const double *x, double *y, size_t n)
{
    for (size_t k = 0; k < n; ++k) {
        long double sr = 0, si = 0;
        for (size_t j = 0; j < n; ++j) {
            size_t e = (j * k) % n;
            long double a = 2.0L * PI_L * (long double)e / (long double)n;
            long double c = cosl(a), s = -sinl(a);
            sr += x[2 * j] * c - x[2 * j + 1] * s;
            si += x[2 * j] * s + x[2 * j + 1] * c;
        }
        y[2 * k] = (double)sr;
        y[2 * k + 1] = (double)si;
    }
}
