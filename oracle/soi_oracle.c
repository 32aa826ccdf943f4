/*
 * soi_oracle.c -- CPU restatement of the SOI FFT hot path.
 *
 * TEST INFRASTRUCTURE: the checker for the CUDA library, never linked into it.
 * Built with -ffp-contract=off and without FMA for the convolution and the
 * demodulation so that its products round exactly like the reference built
 * with -xAVX (Makefile:15; intrinsic.h:24-28 select mul+addsub when AVX2 is
 * absent).  The VLC routines use fma() where compress.c uses _mm256_fmsub_pd /
 * _mm256_fmadd_pd (compress.c:238-261,472-483).
 *
 * Every function cites the reference lines it restates.
 */
#include "soi_oracle.h"
#include "fft_ref.h"

#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* soi.h:308-309: PI as double, VERIFY_PI as a 113-bit quad literal */
static const double PI_D = 3.14159265358979323846;
#define VERIFY_PI_Q 3.141592653589793238462643383279502884197169399375105820974944592307816406286208998628034825342117067982148086q

void oracle_defaults(soi_oracle_params *p)
{
    /* pfft.c:87-91 */
    p->n_mu = 5;
    p->d_mu = 4;
    p->tau = 928 / 1024.;
    p->sigma = 373.7314;
    p->B = 72;
}

/* pfft.c:42-66.  The mixed precision is kept: t in double; the sine/cosine
 * arguments are formed in __float128 and evaluated by the long-double libm;
 * exp() in double; the complex result rounded to double. */
static void w_f(size_t i, const soi_oracle_params *d, double *out)
{
    size_t S = d->S;
    size_t M = d->N / S;
    size_t M_hat = (size_t)d->n_mu * M / (size_t)d->d_mu;
    size_t theta = i / (d->B * S);
    size_t kappa = d->B - (size_t)d->d_mu;
    size_t j = i % (d->B * S);
    double t = ((double)theta / M_hat - (double)j / d->N + (double)kappa / (2 * M)) * M;
    double y;
    if (t == 0) {
        y = 1;
    } else {
        long double sn = sinl((long double)(VERIFY_PI_Q * d->tau * t));
        y = (double)(sn / (PI_D * d->tau * t) * exp(-PI_D * PI_D * t * t / d->sigma));
    }
    double rr = (double)cosl((long double)(VERIFY_PI_Q * t));
    double ri = (double)sinl((long double)(VERIFY_PI_Q * t));
    double mu = (double)d->n_mu / d->d_mu;
    out[0] = rr * y / mu;
    out[1] = ri * y / mu;
}

/* pfft.c:68-82 */
static void W_inv_f(size_t i, const soi_oracle_params *d, double *out)
{
    size_t M = d->N / d->S;
    double t = (double)i / M - 0.5;
    double y = 1 / (2 * d->tau) *
               (erfc(sqrt(d->sigma) * (t - d->tau / 2)) - erfc(sqrt(d->sigma) * (t + d->tau / 2)));
    size_t kappa = d->B - (size_t)d->d_mu;
    double delta = (double)kappa / (2 * M);
    double rr = (double)cosl((long double)(2 * VERIFY_PI_Q * delta * i));
    double ri = -(double)sinl((long double)(2 * VERIFY_PI_Q * delta * i));
    out[0] = rr / y;
    out[1] = ri / y;
}

void oracle_w_table(const soi_oracle_params *p, double *w)
{
    size_t S = p->S, B = p->B;
    size_t total = (size_t)p->n_mu * B * S;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < total; ++i) w_f(i, p, w + 2 * i);
}

void oracle_W_inv_table(const soi_oracle_params *p, double *W_inv)
{
    size_t M = p->N / p->S;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < M; ++i) W_inv_f(i, p, W_inv + 2 * i);
}

/* parallel_filter_subsampling.cpp:218-259 (main loop), :413-425 (K_0 tail),
 * :502-512 (ghost rows).  All three compute, for output row j*n+theta and
 * column s, temp = P(kk=0) then temp = temp + P(kk) for kk = 1..B-1, with
 * P = w*alpha formed as (wr*ar - wi*ai, wr*ai + wi*ar) by mul/mul/addsub.
 * The ghost rows read alpha circularly from the right neighbour
 * (.cpp:101-108); with all rows local that is row index mod R = N/S. */
void oracle_conv(const soi_oracle_params *p, const double *w,
                 const double *alpha, double *G)
{
    size_t S = p->S, B = p->B, n = (size_t)p->n_mu, d = (size_t)p->d_mu;
    size_t M = p->N / S;     /* input rows of S */
    size_t J = M / d;        /* groups of n output rows */
#pragma omp parallel for schedule(static)
    for (size_t j = 0; j < J; ++j) {
        for (size_t th = 0; th < n; ++th) {
            double *g = G + 2 * ((j * n + th) * S);
            for (size_t s = 0; s < S; ++s) {
                double tr = 0, ti = 0;
                for (size_t kk = 0; kk < B; ++kk) {
                    size_t row = (j * d + kk) % M;
                    const double *a = alpha + 2 * (row * S + s);
                    const double *ww = w + 2 * ((th * B + kk) * S + s);
                    double m0 = ww[0] * a[0];
                    double m1 = ww[1] * a[1];
                    double m2 = ww[0] * a[1];
                    double m3 = ww[1] * a[0];
                    double pr = m0 - m1;
                    double pi = m2 + m3;
                    if (kk == 0) { tr = pr; ti = pi; }
                    else { tr = tr + pr; ti = ti + pi; }
                }
                g[2 * s] = tr;
                g[2 * s + 1] = ti;
            }
        }
    }
}

void oracle_row_fft(const soi_oracle_params *p, double *G)
{
    size_t S = p->S;
    size_t Mh = (size_t)p->n_mu * (p->N / S) / (size_t)p->d_mu;
    fftr_plan *pl = fftr_create(S);
#pragma omp parallel for schedule(static)
    for (size_t r = 0; r < Mh; ++r) fftr_execute(pl, G + 2 * r * S);
    fftr_destroy(pl);
}

void oracle_transpose(const soi_oracle_params *p, const double *G, double *T)
{
    size_t S = p->S;
    size_t Mh = (size_t)p->n_mu * (p->N / S) / (size_t)p->d_mu;
#pragma omp parallel for schedule(static)
    for (size_t s = 0; s < S; ++s)
        for (size_t r = 0; r < Mh; ++r) {
            T[2 * (s * Mh + r)] = G[2 * (r * S + s)];
            T[2 * (s * Mh + r) + 1] = G[2 * (r * S + s) + 1];
        }
}

/* pfft.c:642 then :653-660: out = fmaddsub(Wr, g, swap(Wi*g)) which under
 * -xAVX is addsub(mul(Wr,g), swap(mul(Wi,g))). */
void oracle_segment_fft_demod(const soi_oracle_params *p, double *T,
                              const double *W_inv, double *out)
{
    size_t S = p->S, M = p->N / S;
    size_t Mh = (size_t)p->n_mu * M / (size_t)p->d_mu;
    fftr_plan *pl = fftr_create(Mh);
    for (size_t s = 0; s < S; ++s) {
        double *g = T + 2 * s * Mh;
        fftr_execute(pl, g);
        double *o = out + 2 * s * M;
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < M; ++i) {
            double wr = W_inv[2 * i], wi = W_inv[2 * i + 1];
            double gr = g[2 * i], gi = g[2 * i + 1];
            double a = wr * gr, b = wi * gi;
            double c = wr * gi, e = wi * gr;
            o[2 * i] = a - b;
            o[2 * i + 1] = c + e;
        }
    }
    fftr_destroy(pl);
}

static void run_pipeline(const soi_oracle_params *p, size_t chunk_len,
                         const double *alpha, double *out)
{
    size_t S = p->S, M = p->N / S;
    size_t Mh = (size_t)p->n_mu * M / (size_t)p->d_mu;
    double *w = (double *)malloc(sizeof(double) * 2 * (size_t)p->n_mu * p->B * S);
    double *Wi = (double *)malloc(sizeof(double) * 2 * M);
    double *G = (double *)malloc(sizeof(double) * 2 * Mh * S);
    double *T = (double *)malloc(sizeof(double) * 2 * Mh * S);
    oracle_w_table(p, w);
    oracle_W_inv_table(p, Wi);
    oracle_conv(p, w, alpha, G);
    oracle_row_fft(p, G);
    oracle_transpose(p, G, T);
    if (chunk_len) {
        /* pfft.c:316-343: per-segment max exponent (max over the chunks of
         * all ranks after MPI_Allreduce MAX), global max over segments. */
        int *emax = (int *)malloc(sizeof(int) * S);
        int tot = INT_MIN;
        for (size_t s = 0; s < S; ++s) {
            int e = INT_MIN;
            for (size_t c = 0; c < Mh; c += chunk_len) {
                int ec = oracle_max_exponent(T + 2 * (s * Mh + c), (int)(2 * chunk_len));
                if (ec > e) e = ec;
            }
            emax[s] = e;
            if (e > tot) tot = e;
        }
        /* pfft.c:502-506 compress, :624-629 decompress, chunk by chunk */
        int *buf = (int *)malloc(sizeof(int) * (4 * chunk_len + 64));
#pragma omp parallel for schedule(dynamic)
        for (size_t s = 0; s < S; ++s) {
            int *b = (int *)malloc(sizeof(int) * (4 * chunk_len + 64));
            for (size_t c = 0; c < Mh; c += chunk_len) {
                double *x = T + 2 * (s * Mh + c);
                int nw = oracle_compress(b, x, (int)(2 * chunk_len), tot, emax[s]);
                if (nw == 0)
                    memset(x, 0, sizeof(double) * 2 * chunk_len);
                else
                    oracle_decompress(x, b, nw, (int)(2 * chunk_len), tot, emax[s]);
            }
            free(b);
        }
        free(buf);
        free(emax);
    }
    oracle_segment_fft_demod(p, T, Wi, out);
    free(w); free(Wi); free(G); free(T);
}

void oracle_compute_soi(const soi_oracle_params *p, const double *alpha, double *out)
{
    run_pipeline(p, 0, alpha, out);
}

void oracle_compute_soi_vlc(const soi_oracle_params *p, size_t chunk_len,
                            const double *alpha, double *out)
{
    run_pipeline(p, chunk_len, alpha, out);
}

/* ------------------------------------------------------------------ VLC --- */

static inline int biased_exponent(double x)
{
    uint64_t u;
    memcpy(&u, &x, 8);
    return (int)((u >> 52) & 0x7FF);
}

/* compress.c:11-131: the largest biased exponent over the chunk, minus 1023.
 * (The AVX loop reads whole 8-double blocks; for len % 8 != 0 with several
 * OpenMP threads it can read past len -- .c:52-58.  The restatement uses the
 * intended semantics, the max over [0, len).) */
int oracle_max_exponent(const double *x, int len)
{
    int m = INT_MIN;
    for (int i = 0; i < len; ++i) {
        int e = biased_exponent(x[i]);
        if (e > m) m = e;
    }
    return m - 1023;
}

#define VLEN 16
static const int NBITS = 52;   /* compress.c:145 */

static inline uint32_t low_mask(int nbits)
{
    return nbits >= 32 ? 0xFFFFFFFFu : ((1u << nbits) - 1u);
}

/* compress.c:170-203: sixteen lanes share one occupancy counter; lane L of
 * each 16-word group belongs to element 16*g + L. */
static void append16(uint32_t *v, uint32_t *cur, int *occ, int *out, int *outIdx, int nbits)
{
    uint32_t m = low_mask(nbits);
    for (int L = 0; L < VLEN; ++L) v[L] &= m;
    *occ += nbits;
    if (*occ >= 32) {
        int nb = *occ - 32;
        for (int L = 0; L < VLEN; ++L) {
            uint32_t w = cur[L] | (nb ? (v[L] >> nb) : v[L]);
            out[*outIdx + L] = (int)w;
        }
        *outIdx += VLEN;
        uint32_t mk = nb ? ((1u << nb) - 1u) : 0u;
        for (int L = 0; L < VLEN; ++L) {
            v[L] &= mk;
            cur[L] = nb ? (v[L] << (32 - nb)) : 0u;
        }
        *occ = nb;
    } else {
        for (int L = 0; L < VLEN; ++L) cur[L] |= v[L] << (32 - *occ);
    }
}

/* compress.c:147-166, one scalar stream for the tail */
static void append1(uint32_t v, uint32_t *cur, int *occ, int *out, int *outIdx, int nbits)
{
    v &= low_mask(nbits);
    *occ += nbits;
    if (*occ >= 32) {
        int nb = *occ - 32;
        *cur |= nb ? (v >> nb) : v;
        out[*outIdx] = (int)*cur;
        *cur = 0;
        v &= nb ? ((1u << nb) - 1u) : 0u;
        ++*outIdx;
        *occ = nb;
    }
    if (*occ) *cur |= v << (32 - *occ);
}

int oracle_compress(int *out, const double *in, int len, int e_max, int e_max_i)
{
    /* compress.c:207-216 */
    const int i1Len = (NBITS + 3 - 31) - (e_max - e_max_i);
    const int i2Len = (NBITS + 3 - (e_max - e_max_i)) < 32 ? (NBITS + 3 - (e_max - e_max_i)) : 32;
    if (i2Len <= 0) return 0;
    double e1 = pow(2, (NBITS - 31) - e_max);
    double e2 = pow(2, NBITS - e_max);
    double e3 = pow(2, 31);

    uint32_t cur[VLEN] = { 0 };
    int occ = 0, outIdx = 0, i = 0;
    /* :227-322, vector body: _mm256_round_pd(nearest) for i1, fmsub for the
     * remainder, _mm256_cvtpd_epi32 (round to nearest even) for both */
    for (; i < len / VLEN * VLEN; i += VLEN) {
        uint32_t v1[VLEN], v2[VLEN];
        for (int L = 0; L < VLEN; ++L) {
            double x = in[i + L];
            double d1 = nearbyint(x * e1);
            double d2 = fma(x, e2, -(d1 * e3));
            v1[L] = (uint32_t)(int32_t)d1;
            v2[L] = (uint32_t)(int32_t)nearbyint(d2);
        }
        if (i1Len > 0) append16(v1, cur, &occ, out, &outIdx, i1Len);
        append16(v2, cur, &occ, out, &outIdx, i2Len);
    }
    /* :324-328 flush the partial group */
    if (occ) {
        for (int L = 0; L < VLEN; ++L) out[outIdx + L] = (int)cur[L];
        outIdx += VLEN;
    }
    /* :330-369 scalar tail, round() = half away from zero */
    uint32_t c1 = 0;
    occ = 0;
    for (; i < len; ++i) {
        double x = in[i];
        double d1 = round(x * e1);
        double d2 = round(x * e2 - d1 * e3);
        if (i1Len > 0) append1((uint32_t)(int32_t)d1, &c1, &occ, out, &outIdx, i1Len);
        append1((uint32_t)(int32_t)d2, &c1, &occ, out, &outIdx, i2Len);
    }
    if (occ) out[outIdx++] = (int)c1;
    return outIdx;
}

int oracle_vlc_words(int len, int e_max, int e_max_i)
{
    const int i1Len = (NBITS + 3 - 31) - (e_max - e_max_i);
    const int i2Len = (NBITS + 3 - (e_max - e_max_i)) < 32 ? (NBITS + 3 - (e_max - e_max_i)) : 32;
    if (i2Len <= 0) return 0;
    int bits = i2Len + (i1Len > 0 ? i1Len : 0);
    int groups = len / VLEN;
    int words = (int)(((long)groups * bits + 31) / 32) * VLEN;
    int tail = len % VLEN;
    words += (int)(((long)tail * bits + 31) / 32);
    return words;
}

static inline int32_t word_at(const int *in, int in_words, int idx)
{
    return (idx >= 0 && idx < in_words) ? in[idx] : 0;
}

/* compress.c:395-426 */
static void extract16(int32_t *v, uint32_t *cur, int *occ, const int *in, int in_words,
                      int *inIdx, int nbits)
{
    for (int L = 0; L < VLEN; ++L)
        v[L] = (int32_t)(cur[L] << (32 - *occ)) >> (32 - nbits);
    if (nbits <= *occ) {
        *occ -= nbits;
        if (*occ == 0) {
            for (int L = 0; L < VLEN; ++L) cur[L] = (uint32_t)word_at(in, in_words, *inIdx + L);
            *inIdx += VLEN;
            *occ = 32;
        }
    } else {
        int need = nbits - *occ;
        for (int L = 0; L < VLEN; ++L) {
            cur[L] = (uint32_t)word_at(in, in_words, *inIdx + L);
            v[L] |= (int32_t)(cur[L] >> (32 - need));
        }
        *inIdx += VLEN;
        *occ = 32 - need;
    }
}

/* compress.c:374-393 */
static int32_t extract1(uint32_t *cur, int *occ, const int *in, int in_words, int *inIdx, int nbits)
{
    int32_t v = (int32_t)(*cur << (32 - *occ)) >> (32 - nbits);
    if (nbits <= *occ) {
        *occ -= nbits;
        if (*occ == 0) {
            *cur = (uint32_t)word_at(in, in_words, *inIdx);
            ++*inIdx;
            *occ = 32;
        }
    } else {
        int need = nbits - *occ;
        *cur = (uint32_t)word_at(in, in_words, *inIdx);
        /* logicalRightShift, compress.c:133-141 */
        v |= (int32_t)(*cur >> (32 - need));
        ++*inIdx;
        *occ = 32 - need;
    }
    return v;
}

void oracle_decompress(double *out, const int *in, int in_words, int len,
                       int e_max, int e_max_i)
{
    double e1 = pow(2, e_max - (NBITS - 31));
    double e2 = pow(2, e_max - NBITS);
    const int i1Len = (NBITS + 3 - 31) - (e_max - e_max_i);
    const int i2Len = (NBITS + 3 - (e_max - e_max_i)) < 32 ? (NBITS + 3 - (e_max - e_max_i)) : 32;

    uint32_t cur[VLEN];
    for (int L = 0; L < VLEN; ++L) cur[L] = (uint32_t)word_at(in, in_words, L);
    int occ = 32, inIdx = VLEN, i = 0;
    for (; i < len / VLEN * VLEN; i += VLEN) {
        int32_t v1[VLEN] = { 0 }, v2[VLEN];
        if (i1Len > 0) extract16(v1, cur, &occ, in, in_words, &inIdx, i1Len);
        extract16(v2, cur, &occ, in, in_words, &inIdx, i2Len);
        for (int L = 0; L < VLEN; ++L)
            out[i + L] = fma((double)v1[L], e1, (double)v2[L] * e2);   /* :472-483 */
    }
    /* :491-499: the scalar tail is located by this index arithmetic */
    if (occ < 32) inIdx += VLEN;
    else inIdx -= VLEN - 1;
    uint32_t c1 = (uint32_t)word_at(in, in_words, inIdx);
    occ = 32;
    for (; i < len; ++i) {
        int32_t v1 = 0;
        if (i1Len > 0) v1 = extract1(&c1, &occ, in, in_words, &inIdx, i1Len);
        int32_t v2 = extract1(&c1, &occ, in, in_words, &inIdx, i2Len);
        out[i] = (double)v1 * e1 + (double)v2 * e2;               /* :529-532 */
    }
}
