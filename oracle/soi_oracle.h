/*
 * soi_oracle.h -- CPU restatement of the SOI FFT hot path (TEST INFRASTRUCTURE).
 *
 * This is the checker, never the product: only tests/, the smoke check and
 * bench.py's CPU-baseline leg load it.  It restates, in plain C, the algorithm
 * of the reference's pfft.c / parallel_filter_subsampling.cpp / compress.c for
 * one process (the reference's arithmetic per output element does not depend
 * on the MPI rank count P, only on S = k*P).  It is pinned bit-for-bit against
 * the reference sources compiled here (oracle/_ref, see oracle/Makefile) and
 * against the reference's own VLC vectors (tests/golden).
 *
 * Complex buffers are interleaved (re, im) doubles, like cfft_complex_t
 * (soi.h:227).
 */
#ifndef SOI_ORACLE_H
#define SOI_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    size_t N;       /* global length                          */
    size_t S;       /* segments (S = k*P in the reference)     */
    int n_mu, d_mu; /* oversampling mu = n_mu/d_mu            */
    size_t B;       /* window taps                            */
    double tau, sigma;
} soi_oracle_params;

/* set_default_soi_descriptor, pfft.c:84-92 */
void oracle_defaults(soi_oracle_params *p);

/* w[theta][kk][s] = w_f(theta*B*S + kk*S + s), pfft.c:42-66,190-196 */
void oracle_w_table(const soi_oracle_params *p, double *w);
/* W_inv[i], i < M, pfft.c:68-82,207-210 */
void oracle_W_inv_table(const soi_oracle_params *p, double *W_inv);

/* Filter-subsampling convolution (circular), G has M' rows of S:
 * G[row*S + s], row = j*n_mu + theta.  parallel_filter_subsampling.cpp:218-259 */
void oracle_conv(const soi_oracle_params *p, const double *w,
                 const double *alpha, double *G);
/* In-place S-point forward DFT of every row of G (.cpp:308,432,517). */
void oracle_row_fft(const soi_oracle_params *p, double *G);
/* T[s*M' + row] = G[row*S + s] (.cpp:391,437; pfft.c:554-578 with P=1). */
void oracle_transpose(const soi_oracle_params *p, const double *G, double *T);
/* M'-point DFT of each segment then out[s*M+i] = W_inv[i]*T^[s][i], i < M
 * (pfft.c:642,653-685).  T is overwritten. */
void oracle_segment_fft_demod(const soi_oracle_params *p, double *T,
                              const double *W_inv, double *out);
/* Whole compute_soi, out has N complex in natural DFT order. */
void oracle_compute_soi(const soi_oracle_params *p, const double *alpha, double *out);
/* Same, with the VLC round trip of compress.c applied to the transposed
 * data between the S-point and M'-point FFTs, per segment chunk of
 * chunk_len complex (chunk_len = M'/P in the reference).  pfft.c:316-353,
 * 390-447,502-506,618-632. */
void oracle_compute_soi_vlc(const soi_oracle_params *p, size_t chunk_len,
                            const double *alpha, double *out);

/* VLC, compress.c */
int oracle_max_exponent(const double *x, int len);                       /* :11-131  */
int oracle_compress(int *out, const double *in, int len, int e_max, int e_max_i);   /* :205-372 */
void oracle_decompress(double *out, const int *in, int in_words, int len,
                       int e_max, int e_max_i);                          /* :428-544 */
/* number of ints compress() writes for a chunk (pfft.c:397-402 sizing) */
int oracle_vlc_words(int len, int e_max, int e_max_i);

#ifdef __cplusplus
}
#endif
#endif
