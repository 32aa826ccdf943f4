/*
 * fft_ref.h -- FP64 mixed-radix FFT used by the CPU oracle and by the
 * DFTI stand-in that lets the reference's own sources build here.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links this file;
 * only tests/, the smoke check and bench.py's CPU-baseline leg reach it.
 *
 * Convention: forward, unnormalised, X[k] = sum_j x[j] exp(-2*pi*i*j*k/n),
 * the same transform MKL DFTI computes for DftiComputeForward on a
 * DFTI_COMPLEX / DFTI_DOUBLE descriptor (reference call sites:
 * parallel_filter_subsampling.cpp:308,432,517 and pfft.c:642).
 */
#ifndef SOI_ORACLE_FFT_REF_H
#define SOI_ORACLE_FFT_REF_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fftr_plan fftr_plan;

/* Plan a length-n forward transform (any n >= 1). */
fftr_plan *fftr_create(size_t n);
/* In-place transform of n interleaved (re, im) doubles; thread-safe. */
void fftr_execute(const fftr_plan *p, double *x);
void fftr_destroy(fftr_plan *p);
size_t fftr_size(const fftr_plan *p);

/* One-shot helpers for tests. */
void fftr_forward(double *x, size_t n);
/* Naive O(n^2) DFT in long double, for pinning the FFT itself. */
void fftr_naive_dft(const double *x, double *y, size_t n);

#ifdef __cplusplus
}
#endif
#endif
