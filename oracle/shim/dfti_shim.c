/* DFTI stand-in on top of the oracle FFT (oracle/fft_ref.c).  TEST
 * INFRASTRUCTURE: lets the reference's pfft.c and
 * parallel_filter_subsampling.cpp build and run here without MKL. */
#include <stdarg.h>
#include <stdlib.h>
#include "mkl_dfti.h"
#include "../fft_ref.h"

struct soi_dfti_desc { long n; fftr_plan *plan; };

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *h, enum DFTI_CONFIG_VALUE precision,
                              enum DFTI_CONFIG_VALUE domain, MKL_LONG dim, ...)
{
  if (precision != DFTI_DOUBLE || domain != DFTI_COMPLEX || dim != 1) return 1;
  va_list ap;
  va_start(ap, dim);
  long n = va_arg(ap, long);
  va_end(ap);
  struct soi_dfti_desc *d = (struct soi_dfti_desc *)calloc(1, sizeof(*d));
  d->n = n;
  *h = d;
  return DFTI_NO_ERROR;
}
MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE h, enum DFTI_CONFIG_PARAM param, ...)
{
  (void)h; (void)param;
  return DFTI_NO_ERROR;
}
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h)
{
  if (!h->plan) h->plan = fftr_create((size_t)h->n);
  return DFTI_NO_ERROR;
}
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void *x, ...)
{
  fftr_execute(h->plan, (double *)x);
  return DFTI_NO_ERROR;
}
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *h)
{
  if (*h) { fftr_destroy((*h)->plan); free(*h); *h = NULL; }
  return DFTI_NO_ERROR;
}
MKL_LONG DftiErrorClass(MKL_LONG status, MKL_LONG error_class) { return status == error_class; }
char *DftiErrorMessage(MKL_LONG status) { (void)status; return (char *)"dfti shim error"; }
