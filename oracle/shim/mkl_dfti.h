/* Stand-in for MKL's DFTI interface, covering the calls the reference makes:
 *   DftiCreateDescriptor / DftiSetValue / DftiCommitDescriptor  pfft.c:224-228
 *   DftiComputeForward  parallel_filter_subsampling.cpp:308,432,517; pfft.c:642
 *   DftiFreeDescriptor / DftiErrorClass / DftiErrorMessage  pfft.c:246-247; soi.h:182-188
 * Backed by oracle/fft_ref.c (forward, unnormalised).  TEST INFRASTRUCTURE. */
#ifndef SOI_SHIM_MKL_DFTI_H
#define SOI_SHIM_MKL_DFTI_H
#ifdef __cplusplus
extern "C" {
#endif
typedef long MKL_LONG;
typedef struct soi_dfti_desc *DFTI_DESCRIPTOR_HANDLE;
enum DFTI_CONFIG_PARAM {
  DFTI_FORWARD_DOMAIN = 0, DFTI_DIMENSION, DFTI_LENGTHS, DFTI_PRECISION,
  DFTI_PLACEMENT, DFTI_NUMBER_OF_USER_THREADS, DFTI_THREAD_LIMIT,
  DFTI_NUMBER_OF_TRANSFORMS
};
enum DFTI_CONFIG_VALUE {
  DFTI_COMPLEX = 32, DFTI_REAL = 33, DFTI_SINGLE = 35, DFTI_DOUBLE = 36,
  DFTI_INPLACE = 43, DFTI_NOT_INPLACE = 44
};
#define DFTI_NO_ERROR 0
MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE *h, enum DFTI_CONFIG_VALUE precision,
                              enum DFTI_CONFIG_VALUE domain, MKL_LONG dim, ...);
MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE h, enum DFTI_CONFIG_PARAM param, ...);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void *x, ...);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE *h);
MKL_LONG DftiErrorClass(MKL_LONG status, MKL_LONG error_class);
char *DftiErrorMessage(MKL_LONG status);
#ifdef __cplusplus
}
#endif
#endif
