/* Forced-include header (gcc -include) that maps the Intel-compiler spellings
 * used by the reference sources onto GCC ones.  TEST INFRASTRUCTURE for
 * oracle/_ref; the reference files themselves are compiled unmodified.
 *   __declspec(noinline)   soi.h:272, parallel_filter_subsampling.cpp:534
 *   __declspec(align(n))   soi.h:290, compress.c:69, intrinsic.h:61,72
 *   __declspec(aligned(n)) parallel_filter_subsampling.cpp:137,284
 *   __rdtsc()              cpu_freq.c:15, parallel_filter_subsampling.cpp:165
 */
#ifndef SOI_SHIM_COMPAT_H
#define SOI_SHIM_COMPAT_H
#define __declspec(x) __soi_declspec_##x
#define __soi_declspec_noinline __attribute__((noinline))
#define __soi_declspec_align(n) __attribute__((aligned(n)))
#define __soi_declspec_aligned(n) __attribute__((aligned(n)))
#include <x86intrin.h>
#endif
