/* complex.h stand-in for building the reference's C++ translation unit with
 * g++: libstdc++'s <complex.h> undefines the C99 `complex` macro once
 * <complex> is in, but soi.h:227 spells `VAL_TYPE complex`.  C keeps the
 * system header as is.  TEST INFRASTRUCTURE for oracle/_ref. */
#ifndef SOI_SHIM_COMPLEX_H
#define SOI_SHIM_COMPLEX_H
#include_next <complex.h>
#ifdef __cplusplus
#undef complex
#define complex _Complex
#ifndef I
#define I (__extension__ 1.0iF)
#endif
#endif
#endif
