// fft_device.cuh -- complex helpers, radix butterflies and the in-place
// shared-memory decimation-in-frequency FFT used by every SOI kernel.
//
// Forward transforms, exp(-2*pi*i*j*k/L), unnormalised (the DFTI forward
// transform the reference calls at parallel_filter_subsampling.cpp:308 and
// pfft.c:642).  Twiddle tables are generated on the host in long double and
// rounded once to the working precision.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace soi {

template <typename R> struct cplx_of;
template <> struct cplx_of<float> { using type = float2; };
template <> struct cplx_of<double> { using type = double2; };

template <typename V> __device__ __forceinline__ V cmk(decltype(V::x) a, decltype(V::x) b) { V r; r.x = a; r.y = b; return r; }
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return cmk<V>(a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return cmk<V>(a.x - b.x, a.y - b.y); }
// FP32: one packed add (FADD2) per complex add or subtract, the same IEEE
// roundings as two scalar adds in half the instructions (the butterflies are
// mostly adds; measured 1.2 % on stage 1 and 1.7 % on stage 2 at N = 2^29)
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b)
{
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
template <typename V> __device__ __forceinline__ V cmul(V a, V b)
{
  return cmk<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// -i * a
template <typename V> __device__ __forceinline__ V cmi(V a) { return cmk<V>(a.y, -a.x); }
template <typename V> __device__ __forceinline__ V cscale(V a, decltype(V::x) s) { return cmk<V>(a.x * s, a.y * s); }

// Maximum number of radix stages of one in-shared-memory FFT.
constexpr int kMaxStages = 16;

struct FftPlan {
  int L;                    // length
  int nst;                  // stages
  int radix[kMaxStages];    // radix of each DIF stage, first stage first
};

// ---- butterflies (forward) ------------------------------------------------

template <typename V> __device__ __forceinline__ void dft2(V *v)
{
  V a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <typename V> __device__ __forceinline__ void dft4(V *v)
{
  V a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
  V a2 = cadd(v[1], v[3]), a3 = cmi(csub(v[1], v[3]));
  v[0] = cadd(a0, a2);
  v[2] = csub(a0, a2);
  v[1] = cadd(a1, a3);
  v[3] = csub(a1, a3);
}

template <typename V> __device__ __forceinline__ void dft8(V *v)
{
  using R = decltype(V::x);
  const R h = (R)0.70710678118654752440084436210484903928L;
  V e[4] = { v[0], v[2], v[4], v[6] };
  V o[4] = { v[1], v[3], v[5], v[7] };
  dft4(e);
  dft4(o);
  // multiply o[k] by exp(-2 pi i k/8)
  V t1 = cmk<V>(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
  V t2 = cmi(o[2]);
  V t3 = cmk<V>(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
  v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], t1);   v[5] = csub(e[1], t1);
  v[2] = cadd(e[2], t2);   v[6] = csub(e[2], t2);
  v[3] = cadd(e[3], t3);   v[7] = csub(e[3], t3);
}

template <typename V> __device__ __forceinline__ void dft3(V *v)
{
  using R = decltype(V::x);
  const R s3 = (R)0.86602540378443864676372317075293618347L;  // sin(2 pi/3)
  V a = cadd(v[1], v[2]);
  V b = csub(v[1], v[2]);
  V y0 = cadd(v[0], a);
  V t = cmk<V>(v[0].x - (R)0.5 * a.x, v[0].y - (R)0.5 * a.y);
  V u = cmk<V>(s3 * b.y, -s3 * b.x);     // -i * s3 * b
  v[0] = y0;
  v[1] = cadd(t, u);
  v[2] = csub(t, u);
}

template <typename V> __device__ __forceinline__ void dft5(V *v)
{
  using R = decltype(V::x);
  const R c1 = (R)0.30901699437494742410229341718281905886L;   // cos(2 pi/5)
  const R c2 = (R)-0.80901699437494742410229341718281905886L;  // cos(4 pi/5)
  const R s1 = (R)0.95105651629515357211643933337938214340L;   // sin(2 pi/5)
  const R s2 = (R)0.58778525229247312916870595463907276860L;   // sin(4 pi/5)
  V a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  V a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  V y0 = cadd(v[0], cadd(a1, a2));
  V t1 = cmk<V>(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
  V t2 = cmk<V>(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
  V u1 = cmk<V>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);
  V u2 = cmk<V>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);
  v[0] = y0;
  v[1] = csub(t1, cmk<V>(-u1.y, u1.x));   // t1 - i*u1
  v[4] = cadd(t1, cmk<V>(-u1.y, u1.x));
  v[2] = csub(t2, cmk<V>(-u2.y, u2.x));
  v[3] = cadd(t2, cmk<V>(-u2.y, u2.x));
}

// Generic radix R <= 16 by direct O(R^2) sums; wR[k] = exp(-2 pi i k/R).
template <typename V, int RR> __device__ __forceinline__ void dft_generic(V *v, const V *wR)
{
  V o[RR];
#pragma unroll
  for (int k = 0; k < RR; ++k) {
    V acc = v[0];
#pragma unroll
    for (int r = 1; r < RR; ++r) acc = cadd(acc, cmul(v[r], wR[(r * k) % RR]));
    o[k] = acc;
  }
#pragma unroll
  for (int k = 0; k < RR; ++k) v[k] = o[k];
}

template <typename V, int RR> struct Bfly {
  static __device__ __forceinline__ void run(V *v, const V *wR) { dft_generic<V, RR>(v, wR); }
};
template <typename V> struct Bfly<V, 2> { static __device__ __forceinline__ void run(V *v, const V *) { dft2(v); } };
template <typename V> struct Bfly<V, 3> { static __device__ __forceinline__ void run(V *v, const V *) { dft3(v); } };
template <typename V> struct Bfly<V, 4> { static __device__ __forceinline__ void run(V *v, const V *) { dft4(v); } };
template <typename V> struct Bfly<V, 5> { static __device__ __forceinline__ void run(V *v, const V *) { dft5(v); } };
template <typename V> struct Bfly<V, 8> { static __device__ __forceinline__ void run(V *v, const V *) { dft8(v); } };

// ---- one in-place DIF stage over a batch of sequences ----------------------
//
// Element `pos` of sequence `col` lives at buf[pos*pos_stride + col*col_stride].
// Stage of radix RR with previous span span_prev (L for the first stage):
// the butterfly at (block, i) reads positions base + r*span, base =
// block*span_prev + i, and writes output k back at base + k*span multiplied
// by exp(-2 pi i * i*k / span_prev) = tw[i*k*(L/span_prev)].  tw may live in
// shared or global memory (generic loads).
// After all stages position p = sum_s d_s*span_s holds frequency
// k = d_0 + r_0*(d_1 + r_1*(d_2 + ...)), the mixed-radix digit reversal that
// the host precomputes as perm[k] = p.
template <typename V, int RR>
__device__ __forceinline__ void dif_stage(V *buf, int L, int span_prev, int ncol, int pos_stride,
                                          int col_stride, const V *tw, const V *wR)
{
  const int span = span_prev / RR;
  const int tw_scale = L / span_prev;
  const int nbf = (L / RR) * ncol;
  for (int q = threadIdx.x; q < nbf; q += blockDim.x) {
    const int col = q % ncol;
    const int t = q / ncol;
    const int blk = t / span;
    const int i = t - blk * span;
    const int base = blk * span_prev + i;
    V v[RR];
#pragma unroll
    for (int r = 0; r < RR; ++r) v[r] = buf[(base + r * span) * pos_stride + col * col_stride];
    Bfly<V, RR>::run(v, wR);
    if (i) {
#pragma unroll
      for (int k = 1; k < RR; ++k) v[k] = cmul(v[k], tw[i * k * tw_scale]);
    }
#pragma unroll
    for (int r = 0; r < RR; ++r) buf[(base + r * span) * pos_stride + col * col_stride] = v[r];
  }
  __syncthreads();
}

// Whole in-place DIF transform of `ncol` sequences of length plan.L; output in
// digit-reversed positions (see perm).  Must be called by all threads of the
// block; ends with __syncthreads().  wsmall holds exp(-2 pi i k/R) for the
// generic radices 7 and 16 (indices [0,7) and [8,24)).
template <typename V>
__device__ void smem_fft(V *buf, const FftPlan &plan, int ncol, int pos_stride, int col_stride,
                         const V *tw, const V *wsmall)
{
  int span_prev = plan.L;
  for (int s = 0; s < plan.nst; ++s) {
    const int r = plan.radix[s];
    switch (r) {
      case 2: dif_stage<V, 2>(buf, plan.L, span_prev, ncol, pos_stride, col_stride, tw, wsmall); break;
      case 3: dif_stage<V, 3>(buf, plan.L, span_prev, ncol, pos_stride, col_stride, tw, wsmall); break;
      case 4: dif_stage<V, 4>(buf, plan.L, span_prev, ncol, pos_stride, col_stride, tw, wsmall); break;
      case 5: dif_stage<V, 5>(buf, plan.L, span_prev, ncol, pos_stride, col_stride, tw, wsmall); break;
      case 8: dif_stage<V, 8>(buf, plan.L, span_prev, ncol, pos_stride, col_stride, tw, wsmall); break;
      case 7: dif_stage<V, 7>(buf, plan.L, span_prev, ncol, pos_stride, col_stride, tw, wsmall); break;
      default: break;  // the host never plans other radices
    }
    span_prev /= r;
  }
}

}  // namespace soi
