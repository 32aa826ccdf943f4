// soi_kernels.cuh -- the SOI hot path on sm_100a.
//
// Stage 1, k_conv_sfft: the filter-subsampling convolution of
// parallel_filter_subsampling.cpp:134-287 fused with the S-point FFTs
// (:297-311) and with the segment transpose that the reference splits into a
// local transpose (:316-395) and an MPI all-to-all (pfft.c:441-583).
// Stage 2, k_seg_cols + k_seg_rows_demod: the M'-point FFT of every segment
// (pfft.c:642) as a two-pass four-step FFT with the demodulation and the
// oversampling discard (pfft.c:649-694) fused into the last pass.
//
// Data layout in HBM (interleaved complex, precision R):
//   alpha  [M rows][S]          input, row r = alpha[r*S .. r*S+S)
//   T      [S segments][M']     transposed data, one contiguous M'-sequence
//                               per segment (the reference's alpha_tilde)
//   out    [S segments][M]      natural DFT order
// Window factorisation: w[theta][kk][s] = phase[theta][s] * filt[kk][theta][s]
// with filt real (see the host table code), so each tap costs two real FMAs.
#pragma once

#include "fft_device.cuh"

namespace soi {

struct ConvArgs {
  const void *alpha;     // [M][S] complex
  void *T;               // [S][Mh] complex
  const void *filt;      // [atap*d][nmu][S] real, zero beyond B taps
  const void *phase;     // [nmu][S] complex
  const void *twS;       // [S] complex, exp(-2 pi i m/S)
  const int *permS;      // [S]
  const void *wsmall;    // generic-radix roots
  FftPlan planS;
  long long M;           // input rows (N/S)
  long long Mh;          // M' rows of output
  long long J;           // M/d output groups
  int S, d, atap, JT, pitch;
  int seg_lo, seg_hi;    // segments sigma stored (all: 0, S)
};

// Input row index (j*d + kk) mod M for the circular convolution; the ghost
// rows of parallel_filter_subsampling.cpp:495-515 are the rows >= M.
__device__ __forceinline__ long long wrap_row(long long r, long long M) { return r >= M ? r - M : r; }

template <typename R, int NMU, int JR>
__global__ void __launch_bounds__(256) k_conv_sfft(ConvArgs a)
{
  using V = typename cplx_of<R>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int S = a.S;
  const int rows_tile = NMU * a.JT;
  V *tile = reinterpret_cast<V *>(smem_raw);                       // [rows_tile][pitch]
  V *twS = tile + (size_t)rows_tile * a.pitch;                      // [S]
  int *permS = reinterpret_cast<int *>(twS + S);                    // [S]

  const int tid = threadIdx.x;
  for (int i = tid; i < S; i += blockDim.x) {
    twS[i] = reinterpret_cast<const V *>(a.twS)[i];
    permS[i] = a.permS[i];
  }

  const V *__restrict__ alpha = reinterpret_cast<const V *>(a.alpha);
  const R *__restrict__ filt = reinterpret_cast<const R *>(a.filt);
  const int s = tid % S;
  const int jb = tid / S;
  const long long j0 = (long long)blockIdx.x * a.JT;
  const long long jbase = j0 + (long long)jb * JR;
  const bool active = jb * JR < a.JT;
  const int d = a.d;
  const long long M = a.M;

  V acc[JR][NMU];
#pragma unroll
  for (int jj = 0; jj < JR; ++jj)
#pragma unroll
    for (int th = 0; th < NMU; ++th) acc[jj][th] = cmk<V>((R)0, (R)0);

  if (active) {
    const int atap = a.atap;
    const int rem = atap % JR;
    const int amain = atap - rem;
    for (int b = 0; b < d; ++b) {
      // window slot (a + jj) % JR holds x_b[jbase + a + jj] at step a,
      // x_b[t] = alpha[(d*t + b) mod M][s]
      V xw[JR];
#pragma unroll
      for (int jj = 0; jj < JR - 1; ++jj)
        xw[jj] = __ldg(alpha + wrap_row(d * (jbase + jj) + b, M) * S + s);
      for (int a0 = 0; a0 < amain; a0 += JR) {
#pragma unroll
        for (int u = 0; u < JR; ++u) {
          const int astep = a0 + u;
          xw[(u + JR - 1) % JR] = __ldg(alpha + wrap_row(d * (jbase + astep + JR - 1) + b, M) * S + s);
          const R *hp = filt + ((size_t)(astep * d + b) * NMU) * S + s;
          R h[NMU];
#pragma unroll
          for (int th = 0; th < NMU; ++th) h[th] = __ldg(hp + th * S);
#pragma unroll
          for (int jj = 0; jj < JR; ++jj) {
            const V x = xw[(u + jj) % JR];
#pragma unroll
            for (int th = 0; th < NMU; ++th) {
              acc[jj][th].x = fma(h[th], x.x, acc[jj][th].x);
              acc[jj][th].y = fma(h[th], x.y, acc[jj][th].y);
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < JR - 1; ++u) {
        if (u < rem) {
          const int astep = amain + u;
          xw[(u + JR - 1) % JR] = __ldg(alpha + wrap_row(d * (jbase + astep + JR - 1) + b, M) * S + s);
          const R *hp = filt + ((size_t)(astep * d + b) * NMU) * S + s;
          R h[NMU];
#pragma unroll
          for (int th = 0; th < NMU; ++th) h[th] = __ldg(hp + th * S);
#pragma unroll
          for (int jj = 0; jj < JR; ++jj) {
            const V x = xw[(u + jj) % JR];
#pragma unroll
            for (int th = 0; th < NMU; ++th) {
              acc[jj][th].x = fma(h[th], x.x, acc[jj][th].x);
              acc[jj][th].y = fma(h[th], x.y, acc[jj][th].y);
            }
          }
        }
      }
    }
    // epilogue: G = phase * acc into the tile, row (jb*JR + jj)*NMU + theta
    const V *ph = reinterpret_cast<const V *>(a.phase);
#pragma unroll
    for (int th = 0; th < NMU; ++th) {
      const V p = __ldg(ph + th * S + s);
#pragma unroll
      for (int jj = 0; jj < JR; ++jj)
        tile[(size_t)((jb * JR + jj) * NMU + th) * a.pitch + s] = cmul(p, acc[jj][th]);
    }
  }
  __syncthreads();

  // S-point FFT of every row of the tile (rows are the sequences).
  smem_fft<V>(tile, a.planS, rows_tile, 1, a.pitch, reinterpret_cast<const V *>(twS),
              reinterpret_cast<const V *>(a.wsmall));

  // transposed store: T[sigma][rho0 + r] = tile[r][perm(sigma)]
  V *T = reinterpret_cast<V *>(a.T);
  const long long rho0 = (long long)NMU * j0;
  const int total = S * rows_tile;
  for (int idx = tid; idx < total; idx += blockDim.x) {
    const int sg = idx / rows_tile;
    const int r = idx - sg * rows_tile;
    const long long rho = rho0 + r;
    if (rho < a.Mh && sg >= a.seg_lo && sg < a.seg_hi) T[(size_t)sg * a.Mh + rho] = tile[(size_t)r * a.pitch + permS[sg]];
  }
}

// ---------------------------------------------------------------- stage 2 --

struct SegArgs {
  void *T;                 // [S][Mh] complex, in/out of pass 1, input of pass 2
  void *out;               // [S][M] complex
  const void *tw1; const int *perm1; FftPlan plan1;   // length M1
  const void *tw2; const int *perm2; FftPlan plan2;   // length M2
  const double2 *xtw_lo;   // exp(-2 pi i e/Mh), e < 2^lo_bits       (FP64)
  const double2 *xtw_hi;   // exp(-2 pi i (e << lo_bits)/Mh)          (FP64)
  const void *winv;        // [M] complex demodulation table
  const void *wsmall;
  long long Mh, M;
  int M1, M2, C1, C2, lo_bits;
  int seg_lo;              // segment of blockIdx.y == 0
};

// w_{M'}^e computed in FP64 from two tables and rounded once to R.
template <typename V>
__device__ __forceinline__ V cross_twiddle(const SegArgs &a, long long e)
{
  const double2 lo = __ldg(a.xtw_lo + (e & ((1ll << a.lo_bits) - 1)));
  const double2 hi = __ldg(a.xtw_hi + (e >> a.lo_bits));
  const double re = hi.x * lo.x - hi.y * lo.y;
  const double im = hi.x * lo.y + hi.y * lo.x;
  V w;
  w.x = (decltype(w.x))re;
  w.y = (decltype(w.y))im;
  return w;
}

// Pass 1: segment seg_lo + blockIdx.y, columns m2 in [blockIdx.x*C1, +C1): FFT of
// length M1 over m1 of T[m1*M2 + m2], times w_{M'}^(m2*k1), stored in place
// at k1*M2 + m2.
template <typename R>
__global__ void __launch_bounds__(256) k_seg_cols(SegArgs a)
{
  using V = typename cplx_of<R>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *buf = reinterpret_cast<V *>(smem_raw);
  const int C1 = a.C1, M1 = a.M1, M2 = a.M2;
  const int ps = C1 + 1;
  V *seg = reinterpret_cast<V *>(a.T) + (size_t)(a.seg_lo + blockIdx.y) * a.Mh;
  const int m2_0 = blockIdx.x * C1;
  const int total = M1 * C1;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int m1 = idx / C1, c = idx - m1 * C1;
    buf[m1 * ps + c] = seg[(size_t)m1 * M2 + m2_0 + c];
  }
  __syncthreads();
  smem_fft<V>(buf, a.plan1, C1, ps, 1, reinterpret_cast<const V *>(a.tw1),
              reinterpret_cast<const V *>(a.wsmall));
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int k1 = idx / C1, c = idx - k1 * C1;
    V v = buf[__ldg(a.perm1 + k1) * ps + c];
    const long long e = (long long)(m2_0 + c) * k1;
    v = cmul(v, cross_twiddle<V>(a, e));
    seg[(size_t)k1 * M2 + m2_0 + c] = v;
  }
}

// Pass 2: segment seg_lo + blockIdx.y, rows k1 in [blockIdx.x*C2, +C2): FFT of length
// M2 over m2 of row k1, giving X[k1 + M1*k2]; out[seg*M + k] = W_inv[k]*X[k]
// for k < M (pfft.c:653-660), the other M'-M bins are dropped.
template <typename R>
__global__ void __launch_bounds__(256) k_seg_rows_demod(SegArgs a)
{
  using V = typename cplx_of<R>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *buf = reinterpret_cast<V *>(smem_raw);
  const int C2 = a.C2, M1 = a.M1, M2 = a.M2;
  const int ps = C2 + 1;
  const V *seg = reinterpret_cast<const V *>(a.T) + (size_t)(a.seg_lo + blockIdx.y) * a.Mh;
  const int k1_0 = blockIdx.x * C2;
  const int total = M2 * C2;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int c = idx / M2, m2 = idx - c * M2;
    buf[m2 * ps + c] = seg[(size_t)(k1_0 + c) * M2 + m2];
  }
  __syncthreads();
  smem_fft<V>(buf, a.plan2, C2, ps, 1, reinterpret_cast<const V *>(a.tw2),
              reinterpret_cast<const V *>(a.wsmall));
  V *out = reinterpret_cast<V *>(a.out) + (size_t)(a.seg_lo + blockIdx.y) * a.M;
  const V *winv = reinterpret_cast<const V *>(a.winv);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int k2 = idx / C2, c = idx - k2 * C2;
    const long long k = (long long)(k1_0 + c) + (long long)M1 * k2;
    if (k < a.M) {
      const V x = buf[__ldg(a.perm2 + k2) * ps + c];
      out[k] = cmul(__ldg(winv + k), x);
    }
  }
}

// ------------------------------------------------------------ inverse --
// The inverse DFT through the forward pipeline: IDFT(X) = conj(DFT(conj X))/N.
// out[i] = conj(in[i]) * scale, 16 bytes per thread per step (two complex64
// values or one complex128), grid-stride.
template <typename R>
__global__ void k_conj_scale(const void *in, void *out, long long n, R scale)
{
  using V = typename cplx_of<R>::type;
  const V *x = reinterpret_cast<const V *>(in);
  V *y = reinterpret_cast<V *>(out);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const V v = x[i];
    y[i] = cmk<V>(v.x * scale, -v.y * scale);
  }
}

}  // namespace soi
