// fft_reg.cuh -- register-resident DFTs of compile-time size F <= 64 built
// from the radix-2/3/4/5/8 butterflies, with twiddles in constant memory.
//
// RegDFT<V, F>::run(v) transforms v[0..F) in place, natural order in and out,
// forward (exp(-2 pi i jk/F)).  F = A*Bq is split as a four-step in
// registers: A-point DFTs over the stride-Bq subsequences, twiddles
// w_F^(b*ka), Bq-point DFTs, then a compile-time permutation (register
// renaming, no data movement after unrolling).
#pragma once

#include "fft_device.cuh"

namespace soi {

// sizes with a twiddle table in constant memory, and their offsets
constexpr int kRegSizes[] = { 2, 3, 4, 5, 6, 8, 9, 10, 12, 15, 16, 20, 24, 30, 32, 40, 48, 60, 64 };
__host__ __device__ constexpr int reg_tw_offset(int F)
{
  // cumulative sizes of kRegSizes (a table lookup is not usable in device code)
  return F == 2 ? 0 : F == 3 ? 2 : F == 4 ? 5 : F == 5 ? 9 : F == 6 ? 14 : F == 8 ? 20 : F == 9 ? 28
       : F == 10 ? 37 : F == 12 ? 47 : F == 15 ? 59 : F == 16 ? 74 : F == 20 ? 90 : F == 24 ? 110
       : F == 30 ? 134 : F == 32 ? 164 : F == 40 ? 196 : F == 48 ? 236 : F == 60 ? 284 : F == 64 ? 344 : -1;
}
constexpr int kRegTwTotal = 408;

// w_F^m = exp(-2 pi i m/F) at c_regtw[reg_tw_offset(F) + m]; filled by the
// host (long double, rounded once) before the first launch.
__constant__ float2 c_regtw_f[kRegTwTotal];
__constant__ double2 c_regtw_d[kRegTwTotal];

template <typename V> __device__ __forceinline__ V regtw(int idx);
template <> __device__ __forceinline__ float2 regtw<float2>(int idx) { return c_regtw_f[idx]; }
template <> __device__ __forceinline__ double2 regtw<double2>(int idx) { return c_regtw_d[idx]; }

template <int F> struct RegSplit {
  // sizes with a direct butterfly are not split
  static constexpr int A = (F == 2 || F == 3 || F == 4 || F == 5 || F == 8) ? F
                         : (F % 8 == 0 && F > 8) ? 8
                         : (F % 4 == 0 && F > 4) ? 4
                         : (F % 2 == 0 && F > 2) ? 2
                         : (F % 5 == 0 && F > 5) ? 5
                         : (F % 3 == 0 && F > 3) ? 3 : F;
};

template <typename V, int F> struct RegDFT {
  static __device__ __forceinline__ void run(V *v)
  {
    constexpr int A = RegSplit<F>::A;
    constexpr int Bq = F / A;
    if constexpr (Bq == 1) {
      Bfly<V, F>::run(v, nullptr);
    } else {
      constexpr int off = reg_tw_offset(F);
      static_assert(off >= 0, "register DFT size without a twiddle table");
#pragma unroll
      for (int b = 0; b < Bq; ++b) {
        V u[A];
#pragma unroll
        for (int a = 0; a < A; ++a) u[a] = v[b + Bq * a];
        Bfly<V, A>::run(u, nullptr);
#pragma unroll
        for (int a = 0; a < A; ++a) v[b + Bq * a] = (b * a == 0) ? u[a] : cmul(u[a], regtw<V>(off + b * a));
      }
      // for each ka the Bq values v[b + Bq*ka] are contiguous: transform them
#pragma unroll
      for (int a = 0; a < A; ++a) RegDFT<V, Bq>::run(v + Bq * a);
      // v[Bq*ka + kb] = X[ka + A*kb]
      V t[F];
#pragma unroll
      for (int ka = 0; ka < A; ++ka)
#pragma unroll
        for (int kb = 0; kb < Bq; ++kb) t[ka + A * kb] = v[Bq * ka + kb];
#pragma unroll
      for (int i = 0; i < F; ++i) v[i] = t[i];
    }
  }
};

// In-place tile FFT on a shared-memory tile already holding the input (the
// caller prefetched it with cp.async).  Radices R0, R1, R2 (R2 = 1: two
// stages).  Shared index of (col, pos): (pos + pos/RL)*PP + col*PC with RL the
// last radix (one pad element per last-stage group).  The last stage hands each
// thread RL outputs of one column in frequency order f = fbase + (L/RL)*k to
// `emit`, which loads its epilogue factors before storing.
template <typename V, int R0, int R1, int R2, class Emit>
__device__ __forceinline__ void tile_fft_smem(V *sm, int C, int PP, int PC, const V *__restrict__ tw,
                                              const Emit &emit)
{
  constexpr int RL = (R2 > 1) ? R2 : R1;
  constexpr int L = R0 * R1 * R2;
  constexpr int span0 = L / R0;
  auto sidx = [&](int col, int pos) { return (pos + pos / RL) * PP + col * PC; };
  // item q = i*C + col; (col, i) advance by the block size without dividing
  const int nt = blockDim.x, dcol = nt % C, di = nt / C;
  {
    const int n = C * span0;
    int col = threadIdx.x % C, i = threadIdx.x / C;
    // the R0 values of a butterfly sit at one base plus multiples of the
    // shared distance of span0 positions (span0 is a whole number of pad groups)
    static_assert(span0 % RL == 0, "first-stage stride is a whole number of pad groups");
    const int D0 = (span0 + span0 / RL) * PP;
    for (int q = threadIdx.x; q < n; q += nt, col += dcol, i += di) {
      if (col >= C) { col -= C; ++i; }
      V *p = sm + sidx(col, i);
      V v[R0];
#pragma unroll
      for (int r = 0; r < R0; ++r) v[r] = p[r * D0];
      RegDFT<V, R0>::run(v);
      p[0] = v[0];
#pragma unroll
      for (int k = 1; k < R0; ++k) p[k * D0] = cmul(v[k], tw[i * k]);     // tw[0] = 1 exactly
    }
  }
  __syncthreads();
  if constexpr (R2 > 1) {
    constexpr int span1 = span0 / R1;
    const int n = C * (L / R1);
    int col = threadIdx.x % C, t = threadIdx.x / C;
    for (int q = threadIdx.x; q < n; q += nt, col += dcol, t += di) {
      if (col >= C) { col -= C; ++t; }
      const int blk = t / span1, i = t - blk * span1;
      const int base = blk * span0 + i;
      V v[R1];
#pragma unroll
      for (int r = 0; r < R1; ++r) v[r] = sm[sidx(col, base + r * span1)];
      RegDFT<V, R1>::run(v);
#pragma unroll
      for (int k = 0; k < R1; ++k) sm[sidx(col, base + k * span1)] = (k && i) ? cmul(v[k], tw[i * k * R0]) : v[k];
    }
    __syncthreads();
  }
  {
    const int n = C * (L / RL);
    int col = threadIdx.x % C, blk = threadIdx.x / C;
    for (int q = threadIdx.x; q < n; q += nt, col += dcol, blk += di) {
      if (col >= C) { col -= C; ++blk; }
      const V *p = sm + blk * (RL + 1) * PP + col * PC;
      V v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) v[r] = p[r * PP];
      RegDFT<V, RL>::run(v);
      int fbase;
      if constexpr (R2 > 1) fbase = (blk / R1) + R0 * (blk % R1);
      else fbase = blk;
      emit.template run<RL>(col, fbase, L / RL, v);
    }
  }
}

}  // namespace soi

namespace soi {

// tile_fft_smem with the tile geometry known at compile time: C columns,
// shared index (pos + pos/RL)*PP + col*PC, NT threads.  Every register radix
// reads and writes its R values at compile-time offsets from one base address
// (the positions of a butterfly never straddle a pad differently), and the
// twiddle of the i = 0 butterflies is tw[0] = 1 exactly, so no lane takes a
// separate path.
template <typename V, int R0, int R1, int R2, int C, int PP, int PC, int NT, class Emit>
__device__ __forceinline__ void tile_fft_ct(V *sm, const V *__restrict__ tw, const Emit &emit)
{
  constexpr int RL = (R2 > 1) ? R2 : R1;
  constexpr int L = R0 * R1 * R2;
  constexpr int span0 = L / R0;
  static_assert(span0 % RL == 0, "first-stage stride is a whole number of pad groups");
  constexpr int D0 = (span0 + span0 / RL) * PP;             // shared distance of span0 positions
  constexpr int DL = (RL + 1) * PP;                         // shared distance of RL positions
  {
    constexpr int n = C * span0;
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int col = q % C, i = q / C;
      V *p = sm + (i + i / RL) * PP + col * PC;
      V v[R0];
#pragma unroll
      for (int r = 0; r < R0; ++r) v[r] = p[r * D0];
      RegDFT<V, R0>::run(v);
      p[0] = v[0];
#pragma unroll
      for (int k = 1; k < R0; ++k) p[k * D0] = cmul(v[k], __ldg(tw + (k - 1) * span0 + i));
    }
  }
  __syncthreads();
  if constexpr (R2 > 1) {
    constexpr int span1 = span0 / R1;                       // = RL
    constexpr int n = C * (L / R1);
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int col = q % C, t = q / C;
      const int blk = t / span1, i = t - blk * span1;
      V *p = sm + (blk * span0 + blk * (span0 / RL) + i) * PP + col * PC;
      V v[R1];
#pragma unroll
      for (int r = 0; r < R1; ++r) v[r] = p[r * DL];
      RegDFT<V, R1>::run(v);
      p[0] = v[0];
#pragma unroll
      for (int k = 1; k < R1; ++k) p[k * DL] = cmul(v[k], __ldg(tw + (R0 - 1) * span0 + (k - 1) * span1 + i));
    }
    __syncthreads();
  }
  {
    constexpr int n = C * (L / RL);
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int col = q % C, blk = q / C;
      const V *p = sm + blk * DL + col * PC;
      int fbase;
      if constexpr (R2 > 1) fbase = (blk / R1) + R0 * (blk % R1);
      else fbase = blk;
      // the epilogue's own loads go out before the last radix's arithmetic
      const auto pre = emit.prepare(col, fbase, blk);
      V v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) v[r] = p[r * PP];
      RegDFT<V, RL>::run(v);
      emit.template run<RL>(col, fbase, L / RL, v, pre, blk);
    }
  }
}

// The same tile FFT on a dense tile of C-element rows (32 bytes each) as a
// tensor copy lays it out without swizzling: element (m, col) at m*C + col.
// Rows visited: first stage i + r*span0, middle stage blk*span0 + i + r*RL,
// last stage blk*RL + r, as in tile_fft_ct.  A half-warp of the first and
// middle stages reads 4 consecutive rows x C columns (conflict-free); the last
// stage's half-warp (4 butterflies 16 rows apart) reads in a per-butterfly
// row order that keeps it conflict-free too.
template <typename V, int C>
__device__ __forceinline__ V *dense_at(V *base, int m, int col)
{
  return base + m * C + col;
}

template <typename V, int R0, int R1, int R2, int C, int NT, class Emit>
__device__ __forceinline__ void tile_fft_ct_dense(V *sm, const V *__restrict__ tw, const Emit &emit)
{
  static_assert(C * sizeof(V) == 32, "rows of 32 bytes");
  constexpr int RL = (R2 > 1) ? R2 : R1;
  constexpr int L = R0 * R1 * R2;
  constexpr int span0 = L / R0;
  {
    constexpr int n = C * span0;
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int col = q % C, i = q / C;
      V v[R0];
#pragma unroll
      for (int r = 0; r < R0; ++r) v[r] = *dense_at<V, C>(sm, i + r * span0, col);
      RegDFT<V, R0>::run(v);
      *dense_at<V, C>(sm, i, col) = v[0];
#pragma unroll
      for (int k = 1; k < R0; ++k) *dense_at<V, C>(sm, i + k * span0, col) = cmul(v[k], __ldg(tw + (k - 1) * span0 + i));
    }
  }
  __syncthreads();
  if constexpr (R2 > 1) {
    constexpr int span1 = span0 / R1;                       // = RL
    constexpr int n = C * (L / R1);
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int col = q % C, t = q / C;
      const int blk = t / span1, i = t - blk * span1;
      const int m0 = blk * span0 + i;
      V v[R1];
#pragma unroll
      for (int r = 0; r < R1; ++r) v[r] = *dense_at<V, C>(sm, m0 + r * RL, col);
      RegDFT<V, R1>::run(v);
      *dense_at<V, C>(sm, m0, col) = v[0];
#pragma unroll
      for (int k = 1; k < R1; ++k)
        *dense_at<V, C>(sm, m0 + k * RL, col) = cmul(v[k], __ldg(tw + (R0 - 1) * span0 + (k - 1) * span1 + i));
    }
    __syncthreads();
  }
  {
    constexpr int n = C * (L / RL);
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int col = q % C, blk = q / C;
      int fbase;
      if constexpr (R2 > 1) fbase = (blk / R1) + R0 * (blk % R1);
      else fbase = blk;
      const auto pre = emit.prepare(col, fbase, blk);
      // a half-warp holds 4 butterflies 16 rows apart, whose rows share banks:
      // each reads its rows in the order r ^ (blk & 3), which puts the four
      // on different banks, and two conditional swaps restore the order
      const int x = blk & 3;
      V u[RL], v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) u[r] = *dense_at<V, C>(sm, blk * RL + (r ^ x), col);
#pragma unroll
      for (int r = 0; r < RL; ++r) v[r] = (x & 1) ? u[r ^ 1] : u[r];
#pragma unroll
      for (int r = 0; r < RL; ++r) u[r] = (x & 2) ? v[r ^ 2] : v[r];
      RegDFT<V, RL>::run(u);
      emit.template run<RL>(col, fbase, L / RL, u, pre, blk);
    }
  }
}

// The tile FFT on C dense rows of L elements at row pitch PR, as bulk copies
// lay whole rows out: element (col, pos) at col*PR + pos, no pad inside a row.
// With 8-byte elements and PR = 4 (mod 16), a half-warp of the first and
// middle stages (4 columns x 4 consecutive butterflies) falls on distinct
// banks; the last stage's half-warp (4 columns x 4 butterflies RL positions
// apart) reads its positions in the order r ^ (blk & 3), which keeps it on
// distinct banks too, and two conditional swaps restore the order.  Same
// stages, twiddles and epilogue as tile_fft_ct.
template <typename V, int R0, int R1, int R2, int C, int PR, int NT, class Emit>
__device__ __forceinline__ void tile_fft_rows(V *sm, const V *__restrict__ tw, const Emit &emit)
{
  constexpr int RL = (R2 > 1) ? R2 : R1;
  constexpr int L = R0 * R1 * R2;
  constexpr int span0 = L / R0;
  static_assert(RL % 4 == 0, "the last stage's read order needs RL a multiple of 4");
  {
    constexpr int n = C * span0;
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int col = q % C, i = q / C;
      V *p = sm + col * PR + i;
      V v[R0];
#pragma unroll
      for (int r = 0; r < R0; ++r) v[r] = p[r * span0];
      RegDFT<V, R0>::run(v);
      p[0] = v[0];
#pragma unroll
      for (int k = 1; k < R0; ++k) p[k * span0] = cmul(v[k], __ldg(tw + (k - 1) * span0 + i));
    }
  }
  __syncthreads();
  if constexpr (R2 > 1) {
    constexpr int span1 = span0 / R1;                       // = RL
    constexpr int n = C * (L / R1);
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int col = q % C, t = q / C;
      const int blk = t / span1, i = t - blk * span1;
      V *p = sm + col * PR + blk * span0 + i;
      V v[R1];
#pragma unroll
      for (int r = 0; r < R1; ++r) v[r] = p[r * RL];
      RegDFT<V, R1>::run(v);
      p[0] = v[0];
#pragma unroll
      for (int k = 1; k < R1; ++k) p[k * RL] = cmul(v[k], __ldg(tw + (R0 - 1) * span0 + (k - 1) * span1 + i));
    }
    __syncthreads();
  }
  {
    constexpr int n = C * (L / RL);
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int col = q % C, blk = q / C;
      const V *p = sm + col * PR + blk * RL;
      int fbase;
      if constexpr (R2 > 1) fbase = (blk / R1) + R0 * (blk % R1);
      else fbase = blk;
      const auto pre = emit.prepare(col, fbase, blk);
      const int x = blk & 3;
      V u[RL], v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) u[r] = p[r ^ x];
#pragma unroll
      for (int r = 0; r < RL; ++r) v[r] = (x & 1) ? u[r ^ 1] : u[r];
#pragma unroll
      for (int r = 0; r < RL; ++r) u[r] = (x & 2) ? v[r ^ 2] : v[r];
      RegDFT<V, RL>::run(u);
      emit.template run<RL>(col, fbase, L / RL, u, pre, blk);
    }
  }
}

// tile_fft_rows for FP32 tasks of C = 4 rows with each thread on a pair of
// rows (2*cp, 2*cp + 1): every twiddle, and in the epilogue every
// ph(M1*k2) and amplitude pair, is loaded once for both rows, and the two
// outputs of a position leave as one 16-byte store.  First and middle stages:
// a half-warp is 2 pairs x 8 consecutive butterflies, rows 2*cp at 8-byte
// slots 0 / 8 of a 128-byte group (PR = 4 mod 16) and rows 2*cp + 1 at 4 / 12,
// so both loads of a position are conflict-free.  Last stage: 16-byte loads
// of position pairs (2m, 2m + 1) in the pair order m ^ (blk & 3) (a quarter-
// warp, 2 row pairs x 4 butterflies, on 8 distinct 16-byte slots), two
// conditional swaps restore the order.  Same arithmetic, in the same order,
// as tile_fft_rows.
template <typename V, int R0, int R1, int R2, int PR, int NT, class Emit>
__device__ __forceinline__ void tile_fft_rows2(V *sm, const V *__restrict__ tw, const Emit &emit)
{
  constexpr int CH = 2;                                      // row pairs per task
  constexpr int RL = (R2 > 1) ? R2 : R1;
  constexpr int L = R0 * R1 * R2;
  constexpr int span0 = L / R0;
  constexpr int NP = RL / 2;                                 // position pairs of a last-stage butterfly
  static_assert(sizeof(V) == 8 && RL % 8 == 0 && PR % 16 == 4, "FP32 rows, pair order over 4 pairs");
  {
    constexpr int n = CH * span0;
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int cp = q % CH, i = q / CH;
      V *p0 = sm + 2 * cp * PR + i;
      V *p1 = p0 + PR;
      V v[R0], w[R0];
#pragma unroll
      for (int r = 0; r < R0; ++r) { v[r] = p0[r * span0]; w[r] = p1[r * span0]; }
      RegDFT<V, R0>::run(v);
      RegDFT<V, R0>::run(w);
      p0[0] = v[0];
      p1[0] = w[0];
#pragma unroll
      for (int k = 1; k < R0; ++k) {
        const V t = __ldg(tw + (k - 1) * span0 + i);
        p0[k * span0] = cmul(v[k], t);
        p1[k * span0] = cmul(w[k], t);
      }
    }
  }
  __syncthreads();
  if constexpr (R2 > 1) {
    constexpr int span1 = span0 / R1;                       // = RL
    constexpr int n = CH * (L / R1);
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int cp = q % CH, t = q / CH;
      const int blk = t / span1, i = t - blk * span1;
      V *p0 = sm + 2 * cp * PR + blk * span0 + i;
      V *p1 = p0 + PR;
      V v[R1], w[R1];
#pragma unroll
      for (int r = 0; r < R1; ++r) { v[r] = p0[r * RL]; w[r] = p1[r * RL]; }
      RegDFT<V, R1>::run(v);
      RegDFT<V, R1>::run(w);
      p0[0] = v[0];
      p1[0] = w[0];
#pragma unroll
      for (int k = 1; k < R1; ++k) {
        const V t = __ldg(tw + (R0 - 1) * span0 + (k - 1) * span1 + i);
        p0[k * RL] = cmul(v[k], t);
        p1[k * RL] = cmul(w[k], t);
      }
    }
    __syncthreads();
  }
  {
    constexpr int n = CH * (L / RL);
#pragma unroll 1
    for (int q = threadIdx.x; q < n; q += NT) {
      const int cp = q % CH, blk = q / CH;
      const float4 *p0 = reinterpret_cast<const float4 *>(sm + 2 * cp * PR + blk * RL);
      const float4 *p1 = reinterpret_cast<const float4 *>(sm + (2 * cp + 1) * PR + blk * RL);
      int fbase;
      if constexpr (R2 > 1) fbase = (blk / R1) + R0 * (blk % R1);
      else fbase = blk;
      const int x = blk & 3;
      float4 a[NP], b[NP], c[NP], d[NP];
#pragma unroll
      for (int m = 0; m < NP; ++m) { a[m] = p0[m ^ x]; c[m] = p1[m ^ x]; }
#pragma unroll
      for (int m = 0; m < NP; ++m) { b[m] = (x & 1) ? a[m ^ 1] : a[m]; d[m] = (x & 1) ? c[m ^ 1] : c[m]; }
#pragma unroll
      for (int m = 0; m < NP; ++m) { a[m] = (x & 2) ? b[m ^ 2] : b[m]; c[m] = (x & 2) ? d[m ^ 2] : d[m]; }
      V v[RL], w[RL];
#pragma unroll
      for (int m = 0; m < NP; ++m) {
        v[2 * m] = cmk<V>(a[m].x, a[m].y);
        v[2 * m + 1] = cmk<V>(a[m].z, a[m].w);
        w[2 * m] = cmk<V>(c[m].x, c[m].y);
        w[2 * m + 1] = cmk<V>(c[m].z, c[m].w);
      }
      RegDFT<V, RL>::run(v);
      RegDFT<V, RL>::run(w);
      emit.template run2<RL>(cp, fbase, L / RL, v, w, blk);
    }
  }
}

}  // namespace soi
