// stage1_fast.cuh -- filter-subsampling convolution fused with the S-point
// FFTs and the transposed store, with shared-memory staging.
//
// Same arithmetic as k_conv_sfft (parallel_filter_subsampling.cpp:134-287,
// :297-311, :316-395 and the all-to-all of pfft.c:441-583), organised for
// memory-level parallelism: the work of a tile (JT output groups x all S
// columns) is split into phases (polyphase branch b, chunk of AC taps).  For
// each phase the CTA copies the input rows d*t + b it needs and the matching
// filter slice into shared memory with cp.async, one phase ahead of the
// compute (double buffering), and the FMA loop reads only shared memory and
// registers.  The staging buffers are reused for the output tile once the
// convolution is done.
#pragma once

#include "async_copy.cuh"
#include "fft_reg.cuh"

namespace soi {

struct Conv2Args {
  const void *alpha;     // [M][S] complex
  void *T;               // [S][Mh] complex
  const void *filt;      // [d][atap][nmu][S] real (branch-major), zero beyond B taps
  const void *phase;     // [nmu][S] complex
  const void *twS;       // [S] complex
  const int *permS;      // [S]
  const void *wsmall;
  FftPlan planS;
  long long M, Mh, J;
  int S, d, atap, JT, pitch, AC;
  int buf_elems;         // complex elements per staging buffer (rows + filter, rounded)
  int seg_lo, seg_hi;    // segments sigma stored (all: 0, S)
  int *err;              // set to 1 when a staging wait gives up (bulk copies)
  int tma_rows = 0;      // the kernel's tensor map describes alpha (bulk staging)
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
  const unsigned int s = (unsigned int)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// acc += h * x (real h, complex x)
__device__ __forceinline__ void macc(float2 &acc, float h, float2 x) { acc = __ffma2_rn(make_float2(h, h), x, acc); }
__device__ __forceinline__ void macc(double2 &acc, double h, double2 x)
{
  acc.x = fma(h, x.x, acc.x);
  acc.y = fma(h, x.y, acc.y);
}

template <typename R, int NMU, int JR>
__global__ void __launch_bounds__(512, 1) k_conv_sfft_staged(Conv2Args a)
{
  using V = typename cplx_of<R>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int S = a.S;
  const int JT = a.JT;
  const int rows_tile = NMU * JT;
  V *buf0 = reinterpret_cast<V *>(smem_raw);
  V *buf1 = buf0 + a.buf_elems;
  V *tile = buf0;                                            // output tile aliases the staging
  V *twS = buf0 + 2 * (size_t)a.buf_elems;
  int *permS = reinterpret_cast<int *>(twS + S);
  const int tid = threadIdx.x;
  for (int i = tid; i < S; i += blockDim.x) {
    twS[i] = reinterpret_cast<const V *>(a.twS)[i];
    permS[i] = a.permS[i];
  }
  const int s = tid % S;
  const int jb = tid / S;
  const bool active = jb * JR < JT;
  const long long j0 = (long long)blockIdx.x * JT;
  const int d = a.d;
  const long long M = a.M;
  const int nch = (a.atap + a.AC - 1) / a.AC;
  const int nphase = d * nch;
  const V *alpha = reinterpret_cast<const V *>(a.alpha);
  const R *filt = reinterpret_cast<const R *>(a.filt);
  const int rowbytes = S * (int)sizeof(V);

  // copy phase p (branch b = p / nch, taps [a_lo, a_hi)) into dst
  auto issue = [&](int p, V *dst) {
    const int b = p / nch, a_lo = (p % nch) * a.AC;
    const int n_a = min(a.AC, a.atap - a_lo);
    const int nrows = JT + n_a - 1;
    const int cpr = rowbytes / 16;                           // 16-byte chunks per row
    const int nrow_chunks = nrows * cpr;
    for (int c = tid; c < nrow_chunks; c += blockDim.x) {
      const int t = c / cpr, off = c - t * cpr;
      long long r = (long long)d * (j0 + a_lo + t) + b;
      if (r >= M) r -= M;                                    // circular (ghost rows, .cpp:495-515)
      cp_async16(reinterpret_cast<char *>(dst) + (size_t)t * rowbytes + off * 16,
                 reinterpret_cast<const char *>(alpha + r * S) + off * 16);
    }
    R *fdst = reinterpret_cast<R *>(dst + (size_t)nrows * S);
    const char *fsrc = reinterpret_cast<const char *>(filt + ((size_t)(b * a.atap + a_lo) * NMU) * S);
    const int fchunks = (int)((size_t)n_a * NMU * S * sizeof(R) / 16);
    for (int c = tid; c < fchunks; c += blockDim.x)
      cp_async16(reinterpret_cast<char *>(fdst) + c * 16, fsrc + c * 16);
  };

  V acc[JR][NMU];
#pragma unroll
  for (int jj = 0; jj < JR; ++jj)
#pragma unroll
    for (int th = 0; th < NMU; ++th) acc[jj][th] = cmk<V>((R)0, (R)0);

  issue(0, buf0);
  cp_async_commit();
  for (int p = 0; p < nphase; ++p) {
    V *cur = (p & 1) ? buf1 : buf0;
    if (p + 1 < nphase) {
      issue(p + 1, (p & 1) ? buf0 : buf1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (active) {
      const int a_lo = (p % nch) * a.AC;
      const int n_a = min(a.AC, a.atap - a_lo);
      const int nrows = JT + n_a - 1;
      const V *rows = cur;                                   // rows[t][s] = x_b[j0 + a_lo + t]
      const R *fb = reinterpret_cast<const R *>(cur + (size_t)nrows * S);   // fb[u][theta][s]
      const int rb = jb * JR;
      V xw[JR];
#pragma unroll
      for (int jj = 0; jj < JR - 1; ++jj) xw[jj] = rows[(rb + jj) * S + s];
      const int nmain = n_a - n_a % JR;
      for (int u0 = 0; u0 < nmain; u0 += JR) {
#pragma unroll
        for (int u = 0; u < JR; ++u) {
          xw[(u + JR - 1) % JR] = rows[(rb + u0 + u + JR - 1) * S + s];
          R h[NMU];
#pragma unroll
          for (int th = 0; th < NMU; ++th) h[th] = fb[((u0 + u) * NMU + th) * S + s];
#pragma unroll
          for (int jj = 0; jj < JR; ++jj)
#pragma unroll
            for (int th = 0; th < NMU; ++th) macc(acc[jj][th], h[th], xw[(u + jj) % JR]);
        }
      }
#pragma unroll
      for (int u = 0; u < JR - 1; ++u) {
        if (u < n_a - nmain) {
          xw[(u + JR - 1) % JR] = rows[(rb + nmain + u + JR - 1) * S + s];
          R h[NMU];
#pragma unroll
          for (int th = 0; th < NMU; ++th) h[th] = fb[((nmain + u) * NMU + th) * S + s];
#pragma unroll
          for (int jj = 0; jj < JR; ++jj)
#pragma unroll
            for (int th = 0; th < NMU; ++th) macc(acc[jj][th], h[th], xw[(u + jj) % JR]);
        }
      }
    }
    __syncthreads();
  }

  // epilogue: G = phase * acc into the tile (aliases the staging buffers)
  if (active) {
    const V *ph = reinterpret_cast<const V *>(a.phase);
#pragma unroll
    for (int th = 0; th < NMU; ++th) {
      const V pz = __ldg(ph + th * S + s);
#pragma unroll
      for (int jj = 0; jj < JR; ++jj)
        tile[(size_t)((jb * JR + jj) * NMU + th) * a.pitch + s] = cmul(pz, acc[jj][th]);
    }
  }
  __syncthreads();
  smem_fft<V>(tile, a.planS, rows_tile, 1, a.pitch, twS, reinterpret_cast<const V *>(a.wsmall));
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


// Stores of the tile FFT's last stage: T[f][rho0 + col] (the transposed
// store of .cpp:391 / the all-to-all of pfft.c:554-578), consecutive threads
// on consecutive rows rho.
struct NoPrep {};

template <typename V> struct EmitTransposed {
  V *T; long long Mh, rho0; int lo, hi;   // segments f in [lo, hi) are stored
  bool all;                                // [lo, hi) covers every segment
  __device__ __forceinline__ NoPrep prepare(int, int) const { return NoPrep{}; }
  template <int RL> __device__ __forceinline__ void run(int col, int fbase, int fstep, V *v, NoPrep = NoPrep{}) const
  {
    const long long rho = rho0 + col;
    if (rho < Mh) {
      V *dst = T + (size_t)fbase * Mh + rho;
      if (all) {
#pragma unroll
        for (int k = 0; k < RL; ++k) dst[(size_t)k * fstep * Mh] = v[k];
      } else {
#pragma unroll
        for (int k = 0; k < RL; ++k) {
          const int f = fbase + fstep * k;
          if (f >= lo && f < hi) dst[(size_t)k * fstep * Mh] = v[k];
        }
      }
    }
  }
};

// Same kernel with the segment count S = R0*R1 and the block size NT known at
// compile time (NT = 256 runs two CTAs per SM, so one CTA's convolution
// overlaps the other's FFT and stores): shared
// addressing becomes immediate offsets, and the S-point FFT runs as two
// register-radix stages (RegDFT) whose last stage writes the transposed
// output straight to HBM.  Tile layout: row r, column s at
// r*PITCH + s + s/R1, PITCH odd.
//
// BULK: thread 0 stages each phase with one tensor copy (TMA) of the
// phase's JT + AC - 1 input rows -- a box of [rows][1 branch][S values] of
// the input viewed as [J][d][S] -- and one bulk copy of the filter slice,
// both completing on the buffer's mbarrier; all threads wait on the
// mbarrier's phase parity (bounded: a wait that gives up sets a.err and then
// drains).  A tile whose rows wrap around the input (the ghost rows of
// .cpp:495-515) takes its rows by one bulk copy per row from warp 0 instead.
// The buffers start on 128-byte boundaries (the tensor copy's destination
// rule), and the filter slice sits after JT + AC - 1 rows in every phase.
// Otherwise every thread issues 16-byte cp.async.
template <typename R, int NMU, int JR, int R0, int R1, int NT, bool BULK>
__global__ void __launch_bounds__(NT, 512 / NT) k_conv_sfft_tS(Conv2Args a, const __grid_constant__ CUtensorMap rmap)
{
  using V = typename cplx_of<R>::type;
  constexpr int S = R0 * R1;
  constexpr int PITCH = (S + S / R1) | 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int JT = a.JT;
  const int rows_tile = NMU * JT;
  // 128-byte aligned start (the host reserves the slack when BULK)
  unsigned char *smem_base = smem_raw;
  if (BULK) smem_base += (128u - (smem_u32(smem_raw) & 127u)) & 127u;
  V *buf0 = reinterpret_cast<V *>(smem_base);
  V *buf1 = buf0 + a.buf_elems;
  V *tile = buf0;
  V *twS = buf0 + 2 * (size_t)a.buf_elems;
  const int tid = threadIdx.x;
  for (int i = tid; i < S; i += blockDim.x) twS[i] = reinterpret_cast<const V *>(a.twS)[i];
  const int s = tid % S;
  const int jb = tid / S;
  const bool active = jb * JR < JT;
  const long long j0 = (long long)blockIdx.x * JT;
  const int d = a.d;
  const long long M = a.M;
  const int nch = (a.atap + a.AC - 1) / a.AC;
  const int nphase = d * nch;
  const V *alpha = reinterpret_cast<const V *>(a.alpha);
  const R *filt = reinterpret_cast<const R *>(a.filt);
  constexpr int CPR = S * (int)sizeof(V) / 16;                // 16-byte chunks per input row
  static_assert(NT % CPR == 0, "row chunks must tile the block");

  // copy phase p (branch b = p / nch, taps [a_lo, a_lo + n_a)) into dst:
  // input row t of the phase is x_b[j0 + a_lo + t] = alpha row d*(j0 + a_lo + t) + b,
  // read circularly (the ghost rows of .cpp:495-515); each thread steps its
  // source and destination pointers by NT/CPR rows
  constexpr size_t ROWB = (size_t)S * sizeof(V);
  const char *alpha_end = reinterpret_cast<const char *>(alpha) + (size_t)M * ROWB;
  auto issue = [&](int p, V *dst) {
    const int b = p / nch, a_lo = (p % nch) * a.AC;
    const int n_a = min(a.AC, a.atap - a_lo);
    const int nrows = JT + n_a - 1;
    const int off = tid % CPR;
    int t = tid / CPR;
    long long r = (long long)d * (j0 + a_lo + t) + b;
    if (r >= M) r -= M;
    const char *src = reinterpret_cast<const char *>(alpha) + (size_t)r * ROWB + off * 16;
    char *dp = reinterpret_cast<char *>(dst) + (size_t)t * ROWB + off * 16;
    const size_t dsrc = (size_t)d * (NT / CPR) * ROWB;
    for (; t < nrows; t += NT / CPR) {
      cp_async16(dp, src);
      dp += (NT / CPR) * ROWB;
      src += dsrc;
      if (src >= alpha_end) src -= (size_t)M * ROWB;          // the wrap happens at most once per tile
    }
    const char *fs = reinterpret_cast<const char *>(filt + ((size_t)(b * a.atap + a_lo) * NMU) * S) + tid * 16;
    char *fd = reinterpret_cast<char *>(dst + (size_t)nrows * S) + tid * 16;
    const int fchunks = n_a * NMU * S * (int)sizeof(R) / 16;
    for (int c = tid; c < fchunks; c += NT, fs += NT * 16, fd += NT * 16) cp_async16(fd, fs);
  };
  __shared__ unsigned long long s_mbar[2];
  // the same phase as bulk copies issued by warp 0 onto the buffer's mbarrier
  // rows of the box: JT + AC - 1 (the phase with fewer taps uses a prefix);
  // a tile takes the tensor copy when every phase's box ends inside [0, J)
  const int NR = JT + a.AC - 1;
  const bool tma_rows = a.tma_rows && j0 + (nch - 1) * a.AC + NR <= a.J;
  auto issue_bulk = [&](int p, V *dst, unsigned long long *bar) {
    if (tid >= 32) return;
    const int b = p / nch, a_lo = (p % nch) * a.AC;
    const int n_a = min(a.AC, a.atap - a_lo);
    const int nrows = JT + n_a - 1;
    const unsigned fbytes = (unsigned)(n_a * NMU * S * (int)sizeof(R));
    const R *fsrc = filt + ((size_t)(b * a.atap + a_lo) * NMU) * S;
    if (tma_rows) {
      if (tid == 0) {
        mbar_expect_tx(bar, (unsigned)(NR * ROWB) + fbytes);
        fence_proxy_async_smem();
        tma_load_3d(dst, &rmap, 0, b, (int)(j0 + a_lo), bar);
        bulk_g2s(dst + (size_t)NR * S, fsrc, fbytes, bar);
      }
      return;
    }
    if (tid == 0) mbar_expect_tx(bar, (unsigned)(nrows * ROWB) + fbytes);
    __syncwarp();
    fence_proxy_async_smem();
    for (int t = tid; t < nrows; t += 32) {
      long long r = (long long)d * (j0 + a_lo + t) + b;
      if (r >= M) r -= M;                                    // circular (ghost rows, .cpp:495-515)
      bulk_g2s(dst + (size_t)t * S, alpha + r * S, (unsigned)ROWB, bar);
    }
    if (tid == 31) bulk_g2s(dst + (size_t)NR * S, fsrc, fbytes, bar);
  };
  // phase p's data has arrived: buffer p & 1, used for the (p >> 1)-th time
  auto wait_bulk = [&](int p) {
    long long it = 0;
    while (!mbar_try_wait(&s_mbar[p & 1], (unsigned)((p >> 1) & 1))) {
      if (++it > kBulkWaitLimit) {
        // late copies: flag them, then wait for them to land (bounded, 16x
        // longer) so that none is still writing shared memory when the
        // buffer is refilled or the CTA leaves
        if (tid == 0) atomicExch(a.err, 1);
        long long drain = 0;
        while (!mbar_try_wait(&s_mbar[p & 1], (unsigned)((p >> 1) & 1)) && ++drain <= 16 * kBulkWaitLimit) {}
        break;
      }
    }
  };
  if (BULK) {
    if (tid == 0) {
      mbar_init(&s_mbar[0], 1);
      mbar_init(&s_mbar[1], 1);
      mbar_init_fence();
    }
    __syncthreads();
  }

  V acc[JR][NMU];
#pragma unroll
  for (int jj = 0; jj < JR; ++jj)
#pragma unroll
    for (int th = 0; th < NMU; ++th) acc[jj][th] = cmk<V>((R)0, (R)0);

  if (BULK) {
    issue_bulk(0, buf0, &s_mbar[0]);
  } else {
    issue(0, buf0);
    cp_async_commit();
  }
  for (int p = 0; p < nphase; ++p) {
    V *cur = (p & 1) ? buf1 : buf0;
    if (BULK) {
      if (p + 1 < nphase) issue_bulk(p + 1, (p & 1) ? buf0 : buf1, &s_mbar[(p + 1) & 1]);
      wait_bulk(p);
    } else if (p + 1 < nphase) {
      issue(p + 1, (p & 1) ? buf0 : buf1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    // cp.async: the barrier makes every thread's copies visible to all; bulk
    // staging needs none here, every thread has waited on the phase's
    // mbarrier, which makes the copy's bytes visible to it
    if (!BULK) __syncthreads();
    if (active) {
      const int a_lo = (p % nch) * a.AC;
      const int n_a = min(a.AC, a.atap - a_lo);
      const int nrows = JT + n_a - 1;
      const V *rows = cur + (size_t)(jb * JR) * S + s;        // rows[t*S] = x_b[j0 + a_lo + jb*JR + t]
      const R *fb = reinterpret_cast<const R *>(cur + (size_t)(BULK ? NR : nrows) * S) + s;   // fb[(u*NMU + th)*S]
      V xw[JR];
#pragma unroll
      for (int jj = 0; jj < JR - 1; ++jj) xw[jj] = rows[jj * S];
      const int nmain = n_a - n_a % JR;
      for (int u0 = 0; u0 < nmain; u0 += JR) {
        const V *rp = rows + (size_t)u0 * S;
        const R *fp = fb + (size_t)u0 * NMU * S;
#pragma unroll
        for (int u = 0; u < JR; ++u) {
          xw[(u + JR - 1) % JR] = rp[(u + JR - 1) * S];
          R h[NMU];
#pragma unroll
          for (int th = 0; th < NMU; ++th) h[th] = fp[(u * NMU + th) * S];
#pragma unroll
          for (int jj = 0; jj < JR; ++jj)
#pragma unroll
            for (int th = 0; th < NMU; ++th) macc(acc[jj][th], h[th], xw[(u + jj) % JR]);
        }
      }
      const V *rp = rows + (size_t)nmain * S;
      const R *fp = fb + (size_t)nmain * NMU * S;
#pragma unroll
      for (int u = 0; u < JR - 1; ++u) {
        if (u < n_a - nmain) {
          xw[(u + JR - 1) % JR] = rp[(u + JR - 1) * S];
          R h[NMU];
#pragma unroll
          for (int th = 0; th < NMU; ++th) h[th] = fp[(u * NMU + th) * S];
#pragma unroll
          for (int jj = 0; jj < JR; ++jj)
#pragma unroll
            for (int th = 0; th < NMU; ++th) macc(acc[jj][th], h[th], xw[(u + jj) % JR]);
        }
      }
    }
    __syncthreads();
  }
  if (active) {
    const V *ph = reinterpret_cast<const V *>(a.phase);
#pragma unroll
    for (int th = 0; th < NMU; ++th) {
      const V pz = __ldg(ph + th * S + s);
#pragma unroll
      for (int jj = 0; jj < JR; ++jj)
        tile[(size_t)((jb * JR + jj) * NMU + th) * PITCH + s + s / R1] = cmul(pz, acc[jj][th]);
    }
  }
  __syncthreads();
  EmitTransposed<V> e{ reinterpret_cast<V *>(a.T), a.Mh, (long long)NMU * j0, a.seg_lo, a.seg_hi,
                      a.seg_lo == 0 && a.seg_hi >= S };
  tile_fft_smem<V, R0, R1, 1>(tile, rows_tile, 1, PITCH, twS, e);
}

}  // namespace soi
