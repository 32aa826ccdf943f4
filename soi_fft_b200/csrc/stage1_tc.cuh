// stage1_tc.cuh -- the split-precision filter-subsampling convolution on the
// 5th-generation tensor cores (tcgen05, accumulators in tensor memory), fused
// with the S-point FFTs and the transposed store like k_conv_sfft_tS.
//
// The convolution of parallel_filter_subsampling.cpp:134-287 for one column s
// and a tile of JT output groups j is a product of a Hankel matrix of the
// column's inputs with the column's filter:
//
//   G[j][theta][s] = phase[theta][s] * sum_q x_s[d*j + q] * F[q][theta][s],
//
// q = 0 .. KP-1 (KP = taps rounded up to a multiple of 8, zero beyond B).
// With d = 4 the rows of X_s[j][q] = x_s[4j + q] are 4 elements = 16 bytes
// apart, which is exactly the row pitch of a K-major core matrix without
// swizzle: a shared-memory descriptor with LBO (next 4 taps) and SBO (next 8
// rows) describes the Hankel matrix without materialising it.
//
// 3xTF32: x = x_hi + x_lo and F = F_hi + F_lo, each term rounded to TF32.
// The A operand's 128 rows are (j, t, c) for 32 output groups, t in {hi, lo}
// and c in {re, im}; the B operand's 16 rows are (theta, t') for t' in {hi, lo}
// (10 used).  One MMA chain of KP/8 instructions (M = 128, N = 16, K = 8)
// yields every product x_t * F_t'; the epilogue adds the four (the lo*lo term
// is free) and pairs re with im.  Shared-memory layout of one column's A
// operand: 16-byte chunk 4*jj + 2*t + c holds x_{t,c}[4*jj .. 4*jj + 3]
// (tile-local rows), so row m = 4*jj + 2*t + c of K block a is chunk m + 4a.
//
// Warp-specialised pipeline over column pairs, on mbarriers (no block-wide
// barrier until the FFT):
//   thread 511: prefetches the tile's input rows into L2, then, as soon as a
//     shared-memory stage is free, starts a bulk copy (TMA engine) of the
//     pair's two B operands onto the stage's "bfull" barrier;
//   converter warps 8-11: hold the pair's inputs in registers (loaded two
//     pairs ahead), split them into the A chunks (TF32 hi/lo) once the stage
//     is free, and arrive on the stage's "full" barrier;
//   warps 4-6, one thread each: wait for a full stage and a free TMEM slot,
//     issue the MMAs of one third of the taps for both columns (into their
//     own accumulators), and commit them to the stage's "empty" barrier and
//     the slot's "done" barrier;
//   warps 0-3 and 12, 13, 14, 7 (TMEM lane quadrants 0-3, one column of the
//     pair each): wait for a done slot, read the accumulators (tcgen05.ld),
//     add the split products and the K parts, multiply by the phase, write
//     the FFT tile and free the slot.
// Every wait is bounded; one that gives up sets the error flag, every role
// leaves its loop, and the CTA drains its MMAs and copies before it returns.
//
// Measured (N = 2^29, S = 128): 14.3 ms against 5.78 ms for the packed-FMA
// kernel, with the tensor pipe ~8 % active.  The 175 KB output tile of the
// fused S-point FFT leaves room for three 15.5 KB stages only, and an
// M = 128, N = 16 MMA carries 5 useful outputs per A row (depthwise filter:
// no operand is shared between columns), so the pipeline waits on its
// operand refills rather than on the tensor cores.  Kept behind
// SOI_STAGE1_TC=1; the packed-FMA kernel is the default.
#pragma once

#include "async_copy.cuh"
#include "fft_reg.cuh"
#include "stage1_fast.cuh"

namespace soi {

__device__ __forceinline__ float tf32_rna(float x)
{
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// K-major, no swizzle: 8-row core matrices of 16-byte rows; lbo = byte
// distance of K-adjacent core matrices, sbo = of 8-row groups
__device__ __forceinline__ unsigned long long umma_desc(unsigned saddr, unsigned lbo, unsigned sbo)
{
  return (unsigned long long)((saddr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);   // version 1 (sm_100)
}

__device__ __forceinline__ void umma_tf32(unsigned dtmem, unsigned long long ad, unsigned long long bd, unsigned idesc,
                                          unsigned acc)
{
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
               " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}"
               ::"r"(dtmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u) : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned long long *bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(unsigned taddr, float *v)
{
  unsigned r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
               "%14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Geometry of the tensor-core stage 1: S = R0*R1 columns, JT = 32 output
// groups per tile (M = 128 rows of (j, t, c)), KP taps, column pairs in NST
// shared-memory stages and NSL TMEM slots.
template <int R0, int R1, int KP>
struct TcGeom {
  static constexpr int S = R0 * R1, NMU = 5, D = 4, JT = 32, NT = 512;
  static constexpr int PITCH = (S + S / R1) | 1;
  static constexpr int NA = KP / 4;                        // K blocks of 4 taps (= polyphase taps a)
  static constexpr int NJJ = JT + NA - 1;                  // input row quads a tile reads
  static constexpr int NP = S / 2;                         // column pairs
  static constexpr int NST = 3, NSL = 4;                   // shared-memory stages, TMEM slots (pairs)
  static constexpr int TILE = NMU * JT * PITCH * 8;        // output tile (float2)
  static constexpr int ACOL = 64 * NJJ;                    // one column's A chunks
  static constexpr int ASTR = (ACOL + 127) / 128 * 128;    // their 128-byte aligned stride
  static constexpr int BCOL = 64 * KP;                     // one column's B operand: 16 rows x KP taps
  // stage layout: [A of the pair's second column | A of its first column |
  // B of both]; the second column's A region starts the stage (128-byte
  // aligned, as a tensor copy's shared destination must be) and first holds
  // the pair's raw input rows
  static constexpr int OFF_B = 2 * ASTR;
  static constexpr int STAGE = (OFF_B + 2 * BCOL + 127) / 128 * 128;
  static constexpr int OFF_ST = (TILE + 127) / 128 * 128;
  static constexpr int OFF_TW = OFF_ST + NST * STAGE + 128;   // 128 bytes of slack: the stages are
                                                              // aligned at run time
  static constexpr int SMEM = OFF_TW + S * 8;
  // K split into KS parts with their own accumulators (summed by the
  // epilogue): consecutive MMAs then go to different accumulators, so the
  // tensor pipe does not wait for one MMA's result before the next starts
  static constexpr int KS = (KP / 8) % 3 == 0 ? 3 : 1;
  static constexpr int SLOTW = 2 * KS * 16;                // TMEM columns of one pair
  static constexpr int TMEM_COLS = NSL * SLOTW <= 32 ? 32 : NSL * SLOTW <= 64 ? 64 : NSL * SLOTW <= 128 ? 128
                                   : NSL * SLOTW <= 256 ? 256 : 512;
  static constexpr int NPROD = 2 * NJJ;                    // producer threads that write A chunks
  // instruction descriptor: F32 accumulate, TF32 A and B, both K-major, N = 16, M = 128
  static constexpr unsigned IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);
  static_assert(KP % 8 == 0, "whole MMAs of K = 8");
  static_assert(S % 4 == 0 && NP >= NSL, "whole column pairs, in twos");
  static_assert(ACOL % 16 == 0 && BCOL % 16 == 0 && STAGE % 128 == 0, "aligned operands and stages");
  static_assert(4 * NJJ * 16 == ACOL, "the raw rows fill the second column's A region");
  static_assert(SMEM <= 232448, "shared memory");
  static_assert(NPROD < 256, "producer threads (warps 8-15, the last one starts the B copies)");
  static_assert(NSL * SLOTW <= 512, "TMEM allocation");
};

template <int R0, int R1, int KP>
__global__ void __launch_bounds__(512, 1) k_conv_sfft_tc(Conv2Args a, const float *__restrict__ btab)
{
  using Gm = TcGeom<R0, R1, KP>;
  using V = float2;
  constexpr int S = Gm::S, NMU = Gm::NMU, JT = Gm::JT, NT = Gm::NT, PITCH = Gm::PITCH, NP = Gm::NP;
  constexpr int NST = Gm::NST, NSL = Gm::NSL;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // full[NST] (A chunks written), bfull[NST] (B copies landed), empty[NST],
  // done[NSL], freed[NSL], fin
  __shared__ __align__(8) unsigned long long s_bar[3 * NST + 2 * NSL + 1];
  __shared__ unsigned s_tmem;
  __shared__ volatile int s_bad;
  unsigned long long *full = s_bar, *bfull = s_bar + NST, *empty = s_bar + 2 * NST, *done = s_bar + 3 * NST;
  unsigned long long *freed = done + NSL;
  unsigned long long *fin = freed + NSL;
  V *tile = reinterpret_cast<V *>(smem_raw);
  V *twS = reinterpret_cast<V *>(smem_raw + Gm::OFF_TW);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long j0 = (long long)blockIdx.x * JT;
  const long long M = a.M;
  const V *alpha = reinterpret_cast<const V *>(a.alpha);
  const V *phase = reinterpret_cast<const V *>(a.phase);

  for (int i = tid; i < S; i += NT) twS[i] = reinterpret_cast<const V *>(a.twS)[i];
  if (tid == 0) {
    for (int k = 0; k < NST; ++k) {
      mbar_init(&full[k], Gm::NPROD);                        // the A writers
      mbar_init(&bfull[k], 1);                               // the B copy's expect_tx (+ its bytes)
      mbar_init(&empty[k], Gm::KS);                          // one commit per MMA-issuing thread
    }
    for (int k = 0; k < NSL; ++k) {
      mbar_init(&done[k], Gm::KS);                           // one commit per MMA-issuing thread
      mbar_init(&freed[k], 8);                               // the eight epilogue warps
    }
    mbar_init(fin, Gm::KS);
    mbar_init_fence();
    s_bad = 0;
  }
  if (warp == 4) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"((unsigned)Gm::TMEM_COLS) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = s_tmem;

  // bounded, warp-uniform wait for the phase of parity `par` of barrier b;
  // false when it gave up (or another role did)
  auto wait_bar = [&](unsigned long long *b, unsigned par) {
    long long it = 0;
    while (!__all_sync(0xffffffffu, mbar_try_wait(b, par))) {
      if (s_bad) return false;
      if (++it > kBulkWaitLimit) {
        if (lane == 0) {
          atomicExch(a.err, 1);
          s_bad = 1;
        }
        return false;
      }
    }
    return true;
  };
  // the stages start on a 128-byte boundary of the shared window (a tensor
  // copy's destination must), whatever the dynamic region's own alignment
  unsigned char *stbase = smem_raw + Gm::OFF_ST;
  stbase += (128u - (smem_u32(stbase) & 127u)) & 127u;
  auto stage_ptr = [&](int k) { return stbase + k * Gm::STAGE; };

  int nbcopy[NST] = {};                                      // stage fills started per stage (thread 511)
  // the tile's input rows 4*j0 .. 4*j0 + 4*NJJ - 1 wrap past M only in the
  // last tile; that tile's converters read global memory themselves
  const bool wrap = 4 * j0 + 4 * Gm::NJJ > M;
  if (warp < 4 || warp == 7 || (warp >= 12 && warp < 15)) {
    // ---- epilogue: warps 0-3 the pair's first column, warps 12, 13, 14, 7 its
    // second; TMEM lane quadrant = warp % 4, lane -> row m = 32*qd + lane = (jj, t, c)
    const int qd = warp & 3;
    const int c = warp < 4 ? 0 : 1;
    for (int p = 0; p < NP; ++p) {
      const int sl = p % NSL;
      const int s = 2 * p + c;
      V pz[NMU];                                             // the column's phases, loaded before the wait
#pragma unroll
      for (int th = 0; th < NMU; ++th) pz[th] = __ldg(phase + th * S + s);
      if (!wait_bar(&done[sl], (unsigned)((p / NSL) & 1))) break;
      tc_fence_after();
      {
        float v[16];
        tmem_ld16(tmem + ((unsigned)(32 * qd) << 16) + (unsigned)(sl * Gm::SLOTW + c * Gm::KS * 16), v);
#pragma unroll
        for (int q = 1; q < Gm::KS; ++q) {                   // the other K parts' accumulators
          float vq[16];
          tmem_ld16(tmem + ((unsigned)(32 * qd) << 16) + (unsigned)(sl * Gm::SLOTW + (c * Gm::KS + q) * 16), vq);
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] += vq[i];
        }
        float u[NMU], w[NMU];
#pragma unroll
        for (int th = 0; th < NMU; ++th) {
          u[th] = v[th] + v[th + NMU];                       // x_t * (F_hi + F_lo)
          u[th] += __shfl_xor_sync(0xffffffffu, u[th], 2);   // + the other t
        }
#pragma unroll
        for (int th = 0; th < NMU; ++th) w[th] = __shfl_xor_sync(0xffffffffu, u[th], 1);   // the other c
        if ((lane & 3) == 0) {
          const int jr = 8 * qd + (lane >> 2);
#pragma unroll
          for (int th = 0; th < NMU; ++th)
            tile[(size_t)(jr * NMU + th) * PITCH + s + s / R1] = cmul(pz[th], make_float2(u[th], w[th]));
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&freed[sl]);
    }
  } else if (warp >= 4 && warp < 4 + Gm::KS) {
    // ---- MMA issue: lane 0 of warp 4 + q issues the MMAs of K part q of both
    // columns (KS threads issue side by side; each commits its own MMAs)
    const int q = warp - 4;
    if (lane == 0) {
      for (int p = 0; p < NP; ++p) {
        const int k = p % NST, sl = p % NSL;
        bool ok = true;
        {
          long long it = 0;
          while (!mbar_try_wait(&full[k], (unsigned)((p / NST) & 1))) {
            if (s_bad || ++it > kBulkWaitLimit) { ok = false; break; }
          }
          it = 0;
          while (ok && !mbar_try_wait(&bfull[k], (unsigned)((p / NST) & 1))) {
            if (s_bad || ++it > kBulkWaitLimit) { ok = false; break; }
          }
          if (ok && p >= NSL) {
            it = 0;
            while (!mbar_try_wait(&freed[sl], (unsigned)((p / NSL - 1) & 1))) {
              if (s_bad || ++it > kBulkWaitLimit) { ok = false; break; }
            }
          }
        }
        if (!ok) {
          atomicExch(a.err, 1);
          s_bad = 1;
          break;
        }
        tc_fence_after();
        const unsigned sbase = smem_u32(stage_ptr(k)), bbase = sbase + Gm::OFF_B;
        // descriptors of K step 0 of each column; step kk adds kk*128 (A) and
        // kk*256 (B) bytes to the start address field (bits 0-13, in 16-byte
        // units, no carry out: shared addresses stay below 256 KB)
        const unsigned long long a0[2] = { umma_desc(sbase + Gm::ASTR, 64, 128), umma_desc(sbase, 64, 128) };
        const unsigned long long b0[2] = { umma_desc(bbase, 128, 128 * Gm::NA),
                                           umma_desc(bbase + Gm::BCOL, 128, 128 * Gm::NA) };
        constexpr int KPART = KP / 8 / Gm::KS;
        // round r: K step q*KPART + r of both columns (two accumulators)
#pragma unroll
        for (int r = 0; r < KPART; ++r)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const int kk = q * KPART + r;
            umma_tf32(tmem + (unsigned)(sl * Gm::SLOTW + (c * Gm::KS + q) * 16), a0[c] + (unsigned long long)(kk * 8),
                      b0[c] + (unsigned long long)(kk * 16), Gm::IDESC, r > 0 ? 1u : 0u);
          }
        umma_commit(&empty[k]);                              // the stage may be refilled once these finish
        umma_commit(&done[sl]);                              // the slot's accumulators are final
      }
    }
    __syncwarp();
  } else if (warp >= 8) {
    // ---- stage fills (thread 511): one bulk copy of the pair's two B
    // operands onto the stage's bfull barrier, as soon as the stage is free
    if (tid == 511) {
      // the tile's input rows (4*NJJ consecutive rows of S values) into L2
      // first: the pair copies below then read L2, not DRAM
      {
        const char *rows = reinterpret_cast<const char *>(alpha + 4 * j0 * S);
        const long long nrow = wrap ? M - 4 * j0 : 4 * Gm::NJJ;
        const long long bytes = nrow * S * (long long)sizeof(V);
        for (long long off = 0; off < bytes; off += 32768) {
          const unsigned len = (unsigned)(bytes - off < 32768 ? bytes - off : 32768);
          asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(rows + off), "r"(len) : "memory");
        }
      }
      for (int p = 0; p < NP; ++p) {
        const int k = p % NST;
        if (p >= NST) {
          long long it = 0;
          bool ok = true;
          while (!mbar_try_wait(&empty[k], (unsigned)((p / NST - 1) & 1))) {
            if (s_bad || ++it > kBulkWaitLimit) { ok = false; break; }
          }
          if (!ok) {
            atomicExch(a.err, 1);
            s_bad = 1;
            break;
          }
        }
        unsigned char *st = stage_ptr(k);
        mbar_expect_tx(&bfull[k], 2 * Gm::BCOL);
        bulk_g2s(st + Gm::OFF_B, btab + (size_t)2 * p * (Gm::BCOL / 4), 2 * Gm::BCOL, &bfull[k]);
        ++nbcopy[k];
      }
    } else if (warp < 12) {
      // ---- converters, warps 8-11: thread t < 2*NJJ owns row quad jj = t/2 of
      // column t%2 of the pair: x_{t,c}[4jj .. 4jj+3] become chunks 4jj + 2t + c.
      // The inputs are loaded into registers two pairs ahead (from L2, where
      // the loader prefetched the tile's rows); a stage is written once its
      // previous MMAs have finished
      const int t = tid - 256;
      const bool active = t < Gm::NPROD;
      const int jj = t >> 1, cs = t & 1;
      const V *src[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        long long r = 4 * (j0 + jj) + e;
        if (r >= M) r -= M;                                  // circular (ghost rows, .cpp:495-515)
        src[e] = alpha + r * S + cs;
      }
      V xa[4], xb[4];
      auto ld = [&](int p, V *x) {
#pragma unroll
        for (int e = 0; e < 4; ++e) x[e] = __ldg(src[e] + 2 * p);
      };
      auto put = [&](int p, V *x) {
        const int k = p % NST;
        if (p >= NST && !wait_bar(&empty[k], (unsigned)((p / NST - 1) & 1))) return false;
        if (active) {
          unsigned char *st = stage_ptr(k);
          float4 hr, hi, lr, li;
          float *h0 = &hr.x, *h1 = &hi.x, *l0 = &lr.x, *l1 = &li.x;
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            h0[e] = tf32_rna(x[e].x);
            h1[e] = tf32_rna(x[e].y);
            l0[e] = tf32_rna(x[e].x - h0[e]);
            l1[e] = tf32_rna(x[e].y - h1[e]);
          }
          float4 *c4 = reinterpret_cast<float4 *>(st + (1 - cs) * Gm::ASTR) + 4 * jj;
          c4[0] = hr;
          c4[1] = hi;
          c4[2] = lr;
          c4[3] = li;
          fence_proxy_async_smem();                          // the chunks, for the tensor cores
          mbar_arrive(&full[k]);
          if (p + 2 < NP) ld(p + 2, x);
        }
        return true;
      };
      if (active) {
        ld(0, xa);
        ld(1, xb);
      }
      for (int p = 0; p < NP; p += 2) {
        if (!put(p, xa)) break;
        if (!put(p + 1, xb)) break;
      }
    }
  }
  // drain: every MMA this CTA issued and every copy it started completes
  // before the tensor memory is released or the CTA leaves (each warp
  // reconverges first: the roles of warps 4-6 and 15 run in one lane)
  __syncwarp();
  __syncthreads();
  if (warp >= 4 && warp < 4 + Gm::KS && lane == 0) umma_commit(fin);
  {
    long long it = 0;
    while (!mbar_try_wait(fin, 0u) && ++it <= 4 * kBulkWaitLimit) {}
  }
  if (tid == 511) {
    // the stage fills: each stage's last one has landed (in a normal run the
    // converters and the MMAs already waited for all of them)
    for (int k = 0; k < NST; ++k) {
      long long it = 0;
      if (nbcopy[k] > 0)
        while (!mbar_try_wait(&bfull[k], (unsigned)((nbcopy[k] - 1) & 1)) && ++it <= 4 * kBulkWaitLimit) {}
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 4) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((unsigned)Gm::TMEM_COLS)
                 : "memory");
  }
  if (s_bad) return;
  EmitTransposed<V> e{ reinterpret_cast<V *>(a.T), a.Mh, (long long)NMU * j0, a.seg_lo, a.seg_hi,
                      a.seg_lo == 0 && a.seg_hi >= S };
  tile_fft_smem<V, R0, R1, 1>(tile, NMU * JT, 1, PITCH, twS, e);
}

}  // namespace soi
