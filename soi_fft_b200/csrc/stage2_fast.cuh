// stage2_fast.cuh -- the M'-point FFT of every segment with the demodulation
// epilogue (pfft.c:642,649-694), as one persistent kernel with the tile
// geometry fixed at compile time.
//
// Four-step split M' = M1*M2.  Pass 1 of segment s (tile = C columns m2):
// FFT of length M1 over m1 of T[s][m1*M2 + m2], times w_{M'}^(m2*k1), written
// in place.  Pass 2 (tile = C rows k1): FFT of length M2 of row k1, output
// k = k1 + M1*k2, times W_inv[k], stored for k < M (the discard).
//
// Pass-1 tiles (M1 rows of one 32-byte run each) arrive by 2-D tensor copies;
// pass-2 tiles (C whole rows of M2 contiguous elements) by C bulk copies into
// rows at a bank-skewed pitch (FP32 instances; cp.async into a padded tile
// otherwise), both off the load/store path.
//
// Each tile FFT is an in-place decimation-in-frequency transform with "fat"
// radices held in registers (RegDFT), two or three radix stages with one pass
// through shared memory between stages; the last stage stores straight to
// global memory through the epilogue.
//
// C = 32 bytes / element size: every strided row run of a tile (pass-1 loads
// and stores, pass-2 output stores) is one full 32-byte sector, so each L2
// request moves a whole sector.
//
// Epilogue factors come from tables instead of scattered lookups.  Pass 1:
// w_{M'}^(m2*f) for f = fbase + fstep*k is base(m2*fbase) times
// step[col][k] = w_{M'}^(m2*fstep*k); both come from tables laid out in the
// order the warps read them, the task's C x RL steps copied into shared memory
// (row pitch RL + 1).  Pass 2: W_inv[k], k = k1 + M1*k2, is
// amp[min(k, M-k)] * ph(k1) * ph(M1*k2) with ph(k) = exp(-i pi kappa k/M);
// ph(k1) per task in shared memory, amp and ph(M1*k2) from tables laid out in
// the order the last radix stage stores its outputs, and the tile twiddles
// from tables in the order the radix stages read them, so that every table
// load of a warp is one cache line (the SM's load/store data path is this
// kernel's busiest unit).  Every table entry is FP64-generated and rounded
// once; the products are formed in the working precision.
//
// Schedule: CTAs take tasks from a global counter in the order
//   P1(0), P1(1), P2(0), P1(2), P2(1), ..., P2(S-1),
// so that only two segments' intermediates (2 * M' * 8 bytes, 84 MB at
// N = 2^29 in FP32) are live; they stay in L2 between the passes.  A pass-2
// task of segment s waits, with an iteration limit, until all pass-1 tasks of
// s have published their tiles (per-segment counter, release/acquire at gpu
// scope).  Pass-2 tasks then drop the lines they consumed from L2 without
// write-back (discard.global.L2), so the dead intermediate never returns to
// HBM.  The CTA claims its next task while it works on the current one.  A
// CTA holds at most one claimed task it has not started, and a pass-2 task
// only waits on tasks with smaller indices, so the lowest unfinished task can
// always run.  A wait that gives up sets the error flag, and every CTA then
// stops taking tasks; the host reads the flag (SOI_ERR_TIMEOUT).
//
// The kernel works on the segment range [seg_lo, seg_lo + S) of the buffers
// (all segments for a full transform, a band of segments for a
// segments-of-interest transform).
#pragma once

#include "async_copy.cuh"
#include "fft_reg.cuh"

namespace soi {

constexpr long long kWaitLimit = 1ll << 22;   // ~1 s of 256 ns sleeps

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p)
{
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void discard_l2_line(const void *p)
{
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

template <typename V> __device__ __forceinline__ void stcs(V *p, V v);
template <> __device__ __forceinline__ void stcs<float2>(float2 *p, float2 v) { __stcs(p, v); }
template <> __device__ __forceinline__ void stcs<double2>(double2 *p, double2 v) { __stcs(p, v); }

__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem)
{
  const unsigned int s = (unsigned int)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_16cg(void *smem, const void *gmem)
{
  const unsigned int s = (unsigned int)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

struct S2ArgsCT {
  void *T;                    // [S][Mh] pass-1 input, intermediate in place
  void *out;                  // [S][M]
  const void *tw1, *tw2;      // tile twiddles of the two passes, warp read order
  const void *base1;          // [M2/C][M1/RL][C] pass-1 epilogue bases w_{M'}^(m2*fbase), warp read order
  const void *step1;          // [M2][RL] pass-1 epilogue steps w_{M'}^(m2*(M1/RL)*k)
  const void *amp;            // [M1][M2] real, pass-2 store order per task
  const double2 *dlo, *dhi;   // exp(-i pi kappa k/M) two-level, FP64
  const void *ph2;            // [M2] complex exp(-i pi kappa M1 k2 / M), pass-2 store order
  int dlo_bits;
  int M;
  int S;                      // segments in this launch
  int seg_lo;                 // first segment of this launch
  int discard;
  int tma;                    // 1: pass-1 tiles come by tensor copy (the map in the launch's second argument)
  int wait_extra;             // 0; a test sets 1 to make every pass-2 wait run out
  int tail;                   // pass-2 tasks that end a block after its interleaved part (0 .. M1/C)
  int amp_keep;               // 1: amp loads carry an L2 evict_last hint
  int bulk2;                  // 1: pass-2 rows arrive by bulk copies
  int rows2;                  // 1: FP32 pass-2 threads on row pairs (tile_fft_rows2)
  unsigned int *counter, *done1;
  int *err;
};

// a read-only load with an L2 eviction-priority hint (createpolicy); used
// to keep a table that every segment re-reads resident in L2
__device__ __forceinline__ float ldg_hint(const float *p, unsigned long long pol)
{
  float v;
  asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ldg_hint(const double *p, unsigned long long pol)
{
  double v;
  asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ unsigned long long l2_evict_last_policy()
{
  unsigned long long pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

template <typename V>
__device__ __forceinline__ V two_level(const double2 *lo, const double2 *hi, int bits, int e)
{
  const double2 l = __ldg(lo + (e & ((1 << bits) - 1)));
  const double2 h = __ldg(hi + (e >> bits));
  return cmk<V>((decltype(V::x))(h.x * l.x - h.y * l.y), (decltype(V::x))(h.x * l.y + h.y * l.x));
}

template <typename V, int C1, int M2, int RL> struct EmitColsCT {
  V *Tseg; int m2_0; const V *step; const V *base; const S2ArgsCT *a;
  // w_{M'}^(m2*fbase) of butterfly blk: base[blk*C + col], the task's slice of a
  // table in the order the last radix stage's warps read it (one cache line per
  // warp load), loaded before the last radix
  __device__ __forceinline__ V prepare(int col, int, int blk) const
  {
    return __ldg(base + blk * C1 + col);
  }
  template <int RLx> __device__ __forceinline__ void run(int col, int fbase, int fstep, V *v, V base_f, int) const
  {
    static_assert(RLx == RL, "last radix");
    const int m2 = m2_0 + col;
    V *dst = Tseg + fbase * M2 + m2;
    dst[0] = cmul(v[0], base_f);
#pragma unroll
    for (int k = 1; k < RL; ++k) dst[k * fstep * M2] = cmul(v[k], cmul(base_f, step[col * (RL + 1) + k]));
  }
};

struct NoPre {};

// amp and ph(M1*k2) come from tables in this stage's store order: output j of
// butterfly blk is position pos = blk + fstep*j, and the task's rows k1_0 ..
// k1_0 + C-1 own amp[(k1_0*M2 + pos*C) + col], so that a warp's loads (8
// consecutive butterflies x C rows) are one cache line each
template <typename V, int M1, int M2, int C, int RL, bool BATCH> struct EmitRowsCT {
  V *oseg; int k1_0; const V *ph1; const S2ArgsCT *a; unsigned long long pol;
  __device__ __forceinline__ NoPre prepare(int, int, int) const { return NoPre{}; }
  template <int RLx> __device__ __forceinline__ void run(int col, int fbase, int fstep, V *v, NoPre, int blk) const
  {
    static_assert(RLx == RL, "last radix");
    using Rr = decltype(V::x);
    const int k1 = k1_0 + col;
    const int M = a->M;
    const V p1 = ph1[col];
    const V *ph2 = reinterpret_cast<const V *>(a->ph2);
    const Rr *amp = reinterpret_cast<const Rr *>(a->amp) + (size_t)k1_0 * M2 + col;
    if constexpr (sizeof(V) == 8 && BATCH) {
      // FP32 with registers to spare: all RL factors in flight before the
      // first store
      V w[RL];
#pragma unroll
      for (int j = 0; j < RL; ++j) {
        const int pos = blk + fstep * j;
        w[j] = cscale(cmul(p1, __ldg(ph2 + pos)), (a->amp_keep ? ldg_hint(amp + pos * C, pol) : __ldg(amp + pos * C)));
      }
#pragma unroll
      for (int j = 0; j < RL; ++j) {
        const int k = k1 + M1 * (fbase + fstep * j);
        if (k < M) stcs(oseg + k, cmul(v[j], w[j]));
      }
    } else {
      // FP64, or a tight register budget: RL factors would not fit beside
      // the data
#pragma unroll
      for (int j = 0; j < RL; ++j) {
        const int pos = blk + fstep * j;
        const int k = k1 + M1 * (fbase + fstep * j);
        const V w = cscale(cmul(p1, __ldg(ph2 + pos)), (a->amp_keep ? ldg_hint(amp + pos * C, pol) : __ldg(amp + pos * C)));
        if (k < M) stcs(oseg + k, cmul(v[j], w));
      }
    }
  }
};

// EmitRowsCT for a pair of rows (2*cp, 2*cp + 1) of an FP32 task of C = 4
// rows: ph(M1*k2) and the two rows' amplitudes (adjacent in the table) are
// loaded once per position, and outputs k and k + 1 (k even, so both or
// neither below M) leave as one 16-byte streaming store.  The same products,
// in the same order, as EmitRowsCT.
template <int M1, int M2, int RL> struct EmitRowsCT2 {
  float2 *oseg; int k1_0; const float2 *ph1; const S2ArgsCT *a;
  template <int RLx> __device__ __forceinline__ void run2(int cp, int fbase, int fstep, const float2 *v,
                                                          const float2 *w, int blk) const
  {
    static_assert(RLx == RL, "last radix");
    constexpr int C = 4;
    const int ka = k1_0 + 2 * cp;
    const int M = a->M;
    const float2 pa = ph1[2 * cp], pb = ph1[2 * cp + 1];
    const float2 *ph2 = reinterpret_cast<const float2 *>(a->ph2);
    const float2 *amp = reinterpret_cast<const float2 *>(reinterpret_cast<const float *>(a->amp) +
                                                        (size_t)k1_0 * M2 + 2 * cp);
#pragma unroll
    for (int j = 0; j < RL; ++j) {
      const int pos = blk + fstep * j;
      const float2 ph = __ldg(ph2 + pos);
      const float2 am = __ldg(amp + pos * (C / 2));
      const float2 wa = cscale(cmul(pa, ph), am.x), wb = cscale(cmul(pb, ph), am.y);
      const int k = ka + M1 * (fbase + fstep * j);
      if (k < M) {
        const float2 ya = cmul(v[j], wa), yb = cmul(w[j], wb);
        __stcs(reinterpret_cast<float4 *>(oseg + k), make_float4(ya.x, ya.y, yb.x, yb.y));
      }
    }
  }
};

template <int base, int mod, int rem> constexpr int round_up_to_residue()
{
  int x = base;
  while (x % mod != rem) ++x;
  return x;
}

template <typename R, int A0, int A1, int A2, int B0, int B1, int B2, int NT, int CC>
struct S2Geom {
  using V = typename cplx_of<R>::type;
  static constexpr int E = (int)sizeof(V);
  static constexpr int C = CC;                              // columns (rows) per task
  static_assert(C * E == 32 || C * E == 16, "a task's row run is a whole or a half 32-byte sector");
  static constexpr int CPR1 = C * E / 16;                   // 16-byte chunks per pass-1 row run
  static constexpr int M1 = A0 * A1 * A2, M2 = B0 * B1 * B2;
  static constexpr int RLA = A2 > 1 ? A2 : A1, RLB = B2 > 1 ? B2 : B1;
  static constexpr int NT1 = M2 / C, NT2 = M1 / C, PER = NT1 + NT2;
  // pass-2 row pitch: the C rows land on disjoint banks in the last stage,
  // whose loads the hardware splits into groups of 128 bytes (16 eight-byte
  // or 8 sixteen-byte slots): pitch = (slots / C) mod slots
  static constexpr int SLOTS = 128 / E;
  static constexpr int PS2 = round_up_to_residue<M2 + M2 / RLB, SLOTS, (SLOTS / C) % SLOTS>();
  // pass-2 rows by bulk copies: whole rows at pitch PR2 = 4 (mod SLOTS)
  // elements, so the C rows of a task start SLOTS / C slots apart (FP32, C = 4:
  // 4 of 16 eight-byte slots; FP64, C = 2: 4 of 8 sixteen-byte slots), and the
  // last radix's XOR read order spreads a group of 4 butterflies over 4 slots
  static constexpr int PR2 = M2 + 4;
  static constexpr bool BULK2 = ((E == 8 && C == 4) || (E == 16 && C == 2)) && RLB % 4 == 0 && M2 % 16 == 0;
  // pass-1 tensor copies: boxes of BOXR rows (the largest divisor of M1 of at
  // most 256 rows that is a multiple of 32 rows, so every box starts 1024-byte
  // aligned), into a dense tile aligned to 1024 bytes inside the buffer
  // (slack reserved)
  static constexpr int BOXR = [] {
    int b = 0;
    for (int d = 32; d <= 256; d += 32)
      if (M1 % d == 0) b = d;
    return b;
  }();
  static constexpr int BUF1 = (M1 + M1 / RLA) * C, BUF2 = PS2 * C, BUFT = M1 * C + 1024 / E;
  static constexpr int BUF = (BUF1 > BUF2 ? BUF1 : BUF2) > BUFT ? (BUF1 > BUF2 ? BUF1 : BUF2) : BUFT;
  // shared table entries: the pass-1 step table, one row of RLA + 1 per
  // column (the pad puts a warp's C columns on different banks; at a pitch of
  // RLA every read of the table was a C-way bank conflict)
  static constexpr int TAB = C * (RLA + 1);
};

template <typename R, int A0, int A1, int A2, int B0, int B1, int B2, int NT, int CC, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_stage2_ct(S2ArgsCT a, const __grid_constant__ CUtensorMap tmap)
{
  using G = S2Geom<R, A0, A1, A2, B0, B1, B2, NT, CC>;
  using V = typename G::V;
  constexpr int C = G::C, M1 = G::M1, M2 = G::M2, RLA = G::RLA, RLB = G::RLB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *buf = reinterpret_cast<V *>(smem_raw);
  __shared__ V s_tab[G::TAB];
  __shared__ __align__(8) unsigned long long s_bar;   // pass-1 tensor copies complete here
  __shared__ unsigned int s_task[2];
  __shared__ int s_ok[2];
  const int tid = threadIdx.x;
  const unsigned int total = (unsigned int)a.S * G::PER;
  // task index -> (pass, segment, tile): P1(0); then per block b = 0 .. S-2
  // the pass-1 tasks of segment b+1 interleaved in proportion with the first
  // NT2 - tail pass-2 tasks of segment b, followed by its last `tail` pass-2
  // tasks; then P2(S-1).  Segment b+1's intermediate grows while b's is
  // consumed (and discarded), so about one segment's intermediate is live in
  // L2, and a segment's pass-2 tasks come at least `tail` claims after its
  // last pass-1 task, by when that task has usually finished (with tail =
  // NT2 every pass-1 task of b+1 comes before the pass-2 tasks of b).
  const int tail = a.tail;
  auto decode = [&](unsigned int t, int &kind, int &seg, int &tile) {
    if (t < (unsigned int)G::NT1) { kind = 1; seg = 0; tile = (int)t; return; }
    const unsigned int u = t - G::NT1;
    const int blk = (int)(u / G::PER), r = (int)(u % G::PER);
    if (blk >= a.S - 1) { kind = 2; seg = blk; tile = r; return; }
    const int n2i = G::NT2 - tail, ni = G::NT1 + n2i;    // the interleaved part
    if (r >= ni) { kind = 2; seg = blk; tile = n2i + (r - ni); return; }
    const int c0 = r * G::NT1 / ni, c1 = (r + 1) * G::NT1 / ni;   // pass-1 tasks among the first r (r + 1)
    if (c1 > c0) { kind = 1; seg = blk + 1; tile = c0; }
    else { kind = 2; seg = blk; tile = r - c0; }
  };
  const unsigned long long amp_pol = l2_evict_last_policy();
  unsigned int next = 0;
  // thread 0: take the claimed task, claim the one after it, and for a
  // pass-2 task wait (bounded) until its segment's pass 1 is complete; the
  // result goes to slot `slot`, read by all threads after the next barrier
  auto take = [&](int slot) {
    unsigned int t = next;
    if (t < total) next = atomicAdd(a.counter, 1u);
    if (*(volatile int *)a.err) t = total;
    int ok = 1;
    if (t < total) {
      int kind, seg, tile;
      decode(t, kind, seg, tile);
      if (kind == 2) {                                      // pass-2 task of segment seg
        long long it = 0;
        while (ld_acquire_u32(a.done1 + seg) < (unsigned int)(G::NT1 + a.wait_extra)) {
          if (++it > kWaitLimit) { atomicExch(a.err, 1); ok = 0; break; }
          if (*(volatile int *)a.err) { ok = 0; break; }   // another CTA gave up
          __nanosleep(128);
        }
      }
    }
    s_task[slot] = t;
    s_ok[slot] = ok;
  };
  if (tid == 0) {
    mbar_init(&s_bar, 1);
    mbar_init_fence();
    next = atomicAdd(a.counter, 1u);
    take(0);
  }
  __syncthreads();
  // the dense pass-1 tile of the tensor-copy path (rows of C elements), 1024-byte aligned
  V *tile1 = reinterpret_cast<V *>(smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u));
  unsigned int bphase = 0;                                  // parity of s_bar's current phase

  for (int iter = 0;; ++iter) {
    const int slot = iter & 1;
    const unsigned int t = s_task[slot];
    if (t >= total || !s_ok[slot]) break;
    int kind, seg, tile;
    decode(t, kind, seg, tile);
    V *Tseg = reinterpret_cast<V *>(a.T) + (size_t)(a.seg_lo + seg) * ((size_t)M1 * M2);
    if (kind == 1) {
      const int m2_0 = tile * C;
      EmitColsCT<V, C, M2, RLA> e{ Tseg, m2_0, s_tab,
                                   reinterpret_cast<const V *>(a.base1) + (size_t)tile * (M1 / RLA) * C, &a };
      if (a.tma) {
        // C columns x M1 rows (32-byte runs 16 KB apart) by M1 / BOXR tensor
        // copies: the TMA engine gathers the rows, off the load/store path
        if (tid == 0) {
          static_assert(G::BOXR > 0 && M1 % G::BOXR == 0, "whole boxes");
          fence_proxy_async_smem();                         // the previous task's reads of the tile come first
          mbar_expect_tx(&s_bar, (unsigned int)(M1 * C * G::E));
          const int y0 = (a.seg_lo + seg) * M1;
#pragma unroll 1
          for (int b = 0; b < M1 / G::BOXR; ++b)
            tma_load_2d(tile1 + b * G::BOXR * C, &tmap, 2 * m2_0, y0 + b * G::BOXR, &s_bar);
        }
        if (tid < C * RLA) {
          const int col = tid / RLA, k = tid % RLA;
          s_tab[col * (RLA + 1) + k] = __ldg(reinterpret_cast<const V *>(a.step1) + (m2_0 + col) * RLA + k);
        }
        long long it = 0;
        while (!mbar_try_wait(&s_bar, bphase)) {
          if (++it > kBulkWaitLimit) {
            // the copy is late: flag it (no further tasks are taken), then
            // wait for it to land (bounded, 16x longer), so that no copy is
            // still writing this CTA's shared memory when the tile buffer is
            // reused or the CTA leaves; the tile computed from it is discarded
            // with the transform (SOI_ERR_TIMEOUT)
            if (tid == 0) atomicExch(a.err, 1);
            long long drain = 0;
            while (!mbar_try_wait(&s_bar, bphase) && ++drain <= 16 * kBulkWaitLimit) {}
            break;
          }
        }
        bphase ^= 1u;
        __syncthreads();
        tile_fft_ct_dense<V, A0, A1, A2, C, NT>(tile1, reinterpret_cast<const V *>(a.tw1), e);
      } else {
        // rows m1 of C columns: CPR1 chunks of 16 bytes each
        constexpr int EPC = 16 / G::E;                        // elements per 16-byte chunk
        constexpr int CPR1 = G::CPR1;
        for (int q = tid; q < M1 * CPR1; q += NT) {
          const int row = q / CPR1, h = q % CPR1;
          cp_async_16cg(buf + (row + row / RLA) * C + h * EPC, Tseg + row * M2 + m2_0 + h * EPC);
        }
        cp_commit();
        if (tid < C * RLA) {
          const int col = tid / RLA, k = tid % RLA;
          s_tab[col * (RLA + 1) + k] = __ldg(reinterpret_cast<const V *>(a.step1) + (m2_0 + col) * RLA + k);
        }
        cp_wait_all();
        __syncthreads();
        tile_fft_ct<V, A0, A1, A2, C, C, 1, NT>(buf, reinterpret_cast<const V *>(a.tw1), e);
      }
      __syncthreads();                                        // every store of the tile is issued
      if (tid == 0) {
        __threadfence();
        atomicAdd(a.done1 + seg, 1u);                         // publish, then take the next task
        take(slot ^ 1);
      }
    } else if (G::BULK2 && a.bulk2) {
      // C whole rows k1 (C*M2 contiguous elements) by C bulk copies into rows
      // at pitch PR2, onto the same mbarrier as pass 1's tensor copies
      const int k1_0 = tile * C;
      const V *src = Tseg + k1_0 * M2;
      static_assert(!G::BULK2 || C * G::PR2 <= G::BUF, "pass-2 rows fit the tile buffer");
      if (tid == 0) {
        fence_proxy_async_smem();                           // the previous task's accesses of the buffer come first
        mbar_expect_tx(&s_bar, (unsigned int)(C * M2 * G::E));
#pragma unroll
        for (int c = 0; c < C; ++c) bulk_g2s(buf + c * G::PR2, src + c * M2, (unsigned)(M2 * G::E), &s_bar);
      }
      if (tid < C) s_tab[tid] = two_level<V>(a.dlo, a.dhi, a.dlo_bits, k1_0 + tid);
      long long it = 0;
      while (!mbar_try_wait(&s_bar, bphase)) {
        if (++it > kBulkWaitLimit) {
          // late copies: flag them (no further tasks are taken), then wait for
          // them to land (bounded, 16x longer) before the buffer is reused or
          // the CTA leaves
          if (tid == 0) atomicExch(a.err, 1);
          long long drain = 0;
          while (!mbar_try_wait(&s_bar, bphase) && ++drain <= 16 * kBulkWaitLimit) {}
          break;
        }
      }
      bphase ^= 1u;
      __syncthreads();
      if (a.discard) {
        const char *base = reinterpret_cast<const char *>(src);
        constexpr int nlines = C * M2 * G::E / 128;
        for (int l = tid; l < nlines; l += NT) discard_l2_line(base + l * 128);
      }
      EmitRowsCT<V, M1, M2, C, RLB, (MINB <= 2)> e{ reinterpret_cast<V *>(a.out) + (size_t)(a.seg_lo + seg) * a.M, k1_0, s_tab, &a,
                                                    amp_pol };
      if constexpr (G::BULK2) {
        if constexpr (G::E == 8 && C == 4) {
          if (a.rows2) {
            EmitRowsCT2<M1, M2, RLB> e2{ reinterpret_cast<float2 *>(a.out) + (size_t)(a.seg_lo + seg) * a.M, k1_0,
                                         reinterpret_cast<const float2 *>(s_tab), &a };
            tile_fft_rows2<V, B0, B1, B2, G::PR2, NT>(buf, reinterpret_cast<const V *>(a.tw2), e2);
          } else {
            tile_fft_rows<V, B0, B1, B2, C, G::PR2, NT>(buf, reinterpret_cast<const V *>(a.tw2), e);
          }
        } else {
          tile_fft_rows<V, B0, B1, B2, C, G::PR2, NT>(buf, reinterpret_cast<const V *>(a.tw2), e);
        }
      }
      if (tid == 0) take(slot ^ 1);                           // after thread 0's own stores
    } else {
      const int k1_0 = tile * C;
      const V *src = Tseg + k1_0 * M2;
      if constexpr (G::E == 16) {
        for (int q = tid; q < C * M2; q += NT) {
          const int col = q / M2, pos = q % M2;
          cp_async_16cg(buf + (pos + pos / RLB) + col * G::PS2, src + q);
        }
      } else {
        for (int q = tid; q < C * M2; q += NT) {
          const int col = q / M2, pos = q % M2;
          cp_async_8(buf + (pos + pos / RLB) + col * G::PS2, src + q);
        }
      }
      cp_commit();
      if (tid < C) s_tab[tid] = two_level<V>(a.dlo, a.dhi, a.dlo_bits, k1_0 + tid);
      cp_wait_all();
      __syncthreads();
      if (a.discard) {
        // the tile's rows are in shared memory now; their L2 lines are dead
        const char *base = reinterpret_cast<const char *>(src);
        constexpr int nlines = C * M2 * G::E / 128;
        for (int l = tid; l < nlines; l += NT) discard_l2_line(base + l * 128);
      }
      EmitRowsCT<V, M1, M2, C, RLB, (MINB <= 2)> e{ reinterpret_cast<V *>(a.out) + (size_t)(a.seg_lo + seg) * a.M, k1_0, s_tab, &a,
                                                    amp_pol };
      tile_fft_ct<V, B0, B1, B2, C, 1, G::PS2, NT>(buf, reinterpret_cast<const V *>(a.tw2), e);
      if (tid == 0) take(slot ^ 1);                           // after thread 0's own stores
    }
    __syncthreads();                                          // the tile buffer is free, the next task is known
  }
}

}  // namespace soi
