// soi_b200.cu -- host side of libsoi_b200.so: the C ABI of include/soi_b200.h,
// descriptor/plan lifecycle (pfft.c:84-267), long-double table generation
// and the launches of the stage-1/stage-2 kernels (soi_kernels.cuh).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <math.h>
#include <cmath>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <vector>

#include "../../include/soi_b200.h"
#include "soi_kernels.cuh"
#include "vlc_kernels.cuh"
#include "stage2_fast.cuh"
#include "stage1_fast.cuh"
#include "stage1_tc.cuh"
#include "mlp_kernels.cuh"

using namespace soi;

namespace {

const long double kPi = 3.141592653589793238462643383279502884197169399375L;

struct Plan {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int prec = SOI_PRECISION_FP64;
  size_t elem = 16;            // bytes per complex element
  size_t N = 0, S = 0, M = 0, Mh = 0, J = 0, B = 0;
  int nmu = 5, dmu = 4;
  double tau = 0, sigma = 0;
  int atap = 0, JR = 8, JT = 0, pitch = 0;
  size_t smem1 = 0, smem_c = 0, smem_r = 0;
  FftPlan planS{}, plan1{}, plan2{};
  int M1 = 0, M2 = 0, C1 = 0, C2 = 0, lo_bits = 11;
  void *d_filt = nullptr, *d_phase = nullptr, *d_twS = nullptr, *d_tw1 = nullptr, *d_tw2 = nullptr;
  void *d_winv = nullptr, *d_wsmall = nullptr;
  int *d_permS = nullptr, *d_perm1 = nullptr, *d_perm2 = nullptr;
  double2 *d_xlo = nullptr, *d_xhi = nullptr;
  void *d_T = nullptr;         // S*Mh complex
  void *d_io = nullptr;        // N complex staging for host pointers
  void *d_io2 = nullptr;       // second and third staging buffers (streamed host transforms)
  void *d_io3 = nullptr;
  cudaStream_t st_in = nullptr, st_out = nullptr;   // copy streams (streamed host transforms)
  cudaEvent_t sev[9] = {};     // in-copied[3], computed[3], out-copied[3]
  // VLC
  int *d_vlc_words = nullptr, *d_vlc_n = nullptr, *d_vlc_emax = nullptr;
  long vlc_stride = 0;
  // persistent stage 2: compiled radix split and its state
  int fast2 = 0;               // 0: two-kernel stage 2, 3: persistent kernel (4: chosen, not set up)
  int f2_variant = 0;
  int f2_nt = 256;             // threads of the persistent stage-2 instance
  int f2_boxr = 0;             // rows per pass-1 tensor copy
  int f2_tail = 0;             // stage-2 schedule: pass-2 tasks that end a block
  bool tma1 = false;           // tmap1 describes d_T: pass-1 tiles come by tensor copy
  CUtensorMap tmap1;           // d_T as (2*M2 values) x (S*M1 rows), 32-byte boxes, no swizzle
  int f2_grid = 0;
  size_t f2_smem = 0;
  int discard = 1;             // drop consumed intermediate lines from L2
  int amp_keep = 0;            // demodulation amplitude loads hint L2 evict_last
  int bulk2 = 0;               // pass-2 rows by bulk copies
  int rows2 = 0;               // FP32 pass-2 threads on row pairs
  int wait_extra = 0;          // failure test: pass-2 waits for a count that never comes
  void *d_amp = nullptr;            // [M1][M2] real demodulation amplitude, pass-2 store order
  void *d_ctw1 = nullptr, *d_ctw2 = nullptr;   // tile-FFT twiddles of the two passes, warp read order
  void *d_base1 = nullptr, *d_step1 = nullptr; // pass-1 epilogue bases and steps, warp read order
  double2 *d_dlo = nullptr, *d_dhi = nullptr;
  int dlo_bits = 11;
  void (*f2ct_kernel)(S2ArgsCT, const CUtensorMap) = nullptr;
  void *d_ph2 = nullptr;            // [M2] complex exp(-i pi kappa M1 k2 / M), pass-2 store order
  unsigned int *d_sync = nullptr;   // [0] err, [1] counter, [2..2+S) done1
  // staged stage 1
  int s1fast = 0, JR2 = 0, JT2 = 0, AC = 0, buf_elems = 0;
  int s1_tS = 0;                    // compile-time-S stage-1 instance available
  int s1_nt = 512;                  // its block size (256: two CTAs per SM)
  int s1_bulk = 0;                  // its staging by tensor copies
  size_t smem1b = 0;
  void *d_filt2 = nullptr;          // [d][atap][nmu][S] real
  // variant choices forced by the batch tuner (-1: defaults / SOI_* switches)
  int knob_s1_nt = -1;              // 256 or 512 threads for the compile-time-S stage 1
  int knob_s2 = -1;                 // 1 persistent stage 2, 0 two-kernel stage 2
  int knob_s1_bulk = -1;            // 1/0: stage-1 staging by bulk copies or cp.async
  // tensor-core stage 1 (split form, n = 5, d = 4, S in {32, 64, 128}, B <= 72 taps)
  int s1_tc = 0;
  void *d_btc = nullptr;            // [S][16 rows][72 taps] TF32 hi/lo filter, the MMA's B layout
  // a caller's window (soi_init_window_status): y(t) at the taps, [B][n][S],
  // and its transform at xi = j/M - 1/2, j <= M/2; empty: the analytic window
  std::vector<double> cw_time, cw_freq;
  bool timing = false;
  cudaEvent_t ev[5] = {};
  float ms[4] = {0, 0, 0, 0};
};

// One execution of the transform (or of a band of its segments): device
// buffers, stage-2 synchronisation words and the stream.  A plan's own
// compute uses the plan's scratch; the batch driver gives each concurrent
// chain its own.
struct Exec {
  const void *in;              // N inputs [M rows][S]
  void *T;                     // S x M' transposed data
  void *out;                   // N outputs [S][M] (rows of segments outside [lo, hi) untouched)
  unsigned int *sync;          // [0] error flag (sticky), [1] task counter, [2 .. 2 + S) pass-1 counts
  int lo, hi;                  // segments computed
  cudaStream_t st;
  const CUtensorMap *tmap = nullptr;   // T for the pass-1 tensor copies (null: cp.async staging)
};

#define CK(x)                                                                    \
  do {                                                                           \
    cudaError_t e__ = (x);                                                       \
    if (e__ != cudaSuccess) {                                                    \
      fprintf(stderr, "soi_b200: %s failed: %s\n", #x, cudaGetErrorString(e__)); \
      return SOI_ERR_CUDA;                                                       \
    }                                                                            \
  } while (0)

int env_int(const char *name, int dflt)
{
  const char *v = getenv(name);
  return v ? atoi(v) : dflt;
}

// ---- FFT planning ------------------------------------------------------------

bool make_fft_plan(int L, FftPlan &p)
{
  memset(&p, 0, sizeof(p));
  p.L = L;
  int n = L, t = 0;
  while (n % 8 == 0 && n > 8 && t < kMaxStages) { p.radix[t++] = 8; n /= 8; }
  if (n == 8 && t < kMaxStages) { p.radix[t++] = 8; n = 1; }
  while (n % 4 == 0 && t < kMaxStages) { p.radix[t++] = 4; n /= 4; }
  while (n % 2 == 0 && t < kMaxStages) { p.radix[t++] = 2; n /= 2; }
  while (n % 5 == 0 && t < kMaxStages) { p.radix[t++] = 5; n /= 5; }
  while (n % 3 == 0 && t < kMaxStages) { p.radix[t++] = 3; n /= 3; }
  while (n % 7 == 0 && t < kMaxStages) { p.radix[t++] = 7; n /= 7; }
  p.nst = t;
  return n == 1 && L >= 1;
}

// perm[k] = position of frequency k after the in-place DIF stages.
std::vector<int> digit_reversal(const FftPlan &p)
{
  std::vector<int> perm(p.L);
  for (int k = 0; k < p.L; ++k) {
    int rem = k, span = p.L, pos = 0;
    for (int s = 0; s < p.nst; ++s) {
      span /= p.radix[s];
      pos += (rem % p.radix[s]) * span;
      rem /= p.radix[s];
    }
    perm[k] = pos;
  }
  return perm;
}

// ---- tables (long double, rounded once to the working precision) -----------

// time window (pfft.c:42-66) factorised as phase * real filter:
//   t = theta*d/n - kk - s/S + kappa/2, w = exp(i pi t) * y(t) / mu,
//   exp(i pi t) = exp(i pi (theta*d/n + kappa/2 - s/S)) * (-1)^kk.
long double window_y(long double t, double tau, double sigma)
{
  if (t == 0) return 1.0L;
  long double a = kPi * (long double)tau * t;
  return sinl(a) / a * expl(-kPi * kPi * t * t / (long double)sigma);
}

// With ytime / yfreq (a caller's window, soi_init_window_status) the real
// window y(t) at the taps and its Fourier transform at xi = j/M - 1/2,
// j <= M/2, replace the analytic y and y_W.
void host_tables(size_t N, size_t S, int n, int d, size_t B, double tau, double sigma, int atap,
                 std::vector<long double> *filt, std::vector<long double> *ph_re,
                 std::vector<long double> *ph_im, std::vector<long double> *wi_re,
                 std::vector<long double> *wi_im, const double *ytime = nullptr, const double *yfreq = nullptr)
{
  const long long kappa = (long long)B - d;
  const long double mu = (long double)n / d;
  const long long den = 2LL * n * (long long)S;  // t = num / den
  size_t ntap = atap ? (size_t)atap * d : B;
  if (filt) {
    filt->assign(ntap * n * S, 0.0L);
    for (size_t kk = 0; kk < B; ++kk)
      for (int th = 0; th < n; ++th)
        for (size_t s = 0; s < S; ++s) {
          long long num = 2LL * th * d * (long long)S - 2LL * (long long)kk * n * (long long)S -
                          2LL * (long long)s * n + kappa * n * (long long)S;
          long double t = (long double)num / (long double)den;
          long double y = (ytime ? (long double)ytime[(kk * n + th) * S + s] : window_y(t, tau, sigma)) / mu;
          (*filt)[(kk * n + th) * S + s] = (kk & 1) ? -y : y;
        }
  }
  if (ph_re) {
    ph_re->assign((size_t)n * S, 0);
    ph_im->assign((size_t)n * S, 0);
    const long long period = 2 * den;  // exp(i pi q/den) has period 2*den in q
    for (int th = 0; th < n; ++th)
      for (size_t s = 0; s < S; ++s) {
        long long q = 2LL * th * d * (long long)S + kappa * n * (long long)S - 2LL * (long long)s * n;
        q %= period;
        if (q < 0) q += period;
        long double ang = kPi * (long double)q / (long double)den;
        (*ph_re)[th * S + s] = cosl(ang);
        (*ph_im)[th * S + s] = sinl(ang);
      }
  }
  if (wi_re) {
    // pfft.c:68-82: W_inv[i] = exp(-i pi kappa i / M) / y_W(i/M - 1/2)
    size_t M = N / S;
    wi_re->assign(M, 0);
    wi_im->assign(M, 0);
    const long double sq = sqrtl((long double)sigma);
    for (size_t i = 0; i < M; ++i) {
      long double t = (long double)i / (long double)M - 0.5L;
      long double y = yfreq ? (long double)yfreq[std::min(i, M - i)]
                            : (erfcl(sq * (t - tau / 2.0L)) - erfcl(sq * (t + tau / 2.0L))) / (2.0L * tau);
      long long q = (long long)(((unsigned long long)kappa * i) % (2ULL * M));
      long double ang = -kPi * (long double)q / (long double)M;
      (*wi_re)[i] = cosl(ang) / y;
      (*wi_im)[i] = sinl(ang) / y;
    }
  }
}

template <typename R>
void round_complex(const std::vector<long double> &re, const std::vector<long double> &im, std::vector<R> &out)
{
  out.resize(2 * re.size());
  for (size_t i = 0; i < re.size(); ++i) { out[2 * i] = (R)re[i]; out[2 * i + 1] = (R)im[i]; }
}

template <typename R>
std::vector<R> roots_table(long long L)
{
  std::vector<R> t(2 * L);
  for (long long m = 0; m < L; ++m) {
    long double a = -2.0L * kPi * (long double)m / (long double)L;
    t[2 * m] = (R)cosl(a);
    t[2 * m + 1] = (R)sinl(a);
  }
  return t;
}

int upload(void **dst, const void *src, size_t bytes)
{
  CK(cudaMalloc(dst, bytes ? bytes : 16));
  if (bytes) CK(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
  return SOI_OK;
}

// ---- kernel dispatch ---------------------------------------------------------

template <typename R, int NMU, int JR>
int launch_conv_t(Plan &p, const Exec &ex)
{
  ConvArgs a;
  a.alpha = ex.in; a.T = ex.T; a.filt = p.d_filt; a.seg_lo = ex.lo; a.seg_hi = ex.hi; a.phase = p.d_phase; a.twS = p.d_twS;
  a.permS = p.d_permS; a.wsmall = p.d_wsmall; a.planS = p.planS;
  a.M = (long long)p.M; a.Mh = (long long)p.Mh; a.J = (long long)p.J;
  a.S = (int)p.S; a.d = p.dmu; a.atap = p.atap; a.JT = p.JT; a.pitch = p.pitch;
  auto kern = k_conv_sfft<R, NMU, JR>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem1));
  dim3 grid((unsigned)((p.J + p.JT - 1) / p.JT));
  kern<<<grid, 256, p.smem1, ex.st>>>(a);
  CK(cudaGetLastError());
  return SOI_OK;
}

template <typename R>
int launch_conv_r(Plan &p, const Exec &ex)
{
  switch (p.nmu) {
    case 2: return launch_conv_t<R, 2, 8>(p, ex);
    case 3: return launch_conv_t<R, 3, 8>(p, ex);
    case 5: return launch_conv_t<R, 5, 8>(p, ex);
    case 8: return launch_conv_t<R, 8, 4>(p, ex);
    case 9: return launch_conv_t<R, 9, 4>(p, ex);
    default: return SOI_ERR_UNSUPPORTED;
  }
}

int jr_for(int nmu) { return nmu >= 8 ? 4 : 8; }
bool nmu_supported(int nmu) { return nmu == 2 || nmu == 3 || nmu == 5 || nmu == 8 || nmu == 9; }

template <typename R>
int launch_seg_t(Plan &p, const Exec &ex)
{
  SegArgs a;
  a.T = ex.T; a.out = ex.out; a.seg_lo = ex.lo;
  cudaStream_t st = ex.st;
  a.tw1 = p.d_tw1; a.perm1 = p.d_perm1; a.plan1 = p.plan1;
  a.tw2 = p.d_tw2; a.perm2 = p.d_perm2; a.plan2 = p.plan2;
  a.xtw_lo = p.d_xlo; a.xtw_hi = p.d_xhi; a.winv = p.d_winv; a.wsmall = p.d_wsmall;
  a.Mh = (long long)p.Mh; a.M = (long long)p.M;
  a.M1 = p.M1; a.M2 = p.M2; a.C1 = p.C1; a.C2 = p.C2; a.lo_bits = p.lo_bits;
  CK(cudaFuncSetAttribute(k_seg_cols<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_c));
  CK(cudaFuncSetAttribute(k_seg_rows_demod<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_r));
  dim3 g1((unsigned)(p.M2 / p.C1), (unsigned)(ex.hi - ex.lo));
  k_seg_cols<R><<<g1, 256, p.smem_c, st>>>(a);
  CK(cudaGetLastError());
  dim3 g2((unsigned)(p.M1 / p.C2), (unsigned)(ex.hi - ex.lo));
  k_seg_rows_demod<R><<<g2, 256, p.smem_r, st>>>(a);
  CK(cudaGetLastError());
  return SOI_OK;
}

// Register-DFT twiddles in constant memory (long double, rounded once).
// Every kernel built on RegDFT reads them, so every plan uploads them to its
// device.
int upload_regtw()
{
  std::vector<float2> tf(kRegTwTotal);
  std::vector<double2> td(kRegTwTotal);
  for (int F : kRegSizes) {
    const int off = reg_tw_offset(F);
    for (int m = 0; m < F; ++m) {
      long double ang = -2.0L * kPi * (long double)m / (long double)F;
      tf[off + m] = make_float2((float)cosl(ang), (float)sinl(ang));
      td[off + m] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
  }
  CK(cudaMemcpyToSymbol(c_regtw_f, tf.data(), tf.size() * sizeof(float2)));
  CK(cudaMemcpyToSymbol(c_regtw_d, td.data(), td.size() * sizeof(double2)));
  return SOI_OK;
}

// ---- stage 2 with compile-time geometry ----------------------------------------

using S2KernelCT = void (*)(S2ArgsCT, const CUtensorMap);
struct S2ChoiceCT { int M1, M2, elem, nt, C; int ra[3], rb[3]; int boxr; size_t smem; S2KernelCT k; };

// one instance: pass-1 radices (a0, a1, a2), pass-2 radices (b0, b1, b2),
// NT threads, C columns per task, at least MINB CTAs per SM (register bound)
#define SOI_S2CTV(R, a0, a1, a2, b0, b1, b2, NT, C, MINB)                                         \
  { a0 * a1 * a2, b0 * b1 * b2, (int)sizeof(typename cplx_of<R>::type), NT, C, { a0, a1, a2 }, { b0, b1, b2 }, \
    S2Geom<R, a0, a1, a2, b0, b1, b2, NT, C>::BOXR,                                             \
    (size_t)S2Geom<R, a0, a1, a2, b0, b1, b2, NT, C>::BUF * S2Geom<R, a0, a1, a2, b0, b1, b2, NT, C>::E, \
    k_stage2_ct<R, a0, a1, a2, b0, b1, b2, NT, C, MINB> }
// the default instance: 256 threads, a whole 32-byte sector per row run, two CTAs per SM
#define SOI_S2CT(R, a0, a1, a2, b0, b1, b2) \
  SOI_S2CTV(R, a0, a1, a2, b0, b1, b2, 256, 32 / (int)sizeof(typename cplx_of<R>::type), 2)

const S2ChoiceCT kS2CT[] = {
  SOI_S2CT(float, 10, 16, 16, 8, 16, 16),   // M' = 2560 x 2048 (N = 2^29, S = 128; 2^28, 64)
  SOI_S2CT(float, 10, 16, 16, 4, 16, 16),   // 2560 x 1024
  SOI_S2CT(float, 5, 16, 16, 4, 16, 16),    // 1280 x 1024
  SOI_S2CT(float, 5, 16, 16, 8, 8, 8),      // 1280 x 512
  SOI_S2CT(float, 10, 8, 8, 4, 16, 16),     // 640 x 1024
  SOI_S2CT(float, 10, 8, 8, 8, 8, 8),       // 640 x 512
  SOI_S2CT(float, 5, 8, 8, 8, 8, 8),        // 320 x 512
  SOI_S2CT(float, 5, 8, 8, 4, 8, 8),        // 320 x 256
  SOI_S2CT(float, 8, 16, 16, 8, 16, 16),    // 2048 x 2048 (mu = 8/7: N = 7*2^26, S = 128)
  SOI_S2CT(float, 9, 16, 16, 8, 16, 16),    // 2304 x 2048 (mu = 9/8: N = 2^29, S = 128)
  SOI_S2CT(float, 8, 8, 8, 4, 16, 16),      // 512 x 1024  (mu = 8/7: N = 7*2^23, S = 128)
  SOI_S2CT(float, 9, 8, 16, 8, 8, 8),       // 1152 x 512  (mu = 9/8: N = 2^26, S = 128)
  SOI_S2CT(double, 10, 16, 16, 8, 16, 16),
  SOI_S2CT(double, 10, 16, 16, 4, 16, 16),
  SOI_S2CT(double, 5, 16, 16, 4, 16, 16),
  SOI_S2CT(double, 5, 16, 16, 8, 8, 8),
  SOI_S2CT(double, 10, 8, 8, 4, 16, 16),
  SOI_S2CT(double, 10, 8, 8, 8, 8, 8),
  SOI_S2CT(double, 5, 8, 8, 8, 8, 8),
  SOI_S2CT(double, 5, 8, 8, 4, 8, 8),
  SOI_S2CT(double, 8, 16, 16, 8, 16, 16),
  SOI_S2CT(double, 9, 16, 16, 8, 16, 16),
  SOI_S2CT(double, 8, 8, 8, 4, 16, 16),
  SOI_S2CT(double, 9, 8, 16, 8, 8, 8),
};
#undef SOI_S2CT
#undef SOI_S2CTV

// index into kS2CT for M' and the element size, or -1
int pick_s2ct(const Plan &p)
{
  // SOI_STAGE2_FAST=0 (or the tuner) selects the two-kernel path
  if (p.knob_s2 == 0 || (p.knob_s2 < 0 && env_int("SOI_STAGE2_FAST", 1) == 0)) return -1;
  for (int i = 0; i < (int)(sizeof(kS2CT) / sizeof(kS2CT[0])); ++i)
    if ((long long)kS2CT[i].M1 * kS2CT[i].M2 == (long long)p.Mh && kS2CT[i].elem == (int)p.elem) return i;
  return -1;
}

// Twiddles of a tile FFT with radices (r0, r1, r2) over L = r0*r1*r2 points,
// in the order the warps read them (8 consecutive butterflies of a warp read
// 8 consecutive entries, one cache line): first stage w_L^(i*k) at
// [(k-1)*span0 + i], span0 = L/r0; second stage (r2 > 1) w_L^(i*k*r0) at
// [(r0-1)*span0 + (k-1)*r2 + i].  Same values as roots_table(L).
template <typename R>
std::vector<R> tile_twiddles(int r0, int r1, int r2)
{
  const long long L = (long long)r0 * r1 * r2, span0 = L / r0;
  std::vector<R> t;
  auto push = [&](long long m) {
    long double a = -2.0L * kPi * (long double)m / (long double)L;
    t.push_back((R)cosl(a));
    t.push_back((R)sinl(a));
  };
  for (int k = 1; k < r0; ++k)
    for (long long i = 0; i < span0; ++i) push(i * k);
  if (r2 > 1)
    for (int k = 1; k < r1; ++k)
      for (long long i = 0; i < r2; ++i) push(i * k * r0);
  return t;
}

// Output k2 of pass 2's last radix stage at store position pos = blk + nb*j
// (butterfly blk of nb = M2/RL, its output j), for radices (b0, b1, b2).
inline long long pass2_k2(const int *rb, long long pos)
{
  const long long M2 = (long long)rb[0] * rb[1] * rb[2];
  const long long RL = rb[2] > 1 ? rb[2] : rb[1], nb = M2 / RL;
  const long long blk = pos % nb, j = pos / nb;
  const long long fbase = rb[2] > 1 ? blk / rb[1] + rb[0] * (blk % rb[1]) : blk;
  return fbase + nb * j;
}

// Tables of the persistent stage 2.  Demodulation: amp(k) = 1/y_W(k/M - 1/2)
// (even about M/2) and exp(-i pi kappa k/M) = ph(k1) * ph(M1*k2), ph(k1) two-level
// in FP64, ph(M1*k2) per k2.  amp and ph(M1*k2) are stored in the order pass 2's
// last radix stores its outputs: for the task of rows k1 = C*t .. C*t + C-1,
// amp[(t*M2 + pos)*C + col] is amp at k = C*t + col + M1*k2(pos), and
// ph2[pos] is ph(M1*k2(pos)), so that a warp's loads are one cache line each.
// Tile twiddles of both passes in warp read order (tile_twiddles).
template <typename R>
int build_ct_tables(Plan &p, const S2ChoiceCT &c)
{
  const size_t M = p.M, half = M / 2 + 1;
  const long double sq = sqrtl((long double)p.sigma);
  std::vector<R> af(half);
  for (size_t i = 0; i < half; ++i) {
    long double t = (long double)i / (long double)M - 0.5L;
    long double y = !p.cw_freq.empty() ? (long double)p.cw_freq[i]
                                       : (erfcl(sq * (t - p.tau / 2.0L)) - erfcl(sq * (t + p.tau / 2.0L))) / (2.0L * p.tau);
    af[i] = (R)(1.0L / y);
  }
  const long long M1 = c.M1, M2 = c.M2, C = c.C;
  std::vector<long long> k2of(M2);
  for (long long pos = 0; pos < M2; ++pos) k2of[pos] = pass2_k2(c.rb, pos);
  std::vector<R> amp((size_t)M1 * M2);
  for (long long t = 0; t < M1 / C; ++t)
    for (long long pos = 0; pos < M2; ++pos)
      for (long long col = 0; col < C; ++col) {
        const long long k = C * t + col + M1 * k2of[pos];
        const long long km = k >= (long long)M ? 0 : std::min(k, (long long)M - k);
        amp[(size_t)((t * M2 + pos) * C + col)] = af[(size_t)km];
      }
  int rc;
  if ((rc = upload(&p.d_amp, amp.data(), amp.size() * sizeof(R)))) return rc;
  const long long kappa = (long long)p.B - p.dmu;
  auto phase = [&](long long k, long double *o) {
    long long q = (long long)(((unsigned long long)kappa * (unsigned long long)k) % (2ULL * M));
    long double ang = -kPi * (long double)q / (long double)M;
    o[0] = cosl(ang);
    o[1] = sinl(ang);
  };
  const long long nlo = 1LL << p.dlo_bits, nhi = (long long)(M >> p.dlo_bits) + 2;
  std::vector<double> lo(2 * nlo), hi(2 * nhi);
  long double o[2];
  for (long long e = 0; e < nlo; ++e) { phase(e, o); lo[2 * e] = (double)o[0]; lo[2 * e + 1] = (double)o[1]; }
  for (long long h = 0; h < nhi; ++h) { phase(h * nlo, o); hi[2 * h] = (double)o[0]; hi[2 * h + 1] = (double)o[1]; }
  if ((rc = upload((void **)&p.d_dlo, lo.data(), lo.size() * sizeof(double)))) return rc;
  if ((rc = upload((void **)&p.d_dhi, hi.data(), hi.size() * sizeof(double)))) return rc;
  std::vector<R> ph(2 * (size_t)M2);
  for (long long pos = 0; pos < M2; ++pos) {
    phase(M1 * k2of[pos], o);
    ph[2 * pos] = (R)o[0];
    ph[2 * pos + 1] = (R)o[1];
  }
  if ((rc = upload(&p.d_ph2, ph.data(), ph.size() * sizeof(R)))) return rc;
  // pass-1 epilogue: base w_{M'}^(m2*fbase(blk)) at [(t*NB + blk)*C + col]
  // (m2 = C*t + col, NB = M1/RL butterflies of the last radix) and steps
  // w_{M'}^(m2*(M1/RL)*k) at [m2*RL + k], in long double, rounded once
  {
    const long long RLA = c.ra[2] > 1 ? c.ra[2] : c.ra[1], NB = M1 / RLA, Mp = M1 * M2;
    auto root = [&](long long e, R *o) {
      long double ang = -2.0L * kPi * (long double)(e % Mp) / (long double)Mp;
      o[0] = (R)cosl(ang);
      o[1] = (R)sinl(ang);
    };
    std::vector<R> bt(2 * (size_t)M2 * NB), st(2 * (size_t)M2 * RLA);
    for (long long t = 0; t < M2 / C; ++t)
      for (long long blk = 0; blk < NB; ++blk) {
        const long long fbase = c.ra[2] > 1 ? blk / c.ra[1] + c.ra[0] * (blk % c.ra[1]) : blk;
        for (long long col = 0; col < C; ++col) root((C * t + col) * fbase, &bt[2 * (size_t)((t * NB + blk) * C + col)]);
      }
    for (long long m2 = 0; m2 < M2; ++m2)
      for (long long k = 0; k < RLA; ++k) root(m2 * NB * k, &st[2 * (size_t)(m2 * RLA + k)]);
    if ((rc = upload(&p.d_base1, bt.data(), bt.size() * sizeof(R)))) return rc;
    if ((rc = upload(&p.d_step1, st.data(), st.size() * sizeof(R)))) return rc;
  }
  std::vector<R> w1 = tile_twiddles<R>(c.ra[0], c.ra[1], c.ra[2]), w2 = tile_twiddles<R>(c.rb[0], c.rb[1], c.rb[2]);
  if ((rc = upload(&p.d_ctw1, w1.data(), w1.size() * sizeof(R)))) return rc;
  if ((rc = upload(&p.d_ctw2, w2.data(), w2.size() * sizeof(R)))) return rc;
  return SOI_OK;
}

int setup_s2ct(Plan &p, int idx)
{
  const S2ChoiceCT &c = kS2CT[idx];
  p.M1 = c.M1; p.M2 = c.M2;
  p.C1 = p.C2 = c.C;
  p.f2_nt = c.nt;
  p.f2_boxr = c.boxr;
  p.f2_smem = c.smem;
  p.f2ct_kernel = c.k;
  CK(cudaFuncSetAttribute(c.k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.f2_smem));
  int occ = 0, nsm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, c.k, c.nt, p.f2_smem));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, p.device));
  if (occ < 1) return SOI_ERR_UNSUPPORTED;
  p.f2_grid = occ * nsm;
  {
    // schedule tail: a segment's pass-2 tasks must not be claimed before its
    // last pass-1 task has had time to finish, about one task per resident
    // CTA later; ending each block with that many pass-2 tasks keeps most
    // waits away while the rest of the block interleaves the two passes.
    // Measured in the split form: N = 2^29 (NT2 = 640) 5.90 ms with a tail of
    // 296 (the grid), 6.18 with 640, 6.00 with 150; N = 2^26 (NT2 = 320) 0.98
    // ms with 320, 1.11 with 296.  With every CTA holding one claimed task
    // ahead of the running one, a block needs about two tasks per CTA of
    // pass 2 for the interleave to pay; smaller blocks, and FP64 (8.54 ms
    // interleaved against 8.22-8.29 at N = 2^28), keep every pass-1 task of a
    // block ahead of its pass-2 tasks (tail = NT2).
    const int nt2 = c.M1 / c.C;
    const int dflt = (p.prec == SOI_PRECISION_FP64 || nt2 < 2 * p.f2_grid) ? nt2 : p.f2_grid;
    const int tail = env_int("SOI_STAGE2_TAIL", dflt);
    p.f2_tail = tail < 0 ? 0 : tail > nt2 ? nt2 : tail;
  }
  int rc = p.prec == SOI_PRECISION_FP64 ? build_ct_tables<double>(p, c) : build_ct_tables<float>(p, c);
  if (rc) return rc;
  p.discard = env_int("SOI_STAGE2_DISCARD", 1);
  p.amp_keep = env_int("SOI_STAGE2_AMP_KEEP", 0) ? 1 : 0;
  // pass-2 rows by bulk copies: 5.64 vs 5.82 ms at N = 2^29, S = 128 (split),
  // 6.69 vs 7.01 ms at N = 2^28, S = 64 (FP64), bit-identical output;
  // SOI_STAGE2_BULK2=0 selects cp.async
  p.bulk2 = env_int("SOI_STAGE2_BULK2", 1) ? 1 : 0;
  // FP32 pass 2 with each thread on a pair of rows (tile_fft_rows2): the
  // twiddles, ph(M1*k2) and amplitude pairs loaded once for both rows, one
  // 16-byte store per output pair: 5.43 vs 5.63 ms at N = 2^29, S = 128;
  // SOI_STAGE2_ROWS2=0 selects one row per thread
  p.rows2 = env_int("SOI_STAGE2_ROWS2", 1) ? 1 : 0;
  // failure-detection test only: every pass-2 task then waits for one more
  // pass-1 completion than exists, runs out its iteration limit and the
  // compute returns SOI_ERR_TIMEOUT
  p.wait_extra = env_int("SOI_TEST_STAGE2_WAIT_EXTRA", 0) ? 1 : 0;
  p.fast2 = 3;
  return SOI_OK;
}

int launch_s2ct(Plan &p, const Exec &ex)
{
  S2ArgsCT a;
  a.T = ex.T; a.out = ex.out; a.tw1 = p.d_ctw1; a.tw2 = p.d_ctw2; a.base1 = p.d_base1; a.step1 = p.d_step1;
  a.amp = p.d_amp; a.dlo = p.d_dlo; a.dhi = p.d_dhi; a.ph2 = p.d_ph2;
  a.dlo_bits = p.dlo_bits; a.M = (int)p.M;
  a.S = ex.hi - ex.lo; a.seg_lo = ex.lo;
  a.discard = p.discard;
  a.wait_extra = p.wait_extra;
  a.tail = p.f2_tail;
  a.amp_keep = p.amp_keep;
  a.bulk2 = p.bulk2;
  // row pairs store outputs k, k + 1 (k even) as one 16-byte store: M even
  // and the output 16-byte aligned, else one row per thread
  a.rows2 = p.rows2 && p.M % 2 == 0 && p.M1 % 2 == 0 && ((uintptr_t)ex.out & 15) == 0 ? 1 : 0;
  a.err = (int *)ex.sync; a.counter = ex.sync + 1; a.done1 = ex.sync + 2;
  // counters restart; the error flag stays set until the owner clears it
  CK(cudaMemsetAsync(ex.sync + 1, 0, (size_t)(a.S + 1) * sizeof(unsigned int), ex.st));
  a.tma = ex.tmap ? 1 : 0;
  CUtensorMap none;
  memset(&none, 0, sizeof none);
  p.f2ct_kernel<<<p.f2_grid, p.f2_nt, p.f2_smem, ex.st>>>(a, ex.tmap ? *ex.tmap : none);
  CK(cudaGetLastError());
  return SOI_OK;
}

// Error word of an execution (a stage-1 staging wait or a stage-2
// dependency wait that gave up); synchronises the stream.
int check_stage2(Plan &p, const unsigned int *sync, cudaStream_t st)
{
  (void)p;
  if (!sync) return SOI_OK;
  int err = 0;
  CK(cudaMemcpyAsync(&err, sync, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return err ? SOI_ERR_TIMEOUT : SOI_OK;
}

template <typename R, int NMU, int JR>
int launch_conv2_t(Plan &p, const Exec &ex)
{
  Conv2Args a;
  a.alpha = ex.in; a.T = ex.T; a.seg_lo = ex.lo; a.seg_hi = ex.hi; a.filt = p.d_filt2; a.phase = p.d_phase; a.twS = p.d_twS;
  a.permS = p.d_permS; a.wsmall = p.d_wsmall; a.planS = p.planS;
  a.M = (long long)p.M; a.Mh = (long long)p.Mh; a.J = (long long)p.J;
  a.S = (int)p.S; a.d = p.dmu; a.atap = p.atap; a.JT = p.JT2; a.pitch = p.pitch; a.AC = p.AC;
  a.buf_elems = p.buf_elems;
  auto kern = k_conv_sfft_staged<R, NMU, JR>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem1b));
  dim3 grid((unsigned)((p.J + p.JT2 - 1) / p.JT2));
  kern<<<grid, 512, p.smem1b, ex.st>>>(a);
  CK(cudaGetLastError());
  return SOI_OK;
}

// staged stage-1 instances: (precision, n_mu) -> JR
int staged_jr(int prec, int nmu)
{
  if (prec == SOI_PRECISION_SPLIT_FP32) return nmu == 5 ? 8 : nmu == 3 ? 6 : (nmu == 8 || nmu == 9) ? 4 : 0;
  return nmu == 5 ? 4 : nmu == 3 ? 4 : (nmu == 8 || nmu == 9) ? 2 : 0;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// The stage-1 input as a 3-D tensor [J][d][S values] of 8-byte elements
// (a split complex is one element, an FP64 complex two), with boxes of
// JT + AC - 1 rows of one branch: one phase's rows x_b[j0 + a_lo + t] =
// alpha row d*(j0 + a_lo + t) + b.  False when the encoder refuses (the
// input's address or the sizes break the tensor-copy rules); the kernel then
// copies row by row.
bool input_rows_map(const Plan &p, const void *in, CUtensorMap *map)
{
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  const size_t e8 = p.elem / 8;
  const size_t nr = (size_t)p.JT2 + p.AC - 1;
  if (!enc || !in || p.S * e8 > 256 || nr > 256 || p.J > (size_t)INT32_MAX) return false;
  const cuuint64_t dims[3] = { (cuuint64_t)(p.S * e8), (cuuint64_t)p.dmu, (cuuint64_t)p.J };
  const cuuint64_t strides[2] = { (cuuint64_t)(p.S * p.elem), (cuuint64_t)(p.dmu * p.S * p.elem) };
  const cuuint32_t box[3] = { (cuuint32_t)(p.S * e8), 1, (cuuint32_t)nr };
  const cuuint32_t estr[3] = { 1, 1, 1 };
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, const_cast<void *>(in), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename R, int NMU, int JR, int R0, int R1, int NT, bool BULK>
int launch_conv_tS(Plan &p, const Exec &ex)
{
  Conv2Args a;
  a.alpha = ex.in; a.T = ex.T; a.seg_lo = ex.lo; a.seg_hi = ex.hi; a.filt = p.d_filt2; a.phase = p.d_phase; a.twS = p.d_twS;
  a.permS = p.d_permS; a.wsmall = p.d_wsmall; a.planS = p.planS;
  a.M = (long long)p.M; a.Mh = (long long)p.Mh; a.J = (long long)p.J;
  a.S = (int)p.S; a.d = p.dmu; a.atap = p.atap; a.JT = p.JT2; a.pitch = p.pitch; a.AC = p.AC;
  a.buf_elems = p.buf_elems;
  a.err = (int *)ex.sync;
  CUtensorMap rmap;
  memset(&rmap, 0, sizeof rmap);
  if (BULK) a.tma_rows = input_rows_map(p, ex.in, &rmap) ? 1 : 0;
  auto kern = k_conv_sfft_tS<R, NMU, JR, R0, R1, NT, BULK>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem1b));
  dim3 grid((unsigned)((p.J + p.JT2 - 1) / p.JT2));
  kern<<<grid, NT, p.smem1b, ex.st>>>(a, rmap);
  CK(cudaGetLastError());
  return SOI_OK;
}

// compile-time-S instances: n_mu = 5, S in {8..256} (R0*R1 split of S)
template <typename R, int JR, int NT, bool BULK>
int launch_tS_switch_nt(Plan &p, const Exec &ex)
{
  switch (p.S) {
    case 8: return launch_conv_tS<R, 5, JR, 2, 4, NT, BULK>(p, ex);
    case 16: return launch_conv_tS<R, 5, JR, 4, 4, NT, BULK>(p, ex);
    case 32: return launch_conv_tS<R, 5, JR, 4, 8, NT, BULK>(p, ex);
    case 64: return launch_conv_tS<R, 5, JR, 8, 8, NT, BULK>(p, ex);
    case 128: return launch_conv_tS<R, 5, JR, 8, 16, NT, BULK>(p, ex);
    case 256: return launch_conv_tS<R, 5, JR, 16, 16, NT, BULK>(p, ex);
  }
  return SOI_ERR_UNSUPPORTED;
}

template <typename R, int JR>
int launch_tS_switch(Plan &p, const Exec &ex)
{
  if (p.s1_nt == 256)
    return p.s1_bulk ? launch_tS_switch_nt<R, JR, 256, true>(p, ex) : launch_tS_switch_nt<R, JR, 256, false>(p, ex);
  return p.s1_bulk ? launch_tS_switch_nt<R, JR, 512, true>(p, ex) : launch_tS_switch_nt<R, JR, 512, false>(p, ex);
}

bool tS_available(const Plan &p)
{
  if (p.nmu != 5 || env_int("SOI_STAGE1_TS", 1) == 0) return false;
  return p.S == 8 || p.S == 16 || p.S == 32 || p.S == 64 || p.S == 128 || p.S == 256;
}

// last radix of the compile-time-S split (the tile layout pads every R1)
int tS_r1(size_t S) { return S == 8 ? 4 : S == 16 ? 4 : S == 32 ? 8 : S == 64 ? 8 : 16; }

int launch_conv2(Plan &p, const Exec &ex)
{
  if (p.s1_tS)
    return p.prec == SOI_PRECISION_SPLIT_FP32 ? launch_tS_switch<float, 8>(p, ex)
                                              : launch_tS_switch<double, 4>(p, ex);
  if (p.prec == SOI_PRECISION_SPLIT_FP32) {
    switch (p.nmu) {
      case 5: return launch_conv2_t<float, 5, 8>(p, ex);
      case 3: return launch_conv2_t<float, 3, 6>(p, ex);
      case 8: return launch_conv2_t<float, 8, 4>(p, ex);
      case 9: return launch_conv2_t<float, 9, 4>(p, ex);
    }
  } else {
    switch (p.nmu) {
      case 5: return launch_conv2_t<double, 5, 4>(p, ex);
      case 3: return launch_conv2_t<double, 3, 4>(p, ex);
      case 8: return launch_conv2_t<double, 8, 2>(p, ex);
      case 9: return launch_conv2_t<double, 9, 2>(p, ex);
    }
  }
  return SOI_ERR_UNSUPPORTED;
}

// tile geometry of the staged kernel; leaves s1fast = 0 when it does not apply
void plan_stage1_staged(Plan &p)
{
  p.s1fast = 0;
  if (env_int("SOI_STAGE1_FAST", 1) == 0) return;
  const int jr = staged_jr(p.prec, p.nmu);
  if (!jr || p.S > 512 || (p.S * p.nmu) % 4) return;
  const bool ts = tS_available(p);
  // compile-time-S kernel: 512 threads and 200 KB (one CTA per SM), or 256
  // threads and <= 110 KB (two CTAs per SM: one CTA's convolution overlaps
  // the other's S-point FFT and stores; smaller tiles, more halo rows per
  // output) where two thread rows fit.  Staged by tensor copies (one per
  // phase, issued by one thread onto an mbarrier) instead of every thread's
  // 16-byte cp.async, 256 threads measured fastest (stage 1 at N = 2^29,
  // S = 128: 5.36 ms against 5.52 at 512 threads and 5.77 / 6.09 with
  // cp.async; split S = 64 / 32 / 16 and FP64 S = 64 / 32 likewise), except
  // FP64 at S = 128 (6.30 ms at 512 against 6.37).  The batch tuner tries both.
  // A phase's rows are one tensor-copy box: at most 256 values of 8 bytes
  // per row and 256 rows, so wider rows stay with cp.async and the tile
  // search below keeps JT + B/d - 1 <= 256.  Rows of 64 bytes (split, S = 8)
  // measured faster with cp.async (2^24: 0.179 vs 0.205 ms; 2^20: 0.022 vs
  // 0.050), and 256 threads there too.
  const bool bulk = ts && (p.knob_s1_bulk >= 0 ? p.knob_s1_bulk : env_int("SOI_STAGE1_BULK", 1)) != 0 &&
                    p.S * (p.elem / 8) <= 256 && p.S * p.elem >= 128;
  int nt = 512;
  if (ts && 2 * (int)p.S <= 256) {
    const int dflt = p.prec == SOI_PRECISION_FP64 && p.S == 128 ? 512 : (bulk || p.S <= 64) ? 256 : 512;
    nt = (p.knob_s1_nt > 0 ? p.knob_s1_nt : env_int("SOI_STAGE1_NT", dflt)) == 256 ? 256 : 512;
  }
  const int groups = nt / (int)p.S;
  // tensor-copy staging: buffers on 128-byte boundaries, 128 bytes of
  // alignment slack
  const size_t align = bulk ? 128 : 16;
  const size_t budget = (nt == 256 ? 110 * 1024 : 200 * 1024) - p.S * (p.elem + sizeof(int)) - (bulk ? 128 : 0);
  const size_t real = p.elem / 2;
  const size_t pitch = ts ? ((p.S + p.S / tS_r1(p.S)) | 1) : (size_t)p.pitch;
  for (int jt = groups * jr; jt >= jr; jt -= jr) {
    if ((long long)jt > (long long)p.J - p.atap - jt) continue;     // keep the wrap single-step
    if (bulk && jt + p.atap - 1 > 256) continue;               // every tap count fits one box
    for (int ac = p.atap; ac >= 1; --ac) {
      const size_t rows = (size_t)(jt + ac - 1) * p.S;
      const size_t fel = ((size_t)ac * p.nmu * p.S * real + p.elem - 1) / p.elem;
      size_t be = rows + fel;
      const size_t tile = (size_t)p.nmu * jt * pitch;
      be = std::max(be, (tile + 1) / 2);                        // the FFT tile aliases the buffers
      be = (be * p.elem + align - 1) / align * align / p.elem;   // both buffers start aligned
      if (2 * be * p.elem <= budget) {
        p.JR2 = jr; p.JT2 = jt; p.AC = ac; p.buf_elems = (int)be;
        p.smem1b = 2 * be * p.elem + p.S * (p.elem + sizeof(int)) + (bulk ? 128 : 0);
        p.s1fast = 1;
        p.s1_tS = ts ? 1 : 0;
        p.s1_nt = ts ? nt : 512;
        p.s1_bulk = bulk ? 1 : 0;
        return;
      }
    }
  }
}

// ---- tensor-core stage 1 --------------------------------------------------

constexpr int kTcKP = 72;      // taps of the compiled instances (B <= 72, zero beyond B)

// The tensor-core kernel applies to the split form with n = 5, d = 4, S in
// {32, 64, 128}, at most 72 taps and whole 32-group tiles; SOI_STAGE1_TC=1
// selects it (the packed-FMA kernel measured faster, so it is off by default).
bool tc_available(const Plan &p)
{
  if (p.prec != SOI_PRECISION_SPLIT_FP32 || p.nmu != 5 || p.dmu != 4) return false;
  if (!(p.S == 32 || p.S == 64 || p.S == 128)) return false;
  if ((size_t)p.atap * 4 > (size_t)kTcKP || p.J % 32 || p.J < 64) return false;
  return true;
}

// x rounded to 11 significant bits (TF32), ties away from zero like cvt.rna
long double tf32_round(long double x)
{
  if (x == 0) return 0;
  const int e = ilogbl(x);
  const long double sc = ldexpl(1.0L, 10 - e);
  return roundl(x * sc) / sc;
}

// B operand of every column: rows n = theta + 5*t' (t' = 0: F_hi, 1: F_lo;
// rows 10..15 zero) by KP taps q, K-major core matrices of 8 rows x 4 taps:
// byte offset (n/8)*(KP/4)*128 + (q/4)*128 + (n%8)*16 + (q%4)*4 within the
// column's 64*KP bytes.  F[q][theta][s] is the long-double filter tap q.
std::vector<float> tc_filter_table(const Plan &p, const std::vector<long double> &filt)
{
  const int KP = kTcKP, NA = KP / 4;
  std::vector<float> t((size_t)p.S * 16 * KP, 0.0f);
  for (size_t s = 0; s < p.S; ++s)
    for (int th = 0; th < p.nmu; ++th)
      for (int q = 0; q < KP && (size_t)q < p.B; ++q) {
        const long double F = filt[((size_t)q * p.nmu + th) * p.S + s];
        const long double hi = tf32_round(F), lo = tf32_round(F - hi);
        for (int tp = 0; tp < 2; ++tp) {
          const int n = th + 5 * tp;
          const size_t off = (size_t)(n / 8) * NA * 32 + (size_t)(q / 4) * 32 + (n % 8) * 4 + (q % 4);
          t[s * 16 * KP + off] = (float)(tp ? lo : hi);
        }
      }
  return t;
}

template <int R0, int R1>
int launch_tc_t(Plan &p, const Exec &ex)
{
  using Gm = TcGeom<R0, R1, kTcKP>;
  Conv2Args a;
  memset(&a, 0, sizeof a);
  a.alpha = ex.in; a.T = ex.T; a.seg_lo = ex.lo; a.seg_hi = ex.hi; a.phase = p.d_phase; a.twS = p.d_twS;
  a.M = (long long)p.M; a.Mh = (long long)p.Mh; a.J = (long long)p.J;
  a.S = (int)p.S; a.d = p.dmu; a.atap = p.atap; a.JT = Gm::JT;
  a.err = (int *)ex.sync;
  auto kern = k_conv_sfft_tc<R0, R1, kTcKP>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Gm::SMEM));
  kern<<<(unsigned)(p.J / Gm::JT), Gm::NT, Gm::SMEM, ex.st>>>(a, (const float *)p.d_btc);
  CK(cudaGetLastError());
  return SOI_OK;
}

int launch_tc(Plan &p, const Exec &ex)
{
  switch (p.S) {
    case 32: return launch_tc_t<4, 8>(p, ex);
    case 64: return launch_tc_t<8, 8>(p, ex);
    case 128: return launch_tc_t<8, 16>(p, ex);
  }
  return SOI_ERR_UNSUPPORTED;
}

int run_stage1(Plan &p, const Exec &ex)
{
  if (p.s1_tc) return launch_tc(p, ex);
  if (p.s1fast) return launch_conv2(p, ex);
  return p.prec == SOI_PRECISION_FP64 ? launch_conv_r<double>(p, ex) : launch_conv_r<float>(p, ex);
}

int run_stage2(Plan &p, const Exec &ex)
{
  if (p.fast2) return launch_s2ct(p, ex);
  return p.prec == SOI_PRECISION_FP64 ? launch_seg_t<double>(p, ex) : launch_seg_t<float>(p, ex);
}

int run_vlc(Plan &p, const Exec &ex);

// ---- plan construction -------------------------------------------------------

int validate(const soi_desc_t *d, size_t k)
{
  if (!d) return SOI_ERR_INVALID;
  if (d->P != 1 || d->rank != 0) return SOI_ERR_UNSUPPORTED;
  if (k < 1 || d->N == 0 || d->n_mu < 1 || d->d_mu < 1 || d->B < (size_t)d->d_mu) return SOI_ERR_INVALID;
  if (d->precision != SOI_PRECISION_FP64 && d->precision != SOI_PRECISION_SPLIT_FP32) return SOI_ERR_INVALID;
  size_t S = k;
  if (d->N % S) return SOI_ERR_INVALID;
  size_t M = d->N / S;
  if (M % (size_t)d->d_mu) return SOI_ERR_INVALID;              // M' = n*M/d integral
  if (M < d->B) return SOI_ERR_INVALID;                         // .cpp:89-94
  if (!nmu_supported(d->n_mu)) return SOI_ERR_UNSUPPORTED;
  if (S > 256 || S < 2) return SOI_ERR_UNSUPPORTED;
  return SOI_OK;
}

int choose_split(Plan &p)
{
  // M' = M1*M2; pass-1 tile M1 x C1, pass-2 tile M2 x C2; each <= ~110 KB and
  // C*elem >= 32 bytes (a full DRAM sector per row of the tile).
  const size_t budget = p.elem == 16 ? 200 * 1024 : 110 * 1024;
  const int cmin = (int)(32 / p.elem);
  long long best = -1;
  double bestscore = 1e300;
  const long long Mh = (long long)p.Mh;
  for (long long m1 = 2; m1 * 2 <= Mh; ++m1) {
    if (Mh % m1) continue;
    long long m2 = Mh / m1;
    if (m1 > 16384 || m2 > 16384) continue;
    FftPlan a, b;
    if (!make_fft_plan((int)m1, a) || !make_fft_plan((int)m2, b)) continue;
    if ((size_t)m1 * (cmin + 1) * p.elem > budget || (size_t)m2 * (cmin + 1) * p.elem > budget) continue;
    if (m2 % cmin || m1 % cmin) continue;
    double score = fabs(log((double)m1 / (double)m2) - 0.2);
    if (score < bestscore) { bestscore = score; best = m1; }
  }
  if (best < 0) return SOI_ERR_UNSUPPORTED;
  p.M1 = (int)best;
  p.M2 = (int)(Mh / best);
  p.C1 = cmin;
  p.C2 = cmin;
  // grow the column count while the tile stays in budget (fewer, fuller CTAs)
  while ((size_t)p.M1 * (2 * p.C1 + 1) * p.elem <= budget && p.M2 % (2 * p.C1) == 0 && p.C1 < 16) p.C1 *= 2;
  while ((size_t)p.M2 * (2 * p.C2 + 1) * p.elem <= budget && p.M1 % (2 * p.C2) == 0 && p.C2 < 16) p.C2 *= 2;
  make_fft_plan(p.M1, p.plan1);
  make_fft_plan(p.M2, p.plan2);
  p.smem_c = (size_t)p.M1 * (p.C1 + 1) * p.elem;
  p.smem_r = (size_t)p.M2 * (p.C2 + 1) * p.elem;
  return SOI_OK;
}

template <typename R>
int build_tables(Plan &p)
{
  std::vector<long double> filt, phr, phi, wir, wii;
  host_tables(p.N, p.S, p.nmu, p.dmu, p.B, p.tau, p.sigma, p.atap, &filt, &phr, &phi, &wir, &wii,
              p.cw_time.empty() ? nullptr : p.cw_time.data(), p.cw_freq.empty() ? nullptr : p.cw_freq.data());
  std::vector<R> f(filt.size());
  for (size_t i = 0; i < filt.size(); ++i) f[i] = (R)filt[i];
  std::vector<R> ph, wi;
  round_complex<R>(phr, phi, ph);
  round_complex<R>(wir, wii, wi);
  int rc;
  if ((rc = upload(&p.d_filt, f.data(), f.size() * sizeof(R)))) return rc;
  if (p.s1fast) {
    // branch-major copy for the staged kernel: [b][a][theta][s] = filt[d*a + b][theta][s]
    std::vector<R> f2((size_t)p.dmu * p.atap * p.nmu * p.S, (R)0);
    for (int b = 0; b < p.dmu; ++b)
      for (int aa = 0; aa < p.atap; ++aa) {
        const size_t kk = (size_t)p.dmu * aa + b;
        for (int th = 0; th < p.nmu; ++th)
          for (size_t sc = 0; sc < p.S; ++sc)
            f2[(((size_t)b * p.atap + aa) * p.nmu + th) * p.S + sc] = f[(kk * p.nmu + th) * p.S + sc];
      }
    if ((rc = upload(&p.d_filt2, f2.data(), f2.size() * sizeof(R)))) return rc;
  }
  if (p.s1_tc) {
    std::vector<float> bt = tc_filter_table(p, filt);
    if ((rc = upload(&p.d_btc, bt.data(), bt.size() * sizeof(float)))) return rc;
  }
  if ((rc = upload(&p.d_phase, ph.data(), ph.size() * sizeof(R)))) return rc;
  if ((rc = upload(&p.d_winv, wi.data(), wi.size() * sizeof(R)))) return rc;
  std::vector<R> tS = roots_table<R>((long long)p.S), t1 = roots_table<R>(p.M1), t2 = roots_table<R>(p.M2);
  std::vector<R> w7 = roots_table<R>(7);
  if ((rc = upload(&p.d_twS, tS.data(), tS.size() * sizeof(R)))) return rc;
  if ((rc = upload(&p.d_tw1, t1.data(), t1.size() * sizeof(R)))) return rc;
  if ((rc = upload(&p.d_tw2, t2.data(), t2.size() * sizeof(R)))) return rc;
  if ((rc = upload(&p.d_wsmall, w7.data(), w7.size() * sizeof(R)))) return rc;
  std::vector<int> pS = digit_reversal(p.planS), p1 = digit_reversal(p.plan1), p2 = digit_reversal(p.plan2);
  if ((rc = upload((void **)&p.d_permS, pS.data(), pS.size() * sizeof(int)))) return rc;
  if ((rc = upload((void **)&p.d_perm1, p1.data(), p1.size() * sizeof(int)))) return rc;
  if ((rc = upload((void **)&p.d_perm2, p2.data(), p2.size() * sizeof(int)))) return rc;
  // cross twiddles w_{M'}^e = hi[e >> lo_bits] * lo[e & mask], FP64
  const long long Mh = (long long)p.Mh;
  const long long nlo = 1LL << p.lo_bits, nhi = (Mh + nlo - 1) / nlo + 1;
  std::vector<double> lo(2 * nlo), hi(2 * nhi);
  for (long long e = 0; e < nlo; ++e) {
    long double a = -2.0L * kPi * (long double)(e % Mh) / (long double)Mh;
    lo[2 * e] = (double)cosl(a); lo[2 * e + 1] = (double)sinl(a);
  }
  for (long long h = 0; h < nhi; ++h) {
    long double a = -2.0L * kPi * (long double)((h * nlo) % Mh) / (long double)Mh;
    hi[2 * h] = (double)cosl(a); hi[2 * h + 1] = (double)sinl(a);
  }
  if ((rc = upload((void **)&p.d_xlo, lo.data(), lo.size() * sizeof(double)))) return rc;
  if ((rc = upload((void **)&p.d_xhi, hi.data(), hi.size() * sizeof(double)))) return rc;
  return SOI_OK;
}

void free_plan(Plan *p)
{
  if (!p) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(p->device);
  void *bufs[] = { p->d_filt, p->d_phase, p->d_twS, p->d_tw1, p->d_tw2, p->d_winv, p->d_wsmall,
                   p->d_permS, p->d_perm1, p->d_perm2, p->d_xlo, p->d_xhi, p->d_T, p->d_io, p->d_io2, p->d_io3,
                   p->d_vlc_words, p->d_vlc_n, p->d_vlc_emax, p->d_sync, p->d_filt2, p->d_amp, p->d_dlo, p->d_dhi, p->d_ph2, p->d_ctw1, p->d_ctw2, p->d_base1, p->d_step1, p->d_btc };
  for (void *b : bufs) if (b) cudaFree(b);
  for (auto &e : p->ev) if (e) cudaEventDestroy(e);
  for (auto &e : p->sev) if (e) cudaEventDestroy(e);
  if (p->st_in) cudaStreamDestroy(p->st_in);
  if (p->st_out) cudaStreamDestroy(p->st_out);
  if (p->own_stream && p->stream) cudaStreamDestroy(p->stream);
  cudaSetDevice(cur);
  delete p;
}

// Geometry of the plan (no CUDA calls): tile shapes, FFT factorisations.
int plan_geometry(const soi_desc_t *d, size_t k, Plan &p)
{
  int rc = validate(d, k);
  if (rc) return rc;
  p.device = d->device;
  p.prec = d->precision;
  p.elem = p.prec == SOI_PRECISION_FP64 ? 16 : 8;
  p.N = d->N; p.S = k; p.M = d->N / k; p.nmu = d->n_mu; p.dmu = d->d_mu;
  p.Mh = (size_t)p.nmu * p.M / (size_t)p.dmu; p.J = p.M / (size_t)p.dmu;
  p.B = d->B; p.tau = d->tau; p.sigma = d->sigma;
  p.atap = (int)((d->B + d->d_mu - 1) / d->d_mu);
  p.JR = jr_for(p.nmu);
  p.pitch = (int)p.S + 1;
  if (!make_fft_plan((int)p.S, p.planS)) return SOI_ERR_UNSUPPORTED;
  // stage-1 tile: JT output groups x all S columns, bounded by the thread
  // count (256 / S groups of JR), shared memory and the circular wrap
  long long jt = (long long)(256 / (int)p.S) * p.JR;
  const size_t budget1 = 200 * 1024 - p.S * (p.elem + sizeof(int));
  long long jt_smem = (long long)(budget1 / ((size_t)p.nmu * p.pitch * p.elem)) / p.JR * p.JR;
  long long jt_wrap = ((long long)p.J - p.atap - p.JR) / p.JR * p.JR;
  jt = std::min(jt, std::min(jt_smem, jt_wrap));
  if (jt < p.JR) return SOI_ERR_UNSUPPORTED;
  p.JT = (int)jt;
  p.smem1 = (size_t)p.nmu * p.JT * p.pitch * p.elem + p.S * (p.elem + sizeof(int));
  plan_stage1_staged(p);
  p.s1_tc = tc_available(p) && env_int("SOI_STAGE1_TC", 0) == 1 ? 1 : 0;
  const int ict = pick_s2ct(p);
  if (ict >= 0) {
    p.f2_variant = ict;
    p.M1 = kS2CT[ict].M1;
    p.M2 = kS2CT[ict].M2;
    p.C1 = p.C2 = kS2CT[ict].C;
    p.fast2 = 4;                 // chosen; set up when the device plan is built
    make_fft_plan(p.M1, p.plan1);
    make_fft_plan(p.M2, p.plan2);
    return SOI_OK;
  }
  return choose_split(p);
}

// A device plan for k segments of d's transform.  with_stream: the plan gets
// the descriptor's stream (or its own) and timing events, as a descriptor's
// plan; the batch driver's plans run on the batch's streams instead.
// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links no driver import library); null when the driver lacks it
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// The pass-1 tensor map of a persistent stage-2 plan over its own T: rows of
// 2*M2 values (M2 complex, M2*elem bytes apart), S*M1 rows (every segment),
// boxes of one 32-byte run (C complex) x f2_boxr rows, no swizzle: a box lands
// as f2_boxr packed 32-byte rows.  (With a swizzle mode each 32-byte row is
// laid out over the whole swizzle span, which the dense tile has no room
// for.)  The encoder checks base, strides and box against the hardware's
// rules; if it refuses, the kernel stages pass-1 tiles with cp.async.
// The pass-1 tensor map of a persistent stage-2 plan over the T buffer `T`
// (the plan's own, or a batch chain's); false where the plan stages pass 1
// with cp.async.  Measured against cp.async staging: 6.09 vs 6.36 ms at
// N = 2^29 (split), 0.99 vs 1.00 ms at 2^26, 8.09 vs 8.33 ms at 2^28 in FP64;
// SOI_STAGE2_TMA=0 selects cp.async (tests compare the two).
bool pass1_map(const Plan &p, void *T, CUtensorMap *map)
{
  if (p.fast2 != 3 || !T || p.f2_boxr <= 0 || !env_int("SOI_STAGE2_TMA", 1)) return false;
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const bool f64 = p.prec == SOI_PRECISION_FP64;
  const cuuint64_t dims[2] = { (cuuint64_t)2 * p.M2, (cuuint64_t)p.S * p.M1 };
  const cuuint64_t strides[1] = { (cuuint64_t)p.M2 * p.elem };
  const cuuint32_t box[2] = { (cuuint32_t)(32 / (f64 ? 8 : 4)), (cuuint32_t)p.f2_boxr };
  const cuuint32_t estr[2] = { 1, 1 };
  return enc(map, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, T, dims, strides, box,
             estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void make_pass1_map(Plan &p)
{
  p.tma1 = pass1_map(p, p.d_T, &p.tmap1);
}

int make_plan(const soi_desc_t *d, size_t k, int knob_s1_nt, int knob_s2, bool with_stream, Plan **out,
              const double *y_time = nullptr, const double *y_freq = nullptr)
{
  Plan *p = new Plan();
  p->knob_s1_nt = knob_s1_nt;
  p->knob_s2 = knob_s2;
  int rc = plan_geometry(d, k, *p);
  if (rc) { delete p; return rc; }
  if (y_time && y_freq) {
    p->cw_time.assign(y_time, y_time + p->B * (size_t)p->nmu * p->S);
    p->cw_freq.assign(y_freq, y_freq + p->M / 2 + 1);
    for (double v : p->cw_freq)
      if (!(v > 0) || !std::isfinite(v)) { delete p; return SOI_ERR_INVALID; }   // 1/y_W must exist
  }
  cudaError_t ce = cudaSetDevice(d->device);
  if (ce != cudaSuccess) { delete p; return SOI_ERR_CUDA; }
  rc = p->prec == SOI_PRECISION_FP64 ? build_tables<double>(*p) : build_tables<float>(*p);
  if (rc) { free_plan(p); return rc; }
  if ((rc = upload_regtw())) { free_plan(p); return rc; }
  // error word and stage-2 counters: [0] error flag, [1] task counter, [2 .. 2 + S) pass-1 counts
  if (cudaMalloc(&p->d_sync, (p->S + 2) * sizeof(unsigned int)) != cudaSuccess ||
      cudaMemset(p->d_sync, 0, (p->S + 2) * sizeof(unsigned int)) != cudaSuccess) {
    free_plan(p);
    return SOI_ERR_CUDA;
  }
  if (p->fast2 == 4) {
    p->fast2 = 0;
    if ((rc = setup_s2ct(*p, p->f2_variant))) { free_plan(p); return rc; }
  }
  if (!with_stream) {
    *out = p;
    return SOI_OK;
  }
  if (cudaMalloc(&p->d_T, p->S * p->Mh * p->elem) != cudaSuccess) { free_plan(p); return SOI_ERR_CUDA; }
  make_pass1_map(*p);
  if (d->stream) {
    p->stream = (cudaStream_t)d->stream;
  } else {
    // a blocking stream: it is ordered with the legacy default stream, so a
    // device input written there (a copy, a producer kernel) is complete
    // before stage 1 reads it, as the reference's synchronous compute_soi
    // implies; a non-blocking stream let stage 1 read the circular halo at
    // the end of an input that was still being written
    if (cudaStreamCreate(&p->stream) != cudaSuccess) { free_plan(p); return SOI_ERR_CUDA; }
    p->own_stream = true;
  }
  for (auto &e : p->ev)
    if (cudaEventCreate(&e) != cudaSuccess) { free_plan(p); return SOI_ERR_CUDA; }
  *out = p;
  return SOI_OK;
}

int init_plan(soi_desc_t *d, size_t k, const double *y_time = nullptr, const double *y_freq = nullptr)
{
  Plan *p = nullptr;
  int rc = make_plan(d, k, -1, -1, true, &p, y_time, y_freq);
  if (rc) return rc;
  d->plan = p;
  return SOI_OK;
}

Plan *plan_of(soi_desc_t *d) { return d ? (Plan *)d->plan : nullptr; }

// One transform: in -> out (they may alias, the reference's in-place form),
// for segments [seg_lo, seg_hi).  Host pointers are staged through the
// plan's device buffer.  With
// sync_after false the work is only enqueued (nothing waits on the stream,
// so it can be captured into a CUDA graph); soi_check_status reads the
// stage-2 error flag afterwards.
int compute_impl(soi_desc_t *d, const void *in, void *out, bool stage1_only, int seg_lo = 0, int seg_hi = -1,
                 bool sync_after = true)
{
  Plan *p = plan_of(d);
  if (!p) return SOI_ERR_NOT_INITIALISED;
  if (seg_hi < 0) seg_hi = (int)p->S;
  if (seg_lo < 0 || seg_hi > (int)p->S || seg_lo >= seg_hi) return SOI_ERR_INVALID;
  if (!sync_after && !d->device_ptr) return SOI_ERR_INVALID;     // host buffers need the copies to finish
  // stage 1 stages its input rows with 16-byte copies: a device input must
  // start on a 16-byte boundary (host inputs go through an aligned buffer)
  if (d->device_ptr && ((uintptr_t)in & 15)) return SOI_ERR_INVALID;
  if (cudaSetDevice(p->device) != cudaSuccess) return SOI_ERR_CUDA;
  cudaStream_t st = p->stream;
  const size_t bytes = p->N * p->elem;
  const void *src = in;
  void *dst = out;
  if (!d->device_ptr) {
    if (!p->d_io) CK(cudaMalloc(&p->d_io, bytes));
    CK(cudaMemcpyAsync(p->d_io, in, bytes, cudaMemcpyHostToDevice, st));
    src = p->d_io;
    dst = p->d_io;
  }
  int rc;
  const Exec ex{ src, p->d_T, dst, p->d_sync, seg_lo, seg_hi, st, p->tma1 ? &p->tmap1 : nullptr };
  CK(cudaMemsetAsync(p->d_sync, 0, sizeof(unsigned int), st));   // error flag
  if (p->timing) CK(cudaEventRecord(p->ev[0], st));
  if ((rc = run_stage1(*p, ex))) return rc;
  if (p->timing) CK(cudaEventRecord(p->ev[1], st));
  if (stage1_only) {
    if (!sync_after) return SOI_OK;
    CK(cudaStreamSynchronize(st));
    return check_stage2(*p, p->d_sync, st);
  }
  if (d->use_vlc && (rc = run_vlc(*p, ex))) return rc;
  if (p->timing) CK(cudaEventRecord(p->ev[2], st));
  if ((rc = run_stage2(*p, ex))) return rc;
  if (p->timing) CK(cudaEventRecord(p->ev[3], st));
  if (!d->device_ptr) {
    // only the computed segments are copied back
    const size_t seg_bytes = p->M * p->elem;
    CK(cudaMemcpyAsync((char *)out + seg_lo * seg_bytes, (const char *)p->d_io + seg_lo * seg_bytes,
                       (size_t)(seg_hi - seg_lo) * seg_bytes, cudaMemcpyDeviceToHost, st));
  }
  if (!sync_after) return SOI_OK;
  CK(cudaStreamSynchronize(st));
  if ((rc = check_stage2(*p, p->d_sync, st))) return rc;
  if (p->timing) {
    cudaEventElapsedTime(&p->ms[0], p->ev[0], p->ev[1]);
    cudaEventElapsedTime(&p->ms[2], p->ev[1], p->ev[2]);
    cudaEventElapsedTime(&p->ms[1], p->ev[2], p->ev[3]);
    cudaEventElapsedTime(&p->ms[3], p->ev[0], p->ev[3]);
  }
  return SOI_OK;
}

// ---- VLC on the transposed data (pfft.c:316-353, 390-447, 476-543, 618-632) --
// With one process the all-to-all is the identity, so the round trip is
// max_exponent per segment -> global max -> compress -> decompress, one chunk
// per segment (chunk length l = M'/P = M').
// VLC buffers of a plan (words, counts, exponents; the promoted copy in the
// split form), allocated once
int vlc_alloc(Plan &p)
{
  if (p.d_vlc_words) return SOI_OK;
  const size_t S = p.S;
  p.vlc_stride = (long)(4 * p.Mh + 64);
  CK(cudaMalloc(&p.d_vlc_words, (size_t)p.vlc_stride * S * sizeof(int)));
  CK(cudaMalloc(&p.d_vlc_n, S * sizeof(int)));
  CK(cudaMalloc(&p.d_vlc_emax, (S + 1) * sizeof(int)));
  return SOI_OK;
}

int run_vlc(Plan &p, const Exec &ex)
{
  const int len = (int)(2 * p.Mh);
  if (len % 16) return SOI_ERR_UNSUPPORTED;
  cudaStream_t st = ex.st;
  // the computed segments only (all S for a full transform)
  void *T = (char *)ex.T + (size_t)ex.lo * p.Mh * p.elem;
  const int ns = ex.hi - ex.lo;
  int rc;
  if ((rc = vlc_alloc(p))) return rc;
  // the split form's floats are read and written in place (widened to double
  // in the kernels, exactly), so no promoted copy is made
  CK(p.prec == SOI_PRECISION_FP64 ? vlc_max_exponent((const double *)T, len, ns, p.d_vlc_emax, st)
                                  : vlc_max_exponent((const float *)T, len, ns, p.d_vlc_emax, st));
  vlc_global_max<<<1, 256, 0, st>>>(p.d_vlc_emax, ns, p.d_vlc_emax + ns);
  CK(cudaGetLastError());
  dim3 gv(64, (unsigned)ns);
  if (p.prec == SOI_PRECISION_FP64) {
    vlc_compress_kernel<double><<<gv, 256, vlc_compress_smem(), st>>>((const double *)T, len, 0, p.d_vlc_emax + ns,
                                                                      p.d_vlc_emax, p.d_vlc_words, p.vlc_stride,
                                                                      p.d_vlc_n);
    CK(cudaGetLastError());
    vlc_decompress_kernel<double><<<gv, 256, vlc_decompress_smem(), st>>>(p.d_vlc_words, p.vlc_stride, len, 0,
                                                                          p.d_vlc_emax + ns, p.d_vlc_emax,
                                                                          (double *)T);
  } else {
    vlc_compress_kernel<float><<<gv, 256, vlc_compress_smem(), st>>>((const float *)T, len, 0, p.d_vlc_emax + ns,
                                                                     p.d_vlc_emax, p.d_vlc_words, p.vlc_stride,
                                                                     p.d_vlc_n);
    CK(cudaGetLastError());
    vlc_decompress_kernel<float><<<gv, 256, vlc_decompress_smem(), st>>>(p.d_vlc_words, p.vlc_stride, len, 0,
                                                                         p.d_vlc_emax + ns, p.d_vlc_emax,
                                                                         (float *)T);
  }
  CK(cudaGetLastError());
  return SOI_OK;
}

void die_on(int rc, const char *what)
{
  if (rc == SOI_OK) return;
  fprintf(stderr, "%s: %s\n", what, soi_status_string(rc));
  exit(-1);
}

// ---- batch driver ---------------------------------------------------------------
//
// Many independent transforms (of different lengths, segment counts and
// segment bands) as one CUDA graph.  One plan per distinct (N, k), shared by
// all transforms of that shape; with tuning, the plan is the fastest of its
// variants (stage-1 block size, persistent or two-kernel stage 2) timed on
// the first transform of that shape.  The transforms are spread over
// `chains` streams by estimated work (largest first onto the least-loaded
// chain); each chain has its own transposed-data scratch and stage-2
// synchronisation words, so chains run concurrently and the transforms of a
// chain run in order.  The graph forks the chains from the launch stream and
// joins them back.

struct BatchItem {
  size_t N, k;
  int lo, hi;
  const void *in;
  void *out;
  int plan = -1, chain = -1;
  double work = 0;
};

struct Batch {
  int device = 0;
  soi_desc_t tmpl{};
  std::vector<Plan *> plans;
  std::vector<BatchItem> items;
  int nchain = 1;
  std::vector<void *> T;
  std::vector<size_t> Tbytes;
  std::vector<unsigned int *> sync;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t last = nullptr;
  std::vector<float> tuned_ms;          // per plan: best time of the chosen variant (tuning on)
  std::vector<int> variant;             // per plan: 2 * (s1_nt == 256) + (persistent stage 2)
};

void batch_free(Batch *b)
{
  if (!b) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(b->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (void *t : b->T) if (t) cudaFree(t);
  for (unsigned int *q : b->sync) if (q) cudaFree(q);
  for (cudaStream_t s : b->streams) if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->joins) if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  for (Plan *p : b->plans) free_plan(p);
  cudaSetDevice(cur);
  delete b;
}

// enqueue one transform of the batch on its chain's stream
int batch_enqueue(Batch &b, const BatchItem &it)
{
  Plan &p = *b.plans[it.plan];
  // pass-1 tiles by tensor copies over this chain's T (the launch copies the
  // map into the kernel's parameters, so a local map outlives its use)
  CUtensorMap map;
  const bool tma = pass1_map(p, b.T[it.chain], &map);
  const Exec ex{ it.in, b.T[it.chain], it.out, b.sync[it.chain], it.lo, it.hi, b.streams[it.chain],
                 tma ? &map : nullptr };
  int rc;
  if ((rc = run_stage1(p, ex))) return rc;
  if (b.tmpl.use_vlc && (rc = run_vlc(p, ex))) return rc;
  return run_stage2(p, ex);
}

// time one plan variant on a transform (min of `reps` runs after a warm-up)
int batch_time_variant(Batch &b, Plan &p, const BatchItem &it, void *out, float *ms)
{
  cudaStream_t st = b.streams[0];
  CUtensorMap map;
  const bool tma = pass1_map(p, b.T[0], &map);
  const Exec ex{ it.in, b.T[0], out, b.sync[0], it.lo, it.hi, st, tma ? &map : nullptr };
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best = 1e30f;
  int rc = SOI_OK;
  for (int r = 0; r < 4 && rc == SOI_OK; ++r) {
    CK(cudaEventRecord(e0, st));
    rc = run_stage1(p, ex);
    if (rc == SOI_OK && b.tmpl.use_vlc) rc = run_vlc(p, ex);
    if (rc == SOI_OK) rc = run_stage2(p, ex);
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    if (r > 0) best = std::min(best, t);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc == SOI_OK) rc = check_stage2(p, b.sync[0], st);
  *ms = best;
  return rc;
}

int batch_build(Batch &b, int tune)
{
  // plans: one per distinct (N, k); tuning picks the fastest variant
  std::vector<std::pair<size_t, size_t>> shapes;
  for (auto &it : b.items) {
    size_t i = 0;
    while (i < shapes.size() && !(shapes[i].first == it.N && shapes[i].second == it.k)) ++i;
    if (i == shapes.size()) shapes.push_back({ it.N, it.k });
    it.plan = (int)i;
  }
  b.nchain = std::max(1, std::min(b.nchain, (int)b.items.size()));
  if (b.tmpl.use_vlc) b.nchain = 1;              // VLC buffers belong to the plan
  // chains: largest transforms first onto the least-loaded chain
  std::vector<int> order(b.items.size());
  for (size_t i = 0; i < order.size(); ++i) {
    order[i] = (int)i;
    BatchItem &it = b.items[i];
    it.work = (double)it.N * std::log2((double)it.N);
  }
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b.items[x].work > b.items[y].work; });
  std::vector<double> load(b.nchain, 0.0);
  std::vector<size_t> tmax(b.nchain, 0), smax(b.nchain, 0);
  for (int i : order) {
    int c = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    BatchItem &it = b.items[i];
    it.chain = c;
    load[c] += it.work;
    const size_t Mh = (size_t)b.tmpl.n_mu * (it.N / it.k) / (size_t)b.tmpl.d_mu;
    const size_t elem = b.tmpl.precision == SOI_PRECISION_FP64 ? 16 : 8;
    tmax[c] = std::max(tmax[c], it.k * Mh * elem);
    smax[c] = std::max(smax[c], it.k);
  }
  b.T.assign(b.nchain, nullptr);
  b.Tbytes = tmax;
  b.sync.assign(b.nchain, nullptr);
  b.streams.assign(b.nchain, nullptr);
  b.joins.assign(b.nchain, nullptr);
  for (int c = 0; c < b.nchain; ++c) {
    CK(cudaMalloc(&b.T[c], std::max<size_t>(tmax[c], 16)));
    CK(cudaMalloc(&b.sync[c], (smax[c] + 2) * sizeof(unsigned int)));
    CK(cudaMemset(b.sync[c], 0, (smax[c] + 2) * sizeof(unsigned int)));
    CK(cudaStreamCreateWithFlags(&b.streams[c], cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&b.joins[c], cudaEventDisableTiming));
  }
  CK(cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming));
  // tuning needs chain 0's scratch to hold every shape
  if (tune) {
    size_t need = 0;
    for (auto &it : b.items)
      need = std::max(need, it.k * ((size_t)b.tmpl.n_mu * (it.N / it.k) / (size_t)b.tmpl.d_mu) *
                                (b.tmpl.precision == SOI_PRECISION_FP64 ? 16 : 8));
    if (need > tmax[0]) {
      CK(cudaFree(b.T[0]));
      CK(cudaMalloc(&b.T[0], need));
      tmax[0] = need;
      b.Tbytes[0] = need;
    }
    size_t kmax = 0;
    for (auto &it : b.items) kmax = std::max(kmax, it.k);
    if (kmax > smax[0]) {
      CK(cudaFree(b.sync[0]));
      CK(cudaMalloc(&b.sync[0], (kmax + 2) * sizeof(unsigned int)));
      CK(cudaMemset(b.sync[0], 0, (kmax + 2) * sizeof(unsigned int)));
    }
  }
  void *scratch_out = nullptr;
  if (tune) {
    size_t nmax = 0;
    for (auto &it : b.items) nmax = std::max(nmax, it.N);
    CK(cudaMalloc(&scratch_out, nmax * (b.tmpl.precision == SOI_PRECISION_FP64 ? 16 : 8)));
  }
  int rc = SOI_OK;
  for (size_t si = 0; si < shapes.size() && rc == SOI_OK; ++si) {
    soi_desc_t d = b.tmpl;
    d.N = shapes[si].first;
    const BatchItem *first = nullptr;
    for (auto &it : b.items) if (it.plan == (int)si) { first = &it; break; }
    Plan *best = nullptr;
    float best_ms = 0;
    int best_var = 0;
    const int nts[2] = { 256, 512 }, s2s[2] = { 1, 0 };
    std::vector<int> tried;             // variant signatures already timed
    for (int a = 0; a < (tune ? 2 : 1) && rc == SOI_OK; ++a)
      for (int c = 0; c < (tune ? 2 : 1) && rc == SOI_OK; ++c) {
        Plan *p = nullptr;
        rc = make_plan(&d, shapes[si].second, tune ? nts[a] : -1, tune ? s2s[c] : -1, false, &p);
        if (rc) break;
        if (b.tmpl.use_vlc && (rc = vlc_alloc(*p))) { free_plan(p); break; }
        if (!tune) { best = p; break; }
        // a shape without a given variant falls back to another one: time each
        // distinct kernel choice once
        const int sig = (p->s1fast ? 1 : 0) + 2 * p->s1_tS + 4 * (p->s1_nt == 256) + 8 * (p->fast2 ? 1 : 0);
        if (std::find(tried.begin(), tried.end(), sig) != tried.end()) { free_plan(p); continue; }
        tried.push_back(sig);
        float ms = 0;
        rc = batch_time_variant(b, *p, *first, scratch_out, &ms);
        if (rc) { free_plan(p); break; }
        if (!best || ms < best_ms) {
          if (best) free_plan(best);
          best = p; best_ms = ms; best_var = 2 * (p->s1_nt == 256) + (p->fast2 ? 1 : 0);
        } else {
          free_plan(p);
        }
      }
    if (rc) { if (best) free_plan(best); break; }
    b.plans.push_back(best);
    b.tuned_ms.push_back(best_ms);
    b.variant.push_back(tune ? best_var : 2 * (best->s1_nt == 256) + (best->fast2 ? 1 : 0));
  }
  if (scratch_out) cudaFree(scratch_out);
  if (rc) return rc;
  CK(cudaDeviceSynchronize());
  // capture: fork every chain from the capture stream, enqueue, join
  cudaStream_t cap = nullptr;
  CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  rc = SOI_OK;
  if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = SOI_ERR_CUDA;
  if (rc == SOI_OK && cudaEventRecord(b.fork, cap) != cudaSuccess) rc = SOI_ERR_CUDA;
  for (int c = 0; c < b.nchain && rc == SOI_OK; ++c) {
    if (cudaStreamWaitEvent(b.streams[c], b.fork, 0) != cudaSuccess) { rc = SOI_ERR_CUDA; break; }
    // the error flag of a chain starts clear at every launch of the graph
    if (cudaMemsetAsync(b.sync[c], 0, sizeof(unsigned int), b.streams[c]) != cudaSuccess) rc = SOI_ERR_CUDA;
  }
  for (size_t i = 0; i < b.items.size() && rc == SOI_OK; ++i) rc = batch_enqueue(b, b.items[i]);
  for (int c = 0; c < b.nchain && rc == SOI_OK; ++c) {
    if (cudaEventRecord(b.joins[c], b.streams[c]) != cudaSuccess ||
        cudaStreamWaitEvent(cap, b.joins[c], 0) != cudaSuccess) rc = SOI_ERR_CUDA;
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(cap, &g);
  cudaStreamDestroy(cap);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (ce != cudaSuccess || !g) return SOI_ERR_CUDA;
  b.graph = g;
  CK(cudaGraphInstantiate(&b.exec, b.graph, 0));
  return SOI_OK;
}

}  // namespace

// ============================================================ C ABI ==========

extern "C" {

const char *soi_b200_version(void) { return "soi_b200 0.1 (sm_100a)"; }

const char *soi_status_string(int s)
{
  switch (s) {
    case SOI_OK: return "ok";
    case SOI_ERR_INVALID: return "invalid parameters";
    case SOI_ERR_UNSUPPORTED: return "configuration not supported by this build";
    case SOI_ERR_CUDA: return "CUDA runtime error";
    case SOI_ERR_NOT_INITIALISED: return "descriptor not initialised";
    case SOI_ERR_TIMEOUT: return "device-side wait timed out";
    default: return "unknown status";
  }
}

void set_default_soi_descriptor(soi_desc_t *d)
{
  memset(d, 0, sizeof(*d));
  d->n_mu = 5;                 // pfft.c:87-91
  d->d_mu = 4;
  d->tau = 928 / 1024.;
  d->sigma = 373.7314;
  d->B = 72;
  d->use_vlc = 0;              // pfft.c:93-94
  d->comm_to_comp_cost_ratio = 1;
  d->P = 1;
  d->rank = 0;
  d->precision = SOI_PRECISION_FP64;
}

int soi_init_status(soi_desc_t *d, soi_comm_t comm, cfft_size_t k)
{
  if (!d) return SOI_ERR_INVALID;
  d->comm = comm;
  d->k = k;
  if (d->plan) { free_plan((Plan *)d->plan); d->plan = nullptr; }
  int rc = init_plan(d, k);
  if (rc == SOI_OK) {
    free(d->segmentBoundaries);
    d->segmentBoundaries = (int *)malloc(sizeof(int) * 2);   // pfft.c:144-147 with P = 1
    d->segmentBoundaries[0] = 0;
    d->segmentBoundaries[1] = (int)k;
  }
  d->last_status = rc;
  return rc;
}

int soi_init_window_status(soi_desc_t *d, soi_comm_t comm, cfft_size_t k, const double *y_time, const double *y_freq)
{
  if (!y_time || !y_freq) return SOI_ERR_INVALID;
  if (!d) return SOI_ERR_INVALID;
  d->comm = comm;
  d->k = k;
  if (d->plan) { free_plan((Plan *)d->plan); d->plan = nullptr; }
  int rc = init_plan(d, k, y_time, y_freq);
  if (rc == SOI_OK) {
    free(d->segmentBoundaries);
    d->segmentBoundaries = (int *)malloc(sizeof(int) * 2);   // pfft.c:144-147 with P = 1
    d->segmentBoundaries[0] = 0;
    d->segmentBoundaries[1] = (int)k;
  }
  d->last_status = rc;
  return rc;
}

void init_soi_descriptor(soi_desc_t *d, soi_comm_t comm, cfft_size_t k)
{
  die_on(soi_init_status(d, comm, k), "init_soi_descriptor");
}

int soi_compute_status(soi_desc_t *d, void *alpha)
{
  if (!d) return SOI_ERR_INVALID;
  int rc = alpha ? compute_impl(d, alpha, alpha, false) : SOI_ERR_INVALID;
  d->last_status = rc;
  return rc;
}

void compute_soi(soi_desc_t *d, void *alpha) { die_on(soi_compute_status(d, alpha), "compute_soi"); }

int soi_compute_oop_status(soi_desc_t *d, const void *in, void *out)
{
  if (!d) return SOI_ERR_INVALID;
  int rc = (in && out) ? compute_impl(d, in, out, false) : SOI_ERR_INVALID;
  d->last_status = rc;
  return rc;
}

int soi_compute_segments_status(soi_desc_t *d, const void *in, void *out, int seg_lo, int seg_hi)
{
  if (!d) return SOI_ERR_INVALID;
  int rc = (in && out) ? compute_impl(d, in, out, false, seg_lo, seg_hi) : SOI_ERR_INVALID;
  d->last_status = rc;
  return rc;
}

// Streamed host transforms: ins[i] -> outs[i] for i < count, host buffers
// (pinned for the copies to overlap).  Two device staging buffers; transform
// i's upload (copy stream in), kernels (the plan's stream) and download (copy
// stream out) overlap with its neighbours', so PCIe carries both directions
// at once.  Each transform runs in place in its staging buffer; a buffer is
// refilled only after its previous download finished.
int compute_stream_impl(soi_desc_t *d, const void *const *ins, void *const *outs, int count)
{
  Plan *p = plan_of(d);
  if (!p) return SOI_ERR_NOT_INITIALISED;
  if (count < 1 || !ins || !outs) return SOI_ERR_INVALID;
  for (int i = 0; i < count; ++i) if (!ins[i] || !outs[i]) return SOI_ERR_INVALID;
  if (cudaSetDevice(p->device) != cudaSuccess) return SOI_ERR_CUDA;
  const size_t bytes = p->N * p->elem;
  if (!p->d_io) CK(cudaMalloc(&p->d_io, bytes));
  if (!p->d_io2) CK(cudaMalloc(&p->d_io2, bytes));
  if (!p->d_io3) CK(cudaMalloc(&p->d_io3, bytes));
  if (!p->st_in) CK(cudaStreamCreateWithFlags(&p->st_in, cudaStreamNonBlocking));
  if (!p->st_out) CK(cudaStreamCreateWithFlags(&p->st_out, cudaStreamNonBlocking));
  for (auto &e : p->sev)
    if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaStream_t st = p->stream;
  // three buffers: the upload of transform i + 1 never waits for a download
  // (buffer i + 1 was last downloaded as transform i - 2), so in steady state
  // the copies in both directions run back to back and the kernels hide
  // between them
  void *buf[3] = { p->d_io, p->d_io2, p->d_io3 };
  cudaEvent_t *in_done = p->sev, *comp_done = p->sev + 3, *out_done = p->sev + 6;
  CK(cudaMemsetAsync(p->d_sync, 0, sizeof(unsigned int), st));
  // the copy streams start after everything already queued on the plan's stream
  CK(cudaEventRecord(comp_done[0], st));
  CK(cudaStreamWaitEvent(p->st_in, comp_done[0], 0));
  CK(cudaStreamWaitEvent(p->st_out, comp_done[0], 0));
  for (int i = 0; i < count; ++i) {
    const int b = i % 3;
    if (i >= 3) CK(cudaStreamWaitEvent(p->st_in, out_done[b], 0));   // buffer b drained
    CK(cudaMemcpyAsync(buf[b], ins[i], bytes, cudaMemcpyHostToDevice, p->st_in));
    CK(cudaEventRecord(in_done[b], p->st_in));
    CK(cudaStreamWaitEvent(st, in_done[b], 0));
    const Exec ex{ buf[b], p->d_T, buf[b], p->d_sync, 0, (int)p->S, st, p->tma1 ? &p->tmap1 : nullptr };
    int rc;
    if ((rc = run_stage1(*p, ex))) return rc;
    if (d->use_vlc && (rc = run_vlc(*p, ex))) return rc;
    if ((rc = run_stage2(*p, ex))) return rc;
    CK(cudaEventRecord(comp_done[b], st));
    CK(cudaStreamWaitEvent(p->st_out, comp_done[b], 0));
    CK(cudaMemcpyAsync(outs[i], buf[b], bytes, cudaMemcpyDeviceToHost, p->st_out));
    CK(cudaEventRecord(out_done[b], p->st_out));
  }
  // the plan's stream ends after the last download
  CK(cudaStreamWaitEvent(st, out_done[(count - 1) % 3], 0));
  CK(cudaStreamSynchronize(st));
  CK(cudaStreamSynchronize(p->st_out));
  return check_stage2(*p, p->d_sync, st);
}

int soi_compute_async_status(soi_desc_t *d, const void *in, void *out)
{
  if (!d) return SOI_ERR_INVALID;
  int rc = (in && out) ? compute_impl(d, in, out, false, 0, -1, false) : SOI_ERR_INVALID;
  d->last_status = rc;
  return rc;
}

// conj(x) * scale over n complex values on the plan's stream
int conj_scale(Plan &p, const void *in, void *out, size_t n, double scale, cudaStream_t st)
{
  int nsm = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, p.device));
  const unsigned grid = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)nsm * 8);
  if (p.prec == SOI_PRECISION_FP64)
    k_conj_scale<double><<<grid, 256, 0, st>>>(in, out, (long long)n, scale);
  else
    k_conj_scale<float><<<grid, 256, 0, st>>>(in, out, (long long)n, (float)scale);
  CK(cudaGetLastError());
  return SOI_OK;
}

// Inverse transform in -> out: out = conj(in) on the device, the forward
// transform in place, then out = conj(out) / N.
int compute_inverse_impl(soi_desc_t *d, const void *in, void *out)
{
  Plan *p = plan_of(d);
  if (!p) return SOI_ERR_NOT_INITIALISED;
  if (cudaSetDevice(p->device) != cudaSuccess) return SOI_ERR_CUDA;
  cudaStream_t st = p->stream;
  const size_t bytes = p->N * p->elem;
  void *buf = out;
  if (!d->device_ptr) {
    if (!p->d_io) CK(cudaMalloc(&p->d_io, bytes));
    CK(cudaMemcpyAsync(p->d_io, in, bytes, cudaMemcpyHostToDevice, st));
    buf = p->d_io;
    in = p->d_io;
  }
  int rc;
  if ((rc = conj_scale(*p, in, buf, p->N, 1.0, st))) return rc;
  CK(cudaMemsetAsync(p->d_sync, 0, sizeof(unsigned int), st));
  const Exec ex{ buf, p->d_T, buf, p->d_sync, 0, (int)p->S, st, p->tma1 ? &p->tmap1 : nullptr };
  if ((rc = run_stage1(*p, ex))) return rc;
  if (d->use_vlc && (rc = run_vlc(*p, ex))) return rc;
  if ((rc = run_stage2(*p, ex))) return rc;
  if ((rc = conj_scale(*p, buf, buf, p->N, 1.0 / (double)p->N, st))) return rc;
  if (!d->device_ptr) CK(cudaMemcpyAsync(out, buf, bytes, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return check_stage2(*p, p->d_sync, st);
}

int soi_compute_inverse_status(soi_desc_t *d, const void *in, void *out)
{
  if (!d) return SOI_ERR_INVALID;
  if (d->device_ptr && ((uintptr_t)out & 15)) return SOI_ERR_INVALID;   // the conjugated input is staged in out
  int rc = (in && out) ? compute_inverse_impl(d, in, out) : SOI_ERR_INVALID;
  d->last_status = rc;
  return rc;
}

int soi_compute_stream_status(soi_desc_t *d, const void *const *ins, void *const *outs, int count)
{
  if (!d) return SOI_ERR_INVALID;
  if (d->device_ptr) return SOI_ERR_INVALID;                     // host buffers only
  int rc = compute_stream_impl(d, ins, outs, count);
  d->last_status = rc;
  return rc;
}

int soi_check_status(soi_desc_t *d)
{
  Plan *p = plan_of(d);
  if (!p) return SOI_ERR_NOT_INITIALISED;
  if (cudaSetDevice(p->device) != cudaSuccess) return SOI_ERR_CUDA;
  CK(cudaStreamSynchronize(p->stream));
  return check_stage2(*p, p->d_sync, p->stream);
}

int soi_filter_subsampling_status(soi_desc_t *d, void *alpha)
{
  if (!d) return SOI_ERR_INVALID;
  int rc = alpha ? compute_impl(d, alpha, alpha, true) : SOI_ERR_INVALID;
  d->last_status = rc;
  return rc;
}

void parallel_filter_subsampling(soi_desc_t *d, void *alpha)
{
  die_on(soi_filter_subsampling_status(d, alpha), "parallel_filter_subsampling");
}

int soi_get_transposed(soi_desc_t *d, void *dst)
{
  Plan *p = plan_of(d);
  if (!p) return SOI_ERR_NOT_INITIALISED;
  if (cudaSetDevice(p->device) != cudaSuccess) return SOI_ERR_CUDA;
  CK(cudaMemcpyAsync(dst, p->d_T, p->S * p->Mh * p->elem,
                     d->device_ptr ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  return SOI_OK;
}

int soi_free_status(soi_desc_t *d)
{
  if (!d) return SOI_ERR_INVALID;
  if (d->plan) free_plan((Plan *)d->plan);
  d->plan = nullptr;
  free(d->segmentBoundaries);
  d->segmentBoundaries = nullptr;
  return SOI_OK;
}

void free_soi_descriptor(soi_desc_t *d) { soi_free_status(d); }

int soi_filter_subsample_device(soi_desc_t *d, const void *alpha_dev, void *T_dev)
{
  Plan *p = plan_of(d);
  if (!p) return SOI_ERR_NOT_INITIALISED;
  if (cudaSetDevice(p->device) != cudaSuccess) return SOI_ERR_CUDA;
  if ((uintptr_t)alpha_dev & 15) return SOI_ERR_INVALID;
  const Exec ex{ alpha_dev, T_dev, nullptr, p->d_sync, 0, (int)p->S, p->stream };
  return run_stage1(*p, ex);
}

int soi_segment_fft_demod_device(soi_desc_t *d, void *T_dev, void *out_dev)
{
  Plan *p = plan_of(d);
  if (!p) return SOI_ERR_NOT_INITIALISED;
  if (cudaSetDevice(p->device) != cudaSuccess) return SOI_ERR_CUDA;
  const Exec ex{ nullptr, T_dev, out_dev, p->d_sync, 0, (int)p->S, p->stream };
  CK(cudaMemsetAsync(p->d_sync, 0, sizeof(unsigned int), p->stream));
  int rc = run_stage2(*p, ex);
  if (rc == SOI_OK) rc = check_stage2(*p, p->d_sync, p->stream);
  return rc;
}

int soi_plan_geometry(const soi_desc_t *d, cfft_size_t k, long long *info)
{
  if (!info) return SOI_ERR_INVALID;
  Plan p;
  int rc = plan_geometry(d, k, p);
  if (rc) return rc;
  long long v[16] = { (long long)p.S, (long long)p.M, (long long)p.Mh, p.s1fast ? p.JT2 : p.JT, p.atap,
                      p.s1fast ? p.JR2 : p.JR, (long long)(p.s1fast ? p.smem1b : p.smem1), p.M1, p.M2,
                      p.C1, p.C2, (long long)p.smem_c, (long long)p.smem_r, p.planS.nst, p.plan1.nst,
                      p.plan2.nst };
  memcpy(info, v, sizeof(v));
  return SOI_OK;
}

int soi_plan_variant(const soi_desc_t *d, cfft_size_t k, int *info)
{
  if (!info) return SOI_ERR_INVALID;
  Plan p;
  int rc = plan_geometry(d, k, p);
  if (rc) return rc;
  info[0] = p.s1_tc ? 3 : p.s1_tS ? 2 : p.s1fast ? 1 : 0;
  info[1] = p.s1_tc ? 512 : p.s1_tS ? p.s1_nt : (p.s1fast ? 512 : 0);
  info[2] = p.s1_tS && p.s1_bulk ? 1 : 0;
  info[3] = p.fast2 ? 1 : 0;
  // the persistent kernel's pass-2 bulk rows: on unless SOI_STAGE2_BULK2=0
  // (the switch is read when the device plan is set up)
  info[4] = p.fast2 && env_int("SOI_STAGE2_BULK2", 1) ? 1 : 0;
  return SOI_OK;
}

int soi_kernels_per_compute(soi_desc_t *d)
{
  Plan *p = plan_of(d);
  if (!p) return -SOI_ERR_NOT_INITIALISED;
  int n = 1 + (p->fast2 ? 1 : 2);
  if (d->use_vlc) n += 4;                                       // run_vlc
  return n;
}

int soi_set_timing(soi_desc_t *d, int enable)
{
  Plan *p = plan_of(d);
  if (!p) return SOI_ERR_NOT_INITIALISED;
  p->timing = enable != 0;
  return SOI_OK;
}

int soi_last_timings(soi_desc_t *d, float *ms4)
{
  Plan *p = plan_of(d);
  if (!p) return SOI_ERR_NOT_INITIALISED;
  for (int i = 0; i < 4; ++i) ms4[i] = p->ms[i];
  return SOI_OK;
}

int soi_window_tables(cfft_size_t N, cfft_size_t S, int n_mu, int d_mu, cfft_size_t B, double tau,
                      double sigma, double *filt, double *phase, double *W_inv)
{
  if (!N || !S || N % S || n_mu < 1 || d_mu < 1 || B < (size_t)d_mu) return SOI_ERR_INVALID;
  std::vector<long double> f, pr, pi, wr, wi;
  host_tables(N, S, n_mu, d_mu, B, tau, sigma, 0, filt ? &f : nullptr, phase ? &pr : nullptr,
              phase ? &pi : nullptr, W_inv ? &wr : nullptr, W_inv ? &wi : nullptr);
  if (filt) for (size_t i = 0; i < f.size(); ++i) filt[i] = (double)f[i];
  if (phase) for (size_t i = 0; i < pr.size(); ++i) { phase[2 * i] = (double)pr[i]; phase[2 * i + 1] = (double)pi[i]; }
  if (W_inv) for (size_t i = 0; i < wr.size(); ++i) { W_inv[2 * i] = (double)wr[i]; W_inv[2 * i + 1] = (double)wi[i]; }
  return SOI_OK;
}

int soi_mlp_param_count(void) { return kMlpParams; }

int soi_wmlp_param_count(void) { return wmlp::kParams; }

int soi_wmlp_forward_device(const float *params, const float *x, float *y, int n, void *stream)
{
  if (!params || !x || !y || n <= 0) return SOI_ERR_INVALID;
  const int blocks = std::min(1024, (n + 63) / 64);
  wmlp::forward_kernel<wmlp::kIn, wmlp::kOut><<<blocks, 64, 0, (cudaStream_t)stream>>>(params, x, y, n);
  CK(cudaGetLastError());
  return SOI_OK;
}

int soi_wmlp_grad_device(const float *params, const float *x, const float *y, int n, float *grad, float *loss,
                         void *stream)
{
  if (!params || !x || !y || !grad || !loss || n <= 0) return SOI_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemsetAsync(grad, 0, wmlp::kParams * sizeof(float), st));
  CK(cudaMemsetAsync(loss, 0, sizeof(float), st));
  wmlp::grad_kernel<wmlp::kIn, wmlp::kOut><<<(n + wmlp::kBlock - 1) / wmlp::kBlock, wmlp::kBlock, 0, st>>>(
      params, x, y, n, grad, loss);
  CK(cudaGetLastError());
  return SOI_OK;
}

int soi_adam_device(float *params, float *m, float *v, const float *grad, int count, float lr, int step,
                    void *stream)
{
  if (!params || !m || !v || !grad || count <= 0 || step < 1) return SOI_ERR_INVALID;
  mlp_adam_kernel<<<std::min(1024, (count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(params, m, v, grad, count,
                                                                                         lr, 0.9f, 0.999f, 1e-8f,
                                                                                         step);
  CK(cudaGetLastError());
  return SOI_OK;
}

int soi_mlp_forward_device(const float *params, const float *x, float *y, int n, void *stream)
{
  if (!params || !x || !y || n <= 0) return SOI_ERR_INVALID;
  const int blocks = std::min(1024, (n + 127) / 128);
  mlp_forward_kernel<<<blocks, 128, 0, (cudaStream_t)stream>>>(params, x, y, n);
  CK(cudaGetLastError());
  return SOI_OK;
}

int soi_mlp_grad_device(const float *params, const float *x, const float *y, int n, float *grad, float *loss,
                        void *stream)
{
  if (!params || !x || !y || !grad || !loss || n <= 0) return SOI_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  CK(cudaMemsetAsync(grad, 0, kMlpParams * sizeof(float), st));
  CK(cudaMemsetAsync(loss, 0, sizeof(float), st));
  mlp_grad_kernel<<<(n + kMlpBlock - 1) / kMlpBlock, kMlpBlock, 0, st>>>(params, x, y, n, grad, loss);
  CK(cudaGetLastError());
  return SOI_OK;
}

int soi_mlp_adam_device(float *params, float *m, float *v, const float *grad, float lr, int step, void *stream)
{
  if (!params || !m || !v || !grad || step < 1) return SOI_ERR_INVALID;
  mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, m, v, grad, kMlpParams, lr,
                                                                               0.9f, 0.999f, 1e-8f, step);
  CK(cudaGetLastError());
  return SOI_OK;
}

// Words compress() writes for one chunk of len doubles (pfft.c:397-402), in
// 64 bits: 3.5 words per double at full width, so an int overflows past
// ~613M doubles.
static long long vlc_words_ll(long long len, int e_max, int e_max_i)
{
  const int delta = e_max - e_max_i;
  const int i1 = (52 + 3 - 31) - delta, i2 = std::min(32, 52 + 3 - delta);
  if (len < 0) return -1;
  if (i2 <= 0) return 0;
  const long long nb = (i1 > 0 ? i1 : 0) + i2;
  const long long lanes = (len / 16) * nb;
  long long w = (lanes + 31) / 32 * 16;
  w += ((len % 16) * nb + 31) / 32;
  return w;
}

// The same count as an int, or -1 when it does not fit in one.
int soi_vlc_words(int len, int e_max, int e_max_i)
{
  const long long w = vlc_words_ll(len, e_max, e_max_i);
  return w > 2147483647LL ? -1 : (int)w;
}

int soi_vlc_max_exponent_device(const double *x, int len, int nchunks, int *e_max_out, void *stream)
{
  if (!x || !e_max_out || len <= 0 || nchunks <= 0) return SOI_ERR_INVALID;
  CK(vlc_max_exponent(x, len, nchunks, e_max_out, (cudaStream_t)stream));
  return SOI_OK;
}

int soi_vlc_compress_device(const double *x, int len, int nchunks, int e_max, const int *e_max_i,
                            int *words, long stride_words, int *nwords, void *stream)
{
  if (!x || !e_max_i || !words || !nwords || len <= 0 || nchunks <= 0) return SOI_ERR_INVALID;
  if (len % 16) return SOI_ERR_UNSUPPORTED;
  dim3 g(64, (unsigned)nchunks);
  vlc_compress_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(x, len, e_max, nullptr, e_max_i, words, stride_words, nwords);
  CK(cudaGetLastError());
  return SOI_OK;
}

int soi_vlc_decompress_device(const int *words, long stride_words, int len, int nchunks, int e_max,
                              const int *e_max_i, double *out, void *stream)
{
  if (!words || !e_max_i || !out || len <= 0 || nchunks <= 0) return SOI_ERR_INVALID;
  if (len % 16) return SOI_ERR_UNSUPPORTED;
  dim3 g(64, (unsigned)nchunks);
  vlc_decompress_kernel<<<g, 256, 0, (cudaStream_t)stream>>>(words, stride_words, len, e_max, nullptr, e_max_i, out);
  CK(cudaGetLastError());
  return SOI_OK;
}

int soi_batch_create(soi_batch_t **batch, const soi_desc_t *tmpl, const soi_batch_item_t *items, int count,
                     int chains, int tune)
{
  if (!batch || !tmpl || !items || count < 1 || chains < 1) return SOI_ERR_INVALID;
  *batch = nullptr;
  Batch *b = new Batch();
  b->tmpl = *tmpl;
  b->tmpl.plan = nullptr;
  b->tmpl.segmentBoundaries = nullptr;
  b->tmpl.P = 1;
  b->tmpl.rank = 0;
  b->device = tmpl->device;
  b->nchain = chains;
  for (int i = 0; i < count; ++i) {
    const soi_batch_item_t &x = items[i];
    if (!x.in || !x.out || x.k < 1) { delete b; return SOI_ERR_INVALID; }
    if ((uintptr_t)x.in & 15) { delete b; return SOI_ERR_INVALID; }   // 16-byte staging copies
    BatchItem it;
    it.N = x.N; it.k = x.k; it.in = x.in; it.out = x.out;
    it.lo = x.seg_hi <= 0 ? 0 : x.seg_lo;
    it.hi = x.seg_hi <= 0 ? (int)x.k : x.seg_hi;
    if (it.lo < 0 || it.hi > (int)x.k || it.lo >= it.hi) { delete b; return SOI_ERR_INVALID; }
    soi_desc_t d = b->tmpl;
    d.N = x.N;
    int rc = validate(&d, x.k);
    if (rc) { delete b; return rc; }
    b->items.push_back(it);
  }
  if (cudaSetDevice(b->device) != cudaSuccess) { delete b; return SOI_ERR_CUDA; }
  int rc = batch_build(*b, tune);
  if (rc) { batch_free(b); return rc; }
  *batch = (soi_batch_t *)b;
  return SOI_OK;
}

int soi_batch_execute(soi_batch_t *batch, void *stream)
{
  Batch *b = (Batch *)batch;
  if (!b || !b->exec) return SOI_ERR_NOT_INITIALISED;
  if (cudaSetDevice(b->device) != cudaSuccess) return SOI_ERR_CUDA;
  CK(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  b->last = (cudaStream_t)stream;
  return SOI_OK;
}

int soi_batch_check(soi_batch_t *batch)
{
  Batch *b = (Batch *)batch;
  if (!b) return SOI_ERR_NOT_INITIALISED;
  if (cudaSetDevice(b->device) != cudaSuccess) return SOI_ERR_CUDA;
  CK(cudaStreamSynchronize(b->last));
  for (int c = 0; c < b->nchain; ++c) {
    unsigned int err = 0;
    CK(cudaMemcpy(&err, b->sync[c], sizeof(err), cudaMemcpyDeviceToHost));
    if (err) return SOI_ERR_TIMEOUT;
  }
  return SOI_OK;
}

int soi_batch_info(soi_batch_t *batch, long long *info)
{
  Batch *b = (Batch *)batch;
  if (!b || !info) return SOI_ERR_INVALID;
  size_t nodes = 0;
  if (b->graph) cudaGraphGetNodes(b->graph, nullptr, &nodes);
  info[0] = (long long)b->items.size();
  info[1] = (long long)b->plans.size();
  info[2] = b->nchain;
  info[3] = (long long)nodes;
  long long launches = 0;
  for (auto &it : b->items) {
    const Plan &p = *b->plans[it.plan];
    launches += 1 + (p.fast2 ? 1 : 2) + (b->tmpl.use_vlc ? 4 : 0);
  }
  info[4] = launches;
  size_t scratch = 0;
  for (size_t t : b->Tbytes) scratch += t;
  info[5] = (long long)scratch;
  info[6] = 0;
  info[7] = 0;
  return SOI_OK;
}

int soi_batch_plan_info(soi_batch_t *batch, int plan, long long *info)
{
  Batch *b = (Batch *)batch;
  if (!b || !info || plan < 0 || plan >= (int)b->plans.size()) return SOI_ERR_INVALID;
  const Plan &p = *b->plans[plan];
  info[0] = (long long)p.N;
  info[1] = (long long)p.S;
  info[2] = p.s1fast ? (p.s1_tS ? p.s1_nt : 512) : 256;
  info[3] = p.fast2 ? 1 : 0;
  info[4] = p.M1;
  info[5] = p.M2;
  info[6] = (long long)(b->tuned_ms[plan] * 1000.0f);
  info[7] = b->variant[plan];
  return SOI_OK;
}

int soi_batch_destroy(soi_batch_t *batch)
{
  batch_free((Batch *)batch);
  return SOI_OK;
}

}  // extern "C"

// ======================================== VLC round trip without allocation ==
//
// soi_vlc_roundtrip_noalloc_device: the same max_exponent -> compress ->
// decompress round trip as the three soi_vlc_*_device entry points, for
// callers that cannot call cudaMalloc: a host program whose device memory is
// already handed out to its own pool (a framework's caching allocator that
// reserves the GPU at start-up), or a latency-critical loop in which the
// device-wide synchronisation of cudaMalloc/cudaFree is not acceptable.  Its
// scratch (per-chunk exponents, word counts and the compressed words) lives in
// the file-scope array below, which every GPU that loads this library holds
// until the process exits.

namespace {

constexpr long long kNoallocHeaderInts = 4096;              // e_max[<=2047], gmax, nwords[<=2047]
constexpr long long kNoallocWordInts = 8ll << 20;            // 32 MiB of compressed words
constexpr int kNoallocMaxChunks = 2047;
constexpr int kNoallocMaxDevices = 64;

static __device__ __align__(256) int g_noalloc_scratch[kNoallocHeaderInts + kNoallocWordInts];

int *g_noalloc_ptr[kNoallocMaxDevices] = {};
std::atomic<int> g_noalloc_lock{0};

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (cudaGetSymbolAddress with that device current) and cached.
int noalloc_scratch(int **ptr)
{
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoallocMaxDevices) return SOI_ERR_UNSUPPORTED;
  while (g_noalloc_lock.exchange(1)) {}
  int rc = SOI_OK;
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      fprintf(stderr, "soi_b200: cudaGetSymbolAddress(g_noalloc_scratch) failed: %s\n", cudaGetErrorString(e));
      rc = SOI_ERR_CUDA;
    } else {
      g_noalloc_ptr[dev] = (int *)p;
    }
  }
  *ptr = g_noalloc_ptr[dev];
  g_noalloc_lock.store(0);
  return rc;
}

}  // namespace

extern "C" int soi_vlc_roundtrip_noalloc_device(const double *x_dev, double *out_dev, int len, int nchunks,
                                                void *stream)
{
  if (!x_dev || !out_dev || len <= 0 || nchunks <= 0) return SOI_ERR_INVALID;
  if (len % 16) return SOI_ERR_UNSUPPORTED;
  // worst case of compress(): every element at full width (56 bits), counted
  // in 64 bits (len * 3.5 words does not fit an int past ~613M doubles)
  const long long per_chunk = vlc_words_ll(len, 0, 0);
  if (nchunks > kNoallocMaxChunks || per_chunk <= 0 || per_chunk > kNoallocWordInts ||
      per_chunk * nchunks > kNoallocWordInts) {
    fprintf(stderr,
            "soi_vlc_roundtrip_noalloc_device: %d chunks of %d doubles need %lld scratch words; the static "
            "scratch holds %lld words in at most %d chunks\n",
            nchunks, len, per_chunk * nchunks, kNoallocWordInts, kNoallocMaxChunks);
    return SOI_ERR_INVALID;
  }
  int *scr = nullptr;
  int rc = noalloc_scratch(&scr);
  if (rc) return rc;
  int *e_max_i = scr;                       // [nchunks]
  int *g_max = scr + kNoallocMaxChunks;     // [1]
  int *nwords = scr + kNoallocMaxChunks + 1;
  int *words = scr + kNoallocHeaderInts;    // [nchunks][per_chunk]
  cudaStream_t st = (cudaStream_t)stream;
  // every scratch entry read below is written earlier in this call (the
  // exponents, preset and then maximised by vlc_max_exponent, the maximum, the
  // counts, and each compressed word including its zero padding), so nothing
  // else has to be cleared first
  CK(vlc_max_exponent(x_dev, len, nchunks, e_max_i, st));
  vlc_global_max<<<1, 256, 0, st>>>(e_max_i, nchunks, g_max);
  CK(cudaGetLastError());
  dim3 g(64, (unsigned)nchunks);
  vlc_compress_kernel<<<g, 256, 0, st>>>(x_dev, len, 0, g_max, e_max_i, words, (long)per_chunk, nwords);
  CK(cudaGetLastError());
  vlc_decompress_kernel<<<g, 256, 0, st>>>(words, (long)per_chunk, len, 0, g_max, e_max_i, out_dev);
  CK(cudaGetLastError());
  return SOI_OK;
}
