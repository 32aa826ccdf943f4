// vlc_kernels.cuh -- the variable-length compression of compress.c on the GPU,
// bit-exact to the reference's stream for chunks whose length (in doubles) is
// a multiple of 16, which is every chunk on the SOI path (2*M'/P doubles).
//
// Stream format (compress.c:170-203,227-328): element e = 16*g + L goes to
// lane L; each element contributes one field of nb = max(i1Len,0) + i2Len
// bits, i1 (i1Len bits) then i2 (i2Len bits), appended MSB-first to the
// lane's 32-bit words; lane L's word w is stored at out[16*w + L]; a partial
// last word group is flushed with zero padding.  Because every lane receives
// the same number of bits, bit b of lane L's stream is simply bit (b mod 32,
// from the top) of word floor(b/32).  32 consecutive fields of a lane fill
// exactly nb whole words, so a lane's stream splits into independent units of
// 32 fields / nb words: the kernels give each thread one unit (lane L, block
// k), which it packs or unpacks sequentially with no division and no word
// shared with another thread; only a chunk's last unit may be partial (its
// last word zero-padded).
#pragma once

#include <cuda_runtime.h>
#include <limits.h>
#include <stdint.h>

namespace soi {

constexpr int kVlcLanes = 16;

struct VlcBits {
  int i1Len, i2Len, nb;
  double e1, e2, e3;        // quantisation scales (compress.c:214-216)
  double d1, d2;            // reconstruction scales (compress.c:430-431)
};

__device__ __forceinline__ VlcBits vlc_bits(int e_max, int e_max_i)
{
  VlcBits b;
  const int delta = e_max - e_max_i;
  b.i1Len = (52 + 3 - 31) - delta;                          // compress.c:207
  b.i2Len = min(32, 52 + 3 - delta);                        // compress.c:208
  b.nb = (b.i1Len > 0 ? b.i1Len : 0) + b.i2Len;
  b.e1 = ldexp(1.0, (52 - 31) - e_max);
  b.e2 = ldexp(1.0, 52 - e_max);
  b.e3 = ldexp(1.0, 31);
  b.d1 = ldexp(1.0, e_max - (52 - 31));
  b.d2 = ldexp(1.0, e_max - 52);
  return b;
}

// The packed field of one element (vector-path rounding: round-to-nearest-even
// for i1, a fused multiply-subtract then round-to-nearest-even for i2,
// compress.c:235-280).
__device__ __forceinline__ uint64_t vlc_field(double x, const VlcBits &b)
{
  const double r1 = rint(__dmul_rn(x, b.e1));
  const double r2 = fma(x, b.e2, -__dmul_rn(r1, b.e3));
  const int32_t i1 = (int32_t)r1;
  const int32_t i2 = (int32_t)rint(r2);
  const uint64_t m2 = b.i2Len >= 32 ? 0xFFFFFFFFull : ((1ull << b.i2Len) - 1);
  uint64_t f = (uint64_t)(uint32_t)i2 & m2;
  if (b.i1Len > 0) {
    const uint64_t m1 = (1ull << b.i1Len) - 1;
    f |= ((uint64_t)(uint32_t)i1 & m1) << b.i2Len;
  }
  return f;
}

// compress.c:11-131: per chunk (blockIdx.y), max biased exponent - 1023.
// Several blocks per chunk (blockIdx.x, grid-stride); each folds its maximum
// into e_max[chunk] with atomicMax, so e_max must start below any result
// (vlc_max_exponent below presets it).
// X = double, or float for the split form's data (each value widened to
// double exactly, as the round trip defines it on doubles).
template <typename X>
__global__ void vlc_max_exponent_kernel(const X *x, int len, int *e_max)
{
  const X *c = x + (size_t)blockIdx.y * len;
  int m = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const unsigned long long u = (unsigned long long)__double_as_longlong((double)c[i]);
    m = max(m, (int)((u >> 52) & 0x7FF));
  }
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ int wm[32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = threadIdx.x < (blockDim.x + 31) / 32 ? wm[threadIdx.x] : 0;
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) atomicMax(e_max + blockIdx.y, v - 1023);
  }
}

// Per-chunk maximum exponents of nchunks chunks of len doubles into e_max.
template <typename X>
inline cudaError_t vlc_max_exponent(const X *x, int len, int nchunks, int *e_max, cudaStream_t st)
{
  // 0x80 bytes: every preset word is far below -1023, the smallest result
  cudaError_t e = cudaMemsetAsync(e_max, 0x80, (size_t)nchunks * sizeof(int), st);
  if (e != cudaSuccess) return e;
  const long long per = ((long long)len + 2047) / 2048;
  dim3 g((unsigned)(per < 64 ? per : 64), (unsigned)nchunks);
  vlc_max_exponent_kernel<X><<<g, 256, 0, st>>>(x, len, e_max);
  return cudaGetLastError();
}

// max over chunks (pfft.c:340-343, after the MPI_Allreduce MAX of :331-333)
__global__ void vlc_global_max(const int *e, int n, int *out)
{
  int m = INT_MIN;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = max(m, e[i]);
  for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ int wm[32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = threadIdx.x < (blockDim.x + 31) / 32 ? wm[threadIdx.x] : INT_MIN;
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) *out = v;
  }
}

inline size_t vlc_compress_smem() { return 0; }
inline size_t vlc_decompress_smem() { return 0; }

// Words per lane for a chunk of len doubles (len % 16 == 0).
__host__ __device__ __forceinline__ long long vlc_words_per_lane(int len, int nb)
{
  const long long groups = len / kVlcLanes;
  return (groups * nb + 31) / 32;
}

// compress.c:205-372, one chunk per blockIdx.y; one thread per unit (lane L,
// block k of 32 fields), grid-stride over the chunk's units.  e_max =
// *e_max_dev when given, else e_max_host; e_max_i[c] per chunk.
template <typename X>
__global__ void vlc_compress_kernel(const X *x, int len, int e_max_host, const int *e_max_dev,
                                    const int *e_max_i, int *words, long stride, int *nwords)
{
  const int c = blockIdx.y;
  const int e_max = e_max_dev ? *e_max_dev : e_max_host;
  const VlcBits b = vlc_bits(e_max, e_max_i[c]);
  const X *xc = x + (size_t)c * len;
  uint32_t *wc = reinterpret_cast<uint32_t *>(words + (size_t)c * stride);
  if (b.i2Len <= 0) {                        // compress.c:210-212
    if (blockIdx.x == 0 && threadIdx.x == 0) nwords[c] = 0;
    return;
  }
  const int nb = b.nb;
  const long long groups = len / kVlcLanes;
  const long long nblk = (groups + 31) / 32;
  if (blockIdx.x == 0 && threadIdx.x == 0) nwords[c] = (int)(vlc_words_per_lane(len, nb) * kVlcLanes);
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < nblk * kVlcLanes;
       u += (long long)gridDim.x * blockDim.x) {
    const int L = (int)(u % kVlcLanes);
    const long long k = u / kVlcLanes;
    const long long g0 = 32 * k;
    const int nf = (int)(groups - g0 < 32 ? groups - g0 : 32);
    const X *src = xc + g0 * kVlcLanes + L;
    uint32_t *dst = wc + (size_t)k * nb * kVlcLanes + L;          // word k*nb of lane L
    uint32_t cur = 0;
    int have = 0;                                                // bits placed in cur, from the top
    for (int j = 0; j < nf; ++j) {
      const uint64_t f = vlc_field((double)src[(size_t)j * kVlcLanes], b);
      int rem = nb;
      while (rem > 0) {
        const int take = min(32 - have, rem);
        const uint32_t part = (uint32_t)((f >> (rem - take)) & ((1ull << take) - 1));
        cur |= part << (32 - have - take);
        have += take;
        rem -= take;
        if (have == 32) {
          *dst = cur;
          dst += kVlcLanes;
          cur = 0;
          have = 0;
        }
      }
    }
    if (have > 0) *dst = cur;                                    // last unit: zero-padded word
  }
}

// compress.c:428-544 (vector body, :395-426 and :450-489), one chunk per
// blockIdx.y; one thread per unit (lane L, block k of 32 fields).  e_max =
// *e_max_dev when given, else e_max_host; e_max_i[c] per chunk.
// Y = double, or float for the split form (the decoded double rounded to float)
template <typename Y>
__global__ void vlc_decompress_kernel(const int *words, long stride, int len, int e_max_host,
                                      const int *e_max_dev, const int *e_max_i, Y *out)
{
  const int c = blockIdx.y;
  const int e_max = e_max_dev ? *e_max_dev : e_max_host;
  const VlcBits b = vlc_bits(e_max, e_max_i[c]);
  Y *oc = out + (size_t)c * len;
  const uint32_t *wc = reinterpret_cast<const uint32_t *>(words + (size_t)c * stride);
  const int nb = b.nb;
  const long long groups = len / kVlcLanes;
  const long long nblk = (groups + 31) / 32;
  for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < nblk * kVlcLanes;
       u += (long long)gridDim.x * blockDim.x) {
    const int L = (int)(u % kVlcLanes);
    const long long k = u / kVlcLanes;
    const long long g0 = 32 * k;
    const int nf = (int)(groups - g0 < 32 ? groups - g0 : 32);
    Y *dst = oc + g0 * kVlcLanes + L;
    if (b.i2Len <= 0) {
      for (int j = 0; j < nf; ++j) dst[(size_t)j * kVlcLanes] = (Y)0;
      continue;
    }
    const uint32_t *src = wc + (size_t)k * nb * kVlcLanes + L;
    uint32_t cur = 0;
    int left = 0;                                                // unread bits of cur, at its bottom
    for (int j = 0; j < nf; ++j) {
      // gather nb bits MSB-first into f
      uint64_t f = 0;
      int need = nb;
      while (need > 0) {
        if (left == 0) {
          cur = __ldg(src);
          src += kVlcLanes;
          left = 32;
        }
        const int take = min(left, need);
        f = (f << take) | (((uint64_t)cur >> (left - take)) & ((1ull << take) - 1));
        left -= take;
        need -= take;
      }
      int32_t i1 = 0;
      if (b.i1Len > 0) {
        const uint32_t top = (uint32_t)(f >> b.i2Len);
        i1 = (int32_t)(top << (32 - b.i1Len)) >> (32 - b.i1Len);
      }
      const uint32_t low = (uint32_t)(f & (b.i2Len >= 32 ? 0xFFFFFFFFull : ((1ull << b.i2Len) - 1)));
      const int32_t i2 = b.i2Len >= 32 ? (int32_t)low : ((int32_t)(low << (32 - b.i2Len)) >> (32 - b.i2Len));
      dst[(size_t)j * kVlcLanes] = (Y)fma((double)i1, b.d1, __dmul_rn((double)i2, b.d2));
    }
  }
}

}  // namespace soi
