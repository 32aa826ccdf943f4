/*
 * soi_b200.h -- C ABI of the B200 (sm_100a) SOI FFT library, libsoi_b200.so.
 *
 * Drop-in for the reference's public API, soi.h:236-280 (IntelLabs/SOI_FFT):
 * the same descriptor field names and the same four entry points, plus
 * status-returning variants and device-level entry points.  Plain C types
 * only: pointers, sizes, ints, doubles.
 *
 * Differences a caller of the reference must know:
 *   - One process, one GPU.  P (MPI ranks) must be 1 and rank 0; the segment
 *     count is S = k (the reference's S = k*P).  `comm` stands in for
 *     MPI_Comm and is not used.
 *   - alpha_dt holds N complex inputs and receives N complex outputs in
 *     natural DFT order (the reference's rank r holds N/P inputs and gets
 *     segments [segmentBoundaries[r], segmentBoundaries[r+1]) * M outputs).
 *   - precision selects the element type of alpha_dt:
 *       SOI_PRECISION_FP64       double complex (cfft_complex_t, soi.h:227)
 *       SOI_PRECISION_SPLIT_FP32 float complex (complex64 storage)
 *   - device_ptr = 0: alpha_dt is host memory, copied in and out inside
 *     compute_soi.  device_ptr = 1: alpha_dt is device memory.
 *   - The void entry points print a message and exit(-1) on an unsupported
 *     configuration, as the reference does (pfft.c:157-183,
 *     parallel_filter_subsampling.cpp:89-94,543-548).  The *_status
 *     variants return a soi_status_t instead.
 */
#ifndef SOI_B200_H
#define SOI_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t cfft_size_t;        /* soi.h:220 */
typedef void *soi_comm_t;          /* stands in for MPI_Comm (soi.h:238) */
/* soi.h:227: one interleaved (re, im) pair of doubles.  C sees the C99 complex
 * type the reference uses; C++ (no _Complex) a struct of the same layout. */
#ifdef __cplusplus
typedef struct { double re, im; } cfft_complex_t;
#else
typedef double _Complex cfft_complex_t;
#endif

typedef enum {
  SOI_PRECISION_FP64 = 0,          /* plain method, FP64 complex throughout        */
  SOI_PRECISION_SPLIT_FP32 = 1     /* complex64 storage, FP32 arithmetic,
                                      FP64-generated tables rounded once          */
} soi_precision_t;

typedef enum {
  SOI_OK = 0,
  SOI_ERR_INVALID = 1,             /* bad sizes / parameters                      */
  SOI_ERR_UNSUPPORTED = 2,         /* valid for the reference, not built here     */
  SOI_ERR_CUDA = 3,                /* a CUDA runtime call failed                  */
  SOI_ERR_NOT_INITIALISED = 4,
  SOI_ERR_TIMEOUT = 5              /* a bounded device-side wait gave up          */
} soi_status_t;

/* Descriptor.  Field names follow soi_desc_t, soi.h:236-270. */
typedef struct {
  soi_comm_t comm;        /* soi.h:238, unused                                   */
  int P;                  /* soi.h:239, must be 1                                */
  int rank;               /* soi.h:240, must be 0                                */
  cfft_size_t k;          /* soi.h:241, segments (S = k*P)                       */
  cfft_size_t N;          /* soi.h:242, transform length                         */
  /* soi.h:243-251: the reference's host tables and work buffers.  Present so
   * that its callers compile and run unchanged (test.c:409-420 frees them and
   * sets them to NULL after every compute).  This library keeps its tables
   * and buffers on the device, inside `plan`: set_default_soi_descriptor sets
   * these to NULL, and nothing in the library reads, writes or frees them. */
  cfft_complex_t *W_inv;
  cfft_complex_t *w;
  void *w_dup;            /* SIMDFPTYPE * in soi.h:245                           */
  cfft_complex_t *gamma_tilde;
  cfft_complex_t *alpha_tilde;
  cfft_complex_t *beta_tilde;
  cfft_complex_t *alpha_ghost;
  int *delta, *epsilon;
  int n_mu;               /* soi.h:252, oversampling numerator                   */
  int d_mu;               /* soi.h:253, oversampling denominator                 */
  cfft_size_t B;          /* soi.h:254, window taps                              */
  double tau;             /* soi.h:255                                           */
  double sigma;           /* soi.h:256                                           */
  int use_vlc;            /* soi.h:266, VLC round trip of the transposed data    */
  int *segmentBoundaries; /* soi.h:267, [0, S] after init                        */
  double comm_to_comp_cost_ratio; /* soi.h:269, kept for source compatibility    */
  /* additions */
  int precision;          /* soi_precision_t                                     */
  int device_ptr;         /* alpha_dt is a device pointer                        */
  int device;             /* CUDA device ordinal                                 */
  void *stream;           /* cudaStream_t to run on (NULL: the library's own,
                             a blocking stream, ordered with the legacy
                             default stream; with any other stream the caller
                             orders the input's producer before the call)    */
  int last_status;        /* soi_status_t of the last call                       */
  void *plan;             /* opaque device state                                 */
} soi_desc_t;

/* ---- reference entry points (soi.h:272-280) --------------------------- */

/* pfft.c:84-138: n_mu=5, d_mu=4, tau=928/1024, sigma=373.7314, B=72,
 * use_vlc=0, plus P=1, rank=0, precision=FP64, device_ptr=0, device=0. */
void set_default_soi_descriptor(soi_desc_t *desc);

/* pfft.c:140-232: tabulates the windows and sets up the device plan. */
void init_soi_descriptor(soi_desc_t *desc, soi_comm_t comm, cfft_size_t k);

/* pfft.c:276-721: in-place transform of alpha_dt (see precision, device_ptr). */
void compute_soi(soi_desc_t *desc, void *alpha_dt);

/* pfft.c:234-267 */
void free_soi_descriptor(soi_desc_t *desc);

/* parallel_filter_subsampling.cpp:535-550: stage 1 only (convolution, S-point
 * FFTs and segment transpose) into the descriptor's device buffer; fetch it
 * with soi_get_transposed. */
void parallel_filter_subsampling(soi_desc_t *desc, void *alpha_dt);

/* ---- status-returning variants ---------------------------------------- */
/* Device inputs (device_ptr = 1) must start on a 16-byte boundary (memory
 * from cudaMalloc does); a misaligned input returns SOI_ERR_INVALID. */
int soi_init_status(soi_desc_t *desc, soi_comm_t comm, cfft_size_t k);
/* init_soi_descriptor with a caller's window in place of the analytic one
 * (pfft.c:42-82): y_time[(kk*n_mu + theta)*k + s] is the real window y(t) at
 * t = theta*d_mu/n_mu - kk - s/k + (B - d_mu)/2 for kk < B, theta < n_mu,
 * s < k (the points where the reference evaluates w_f), and y_freq[j] is
 * its Fourier transform at xi = j/M - 1/2, j = 0 .. M/2 (M = N/k; the
 * transform is even, and must be positive there: the demodulation divides
 * by it, SOI_ERR_INVALID otherwise).  tau and sigma are not used.  No
 * counterpart in the reference. */
int soi_init_window_status(soi_desc_t *desc, soi_comm_t comm, cfft_size_t k, const double *y_time,
                           const double *y_freq);
int soi_compute_status(soi_desc_t *desc, void *alpha_dt);
/* Out-of-place compute_soi: `in` (N inputs) is left untouched, `out`
 * receives the N outputs; both host or both device memory per device_ptr.
 * No counterpart in the reference, whose compute_soi is in-place only. */
int soi_compute_oop_status(soi_desc_t *desc, const void *in, void *out);
/* Segments of interest: the outputs of segments [seg_lo, seg_hi) only
 * (out[seg_lo*M .. seg_hi*M), M = N/k); the rest of `out` is left as it was.
 * The convolution still reads all N inputs, but the transposed store, the
 * M'-point FFTs and the demodulation run for those segments only, so a band
 * of the spectrum costs its share of stage 2.  Results are bit-identical to
 * the same segments of a full compute.  Host or device buffers per
 * device_ptr.  No counterpart in the reference, where each rank computes the
 * segments it owns (pfft.c:584-694). */
int soi_compute_segments_status(soi_desc_t *desc, const void *in, void *out, int seg_lo, int seg_hi);
/* Out-of-place compute on device buffers (device_ptr = 1) that only enqueues
 * work on the descriptor's stream and never waits on it, so it can be
 * recorded into a CUDA graph.  A persistent-kernel wait that gave up is
 * reported by the next soi_check_status.  No counterpart in the reference. */
int soi_compute_async_status(soi_desc_t *desc, const void *in, void *out);
/* Inverse transform: out[n] = (1/N) sum_k in[k] exp(+2 pi i k n / N), computed
 * as conj(forward(conj(in)))/N with the same plan (window, precision,
 * segments); `in` is left untouched; host or device buffers per device_ptr.
 * No counterpart in the reference, which has no inverse. */
int soi_compute_inverse_status(soi_desc_t *desc, const void *in, void *out);
/* Several transforms of host buffers (device_ptr = 0): outs[i] receives the
 * transform of ins[i], i < count.  Uploads, kernels and downloads of
 * neighbouring transforms overlap on separate streams (PCIe carries both
 * directions at once), so with pinned buffers the cost per transform
 * approaches one copy time instead of two plus the kernels.  Three N-element
 * device staging buffers, allocated on first use.  Returns after the last
 * download.  No counterpart in the reference. */
int soi_compute_stream_status(soi_desc_t *desc, const void *const *ins, void *const *outs, int count);
/* Waits for the descriptor's stream and returns SOI_ERR_TIMEOUT if a
 * stage-2 dependency wait gave up since the last compute, else SOI_OK. */
int soi_check_status(soi_desc_t *desc);
int soi_filter_subsampling_status(soi_desc_t *desc, void *alpha_dt);
int soi_free_status(soi_desc_t *desc);
const char *soi_status_string(int status);

/* Copy the transposed data (alpha_tilde of the reference: S segments of
 * M' = n_mu*M/d_mu elements, segment-major) to dst (host or device per
 * desc->device_ptr), element type per desc->precision. */
int soi_get_transposed(soi_desc_t *desc, void *dst);

/* ---- device-level entry points (device pointers, desc->stream) --------- */

/* Stage 1 from a device input to a device transposed buffer (S x M'). */
int soi_filter_subsample_device(soi_desc_t *desc, const void *alpha_dev, void *transposed_dev);
/* Stage 2: M'-point FFT of each segment, demodulation, discard; reads and
 * overwrites transposed_dev, writes N outputs to out_dev. */
int soi_segment_fft_demod_device(soi_desc_t *desc, void *transposed_dev, void *out_dev);

/* Plan geometry without touching a GPU (host logic, for tests and tuning):
 * info[0..15] = S, M, M', stage-1 groups per tile JT, taps per phase,
 * groups per thread JR, stage-1 shared bytes, M1, M2, C1, C2, pass-1 and
 * pass-2 shared bytes, radix stages of the S-, M1- and M2-point FFTs. */
int soi_plan_geometry(const soi_desc_t *desc, cfft_size_t k, long long *info);
/* The kernels a plan runs, without touching a GPU: info[0] = stage-1 kernel
 * (0 general, 1 staged, 2 compile-time S, 3 tensor cores), info[1] = its
 * threads per CTA, info[2] = its staging (0 cp.async, 1 one tensor copy per
 * phase), info[3] = stage 2 (0 two kernels, 1 persistent four-step),
 * info[4] = pass-2 rows by bulk copies (1) or cp.async (0). */
int soi_plan_variant(const soi_desc_t *desc, cfft_size_t k, int *info);

/* Kernel timings of the last compute (milliseconds, CUDA events on the
 * launching stream): [0] stage 1, [1] stage 2, [2] VLC, [3] whole compute. */
int soi_last_timings(soi_desc_t *desc, float *ms4);
/* Enable/disable event timing (off by default). */
int soi_set_timing(soi_desc_t *desc, int enable);
/* Number of this library's kernels one compute launches on the device
 * (stage 1, stage 2, and the VLC round trip when use_vlc is set); < 0 is a
 * soi_status_t error.  No counterpart in the reference (no GPU there). */
int soi_kernels_per_compute(soi_desc_t *desc);

/* ---- batched transforms ------------------------------------------------ */
/* No counterpart in the reference, which transforms one signal per call.
 * A batch is a fixed set of transforms on device buffers, replayed as one
 * CUDA graph: one plan per distinct (N, k) (with `tune`, the fastest of the
 * plan's kernel variants, timed once on the first transform of that shape),
 * the transforms spread over `chains` concurrent streams (each with its own
 * scratch, in order within a chain).  Window, oversampling, precision,
 * device and use_vlc come from `tmpl` (a descriptor set up as for
 * init_soi_descriptor; its N is ignored).  With use_vlc the batch runs one
 * chain. */
typedef struct soi_batch soi_batch_t;
typedef struct {
  cfft_size_t N;          /* transform length                                  */
  cfft_size_t k;          /* segments (the reference's k with P = 1)           */
  int seg_lo, seg_hi;     /* segments of interest; seg_hi <= 0: all k           */
  const void *in;         /* device input, N complex (complex64 in split form)  */
  void *out;              /* device output, N complex; may equal in            */
} soi_batch_item_t;
int soi_batch_create(soi_batch_t **batch, const soi_desc_t *tmpl, const soi_batch_item_t *items, int count,
                     int chains, int tune);
/* Launches the batch's graph on `stream` (a cudaStream_t; NULL = legacy). */
int soi_batch_execute(soi_batch_t *batch, void *stream);
/* Waits for the last execute; SOI_ERR_TIMEOUT if a stage-2 wait gave up. */
int soi_batch_check(soi_batch_t *batch);
/* info[0..7] = transforms, plans, chains, graph nodes, kernel launches per
 * execute, scratch bytes, 0, 0. */
int soi_batch_info(soi_batch_t *batch, long long *info);
/* Plan `plan`: info[0..7] = N, k, stage-1 block size, persistent stage 2
 * (1/0), M1, M2, tuned time (microseconds, 0 untuned), variant code. */
int soi_batch_plan_info(soi_batch_t *batch, int plan, long long *info);
int soi_batch_destroy(soi_batch_t *batch);

/* ---- VLC (compress.c) on the device ------------------------------------ */

/* compress.c:11-131 over nchunks chunks of `len` doubles each (device
 * pointers): e_max_out[c] = max biased exponent of chunk c minus 1023. */
int soi_vlc_max_exponent_device(const double *x_dev, int len, int nchunks,
                                int *e_max_out_dev, void *stream);
/* compress.c:205-372 for each chunk: words_dev + c*stride_words receives the
 * compressed words, nwords_dev[c] their count.  e_max is the global maximum
 * exponent, e_max_i_dev[c] the chunk's.  len must be a multiple of 16. */
int soi_vlc_compress_device(const double *x_dev, int len, int nchunks, int e_max,
                            const int *e_max_i_dev, int *words_dev, long stride_words,
                            int *nwords_dev, void *stream);
/* compress.c:428-544 for each chunk (len a multiple of 16). */
int soi_vlc_decompress_device(const int *words_dev, long stride_words, int len, int nchunks,
                              int e_max, const int *e_max_i_dev, double *out_dev, void *stream);
/* The same round trip (max_exponent, global maximum, compress, decompress)
 * for callers that cannot call cudaMalloc -- a process whose device memory is
 * already reserved by its own pool allocator, or a latency-critical loop that
 * must not pay cudaMalloc/cudaFree's device-wide synchronisation.  No
 * counterpart in the reference.  It allocates nothing: its scratch is a
 * static device array of 32 MiB of compressed words (plus 16 KiB of
 * per-chunk exponents and counts) that every GPU loading this library holds
 * until the process exits.  Limits: len a multiple of 16, nchunks <= 2047,
 * nchunks * soi_vlc_words(len, 0, 0) <= 8388608 (about 4.8M doubles in
 * total); larger requests return SOI_ERR_INVALID with a message on stderr.
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress), so make that first call before any stream capture.
 * All calls share the one array: calls that overlap on the GPU (different
 * streams, or host threads without ordering) race and corrupt each other.
 * x_dev: nchunks*len doubles in, out_dev: nchunks*len doubles out, on
 * `stream`; the call returns without synchronising. */
int soi_vlc_roundtrip_noalloc_device(const double *x_dev, double *out_dev, int len, int nchunks,
                                     void *stream);
/* Words compress() writes for one chunk (pfft.c:397-402 sizing); -1 when the
 * count does not fit in an int (len above ~613M doubles at full width). */
int soi_vlc_words(int len, int e_max, int e_max_i);

/* ---- learned window surrogate (no counterpart in the reference) --------- */

/* A 4-64-64-1 GELU MLP (FP32) predicting log10 of the transform's relative L2
 * error for a window (inputs normalised by soi_fft_b200/window_mlp.py).
 * Parameters: soi_mlp_param_count() floats, layout W1[64][4] b1 W2[64][64]
 * b2 W3[64] b3.  All pointers are device pointers. */
int soi_mlp_param_count(void);
/* y[i] = MLP(x[i][0..4)) for i < n */
int soi_mlp_forward_device(const float *params, const float *x, float *y, int n, void *stream);
/* grad = d/dparams of mean((MLP(x) - y)^2), loss = that mean; both overwritten */
int soi_mlp_grad_device(const float *params, const float *x, const float *y, int n, float *grad, float *loss,
                        void *stream);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) at 1-based step count */
int soi_mlp_adam_device(float *params, float *m, float *v, const float *grad, float lr, int step, void *stream);

/* ---- learned window proposer (no counterpart in the reference) ---------- */

/* A 2-64-64-32 GELU MLP (FP32) mapping (mu, log10 target error), normalised by
 * soi_fft_b200/window_cheb.py, to 32 Chebyshev coefficients of a window's
 * frequency-response profile.  Layout W1[64][2] b1[64] W2[64][64] b2[64]
 * W3[32][64] b3[32].  Device pointers. */
int soi_wmlp_param_count(void);
/* y[i][0..32) = MLP(x[i][0..2)) for i < n */
int soi_wmlp_forward_device(const float *params, const float *x, float *y, int n, void *stream);
/* grad = d/dparams of mean((MLP(x) - y)^2) over the n x 32 outputs, loss = that mean */
int soi_wmlp_grad_device(const float *params, const float *x, const float *y, int n, float *grad, float *loss,
                         void *stream);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) over `count` parameters */
int soi_adam_device(float *params, float *m, float *v, const float *grad, int count, float lr, int step,
                    void *stream);

/* ---- host-side tables (no GPU needed) ---------------------------------- */

/* The factorised window the kernels use: for output phase theta, tap kk and
 * column s the reference's w[theta][kk][s] (pfft.c:42-66) equals
 * phase[theta][s] * filt[kk][theta][s], with filt real.  filt: B*n_mu*S
 * doubles ([kk][theta][s]), phase: n_mu*S complex ([theta][s]),
 * W_inv: N/S complex (pfft.c:68-82).  Any pointer may be NULL. */
int soi_window_tables(cfft_size_t N, cfft_size_t S, int n_mu, int d_mu, cfft_size_t B,
                      double tau, double sigma, double *filt, double *phase, double *W_inv);

/* Library version string. */
const char *soi_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif
