/*
 * A C caller of libsoi_b200.so written the way the reference's own driver
 * calls soi.h (test.c:199-207,373-429): set_default_soi_descriptor, fields set
 * directly in the struct (test.c:91-101,125-128), init_soi_descriptor with a
 * communicator, compute_soi on a cfft_complex_t buffer of M_hat*k elements
 * (test.c:380), the table and work-buffer fields freed and set to NULL after
 * the compute (test.c:409-420), segmentBoundaries read for the owned
 * segments (test.c:423-424), free_soi_descriptor.  Only the header differs:
 * soi_b200.h in place of soi.h, and a stand-in for MPI_COMM_WORLD.
 *
 *   soi_caller validate            checks defaults and init's argument
 *                                  validation (no GPU needed)
 *   soi_caller compute N k seed out.bin
 *                                  transforms a seeded input and writes the
 *                                  N outputs (complex128) to out.bin
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "soi_b200.h"

#define MPI_COMM_WORLD ((soi_comm_t)0)

/* splitmix64 -> uniform doubles in [-1, 1) */
static uint64_t next_u64(uint64_t *s)
{
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static double uniform(uint64_t *s) { return (double)(next_u64(s) >> 11) * 0x1.0p-52 - 1.0; }

static int validate(void)
{
  soi_desc_t d;
  set_default_soi_descriptor(&d);
  /* pfft.c:87-94 defaults, and the soi.h:243-251 fields start NULL */
  if (d.n_mu != 5 || d.d_mu != 4 || d.B != 72 || d.tau != 928 / 1024. || d.sigma != 373.7314 || d.use_vlc) return 1;
  if (d.W_inv || d.w || d.w_dup || d.gamma_tilde || d.alpha_tilde || d.beta_tilde || d.alpha_ghost || d.delta ||
      d.epsilon)
    return 2;
  /* the fields test.c's parseArgs sets */
  d.N = 1000; d.P = 1; d.rank = 0;
  if (soi_init_status(&d, MPI_COMM_WORLD, 8) != SOI_ERR_INVALID) return 3;     /* S does not divide N */
  d.N = 1 << 16; d.n_mu = 7;
  if (soi_init_status(&d, MPI_COMM_WORLD, 8) != SOI_ERR_UNSUPPORTED) return 4; /* mu = 7/4 not built */
  d.n_mu = 5; d.P = 2;
  if (soi_init_status(&d, MPI_COMM_WORLD, 8) != SOI_ERR_UNSUPPORTED) return 5; /* several ranks */
  d.P = 1;
  if (soi_init_status(&d, MPI_COMM_WORLD, 0) != SOI_ERR_INVALID) return 6;     /* k = 0 */
  free_soi_descriptor(&d);
  printf("validate ok\n");
  return 0;
}

static int compute(size_t N, size_t k, uint64_t seed, const char *path)
{
  soi_desc_t d;
  set_default_soi_descriptor(&d);
  d.N = N; d.P = 1; d.rank = 0;
  d.n_mu = 5; d.d_mu = 4; d.B = 72;
  init_soi_descriptor(&d, MPI_COMM_WORLD, k);

  cfft_size_t S = d.k * d.P;                 /* test.c:375-377 */
  cfft_size_t M = d.N / S;
  cfft_size_t M_hat = d.n_mu * M / d.d_mu;
  cfft_complex_t *in_buf = NULL;
  size_t in_buf_size = sizeof(cfft_complex_t) * M_hat * d.k;
  if (posix_memalign((void **)&in_buf, 4096, in_buf_size) || !in_buf) return 10;
  uint64_t s = seed;
  for (size_t i = 0; i < d.N / d.P; ++i) {
    double re = uniform(&s), im = uniform(&s);
    in_buf[i] = re + im * I;
  }

  compute_soi(&d, in_buf);

  free(d.w); d.w = NULL;                      /* test.c:409-420 */
  free(d.w_dup); d.w_dup = NULL;
  free(d.W_inv); d.W_inv = NULL;
  free(d.alpha_ghost); d.alpha_ghost = NULL;
  if (d.use_vlc && d.epsilon) {
    free(d.epsilon); d.epsilon = NULL;
  }
  d.alpha_tilde = NULL;
  d.beta_tilde = NULL;
  d.gamma_tilde = NULL;

  int firstSegment = d.segmentBoundaries[d.rank];   /* test.c:423-424 */
  int nSegments = d.segmentBoundaries[d.rank + 1] - firstSegment;
  if (firstSegment != 0 || (size_t)nSegments != S) return 11;

  FILE *f = fopen(path, "wb");
  if (!f) return 12;
  size_t w = fwrite(in_buf + M * firstSegment, sizeof(cfft_complex_t), M * nSegments, f);
  fclose(f);
  free_soi_descriptor(&d);
  free(in_buf);
  if (w != M * (size_t)nSegments) return 13;
  printf("compute ok\n");
  return 0;
}

int main(int argc, char **argv)
{
  if (argc >= 2 && !strcmp(argv[1], "validate")) return validate();
  if (argc >= 6 && !strcmp(argv[1], "compute"))
    return compute((size_t)strtoull(argv[2], 0, 10), (size_t)strtoull(argv[3], 0, 10),
                   (uint64_t)strtoull(argv[4], 0, 10), argv[5]);
  fprintf(stderr, "usage: soi_caller validate | compute N k seed out.bin\n");
  return 2;
}
