/*
 * ref_run.c -- harness that drives the reference's own compute_soi (pfft.c,
 * parallel_filter_subsampling.cpp, compress.c compiled unmodified from the
 * reference tree) on P forked ranks.  It replaces test.c:197-472 (which needs
 * MKL's cluster DFT) for one purpose: feed a given input, return the output in
 * natural order and the best wall time.  TEST INFRASTRUCTURE / CPU baseline.
 *
 * usage: soi_ref_run --N n --P p --k k [--n_mu 5 --d_mu 4 --B 72 --tau t
 *                    --sigma s --vlc --ratio r --threads T --repeat R]
 *                    --in file --out file
 * Input and output are raw interleaved complex128.  The last stdout line is
 * "SOI_REF_RESULT best_s=<seconds> ranks=<P> threads=<T>".
 */
#define _GNU_SOURCE
#include <fcntl.h>
#include <limits.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "soi.h"

typedef struct {
  size_t N; int P; size_t k; int n_mu, d_mu; size_t B; double tau, sigma;
  int vlc; double ratio; int threads; int repeat;
  const double *in; double *out; double *times;   /* times[0] best, times[1+r] repeat r */
} job_t;

static int rank_body(int rank, void *arg)
{
  job_t *j = (job_t *)arg;
  soi_desc_t d;
  set_default_soi_descriptor(&d);
  d.N = j->N; d.P = j->P; d.rank = rank;
  d.n_mu = j->n_mu; d.d_mu = j->d_mu; d.B = j->B;
  if (j->tau > 0) d.tau = j->tau;
  if (j->sigma > 0) d.sigma = j->sigma;
  d.use_vlc = j->vlc; d.comm_to_comp_cost_ratio = j->ratio;
  omp_set_num_threads(j->threads);
  size_t S = j->k * (size_t)j->P, M = j->N / S, Mh = (size_t)j->n_mu * M / (size_t)j->d_mu;
  cfft_complex_t *buf = NULL;
  if (posix_memalign((void **)&buf, 4096, sizeof(cfft_complex_t) * Mh * j->k)) return 2;
  init_soi_descriptor(&d, MPI_COMM_WORLD, j->k);
  double best = 1e300;
  size_t local = j->N / (size_t)j->P;
  for (int r = 0; r < j->repeat; ++r) {
    memcpy(buf, j->in + 2 * rank * local, sizeof(cfft_complex_t) * local);
    MPI_Barrier(MPI_COMM_WORLD);
    double t0 = MPI_Wtime();
    compute_soi(&d, buf);
    MPI_Barrier(MPI_COMM_WORLD);
    double t = MPI_Wtime() - t0;
    if (t < best) best = t;
    if (rank == 0 && r < 62) j->times[1 + r] = t;
  }
  int s0 = d.segmentBoundaries[rank], ns = d.segmentBoundaries[rank + 1] - s0;
  memcpy(j->out + 2 * (size_t)s0 * M, buf, sizeof(cfft_complex_t) * (size_t)ns * M);
  if (rank == 0) j->times[0] = best;
  free_soi_descriptor(&d);
  free(buf);
  return 0;
}

int main(int argc, char **argv)
{
  job_t j;
  memset(&j, 0, sizeof(j));
  j.P = 1; j.k = 1; j.n_mu = 5; j.d_mu = 4; j.B = 72; j.ratio = 1; j.threads = 1; j.repeat = 1;
  const char *fin = NULL, *fout = NULL;
  for (int i = 1; i < argc; ++i) {
    const char *a = argv[i];
    const char *v = i + 1 < argc ? argv[i + 1] : "";
    if (!strcmp(a, "--N")) { j.N = strtoull(v, 0, 10); ++i; }
    else if (!strcmp(a, "--P")) { j.P = atoi(v); ++i; }
    else if (!strcmp(a, "--k")) { j.k = strtoull(v, 0, 10); ++i; }
    else if (!strcmp(a, "--n_mu")) { j.n_mu = atoi(v); ++i; }
    else if (!strcmp(a, "--d_mu")) { j.d_mu = atoi(v); ++i; }
    else if (!strcmp(a, "--B")) { j.B = strtoull(v, 0, 10); ++i; }
    else if (!strcmp(a, "--tau")) { j.tau = atof(v); ++i; }
    else if (!strcmp(a, "--sigma")) { j.sigma = atof(v); ++i; }
    else if (!strcmp(a, "--vlc")) { j.vlc = 1; }
    else if (!strcmp(a, "--ratio")) { j.ratio = atof(v); ++i; }
    else if (!strcmp(a, "--threads")) { j.threads = atoi(v); ++i; }
    else if (!strcmp(a, "--repeat")) { j.repeat = atoi(v); ++i; }
    else if (!strcmp(a, "--in")) { fin = v; ++i; }
    else if (!strcmp(a, "--out")) { fout = v; ++i; }
    else { fprintf(stderr, "unknown argument %s\n", a); return 2; }
  }
  if (!j.N || !fin || !fout) { fprintf(stderr, "need --N --in --out\n"); return 2; }
  size_t S = j.k * (size_t)j.P;
  /* the reference's own preconditions (test.c:130; .cpp:89,128-132,537-548) */
  if (j.N % ((size_t)j.d_mu * S * 16)) { fprintf(stderr, "d_mu*S*16 must divide N\n"); return 2; }
  size_t ntg = S / 4 < 8 ? S / 4 : 8;
  if (ntg == 0 || j.threads % (int)ntg) { fprintf(stderr, "threads must be a multiple of %zu\n", ntg); return 2; }
  size_t bytes = sizeof(double) * 2 * j.N;
  int fd = open(fin, O_RDONLY);
  if (fd < 0) { perror("open in"); return 2; }
  j.in = (const double *)mmap(NULL, bytes, PROT_READ, MAP_SHARED, fd, 0);
  if (j.in == MAP_FAILED) { perror("mmap in"); return 2; }
  double *shared = (double *)mmap(NULL, bytes + 4096, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  if (shared == MAP_FAILED) { perror("mmap out"); return 2; }
  j.out = shared;
  j.times = shared + 2 * j.N;
  size_t Mh = (size_t)j.n_mu * (j.N / S) / (size_t)j.d_mu;
  size_t arena = 2 * sizeof(double) * 2 * Mh * S + ((size_t)64 << 20);
  int rc = soi_mpi_run(j.P, arena, rank_body, &j);
  if (rc) { fprintf(stderr, "a rank failed\n"); return 3; }
  FILE *fo = fopen(fout, "wb");
  if (!fo) { perror("open out"); return 2; }
  fwrite(j.out, 1, bytes, fo);
  fclose(fo);
  fflush(stdout);
  printf("\nSOI_REF_RESULT best_s=%.9f ranks=%d threads=%d times=", j.times[0], j.P, j.threads);
  for (int r = 0; r < j.repeat && r < 62; ++r) printf("%s%.9f", r ? "," : "", j.times[1 + r]);
  printf("\n");
  return 0;
}
