/* Times the reference's bundled CPU presolver (PSLP 0.0.11, built from its
 * sources by oracle/pslp.mk) on one LP file with the settings the reference's
 * experiment driver uses (default_settings, verbose off;
 * solver_interface/adapters/pslp.cpp:232-240).  CPU BASELINE ONLY.
 *
 * Every run presolves, then postsolves one reduced point (x at the reduced
 * bounds nearest 0, y = 0, z = 0), the same kind of point the engine's
 * benchmark postsolves, so presolve + postsolve are timed as one step.
 *
 * usage: pslp_driver <lp.bin> [repeat]
 * prints: one line per run "pslp run=<k> presolve_s=<stats> wall_s=<wall>
 *         postsolve_s=<wall> rows=<m'> cols=<n'> nnz=<nnz'> status=<s>" */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "PSLP/PSLP_API.h"
#include "PSLP/PSLP_stats.h"

static double now(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static void* read_block(FILE* f, size_t bytes) {
  void* p = malloc(bytes ? bytes : 1);
  if (!p || fread(p, 1, bytes, f) != bytes) { fprintf(stderr, "read failed\n"); exit(1); }
  return p;
}

int main(int argc, char** argv) {
  if (argc < 2) { fprintf(stderr, "usage: pslp_driver <lp.bin> [repeat]\n"); return 2; }
  const int repeat = argc > 2 ? atoi(argv[2]) : 1;
  FILE* f = fopen(argv[1], "rb");
  if (!f) { perror("open"); return 1; }
  char magic[8];
  int64_t m, n, nnz;
  double obj;
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "GPPLP001", 8)) { fprintf(stderr, "bad LP file\n"); return 1; }
  if (fread(&m, 8, 1, f) != 1 || fread(&n, 8, 1, f) != 1 || fread(&nnz, 8, 1, f) != 1 || fread(&obj, 8, 1, f) != 1) return 1;
  int* ptr = read_block(f, sizeof(int) * (size_t)(m + 1));
  int* idx = read_block(f, sizeof(int) * (size_t)nnz);
  double* val = read_block(f, sizeof(double) * (size_t)nnz);
  double* c = read_block(f, sizeof(double) * (size_t)n);
  double* l = read_block(f, sizeof(double) * (size_t)n);
  double* u = read_block(f, sizeof(double) * (size_t)n);
  double* AL = read_block(f, sizeof(double) * (size_t)m);
  double* AU = read_block(f, sizeof(double) * (size_t)m);
  fclose(f);
  for (int r = 0; r < repeat; ++r) {
    Settings* stgs = default_settings();
    stgs->verbose = false;
    const double t0 = now();
    Presolver* p = new_presolver(val, idx, ptr, (size_t)m, (size_t)n, (size_t)nnz, AL, AU, l, u, c, stgs);
    if (!p) { fprintf(stderr, "new_presolver failed\n"); return 1; }
    const PresolveStatus st = run_presolver(p);
    const double wall = now() - t0;
    const size_t m1 = p->reduced_prob->m, n1 = p->reduced_prob->n;
    double* xr = calloc(n1 ? n1 : 1, sizeof(double));
    double* yr = calloc(m1 ? m1 : 1, sizeof(double));
    double* zr = calloc(n1 ? n1 : 1, sizeof(double));
    for (size_t j = 0; j < n1; ++j) {
      const double lo = p->reduced_prob->lbs[j], hi = p->reduced_prob->ubs[j];
      xr[j] = 0.0 < lo ? lo : (0.0 > hi ? hi : 0.0);
    }
    const double t1 = now();
    postsolve(p, xr, yr, zr);
    const double post = now() - t1;
    printf("pslp run=%d presolve_s=%.6f wall_s=%.6f postsolve_s=%.6f rows=%zu cols=%zu nnz=%zu status=%d\n", r,
           p->stats->time_presolve, wall, post, m1, n1, p->reduced_prob->nnz, (int)st);
    free(xr); free(yr); free(zr);
    fflush(stdout);
    free_presolver(p);
    free_settings(stgs);
  }
  free(ptr); free(idx); free(val); free(c); free(l); free(u); free(AL); free(AU);
  return 0;
}
