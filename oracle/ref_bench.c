/*
 * CPU-baseline timing harness for the unmodified reference step (test
 * infrastructure; this repository's own code).  It builds a case through
 * ref_fixture.c (reference setup API), then times only the step loop of the
 * reference Earth driver shape (test_cubedsphere_dipole_background.c:
 * 589-692): dt = min(0.5 * min_f local_timestep, 1.25 * dt_prev), predictor
 * ratio 0.5 * dt / dt_prev (0 on the first step), one planned six-face step.
 *
 * usage: ref_bench KIND NR N WARMUP STEPS [SEED]
 * prints one JSON object on stdout.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct fx_case fx_case;
fx_case *fx_create(int kind, size_t nr, size_t n, unsigned long long seed);
void fx_destroy(fx_case *c);
int fx_local_timestep(fx_case *c, double *dt);
int fx_step(fx_case *c, double ratio, double dt);

static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

int main(int argc, char **argv) {
  if (argc < 6) {
    fprintf(stderr, "usage: %s KIND NR N WARMUP STEPS [SEED]\n", argv[0]);
    return 2;
  }
  const int kind = atoi(argv[1]);
  const size_t nr = (size_t)atol(argv[2]);
  const size_t n = (size_t)atol(argv[3]);
  const int warmup = atoi(argv[4]);
  const int steps = atoi(argv[5]);
  const unsigned long long seed = argc > 6 ? strtoull(argv[6], NULL, 10) : 1;
  const double t0 = now_s();
  fx_case *c = fx_create(kind, nr, n, seed);
  if (c == NULL) { fprintf(stderr, "setup failed\n"); return 1; }
  const double setup = now_s() - t0;
  double dt_prev = 0.0, loop = 0.0;
  for (int s = 0; s < warmup + steps; ++s) {
    const double start = now_s();
    double local;
    if (fx_local_timestep(c, &local) != 0) { fprintf(stderr, "cfl\n"); return 1; }
    double dt = 0.5 * local;
    if (dt_prev > 0.0) dt = fmin(dt, 1.25 * dt_prev);
    const double ratio = dt_prev > 0.0 ? 0.5 * dt / dt_prev : 0.0;
    if (fx_step(c, ratio, dt) != 0) { fprintf(stderr, "step %d\n", s); return 1; }
    dt_prev = dt;
    if (s >= warmup) loop += now_s() - start;
  }
  int threads = 1;
#ifdef _OPENMP
  threads = omp_get_max_threads();
#endif
  const double cells = 6.0 * (double)nr * (double)n * (double)n;
  printf("{\"cells\": %.0f, \"steps\": %d, \"seconds\": %.6f, "
         "\"setup_seconds\": %.3f, \"threads\": %d, "
         "\"cell_updates_per_s\": %.6e, \"last_dt\": %.17g}\n",
         cells, steps, loop, setup, threads,
         cells * (double)steps / loop, dt_prev);
  fx_destroy(c);
  return 0;
}
