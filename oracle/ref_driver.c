/*
 * N-step driver for the reference solver built against the single-rank shims
 * (oracle build only: it links the reference's own .c files under src/).
 *
 * The reference main loop (src/main.c:87-118) has no step-count limit and
 * interleaves logging/saving, so this driver restates only its start-up
 * (src/main.c:46-85: step/time NPYs, domain_init, fluid_init) and then calls
 * integrate() (src/integrate.c:9-35) a fixed number of times.
 *
 *   tcref_<cfg> <ic_dir> <warmup_steps> <timed_steps> [<out_dir> [<steps>]]
 *
 * Environment (as the reference reads it): Re, Pr, coef_dt_adv, coef_dt_dif.
 * The warm-up steps absorb the reference's first-call lazy initialisation
 * (FFT plans, linear-system buffers, Laplacian tables); only the timed steps
 * are clocked, and the seconds spent in the FFT shim's transforms within them
 * are reported beside the total. With <out_dir>, the final state is written in the reference's
 * save layout (src/save.c:74-110) so it can be compared or restarted from;
 * <steps>, a comma-separated list of step counts, also saves the states after
 * those steps (counted from the start, warm-up included) to
 * <out_dir>/step<10 digits>.
 * Prints one JSON line on stdout.
 */
#define _POSIX_C_SOURCE 200809L
#include <stdio.h>
#include <stdlib.h>
#include <time.h>
#include <sys/stat.h>
#include <mpi.h>
#include "domain.h"
#include "fluid.h"
#include "fluid_solver.h"
#include "integrate.h"
#include "fileio.h"
#include "fftw3.h"   /* the shim's tcref_fft_seconds */

static int save_state(const char * dir, size_t step, double time, const domain_t * domain, const fluid_t * fluid){
  mkdir(dir, 0755);
  fileio.w_serial(dir, "step", 0, NULL, fileio.npy_size_t, sizeof(size_t), &step);
  fileio.w_serial(dir, "time", 0, NULL, fileio.npy_double, sizeof(double), &time);
  if(0 != domain_save(dir, domain)) return 1;
  if(0 != fluid_save(dir, domain, fluid)) return 1;
  return 0;
}

/* is n in the comma-separated list s? */
static int listed(const char * s, long n){
  while(NULL != s && '\0' != *s){
    char * end = NULL;
    const long v = strtol(s, &end, 10);
    if(end == s) return 0;
    if(v == n) return 1;
    s = ',' == *end ? end + 1 : end;
  }
  return 0;
}

static double now(void){
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1.e-9 * (double)ts.tv_nsec;
}

int main(int argc, char * argv[]){
  if(argc < 4){
    fprintf(stderr, "usage: %s <ic_dir> <warmup_steps> <timed_steps> [<out_dir> [<steps>]]\n", argv[0]);
    return 2;
  }
  const char * dirname_ic = argv[1];
  const long warmup = atol(argv[2]);
  const long nsteps = atol(argv[3]);
  const char * outdir = argc > 4 ? argv[4] : NULL;
  const char * save_list = argc > 5 ? argv[5] : NULL;
  char stepdir[4096];
  MPI_Init(NULL, NULL);
  if(0 != fileio.init()) return 1;
  size_t step = 0;
  if(0 != fileio.r_serial(dirname_ic, "step", 0, NULL, fileio.npy_size_t, sizeof(size_t), &step)) return 1;
  double time = 0.;
  if(0 != fileio.r_serial(dirname_ic, "time", 0, NULL, fileio.npy_double, sizeof(double), &time)) return 1;
  domain_t domain = {0};
  if(0 != domain_init(dirname_ic, &domain)) return 1;
  fluid_t fluid = {0};
  if(0 != fluid_init(dirname_ic, &domain, &fluid)) return 1;
  double dt = 0.;
  for(long n = 0; n < warmup; n++){
    if(0 != integrate(&domain, &fluid, &dt)) return 1;
    step += 1;
    time += dt;
  }
  const double tic = now();
  const double fft0 = tcref_fft_seconds;
  double saving = 0.;
  for(long n = 0; n < nsteps; n++){
    if(0 != integrate(&domain, &fluid, &dt)) return 1;
    step += 1;
    time += dt;
    if(NULL != outdir && listed(save_list, warmup + n + 1)){
      const double t0 = now();
      mkdir(outdir, 0755);
      snprintf(stepdir, sizeof(stepdir), "%s/step%010ld", outdir, warmup + n + 1);
      if(0 != save_state(stepdir, step, time, &domain, &fluid)) return 1;
      saving += now() - t0;
    }
  }
  const double toc = now() - saving;
  const double fft_seconds = tcref_fft_seconds - fft0;
  if(NULL != outdir){
    if(0 != save_state(outdir, step, time, &domain, &fluid)) return 1;
  }
  const size_t ncells = domain.glsizes[0] * domain.glsizes[1] * domain.glsizes[2];
  printf("{\"cells\": %zu, \"warmup\": %ld, \"steps\": %ld, \"seconds\": %.9e, \"fft_seconds\": %.9e, "
      "\"dt_last\": %.17e, \"time\": %.17e}\n", ncells, warmup, nsteps, toc - tic, fft_seconds, dt, time);
  MPI_Finalize();
  return 0;
}
