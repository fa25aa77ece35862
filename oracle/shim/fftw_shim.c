/*
 * FP64 discrete Fourier transforms for oracle/shim/fftw3.h (oracle build
 * only). Power-of-two lengths use an iterative radix-2 Cooley-Tukey
 * transform (bit-reversal permutation, then log2(N) butterfly passes with
 * twiddles exp(-+2 pi i k / N) from libm cos/sin); other lengths fall back to
 * the direct O(N^2) sum. Not bitwise equal to FFTW, which itself picks
 * algorithms at run time under FFTW_MEASURE.
 */
#define _POSIX_C_SOURCE 200809L
#include <stdio.h>
#include <stdlib.h>
#include <time.h>
#include <string.h>
#include <math.h>
#include "fftw3.h"

typedef enum { KIND_R2C, KIND_C2R, KIND_C2C } kind_t;

struct fftw_plan_s {
  kind_t kind;
  int n;
  int howmany;
  void * in;
  int istride, idist;
  void * out;
  int ostride, odist;
  int sign;
  double _Complex * tw;   /* exp(sign 2 pi i k / n), k < n */
  double _Complex * work; /* one line of length n */
};

static const double shim_pi = 3.14159265358979323846;

void * fftw_malloc(size_t n){
  return malloc(n > 0 ? n : 1);
}

void fftw_free(void * p){
  free(p);
}

static int is_pow2(int n){
  return n > 0 && 0 == (n & (n - 1));
}

/* in-place transform of one contiguous line, twiddles precomputed */
static void dft_line(const int n, const double _Complex * tw, double _Complex * x, double _Complex * scratch){
  if(1 == n){
    return;
  }
  if(is_pow2(n)){
    /* bit-reversal permutation */
    for(int i = 1, j = 0; i < n; i++){
      int bit = n >> 1;
      for(; j & bit; bit >>= 1){
        j ^= bit;
      }
      j ^= bit;
      if(i < j){
        const double _Complex t = x[i];
        x[i] = x[j];
        x[j] = t;
      }
    }
    for(int len = 2; len <= n; len <<= 1){
      const int half = len >> 1;
      const int step = n / len;
      for(int s = 0; s < n; s += len){
        for(int k = 0; k < half; k++){
          const double _Complex w = tw[k * step];
          const double _Complex a = x[s + k];
          const double _Complex b = x[s + k + half] * w;
          x[s + k] = a + b;
          x[s + k + half] = a - b;
        }
      }
    }
    return;
  }
  for(int k = 0; k < n; k++){
    double _Complex acc = 0.;
    for(int m = 0; m < n; m++){
      acc += x[m] * tw[(int)(((long)k * m) % n)];
    }
    scratch[k] = acc;
  }
  memcpy(x, scratch, sizeof(double _Complex) * (size_t)n);
}

static fftw_plan make_plan(kind_t kind, const int * n, int howmany, void * in, int istride, int idist, void * out, int ostride, int odist, int sign){
  fftw_plan p = calloc(1, sizeof(struct fftw_plan_s));
  p->kind = kind;
  p->n = n[0];
  p->howmany = howmany;
  p->in = in;
  p->istride = istride;
  p->idist = idist;
  p->out = out;
  p->ostride = ostride;
  p->odist = odist;
  p->sign = sign;
  p->tw = malloc(sizeof(double _Complex) * (size_t)p->n);
  for(int k = 0; k < p->n; k++){
    const double arg = 2. * shim_pi * (double)k / (double)p->n;
    p->tw[k] = cos(arg) + (double)sign * sin(arg) * I;
  }
  p->work = malloc(sizeof(double _Complex) * 2 * (size_t)p->n);
  return p;
}

fftw_plan fftw_plan_many_dft_r2c(
    int rank, const int * n, int howmany,
    double * in, const int * inembed, int istride, int idist,
    fftw_complex * out, const int * onembed, int ostride, int odist,
    unsigned flags){
  (void)inembed; (void)onembed; (void)flags;
  if(1 != rank) return NULL;
  return make_plan(KIND_R2C, n, howmany, in, istride, idist, out, ostride, odist, FFTW_FORWARD);
}

fftw_plan fftw_plan_many_dft_c2r(
    int rank, const int * n, int howmany,
    fftw_complex * in, const int * inembed, int istride, int idist,
    double * out, const int * onembed, int ostride, int odist,
    unsigned flags){
  (void)inembed; (void)onembed; (void)flags;
  if(1 != rank) return NULL;
  return make_plan(KIND_C2R, n, howmany, in, istride, idist, out, ostride, odist, FFTW_BACKWARD);
}

fftw_plan fftw_plan_many_dft(
    int rank, const int * n, int howmany,
    fftw_complex * in, const int * inembed, int istride, int idist,
    fftw_complex * out, const int * onembed, int ostride, int odist,
    int sign, unsigned flags){
  (void)inembed; (void)onembed; (void)flags;
  if(1 != rank) return NULL;
  return make_plan(KIND_C2C, n, howmany, in, istride, idist, out, ostride, odist, sign);
}

double tcref_fft_seconds = 0.;

static double shim_now(void){
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1.e-9 * (double)ts.tv_nsec;
}

static void execute(const fftw_plan p);

void fftw_execute(const fftw_plan p){
  const double t0 = shim_now();
  execute(p);
  tcref_fft_seconds += shim_now() - t0;
}

static void execute(const fftw_plan p){
  const int n = p->n;
  const int nh = n / 2 + 1;
  double _Complex * x = p->work;
  double _Complex * scratch = p->work + n;
  for(int m = 0; m < p->howmany; m++){
    switch(p->kind){
      case KIND_R2C: {
        const double * in = (const double *)p->in + (size_t)m * p->idist;
        double _Complex * out = (double _Complex *)p->out + (size_t)m * p->odist;
        for(int k = 0; k < n; k++){
          x[k] = in[(size_t)k * p->istride];
        }
        dft_line(n, p->tw, x, scratch);
        for(int k = 0; k < nh; k++){
          out[(size_t)k * p->ostride] = x[k];
        }
        break;
      }
      case KIND_C2R: {
        const double _Complex * in = (const double _Complex *)p->in + (size_t)m * p->idist;
        double * out = (double *)p->out + (size_t)m * p->odist;
        /* Hermitian extension; DC and Nyquist are taken as real */
        for(int k = 0; k < nh; k++){
          x[k] = in[(size_t)k * p->istride];
        }
        x[0] = creal(x[0]);
        if(0 == n % 2){
          x[n / 2] = creal(x[n / 2]);
        }
        for(int k = nh; k < n; k++){
          x[k] = conj(x[n - k]);
        }
        dft_line(n, p->tw, x, scratch);
        for(int k = 0; k < n; k++){
          out[(size_t)k * p->ostride] = creal(x[k]);
        }
        break;
      }
      case KIND_C2C: {
        const double _Complex * in = (const double _Complex *)p->in + (size_t)m * p->idist;
        double _Complex * out = (double _Complex *)p->out + (size_t)m * p->odist;
        for(int k = 0; k < n; k++){
          x[k] = in[(size_t)k * p->istride];
        }
        dft_line(n, p->tw, x, scratch);
        for(int k = 0; k < n; k++){
          out[(size_t)k * p->ostride] = x[k];
        }
        break;
      }
    }
  }
}

void fftw_destroy_plan(fftw_plan p){
  if(NULL == p) return;
  free(p->tw);
  free(p->work);
  free(p);
}
