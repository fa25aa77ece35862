/*
 * Stand-in for the FFTW3 calls SimpleTCSolver makes (oracle build only;
 * FFTW is a system dependency of the reference, not vendored with it, and
 * absent here). Conventions follow FFTW3's documentation:
 *   - transforms are unnormalised;
 *   - forward (sign -1) computes X[k] = sum_n x[n] exp(-2 pi i n k / N),
 *     backward (sign +1) the same with exp(+2 pi i n k / N);
 *   - r2c keeps the N/2+1 non-negative frequencies;
 *   - c2r reads the N/2+1 frequencies, treats them as Hermitian and ignores
 *     the imaginary parts of the DC and (even N) Nyquist terms.
 * Call sites: src/fluid/compute_potential.c:247-309 (plans), :519-580 (execute).
 */
#if !defined(TCREF_SHIM_FFTW3_H)
#define TCREF_SHIM_FFTW3_H

#include <stddef.h>
#include <complex.h>

typedef double _Complex fftw_complex;
typedef struct fftw_plan_s * fftw_plan;

#define FFTW_FORWARD  (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE  (0U)
#define FFTW_ESTIMATE (1U << 6)

void * fftw_malloc(size_t n);
void fftw_free(void * p);

fftw_plan fftw_plan_many_dft_r2c(
    int rank, const int * n, int howmany,
    double * in, const int * inembed, int istride, int idist,
    fftw_complex * out, const int * onembed, int ostride, int odist,
    unsigned flags);

fftw_plan fftw_plan_many_dft_c2r(
    int rank, const int * n, int howmany,
    fftw_complex * in, const int * inembed, int istride, int idist,
    double * out, const int * onembed, int ostride, int odist,
    unsigned flags);

fftw_plan fftw_plan_many_dft(
    int rank, const int * n, int howmany,
    fftw_complex * in, const int * inembed, int istride, int idist,
    fftw_complex * out, const int * onembed, int ostride, int odist,
    int sign, unsigned flags);

void fftw_execute(const fftw_plan plan);

/* not part of FFTW: wall seconds spent inside fftw_execute so far, so that a
 * timing driver can state the transforms' share of a step */
extern double tcref_fft_seconds;
void fftw_destroy_plan(fftw_plan plan);

#endif // TCREF_SHIM_FFTW3_H
