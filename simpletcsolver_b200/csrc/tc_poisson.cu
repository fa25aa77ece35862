// Pressure Poisson solver: fluid_compute_potential
// (src/fluid/compute_potential.c:382-583).
//
//   div_ffty_kernel  div(u) / (gamma dt ny nz) at cell centres (assign_input,
//                    :382-425) fused with the real-to-complex DFT along y; two real
//                    lines travel as one complex FFT and are separated afterwards
//   fftz_kernel      complex DFT along z, forward (-1) or backward (+1), in place
//   tdm_kernel       per wavenumber pair (ky, kz) the radial Thomas solve with
//                    c_i = -l_i - u_i + ey/hyxc_i^2 + ez/hz^2 and Neumann ends
//                    (:445-488); the singular (0, 0) system is solved with its last
//                    unknown pinned to zero
//   iffty_kernel     complex-to-real DFT along y (imaginary parts of the DC and
//                    Nyquist terms ignored, as FFTW's c2r does) writing psi with its
//                    Neumann x ghosts and periodic images (extract_output, :427-443)
//
// Transforms are unnormalised like FFTW's; the 1/(ny nz) factor sits in the
// right-hand side as in the reference. FFTs are in-place Stockham passes over
// lines held in shared memory, 16 elements per thread, radix-16 butterflies in
// registers (N = 1024: passes of 16, 16, 4), twiddles exp(-2 pi i m / N)
// tabulated on the host from libm.
//
// Spectral layout: spec[i][kz][ky] (ky fastest), so the y and z transforms read
// and write rows of contiguous wavenumbers and the radial solve, one thread per
// (kz, ky) line, walks i with fully coalesced steps.
#include <type_traits>

#include "tc_common.cuh"
#include "tc_kernels.h"

// resident CTAs per SM requested from the register allocator (measured best
// at 256 x 1024 x 512: 2 for the divergence + y transform, whose version at 3
// spills 296 bytes and takes 2.36 ms against 1.25 (with 8 rows of loads in
// flight 1.30); 2 for the inverse y transform with its spectrum rows staged by
// bulk copies (FP64), 0.68 ms against 0.74 at 3, which spills; the staged rows
// against per-thread loads at 3: 0.74 against 0.84 ms; 3 for the inverse
// transform of FP32 spectra (per-thread loads), 0.77 against 0.83 at 2; a persistent,
// double-buffered version over tiles of two lines at 3 CTAs per SM: 1.00 ms;
// the divergence with its field rows staged in chunks of 512 cells by
// 16-byte asynchronous copies, two chunks in flight: 1.94 ms against 1.25,
// since the per-thread loads already keep more bytes in flight; a persistent
// divergence transform with two roles (256 threads forming the divergence of
// the next tile into one of two line buffers while 256 transform the current
// one, at named barriers, one CTA per SM): 1.31 ms)
// y transforms (divergence + forward, inverse): elements per thread and
// threads per CTA. Measured at 256 x 1024 x 512 (ms, divergence + forward /
// inverse): 16 / 256 1.32 / 0.96; 8 / 512 1.59-1.68 / 1.02; 8 / 256 1.68 / 0.97.
#ifndef TC_DIV_UNROLL
#define TC_DIV_UNROLL 4     // rows of the divergence loads in flight per thread
#endif
#ifndef TC_IFFTY_UNROLL
#define TC_IFFTY_UNROLL 4   // spectrum loads in flight per thread, inverse y transform
#endif
// inverse y transform: strength-reduced psi stores (measured at 256 x 1024 x
// 512: 0.95 -> 0.89 ms per launch; with the stores skipped 0.73 ms, the FFT
// and the spectrum loads). A first FFT pass reading the spectrum straight into
// registers instead of through shared memory measured 1.10 ms (spills).
#ifndef TC_IFFTY_STREAM
#define TC_IFFTY_STREAM 1
#endif
#ifndef TC_FFT_SMEM_MAX
#define TC_FFT_SMEM_MAX (80 * 1024)   // dynamic shared memory the FFT kernels may ask for
#endif
#ifndef TC_FFTY_EPT
#define TC_FFTY_EPT 16
#endif
#ifndef TC_FFTY_THREADS
#define TC_FFTY_THREADS 256
#endif
// z transforms: elements per thread (the largest radix), threads per CTA and
// resident CTAs requested from the register allocator. Measured at
// 256 x 1024 x 512 (ms per launch): 16 / 256 / 2 0.65; 8 / 512 / 2 0.66;
// 8 / 256 / 3 0.58; 8 / 256 / 4 0.67; 8 / 128 / 6 0.72.
#ifndef TC_FFTZ_EPT
#define TC_FFTZ_EPT 8
#endif
#ifndef TC_FFTZ_THREADS
#define TC_FFTZ_THREADS 256
#endif
// z transforms: CTAs of neighbouring wavenumber groups launched back to back
// (grid x over the groups, y over the radial index), so the 32-byte sectors
// that two groups' columns share (rows of nyh = ny/2 + 1 complex values start
// 16 bytes off a sector every other row) are still in L2 for the second.
// Measured at 256 x 1024 x 512: 0.58 -> 0.53 ms per launch.
#ifndef TC_FFTZ_MFAST
#define TC_FFTZ_MFAST 1
#endif
#ifndef TC_FFTZ_MIN_BLOCKS
#define TC_FFTZ_MIN_BLOCKS 3
#endif
#ifndef TC_IFFTY_MIN_BLOCKS
#define TC_IFFTY_MIN_BLOCKS 3
#endif
#ifndef TC_IFFTY_BULK_MIN_BLOCKS
#define TC_IFFTY_BULK_MIN_BLOCKS 2
#endif
#ifndef TC_DIVFFT_MIN_BLOCKS
#define TC_DIVFFT_MIN_BLOCKS 2
#endif
// the same for the float transforms of the FP32-storage mode
#ifndef TC_DIVFFT_MIN_BLOCKS32
#define TC_DIVFFT_MIN_BLOCKS32 3
#endif
#ifndef TC_FFTZ_MIN_BLOCKS32
#define TC_FFTZ_MIN_BLOCKS32 4
#endif
#ifndef TC_IFFTY_MIN_BLOCKS32
#define TC_IFFTY_MIN_BLOCKS32 3
#endif

namespace tcgpu {

constexpr int kDivUnroll = TC_DIV_UNROLL, kIfftyUnroll = TC_IFFTY_UNROLL;

// spectral values as stored: double2, or float2 in the FP32-storage mode
// (arithmetic in double either way)
__device__ __forceinline__ double2 zget(const double2 * p) { return *p; }
__device__ __forceinline__ double2 zget(const float2 * p) {
  const float2 v = *p;
  return make_double2((double)v.x, (double)v.y);
}
__device__ __forceinline__ void zput(double2 * p, double2 v) { *p = v; }
__device__ __forceinline__ void zput(float2 * p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }

// The power-of-two transforms compute in the stored precision: double2, or
// float2 in the FP32-storage mode (the radial Poisson eliminations, the
// divergence and the direct transforms stay double).
template <class CX> struct CxT;
template <> struct CxT<double2> {
  using R = double;
  __device__ static double2 mk(double x, double y) { return make_double2(x, y); }
};
template <> struct CxT<float2> {
  using R = float;
  __device__ static float2 mk(float x, float y) { return make_float2(x, y); }
};
template <class CX>
__device__ __forceinline__ CX mkc(typename CxT<CX>::R x, typename CxT<CX>::R y) { return CxT<CX>::mk(x, y); }
template <class CX>
__device__ __forceinline__ CX cmul(CX a, CX b) {
  return mkc<CX>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// twiddle tables in the transforms' precision
template <class CX> __device__ __forceinline__ const CX * tw_y_of(const Poisson & ps);
template <> __device__ __forceinline__ const double2 * tw_y_of<double2>(const Poisson & ps) { return ps.tw_y; }
template <> __device__ __forceinline__ const float2 * tw_y_of<float2>(const Poisson & ps) { return ps.tw_y32; }
template <class CX> __device__ __forceinline__ const CX * tw_z_of(const Poisson & ps);
template <> __device__ __forceinline__ const double2 * tw_z_of<double2>(const Poisson & ps) { return ps.tw_z; }
template <> __device__ __forceinline__ const float2 * tw_z_of<float2>(const Poisson & ps) { return ps.tw_z32; }

// Shared-memory lines are padded by one slot per 16 complex values so that the
// strided stores of the first pass and the unit-stride accesses of the others
// are both free of bank conflicts.
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int n) { return n + (n >> 4) + 1; }

template <int SIGN, class CX>
__device__ __forceinline__ CX twid(const CX * __restrict__ tw, int m) {
  CX w = __ldg(tw + m);
  if (SIGN > 0) w.y = -w.y;
  return w;
}

// multiply by exp(SIGN i pi / 2) = SIGN i
template <int SIGN, class CX>
__device__ __forceinline__ CX quarter(CX z) {
  return SIGN < 0 ? mkc<CX>(z.y, -z.x) : mkc<CX>(-z.y, z.x);
}

template <int R>
__host__ __device__ constexpr int brev(int a) {
  int b = 0;
  for (int m = 1; m < R; m <<= 1) b = (b << 1) | ((a & m) ? 1 : 0);
  return b;
}

// exp(-2 pi i m / 16), m = 0 .. 7: the twiddles inside the 16-point DFTs,
// cos and sin of multiples of pi/8 (sqrt(2 + sqrt 2)/2, sqrt(2)/2,
// sqrt(2 - sqrt 2)/2), correctly rounded
__device__ constexpr double kC1 = 0.92387953251128674, kC2 = 0.70710678118654752, kC3 = 0.38268343236508977;
template <int SIGN, class CX>
__device__ __forceinline__ CX twid16(int m) {
  using R = typename CxT<CX>::R;
  const double c = m == 0 ? 1. : m == 1 ? kC1 : m == 2 ? kC2 : m == 3 ? kC3 : m == 4 ? 0. : m == 5 ? -kC3
                 : m == 6 ? -kC2 : -kC1;
  const double sn = m == 0 ? 0. : m == 1 ? kC3 : m == 2 ? kC2 : m == 3 ? kC1 : m == 4 ? 1. : m == 5 ? kC1
                  : m == 6 ? kC2 : kC3;
  return mkc<CX>((R)c, (R)(SIGN < 0 ? -sn : sn));
}

// In-register DFT of R points: v[s] <- sum_r v[r] exp(SIGN 2 pi i r s / R),
// iterative radix-2 decimation in time; twiddles exp(SIGN 2 pi i k / len) are
// compile-time constants (R <= 16).
template <int R, int SIGN, class CX>
__device__ __forceinline__ void dft_reg(CX * v, const CX * __restrict__ tw, int N) {
#pragma unroll
  for (int a = 0; a < R; a++) {
    const int b = brev<R>(a);
    if (a < b) {
      const CX t = v[a];
      v[a] = v[b];
      v[b] = t;
    }
  }
#pragma unroll
  for (int len = 2; len <= R; len <<= 1) {
    const int half = len >> 1;
#pragma unroll
    for (int k = 0; k < half; k++) {
      CX w = mkc<CX>(1, 0);
      if (k != 0 && 4 * k != len) w = twid16<SIGN, CX>(k * (16 / len));
#pragma unroll
      for (int s = 0; s < R; s += len) {
        const CX a = v[s + k];
        CX b = v[s + k + half];
        if (4 * k == len) b = quarter<SIGN>(b);
        else if (k != 0) b = cmul(b, w);
        v[s + k] = mkc<CX>(a.x + b.x, a.y + b.y);
        v[s + k + half] = mkc<CX>(a.x - b.x, a.y - b.y);
      }
    }
  }
}

// v[r] *= w^r, r = 1 .. R-1, w = exp(SIGN 2 pi i step / N): with
// TC_FFT_TWIDDLE_PRODUCTS the powers of two of w come from the table and the
// others are their products (fewer loads and registers, up to three extra
// roundings; measured at 256 x 1024 x 512 the y and z transforms 5-11%
// faster); otherwise every power from the table.
#ifndef TC_FFT_TWIDDLE_PRODUCTS
#define TC_FFT_TWIDDLE_PRODUCTS 1
#endif
// twiddle v[r] and v[r + 8] together (radix 16): the products are the same,
// fewer of them are live at once
#ifndef TC_FFT_TWIDDLE_PAIRED
#define TC_FFT_TWIDDLE_PAIRED 1
#endif
template <int R, int SIGN, class CX>
__device__ __forceinline__ void apply_twiddles(CX * v, const CX * __restrict__ tw, int step) {
  if (TC_FFT_TWIDDLE_PRODUCTS) {
    CX p2[4];   // w^1, w^2, w^4, w^8
#pragma unroll
    for (int b = 0; (1 << b) < R; b++) p2[b] = twid<SIGN>(tw, (1 << b) * step);
    CX low[8];  // w^0 .. w^7 as products of p2
    low[0] = mkc<CX>(1, 0);
#pragma unroll
    for (int r = 1; r < R && r < 8; r++) {
      const int hb = 31 - __clz(r);
      low[r] = (r == (1 << hb)) ? p2[hb] : cmul(p2[hb], low[r - (1 << hb)]);
      v[r] = cmul(v[r], low[r]);
#if TC_FFT_TWIDDLE_PAIRED
      // w^(r+8) right away, so that low[r] dies with its last product
      if (R == 16) v[r + 8] = cmul(v[r + 8], cmul(p2[3], low[r]));
#endif
    }
#if TC_FFT_TWIDDLE_PAIRED
    if (R == 16) v[8] = cmul(v[8], p2[3]);
#else
#pragma unroll
    for (int r = 8; r < R; r++) v[r] = cmul(v[r], r == 8 ? p2[3] : cmul(p2[3], low[r - 8]));
#endif
  } else {
#pragma unroll
    for (int r = 1; r < R; r++) v[r] = cmul(v[r], twid<SIGN>(tw, r * step));
  }
}

// Barrier between the passes of one line's transform. LB: the caller's lines
// are contiguous thread ranges (line p = threads p TPL .. p TPL + TPL - 1).
// When TPL is then a multiple of 32 the line's warps wait only for each other
// (named barrier 1 + line; the CTA holds at most 8 lines), so the lines of a
// CTA advance independently; otherwise the whole CTA waits. A caller that
// reads across lines after the transform synchronises the CTA itself.
// Measured at 256 x 1024 x 512 (ms per launch, divergence + y / inverse y):
// CTA barriers 1.29 / 0.89, line barriers 1.27 / 0.86, line barriers and
// paired twiddles 1.26 / 0.83.
#ifndef TC_FFT_LINE_BARRIER
#define TC_FFT_LINE_BARRIER 1
#endif
template <bool LB>
__device__ __forceinline__ void line_barrier(int TPL) {
#if TC_FFT_LINE_BARRIER
  if (LB && (TPL & 31) == 0 && (int)blockDim.x <= 8 * TPL) {
    asm volatile("bar.sync %0, %1;" : : "r"(1 + (int)threadIdx.x / TPL), "r"(TPL) : "memory");
    return;
  }
#endif
  __syncthreads();
}

// One in-place Stockham pass of radix R over a padded line x of length N: the
// thread owns butterflies j = t + b TPL (b < B); Ns is the product of the
// radices already applied. All inputs are read before anything is written.
template <int R, int B, int SIGN, bool LB, class CX>
__device__ __forceinline__ void stockham_pass(CX * x, int N, int Ns, int t, int TPL, const CX * __restrict__ tw) {
  CX v[B][R];
  const int NR = N / R;
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * TPL;
#pragma unroll
    for (int r = 0; r < R; r++) v[b][r] = x[pad(j + r * NR)];
  }
  line_barrier<LB>(TPL);
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * TPL;
    const int k = j & (Ns - 1);
    if (Ns > 1) {
      const int step = k * (N / (Ns * R));
      apply_twiddles<R, SIGN>(v[b], tw, step);
    }
    dft_reg<R, SIGN>(v[b], tw, N);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) x[pad(base + r * Ns)] = v[b][r];
  }
  line_barrier<LB>(TPL);
}

// Full transform of the CTA's lines (N = 2^lg): EPT elements per thread,
// radix-16 passes then the remainder; natural-order output in place.
template <int EPT, int SIGN, bool LB = false, class CX>
__device__ void fft_inplace(CX * x, int N, int lg, int t, int TPL, const CX * __restrict__ tw) {
  int Ns = 1;
  int left = lg;
  while (left > 0) {
    // radix 2^rl, at most EPT (one butterfly's points per thread)
    constexpr int LGE = EPT >= 16 ? 4 : EPT >= 8 ? 3 : EPT >= 4 ? 2 : 1;
    const int rl = left >= LGE ? LGE : left;
    if (EPT == 16) {
      if (rl == 4) stockham_pass<16, 1, SIGN, LB>(x, N, Ns, t, TPL, tw);
      else if (rl == 3) stockham_pass<8, 2, SIGN, LB>(x, N, Ns, t, TPL, tw);
      else if (rl == 2) stockham_pass<4, 4, SIGN, LB>(x, N, Ns, t, TPL, tw);
      else stockham_pass<2, 8, SIGN, LB>(x, N, Ns, t, TPL, tw);
    } else if (EPT == 8) {
      if (rl == 3) stockham_pass<8, 1, SIGN, LB>(x, N, Ns, t, TPL, tw);
      else if (rl == 2) stockham_pass<4, 2, SIGN, LB>(x, N, Ns, t, TPL, tw);
      else stockham_pass<2, 4, SIGN, LB>(x, N, Ns, t, TPL, tw);
    } else {
      if (rl == 2) stockham_pass<4, 1, SIGN, LB>(x, N, Ns, t, TPL, tw);
      else stockham_pass<2, 2, SIGN, LB>(x, N, Ns, t, TPL, tw);
    }
    Ns <<= rl;
    left -= rl;
  }
}

// Stockham pass reading its inputs through ld(e) (IN) instead of from the
// shared line x, and/or writing its outputs through st(e, v) (OUT): the first
// and last passes of a transform whose input or output lives elsewhere, so
// the data crosses shared memory only between passes. A pass that reads and
// writes the shared line synchronises like stockham_pass.
template <int R, int B, int SIGN, bool IN, bool OUT, bool LB, class CX, class Ld, class St>
__device__ __forceinline__ void stockham_pass_io(CX * x, const Ld & ld, const St & st, int N, int Ns, int t,
                                                 int TPL, const CX * __restrict__ tw) {
  CX v[B][R];
  const int NR = N / R;
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * TPL;
#pragma unroll
    for (int r = 0; r < R; r++) v[b][r] = IN ? ld(j + r * NR) : x[pad(j + r * NR)];
  }
  if (!IN && !OUT) line_barrier<LB>(TPL);
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * TPL;
    const int k = j & (Ns - 1);
    if (Ns > 1) {
      const int step = k * (N / (Ns * R));
      apply_twiddles<R, SIGN>(v[b], tw, step);
    }
    dft_reg<R, SIGN>(v[b], tw, N);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) {
      if (OUT) st(base + r * Ns, v[b][r]);
      else x[pad(base + r * Ns)] = v[b][r];
    }
  }
  if (!OUT) line_barrier<LB>(TPL);
}

// Full transform of one line (N = 2^lg) whose input comes from ld (IN_LD) or
// the shared line x, and whose output goes to st (OUT_ST) or back to x; the
// passes between go through x.
template <int EPT, int SIGN, bool IN_LD, bool OUT_ST, bool LB = false, class CX, class Ld, class St>
__device__ void fft_io(CX * x, const Ld & ld, const St & st, int N, int lg, int t, int TPL,
                       const CX * __restrict__ tw) {
  int Ns = 1;
  int left = lg;
  auto pass = [&](auto rc, auto bc) {
    constexpr int R = decltype(rc)::value, B = decltype(bc)::value;
    const bool first = IN_LD && Ns == 1, last = OUT_ST && left == 0;
    if (first && last) stockham_pass_io<R, B, SIGN, true, true, LB>(x, ld, st, N, Ns, t, TPL, tw);
    else if (first) stockham_pass_io<R, B, SIGN, true, false, LB>(x, ld, st, N, Ns, t, TPL, tw);
    else if (last) stockham_pass_io<R, B, SIGN, false, true, LB>(x, ld, st, N, Ns, t, TPL, tw);
    else stockham_pass_io<R, B, SIGN, false, false, LB>(x, ld, st, N, Ns, t, TPL, tw);
  };
  using I = int;
  while (left > 0) {
    // radix 2^rl, at most EPT (one butterfly's points per thread)
    constexpr int LGE = EPT >= 16 ? 4 : EPT >= 8 ? 3 : EPT >= 4 ? 2 : 1;
    const int rl = left >= LGE ? LGE : left;
    left -= rl;
    if (EPT == 16) {
      if (rl == 4) pass(std::integral_constant<I, 16>(), std::integral_constant<I, 1>());
      else if (rl == 3) pass(std::integral_constant<I, 8>(), std::integral_constant<I, 2>());
      else if (rl == 2) pass(std::integral_constant<I, 4>(), std::integral_constant<I, 4>());
      else pass(std::integral_constant<I, 2>(), std::integral_constant<I, 8>());
    } else if (EPT == 8) {
      if (rl == 3) pass(std::integral_constant<I, 8>(), std::integral_constant<I, 1>());
      else if (rl == 2) pass(std::integral_constant<I, 4>(), std::integral_constant<I, 2>());
      else pass(std::integral_constant<I, 2>(), std::integral_constant<I, 4>());
    } else {
      if (rl == 2) pass(std::integral_constant<I, 4>(), std::integral_constant<I, 1>());
      else pass(std::integral_constant<I, 2>(), std::integral_constant<I, 2>());
    }
    Ns <<= rl;
  }
}

// --------------------------------------------------------------- forward y
// CTA: P complex lines (radial indices i0 .. i0+2P-1) x all j at one k;
// TPL = ny / EPT threads per line.
template <int EPT, class T, class Z>
__global__ void __launch_bounds__(TC_FFTY_THREADS, sizeof(Z) == 8 ? TC_DIVFFT_MIN_BLOCKS32 : TC_DIVFFT_MIN_BLOCKS)
div_ffty_kernel(Geo g, Coefs cf, Poisson ps, int P, int lg,
                const T * __restrict__ ux, const T * __restrict__ uy,
                const T * __restrict__ uz, const double * __restrict__ dtp, int rkstep) {
  extern __shared__ double2 smem[];
  using R = typename CxT<Z>::R;   // the transform's precision
  Z * const zsm = reinterpret_cast<Z *>(smem);
  const int ny = g.ny, nx = g.nx, nz = g.nz;
  const int TI = 2 * P;
  const int TPL = ny / EPT;
  const int LS = padded_len(ny);
  const int i0 = blockIdx.x * TI + 1;
  const int k = blockIdx.y + 1;
  const double norm = 1. * ny * nz;
  const double prefactor = 1. / (rk_gamma(rkstep) * (*dtp)) / norm;
  // When TI divides the block size (ny >= 2 EPT) each thread keeps one radial
  // index and visits rows j = j0, j0 + blockDim / TI, ... (2 EPT of them);
  // otherwise (short lines) the plain element loop.
  if (blockDim.x % TI != 0) {
    for (int idx = threadIdx.x; idx < TI * ny; idx += blockDim.x) {
      const int ii = idx % TI;
      const int j = idx / TI + 1;
      const int i = i0 + ii;
      double val = 0.;
      if (i <= nx) {
        const double ux_xm = __ldg(ux + sidx_f<T>(g, i, j, k));
        const double ux_xp = __ldg(ux + sidx_f<T>(g, i + 1, j, k));
        const double uy_ym = __ldg(uy + sidx_c<T>(g, i, j, k));
        const double uy_yp = __ldg(uy + sidx_c<T>(g, i, j + 1, k));
        const double uz_zm = __ldg(uz + sidx_c<T>(g, i, j, k));
        const double uz_zp = __ldg(uz + sidx_c<T>(g, i, j, k + 1));
        const double jxm = __ldg(cf.c_jf + i), jxp = __ldg(cf.c_jf + i + 1);
        const double jy = __ldg(cf.c_e1 + i), jz = __ldg(cf.c_e2 + i);
        const double div = __ldg(cf.c_invjdxc + i) * (
            -jxm * ux_xm + jxp * ux_xp
            - jy * uy_ym + jy * uy_yp
            - jz * uz_zm + jz * uz_zp);
        val = prefactor * div;
      }
      R * line = reinterpret_cast<R *>(zsm + (size_t)(ii >> 1) * LS);
      line[2 * pad(j - 1) + (ii & 1)] = (R)val;
    }
  } else {
    const int ii = threadIdx.x % TI;
    const int j0 = threadIdx.x / TI + 1;
    const int jstep = blockDim.x / TI;
    const int i = i0 + ii;
    R * line = reinterpret_cast<R *>(zsm + (size_t)(ii >> 1) * LS);
    if (i <= nx) {
      const double jxm = __ldg(cf.c_jf + i), jxp = __ldg(cf.c_jf + i + 1);
      const double jy = __ldg(cf.c_e1 + i), jz = __ldg(cf.c_e2 + i);
      const double ijd = __ldg(cf.c_invjdxc + i);
      const T * __restrict__ pxm = ux + sidx_f<T>(g, i, 0, k);
      const T * __restrict__ pym = uy + sidx_c<T>(g, i, 0, k);
      const T * __restrict__ pzm = uz + sidx_c<T>(g, i, 0, k);
      const T * __restrict__ pzp = uz + sidx_c<T>(g, i, 0, k + 1);
      const int sf = srow_f<T>(g), sc = srow_c<T>(g);
#pragma unroll kDivUnroll
      for (int r = 0; r < 2 * EPT; r++) {
        const int j = j0 + r * jstep;
        const double ux_xm = __ldg(pxm + (size_t)j * sf);
        const double ux_xp = __ldg(pxm + (size_t)j * sf + 1);
        const double uy_ym = __ldg(pym + (size_t)j * sc);
        const double uy_yp = __ldg(pym + (size_t)(j + 1) * sc);
        const double uz_zm = __ldg(pzm + (size_t)j * sc);
        const double uz_zp = __ldg(pzp + (size_t)j * sc);
        const double div = ijd * (
            -jxm * ux_xm + jxp * ux_xp
            - jy * uy_ym + jy * uy_yp
            - jz * uz_zm + jz * uz_zp);
        line[2 * pad(j - 1) + (ii & 1)] = (R)(prefactor * div);
      }
    } else {
#pragma unroll 8
      for (int r = 0; r < 2 * EPT; r++) line[2 * pad(j0 + r * jstep - 1) + (ii & 1)] = 0.;
    }
  }
  __syncthreads();
  const int p = threadIdx.x / TPL, t = threadIdx.x % TPL;
  fft_inplace<EPT, -1, true>(zsm + (size_t)p * LS, ny, lg, t, TPL, tw_y_of<Z>(ps));
  if (TC_FFT_LINE_BARRIER) __syncthreads();
  // separate the two real transforms and store the ny/2+1 non-negative
  // wavenumbers: m < ny/2 for every radial index (power-of-two index
  // arithmetic), then the Nyquist terms
  const int nyh = ps.nyh, half = ny >> 1;
  auto put = [&](int ii, int m) {
    const int i = i0 + ii;
    if (i > nx) return;
    const Z * z = zsm + (size_t)(ii >> 1) * LS;
    const Z zm = z[pad(m)];
    const Z zn = z[pad((ny - m) & (ny - 1))];
    Z out;
    if ((ii & 1) == 0) out = mkc<Z>(R(0.5) * (zm.x + zn.x), R(0.5) * (zm.y - zn.y));
    else out = mkc<Z>(R(0.5) * (zm.y + zn.y), R(-0.5) * (zm.x - zn.x));
    static_cast<Z *>(ps.spec)[((size_t)(i - 1) * nz + (k - 1)) * nyh + m] = out;
  };
  for (int idx = threadIdx.x; idx < TI * half; idx += blockDim.x) put(idx >> (lg - 1), idx & (half - 1));
  for (int ii = threadIdx.x; ii < TI; ii += blockDim.x) put(ii, half);
}

// --------------------------------------------------------------- z transforms
// CTA: P lines (wavenumbers m0 .. m0+P-1) of one radial index, all kz. Thread
// (p, t) = (tid mod P, tid / P): lanes run along the contiguous wavenumbers, so
// the first pass reads and the last pass writes rows of P values straight from
// and to the spectral array.
template <int EPT, int SIGN, class Z>
__global__ void __launch_bounds__(TC_FFTZ_THREADS, sizeof(Z) == 8 ? TC_FFTZ_MIN_BLOCKS32 : TC_FFTZ_MIN_BLOCKS)
fftz_kernel(Geo g, Poisson ps, int P, int lg) {
  extern __shared__ double2 smem[];
  const int nz = g.nz, nyh = ps.nyh;
  const int TPL = nz / EPT;
  const int LS = padded_len(nz);
#if TC_FFTZ_MFAST
  const int i = blockIdx.y;          // 0..nx-1
  const int p = threadIdx.x % P, t = threadIdx.x / P;
  const int m = blockIdx.x * P + p;
#else
  const int i = blockIdx.x;          // 0..nx-1
  const int p = threadIdx.x % P, t = threadIdx.x / P;
  const int m = blockIdx.y * P + p;
#endif
  Z * col = static_cast<Z *>(ps.spec) + (size_t)i * nz * nyh + m;
  const bool gv = m < nyh;
  auto ld = [&](int e) { return gv ? col[(size_t)e * nyh] : mkc<Z>(0, 0); };
  auto st = [&](int e, Z v) { if (gv) col[(size_t)e * nyh] = v; };
  fft_io<EPT, SIGN, true, true>(reinterpret_cast<Z *>(smem) + (size_t)p * LS, ld, st, nz, lg, t, TPL, tw_z_of<Z>(ps));
}

// --------------------------------------------------------------- radial solve
// rows fetched ahead of the recurrence (measured at 256 x 1024 x 512: 2 rows
// 0.89 ms, 4 rows 0.92 ms, none 1.00 ms)
#ifndef TC_TDM_PREFETCH
#define TC_TDM_PREFETCH 2
#endif
template <class Z>
__global__ void __launch_bounds__(128, 8)
tdm_kernel(Geo g, Poisson ps, const double * __restrict__ tab_y, const double * __restrict__ tab_z,
           const double * __restrict__ base) {
  const int nyh = ps.nyh, nz = g.nz, n = g.nx;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)nyh * nz) return;
  const int m = (int)(tid % nyh);
  const int kz = (int)(tid / nyh);
  const size_t st = (size_t)nz * nyh;
  Z * q = static_cast<Z *>(ps.spec) + (size_t)kz * nyh + m;
  double * v = ps.vscr + (size_t)kz * nyh + m;
  const double tz = __ldg(tab_z + kz);
  const bool pin = (m == 0 && kz == 0);
  // c_i = -l_i - u_i + ey/hyxc/hyxc + ez/hz/hz, c_0 += l_0, c_{n-1} += u_{n-1}
  auto cdiag = [&](int i) {
    double c = __ldg(base + i) + __ldg(tab_y + (size_t)i * nyh + m) + tz;
    if (i == 0) c += __ldg(ps.tl);
    if (i == n - 1) c += __ldg(ps.tu + n - 1);
    return c;
  };
  if (n == 1) {
    const double c = cdiag(0);
    const double2 x = zget(q);
    zput(q, pin ? make_double2(0., 0.) : make_double2(x.x / c, x.y / c));
    return;
  }
  // forward elimination (src/tdm.c:24-44)
  double c0 = cdiag(0);
  double vprev = __ldg(ps.tu) / c0;
  v[0] = vprev;
  double2 qprev = zget(q);
  qprev = make_double2(qprev.x / c0, qprev.y / c0);
  zput(q, qprev);
  // rows are fetched G at a time ahead of the recurrence, so G loads per
  // thread are in flight together
  constexpr int G = TC_TDM_PREFETCH;
  for (int ib = 1; ib < n - 1; ib += G) {
    double2 r[G];
    double cd[G];
#pragma unroll
    for (int u = 0; u < G; u++) {
      const int i = ib + u;
      if (i < n - 1) {
        r[u] = zget(q + (size_t)i * st);
        cd[u] = cdiag(i);
      }
    }
#pragma unroll
    for (int u = 0; u < G; u++) {
      const int i = ib + u;
      if (i < n - 1) {
        const double l = __ldg(ps.tl + i);
        const double val = 1. / (cd[u] - l * vprev);
        vprev = val * __ldg(ps.tu + i);
        v[(size_t)i * st] = vprev;
        qprev = make_double2(val * (r[u].x - l * qprev.x), val * (r[u].y - l * qprev.y));
        zput(q + (size_t)i * st, qprev);
      }
    }
  }
  {
    const int i = n - 1;
    const double l = __ldg(ps.tl + i);
    const double val = cdiag(i) - l * vprev;
    const double2 r = zget(q + (size_t)i * st);
    double2 x;
    if (pin) x = make_double2(0., 0.);
    else {
      const double iv = 1. / val;
      x = make_double2(iv * (r.x - l * qprev.x), iv * (r.y - l * qprev.y));
    }
    zput(q + (size_t)i * st, x);
    qprev = x;
  }
  // back substitution
  for (int ib = n - 2; ib >= 0; ib -= G) {
    double2 r[G];
    double vi[G];
#pragma unroll
    for (int u = 0; u < G; u++) {
      const int i = ib - u;
      if (i >= 0) {
        vi[u] = v[(size_t)i * st];
        r[u] = zget(q + (size_t)i * st);
      }
    }
#pragma unroll
    for (int u = 0; u < G; u++) {
      const int i = ib - u;
      if (i >= 0) {
        qprev = make_double2(r[u].x - vi[u] * qprev.x, r[u].y - vi[u] * qprev.y);
        zput(q + (size_t)i * st, qprev);
      }
    }
  }
}

// ---------------------------------------------------- radial solves by warps
// Factors of line l = kz nyh + m (the forward elimination of src/tdm.c:24-44
// with the Neumann ends folded into the diagonal, as in tdm_kernel): the
// forward sweep y_i = w_i (q_i - l_i y_{i-1}), y_{-1} = 0, and the back
// substitution x_i = y_i - v_i x_{i+1}, x_n = 0 (v_{n-1} = 0). The pinned mode
// (line 0) has w_{n-1} = 0, which sets its last unknown to zero.
__global__ void tdm_factor_kernel(Geo g, Poisson ps, const double * __restrict__ tab_y,
                                  const double * __restrict__ tab_z, const double * __restrict__ base) {
  const int nyh = ps.nyh, nz = g.nz, n = g.nx, fe = ps.fe;
  const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= (long long)nyh * nz) return;
  const int m = (int)(l % nyh), kz = (int)(l / nyh);
  const double tz = tab_z[kz];
  auto cdiag = [&](int i) {
    double c = base[i] + tab_y[(size_t)i * nyh + m] + tz;
    if (i == 0) c += ps.tl[0];
    if (i == n - 1) c += ps.tu[n - 1];
    return c;
  };
  double * w = ps.fw + (size_t)l * n;
  double * v = ps.fv + (size_t)l * n;
  auto at = [&](int i) { return (i % fe) * 32 + i / fe; };
  const double c0 = cdiag(0);
  double vprev = ps.tu[0] / c0;
  w[at(0)] = 1. / c0;
  v[at(0)] = vprev;
  for (int i = 1; i < n - 1; i++) {
    const double val = 1. / (cdiag(i) - ps.tl[i] * vprev);
    vprev = val * ps.tu[i];
    w[at(i)] = val;
    v[at(i)] = vprev;
  }
  const double last = cdiag(n - 1) - ps.tl[n - 1] * vprev;
  w[at(n - 1)] = (l == 0) ? 0. : 1. / last;
  v[at(n - 1)] = 0.;
}

void launch_tdm_factors(const Geo & g, const Poisson & ps, const double * tab_y, const double * tab_z,
                        const double * base, cudaStream_t st) {
  const long long nl = (long long)ps.nyh * g.nz;
  tdm_factor_kernel<<<(unsigned)((nl + 127) / 128), 128, 0, st>>>(g, ps, tab_y, tab_z, base);
}

// The radial systems of 16 consecutive lines (kz, m) as one tile: for every i
// their 16 complex values are contiguous (256 bytes), loaded and stored once;
// each warp solves whole lines from shared memory with the affine-map scans
// (E = n / 32 points per lane, in-register prefix + 5-level shuffle scan).
constexpr int TDM_PT = 16;
// resident CTAs per SM requested from the register allocator (0: the
// allocator's own choice), and the factor rows loaded ahead of their use: the
// warp's first w row with the tile, each line's v row before its forward scan.
// Measured at 256 x 1024 x 512 (ms per launch): 0.58, prefetched 0.56; 3
// resident CTAs (80 registers, 64 bytes spilled) 0.58.
#ifndef TC_TDM_LINES_MB
#define TC_TDM_LINES_MB 0
#endif
#if TC_TDM_LINES_MB > 0
#define TC_TDM_LINES_BOUNDS __launch_bounds__(256, TC_TDM_LINES_MB)
#else
#define TC_TDM_LINES_BOUNDS __launch_bounds__(256)
#endif
#ifndef TC_TDM_LINES_PREFETCH
#define TC_TDM_LINES_PREFETCH 1
#endif

template <int E, class Z>
__global__ void TC_TDM_LINES_BOUNDS tdm_lines_kernel(Geo g, Poisson ps) {
  constexpr int N = 32 * E, NT = 256, PER = N * TDM_PT / NT;
  extern __shared__ double2 tq[];
  const int nyh = ps.nyh;
  const long long nlines = (long long)nyh * g.nz;
  const long long l0 = (long long)blockIdx.x * TDM_PT;
  const int nt = (int)min((long long)TDM_PT, nlines - l0);
  const size_t st = (size_t)nlines;               // complex values between radial indices
  Z * spec = static_cast<Z *>(ps.spec);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#if TC_TDM_LINES_PREFETCH
  double wq[E];   // w of the warp's first line, in flight with the tile
  if (wid < nt) {
    const double * w = ps.fw + (size_t)(l0 + wid) * N;
#pragma unroll
    for (int e = 0; e < E; e++) wq[e] = w[e * 32 + lane];
  }
#endif
  {
    double2 buf[PER];
#pragma unroll
    for (int r = 0; r < PER; r++) {
      const int q = threadIdx.x + r * NT, t = q % TDM_PT, i = q / TDM_PT;
      buf[r] = t < nt ? zget(spec + (size_t)i * st + l0 + t) : make_double2(0., 0.);
    }
#pragma unroll
    for (int r = 0; r < PER; r++) {
      const int q = threadIdx.x + r * NT, t = q % TDM_PT, i = q / TDM_PT;
      tq[i * TDM_PT + (t ^ ((i / E) & (TDM_PT - 1)))] = buf[r];
    }
  }
  __syncthreads();
  double ll[E];
#pragma unroll
  for (int e = 0; e < E; e++) ll[e] = ps.tl[lane * E + e];
  for (int t = wid; t < nt; t += NT / 32) {
    const long long l = l0 + t;
    const double * w = ps.fw + (size_t)l * N;
    const double * v = ps.fv + (size_t)l * N;
    const int sw = t ^ (lane & (TDM_PT - 1));
    double fa[E], bre[E], bim[E];
#if TC_TDM_LINES_PREFETCH
    double vq[E];
#pragma unroll
    for (int e = 0; e < E; e++) vq[e] = v[e * 32 + lane];
#endif
#pragma unroll
    for (int e = 0; e < E; e++) {
      const double2 qv = tq[(lane * E + e) * TDM_PT + sw];
#if TC_TDM_LINES_PREFETCH
      const double we = (t == wid) ? wq[e] : w[e * 32 + lane];
#else
      const double we = w[e * 32 + lane];
#endif
      fa[e] = -we * ll[e];
      bre[e] = we * qv.x;
      bim[e] = we * qv.y;
    }
    // forward: prefix of the lane's maps, then across lanes
#pragma unroll
    for (int d = 1; d < E; d <<= 1) {
#pragma unroll
      for (int e = E - 1; e >= d; e--) {
        bre[e] = fa[e] * bre[e - d] + bre[e];
        bim[e] = fa[e] * bim[e - d] + bim[e];
        fa[e] = fa[e] * fa[e - d];
      }
    }
    double A = fa[E - 1], Bre = bre[E - 1], Bim = bim[E - 1];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double oa = __shfl_up_sync(0xffffffffu, A, off);
      const double ore = __shfl_up_sync(0xffffffffu, Bre, off);
      const double oim = __shfl_up_sync(0xffffffffu, Bim, off);
      if (lane >= off) { Bre = A * ore + Bre; Bim = A * oim + Bim; A = A * oa; }
    }
    double yre = __shfl_up_sync(0xffffffffu, Bre, 1), yim = __shfl_up_sync(0xffffffffu, Bim, 1);
    if (lane == 0) { yre = 0.; yim = 0.; }
#pragma unroll
    for (int e = 0; e < E; e++) {
      bre[e] = fa[e] * yre + bre[e];
      bim[e] = fa[e] * yim + bim[e];
    }
    // backward: x_i = y_i - v_i x_{i+1}, suffix maps
#pragma unroll
#if TC_TDM_LINES_PREFETCH
    for (int e = 0; e < E; e++) fa[e] = -vq[e];
#else
    for (int e = 0; e < E; e++) fa[e] = -v[e * 32 + lane];
#endif
#pragma unroll
    for (int d = 1; d < E; d <<= 1) {
#pragma unroll
      for (int e = 0; e + d < E; e++) {
        bre[e] = fa[e] * bre[e + d] + bre[e];
        bim[e] = fa[e] * bim[e + d] + bim[e];
        fa[e] = fa[e] * fa[e + d];
      }
    }
    A = fa[0];
    Bre = bre[0];
    Bim = bim[0];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double oa = __shfl_down_sync(0xffffffffu, A, off);
      const double ore = __shfl_down_sync(0xffffffffu, Bre, off);
      const double oim = __shfl_down_sync(0xffffffffu, Bim, off);
      if (lane + off < 32) { Bre = A * ore + Bre; Bim = A * oim + Bim; A = A * oa; }
    }
    double xre = __shfl_down_sync(0xffffffffu, Bre, 1), xim = __shfl_down_sync(0xffffffffu, Bim, 1);
    if (lane == 31) { xre = 0.; xim = 0.; }
#pragma unroll
    for (int e = 0; e < E; e++)
      tq[(lane * E + e) * TDM_PT + sw] = make_double2(fa[e] * xre + bre[e], fa[e] * xim + bim[e]);
  }
  __syncthreads();
#pragma unroll 8
  for (int r = 0; r < PER; r++) {
    const int q = threadIdx.x + r * NT, t = q % TDM_PT, i = q / TDM_PT;
    if (t < nt) zput(spec + (size_t)i * st + l0 + t, tq[i * TDM_PT + (t ^ ((i / E) & (TDM_PT - 1)))]);
  }
}

template <class Z>
static bool launch_tdm_lines(const Geo & g, const Poisson & ps, cudaStream_t st) {
  const long long nl = (long long)ps.nyh * g.nz;
  const unsigned nblk = (unsigned)((nl + TDM_PT - 1) / TDM_PT);
  const size_t smem = sizeof(double2) * (size_t)g.nx * TDM_PT;
  switch (ps.fe) {
    case 2: tdm_lines_kernel<2, Z><<<nblk, 256, smem, st>>>(g, ps); return true;
    case 4: tdm_lines_kernel<4, Z><<<nblk, 256, smem, st>>>(g, ps); return true;
    case 8: tdm_lines_kernel<8, Z><<<nblk, 256, smem, st>>>(g, ps); return true;
    default: return false;
  }
}

// --------------------------------------------------------------- inverse y
// BULK (FP64 spectra): one thread copies the two spectrum rows of each line
// pair (nyh values each, 16-byte aligned) straight into the pair's line buffer
// with bulk asynchronous copies, all rows of the CTA in flight at once; every
// thread then reads the values its extension needs from shared memory, and
// after a barrier writes the extended lines over the staged rows. Otherwise
// each thread loads its values from global memory.
template <int EPT, class Z, bool BULK>
__global__ void __launch_bounds__(TC_FFTY_THREADS, BULK ? TC_IFFTY_BULK_MIN_BLOCKS
                                                  : sizeof(Z) == 8 ? TC_IFFTY_MIN_BLOCKS32 : TC_IFFTY_MIN_BLOCKS)
iffty_kernel(Geo g, Poisson ps, int P, int lg, double * __restrict__ psi) {
  static_assert(!BULK || sizeof(Z) == 16, "bulk rows: FP64 spectra (16-byte values)");
  extern __shared__ double2 smem[];
  using R = typename CxT<Z>::R;   // the transform's precision
  Z * const zsm = reinterpret_cast<Z *>(smem);
  const int ny = g.ny, nx = g.nx, nz = g.nz, nyh = ps.nyh;
  const int TI = 2 * P;
  const int TPL = ny / EPT;
  const int LS = padded_len(ny);
  const int i0 = blockIdx.x * TI + 1;
  const int k = blockIdx.y + 1;
  // Hermitian extension of the two packed real lines: each stored wavenumber
  // mr < ny/2 gives the line's values at m = mr and m = ny - mr; the Nyquist
  // terms follow (imaginary parts of DC and Nyquist ignored, as FFTW's c2r
  // does)
  const int half = ny >> 1;
  const Z * sp = static_cast<const Z *>(ps.spec);
  if constexpr (BULK) {
    unsigned long long * bar = reinterpret_cast<unsigned long long *>(smem + (size_t)P * LS);
    if (threadIdx.x == 0) {
      mbar_init(bar, 1);
      fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned row = (unsigned)(nyh * sizeof(double2));
      unsigned total = 0;
      for (int q = 0; q < TI; q++)
        if (i0 + q <= nx) total += row;
      mbar_expect_tx(bar, total);
      for (int q = 0; q < TI; q++)
        if (i0 + q <= nx)
          bulk_g2s(smem + (size_t)(q >> 1) * LS + (q & 1) * nyh, sp + ((size_t)(i0 + q - 1) * nz + (k - 1)) * nyh, row,
                   bar);
    }
    if (!mbar_wait(bar, 0)) {   // the copies did not land: report, store nothing
      if (threadIdx.x == 0) atomicOr(ps.status, ST_TIMEOUT);
      return;
    }
    double2 xa[EPT / 2], xb[EPT / 2];
#pragma unroll
    for (int r = 0; r < EPT / 2; r++) {
      const int u = threadIdx.x + r * blockDim.x;
      const int mr = u & (half - 1), pp = u >> (lg - 1);
      const double2 * rows = smem + (size_t)pp * LS;
      xa[r] = i0 + 2 * pp <= nx ? rows[mr] : make_double2(0., 0.);
      xb[r] = i0 + 2 * pp + 1 <= nx ? rows[nyh + mr] : make_double2(0., 0.);
    }
    double qa = 0., qb = 0.;
    const int pq = threadIdx.x;
    if (pq < P) {
      const double2 * rows = smem + (size_t)pq * LS;
      if (i0 + 2 * pq <= nx) qa = rows[half].x;
      if (i0 + 2 * pq + 1 <= nx) qb = rows[nyh + half].x;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < EPT / 2; r++) {
      const int u = threadIdx.x + r * blockDim.x;
      const int mr = u & (half - 1), pp = u >> (lg - 1);
      double2 a = xa[r], b = xb[r];
      if (mr == 0) { a.y = 0.; b.y = 0.; }
      double2 * line = smem + (size_t)pp * LS;
      line[pad(mr)] = make_double2(a.x - b.y, a.y + b.x);
      if (mr != 0) line[pad(ny - mr)] = make_double2(a.x + b.y, -a.y + b.x);
    }
    if (pq < P) smem[(size_t)pq * LS + pad(half)] = make_double2(qa, qb);
  } else {
#pragma unroll kIfftyUnroll
    for (int r = 0; r < EPT / 2; r++) {     // P half = blockDim EPT / 2 items
      const int u = threadIdx.x + r * blockDim.x;
      const int mr = u & (half - 1);
      const int pp = u >> (lg - 1);
      const int ia = i0 + 2 * pp, ib = ia + 1;
      Z xa = mkc<Z>(0, 0), xb = mkc<Z>(0, 0);
      if (ia <= nx) xa = sp[((size_t)(ia - 1) * nz + (k - 1)) * nyh + mr];
      if (ib <= nx) xb = sp[((size_t)(ib - 1) * nz + (k - 1)) * nyh + mr];
      if (mr == 0) { xa.y = 0; xb.y = 0; }
      Z * line = zsm + (size_t)pp * LS;
      line[pad(mr)] = mkc<Z>(xa.x - xb.y, xa.y + xb.x);
      if (mr != 0) line[pad(ny - mr)] = mkc<Z>(xa.x + xb.y, -xa.y + xb.x);
    }
    for (int pp = threadIdx.x; pp < P; pp += blockDim.x) {
      const int ia = i0 + 2 * pp, ib = ia + 1;
      const R xa = ia <= nx ? sp[((size_t)(ia - 1) * nz + (k - 1)) * nyh + half].x : R(0);
      const R xb = ib <= nx ? sp[((size_t)(ib - 1) * nz + (k - 1)) * nyh + half].x : R(0);
      zsm[(size_t)pp * LS + pad(half)] = mkc<Z>(xa, xb);
    }
  }
  __syncthreads();
  {
    const int p = threadIdx.x / TPL, t = threadIdx.x % TPL;
    fft_inplace<EPT, +1, true>(zsm + (size_t)p * LS, ny, lg, t, TPL, tw_y_of<Z>(ps));
  }
  if (TC_FFT_LINE_BARRIER) __syncthreads();
  // one radial index per thread when TI divides the block size (ny >= 2 EPT),
  // else the plain element loop
  // (TI and the block size are powers of two)
  const int lgt = __ffs(TI) - 1;
  const bool fixed_i = blockDim.x % TI == 0;
#if TC_IFFTY_STREAM
  if (fixed_i) {
    // the thread's radial index is fixed and its rows j advance by a constant
    // stride: one pointer step per store, the images only on edge rows/planes
    const int ii = threadIdx.x & (TI - 1), i = i0 + ii;
    if (i > nx) return;
    const int js = blockDim.x >> lgt;
    const Z * zs = zsm + (size_t)(ii >> 1) * LS;
    const bool hi = (ii & 1) != 0, kedge = k == 1 || k == nz;
    int j = (threadIdx.x >> lgt) + 1;
    double * out = psi + cidx(g, i, j, k);
    const size_t step = (size_t)js * (nx + 2);
#pragma unroll 4
    for (int r = 0; r < 2 * EPT; r++, j += js, out += step) {
      const Z z = zs[pad(j - 1)];
      const double val = (double)(hi ? z.y : z.x);
      *out = val;
      if (i == 1) out[-1] = val;
      if (i == nx) out[1] = val;
      if (kedge || j == 1 || j == ny)
        for_images(j, k, ny, nz, [&](int jj, int kk) {
          const size_t q = cidx(g, i, jj, kk);
          psi[q] = val;
          if (i == 1) psi[q - 1] = val;
          if (i == nx) psi[q + 1] = val;
        });
    }
    return;
  }
#endif
  const int nr = fixed_i ? 2 * EPT : (TI * ny + blockDim.x - 1) / blockDim.x;
#pragma unroll 4
  for (int r = 0; r < nr; r++) {
    const int idx = fixed_i ? threadIdx.x : threadIdx.x + r * blockDim.x;
    if (idx >= TI * ny) break;
    const int ii = idx & (TI - 1);
    const int j = fixed_i ? (idx >> lgt) + 1 + r * (blockDim.x >> lgt) : (idx >> lgt) + 1;
    const int i = i0 + ii;
    if (i > nx) continue;
    const Z z = zsm[(size_t)(ii >> 1) * LS + pad(j - 1)];
    const double val = (double)((ii & 1) ? z.y : z.x);
    auto put = [&](int jj, int kk) {
      psi[cidx(g, i, jj, kk)] = val;
      if (i == 1) psi[cidx(g, 0, jj, kk)] = val;
      if (i == nx) psi[cidx(g, nx + 1, jj, kk)] = val;
    };
    put(j, k);
    for_images(j, k, ny, nz, put);
  }
}

// --------------------------------------------------------------- direct DFTs
// Lengths that are not powers of two (even ny, nz a multiple of 4, as FFTW
// plans any length: compute_potential.c:247-309) take direct transforms: each
// output wavenumber is the sum over the line with twiddles tw[(j m) mod N] =
// exp(-2 pi i (j m mod N) / N) from the same tables. O(N^2) per line, FP64
// accumulation, FFTW's conventions (unnormalised, r2c keeps N/2+1 terms, c2r
// ignores the imaginary parts of the DC and Nyquist terms).

// divergence (as div_ffty_kernel) of one (i, k) line into shared memory, then
// its r2c transform along y
template <class T, class Z>
__global__ void div_dfty_kernel(Geo g, Coefs cf, Poisson ps, const T * __restrict__ ux, const T * __restrict__ uy,
                                const T * __restrict__ uz, const double * __restrict__ dtp, int rkstep) {
  extern __shared__ double line[];
  const int ny = g.ny, nz = g.nz, nyh = ps.nyh;
  const int i = blockIdx.x + 1, k = blockIdx.y + 1;
  const double prefactor = 1. / (rk_gamma(rkstep) * (*dtp)) / (1. * ny * nz);
  const double jxm = __ldg(cf.c_jf + i), jxp = __ldg(cf.c_jf + i + 1);
  const double jy = __ldg(cf.c_e1 + i), jz = __ldg(cf.c_e2 + i), ijd = __ldg(cf.c_invjdxc + i);
  for (int j = threadIdx.x + 1; j <= ny; j += blockDim.x) {
    const double div = ijd * (
        -jxm * (double)ux[sidx_f<T>(g, i, j, k)] + jxp * (double)ux[sidx_f<T>(g, i + 1, j, k)]
        - jy * (double)uy[sidx_c<T>(g, i, j, k)] + jy * (double)uy[sidx_c<T>(g, i, j + 1, k)]
        - jz * (double)uz[sidx_c<T>(g, i, j, k)] + jz * (double)uz[sidx_c<T>(g, i, j, k + 1)]);
    line[j - 1] = prefactor * div;
  }
  __syncthreads();
  Z * out = static_cast<Z *>(ps.spec) + ((size_t)(i - 1) * nz + (k - 1)) * nyh;
  for (int m = threadIdx.x; m < nyh; m += blockDim.x) {
    double re = 0., im = 0.;
    int q = 0;   // j m mod ny
    for (int j = 0; j < ny; j++) {
      const double2 w = ps.tw_y[q];
      re += line[j] * w.x;
      im += line[j] * w.y;
      q += m;
      if (q >= ny) q -= ny;
    }
    zput(out + m, make_double2(re, im));
  }
}

// complex transform along z of the columns (i, ky), in place; SIGN -1 forward
template <int SIGN, class Z>
__global__ void dftz_kernel(Geo g, Poisson ps) {
  extern __shared__ double2 col[];
  const int nz = g.nz, nyh = ps.nyh;
  const int ky = blockIdx.x, i = blockIdx.y + 1;
  Z * base = static_cast<Z *>(ps.spec) + (size_t)(i - 1) * nz * nyh + ky;
  for (int k = threadIdx.x; k < nz; k += blockDim.x) col[k] = zget(base + (size_t)k * nyh);
  __syncthreads();
  for (int m = threadIdx.x; m < nz; m += blockDim.x) {
    double re = 0., im = 0.;
    int q = 0;   // k m mod nz
    for (int k = 0; k < nz; k++) {
      const double2 w = ps.tw_z[q];
      const double wy = SIGN < 0 ? w.y : -w.y;
      re += col[k].x * w.x - col[k].y * wy;
      im += col[k].x * wy + col[k].y * w.x;
      q += m;
      if (q >= nz) q -= nz;
    }
    zput(base + (size_t)m * nyh, make_double2(re, im));
  }
}

// c2r transform along y of one (i, k) line into psi with its Neumann x ghosts
// and periodic images (as iffty_kernel)
template <class Z>
__global__ void idfty_kernel(Geo g, Poisson ps, double * __restrict__ psi) {
  extern __shared__ double2 spec_line[];
  const int ny = g.ny, nx = g.nx, nz = g.nz, nyh = ps.nyh, half = ny / 2;
  const int i = blockIdx.x + 1, k = blockIdx.y + 1;
  const Z * in = static_cast<const Z *>(ps.spec) + ((size_t)(i - 1) * nz + (k - 1)) * nyh;
  for (int m = threadIdx.x; m < nyh; m += blockDim.x) {
    double2 x = zget(in + m);
    if (m == 0 || m == half) x.y = 0.;
    spec_line[m] = x;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < ny; j += blockDim.x) {
    // X_0 + (-1)^j X_{N/2} + 2 Re sum_{0 < m < N/2} X_m exp(+2 pi i j m / N)
    double acc = 0.;
    int q = j;   // j m mod ny for m = 1
    for (int m = 1; m < half; m++) {
      const double2 w = ps.tw_y[q];     // exp(-2 pi i q / N): conjugated below
      acc += spec_line[m].x * w.x + spec_line[m].y * w.y;
      q += j;
      if (q >= ny) q -= ny;
    }
    const double val = spec_line[0].x + ((j & 1) ? -spec_line[half].x : spec_line[half].x) + 2. * acc;
    auto put = [&](int jj, int kk) {
      psi[cidx(g, i, jj, kk)] = val;
      if (i == 1) psi[cidx(g, 0, jj, kk)] = val;
      if (i == nx) psi[cidx(g, nx + 1, jj, kk)] = val;
    };
    put(j + 1, k);
    for_images(j + 1, k, ny, nz, put);
  }
}

// --------------------------------------------------------------- launchers
static bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return l;
}

// lines per CTA: ceil-free power of two, TPL threads each, at most 256 threads,
// at most `cap` lines
static int lines_per_cta(int n, int cap, int ept_max = 16, int threads = 256) {
  const int ept = n < ept_max ? n : ept_max;
  const int tpl = n / ept;
  int p = threads / tpl;
  while (p > 1 && p > cap) p >>= 1;
  return p < 1 ? 1 : p;
}

template <int EPTY, int EPTZ, class T, class Z>
static void launch_poisson_t(const Geo & g, const Coefs & cf, const Poisson & ps, const FieldsT<T> & f,
                             const double * tab_y, const double * tab_z, const double * base,
                             const double * dtp, int rkstep, cudaStream_t st, const PoissonMarks & pm) {
  auto mark = [&](int kk) { if (pm.mark) pm.mark(kk, 1); };
  const bool fy = pow2(g.ny), fz = pow2(g.nz);   // FFTs; otherwise the direct transforms
  const int lgy = ilog2(g.ny), lgz = ilog2(g.nz);
  const int Py = lines_per_cta(g.ny, (g.nx + 1) / 2, EPTY, TC_FFTY_THREADS);
  const int tply = g.ny / EPTY;
  const size_t smy = sizeof(Z) * (size_t)Py * padded_len(g.ny);
  dim3 gy((g.nx + 2 * Py - 1) / (2 * Py), g.nz);
  const dim3 gl(g.nx, g.nz);   // one CTA per (i, k) line of the direct transforms in y
  if (fy) div_ffty_kernel<EPTY, T, Z><<<gy, Py * tply, smy, st>>>(g, cf, ps, Py, lgy, f.ux, f.uy, f.uz, dtp, rkstep);
  else div_dfty_kernel<T, Z><<<gl, 128, sizeof(double) * g.ny, st>>>(g, cf, ps, f.ux, f.uy, f.uz, dtp, rkstep);
  mark(pm.k_div);
  const int Pz = lines_per_cta(g.nz, ps.nyh, EPTZ, TC_FFTZ_THREADS);
  const int tplz = g.nz / EPTZ;
  const size_t smz = sizeof(Z) * (size_t)Pz * padded_len(g.nz);
#if TC_FFTZ_MFAST
  dim3 gz((ps.nyh + Pz - 1) / Pz, g.nx);
#else
  dim3 gz(g.nx, (ps.nyh + Pz - 1) / Pz);
#endif
  const dim3 gc(ps.nyh, g.nx);   // one CTA per (ky, i) column of the direct transforms in z
  if (fz) fftz_kernel<EPTZ, -1, Z><<<gz, Pz * tplz, smz, st>>>(g, ps, Pz, lgz);
  else dftz_kernel<-1, Z><<<gc, 128, sizeof(double2) * g.nz, st>>>(g, ps);
  mark(pm.k_fwd);
  if (!launch_tdm_lines<Z>(g, ps, st)) {
    const long long nl = (long long)ps.nyh * g.nz;
    tdm_kernel<Z><<<(unsigned)((nl + 127) / 128), 128, 0, st>>>(g, ps, tab_y, tab_z, base);
  }
  mark(pm.k_tdm);
  if (fz) fftz_kernel<EPTZ, +1, Z><<<gz, Pz * tplz, smz, st>>>(g, ps, Pz, lgz);
  else dftz_kernel<+1, Z><<<gc, 128, sizeof(double2) * g.nz, st>>>(g, ps);
  mark(pm.k_inv);
  constexpr bool bulk = sizeof(Z) == 16;   // staged spectrum rows need 16-byte values
  if (fy && bulk && g.ny >= 16)   // two rows of nyh values fit a padded line buffer from ny = 16 on
    iffty_kernel<EPTY, Z, bulk><<<gy, Py * tply, smy + 16, st>>>(g, ps, Py, lgy, f.psi);
  else if (fy)
    iffty_kernel<EPTY, Z, false><<<gy, Py * tply, smy, st>>>(g, ps, Py, lgy, f.psi);
  else idfty_kernel<Z><<<gl, 128, sizeof(double2) * ps.nyh, st>>>(g, ps, f.psi);
  mark(pm.k_ify);
}

template <int EPTY, class T, class Z>
static void launch_poisson_z(const Geo & g, const Coefs & cf, const Poisson & ps, const FieldsT<T> & f,
                             const double * tab_y, const double * tab_z, const double * base,
                             const double * dtp, int rkstep, cudaStream_t st, const PoissonMarks & pm) {
  if (g.nz >= 16 && TC_FFTZ_EPT == 16)
    launch_poisson_t<EPTY, 16, T, Z>(g, cf, ps, f, tab_y, tab_z, base, dtp, rkstep, st, pm);
  else if (g.nz >= 8) launch_poisson_t<EPTY, 8, T, Z>(g, cf, ps, f, tab_y, tab_z, base, dtp, rkstep, st, pm);
  else launch_poisson_t<EPTY, 4, T, Z>(g, cf, ps, f, tab_y, tab_z, base, dtp, rkstep, st, pm);
}

template <class T, class Z>
static void launch_poisson_s(const Geo & g, const Coefs & cf, const Poisson & ps, const FieldsT<T> & f,
                             const double * tab_y, const double * tab_z, const double * base,
                             const double * dtp, int rkstep, cudaStream_t st, const PoissonMarks & pm) {
  if (g.ny >= 16 && TC_FFTY_EPT == 16)
    launch_poisson_z<16, T, Z>(g, cf, ps, f, tab_y, tab_z, base, dtp, rkstep, st, pm);
  else if (g.ny >= 8) launch_poisson_z<8, T, Z>(g, cf, ps, f, tab_y, tab_z, base, dtp, rkstep, st, pm);
  else launch_poisson_z<4, T, Z>(g, cf, ps, f, tab_y, tab_z, base, dtp, rkstep, st, pm);
}

// storage: fields and spectra both double, or both float (FP32-storage mode)
void launch_poisson(const Geo & g, const Coefs & cf, const Poisson & ps, const FieldBufs & f,
                    const double * tab_y, const double * tab_z, const double * base,
                    const double * dtp, int rkstep, cudaStream_t st, const PoissonMarks & pm) {
  if (f.bytes == 4)
    launch_poisson_s<float, float2>(g, cf, ps, f.as<float>(), tab_y, tab_z, base, dtp, rkstep, st, pm);
  else
    launch_poisson_s<double, double2>(g, cf, ps, f.as<double>(), tab_y, tab_z, base, dtp, rkstep, st, pm);
}

template <typename K>
static void allow_dyn_smem(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_FFT_SMEM_MAX);
}

template <class T, class Z>
static void poisson_smem_limits_s() {
  // up to 256 threads x 16 elements of 16 bytes, padded: < 74 KB of dynamic shared memory
  allow_dyn_smem(div_ffty_kernel<16, T, Z>);
  allow_dyn_smem(div_ffty_kernel<8, T, Z>);
  allow_dyn_smem(div_ffty_kernel<4, T, Z>);
  allow_dyn_smem(iffty_kernel<16, Z, false>);
  allow_dyn_smem(iffty_kernel<8, Z, false>);
  allow_dyn_smem(iffty_kernel<4, Z, false>);
  allow_dyn_smem(iffty_kernel<16, Z, sizeof(Z) == 16>);
  allow_dyn_smem(iffty_kernel<8, Z, sizeof(Z) == 16>);
  allow_dyn_smem(iffty_kernel<4, Z, sizeof(Z) == 16>);
  allow_dyn_smem(fftz_kernel<16, -1, Z>);
  allow_dyn_smem(fftz_kernel<16, +1, Z>);
  allow_dyn_smem(fftz_kernel<8, -1, Z>);
  allow_dyn_smem(fftz_kernel<8, +1, Z>);
  allow_dyn_smem(fftz_kernel<4, -1, Z>);
  allow_dyn_smem(fftz_kernel<4, +1, Z>);
}

void poisson_smem_limits() {
  poisson_smem_limits_s<double, double2>();
  poisson_smem_limits_s<float, float2>();
  allow_dyn_smem(tdm_lines_kernel<8, double2>);
  allow_dyn_smem(tdm_lines_kernel<8, float2>);
  allow_dyn_smem(tdm_lines_kernel<4, double2>);
  allow_dyn_smem(tdm_lines_kernel<4, float2>);
}

}  // namespace tcgpu
