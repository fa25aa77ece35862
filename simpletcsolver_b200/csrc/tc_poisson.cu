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
// right-hand side as in the reference. FFTs are radix-2 Stockham passes in shared
// memory with twiddles exp(-2 pi i m / N) tabulated on the host from libm.
//
// Spectral layout: spec[i][kz][ky] (ky fastest), so the y and z transforms read
// and write rows of contiguous wavenumbers and the radial solve, one thread per
// (kz, ky) line, walks i with fully coalesced steps.
#include "tc_common.cuh"
#include "tc_kernels.h"

namespace tcgpu {

__device__ inline double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// radix-2 Stockham autosort over P lines of length N held in a; b is scratch.
// Returns the buffer that holds the result (natural order).
template <int SIGN>
__device__ double2 * fft_lines(double2 * a, double2 * b, int N, int P, const double2 * __restrict__ tw) {
  const int half = N >> 1;
  for (int Ns = 1; Ns < N; Ns <<= 1) {
    const int tws = N / (2 * Ns);
    for (int idx = threadIdx.x; idx < P * half; idx += blockDim.x) {
      const int p = idx / half;
      const int jj = idx - p * half;
      const double2 * x = a + (size_t)p * N;
      double2 * y = b + (size_t)p * N;
      const int kk = jj & (Ns - 1);
      double2 w = __ldg(tw + kk * tws);
      if (SIGN > 0) w.y = -w.y;
      const double2 u0 = x[jj];
      const double2 t = cmul(x[jj + half], w);
      const int o = ((jj - kk) << 1) + kk;
      y[o] = make_double2(u0.x + t.x, u0.y + t.y);
      y[o + Ns] = make_double2(u0.x - t.x, u0.y - t.y);
    }
    __syncthreads();
    double2 * s = a;
    a = b;
    b = s;
  }
  return a;
}

// --------------------------------------------------------------- forward y
__global__ void __launch_bounds__(256)
div_ffty_kernel(Geo g, Coefs cf, Poisson ps, int P,
                const double * __restrict__ ux, const double * __restrict__ uy,
                const double * __restrict__ uz, const double * __restrict__ dtp, int rkstep) {
  extern __shared__ double2 smem[];
  const int ny = g.ny, nx = g.nx, nz = g.nz;
  const int TI = 2 * P;
  const int i0 = blockIdx.x * TI + 1;
  const int k = blockIdx.y + 1;
  double2 * a = smem;
  double2 * b = smem + (size_t)P * ny;
  const double norm = 1. * ny * nz;
  const double prefactor = 1. / (rk_gamma(rkstep) * (*dtp)) / norm;
  for (int idx = threadIdx.x; idx < TI * ny; idx += blockDim.x) {
    const int ii = idx % TI;
    const int j = idx / TI + 1;
    const int i = i0 + ii;
    double val = 0.;
    if (i <= nx) {
      const double ux_xm = __ldg(ux + fidx(g, i, j, k));
      const double ux_xp = __ldg(ux + fidx(g, i + 1, j, k));
      const double uy_ym = __ldg(uy + cidx(g, i, j, k));
      const double uy_yp = __ldg(uy + cidx(g, i, j + 1, k));
      const double uz_zm = __ldg(uz + cidx(g, i, j, k));
      const double uz_zp = __ldg(uz + cidx(g, i, j, k + 1));
      const double jxm = __ldg(cf.c_jf + i), jxp = __ldg(cf.c_jf + i + 1);
      const double jy = __ldg(cf.c_e1 + i), jz = __ldg(cf.c_e2 + i);
      const double div = __ldg(cf.c_invjdxc + i) * (
          -jxm * ux_xm + jxp * ux_xp
          - jy * uy_ym + jy * uy_yp
          - jz * uz_zm + jz * uz_zp);
      val = prefactor * div;
    }
    double * line = reinterpret_cast<double *>(a + (size_t)(ii >> 1) * ny);
    line[2 * (j - 1) + (ii & 1)] = val;
  }
  __syncthreads();
  double2 * r = fft_lines<-1>(a, b, ny, P, ps.tw_y);
  // separate the two real transforms and store the ny/2+1 non-negative wavenumbers
  const int nyh = ps.nyh;
  for (int idx = threadIdx.x; idx < TI * nyh; idx += blockDim.x) {
    const int m = idx % nyh;
    const int ii = idx / nyh;
    const int i = i0 + ii;
    if (i > nx) continue;
    const double2 * z = r + (size_t)(ii >> 1) * ny;
    const double2 zm = z[m];
    const double2 zn = z[(ny - m) & (ny - 1)];
    double2 out;
    if ((ii & 1) == 0) out = make_double2(0.5 * (zm.x + zn.x), 0.5 * (zm.y - zn.y));
    else out = make_double2(0.5 * (zm.y + zn.y), -0.5 * (zm.x - zn.x));
    ps.spec[((size_t)(i - 1) * nz + (k - 1)) * nyh + m] = out;
  }
}

// --------------------------------------------------------------- z transforms
template <int SIGN>
__global__ void __launch_bounds__(256)
fftz_kernel(Geo g, Poisson ps, int TM) {
  extern __shared__ double2 smem[];
  const int nz = g.nz, nyh = ps.nyh;
  const int i = blockIdx.x;          // 0..nx-1
  const int m0 = blockIdx.y * TM;
  double2 * a = smem;
  double2 * b = smem + (size_t)TM * nz;
  double2 * base = ps.spec + (size_t)i * nz * nyh;
  for (int idx = threadIdx.x; idx < TM * nz; idx += blockDim.x) {
    const int mm = idx % TM;
    const int kz = idx / TM;
    const int m = m0 + mm;
    a[(size_t)mm * nz + kz] = (m < nyh) ? base[(size_t)kz * nyh + m] : make_double2(0., 0.);
  }
  __syncthreads();
  double2 * r = fft_lines<SIGN>(a, b, nz, TM, ps.tw_z);
  for (int idx = threadIdx.x; idx < TM * nz; idx += blockDim.x) {
    const int mm = idx % TM;
    const int kz = idx / TM;
    const int m = m0 + mm;
    if (m < nyh) base[(size_t)kz * nyh + m] = r[(size_t)mm * nz + kz];
  }
}

// --------------------------------------------------------------- radial solve
__global__ void __launch_bounds__(128)
tdm_kernel(Geo g, Poisson ps, const double * __restrict__ tab_y, const double * __restrict__ tab_z,
           const double * __restrict__ base) {
  const int nyh = ps.nyh, nz = g.nz, n = g.nx;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)nyh * nz) return;
  const int m = (int)(tid % nyh);
  const int kz = (int)(tid / nyh);
  const size_t st = (size_t)nz * nyh;
  double2 * q = ps.spec + (size_t)kz * nyh + m;
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
    double2 x = q[0];
    q[0] = pin ? make_double2(0., 0.) : make_double2(x.x / c, x.y / c);
    return;
  }
  // forward elimination (src/tdm.c:24-44)
  double c0 = cdiag(0);
  double vprev = __ldg(ps.tu) / c0;
  v[0] = vprev;
  double2 qprev = q[0];
  qprev = make_double2(qprev.x / c0, qprev.y / c0);
  q[0] = qprev;
  for (int i = 1; i < n - 1; i++) {
    const double l = __ldg(ps.tl + i);
    const double val = 1. / (cdiag(i) - l * vprev);
    vprev = val * __ldg(ps.tu + i);
    v[(size_t)i * st] = vprev;
    const double2 r = q[(size_t)i * st];
    qprev = make_double2(val * (r.x - l * qprev.x), val * (r.y - l * qprev.y));
    q[(size_t)i * st] = qprev;
  }
  {
    const int i = n - 1;
    const double l = __ldg(ps.tl + i);
    const double val = cdiag(i) - l * vprev;
    const double2 r = q[(size_t)i * st];
    double2 x;
    if (pin) x = make_double2(0., 0.);
    else {
      const double iv = 1. / val;
      x = make_double2(iv * (r.x - l * qprev.x), iv * (r.y - l * qprev.y));
    }
    q[(size_t)i * st] = x;
    qprev = x;
  }
  // back substitution
  for (int i = n - 2; i >= 0; i--) {
    const double vi = v[(size_t)i * st];
    const double2 r = q[(size_t)i * st];
    qprev = make_double2(r.x - vi * qprev.x, r.y - vi * qprev.y);
    q[(size_t)i * st] = qprev;
  }
}

// --------------------------------------------------------------- inverse y
__global__ void __launch_bounds__(256)
iffty_kernel(Geo g, Poisson ps, int P, double * __restrict__ psi) {
  extern __shared__ double2 smem[];
  const int ny = g.ny, nx = g.nx, nz = g.nz, nyh = ps.nyh;
  const int TI = 2 * P;
  const int i0 = blockIdx.x * TI + 1;
  const int k = blockIdx.y + 1;
  double2 * a = smem;
  double2 * b = smem + (size_t)P * ny;
  // Hermitian extension of the two packed real lines
  for (int idx = threadIdx.x; idx < P * ny; idx += blockDim.x) {
    const int m = idx % ny;
    const int pp = idx / ny;
    const int ia = i0 + 2 * pp, ib = ia + 1;
    const int mr = (m <= ny / 2) ? m : ny - m;
    double2 xa = make_double2(0., 0.), xb = make_double2(0., 0.);
    if (ia <= nx) xa = ps.spec[((size_t)(ia - 1) * nz + (k - 1)) * nyh + mr];
    if (ib <= nx) xb = ps.spec[((size_t)(ib - 1) * nz + (k - 1)) * nyh + mr];
    if (mr == 0 || 2 * mr == ny) { xa.y = 0.; xb.y = 0.; }
    double2 z;
    if (m <= ny / 2) z = make_double2(xa.x - xb.y, xa.y + xb.x);
    else z = make_double2(xa.x + xb.y, -xa.y + xb.x);
    a[(size_t)pp * ny + m] = z;
  }
  __syncthreads();
  double2 * r = fft_lines<+1>(a, b, ny, P, ps.tw_y);
  for (int idx = threadIdx.x; idx < TI * ny; idx += blockDim.x) {
    const int ii = idx % TI;
    const int j = idx / TI + 1;
    const int i = i0 + ii;
    if (i > nx) continue;
    const double2 z = r[(size_t)(ii >> 1) * ny + (j - 1)];
    const double val = (ii & 1) ? z.y : z.x;
    auto put = [&](int jj, int kk) {
      psi[cidx(g, i, jj, kk)] = val;
      if (i == 1) psi[cidx(g, 0, jj, kk)] = val;
      if (i == nx) psi[cidx(g, nx + 1, jj, kk)] = val;
    };
    put(j, k);
    for_images(j, k, ny, nz, put);
  }
}

static int pick_lines(int n, int maxlines) {
  int p = 1;
  while (p * 2 * n <= 2048 && p * 2 <= maxlines) p *= 2;
  return p;
}

void launch_poisson(const Geo & g, const Coefs & cf, const Poisson & ps, const Fields & f,
                    const double * tab_y, const double * tab_z, const double * base,
                    const double * dtp, int rkstep, cudaStream_t st, const PoissonMarks & pm) {
  auto mark = [&](int k) { if (pm.mark) pm.mark(k, 1); };
  const int P = pick_lines(g.ny, 8);
  const size_t smy = sizeof(double2) * 2 * (size_t)P * g.ny;
  dim3 gy((g.nx + 2 * P - 1) / (2 * P), g.nz);
  div_ffty_kernel<<<gy, 256, smy, st>>>(g, cf, ps, P, f.ux, f.uy, f.uz, dtp, rkstep);
  mark(pm.k_div);
  const int TM = pick_lines(g.nz, 16);
  const size_t smz = sizeof(double2) * 2 * (size_t)TM * g.nz;
  dim3 gz(g.nx, (ps.nyh + TM - 1) / TM);
  fftz_kernel<-1><<<gz, 256, smz, st>>>(g, ps, TM);
  mark(pm.k_fwd);
  const long long nl = (long long)ps.nyh * g.nz;
  tdm_kernel<<<(unsigned)((nl + 127) / 128), 128, 0, st>>>(g, ps, tab_y, tab_z, base);
  mark(pm.k_tdm);
  fftz_kernel<+1><<<gz, 256, smz, st>>>(g, ps, TM);
  mark(pm.k_inv);
  iffty_kernel<<<gy, 256, smy, st>>>(g, ps, P, f.psi);
  mark(pm.k_ify);
}

void poisson_smem_limits() {
  // 2 buffers x 2048 complex doubles = 64 KB of dynamic shared memory
  cudaFuncSetAttribute(div_ffty_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536);
  cudaFuncSetAttribute(iffty_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536);
  cudaFuncSetAttribute(fftz_kernel<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536);
  cudaFuncSetAttribute(fftz_kernel<+1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 65536);
}

}  // namespace tcgpu
