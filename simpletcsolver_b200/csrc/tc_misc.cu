// Correction, pressure update, time-step size, boundary conditions, tensors and
// logging reductions.
//
//   correct_kernel   fluid_correct_velocity (src/fluid/correct/*.c) and
//                    fluid_update_pressure (src/fluid/update_pressure.c:23-173)
//                    fused: one pass reads psi once and updates ux, uy, uz and p,
//                    writing walls, Neumann ghosts and periodic images.
//   dtmin_kernel     decide_dt_adv (src/decide_dt.c:32-80): min of h/(|u|+1e-8)
//                    over the interior, warp-shuffle + block reduction, then an
//                    order-independent atomicMin on the bit pattern of the
//                    (positive) double; non-finite velocities raise a status bit.
//   dtfinal_kernel   dt = coef_adv * min(1, that) then the diffusive limits of the
//                    explicit directions (src/decide_dt.c:89-160).
//   bc_kernel        fluid_update_boundaries_* on one field.
//   tensor_kernel    l_ij arrays with halos (src/fluid/predict/l*.c).
//   diag_kernel      src/logging/{divergence,injection,dissipation,total_energy}.c
//                    as a deterministic two-stage reduction.
#include "tc_common.cuh"
#include "tc_kernels.h"

namespace tcgpu {

// --------------------------------------------------------------- correction
__global__ void __launch_bounds__(256)
correct_kernel(Geo g, Bc bc, Coefs cf, Fields f, const double * __restrict__ dtp, int rkstep, double nu, int what) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double dt = *dtp;
  const double pf = rk_gamma(rkstep) * dt;          // correct/main.c:21-22
  const double pp = 0.5 * rk_gamma(rkstep) * dt * nu; // update_pressure.c:161-162
  const double * psi = f.psi;
  const double psi0 = __ldg(psi + cidx(g, i, j, k));
  const double psi_im = __ldg(psi + cidx(g, i - 1, j, k));
  const double psi_jm = __ldg(psi + cidx(g, i, j - 1, k));
  const double psi_km = __ldg(psi + cidx(g, i, j, k - 1));
  // ux, i = 2..nx (correct/ux.c:25-52); walls stay zero
  if (what & CORRECT_VELOCITY) {
    double val = 0.;
    if (i >= 2) {
      const size_t q = fidx(g, i, j, k);
      val = f.ux[q] - pf * __ldg(cf.c_invhxxf + i) * (-psi_im + psi0);
      f.ux[q] = val;
      for_images(j, k, ny, nz, [&](int jj, int kk) { f.ux[fidx(g, i, jj, kk)] = val; });
    } else {
      f.ux[fidx(g, 1, j, k)] = 0.;
      for_images(j, k, ny, nz, [&](int jj, int kk) { f.ux[fidx(g, 1, jj, kk)] = 0.; });
    }
    if (i == nx) {
      f.ux[fidx(g, nx + 1, j, k)] = 0.;
      for_images(j, k, ny, nz, [&](int jj, int kk) { f.ux[fidx(g, nx + 1, jj, kk)] = 0.; });
    }
  }
  // uy (correct/uy.c:25-52) with its walls (boundary/uy.c)
  if (what & CORRECT_VELOCITY) {
    const size_t q = cidx(g, i, j, k);
    const double val = f.uy[q] - pf * __ldg(cf.c_invhyxc + i) * (-psi_jm + psi0);
    auto put = [&](int jj, int kk) {
      f.uy[cidx(g, i, jj, kk)] = val;
      if (i == 1) f.uy[cidx(g, 0, jj, kk)] = bc.uy_xm;
      if (i == nx) f.uy[cidx(g, nx + 1, jj, kk)] = bc.uy_xp;
    };
    put(j, k);
    for_images(j, k, ny, nz, put);
  }
  // uz (correct/uz.c:15-44)
  if (what & CORRECT_VELOCITY) {
    const size_t q = cidx(g, i, j, k);
    const double val = f.uz[q] - pf * cf.inv_hz * (-psi_km + psi0);
    auto put = [&](int jj, int kk) {
      f.uz[cidx(g, i, jj, kk)] = val;
      if (i == 1) f.uz[cidx(g, 0, jj, kk)] = 0.;
      if (i == nx) f.uz[cidx(g, nx + 1, jj, kk)] = 0.;
    };
    put(j, k);
    for_images(j, k, ny, nz, put);
  }
  // p += psi, then the implicit-direction corrections (update_pressure.c:23-136)
  if (what & CORRECT_PRESSURE) {
    const size_t q = cidx(g, i, j, k);
    double val = f.p[q] + psi0;
    const double ijd = __ldg(cf.c_invjdxc + i);
    if (bc.implicit[0]) {
      const double l = __ldg(cf.c_pxl + i), u = __ldg(cf.c_pxu + i), c = -l - u;
      const double psi_ip = __ldg(psi + cidx(g, i + 1, j, k));
      val -= 2. * pp * ijd * (l * psi_im + c * psi0 + u * psi_ip);
    }
    if (bc.implicit[1]) {
      const double l = __ldg(cf.c_pyl + i), c = -l - l;
      const double psi_jp = __ldg(psi + cidx(g, i, j + 1, k));
      val -= 2. * pp * ijd * (l * psi_jm + c * psi0 + l * psi_jp);
    }
    if (bc.implicit[2]) {
      const double l = __ldg(cf.c_pzl + i), c = -l - l;
      const double psi_kp = __ldg(psi + cidx(g, i, j, k + 1));
      val -= 2. * pp * ijd * (l * psi_km + c * psi0 + l * psi_kp);
    }
    auto put = [&](int jj, int kk) {
      f.p[cidx(g, i, jj, kk)] = val;
      if (i == 1) f.p[cidx(g, 0, jj, kk)] = val;
      if (i == nx) f.p[cidx(g, nx + 1, jj, kk)] = val;
    };
    put(j, k);
    for_images(j, k, ny, nz, put);
  }
}

void launch_correct(const Geo & g, const Bc & bc, const Coefs & cf, const Fields & f, const double * dtp,
                    int rkstep, double nu, int what, cudaStream_t st) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
  correct_kernel<<<grid, block, 0, st>>>(g, bc, cf, f, dtp, rkstep, nu, what);
}

// --------------------------------------------------------------- decide_dt
__device__ inline double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void __launch_bounds__(256)
dtmin_kernel(Geo g, const double * __restrict__ ux, const double * __restrict__ uy,
             const double * __restrict__ uz, unsigned long long * dtmin, unsigned * status) {
  const double small = 1.e-8;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  double m = 1.;
  bool bad = false;
  if (i <= g.nx && j <= g.ny) {
    const double hx = __ldg(g.hxxf + i), hy = __ldg(g.hyxc + i), hz = g.hz;
    for (int k = blockIdx.z + 1; k <= g.nz; k += gridDim.z) {
      if (i >= 2) {
        const double v = __ldg(ux + fidx(g, i, j, k));
        bad |= !isfinite(v);
        m = fmin(m, hx / (fabs(v) + small));
      }
      const double vy = __ldg(uy + cidx(g, i, j, k));
      const double vz = __ldg(uz + cidx(g, i, j, k));
      bad |= !isfinite(vy) || !isfinite(vz);
      m = fmin(m, hy / (fabs(vy) + small));
      m = fmin(m, hz / (fabs(vz) + small));
    }
  }
  __shared__ double red[8];
  m = warp_min(m);
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  const int lane = t & 31, wid = t >> 5;
  if (lane == 0) red[wid] = m;
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(status, (unsigned)ST_NONFINITE);
  __syncthreads();
  if (wid == 0) {
    double v = (lane < 8) ? red[lane] : 1.;
    v = warp_min(v);
    if (lane == 0) atomicMin(dtmin, (unsigned long long)__double_as_longlong(v));
  }
}

__global__ void dtfinal_kernel(double coef_adv, const double * caps, unsigned long long * dtmin,
                               double * dtp, unsigned * status) {
  double dt = __longlong_as_double((long long)*dtmin);
  dt = fmin(1., dt);
  dt *= coef_adv;
  for (int d = 0; d < 3; d++) {
    if (caps[d] > 0.) dt = fmin(dt, caps[d]);
  }
  if (!(dt > 0.) || !isfinite(dt)) atomicOr(status, (unsigned)ST_BADDT);
  *dtp = dt;
  *dtmin = 0x3ff0000000000000ull;  // 1.0, the reference's starting value
}

void launch_dtmin(const Geo & g, const Fields & f, unsigned long long * dtmin, unsigned * status, cudaStream_t st) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz < 16 ? g.nz : 16);
  dtmin_kernel<<<grid, block, 0, st>>>(g, f.ux, f.uy, f.uz, dtmin, status);
}

void launch_dtfinal(double coef_adv, const double * dt_caps, unsigned long long * dtmin, double * dtp,
                    unsigned * status, cudaStream_t st) {
  dtfinal_kernel<<<1, 1, 0, st>>>(coef_adv, dt_caps, dtmin, dtp, status);
}

void launch_decide_dt(const Geo & g, const Fields & f, double coef_adv, const double * dt_caps,
                      unsigned long long * dtmin, double * dtp, unsigned * status, cudaStream_t st) {
  launch_dtmin(g, f, dtmin, status, st);
  launch_dtfinal(coef_adv, dt_caps, dtmin, dtp, status, st);
}

// --------------------------------------------------------------- boundary conditions
__global__ void bc_kernel(Geo g, Bc bc, int kind, double * __restrict__ a) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;   // position in the row
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (j > ny) return;
  if (kind == BC_UX) {
    if (e > nx) return;                                  // i = e + 1
    double * row = a + fidx(g, 1, j, k);
    double val = (e == 0 || e == nx) ? 0. : row[e];
    row[e] = val;
    for_images(j, k, ny, nz, [&](int jj, int kk) { a[fidx(g, 1, jj, kk) + e] = val; });
    return;
  }
  if (e > nx + 1) return;                                // i = e
  double * row = a + cidx(g, 0, j, k);
  double val;
  if (e == 0 || e == nx + 1) {
    const bool lo = (e == 0);
    switch (kind) {
      case BC_UY: val = lo ? bc.uy_xm : bc.uy_xp; break;
      case BC_UZ: val = 0.; break;
      case BC_T: val = lo ? bc.t_xm : bc.t_xp; break;
      default: val = lo ? row[1] : row[nx]; break;       // p, psi: Neumann copy
    }
  } else {
    val = row[e];
  }
  row[e] = val;
  for_images(j, k, ny, nz, [&](int jj, int kk) { a[cidx(g, 0, jj, kk) + e] = val; });
}

void launch_bc(const Geo & g, const Bc & bc, BcKind kind, double * a, cudaStream_t st) {
  dim3 block(64, 4, 1);
  dim3 grid((g.nx + 2 + 63) / 64, (g.ny + 3) / 4, g.nz);
  bc_kernel<<<grid, block, 0, st>>>(g, bc, (int)kind, a);
}

// --------------------------------------------------------------- tensors
// Row lengths: face tensors (lxy lxz lyx0 lyx1 lzx) nx+1, centre tensors nx.
__global__ void tensor_kernel(Geo g, Coefs cf, Fields f, Tensors tn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;   // 1..nx+1
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i > nx + 1 || j > ny) return;
  auto fi = [&](int ii, int jj, int kk) { return (size_t)(ii - 1) + (size_t)(nx + 1) * ((size_t)jj + (size_t)(ny + 2) * kk); };
  auto ci = [&](int ii, int jj, int kk) { return (size_t)(ii - 1) + (size_t)nx * ((size_t)jj + (size_t)(ny + 2) * kk); };
  const double * ux = f.ux;
  const double * uy = f.uy;
  const double * uz = f.uz;
  {  // face tensors
    const double ih = __ldg(cf.c_invhxxf + i);
    const double lxy = ih * (-uy[cidx(g, i - 1, j, k)] + uy[cidx(g, i, j, k)]);
    const double lxz = ih * (-uz[cidx(g, i - 1, j, k)] + uz[cidx(g, i, j, k)]);
    const double lyx0 = __ldg(cf.c_invhyxf + i) * (-ux[fidx(g, i, j - 1, k)] + ux[fidx(g, i, j, k)]);
    const double lyx1 = __ldg(cf.c_lyx1f + i) * (__ldg(cf.c_wm + i) * uy[cidx(g, i - 1, j, k)] + __ldg(cf.c_wp + i) * uy[cidx(g, i, j, k)]);
    const double lzx = cf.inv_hz * (-ux[fidx(g, i, j, k - 1)] + ux[fidx(g, i, j, k)]);
    const double vals[5] = {lxy, lxz, lyx0, lyx1, lzx};
    const int slot[5] = {1, 2, 3, 4, 8};
    for (int s = 0; s < 5; s++) {
      double * a = tn.a[slot[s]];
      a[fi(i, j, k)] = vals[s];
      for_images(j, k, ny, nz, [&](int jj, int kk) { a[fi(i, jj, kk)] = vals[s]; });
    }
  }
  if (i <= nx) {  // centre tensors
    const double lxx = (1. / __ldg(g.hxxc + i)) * (-ux[fidx(g, i, j, k)] + ux[fidx(g, i + 1, j, k)]);
    const double ihy = __ldg(cf.c_invhyxc + i);
    const double lyy0 = ihy * (-uy[cidx(g, i, j, k)] + uy[cidx(g, i, j + 1, k)]);
    const double lyy1 = __ldg(cf.c_lyy1 + i) * (0.5 * ux[fidx(g, i, j, k)] + 0.5 * ux[fidx(g, i + 1, j, k)]);
    const double lyz = ihy * (-uz[cidx(g, i, j - 1, k)] + uz[cidx(g, i, j, k)]);
    const double lzy = cf.inv_hz * (-uy[cidx(g, i, j, k - 1)] + uy[cidx(g, i, j, k)]);
    const double lzz = cf.inv_hz * (-uz[cidx(g, i, j, k)] + uz[cidx(g, i, j, k + 1)]);
    const double vals[6] = {lxx, lyy0, lyy1, lyz, lzy, lzz};
    const int slot[6] = {0, 5, 6, 7, 9, 10};
    for (int s = 0; s < 6; s++) {
      double * a = tn.a[slot[s]];
      a[ci(i, j, k)] = vals[s];
      for_images(j, k, ny, nz, [&](int jj, int kk) { a[ci(i, jj, kk)] = vals[s]; });
    }
  }
}

void launch_tensors(const Geo & g, const Coefs & cf, const Fields & f, const Tensors & tn, cudaStream_t st) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 1 + 31) / 32, (g.ny + 7) / 8, g.nz);
  tensor_kernel<<<grid, block, 0, st>>>(g, cf, f, tn);
}

// --------------------------------------------------------------- diagnostics
// partial[b][0..8]: max|div|, inj_m, inj_s, dis_m, dis_s, e_ux, e_uy, e_uz, e_t
constexpr int DIAG_BLOCKS = 296;

__global__ void __launch_bounds__(256)
diag_kernel(Geo g, Coefs cf, Bc bc, Fields f, double * partial) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long total = (long long)(nx + 1) * ny * nz;
  double acc[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
  const double * ux = f.ux;
  const double * uy = f.uy;
  const double * uz = f.uz;
  const double * t = f.t;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
       c += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(c % (nx + 1)) + 1;     // 1..nx+1
    const long long r = c / (nx + 1);
    const int j = (int)(r % ny) + 1;
    const int k = (int)(r / ny) + 1;
    const double jdf = __ldg(g.jdxf + i);
    const double hxf = __ldg(g.hxxf + i);
    // face quantities at i
    const double ih = __ldg(cf.c_invhxxf + i);
    const double uyim = uy[cidx(g, i - 1, j, k)], uyi = uy[cidx(g, i, j, k)];
    const double lxy = ih * (-uyim + uyi);
    const double lxz = ih * (-uz[cidx(g, i - 1, j, k)] + uz[cidx(g, i, j, k)]);
    const double lyx = __ldg(cf.c_invhyxf + i) * (-ux[fidx(g, i, j - 1, k)] + ux[fidx(g, i, j, k)])
                     + __ldg(cf.c_lyx1f + i) * (__ldg(cf.c_wm + i) * uyim + __ldg(cf.c_wp + i) * uyi);
    const double lzx = cf.inv_hz * (-ux[fidx(g, i, j, k - 1)] + ux[fidx(g, i, j, k)]);
    // dissipation.c:40-151 (face contributions)
    acc[3] += jdf * lyx * (lyx + lxy);
    acc[3] += jdf * lzx * (lzx + lxz);
    acc[3] += jdf * lxy * (lxy + lyx);
    acc[3] += jdf * lxz * (lxz + lzx);
    {  // dissipation.c:240-265 (scalar, x)
      const double d = -t[cidx(g, i - 1, j, k)] + t[cidx(g, i, j, k)];
      const double q = d / hxf;
      acc[4] += jdf * (q * q);
    }
    // injection.c:55-98 at the two walls
    if (i == 1 || i == nx + 1) {
      const double sgn = (i == 1) ? -1. : 1.;
      const double uyw = (i == 1) ? uyim : uyi;
      acc[1] += sgn * jdf / hxf * uyw * (lyx + lxy);
      const double tw = (i == 1) ? t[cidx(g, 0, j, k)] : t[cidx(g, nx + 1, j, k)];
      const double dtw = (i == 1) ? (-t[cidx(g, 0, j, k)] + t[cidx(g, 1, j, k)])
                                  : (-t[cidx(g, nx, j, k)] + t[cidx(g, nx + 1, j, k)]);
      acc[2] += sgn * jdf / hxf * tw / hxf * dtw;
    }
    if (i >= 2 && i <= nx) {  // total_energy.c:45-51
      const double v = ux[fidx(g, i, j, k)];
      acc[5] += jdf * 0.5 * (v * v);
    }
    if (i <= nx) {
      const double jdc = __ldg(g.jdxc + i);
      const double ux0 = ux[fidx(g, i, j, k)], ux1 = ux[fidx(g, i + 1, j, k)];
      const double uy0 = uyi, uy1 = uy[cidx(g, i, j + 1, k)];
      const double uz0 = uz[cidx(g, i, j, k)], uz1 = uz[cidx(g, i, j, k + 1)];
      // divergence.c:56-78
      const double div = __ldg(cf.c_invjdxc + i) * (
          -__ldg(cf.c_jf + i) * ux0 + __ldg(cf.c_jf + i + 1) * ux1
          - __ldg(cf.c_e1 + i) * uy0 + __ldg(cf.c_e1 + i) * uy1
          - __ldg(cf.c_e2 + i) * uz0 + __ldg(cf.c_e2 + i) * uz1);
      acc[0] = fmax(acc[0], fabs(div));
      // centre tensors and dissipation contributions
      const double lxx = (1. / __ldg(g.hxxc + i)) * (-ux0 + ux1);
      const double ihy = __ldg(cf.c_invhyxc + i);
      const double lyy = ihy * (-uy0 + uy1) + __ldg(cf.c_lyy1 + i) * (0.5 * ux0 + 0.5 * ux1);
      const double lyz = ihy * (-uz[cidx(g, i, j - 1, k)] + uz0);
      const double lzy = cf.inv_hz * (-uy[cidx(g, i, j, k - 1)] + uy0);
      const double lzz = cf.inv_hz * (-uz0 + uz1);
      acc[3] += jdc * lxx * (lxx + lxx);
      acc[3] += jdc * lyy * (lyy + lyy);
      acc[3] += jdc * lzy * (lzy + lyz);
      acc[3] += jdc * lyz * (lyz + lzy);
      acc[3] += jdc * lzz * (lzz + lzz);
      const double t0 = t[cidx(g, i, j, k)];
      {
        const double q = (-t[cidx(g, i, j - 1, k)] + t0) / __ldg(g.hyxc + i);
        acc[4] += jdc * (q * q);
      }
      {
        const double q = (-t[cidx(g, i, j, k - 1)] + t0) / g.hz;
        acc[4] += jdc * (q * q);
      }
      acc[6] += jdc * 0.5 * (uy0 * uy0);
      acc[7] += jdc * 0.5 * (uz0 * uz0);
      acc[8] += jdc * 0.5 * (t0 * t0);
    }
  }
  __shared__ double red[8][9];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int q = 0; q < 9; q++) {
    double v = acc[q];
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v, o);
      v = (q == 0) ? fmax(v, w) : v + w;
    }
    if (lane == 0) red[wid][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    const int q = threadIdx.x;
    double v = red[0][q];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = (q == 0) ? fmax(v, red[w][q]) : v + red[w][q];
    partial[(size_t)blockIdx.x * 9 + q] = v;
  }
}

__global__ void diag_final_kernel(const double * partial, int nblocks, double nu, double kappa, double * out) {
  const int q = threadIdx.x;
  if (q >= 9) return;
  double v = partial[q];
  for (int b = 1; b < nblocks; b++) v = (q == 0) ? fmax(v, partial[(size_t)b * 9 + q]) : v + partial[(size_t)b * 9 + q];
  if (q == 1 || q == 3) v *= nu;
  if (q == 2 || q == 4) v *= kappa;
  out[q] = v;
}

void launch_diagnostics(const Geo & g, const Coefs & cf, const Bc & bc, const Fields & f, double nu, double kappa,
                        double * out, double * partial, cudaStream_t st) {
  diag_kernel<<<DIAG_BLOCKS, 256, 0, st>>>(g, cf, bc, f, partial);
  diag_final_kernel<<<1, 32, 0, st>>>(partial, DIAG_BLOCKS, nu, kappa, out);
}

}  // namespace tcgpu
