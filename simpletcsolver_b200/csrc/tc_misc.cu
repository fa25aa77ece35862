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
__device__ inline double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Advective limit of a (32, 8) block: the largest |v| + 1e-8 per direction
// over the block's eight rows j of each radial index, one division per index
// and direction (h depends on i only, and correctly rounded division is
// monotonic, so h / max(|v| + 1e-8) is the minimum of the per-cell quotients),
// the minimum over the 32 indices, then an order-independent atomicMin on the
// bit pattern of the positive double into one of DT_SLOTS accumulators (blocks
// spread over them). Non-finite velocities raise ST_NONFINITE. Threads without
// a cell pass a = 0.
__device__ inline void block_cfl(double ax, double ay, double az, double hx, double hy, double hz, bool bad,
                                 unsigned long long * dtmin, unsigned * status) {
  __shared__ double sa[3][8][32];
  const int tx = threadIdx.x, ty = threadIdx.y;
  sa[0][ty][tx] = ax;
  sa[1][ty][tx] = ay;
  sa[2][ty][tx] = az;
  if (__syncthreads_or(bad) && tx == 0 && ty == 0) atomicOr(status, (unsigned)ST_NONFINITE);
  if (ty == 0) {
    double mx = 0., my = 0., mz = 0.;
#pragma unroll
    for (int r = 0; r < 8; r++) {
      mx = fmax(mx, sa[0][r][tx]);
      my = fmax(my, sa[1][r][tx]);
      mz = fmax(mz, sa[2][r][tx]);
    }
    double m = 1.;
    if (mx > 0.) m = fmin(m, hx / mx);
    if (my > 0.) m = fmin(m, hy / my);
    if (mz > 0.) m = fmin(m, hz / mz);
    m = warp_min(m);
    if (tx == 0) {
      const unsigned b = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
      atomicMin(dtmin + (b & (DT_SLOTS - 1)), (unsigned long long)__double_as_longlong(m));
    }
  }
}

// Advective limit of one warp of a (32, 8) block (lanes along i, each lane's
// largest |v| + 1e-8 over its cells): one division per lane and direction, the
// minimum over the warp, atomicMin into one of the DT_SLOTS accumulators. No
// block-wide synchronisation, so the block's other warps are not held up.
__device__ inline void warp_cfl(double ax, double ay, double az, double hx, double hy, double hz, bool bad,
                                unsigned long long * dtmin, unsigned * status) {
  double m = 1.;
  if (ax > 0.) m = fmin(m, hx / ax);
  if (ay > 0.) m = fmin(m, hy / ay);
  if (az > 0.) m = fmin(m, hz / az);
  m = warp_min(m);
  const bool anybad = __any_sync(0xffffffffu, bad);
  if (threadIdx.x == 0) {
    if (anybad) atomicOr(status, (unsigned)ST_NONFINITE);
    const unsigned b = threadIdx.y + 8 * (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z));
    atomicMin(dtmin + (b & (DT_SLOTS - 1)), (unsigned long long)__double_as_longlong(m));
  }
}

// Cells per thread along z in the correction that also takes the advective
// limit (each lane's divisions are shared by its cells; measured at
// 256 x 1024 x 512: 1 cell 2.5 ms, 2-8 cells 2.2 ms per launch).
#ifndef TC_CFL_KZ
#define TC_CFL_KZ 4
#endif

// WHAT: CORRECT_VELOCITY and/or CORRECT_PRESSURE; IMPL: implicit directions
// as a compile-time mask (bit 0 x, 1 y, 2 z) or -1 to read them from bc. A
// thread takes TC_CORRECT_KZ cells along z, TC_CFL_KZ with CFL. With CFL the advective
// limit of decide_dt_adv
// (src/decide_dt.c:32-80) is taken on the corrected velocities as they are
// written, for the next step's dt (the reference computes it at the start of
// that step from the same values).
// Resident blocks requested from the register allocator (plain / with CFL),
// cells per thread along z without CFL (TC_CORRECT_KZ), and the cells whose
// inputs are loaded together before any of them is stored (TC_CORRECT_G with
// CFL, all KZ cells without). Within a group psi at k-1 and k+1 of an inner
// cell is its neighbour's psi at k, loaded once. Measured at 256 x 1024 x 512
// (ms per launch, averaged over a step's three): blocks 6/5, 1 cell 2.23; 5/4
// 2.15; 4/4 2.04 (the CFL kernel spills at 64 registers); 4/3 1.95 (no
// spills); 3/3 with 2 cells 1.88; 4/4 with 2 cells 2.03; 4/2 with CFL groups
// of 2 1.94; 2/3 with 4 cells 1.96. With all loads issued up front the registers holding them buy
// more than the extra warps.
#ifndef TC_CORRECT_MB
#define TC_CORRECT_MB 3
#endif
#ifndef TC_CORRECT_MB_CFL
#define TC_CORRECT_MB_CFL 3
#endif
#ifndef TC_CORRECT_KZ
#define TC_CORRECT_KZ 2
#endif
#ifndef TC_CORRECT_G
#define TC_CORRECT_G 1
#endif
template <int WHAT, int IMPL, bool CFL, class T>
__global__ void __launch_bounds__(256, CFL ? TC_CORRECT_MB_CFL : TC_CORRECT_MB)
correct_kernel(Geo g, Bc bc, Coefs cf, FieldsT<T> f, const double * __restrict__ dtp, int rkstep, double nu,
               unsigned long long * dtmin, unsigned * status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  constexpr int KZ = CFL ? TC_CFL_KZ : TC_CORRECT_KZ;
  constexpr int G = CFL ? TC_CORRECT_G : TC_CORRECT_KZ;
  static_assert(KZ % G == 0, "cells per thread must be a multiple of the load group");
  const bool act = i <= nx && j <= ny;
  const bool ix = IMPL >= 0 ? (IMPL & 1) != 0 : bc.implicit[0] != 0;
  const bool iy = IMPL >= 0 ? (IMPL & 2) != 0 : bc.implicit[1] != 0;
  const bool iz = IMPL >= 0 ? (IMPL & 4) != 0 : bc.implicit[2] != 0;
  const double small = 1.e-8;
  double ax = 0., ay = 0., az = 0.;   // |v| + 1e-8 of the corrected velocities (CFL)
  bool bad = false;
#pragma unroll 1
  for (int k0 = 0; k0 < KZ; k0 += G) {
    if (act) {
      // every input of the group is loaded before the first store (the arrays
      // are distinct, which the compiler cannot know), so a thread's loads are
      // in flight together
      const double * psi = f.psi;
      const size_t sj = (size_t)(nx + 2), sk = (size_t)(nx + 2) * (ny + 2);
      const int kb = blockIdx.z * KZ + k0 + 1;
      double psi0[G], psi_im[G], psi_jm[G], psi_km[G], psi_ip[G], psi_jp[G], psi_kp[G];
      double ux0[G], uy0[G], uz0[G], p0[G];
#pragma unroll
      for (int m = 0; m < G; m++) {
        const size_t qp = cidx(g, i, j, kb + m);                                    // p, psi
        const size_t qc = sidx_c<T>(g, i, j, kb + m), qf = sidx_f<T>(g, i, j, kb + m);  // ux, uy, uz
        psi0[m] = __ldg(psi + qp);
        psi_im[m] = __ldg(psi + qp - 1);
        psi_jm[m] = __ldg(psi + qp - sj);
        psi_km[m] = m == 0 ? __ldg(psi + qp - sk) : psi0[m - 1];
        psi_ip[m] = psi_jp[m] = psi_kp[m] = 0.;
        ux0[m] = uy0[m] = uz0[m] = p0[m] = 0.;
        if (WHAT & CORRECT_VELOCITY) {
          if (i >= 2) ux0[m] = f.ux[qf];
          uy0[m] = f.uy[qc];
          uz0[m] = f.uz[qc];
        }
        if (WHAT & CORRECT_PRESSURE) {
          p0[m] = f.p[qp];
          if (ix) psi_ip[m] = __ldg(psi + qp + 1);
          if (iy) psi_jp[m] = __ldg(psi + qp + sj);
          if (iz && m == G - 1) psi_kp[m] = __ldg(psi + qp + sk);
        }
      }
      if (WHAT & CORRECT_PRESSURE) {
#pragma unroll
        for (int m = 0; m + 1 < G; m++)
          if (iz) psi_kp[m] = psi0[m + 1];
      }
      const double dt = *dtp;
      const double pf = rk_gamma(rkstep) * dt;            // correct/main.c:21-22
      const double pp = 0.5 * rk_gamma(rkstep) * dt * nu;  // update_pressure.c:161-162
#pragma unroll
      for (int m = 0; m < G; m++) {
        const int k = kb + m;
        if (WHAT & CORRECT_VELOCITY) {
          const size_t qf = sidx_f<T>(g, i, j, k);
          // ux, i = 2..nx (correct/ux.c:25-52); walls stay zero
          const double vx = (i >= 2) ? ux0[m] - pf * __ldg(cf.c_invhxxf + i) * (-psi_im[m] + psi0[m]) : 0.;
          f.ux[qf] = (T)vx;
          for_images(j, k, ny, nz, [&](int jj, int kk) { f.ux[sidx_f<T>(g, i, jj, kk)] = (T)vx; });
          if (i == nx) {
            f.ux[qf + 1] = (T)0.;
            for_images(j, k, ny, nz, [&](int jj, int kk) { f.ux[sidx_f<T>(g, nx + 1, jj, kk)] = (T)0.; });
          }
          // uy (correct/uy.c:25-52), uz (correct/uz.c:15-44) with their walls
          const double vy = uy0[m] - pf * __ldg(cf.c_invhyxc + i) * (-psi_jm[m] + psi0[m]);
          const double vz = uz0[m] - pf * cf.inv_hz * (-psi_km[m] + psi0[m]);
          auto put = [&](int jj, int kk) {
            const size_t q = sidx_c<T>(g, i, jj, kk);
            f.uy[q] = (T)vy;
            f.uz[q] = (T)vz;
            if (i == 1) { f.uy[q - 1] = (T)bc.uy_xm; f.uz[q - 1] = (T)0.; }
            if (i == nx) { f.uy[q + 1] = (T)bc.uy_xp; f.uz[q + 1] = (T)0.; }
          };
          put(j, k);
          for_images(j, k, ny, nz, put);
          if (CFL) {
            bad |= !isfinite(vx) || !isfinite(vy) || !isfinite(vz);
            if (i >= 2) ax = fmax(ax, fabs(vx) + small);
            ay = fmax(ay, fabs(vy) + small);
            az = fmax(az, fabs(vz) + small);
          }
        }
        // p += psi, then the implicit-direction corrections (update_pressure.c:23-136)
        if (WHAT & CORRECT_PRESSURE) {
          double val = p0[m] + psi0[m];   // p and psi are double in every storage mode
          const double ijd = __ldg(cf.c_invjdxc + i);
          if (ix) {
            const double l = __ldg(cf.c_pxl + i), u = __ldg(cf.c_pxu + i), c = -l - u;
            val -= 2. * pp * ijd * (l * psi_im[m] + c * psi0[m] + u * psi_ip[m]);
          }
          if (iy) {
            const double l = __ldg(cf.c_pyl + i), c = -l - l;
            val -= 2. * pp * ijd * (l * psi_jm[m] + c * psi0[m] + l * psi_jp[m]);
          }
          if (iz) {
            const double l = __ldg(cf.c_pzl + i), c = -l - l;
            val -= 2. * pp * ijd * (l * psi_km[m] + c * psi0[m] + l * psi_kp[m]);
          }
          auto put = [&](int jj, int kk) {
            const size_t q = cidx(g, i, jj, kk);
            f.p[q] = val;
            if (i == 1) f.p[q - 1] = val;
            if (i == nx) f.p[q + 1] = val;
          };
          put(j, k);
          for_images(j, k, ny, nz, put);
        }
      }
    }
  }
  if (CFL) {
    const bool in = i <= nx;
    warp_cfl(ax, ay, az, in ? __ldg(g.hxxf + i) : 1., in ? __ldg(g.hyxc + i) : 1., g.hz, bad, dtmin, status);
  }
}

template <int WHAT, int IMPL, bool CFL, class T>
static void launch_correct_t(const Geo & g, const Bc & bc, const Coefs & cf, const FieldsT<T> & f, const double * dtp,
                             int rkstep, double nu, unsigned long long * dtmin, unsigned * status, cudaStream_t st) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz / (CFL ? TC_CFL_KZ : TC_CORRECT_KZ));   // nz: power of two >= 4
  correct_kernel<WHAT, IMPL, CFL, T><<<grid, block, 0, st>>>(g, bc, cf, f, dtp, rkstep, nu, dtmin, status);
}

template <bool CFL, class T>
static void launch_correct_both(const Geo & g, const Bc & bc, const Coefs & cf, const FieldsT<T> & f,
                                const double * dtp, int rkstep, double nu, unsigned long long * dtmin,
                                unsigned * status, cudaStream_t st) {
  const int mask = (bc.implicit[0] ? 1 : 0) | (bc.implicit[1] ? 2 : 0) | (bc.implicit[2] ? 4 : 0);
  constexpr int B = CORRECT_VELOCITY | CORRECT_PRESSURE;
  switch (mask) {
    case 1: launch_correct_t<B, 1, CFL, T>(g, bc, cf, f, dtp, rkstep, nu, dtmin, status, st); break;
    case 7: launch_correct_t<B, 7, CFL, T>(g, bc, cf, f, dtp, rkstep, nu, dtmin, status, st); break;
    case 0: launch_correct_t<B, 0, CFL, T>(g, bc, cf, f, dtp, rkstep, nu, dtmin, status, st); break;
    default: launch_correct_t<B, -1, CFL, T>(g, bc, cf, f, dtp, rkstep, nu, dtmin, status, st); break;
  }
}

template <class T>
static void launch_correct_s(const Geo & g, const Bc & bc, const Coefs & cf, const FieldsT<T> & f, const double * dtp,
                             int rkstep, double nu, int what, unsigned long long * cfl_dtmin, unsigned * status,
                             cudaStream_t st) {
  if (what == CORRECT_VELOCITY)
    launch_correct_t<CORRECT_VELOCITY, -1, false, T>(g, bc, cf, f, dtp, rkstep, nu, nullptr, status, st);
  else if (what == CORRECT_PRESSURE)
    launch_correct_t<CORRECT_PRESSURE, -1, false, T>(g, bc, cf, f, dtp, rkstep, nu, nullptr, status, st);
  else if (cfl_dtmin)
    launch_correct_both<true, T>(g, bc, cf, f, dtp, rkstep, nu, cfl_dtmin, status, st);
  else
    launch_correct_both<false, T>(g, bc, cf, f, dtp, rkstep, nu, nullptr, status, st);
}

void launch_correct(const Geo & g, const Bc & bc, const Coefs & cf, const FieldBufs & f, const double * dtp,
                    int rkstep, double nu, int what, unsigned long long * cfl_dtmin, unsigned * status,
                    cudaStream_t st) {
  if (f.bytes == 4) launch_correct_s<float>(g, bc, cf, f.as<float>(), dtp, rkstep, nu, what, cfl_dtmin, status, st);
  else launch_correct_s<double>(g, bc, cf, f.as<double>(), dtp, rkstep, nu, what, cfl_dtmin, status, st);
}

// --------------------------------------------------------------- decide_dt
template <class T>
__global__ void __launch_bounds__(256)
dtmin_kernel(Geo g, const T * __restrict__ ux, const T * __restrict__ uy,
             const T * __restrict__ uz, unsigned long long * dtmin, unsigned * status) {
  const double small = 1.e-8;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  bool bad = false;
  double ax = 0., ay = 0., az = 0., hx = 1., hy = 1., hz = 1.;
  if (i <= g.nx && j <= g.ny) {
    hx = __ldg(g.hxxf + i);
    hy = __ldg(g.hyxc + i);
    hz = g.hz;
    for (int k = blockIdx.z + 1; k <= g.nz; k += gridDim.z) {
      if (i >= 2) {
        const double v = __ldg(ux + sidx_f<T>(g, i, j, k));
        bad |= !isfinite(v);
        ax = fmax(ax, fabs(v) + small);
      }
      const double vy = __ldg(uy + sidx_c<T>(g, i, j, k));
      const double vz = __ldg(uz + sidx_c<T>(g, i, j, k));
      bad |= !isfinite(vy) || !isfinite(vz);
      ay = fmax(ay, fabs(vy) + small);
      az = fmax(az, fabs(vz) + small);
    }
  }
  block_cfl(ax, ay, az, hx, hy, hz, bad, dtmin, status);
}

// sets the accumulators of the advective limit back to 1.0, the reference's
// starting value (src/decide_dt.c:40)
__global__ void dtreset_kernel(unsigned long long * dtmin) { dtmin[threadIdx.x] = 0x3ff0000000000000ull; }

void launch_dtreset(unsigned long long * dtmin, cudaStream_t st) { dtreset_kernel<<<1, DT_SLOTS, 0, st>>>(dtmin); }

// one thread per accumulator: their minimum, then dt, and each thread resets
// its accumulator to 1.0
__global__ void __launch_bounds__(DT_SLOTS)
dtfinal_kernel(double coef_adv, const double * caps, unsigned long long * dtmin, double * dtp, unsigned * status) {
  __shared__ double red[DT_SLOTS / 32];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  double v = warp_min(__longlong_as_double((long long)dtmin[t]));
  dtmin[t] = 0x3ff0000000000000ull;  // 1.0
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (t != 0) return;
  double dt = red[0];
  for (int w = 1; w < DT_SLOTS / 32; w++) dt = fmin(dt, red[w]);
  dt = fmin(1., dt);
  dt *= coef_adv;
  for (int d = 0; d < 3; d++) {
    if (caps[d] > 0.) dt = fmin(dt, caps[d]);
  }
  if (!(dt > 0.) || !isfinite(dt)) atomicOr(status, (unsigned)ST_BADDT);
  *dtp = dt;
}

void launch_dtmin(const Geo & g, const FieldBufs & f, unsigned long long * dtmin, unsigned * status, cudaStream_t st) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz < 16 ? g.nz : 16);
  if (f.bytes == 4) {
    const FieldsT<float> a = f.as<float>();
    dtmin_kernel<float><<<grid, block, 0, st>>>(g, a.ux, a.uy, a.uz, dtmin, status);
  } else {
    const FieldsT<double> a = f.as<double>();
    dtmin_kernel<double><<<grid, block, 0, st>>>(g, a.ux, a.uy, a.uz, dtmin, status);
  }
}

void launch_dtfinal(double coef_adv, const double * dt_caps, unsigned long long * dtmin, double * dtp,
                    unsigned * status, cudaStream_t st) {
  dtfinal_kernel<<<1, DT_SLOTS, 0, st>>>(coef_adv, dt_caps, dtmin, dtp, status);
}

void launch_decide_dt(const Geo & g, const FieldBufs & f, double coef_adv, const double * dt_caps,
                      unsigned long long * dtmin, double * dtp, unsigned * status, cudaStream_t st) {
  launch_dtmin(g, f, dtmin, status, st);
  launch_dtfinal(coef_adv, dt_caps, dtmin, dtp, status, st);
}

// --------------------------------------------------------------- boundary conditions
// T: storage type of the field (p and psi are always double; ux, uy, uz, t
// follow the storage mode)
template <class T>
__global__ void bc_kernel(Geo g, Bc bc, int kind, T * __restrict__ a) {
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;   // position in the row
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (j > ny) return;
  const bool state = kind != BC_P && kind != BC_PSI;     // p, psi: reference layout (double)
  auto ic = [&](int ii, int jj, int kk) { return state ? sidx_c<T>(g, ii, jj, kk) : cidx(g, ii, jj, kk); };
  if (kind == BC_UX) {
    if (e > nx) return;                                  // i = e + 1
    T * row = a + sidx_f<T>(g, 1, j, k);
    const T val = (e == 0 || e == nx) ? (T)0. : row[e];
    row[e] = val;
    for_images(j, k, ny, nz, [&](int jj, int kk) { a[sidx_f<T>(g, 1, jj, kk) + e] = val; });
    return;
  }
  if (e > nx + 1) return;                                // i = e
  T * row = a + ic(0, j, k);
  T val;
  if (e == 0 || e == nx + 1) {
    const bool lo = (e == 0);
    switch (kind) {
      case BC_UY: val = (T)(lo ? bc.uy_xm : bc.uy_xp); break;
      case BC_UZ: val = (T)0.; break;
      case BC_T: val = (T)(lo ? bc.t_xm : bc.t_xp); break;
      default: val = lo ? row[1] : row[nx]; break;       // p, psi: Neumann copy
    }
  } else {
    val = row[e];
  }
  row[e] = val;
  for_images(j, k, ny, nz, [&](int jj, int kk) { a[ic(0, jj, kk) + e] = val; });
}

void launch_bc(const Geo & g, const Bc & bc, BcKind kind, void * a, int bytes, cudaStream_t st) {
  dim3 block(64, 4, 1);
  dim3 grid((g.nx + 2 + 63) / 64, (g.ny + 3) / 4, g.nz);
  if (bytes == 4) bc_kernel<float><<<grid, block, 0, st>>>(g, bc, (int)kind, static_cast<float *>(a));
  else bc_kernel<double><<<grid, block, 0, st>>>(g, bc, (int)kind, static_cast<double *>(a));
}

// --------------------------------------------------------------- tensors
// Row lengths: face tensors (lxy lxz lyx0 lyx1 lzx) nx+1, centre tensors nx.
template <class T>
__global__ void tensor_kernel(Geo g, Coefs cf, FieldsT<T> f, Tensors tn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;   // 1..nx+1
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i > nx + 1 || j > ny) return;
  auto fi = [&](int ii, int jj, int kk) { return (size_t)(ii - 1) + (size_t)(nx + 1) * ((size_t)jj + (size_t)(ny + 2) * kk); };
  auto ci = [&](int ii, int jj, int kk) { return (size_t)(ii - 1) + (size_t)nx * ((size_t)jj + (size_t)(ny + 2) * kk); };
  const T * ux = f.ux;
  const T * uy = f.uy;
  const T * uz = f.uz;
  {  // face tensors
    const double ih = __ldg(cf.c_invhxxf + i);
    const double lxy = ih * (-(double)uy[sidx_c<T>(g, i - 1, j, k)] + (double)uy[sidx_c<T>(g, i, j, k)]);
    const double lxz = ih * (-(double)uz[sidx_c<T>(g, i - 1, j, k)] + (double)uz[sidx_c<T>(g, i, j, k)]);
    const double lyx0 = __ldg(cf.c_invhyxf + i) * (-(double)ux[sidx_f<T>(g, i, j - 1, k)] + (double)ux[sidx_f<T>(g, i, j, k)]);
    const double lyx1 = __ldg(cf.c_lyx1f + i) * (__ldg(cf.c_wm + i) * (double)uy[sidx_c<T>(g, i - 1, j, k)] + __ldg(cf.c_wp + i) * (double)uy[sidx_c<T>(g, i, j, k)]);
    const double lzx = cf.inv_hz * (-(double)ux[sidx_f<T>(g, i, j, k - 1)] + (double)ux[sidx_f<T>(g, i, j, k)]);
    const double vals[5] = {lxy, lxz, lyx0, lyx1, lzx};
    const int slot[5] = {1, 2, 3, 4, 8};
    for (int s = 0; s < 5; s++) {
      double * a = tn.a[slot[s]];
      a[fi(i, j, k)] = vals[s];
      for_images(j, k, ny, nz, [&](int jj, int kk) { a[fi(i, jj, kk)] = vals[s]; });
    }
  }
  if (i <= nx) {  // centre tensors
    const double lxx = (1. / __ldg(g.hxxc + i)) * (-(double)ux[sidx_f<T>(g, i, j, k)] + (double)ux[sidx_f<T>(g, i + 1, j, k)]);
    const double ihy = __ldg(cf.c_invhyxc + i);
    const double lyy0 = ihy * (-(double)uy[sidx_c<T>(g, i, j, k)] + (double)uy[sidx_c<T>(g, i, j + 1, k)]);
    const double lyy1 = __ldg(cf.c_lyy1 + i) * (0.5 * (double)ux[sidx_f<T>(g, i, j, k)] + 0.5 * (double)ux[sidx_f<T>(g, i + 1, j, k)]);
    const double lyz = ihy * (-(double)uz[sidx_c<T>(g, i, j - 1, k)] + (double)uz[sidx_c<T>(g, i, j, k)]);
    const double lzy = cf.inv_hz * (-(double)uy[sidx_c<T>(g, i, j, k - 1)] + (double)uy[sidx_c<T>(g, i, j, k)]);
    const double lzz = cf.inv_hz * (-(double)uz[sidx_c<T>(g, i, j, k)] + (double)uz[sidx_c<T>(g, i, j, k + 1)]);
    const double vals[6] = {lxx, lyy0, lyy1, lyz, lzy, lzz};
    const int slot[6] = {0, 5, 6, 7, 9, 10};
    for (int s = 0; s < 6; s++) {
      double * a = tn.a[slot[s]];
      a[ci(i, j, k)] = vals[s];
      for_images(j, k, ny, nz, [&](int jj, int kk) { a[ci(i, jj, kk)] = vals[s]; });
    }
  }
}

void launch_tensors(const Geo & g, const Coefs & cf, const FieldBufs & f, const Tensors & tn, cudaStream_t st) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 1 + 31) / 32, (g.ny + 7) / 8, g.nz);
  if (f.bytes == 4) tensor_kernel<float><<<grid, block, 0, st>>>(g, cf, f.as<float>(), tn);
  else tensor_kernel<double><<<grid, block, 0, st>>>(g, cf, f.as<double>(), tn);
}

// --------------------------------------------------------------- diagnostics
// partial[b][0..8]: max|div|, inj_m, inj_s, dis_m, dis_s, e_ux, e_uy, e_uz, e_t
constexpr int DIAG_BLOCKS = 296;

// f: the current fields (divergence, energies, the wall velocity of the
// momentum injection, every scalar term); fs: the fields the velocity-gradient
// tensors are formed from (injection and dissipation of momentum). The
// reference logs tensors of the last predict's input fields
// (src/fluid/predict/main.c:56-82, read by src/logging/injection.c:49-51 and
// dissipation.c); fs = f gives the tensors of the current fields.
template <class T>
__global__ void __launch_bounds__(256)
diag_kernel(Geo g, Coefs cf, Bc bc, FieldsT<T> f, FieldsT<T> fs, double * partial) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long total = (long long)(nx + 1) * ny * nz;
  double acc[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
  const T * ux = f.ux;
  const T * uy = f.uy;
  const T * uz = f.uz;
  const T * t = f.t;
  const T * sux = fs.ux;
  const T * suy = fs.uy;
  const T * suz = fs.uz;
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
    const double uyim = (double)uy[sidx_c<T>(g, i - 1, j, k)], uyi = (double)uy[sidx_c<T>(g, i, j, k)];
    const double suyim = (double)suy[sidx_c<T>(g, i - 1, j, k)], suyi = (double)suy[sidx_c<T>(g, i, j, k)];
    const double lxy = ih * (-suyim + suyi);
    const double lxz = ih * (-(double)suz[sidx_c<T>(g, i - 1, j, k)] + (double)suz[sidx_c<T>(g, i, j, k)]);
    const double lyx = __ldg(cf.c_invhyxf + i) * (-(double)sux[sidx_f<T>(g, i, j - 1, k)] + (double)sux[sidx_f<T>(g, i, j, k)])
                     + __ldg(cf.c_lyx1f + i) * (__ldg(cf.c_wm + i) * suyim + __ldg(cf.c_wp + i) * suyi);
    const double lzx = cf.inv_hz * (-(double)sux[sidx_f<T>(g, i, j, k - 1)] + (double)sux[sidx_f<T>(g, i, j, k)]);
    // dissipation.c:40-151 (face contributions)
    acc[3] += jdf * lyx * (lyx + lxy);
    acc[3] += jdf * lzx * (lzx + lxz);
    acc[3] += jdf * lxy * (lxy + lyx);
    acc[3] += jdf * lxz * (lxz + lzx);
    {  // dissipation.c:240-265 (scalar, x)
      const double d = -(double)t[sidx_c<T>(g, i - 1, j, k)] + (double)t[sidx_c<T>(g, i, j, k)];
      const double q = d / hxf;
      acc[4] += jdf * (q * q);
    }
    // injection.c:55-98 at the two walls
    if (i == 1 || i == nx + 1) {
      const double sgn = (i == 1) ? -1. : 1.;
      const double uyw = (i == 1) ? uyim : uyi;
      acc[1] += sgn * jdf / hxf * uyw * (lyx + lxy);
      const double tw = (i == 1) ? (double)t[sidx_c<T>(g, 0, j, k)] : (double)t[sidx_c<T>(g, nx + 1, j, k)];
      const double dtw = (i == 1) ? (-(double)t[sidx_c<T>(g, 0, j, k)] + (double)t[sidx_c<T>(g, 1, j, k)])
                                  : (-(double)t[sidx_c<T>(g, nx, j, k)] + (double)t[sidx_c<T>(g, nx + 1, j, k)]);
      acc[2] += sgn * jdf / hxf * tw / hxf * dtw;
    }
    if (i >= 2 && i <= nx) {  // total_energy.c:45-51
      const double v = (double)ux[sidx_f<T>(g, i, j, k)];
      acc[5] += jdf * 0.5 * (v * v);
    }
    if (i <= nx) {
      const double jdc = __ldg(g.jdxc + i);
      const double ux0 = (double)ux[sidx_f<T>(g, i, j, k)], ux1 = (double)ux[sidx_f<T>(g, i + 1, j, k)];
      const double uy0 = uyi, uy1 = (double)uy[sidx_c<T>(g, i, j + 1, k)];
      const double uz0 = (double)uz[sidx_c<T>(g, i, j, k)], uz1 = (double)uz[sidx_c<T>(g, i, j, k + 1)];
      // divergence.c:56-78
      const double div = __ldg(cf.c_invjdxc + i) * (
          -__ldg(cf.c_jf + i) * ux0 + __ldg(cf.c_jf + i + 1) * ux1
          - __ldg(cf.c_e1 + i) * uy0 + __ldg(cf.c_e1 + i) * uy1
          - __ldg(cf.c_e2 + i) * uz0 + __ldg(cf.c_e2 + i) * uz1);
      acc[0] = fmax(acc[0], fabs(div));
      // centre tensors and dissipation contributions
      const double sux0 = (double)sux[sidx_f<T>(g, i, j, k)], sux1 = (double)sux[sidx_f<T>(g, i + 1, j, k)];
      const double suy0 = suyi, suy1 = (double)suy[sidx_c<T>(g, i, j + 1, k)];
      const double suz0 = (double)suz[sidx_c<T>(g, i, j, k)], suz1 = (double)suz[sidx_c<T>(g, i, j, k + 1)];
      const double lxx = (1. / __ldg(g.hxxc + i)) * (-sux0 + sux1);
      const double ihy = __ldg(cf.c_invhyxc + i);
      const double lyy = ihy * (-suy0 + suy1) + __ldg(cf.c_lyy1 + i) * (0.5 * sux0 + 0.5 * sux1);
      const double lyz = ihy * (-(double)suz[sidx_c<T>(g, i, j - 1, k)] + suz0);
      const double lzy = cf.inv_hz * (-(double)suy[sidx_c<T>(g, i, j, k - 1)] + suy0);
      const double lzz = cf.inv_hz * (-suz0 + suz1);
      acc[3] += jdc * lxx * (lxx + lxx);
      acc[3] += jdc * lyy * (lyy + lyy);
      acc[3] += jdc * lzy * (lzy + lyz);
      acc[3] += jdc * lyz * (lyz + lzy);
      acc[3] += jdc * lzz * (lzz + lzz);
      const double t0 = (double)t[sidx_c<T>(g, i, j, k)];
      {
        const double q = (-(double)t[sidx_c<T>(g, i, j - 1, k)] + t0) / __ldg(g.hyxc + i);
        acc[4] += jdc * (q * q);
      }
      {
        const double q = (-(double)t[sidx_c<T>(g, i, j, k - 1)] + t0) / g.hz;
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

void launch_diagnostics(const Geo & g, const Coefs & cf, const Bc & bc, const FieldBufs & f, const FieldBufs & fs,
                        double nu, double kappa, double * out, double * partial, cudaStream_t st) {
  if (f.bytes == 4) diag_kernel<float><<<DIAG_BLOCKS, 256, 0, st>>>(g, cf, bc, f.as<float>(), fs.as<float>(), partial);
  else diag_kernel<double><<<DIAG_BLOCKS, 256, 0, st>>>(g, cf, bc, f.as<double>(), fs.as<double>(), partial);
  diag_final_kernel<<<1, 32, 0, st>>>(partial, DIAG_BLOCKS, nu, kappa, out);
}

// --------------------------------------------------------------- statistics
// src/statistics.c:124-240: one thread per (i = 0..nx+1, j, k) of the interior
// j, k adds this sample to the eight accumulators. Products and sums are
// rounded separately (no contraction), as the reference's C does, so the
// accumulated values follow its arithmetic.
template <class T>
__global__ void stats_kernel(Geo g, Coefs cf, FieldsT<T> f, FieldsT<T> fs, Stats st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;   // 0..nx+1
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  const int nx = g.nx, ny = g.ny;
  if (i > nx + 1 || j > ny) return;
  const size_t line = (size_t)(j - 1) + (size_t)ny * (k - 1);
  {  // uy, uz at i = 0..nx+1 (statistics.c:146-185)
    const size_t q = (size_t)i + (size_t)(nx + 2) * line;
    const double vy = (double)f.uy[sidx_c<T>(g, i, j, k)], vz = (double)f.uz[sidx_c<T>(g, i, j, k)];
    st.a[2][q] = __dadd_rn(st.a[2][q], vy);
    st.a[3][q] = __dadd_rn(st.a[3][q], __dmul_rn(vy, vy));
    st.a[4][q] = __dadd_rn(st.a[4][q], vz);
    st.a[5][q] = __dadd_rn(st.a[5][q], __dmul_rn(vz, vz));
  }
  if (i < 1) return;
  const size_t q = (size_t)(i - 1) + (size_t)(nx + 1) * line;
  const double vx = (double)f.ux[sidx_f<T>(g, i, j, k)];
  st.a[0][q] = __dadd_rn(st.a[0][q], vx);                 // :126-144
  st.a[1][q] = __dadd_rn(st.a[1][q], __dmul_rn(vx, vx));
  {  // adv (:187-204): ux averaged to the y face times uy averaged to the x face
    const double x = __dadd_rn(__dmul_rn(0.5, (double)f.ux[sidx_f<T>(g, i, j - 1, k)]), __dmul_rn(0.5, vx));
    const double y = __dadd_rn(__dmul_rn(0.5, (double)f.uy[sidx_c<T>(g, i - 1, j, k)]),
                               __dmul_rn(0.5, (double)f.uy[sidx_c<T>(g, i, j, k)]));
    st.a[6][q] = __dadd_rn(st.a[6][q], __dmul_rn(x, y));
  }
  {  // dif (:206-223): lyx0 + lyx1 + lxy (predict/lyx.c:24-83, lxy.c:19-49) of fs
    const double uym = (double)fs.uy[sidx_c<T>(g, i - 1, j, k)], uy0 = (double)fs.uy[sidx_c<T>(g, i, j, k)];
    const double lyx0 = __dmul_rn(__ldg(cf.c_invhyxf + i),
                                  __dadd_rn(-(double)fs.ux[sidx_f<T>(g, i, j - 1, k)], (double)fs.ux[sidx_f<T>(g, i, j, k)]));
    const double lyx1 = __dmul_rn(__ldg(cf.c_lyx1f + i),
                                  __dadd_rn(__dmul_rn(__ldg(cf.c_wm + i), uym), __dmul_rn(__ldg(cf.c_wp + i), uy0)));
    const double lxy = __dmul_rn(__ldg(cf.c_invhxxf + i), __dadd_rn(-uym, uy0));
    st.a[7][q] = __dadd_rn(st.a[7][q], __dadd_rn(__dadd_rn(lyx0, lyx1), lxy));
  }
}

void launch_statistics(const Geo & g, const Coefs & cf, const FieldBufs & f, const FieldBufs & fs, const Stats & s,
                       cudaStream_t st) {
  dim3 block(64, 4, 1);
  dim3 grid((g.nx + 2 + 63) / 64, (g.ny + 3) / 4, g.nz);
  if (f.bytes == 4) stats_kernel<float><<<grid, block, 0, st>>>(g, cf, f.as<float>(), fs.as<float>(), s);
  else stats_kernel<double><<<grid, block, 0, st>>>(g, cf, f.as<double>(), fs.as<double>(), s);
}

// mean uy(r): out[i] = inv_count * sum over j, k of uy1[k][j][i], one block per i
__global__ void stat_profile_kernel(Geo g, const double * __restrict__ uy1, double inv_count, double * out) {
  const int i = blockIdx.x;
  const size_t lines = (size_t)g.ny * g.nz;
  double acc = 0.;
  for (size_t l = threadIdx.x; l < lines; l += blockDim.x) acc += uy1[(size_t)i + (size_t)(g.nx + 2) * l];
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[w];
    out[i] = v * inv_count;
  }
}

void launch_stat_profile(const Geo & g, const double * uy1, double inv_count, double * out, cudaStream_t st) {
  stat_profile_kernel<<<g.nx + 2, 256, 0, st>>>(g, uy1, inv_count, out);
}

// --------------------------------------------------------------- initial field
// A seeded initial field generated on the device: uy and t from radial profiles
// (one value per i, formed on the host), plus uniform noise in [-amp, amp) on
// ux (interior faces), uy, uz and t. The noise of value q of field f is a
// function of (seed, f, q) alone (SplitMix64 finaliser of a counter), so the
// field does not depend on the launch shape. p = 0. Halos are left to the
// boundary kernels.
__device__ __forceinline__ double noise(unsigned long long seed, unsigned f, unsigned long long q, double amp) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (q + 1ull + ((unsigned long long)f << 58));
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const double u = (double)(z >> 11) * 0x1.0p-53;   // [0, 1)
  return amp * (2. * u - 1.);
}

template <class T>
__global__ void initial_field_kernel(Geo g, FieldsT<T> f, const double * __restrict__ uy_prof,
                                     const double * __restrict__ t_prof, unsigned long long seed, double amp_u,
                                     double amp_t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;   // 0..nx+1
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  const int nx = g.nx, ny = g.ny;
  if (i > nx + 1 || j > ny) return;
  const unsigned long long q = (unsigned long long)i + (unsigned long long)(nx + 2) * ((unsigned long long)(j - 1) +
                               (unsigned long long)ny * (unsigned long long)(k - 1));
  f.uy[sidx_c<T>(g, i, j, k)] = (T)(uy_prof[i] + noise(seed, 1, q, amp_u));
  f.uz[sidx_c<T>(g, i, j, k)] = (T)noise(seed, 2, q, amp_u);
  f.t[sidx_c<T>(g, i, j, k)] = (T)(t_prof[i] + (amp_t > 0. ? noise(seed, 3, q, amp_t) : 0.));
  f.p[sidx_c<double>(g, i, j, k)] = 0.;   // p is FP64 in the reference layout in every storage mode
  if (i >= 1) f.ux[sidx_f<T>(g, i, j, k)] = (T)((i == 1 || i == nx + 1) ? 0. : noise(seed, 0, q, amp_u));
}

void launch_initial_field(const Geo & g, const FieldBufs & f, const double * uy_prof, const double * t_prof,
                          unsigned long long seed, double amp_u, double amp_t, cudaStream_t st) {
  dim3 block(64, 4, 1);
  dim3 grid((g.nx + 2 + 63) / 64, (g.ny + 3) / 4, g.nz);
  if (f.bytes == 4)
    initial_field_kernel<float><<<grid, block, 0, st>>>(g, f.as<float>(), uy_prof, t_prof, seed, amp_u, amp_t);
  else
    initial_field_kernel<double><<<grid, block, 0, st>>>(g, f.as<double>(), uy_prof, t_prof, seed, amp_u, amp_t);
}

// --------------------------------------------------------------- radial slabs
// out[((k - 1) ny + j - 1) count + c] = a(i0 + c, j, k) over the interior j, k
template <class T>
__global__ void slab_kernel(Geo g, const T * __restrict__ a, bool face, int i0, int count, double * __restrict__ out) {
  const size_t n = (size_t)count * g.ny * g.nz;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(q % count);
    const size_t line = q / count;
    const int j = (int)(line % g.ny) + 1, k = (int)(line / g.ny) + 1;
    out[q] = (double)a[face ? sidx_f<T>(g, i0 + c, j, k) : sidx_c<T>(g, i0 + c, j, k)];
  }
}

void launch_slab(const Geo & g, const void * a, int bytes, bool face, int i0, int count, double * out,
                 cudaStream_t st) {
  const size_t n = (size_t)count * g.ny * g.nz;
  const unsigned blocks = (unsigned)((n + 255) / 256 < 2368 ? (n + 255) / 256 : 2368);
  if (bytes == 4) slab_kernel<float><<<blocks, 256, 0, st>>>(g, static_cast<const float *>(a), face, i0, count, out);
  else slab_kernel<double><<<blocks, 256, 0, st>>>(g, static_cast<const double *>(a), face, i0, count, out);
}

// --------------------------------------------------------------- FP32 storage
// rows of nref doubles (the reference's layout) <-> rows of pitch floats with
// element e of a row at e + shift (the FP32 layout: shift 1 for ux, whose face
// i sits at element i - 1 of a reference row and at element i of an FP32 row)
__global__ void pack32_kernel(const double * __restrict__ src, float * __restrict__ dst, size_t rows, int nref,
                              int pitch, int shift) {
  const size_t n = rows * (size_t)nref;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const size_t r = q / nref, e = q % nref;
    dst[r * pitch + e + shift] = (float)src[q];
  }
}
__global__ void unpack32_kernel(const float * __restrict__ src, double * __restrict__ dst, size_t rows, int nref,
                                int pitch, int shift) {
  const size_t n = rows * (size_t)nref;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const size_t r = q / nref, e = q % nref;
    dst[q] = (double)src[r * pitch + e + shift];
  }
}
void launch_pack32(const double * src, float * dst, size_t rows, int nref, int pitch, int shift, cudaStream_t st) {
  pack32_kernel<<<2368, 256, 0, st>>>(src, dst, rows, nref, pitch, shift);
}
void launch_unpack32(const float * src, double * dst, size_t rows, int nref, int pitch, int shift, cudaStream_t st) {
  unpack32_kernel<<<2368, 256, 0, st>>>(src, dst, rows, nref, pitch, shift);
}

}  // namespace tcgpu
