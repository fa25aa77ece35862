// Predict stage, the parts around the marching kernel (tc_march.cu):
//
// xfactor_kernel    line-independent Thomas factors of the radial implicit
//                   systems (I - k L_x) for the three substeps, from dt on the device.
// apply_kernel      u + delta after the y / z solves (planar configuration).
// ysolve/zsolve     periodic (Sherman-Morrison, src/tdm.c:66-106) solves in y
//                   and z for the planar configuration, one thread per line.
#include "tc_common.cuh"
#include "tc_kernels.h"

namespace tcgpu {

// ------------------------------------------------------------ Thomas factors
// One thread per (substep, variable, direction): the forward-elimination
// factors of gtsv (src/tdm.c:24-44) for (I - pf L) with
//   l = -pf lap.l, c = 1 - pf lap.c, u = -pf lap.u   (predict/linear_system.c:26-33)
// pf = 0.5 gamma dt diffusivity, doubled for the "diagonal" component
// (ux-x ux.c:502, uy-y uy.c:541, uz-z uz.c:451, t-y t.c:348).
// Output per line family: lo[n] = l (lo[0] = 0), w[n] (w[0] = 1/c[0],
// w[i] = 1/(c - l v)), v[n] (v[n-1] = 0), so every row of the forward sweep
// reads q = w (r - l q_prev). Entries from n on stay zero. Rows are stored
// interleaved for the warp that solves them (XFactors::ne).
__global__ void xfactor_kernel(XFactors xf, const double * __restrict__ dtp, double nu, double kappa) {
  const int tid = threadIdx.x;
  if (tid >= 12) return;
  const int rk = tid / 4, var = tid % 4;
  const double dt = *dtp;
  const double diff = (var == VT) ? kappa : nu;
  double pf = 0.5 * rk_gamma(rk) * dt * diff;
  if (var == VUX) pf = 2. * pf;
  const int n = xf.n[var];
  const double * ll = xf.lap_l[var];
  const double * lc = xf.lap_c[var];
  const double * lu = xf.lap_u[var];
  double * lo = xf.lo + (size_t)(rk * 4 + var) * xf.stride;
  double * w = xf.w + (size_t)(rk * 4 + var) * xf.stride;
  double * v = xf.v + (size_t)(rk * 4 + var) * xf.stride;
  const int ne = xf.ne;
  double vprev = 0.;
  for (int e = 0; e < n; e++) {
    const int pe = (e % ne) * 32 + e / ne;   // interleaved position of element e
    const double l = -pf * ll[e];
    const double c = 1. - pf * lc[e];
    const double u = -pf * lu[e];
    lo[pe] = (e == 0) ? 0. : l;
    if (e == 0) {
      w[pe] = 1. / c;
      vprev = u / c;
      v[pe] = (n > 1) ? vprev : 0.;
    } else if (e < n - 1) {
      const double val = 1. / (c - l * vprev);
      w[pe] = val;
      vprev = val * u;
      v[pe] = vprev;
    } else {
      w[pe] = 1. / (c - l * vprev);
      v[pe] = 0.;
    }
  }
}

// out = in + delta for every cell, walls and images (after the y / z solves)
template <class T>
__global__ void __launch_bounds__(256)
apply_kernel(Geo g, Bc bc, FieldsT<T> in, FieldsT<T> out, DeltaSet ds) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i > nx || j > ny) return;
  const size_t qc = pidx(nx, ny, i - 1, j, k);
  const double vx = (i >= 2) ? (double)in.ux[sidx_f<T>(g, i, j, k)] + ds.d[VUX][pidx(nx - 1, ny, i - 2, j, k)] : 0.;
  const double vy = (double)in.uy[sidx_c<T>(g, i, j, k)] + ds.d[VUY][qc];
  const double vz = (double)in.uz[sidx_c<T>(g, i, j, k)] + ds.d[VUZ][qc];
  const double vt = (double)in.t[sidx_c<T>(g, i, j, k)] + ds.d[VT][qc];
  auto put = [&](int jj, int kk) {
    out.ux[sidx_f<T>(g, i, jj, kk)] = (T)(vx);
    out.uy[sidx_c<T>(g, i, jj, kk)] = (T)(vy);
    out.uz[sidx_c<T>(g, i, jj, kk)] = (T)(vz);
    out.t[sidx_c<T>(g, i, jj, kk)] = (T)(vt);
    if (i == 1) {
      out.uy[sidx_c<T>(g, 0, jj, kk)] = (T)(bc.uy_xm);
      out.uz[sidx_c<T>(g, 0, jj, kk)] = (T)(0.);
      out.t[sidx_c<T>(g, 0, jj, kk)] = (T)(bc.t_xm);
    }
    if (i == nx) {
      out.ux[sidx_f<T>(g, nx + 1, jj, kk)] = (T)(0.);
      out.uy[sidx_c<T>(g, nx + 1, jj, kk)] = (T)(bc.uy_xp);
      out.uz[sidx_c<T>(g, nx + 1, jj, kk)] = (T)(0.);
      out.t[sidx_c<T>(g, nx + 1, jj, kk)] = (T)(bc.t_xp);
    }
  };
  put(j, k);
  for_images(j, k, ny, nz, put);
}

// ------------------------------------------------------------ periodic y / z solves
// One thread per line; coefficients (I - pf L_y) with lapy depending on i
// (predict/linear_system.c:39-70), (I - pf L_z) scalar (:72-103). The
// Sherman-Morrison correction vector q1 and the elimination factors are
// recomputed per line (they depend on i only; lines are cheap here).
__global__ void ysolve_kernel(Geo g, YZFactors yf, int rkstep, int var,
                              double * __restrict__ delta) {
  // lines (ii, k), thread along ii for coalescing (delta is [k][j][ii])
  const int n_i = yf.n_i[var];
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)n_i * g.nz) return;
  const int ii = (int)(tid % n_i);
  const int k = (int)(tid / n_i) + 1;
  const int n = g.ny;
  const size_t so = (size_t)(rkstep * 4 + var) * yf.stride_y;
  // per-ii factors of the reduced (n-1) system and the correction vector
  const int fi = yf.uniform_y ? 0 : ii;
  const double * v = yf.v + so + (size_t)fi * n;
  const double * w = yf.w + so + (size_t)fi * n;
  const double * q1 = yf.q1 + so + (size_t)fi * n;
  const double l = yf.l[(rkstep * 4 + var) * yf.max_i + fi];
  const double c = yf.c[(rkstep * 4 + var) * yf.max_i + fi];
  const double u = yf.u[(rkstep * 4 + var) * yf.max_i + fi];
  double * q = delta + (size_t)ii + (size_t)n_i * (size_t)n * (size_t)(k - 1);
  const size_t st = (size_t)n_i;
  // gtsv on q[0..n-2]
  double prev = q[0] / c;
  q[0] = prev;
  for (int e = 1; e < n - 1; e++) {
    const double r = w[e] * (q[e * st] - l * prev);
    q[e * st] = r;
    prev = r;
  }
  for (int e = n - 3; e >= 0; e--) {
    const double x = q[e * st] - v[e] * q[(e + 1) * st];
    q[e * st] = x;
  }
  const double num = q[(n - 1) * st] - u * q[0] - l * q[(n - 2) * st];
  const double den = c + u * q1[0] + l * q1[n - 2];
  const double last = fabs(den) < 2.220446049250313e-16 ? 0. : num / den;
  q[(n - 1) * st] = last;
  for (int e = 0; e < n - 1; e++) q[e * st] = q[e * st] + last * q1[e];
}

__global__ void zsolve_kernel(Geo g, YZFactors yf, int rkstep, int var,
                              double * __restrict__ delta) {
  // lines (ii, j), thread along ii; delta is [k][j][ii], stride n_i*ny in k
  const int n_i = yf.n_i[var];
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)n_i * g.ny) return;
  const int ii = (int)(tid % n_i);
  const int j = (int)(tid / n_i) + 1;
  const int n = g.nz;
  const size_t so = (size_t)(rkstep * 4 + var) * yf.stride_z;
  const double * v = yf.vz + so;
  const double * w = yf.wz + so;
  const double * q1 = yf.q1z + so;
  const double l = yf.lz[rkstep * 4 + var];
  const double c = yf.cz[rkstep * 4 + var];
  const double u = yf.uz[rkstep * 4 + var];
  double * q = delta + (size_t)ii + (size_t)n_i * (size_t)(j - 1);
  const size_t st = (size_t)n_i * (size_t)g.ny;
  double prev = q[0] / c;
  q[0] = prev;
  for (int e = 1; e < n - 1; e++) {
    const double r = w[e] * (q[e * st] - l * prev);
    q[e * st] = r;
    prev = r;
  }
  for (int e = n - 3; e >= 0; e--) {
    q[e * st] = q[e * st] - v[e] * q[(e + 1) * st];
  }
  const double num = q[(n - 1) * st] - u * q[0] - l * q[(n - 2) * st];
  const double den = c + u * q1[0] + l * q1[n - 2];
  const double last = fabs(den) < 2.220446049250313e-16 ? 0. : num / den;
  q[(n - 1) * st] = last;
  for (int e = 0; e < n - 1; e++) q[e * st] = q[e * st] + last * q1[e];
}

// ------------------------------------------------------------ periodic solves, one warp per line
// The same solves for lines of N = 32 E points: a CTA takes a tile of PT
// consecutive radial indices of one plane (y lines) or one row (z lines) into
// shared memory with coalesced loads, and each warp solves whole lines with
// the forward and backward Thomas recurrences written as affine maps
// (y_j = a_j y_{j-1} + b_j) combined by a 5-level shuffle scan, E points per
// lane; then the Sherman-Morrison correction (src/tdm.c:88-99) and a coalesced
// store. Element (j, t) of the tile sits at j PT + (t ^ (j / E mod PT)), so the
// 32 lanes reading element j = lane E + e of one line hit distinct banks.
#ifndef TC_PLINES_PT
#define TC_PLINES_PT 16
#endif
#ifndef TC_PLINES_THREADS
#define TC_PLINES_THREADS 256
#endif
constexpr int PT = TC_PLINES_PT;

struct PAff { double a, b; };

// element j of a staged factor row: row j / 16, column (j mod 16) ^ (j / 16 mod
// 16), so the lanes reading j = lane E + e (E = 4 .. 16) hit distinct banks
__device__ __forceinline__ int fsw(int j) { return (j & ~15) | ((j & 15) ^ ((j >> 4) & 15)); }

template <int E, bool UNI>
__global__ void __launch_bounds__(TC_PLINES_THREADS) periodic_lines_kernel(
    int n_i, long long outer_stride, long long elem_stride, const double * __restrict__ fl,
    const double * __restrict__ fc, const double * __restrict__ fu, int lcu_stride, const double * __restrict__ fw,
    const double * __restrict__ fv, const double * __restrict__ fq1, int fac_stride, double * __restrict__ delta) {
  constexpr int N = 32 * E;
  extern __shared__ double sq[];
  const int ntile = (n_i + PT - 1) / PT;
  const int tile = (int)(blockIdx.x % ntile);
  const long long outer = blockIdx.x / ntile;
  const int ii0 = tile * PT;
  const int nt = min(PT, n_i - ii0);
  double * base = delta + ii0 + outer_stride * outer;
  // all of a thread's loads in flight at once (PER independent loads)
  constexpr int NT = TC_PLINES_THREADS, PER = N * PT / NT;
  static_assert((N * PT) % NT == 0, "tile size must be a multiple of the thread count");
  {
    double buf[PER];
#pragma unroll
    for (int r = 0; r < PER; r++) {
      const int q = threadIdx.x + r * NT, t = q % PT, j = q / PT;
      buf[r] = t < nt ? base[(long long)j * elem_stride + t] : 0.;
    }
#pragma unroll
    for (int r = 0; r < PER; r++) {
      const int q = threadIdx.x + r * NT, t = q % PT, j = q / PT;
      sq[j * PT + (t ^ ((j / E) & (PT - 1)))] = buf[r];
    }
  }
  // one set of factors for every line: staged once (w, v, q1 after the tile)
  double * sfw = sq + N * PT, * sfv = sfw + N, * sfq = sfv + N;
  if constexpr (UNI) {
    for (int j = threadIdx.x; j < N; j += NT) {
      sfw[fsw(j)] = fw[j];
      sfv[fsw(j)] = fv[j];
      sfq[fsw(j)] = fq1[j];
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int t = wid; t < nt; t += nw) {
    const int ii = ii0 + t;
    const double l = fl[ii * lcu_stride], c = fc[ii * lcu_stride], u = fu[ii * lcu_stride];
    const double * w = fw + (size_t)ii * fac_stride;
    const double * v = fv + (size_t)ii * fac_stride;
    const double * q1 = fq1 + (size_t)ii * fac_stride;
    const int sw = t ^ (lane & (PT - 1));
    double q[E], ww[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      q[e] = sq[(lane * E + e) * PT + sw];
      ww[e] = UNI ? sfw[fsw(lane * E + e)] : w[lane * E + e];
    }
    const double qlast = __shfl_sync(0xffffffffu, q[E - 1], 31);   // right-hand side of row N - 1
    // forward sweep of the reduced system (rows 0 .. N-2): y_0 = q_0 / c,
    // y_j = w_j (q_j - l y_{j-1}); row N - 1 is left as it is
    // the lane's maps y_j = fa_j y_{j-1} + fb_j, combined by an in-register
    // prefix (log2 E levels of independent compositions, not an E-long chain)
    double fa[E], fb[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int j = lane * E + e;
      if (j == 0) { fa[e] = 0.; fb[e] = q[e] / c; }
      else if (j == N - 1) { fa[e] = 1.; fb[e] = 0.; }
      else { fa[e] = -ww[e] * l; fb[e] = ww[e] * q[e]; }
    }
#pragma unroll
    for (int d = 1; d < E; d <<= 1) {
#pragma unroll
      for (int e = E - 1; e >= d; e--) {
        fb[e] = fa[e] * fb[e - d] + fb[e];
        fa[e] = fa[e] * fa[e - d];
      }
    }
    PAff acc{fa[E - 1], fb[E - 1]};
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double oa = __shfl_up_sync(0xffffffffu, acc.a, off);
      const double ob = __shfl_up_sync(0xffffffffu, acc.b, off);
      if (lane >= off) { acc.b = acc.a * ob + acc.b; acc.a = acc.a * oa; }
    }
    double yin = __shfl_up_sync(0xffffffffu, acc.b, 1);
    if (lane == 0) yin = 0.;
#pragma unroll
    for (int e = 0; e < E; e++) q[e] = fa[e] * yin + fb[e];   // row N - 1 is not used below
    // backward sweep: x_{N-2} = y_{N-2}, x_j = y_j - v_j x_{j+1} (v_{N-2} = 0),
    // suffix maps combined the same way
    double vv[E];
#pragma unroll
    for (int e = 0; e < E; e++) vv[e] = UNI ? sfv[fsw(lane * E + e)] : v[lane * E + e];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int j = lane * E + e;
      fa[e] = (j == N - 1) ? 0. : -vv[e];
      fb[e] = (j == N - 1) ? 0. : q[e];
    }
#pragma unroll
    for (int d = 1; d < E; d <<= 1) {
#pragma unroll
      for (int e = 0; e + d < E; e++) {
        fb[e] = fa[e] * fb[e + d] + fb[e];
        fa[e] = fa[e] * fa[e + d];
      }
    }
    PAff bac{fa[0], fb[0]};
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double oa = __shfl_down_sync(0xffffffffu, bac.a, off);
      const double ob = __shfl_down_sync(0xffffffffu, bac.b, off);
      if (lane + off < 32) { bac.b = bac.a * ob + bac.b; bac.a = bac.a * oa; }
    }
    double xin = __shfl_down_sync(0xffffffffu, bac.b, 1);
    if (lane == 31) xin = 0.;
#pragma unroll
    for (int e = 0; e < E; e++) q[e] = fa[e] * xin + fb[e];
    // Sherman-Morrison: the last unknown, then the correction of rows 0 .. N-2
    const double x0 = __shfl_sync(0xffffffffu, q[0], 0);
    const double xn2 = __shfl_sync(0xffffffffu, q[E - 2], 31);
    const double num = qlast - u * x0 - l * xn2;
    const double den = c + u * (UNI ? sfq[fsw(0)] : q1[0]) + l * (UNI ? sfq[fsw(N - 2)] : q1[N - 2]);
    const double last = fabs(den) < 2.220446049250313e-16 ? 0. : num / den;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int j = lane * E + e;
      const double x = (j == N - 1) ? last : q[e] + last * (UNI ? sfq[fsw(j)] : q1[j]);
      sq[j * PT + sw] = x;
    }
  }
  __syncthreads();
#pragma unroll 8
  for (int r = 0; r < PER; r++) {
    const int q = threadIdx.x + r * NT, t = q % PT, j = q / PT;
    if (t < nt) base[(long long)j * elem_stride + t] = sq[j * PT + (t ^ ((j / E) & (PT - 1)))];
  }
}

// lines of n points through the warp kernel when n = 32 E, E in {2, 4, 8, 16};
// false: not handled
static bool launch_periodic_lines(int n, int n_i, long long nouter, long long outer_stride, long long elem_stride,
                                  const double * fl, const double * fc, const double * fu, int lcu_stride,
                                  const double * fw, const double * fv, const double * fq1, int fac_stride,
                                  double * delta, cudaStream_t st) {
  const long long nblk = (long long)((n_i + PT - 1) / PT) * nouter;
  const bool uni = fac_stride == 0;
  const size_t smem = (size_t)n * (PT + (uni ? 3 : 0)) * sizeof(double);
#define PLK(EE)                                                                                              \
  case 32 * EE:                                                                                              \
    if (uni)                                                                                                 \
      periodic_lines_kernel<EE, true><<<(unsigned)nblk, TC_PLINES_THREADS, smem, st>>>(                      \
          n_i, outer_stride, elem_stride, fl, fc, fu, lcu_stride, fw, fv, fq1, fac_stride, delta);           \
    else                                                                                                     \
      periodic_lines_kernel<EE, false><<<(unsigned)nblk, TC_PLINES_THREADS, smem, st>>>(                     \
          n_i, outer_stride, elem_stride, fl, fc, fu, lcu_stride, fw, fv, fq1, fac_stride, delta);           \
    return true;
  switch (n) {
    PLK(2)
    PLK(4)
    PLK(8)
    PLK(16)
    default:
      return false;
  }
#undef PLK
}

void allow_periodic_lines_smem() {
  cudaFuncSetAttribute(periodic_lines_kernel<16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 512 * PT * 8);
  cudaFuncSetAttribute(periodic_lines_kernel<16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 512 * (PT + 3) * 8);
  cudaFuncSetAttribute(periodic_lines_kernel<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 256 * PT * 8);
  cudaFuncSetAttribute(periodic_lines_kernel<8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 256 * (PT + 3) * 8);
  cudaFuncSetAttribute(periodic_lines_kernel<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * PT * 8);
  cudaFuncSetAttribute(periodic_lines_kernel<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * (PT + 3) * 8);
  cudaFuncSetAttribute(periodic_lines_kernel<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * PT * 8);
  cudaFuncSetAttribute(periodic_lines_kernel<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * (PT + 3) * 8);
}

// ------------------------------------------------------------ periodic factors
// Factors of the reduced (n-1) systems of the periodic solves (src/tdm.c:78-87):
// one thread per (substep, variable, radial index) for y, per (substep,
// variable) for z. Doubled prefactor: uy-y and t-y (uy.c:541, t.c:348), uz-z
// (uz.c:451).
__device__ inline void periodic_factors(int n, double l, double c, double u,
                                        double * v, double * w, double * q1) {
  const int m = n - 1;
  v[0] = u / c;
  w[0] = c;
  for (int e = 1; e < m; e++) {
    const double val = 1. / (c - l * v[e - 1]);
    w[e] = val;
    v[e] = (e < m - 1) ? val * u : 0.;
  }
  for (int e = 0; e < m; e++) q1[e] = (e == 0) ? -l : (e == m - 1) ? -u : 0.;
  q1[0] = q1[0] / c;
  for (int e = 1; e < m; e++) q1[e] = w[e] * (q1[e] - l * q1[e - 1]);
  for (int e = m - 2; e >= 0; e--) q1[e] -= v[e] * q1[e + 1];
}

__global__ void yzfactor_kernel(Geo g, YZFactors yf, const double * __restrict__ dtp, double nu, double kappa) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const double dt = *dtp;
  const int total_y = 12 * yf.max_i;
  if (tid < total_y) {
    const int rv = tid / yf.max_i, ii = tid % yf.max_i;
    const int rk = rv / 4, var = rv % 4;
    if (ii >= yf.n_i[var] || (yf.uniform_y && ii > 0)) return;
    const double diff = var == VT ? kappa : nu;
    double pf = 0.5 * rk_gamma(rk) * dt * diff;
    if (var == VUY || var == VT) pf = 2. * pf;
    const double l = -pf * yf.lapy_l[var][ii];
    const double c = 1. - pf * yf.lapy_c[var][ii];
    const double u = -pf * yf.lapy_u[var][ii];
    yf.l[rv * yf.max_i + ii] = l;
    yf.c[rv * yf.max_i + ii] = c;
    yf.u[rv * yf.max_i + ii] = u;
    const size_t o = (size_t)rv * yf.stride_y + (size_t)ii * g.ny;
    periodic_factors(g.ny, l, c, u, yf.v + o, yf.w + o, yf.q1 + o);
  } else if (tid < total_y + 12) {
    const int rv = tid - total_y;
    const int rk = rv / 4, var = rv % 4;
    const double diff = var == VT ? kappa : nu;
    double pf = 0.5 * rk_gamma(rk) * dt * diff;
    if (var == VUZ) pf = 2. * pf;
    const double l = -pf * yf.lapz_l;
    const double c = 1. - pf * yf.lapz_c;
    const double u = -pf * yf.lapz_u;
    yf.lz[rv] = l;
    yf.cz[rv] = c;
    yf.uz[rv] = u;
    const size_t o = (size_t)rv * yf.stride_z;
    periodic_factors(g.nz, l, c, u, yf.vz + o, yf.wz + o, yf.q1z + o);
  }
}

void launch_yzfactors(const Geo & g, const YZFactors & yf, const double * dtp, double nu, double kappa, cudaStream_t st) {
  const int total = 12 * yf.max_i + 12;
  yzfactor_kernel<<<(total + 127) / 128, 128, 0, st>>>(g, yf, dtp, nu, kappa);
}

// ------------------------------------------------------------ launchers
int predict_warps(int nx) {
  int w = 1;
  while (32 * w < nx) w *= 2;
  return w;
}

void launch_xfactors(const XFactors & xf, const double * dtp, double nu, double kappa, cudaStream_t st) {
  xfactor_kernel<<<1, 32, 0, st>>>(xf, dtp, nu, kappa);
}

void launch_apply(const Geo & g, const Bc & bc, const FieldBufs & in, const FieldBufs & out, const DeltaSet & ds,
                  cudaStream_t st) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
  if (in.bytes == 4) apply_kernel<float><<<grid, block, 0, st>>>(g, bc, in.as<float>(), out.as<float>(), ds);
  else apply_kernel<double><<<grid, block, 0, st>>>(g, bc, in.as<double>(), out.as<double>(), ds);
}

void launch_ysolve(const Geo & g, const YZFactors & yf, int rkstep, const DeltaSet & ds, cudaStream_t st) {
  for (int v = 0; v < 4; v++) {
    const int n_i = yf.n_i[v], rv = rkstep * 4 + v;
    const size_t so = (size_t)rv * yf.stride_y;
    const int us = yf.uniform_y ? 0 : 1;   // uniform: every line uses the factors of i = 0
    if (launch_periodic_lines(g.ny, n_i, g.nz, (long long)n_i * g.ny, n_i, yf.l + rv * yf.max_i,
                              yf.c + rv * yf.max_i, yf.u + rv * yf.max_i, us, yf.w + so, yf.v + so, yf.q1 + so,
                              us * g.ny, ds.d[v], st))
      continue;
    const long long n = (long long)n_i * g.nz;
    ysolve_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(g, yf, rkstep, v, ds.d[v]);
  }
}

void launch_zsolve(const Geo & g, const YZFactors & yf, int rkstep, const DeltaSet & ds, cudaStream_t st) {
  for (int v = 0; v < 4; v++) {
    const int n_i = yf.n_i[v], rv = rkstep * 4 + v;
    const size_t so = (size_t)rv * yf.stride_z;
    if (launch_periodic_lines(g.nz, n_i, g.ny, n_i, (long long)n_i * g.ny, yf.lz + rv, yf.cz + rv, yf.uz + rv, 0,
                              yf.wz + so, yf.vz + so, yf.q1z + so, 0, ds.d[v], st))
      continue;
    const long long n = (long long)n_i * g.ny;
    zsolve_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(g, yf, rkstep, v, ds.d[v]);
  }
}

}  // namespace tcgpu
