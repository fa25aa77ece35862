// Predict stage: fluid_predict_field (src/fluid/predict/main.c:35-110).
//
// rhs_delta_kernel  one thread per cell (i, j, k) computes the right-hand sides
//                   of ux (face i), uy, uz and t (centre i) in registers, the
//                   velocity-gradient tensors they need included, and writes the
//                   new explicit source term and the RK increment
//                   delta = dt (alpha srcA + beta srcA_prev + gamma srcG).
//                   srcG (implicit diffusion + pressure gradient) never leaves
//                   registers.
// xfactor_kernel    line-independent Thomas factors of the radial implicit
//                   systems (I - k L_x) for the three substeps, from dt on the device.
// xsolve_kernel     one warp per radial line: the Thomas recurrences of
//                   src/tdm.c:17-50 evaluated as warp-wide scans of affine maps,
//                   then u += delta with the wall values and periodic images
//                   (boundary/*.c, halo.c) written in the same pass.
// ysolve/zsolve     periodic (Sherman-Morrison, src/tdm.c:66-106) solves in y
//                   and z for the planar configuration, one thread per line.
#include "tc_common.cuh"
#include "tc_kernels.h"

namespace tcgpu {

#define LD(p) __ldg(p)

// ------------------------------------------------------------ rhs + delta
__global__ void __launch_bounds__(256)
rhs_delta_kernel(Geo g, Bc bc, Coefs cf, double nu, double kappa,
                 const double * __restrict__ ux, const double * __restrict__ uy,
                 const double * __restrict__ uz, const double * __restrict__ p,
                 const double * __restrict__ t,
                 const double * __restrict__ s_old0, const double * __restrict__ s_old1,
                 const double * __restrict__ s_old2, const double * __restrict__ s_old3,
                 double * __restrict__ s_new0, double * __restrict__ s_new1,
                 double * __restrict__ s_new2, double * __restrict__ s_new3,
                 double * __restrict__ d0, double * __restrict__ d1,
                 double * __restrict__ d2, double * __restrict__ d3,
                 const double * __restrict__ dtp, int rkstep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > g.nx || j > g.ny) return;
  const int nx = g.nx;
  const double dt = *dtp;
  const double ca = rk_alpha(rkstep) * dt;
  const double cb = rk_beta(rkstep) * dt;
  const double cg = rk_gamma(rkstep) * dt;
  const bool use_old = rkstep != 0;
  const bool ix = bc.implicit[0], iy = bc.implicit[1], iz = bc.implicit[2];

#define UXv(I, J, K) LD(ux + fidx(g, (I), (J), (K)))
#define UYv(I, J, K) LD(uy + cidx(g, (I), (J), (K)))
#define UZv(I, J, K) LD(uz + cidx(g, (I), (J), (K)))
#define Pv(I, J, K)  LD(p + cidx(g, (I), (J), (K)))
#define Tv(I, J, K)  LD(t + cidx(g, (I), (J), (K)))
#define CF(name, I) LD(cf.name + (I))

  // ---------------------------------------------------------------- ux at face i
  if (i >= 2) {
    double e = 0., gi = 0.;
    const double ux_m = UXv(i - 1, j, k), ux_0 = UXv(i, j, k), ux_p = UXv(i + 1, j, k);
    const double invj = CF(f_invjd, i);
    {  // advection_x, predict/ux.c:92-121
      const double a1 = CF(f_a1, i), a2 = CF(f_a2, i), a3 = CF(f_a3, i);
      const double ux_xm = a1 * ux_m + a2 * ux_0;
      const double ux_xp = a2 * ux_0 + a3 * ux_p;
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, c = -l - u;
      e -= invj * (l * ux_m + c * ux_0 + u * ux_p);
    }
    const double uy_m0 = UYv(i - 1, j, k), uy_00 = UYv(i, j, k);
    const double uy_m1 = UYv(i - 1, j + 1, k), uy_01 = UYv(i, j + 1, k);
    const double ux_jm = UXv(i, j - 1, k), ux_jp = UXv(i, j + 1, k);
    {  // advection_y :123-155
      const double b1 = CF(f_b1, i), b2 = CF(f_b2, i);
      const double uy_ym = b1 * uy_m0 + b2 * uy_00;
      const double uy_yp = b1 * uy_m1 + b2 * uy_01;
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, c = -l - u;
      e -= invj * (l * ux_jm + c * ux_0 + u * ux_jp);
    }
    const double uz_m0 = UZv(i - 1, j, k), uz_00 = UZv(i, j, k);
    const double uz_m1 = UZv(i - 1, j, k + 1), uz_01 = UZv(i, j, k + 1);
    const double ux_km = UXv(i, j, k - 1), ux_kp = UXv(i, j, k + 1);
    {  // advection_z :157-186
      const double c1 = CF(f_c1, i), c2 = CF(f_c2, i);
      const double uz_zm = c1 * uz_m0 + c2 * uz_00;
      const double uz_zp = c1 * uz_m1 + c2 * uz_01;
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, c = -l - u;
      e -= invj * (l * ux_km + c * ux_0 + u * ux_kp);
    }
    {  // advection_1 (centrifugal) :194-226
      const double uy_xm = 0.5 * uy_m0 + 0.5 * uy_m1;
      const double uy_xp = 0.5 * uy_00 + 0.5 * uy_01;
      e += invj * (CF(f_hd1, i) * uy_xm * uy_xm + CF(f_hd2, i) * uy_xp * uy_xp);
    }
    {  // diffusion_x :228-245
      const double v = 2. * nu * (CF(f_lxl, i) * ux_m + CF(f_lxc, i) * ux_0 + CF(f_lxu, i) * ux_p);
      if (ix) gi += v; else e += v;
    }
    {  // diffusion_y0 :247-264
      const double v = nu * (CF(f_lyl, i) * ux_jm + CF(f_lyc, i) * ux_0 + CF(f_lyu, i) * ux_jp);
      if (iy) gi += v; else e += v;
    }
    const double njd = nu * invj;
    {  // diffusion_y1 :266-290, with lyx1 (lyx.c:64-83) and lxy (lxy.c:28-34)
      const double F = CF(c_lyx1f, i), wm = CF(c_wm, i), wp = CF(c_wp, i), ih = CF(c_invhxxf, i);
      const double lyx1_m = F * (wm * uy_m0 + wp * uy_00);
      const double lyx1_p = F * (wm * uy_m1 + wp * uy_01);
      const double lxy_m = ih * (-uy_m0 + uy_00);
      const double lxy_p = ih * (-uy_m1 + uy_01);
      const double jh = CF(f_e1, i);
      e += njd * (-jh * (lyx1_m + lxy_m) + jh * (lyx1_p + lxy_p));
    }
    {  // diffusion_z0 :292-309
      const double v = nu * (cf.lz_l * ux_km + cf.lz_c * ux_0 + cf.lz_u * ux_kp);
      if (iz) gi += v; else e += v;
    }
    {  // diffusion_z1 :311-332, lxz (lxz.c:19-27)
      const double ih = CF(c_invhxxf, i), jh = CF(f_e2, i);
      const double lxz_m = ih * (-uz_m0 + uz_00);
      const double lxz_p = ih * (-uz_m1 + uz_01);
      e += njd * (-jh * lxz_m + jh * lxz_p);
    }
    {  // diffusion_a :344-375, lyy0/lyy1 (lyy.c) at centres i-1 and i
      const double lyy_xm = CF(c_invhyxc, i - 1) * (-uy_m0 + uy_m1) + CF(c_lyy1, i - 1) * (0.5 * ux_m + 0.5 * ux_0);
      const double lyy_xp = CF(c_invhyxc, i) * (-uy_00 + uy_01) + CF(c_lyy1, i) * (0.5 * ux_0 + 0.5 * ux_p);
      e -= 2. * njd * (CF(f_hd1, i) * lyy_xm + CF(f_hd2, i) * lyy_xp);
    }
    // pressure :377-394
    gi -= CF(c_invhxxf, i) * (-Pv(i - 1, j, k) + Pv(i, j, k));
    const size_t q = pidx(nx - 1, g.ny, i - 2, j, k);
    const double old = use_old ? s_old0[q] : 0.;
    s_new0[q] = e;
    d0[q] = ca * e + cb * old + cg * gi;
  }

  // ---------------------------------------------------------------- uy at centre i
  const double uy_0 = UYv(i, j, k);
  const double uy_im = UYv(i - 1, j, k), uy_ip = UYv(i + 1, j, k);
  const double uy_jm = UYv(i, j - 1, k), uy_jp = UYv(i, j + 1, k);
  const double uy_km = UYv(i, j, k - 1), uy_kp = UYv(i, j, k + 1);
  const double ux_0 = UXv(i, j, k), ux_1 = UXv(i + 1, j, k);          // faces i, i+1 at j
  const double ux_0m = UXv(i, j - 1, k), ux_1m = UXv(i + 1, j - 1, k); // at j-1
  const double ux_0k = UXv(i, j, k - 1), ux_1k = UXv(i + 1, j, k - 1); // at k-1
  const double uz_0 = UZv(i, j, k), uz_kp = UZv(i, j, k + 1);
  const double uz_jm = UZv(i, j - 1, k), uz_jmkp = UZv(i, j - 1, k + 1);
  const double invjc = CF(c_invjdxc, i);
  const double njc = nu * invjc;
  {
    double e = 0., gi = 0.;
    const double a1 = CF(c_a1, i), a2 = CF(c_a2, i);
    {  // advection_x, predict/uy.c:93-123
      const double ux_xm = a1 * ux_0m + a1 * ux_0;
      const double ux_xp = a2 * ux_1m + a2 * ux_1;
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, c = -l - u;
      e -= invjc * (l * uy_im + c * uy_0 + u * uy_ip);
    }
    const double b = CF(c_b, i);
    {  // advection_y :125-151
      const double uy_ym = b * uy_jm + b * uy_0;
      const double uy_yp = b * uy_0 + b * uy_jp;
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, c = -l - u;
      e -= invjc * (l * uy_jm + c * uy_0 + u * uy_jp);
    }
    const double cz = CF(c_cz, i);
    {  // advection_z :153-180
      const double uz_zm = cz * uz_jm + cz * uz_0;
      const double uz_zp = cz * uz_jmkp + cz * uz_kp;
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, c = -l - u;
      e -= invjc * (l * uy_km + c * uy_0 + u * uy_kp);
    }
    {  // advection_1 :188-223
      const double uy_ym = 0.5 * uy_jm + 0.5 * uy_0;
      const double uy_yp = 0.5 * uy_0 + 0.5 * uy_jp;
      const double ux_ym = 0.5 * ux_0m + 0.5 * ux_1m;
      const double ux_yp = 0.5 * ux_0 + 0.5 * ux_1;
      const double hd = CF(c_hd, i);
      e -= invjc * (hd * uy_ym * ux_ym + hd * uy_yp * ux_yp);
    }
    {  // diffusion_x0
      const double v = nu * (CF(c_lxl, i) * uy_im + CF(c_lxc, i) * uy_0 + CF(c_lxu, i) * uy_ip);
      if (ix) gi += v; else e += v;
    }
    // lyx0 (lyx.c:33-39), lyx1 (:64-83), lxy (lxy.c) at faces i and i+1
    const double lyx0_m = CF(c_invhyxf, i) * (-ux_0m + ux_0);
    const double lyx0_p = CF(c_invhyxf, i + 1) * (-ux_1m + ux_1);
    const double lyx1_m = CF(c_lyx1f, i) * (CF(c_wm, i) * uy_im + CF(c_wp, i) * uy_0);
    const double lyx1_p = CF(c_lyx1f, i + 1) * (CF(c_wm, i + 1) * uy_0 + CF(c_wp, i + 1) * uy_ip);
    const double lyx_xm = lyx0_m + lyx1_m;
    const double lyx_xp = lyx0_p + lyx1_p;
    const double jfm = CF(c_jf, i), jfp = CF(c_jf, i + 1);
    // diffusion_x1
    e += njc * (-jfm * lyx_xm + jfp * lyx_xp);
    {  // diffusion_y0
      const double v = 2. * nu * (CF(c_lyl, i) * uy_jm + CF(c_lyc, i) * uy_0 + CF(c_lyu, i) * uy_jp);
      if (iy) gi += v; else e += v;
    }
    {  // diffusion_y1, lyy1 (lyy.c:64-83) at j-1 and j
      const double K = CF(c_lyy1, i);
      const double lyy1_m = K * (0.5 * ux_0m + 0.5 * ux_1m);
      const double lyy1_0 = K * (0.5 * ux_0 + 0.5 * ux_1);
      const double jh = CF(c_e1, i);
      e += 2. * njc * (-jh * lyy1_m + jh * lyy1_0);
    }
    {  // diffusion_z0
      const double v = nu * (cf.lz_l * uy_km + cf.lz_c * uy_0 + cf.lz_u * uy_kp);
      if (iz) gi += v; else e += v;
    }
    {  // diffusion_z1, lyz (lyz.c:19-27) at k and k+1
      const double ih = CF(c_invhyxc, i);
      const double lyz_0 = ih * (-uz_jm + uz_0);
      const double lyz_p = ih * (-uz_jmkp + uz_kp);
      const double jh = CF(c_e2, i);
      e += njc * (-jh * lyz_0 + jh * lyz_p);
    }
    {  // diffusion_a :367-400
      const double lxy_m = CF(c_invhxxf, i) * (-uy_im + uy_0);
      const double lxy_p = CF(c_invhxxf, i + 1) * (-uy_0 + uy_ip);
      e += njc * (CF(c_hda1, i) * (lyx_xm + lxy_m) + CF(c_hda2, i) * (lyx_xp + lxy_p));
    }
    gi -= CF(c_invhyxc, i) * (-Pv(i, j - 1, k) + Pv(i, j, k));
    const size_t q = pidx(nx, g.ny, i - 1, j, k);
    const double old = use_old ? s_old1[q] : 0.;
    s_new1[q] = e;
    d1[q] = ca * e + cb * old + cg * gi;
  }

  // ---------------------------------------------------------------- uz at centre i
  {
    double e = 0., gi = 0.;
    const double uz_im = UZv(i - 1, j, k), uz_ip = UZv(i + 1, j, k);
    const double uz_jp = UZv(i, j + 1, k), uz_km = UZv(i, j, k - 1);
    const double uy_jpkm = UYv(i, j + 1, k - 1);
    {  // advection_x, predict/uz.c:88-118
      const double a1 = CF(c_a1, i), a2 = CF(c_a2, i);
      const double ux_xm = a1 * ux_0k + a1 * ux_0;
      const double ux_xp = a2 * ux_1k + a2 * ux_1;
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, c = -l - u;
      e -= invjc * (l * uz_im + c * uz_0 + u * uz_ip);
    }
    {  // advection_y
      const double b = CF(c_b, i);
      const double uy_ym = b * uy_km + b * uy_0;
      const double uy_yp = b * uy_jpkm + b * uy_jp;
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, c = -l - u;
      e -= invjc * (l * uz_jm + c * uz_0 + u * uz_jp);
    }
    {  // advection_z
      const double cz = CF(c_cz, i);
      const double uz_zm = cz * uz_km + cz * uz_0;
      const double uz_zp = cz * uz_0 + cz * uz_kp;
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, c = -l - u;
      e -= invjc * (l * uz_km + c * uz_0 + u * uz_kp);
    }
    {  // diffusion_x0
      const double v = nu * (CF(c_lxl, i) * uz_im + CF(c_lxc, i) * uz_0 + CF(c_lxu, i) * uz_ip);
      if (ix) gi += v; else e += v;
    }
    {  // diffusion_x1, lzx (lzx.c) at faces i, i+1
      const double ihz = cf.inv_hz;
      const double lzx_m = ihz * (-ux_0k + ux_0);
      const double lzx_p = ihz * (-ux_1k + ux_1);
      e += njc * (-CF(c_jf, i) * lzx_m + CF(c_jf, i + 1) * lzx_p);
    }
    {  // diffusion_y0
      const double v = nu * (CF(c_lyl, i) * uz_jm + CF(c_lyc, i) * uz_0 + CF(c_lyu, i) * uz_jp);
      if (iy) gi += v; else e += v;
    }
    {  // diffusion_y1, lzy (lzy.c) at j, j+1
      const double ihz = cf.inv_hz;
      const double lzy_0 = ihz * (-uy_km + uy_0);
      const double lzy_p = ihz * (-uy_jpkm + uy_jp);
      const double jh = CF(c_e1, i);
      e += njc * (-jh * lzy_0 + jh * lzy_p);
    }
    {  // diffusion_z
      const double v = 2. * nu * (cf.lz_l * uz_km + cf.lz_c * uz_0 + cf.lz_u * uz_kp);
      if (iz) gi += v; else e += v;
    }
    gi -= cf.inv_hz * (-Pv(i, j, k - 1) + Pv(i, j, k));
    const size_t q = pidx(nx, g.ny, i - 1, j, k);
    const double old = use_old ? s_old2[q] : 0.;
    s_new2[q] = e;
    d2[q] = ca * e + cb * old + cg * gi;
  }

  // ---------------------------------------------------------------- t at centre i
  {
    double e = 0., gi = 0.;
    const double t0 = Tv(i, j, k);
    const double tim = Tv(i - 1, j, k), tip = Tv(i + 1, j, k);
    const double tjm = Tv(i, j - 1, k), tjp = Tv(i, j + 1, k);
    const double tkm = Tv(i, j, k - 1), tkp = Tv(i, j, k + 1);
    {  // advection_x, predict/t.c:88-116
      const double ux_xm = CF(c_jf, i) * ux_0;
      const double ux_xp = CF(c_jf, i + 1) * ux_1;
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, c = -l - u;
      e -= invjc * (l * tim + c * t0 + u * tip);
    }
    {  // advection_y
      const double jh = CF(c_e1, i);
      const double uy_ym = jh * uy_0;
      const double uy_yp = jh * uy_jp;
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, c = -l - u;
      e -= invjc * (l * tjm + c * t0 + u * tjp);
    }
    {  // advection_z
      const double jh = CF(c_e2, i);
      const double uz_zm = jh * uz_0;
      const double uz_zp = jh * uz_kp;
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, c = -l - u;
      e -= invjc * (l * tkm + c * t0 + u * tkp);
    }
    {
      const double v = kappa * (CF(c_lxl, i) * tim + CF(c_lxc, i) * t0 + CF(c_lxu, i) * tip);
      if (ix) gi += v; else e += v;
    }
    {
      const double v = kappa * (CF(c_lyl, i) * tjm + CF(c_lyc, i) * t0 + CF(c_lyu, i) * tjp);
      if (iy) gi += v; else e += v;
    }
    {
      const double v = kappa * (cf.lz_l * tkm + cf.lz_c * t0 + cf.lz_u * tkp);
      if (iz) gi += v; else e += v;
    }
    const size_t q = pidx(nx, g.ny, i - 1, j, k);
    const double old = use_old ? s_old3[q] : 0.;
    s_new3[q] = e;
    d3[q] = ca * e + cb * old + cg * gi;
  }
#undef UXv
#undef UYv
#undef UZv
#undef Pv
#undef Tv
#undef CF
}

// ------------------------------------------------------------ Thomas factors
// One thread per (substep, variable, direction): the forward-elimination
// factors of gtsv (src/tdm.c:24-44) for (I - pf L) with
//   l = -pf lap.l, c = 1 - pf lap.c, u = -pf lap.u   (predict/linear_system.c:26-33)
// pf = 0.5 gamma dt diffusivity, doubled for the "diagonal" component
// (ux-x ux.c:502, uy-y uy.c:541, uz-z uz.c:451, t-y t.c:348).
// Output per line family: lo[n] = l, w[n] (w[0] = c[0], w[i] = 1/(c - l v)),
// v[n] (v[n-1] = 0).
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
  double vprev = 0.;
  for (int e = 0; e < n; e++) {
    const double l = -pf * ll[e];
    const double c = 1. - pf * lc[e];
    const double u = -pf * lu[e];
    lo[e] = l;
    if (e == 0) {
      w[0] = c;
      vprev = u / c;
      v[0] = (n > 1) ? vprev : 0.;
    } else if (e < n - 1) {
      const double val = 1. / (c - l * vprev);
      w[e] = val;
      vprev = val * u;
      v[e] = vprev;
    } else {
      w[e] = 1. / (c - l * vprev);
      v[e] = 0.;
    }
  }
}

// ------------------------------------------------------------ radial solve + update
// Affine map composition q -> A q + B. compose(first, then).
struct Aff { double a, b; };

__device__ inline void shfl_up_aff(Aff & x, int off) {
  x.a = __shfl_up_sync(0xffffffffu, x.a, off);
  x.b = __shfl_up_sync(0xffffffffu, x.b, off);
}
__device__ inline void shfl_down_aff(Aff & x, int off) {
  x.a = __shfl_down_sync(0xffffffffu, x.a, off);
  x.b = __shfl_down_sync(0xffffffffu, x.b, off);
}

template <int E>
__device__ inline int spad(int e) { return E > 1 ? e + e / E : e; }

// One warp per (line, variable). Lines: (j, k) interior; var picks the field.
// With SOLVE the radial Thomas system is solved first (implicit x). With APPLY
// the increment is then added and the row's walls and periodic images written;
// without it the solved increment goes back to the delta buffer (for the y/z
// solves that follow in the planar configuration, linear_system.c order).
template <int E, bool SOLVE, bool APPLY>
__global__ void __launch_bounds__(256)
xsolve_kernel(Geo g, Bc bc, XFactors xf, int rkstep, int var_lo,
              double * __restrict__ ux, double * __restrict__ uy,
              double * __restrict__ uz, double * __restrict__ t,
              const double * __restrict__ d0, const double * __restrict__ d1,
              const double * __restrict__ d2, const double * __restrict__ d3) {
  constexpr int WARPS = 8;
  constexpr int SLEN = 32 * E + (E > 1 ? 32 : 0);
  __shared__ double sbuf[WARPS][SLEN];
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  const long long line = (long long)blockIdx.x * WARPS + wid;
  const int ny = g.ny, nz = g.nz, nx = g.nx;
  const long long nlines = (long long)ny * nz;
  const int var = var_lo + blockIdx.y;
  if (line >= nlines) return;
  const int j = (int)(line % ny) + 1;
  const int k = (int)(line / ny) + 1;
  const int n = xf.n[var];
  double * dsrc = const_cast<double *>(var == VUX ? d0 : var == VUY ? d1 : var == VUZ ? d2 : d3);
  double * drow = dsrc + (size_t)n * ((size_t)(j - 1) + (size_t)ny * (size_t)(k - 1));
  double * sb = sbuf[wid];
  for (int r = 0; r < E; r++) {
    const int e = lane + 32 * r;
    if (e < n) sb[spad<E>(e)] = drow[e];
  }
  __syncwarp();
  if (SOLVE) {
    const size_t fo = (size_t)(rkstep * 4 + var) * xf.stride;
    const double * lo = xf.lo + fo;
    const double * w = xf.w + fo;
    const double * v = xf.v + fo;
    double q[E];
#pragma unroll
    for (int m = 0; m < E; m++) {
      const int e = lane * E + m;
      q[m] = (e < n) ? sb[spad<E>(e)] : 0.;
    }
    // forward: q_0 = r_0 / c_0; q_e = w_e (r_e - l_e q_{e-1})
    Aff acc{1., 0.};
#pragma unroll
    for (int m = 0; m < E; m++) {
      const int e = lane * E + m;
      Aff f;
      if (e == 0) { f.a = 0.; f.b = q[m] / LD(w); }
      else if (e < n) { const double we = LD(w + e); f.a = -we * LD(lo + e); f.b = we * q[m]; }
      else { f.a = 0.; f.b = 0.; }
      acc.b = f.a * acc.b + f.b;
      acc.a = f.a * acc.a;
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      Aff o = acc;
      shfl_up_aff(o, off);
      if (lane >= off) { acc.b = acc.a * o.b + acc.b; acc.a = acc.a * o.a; }
    }
    double qin = __shfl_up_sync(0xffffffffu, acc.b, 1);
    if (lane == 0) qin = 0.;
#pragma unroll
    for (int m = 0; m < E; m++) {
      const int e = lane * E + m;
      double r;
      if (e == 0) r = q[m] / LD(w);
      else if (e < n) r = LD(w + e) * (q[m] - LD(lo + e) * qin);
      else r = 0.;
      q[m] = r;
      qin = r;
    }
    // backward: x_e = q_e - v_e x_{e+1}
    Aff bac{1., 0.};
#pragma unroll
    for (int m = E - 1; m >= 0; m--) {
      const int e = lane * E + m;
      Aff f;
      if (e < n) { f.a = -LD(v + e); f.b = q[m]; } else { f.a = 0.; f.b = 0.; }
      bac.b = f.a * bac.b + f.b;
      bac.a = f.a * bac.a;
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      Aff o = bac;
      shfl_down_aff(o, off);
      if (lane + off < 32) { bac.b = bac.a * o.b + bac.b; bac.a = bac.a * o.a; }
    }
    double xin = __shfl_down_sync(0xffffffffu, bac.b, 1);
    if (lane == 31) xin = 0.;
#pragma unroll
    for (int m = E - 1; m >= 0; m--) {
      const int e = lane * E + m;
      double x = 0.;
      if (e < n) x = q[m] - LD(v + e) * xin;
      q[m] = x;
      xin = x;
    }
    __syncwarp();
#pragma unroll
    for (int m = 0; m < E; m++) {
      const int e = lane * E + m;
      if (e < n) sb[spad<E>(e)] = q[m];
    }
    __syncwarp();
  }
  if (!APPLY) {
    for (int r = 0; r < E; r++) {
      const int e = lane + 32 * r;
      if (e < n) drow[e] = sb[spad<E>(e)];
    }
    return;
  }
  // u += delta over the row, walls, periodic images
  if (var == VUX) {
    double * row = ux + fidx(g, 1, j, k);
    for (int r = 0; r < E + 1; r++) {
      const int e = lane + 32 * r;          // e -> i = e + 1, i = 1..nx+1
      if (e > nx) break;
      double val;
      if (e == 0 || e == nx) val = 0.;      // boundary/ux.c:24-26
      else val = row[e] + sb[spad<E>(e - 1)];
      row[e] = val;
      for_images(j, k, ny, nz, [&](int jj, int kk) {
        ux[fidx(g, 1, jj, kk) + e] = val;
      });
    }
  } else {
    double * arr = var == VUY ? uy : var == VUZ ? uz : t;
    const double wm = var == VUY ? bc.uy_xm : var == VUZ ? 0. : bc.t_xm;
    const double wp = var == VUY ? bc.uy_xp : var == VUZ ? 0. : bc.t_xp;
    double * row = arr + cidx(g, 0, j, k);
    for (int r = 0; r < E + 1; r++) {
      const int e = lane + 32 * r;          // e = i, 0..nx+1
      if (e > nx + 1) break;
      double val;
      if (e == 0) val = wm;
      else if (e == nx + 1) val = wp;
      else val = row[e] + sb[spad<E>(e - 1)];
      row[e] = val;
      for_images(j, k, ny, nz, [&](int jj, int kk) {
        arr[cidx(g, 0, jj, kk) + e] = val;
      });
    }
  }
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
  const double * v = yf.v + so + (size_t)ii * n;
  const double * w = yf.w + so + (size_t)ii * n;
  const double * q1 = yf.q1 + so + (size_t)ii * n;
  const double l = yf.l[(rkstep * 4 + var) * yf.max_i + ii];
  const double c = yf.c[(rkstep * 4 + var) * yf.max_i + ii];
  const double u = yf.u[(rkstep * 4 + var) * yf.max_i + ii];
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
    if (ii >= yf.n_i[var]) return;
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
void launch_rhs_delta(const Geo & g, const Bc & bc, const Coefs & cf, double nu, double kappa,
                      const Fields & f, double * const s_old[4], double * const s_new[4],
                      double * const d[4], const double * dtp, int rkstep, cudaStream_t st) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
  rhs_delta_kernel<<<grid, block, 0, st>>>(g, bc, cf, nu, kappa, f.ux, f.uy, f.uz, f.p, f.t,
      s_old[0], s_old[1], s_old[2], s_old[3], s_new[0], s_new[1], s_new[2], s_new[3],
      d[0], d[1], d[2], d[3], dtp, rkstep);
}

void launch_xfactors(const XFactors & xf, const double * dtp, double nu, double kappa, cudaStream_t st) {
  xfactor_kernel<<<1, 32, 0, st>>>(xf, dtp, nu, kappa);
}

template <int E>
static void launch_xsolve_e(const Geo & g, const Bc & bc, const XFactors & xf, int rkstep, int mode,
                            const Fields & f, double * const d[4], cudaStream_t st) {
  const long long nlines = (long long)g.ny * g.nz;
  dim3 grid((unsigned)((nlines + 7) / 8), 4, 1);
  if (mode == XS_SOLVE_APPLY) {
    xsolve_kernel<E, true, true><<<grid, 256, 0, st>>>(g, bc, xf, rkstep, 0, f.ux, f.uy, f.uz, f.t, d[0], d[1], d[2], d[3]);
  } else if (mode == XS_SOLVE) {
    xsolve_kernel<E, true, false><<<grid, 256, 0, st>>>(g, bc, xf, rkstep, 0, f.ux, f.uy, f.uz, f.t, d[0], d[1], d[2], d[3]);
  } else {
    xsolve_kernel<E, false, true><<<grid, 256, 0, st>>>(g, bc, xf, rkstep, 0, f.ux, f.uy, f.uz, f.t, d[0], d[1], d[2], d[3]);
  }
}

int xsolve_elems(int nx) {
  int e = 1;
  while (32 * e < nx) e *= 2;
  return e;
}

void launch_xsolve(const Geo & g, const Bc & bc, const XFactors & xf, int rkstep, int mode,
                   const Fields & f, double * const d[4], cudaStream_t st) {
  switch (xsolve_elems(g.nx)) {
    case 1: launch_xsolve_e<1>(g, bc, xf, rkstep, mode, f, d, st); break;
    case 2: launch_xsolve_e<2>(g, bc, xf, rkstep, mode, f, d, st); break;
    case 4: launch_xsolve_e<4>(g, bc, xf, rkstep, mode, f, d, st); break;
    case 8: launch_xsolve_e<8>(g, bc, xf, rkstep, mode, f, d, st); break;
    default: launch_xsolve_e<16>(g, bc, xf, rkstep, mode, f, d, st); break;
  }
}

void launch_ysolve(const Geo & g, const YZFactors & yf, int rkstep, double * const d[4], cudaStream_t st) {
  for (int v = 0; v < 4; v++) {
    const long long n = (long long)yf.n_i[v] * g.nz;
    ysolve_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(g, yf, rkstep, v, d[v]);
  }
}

void launch_zsolve(const Geo & g, const YZFactors & yf, int rkstep, double * const d[4], cudaStream_t st) {
  for (int v = 0; v < 4; v++) {
    const long long n = (long long)yf.n_i[v] * g.ny;
    zsolve_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(g, yf, rkstep, v, d[v]);
  }
}

}  // namespace tcgpu
