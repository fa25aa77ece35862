// Predict stage: fluid_predict_field (src/fluid/predict/main.c:35-110).
//
// predict_kernel    one CTA row per radial line, one thread per cell: the
//                   right-hand sides of ux (face i), uy, uz and t (centre i) in
//                   registers, velocity-gradient tensors included; the new
//                   explicit source terms; the RK increment
//                   delta = dt (alpha srcA + beta srcA_prev + gamma srcG), srcG
//                   (implicit diffusion + pressure gradient) never leaving
//                   registers; the radial implicit solve (src/tdm.c:17-50) as
//                   block-wide scans of affine maps; u + delta written to the
//                   other buffer with walls and periodic images (boundary/*.c,
//                   halo.c). One pass over the fields per substep.
// xfactor_kernel    line-independent Thomas factors of the radial implicit
//                   systems (I - k L_x) for the three substeps, from dt on the device.
// apply_kernel      u + delta after the y / z solves (planar configuration).
// ysolve/zsolve     periodic (Sherman-Morrison, src/tdm.c:66-106) solves in y
//                   and z for the planar configuration, one thread per line.
#include "tc_common.cuh"
#include "tc_kernels.h"

namespace tcgpu {

#define LD(p) __ldg(p)

// ------------------------------------------------------------ rhs + delta of one cell
// Right-hand sides of ux (face i), uy, uz, t (centre i), the new explicit
// source terms (written to s_new*) and the RK increments dl[0..3]
// (dl[0] is 0 at i = 1, where ux has no unknown). u0 returns the cell's
// current values.
__device__ __forceinline__ void cell_rhs_delta(
    const Geo & g, const Bc & bc, const Coefs & cf, double nu, double kappa,
    const double * __restrict__ ux, const double * __restrict__ uy,
    const double * __restrict__ uz, const double * __restrict__ p,
    const double * __restrict__ t,
    const double * __restrict__ s_old0, const double * __restrict__ s_old1,
    const double * __restrict__ s_old2, const double * __restrict__ s_old3,
    double * __restrict__ s_new0, double * __restrict__ s_new1,
    double * __restrict__ s_new2, double * __restrict__ s_new3,
    int i, int j, int k, double ca, double cb, double cg, bool use_old,
    double dl[4], double u0[4]) {
  const int nx = g.nx;
  const bool ix = bc.implicit[0], iy = bc.implicit[1], iz = bc.implicit[2];
  dl[0] = 0.;
  // neighbours from base pointers: (di, dj, dk) offsets with the row and
  // plane strides of the face (ux) and centre arrays
  const int sjf = nx + 1, skf = (nx + 1) * (g.ny + 2);
  const int sjc = nx + 2, skc = (nx + 2) * (g.ny + 2);
  const double * __restrict__ bx = ux + fidx(g, i, j, k);
  const double * __restrict__ by = uy + cidx(g, i, j, k);
  const double * __restrict__ bz = uz + cidx(g, i, j, k);
  const double * __restrict__ bp = p + cidx(g, i, j, k);
  const double * __restrict__ bt = t + cidx(g, i, j, k);
  const double * __restrict__ bc_ = cf.tab + i;
#define UXv(DI, DJ, DK) LD(bx + ((DI) + (DJ) * sjf + (DK) * skf))
#define UYv(DI, DJ, DK) LD(by + ((DI) + (DJ) * sjc + (DK) * skc))
#define UZv(DI, DJ, DK) LD(bz + ((DI) + (DJ) * sjc + (DK) * skc))
#define Pv(DI, DJ, DK)  LD(bp + ((DI) + (DJ) * sjc + (DK) * skc))
#define Tv(DI, DJ, DK)  LD(bt + ((DI) + (DJ) * sjc + (DK) * skc))
#define CF(T, D) LD(bc_ + ((T) * CSTRIDE + (D)))

  // ---------------------------------------------------------------- ux at face i
  if (i >= 2) {
    double e = 0., gi = 0.;
    const double ux_m = UXv(-1, 0, 0), ux_0 = UXv(0, 0, 0), ux_p = UXv(+1, 0, 0);
    const double invj = CF(F_INVJD, 0);
    {  // advection_x, predict/ux.c:92-121
      const double a1 = CF(F_A1, 0), a2 = CF(F_A2, 0), a3 = CF(F_A3, 0);
      const double ux_xm = a1 * ux_m + a2 * ux_0;
      const double ux_xp = a2 * ux_0 + a3 * ux_p;
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, c = -l - u;
      e -= invj * (l * ux_m + c * ux_0 + u * ux_p);
    }
    const double uy_m0 = UYv(-1, 0, 0), uy_00 = UYv(0, 0, 0);
    const double uy_m1 = UYv(-1, +1, 0), uy_01 = UYv(0, +1, 0);
    const double ux_jm = UXv(0, -1, 0), ux_jp = UXv(0, +1, 0);
    {  // advection_y :123-155
      const double b1 = CF(F_B1, 0), b2 = CF(F_B2, 0);
      const double uy_ym = b1 * uy_m0 + b2 * uy_00;
      const double uy_yp = b1 * uy_m1 + b2 * uy_01;
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, c = -l - u;
      e -= invj * (l * ux_jm + c * ux_0 + u * ux_jp);
    }
    const double uz_m0 = UZv(-1, 0, 0), uz_00 = UZv(0, 0, 0);
    const double uz_m1 = UZv(-1, 0, +1), uz_01 = UZv(0, 0, +1);
    const double ux_km = UXv(0, 0, -1), ux_kp = UXv(0, 0, +1);
    {  // advection_z :157-186
      const double c1 = CF(F_C1, 0), c2 = CF(F_C2, 0);
      const double uz_zm = c1 * uz_m0 + c2 * uz_00;
      const double uz_zp = c1 * uz_m1 + c2 * uz_01;
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, c = -l - u;
      e -= invj * (l * ux_km + c * ux_0 + u * ux_kp);
    }
    {  // advection_1 (centrifugal) :194-226
      const double uy_xm = 0.5 * uy_m0 + 0.5 * uy_m1;
      const double uy_xp = 0.5 * uy_00 + 0.5 * uy_01;
      e += invj * (CF(F_HD1, 0) * uy_xm * uy_xm + CF(F_HD2, 0) * uy_xp * uy_xp);
    }
    {  // diffusion_x :228-245
      const double v = 2. * nu * (CF(F_LXL, 0) * ux_m + CF(F_LXC, 0) * ux_0 + CF(F_LXU, 0) * ux_p);
      if (ix) gi += v; else e += v;
    }
    {  // diffusion_y0 :247-264
      const double v = nu * (CF(F_LYL, 0) * ux_jm + CF(F_LYC, 0) * ux_0 + CF(F_LYU, 0) * ux_jp);
      if (iy) gi += v; else e += v;
    }
    const double njd = nu * invj;
    {  // diffusion_y1 :266-290, with lyx1 (lyx.c:64-83) and lxy (lxy.c:28-34)
      const double F = CF(C_LYX1F, 0), wm = CF(C_WM, 0), wp = CF(C_WP, 0), ih = CF(C_INVHXXF, 0);
      const double lyx1_m = F * (wm * uy_m0 + wp * uy_00);
      const double lyx1_p = F * (wm * uy_m1 + wp * uy_01);
      const double lxy_m = ih * (-uy_m0 + uy_00);
      const double lxy_p = ih * (-uy_m1 + uy_01);
      const double jh = CF(F_E1, 0);
      e += njd * (-jh * (lyx1_m + lxy_m) + jh * (lyx1_p + lxy_p));
    }
    {  // diffusion_z0 :292-309
      const double v = nu * (cf.lz_l * ux_km + cf.lz_c * ux_0 + cf.lz_u * ux_kp);
      if (iz) gi += v; else e += v;
    }
    {  // diffusion_z1 :311-332, lxz (lxz.c:19-27)
      const double ih = CF(C_INVHXXF, 0), jh = CF(F_E2, 0);
      const double lxz_m = ih * (-uz_m0 + uz_00);
      const double lxz_p = ih * (-uz_m1 + uz_01);
      e += njd * (-jh * lxz_m + jh * lxz_p);
    }
    {  // diffusion_a :344-375, lyy0/lyy1 (lyy.c) at centres i-1 and i
      const double lyy_xm = CF(C_INVHYXC, -1) * (-uy_m0 + uy_m1) + CF(C_LYY1, -1) * (0.5 * ux_m + 0.5 * ux_0);
      const double lyy_xp = CF(C_INVHYXC, 0) * (-uy_00 + uy_01) + CF(C_LYY1, 0) * (0.5 * ux_0 + 0.5 * ux_p);
      e -= 2. * njd * (CF(F_HD1, 0) * lyy_xm + CF(F_HD2, 0) * lyy_xp);
    }
    // pressure :377-394
    gi -= CF(C_INVHXXF, 0) * (-Pv(-1, 0, 0) + Pv(0, 0, 0));
    const size_t q = pidx(nx - 1, g.ny, i - 2, j, k);
    const double old = use_old ? s_old0[q] : 0.;
    s_new0[q] = e;
    dl[0] = ca * e + cb * old + cg * gi;
  }

  // ---------------------------------------------------------------- uy at centre i
  const double uy_0 = UYv(0, 0, 0);
  const double uy_im = UYv(-1, 0, 0), uy_ip = UYv(+1, 0, 0);
  const double uy_jm = UYv(0, -1, 0), uy_jp = UYv(0, +1, 0);
  const double uy_km = UYv(0, 0, -1), uy_kp = UYv(0, 0, +1);
  const double ux_0 = UXv(0, 0, 0), ux_1 = UXv(+1, 0, 0);          // faces i, i+1 at j
  const double ux_0m = UXv(0, -1, 0), ux_1m = UXv(+1, -1, 0); // at j-1
  const double ux_0k = UXv(0, 0, -1), ux_1k = UXv(+1, 0, -1); // at k-1
  const double uz_0 = UZv(0, 0, 0), uz_kp = UZv(0, 0, +1);
  const double uz_jm = UZv(0, -1, 0), uz_jmkp = UZv(0, -1, +1);
  const double invjc = CF(C_INVJDXC, 0);
  const double njc = nu * invjc;
  u0[0] = ux_0;
  u0[1] = uy_0;
  u0[2] = uz_0;
  {
    double e = 0., gi = 0.;
    const double a1 = CF(C_A1, 0), a2 = CF(C_A2, 0);
    {  // advection_x, predict/uy.c:93-123
      const double ux_xm = a1 * ux_0m + a1 * ux_0;
      const double ux_xp = a2 * ux_1m + a2 * ux_1;
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, c = -l - u;
      e -= invjc * (l * uy_im + c * uy_0 + u * uy_ip);
    }
    const double b = CF(C_B, 0);
    {  // advection_y :125-151
      const double uy_ym = b * uy_jm + b * uy_0;
      const double uy_yp = b * uy_0 + b * uy_jp;
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, c = -l - u;
      e -= invjc * (l * uy_jm + c * uy_0 + u * uy_jp);
    }
    const double cz = CF(C_CZ, 0);
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
      const double hd = CF(C_HD, 0);
      e -= invjc * (hd * uy_ym * ux_ym + hd * uy_yp * ux_yp);
    }
    {  // diffusion_x0
      const double v = nu * (CF(C_LXL, 0) * uy_im + CF(C_LXC, 0) * uy_0 + CF(C_LXU, 0) * uy_ip);
      if (ix) gi += v; else e += v;
    }
    // lyx0 (lyx.c:33-39), lyx1 (:64-83), lxy (lxy.c) at faces i and i+1
    const double lyx0_m = CF(C_INVHYXF, 0) * (-ux_0m + ux_0);
    const double lyx0_p = CF(C_INVHYXF, +1) * (-ux_1m + ux_1);
    const double lyx1_m = CF(C_LYX1F, 0) * (CF(C_WM, 0) * uy_im + CF(C_WP, 0) * uy_0);
    const double lyx1_p = CF(C_LYX1F, +1) * (CF(C_WM, +1) * uy_0 + CF(C_WP, +1) * uy_ip);
    const double lyx_xm = lyx0_m + lyx1_m;
    const double lyx_xp = lyx0_p + lyx1_p;
    const double jfm = CF(C_JF, 0), jfp = CF(C_JF, +1);
    // diffusion_x1
    e += njc * (-jfm * lyx_xm + jfp * lyx_xp);
    {  // diffusion_y0
      const double v = 2. * nu * (CF(C_LYL, 0) * uy_jm + CF(C_LYC, 0) * uy_0 + CF(C_LYU, 0) * uy_jp);
      if (iy) gi += v; else e += v;
    }
    {  // diffusion_y1, lyy1 (lyy.c:64-83) at j-1 and j
      const double K = CF(C_LYY1, 0);
      const double lyy1_m = K * (0.5 * ux_0m + 0.5 * ux_1m);
      const double lyy1_0 = K * (0.5 * ux_0 + 0.5 * ux_1);
      const double jh = CF(C_E1, 0);
      e += 2. * njc * (-jh * lyy1_m + jh * lyy1_0);
    }
    {  // diffusion_z0
      const double v = nu * (cf.lz_l * uy_km + cf.lz_c * uy_0 + cf.lz_u * uy_kp);
      if (iz) gi += v; else e += v;
    }
    {  // diffusion_z1, lyz (lyz.c:19-27) at k and k+1
      const double ih = CF(C_INVHYXC, 0);
      const double lyz_0 = ih * (-uz_jm + uz_0);
      const double lyz_p = ih * (-uz_jmkp + uz_kp);
      const double jh = CF(C_E2, 0);
      e += njc * (-jh * lyz_0 + jh * lyz_p);
    }
    {  // diffusion_a :367-400
      const double lxy_m = CF(C_INVHXXF, 0) * (-uy_im + uy_0);
      const double lxy_p = CF(C_INVHXXF, +1) * (-uy_0 + uy_ip);
      e += njc * (CF(C_HDA1, 0) * (lyx_xm + lxy_m) + CF(C_HDA2, 0) * (lyx_xp + lxy_p));
    }
    gi -= CF(C_INVHYXC, 0) * (-Pv(0, -1, 0) + Pv(0, 0, 0));
    const size_t q = pidx(nx, g.ny, i - 1, j, k);
    const double old = use_old ? s_old1[q] : 0.;
    s_new1[q] = e;
    dl[1] = ca * e + cb * old + cg * gi;
  }

  // ---------------------------------------------------------------- uz at centre i
  {
    double e = 0., gi = 0.;
    const double uz_im = UZv(-1, 0, 0), uz_ip = UZv(+1, 0, 0);
    const double uz_jp = UZv(0, +1, 0), uz_km = UZv(0, 0, -1);
    const double uy_jpkm = UYv(0, +1, -1);
    {  // advection_x, predict/uz.c:88-118
      const double a1 = CF(C_A1, 0), a2 = CF(C_A2, 0);
      const double ux_xm = a1 * ux_0k + a1 * ux_0;
      const double ux_xp = a2 * ux_1k + a2 * ux_1;
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, c = -l - u;
      e -= invjc * (l * uz_im + c * uz_0 + u * uz_ip);
    }
    {  // advection_y
      const double b = CF(C_B, 0);
      const double uy_ym = b * uy_km + b * uy_0;
      const double uy_yp = b * uy_jpkm + b * uy_jp;
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, c = -l - u;
      e -= invjc * (l * uz_jm + c * uz_0 + u * uz_jp);
    }
    {  // advection_z
      const double cz = CF(C_CZ, 0);
      const double uz_zm = cz * uz_km + cz * uz_0;
      const double uz_zp = cz * uz_0 + cz * uz_kp;
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, c = -l - u;
      e -= invjc * (l * uz_km + c * uz_0 + u * uz_kp);
    }
    {  // diffusion_x0
      const double v = nu * (CF(C_LXL, 0) * uz_im + CF(C_LXC, 0) * uz_0 + CF(C_LXU, 0) * uz_ip);
      if (ix) gi += v; else e += v;
    }
    {  // diffusion_x1, lzx (lzx.c) at faces i, i+1
      const double ihz = cf.inv_hz;
      const double lzx_m = ihz * (-ux_0k + ux_0);
      const double lzx_p = ihz * (-ux_1k + ux_1);
      e += njc * (-CF(C_JF, 0) * lzx_m + CF(C_JF, +1) * lzx_p);
    }
    {  // diffusion_y0
      const double v = nu * (CF(C_LYL, 0) * uz_jm + CF(C_LYC, 0) * uz_0 + CF(C_LYU, 0) * uz_jp);
      if (iy) gi += v; else e += v;
    }
    {  // diffusion_y1, lzy (lzy.c) at j, j+1
      const double ihz = cf.inv_hz;
      const double lzy_0 = ihz * (-uy_km + uy_0);
      const double lzy_p = ihz * (-uy_jpkm + uy_jp);
      const double jh = CF(C_E1, 0);
      e += njc * (-jh * lzy_0 + jh * lzy_p);
    }
    {  // diffusion_z
      const double v = 2. * nu * (cf.lz_l * uz_km + cf.lz_c * uz_0 + cf.lz_u * uz_kp);
      if (iz) gi += v; else e += v;
    }
    gi -= cf.inv_hz * (-Pv(0, 0, -1) + Pv(0, 0, 0));
    const size_t q = pidx(nx, g.ny, i - 1, j, k);
    const double old = use_old ? s_old2[q] : 0.;
    s_new2[q] = e;
    dl[2] = ca * e + cb * old + cg * gi;
  }

  // ---------------------------------------------------------------- t at centre i
  {
    double e = 0., gi = 0.;
    const double t0 = Tv(0, 0, 0);
    const double tim = Tv(-1, 0, 0), tip = Tv(+1, 0, 0);
    const double tjm = Tv(0, -1, 0), tjp = Tv(0, +1, 0);
    const double tkm = Tv(0, 0, -1), tkp = Tv(0, 0, +1);
    u0[3] = t0;
    {  // advection_x, predict/t.c:88-116
      const double ux_xm = CF(C_JF, 0) * ux_0;
      const double ux_xp = CF(C_JF, +1) * ux_1;
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, c = -l - u;
      e -= invjc * (l * tim + c * t0 + u * tip);
    }
    {  // advection_y
      const double jh = CF(C_E1, 0);
      const double uy_ym = jh * uy_0;
      const double uy_yp = jh * uy_jp;
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, c = -l - u;
      e -= invjc * (l * tjm + c * t0 + u * tjp);
    }
    {  // advection_z
      const double jh = CF(C_E2, 0);
      const double uz_zm = jh * uz_0;
      const double uz_zp = jh * uz_kp;
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, c = -l - u;
      e -= invjc * (l * tkm + c * t0 + u * tkp);
    }
    {
      const double v = kappa * (CF(C_LXL, 0) * tim + CF(C_LXC, 0) * t0 + CF(C_LXU, 0) * tip);
      if (ix) gi += v; else e += v;
    }
    {
      const double v = kappa * (CF(C_LYL, 0) * tjm + CF(C_LYC, 0) * t0 + CF(C_LYU, 0) * tjp);
      if (iy) gi += v; else e += v;
    }
    {
      const double v = kappa * (cf.lz_l * tkm + cf.lz_c * t0 + cf.lz_u * tkp);
      if (iz) gi += v; else e += v;
    }
    const size_t q = pidx(nx, g.ny, i - 1, j, k);
    const double old = use_old ? s_old3[q] : 0.;
    s_new3[q] = e;
    dl[3] = ca * e + cb * old + cg * gi;
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

// ------------------------------------------------------------ fused predict
// Affine map q -> a q + b; compositions of the Thomas recurrences.
struct Aff { double a, b; };

template <int E>
__device__ __forceinline__ int spad(int e) { return E > 1 ? e + e / E : e; }

// Radial Thomas solve of one line by one warp (src/tdm.c:24-48), the line held
// in shared memory (padded by one slot per E elements against bank
// conflicts). Lane t owns elements tE .. tE+E-1: it composes their affine maps,
// a 5-level shuffle scan supplies the value entering its chunk, then the
// recurrence runs in the reference's form q = w (r - l q_prev) (forward) and
// x = q - v x_next (backward).
template <int E>
__device__ __forceinline__ void solve_line(double * sb, const XFactors & xf, int rkstep, int var, int lane) {
  const int n = xf.n[var];
  const size_t fo = (size_t)(rkstep * 4 + var) * xf.stride;
  const double * __restrict__ lo = xf.lo + fo;
  const double * __restrict__ w = xf.w + fo;
  const double * __restrict__ v = xf.v + fo;
  double q[E], ll[E], ww[E];
#pragma unroll
  for (int m = 0; m < E; m++) {
    const int e = lane * E + m;
    const bool el = e < n;
    q[m] = el ? sb[spad<E>(e)] : 0.;
    ll[m] = el ? LD(lo + e) : 0.;
    ww[m] = el ? LD(w + e) : 0.;
  }
  Aff acc{1., 0.};
#pragma unroll
  for (int m = 0; m < E; m++) {
    const int e = lane * E + m;
    double fa, fb;
    if (e == 0) { fa = 0.; fb = q[m] / ww[m]; }          // w[0] holds c[0]
    else if (e < n) { fa = -ww[m] * ll[m]; fb = ww[m] * q[m]; }
    else { fa = 0.; fb = 0.; }
    acc.b = fa * acc.b + fb;
    acc.a = fa * acc.a;
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double oa = __shfl_up_sync(0xffffffffu, acc.a, off);
    const double ob = __shfl_up_sync(0xffffffffu, acc.b, off);
    if (lane >= off) { acc.b = acc.a * ob + acc.b; acc.a = acc.a * oa; }
  }
  double qin = __shfl_up_sync(0xffffffffu, acc.b, 1);
  if (lane == 0) qin = 0.;
#pragma unroll
  for (int m = 0; m < E; m++) {
    const int e = lane * E + m;
    double r;
    if (e == 0) r = q[m] / ww[m];
    else if (e < n) r = ww[m] * (q[m] - ll[m] * qin);
    else r = 0.;
    q[m] = r;
    qin = r;
  }
  double vv[E];
  Aff bac{1., 0.};
#pragma unroll
  for (int m = E - 1; m >= 0; m--) {
    const int e = lane * E + m;
    vv[m] = (e < n) ? LD(v + e) : 0.;
    const double fa = (e < n) ? -vv[m] : 0.;
    const double fb = (e < n) ? q[m] : 0.;
    bac.b = fa * bac.b + fb;
    bac.a = fa * bac.a;
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double oa = __shfl_down_sync(0xffffffffu, bac.a, off);
    const double ob = __shfl_down_sync(0xffffffffu, bac.b, off);
    if (lane + off < 32) { bac.b = bac.a * ob + bac.b; bac.a = bac.a * oa; }
  }
  double xin = __shfl_down_sync(0xffffffffu, bac.b, 1);
  if (lane == 31) xin = 0.;
#pragma unroll
  for (int m = E - 1; m >= 0; m--) {
    const int e = lane * E + m;
    const double x = (e < n) ? q[m] - vv[m] * xin : 0.;
    if (e < n) sb[spad<E>(e)] = x;
    xin = x;
  }
}

// One CTA row per radial line (j, k), one thread per radial index i. Each
// thread computes the four right-hand sides and increments of its cell; the
// increments are staged in shared memory and the radial implicit systems of
// the CTA's lines are solved one per warp (line-independent factors from
// xfactor_kernel). The new fields go to the other buffer of the pair (the old
// ones are still read by neighbouring lines), walls and periodic images
// included. PREDICT_DELTA writes the radially solved increments instead, for
// the y and z solves of the planar configuration.
#ifndef TC_PREDICT_MIN_BLOCKS
#define TC_PREDICT_MIN_BLOCKS 4
#endif
template <int NW>   // warps per line; also the elements per lane of the solves
__global__ void __launch_bounds__(256, TC_PREDICT_MIN_BLOCKS)
predict_kernel(Geo g, Bc bc, Coefs cf, XFactors xf, double nu, double kappa,
               Fields in, Fields out, SrcSet ss, DeltaSet ds, const double * __restrict__ dtp,
               int rkstep, int mode) {
  constexpr int NT = 32 * NW;
  constexpr int LPB = 256 / NT;
  constexpr int E = NW;
  constexpr int SL = 32 * E + (E > 1 ? 32 : 0);
  __shared__ double sd[LPB][4][SL];
  const int tx = threadIdx.x;
  const int ly = threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long nlines = (long long)ny * nz;
  const long long line = (long long)blockIdx.x * LPB + ly;
  const bool vline = line < nlines;
  const int j = vline ? (int)(line % ny) + 1 : 1;
  const int k = vline ? (int)(line / ny) + 1 : 1;
  const int i = tx + 1;
  const bool cell = vline && i <= nx;
  const double dt = *dtp;
  const double ca = rk_alpha(rkstep) * dt;
  const double cb = rk_beta(rkstep) * dt;
  const double cg = rk_gamma(rkstep) * dt;
  double dl[4] = {0., 0., 0., 0.}, u0[4] = {0., 0., 0., 0.};
  if (cell) {
    cell_rhs_delta(g, bc, cf, nu, kappa, in.ux, in.uy, in.uz, in.p, in.t,
                   ss.old_[0], ss.old_[1], ss.old_[2], ss.old_[3], ss.new_[0], ss.new_[1], ss.new_[2], ss.new_[3],
                   i, j, k, ca, cb, cg, rkstep != 0, dl, u0);
  }
  if (bc.implicit[0]) {
    if (cell) {
      if (i >= 2) sd[ly][VUX][spad<E>(i - 2)] = dl[VUX];
      sd[ly][VUY][spad<E>(i - 1)] = dl[VUY];
      sd[ly][VUZ][spad<E>(i - 1)] = dl[VUZ];
      sd[ly][VT][spad<E>(i - 1)] = dl[VT];
    }
    __syncthreads();
    const int wid = (ly * NT + tx) >> 5;
    const int lane = tx & 31;
    for (int s = wid; s < 4 * LPB; s += 8) {
      const int l = s >> 2, v = s & 3;
      if ((long long)blockIdx.x * LPB + l >= nlines) continue;
      solve_line<E>(sd[l][v], xf, rkstep, v, lane);
    }
    __syncthreads();
    if (cell) {
      dl[VUX] = (i >= 2) ? sd[ly][VUX][spad<E>(i - 2)] : 0.;
      dl[VUY] = sd[ly][VUY][spad<E>(i - 1)];
      dl[VUZ] = sd[ly][VUZ][spad<E>(i - 1)];
      dl[VT] = sd[ly][VT][spad<E>(i - 1)];
    }
  }
  if (!cell) return;
  if (mode == PREDICT_DELTA) {
    if (i >= 2) ds.d[VUX][pidx(nx - 1, ny, i - 2, j, k)] = dl[VUX];
    const size_t qc = pidx(nx, ny, i - 1, j, k);
    ds.d[VUY][qc] = dl[VUY];
    ds.d[VUZ][qc] = dl[VUZ];
    ds.d[VT][qc] = dl[VT];
    return;
  }
  // u += delta into the other buffer, walls (boundary/*.c) and images (halo.c)
  const double vx = (i >= 2) ? u0[VUX] + dl[VUX] : 0.;
  const double vy = u0[VUY] + dl[VUY];
  const double vz = u0[VUZ] + dl[VUZ];
  const double vt = u0[VT] + dl[VT];
  auto put = [&](int jj, int kk) {
    out.ux[fidx(g, i, jj, kk)] = vx;
    out.uy[cidx(g, i, jj, kk)] = vy;
    out.uz[cidx(g, i, jj, kk)] = vz;
    out.t[cidx(g, i, jj, kk)] = vt;
    if (i == 1) {
      out.uy[cidx(g, 0, jj, kk)] = bc.uy_xm;
      out.uz[cidx(g, 0, jj, kk)] = 0.;
      out.t[cidx(g, 0, jj, kk)] = bc.t_xm;
    }
    if (i == nx) {
      out.ux[fidx(g, nx + 1, jj, kk)] = 0.;
      out.uy[cidx(g, nx + 1, jj, kk)] = bc.uy_xp;
      out.uz[cidx(g, nx + 1, jj, kk)] = 0.;
      out.t[cidx(g, nx + 1, jj, kk)] = bc.t_xp;
    }
  };
  put(j, k);
  for_images(j, k, ny, nz, put);
}

// out = in + delta for every cell, walls and images (after the y / z solves)
__global__ void __launch_bounds__(256)
apply_kernel(Geo g, Bc bc, Fields in, Fields out, DeltaSet ds) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (i > nx || j > ny) return;
  const size_t qc = pidx(nx, ny, i - 1, j, k);
  const double vx = (i >= 2) ? in.ux[fidx(g, i, j, k)] + ds.d[VUX][pidx(nx - 1, ny, i - 2, j, k)] : 0.;
  const double vy = in.uy[cidx(g, i, j, k)] + ds.d[VUY][qc];
  const double vz = in.uz[cidx(g, i, j, k)] + ds.d[VUZ][qc];
  const double vt = in.t[cidx(g, i, j, k)] + ds.d[VT][qc];
  auto put = [&](int jj, int kk) {
    out.ux[fidx(g, i, jj, kk)] = vx;
    out.uy[cidx(g, i, jj, kk)] = vy;
    out.uz[cidx(g, i, jj, kk)] = vz;
    out.t[cidx(g, i, jj, kk)] = vt;
    if (i == 1) {
      out.uy[cidx(g, 0, jj, kk)] = bc.uy_xm;
      out.uz[cidx(g, 0, jj, kk)] = 0.;
      out.t[cidx(g, 0, jj, kk)] = bc.t_xm;
    }
    if (i == nx) {
      out.ux[fidx(g, nx + 1, jj, kk)] = 0.;
      out.uy[cidx(g, nx + 1, jj, kk)] = bc.uy_xp;
      out.uz[cidx(g, nx + 1, jj, kk)] = 0.;
      out.t[cidx(g, nx + 1, jj, kk)] = bc.t_xp;
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
template <int NW>
static void launch_predict_nw(const Geo & g, const Bc & bc, const Coefs & cf, const XFactors & xf, double nu,
                              double kappa, const Fields & in, const Fields & out, const SrcSet & ss,
                              const DeltaSet & ds, const double * dtp, int rkstep, int mode, cudaStream_t st) {
  constexpr int NT = 32 * NW;
  constexpr int LPB = 256 / NT;
  const long long nlines = (long long)g.ny * g.nz;
  dim3 block(NT, LPB, 1);
  dim3 grid((unsigned)((nlines + LPB - 1) / LPB), 1, 1);
  predict_kernel<NW><<<grid, block, 0, st>>>(g, bc, cf, xf, nu, kappa, in, out, ss, ds, dtp, rkstep, mode);
}

int predict_warps(int nx) {
  int w = 1;
  while (32 * w < nx) w *= 2;
  return w;
}

void launch_predict(const Geo & g, const Bc & bc, const Coefs & cf, const XFactors & xf, double nu, double kappa,
                    const Fields & in, const Fields & out, const SrcSet & ss, const DeltaSet & ds,
                    const double * dtp, int rkstep, int mode, cudaStream_t st) {
  switch (predict_warps(g.nx)) {
    case 1: launch_predict_nw<1>(g, bc, cf, xf, nu, kappa, in, out, ss, ds, dtp, rkstep, mode, st); break;
    case 2: launch_predict_nw<2>(g, bc, cf, xf, nu, kappa, in, out, ss, ds, dtp, rkstep, mode, st); break;
    case 4: launch_predict_nw<4>(g, bc, cf, xf, nu, kappa, in, out, ss, ds, dtp, rkstep, mode, st); break;
    default: launch_predict_nw<8>(g, bc, cf, xf, nu, kappa, in, out, ss, ds, dtp, rkstep, mode, st); break;
  }
}

void launch_xfactors(const XFactors & xf, const double * dtp, double nu, double kappa, cudaStream_t st) {
  xfactor_kernel<<<1, 32, 0, st>>>(xf, dtp, nu, kappa);
}

void launch_apply(const Geo & g, const Bc & bc, const Fields & in, const Fields & out, const DeltaSet & ds,
                  cudaStream_t st) {
  dim3 block(32, 8, 1);
  dim3 grid((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
  apply_kernel<<<grid, block, 0, st>>>(g, bc, in, out, ds);
}

void launch_ysolve(const Geo & g, const YZFactors & yf, int rkstep, const DeltaSet & ds, cudaStream_t st) {
  for (int v = 0; v < 4; v++) {
    const long long n = (long long)yf.n_i[v] * g.nz;
    ysolve_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(g, yf, rkstep, v, ds.d[v]);
  }
}

void launch_zsolve(const Geo & g, const YZFactors & yf, int rkstep, const DeltaSet & ds, cudaStream_t st) {
  for (int v = 0; v < 4; v++) {
    const long long n = (long long)yf.n_i[v] * g.ny;
    zsolve_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(g, yf, rkstep, v, ds.d[v]);
  }
}

}  // namespace tcgpu
