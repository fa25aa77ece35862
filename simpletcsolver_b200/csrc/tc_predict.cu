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

// ------------------------------------------------------------ rhs + delta of KP cells
// Right-hand sides of ux (face i), uy, uz, t (centre i) of the KP cells
// (i, j, k + c), c < KP, the new explicit source terms (written to s_new*)
// and the RK increments dl[c][0..3] (dl[c][0] is 0 at i = 1, where ux has no
// unknown). u0 returns the cells' current values. The KP cells share every
// metric coefficient load (the tables depend on i only) and the field values
// their stencils have in common; each term runs over the KP cells in turn.
#define FC _Pragma("unroll") for (int c = 0; c < KP; c++)
template <int KP>
__device__ __forceinline__ void cells_rhs_delta(
    const Geo & g, const Bc & bc, const Coefs & cf, double nu, double kappa,
    const double * __restrict__ ux, const double * __restrict__ uy,
    const double * __restrict__ uz, const double * __restrict__ p,
    const double * __restrict__ t,
    const double * __restrict__ s_old0, const double * __restrict__ s_old1,
    const double * __restrict__ s_old2, const double * __restrict__ s_old3,
    double * __restrict__ s_new0, double * __restrict__ s_new1,
    double * __restrict__ s_new2, double * __restrict__ s_new3,
    int i, int j, int k, double ca, double cb, double cg, bool use_old,
    double (&dl)[KP][4], double (&u0)[KP][4]) {
  const int nx = g.nx;
  const bool ix = bc.implicit[0], iy = bc.implicit[1], iz = bc.implicit[2];
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
  // packed source-term offsets of the first cell, and their plane stride
  const size_t qf0 = pidx(nx - 1, g.ny, i - 2, j, k), qc0 = pidx(nx, g.ny, i - 1, j, k);
  const size_t pf = (size_t)(nx - 1) * g.ny, pc = (size_t)nx * g.ny;
#define UXv(DI, DJ, DK) LD(bx + ((DI) + (DJ) * sjf + (DK) * skf))
#define UYv(DI, DJ, DK) LD(by + ((DI) + (DJ) * sjc + (DK) * skc))
#define UZv(DI, DJ, DK) LD(bz + ((DI) + (DJ) * sjc + (DK) * skc))
#define Pv(DI, DJ, DK)  LD(bp + ((DI) + (DJ) * sjc + (DK) * skc))
#define Tv(DI, DJ, DK)  LD(bt + ((DI) + (DJ) * sjc + (DK) * skc))
#define CF(T, D) LD(bc_ + ((T) * CSTRIDE + (D)))

  FC { dl[c][0] = 0.; }
  // ---------------------------------------------------------------- ux at face i
  if (i >= 2) {
    double e[KP], gi[KP];
    double ux_m[KP], ux_0[KP], ux_p[KP];
    FC {
      e[c] = 0.; gi[c] = 0.;
      ux_m[c] = UXv(-1, 0, c); ux_0[c] = UXv(0, 0, c); ux_p[c] = UXv(+1, 0, c);
    }
    const double invj = CF(F_INVJD, 0);
    {  // advection_x, predict/ux.c:92-121
      const double a1 = CF(F_A1, 0), a2 = CF(F_A2, 0), a3 = CF(F_A3, 0);
      FC {
        const double ux_xm = a1 * ux_m[c] + a2 * ux_0[c];
        const double ux_xp = a2 * ux_0[c] + a3 * ux_p[c];
        const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, cc = -l - u;
        e[c] -= invj * (l * ux_m[c] + cc * ux_0[c] + u * ux_p[c]);
      }
    }
    double uy_m0[KP], uy_00[KP], uy_m1[KP], uy_01[KP], ux_jm[KP], ux_jp[KP];
    FC {
      uy_m0[c] = UYv(-1, 0, c); uy_00[c] = UYv(0, 0, c);
      uy_m1[c] = UYv(-1, +1, c); uy_01[c] = UYv(0, +1, c);
      ux_jm[c] = UXv(0, -1, c); ux_jp[c] = UXv(0, +1, c);
    }
    {  // advection_y :123-155
      const double b1 = CF(F_B1, 0), b2 = CF(F_B2, 0);
      FC {
        const double uy_ym = b1 * uy_m0[c] + b2 * uy_00[c];
        const double uy_yp = b1 * uy_m1[c] + b2 * uy_01[c];
        const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, cc = -l - u;
        e[c] -= invj * (l * ux_jm[c] + cc * ux_0[c] + u * ux_jp[c]);
      }
    }
    double uz_m0[KP], uz_00[KP], uz_m1[KP], uz_01[KP], ux_km[KP], ux_kp[KP];
    FC {
      uz_m0[c] = UZv(-1, 0, c); uz_00[c] = UZv(0, 0, c);
      uz_m1[c] = UZv(-1, 0, c + 1); uz_01[c] = UZv(0, 0, c + 1);
      ux_km[c] = UXv(0, 0, c - 1); ux_kp[c] = UXv(0, 0, c + 1);
    }
    {  // advection_z :157-186
      const double c1 = CF(F_C1, 0), c2 = CF(F_C2, 0);
      FC {
        const double uz_zm = c1 * uz_m0[c] + c2 * uz_00[c];
        const double uz_zp = c1 * uz_m1[c] + c2 * uz_01[c];
        const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, cc = -l - u;
        e[c] -= invj * (l * ux_km[c] + cc * ux_0[c] + u * ux_kp[c]);
      }
    }
    {  // advection_1 (centrifugal) :194-226
      const double hd1 = CF(F_HD1, 0), hd2 = CF(F_HD2, 0);
      FC {
        const double uy_xm = 0.5 * uy_m0[c] + 0.5 * uy_m1[c];
        const double uy_xp = 0.5 * uy_00[c] + 0.5 * uy_01[c];
        e[c] += invj * (hd1 * uy_xm * uy_xm + hd2 * uy_xp * uy_xp);
      }
    }
    {  // diffusion_x :228-245
      const double ll = CF(F_LXL, 0), lc = CF(F_LXC, 0), lu = CF(F_LXU, 0);
      FC {
        const double v = 2. * nu * (ll * ux_m[c] + lc * ux_0[c] + lu * ux_p[c]);
        if (ix) gi[c] += v; else e[c] += v;
      }
    }
    {  // diffusion_y0 :247-264
      const double ll = CF(F_LYL, 0), lc = CF(F_LYC, 0), lu = CF(F_LYU, 0);
      FC {
        const double v = nu * (ll * ux_jm[c] + lc * ux_0[c] + lu * ux_jp[c]);
        if (iy) gi[c] += v; else e[c] += v;
      }
    }
    const double njd = nu * invj;
    const double ih = CF(C_INVHXXF, 0);
    {  // diffusion_y1 :266-290, with lyx1 (lyx.c:64-83) and lxy (lxy.c:28-34)
      const double F = CF(C_LYX1F, 0), wm = CF(C_WM, 0), wp = CF(C_WP, 0);
      const double jh = CF(F_E1, 0);
      FC {
        const double lyx1_m = F * (wm * uy_m0[c] + wp * uy_00[c]);
        const double lyx1_p = F * (wm * uy_m1[c] + wp * uy_01[c]);
        const double lxy_m = ih * (-uy_m0[c] + uy_00[c]);
        const double lxy_p = ih * (-uy_m1[c] + uy_01[c]);
        e[c] += njd * (-jh * (lyx1_m + lxy_m) + jh * (lyx1_p + lxy_p));
      }
    }
    {  // diffusion_z0 :292-309
      FC {
        const double v = nu * (cf.lz_l * ux_km[c] + cf.lz_c * ux_0[c] + cf.lz_u * ux_kp[c]);
        if (iz) gi[c] += v; else e[c] += v;
      }
    }
    {  // diffusion_z1 :311-332, lxz (lxz.c:19-27)
      const double jh = CF(F_E2, 0);
      FC {
        const double lxz_m = ih * (-uz_m0[c] + uz_00[c]);
        const double lxz_p = ih * (-uz_m1[c] + uz_01[c]);
        e[c] += njd * (-jh * lxz_m + jh * lxz_p);
      }
    }
    {  // diffusion_a :344-375, lyy0/lyy1 (lyy.c) at centres i-1 and i
      const double hm = CF(C_INVHYXC, -1), km = CF(C_LYY1, -1), h0 = CF(C_INVHYXC, 0), k0 = CF(C_LYY1, 0);
      const double hd1 = CF(F_HD1, 0), hd2 = CF(F_HD2, 0);
      FC {
        const double lyy_xm = hm * (-uy_m0[c] + uy_m1[c]) + km * (0.5 * ux_m[c] + 0.5 * ux_0[c]);
        const double lyy_xp = h0 * (-uy_00[c] + uy_01[c]) + k0 * (0.5 * ux_0[c] + 0.5 * ux_p[c]);
        e[c] -= 2. * njd * (hd1 * lyy_xm + hd2 * lyy_xp);
      }
    }
    // pressure :377-394
    FC {
      gi[c] -= ih * (-Pv(-1, 0, c) + Pv(0, 0, c));
      const size_t q = qf0 + c * pf;
      const double old = use_old ? s_old0[q] : 0.;
      s_new0[q] = e[c];
      dl[c][0] = ca * e[c] + cb * old + cg * gi[c];
    }
  }

  // ---------------------------------------------------------------- uy at centre i
  double uy_0[KP], uy_im[KP], uy_ip[KP], uy_jm[KP], uy_jp[KP], uy_km[KP], uy_kp[KP];
  double ux_0[KP], ux_1[KP], ux_0m[KP], ux_1m[KP], ux_0k[KP], ux_1k[KP];
  double uz_0[KP], uz_kp[KP], uz_jm[KP], uz_jmkp[KP];
  FC {
    uy_0[c] = UYv(0, 0, c);
    uy_im[c] = UYv(-1, 0, c); uy_ip[c] = UYv(+1, 0, c);
    uy_jm[c] = UYv(0, -1, c); uy_jp[c] = UYv(0, +1, c);
    uy_km[c] = UYv(0, 0, c - 1); uy_kp[c] = UYv(0, 0, c + 1);
    ux_0[c] = UXv(0, 0, c); ux_1[c] = UXv(+1, 0, c);          // faces i, i+1 at j
    ux_0m[c] = UXv(0, -1, c); ux_1m[c] = UXv(+1, -1, c);      // at j-1
    ux_0k[c] = UXv(0, 0, c - 1); ux_1k[c] = UXv(+1, 0, c - 1);  // at k-1
    uz_0[c] = UZv(0, 0, c); uz_kp[c] = UZv(0, 0, c + 1);
    uz_jm[c] = UZv(0, -1, c); uz_jmkp[c] = UZv(0, -1, c + 1);
    u0[c][0] = ux_0[c];
    u0[c][1] = uy_0[c];
    u0[c][2] = uz_0[c];
  }
  const double invjc = CF(C_INVJDXC, 0);
  const double njc = nu * invjc;
  const double a1 = CF(C_A1, 0), a2 = CF(C_A2, 0);
  const double bb = CF(C_B, 0), cz = CF(C_CZ, 0);
  const double jf0 = CF(C_JF, 0), jf1 = CF(C_JF, +1);
  const double e1 = CF(C_E1, 0), e2 = CF(C_E2, 0);
  {
    double e[KP], gi[KP];
    FC { e[c] = 0.; gi[c] = 0.; }
    FC {  // advection_x, predict/uy.c:93-123
      const double ux_xm = a1 * ux_0m[c] + a1 * ux_0[c];
      const double ux_xp = a2 * ux_1m[c] + a2 * ux_1[c];
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, cc = -l - u;
      e[c] -= invjc * (l * uy_im[c] + cc * uy_0[c] + u * uy_ip[c]);
    }
    FC {  // advection_y :125-151
      const double uy_ym = bb * uy_jm[c] + bb * uy_0[c];
      const double uy_yp = bb * uy_0[c] + bb * uy_jp[c];
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, cc = -l - u;
      e[c] -= invjc * (l * uy_jm[c] + cc * uy_0[c] + u * uy_jp[c]);
    }
    FC {  // advection_z :153-180
      const double uz_zm = cz * uz_jm[c] + cz * uz_0[c];
      const double uz_zp = cz * uz_jmkp[c] + cz * uz_kp[c];
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, cc = -l - u;
      e[c] -= invjc * (l * uy_km[c] + cc * uy_0[c] + u * uy_kp[c]);
    }
    {  // advection_1 :188-223
      const double hd = CF(C_HD, 0);
      FC {
        const double uy_ym = 0.5 * uy_jm[c] + 0.5 * uy_0[c];
        const double uy_yp = 0.5 * uy_0[c] + 0.5 * uy_jp[c];
        const double ux_ym = 0.5 * ux_0m[c] + 0.5 * ux_1m[c];
        const double ux_yp = 0.5 * ux_0[c] + 0.5 * ux_1[c];
        e[c] -= invjc * (hd * uy_ym * ux_ym + hd * uy_yp * ux_yp);
      }
    }
    {  // diffusion_x0
      const double ll = CF(C_LXL, 0), lc = CF(C_LXC, 0), lu = CF(C_LXU, 0);
      FC {
        const double v = nu * (ll * uy_im[c] + lc * uy_0[c] + lu * uy_ip[c]);
        if (ix) gi[c] += v; else e[c] += v;
      }
    }
    // lyx0 (lyx.c:33-39), lyx1 (:64-83) at faces i and i+1
    double lyx_xm[KP], lyx_xp[KP];
    {
      const double hf0 = CF(C_INVHYXF, 0), hf1 = CF(C_INVHYXF, +1);
      const double F0 = CF(C_LYX1F, 0), F1 = CF(C_LYX1F, +1);
      const double wm0 = CF(C_WM, 0), wp0 = CF(C_WP, 0), wm1 = CF(C_WM, +1), wp1 = CF(C_WP, +1);
      FC {
        const double lyx0_m = hf0 * (-ux_0m[c] + ux_0[c]);
        const double lyx0_p = hf1 * (-ux_1m[c] + ux_1[c]);
        const double lyx1_m = F0 * (wm0 * uy_im[c] + wp0 * uy_0[c]);
        const double lyx1_p = F1 * (wm1 * uy_0[c] + wp1 * uy_ip[c]);
        lyx_xm[c] = lyx0_m + lyx1_m;
        lyx_xp[c] = lyx0_p + lyx1_p;
        // diffusion_x1
        e[c] += njc * (-jf0 * lyx_xm[c] + jf1 * lyx_xp[c]);
      }
    }
    {  // diffusion_y0
      const double ll = CF(C_LYL, 0), lc = CF(C_LYC, 0), lu = CF(C_LYU, 0);
      FC {
        const double v = 2. * nu * (ll * uy_jm[c] + lc * uy_0[c] + lu * uy_jp[c]);
        if (iy) gi[c] += v; else e[c] += v;
      }
    }
    {  // diffusion_y1, lyy1 (lyy.c:64-83) at j-1 and j
      const double K = CF(C_LYY1, 0);
      FC {
        const double lyy1_m = K * (0.5 * ux_0m[c] + 0.5 * ux_1m[c]);
        const double lyy1_0 = K * (0.5 * ux_0[c] + 0.5 * ux_1[c]);
        e[c] += 2. * njc * (-e1 * lyy1_m + e1 * lyy1_0);
      }
    }
    FC {  // diffusion_z0
      const double v = nu * (cf.lz_l * uy_km[c] + cf.lz_c * uy_0[c] + cf.lz_u * uy_kp[c]);
      if (iz) gi[c] += v; else e[c] += v;
    }
    const double ihc = CF(C_INVHYXC, 0);
    FC {  // diffusion_z1, lyz (lyz.c:19-27) at k and k+1
      const double lyz_0 = ihc * (-uz_jm[c] + uz_0[c]);
      const double lyz_p = ihc * (-uz_jmkp[c] + uz_kp[c]);
      e[c] += njc * (-e2 * lyz_0 + e2 * lyz_p);
    }
    {  // diffusion_a :367-400, lxy (lxy.c) at faces i and i+1
      const double hx0 = CF(C_INVHXXF, 0), hx1 = CF(C_INVHXXF, +1);
      const double hda1 = CF(C_HDA1, 0), hda2 = CF(C_HDA2, 0);
      FC {
        const double lxy_m = hx0 * (-uy_im[c] + uy_0[c]);
        const double lxy_p = hx1 * (-uy_0[c] + uy_ip[c]);
        e[c] += njc * (hda1 * (lyx_xm[c] + lxy_m) + hda2 * (lyx_xp[c] + lxy_p));
      }
    }
    FC {
      gi[c] -= ihc * (-Pv(0, -1, c) + Pv(0, 0, c));
      const size_t q = qc0 + c * pc;
      const double old = use_old ? s_old1[q] : 0.;
      s_new1[q] = e[c];
      dl[c][1] = ca * e[c] + cb * old + cg * gi[c];
    }
  }

  // ---------------------------------------------------------------- uz at centre i
  {
    double e[KP], gi[KP];
    double uz_im[KP], uz_ip[KP], uz_jp[KP], uz_km[KP], uy_jpkm[KP];
    FC {
      e[c] = 0.; gi[c] = 0.;
      uz_im[c] = UZv(-1, 0, c); uz_ip[c] = UZv(+1, 0, c);
      uz_jp[c] = UZv(0, +1, c); uz_km[c] = UZv(0, 0, c - 1);
      uy_jpkm[c] = UYv(0, +1, c - 1);
    }
    FC {  // advection_x, predict/uz.c:88-118
      const double ux_xm = a1 * ux_0k[c] + a1 * ux_0[c];
      const double ux_xp = a2 * ux_1k[c] + a2 * ux_1[c];
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, cc = -l - u;
      e[c] -= invjc * (l * uz_im[c] + cc * uz_0[c] + u * uz_ip[c]);
    }
    FC {  // advection_y
      const double uy_ym = bb * uy_km[c] + bb * uy_0[c];
      const double uy_yp = bb * uy_jpkm[c] + bb * uy_jp[c];
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, cc = -l - u;
      e[c] -= invjc * (l * uz_jm[c] + cc * uz_0[c] + u * uz_jp[c]);
    }
    FC {  // advection_z
      const double uz_zm = cz * uz_km[c] + cz * uz_0[c];
      const double uz_zp = cz * uz_0[c] + cz * uz_kp[c];
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, cc = -l - u;
      e[c] -= invjc * (l * uz_km[c] + cc * uz_0[c] + u * uz_kp[c]);
    }
    {  // diffusion_x0
      const double ll = CF(C_LXL, 0), lc = CF(C_LXC, 0), lu = CF(C_LXU, 0);
      FC {
        const double v = nu * (ll * uz_im[c] + lc * uz_0[c] + lu * uz_ip[c]);
        if (ix) gi[c] += v; else e[c] += v;
      }
    }
    const double ihz = cf.inv_hz;
    FC {  // diffusion_x1, lzx (lzx.c) at faces i, i+1
      const double lzx_m = ihz * (-ux_0k[c] + ux_0[c]);
      const double lzx_p = ihz * (-ux_1k[c] + ux_1[c]);
      e[c] += njc * (-jf0 * lzx_m + jf1 * lzx_p);
    }
    {  // diffusion_y0
      const double ll = CF(C_LYL, 0), lc = CF(C_LYC, 0), lu = CF(C_LYU, 0);
      FC {
        const double v = nu * (ll * uz_jm[c] + lc * uz_0[c] + lu * uz_jp[c]);
        if (iy) gi[c] += v; else e[c] += v;
      }
    }
    FC {  // diffusion_y1, lzy (lzy.c) at j, j+1
      const double lzy_0 = ihz * (-uy_km[c] + uy_0[c]);
      const double lzy_p = ihz * (-uy_jpkm[c] + uy_jp[c]);
      e[c] += njc * (-e1 * lzy_0 + e1 * lzy_p);
    }
    FC {  // diffusion_z
      const double v = 2. * nu * (cf.lz_l * uz_km[c] + cf.lz_c * uz_0[c] + cf.lz_u * uz_kp[c]);
      if (iz) gi[c] += v; else e[c] += v;
    }
    FC {
      gi[c] -= ihz * (-Pv(0, 0, c - 1) + Pv(0, 0, c));
      const size_t q = qc0 + c * pc;
      const double old = use_old ? s_old2[q] : 0.;
      s_new2[q] = e[c];
      dl[c][2] = ca * e[c] + cb * old + cg * gi[c];
    }
  }

  // ---------------------------------------------------------------- t at centre i
  {
    double e[KP], gi[KP];
    double t0[KP], tim[KP], tip[KP], tjm[KP], tjp[KP], tkm[KP], tkp[KP];
    FC {
      e[c] = 0.; gi[c] = 0.;
      t0[c] = Tv(0, 0, c);
      tim[c] = Tv(-1, 0, c); tip[c] = Tv(+1, 0, c);
      tjm[c] = Tv(0, -1, c); tjp[c] = Tv(0, +1, c);
      tkm[c] = Tv(0, 0, c - 1); tkp[c] = Tv(0, 0, c + 1);
      u0[c][3] = t0[c];
    }
    FC {  // advection_x, predict/t.c:88-116
      const double ux_xm = jf0 * ux_0[c];
      const double ux_xp = jf1 * ux_1[c];
      const double l = -0.5 * ux_xm, u = 0.5 * ux_xp, cc = -l - u;
      e[c] -= invjc * (l * tim[c] + cc * t0[c] + u * tip[c]);
    }
    FC {  // advection_y
      const double uy_ym = e1 * uy_0[c];
      const double uy_yp = e1 * uy_jp[c];
      const double l = -0.5 * uy_ym, u = 0.5 * uy_yp, cc = -l - u;
      e[c] -= invjc * (l * tjm[c] + cc * t0[c] + u * tjp[c]);
    }
    FC {  // advection_z
      const double uz_zm = e2 * uz_0[c];
      const double uz_zp = e2 * uz_kp[c];
      const double l = -0.5 * uz_zm, u = 0.5 * uz_zp, cc = -l - u;
      e[c] -= invjc * (l * tkm[c] + cc * t0[c] + u * tkp[c]);
    }
    {
      const double ll = CF(C_LXL, 0), lc = CF(C_LXC, 0), lu = CF(C_LXU, 0);
      FC {
        const double v = kappa * (ll * tim[c] + lc * t0[c] + lu * tip[c]);
        if (ix) gi[c] += v; else e[c] += v;
      }
    }
    {
      const double ll = CF(C_LYL, 0), lc = CF(C_LYC, 0), lu = CF(C_LYU, 0);
      FC {
        const double v = kappa * (ll * tjm[c] + lc * t0[c] + lu * tjp[c]);
        if (iy) gi[c] += v; else e[c] += v;
      }
    }
    FC {
      const double v = kappa * (cf.lz_l * tkm[c] + cf.lz_c * t0[c] + cf.lz_u * tkp[c]);
      if (iz) gi[c] += v; else e[c] += v;
      const size_t q = qc0 + c * pc;
      const double old = use_old ? s_old3[q] : 0.;
      s_new3[q] = e[c];
      dl[c][3] = ca * e[c] + cb * old + cg * gi[c];
    }
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
// Lane's chunk of a factor row: E consecutive values, as 16-byte pairs when
// E > 1 (rows start 16-byte aligned and hold at least 32 E values).
template <int E>
__device__ __forceinline__ void load_chunk(double (&r)[E], const double * __restrict__ row, int lane) {
  if constexpr (E == 1) {
    r[0] = LD(row + lane);
  } else {
    const double2 * p2 = reinterpret_cast<const double2 *>(row + lane * E);
#pragma unroll
    for (int m = 0; m < E / 2; m++) {
      const double2 t = __ldg(p2 + m);
      r[2 * m] = t.x;
      r[2 * m + 1] = t.y;
    }
  }
}

template <int E>
__device__ __forceinline__ void solve_line(double * sb, const XFactors & xf, int rkstep, int var, int lane) {
  const int n = xf.n[var];
  const size_t fo = (size_t)(rkstep * 4 + var) * xf.stride;
  const double * __restrict__ lo = xf.lo + fo;
  const double * __restrict__ w = xf.w + fo;
  const double * __restrict__ v = xf.v + fo;
  double q[E], ll[E], ww[E];
  load_chunk<E>(ll, lo, lane);
  load_chunk<E>(ww, w, lane);
#pragma unroll
  for (int m = 0; m < E; m++) {
    const int e = lane * E + m;
    const bool el = e < n;
    q[m] = el ? sb[spad<E>(e)] : 0.;
    ll[m] = el ? ll[m] : 0.;
    ww[m] = el ? ww[m] : 0.;
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
  load_chunk<E>(vv, v, lane);
  Aff bac{1., 0.};
#pragma unroll
  for (int m = E - 1; m >= 0; m--) {
    const int e = lane * E + m;
    vv[m] = (e < n) ? vv[m] : 0.;
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

// One CTA row per group of KP radial lines (j, k..k+KP-1), one thread per
// radial index i. Each thread computes the four right-hand sides and
// increments of its KP cells; the increments are staged in shared memory and
// the radial implicit systems of the CTA's lines are solved one per warp
// (line-independent factors from xfactor_kernel). The new fields go to the
// other buffer of the pair (the old ones are still read by neighbouring
// lines), walls and periodic images included. PREDICT_DELTA writes the
// radially solved increments instead, for the y and z solves of the planar
// configuration.
// Measured at 256 x 1024 x 512 (ms per launch): KP 1 with 3 resident CTAs
// (80 registers) 10.8; KP 1 / 4 CTAs 11.6; KP 2 / 2 CTAs 11.1; KP 2 / 3 CTAs
// 13.3; KP 4 / 2 CTAs 13.5. Sharing coefficient loads between lines halves
// the global load instructions, but the register growth costs more occupancy
// than the loads save.
#ifndef TC_PREDICT_MIN_BLOCKS
#define TC_PREDICT_MIN_BLOCKS 3
#endif
#ifndef TC_PREDICT_KP
#define TC_PREDICT_KP 1
#endif
template <int NW, int KP>   // warps per line (also the elements per lane of the solves); lines per thread
__global__ void __launch_bounds__(256, TC_PREDICT_MIN_BLOCKS)
predict_kernel(Geo g, Bc bc, Coefs cf, XFactors xf, double nu, double kappa,
               Fields in, Fields out, SrcSet ss, DeltaSet ds, const double * __restrict__ dtp,
               int rkstep, int mode) {
  constexpr int NT = 32 * NW;
  constexpr int LPB = 256 / NT;
  constexpr int E = NW;
  constexpr int SL = 32 * E + (E > 1 ? 32 : 0);
  __shared__ double sd[LPB][KP][4][SL];
  const int tx = threadIdx.x;
  const int ly = threadIdx.y;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const long long ngroups = (long long)ny * (nz / KP);
  const long long grp = (long long)blockIdx.x * LPB + ly;
  const bool vgrp = grp < ngroups;
  const int j = vgrp ? (int)(grp % ny) + 1 : 1;
  const int k = vgrp ? (int)(grp / ny) * KP + 1 : 1;
  const int i = tx + 1;
  const bool cell = vgrp && i <= nx;
  const double dt = *dtp;
  const double ca = rk_alpha(rkstep) * dt;
  const double cb = rk_beta(rkstep) * dt;
  const double cg = rk_gamma(rkstep) * dt;
  double dl[KP][4], u0[KP][4];
  FC {
#pragma unroll
    for (int v = 0; v < 4; v++) { dl[c][v] = 0.; u0[c][v] = 0.; }
  }
  if (cell) {
    cells_rhs_delta<KP>(g, bc, cf, nu, kappa, in.ux, in.uy, in.uz, in.p, in.t,
                        ss.old_[0], ss.old_[1], ss.old_[2], ss.old_[3], ss.new_[0], ss.new_[1], ss.new_[2],
                        ss.new_[3], i, j, k, ca, cb, cg, rkstep != 0, dl, u0);
  }
  if (bc.implicit[0]) {
    if (cell) {
      FC {
        if (i >= 2) sd[ly][c][VUX][spad<E>(i - 2)] = dl[c][VUX];
        sd[ly][c][VUY][spad<E>(i - 1)] = dl[c][VUY];
        sd[ly][c][VUZ][spad<E>(i - 1)] = dl[c][VUZ];
        sd[ly][c][VT][spad<E>(i - 1)] = dl[c][VT];
      }
    }
    __syncthreads();
    const int wid = (ly * NT + tx) >> 5;
    const int lane = tx & 31;
    for (int s = wid; s < 4 * KP * LPB; s += 8) {
      const int l = s / (4 * KP), c = (s >> 2) % KP, v = s & 3;
      if ((long long)blockIdx.x * LPB + l >= ngroups) continue;
      solve_line<E>(sd[l][c][v], xf, rkstep, v, lane);
    }
    __syncthreads();
    if (cell) {
      FC {
        dl[c][VUX] = (i >= 2) ? sd[ly][c][VUX][spad<E>(i - 2)] : 0.;
        dl[c][VUY] = sd[ly][c][VUY][spad<E>(i - 1)];
        dl[c][VUZ] = sd[ly][c][VUZ][spad<E>(i - 1)];
        dl[c][VT] = sd[ly][c][VT][spad<E>(i - 1)];
      }
    }
  }
  if (!cell) return;
  if (mode == PREDICT_DELTA) {
    FC {
      if (i >= 2) ds.d[VUX][pidx(nx - 1, ny, i - 2, j, k + c)] = dl[c][VUX];
      const size_t qc = pidx(nx, ny, i - 1, j, k + c);
      ds.d[VUY][qc] = dl[c][VUY];
      ds.d[VUZ][qc] = dl[c][VUZ];
      ds.d[VT][qc] = dl[c][VT];
    }
    return;
  }
  // u += delta into the other buffer, walls (boundary/*.c) and images (halo.c)
  FC {
    const double vx = (i >= 2) ? u0[c][VUX] + dl[c][VUX] : 0.;
    const double vy = u0[c][VUY] + dl[c][VUY];
    const double vz = u0[c][VUZ] + dl[c][VUZ];
    const double vt = u0[c][VT] + dl[c][VT];
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
    put(j, k + c);
    for_images(j, k + c, ny, nz, put);
  }
}
#undef FC

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
  constexpr int KP = TC_PREDICT_KP;   // nz is a power of two >= 4
  const long long ngroups = (long long)g.ny * (g.nz / KP);
  dim3 block(NT, LPB, 1);
  dim3 grid((unsigned)((ngroups + LPB - 1) / LPB), 1, 1);
  predict_kernel<NW, KP><<<grid, block, 0, st>>>(g, bc, cf, xf, nu, kappa, in, out, ss, ds, dtp, rkstep, mode);
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
