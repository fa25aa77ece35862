// Predict stage: fluid_predict_field (src/fluid/predict/main.c:35-110) for JT
// neighbouring radial lines (j .. j+JT-1) per CTA, marching through a chunk of
// KC planes in z. One pass over the fields per substep: right-hand sides of ux
// (face i), uy, uz, t (centre i), the new explicit source terms, the RK
// increment delta = dt (alpha srcA + beta srcA_prev + gamma srcG) with srcG
// (implicit diffusion + pressure gradient) kept in registers, the radial
// implicit solve (src/tdm.c:17-50), and u + delta into the other buffer of the
// pair with walls and periodic images (boundary/*.c, halo.c).
//
// Per CTA, a ring of four plane slots in shared memory holds the rows
// j-1 .. j+JT of ux, uy, uz, t and j-1 .. j+JT-1 of p for planes k and k+1,
// while planes k+2 and k+3 stream in: one bulk asynchronous copy
// (cp.async.bulk, completion counted in bytes on an mbarrier) per row, issued
// two planes ahead by one thread; the previous substep's source terms of the
// CTA's lines arrive one plane ahead into a buffer of their own. Values a cell
// needs from plane k-1 (ux at faces i, i+1; uy at rows j, j+1; uz, p, t at j)
// are the ones the same thread read one plane earlier and stay in registers;
// the metric coefficients depend on i only, are folded into one product per
// stencil term on the host (the P_* tables) and are loaded once per thread.
// The radial systems are solved by a warpgroup of their own (one warp per
// variable, shuffle scans of affine maps) while the other warps form the next
// plane's right-hand sides; the roles split the register file unevenly
// (setmaxnreg) and meet only at mbarriers.
//
// Row copies start and end on 16-byte boundaries as bulk copies require: a row
// of n doubles starting at element s is copied from s & ~1 up to the even
// bound above s + n, and read at offset s & 1. The parity of s depends only on
// the row's j (ny + 2 is even), so each row keeps one offset for the whole
// march. Every array holds an even number of doubles, so the widened copies
// stay inside their allocations. The packed source-term rows of JT (even)
// consecutive lines start and end on 16-byte boundaries as they are.
#include <type_traits>

#include "tc_common.cuh"
#include "tc_kernels.h"

// FP32-storage mode: right-hand sides in float arithmetic (1), or double (0)
#ifndef TC_MARCH_FP32_ARITH
#define TC_MARCH_FP32_ARITH 1
#endif

namespace tcgpu {
namespace {

#define LD(p) __ldg(p)

// fields of a slot, in row-block order
enum SlotField { SF_UX = 0, SF_UY = 1, SF_UZ = 2, SF_T = 3, SF_P = 4 };

// Two thread groups per radial line: group A (ux at face i, t at centre i)
// and group B (uy, uz at centre i), each with the coefficients of its own
// variables in registers, loaded once (they depend on i only). The
// coefficients are products of the metric tables taken once on the host
// (P_* tables); each is spelled out below where it is used.
// C is the arithmetic type of the right-hand sides: double, or float in the
// FP32-storage mode (the increments, the radial solves and the update stay
// double).
template <class C>
struct CoefA {
  C xa1, xa2, xa3, yb1, yb2, zc1, zc2, h1, h2;        // ux advection
  C lxl, lxu, ly;                                     // ux Laplacian, x and y (carry 2 nu, nu)
  C cy1, cy2, ca1, ca2, cz1, px;                      // ux cross diffusion, pressure gradient
  C tx0, tx1, ty, tz;                                 // t advection
};
template <class C>
struct CoefB {
  C a1, a2, b, c, h;                                  // uy / uz advection
  C lxl, lxu, ly;                                     // centred Laplacian, x and y (carry nu; t: x kappa/nu)
  C p1, p2, qm, q0, qp, yk, yz, py;                   // uy cross diffusion, pressure gradient
  C zx0, zx1, zy;                                     // uz cross diffusion
};
// the z Laplacian's coefficients and 1/hz, shared by every cell
template <class C>
struct CoefZ {
  C l, c, u, ihz;
};
// The Laplacians in x and y are applied as differences from the centre value:
// the centre coefficients of the tables are the negated sums of the others
// (F_LXC = -F_LXL - F_LXU, F_LYC = -2 F_LYL = -2 F_LYU, likewise for C_*), so
// l a + c b + u d = l (a - b) + u (d - b) and only l and u are held.

template <class C>
__device__ __forceinline__ void load_coefs(CoefA<C> & q, const Coefs & cf, int i) {
  const double * __restrict__ b = cf.tab + i;
#define CF(T) (C)LD(b + (T) * CSTRIDE)
  q.xa1 = CF(P_XA1); q.xa2 = CF(P_XA2); q.xa3 = CF(P_XA3); q.yb1 = CF(P_YB1); q.yb2 = CF(P_YB2);
  q.zc1 = CF(P_ZC1); q.zc2 = CF(P_ZC2); q.h1 = CF(P_H1); q.h2 = CF(P_H2);
  q.lxl = CF(F_LXL); q.lxu = CF(F_LXU); q.ly = CF(F_LYL);
  q.cy1 = CF(P_CY1); q.cy2 = CF(P_CY2); q.ca1 = CF(P_CA1); q.ca2 = CF(P_CA2); q.cz1 = CF(P_CZ1);
  q.px = CF(C_INVHXXF);
  q.tx0 = CF(P_TX0); q.tx1 = CF(P_TX1); q.ty = CF(P_TY); q.tz = CF(P_TZ);
#undef CF
}
template <class C>
__device__ __forceinline__ void load_coefs(CoefB<C> & q, const Coefs & cf, int i) {
  const double * __restrict__ b = cf.tab + i;
#define CF(T) (C)LD(b + (T) * CSTRIDE)
  q.a1 = CF(P_UA1); q.a2 = CF(P_UA2); q.b = CF(P_UB); q.c = CF(P_UC); q.h = CF(P_UH);
  q.lxl = CF(C_LXL); q.lxu = CF(C_LXU); q.ly = CF(C_LYL);
  q.p1 = CF(P_P1); q.p2 = CF(P_P2); q.qm = CF(P_QM); q.q0 = CF(P_Q0); q.qp = CF(P_QP);
  q.yk = CF(P_YK); q.yz = CF(P_YZ); q.py = CF(C_INVHYXC);
  q.zx0 = CF(P_ZX0); q.zx1 = CF(P_ZX1); q.zy = CF(P_ZY);
#undef CF
}

// A cell's view of three plane slots (k-1, k and k+1): base pointers already
// moved to the cell's radial index and, for rows of odd parity, to the widened
// copy's offset. Field rows hold the storage type T (ux at element i - 1 in the
// reference layout, at element i in the FP32 layout); p rows are double.
template <class T>
struct SlotView {
  const T * cb;        // plane k, centre fields
  const T * cbo;       // plane k, centre fields, odd rows
  const T * fb;        // plane k, ux
  const T * fbo;       // plane k, ux, odd rows
  const T * nb;        // plane k+1, centre fields
  const T * nbo;
  const T * nf;        // plane k+1, ux
  const T * nfo;
  const T * mb;        // plane k-1, centre fields
  const T * mbo;
  const T * mf;        // plane k-1, ux
  const T * mfo;
  const double * pb;   // plane k, p
  const double * pbo;  // plane k, p, odd rows
  const double * mp;   // plane k-1, p
  const double * mpo;
};

// Slot rows: field f, row r (j - 1 + r for the CTA's first line j) starts at
// (f (JT + 2) + r) RL values of the field block, p row r at r RL of the p
// block; odd rows read at the widened copy's offset. JL is the cell's line
// within the CTA.
#define ROW_(F, DJ) (((F) * (JT + 2) + JL + 1 + (DJ)) * RL)
#define ODD_(DJ) (((JL + 1 + (DJ)) & 1) != 0)
#define UX(DI, DJ) (ODD_(DJ) ? V.fbo : V.fb)[ROW_(SF_UX, DJ) + (DI)]
#define UY(DI, DJ) (ODD_(DJ) ? V.cbo : V.cb)[ROW_(SF_UY, DJ) + (DI)]
#define UZ(DI, DJ) (ODD_(DJ) ? V.cbo : V.cb)[ROW_(SF_UZ, DJ) + (DI)]
#define TT(DI, DJ) (ODD_(DJ) ? V.cbo : V.cb)[ROW_(SF_T, DJ) + (DI)]
#define PP(DI, DJ) (ODD_(DJ) ? V.pbo : V.pb)[(JL + 1 + (DJ)) * RL + (DI)]
#define NUX(DI) (ODD_(0) ? V.nfo : V.nf)[ROW_(SF_UX, 0) + (DI)]
#define NUY(DI) (ODD_(0) ? V.nbo : V.nb)[ROW_(SF_UY, 0) + (DI)]
#define NUZ(DI, DJ) (ODD_(DJ) ? V.nbo : V.nb)[ROW_(SF_UZ, DJ) + (DI)]
#define NTT(DI) (ODD_(0) ? V.nbo : V.nb)[ROW_(SF_T, 0) + (DI)]
#define MUX(DI) (ODD_(0) ? V.mfo : V.mf)[ROW_(SF_UX, 0) + (DI)]
#define MUY(DJ) (ODD_(DJ) ? V.mbo : V.mb)[ROW_(SF_UY, DJ)]
#define MUZ() (ODD_(0) ? V.mbo : V.mb)[ROW_(SF_UZ, 0)]
#define MTT() (ODD_(0) ? V.mbo : V.mb)[ROW_(SF_T, 0)]
#define MPP() (ODD_(0) ? V.mpo : V.mp)[(JL + 1) * RL]
// diffusion in direction D goes to the implicit part when D is implicit
#define ROUTE(D, V_) do { if (D) gi += (V_); else e += (V_); } while (0)

// the z Laplacian's coefficients and 1/hz: kernel parameters in double
// arithmetic, per-thread float copies in float arithmetic
#define ZL (std::is_same<C, double>::value ? (C)cf.lz_l : lz.l)
#define ZC (std::is_same<C, double>::value ? (C)cf.lz_c : lz.c)
#define ZU (std::is_same<C, double>::value ? (C)cf.lz_u : lz.u)
#define ZIH (std::is_same<C, double>::value ? (C)cf.inv_hz : lz.ihz)
// Group A: right-hand sides of ux at face i (src/fluid/predict/ux.c) and t at
// centre i (t.c) of cell (i, j, k); new source terms to ss.new_, increments
// dl[0] (ux, 0 at i = 1 where ux has no unknown) and dl[1] (t), current
// values u0[0] (ux) and u0[1] (t).
template <int JT, int RL, int JL, int IMPL, class T, class C>
__device__ __forceinline__ void cell_a(const CoefA<C> & q, const CoefB<C> & qc_, const SlotView<T> & V, const Bc & bc,
                                       const Coefs & cf, const CoefZ<C> & lz, C nu, C kappa, C rpr, int i, size_t qf,
                                       size_t qc,
                                       const SrcSetT<T> & ss, C ca, C cb, C cg, C old_x, C old_t, double dl[2],
                                       double u0[2]) {
  const bool ix = IMPL >= 0 ? (IMPL & 1) != 0 : bc.implicit[0] != 0;
  const bool iy = IMPL >= 0 ? (IMPL & 2) != 0 : bc.implicit[1] != 0;
  const bool iz = IMPL >= 0 ? (IMPL & 4) != 0 : bc.implicit[2] != 0;
  const C ux_0 = UX(0, 0), ux_p = UX(1, 0);
  const C uy_00 = UY(0, 0), uy_01 = UY(0, 1);
  const C uz_00 = UZ(0, 0), uz_01 = NUZ(0, 0);
  // ux has no unknown at i = 1 (face 1 is the wall): its value there is
  // formed from in-bounds shared-memory neighbours and discarded, so the
  // whole cell stays one branch-free block the scheduler can interleave
  {
    const C ux_m = UX(-1, 0);
    const C ux_jm = UX(0, -1), ux_jp = UX(0, 1);
    const C ux_km = MUX(0), ux_kp = NUX(0);
    const C uy_m0 = UY(-1, 0), uy_m1 = UY(-1, 1);
    const C uz_m0 = UZ(-1, 0), uz_m1 = NUZ(-1, 0);
    C e, gi;
    // advection (ux.c:92-186): invj (l q_m + c q_0 + u q_p) with c = -l - u,
    // l = -0.5 (a q_m' + a' q_0'), u = 0.5 (...), as differences from q_0
    e = (q.xa1 * ux_m + q.xa2 * ux_0) * (ux_m - ux_0) - (q.xa2 * ux_0 + q.xa3 * ux_p) * (ux_p - ux_0);
    e += (q.yb1 * uy_m0 + q.yb2 * uy_00) * (ux_jm - ux_0) - (q.yb1 * uy_m1 + q.yb2 * uy_01) * (ux_jp - ux_0);
    e += (q.zc1 * uz_m0 + q.zc2 * uz_00) * (ux_km - ux_0) - (q.zc1 * uz_m1 + q.zc2 * uz_01) * (ux_kp - ux_0);
    // centrifugal term (:194-226): invj hd (uy averaged to the face)^2
    const C sm = uy_m0 + uy_m1, sp = uy_00 + uy_01;
    e += q.h1 * sm * sm + q.h2 * sp * sp;
    // cross diffusion (:266-375): diffusion_y1 and the uy part of diffusion_a
    // as differences of uy across j, the ux part of diffusion_a, diffusion_z1
    e += q.cy1 * (uy_m1 - uy_m0) + q.cy2 * (uy_01 - uy_00) + q.ca1 * (ux_m + ux_0) +
         q.ca2 * (ux_0 + ux_p) + q.cz1 * ((uz_01 - uz_m1) - (uz_00 - uz_m0));   // coefficients carry nu
    // pressure gradient (:377-394)
    gi = -q.px * (C)(PP(0, 0) - PP(-1, 0));
    ROUTE(ix, q.lxl * (ux_m - ux_0) + q.lxu * (ux_p - ux_0));        // carries 2 nu
    ROUTE(iy, q.ly * ((ux_jm - ux_0) + (ux_jp - ux_0)));             // carries nu
    ROUTE(iz, nu * (ZL * ux_km + ZC * ux_0 + ZU * ux_kp));
    if constexpr (IMPL == -2) e += (i >= 2) ? (C)ss.frc[VUX][qf] : C(0);   // closure forcing
    if (i >= 2) ss.new_[VUX][qf] = (T)e;
    dl[0] = (i >= 2) ? (double)(ca * e + cb * old_x + cg * gi) : 0.;
  }
  {
    const C t_0 = TT(0, 0);
    const C tim = TT(-1, 0), tip = TT(1, 0), tjm = TT(0, -1), tjp = TT(0, 1);
    const C tkm = MTT(), tkp = NTT(0);
    C e, gi = 0;
    // advection (t.c:88-116) with face velocities ux_0, ux_p, uy_00, uy_01, uz_00, uz_01
    e = q.tx0 * ux_0 * (tim - t_0) - q.tx1 * ux_p * (tip - t_0);
    e += q.ty * uy_00 * (tjm - t_0) - q.ty * uy_01 * (tjp - t_0);
    e += q.tz * uz_00 * (tkm - t_0) - q.tz * uz_01 * (tkp - t_0);
    ROUTE(ix, rpr * (qc_.lxl * (tim - t_0) + qc_.lxu * (tip - t_0)));   // nu kappa/nu
    ROUTE(iy, rpr * (qc_.ly * ((tjm - t_0) + (tjp - t_0))));
    ROUTE(iz, kappa * (ZL * tkm + ZC * t_0 + ZU * tkp));
    ss.new_[VT][qc] = (T)e;
    dl[1] = ca * e + cb * old_t + cg * gi;
    u0[1] = t_0;
  }
  u0[0] = ux_0;
}

// Group B: right-hand sides of uy (src/fluid/predict/uy.c) and uz (uz.c) at
// centre i of cell (i, j, k); increments dl[0] (uy), dl[1] (uz), current
// values u0[0], u0[1].
template <int JT, int RL, int JL, int IMPL, class T, class C>
__device__ __forceinline__ void cell_b(const CoefB<C> & q, const SlotView<T> & V, const Bc & bc,
                                       const Coefs & cf, const CoefZ<C> & lz, C nu, int i, size_t qc,
                                       const SrcSetT<T> & ss,
                                       C ca, C cb, C cg, C old_y, C old_z, double dl[2], double u0[2]) {
  const bool ix = IMPL >= 0 ? (IMPL & 1) != 0 : bc.implicit[0] != 0;
  const bool iy = IMPL >= 0 ? (IMPL & 2) != 0 : bc.implicit[1] != 0;
  const bool iz = IMPL >= 0 ? (IMPL & 4) != 0 : bc.implicit[2] != 0;
  const C ux_0 = UX(0, 0), ux_1 = UX(1, 0);
  const C uy_0 = UY(0, 0), uy_jp = UY(0, 1);
  const C uz_0 = UZ(0, 0), uz_kp = NUZ(0, 0);
  const double p_0 = PP(0, 0);   // p is double in both modes
  {  // uy
    const C uy_im = UY(-1, 0), uy_ip = UY(1, 0), uy_jm = UY(0, -1);
    const C uy_km = MUY(0), uy_kp = NUY(0);
    const C ux_0m = UX(0, -1), ux_1m = UX(1, -1);
    const C uz_jm = UZ(0, -1), uz_jmkp = NUZ(0, -1);
    C e, gi;
    // advection (uy.c:93-180), as differences from uy_0
    e = q.a1 * (ux_0m + ux_0) * (uy_im - uy_0) - q.a2 * (ux_1m + ux_1) * (uy_ip - uy_0);
    e += q.b * (uy_jm + uy_0) * (uy_jm - uy_0) - q.b * (uy_0 + uy_jp) * (uy_jp - uy_0);
    e += q.c * (uz_jm + uz_0) * (uy_km - uy_0) - q.c * (uz_jmkp + uz_kp) * (uy_kp - uy_0);
    // advection_1 (:188-223): -invjc hd (uy ux averaged to j -/+ 1/2)
    e -= q.h * ((uy_jm + uy_0) * (ux_0m + ux_1m) + (uy_0 + uy_jp) * (ux_0 + ux_1));
    // diffusion_x1 + diffusion_a (lyx at faces i, i+1 and lxy), diffusion_y1
    // (lyy1 at j-1, j), diffusion_z1 (lyz at k, k+1)
    e += q.p1 * (ux_0 - ux_0m) + q.p2 * (ux_1 - ux_1m) + q.qm * uy_im + q.q0 * uy_0 + q.qp * uy_ip +
         q.yk * ((ux_0 + ux_1) - (ux_0m + ux_1m)) + q.yz * ((uz_kp - uz_jmkp) - (uz_0 - uz_jm));   // carry nu
    gi = -q.py * (C)(p_0 - PP(0, -1));
    ROUTE(ix, q.lxl * (uy_im - uy_0) + q.lxu * (uy_ip - uy_0));      // carry nu
    ROUTE(iy, C(2) * (q.ly * ((uy_jm - uy_0) + (uy_jp - uy_0))));
    ROUTE(iz, nu * (ZL * uy_km + ZC * uy_0 + ZU * uy_kp));
    if constexpr (IMPL == -2) e += (C)ss.frc[VUY][qc];
    ss.new_[VUY][qc] = (T)e;
    dl[0] = ca * e + cb * old_y + cg * gi;
  }
  {  // uz
    const C uz_im = UZ(-1, 0), uz_ip = UZ(1, 0), uz_jm = UZ(0, -1), uz_jp = UZ(0, 1);
    const C uz_km = MUZ();
    const C uy_km = MUY(0), uy_jpkm = MUY(1);
    const C ux_0k = MUX(0), ux_1k = MUX(1);
    C e, gi;
    // advection (uz.c:88-180), as differences from uz_0
    e = q.a1 * (ux_0k + ux_0) * (uz_im - uz_0) - q.a2 * (ux_1k + ux_1) * (uz_ip - uz_0);
    e += q.b * (uy_km + uy_0) * (uz_jm - uz_0) - q.b * (uy_jpkm + uy_jp) * (uz_jp - uz_0);
    e += q.c * (uz_km + uz_0) * (uz_km - uz_0) - q.c * (uz_0 + uz_kp) * (uz_kp - uz_0);
    // diffusion_x1 (lzx at faces i, i+1), diffusion_y1 (lzy at j, j+1)
    e += q.zx1 * (ux_1 - ux_1k) - q.zx0 * (ux_0 - ux_0k) + q.zy * ((uy_jp - uy_jpkm) - (uy_0 - uy_km));   // carry nu
    gi = -ZIH * (C)(p_0 - MPP());
    ROUTE(ix, q.lxl * (uz_im - uz_0) + q.lxu * (uz_ip - uz_0));
    ROUTE(iy, q.ly * ((uz_jm - uz_0) + (uz_jp - uz_0)));
    ROUTE(iz, C(2) * nu * (ZL * uz_km + ZC * uz_0 + ZU * uz_kp));
    if constexpr (IMPL == -2) e += (C)ss.frc[VUZ][qc];
    ss.new_[VUZ][qc] = (T)e;
    dl[1] = ca * e + cb * old_z + cg * gi;
  }
  u0[0] = uy_0;
  u0[1] = uz_0;
}
#undef ZL
#undef ZC
#undef ZU
#undef ZIH
#undef ROW_
#undef ODD_
#undef UX
#undef UY
#undef UZ
#undef TT
#undef PP
#undef NUX
#undef NUY
#undef NUZ
#undef NTT
#undef MPP
#undef MTT
#undef MUZ
#undef MUY
#undef MUX
#undef ROUTE

template <int E>
__device__ __forceinline__ int spad(int e) { return E > 1 ? e + e / E : e; }

struct Aff { double a, b; };

// Lane's chunk of a factor row: the E values of elements lane E .. lane E + E-1
// (rows hold at least 32 E values).
template <int E>
__device__ __forceinline__ void load_chunk(double (&r)[E], const double * __restrict__ row, int lane) {
  // rows are stored interleaved (element lane E + m at m 32 + lane): one
  // coalesced 256-byte load per m
#pragma unroll
  for (int m = 0; m < E; m++) r[m] = LD(row + m * 32 + lane);
}

// Radial Thomas solve of one line by one warp (src/tdm.c:24-48): lane t owns
// elements tE .. tE+E-1. The forward sweep q_m = w_m (r_m - l_m q_{m-1}) is the
// affine map q_{m-1} -> fa_m q_{m-1} + fb_m with fa = -w l, fb = w r; each lane
// composes its maps, a 5-level shuffle scan supplies the value entering its
// chunk, and the chunk's q follow from (fa, fb). The back substitution
// x_m = q_m - v_m x_{m+1} runs the same way from the other end. The factor rows
// have w[0] = 1 / c[0] and l[0] = 0, and zeros from n on; the staging line is
// zero from n on as well, so elements past the end map to zero without tests.
// Only (fa, fb), then (q, v), stay live across a scan.
template <int E>
__device__ __forceinline__ void solve_line(double * sb, const double * __restrict__ lrow,
                                           const double * __restrict__ wrow, const double * __restrict__ vrow,
                                           int lane) {
  double fa[E], fb[E];
  {
    double ll[E], ww[E];
    load_chunk<E>(ll, lrow, lane);
    load_chunk<E>(ww, wrow, lane);
#pragma unroll
    for (int m = 0; m < E; m++) {
      fa[m] = -ww[m] * ll[m];
      fb[m] = ww[m] * sb[spad<E>(lane * E + m)];
    }
  }
  Aff acc{1., 0.};
#pragma unroll
  for (int m = 0; m < E; m++) {
    acc.b = fa[m] * acc.b + fb[m];
    acc.a = fa[m] * acc.a;
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double oa = __shfl_up_sync(0xffffffffu, acc.a, off);
    const double ob = __shfl_up_sync(0xffffffffu, acc.b, off);
    if (lane >= off) { acc.b = acc.a * ob + acc.b; acc.a = acc.a * oa; }
  }
  double qin = __shfl_up_sync(0xffffffffu, acc.b, 1);
  if (lane == 0) qin = 0.;
  double * q = fb;
#pragma unroll
  for (int m = 0; m < E; m++) {
    q[m] = fa[m] * qin + fb[m];
    qin = q[m];
  }
  double vv[E];
  load_chunk<E>(vv, vrow, lane);
  Aff bac{1., 0.};
#pragma unroll
  for (int m = E - 1; m >= 0; m--) {
    bac.b = -vv[m] * bac.b + q[m];
    bac.a = -vv[m] * bac.a;
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
    const double x = q[m] - vv[m] * xin;
    sb[spad<E>(lane * E + m)] = x;
    xin = x;
  }
}

// Thread roles. The CTA is NRW "field" warps (one thread per radial index,
// whole warpgroups) followed by one warpgroup of four "solve" warps (warp v
// solves variable v of the CTA's lines). Per plane k the field warps form the
// right-hand sides and increments of every cell and hand them to the solve
// warps through a double-buffered staging area (mbarrier full[k & 1]); while
// the solve warps run the radial systems of plane k, the field warps go on to
// plane k + 1 and then take plane k's solutions back (mbarrier done[k & 1]) to
// add them to the values they kept and store the new fields. So no block-wide
// barrier separates the right-hand sides from the solves.
//
// Shared memory, in bytes, shared by the kernel and its launcher. Row buffers
// are sized for the widest radial line of the warp count (nx <= 32 NW), so
// every stencil offset is a compile-time constant. A ring slot holds the field
// rows (storage type T) and the p rows (double) of one plane; the previous
// substep's source terms of the CTA's lines arrive one plane ahead by bulk
// copies into a two-plane buffer of their own.
template <int NW, int JT, class T>
struct MarchLayout {
  static_assert(JT == 2, "line pairs start at odd j, so rows of even index have even j");
  static constexpr int E = NW;
  static constexpr int NSLOT = 4;                             // planes k .. k+3 in the ring
  static constexpr int RL = 32 * NW + 4;                      // values per row: >= nx + 4, multiple of 4
  static constexpr int NRW = NW < 4 ? 4 : NW;                 // field warps
  static constexpr int NRT = 32 * NRW;
  static constexpr int THREADS = NRT + 128;                   // + the solve warpgroup
  static constexpr int NFROW = 4 * (JT + 2);                  // ux, uy, uz, t: JT + 2 rows each
  static constexpr size_t POFF = (size_t)NFROW * RL * sizeof(T);          // p: JT + 1 rows of double
  static constexpr size_t SLOT = POFF + (size_t)(JT + 1) * RL * sizeof(double);
  static constexpr int SL = 32 * E + (E > 1 ? 32 : 0);        // staging line (padded for the solves)
  static constexpr size_t STAGE = NSLOT * SLOT;               // [2][JT][4][SL] doubles after the ring
  static constexpr int OL = 32 * NW;                          // old source terms per line and variable
  static constexpr size_t OLDS = STAGE + sizeof(double) * 2 * JT * 4 * SL;   // [2][4][JT OL] T
  static constexpr size_t BAR = OLDS + sizeof(T) * 2 * 4 * JT * OL;
  // mbarriers: NSLOT ring slots, full[2], done[2], olds[2]; then the abort
  // flag, the last plane issued and a release counter per slot
  static constexpr int NBAR = NSLOT + 6;
  static constexpr size_t BYTES = BAR + NBAR * sizeof(unsigned long long) + 8 + 4 * NSLOT;
  // registers per thread at launch, and after the split (field, solve): the
  // warpgroups' shares add up to the launch total (THREADS x REGS)
  static constexpr int REGS = NRW == 8 ? 168 : 0;
  static constexpr int REGS_FIELD = 200, REGS_SOLVE = 104;
  static_assert(REGS == 0 || NRT * REGS_FIELD + 128 * REGS_SOLVE <= THREADS * REGS, "register split");
};

// Everything the roles need besides their coefficients.
template <class T>
struct MarchArgs {
  Geo g;
  Bc bc;
  Coefs cf;
  XFactors xf;
  double nu, kappa;
  FieldsT<T> in, out;
  SrcSetT<T> ss;
  DeltaSet ds;
  int rkstep, mode, KC;
  unsigned * status;
};

__device__ __forceinline__ void mbar_arrive(unsigned long long * bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// barrier among the field warps only (id 1; id 0 is __syncthreads)
template <int N>
__device__ __forceinline__ void field_barrier() {
  asm volatile("bar.sync 1, %0;" ::"n"(N) : "memory");
}

// the slot of plane kp and the parity of its fill (planes k0 - 1 .. k1 pass
// through the NSLOT slots in turn)
__device__ __forceinline__ int slot_of(int kp, int k0, int nslot) { return (kp - k0 + 1) % nslot; }
__device__ __forceinline__ unsigned fill_parity(int kp, int k0, int nslot) { return ((kp - k0 + 1) / nslot) & 1u; }

// The field warps: one thread per radial index i of the CTA's JT lines.
// TILE: radial lines longer than the field warps (nx > 32 NW). The CTA then
// covers the radial indices ib + 1 .. ib + NRT of its lines (ib = tile x NRT),
// its rows hold i = ib .. ib + NRT + 1 (ux faces ib .. ib + NRT + 1), the old
// source terms are read from global memory, and the increments go to the
// delta buffers before any radial solve (a separate line solve follows).
template <int NW, int JT, int IMPL, class T, bool TILE = false>
__device__ __forceinline__ void march_fields(const MarchArgs<T> & A, char * ring, double * stage, T * olds,
                                             unsigned long long * bar, volatile int * abort_flag,
                                             int * release_cnt, volatile int * issued_p, int j0, int k0, int k1,
                                             double dt, int ib = 0) {
  using L = MarchLayout<NW, JT, T>;
  constexpr int E = L::E, RL = L::RL, SL = L::SL, NS = L::NSLOT, OL = L::OL;
  const Geo & g = A.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tx = threadIdx.x;
  const int i = ib + tx + 1;
  const bool act = i <= nx;
  unsigned long long * full = bar + NS;
  unsigned long long * done = bar + NS + 2;
  unsigned long long * obar = bar + NS + 4;
  // element offsets in the widened copies of even and odd rows: ux (fe, of),
  // centre fields (0, oc) and p (0, op); none in the FP32 layout, whose rows
  // and tiles start on 16-byte boundaries. A tile's rows start at centre
  // index ib (even) and ux face ib (element ib - 1).
  constexpr bool D64 = sizeof(T) == 8;
  const int e0f = (D64 && ib > 0) ? ib - 1 : ib;   // first ux element of the tile's rows
  const int fe = D64 ? e0f & 1 : 0;
  const int of = D64 ? ((nx + 1) & 1) ^ (e0f & 1) : 0, oc = D64 ? (nx + 2) & 1 : 0, op = (nx + 2) & 1;
  const int fsh = (D64 && ib == 0) ? 1 : 0;   // ux face i at smem element i - ib - fsh of its row
  const size_t sjc = (size_t)ny + 2;
  auto frow = [&](char * slot, int f, int r) { return reinterpret_cast<T *>(slot) + (size_t)(f * (JT + 2) + r) * RL; };
  auto prow = [&](char * slot, int r) { return reinterpret_cast<double *>(slot + L::POFF) + (size_t)r * RL; };

  // Copies of plane kp into slot sl: every row of the five arrays (4 = p, in
  // double), widened to 16-byte bounds; one thread counts the bytes, expects
  // them on the slot's mbarrier and issues the copies.
  auto issue = [&](int kp, int sl) {
    char * base = ring + (size_t)sl * L::SLOT;
    const char * src[5] = {reinterpret_cast<const char *>(A.in.ux), reinterpret_cast<const char *>(A.in.uy),
                           reinterpret_cast<const char *>(A.in.uz), reinterpret_cast<const char *>(A.in.t),
                           reinterpret_cast<const char *>(A.in.p)};
    auto all = [&](bool go, unsigned & total) {
      for (int f = 0; f < 5; f++) {
        const size_t es = f == SF_P ? sizeof(double) : sizeof(T), al = 16 / es;
        const size_t len = (f == SF_P || (D64 && f != SF_UX)) ? (size_t)nx + 2 : D64 ? (size_t)nx + 1 : (size_t)pitch32(nx);
        // the part of the row the tile reads (the whole row without tiles)
        const size_t e0 = f == SF_UX ? (size_t)e0f : (size_t)ib;
        const size_t want = (f == SF_UX && D64) ? (size_t)L::NRT + 1 + (ib > 0 ? 1 : 0) : (size_t)L::NRT + 2;
        const size_t n = TILE ? (len - e0 < want ? len - e0 : want) : len;
        for (int r = 0; r < (f == SF_P ? JT + 1 : JT + 2); r++) {
          const size_t s0 = len * ((size_t)(j0 - 1 + r) + sjc * kp) + (TILE ? e0 : 0);
          const size_t a = s0 & ~(al - 1), b = (s0 + n + al - 1) & ~(al - 1);
          const unsigned by = (unsigned)((b - a) * es);
          const size_t off = (D64 || f != SF_P) ? (size_t)(f * (JT + 2) + r) * RL * sizeof(T)
                                                : L::POFF + (size_t)r * RL * sizeof(double);
          if (go) bulk_g2s(base + off, src[f] + a * es, by, &bar[sl]);
          else total += by;
        }
      }
    };
    unsigned total = 0;
    all(false, total);
    mbar_expect_tx(&bar[sl], total);
    all(true, total);
  };
  // bounded wait; after any wait of the CTA has given up, no thread waits any
  // more (the CTA runs to its end without storing anything)
  auto wait = [&](unsigned long long * b, unsigned parity) {
    if (*abort_flag) return false;
    if (mbar_wait(b, parity)) return true;
    *abort_flag = 1;
    return false;
  };
  if (tx == 0) {
    for (int s = 0; s < NS && k0 - 1 + s <= k1; s++) issue(k0 - 1 + s, s);
    *issued_p = k0 - 2 + (k1 - k0 + 2 < NS ? k1 - k0 + 2 : NS);
  }

  // the previous substep's source terms of the CTA's lines, one plane ahead:
  // the JT lines of a variable are consecutive in the packed layout and start
  // on a 16-byte boundary (even line index), so one bulk copy per variable
  const bool use_old = A.rkstep != 0;
  const int lf = D64 ? nx - 1 : spitch32(nx), lc = D64 ? nx : spitch32(nx);   // source-term lines (sline)
  auto fetch_olds = [&](int kp, int buf) {
    const unsigned total = (unsigned)((size_t)JT * (lf + 3 * lc) * sizeof(T));
    mbar_expect_tx(&obar[buf], total);
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int li = v == VUX ? lf : lc;
      bulk_g2s(olds + (size_t)(buf * 4 + v) * JT * OL, A.ss.old_[v] + pidx(li, ny, 0, j0, kp),
               (unsigned)((size_t)JT * li * sizeof(T)), &obar[buf]);
    }
  };
  const bool olds_smem = use_old && !TILE;   // tiles read the old terms from global memory
  if (tx == 0 && olds_smem) {
    fetch_olds(k0, 0);
    if (k0 + 1 < k1) fetch_olds(k0 + 1, 1);
  }

  // arithmetic type of the right-hand sides
  using C = typename std::conditional<sizeof(T) == 4 && TC_MARCH_FP32_ARITH, float, double>::type;
  CoefA<C> qa;
  CoefB<C> qb;
  load_coefs(qa, A.cf, act ? i : 1);
  load_coefs(qb, A.cf, act ? i : 1);
  const CoefZ<C> qz{(C)A.cf.lz_l, (C)A.cf.lz_c, (C)A.cf.lz_u, (C)A.cf.inv_hz};
  // the diffusivities folded into the per-thread coefficients once, so the
  // cell updates multiply by them no more (the z Laplacian, a shared scalar
  // set, keeps its factor)
  {
    const C nu = (C)A.nu, n2 = (C)(2. * A.nu);
    qa.lxl *= n2; qa.lxu *= n2; qa.ly *= nu;
    qa.cy1 *= nu; qa.cy2 *= nu; qa.ca1 *= nu; qa.ca2 *= nu; qa.cz1 *= nu;
    qb.lxl *= nu; qb.lxu *= nu; qb.ly *= nu;
    qb.p1 *= nu; qb.p2 *= nu; qb.qm *= nu; qb.q0 *= nu; qb.qp *= nu; qb.yk *= nu; qb.yz *= nu;
    qb.zx0 *= nu; qb.zx1 *= nu; qb.zy *= nu;
  }
  const C rpr = (C)(A.kappa / A.nu);   // the scalar's Laplacians use the centred tables with kappa
  const int rk = A.rkstep;
  const C ca = (C)(rk_alpha(rk) * dt), cb = (C)(rk_beta(rk) * dt), cg = (C)(rk_gamma(rk) * dt);
  const C nu_c = (C)A.nu, kappa_c = (C)A.kappa;

  // planes k0 - 1 and k0
  wait(&bar[0], 0);
  wait(&bar[1], 0);

  // u += delta into the other buffer, walls (boundary/*.c) and images
  // (halo.c); or the increments themselves (planar y / z solves follow)
  auto store = [&](int k, const double (&dl)[JT][4], const double (&u0)[JT][4]) {
    if (!act || *abort_flag) return;
#pragma unroll
    for (int jl = 0; jl < JT; jl++) {
      const int j = j0 + jl;
      if (A.mode == PREDICT_DELTA) {
        const size_t qc = pidx(nx, ny, i - 1, j, k);
        if (i >= 2) A.ds.d[VUX][pidx(nx - 1, ny, i - 2, j, k)] = dl[jl][VUX];
        A.ds.d[VT][qc] = dl[jl][VT];
        A.ds.d[VUY][qc] = dl[jl][VUY];
        A.ds.d[VUZ][qc] = dl[jl][VUZ];
        continue;
      }
      const double vx = (i < 2) ? 0. : u0[jl][VUX] + dl[jl][VUX];
      const double vt = u0[jl][VT] + dl[jl][VT];
      const double vy = u0[jl][VUY] + dl[jl][VUY];
      const double vz = u0[jl][VUZ] + dl[jl][VUZ];
      auto put = [&](int jj, int kk) {
        A.out.ux[sidx_f<T>(g, i, jj, kk)] = (T)vx;
        A.out.t[sidx_c<T>(g, i, jj, kk)] = (T)vt;
        A.out.uy[sidx_c<T>(g, i, jj, kk)] = (T)vy;
        A.out.uz[sidx_c<T>(g, i, jj, kk)] = (T)vz;
        if (i == 1) {
          A.out.t[sidx_c<T>(g, 0, jj, kk)] = (T)A.bc.t_xm;
          A.out.uy[sidx_c<T>(g, 0, jj, kk)] = (T)A.bc.uy_xm;
          A.out.uz[sidx_c<T>(g, 0, jj, kk)] = (T)0.;
        }
        if (i == nx) {
          A.out.ux[sidx_f<T>(g, nx + 1, jj, kk)] = (T)0.;
          A.out.t[sidx_c<T>(g, nx + 1, jj, kk)] = (T)A.bc.t_xp;
          A.out.uy[sidx_c<T>(g, nx + 1, jj, kk)] = (T)A.bc.uy_xp;
          A.out.uz[sidx_c<T>(g, nx + 1, jj, kk)] = (T)0.;
        }
      };
      put(j, k);
      for_images(j, k, ny, nz, put);
    }
  };
  // staging positions: ux unknowns are faces 2..nx (element i - 2), the
  // centred ones cells 1..nx (element i - 1)
  auto stage_pos = [&](int v) { return v == VUX ? spad<E>(i - 2) : spad<E>(i - 1); };
  // plane k's solutions from the solve warps, added to the values kept
  auto finish_plane = [&](int k, int step, const double (&u0)[JT][4]) {
    const int b = step & 1;
    wait(&done[b], (unsigned)(step >> 1) & 1u);
    double x[JT][4];
    const double * sdb = stage + (size_t)b * JT * 4 * SL;
#pragma unroll
    for (int jl = 0; jl < JT; jl++)
#pragma unroll
      for (int v = 0; v < 4; v++)
        x[jl][v] = (act && (v != VUX || i >= 2)) ? sdb[(size_t)(jl * 4 + v) * SL + stage_pos(v)] : 0.;
    store(k, x, u0);
  };

  // tiles leave the radial solve to the line kernel that follows
  const bool solve_x = !TILE && (IMPL >= 0 ? (IMPL & 1) != 0 : A.bc.implicit[0] != 0);
  double up[JT][4];   // values of the previous plane's cells, until its solutions arrive
  for (int k = k0; k < k1; k++) {
    const int step = k - k0;
    wait(&bar[slot_of(k + 1, k0, NS)], fill_parity(k + 1, k0, NS));
    if (olds_smem) wait(&obar[step & 1], (unsigned)(step >> 1) & 1u);
    double dl[JT][4], u0[JT][4];   // indexed by Var
#pragma unroll
    for (int jl = 0; jl < JT; jl++)
#pragma unroll
      for (int v = 0; v < 4; v++) dl[jl][v] = u0[jl][v] = 0.;
    if (act) {
      char * ms = ring + (size_t)slot_of(k - 1, k0, NS) * L::SLOT;
      char * cs = ring + (size_t)slot_of(k, k0, NS) * L::SLOT;
      char * ns = ring + (size_t)slot_of(k + 1, k0, NS) * L::SLOT;
      SlotView<T> V;
      const int is = i - ib;   // the cell's element in the tile's rows
      V.cb = reinterpret_cast<const T *>(cs) + is;
      V.cbo = V.cb + oc;
      V.fb = V.cb - fsh + fe;
      V.fbo = V.cb - fsh + of;
      V.nb = reinterpret_cast<const T *>(ns) + is;
      V.nbo = V.nb + oc;
      V.nf = V.nb - fsh + fe;
      V.nfo = V.nb - fsh + of;
      V.mb = reinterpret_cast<const T *>(ms) + is;
      V.mbo = V.mb + oc;
      V.mf = V.mb - fsh + fe;
      V.mfo = V.mb - fsh + of;
      if constexpr (D64) {   // p rows follow the field rows: same base registers, constant offsets
        V.pb = reinterpret_cast<const double *>(V.cb) + L::NFROW * RL;
        V.pbo = reinterpret_cast<const double *>(V.cbo) + L::NFROW * RL;
        V.mp = reinterpret_cast<const double *>(V.mb) + L::NFROW * RL;
        V.mpo = reinterpret_cast<const double *>(V.mbo) + L::NFROW * RL;
      } else {
        V.pb = prow(cs, 0) + is;
        V.pbo = V.pb + op;
        V.mp = prow(ms, 0) + is;
        V.mpo = V.mp + op;
      }
      const size_t qf = pidx(lf, ny, i - 2, j0, k), qc = pidx(lc, ny, i - 1, j0, k);
      const T * ob = olds + (size_t)(step & 1) * 4 * JT * OL;   // this plane's old terms
      auto cells = [&](auto jlc) {
        constexpr int JL = decltype(jlc)::value;
        double d2[2], w2[2];
        auto old = [&](int v) {
          if (!use_old) return 0.;
          if constexpr (TILE) {   // from global memory (ux at i = 1 has none)
            if (v == VUX && i < 2) return 0.;
            const int li = v == VUX ? lf : lc;
            return (double)A.ss.old_[v][pidx(li, ny, v == VUX ? i - 2 : i - 1, j0 + JL, k)];
          } else {
            return (double)ob[(size_t)v * JT * OL + JL * (v == VUX ? lf : lc) + (v == VUX ? i - 2 : i - 1)];
          }
        };
        // old(VUX) at i = 1 reads the shared-memory word before the line (discarded)
        cell_a<JT, RL, JL, IMPL>(qa, qb, V, A.bc, A.cf, qz, nu_c, kappa_c, rpr, i, qf + (size_t)JL * lf,
                                 qc + (size_t)JL * lc, A.ss, ca, cb, cg, (C)old(VUX), (C)old(VT), d2, w2);
        dl[JL][VUX] = d2[0]; dl[JL][VT] = d2[1]; u0[JL][VUX] = w2[0]; u0[JL][VT] = w2[1];
        cell_b<JT, RL, JL, IMPL>(qb, V, A.bc, A.cf, qz, nu_c, i, qc + (size_t)JL * lc, A.ss, ca, cb, cg,
                                 (C)old(VUY), (C)old(VUZ), d2, w2);
        dl[JL][VUY] = d2[0]; dl[JL][VUZ] = d2[1]; u0[JL][VUY] = w2[0]; u0[JL][VUZ] = w2[1];
      };
      cells(std::integral_constant<int, 0>());
      cells(std::integral_constant<int, 1>());
    }
    // This warp is done with the slot of plane k - 1 and with the old terms'
    // buffer of plane k; the last field warp to get here refills them with
    // planes k + 3 and k + 2 (no warp waits for the others).
    __syncwarp();
    if ((tx & 31) == 0) {
      __threadfence_block();
      int * cnt = release_cnt + slot_of(k - 1, k0, NS);
      if (atomicAdd(cnt, 1) == L::NRW - 1) {
        *cnt = 0;
        __threadfence_block();
        if (!*abort_flag) {
          fence_async_smem();
          if (k + 3 <= k1) {
            issue(k + 3, slot_of(k + 3, k0, NS));
            *issued_p = k + 3;
          }
          if (olds_smem && k + 2 < k1) fetch_olds(k + 2, step & 1);
        }
      }
    }
    if (solve_x) {
      const int b = step & 1;
      double * sdb = stage + (size_t)b * JT * 4 * SL;
      if (act) {
#pragma unroll
        for (int jl = 0; jl < JT; jl++)
#pragma unroll
          for (int v = 0; v < 4; v++)
            if (v != VUX || i >= 2) sdb[(size_t)(jl * 4 + v) * SL + stage_pos(v)] = dl[jl][v];
      }
      mbar_arrive(&full[b]);
      if (step > 0) finish_plane(k - 1, step - 1, up);
#pragma unroll
      for (int jl = 0; jl < JT; jl++)
#pragma unroll
        for (int v = 0; v < 4; v++) up[jl][v] = u0[jl][v];
    } else {
      store(k, dl, u0);
    }
  }
  if (solve_x) finish_plane(k1 - 1, k1 - 1 - k0, up);
  field_barrier<L::NRT>();   // every issue is done
  if (*abort_flag && tx == 0) {
    // copies may still be in flight into the ring and the olds buffers: wait,
    // bounded, for the latest fill of each before the CTA exits
    const int issued = *issued_p;
    for (int kp = (issued - NS + 1 > k0 - 1 ? issued - NS + 1 : k0 - 1); kp <= issued; kp++)
      mbar_wait(&bar[slot_of(kp, k0, NS)], fill_parity(kp, k0, NS));
    if (olds_smem) {
      for (int kp = k1 - 2 > k0 ? k1 - 2 : k0; kp < k1; kp++)
        mbar_wait(&obar[(kp - k0) & 1], (unsigned)((kp - k0) >> 1) & 1u);
    }
  }
}

// The solve warpgroup: warp v solves variable v of the CTA's JT lines, plane
// after plane.
template <int NW, int JT, class T>
__device__ __forceinline__ void march_solves(const MarchArgs<T> & A, double * stage, unsigned long long * bar,
                                             volatile int * abort_flag, int KC) {
  using L = MarchLayout<NW, JT, T>;
  constexpr int E = L::E, SL = L::SL, NS = L::NSLOT;
  const int lane = threadIdx.x & 31;
  const int v = (threadIdx.x - L::NRT) >> 5;
  unsigned long long * full = bar + NS;
  unsigned long long * done = bar + NS + 2;
  const size_t fo = (size_t)(A.rkstep * 4 + v) * A.xf.stride;
  for (int step = 0; step < KC; step++) {
    const int b = step & 1;
    if (!*abort_flag && !mbar_wait(&full[b], (unsigned)(step >> 1) & 1u)) *abort_flag = 1;
    double * sdb = stage + (size_t)b * JT * 4 * SL;
    // one line at a time; the factor rows (6 KB per variable) stay in L1
#pragma unroll 1
    for (int jl = 0; jl < JT; jl++)
      solve_line<E>(sdb + (size_t)(jl * 4 + v) * SL, A.xf.lo + fo, A.xf.w + fo, A.xf.v + fo, lane);
    mbar_arrive(&done[b]);
  }
}

template <int R>
__device__ __forceinline__ void regs_inc() { asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(R)); }
template <int R>
__device__ __forceinline__ void regs_dec() { asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(R)); }

// CTA = JT lines (j0 .. j0+JT-1) x KC planes; field warps and the solve
// warpgroup as above.
template <int NW, int JT, int IMPL, class T, bool TILE = false>
__global__ void __launch_bounds__(MarchLayout<NW, JT, T>::THREADS, 1)
march_predict_kernel(MarchArgs<T> A, const double * __restrict__ dtp) {
  using L = MarchLayout<NW, JT, T>;
  extern __shared__ __align__(16) double sm[];
  char * ring = reinterpret_cast<char *>(sm);
  double * stage = reinterpret_cast<double *>(ring + L::STAGE);
  T * olds = reinterpret_cast<T *>(ring + L::OLDS);
  unsigned long long * bar = reinterpret_cast<unsigned long long *>(ring + L::BAR);
  volatile int * abort_flag = reinterpret_cast<volatile int *>(bar + L::NBAR);
  volatile int * issued_p = abort_flag + 1;
  int * release_cnt = const_cast<int *>(abort_flag + 2);
  const int tx = threadIdx.x;
  const int njg = A.g.ny / JT;
  const int ntile = TILE ? (A.g.nx + L::NRT - 1) / L::NRT : 1;
  const int tile = TILE ? (int)(blockIdx.x % ntile) : 0;
  const unsigned bl = TILE ? blockIdx.x / ntile : blockIdx.x;
  const int j0 = (int)(bl % njg) * JT + 1;   // odd
  const int k0 = (int)(bl / njg) * A.KC + 1;
  const int k1 = k0 + A.KC;   // planes k0 .. k1-1 are computed; k0-1 .. k1 are read
  if (tx == 0) {
    for (int s = 0; s < L::NSLOT; s++) mbar_init(&bar[s], 1);
    mbar_init(&bar[L::NSLOT + 0], L::NRT);   // full: every field thread
    mbar_init(&bar[L::NSLOT + 1], L::NRT);
    mbar_init(&bar[L::NSLOT + 2], 128);      // done: every solve thread
    mbar_init(&bar[L::NSLOT + 3], 128);
    mbar_init(&bar[L::NSLOT + 4], 1);        // olds: the issuing thread's expected bytes
    mbar_init(&bar[L::NSLOT + 5], 1);
    *abort_flag = 0;
    for (int sl = 0; sl < L::NSLOT; sl++) release_cnt[sl] = 0;
    fence_mbar_init();
  }
  // staging lines are zero past each line's unknowns for the whole march
  for (int e = tx; e < 2 * JT * 4 * L::SL; e += blockDim.x) stage[e] = 0.;
  __syncthreads();
  const double dt = *dtp;
  if (tx < L::NRT) {
    if constexpr (L::REGS > 0) regs_inc<L::REGS_FIELD>();
    march_fields<NW, JT, IMPL, T, TILE>(A, ring, stage, olds, bar, abort_flag, release_cnt, issued_p, j0, k0, k1,
                                        dt, tile * L::NRT);
  } else {
    if constexpr (L::REGS > 0) regs_dec<L::REGS_SOLVE>();
    const bool solve_x = !TILE && (IMPL >= 0 ? (IMPL & 1) != 0 : A.bc.implicit[0] != 0);
    if (solve_x) march_solves<NW, JT, T>(A, stage, bar, abort_flag, A.KC);
  }
  __syncthreads();
  if (tx == 0 && *abort_flag) atomicOr(A.status, ST_TIMEOUT);
}

#ifndef TC_MARCH_JT
#define TC_MARCH_JT 2
#endif
// Planes per CTA, at most: each CTA's start (coefficients, barriers, the first
// planes' copies) overlaps nothing at one CTA per SM, and its two halo planes
// are read twice. Smaller grids take fewer planes per CTA when the last wave
// of CTAs would leave SMs idle (march_planes).
#ifndef TC_MARCH_KC
#define TC_MARCH_KC 64
#endif

// The largest chunk of planes, from TC_MARCH_KC down to 16, whose last partial
// wave of CTAs wastes at most 5% of the launch (at 256 x 512 x 128: 64 planes
// are 3.5 waves, 32 planes 6.9).
template <int NW, class T>
static int march_planes(const Geo & g) {
  constexpr int JT = TC_MARCH_JT;
  using L = MarchLayout<NW, JT, T>;
  static int per_sm[16], sms[16];   // per device: resident CTAs of this instance, SM count
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 15;
  if (per_sm[dev] == 0) {
    int b = 0, n = 0;
    // a failed query falls back to one CTA on 148 SMs and clears its own error
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, march_predict_kernel<NW, JT, 1, T>, L::THREADS, L::BYTES) !=
        cudaSuccess) {
      b = 0;
      cudaGetLastError();
    }
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      n = 0;
      cudaGetLastError();
    }
    sms[dev] = n > 0 ? n : 148;
    per_sm[dev] = b > 0 ? b : 1;
  }
  const long long slots = (long long)sms[dev] * per_sm[dev], lines = g.ny / JT;
  // chunks divide nz: the largest divisor of nz up to TC_MARCH_KC, then
  // smaller divisors down to 16 while the last wave is too empty (for a power
  // of two nz: halving)
  auto below = [&](int c) {   // the largest divisor of nz below c, or 0
    for (int d = c - 1; d >= 1; d--)
      if (g.nz % d == 0) return d;
    return 0;
  };
  int kc = g.nz < TC_MARCH_KC ? g.nz : TC_MARCH_KC;
  if (g.nz % kc) kc = below(kc);
  for (;;) {
    const long long nblk = lines * (g.nz / kc), waves = (nblk + slots - 1) / slots;
    if (waves * slots * 100 <= nblk * 105) break;
    const int next = below(kc);
    if (kc <= 16 || next < 16) break;
    kc = next;
  }
  return kc;
}

template <int NW, class T>
void launch_march_nw(MarchArgs<T> A, const double * dtp, cudaStream_t st) {
  constexpr int JT = TC_MARCH_JT;   // ny is even
  using L = MarchLayout<NW, JT, T>;
  A.KC = march_planes<NW, T>(A.g);
  const long long nblk = (long long)(A.g.ny / JT) * (A.g.nz / A.KC);
  const int mask = (A.bc.implicit[0] ? 1 : 0) | (A.bc.implicit[1] ? 2 : 0) | (A.bc.implicit[2] ? 4 : 0);
  const unsigned grid = (unsigned)nblk, block = L::THREADS;
  const size_t smem = L::BYTES;
  if constexpr (sizeof(T) == 8) {   // IMPL -2: run-time implicit flags plus the closure forcing
    if (A.ss.frc[0]) {
      march_predict_kernel<NW, JT, -2, T><<<grid, block, smem, st>>>(A, dtp);
      return;
    }
  }
  switch (mask) {
    case 1: march_predict_kernel<NW, JT, 1, T><<<grid, block, smem, st>>>(A, dtp); break;
    case 7: march_predict_kernel<NW, JT, 7, T><<<grid, block, smem, st>>>(A, dtp); break;
    case 0: march_predict_kernel<NW, JT, 0, T><<<grid, block, smem, st>>>(A, dtp); break;
    default: march_predict_kernel<NW, JT, -1, T><<<grid, block, smem, st>>>(A, dtp); break;
  }
}

template <int NW, class T>
void allow_march_smem() {
  constexpr int JT = TC_MARCH_JT;
  const int bytes = (int)MarchLayout<NW, JT, T>::BYTES;
  cudaFuncSetAttribute(march_predict_kernel<NW, JT, 1, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(march_predict_kernel<NW, JT, 7, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(march_predict_kernel<NW, JT, 0, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(march_predict_kernel<NW, JT, -1, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if constexpr (sizeof(T) == 8)
    cudaFuncSetAttribute(march_predict_kernel<NW, JT, -2, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if constexpr (NW == 8) {
    cudaFuncSetAttribute(march_predict_kernel<NW, JT, -1, T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if constexpr (sizeof(T) == 8)
      cudaFuncSetAttribute(march_predict_kernel<NW, JT, -2, T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           bytes);
  }
}

// radial lines longer than one CTA's field threads: tiles of 256 radial
// indices, increments to the delta buffers (the radial solve is launched
// separately), implicit flags and the closure forcing read at run time
template <class T>
void launch_march_tiles(MarchArgs<T> A, const double * dtp, cudaStream_t st) {
  constexpr int NW = 8, JT = TC_MARCH_JT;
  using L = MarchLayout<NW, JT, T>;
  A.KC = march_planes<NW, T>(A.g);
  A.mode = PREDICT_DELTA;
  const int ntile = (A.g.nx + L::NRT - 1) / L::NRT;
  const long long nblk = (long long)ntile * (A.g.ny / JT) * (A.g.nz / A.KC);
  if constexpr (sizeof(T) == 8) {
    if (A.ss.frc[0]) {
      march_predict_kernel<NW, JT, -2, T, true><<<(unsigned)nblk, L::THREADS, L::BYTES, st>>>(A, dtp);
      return;
    }
  }
  march_predict_kernel<NW, JT, -1, T, true><<<(unsigned)nblk, L::THREADS, L::BYTES, st>>>(A, dtp);
}

// Radial implicit solves of lines longer than one CTA's field threads (the
// tile mode above leaves its increments unsolved): one warp per (variable,
// j, k) line of the delta buffers, staged in shared memory, with the factor
// rows and scans of the march kernel (solve_line).
template <int E>
__global__ void __launch_bounds__(256) xsolve_kernel(Geo g, XFactors xf, int rk, DeltaSet ds) {
  extern __shared__ double xs_stage[];
  constexpr int SL = 32 * E + 32;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long lines = (long long)g.ny * g.nz;
  const long long q = (long long)blockIdx.x * 8 + w;   // (variable, line)
  if (q >= 4 * lines) return;                          // whole warps
  const int v = (int)(q / lines);
  const long long line = q % lines;
  const int n = xf.n[v];
  double * sb = xs_stage + (size_t)w * SL;
  double * d = ds.d[v] + (size_t)line * n;   // packed layout: line (j, k) holds n values
  for (int e = lane; e < 32 * E; e += 32) sb[spad<E>(e)] = e < n ? d[e] : 0.;
  __syncwarp();
  const size_t fo = (size_t)(rk * 4 + v) * xf.stride;
  solve_line<E>(sb, xf.lo + fo, xf.w + fo, xf.v + fo, lane);
  __syncwarp();
  for (int e = lane; e < n; e += 32) d[e] = sb[spad<E>(e)];
}

template <class T>
void launch_march_t(const Geo & g, const Bc & bc, const Coefs & cf, const XFactors & xf, double nu,
                    double kappa, const FieldBufs & in, const FieldBufs & out, const SrcBufs & ss,
                    const DeltaSet & ds, const double * dtp, int rkstep, int mode, unsigned * status,
                    cudaStream_t st) {
  MarchArgs<T> A{g, bc, cf, xf, nu, kappa, in.as<T>(), out.as<T>(), ss.as<T>(), ds, rkstep, mode, 0, status};
  if (g.nx > MarchLayout<8, TC_MARCH_JT, T>::NRT) {
    launch_march_tiles<T>(A, dtp, st);
    return;
  }
  switch (predict_warps(g.nx)) {
    case 1: launch_march_nw<1>(A, dtp, st); break;
    case 2: launch_march_nw<2>(A, dtp, st); break;
    case 4: launch_march_nw<4>(A, dtp, st); break;
    default: launch_march_nw<8>(A, dtp, st); break;
  }
}

}  // namespace

void launch_predict_march(const Geo & g, const Bc & bc, const Coefs & cf, const XFactors & xf, double nu,
                          double kappa, const FieldBufs & in, const FieldBufs & out, const SrcBufs & ss,
                          const DeltaSet & ds, const double * dtp, int rkstep, int mode, unsigned * status,
                          cudaStream_t st) {
  if (in.bytes == 4) launch_march_t<float>(g, bc, cf, xf, nu, kappa, in, out, ss, ds, dtp, rkstep, mode, status, st);
  else launch_march_t<double>(g, bc, cf, xf, nu, kappa, in, out, ss, ds, dtp, rkstep, mode, status, st);
}

// Self-test of the bounded waits: an mbarrier expects 16 bytes that no copy
// will ever deliver; every thread's wait must give up after kWaitCycles and the
// kernel report ST_TIMEOUT and return (the same wait the predict kernel uses).
__global__ void wait_selftest_kernel(unsigned * status) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_expect_tx(&bar, 16);   // the only arrival; its bytes never come
  __syncthreads();
  const bool ok = mbar_wait(&bar, 0);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(status, ST_TIMEOUT);
}

void launch_wait_selftest(unsigned * status, cudaStream_t st) { wait_selftest_kernel<<<1, 64, 0, st>>>(status); }

void launch_xsolve(const Geo & g, const XFactors & xf, int rkstep, const DeltaSet & ds, cudaStream_t st) {
  const long long lines = 4LL * g.ny * g.nz;
  const unsigned blocks = (unsigned)((lines + 7) / 8);
  if (xf.ne <= 16) xsolve_kernel<16><<<blocks, 256, 8 * (32 * 16 + 32) * sizeof(double), st>>>(g, xf, rkstep, ds);
  else xsolve_kernel<32><<<blocks, 256, 8 * (32 * 32 + 32) * sizeof(double), st>>>(g, xf, rkstep, ds);
}

void march_smem_limits() {
  cudaFuncSetAttribute(xsolve_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, 8 * (32 * 32 + 32) * 8);
  allow_march_smem<1, double>();
  allow_march_smem<2, double>();
  allow_march_smem<4, double>();
  allow_march_smem<8, double>();
  allow_march_smem<1, float>();
  allow_march_smem<2, float>();
  allow_march_smem<4, float>();
  allow_march_smem<8, float>();
}

}  // namespace tcgpu
