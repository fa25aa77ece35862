// Predict stage: fluid_predict_field (src/fluid/predict/main.c:35-110) for JT
// neighbouring radial lines (j .. j+JT-1) per CTA, marching through a chunk of
// KC planes in z. One pass over the fields per substep: right-hand sides of ux
// (face i), uy, uz, t (centre i), the new explicit source terms, the RK
// increment delta = dt (alpha srcA + beta srcA_prev + gamma srcG) with srcG
// (implicit diffusion + pressure gradient) kept in registers, the radial
// implicit solve (src/tdm.c:17-50), and u + delta into the other buffer of the
// pair with walls and periodic images (boundary/*.c, halo.c).
//
// Per CTA, a ring of three plane slots in shared memory holds the rows
// j-1 .. j+JT of ux, uy, uz, t, j-1 .. j+JT-1 of p and the previous
// substep's source terms of the CTA's lines for planes k and k+1, while plane
// k+2 streams in: one bulk asynchronous copy (cp.async.bulk, completion counted
// in bytes on an mbarrier) per row, issued one plane ahead by one thread.
// Values a cell needs from plane k-1 (ux at faces i, i+1; uy at rows j, j+1;
// uz, p, t at j) are the ones the same thread read one plane earlier and stay
// in registers; the metric coefficients depend on i only, are folded into one
// product per stencil term on the host (the P_* tables) and are loaded once
// per thread. The radial systems of the JT lines are solved one per warp with
// shuffle scans of affine maps.
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

namespace tcgpu {
namespace {

#define LD(p) __ldg(p)

constexpr int NSLOT = 3;
// wait limit on a plane's arrival, in SM clock cycles (about two seconds)
constexpr long long kWaitCycles = 4000000000LL;

__device__ __forceinline__ unsigned smem_u32(const void * p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long * bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long * bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long * bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false if the phase did not complete within kWaitCycles
__device__ __forceinline__ bool mbar_wait(unsigned long long * bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > kWaitCycles) return false;
  }
  return true;
}
__device__ __forceinline__ void bulk_g2s(void * dst, const void * src, unsigned bytes, unsigned long long * bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// fields of a slot, in row-block order
enum SlotField { SF_UX = 0, SF_UY = 1, SF_UZ = 2, SF_T = 3, SF_P = 4 };

// Two thread groups per radial line: group A (ux at face i, t at centre i)
// and group B (uy, uz at centre i), each with the coefficients of its own
// variables in registers, loaded once (they depend on i only). The
// coefficients are products of the metric tables taken once on the host
// (P_* tables); each is spelled out below where it is used.
struct CoefA {
  double xa1, xa2, xa3, yb1, yb2, zc1, zc2, h1, h2;   // ux advection
  double lxl, lxc, lxu, lyl, lyc, lyu;                // ux Laplacian, x and y
  double cy1, cy2, ca1, ca2, cz1, px;                 // ux cross diffusion, pressure gradient
  double tx0, tx1, ty, tz;                            // t advection
  double clxl, clxc, clxu, clyl, clyc, clyu;          // t Laplacian, x and y
};
struct CoefB {
  double a1, a2, b, c, h;                             // uy / uz advection
  double lxl, lxc, lxu, lyl, lyc, lyu;                // centred Laplacian, x and y
  double p1, p2, qm, q0, qp, yk, yz, py;              // uy cross diffusion, pressure gradient
  double zx0, zx1, zy;                                // uz cross diffusion
};

__device__ __forceinline__ void load_coefs(CoefA & q, const Coefs & cf, int i) {
  const double * __restrict__ b = cf.tab + i;
#define CF(T) LD(b + (T) * CSTRIDE)
  q.xa1 = CF(P_XA1); q.xa2 = CF(P_XA2); q.xa3 = CF(P_XA3); q.yb1 = CF(P_YB1); q.yb2 = CF(P_YB2);
  q.zc1 = CF(P_ZC1); q.zc2 = CF(P_ZC2); q.h1 = CF(P_H1); q.h2 = CF(P_H2);
  q.lxl = CF(F_LXL); q.lxc = CF(F_LXC); q.lxu = CF(F_LXU); q.lyl = CF(F_LYL); q.lyc = CF(F_LYC); q.lyu = CF(F_LYU);
  q.cy1 = CF(P_CY1); q.cy2 = CF(P_CY2); q.ca1 = CF(P_CA1); q.ca2 = CF(P_CA2); q.cz1 = CF(P_CZ1);
  q.px = CF(C_INVHXXF);
  q.tx0 = CF(P_TX0); q.tx1 = CF(P_TX1); q.ty = CF(P_TY); q.tz = CF(P_TZ);
  q.clxl = CF(C_LXL); q.clxc = CF(C_LXC); q.clxu = CF(C_LXU); q.clyl = CF(C_LYL); q.clyc = CF(C_LYC);
  q.clyu = CF(C_LYU);
#undef CF
}
__device__ __forceinline__ void load_coefs(CoefB & q, const Coefs & cf, int i) {
  const double * __restrict__ b = cf.tab + i;
#define CF(T) LD(b + (T) * CSTRIDE)
  q.a1 = CF(P_UA1); q.a2 = CF(P_UA2); q.b = CF(P_UB); q.c = CF(P_UC); q.h = CF(P_UH);
  q.lxl = CF(C_LXL); q.lxc = CF(C_LXC); q.lxu = CF(C_LXU); q.lyl = CF(C_LYL); q.lyc = CF(C_LYC); q.lyu = CF(C_LYU);
  q.p1 = CF(P_P1); q.p2 = CF(P_P2); q.qm = CF(P_QM); q.q0 = CF(P_Q0); q.qp = CF(P_QP);
  q.yk = CF(P_YK); q.yz = CF(P_YZ); q.py = CF(C_INVHYXC);
  q.zx0 = CF(P_ZX0); q.zx1 = CF(P_ZX1); q.zy = CF(P_ZY);
#undef CF
}

// values of plane k-1 a cell needs, carried from the previous plane
struct PrevA { double ux0, t0; };
struct PrevB { double ux0, ux1, uy0, uyjp, uz0, p0; };

// A cell's view of two plane slots (k and k+1): base pointers already moved to
// the cell's radial index and, for rows of odd parity, to the widened copy's
// offset. Field rows hold the storage type T (ux at element i - 1 in the
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
  const double * pb;   // plane k, p
  const double * pbo;  // plane k, p, odd rows
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
// diffusion in direction D goes to the implicit part when D is implicit
#define ROUTE(D, V_) do { if (D) gi += (V_); else e += (V_); } while (0)

// Group A: right-hand sides of ux at face i (src/fluid/predict/ux.c) and t at
// centre i (t.c) of cell (i, j, k); new source terms to ss.new_, increments
// dl[0] (ux, 0 at i = 1 where ux has no unknown) and dl[1] (t), current
// values u0[0] (ux) and u0[1] (t).
template <int JT, int RL, int JL, int IMPL, class T>
__device__ __forceinline__ void cell_a(const CoefA & q, const SlotView<T> & V, PrevA & pv, const Bc & bc,
                                       const Coefs & cf, double nu, double kappa, int i, size_t qf, size_t qc,
                                       const SrcSetT<T> & ss, double ca, double cb, double cg, double old_x,
                                       double old_t, double dl[2], double u0[2]) {
  const bool ix = IMPL >= 0 ? (IMPL & 1) != 0 : bc.implicit[0] != 0;
  const bool iy = IMPL >= 0 ? (IMPL & 2) != 0 : bc.implicit[1] != 0;
  const bool iz = IMPL >= 0 ? (IMPL & 4) != 0 : bc.implicit[2] != 0;
  const double ux_0 = UX(0, 0), ux_p = UX(1, 0);
  const double uy_00 = UY(0, 0), uy_01 = UY(0, 1);
  const double uz_00 = UZ(0, 0), uz_01 = NUZ(0, 0);
  dl[0] = 0.;
  if (i >= 2) {
    const double ux_m = UX(-1, 0);
    const double ux_jm = UX(0, -1), ux_jp = UX(0, 1);
    const double ux_km = pv.ux0, ux_kp = NUX(0);
    const double uy_m0 = UY(-1, 0), uy_m1 = UY(-1, 1);
    const double uz_m0 = UZ(-1, 0), uz_m1 = NUZ(-1, 0);
    double e, gi;
    // advection (ux.c:92-186): invj (l q_m + c q_0 + u q_p) with c = -l - u,
    // l = -0.5 (a q_m' + a' q_0'), u = 0.5 (...), as differences from q_0
    e = (q.xa1 * ux_m + q.xa2 * ux_0) * (ux_m - ux_0) - (q.xa2 * ux_0 + q.xa3 * ux_p) * (ux_p - ux_0);
    e += (q.yb1 * uy_m0 + q.yb2 * uy_00) * (ux_jm - ux_0) - (q.yb1 * uy_m1 + q.yb2 * uy_01) * (ux_jp - ux_0);
    e += (q.zc1 * uz_m0 + q.zc2 * uz_00) * (ux_km - ux_0) - (q.zc1 * uz_m1 + q.zc2 * uz_01) * (ux_kp - ux_0);
    // centrifugal term (:194-226): invj hd (uy averaged to the face)^2
    const double sm = uy_m0 + uy_m1, sp = uy_00 + uy_01;
    e += q.h1 * sm * sm + q.h2 * sp * sp;
    // cross diffusion (:266-375): diffusion_y1 and the uy part of diffusion_a
    // as differences of uy across j, the ux part of diffusion_a, diffusion_z1
    e += q.cy1 * (uy_m1 - uy_m0) + q.cy2 * (uy_01 - uy_00) + q.ca1 * (ux_m + ux_0) +
         q.ca2 * (ux_0 + ux_p) + q.cz1 * ((uz_01 - uz_m1) - (uz_00 - uz_m0));   // coefficients carry nu
    // pressure gradient (:377-394)
    gi = -q.px * (PP(0, 0) - PP(-1, 0));
    ROUTE(ix, q.lxl * ux_m + q.lxc * ux_0 + q.lxu * ux_p);          // carries 2 nu
    ROUTE(iy, q.lyl * ux_jm + q.lyc * ux_0 + q.lyu * ux_jp);          // carries nu
    ROUTE(iz, nu * (cf.lz_l * ux_km + cf.lz_c * ux_0 + cf.lz_u * ux_kp));
    if constexpr (IMPL == -2) e += ss.frc[VUX][qf];   // closure forcing
    ss.new_[VUX][qf] = (T)e;
    dl[0] = ca * e + cb * old_x + cg * gi;
  }
  {
    const double t_0 = TT(0, 0);
    const double tim = TT(-1, 0), tip = TT(1, 0), tjm = TT(0, -1), tjp = TT(0, 1);
    const double tkm = pv.t0, tkp = NTT(0);
    double e, gi = 0.;
    // advection (t.c:88-116) with face velocities ux_0, ux_p, uy_00, uy_01, uz_00, uz_01
    e = q.tx0 * ux_0 * (tim - t_0) - q.tx1 * ux_p * (tip - t_0);
    e += q.ty * uy_00 * (tjm - t_0) - q.ty * uy_01 * (tjp - t_0);
    e += q.tz * uz_00 * (tkm - t_0) - q.tz * uz_01 * (tkp - t_0);
    ROUTE(ix, q.clxl * tim + q.clxc * t_0 + q.clxu * tip);            // carry kappa
    ROUTE(iy, q.clyl * tjm + q.clyc * t_0 + q.clyu * tjp);
    ROUTE(iz, kappa * (cf.lz_l * tkm + cf.lz_c * t_0 + cf.lz_u * tkp));
    ss.new_[VT][qc] = (T)e;
    dl[1] = ca * e + cb * old_t + cg * gi;
    u0[1] = t_0;
    pv.t0 = t_0;
  }
  u0[0] = ux_0;
  pv.ux0 = ux_0;
}

// Group B: right-hand sides of uy (src/fluid/predict/uy.c) and uz (uz.c) at
// centre i of cell (i, j, k); increments dl[0] (uy), dl[1] (uz), current
// values u0[0], u0[1].
template <int JT, int RL, int JL, int IMPL, class T>
__device__ __forceinline__ void cell_b(const CoefB & q, const SlotView<T> & V, PrevB & pv, const Bc & bc,
                                       const Coefs & cf, double nu, int i, size_t qc, const SrcSetT<T> & ss,
                                       double ca, double cb, double cg, double old_y, double old_z, double dl[2],
                                       double u0[2]) {
  const bool ix = IMPL >= 0 ? (IMPL & 1) != 0 : bc.implicit[0] != 0;
  const bool iy = IMPL >= 0 ? (IMPL & 2) != 0 : bc.implicit[1] != 0;
  const bool iz = IMPL >= 0 ? (IMPL & 4) != 0 : bc.implicit[2] != 0;
  const double ux_0 = UX(0, 0), ux_1 = UX(1, 0);
  const double uy_0 = UY(0, 0), uy_jp = UY(0, 1);
  const double uz_0 = UZ(0, 0), uz_kp = NUZ(0, 0);
  const double p_0 = PP(0, 0);
  {  // uy
    const double uy_im = UY(-1, 0), uy_ip = UY(1, 0), uy_jm = UY(0, -1);
    const double uy_km = pv.uy0, uy_kp = NUY(0);
    const double ux_0m = UX(0, -1), ux_1m = UX(1, -1);
    const double uz_jm = UZ(0, -1), uz_jmkp = NUZ(0, -1);
    double e, gi;
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
    gi = -q.py * (p_0 - PP(0, -1));
    ROUTE(ix, q.lxl * uy_im + q.lxc * uy_0 + q.lxu * uy_ip);          // carry nu
    ROUTE(iy, 2. * (q.lyl * uy_jm + q.lyc * uy_0 + q.lyu * uy_jp));
    ROUTE(iz, nu * (cf.lz_l * uy_km + cf.lz_c * uy_0 + cf.lz_u * uy_kp));
    if constexpr (IMPL == -2) e += ss.frc[VUY][qc];
    ss.new_[VUY][qc] = (T)e;
    dl[0] = ca * e + cb * old_y + cg * gi;
  }
  {  // uz
    const double uz_im = UZ(-1, 0), uz_ip = UZ(1, 0), uz_jm = UZ(0, -1), uz_jp = UZ(0, 1);
    const double uz_km = pv.uz0;
    const double uy_km = pv.uy0, uy_jpkm = pv.uyjp;
    const double ux_0k = pv.ux0, ux_1k = pv.ux1;
    double e, gi;
    // advection (uz.c:88-180), as differences from uz_0
    e = q.a1 * (ux_0k + ux_0) * (uz_im - uz_0) - q.a2 * (ux_1k + ux_1) * (uz_ip - uz_0);
    e += q.b * (uy_km + uy_0) * (uz_jm - uz_0) - q.b * (uy_jpkm + uy_jp) * (uz_jp - uz_0);
    e += q.c * (uz_km + uz_0) * (uz_km - uz_0) - q.c * (uz_0 + uz_kp) * (uz_kp - uz_0);
    // diffusion_x1 (lzx at faces i, i+1), diffusion_y1 (lzy at j, j+1)
    e += q.zx1 * (ux_1 - ux_1k) - q.zx0 * (ux_0 - ux_0k) + q.zy * ((uy_jp - uy_jpkm) - (uy_0 - uy_km));   // carry nu
    gi = -cf.inv_hz * (p_0 - pv.p0);
    ROUTE(ix, q.lxl * uz_im + q.lxc * uz_0 + q.lxu * uz_ip);
    ROUTE(iy, q.lyl * uz_jm + q.lyc * uz_0 + q.lyu * uz_jp);
    ROUTE(iz, 2. * nu * (cf.lz_l * uz_km + cf.lz_c * uz_0 + cf.lz_u * uz_kp));
    if constexpr (IMPL == -2) e += ss.frc[VUZ][qc];
    ss.new_[VUZ][qc] = (T)e;
    dl[1] = ca * e + cb * old_z + cg * gi;
  }
  u0[0] = uy_0;
  u0[1] = uz_0;
  pv.ux0 = ux_0;
  pv.ux1 = ux_1;
  pv.uy0 = uy_0;
  pv.uyjp = uy_jp;
  pv.uz0 = uz_0;
  pv.p0 = p_0;
}
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
// elements tE .. tE+E-1, composes their affine maps, a 5-level shuffle scan
// supplies the value entering its chunk, then the recurrences run in the
// reference's form q = w (r - l q_prev) and x = q - v x_next. The factor rows
// hold w[0] = 1 / c[0] and l[0] = 0, and zeros from n on; the staging line is
// zero from n on as well, so elements past the end map to zero without tests.
template <int E>
__device__ __forceinline__ void solve_line(double * sb, const XFactors & xf, int rkstep, int var, int lane) {
  const size_t fo = (size_t)(rkstep * 4 + var) * xf.stride;
  double q[E], ll[E], ww[E];
  load_chunk<E>(ll, xf.lo + fo, lane);
  load_chunk<E>(ww, xf.w + fo, lane);
#pragma unroll
  for (int m = 0; m < E; m++) q[m] = sb[spad<E>(lane * E + m)];
  Aff acc{1., 0.};
#pragma unroll
  for (int m = 0; m < E; m++) {
    const double fa = -ww[m] * ll[m], fb = ww[m] * q[m];
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
    const double r = ww[m] * (q[m] - ll[m] * qin);
    q[m] = r;
    qin = r;
  }
  double vv[E];
  load_chunk<E>(vv, xf.v + fo, lane);
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

// Shared-memory layout in bytes, shared by the kernel and its launcher. Row
// buffers are sized for the widest radial line of the warp count (nx <= 32 NW),
// so every stencil offset is a compile-time constant. A slot holds the field
// rows (storage type T), the p rows (double) and the previous substep's source
// terms (T).
template <int NW, int JT, class T>
struct MarchLayout {
  static_assert(JT == 2 || JT == 4, "line groups start at odd j, so rows of even index have even j");
  static constexpr int E = NW;
  static constexpr int RL = 32 * NW + 4;                      // values per row: >= nx + 4, multiple of 4
  static constexpr int NFROW = 4 * (JT + 2);                  // ux, uy, uz, t: JT + 2 rows each
  static constexpr size_t POFF = (size_t)NFROW * RL * sizeof(T);          // p: JT + 1 rows of double
  static constexpr size_t OLDOFF = POFF + (size_t)(JT + 1) * RL * sizeof(double);
  static constexpr size_t SLOT = OLDOFF + (size_t)4 * JT * RL * sizeof(T);  // JT lines per variable
  static constexpr int SL = 32 * E + (E > 1 ? 32 : 0);        // staging line (padded for the solves)
  static constexpr size_t STAGE = NSLOT * SLOT;               // [2][JT][4][SL] doubles after the ring
  static constexpr size_t BAR = STAGE + sizeof(double) * 2 * JT * 4 * SL;   // NSLOT mbarriers
  static constexpr size_t BYTES = BAR + NSLOT * sizeof(unsigned long long);
};

// Everything a group's march needs besides its coefficients.
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

// The plane loop of one thread group: G = 0 computes ux and t, G = 1 uy and
// uz, G = 2 all four (one group per line). With two groups both pass the same
// barriers in the same order.
template <int NW, int JT, int IMPL, int G, class T>
__device__ __forceinline__ void march_group(const MarchArgs<T> & A, char * ring, double * stage,
                                            unsigned long long * bar, int j0, int k0, int k1, double dt) {
  using L = MarchLayout<NW, JT, T>;
  constexpr int E = L::E, RL = L::RL, SL = L::SL, NT = 32 * NW;
  constexpr bool GA = G != 1, GB = G != 0;   // group computes ux and t / uy and uz
  constexpr int NGRP = G == 2 ? 1 : 2;
  const Geo & g = A.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int tx = threadIdx.x;
  const int lane = tx & 31, wid = tx >> 5;
  const int i = tx - (G == 1 ? NT : 0) + 1;
  const bool act = i <= nx;
  // element offsets of odd rows in their widened copies: ux / centre fields
  // (none in the FP32 layout, whose rows start on 16-byte boundaries) and p
  constexpr bool D64 = sizeof(T) == 8;
  const int of = D64 ? (nx + 1) & 1 : 0, oc = D64 ? (nx + 2) & 1 : 0, op = (nx + 2) & 1;
  constexpr int FSH = D64 ? 1 : 0;   // ux face i at element i - FSH of its row
  const size_t sjc = (size_t)ny + 2;
  auto frow = [&](char * slot, int f, int r) { return reinterpret_cast<T *>(slot) + (size_t)(f * (JT + 2) + r) * RL; };
  auto prow = [&](char * slot, int r) { return reinterpret_cast<double *>(slot + L::POFF) + (size_t)r * RL; };
  auto orow = [&](char * slot, int v) { return reinterpret_cast<T *>(slot + L::OLDOFF) + (size_t)v * JT * RL; };

  // Copies of plane kp into slot sl: the field rows and, for planes that are
  // computed in a substep with beta != 0, the source terms of the previous
  // substep at the JT lines (consecutive in the packed layout, 16-byte
  // aligned as JT is even).
  const bool use_old = A.rkstep != 0;
  auto issue = [&](int kp, int sl) {
    char * base = ring + (size_t)sl * L::SLOT;
    const bool olds = use_old && kp >= k0 && kp < k1;
    // every row of the five arrays (4 = p, in double), widened to 16-byte
    // bounds: counts the bytes or issues the copies. With 8-byte storage the
    // p rows continue the field rows' layout.
    const char * src[5] = {reinterpret_cast<const char *>(A.in.ux), reinterpret_cast<const char *>(A.in.uy),
                           reinterpret_cast<const char *>(A.in.uz), reinterpret_cast<const char *>(A.in.t),
                           reinterpret_cast<const char *>(A.in.p)};
    auto all = [&](bool go, unsigned & total) {
      for (int f = 0; f < 5; f++) {
        const size_t es = f == SF_P ? sizeof(double) : sizeof(T), al = 16 / es;
        const size_t n = (f == SF_P || (D64 && f != SF_UX)) ? (size_t)nx + 2 : D64 ? (size_t)nx + 1 : (size_t)pitch32(nx);
        for (int r = 0; r < (f == SF_P ? JT + 1 : JT + 2); r++) {
          const size_t s0 = n * ((size_t)(j0 - 1 + r) + sjc * kp);
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
    if (olds) total += (unsigned)(JT * (D64 ? 4 * nx - 1 : 4 * spitch32(nx)) * sizeof(T));
    mbar_expect_tx(&bar[sl], total);
    if (olds) {
      for (int v = 0; v < 4; v++) {
        const int ni = (v == VUX) ? nx - 1 : nx;
        const int li = D64 ? ni : spitch32(nx);   // packed line length (sline)
        bulk_g2s(orow(base, v), A.ss.old_[v] + pidx(li, ny, 0, j0, kp), (unsigned)(JT * li * sizeof(T)), &bar[sl]);
      }
    }
    all(true, total);
  };
  if (tx == 0) {
    issue(k0 - 1, 0);
    issue(k0, 1);
    issue(k0 + 1, 2);
  }
  unsigned par[NSLOT] = {0u, 0u, 0u};
  bool late = false;
  auto wait_slot = [&](int sl) {
    if (!mbar_wait(&bar[sl], par[sl])) late = true;
    par[sl] ^= 1u;
  };

  CoefA qa;
  CoefB qb;
  if constexpr (GA) load_coefs(qa, A.cf, act ? i : 1);
  if constexpr (GB) load_coefs(qb, A.cf, act ? i : 1);
  // the diffusivities folded into the per-thread coefficients once, so the
  // cell updates multiply by them no more (the z Laplacian, a shared scalar
  // set, keeps its factor)
  if constexpr (GA) {
    const double nu = A.nu, n2 = 2. * A.nu, ka = A.kappa;
    qa.lxl *= n2; qa.lxc *= n2; qa.lxu *= n2;
    qa.lyl *= nu; qa.lyc *= nu; qa.lyu *= nu;
    qa.cy1 *= nu; qa.cy2 *= nu; qa.ca1 *= nu; qa.ca2 *= nu; qa.cz1 *= nu;
    qa.clxl *= ka; qa.clxc *= ka; qa.clxu *= ka; qa.clyl *= ka; qa.clyc *= ka; qa.clyu *= ka;
  }
  if constexpr (GB) {
    const double nu = A.nu;
    qb.lxl *= nu; qb.lxc *= nu; qb.lxu *= nu; qb.lyl *= nu; qb.lyc *= nu; qb.lyu *= nu;
    qb.p1 *= nu; qb.p2 *= nu; qb.qm *= nu; qb.q0 *= nu; qb.qp *= nu; qb.yk *= nu; qb.yz *= nu;
    qb.zx0 *= nu; qb.zx1 *= nu; qb.zy *= nu;
  }
  const int rk = A.rkstep;
  const double ca = rk_alpha(rk) * dt, cb = rk_beta(rk) * dt, cg = rk_gamma(rk) * dt;

  // plane k0 - 1: the carried values
  wait_slot(0);
  wait_slot(1);
  PrevA pa[JT];
  PrevB pb[JT];
  if (act) {
#pragma unroll
    for (int jl = 0; jl < JT; jl++) {
      const int r1 = jl + 1, r2 = jl + 2;   // rows j and j + 1
      const int o1c = (r1 & 1) ? oc : 0, o1f = (r1 & 1) ? of : 0, o2c = (r2 & 1) ? oc : 0;
      const int o1p = (r1 & 1) ? op : 0;
      const T * ux1 = frow(ring, SF_UX, r1) + o1f + i - FSH;
      if constexpr (GA) {
        pa[jl].ux0 = ux1[0];
        pa[jl].t0 = frow(ring, SF_T, r1)[o1c + i];
      }
      if constexpr (GB) {
        pb[jl].ux0 = ux1[0];
        pb[jl].ux1 = ux1[1];
        pb[jl].uy0 = frow(ring, SF_UY, r1)[o1c + i];
        pb[jl].uyjp = frow(ring, SF_UY, r2)[o2c + i];
        pb[jl].uz0 = frow(ring, SF_UZ, r1)[o1c + i];
        pb[jl].p0 = prow(ring, r1)[o1p + i];
      }
    }
  }
  __syncthreads();

  const bool solve_x = IMPL >= 0 ? (IMPL & 1) != 0 : A.bc.implicit[0] != 0;
  for (int k = k0; k < k1; k++) {
    const int step = k - k0;
    const int cur = (step + 1) % NSLOT, nxt = (step + 2) % NSLOT, fre = step % NSLOT;
    // plane k + 2 into the slot of plane k - 1, which every thread finished
    // reading before the previous plane's first barrier
    if (tx == 0 && k + 2 <= k1) {
      fence_async_smem();
      issue(k + 2, fre);
    }
    wait_slot(nxt);
    double * sdb = stage + (size_t)(step & 1) * JT * 4 * SL;
    double dl[JT][4], u0[JT][4];   // indexed by Var
#pragma unroll
    for (int jl = 0; jl < JT; jl++)
#pragma unroll
      for (int v = 0; v < 4; v++) dl[jl][v] = u0[jl][v] = 0.;
    if (act) {
      char * cs = ring + (size_t)cur * L::SLOT;
      char * ns = ring + (size_t)nxt * L::SLOT;
      SlotView<T> V;
      V.cb = reinterpret_cast<const T *>(cs) + i;
      V.cbo = V.cb + oc;
      V.fb = V.cb - FSH;
      V.fbo = V.fb + of;
      V.nb = reinterpret_cast<const T *>(ns) + i;
      V.nbo = V.nb + oc;
      V.nf = V.nb - FSH;
      V.nfo = V.nf + of;
      if constexpr (D64) {   // p rows follow the field rows: same base registers, constant offsets
        V.pb = reinterpret_cast<const double *>(V.cb) + L::NFROW * RL;
        V.pbo = reinterpret_cast<const double *>(V.cbo) + L::NFROW * RL;
      } else {
        V.pb = prow(cs, 0) + i;
        V.pbo = V.pb + op;
      }
      const int lf = D64 ? nx - 1 : spitch32(nx), lc = D64 ? nx : spitch32(nx);   // source-term lines (sline)
      const size_t qf = pidx(lf, ny, i - 2, j0, k), qc = pidx(lc, ny, i - 1, j0, k);
      const T * ob = orow(cs, 0);   // old source terms of plane k
      auto cells = [&](auto jlc) {
        constexpr int JL = decltype(jlc)::value;
        double d2[2], w2[2];
        auto old = [&](int v, int e) {
          return use_old ? (double)ob[v * JT * RL + JL * (v == VUX ? lf : lc) + e] : 0.;
        };
        if constexpr (GA) {
          cell_a<JT, RL, JL, IMPL>(qa, V, pa[JL], A.bc, A.cf, A.nu, A.kappa, i, qf + (size_t)JL * lf,
                                   qc + (size_t)JL * lc, A.ss, ca, cb, cg, i >= 2 ? old(VUX, i - 2) : 0.,
                                   old(VT, i - 1), d2, w2);
          dl[JL][VUX] = d2[0]; dl[JL][VT] = d2[1]; u0[JL][VUX] = w2[0]; u0[JL][VT] = w2[1];
        }
        if constexpr (GB) {
          cell_b<JT, RL, JL, IMPL>(qb, V, pb[JL], A.bc, A.cf, A.nu, i, qc + (size_t)JL * lc, A.ss, ca, cb, cg,
                                   old(VUY, i - 1), old(VUZ, i - 1), d2, w2);
          dl[JL][VUY] = d2[0]; dl[JL][VUZ] = d2[1]; u0[JL][VUY] = w2[0]; u0[JL][VUZ] = w2[1];
        }
      };
      cells(std::integral_constant<int, 0>());
      cells(std::integral_constant<int, 1>());
      if constexpr (JT == 4) {
        cells(std::integral_constant<int, 2>());
        cells(std::integral_constant<int, 3>());
      }
    }
    // staging positions: ux unknowns are faces 2..nx (element i - 2), the
    // centred ones cells 1..nx (element i - 1)
    if (solve_x) {
      if (act) {
#pragma unroll
        for (int jl = 0; jl < JT; jl++) {
          double * s = sdb + (size_t)jl * 4 * SL;
          if constexpr (GA) {
            if (i >= 2) s[VUX * SL + spad<E>(i - 2)] = dl[jl][VUX];
            s[VT * SL + spad<E>(i - 1)] = dl[jl][VT];
          }
          if constexpr (GB) {
            s[VUY * SL + spad<E>(i - 1)] = dl[jl][VUY];
            s[VUZ * SL + spad<E>(i - 1)] = dl[jl][VUZ];
          }
        }
      }
      __syncthreads();
      for (int s = wid; s < 4 * JT; s += NGRP * NW) solve_line<E>(sdb + (size_t)s * SL, A.xf, rk, s & 3, lane);
      __syncthreads();
      if (act) {
#pragma unroll
        for (int jl = 0; jl < JT; jl++) {
          const double * s = sdb + (size_t)jl * 4 * SL;
          if constexpr (GA) {
            dl[jl][VUX] = (i >= 2) ? s[VUX * SL + spad<E>(i - 2)] : 0.;
            dl[jl][VT] = s[VT * SL + spad<E>(i - 1)];
          }
          if constexpr (GB) {
            dl[jl][VUY] = s[VUY * SL + spad<E>(i - 1)];
            dl[jl][VUZ] = s[VUZ * SL + spad<E>(i - 1)];
          }
        }
      }
    } else {
      // no radial solve: this barrier alone orders the plane's slot reads
      // before the copy into that slot two planes on
      __syncthreads();
    }
    if (!act) continue;
#pragma unroll
    for (int jl = 0; jl < JT; jl++) {
      const int j = j0 + jl;
      if (A.mode == PREDICT_DELTA) {
        const size_t qc = pidx(nx, ny, i - 1, j, k);
        if constexpr (GA) {
          if (i >= 2) A.ds.d[VUX][pidx(nx - 1, ny, i - 2, j, k)] = dl[jl][VUX];
          A.ds.d[VT][qc] = dl[jl][VT];
        }
        if constexpr (GB) {
          A.ds.d[VUY][qc] = dl[jl][VUY];
          A.ds.d[VUZ][qc] = dl[jl][VUZ];
        }
        continue;
      }
      // u += delta into the other buffer, walls (boundary/*.c) and images (halo.c)
      const double vx = (i < 2) ? 0. : u0[jl][VUX] + dl[jl][VUX];
      const double vt = u0[jl][VT] + dl[jl][VT];
      const double vy = u0[jl][VUY] + dl[jl][VUY];
      const double vz = u0[jl][VUZ] + dl[jl][VUZ];
      auto put = [&](int jj, int kk) {
        if constexpr (GA) {
          A.out.ux[sidx_f<T>(g, i, jj, kk)] = (T)vx;
          A.out.t[sidx_c<T>(g, i, jj, kk)] = (T)vt;
          if (i == 1) A.out.t[sidx_c<T>(g, 0, jj, kk)] = (T)A.bc.t_xm;
          if (i == nx) {
            A.out.ux[sidx_f<T>(g, nx + 1, jj, kk)] = (T)0.;
            A.out.t[sidx_c<T>(g, nx + 1, jj, kk)] = (T)A.bc.t_xp;
          }
        }
        if constexpr (GB) {
          A.out.uy[sidx_c<T>(g, i, jj, kk)] = (T)vy;
          A.out.uz[sidx_c<T>(g, i, jj, kk)] = (T)vz;
          if (i == 1) {
            A.out.uy[sidx_c<T>(g, 0, jj, kk)] = (T)A.bc.uy_xm;
            A.out.uz[sidx_c<T>(g, 0, jj, kk)] = (T)0.;
          }
          if (i == nx) {
            A.out.uy[sidx_c<T>(g, nx + 1, jj, kk)] = (T)A.bc.uy_xp;
            A.out.uz[sidx_c<T>(g, nx + 1, jj, kk)] = (T)0.;
          }
        }
      };
      put(j, k);
      for_images(j, k, ny, nz, put);
    }
  }
  if (late) atomicOr(A.status, ST_TIMEOUT);
}

// Thread groups per line. With 2, ux and t are computed by one thread and uy
// and uz by another, so the coefficients of each fit in 128 registers and twice
// as many warps are resident; measured at 256 x 1024 x 512 the single group
// (up to 255 registers, 8 warps per SM) is faster (7.9 against 9.4 ms per
// launch, the two groups waiting on each other at the barriers).
#ifndef TC_MARCH_GROUPS
#define TC_MARCH_GROUPS 1
#endif
// NG groups of 32 NW threads, one thread per radial index in each; CTA = JT
// lines (j0 .. j0+JT-1) x KC planes.
template <int NW, int JT, int IMPL, class T>
__global__ void __launch_bounds__(32 * NW * TC_MARCH_GROUPS, 1)
march_predict_kernel(MarchArgs<T> A, const double * __restrict__ dtp) {
  using L = MarchLayout<NW, JT, T>;
  extern __shared__ __align__(16) double sm[];
  char * ring = reinterpret_cast<char *>(sm);
  double * stage = reinterpret_cast<double *>(ring + L::STAGE);
  unsigned long long * bar = reinterpret_cast<unsigned long long *>(ring + L::BAR);
  const int tx = threadIdx.x;
  const int njg = A.g.ny / JT;
  const int j0 = (int)(blockIdx.x % njg) * JT + 1;   // odd
  const int k0 = (int)(blockIdx.x / njg) * A.KC + 1;
  const int k1 = k0 + A.KC;   // planes k0 .. k1-1 are computed; k0-1 .. k1 are read
  if (tx == 0) {
    for (int s = 0; s < NSLOT; s++) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  // staging lines are zero past each line's unknowns for the whole march
  for (int e = tx; e < 2 * JT * 4 * L::SL; e += blockDim.x) stage[e] = 0.;
  __syncthreads();
  const double dt = *dtp;
  if constexpr (TC_MARCH_GROUPS == 1) {
    march_group<NW, JT, IMPL, 2>(A, ring, stage, bar, j0, k0, k1, dt);
  } else {
    if (tx < 32 * NW) march_group<NW, JT, IMPL, 0>(A, ring, stage, bar, j0, k0, k1, dt);
    else march_group<NW, JT, IMPL, 1>(A, ring, stage, bar, j0, k0, k1, dt);
  }
}

#ifndef TC_MARCH_JT
#define TC_MARCH_JT 2
#endif
// Planes per CTA, at most: each CTA's start (coefficients, barriers, the first
// planes' copies) overlaps nothing at one CTA per SM, and its two halo planes
// are read twice. Measured at 256 x 1024 x 512 (ms per launch): 16 7.01, 32
// 6.86, 64 6.82, 128 6.81-7.03. Smaller grids take fewer planes per CTA when
// the last wave of CTAs would leave SMs idle (march_planes).
#ifndef TC_MARCH_KC
#define TC_MARCH_KC 64
#endif

// The largest chunk of planes, from TC_MARCH_KC down to 16, whose last partial
// wave of CTAs wastes at most 5% of the launch (at 256 x 512 x 128: 64 planes
// are 3.5 waves, 32 planes 6.9).
template <int NW, class T>
static int march_planes(const Geo & g) {
  constexpr int JT = TC_MARCH_JT;
  static int per_sm[16], sms[16];   // per device: resident CTAs of this instance, SM count
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 15;
  if (per_sm[dev] == 0) {
    int b = 0, n = 0;
    // a failed query falls back to one CTA on 148 SMs and clears its own error
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, march_predict_kernel<NW, JT, 1, T>,
                                                      32 * NW * TC_MARCH_GROUPS, MarchLayout<NW, JT, T>::BYTES) !=
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
  int kc = g.nz < TC_MARCH_KC ? g.nz : TC_MARCH_KC;
  for (; kc > 16; kc >>= 1) {
    const long long nblk = lines * (g.nz / kc), waves = (nblk + slots - 1) / slots;
    if (waves * slots * 100 <= nblk * 105) break;
  }
  return kc;
}

template <int NW, class T>
void launch_march_nw(MarchArgs<T> A, const double * dtp, cudaStream_t st) {
  constexpr int JT = TC_MARCH_JT;   // ny is a power of two >= 4
  A.KC = march_planes<NW, T>(A.g);
  const long long nblk = (long long)(A.g.ny / JT) * (A.g.nz / A.KC);
  const int mask = (A.bc.implicit[0] ? 1 : 0) | (A.bc.implicit[1] ? 2 : 0) | (A.bc.implicit[2] ? 4 : 0);
  const unsigned grid = (unsigned)nblk, block = 32 * NW * TC_MARCH_GROUPS;
  const size_t smem = MarchLayout<NW, JT, T>::BYTES;
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
}

template <class T>
void launch_march_t(const Geo & g, const Bc & bc, const Coefs & cf, const XFactors & xf, double nu,
                    double kappa, const FieldBufs & in, const FieldBufs & out, const SrcBufs & ss,
                    const DeltaSet & ds, const double * dtp, int rkstep, int mode, unsigned * status,
                    cudaStream_t st) {
  MarchArgs<T> A{g, bc, cf, xf, nu, kappa, in.as<T>(), out.as<T>(), ss.as<T>(), ds, rkstep, mode, 0, status};
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

void march_smem_limits() {
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
