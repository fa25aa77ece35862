// Kernel-side data structures and launchers of the tcgpu library.
#pragma once

#include "tc_common.cuh"

namespace tcgpu {

// Device pointers of the state fields (reference layout with halos). ux, uy,
// uz and t are stored in T: double, or float in the FP32-storage mode (all
// arithmetic stays FP64); p and psi are always double.
template <class T>
struct FieldsT {
  T * ux;
  T * uy;
  T * uz;
  double * p;
  double * psi;
  T * t;
};
using Fields = FieldsT<double>;
// the host's type-erased form: bytes = 8 or 4 per stored value
struct FieldBufs {
  void * ux;
  void * uy;
  void * uz;
  double * p;
  double * psi;
  void * t;
  int bytes;
  template <class T>
  FieldsT<T> as() const {
    return FieldsT<T>{static_cast<T *>(ux), static_cast<T *>(uy), static_cast<T *>(uz), p, psi,
                      static_cast<T *>(t)};
  }
};

// Per-radial-index coefficient tables (length nx+2, indexed by the reference
// i), computed on the host once per context with the reference's operand
// order. f_* belong to ux at face i, c_* to the cell-centred variables at i.
// All tables live in one allocation laid out [table][CSTRIDE] so that a
// thread's coefficients are reached from one base pointer with compile-time
// offsets (tab + table * CSTRIDE + i); nx + 2 <= CSTRIDE.
constexpr int CSTRIDE = 1032;
enum CoefTable {
  F_INVJD, F_A1, F_A2, F_A3, F_B1, F_B2, F_C1, F_C2, F_HD1, F_HD2, F_LXL, F_LXC, F_LXU, F_LYL, F_LYC, F_LYU,
  F_E1, F_E2, C_LYX1F, C_WM, C_WP, C_INVHXXF, C_INVHYXC, C_INVHYXF, C_LYY1, C_INVJDXC, C_A1, C_A2, C_B, C_CZ,
  C_HD, C_LXL, C_LXC, C_LXU, C_LYL, C_LYC, C_LYU, C_JF, C_E1, C_E2, C_HDA1, C_HDA2, C_PXL, C_PXU, C_PYL, C_PZL,
  // Products of the tables above, one per stencil term of the marching
  // predict kernel (the viscosity factor stays out, applied in the kernel).
  // ux at face i:
  P_XA1, P_XA2, P_XA3,   // 0.5 F_INVJD F_A1..3        advection in x
  P_YB1, P_YB2,          // 0.5 F_INVJD F_B1..2        advection in y
  P_ZC1, P_ZC2,          // 0.5 F_INVJD F_C1..2        advection in z
  P_H1, P_H2,            // 0.25 F_INVJD F_HD1..2      centrifugal term
  P_CY1, P_CY2,          // uy differences of diffusion_y1 + diffusion_a, / nu
  P_CA1, P_CA2,          // ux sums of diffusion_a, / nu
  P_CZ1,                 // uz differences of diffusion_z1, / nu
  // t at centre i:
  P_TX0, P_TX1, P_TY, P_TZ,  // 0.5 C_INVJDXC {C_JF(i), C_JF(i+1), C_E1, C_E2}
  // uy, uz at centre i:
  P_UA1, P_UA2, P_UB, P_UC,  // 0.5 C_INVJDXC {C_A1, C_A2, C_B, C_CZ}
  P_UH,                      // 0.25 C_INVJDXC C_HD
  P_P1, P_P2,                // uy: ux differences of diffusion_x1 + diffusion_a, / nu
  P_QM, P_Q0, P_QP,          // uy: uy values of diffusion_x1 + diffusion_a, / nu
  P_YK, P_YZ,                // uy: diffusion_y1, diffusion_z1, / nu
  P_ZX0, P_ZX1, P_ZY,        // uz: diffusion_x1, diffusion_y1, / nu
  NCOEF_TABLES
};
struct Coefs {
  const double * tab;      // base of the [table][CSTRIDE] block
  const double * f_invjd;  // 1 / JDXF(i)
  const double * f_a1;     // 0.5 JDXF(i-1) / HXXF(i-1)
  const double * f_a2;     // 0.5 JDXF(i)   / HXXF(i)
  const double * f_a3;     // 0.5 JDXF(i+1) / HXXF(i+1)
  const double * f_b1;     // 0.5 JDXC(i-1) / HYXC(i-1)
  const double * f_b2;     // 0.5 JDXC(i)   / HYXC(i)
  const double * f_c1;     // 0.5 JDXC(i-1) / hz
  const double * f_c2;     // 0.5 JDXC(i)   / hz
  const double * f_hd1;    // 0.5 (-JDXF(i-1)/HXXF(i-1) + JDXF(i)/HXXF(i))
  const double * f_hd2;    // 0.5 (-JDXF(i)/HXXF(i) + JDXF(i+1)/HXXF(i+1))
  const double * f_lxl;    // ux Laplacian in x (ux.c:34-47)
  const double * f_lxc;
  const double * f_lxu;
  const double * f_lyl;    // ux Laplacian in y (ux.c:48-58)
  const double * f_lyc;
  const double * f_lyu;
  const double * f_e1;     // JDXF(i) / HYXF(i)
  const double * f_e2;     // JDXF(i) / hz
  const double * c_lyx1f;  // -1/JDXF(i) (-JDXC(i-1)/HXXC(i-1) + JDXC(i)/HXXC(i))   lyx.c:70-83
  const double * c_wm;     // 0 at i = 1, else 0.5
  const double * c_wp;     // 0 at i = nx+1, else 0.5
  const double * c_invhxxf;
  const double * c_invhyxc;
  const double * c_invhyxf;
  const double * c_lyy1;   // 1/JDXC(i) (-JDXF(i)/HXXF(i) + JDXF(i+1)/HXXF(i+1))    lyy.c:70-83
  const double * c_invjdxc;
  const double * c_a1;     // 0.5 JDXF(i)   / HXXF(i)
  const double * c_a2;     // 0.5 JDXF(i+1) / HXXF(i+1)
  const double * c_b;      // 0.5 JDXC(i) / HYXC(i)
  const double * c_cz;     // 0.5 JDXC(i) / hz
  const double * c_hd;     // 0.5 (-JDXF(i)/HXXF(i) + JDXF(i+1)/HXXF(i+1))
  const double * c_lxl;    // centred Laplacian in x (uy.c:34-47, uz.c, t.c)
  const double * c_lxc;
  const double * c_lxu;
  const double * c_lyl;    // centred Laplacian in y
  const double * c_lyc;
  const double * c_lyu;
  const double * c_jf;     // JDXF(i) / HXXF(i)
  const double * c_e1;     // JDXC(i) / HYXC(i)
  const double * c_e2;     // JDXC(i) / hz
  const double * c_hda1;   // 0.5 (-JDXC(i-1)/HXXC(i-1) + JDXC(i)/HXXC(i))
  const double * c_hda2;   // 0.5 (-JDXC(i)/HXXC(i) + JDXC(i+1)/HXXC(i+1))
  const double * c_pxl;    // JDXF(i)/HXXF(i)/HXXF(i)        update_pressure.c:51-56
  const double * c_pxu;    // JDXF(i+1)/HXXF(i+1)/HXXF(i+1)
  const double * c_pyl;    // JDXC(i)/HYXC(i)/HYXC(i)        :86-90
  const double * c_pzl;    // JDXC(i)/hz/hz                  :118-122
  double lz_l, lz_c, lz_u; // Laplacian in z
  double inv_hz;
};

// Radial Thomas factors for the three substeps x four variables.
struct XFactors {
  int n[4];                 // nx-1 for ux, nx otherwise
  size_t stride;            // >= nx
  const double * lap_l[4];  // per-variable Laplacian coefficients, packed e = i - i0
  const double * lap_c[4];
  const double * lap_u[4];
  double * lo;              // [12][stride], element e of a row at (e % ne) 32 + e / ne: the
  double * w;               // ne elements a lane of the solving warp owns (e = lane ne + m)
  double * v;               // are read with one coalesced load per m
  int ne;                   // elements per lane of the radial solves (warps of the predict kernel)
};

// Periodic y / z factors (planar configuration with implicit y and z).
struct YZFactors {
  int n_i[4];
  int max_i;
  int uniform_y;            // the y operators do not depend on i (planar grids): factors of i = 0 serve all
  size_t stride_y;          // max_i * ny
  size_t stride_z;          // nz
  const double * lapy_l[4];
  const double * lapy_c[4];
  const double * lapy_u[4];
  double lapz_l, lapz_c, lapz_u;
  double * l;               // [12][max_i]
  double * c;
  double * u;
  double * v;               // [12][max_i][ny]
  double * w;
  double * q1;
  double * lz;              // [12]
  double * cz;
  double * uz;
  double * vz;              // [12][nz]
  double * wz;
  double * q1z;
};

// Poisson solver state.
struct Poisson {
  int nyh;                  // ny/2 + 1
  void * spec;              // [nx][nz][nyh] complex spectra: double2, or float2 (spec_bytes 8)
  int spec_bytes;           // 16 or 8 per complex value
  double * vscr;            // [nx][nz][nyh] elimination factors
  // Radial solves by warps over tiles of lines (nx = 32 fe, fe in {2, 4, 8}):
  // the factors of every line (kz, m) computed once per context, since the
  // Poisson matrix does not change; [line][nx] with element i at
  // (i % fe) 32 + i / fe (the fe elements a lane owns arrive coalesced).
  // fe = 0: the per-column kernel with factors from each call.
  int fe;
  double * fw;              // multipliers of the forward sweep
  double * fv;              // back-substitution factors
  const double2 * tw_y;     // exp(-2 pi i m / ny), m < ny
  const double2 * tw_z;     // exp(-2 pi i m / nz), m < nz
  const float2 * tw_y32;    // the same rounded to float (FP32-storage contexts, whose transforms run in float)
  const float2 * tw_z32;
  const double * tl;        // radial l_i (compute_potential.c:197-200), length nx
  const double * tu;        // radial u_i
  const double * ihy2;      // 1 / HYXC(i)^2 as (1/HYXC)/HYXC, length nx (index i-1)
  const double * hyxc;      // HYXC(i), length nx (index i-1)
  const double * eval_y;    // -4 sin^2(pi m / ny), m < nyh
  const double * eval_z;    // -4 sin^2(pi m / nz), m < nz
  unsigned * status;        // the context's error word (ST_TIMEOUT from a bounded wait)
};

// RK source terms of one substep: old_ (srcA of the previous substep) and new_,
// stored like the state fields; frc: optional forcing added to the new
// explicit terms of ux, uy, uz (FP64, packed interior layout; the learned
// closure of a coarse grid), null when off
template <class T>
struct SrcSetT {
  const T * old_[4];
  T * new_[4];
  const double * frc[4];
};
using SrcSet = SrcSetT<double>;
struct SrcBufs {
  const void * old_[4];
  void * new_[4];
  int bytes;
  const double * frc[4];
  template <class T>
  SrcSetT<T> as() const {
    SrcSetT<T> s;
    for (int v = 0; v < 4; v++) {
      s.old_[v] = static_cast<const T *>(old_[v]);
      s.new_[v] = static_cast<T *>(new_[v]);
      s.frc[v] = frc[v];
    }
    return s;
  }
};
// increments (packed interior layout), used by the planar y / z solves
struct DeltaSet {
  double * d[4];
};
enum { PREDICT_APPLY = 0, PREDICT_DELTA = 1 };
int predict_warps(int nx);
// marching form of the predict stage (tc_march.cu); sets ST_TIMEOUT in
// *status if a plane's copy does not arrive within its wait limit
void launch_predict_march(const Geo & g, const Bc & bc, const Coefs & cf, const XFactors & xf, double nu,
                          double kappa, const FieldBufs & in, const FieldBufs & out, const SrcBufs & ss,
                          const DeltaSet & ds, const double * dtp, int rkstep, int mode, unsigned * status,
                          cudaStream_t st);
void march_smem_limits();
// radial implicit solves of the delta buffers, lines of up to 1024 points
// (after the predict's tile mode, nx > 256)
void launch_xsolve(const Geo & g, const XFactors & xf, int rkstep, const DeltaSet & ds, cudaStream_t st);
// one CTA whose mbarrier wait can never complete: sets ST_TIMEOUT in *status
void launch_wait_selftest(unsigned * status, cudaStream_t st);
void launch_xfactors(const XFactors & xf, const double * dtp, double nu, double kappa, cudaStream_t st);
void launch_apply(const Geo & g, const Bc & bc, const FieldBufs & in, const FieldBufs & out, const DeltaSet & ds,
                  cudaStream_t st);
void launch_yzfactors(const Geo & g, const YZFactors & yf, const double * dtp, double nu, double kappa, cudaStream_t st);
void launch_ysolve(const Geo & g, const YZFactors & yf, int rkstep, const DeltaSet & ds, cudaStream_t st);
void launch_zsolve(const Geo & g, const YZFactors & yf, int rkstep, const DeltaSet & ds, cudaStream_t st);
void allow_periodic_lines_smem();

// optional per-launch callback of the host's kernel accounting
struct PoissonMarks {
  void (*mark)(int kind, int n) = nullptr;
  int k_div = 0, k_fwd = 0, k_tdm = 0, k_inv = 0, k_ify = 0;
};
// tab_y[i][ky] = ey/hyxc/hyxc, tab_z[kz] = ez/hz/hz, base[i] = -l_i - u_i
void launch_poisson(const Geo & g, const Coefs & cf, const Poisson & ps, const FieldBufs & f,
                    const double * tab_y, const double * tab_z, const double * base,
                    const double * dtp, int rkstep, cudaStream_t st, const PoissonMarks & pm = PoissonMarks());
void poisson_smem_limits();
// per-line factors of the warp radial solves (Poisson::fe > 0), once per context
void launch_tdm_factors(const Geo & g, const Poisson & ps, const double * tab_y, const double * tab_z,
                        const double * base, cudaStream_t st);
enum { CORRECT_VELOCITY = 1, CORRECT_PRESSURE = 2 };
// cfl_dtmin: when non-null (velocity and pressure together), the advective
// time-step limit of the corrected velocities is folded into it
void launch_correct(const Geo & g, const Bc & bc, const Coefs & cf, const FieldBufs & f, const double * dtp,
                    int rkstep, double nu, int what, unsigned long long * cfl_dtmin, unsigned * status,
                    cudaStream_t st);
// the advective limit is gathered in DT_SLOTS accumulators (blocks spread
// their atomicMin over them); dtfinal takes their minimum and resets them
constexpr int DT_SLOTS = 256;
void launch_dtreset(unsigned long long * dtmin, cudaStream_t st);

// decide_dt: dt_caps[0..2] are the diffusive limits (0 when that direction is
// implicit), written to *dtp together with status bits in *status
void launch_decide_dt(const Geo & g, const FieldBufs & f, double coef_adv, const double * dt_caps,
                      unsigned long long * dtmin, double * dtp, unsigned * status, cudaStream_t st);
void launch_dtmin(const Geo & g, const FieldBufs & f, unsigned long long * dtmin, unsigned * status, cudaStream_t st);
void launch_dtfinal(double coef_adv, const double * dt_caps, unsigned long long * dtmin, double * dtp,
                    unsigned * status, cudaStream_t st);

// boundary conditions + periodic images of a single field (boundary/*.c)
enum BcKind { BC_UX = 0, BC_UY, BC_UZ, BC_P, BC_PSI, BC_T };
// a: the field, bytes per value 8 or 4 (p and psi are always double)
void launch_bc(const Geo & g, const Bc & bc, BcKind kind, void * a, int bytes, cudaStream_t st);

// velocity-gradient tensors with halos (predict/l*.c), for logging/statistics
struct Tensors { double * a[11]; };  // lxx lxy lxz lyx0 lyx1 lyy0 lyy1 lyz lzx lzy lzz
void launch_tensors(const Geo & g, const Coefs & cf, const FieldBufs & f, const Tensors & tn, cudaStream_t st);

// logging reductions (src/logging/*.c); out: 9 doubles on the device,
// partial: DIAG_BLOCKS x 9 doubles of scratch; f: current fields, fs: the
// fields the momentum injection / dissipation tensors are formed from
constexpr int DIAG_BLOCKS_MAX = 296;
void launch_diagnostics(const Geo & g, const Coefs & cf, const Bc & bc, const FieldBufs & f, const FieldBufs & fs,
                        double nu, double kappa, double * out, double * partial, cudaStream_t st);

// statistics of src/statistics.c:124-240 accumulated on the device, in the
// reference's dump layouts: ux1, ux2 [k][j][i = 1..nx+1]; uy1, uy2, uz1, uz2
// [k][j][i = 0..nx+1]; adv, dif [k][j][i = 1..nx+1] (interior j, k only).
// f: current fields (means, adv); fs: the fields dif's tensors are formed from
struct Stats { double * a[8]; };     // ux1 ux2 uy1 uy2 uz1 uz2 adv dif
void launch_statistics(const Geo & g, const Coefs & cf, const FieldBufs & f, const FieldBufs & fs, const Stats & s,
                       cudaStream_t st);
// mean of uy1 over j and k, divided by the sample count: nx + 2 values
void launch_stat_profile(const Geo & g, const double * uy1, double inv_count, double * out, cudaStream_t st);

// seeded initial field on the device: uy_prof[i], t_prof[i] (i = 0..nx+1,
// device arrays) plus uniform noise of amplitude amp_u (ux, uy, uz) and amp_t (t)
void launch_initial_field(const Geo & g, const FieldBufs & f, const double * uy_prof, const double * t_prof,
                          unsigned long long seed, double amp_u, double amp_t, cudaStream_t st);

// values of one field at radial indices i0 .. i0+count-1 over the interior
// j, k into out[((k-1) ny + j-1) count + c] (doubles; a: 8 or 4 bytes per value)
void launch_slab(const Geo & g, const void * a, int bytes, bool face, int i0, int count, double * out,
                 cudaStream_t st);

// FP32-storage mode: rows of nref doubles in the reference's layout to and from
// rows of pitch floats (element e at e + shift)
void launch_pack32(const double * src, float * dst, size_t rows, int nref, int pitch, int shift, cudaStream_t st);
void launch_unpack32(const float * src, double * dst, size_t rows, int nref, int pitch, int shift, cudaStream_t st);

// learned closure (tc_closure.cu): 4x restriction of a fine state, network
// input of a coarse state, network output into the predict forcing
void launch_coarsen(const Geo & gf, const FieldsT<double> & f, const Geo & gc, const FieldsT<double> & c,
                    cudaStream_t st);
void launch_closure_input(const Geo & g, const double * ux, const double * uy, const double * uz, const double s[3],
                          int cp, void * out, cudaStream_t st);
void launch_closure_forcing(int nx, int ny, int nz, const float * f, int nc, const double s[3], double * fux,
                            double * fuy, double * fuz, cudaStream_t st);
void launch_closure_target(const Geo & g, const FieldsT<double> & pred, const FieldsT<double> & ref, double tau,
                           float * out, cudaStream_t st);

}  // namespace tcgpu
