// Host runtime of tcgpu: per-fluid device contexts, the step schedule (one
// CUDA stream, the full time step captured once as a CUDA graph), host<->device
// coherence, and the exported C entry points of include/tcgpu.h.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <chrono>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "tcgpu.h"
#include "tc_common.cuh"
#include "tc_kernels.h"

using namespace tcgpu;

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

static int fail(const char * fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  fprintf(stderr, "tcgpu: %s\n", buf);
  fflush(stderr);
  return 1;
}

#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) return fail("%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// ------------------------------------------------------------------ parameters
// defaults: the reference's shipped src/param/boundary-condition.c and implicit.c
static tcgpu_params_t g_params = {1.0, 0.0, 0.5, -0.5, 1, 0, 0, -1.0, -1.0};
static std::mutex g_mutex;

// a variable that is set to anything but "" or "0"
static bool env_flag(const char * name) {
  const char * s = getenv(name);
  return s != nullptr && s[0] != '\0' && strcmp(s, "0") != 0;
}

static int env_double(const char * name, double * value) {
  // src/config.c:14-46
  const char * s = getenv(name);
  if (s == nullptr) return fail("%s not found", name);
  errno = 0;
  *value = strtod(s, nullptr);
  if (errno != 0) return fail("%s: invalid value as double", name);
  return 0;
}

// ------------------------------------------------------------------ context
struct Ctx {
  const fluid_t * key = nullptr;
  int nx = 0, ny = 0, nz = 0;
  size_t nc = 0, nf = 0;
  Geo g{};
  Bc bc{};
  Coefs cf{};
  XFactors xf{};
  YZFactors yf{};
  Poisson ps{};
  int sb = 8;           // bytes per stored value of ux, uy, uz, t, sources, spectra: 8, or 4 (FP32 storage)
  FieldBufs fb[2]{};    // ux, uy, uz, t double-buffered; p and psi shared
  int cur = 0;          // buffer holding the current state
  void * src[4][2]{};
  double * stage = nullptr;   // FP32 storage: reference-layout doubles between host and device
  double * frc[4]{};          // closure forcing of ux, uy, uz (packed interior layout; frc[3] unused)
  bool forcing = false;       // add frc to the explicit terms in every predict
  DeltaSet ds{};
  double * tab_y = nullptr;
  double * tab_z = nullptr;
  double * base = nullptr;
  double * dt_caps = nullptr;
  double * dtp = nullptr;
  unsigned long long * dtmin = nullptr;
  // dtmin holds the advective limit of the current fields, folded in by the
  // last correction of the previous step (reset to 1.0 whenever that stops
  // being true)
  bool dt_ready = false;
  unsigned * status = nullptr;
  double * diag_out = nullptr;
  double * diag_part = nullptr;
  Tensors tn{};
  bool have_tn = false;
  // fb[cur ^ 1] holds the input fields of the last predict: every predict
  // writes the other buffer of the pair and leaves its input in place until the
  // next predict, and nothing else writes that buffer. The reference's logging
  // and statistics read the velocity-gradient tensors of exactly those fields
  // (src/fluid/predict/main.c:56-82 is their only writer).
  bool have_prev = false;
  double * slab = nullptr;    // tcgpu_radial_slab staging, slab_n doubles
  size_t slab_n = 0;
  Stats stats{};              // device statistics (src/statistics.c), allocated on first use
  size_t stat_num = 0;
  double * stat_prof = nullptr;
  double coef_adv = 0., coef_dif = 0.;
  double Re = 0., Pr = 0., nu = 0., kappa = 0.;
  double caps_h[3] = {0., 0., 0.};
  unsigned coherence = 0;
  cudaStream_t st = nullptr;
  cudaGraphExec_t step_graph[2] = {nullptr, nullptr};   // one per starting buffer
  int graph_launches[TCGPU_K_COUNT] = {0};
  FieldBufs & f() { return fb[cur]; }
  std::vector<void *> pinned;     // caller arrays registered with cudaHostRegister
  double * h_scalar = nullptr;    // pinned: dt in / out
  unsigned * h_status = nullptr;  // pinned
  std::vector<void *> allocs;
};

static std::map<const fluid_t *, Ctx *> g_ctx;
static int g_storage_bytes = 8;   // storage of contexts created from now on

static void * valloc(Ctx & c, size_t bytes) {
  void * p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, bytes);
  c.allocs.push_back(p);
  return p;
}

static double * dalloc(Ctx & c, size_t n) {
  void * p = nullptr;
  if (cudaMalloc(&p, n * sizeof(double)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, n * sizeof(double));
  c.allocs.push_back(p);
  return static_cast<double *>(p);
}

static void destroy_ctx(Ctx * c) {
  if (c == nullptr) return;
  if (c->st) cudaStreamSynchronize(c->st);
  for (int b = 0; b < 2; b++) if (c->step_graph[b]) cudaGraphExecDestroy(c->step_graph[b]);
  for (void * p : c->pinned) cudaHostUnregister(p);
  for (void * p : c->allocs) cudaFree(p);
  if (c->h_scalar) cudaFreeHost(c->h_scalar);
  if (c->h_status) cudaFreeHost(c->h_status);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}


// metric accessors of the reference's domain_t (array_macros/domain/*.h)
struct Metric {
  std::vector<double> hxxf, hxxc, hyxf, hyxc, jdxf, jdxc;  // length nx+2, index = i
};

static void read_metric(const domain_t * d, int nx, Metric & m) {
  m.hxxf.assign(nx + 3, 0.);
  m.hxxc.assign(nx + 3, 0.);
  m.hyxf.assign(nx + 3, 0.);
  m.hyxc.assign(nx + 3, 0.);
  m.jdxf.assign(nx + 3, 0.);
  m.jdxc.assign(nx + 3, 0.);
  for (int i = 1; i <= nx + 1; i++) {
    m.hxxf[i] = d->hxxf[i - 1];
    m.hyxf[i] = d->hyxf[i - 1];
    m.jdxf[i] = d->jdxf[i - 1];
  }
  for (int i = 0; i <= nx + 1; i++) {
    m.hxxc[i] = d->hxxc[i];
    m.hyxc[i] = d->hyxc[i];
    m.jdxc[i] = d->jdxc[i];
  }
}

static int resolve_coefs(Ctx & c) {
  if (g_params.coef_dt_adv >= 0.) c.coef_adv = g_params.coef_dt_adv;
  else if (env_double("coef_dt_adv", &c.coef_adv)) return 1;
  if (g_params.coef_dt_dif >= 0.) c.coef_dif = g_params.coef_dt_dif;
  else if (env_double("coef_dt_dif", &c.coef_dif)) return 1;
  return 0;
}

// diffusivities and the diffusive dt limits (src/decide_dt.c:89-115)
static int set_physics(Ctx & c, const fluid_t * fl, const domain_t * d) {
  if (c.Re == fl->Re && c.Pr == fl->Pr && c.nu != 0.) return 0;
  c.Re = fl->Re;
  c.Pr = fl->Pr;
  c.nu = 1. / fl->Re;                      // compute_diffusivity.c
  c.kappa = 1. / fl->Re / fl->Pr;
  const double diffusivity = fmax(c.nu, c.kappa);
  double gs[3];
  gs[0] = 1.7976931348623157e308;
  for (int i = 0; i <= c.nx + 1; i++) gs[0] = fmin(gs[0], d->hxxc[i]);
  gs[1] = d->hyxc[1];
  gs[2] = d->hz;
  for (int dim = 0; dim < 3; dim++) {
    const double v = c.coef_dif / diffusivity * 0.5 / 3 * pow(gs[dim], 2.);
    c.caps_h[dim] = c.bc.implicit[dim] ? 0. : v;
  }
  CK(cudaMemcpy(c.dt_caps, c.caps_h, sizeof(c.caps_h), cudaMemcpyHostToDevice));
  for (int b = 0; b < 2; b++) {
    if (c.step_graph[b]) {
      cudaGraphExecDestroy(c.step_graph[b]);
      c.step_graph[b] = nullptr;
    }
  }
  return 0;
}

static int build_tables(Ctx & c, const domain_t * d) {
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  const size_t L = (size_t)nx + 2;
  Metric m;
  read_metric(d, nx, m);
  const double hz = d->hz;
  auto HXXF = [&](int i) { return m.hxxf[i]; };
  auto HXXC = [&](int i) { return m.hxxc[i]; };
  auto HYXF = [&](int i) { return m.hyxf[i]; };
  auto HYXC = [&](int i) { return m.hyxc[i]; };
  auto JDXF = [&](int i) { return m.jdxf[i]; };
  auto JDXC = [&](int i) { return m.jdxc[i]; };
  if (L > (size_t)CSTRIDE) return fail("nx = %d too large for the coefficient tables", nx);
  std::vector<double> T((size_t)NCOEF_TABLES * CSTRIDE, 0.);
  auto col = [&](int n) { return T.data() + (size_t)n * CSTRIDE; };
  constexpr int NCOL = NCOEF_TABLES;
  for (int i = 2; i <= nx; i++) {   // ux at face i (ux.c)
    col(F_INVJD)[i] = 1. / JDXF(i);
    col(F_A1)[i] = 0.5 * JDXF(i - 1) / HXXF(i - 1);
    col(F_A2)[i] = 0.5 * JDXF(i) / HXXF(i);
    col(F_A3)[i] = 0.5 * JDXF(i + 1) / HXXF(i + 1);
    col(F_B1)[i] = 0.5 * JDXC(i - 1) / HYXC(i - 1);
    col(F_B2)[i] = 0.5 * JDXC(i) / HYXC(i);
    col(F_C1)[i] = 0.5 * JDXC(i - 1) / hz;
    col(F_C2)[i] = 0.5 * JDXC(i) / hz;
    const double djdhx_xm = -JDXF(i - 1) / HXXF(i - 1) + JDXF(i) / HXXF(i);
    const double djdhx_xp = -JDXF(i) / HXXF(i) + JDXF(i + 1) / HXXF(i + 1);
    col(F_HD1)[i] = 0.5 * djdhx_xm;
    col(F_HD2)[i] = 0.5 * djdhx_xp;
    const double l = 1. / JDXF(i) * JDXC(i - 1) / HXXC(i - 1) / HXXC(i - 1);   // ux.c:38-43
    const double u = 1. / JDXF(i) * JDXC(i) / HXXC(i) / HXXC(i);
    col(F_LXL)[i] = l;
    col(F_LXC)[i] = -l - u;
    col(F_LXU)[i] = u;
    const double ly = 1. / HYXF(i) / HYXF(i);                                 // ux.c:52-54
    col(F_LYL)[i] = ly;
    col(F_LYC)[i] = -ly - ly;
    col(F_LYU)[i] = ly;
    col(F_E1)[i] = JDXF(i) / HYXF(i);
    col(F_E2)[i] = JDXF(i) / hz;
  }
  for (int i = 1; i <= nx + 1; i++) {  // face quantities
    const double djdhx = -JDXC(i - 1) / HXXC(i - 1) + JDXC(i) / HXXC(i);
    col(C_LYX1F)[i] = -1. / JDXF(i) * djdhx;                                  // lyx.c:79-82
    col(C_WM)[i] = (i == 1) ? 0. : 0.5;
    col(C_WP)[i] = (i == nx + 1) ? 0. : 0.5;
    col(C_INVHXXF)[i] = 1. / HXXF(i);
    col(C_INVHYXF)[i] = 1. / HYXF(i);
    col(C_JF)[i] = JDXF(i) / HXXF(i);
  }
  for (int i = 1; i <= nx; i++) {      // cell-centred variables at i
    col(C_INVHYXC)[i] = 1. / HYXC(i);
    const double djdhx = -JDXF(i) / HXXF(i) + JDXF(i + 1) / HXXF(i + 1);
    col(C_LYY1)[i] = 1. / JDXC(i) * djdhx;                                    // lyy.c:79-82
    col(C_INVJDXC)[i] = 1. / JDXC(i);
    col(C_A1)[i] = 0.5 * JDXF(i) / HXXF(i);
    col(C_A2)[i] = 0.5 * JDXF(i + 1) / HXXF(i + 1);
    col(C_B)[i] = 0.5 * JDXC(i) / HYXC(i);
    col(C_CZ)[i] = 0.5 * JDXC(i) / hz;
    col(C_HD)[i] = 0.5 * djdhx;
    const double l = 1. / JDXC(i) * JDXF(i) / HXXF(i) / HXXF(i);              // uy.c:38-43
    const double u = 1. / JDXC(i) * JDXF(i + 1) / HXXF(i + 1) / HXXF(i + 1);
    col(C_LXL)[i] = l;
    col(C_LXC)[i] = -l - u;
    col(C_LXU)[i] = u;
    const double ly = 1. / HYXC(i) / HYXC(i);
    col(C_LYL)[i] = ly;
    col(C_LYC)[i] = -ly - ly;
    col(C_LYU)[i] = ly;
    col(C_E1)[i] = JDXC(i) / HYXC(i);
    col(C_E2)[i] = JDXC(i) / hz;
    const double dm = -JDXC(i - 1) / HXXC(i - 1) + JDXC(i) / HXXC(i);
    const double dp = -JDXC(i) / HXXC(i) + JDXC(i + 1) / HXXC(i + 1);
    col(C_HDA1)[i] = 0.5 * dm;
    col(C_HDA2)[i] = 0.5 * dp;
    col(C_PXL)[i] = JDXF(i) / HXXF(i) / HXXF(i);
    col(C_PXU)[i] = JDXF(i + 1) / HXXF(i + 1) / HXXF(i + 1);
    col(C_PYL)[i] = JDXC(i) / HYXC(i) / HYXC(i);
    col(C_PZL)[i] = JDXC(i) / hz / hz;
  }
  // products for the marching predict kernel (tc_march.cu); each term's
  // derivation is beside its use there
  for (int i = 2; i <= nx; i++) {
    const double invj = col(F_INVJD)[i];
    col(P_XA1)[i] = 0.5 * invj * col(F_A1)[i];
    col(P_XA2)[i] = 0.5 * invj * col(F_A2)[i];
    col(P_XA3)[i] = 0.5 * invj * col(F_A3)[i];
    col(P_YB1)[i] = 0.5 * invj * col(F_B1)[i];
    col(P_YB2)[i] = 0.5 * invj * col(F_B2)[i];
    col(P_ZC1)[i] = 0.5 * invj * col(F_C1)[i];
    col(P_ZC2)[i] = 0.5 * invj * col(F_C2)[i];
    col(P_H1)[i] = 0.25 * invj * col(F_HD1)[i];
    col(P_H2)[i] = 0.25 * invj * col(F_HD2)[i];
    const double jh = col(F_E1)[i], F = col(C_LYX1F)[i], wm = col(C_WM)[i], wp = col(C_WP)[i];
    const double ih = col(C_INVHXXF)[i];
    const double hm = col(C_INVHYXC)[i - 1], h0 = col(C_INVHYXC)[i];
    const double km = col(C_LYY1)[i - 1], k0 = col(C_LYY1)[i];
    const double hd1 = col(F_HD1)[i], hd2 = col(F_HD2)[i];
    col(P_CY1)[i] = invj * (jh * (F * wm - ih) - 2. * hd1 * hm);
    col(P_CY2)[i] = invj * (jh * (F * wp + ih) - 2. * hd2 * h0);
    col(P_CA1)[i] = -invj * hd1 * km;
    col(P_CA2)[i] = -invj * hd2 * k0;
    col(P_CZ1)[i] = invj * col(F_E2)[i] * ih;
  }
  for (int i = 1; i <= nx; i++) {
    const double invjc = col(C_INVJDXC)[i];
    col(P_TX0)[i] = 0.5 * invjc * col(C_JF)[i];
    col(P_TX1)[i] = 0.5 * invjc * col(C_JF)[i + 1];
    col(P_TY)[i] = 0.5 * invjc * col(C_E1)[i];
    col(P_TZ)[i] = 0.5 * invjc * col(C_E2)[i];
    col(P_UA1)[i] = 0.5 * invjc * col(C_A1)[i];
    col(P_UA2)[i] = 0.5 * invjc * col(C_A2)[i];
    col(P_UB)[i] = 0.5 * invjc * col(C_B)[i];
    col(P_UC)[i] = 0.5 * invjc * col(C_CZ)[i];
    col(P_UH)[i] = 0.25 * invjc * col(C_HD)[i];
    const double hf0 = col(C_INVHYXF)[i], hf1 = col(C_INVHYXF)[i + 1];
    const double F0 = col(C_LYX1F)[i], F1 = col(C_LYX1F)[i + 1];
    const double wm0 = col(C_WM)[i], wp0 = col(C_WP)[i], wm1 = col(C_WM)[i + 1], wp1 = col(C_WP)[i + 1];
    const double jf0 = col(C_JF)[i], jf1 = col(C_JF)[i + 1];
    const double hx0 = col(C_INVHXXF)[i], hx1 = col(C_INVHXXF)[i + 1];
    const double a1 = col(C_HDA1)[i] - jf0, a2 = col(C_HDA2)[i] + jf1;
    col(P_P1)[i] = invjc * a1 * hf0;
    col(P_P2)[i] = invjc * a2 * hf1;
    col(P_QM)[i] = invjc * (a1 * F0 * wm0 - col(C_HDA1)[i] * hx0);
    col(P_Q0)[i] = invjc * (a1 * F0 * wp0 + a2 * F1 * wm1 + col(C_HDA1)[i] * hx0 - col(C_HDA2)[i] * hx1);
    col(P_QP)[i] = invjc * (a2 * F1 * wp1 + col(C_HDA2)[i] * hx1);
    col(P_YK)[i] = invjc * col(C_E1)[i] * col(C_LYY1)[i];
    col(P_YZ)[i] = invjc * col(C_E2)[i] * col(C_INVHYXC)[i];
    col(P_ZX0)[i] = invjc * jf0 / hz;
    col(P_ZX1)[i] = invjc * jf1 / hz;
    col(P_ZY)[i] = invjc * col(C_E1)[i] / hz;
  }
  double * dT = dalloc(c, T.size());
  if (!dT) return fail("cudaMalloc of coefficient tables failed");
  CK(cudaMemcpy(dT, T.data(), T.size() * sizeof(double), cudaMemcpyHostToDevice));
  const double * cols[NCOL];
  for (int n = 0; n < NCOL; n++) cols[n] = dT + (size_t)n * CSTRIDE;
  Coefs & cf = c.cf;
  cf.tab = dT;
  // tables reached through named pointers: F_INVJD .. C_PZL (the P_* tables
  // are read from tab with their offsets)
  constexpr int NNAMED = C_PZL + 1;
  const double ** dst[] = {&cf.f_invjd, &cf.f_a1, &cf.f_a2, &cf.f_a3, &cf.f_b1, &cf.f_b2, &cf.f_c1, &cf.f_c2,
      &cf.f_hd1, &cf.f_hd2, &cf.f_lxl, &cf.f_lxc, &cf.f_lxu, &cf.f_lyl, &cf.f_lyc, &cf.f_lyu, &cf.f_e1, &cf.f_e2,
      &cf.c_lyx1f, &cf.c_wm, &cf.c_wp, &cf.c_invhxxf, &cf.c_invhyxc, &cf.c_invhyxf, &cf.c_lyy1, &cf.c_invjdxc,
      &cf.c_a1, &cf.c_a2, &cf.c_b, &cf.c_cz, &cf.c_hd, &cf.c_lxl, &cf.c_lxc, &cf.c_lxu, &cf.c_lyl, &cf.c_lyc,
      &cf.c_lyu, &cf.c_jf, &cf.c_e1, &cf.c_e2, &cf.c_hda1, &cf.c_hda2, &cf.c_pxl, &cf.c_pxu, &cf.c_pyl, &cf.c_pzl};
  static_assert(sizeof(dst) / sizeof(dst[0]) == NNAMED, "one named pointer per table F_INVJD .. C_PZL");
  for (int n = 0; n < NNAMED; n++) *dst[n] = cols[n];
  const double lz = 1. / hz / hz;
  cf.lz_l = lz;
  cf.lz_c = -lz - lz;
  cf.lz_u = lz;
  cf.inv_hz = 1. / hz;

  // geometry tables
  std::vector<double> G(6 * L, 0.);
  for (int i = 0; i <= nx + 1; i++) {
    G[0 * L + i] = m.hxxf[i];
    G[1 * L + i] = m.hxxc[i];
    G[2 * L + i] = m.hyxf[i];
    G[3 * L + i] = m.hyxc[i];
    G[4 * L + i] = m.jdxf[i];
    G[5 * L + i] = m.jdxc[i];
  }
  double * dG = dalloc(c, G.size());
  if (!dG) return fail("cudaMalloc failed");
  CK(cudaMemcpy(dG, G.data(), G.size() * sizeof(double), cudaMemcpyHostToDevice));
  c.g.nx = nx;
  c.g.ny = ny;
  c.g.nz = nz;
  c.g.hz = hz;
  c.g.hxxf = dG;
  c.g.hxxc = dG + L;
  c.g.hyxf = dG + 2 * L;
  c.g.hyxc = dG + 3 * L;
  c.g.jdxf = dG + 4 * L;
  c.g.jdxc = dG + 5 * L;

  // packed per-variable Laplacians for the implicit solves
  std::vector<double> P((size_t)4 * 6 * L, 0.);  // [var][lx l c u, ly l c u][L]
  for (int v = 0; v < 4; v++) {
    const int i0 = (v == VUX) ? 2 : 1;
    const int n = nx - i0 + 1;
    for (int e = 0; e < n; e++) {
      const int i = e + i0;
      double * b = P.data() + (size_t)v * 6 * L;
      if (v == VUX) {
        b[0 * L + e] = col(F_LXL)[i]; b[1 * L + e] = col(F_LXC)[i]; b[2 * L + e] = col(F_LXU)[i];
        b[3 * L + e] = col(F_LYL)[i]; b[4 * L + e] = col(F_LYC)[i]; b[5 * L + e] = col(F_LYU)[i];
      } else {
        b[0 * L + e] = col(C_LXL)[i]; b[1 * L + e] = col(C_LXC)[i]; b[2 * L + e] = col(C_LXU)[i];
        b[3 * L + e] = col(C_LYL)[i]; b[4 * L + e] = col(C_LYC)[i]; b[5 * L + e] = col(C_LYU)[i];
      }
    }
  }
  double * dP = dalloc(c, P.size());
  if (!dP) return fail("cudaMalloc failed");
  CK(cudaMemcpy(dP, P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice));
  // factor rows cover every element a solving warp touches (32 lanes x
  // elements per lane) and start on 16-byte boundaries for paired loads
  const size_t LX = ((std::max(L, (size_t)32 * predict_warps(nx)) + 1) / 2) * 2;
  c.xf.stride = LX;
  c.xf.ne = predict_warps(nx);   // the march kernel solves with E = its warp count elements per lane
  for (int v = 0; v < 4; v++) {
    c.xf.n[v] = (v == VUX) ? nx - 1 : nx;
    c.xf.lap_l[v] = dP + (size_t)v * 6 * L;
    c.xf.lap_c[v] = dP + (size_t)v * 6 * L + L;
    c.xf.lap_u[v] = dP + (size_t)v * 6 * L + 2 * L;
  }
  c.xf.lo = dalloc(c, 12 * LX);
  c.xf.w = dalloc(c, 12 * LX);
  c.xf.v = dalloc(c, 12 * LX);
  if (c.bc.implicit[1] || c.bc.implicit[2]) {
    YZFactors & yf = c.yf;
    yf.max_i = nx;
    yf.stride_y = (size_t)nx * ny;
    yf.stride_z = (size_t)nz;
    for (int v = 0; v < 4; v++) {
      yf.n_i[v] = (v == VUX) ? nx - 1 : nx;
      yf.lapy_l[v] = dP + (size_t)v * 6 * L + 3 * L;
      yf.lapy_c[v] = dP + (size_t)v * 6 * L + 4 * L;
      yf.lapy_u[v] = dP + (size_t)v * 6 * L + 5 * L;
    }
    yf.uniform_y = 1;
    for (int v = 0; v < 4; v++) {
      const double * b = P.data() + (size_t)v * 6 * L;
      for (int e = 1; e < yf.n_i[v]; e++)
        for (int r = 3; r < 6; r++)
          if (b[r * L + e] != b[r * L]) yf.uniform_y = 0;
    }
    yf.lapz_l = cf.lz_l;
    yf.lapz_c = cf.lz_c;
    yf.lapz_u = cf.lz_u;
    yf.l = dalloc(c, 12 * (size_t)nx);
    yf.c = dalloc(c, 12 * (size_t)nx);
    yf.u = dalloc(c, 12 * (size_t)nx);
    yf.v = dalloc(c, 12 * yf.stride_y);
    yf.w = dalloc(c, 12 * yf.stride_y);
    yf.q1 = dalloc(c, 12 * yf.stride_y);
    yf.lz = dalloc(c, 12);
    yf.cz = dalloc(c, 12);
    yf.uz = dalloc(c, 12);
    yf.vz = dalloc(c, 12 * (size_t)nz);
    yf.wz = dalloc(c, 12 * (size_t)nz);
    yf.q1z = dalloc(c, 12 * (size_t)nz);
  }

  // Poisson tables (compute_potential.c:173-211, 311-349)
  const int nyh = ny / 2 + 1;
  c.ps.nyh = nyh;
  c.ps.status = c.status;
  std::vector<double> tl(nx), tu(nx), base(nx), tz(nz), ty((size_t)nx * nyh);
  for (int i = 1; i <= nx; i++) {
    tl[i - 1] = 1. / JDXC(i) * JDXF(i) / HXXF(i) / HXXF(i);
    tu[i - 1] = 1. / JDXC(i) * JDXF(i + 1) / HXXF(i + 1) / HXXF(i + 1);
    base[i - 1] = -tl[i - 1] - tu[i - 1];
  }
  const double g_pi = 3.14159265358979324;
  std::vector<double> ey(nyh), ez(nz);
  for (int n = 0; n < nyh; n++) {
    const double s = sin(g_pi * n / ny);
    ey[n] = -4. * (s * s);
  }
  for (int n = 0; n < nz; n++) {
    const double s = sin(g_pi * n / nz);
    ez[n] = -4. * (s * s);
    tz[n] = ez[n] / hz / hz;
  }
  for (int i = 1; i <= nx; i++)
    for (int n = 0; n < nyh; n++) ty[(size_t)(i - 1) * nyh + n] = ey[n] / HYXC(i) / HYXC(i);
  double * dtl = dalloc(c, nx);
  double * dtu = dalloc(c, nx);
  c.base = dalloc(c, nx);
  c.tab_z = dalloc(c, nz);
  c.tab_y = dalloc(c, (size_t)nx * nyh);
  if (!dtl || !dtu || !c.base || !c.tab_z || !c.tab_y) return fail("cudaMalloc failed");
  CK(cudaMemcpy(dtl, tl.data(), nx * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dtu, tu.data(), nx * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c.base, base.data(), nx * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c.tab_z, tz.data(), nz * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c.tab_y, ty.data(), ty.size() * sizeof(double), cudaMemcpyHostToDevice));
  c.ps.tl = dtl;
  c.ps.tu = dtu;
  // twiddles exp(-2 pi i m / N), m < N, from libm
  auto twiddles = [&](int N) -> double2 * {
    std::vector<double> tw(2 * (size_t)N);
    for (int k = 0; k < N; k++) {
      const double a = 2. * g_pi * k / N;
      tw[2 * k] = cos(a);
      tw[2 * k + 1] = -sin(a);
    }
    double * p = dalloc(c, 2 * (size_t)N);
    if (p) cudaMemcpy(p, tw.data(), 2 * (size_t)N * sizeof(double), cudaMemcpyHostToDevice);
    return reinterpret_cast<double2 *>(p);
  };
  c.ps.tw_y = twiddles(ny);
  c.ps.tw_z = twiddles(nz);
  // FP32-storage contexts transform in float: the same tables rounded once
  auto twiddles32 = [&](int N) -> float2 * {
    std::vector<float> tw(2 * (size_t)N);
    for (int k = 0; k < N; k++) {
      const double a = 2. * g_pi * k / N;
      tw[2 * k] = (float)cos(a);
      tw[2 * k + 1] = (float)-sin(a);
    }
    float * p = static_cast<float *>(valloc(c, 2 * (size_t)N * sizeof(float)));
    if (p) cudaMemcpy(p, tw.data(), 2 * (size_t)N * sizeof(float), cudaMemcpyHostToDevice);
    return reinterpret_cast<float2 *>(p);
  };
  if (c.sb == 4) {
    c.ps.tw_y32 = twiddles32(ny);
    c.ps.tw_z32 = twiddles32(nz);
    if (!c.ps.tw_y32 || !c.ps.tw_z32) return fail("cudaMalloc of Poisson buffers failed");
  }
  const size_t nspec = (size_t)nx * nz * nyh;
  c.ps.spec_bytes = 2 * c.sb;
  c.ps.spec = valloc(c, nspec * c.ps.spec_bytes);
  c.ps.vscr = dalloc(c, nspec);
  if (!c.ps.tw_y || !c.ps.tw_z || !c.ps.spec || !c.ps.vscr) return fail("cudaMalloc of Poisson buffers failed");
  // radial solves by warps when nx = 32 E: per-line factors computed once
  c.ps.fe = (nx == 64 || nx == 128 || nx == 256) ? nx / 32 : 0;
  if (c.ps.fe) {
    c.ps.fw = dalloc(c, nspec);
    c.ps.fv = c.ps.vscr;   // not otherwise used on this path
    if (!c.ps.fw) return fail("cudaMalloc of Poisson buffers failed");
    launch_tdm_factors(c.g, c.ps, c.tab_y, c.tab_z, c.base, c.st);
    CK(cudaGetLastError());
  }
  return 0;
}

static int check_domain(const domain_t * d) {
  if (d == nullptr) return fail("domain is NULL");
  for (int dim = 0; dim < 3; dim++) {
    if (d->mysizes[dim] != d->glsizes[dim] || d->offsets[dim] != 0)
      return fail("only a single rank owning the whole domain is supported (dim %d: mysize %zu, glsize %zu, offset %zu)",
                  dim, d->mysizes[dim], d->glsizes[dim], d->offsets[dim]);
  }
  const size_t nx = d->glsizes[0], ny = d->glsizes[1], nz = d->glsizes[2];
  if (nx < 2 || nx > 1024) return fail("nx = %zu outside the supported range [2, 1024]", nx);
  // any even ny and any nz that is a multiple of 4 (powers of two take the
  // FFT kernels, other lengths direct transforms)
  if (ny < 4 || ny > 2048 || ny % 2 || nz < 4 || nz > 2048 || nz % 4)
    return fail("ny = %zu must be even and nz = %zu a multiple of 4, both in [4, 2048]", ny, nz);
  if (!d->hxxf || !d->hxxc || !d->hyxf || !d->hyxc || !d->jdxf || !d->jdxc)
    return fail("domain metric arrays are not initialised");
  return 0;
}

static Ctx * create_ctx(const domain_t * d, const fluid_t * fl) {
  if (check_domain(d)) return nullptr;
  Ctx * c = new Ctx();
  c->key = fl;
  c->nx = (int)d->glsizes[0];
  c->ny = (int)d->glsizes[1];
  c->nz = (int)d->glsizes[2];
  c->nc = (size_t)(c->nx + 2) * (c->ny + 2) * (c->nz + 2);
  c->nf = (size_t)(c->nx + 1) * (c->ny + 2) * (c->nz + 2);
  c->g.nx = c->nx;
  c->g.ny = c->ny;
  c->g.nz = c->nz;
  c->sb = g_storage_bytes;
  c->bc.uy_xm = g_params.uy_xm;
  c->bc.uy_xp = g_params.uy_xp;
  c->bc.t_xm = g_params.t_xm;
  c->bc.t_xp = g_params.t_xp;
  c->bc.implicit[0] = g_params.implicit_x ? 1 : 0;
  c->bc.implicit[1] = g_params.implicit_y ? 1 : 0;
  c->bc.implicit[2] = g_params.implicit_z ? 1 : 0;
  // a host that cannot call tcgpu_set_coherence (the reference's own main.c)
  // opts in to the extra copies through the environment
  if (env_flag("TCGPU_SYNC_TENSORS")) c->coherence |= TCGPU_SYNC_TENSORS;
  if (env_flag("TCGPU_SYNC_SRCS")) c->coherence |= TCGPU_SYNC_SRCS;
  auto bad = [&](const char * what) { fail("%s", what); destroy_ctx(c); return (Ctx *)nullptr; };
  if (resolve_coefs(*c)) { destroy_ctx(c); return nullptr; }
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) return bad("cudaStreamCreate failed");
  double * p = dalloc(*c, c->nc);
  double * psi = dalloc(*c, c->nc);
  if (!p || !psi) return bad("cudaMalloc of fields failed");
  const bool f32 = c->sb == 4;
  const size_t nsf = f32 ? scount_f<float>(c->g) : c->nf, nsc = f32 ? scount_c<float>(c->g) : c->nc;
  for (int b = 0; b < 2; b++) {
    FieldBufs & F = c->fb[b];
    F.ux = valloc(*c, nsf * c->sb);
    F.uy = valloc(*c, nsc * c->sb);
    F.uz = valloc(*c, nsc * c->sb);
    F.t = valloc(*c, nsc * c->sb);
    F.p = p;
    F.psi = psi;
    F.bytes = c->sb;
    if (!F.ux || !F.uy || !F.uz || !F.t) return bad("cudaMalloc of fields failed");
  }
  if (f32) {
    c->stage = dalloc(*c, c->nc);
    if (!c->stage) return bad("cudaMalloc of the staging buffer failed");
  }
  const size_t nin = (size_t)c->nx * c->ny * c->nz;
  // increments between the predict and separate line solves: implicit y or z,
  // or radial lines longer than the predict kernel's 256 field threads
  const bool need_delta = c->bc.implicit[1] || c->bc.implicit[2] || c->nx > 256;
  for (int v = 0; v < 4; v++) {
    const size_t n = (v == VUX) ? (size_t)(c->nx - 1) * c->ny * c->nz : nin;
    const size_t ns = f32 ? (size_t)spitch32(c->nx) * c->ny * c->nz : n;
    c->src[v][0] = valloc(*c, ns * c->sb);
    c->src[v][1] = valloc(*c, ns * c->sb);
    if (!c->src[v][0] || !c->src[v][1]) return bad("cudaMalloc of source terms failed");
    if (need_delta) {
      c->ds.d[v] = dalloc(*c, n);
      if (!c->ds.d[v]) return bad("cudaMalloc of increments failed");
    }
  }
  c->dt_caps = dalloc(*c, 3);
  c->dtp = dalloc(*c, 1);
  c->dtmin = reinterpret_cast<unsigned long long *>(dalloc(*c, DT_SLOTS));
  c->status = reinterpret_cast<unsigned *>(dalloc(*c, 1));
  c->diag_out = dalloc(*c, 16);
  c->diag_part = dalloc(*c, (size_t)DIAG_BLOCKS_MAX * 9);
  if (!c->dt_caps || !c->dtp || !c->dtmin || !c->status || !c->diag_out || !c->diag_part) return bad("cudaMalloc failed");
  const std::vector<unsigned long long> ones(DT_SLOTS, 0x3ff0000000000000ull);   // 1.0
  if (cudaMemcpy(c->dtmin, ones.data(), DT_SLOTS * sizeof(ones[0]), cudaMemcpyHostToDevice) != cudaSuccess)
    return bad("cudaMemcpy failed");
  if (cudaMallocHost(&c->h_scalar, 64 * sizeof(double)) != cudaSuccess) return bad("cudaMallocHost failed");
  if (cudaMallocHost(&c->h_status, sizeof(unsigned) * 4) != cudaSuccess) return bad("cudaMallocHost failed");
  if (build_tables(*c, d)) { destroy_ctx(c); return nullptr; }
  poisson_smem_limits();
  march_smem_limits();
  allow_periodic_lines_smem();
  c->nu = 0.;
  if (set_physics(*c, fl, d)) { destroy_ctx(c); return nullptr; }
  return c;
}

static Ctx * get_ctx(const domain_t * d, const fluid_t * fl) {
  if (fl == nullptr) { fail("fluid is NULL"); return nullptr; }
  std::lock_guard<std::mutex> lk(g_mutex);
  auto it = g_ctx.find(fl);
  if (it != g_ctx.end()) {
    Ctx * c = it->second;
    if (d != nullptr && (c->nx != (int)d->glsizes[0] || c->ny != (int)d->glsizes[1] || c->nz != (int)d->glsizes[2])) {
      destroy_ctx(c);
      g_ctx.erase(it);
    } else {
      if (d != nullptr && set_physics(*c, fl, d)) return nullptr;
      return c;
    }
  }
  if (d == nullptr) { fail("no device state for this fluid yet"); return nullptr; }
  Ctx * c = create_ctx(d, fl);
  if (c) g_ctx[fl] = c;
  return c;
}

// ------------------------------------------------------------------ schedule
// Optional per-kernel accounting: an event after each launch (instrumented
// runs only) and a launch count per kernel kind.
struct Recorder {
  bool events = false;
  cudaStream_t st = nullptr;
  std::vector<cudaEvent_t> ev;
  std::vector<int> kind;
  size_t used = 0;
  int launches[TCGPU_K_COUNT] = {0};
  void mark(int k, int n = 1) {
    launches[k] += n;
    if (!events) return;
    if (used == ev.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev.push_back(e);
      kind.push_back(k);
    }
    kind[used] = k;
    cudaEventRecord(ev[used++], st);
  }
  ~Recorder() { for (auto e : ev) cudaEventDestroy(e); }
};
static thread_local Recorder * g_rec = nullptr;
static void mark(int k, int n = 1) { if (g_rec) g_rec->mark(k, n); }

static void * s_new(Ctx & c, int v, int rk) { return c.src[v][rk == 1 ? 1 : 0]; }
static void * s_old(Ctx & c, int v, int rk) { return c.src[v][rk == 1 ? 0 : 1]; }

static void enqueue_factors(Ctx & c) {
  if (c.bc.implicit[0]) { launch_xfactors(c.xf, c.dtp, c.nu, c.kappa, c.st); mark(TCGPU_K_FACTORS); }
  if (c.bc.implicit[1] || c.bc.implicit[2]) { launch_yzfactors(c.g, c.yf, c.dtp, c.nu, c.kappa, c.st); mark(TCGPU_K_FACTORS); }
}

static void enqueue_predict(Ctx & c, int rk) {
  SrcBufs ss;
  ss.bytes = c.sb;
  for (int v = 0; v < 4; v++) {
    ss.new_[v] = s_new(c, v, rk);
    ss.old_[v] = s_old(c, v, rk);
    ss.frc[v] = c.forcing ? c.frc[v] : nullptr;
  }
  const FieldBufs in = c.fb[c.cur];
  const FieldBufs out = c.fb[c.cur ^ 1];
  const bool iy = c.bc.implicit[1], iz = c.bc.implicit[2], tiles = c.nx > 256;
  c.have_prev = true;
  auto predict = [&](int mode) {
    launch_predict_march(c.g, c.bc, c.cf, c.xf, c.nu, c.kappa, in, out, ss, c.ds, c.dtp, rk, mode, c.status, c.st);
  };
  if (!iy && !iz && !tiles) {
    predict(PREDICT_APPLY);
    mark(TCGPU_K_PREDICT);
  } else {
    predict(PREDICT_DELTA);
    mark(TCGPU_K_PREDICT);
    if (tiles && c.bc.implicit[0]) { launch_xsolve(c.g, c.xf, rk, c.ds, c.st); mark(TCGPU_K_YZSOLVE); }
    if (iy) { launch_ysolve(c.g, c.yf, rk, c.ds, c.st); mark(TCGPU_K_YZSOLVE, 4); }
    if (iz) { launch_zsolve(c.g, c.yf, rk, c.ds, c.st); mark(TCGPU_K_YZSOLVE, 4); }
    launch_apply(c.g, c.bc, in, out, c.ds, c.st);
    mark(TCGPU_K_APPLY);
  }
  c.cur ^= 1;
}

static void enqueue_potential(Ctx & c, int rk) {
  PoissonMarks pm;
  pm.mark = g_rec ? &mark : nullptr;
  pm.k_div = TCGPU_K_DIV_FFTY;
  pm.k_fwd = TCGPU_K_FFTZ_FWD;
  pm.k_tdm = TCGPU_K_TDM;
  pm.k_inv = TCGPU_K_FFTZ_INV;
  pm.k_ify = TCGPU_K_IFFTY;
  launch_poisson(c.g, c.cf, c.ps, c.f(), c.tab_y, c.tab_z, c.base, c.dtp, rk, c.st, pm);
}

static void enqueue_correct(Ctx & c, int rk, int what, bool cfl = false) {
  launch_correct(c.g, c.bc, c.cf, c.f(), c.dtp, rk, c.nu, what, cfl ? c.dtmin : nullptr, c.status, c.st);
  mark(TCGPU_K_CORRECT);
}

static void enqueue_dtmin(Ctx & c) {
  launch_dtmin(c.g, c.f(), c.dtmin, c.status, c.st);
  mark(TCGPU_K_DTMIN);
}

// One step (integrate.c:24-70) after the advective limit of the current
// fields is in dtmin: dt, the factors, three substeps; the last correction
// leaves the next step's advective limit in dtmin.
static void enqueue_step(Ctx & c) {
  launch_dtfinal(c.coef_adv, c.dt_caps, c.dtmin, c.dtp, c.status, c.st);
  mark(TCGPU_K_DTFINAL);
  enqueue_factors(c);
  for (int rk = 0; rk < 3; rk++) {
    enqueue_predict(c, rk);
    enqueue_potential(c, rk);
    enqueue_correct(c, rk, CORRECT_VELOCITY | CORRECT_PRESSURE, rk == 2);
  }
}

static int launch_step(Ctx & c) {
  if (!c.dt_ready) enqueue_dtmin(c);
  const int p = c.cur;
  if (c.step_graph[p] == nullptr) {
    cudaGraph_t graph;
    Recorder count;
    Recorder * prev = g_rec;
    g_rec = &count;
    CK(cudaStreamBeginCapture(c.st, cudaStreamCaptureModeThreadLocal));
    enqueue_step(c);
    CK(cudaStreamEndCapture(c.st, &graph));
    g_rec = prev;
    c.cur = p;   // capture only recorded the launches
    for (int k = 0; k < TCGPU_K_COUNT; k++) c.graph_launches[k] = count.launches[k];
    cudaError_t e = cudaGraphInstantiate(&c.step_graph[p], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail("cudaGraphInstantiate failed: %s", cudaGetErrorString(e));
  }
  CK(cudaGraphLaunch(c.step_graph[p], c.st));
  c.cur = p ^ 1;   // three predicts per step: the state ends in the other buffer
  c.dt_ready = true;
  return 0;
}

// set the device dt from a host value (stage-by-stage entry points)
static int set_dt(Ctx & c, double dt) {
  *c.h_scalar = dt;
  CK(cudaMemcpyAsync(c.dtp, c.h_scalar, sizeof(double), cudaMemcpyHostToDevice, c.st));
  return 0;
}

// the fields are about to change outside a full step: drop the advective limit
// the last step left in dtmin
static void invalidate_dt(Ctx & c) {
  if (!c.dt_ready) return;
  launch_dtreset(c.dtmin, c.st);
  c.dt_ready = false;
}

static int finish(Ctx & c, const char * what) {
  CK(cudaMemcpyAsync(c.h_status, c.status, sizeof(unsigned), cudaMemcpyDeviceToHost, c.st));
  cudaError_t e = cudaStreamSynchronize(c.st);
  if (e != cudaSuccess) return fail("%s: %s", what, cudaGetErrorString(e));
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail("%s: %s", what, cudaGetErrorString(e));
  if (*c.h_status) {
    const unsigned s = *c.h_status;
    cudaMemsetAsync(c.status, 0, sizeof(unsigned), c.st);
    invalidate_dt(c);
    cudaStreamSynchronize(c.st);
    if (s & ST_NONFINITE) return fail("%s: non-finite velocity in the field", what);
    if (s & ST_BADDT) return fail("%s: invalid time step size", what);
    if (s & ST_TIMEOUT) return fail("%s: a device copy did not complete within its wait limit", what);
  }
  return 0;
}

// ------------------------------------------------------------------ coherence
static size_t field_count(const Ctx & c, unsigned bit) { return bit == TCGPU_UX ? c.nf : c.nc; }

static void * dev_field(Ctx & c, unsigned bit) {
  const FieldBufs & f = c.f();
  switch (bit) {
    case TCGPU_UX: return f.ux;
    case TCGPU_UY: return f.uy;
    case TCGPU_UZ: return f.uz;
    case TCGPU_P: return f.p;
    case TCGPU_PSI: return f.psi;
    default: return f.t;
  }
}

static const array_t * host_field(const fluid_t * fl, unsigned bit) {
  switch (bit) {
    case TCGPU_UX: return &fl->ux;
    case TCGPU_UY: return &fl->uy;
    case TCGPU_UZ: return &fl->uz;
    case TCGPU_P: return &fl->p;
    case TCGPU_PSI: return &fl->psi;
    default: return &fl->t;
  }
}

static int check_host_array(const Ctx & c, const array_t * a, size_t n, const char * name) {
  if (a->data == nullptr) return fail("%s: host array is NULL", name);
  if (a->datasize != 0 && a->datasize != n * sizeof(double))
    return fail("%s: host array holds %zu bytes, %zu expected", name, a->datasize, n * sizeof(double));
  (void)c;
  return 0;
}

static const char * field_name(unsigned bit) {
  switch (bit) {
    case TCGPU_UX: return "ux";
    case TCGPU_UY: return "uy";
    case TCGPU_UZ: return "uz";
    case TCGPU_P: return "p";
    case TCGPU_PSI: return "psi";
    default: return "t";
  }
}

// bytes per stored value of a field: p and psi are always double
static int field_bytes(const Ctx & c, unsigned bit) { return (bit == TCGPU_P || bit == TCGPU_PSI) ? 8 : c.sb; }

// FP32 storage: reference-layout rows of a field (nref doubles) and their
// FP32 pitch and shift
static void rows_of(const Ctx & c, unsigned bit, size_t & rows, int & nref, int & pitch, int & shift) {
  rows = (size_t)(c.ny + 2) * (c.nz + 2);
  nref = bit == TCGPU_UX ? c.nx + 1 : c.nx + 2;
  pitch = pitch32(c.nx);
  shift = bit == TCGPU_UX ? 1 : 0;
}

static int push_fields(Ctx & c, const fluid_t * fl, unsigned mask) {
  invalidate_dt(c);
  for (unsigned bit = 1; bit <= TCGPU_T; bit <<= 1) {
    if (!(mask & bit)) continue;
    const array_t * a = host_field(fl, bit);
    const size_t n = field_count(c, bit);
    if (check_host_array(c, a, n, field_name(bit))) return 1;
    if (field_bytes(c, bit) == 8) {
      CK(cudaMemcpyAsync(dev_field(c, bit), a->data, n * sizeof(double), cudaMemcpyHostToDevice, c.st));
    } else {
      size_t rows;
      int nref, pitch, shift;
      rows_of(c, bit, rows, nref, pitch, shift);
      CK(cudaMemcpyAsync(c.stage, a->data, n * sizeof(double), cudaMemcpyHostToDevice, c.st));
      launch_pack32(c.stage, static_cast<float *>(dev_field(c, bit)), rows, nref, pitch, shift, c.st);
    }
  }
  return 0;
}

static int pull_fields(Ctx & c, fluid_t * fl, unsigned mask) {
  for (unsigned bit = 1; bit <= TCGPU_T; bit <<= 1) {
    if (!(mask & bit)) continue;
    const array_t * a = host_field(fl, bit);
    const size_t n = field_count(c, bit);
    if (check_host_array(c, a, n, field_name(bit))) return 1;
    if (field_bytes(c, bit) == 8) {
      CK(cudaMemcpyAsync(a->data, dev_field(c, bit), n * sizeof(double), cudaMemcpyDeviceToHost, c.st));
    } else {
      size_t rows;
      int nref, pitch, shift;
      rows_of(c, bit, rows, nref, pitch, shift);
      launch_unpack32(static_cast<const float *>(dev_field(c, bit)), c.stage, rows, nref, pitch, shift, c.st);
      CK(cudaMemcpyAsync(a->data, c.stage, n * sizeof(double), cudaMemcpyDeviceToHost, c.st));
    }
  }
  return 0;
}

static int ensure_tensors(Ctx & c) {
  if (c.have_tn) return 0;
  const size_t nface = (size_t)(c.nx + 1) * (c.ny + 2) * (c.nz + 2);
  const size_t ncent = (size_t)c.nx * (c.ny + 2) * (c.nz + 2);
  const bool face[11] = {false, true, true, true, true, false, false, false, true, false, false};
  for (int s = 0; s < 11; s++) {
    c.tn.a[s] = dalloc(c, face[s] ? nface : ncent);
    if (!c.tn.a[s]) return fail("cudaMalloc of tensors failed");
  }
  c.have_tn = true;
  return 0;
}

// the fields the reference's tensors belong to: the last predict's input,
// or the current fields before any predict
static const FieldBufs & tensor_fields(Ctx & c) { return c.have_prev ? c.fb[c.cur ^ 1] : c.fb[c.cur]; }

// the eleven tensors of fields f, copied into the caller's arrays
static int pull_tensors(Ctx & c, fluid_t * fl, const FieldBufs & f) {
  if (ensure_tensors(c)) return 1;
  launch_tensors(c.g, c.cf, f, c.tn, c.st);
  const size_t nface = (size_t)(c.nx + 1) * (c.ny + 2) * (c.nz + 2);
  const size_t ncent = (size_t)c.nx * (c.ny + 2) * (c.nz + 2);
  array_t * dst[11] = {&fl->lxx, &fl->lxy, &fl->lxz, &fl->lyx0, &fl->lyx1, &fl->lyy0, &fl->lyy1, &fl->lyz,
                       &fl->lzx, &fl->lzy, &fl->lzz};
  const bool face[11] = {false, true, true, true, true, false, false, false, true, false, false};
  for (int s = 0; s < 11; s++) {
    if (dst[s]->data == nullptr) continue;
    CK(cudaMemcpyAsync(dst[s]->data, c.tn.a[s], (face[s] ? nface : ncent) * sizeof(double),
                       cudaMemcpyDeviceToHost, c.st));
  }
  return 0;
}

// reset_srcs (predict/main.c:8-25): the reference swaps the alpha and beta
// buffers of the caller's fluid_t; the same swap is mirrored there, and with
// TCGPU_SYNC_SRCS the device terms are copied into them.
static int mirror_srcs(Ctx & c, fluid_t * fl, int rk) {
  array_t * arrs[4] = {fl->srcux, fl->srcuy, fl->srcuz, fl->srct};
  for (int v = 0; v < 4; v++) {
    void * tmp = arrs[v][0].data;
    arrs[v][0].data = arrs[v][1].data;
    arrs[v][1].data = tmp;
  }
  if (!(c.coherence & TCGPU_SYNC_SRCS)) return 0;
  for (int v = 0; v < 4; v++) {
    const int ni = (v == VUX) ? c.nx - 1 : c.nx;
    const size_t n = (size_t)ni * c.ny * c.nz;
    auto copy = [&](void * host, const void * dev) -> int {
      if (c.sb == 8) {
        CK(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, c.st));
      } else {
        launch_unpack32(static_cast<const float *>(dev), c.stage, (size_t)c.ny * c.nz, ni, spitch32(c.nx), 0, c.st);
        CK(cudaMemcpyAsync(host, c.stage, n * sizeof(double), cudaMemcpyDeviceToHost, c.st));
      }
      return 0;
    };
    if (arrs[v][0].data && copy(arrs[v][0].data, s_new(c, v, rk))) return 1;
    if (arrs[v][1].data && rk != 0 && copy(arrs[v][1].data, s_old(c, v, rk))) return 1;
  }
  return 0;
}

static bool coherent(const Ctx & c) { return !(c.coherence & TCGPU_NO_COHERENCE); }

static int apply_bcs(Ctx & c, unsigned mask) {
  const BcKind kinds[6] = {BC_UX, BC_UY, BC_UZ, BC_P, BC_PSI, BC_T};
  for (int s = 0; s < 6; s++) {
    const unsigned bit = 1u << s;
    if (mask & bit) launch_bc(c.g, c.bc, kinds[s], dev_field(c, bit), field_bytes(c, bit), c.st);
  }
  return 0;
}

// ------------------------------------------------------------------ exported API
extern "C" {

const uint_fast8_t rk_a = 0;
const uint_fast8_t rk_b = 1;
const uint_fast8_t rk_g = 2;
const rkcoef_t rkcoefs[3] = {
    {32. / 60., 0. / 60., 32. / 60. + 0. / 60.},
    {25. / 60., -17. / 60., 25. / 60. + -17. / 60.},
    {45. / 60., -25. / 60., 45. / 60. + -25. / 60.},
};

const char * tcgpu_last_error(void) { return g_last_error.c_str(); }

int tcgpu_set_params(const tcgpu_params_t * params) {
  if (params == nullptr) return fail("params is NULL");
  std::lock_guard<std::mutex> lk(g_mutex);
  g_params = *params;
  return 0;
}

int tcgpu_get_params(tcgpu_params_t * params) {
  if (params == nullptr) return fail("params is NULL");
  *params = g_params;
  return 0;
}

int tcgpu_set_coherence(const domain_t * domain, fluid_t * fluid, unsigned flags) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  c->coherence = flags;
  if ((flags & TCGPU_PIN_HOST) && c->pinned.empty()) {
    for (unsigned bit = 1; bit <= TCGPU_T; bit <<= 1) {
      const array_t * a = host_field(fluid, bit);
      if (a->data == nullptr) continue;
      const size_t n = field_count(*c, bit) * sizeof(double);
      if (cudaHostRegister(a->data, n, cudaHostRegisterDefault) == cudaSuccess) c->pinned.push_back(a->data);
      else cudaGetLastError();
    }
  }
  return 0;
}

int tcgpu_push(const domain_t * domain, fluid_t * fluid, unsigned fields) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (push_fields(*c, fluid, fields & TCGPU_FIELDS)) return 1;
  apply_bcs(*c, fields & TCGPU_FIELDS);
  return finish(*c, "tcgpu_push");
}

int tcgpu_pull(const domain_t * domain, fluid_t * fluid, unsigned fields) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (pull_fields(*c, fluid, fields & TCGPU_FIELDS)) return 1;
  if ((fields & TCGPU_TENSORS) && pull_tensors(*c, fluid, tensor_fields(*c))) return 1;
  return finish(*c, "tcgpu_pull");
}

int tcgpu_run(const domain_t * domain, fluid_t * fluid, int nsteps, double * dts) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (nsteps > 64 && dts != nullptr) {
    for (int s0 = 0; s0 < nsteps; s0 += 64) {
      const int n = nsteps - s0 < 64 ? nsteps - s0 : 64;
      if (tcgpu_run(domain, fluid, n, dts + s0)) return 1;
    }
    return 0;
  }
  for (int s = 0; s < nsteps; s++) {
    if (launch_step(*c)) return 1;
    if (dts) CK(cudaMemcpyAsync(c->h_scalar + s, c->dtp, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  }
  if (finish(*c, "tcgpu_run")) return 1;
  if (dts) memcpy(dts, c->h_scalar, sizeof(double) * nsteps);
  return 0;
}

int tcgpu_run_timed(const domain_t * domain, fluid_t * fluid, int nsteps, int instrument, double * dts,
                    float * elapsed_ms, double * kernel_ms, int * kernel_launches) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (nsteps < 0 || nsteps > 64) return fail("tcgpu_run_timed: nsteps must be in [0, 64]");
  Recorder rec;
  rec.events = instrument != 0;
  rec.st = c->st;
  if (!instrument && c->step_graph[c->cur] == nullptr) {
    // capture both parities outside the timed region
    if (launch_step(*c) || launch_step(*c) || finish(*c, "tcgpu_run_timed")) return 1;
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaEventRecord(e0, c->st));
  if (instrument) rec.mark(TCGPU_K_DTMIN, 0);   // start marker, counts nothing
  int direct_dtmin = 0;                          // dtmin launches outside the step graphs
  for (int s = 0; s < nsteps; s++) {
    if (instrument) {
      g_rec = &rec;
      if (!c->dt_ready) enqueue_dtmin(*c);
      enqueue_step(*c);
      c->dt_ready = true;
      g_rec = nullptr;
    } else {
      if (!c->dt_ready) direct_dtmin++;
      if (launch_step(*c)) return 1;
    }
    if (dts) CK(cudaMemcpyAsync(c->h_scalar + s, c->dtp, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaEventRecord(e1, c->st));
  if (finish(*c, "tcgpu_run_timed")) return 1;
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (elapsed_ms) *elapsed_ms = ms;
  if (dts) memcpy(dts, c->h_scalar, sizeof(double) * nsteps);
  if (kernel_ms) {
    for (int k = 0; k < TCGPU_K_COUNT; k++) kernel_ms[k] = 0.;
    for (size_t i = 1; i < rec.used; i++) {
      float d = 0.f;
      cudaEventElapsedTime(&d, rec.ev[i - 1], rec.ev[i]);
      kernel_ms[rec.kind[i]] += d;
    }
  }
  if (kernel_launches) {
    for (int k = 0; k < TCGPU_K_COUNT; k++) kernel_launches[k] = instrument ? rec.launches[k] : c->graph_launches[k] * nsteps;
    if (!instrument) kernel_launches[TCGPU_K_DTMIN] += direct_dtmin;
  }
  return 0;
}

int tcgpu_set_storage(int bytes) {
  if (bytes != 8 && bytes != 4) return fail("tcgpu_set_storage: %d bytes per value; 8 or 4 expected", bytes);
  g_storage_bytes = bytes;
  return 0;
}

int tcgpu_get_storage(const fluid_t * fluid) {
  std::lock_guard<std::mutex> lk(g_mutex);
  auto it = g_ctx.find(fluid);
  return it == g_ctx.end() ? g_storage_bytes : it->second->sb;
}

int tcgpu_set_device(int device) {
  CK(cudaSetDevice(device));
  return 0;
}

static int diagnostics(Ctx & c, const FieldBufs & fs, double out[9], const char * what) {
  launch_diagnostics(c.g, c.cf, c.bc, c.f(), fs, c.nu, c.kappa, c.diag_out, c.diag_part, c.st);
  CK(cudaMemcpyAsync(c.h_scalar, c.diag_out, 9 * sizeof(double), cudaMemcpyDeviceToHost, c.st));
  if (finish(c, what)) return 1;
  memcpy(out, c.h_scalar, 9 * sizeof(double));
  return 0;
}

int tcgpu_diagnostics(const domain_t * domain, fluid_t * fluid, double out[9]) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  return diagnostics(*c, c->f(), out, "tcgpu_diagnostics");
}

int tcgpu_log_quantities(const domain_t * domain, fluid_t * fluid, double out[9]) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  return diagnostics(*c, tensor_fields(*c), out, "tcgpu_log_quantities");
}

// ------------------------------------------------------------------ statistics
static int ensure_stats(Ctx & c) {
  if (c.stats.a[0]) return 0;
  const size_t lines = (size_t)c.ny * c.nz;
  for (int s = 0; s < 8; s++) {
    const bool wide = s >= 2 && s <= 5;   // uy, uz: i = 0..nx+1
    c.stats.a[s] = dalloc(c, (wide ? c.nx + 2 : c.nx + 1) * lines);
    if (!c.stats.a[s]) return fail("cudaMalloc of the statistics failed");
  }
  c.stat_prof = dalloc(c, (size_t)c.nx + 2);
  if (!c.stat_prof) return fail("cudaMalloc of the statistics failed");
  return 0;
}

static size_t stat_count(const Ctx & c, int s) {
  return (size_t)((s >= 2 && s <= 5) ? c.nx + 2 : c.nx + 1) * c.ny * c.nz;
}

int tcgpu_statistics_collect(const domain_t * domain, fluid_t * fluid) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (ensure_stats(*c)) return 1;
  launch_statistics(c->g, c->cf, c->f(), tensor_fields(*c), c->stats, c->st);
  CK(cudaGetLastError());
  c->stat_num += 1;
  return 0;
}

int tcgpu_statistics_reset(const domain_t * domain, fluid_t * fluid) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (c->stats.a[0]) {
    for (int s = 0; s < 8; s++) CK(cudaMemsetAsync(c->stats.a[s], 0, stat_count(*c, s) * sizeof(double), c->st));
  }
  c->stat_num = 0;
  return finish(*c, "tcgpu_statistics_reset");
}

int tcgpu_statistics_get(const domain_t * domain, fluid_t * fluid, size_t * num, double * const out[8]) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (ensure_stats(*c)) return 1;
  if (num) *num = c->stat_num;
  if (out) {
    for (int s = 0; s < 8; s++) {
      if (out[s] == nullptr) continue;
      CK(cudaMemcpyAsync(out[s], c->stats.a[s], stat_count(*c, s) * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    }
  }
  return finish(*c, "tcgpu_statistics_get");
}

int tcgpu_io_fluid_alloc(const domain_t * domain, fluid_t * fluid);

int tcgpu_fluid_init_generated(const domain_t * domain, fluid_t * fluid, const tcgpu_ic_t * ic) {
  if (domain == nullptr || fluid == nullptr || ic == nullptr) return fail("tcgpu_fluid_init_generated: NULL argument");
  if (!(ic->noise_u >= 0.) || !(ic->noise_t >= 0.)) return fail("tcgpu_fluid_init_generated: negative noise");
  if (check_domain(domain)) return 1;
  if (tcgpu_io_fluid_alloc(domain, fluid)) return 1;
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  // radial profiles at the cell centres i = 0..nx+1 (the walls included, as
  // initial_condition/main.py lays out xc): circular Couette A r + B / r when
  // curved, linear when planar; the scalar linear between its wall values
  const int nx = c->nx;
  std::vector<double> prof(2 * ((size_t)nx + 2));
  const double ri = domain->xf[0], ro = domain->xf[nx], lx = ro - ri;
  const double ui = c->bc.uy_xm, uo = c->bc.uy_xp;
  const double A = (uo * ro - ui * ri) / (ro * ro - ri * ri), B = (ui - A * ri) * ri;
  for (int i = 0; i <= nx + 1; i++) {
    const double r = domain->xc[i];
    prof[i] = domain->is_curved ? A * r + B / r : ui + (uo - ui) * (r - ri) / lx;
    prof[nx + 2 + i] = c->bc.t_xm + (c->bc.t_xp - c->bc.t_xm) * (r - ri) / lx;
  }
  double * dprof = dalloc(*c, prof.size());
  if (!dprof) return fail("tcgpu_fluid_init_generated: cudaMalloc failed");
  CK(cudaMemcpyAsync(dprof, prof.data(), prof.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
  invalidate_dt(*c);
  launch_initial_field(c->g, c->f(), dprof, dprof + nx + 2, ic->seed, ic->noise_u, ic->noise_t, c->st);
  CK(cudaGetLastError());
  apply_bcs(*c, TCGPU_UX | TCGPU_UY | TCGPU_UZ | TCGPU_P | TCGPU_T);
  // the caller's arrays hold the same field, as after fluid_init
  if (pull_fields(*c, fluid, TCGPU_UX | TCGPU_UY | TCGPU_UZ | TCGPU_P | TCGPU_T)) return 1;
  const int rc = finish(*c, "tcgpu_fluid_init_generated");
  cudaFree(dprof);
  c->allocs.erase(std::remove(c->allocs.begin(), c->allocs.end(), static_cast<void *>(dprof)), c->allocs.end());
  return rc;
}

int tcgpu_radial_slab(const domain_t * domain, fluid_t * fluid, unsigned field, int i0, int count, double * out) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (out == nullptr) return fail("tcgpu_radial_slab: out is NULL");
  if (field != TCGPU_UX && field != TCGPU_UY && field != TCGPU_UZ && field != TCGPU_P && field != TCGPU_PSI &&
      field != TCGPU_T)
    return fail("tcgpu_radial_slab: field must be one of TCGPU_UX, _UY, _UZ, _P, _PSI, _T");
  const int lo = field == TCGPU_UX ? 1 : 0;
  if (count < 1 || i0 < lo || i0 + count - 1 > c->nx + 1)
    return fail("tcgpu_radial_slab: radial range %d..%d outside %d..%d", i0, i0 + count - 1, lo, c->nx + 1);
  const size_t n = (size_t)count * c->ny * c->nz;
  if (n > c->slab_n) {
    c->slab = dalloc(*c, n);
    if (!c->slab) return fail("tcgpu_radial_slab: cudaMalloc failed");
    c->slab_n = n;
  }
  launch_slab(c->g, dev_field(*c, field), field_bytes(*c, field), field == TCGPU_UX, i0, count, c->slab, c->st);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, c->slab, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  return finish(*c, "tcgpu_radial_slab");
}

int tcgpu_io_write_statistics(const char dirname[], const domain_t * domain, size_t num, const double * const a[8]);

int tcgpu_statistics_save(const char dirname[], const domain_t * domain, fluid_t * fluid) {
  if (dirname == nullptr) return fail("tcgpu_statistics_save: dirname is NULL");
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (c->stat_num == 0) return 0;   // statistics.c:256-258: nothing collected, nothing saved
  std::vector<std::vector<double>> host(8);
  const double * ptrs[8];
  for (int s = 0; s < 8; s++) {
    host[s].resize(stat_count(*c, s));
    CK(cudaMemcpyAsync(host[s].data(), c->stats.a[s], host[s].size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    ptrs[s] = host[s].data();
  }
  if (finish(*c, "tcgpu_statistics_save")) return 1;
  return tcgpu_io_write_statistics(dirname, domain, c->stat_num, ptrs);
}

int tcgpu_statistics_mean_uy(const domain_t * domain, fluid_t * fluid, double * profile) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (profile == nullptr) return fail("tcgpu_statistics_mean_uy: profile is NULL");
  if (c->stat_num == 0) return fail("tcgpu_statistics_mean_uy: no samples collected");
  const double inv = 1. / ((double)c->stat_num * (double)c->ny * (double)c->nz);
  launch_stat_profile(c->g, c->stats.a[2], inv, c->stat_prof, c->st);
  std::vector<double> host((size_t)c->nx + 2);
  CK(cudaMemcpyAsync(host.data(), c->stat_prof, host.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  if (finish(*c, "tcgpu_statistics_mean_uy")) return 1;
  memcpy(profile, host.data(), host.size() * sizeof(double));
  return 0;
}

int tcgpu_selftest_wait(double * seconds) {
  unsigned * d = nullptr;
  unsigned h = 0;
  cudaStream_t st = nullptr;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  if (cudaMalloc(&d, sizeof(unsigned)) != cudaSuccess) {
    cudaStreamDestroy(st);
    return fail("tcgpu_selftest_wait: cudaMalloc failed");
  }
  const auto t0 = std::chrono::steady_clock::now();
  cudaMemsetAsync(d, 0, sizeof(unsigned), st);
  launch_wait_selftest(d, st);
  cudaMemcpyAsync(&h, d, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  const auto t1 = std::chrono::steady_clock::now();
  cudaFree(d);
  cudaStreamDestroy(st);
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  if (e != cudaSuccess) return fail("tcgpu_selftest_wait: %s", cudaGetErrorString(e));
  if (!(h & ST_TIMEOUT)) return fail("tcgpu_selftest_wait: the wait did not report giving up");
  return 0;
}

void * tcgpu_stream(const domain_t * domain, fluid_t * fluid) {
  Ctx * c = get_ctx(domain, fluid);
  return c ? static_cast<void *>(c->st) : nullptr;
}

int tcgpu_coarsen(const domain_t * fine_domain, fluid_t * fine, const domain_t * coarse_domain, fluid_t * coarse) {
  Ctx * f = get_ctx(fine_domain, fine);
  Ctx * c = get_ctx(coarse_domain, coarse);
  if (!f || !c) return 1;
  if (f == c) return fail("tcgpu_coarsen: the fine and coarse fluids are the same");
  if (f->sb != 8 || c->sb != 8) return fail("tcgpu_coarsen: both contexts need 8-byte storage");
  if (f->nx != 4 * c->nx || f->ny != 4 * c->ny || f->nz != 4 * c->nz)
    return fail("tcgpu_coarsen: the coarse grid must be 4x coarser in every direction");
  // the coarse stream waits for the fine state
  cudaEvent_t ev;
  CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ev, f->st));
  CK(cudaStreamWaitEvent(c->st, ev, 0));
  launch_coarsen(f->g, f->f().as<double>(), c->g, c->f().as<double>(), c->st);
  apply_bcs(*c, TCGPU_UX | TCGPU_UY | TCGPU_UZ | TCGPU_P | TCGPU_T);
  invalidate_dt(*c);
  const int rc = finish(*c, "tcgpu_coarsen");
  cudaEventDestroy(ev);
  return rc;
}

int tcgpu_closure_input(const domain_t * domain, fluid_t * fluid, const double scale[3], int cp, void * out) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (c->sb != 8) return fail("tcgpu_closure_input: needs 8-byte storage");
  if (!scale || !out || cp < 16 || cp % 16 || (reinterpret_cast<uintptr_t>(out) & 15u))
    return fail("tcgpu_closure_input: bad arguments");
  const FieldsT<double> F = c->f().as<double>();
  launch_closure_input(c->g, F.ux, F.uy, F.uz, scale, cp, out, c->st);
  CK(cudaGetLastError());
  return 0;
}

int tcgpu_closure_target(const domain_t * domain, fluid_t * predicted, fluid_t * reference, double tau, float * out) {
  Ctx * a = get_ctx(domain, predicted);
  Ctx * b = get_ctx(domain, reference);
  if (!a || !b) return 1;
  if (a->sb != 8 || b->sb != 8) return fail("tcgpu_closure_target: needs 8-byte storage");
  if (a->nx != b->nx || a->ny != b->ny || a->nz != b->nz) return fail("tcgpu_closure_target: grids differ");
  if (!(tau > 0.) || !out) return fail("tcgpu_closure_target: bad arguments");
  cudaEvent_t ev;
  CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CK(cudaEventRecord(ev, b->st));
  CK(cudaStreamWaitEvent(a->st, ev, 0));
  launch_closure_target(a->g, a->f().as<double>(), b->f().as<double>(), tau, out, a->st);
  const int rc = finish(*a, "tcgpu_closure_target");
  cudaEventDestroy(ev);
  return rc;
}

int tcgpu_set_forcing(const domain_t * domain, fluid_t * fluid, const float * f, int nc, const double scale[3]) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  const bool on = f != nullptr;
  if (on) {
    if (c->sb != 8) return fail("tcgpu_set_forcing: needs 8-byte storage");
    if (nc < 3 || !scale) return fail("tcgpu_set_forcing: bad arguments");
    if (!c->frc[0]) {
      const size_t nin = (size_t)c->nx * c->ny * c->nz;
      c->frc[0] = dalloc(*c, (size_t)(c->nx - 1) * c->ny * c->nz);
      c->frc[1] = dalloc(*c, nin);
      c->frc[2] = dalloc(*c, nin);
      if (!c->frc[0] || !c->frc[1] || !c->frc[2]) return fail("tcgpu_set_forcing: cudaMalloc failed");
    }
    launch_closure_forcing(c->nx, c->ny, c->nz, f, nc, scale, c->frc[0], c->frc[1], c->frc[2], c->st);
    CK(cudaGetLastError());
  }
  if (on != c->forcing) {   // the captured steps hold the other predict variant
    for (int b = 0; b < 2; b++) {
      if (c->step_graph[b]) {
        cudaGraphExecDestroy(c->step_graph[b]);
        c->step_graph[b] = nullptr;
      }
    }
    c->forcing = on;
  }
  return 0;
}

int tcgpu_release(fluid_t * fluid) {
  std::lock_guard<std::mutex> lk(g_mutex);
  auto it = g_ctx.find(fluid);
  if (it == g_ctx.end()) return 0;
  destroy_ctx(it->second);
  g_ctx.erase(it);
  return 0;
}

double fluid_compute_momentum_diffusivity(const fluid_t * fluid) { return 1. / fluid->Re; }
double fluid_compute_scalar_diffusivity(const fluid_t * fluid) { return 1. / fluid->Re / fluid->Pr; }

int decide_dt(const domain_t * domain, const fluid_t * fluid, double * dt) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  invalidate_dt(*c);
  if (coherent(*c) && push_fields(*c, fluid, TCGPU_UX | TCGPU_UY | TCGPU_UZ)) return 1;
  launch_decide_dt(c->g, c->f(), c->coef_adv, c->dt_caps, c->dtmin, c->dtp, c->status, c->st);
  CK(cudaMemcpyAsync(c->h_scalar, c->dtp, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  if (finish(*c, "decide_dt")) return 1;
  *dt = *c->h_scalar;
  return 0;
}

int fluid_predict_field(const domain_t * domain, const size_t rkstep, const double dt, fluid_t * fluid) {
  if (rkstep > 2) return fail("rkstep %zu out of range", rkstep);
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  invalidate_dt(*c);
  const int rk = (int)rkstep;
  if (coherent(*c) && push_fields(*c, fluid, TCGPU_UX | TCGPU_UY | TCGPU_UZ | TCGPU_P | TCGPU_T)) return 1;
  if (set_dt(*c, dt)) return 1;
  if ((c->coherence & TCGPU_SYNC_TENSORS) && coherent(*c) && pull_tensors(*c, fluid, c->f())) return 1;
  enqueue_factors(*c);
  enqueue_predict(*c, rk);
  if (coherent(*c)) {
    if (pull_fields(*c, fluid, TCGPU_UX | TCGPU_UY | TCGPU_UZ | TCGPU_T)) return 1;
    if (mirror_srcs(*c, fluid, rk)) return 1;
  }
  return finish(*c, "fluid_predict_field");
}

int fluid_compute_potential(const domain_t * domain, const size_t rkstep, const double dt, fluid_t * fluid) {
  if (rkstep > 2) return fail("rkstep %zu out of range", rkstep);
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  invalidate_dt(*c);
  if (coherent(*c) && push_fields(*c, fluid, TCGPU_UX | TCGPU_UY | TCGPU_UZ)) return 1;
  if (set_dt(*c, dt)) return 1;
  enqueue_potential(*c, (int)rkstep);
  if (coherent(*c) && pull_fields(*c, fluid, TCGPU_PSI)) return 1;
  return finish(*c, "fluid_compute_potential");
}

int fluid_correct_velocity(const domain_t * domain, const size_t rkstep, const double dt, fluid_t * fluid) {
  if (rkstep > 2) return fail("rkstep %zu out of range", rkstep);
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  invalidate_dt(*c);
  if (coherent(*c) && push_fields(*c, fluid, TCGPU_UX | TCGPU_UY | TCGPU_UZ | TCGPU_PSI)) return 1;
  if (set_dt(*c, dt)) return 1;
  enqueue_correct(*c, (int)rkstep, CORRECT_VELOCITY);
  if (coherent(*c) && pull_fields(*c, fluid, TCGPU_UX | TCGPU_UY | TCGPU_UZ)) return 1;
  return finish(*c, "fluid_correct_velocity");
}

int fluid_update_pressure(const domain_t * domain, const size_t rkstep, const double dt, fluid_t * fluid) {
  if (rkstep > 2) return fail("rkstep %zu out of range", rkstep);
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  invalidate_dt(*c);
  // inside integrate() this update runs fused with the velocity correction
  if (coherent(*c) && push_fields(*c, fluid, TCGPU_P | TCGPU_PSI)) return 1;
  if (set_dt(*c, dt)) return 1;
  enqueue_correct(*c, (int)rkstep, CORRECT_PRESSURE);
  if (coherent(*c) && pull_fields(*c, fluid, TCGPU_P)) return 1;
  return finish(*c, "fluid_update_pressure");
}

int integrate(const domain_t * domain, fluid_t * fluid, double * dt) {
  Ctx * c = get_ctx(domain, fluid);
  if (!c) return 1;
  if (coherent(*c) && push_fields(*c, fluid, TCGPU_UX | TCGPU_UY | TCGPU_UZ | TCGPU_P | TCGPU_T)) return 1;
  if (launch_step(*c)) return 1;
  CK(cudaMemcpyAsync(c->h_scalar, c->dtp, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  // a rejected step (non-finite field, invalid dt) leaves the caller's arrays untouched
  if (finish(*c, "integrate")) return 1;
  if (coherent(*c)) {
    if (pull_fields(*c, fluid, TCGPU_FIELDS)) return 1;
    // the tensors the reference leaves behind: those of the substep-3 input
    if ((c->coherence & TCGPU_SYNC_TENSORS) && pull_tensors(*c, fluid, tensor_fields(*c))) return 1;
    // three predict calls swap the caller's alpha/beta source buffers three times
    array_t * arrs[4] = {fluid->srcux, fluid->srcuy, fluid->srcuz, fluid->srct};
    for (int v = 0; v < 4; v++) {
      void * tmp = arrs[v][0].data;
      arrs[v][0].data = arrs[v][1].data;
      arrs[v][1].data = tmp;
    }
  }
  if (finish(*c, "integrate")) return 1;
  *dt = *c->h_scalar;
  return 0;
}

// fluid_update_boundaries_* on a single host array: it travels through a
// scratch device buffer; no solver context is needed or touched.
static int bc_entry(const domain_t * domain, array_t * array, BcKind kind, const char * name) {
  if (check_domain(domain)) return 1;
  if (array == nullptr || array->data == nullptr) return fail("%s: array is NULL", name);
  Geo g{};
  g.nx = (int)domain->glsizes[0];
  g.ny = (int)domain->glsizes[1];
  g.nz = (int)domain->glsizes[2];
  Bc bc{};
  bc.uy_xm = g_params.uy_xm;
  bc.uy_xp = g_params.uy_xp;
  bc.t_xm = g_params.t_xm;
  bc.t_xp = g_params.t_xp;
  const size_t n = (kind == BC_UX) ? ncell_f(g) : ncell_c(g);
  if (array->datasize != 0 && array->datasize != n * sizeof(double))
    return fail("%s: array holds %zu bytes, %zu expected", name, array->datasize, n * sizeof(double));
  double * dbuf = nullptr;
  CK(cudaMalloc(&dbuf, n * sizeof(double)));
  cudaError_t e = cudaMemcpy(dbuf, array->data, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    launch_bc(g, bc, kind, dbuf, 8, 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(array->data, dbuf, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dbuf);
  if (e != cudaSuccess) return fail("%s: %s", name, cudaGetErrorString(e));
  return 0;
}

int fluid_update_boundaries_ux(const domain_t * d, array_t * a) { return bc_entry(d, a, BC_UX, "fluid_update_boundaries_ux"); }
int fluid_update_boundaries_uy(const domain_t * d, array_t * a) { return bc_entry(d, a, BC_UY, "fluid_update_boundaries_uy"); }
int fluid_update_boundaries_uz(const domain_t * d, array_t * a) { return bc_entry(d, a, BC_UZ, "fluid_update_boundaries_uz"); }
int fluid_update_boundaries_p(const domain_t * d, array_t * a) { return bc_entry(d, a, BC_P, "fluid_update_boundaries_p"); }
int fluid_update_boundaries_psi(const domain_t * d, array_t * a) { return bc_entry(d, a, BC_PSI, "fluid_update_boundaries_psi"); }
int fluid_update_boundaries_t(const domain_t * d, array_t * a) { return bc_entry(d, a, BC_T, "fluid_update_boundaries_t"); }

}  // extern "C"

extern "C" int tcgpu_report_error(const char * msg) { return fail("%s", msg); }
