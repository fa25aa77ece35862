// The reference's batched tri-diagonal solver object (include/tdm.h,
// src/tdm.c) with solve() on the GPU.
//
// The caller fills l, c, u (host arrays owned by the object) and hands solve()
// nrhs right-hand sides of length `size`, contiguous, real or complex
// (interleaved re/im), in host or device memory. The elimination factors depend
// only on l, c, u, so they are formed once per solve on the host in the
// reference's operation order (src/tdm.c:24-44, 78-87); the device then runs one
// thread per right-hand side with the same operations, rounded one by one (no
// fused multiply-add), which makes the results bit-identical to the reference's.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "tcgpu.h"

extern "C" int tcgpu_report_error(const char * msg);

struct tdm_info_t_ {
  int size;
  int nrhs;
  bool is_periodic;
  bool is_complex;
  double * l;
  double * c;
  double * u;
  double * dcoef;     // device: [l | v | w | q1], length 4 * size
  double * dbuf;      // device staging for host right-hand sides
  size_t dbuf_bytes;
};

namespace {

constexpr double kEps = 2.220446049250313e-16;  // DBL_EPSILON

struct Plan {
  int m;          // size of the non-periodic system that is eliminated
  double c0;      // first pivot (q0 = q0 / c0)
  int singular;   // last pivot |val| <= eps (gtsv sets the last unknown to 0)
  // periodic correction (src/tdm.c:84-96)
  double u_last, l_last, den;
  int den_zero;
};

// one right-hand side component (stride 1 or 2 doubles), reference arithmetic
__device__ void gtsv_dev(int m, const double * l, const double * v, const double * w, double c0, int singular,
                         double * q, int s) {
  q[0] = __ddiv_rn(q[0], c0);
  for (int i = 1; i < m - 1; i++)
    q[i * s] = __dmul_rn(w[i], __dsub_rn(q[i * s], __dmul_rn(l[i], q[(i - 1) * s])));
  if (m > 1) {
    const int i = m - 1;
    q[i * s] = singular ? 0. : __dmul_rn(w[i], __dsub_rn(q[i * s], __dmul_rn(l[i], q[(i - 1) * s])));
  }
  for (int i = m - 2; i >= 0; i--) q[i * s] = __dsub_rn(q[i * s], __dmul_rn(v[i], q[(i + 1) * s]));
}

__global__ void tdm_kernel(int n, int nrhs, int comps, int periodic, const double * __restrict__ coef, Plan pl,
                           double * __restrict__ data) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrhs * comps) return;
  const int line = r / comps, comp = r % comps;
  double * q = data + (size_t)line * n * comps + comp;
  const double * l = coef;
  const double * v = coef + n;
  const double * w = coef + 2 * n;
  const double * q1 = coef + 3 * n;
  const int s = comps;
  gtsv_dev(pl.m, l, v, w, pl.c0, pl.singular, q, s);
  if (periodic) {
    const double num = __dsub_rn(__dsub_rn(q[(n - 1) * s], __dmul_rn(pl.u_last, q[0])),
                                 __dmul_rn(pl.l_last, q[(n - 2) * s]));
    const double last = pl.den_zero ? 0. : __ddiv_rn(num, pl.den);
    q[(n - 1) * s] = last;
    for (int i = 0; i < n - 1; i++) q[i * s] = __dadd_rn(q[i * s], __dmul_rn(last, q1[i]));
  }
}

// host elimination factors of gtsv for size m (src/tdm.c:24-44)
void factors(int m, const double * l, const double * c, const double * u, double * v, double * w, Plan & pl) {
  pl.c0 = c[0];
  v[0] = u[0] / c[0];
  for (int i = 1; i < m - 1; i++) {
    const double val = 1. / (c[i] - l[i] * v[i - 1]);
    w[i] = val;
    v[i] = val * (u[i]);
  }
  pl.singular = 0;
  if (m > 1) {
    const double val = c[m - 1] - l[m - 1] * v[m - 2];
    if (fabs(val) > kEps) w[m - 1] = 1. / val;
    else pl.singular = 1;
  }
}

void host_gtsv(int m, const double * l, const double * c, const double * u, const double * v, const double * w,
               const Plan & pl, double * q) {
  (void)u;
  q[0] = q[0] / c[0];
  for (int i = 1; i < m - 1; i++) q[i] = w[i] * (q[i] - l[i] * q[i - 1]);
  if (m > 1) q[m - 1] = pl.singular ? 0. : w[m - 1] * (q[m - 1] - l[m - 1] * q[m - 2]);
  for (int i = m - 2; i >= 0; i--) q[i] -= v[i] * q[i + 1];
}

int construct(const int size, const int nrhs, const bool is_periodic, const bool is_complex, tdm_info_t ** info) {
  if (size <= 0) {
    printf("ERROR(%s): size should be positive: %d\n", __func__, size);
    *info = nullptr;
    return 1;
  }
  if (nrhs <= 0) {
    printf("ERROR(%s): nrhs should be positive: %d\n", __func__, nrhs);
    *info = nullptr;
    return 1;
  }
  tdm_info_t * t = static_cast<tdm_info_t *>(calloc(1, sizeof(tdm_info_t)));
  t->size = size;
  t->nrhs = nrhs;
  t->is_periodic = is_periodic;
  t->is_complex = is_complex;
  t->l = static_cast<double *>(calloc(size, sizeof(double)));
  t->c = static_cast<double *>(calloc(size, sizeof(double)));
  t->u = static_cast<double *>(calloc(size, sizeof(double)));
  if (cudaMalloc(&t->dcoef, 4 * (size_t)size * sizeof(double)) != cudaSuccess) {
    tcgpu_report_error("tdm.construct: cudaMalloc failed");
    *info = nullptr;
    return 1;
  }
  *info = t;
  return 0;
}

int get_l(const tdm_info_t * info, double ** l) {
  if (info == nullptr) { printf("ERROR(%s): info is NULL\n", __func__); return 1; }
  *l = info->l;
  return 0;
}
int get_c(const tdm_info_t * info, double ** c) {
  if (info == nullptr) { printf("ERROR(%s): info is NULL\n", __func__); return 1; }
  *c = info->c;
  return 0;
}
int get_u(const tdm_info_t * info, double ** u) {
  if (info == nullptr) { printf("ERROR(%s): info is NULL\n", __func__); return 1; }
  *u = info->u;
  return 0;
}
int get_size(const tdm_info_t * info, int * size) {
  if (info == nullptr) { printf("ERROR(%s): info is NULL\n", __func__); return 1; }
  *size = info->size;
  return 0;
}
int get_nrhs(const tdm_info_t * info, int * nrhs) {
  if (info == nullptr) { printf("ERROR(%s): info is NULL\n", __func__); return 1; }
  *nrhs = info->nrhs;
  return 0;
}

int solve(const tdm_info_t * info_c, void * data) {
  if (info_c == nullptr) { printf("ERROR(%s): info is NULL\n", __func__); return 1; }
  tdm_info_t * info = const_cast<tdm_info_t *>(info_c);
  const int n = info->size;
  const int comps = info->is_complex ? 2 : 1;
  const size_t bytes = (size_t)n * info->nrhs * comps * sizeof(double);
  // elimination factors on the host
  const int m = info->is_periodic ? n - 1 : n;
  std::vector<double> coef(4 * (size_t)n, 0.);
  double * l = coef.data();
  double * v = l + n;
  double * w = l + 2 * n;
  double * q1 = l + 3 * n;
  memcpy(l, info->l, n * sizeof(double));
  Plan pl{};
  pl.m = m;
  factors(m, info->l, info->c, info->u, v, w, pl);
  if (info->is_periodic) {
    // src/tdm.c:78-86: the additional system coming from periodicity
    for (int i = 0; i < n - 1; i++) q1[i] = i == 0 ? -info->l[i] : i == n - 2 ? -info->u[i] : 0.;
    host_gtsv(m, info->l, info->c, info->u, v, w, pl, q1);
    pl.u_last = info->u[n - 1];
    pl.l_last = info->l[n - 1];
    pl.den = info->c[n - 1] + info->u[n - 1] * q1[0] + info->l[n - 1] * q1[n - 2];
    pl.den_zero = fabs(pl.den) < kEps;
  }
  cudaPointerAttributes attr{};
  const bool on_device = cudaPointerGetAttributes(&attr, data) == cudaSuccess &&
                         (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
  cudaGetLastError();
  double * d = static_cast<double *>(data);
  if (cudaMemcpy(info->dcoef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return tcgpu_report_error("tdm.solve: cudaMemcpy failed");
  if (!on_device) {
    if (info->dbuf_bytes < bytes) {
      cudaFree(info->dbuf);
      info->dbuf = nullptr;
      if (cudaMalloc(&info->dbuf, bytes) != cudaSuccess) return tcgpu_report_error("tdm.solve: cudaMalloc failed");
      info->dbuf_bytes = bytes;
    }
    if (cudaMemcpy(info->dbuf, data, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      return tcgpu_report_error("tdm.solve: cudaMemcpy failed");
    d = info->dbuf;
  }
  const int threads = info->nrhs * comps;
  tdm_kernel<<<(threads + 127) / 128, 128>>>(n, info->nrhs, comps, info->is_periodic ? 1 : 0, info->dcoef, pl, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && !on_device) e = cudaMemcpy(data, info->dbuf, bytes, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    char msg[256];
    snprintf(msg, sizeof(msg), "tdm.solve: %s", cudaGetErrorString(e));
    return tcgpu_report_error(msg);
  }
  return 0;
}

int destruct(tdm_info_t * info) {
  if (info == nullptr) { printf("ERROR(%s): info is NULL\n", __func__); return 1; }
  free(info->l);
  free(info->c);
  free(info->u);
  cudaFree(info->dcoef);
  cudaFree(info->dbuf);
  free(info);
  return 0;
}

}  // namespace

extern "C" const tdm_t tdm = {
    construct, get_l, get_c, get_u, get_size, get_nrhs, solve, destruct,
};

// ---------------------------------------------------------------- allocation-free solve
// For callers that must not allocate device memory themselves or have the
// library do it: a framework that owns the whole device memory pool, a
// real-time host that reserves all device memory up front and may not allocate
// afterwards, or a plugin whose allocator belongs to someone else. The
// elimination-factor table that tdm.solve() keeps in cudaMalloc'd memory lives
// here in a fixed static device array instead; the caller supplies the
// coefficients (host) and the right-hand sides (device memory of the current
// device, solved in place). The work is ordered on the legacy default stream
// and finished before the call returns.
namespace {

constexpr int kNoAllocMax = TCGPU_TDM_NOALLOC_MAX_SIZE;
// [l | v | w | q1], kNoAllocMax each; every loaded GPU holds it until exit
static __device__ __align__(256) double g_noalloc_factors[4 * kNoAllocMax];
static double g_noalloc_host[4 * kNoAllocMax];     // staging of the factors
static double * g_noalloc_dev[128];                // device address per device ordinal
static std::mutex g_noalloc_mutex;

}  // namespace

extern "C" int tcgpu_tdm_solve_noalloc(int size, int nrhs, bool is_periodic, bool is_complex, const double * l,
                                       const double * c, const double * u, double * data) {
  if (size < 1 || size > kNoAllocMax || (is_periodic && size < 3))
    return tcgpu_report_error(is_periodic && size < 3 && size >= 1
                                  ? "tcgpu_tdm_solve_noalloc: periodic systems need size >= 3"
                                  : "tcgpu_tdm_solve_noalloc: size outside [1, TCGPU_TDM_NOALLOC_MAX_SIZE]");
  if (nrhs < 1) return tcgpu_report_error("tcgpu_tdm_solve_noalloc: nrhs must be positive");
  if (l == nullptr || c == nullptr || u == nullptr || data == nullptr)
    return tcgpu_report_error("tcgpu_tdm_solve_noalloc: NULL argument");
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, data) != cudaSuccess ||
      (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)) {
    cudaGetLastError();
    return tcgpu_report_error("tcgpu_tdm_solve_noalloc: data must be device memory");
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mutex);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
    return tcgpu_report_error("tcgpu_tdm_solve_noalloc: no current device");
  if (attr.type == cudaMemoryTypeDevice && attr.device != dev)
    return tcgpu_report_error("tcgpu_tdm_solve_noalloc: data is device memory of another device than the current one");
  if (g_noalloc_dev[dev] == nullptr) {
    // set-up once per device, with that device current: the symbol's device
    // address (the name itself is only a host-side stand-in)
    double * p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noalloc_factors);
    if (e != cudaSuccess) {
      char msg[256];
      snprintf(msg, sizeof(msg), "tcgpu_tdm_solve_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return tcgpu_report_error(msg);
    }
    g_noalloc_dev[dev] = p;
  }
  const int n = size;
  const int m = is_periodic ? n - 1 : n;
  double * hl = g_noalloc_host;
  double * hv = hl + n;
  double * hw = hl + 2 * n;
  double * hq1 = hl + 3 * n;
  // every entry the kernel reads is rewritten here; nothing from an earlier call survives
  for (int i = 0; i < 4 * n; i++) hl[i] = 0.;
  memcpy(hl, l, n * sizeof(double));
  Plan pl{};
  pl.m = m;
  factors(m, l, c, u, hv, hw, pl);
  if (is_periodic) {
    for (int i = 0; i < n - 1; i++) hq1[i] = i == 0 ? -l[i] : i == n - 2 ? -u[i] : 0.;
    host_gtsv(m, l, c, u, hv, hw, pl, hq1);
    pl.u_last = u[n - 1];
    pl.l_last = l[n - 1];
    pl.den = c[n - 1] + u[n - 1] * hq1[0] + l[n - 1] * hq1[n - 2];
    pl.den_zero = fabs(pl.den) < kEps;
  }
  double * dcoef = g_noalloc_dev[dev];
  cudaError_t e = cudaMemcpy(dcoef, hl, 4 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const int comps = is_complex ? 2 : 1;
    const int threads = nrhs * comps;
    tdm_kernel<<<(threads + 127) / 128, 128>>>(n, nrhs, comps, is_periodic ? 1 : 0, dcoef, pl, data);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) {
    char msg[256];
    snprintf(msg, sizeof(msg), "tcgpu_tdm_solve_noalloc: %s", cudaGetErrorString(e));
    return tcgpu_report_error(msg);
  }
  return 0;
}
