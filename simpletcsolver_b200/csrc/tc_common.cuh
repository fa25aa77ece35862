// Shared definitions of the tcgpu kernels.
//
// HBM layout of the fields is the reference's own (array_macros/fluid/*.h):
// x fastest, one halo layer in y and z, and in x either the two walls/ghosts
// (uy, uz, p, psi, t: i = 0..nx+1, row length nx+2) or the faces only
// (ux: i = 1..nx+1, row length nx+1). Keeping the reference layout makes the
// host<->device copies of the drop-in entry points single memcpys. Every kernel
// that writes a cell also writes its periodic images in the y/z halo and the
// wall value of its row, which is what halo.c and boundary/*.c do on the CPU.
//
// RK source terms and increments use the reference's packed interior layout
// (srcux: i = 2..nx, others i = 1..nx; src/fluid/predict/*.c BEGIN loops).
#pragma once

#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

namespace tcgpu {

// Wray RK3, src/runge_kutta.c:8-15
__host__ __device__ constexpr double rk_alpha(int s) { return s == 0 ? 32. / 60. : s == 1 ? 25. / 60. : 45. / 60.; }
__host__ __device__ constexpr double rk_beta(int s)  { return s == 0 ? 0. / 60. : s == 1 ? -17. / 60. : -25. / 60.; }
__host__ __device__ constexpr double rk_gamma(int s) { return rk_alpha(s) + rk_beta(s); }

enum Var { VUX = 0, VUY = 1, VUZ = 2, VT = 3 };

// sizes and metric tables, passed to every kernel by value
struct Geo {
  int nx, ny, nz;
  double hz;
  // length nx+2, indexed by the reference's i (unused entries are zero)
  const double * hxxf;
  const double * hxxc;
  const double * hyxf;
  const double * hyxc;
  const double * jdxf;
  const double * jdxc;
};

// runtime replacement of src/param/*.c
struct Bc {
  double uy_xm, uy_xp, t_xm, t_xp;
  int implicit[3];
};

__host__ __device__ inline size_t cidx(const Geo & g, int i, int j, int k) {
  return (size_t)i + (size_t)(g.nx + 2) * ((size_t)j + (size_t)(g.ny + 2) * (size_t)k);
}
__host__ __device__ inline size_t fidx(const Geo & g, int i, int j, int k) {
  return (size_t)(i - 1) + (size_t)(g.nx + 1) * ((size_t)j + (size_t)(g.ny + 2) * (size_t)k);
}
__host__ __device__ inline size_t ncell_c(const Geo & g) { return (size_t)(g.nx + 2) * (g.ny + 2) * (g.nz + 2); }
__host__ __device__ inline size_t ncell_f(const Geo & g) { return (size_t)(g.nx + 1) * (g.ny + 2) * (g.nz + 2); }
// packed interior index; i0 = 2 for ux, 1 otherwise
__host__ __device__ inline size_t pidx(int n_i, int ny, int ii, int j, int k) {
  return (size_t)ii + (size_t)n_i * ((size_t)(j - 1) + (size_t)ny * (size_t)(k - 1));
}

// Layout of the state arrays (ux, uy, uz, t) and RK source terms by storage
// type. double: the reference's layout above (host copies are single
// memcpys). float (FP32-storage mode, device only, converted on every host
// copy): rows of P = nx + 2 rounded up to a multiple of 4 values so that every
// row starts on a 16-byte boundary; ux keeps face i at element i (element 0
// unused), so all four fields share one index; source-term lines are padded
// to PS = nx rounded up to a multiple of 4.
__host__ __device__ constexpr int pitch32(int nx) { return (nx + 2 + 3) & ~3; }
__host__ __device__ constexpr int spitch32(int nx) { return (nx + 3) & ~3; }
template <class T>
__host__ __device__ inline size_t sidx_c(const Geo & g, int i, int j, int k) {
  if (sizeof(T) == 8) return cidx(g, i, j, k);
  return (size_t)i + (size_t)pitch32(g.nx) * ((size_t)j + (size_t)(g.ny + 2) * (size_t)k);
}
template <class T>
__host__ __device__ inline size_t sidx_f(const Geo & g, int i, int j, int k) {
  if (sizeof(T) == 8) return fidx(g, i, j, k);
  return (size_t)i + (size_t)pitch32(g.nx) * ((size_t)j + (size_t)(g.ny + 2) * (size_t)k);
}
// row strides (elements) of the state arrays
template <class T> __host__ __device__ inline int srow_c(const Geo & g) { return sizeof(T) == 8 ? g.nx + 2 : pitch32(g.nx); }
template <class T> __host__ __device__ inline int srow_f(const Geo & g) { return sizeof(T) == 8 ? g.nx + 1 : pitch32(g.nx); }
// element count of a state array
template <class T> __host__ __device__ inline size_t scount_c(const Geo & g) {
  return (size_t)srow_c<T>(g) * (g.ny + 2) * (g.nz + 2);
}
template <class T> __host__ __device__ inline size_t scount_f(const Geo & g) {
  return (size_t)srow_f<T>(g) * (g.ny + 2) * (g.nz + 2);
}
// packed source-term index (ii from 0; n_i = nx - 1 for ux, nx otherwise)
template <class T>
__host__ __device__ inline size_t sidx_s(const Geo & g, int n_i, int ii, int j, int k) {
  return pidx(sizeof(T) == 8 ? n_i : spitch32(g.nx), g.ny, ii, j, k);
}
template <class T> __host__ __device__ inline int sline(const Geo & g, int n_i) {
  return sizeof(T) == 8 ? n_i : spitch32(g.nx);
}

// periodic images of interior (j, k) in the one-layer halo, including the
// corner written by the z exchange after the y exchange (src/halo.c:18-142);
// ny, nz >= 2 (the FFTs require powers of two >= 4)
template <typename F>
__device__ inline void for_images(int j, int k, int ny, int nz, F && f) {
  const int jj = (j == 1) ? ny + 1 : (j == ny) ? 0 : -1;
  const int kk = (k == 1) ? nz + 1 : (k == nz) ? 0 : -1;
  if (jj >= 0) f(jj, k);
  if (kk >= 0) f(j, kk);
  if (jj >= 0 && kk >= 0) f(jj, kk);
}

// device-side status word: set by kernels, read by the host after a step
enum : unsigned { ST_NONFINITE = 1u, ST_BADDT = 2u, ST_TIMEOUT = 4u };

// ---- mbarriers and bulk asynchronous copies (sm_90+) ----------------------
// wait limit on an mbarrier phase, in SM clock cycles (about two seconds)
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
// global -> shared bulk copy (16-byte aligned addresses, size a multiple of
// 16), completion counted in bytes on bar
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

}  // namespace tcgpu
