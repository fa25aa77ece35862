// Learned closure of the coarse solver: 3x3x3 convolutions on the 5th-generation
// tensor cores (tcgen05.mma, BF16 operands from shared memory, FP32 accumulators
// in tensor memory), their backward passes, Adam, and the grid-side kernels
// (4x box filter of fine fields, network input assembly, forcing hand-off).
// No counterpart in the reference.
//
// Activations are channels-last BF16, act[((k ny + j) nx + i) C + c] over the
// interior cells of the coarse grid; x (radial) is zero-padded at the walls,
// y and z are periodic.
//
// One convolution = an implicit GEMM per output tile of 8 (x) x 16 (y) cells of
// one z plane: M = 128 cells, N = the output channels, K = 27 taps x the input
// channels. A CTA keeps the tile's (x, y) block and marches through a chunk of
// z planes. The halo of three planes (10 x 18 cells each) sits in shared memory
// in the tensor cores' no-swizzle layout, 16-byte units ordered
// [y][channel chunk][x] (a unit = 8 channels of one cell), so every tap's A
// operand is the same halo seen from a shifted start address:
//   K-major A (forward, input gradient): 8-row core matrices = 8 consecutive x
//     of one y row; row groups (y) at stride ROWB, channel chunks at CHB;
//   MN-major A (weight gradient): a unit is 8 channels (M) of one cell (K);
//     channel chunks at CHB continue into the next y row, so one M = 128
//     operand spans 128 / C consecutive y shifts of the tap.
#include <cuda_bf16.h>
#include <stdint.h>
#include <stdio.h>

#include "tc_common.cuh"
#include "tc_kernels.h"

namespace tcgpu {
namespace {

// wait limit on an mbarrier phase, in SM clock cycles (about two seconds)
constexpr long long kNnWaitCycles = 4000000000LL;

__device__ __forceinline__ unsigned su32(const void * p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void nn_mbar_init(unsigned long long * bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool nn_mbar_try(unsigned long long * bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false if the phase did not complete within kNnWaitCycles
__device__ __forceinline__ bool nn_mbar_wait(unsigned long long * bar, unsigned parity) {
  if (nn_mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!nn_mbar_try(bar, parity)) {
    if (clock64() - t0 > kNnWaitCycles) return false;
  }
  return true;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16-byte asynchronous copy global -> shared; zero-filled when !valid (the
// source address is then not read)
__device__ __forceinline__ void cp16(void * dst, const void * src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(su32(dst)), "l"(src), "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---- tensor memory ------------------------------------------------------
// allocation by one full warp; the address lands in *slot
__device__ __forceinline__ void tmem_alloc(unsigned * slot, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- tcgen05.mma --------------------------------------------------------
// Shared-memory matrix descriptor, no swizzle: start address, leading and
// stride byte offsets (16-byte units), descriptor version 1 (bits 46-47).
__device__ __forceinline__ uint64_t smem_desc(unsigned saddr, unsigned lbo, unsigned sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;   // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// K-major (0) or MN-major (1) operands, N and M.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4)                       // D format F32
         | (1u << 7)                     // A format BF16
         | (1u << 10)                    // B format BF16
         | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16)
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(M >> 4) << 24);   // M / 16
}
// D (tensor memory) [+]= A (smem) x B (smem), issued by one thread
__device__ __forceinline__ void mma_bf16(unsigned dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1u : 0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
// arrive on the mbarrier once all previously issued MMAs of this thread completed
__device__ __forceinline__ void mma_commit(unsigned long long * bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}
// 32 lanes x 16 / 32 consecutive 32-bit columns, one lane per thread of the warp
__device__ __forceinline__ void tmem_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

// GELU in its tanh form (Hendrycks and Gimpel 2016),
//   gelu(z) = 0.5 z (1 + tanh(u)), u = sqrt(2/pi) (z + 0.044715 z^3),
// with the hardware tanh approximation (tanh.approx.f32, about 2^-11
// relative), and its derivative
//   0.5 (1 + t) + 0.5 z (1 - t^2) sqrt(2/pi) (1 + 3 0.044715 z^2), t = tanh(u).
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
constexpr float kGeluS = 0.79788456080286536f, kGeluC = 0.044715f;
__device__ __forceinline__ float gelu(float z) {
  const float t = tanh_hw(kGeluS * z * fmaf(kGeluC * z, z, 1.f));
  const float h = 0.5f * z;
  return fmaf(h, t, h);
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float z2 = z * z;
  const float t = tanh_hw(kGeluS * z * fmaf(kGeluC, z2, 1.f));
  return fmaf(0.5f, 1.f + t, 0.5f * z * (1.f - t * t) * kGeluS * fmaf(3.f * kGeluC, z2, 1.f));
}

// ---- convolution: forward and input gradient ------------------------------
constexpr int TX = 8, TY = 16;             // output tile: 8 x, 16 y, one z plane (M = 128)
constexpr int HX = TX + 2, HY = TY + 2;    // halo of one plane
constexpr int NN_THREADS = 128;            // weight gradient: 4 warps, one TMEM lane quarter each
// epilogue warps: groups of four (one per TMEM lane quarter), each group
// draining every NGRP-th output plane; halo loader warps
#ifndef TC_CONV_EPI_GROUPS
#define TC_CONV_EPI_GROUPS 2
#endif
#ifndef TC_CONV_LOADERS
#define TC_CONV_LOADERS 2
#endif
constexpr int NGRP = TC_CONV_EPI_GROUPS;
constexpr int NEPI = 4 * NGRP;
constexpr int NLD = TC_CONV_LOADERS;
constexpr int CONV_THREADS = 32 * (NEPI + 1 + NLD);   // + the MMA warp and the loaders

enum ConvEpilogue { EPI_GELU = 0, EPI_LINEAR = 1, EPI_DGELU = 2 };

// The three z taps are stacked along N: one MMA multiplies the halo of input
// plane p, shifted by (dy, dx), with the weights of taps dz = -1, 0, +1 side
// by side (N = 3 COUT) and adds into the accumulators of output planes p + 1,
// p and p - 1, which sit side by side in tensor memory. Output plane number g
// of the CTA (counted over all its segments) owns the accumulator at column
// block c(g) = S - 1 - g mod S of a ring of S blocks of COUT columns; the
// window of step p starts at c(g(p + 1)) and runs on into two overflow blocks
// S and S + 1 past the ring instead of wrapping, so every step is one MMA per
// shift. A plane whose block is 0 or 1 therefore also collects in block S or
// S + 1, which the epilogue adds. Accumulators start at zero and are zeroed
// again by the epilogue that drains them, so every MMA accumulates.
template <int CIN, int COUT>
struct ConvLayout {
  static_assert(CIN == 16 || CIN == 32, "input channels: 16 or 32");
  static_assert(COUT == 16 || COUT == 32, "output channels: 16 or 32");
  static constexpr int CC = CIN / 8;                     // 16-byte channel chunks per cell
  static constexpr int CHB = HX * 16;                    // bytes between channel chunks of a halo row
  static constexpr int ROWB = CC * CHB;                  // bytes between halo rows (y)
  static constexpr int SLOTB = HY * ROWB;                // one halo plane
  static constexpr int WB = 27 * CIN * COUT * 2;         // packed BF16 weights
  static constexpr int WSH = 3 * COUT * 16;              // bytes per (dy, dx, channel chunk): 3 COUT rows of 8
  static constexpr int HALO = WB;                        // halo slots after the weights
  static constexpr int NSL = 5;                          // halo planes in the ring
  static constexpr int LAG = 2;                          // planes between a plane's copies and its announcement
  static constexpr int S = 6;                            // output-plane accumulators in the ring
  static constexpr int TCOLS = (S + 2) * COUT;           // + two overflow blocks
  static constexpr int BAR = HALO + NSL * SLOTB;         // mbarriers, TMEM address, abort flag
  static constexpr int NBAR = 2 * NSL + 2 * S + 1;
  static constexpr int BIAS = BAR + NBAR * 8 + 16;       // COUT floats
  static constexpr int BYTES = BIAS + COUT * 4;
  static_assert(TCOLS == 128 || TCOLS == 256, "tensor-memory allocation: a power of two");
  static_assert(S % NGRP == 0, "each accumulator belongs to one epilogue group");
};

struct ConvArgs {
  int nx, ny, nz;                 // coarse interior
  const __nv_bfloat16 * in;       // [cell][CIN]
  const __nv_bfloat16 * w;        // packed [dy+1][dx+1][CIN/8][3 COUT][8], rows (dz+1) COUT + co
  const float * bias;             // [COUT] (forward epilogues)
  const __nv_bfloat16 * zsave;    // [cell][COUT] pre-activations (EPI_DGELU)
  __nv_bfloat16 * out;            // [cell][COUT] (EPI_GELU, EPI_DGELU)
  __nv_bfloat16 * pre;            // [cell][COUT] pre-activations to keep (EPI_GELU, optional)
  float * outf;                   // [cell][nout] (EPI_LINEAR)
  int nout;
  unsigned * status;
};

__device__ __forceinline__ int wrapi(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

__device__ __forceinline__ void nn_arrive(unsigned long long * bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(bar)) : "memory");
}
// The loader threads' share (thread lt of 32 NLD) of one halo plane (global
// plane kp) into a slot: 16-byte units, coalesced over the channel chunks of
// consecutive cells, written to [y][chunk][x]; cells outside 0 <= x < nx are
// zero-filled (the walls), y wraps around.
template <int CIN>
__device__ __forceinline__ void load_halo_part(char * slot, const __nv_bfloat16 * in, int nx, int ny, int x0, int y0,
                                               int kp, int lt) {
  constexpr int CC = CIN / 8;
  for (int u = lt; u < HY * HX * CC; u += 32 * NLD) {
    const int cc = u % CC, xh = (u / CC) % HX, yh = u / (CC * HX);
    const int i = x0 - 1 + xh, j = wrapi(y0 - 1 + yh, ny);
    const bool valid = i >= 0 && i < nx;
    const __nv_bfloat16 * src = in + ((size_t)((size_t)kp * ny + j) * nx + (valid ? i : 0)) * CIN + cc * 8;
    cp16(slot + ((yh * CC + cc) * HX + xh) * 16, src, valid);
  }
}
// zeros into 32 lanes x N consecutive columns (one lane per thread of the warp)
template <int N>
__device__ __forceinline__ void tmem_zero(unsigned taddr) {
  static_assert(N == 8 || N == 16, "8 or 16 columns");
  const unsigned z = 0u;
  if constexpr (N == 16)
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
        "%1};" ::"r"(taddr), "r"(z)
        : "memory");
  else
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1};" ::"r"(taddr), "r"(z)
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// bounded wait that also gives up once another role of the CTA has given up
__device__ __forceinline__ bool conv_wait(unsigned long long * bar, unsigned parity, volatile int * abort_flag) {
  if (nn_mbar_try(bar, parity)) return true;
  const long long t0 = clock64();
  while (!nn_mbar_try(bar, parity)) {
    if (*abort_flag) return false;
    if (clock64() - t0 > kNnWaitCycles) {
      *abort_flag = 1;
      return false;
    }
  }
  return true;
}

// The CTA's output planes: q0 <= q < q1 in the order q = tile nz + z (the
// 128-cell column tiles, x fastest), an equal share of all of them, walked as
// segments of one tile each (a z range that the CTA marches through).
struct ConvSeg { int x0, y0, z0, z1; };
struct ConvCursor {
  long long q, q1;
  __device__ __forceinline__ ConvCursor(const ConvArgs & A) {
    const long long total = (long long)(A.nx / TX) * (A.ny / TY) * A.nz;
    q = total * blockIdx.x / gridDim.x;
    q1 = total * (blockIdx.x + 1) / gridDim.x;
  }
  __device__ __forceinline__ bool next(const ConvArgs & A, ConvSeg & s) {
    if (q >= q1) return false;
    const int nbx = A.nx / TX;
    const int tile = (int)(q / A.nz), z0 = (int)(q % A.nz);
    const long long rest = q1 - q;
    const int z1 = rest < (long long)(A.nz - z0) ? z0 + (int)rest : A.nz;
    s.x0 = (tile % nbx) * TX;
    s.y0 = (tile / nbx) * TY;
    s.z0 = z0;
    s.z1 = z1;
    q += z1 - z0;
    return true;
  }
};

// Accumulator rows = TMEM lanes: warp w drains lane quarter w % 4 of block blk
// (and of its overflow block), all COUT columns in chunks of 16 (bias bias[]
// in shared memory), and zeroes what it read; the zeros land while it
// computes. The epilogue warps form NGRP groups of four that take the output
// planes in turn, so that NGRP planes are drained at a time.
template <int CIN, int COUT, int EPI>
__device__ __forceinline__ void conv_epilogue(const ConvArgs & A, unsigned tmem, int blk, int warp, size_t cell,
                                              unsigned long long * empty, int lane, const float * bias) {
  constexpr int S = ConvLayout<CIN, COUT>::S;
  const unsigned tq = tmem + ((unsigned)((warp & 3) * 32) << 16) + (unsigned)(blk * COUT);
#pragma unroll
  for (int c0 = 0; c0 < COUT; c0 += 16) {
    const unsigned ta = tq + c0;
    float v[16];
    tmem_ld16(ta, v);
    tmem_zero<16>(ta);
    if (blk < 2) {   // the part collected in the overflow block
      const unsigned tb = ta + (unsigned)(S * COUT);
      float w[16];
      tmem_ld16(tb, w);
      tmem_zero<16>(tb);
#pragma unroll
      for (int q = 0; q < 16; q++) v[q] += w[q];
    }
    if constexpr (EPI == EPI_LINEAR) {
#pragma unroll
      for (int q = 0; q < 16; q++)
        if (c0 + q < A.nout) A.outf[cell * A.nout + c0 + q] = v[q] + bias[c0 + q];
    } else {
      alignas(16) __nv_bfloat162 o[8];
      if constexpr (EPI == EPI_GELU) {
        alignas(16) __nv_bfloat162 zp[8];
#pragma unroll
        for (int q = 0; q < 16; q += 2) {
          const float za = v[q] + bias[c0 + q], zb = v[q + 1] + bias[c0 + q + 1];
          zp[q / 2] = __floats2bfloat162_rn(za, zb);
          o[q / 2] = __floats2bfloat162_rn(gelu(za), gelu(zb));
        }
        if (A.pre) {
          uint4 * dp = reinterpret_cast<uint4 *>(A.pre + cell * COUT + c0);
          dp[0] = reinterpret_cast<const uint4 *>(zp)[0];
          dp[1] = reinterpret_cast<const uint4 *>(zp)[1];
        }
      } else {
        alignas(16) __nv_bfloat162 zs[8];
        const uint4 * sp = reinterpret_cast<const uint4 *>(A.zsave + cell * COUT + c0);
        reinterpret_cast<uint4 *>(zs)[0] = sp[0];
        reinterpret_cast<uint4 *>(zs)[1] = sp[1];
#pragma unroll
        for (int q = 0; q < 16; q += 2) {
          const float2 zf = __bfloat1622float2(zs[q / 2]);
          o[q / 2] = __floats2bfloat162_rn(v[q] * gelu_grad(zf.x), v[q + 1] * gelu_grad(zf.y));
        }
      }
      uint4 * op = reinterpret_cast<uint4 *>(A.out + cell * COUT + c0);
      op[0] = reinterpret_cast<const uint4 *>(o)[0];
      op[1] = reinterpret_cast<const uint4 *>(o)[1];
    }
  }
  // the accumulator may be written again once every warp of the group has
  // read and zeroed its part
  tmem_wait_st();
  tc_fence_before();
  __syncwarp();
  if (lane == 0) nn_arrive(empty);
}

// Persistent CTAs, each over its share of the output planes (ConvCursor).
// Loader warps (NLD): the input planes of its segments, in order, into a ring
// of NSL slots (16-byte asynchronous copies; each thread arrives on full once its
// copies of a plane landed). MMA warp (warp NEPI, one thread): per input plane
// the MMAs of its 9 shifts into the accumulators of the output planes it
// feeds; tcgen05.commit then releases the slot (slot_free) and, when an output
// plane got its last contribution, hands it to the epilogue (acc_full). Before
// an output plane's first contribution its accumulator must have been drained
// and zeroed (acc_empty). Epilogue warps 0 .. NEPI-1: per output plane, wait
// acc_full, read and zero the accumulator, release it, apply the epilogue and
// store. Every wait is bounded; a CTA whose wait gave up stops issuing and
// storing, waits (bounded) for the copies and MMAs it started, and reports
// ST_TIMEOUT.
template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(CONV_THREADS, 2) conv3_kernel(ConvArgs A) {
  using L = ConvLayout<CIN, COUT>;
  constexpr int NS = L::NSL, S = L::S;
  extern __shared__ __align__(128) char smc[];
  char * wsm = smc;
  char * halo = smc + L::HALO;
  unsigned long long * full = reinterpret_cast<unsigned long long *>(smc + L::BAR);
  unsigned long long * sfree = full + NS;
  unsigned long long * accf = sfree + NS;
  unsigned long long * acce = accf + S;
  unsigned long long * fin = acce + S;
  unsigned * tslot = reinterpret_cast<unsigned *>(fin + 1);
  volatile int * abort_flag = reinterpret_cast<volatile int *>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == NEPI) tmem_alloc(tslot, L::TCOLS);
  if (tid == 0) {
    for (int s = 0; s < NS; s++) {
      nn_mbar_init(&full[s], 32 * NLD);
      nn_mbar_init(&sfree[s], 1);
    }
    for (int a = 0; a < S; a++) {
      nn_mbar_init(&accf[a], 1);
      nn_mbar_init(&acce[a], 4);
    }
    nn_mbar_init(fin, 1);
    *abort_flag = 0;
    fence_barrier_init();
  }
  float * bias_s = reinterpret_cast<float *>(smc + L::BIAS);
  if (tid < COUT) bias_s[tid] = (EPI != EPI_DGELU) ? A.bias[tid] : 0.f;
  // weights: the exact shared-memory image, read by the tensor cores
  for (int u = tid; u < L::WB / 16; u += CONV_THREADS) cp16(wsm + u * 16, reinterpret_cast<const char *>(A.w) + u * 16, true);
  cp_commit();
  cp_wait<0>();
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tslot;
  if (warp < NEPI) {   // every accumulator starts at zero
    const unsigned tl = tmem + ((unsigned)((warp & 3) * 32) << 16);
    for (int c = warp >> 2; c < S + 2; c += NGRP)
      for (int c0 = 0; c0 < COUT; c0 += 16) tmem_zero<16>(tl + c * COUT + c0);
    tmem_wait_st();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  auto colslot = [&](int g) { return S - 1 - (g % S); };
  if (warp == NEPI) {
    if (lane == 0) {
      // K-major weights: channel chunks (K) at WSH, groups of 8 rows (N) at 128 bytes
      const uint64_t bdesc0 = smem_desc(su32(wsm), L::WSH, 128);
      const unsigned hb = su32(halo);
      bool ok = true;
      int hc = 0, gb = 0;   // input planes consumed; output planes of the segments before this one
      ConvCursor cur(A);
      ConvSeg it;
      while (ok && cur.next(A, it)) {
        for (int p = it.z0 - 1; p <= it.z1 && ok; p++, hc++) {
          ok = conv_wait(&full[hc % NS], (unsigned)(hc / NS) & 1u, abort_flag);
          // first contribution to output plane p + 1: its accumulator drained
          const int gn = gb + (p + 1 - it.z0);
          if (ok && p + 1 < it.z1 && gn >= S) ok = conv_wait(&acce[gn % S], (unsigned)(gn / S - 1) & 1u, abort_flag);
          if (!ok) break;
          tc_fence_after();
          // outputs ohi .. olo (descending: ascending accumulator blocks), taps
          // dz = p - o; the window starts at block c(g(p + 1))
          const int ohi = min(p + 1, it.z1 - 1), olo = max(p - 1, it.z0);
          const int n = ohi - olo + 1;
          const int blk = colslot(gb + (p + 1 - it.z0)) + (p + 1 - ohi);
          const uint64_t adesc = smem_desc(hb + (unsigned)((hc % NS) * L::SLOTB), L::CHB, L::ROWB);
          const unsigned d = tmem + (unsigned)(blk * COUT);
          const uint32_t idesc = n == 1 ? instr_desc_bf16(128, COUT, 0, 0)
                               : n == 2 ? instr_desc_bf16(128, 2 * COUT, 0, 0)
                                        : instr_desc_bf16(128, 3 * COUT, 0, 0);
          const uint64_t bd0 = bdesc0 + (uint64_t)(((p - ohi + 1) * COUT * 16) >> 4);   // rows of tap dz = p - ohi
#pragma unroll
          for (int sh = 0; sh < 9; sh++) {
            const int dy = sh / 3, dx = sh % 3;   // offsets + 1
#pragma unroll
            for (int kk = 0; kk < CIN / 16; kk++) {
              // start addresses advance in 16-byte units in the low bits of the descriptors
              const uint64_t a = adesc + (uint64_t)((dy * L::ROWB + dx * 16 + kk * 2 * L::CHB) >> 4);
              const uint64_t b = bd0 + (uint64_t)(((sh * L::CC + 2 * kk) * L::WSH) >> 4);
              mma_bf16(d, a, b, idesc, true);
            }
          }
          mma_commit(&sfree[hc % NS]);
          if (p - 1 >= it.z0) mma_commit(&accf[(gb + p - 1 - it.z0) % S]);   // output plane p - 1 complete
        }
        gb += it.z1 - it.z0;
      }
      if (!ok) atomicOr(A.status, ST_TIMEOUT);
      // drain: the MMAs issued and the arrivals of their last slot releases
      mma_commit(fin);
      nn_mbar_wait(fin, 0);
      for (int h = hc - 1; h >= 0 && h >= hc - NS; h--) nn_mbar_wait(&sfree[h % NS], (unsigned)(h / NS) & 1u);
    }
    __syncwarp();
  } else if (warp > NEPI) {
    // loaders: plane h into slot h % NS once the MMAs of plane h - NS are done.
    // Plane h - LAG is announced (each thread: its copies landed, made visible
    // to the tensor cores, one arrival) before that wait, so the announcement
    // never waits on recent MMAs: while the loaders wait for a slot, the MMA
    // warp has the planes up to h - LAG
    constexpr int LAG = L::LAG;
    const int lt = tid - 32 * (NEPI + 1);
    int h = 0;
    bool ok = true;
    ConvCursor cur(A);
    ConvSeg it;
    while (ok && cur.next(A, it)) {
      for (int p = it.z0 - 1; p <= it.z1; p++, h++) {
        if (h >= LAG) {
          cp_wait<LAG - 1>();
          fence_proxy_async();
          nn_arrive(&full[(h - LAG) % NS]);
        }
        if (h >= NS && !conv_wait(&sfree[h % NS], (unsigned)((h - NS) / NS) & 1u, abort_flag)) {
          ok = false;
          break;
        }
        load_halo_part<CIN>(halo + (h % NS) * L::SLOTB, A.in, A.nx, A.ny, it.x0, it.y0, wrapi(p, A.nz), lt);
        cp_commit();
      }
    }
    cp_wait<0>();
    fence_proxy_async();
    if (ok)
      for (int q = h - LAG < 0 ? 0 : h - LAG; q < h; q++) nn_arrive(&full[q % NS]);
    if (!ok && lane == 0) atomicOr(A.status, ST_TIMEOUT);
  } else {
    const int m = (warp & 3) * 32 + lane;   // accumulator row = TMEM lane of this thread
    const int grp = warp >> 2;              // this warp's group takes planes g with g % NGRP == grp
    int g = 0;
    bool ok = true;
    ConvCursor cur(A);
    ConvSeg it;
    while (ok && cur.next(A, it)) {
      const int xi = it.x0 + (m & 7), yj = it.y0 + (m >> 3);
      for (int z = it.z0; z < it.z1; z++, g++) {
        if (g % NGRP != grp) continue;
        if (!conv_wait(&accf[g % S], (unsigned)(g / S) & 1u, abort_flag)) {
          if (lane == 0) atomicOr(A.status, ST_TIMEOUT);
          ok = false;
          break;
        }
        tc_fence_after();
        const size_t cell = ((size_t)z * A.ny + yj) * A.nx + xi;
        conv_epilogue<CIN, COUT, EPI>(A, tmem, colslot(g), warp, cell, &acce[g % S], lane, bias_s);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == NEPI) tmem_free(tmem, L::TCOLS);
}

// ---- convolution: weight gradient -----------------------------------------
// dW[t][co][ci] = sum over cells of X[cell + tap t][ci] dY[cell][co] as
// D (M = 128, N = COUT) += A (M x K = 16 cells) B^T, both operands MN-major:
// A is the input halo (a 16-byte unit = 8 channels of one cell; channel chunks
// at CHB continue into the next halo row, so rows m = (y shift s, ci) cover
// NSH = 128 / CIN shifts s = dy + 1 of one (dz, dx) pair); B is the gradient
// tile of the plane, units [y][co chunk][x]. Nine accumulators (dz, dx) of
// COUT columns each live in tensor memory for the whole life of the CTA,
// which loops over (column tile, z chunk) work items; the CTA writes its raw
// partial sums, reduced afterwards by wgrad_reduce_kernel.
template <int CIN, int COUT>
struct WgradLayout {
  static constexpr int NSH = 128 / CIN;                  // y shifts per accumulator
  static constexpr int HYW = TY + NSH - 1;               // halo rows y0 - 1 .. y0 + TY + NSH - 3
  static constexpr int CHB = HX * 16;
  static constexpr int ROWB = (CIN / 8) * CHB;
  static constexpr int SLOTB = HYW * ROWB;
  static constexpr int GB = TY * (COUT / 8) * TX * 16;   // gradient tile of one plane
  static constexpr int NSW = 5, NGS = 3;                 // halo and gradient slots: MMAs of two planes in flight
  static constexpr int GOFF = NSW * SLOTB;               // gradient slots after the halo ring
  static constexpr int BAR = GOFF + NGS * GB;            // two mbarriers, then the TMEM address
  static constexpr int USED = BAR + 32;
  static constexpr int TCOLS = 9 * COUT > 256 ? 512 : 256;
  // one CTA per SM, so that its tensor-memory allocation never waits on
  // another CTA's: ask for more than half of the shared memory
  static constexpr int BYTES = USED < 120 * 1024 ? 120 * 1024 : USED;
};

struct WgradArgs {
  int nx, ny, nz, zc, nitems;
  const __nv_bfloat16 * x;    // [cell][CIN] layer input
  const __nv_bfloat16 * dy;   // [cell][COUT] gradient of the layer's pre-activation
  float * part;               // [gridDim.x][9][128][COUT] raw sums, then [gridDim.x][COUT] bias sums
  unsigned * status;
};

template <int CIN>
__device__ __forceinline__ void load_halo_w(char * slot, const __nv_bfloat16 * in, int nx, int ny, int x0, int y0,
                                            int kp, int hyw) {
  constexpr int CC = CIN / 8;
  for (int u = threadIdx.x; u < hyw * HX * CC; u += NN_THREADS) {
    const int cc = u % CC, xh = (u / CC) % HX, yh = u / (CC * HX);
    const int i = x0 - 1 + xh;
    int j = (y0 - 1 + yh) % ny;
    if (j < 0) j += ny;
    const bool valid = i >= 0 && i < nx;
    const __nv_bfloat16 * src = in + ((size_t)((size_t)kp * ny + j) * nx + (valid ? i : 0)) * CIN + cc * 8;
    cp16(slot + ((yh * CC + cc) * HX + xh) * 16, src, valid);
  }
}
template <int COUT>
__device__ __forceinline__ void load_grad_tile(char * slot, const __nv_bfloat16 * dy, int nx, int ny, int x0, int y0,
                                               int z) {
  constexpr int CC = COUT / 8;
  for (int u = threadIdx.x; u < TY * TX * CC; u += NN_THREADS) {
    const int cc = u % CC, x = (u / CC) % TX, y = u / (CC * TX);
    const __nv_bfloat16 * src = dy + ((size_t)((size_t)z * ny + y0 + y) * nx + x0 + x) * COUT + cc * 8;
    cp16(slot + ((y * CC + cc) * TX + x) * 16, src, true);
  }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(NN_THREADS, 1) conv3_wgrad_kernel(WgradArgs A) {
  using L = WgradLayout<CIN, COUT>;
  extern __shared__ __align__(128) char smw[];
  char * halo = smw;
  char * gsl = smw + L::GOFF;
  unsigned long long * bar = reinterpret_cast<unsigned long long *>(smw + L::BAR);   // two
  unsigned * tslot = reinterpret_cast<unsigned *>(smw + L::BAR + 16);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nbx = A.nx / TX, ncol = nbx * (A.ny / TY);

  if (warp == 0) tmem_alloc(tslot, L::TCOLS);
  if (tid == 0) {
    nn_mbar_init(&bar[0], 1);
    nn_mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tslot;
  constexpr uint32_t IDESC = instr_desc_bf16(128, COUT, 1, 1);
  float bsum = 0.f;                 // bias gradient of channel tid (tid < COUT)
  bool first = true;                // no accumulator written yet
  unsigned phase[2] = {0u, 0u};
  int pending[2] = {0, 0};          // commits on each barrier not yet waited for
  bool bad = false;
  // wait for the MMAs committed on barrier b (bounded)
  auto drain = [&](int b) {
    if (!pending[b]) return;
    const bool ok = nn_mbar_wait(&bar[b], phase[b]);
    phase[b] ^= 1u;
    pending[b] = 0;
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(A.status, ST_TIMEOUT);
      bad = true;
    }
  };

  // Per plane z: (a) the MMAs of plane z - 2 have finished (their barrier is
  // the one plane z commits on), so the halo slot of z + 2 and the gradient
  // slot of z + 1 are free; (b) issue those copies; (c) wait for the planes up
  // to z + 1 and the tile of z; (d) issue the plane's 72 MMAs; the MMAs of
  // z - 1 and z overlap the copies of the next planes.
  for (int item = blockIdx.x; item < A.nitems && !bad; item += gridDim.x) {
    const int col = item % ncol, zch = item / ncol;
    const int x0 = (col % nbx) * TX, y0 = (col / nbx) * TY;
    const int z0 = zch * A.zc, z1 = min(z0 + A.zc, A.nz);
    drain(0);
    drain(1);
    if (bad) break;
    load_halo_w<CIN>(halo + 0 * L::SLOTB, A.x, A.nx, A.ny, x0, y0, wrapi(z0 - 1, A.nz), L::HYW);
    load_halo_w<CIN>(halo + 1 * L::SLOTB, A.x, A.nx, A.ny, x0, y0, z0, L::HYW);
    load_halo_w<CIN>(halo + 2 * L::SLOTB, A.x, A.nx, A.ny, x0, y0, wrapi(z0 + 1, A.nz), L::HYW);
    load_grad_tile<COUT>(gsl + 1 * L::GB, A.dy, A.nx, A.ny, x0, y0, z0);   // tile of plane z in slot r % 3
    cp_commit();
    for (int z = z0, it = 0; z < z1; z++, it++) {
      const int r = z - z0 + 1;
      drain(it & 1);
      if (bad) break;
      if (z + 2 <= z1) load_halo_w<CIN>(halo + ((r + 2) % L::NSW) * L::SLOTB, A.x, A.nx, A.ny, x0, y0,
                                        wrapi(z + 2, A.nz), L::HYW);
      if (z + 1 < z1) load_grad_tile<COUT>(gsl + ((r + 1) % L::NGS) * L::GB, A.dy, A.nx, A.ny, x0, y0, z + 1);
      cp_commit();
      cp_wait<1>();
      fence_proxy_async();
      __syncthreads();
      const char * g = gsl + (r % L::NGS) * L::GB;
      if (tid == 0) {
        tc_fence_after();
        const unsigned hb = su32(halo), gb = su32(g);
        const unsigned sb[3] = {hb + ((r - 1) % L::NSW) * L::SLOTB, hb + (r % L::NSW) * L::SLOTB,
                                hb + ((r + 1) % L::NSW) * L::SLOTB};
#pragma unroll
        for (int a = 0; a < 9; a++) {
          const int dz = a / 3 - 1, dx = a % 3 - 1;
          const unsigned a0 = sb[dz + 1] + (1 + dx) * 16;
#pragma unroll
          for (int s = 0; s < TY / 2; s++) {
            const uint64_t ad = smem_desc(a0 + 2 * s * L::ROWB, L::ROWB, L::CHB);
            const uint64_t bd = smem_desc(gb + 2 * s * (COUT / 8) * TX * 16, (COUT / 8) * TX * 16, TX * 16);
            mma_bf16(tmem + a * COUT, ad, bd, IDESC, !(first && s == 0));
          }
        }
        mma_commit(&bar[it & 1]);
      }
      pending[it & 1] = 1;
      if (tid < COUT) {   // bias gradient from the same tile
        constexpr int CC = COUT / 8;
        const __nv_bfloat16 * gv = reinterpret_cast<const __nv_bfloat16 *>(g);
        float acc = 0.f;
        for (int c = 0; c < TX * TY; c++) {
          const int x = c % TX, y = c / TX;
          acc += __bfloat162float(gv[((y * CC + tid / 8) * TX + x) * 8 + tid % 8]);
        }
        bsum += acc;
      }
      first = false;
      tc_fence_before();
      __syncthreads();
    }
    cp_wait<0>();
    __syncthreads();
  }
  drain(0);
  drain(1);
  tc_fence_after();
  // raw partial sums of this CTA: [a][m][co]
  float * dst = A.part + (size_t)blockIdx.x * 9 * 128 * COUT;
  const int m = warp * 32 + lane;
  for (int a = 0; a < 9; a++) {
#pragma unroll
    for (int h = 0; h < COUT / 16; h++) {
      float v[16];
      tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + a * COUT + h * 16, v);
#pragma unroll
      for (int q = 0; q < 16; q++) dst[((size_t)a * 128 + m) * COUT + h * 16 + q] = first ? 0.f : v[q];
    }
  }
  float * bdst = A.part + (size_t)gridDim.x * 9 * 128 * COUT + (size_t)blockIdx.x * COUT;
  if (tid < COUT) bdst[tid] = bsum;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_free(tmem, L::TCOLS);
}

// Sum of the CTAs' raw partials into the master-layout gradients
// dw[t][co][ci] (real channel counts) and db[co]; beta = 0 overwrites,
// 1 accumulates.
__global__ void wgrad_reduce_kernel(const float * __restrict__ part, int nblk, int cinp, int coutp, int cin, int cout,
                                    float * __restrict__ dw, float * __restrict__ db, float beta) {
  const int nw = 27 * cout * cin;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nw + cout; q += gridDim.x * blockDim.x) {
    if (q < nw) {
      const int ci = q % cin, co = (q / cin) % cout, t = q / (cin * cout);
      const int dz = t / 9, dyi = (t / 3) % 3, dx = t % 3;   // dyi = dy + 1
      const int a = dz * 3 + dx, m = (dyi * (cinp / 8) + ci / 8) * 8 + ci % 8;
      float acc = 0.f;
      for (int b = 0; b < nblk; b++) acc += part[(((size_t)b * 9 + a) * 128 + m) * coutp + co];
      dw[q] = beta * dw[q] + acc;
    } else {
      const int co = q - nw;
      float acc = 0.f;
      const float * bp = part + (size_t)nblk * 9 * 128 * coutp;
      for (int b = 0; b < nblk; b++) acc += bp[(size_t)b * coutp + co];
      db[co] = beta * db[co] + acc;
    }
  }
}

template <int CIN, int COUT>
int launch_wgrad(WgradArgs a, int nblk, cudaStream_t st) {
  using L = WgradLayout<CIN, COUT>;
  if (cudaFuncSetAttribute(conv3_wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES) !=
      cudaSuccess)
    return 1;
  conv3_wgrad_kernel<CIN, COUT><<<nblk, NN_THREADS, L::BYTES, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

// ---- loss, optimiser -------------------------------------------------------
// Mean squared error of the predicted forcing against the target over n
// cells x nc channels (FP32, [cell][nc]), optional per-cell weight (NULL: 1):
// loss += sum w (f - t)^2 / (n nc) (double accumulator) and the gradient with
// respect to f, 2 w (f - t) / (n nc), as BF16 [cell][cp] (channels >= nc zero).
__global__ void mse_kernel(const float * __restrict__ f, const float * __restrict__ t, const float * __restrict__ w,
                           size_t n, int nc, int cp, float scale, __nv_bfloat16 * __restrict__ g,
                           double * __restrict__ loss) {
  double acc = 0.;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const float wc = w ? w[q] : 1.f;
    alignas(16) __nv_bfloat16 o[16];
    for (int c = 0; c < 16; c++) o[c] = __float2bfloat16_rn(0.f);
    for (int c = 0; c < nc; c++) {
      const float d = f[q * nc + c] - t[q * nc + c];
      acc += (double)(wc * d * d);
      o[c] = __float2bfloat16_rn(2.f * wc * d * scale);
    }
    for (int c0 = 0; c0 < cp; c0 += 16) {
      uint4 * dp = reinterpret_cast<uint4 *>(g + q * cp + c0);
      if (c0 == 0) {
        dp[0] = reinterpret_cast<const uint4 *>(o)[0];
        dp[1] = reinterpret_cast<const uint4 *>(o)[1];
      } else {
        dp[0] = make_uint4(0, 0, 0, 0);
        dp[1] = make_uint4(0, 0, 0, 0);
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];
    atomicAdd(loss, s * (double)scale);
  }
}

// Adam (Kingma and Ba 2015) on FP32 master parameters; step >= 1 is the
// update count, bias corrections 1 - beta^step.
__global__ void adam_kernel(float * __restrict__ p, const float * __restrict__ g, float * __restrict__ m,
                            float * __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
  }
}

// ---- weights ---------------------------------------------------------------
// Master weights (FP32) w[t][co][ci], t = 9 (dz+1) + 3 (dy+1) + (dx+1), real
// channel counts cin x cout, into the BF16 shared-memory images of the forward
// convolution, [dy+1][dx+1][ci/8][(dz+1) COUTP + co][ci%8] over padded counts
// CINP x COUTP (the three z taps of a shift side by side along N), and of the
// input-gradient convolution (taps mirrored, channels swapped),
// [1-dy][1-dx][co/8][(1-dz) CINP + ci][co%8]. Padding channels are zero.
__global__ void pack_weights_kernel(const float * __restrict__ w, int cin, int cout, int cinp, int coutp,
                                    __nv_bfloat16 * __restrict__ fwd, __nv_bfloat16 * __restrict__ bwd) {
  const int n = 27 * cinp * coutp;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int ci = q % cinp, co = (q / cinp) % coutp, t = q / (cinp * coutp);
    const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;   // offsets + 1
    const float v = (ci < cin && co < cout) ? w[((size_t)t * cout + co) * cin + ci] : 0.f;
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    fwd[((size_t)((dy * 3 + dx) * (cinp / 8) + ci / 8) * 3 * coutp + dz * coutp + co) * 8 + ci % 8] = b;
    if (bwd)
      bwd[((size_t)(((2 - dy) * 3 + (2 - dx)) * (coutp / 8) + co / 8) * 3 * cinp + (2 - dz) * cinp + ci) * 8 + co % 8] =
          b;
  }
}

// SMs of the current device
static int device_sms() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 0;
  return n;
}

// CTAs of a kernel that fit on one SM: registers (allocated per warp in units
// of 256), shared memory (plus the per-block reservation), threads, and at
// most 512 tensor-memory columns, so that no allocation has to wait
static int conv_ctas_per_sm(const void * kern, int threads, int smem, int tcols) {
  int dev = 0, regs_sm = 0, smem_sm = 0, resv = 0, thr_sm = 0;
  cudaFuncAttributes fa;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaFuncGetAttributes(&fa, kern) != cudaSuccess ||
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess)
    return 0;
  const int warps = (threads + 31) / 32;
  const int regs_cta = warps * ((fa.numRegs * 32 + 255) / 256 * 256);
  int n = 512 / tcols;
  if (regs_cta > 0 && regs_sm / regs_cta < n) n = regs_sm / regs_cta;
  if (smem_sm / (smem + resv) < n) n = smem_sm / (smem + resv);
  if (thr_sm / (32 * warps) < n) n = thr_sm / (32 * warps);
  return n;
}

template <int CIN, int COUT, int EPI>
int launch_conv3(ConvArgs a, cudaStream_t st) {
  using L = ConvLayout<CIN, COUT>;
  auto kern = conv3_kernel<CIN, COUT, EPI>;
  // once per instantiation: the whole unified L1 as shared memory, so that two
  // CTAs fit per SM, and the resident CTAs per SM from the kernel's registers,
  // shared memory and tensor-memory columns (the occupancy query reports one
  // CTA here, which leaves half of every SM idle)
  static const int per_sm = [&] {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES) != cudaSuccess ||
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared) !=
            cudaSuccess)
      return 0;
    return conv_ctas_per_sm(reinterpret_cast<const void *>(kern), CONV_THREADS, L::BYTES, L::TCOLS);
  }();
  if (per_sm < 1) return 1;
  const long long total = (long long)(a.nx / TX) * (a.ny / TY) * a.nz;   // output planes of all tiles
  const int g = per_sm * device_sms();
  if (g < 1) return 1;
  const int grid = total < g ? (int)total : g;
  kern<<<grid, CONV_THREADS, L::BYTES, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

template <int EPI>
int dispatch_conv3(int cin, int cout, const ConvArgs & a, cudaStream_t st) {
  if (cin == 16 && cout == 32) return launch_conv3<16, 32, EPI>(a, st);
  if (cin == 32 && cout == 32) return launch_conv3<32, 32, EPI>(a, st);
  if (cin == 32 && cout == 16) return launch_conv3<32, 16, EPI>(a, st);
  if (cin == 16 && cout == 16) return launch_conv3<16, 16, EPI>(a, st);
  return 1;
}

// weight gradient: (column tile, z chunk) work items and the CTAs over them
void wgrad_split(int nx, int ny, int nz, int & zc, int & nitems, int & nblk) {
  const int ncol = (nx / TX) * (ny / TY);
  zc = nz;
  while (zc > 4 && (long)ncol * ((nz + zc - 1) / zc) < 148L * 2) zc = (zc + 1) / 2;
  nitems = ncol * ((nz + zc - 1) / zc);
  nblk = nitems < 148 ? nitems : 148;
}

}  // namespace

// ---- grid side: 4x restriction, network input, forcing --------------------
// Restriction of a fine state to the grid coarser by R in every direction
// (coarse cell = R^3 fine cells, coarse radial faces = every R-th fine face):
// every coarse face flux is the sum of the fine fluxes through it, so a
// discretely divergence-free fine field stays divergence-free. ux at coarse
// face I: the mean of the R^2 fine faces (their flux weights J/hx do not vary
// on a radial face); uy at coarse y-face J: weights J/hy = hx hz of the fine
// faces' cells; uz at coarse z-face K: weights J/hz = hx hy; t and p: volume
// (J) weighted cell means. Interior only; walls and images follow from the
// boundary kernels.
template <int R>
__global__ void coarsen_kernel(Geo gf, FieldsT<double> f, Geo gc, FieldsT<double> c) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int J = blockIdx.y + 1, K = blockIdx.z + 1;
  if (I > gc.nx) return;
  const int i0 = R * (I - 1) + 1, j0 = R * (J - 1) + 1, k0 = R * (K - 1) + 1;
  double sux = 0., suy = 0., wy = 0., suz = 0., wz = 0., st = 0., sp = 0., wv = 0.;
  for (int a = 0; a < R; a++) {
    const int i = i0 + a;
    const double hxz = gf.jdxc[i] / gf.hyxc[i], hxy = gf.jdxc[i] / gf.hz, vol = gf.jdxc[i];
    for (int b = 0; b < R; b++) {
      if (a == 0) {   // x face i0: (j0 + b, k0 + e)
        for (int e = 0; e < R; e++) sux += f.ux[fidx(gf, i0, j0 + b, k0 + e)];
      }
      suy += hxz * f.uy[cidx(gf, i, j0, k0 + b)];
      suz += hxy * f.uz[cidx(gf, i, j0 + b, k0)];
      for (int e = 0; e < R; e++) {
        st += vol * f.t[cidx(gf, i, j0 + b, k0 + e)];
        sp += vol * f.p[cidx(gf, i, j0 + b, k0 + e)];
      }
    }
    wy += R * hxz;
    wz += R * hxy;
    wv += R * R * vol;
  }
  c.ux[fidx(gc, I, J, K)] = I == 1 ? 0. : sux / (R * R);
  c.uy[cidx(gc, I, J, K)] = suy / wy;
  c.uz[cidx(gc, I, J, K)] = suz / wz;
  c.t[cidx(gc, I, J, K)] = st / wv;
  c.p[cidx(gc, I, J, K)] = sp / wv;
}

void launch_coarsen(const Geo & gf, const FieldsT<double> & f, const Geo & gc, const FieldsT<double> & c,
                    cudaStream_t st) {
  const dim3 block(64), grid((gc.nx + 63) / 64, gc.ny, gc.nz);
  coarsen_kernel<4><<<grid, block, 0, st>>>(gf, f, gc, c);
}

// Network input of the coarse state, BF16 [cell][cp] over interior cells
// (i, j, k from 0): ux averaged to the centre, uy, uz, each divided by its
// scale, and the radial index coordinate 2 (i + 1/2) / nx - 1; channels
// 4 .. cp-1 zero.
__global__ void closure_input_kernel(Geo g, const double * __restrict__ ux, const double * __restrict__ uy,
                                     const double * __restrict__ uz, double s0, double s1, double s2, int cp,
                                     __nv_bfloat16 * __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const int I = i + 1, J = j + 1, K = k + 1;
  alignas(16) __nv_bfloat16 o[16];
  for (int q = 0; q < 16; q++) o[q] = __float2bfloat16_rn(0.f);
  o[0] = __float2bfloat16_rn((float)(0.5 * (ux[fidx(g, I, J, K)] + ux[fidx(g, I + 1, J, K)]) / s0));
  o[1] = __float2bfloat16_rn((float)(uy[cidx(g, I, J, K)] / s1));
  o[2] = __float2bfloat16_rn((float)(uz[cidx(g, I, J, K)] / s2));
  o[3] = __float2bfloat16_rn((float)(2.0 * (i + 0.5) / g.nx - 1.0));
  uint4 * dp = reinterpret_cast<uint4 *>(out + (((size_t)k * g.ny + j) * g.nx + i) * cp);
  dp[0] = reinterpret_cast<const uint4 *>(o)[0];
  dp[1] = reinterpret_cast<const uint4 *>(o)[1];
  for (int c0 = 16; c0 < cp; c0 += 8) dp[c0 / 8] = make_uint4(0, 0, 0, 0);
}

void launch_closure_input(const Geo & g, const double * ux, const double * uy, const double * uz, const double s[3],
                          int cp, void * out, cudaStream_t st) {
  const dim3 block(64), grid((g.nx + 63) / 64, g.ny, g.nz);
  closure_input_kernel<<<grid, block, 0, st>>>(g, ux, uy, uz, s[0], s[1], s[2], cp,
                                               static_cast<__nv_bfloat16 *>(out));
}

// Network output f (FP32 [cell][nc], nc >= 3) times the scales into the
// packed forcing of ux (faces 2..nx: channel 0 of cell i = face i + 1 of the
// reference's numbering), uy and uz (channels 1, 2).
__global__ void closure_forcing_kernel(int nx, int ny, int nz, const float * __restrict__ f, int nc, double s0,
                                       double s1, double s2, double * __restrict__ fux, double * __restrict__ fuy,
                                       double * __restrict__ fuz) {
  const size_t n = (size_t)nx * ny * nz;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const size_t line = q / nx;
    fuy[q] = s1 * (double)f[q * nc + 1];
    fuz[q] = s2 * (double)f[q * nc + 2];
    if (i >= 1) fux[(size_t)(i - 1) + (size_t)(nx - 1) * line] = s0 * (double)f[q * nc];
  }
}

void launch_closure_forcing(int nx, int ny, int nz, const float * f, int nc, const double s[3], double * fux,
                            double * fuy, double * fuz, cudaStream_t st) {
  closure_forcing_kernel<<<1184, 256, 0, st>>>(nx, ny, nz, f, nc, s[0], s[1], s[2], fux, fuy, fuz);
}

// Closure target of one sample: (reference - predicted) / tau for ux (channel
// 0 of cell i = face i + 1; zero at the wall face), uy, uz, FP32 [cell][3].
__global__ void closure_target_kernel(Geo g, const double * __restrict__ pux, const double * __restrict__ puy,
                                      const double * __restrict__ puz, const double * __restrict__ rux,
                                      const double * __restrict__ ruy, const double * __restrict__ ruz,
                                      double inv_tau, float * __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= g.nx) return;
  const int I = i + 1, J = j + 1, K = k + 1;
  const size_t q = ((size_t)k * g.ny + j) * g.nx + i;
  const size_t f = fidx(g, I, J, K), c = cidx(g, I, J, K);
  out[q * 3 + 0] = i == 0 ? 0.f : (float)((rux[f] - pux[f]) * inv_tau);
  out[q * 3 + 1] = (float)((ruy[c] - puy[c]) * inv_tau);
  out[q * 3 + 2] = (float)((ruz[c] - puz[c]) * inv_tau);
}

void launch_closure_target(const Geo & g, const FieldsT<double> & pred, const FieldsT<double> & ref, double tau,
                           float * out, cudaStream_t st) {
  const dim3 block(64), grid((g.nx + 63) / 64, g.ny, g.nz);
  closure_target_kernel<<<grid, block, 0, st>>>(g, pred.ux, pred.uy, pred.uz, ref.ux, ref.uy, ref.uz, 1.0 / tau, out);
}

}  // namespace tcgpu

using namespace tcgpu;

static __device__ unsigned g_nn_status;   // error bits of the network kernels (ST_TIMEOUT)

static thread_local char g_nn_err[256];
static int nn_fail(const char * msg) {
  snprintf(g_nn_err, sizeof(g_nn_err), "%s", msg);
  fprintf(stderr, "tcgpu: %s\n", msg);
  return 1;
}
static bool aligned16(const void * p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
static unsigned * nn_status_ptr() {
  unsigned * p = nullptr;
  if (cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_nn_status) != cudaSuccess) return nullptr;
  return p;
}

extern "C" {

const char * tcgpu_nn_last_error(void) { return g_nn_err; }

int tcgpu_nn_pack_weights(const float * w, int cin, int cout, int cinp, int coutp, void * fwd, void * bwd,
                          void * stream) {
  if (cin > cinp || cout > coutp || cinp % 16 || coutp % 16 || !fwd) return nn_fail("nn_pack_weights: bad sizes");
  const int n = 27 * cinp * coutp;
  pack_weights_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      w, cin, cout, cinp, coutp, static_cast<__nv_bfloat16 *>(fwd), static_cast<__nv_bfloat16 *>(bwd));
  return cudaGetLastError() == cudaSuccess ? 0 : nn_fail("nn_pack_weights: launch failed");
}

int tcgpu_nn_conv3(int mode, int cin, int cout, int nx, int ny, int nz, const void * in, const void * wpacked,
                   const float * bias, const void * zsave, void * out, void * pre, float * outf, int nout,
                   void * stream) {
  if (nx % TX || ny % TY || nx <= 0 || ny <= 0 || nz <= 0)
    return nn_fail("nn_conv3: nx must be a multiple of 8 and ny of 16");
  if (!in || !wpacked || !aligned16(in) || !aligned16(wpacked)) return nn_fail("nn_conv3: inputs not 16-byte aligned");
  ConvArgs a{};
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.in = static_cast<const __nv_bfloat16 *>(in);
  a.w = static_cast<const __nv_bfloat16 *>(wpacked);
  a.bias = bias;
  a.zsave = static_cast<const __nv_bfloat16 *>(zsave);
  a.out = static_cast<__nv_bfloat16 *>(out);
  a.pre = static_cast<__nv_bfloat16 *>(pre);
  a.outf = outf;
  a.nout = nout;
  a.status = nn_status_ptr();
  if (!a.status) return nn_fail("nn_conv3: status word unavailable");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = 1;
  switch (mode) {
    case 0:
      if (!bias || !out || !aligned16(out) || (pre && !aligned16(pre))) return nn_fail("nn_conv3: bad outputs");
      rc = dispatch_conv3<EPI_GELU>(cin, cout, a, st);
      break;
    case 1:
      if (!bias || !outf || nout < 1 || nout > cout) return nn_fail("nn_conv3: bad outputs");
      rc = dispatch_conv3<EPI_LINEAR>(cin, cout, a, st);
      break;
    case 2:
      if (!zsave || !out || !aligned16(out) || !aligned16(zsave)) return nn_fail("nn_conv3: bad outputs");
      rc = dispatch_conv3<EPI_DGELU>(cin, cout, a, st);
      break;
    default:
      return nn_fail("nn_conv3: mode 0 (forward, GELU), 1 (forward, linear) or 2 (input gradient)");
  }
  return rc ? nn_fail("nn_conv3: unsupported channel counts or launch failure") : 0;
}

size_t tcgpu_nn_wgrad_workspace(int nx, int ny, int nz, int coutp) {
  if (nx % TX || ny % TY || nx <= 0 || ny <= 0 || nz <= 0) return 0;
  int zc, nitems, nblk;
  wgrad_split(nx, ny, nz, zc, nitems, nblk);
  return (size_t)nblk * (9 * 128 + 1) * coutp * sizeof(float);
}

int tcgpu_nn_conv3_wgrad(int cinp, int coutp, int cin, int cout, int nx, int ny, int nz, const void * x,
                         const void * dy, float * dw, float * db, float beta, void * workspace, size_t ws_bytes,
                         void * stream) {
  if (nx % TX || ny % TY || nx <= 0 || ny <= 0 || nz <= 0)
    return nn_fail("nn_conv3_wgrad: nx must be a multiple of 8 and ny of 16");
  if (cin > cinp || cout > coutp || !x || !dy || !dw || !db || !aligned16(x) || !aligned16(dy))
    return nn_fail("nn_conv3_wgrad: bad arguments");
  if (!workspace || ws_bytes < tcgpu_nn_wgrad_workspace(nx, ny, nz, coutp))
    return nn_fail("nn_conv3_wgrad: workspace smaller than tcgpu_nn_wgrad_workspace()");
  WgradArgs a{};
  a.nx = nx; a.ny = ny; a.nz = nz;
  int nblk;
  wgrad_split(nx, ny, nz, a.zc, a.nitems, nblk);
  a.x = static_cast<const __nv_bfloat16 *>(x);
  a.dy = static_cast<const __nv_bfloat16 *>(dy);
  a.part = static_cast<float *>(workspace);
  a.status = nn_status_ptr();
  if (!a.status) return nn_fail("nn_conv3_wgrad: status word unavailable");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = 1;
  if (cinp == 16 && coutp == 32) rc = launch_wgrad<16, 32>(a, nblk, st);
  else if (cinp == 32 && coutp == 32) rc = launch_wgrad<32, 32>(a, nblk, st);
  else if (cinp == 32 && coutp == 16) rc = launch_wgrad<32, 16>(a, nblk, st);
  else if (cinp == 16 && coutp == 16) rc = launch_wgrad<16, 16>(a, nblk, st);
  if (rc) return nn_fail("nn_conv3_wgrad: unsupported channel counts or launch failure");
  const int nred = 27 * cout * cin + cout;
  wgrad_reduce_kernel<<<(nred + 255) / 256, 256, 0, st>>>(a.part, nblk, cinp, coutp, cin, cout, dw, db, beta);
  return cudaGetLastError() == cudaSuccess ? 0 : nn_fail("nn_conv3_wgrad: reduction launch failed");
}

int tcgpu_nn_mse(const float * f, const float * t, const float * w, size_t ncell, int nc, int cp, void * grad,
                 double * loss, void * stream) {
  if (!f || !t || !grad || !loss || nc < 1 || nc > 16 || cp % 16 || cp < 16 || !aligned16(grad))
    return nn_fail("nn_mse: bad arguments");
  const float scale = 1.f / (float)((double)ncell * nc);
  mse_kernel<<<1184, 256, 0, static_cast<cudaStream_t>(stream)>>>(f, t, w, ncell, nc, cp, scale,
                                                                     static_cast<__nv_bfloat16 *>(grad), loss);
  return cudaGetLastError() == cudaSuccess ? 0 : nn_fail("nn_mse: launch failed");
}

int tcgpu_nn_adam(float * p, const float * g, float * m, float * v, size_t n, float lr, float beta1, float beta2,
                  float eps, int step, void * stream) {
  if (!p || !g || !m || !v || step < 1) return nn_fail("nn_adam: bad arguments");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<(int)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      p, g, m, v, n, lr, beta1, beta2, eps, c1, c2);
  return cudaGetLastError() == cudaSuccess ? 0 : nn_fail("nn_adam: launch failed");
}

// error bits raised by the network kernels since the last clear (synchronises the device)
int tcgpu_nn_status(int clear) {
  unsigned v = 0;
  if (cudaMemcpyFromSymbol(&v, g_nn_status, sizeof(v)) != cudaSuccess) return -1;
  if (clear) {
    const unsigned z = 0;
    if (cudaMemcpyToSymbol(g_nn_status, &z, sizeof(z)) != cudaSuccess) return -1;
  }
  return (int)v;
}

}  // extern "C"
