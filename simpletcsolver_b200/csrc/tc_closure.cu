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

// GELU, erf form: 0.5 z (1 + erf(z / sqrt 2)), and its derivative
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}


// ---- convolution: forward and input gradient ------------------------------
constexpr int TX = 8, TY = 16;             // output tile: 8 x, 16 y, one z plane (M = 128)
constexpr int HX = TX + 2, HY = TY + 2;    // halo of one plane
constexpr int NN_THREADS = 128;            // 4 warps: one TMEM lane quarter each
constexpr int NSLOT_NN = 4;                // halo planes z-1, z, z+1 and the one streaming in

enum ConvEpilogue { EPI_GELU = 0, EPI_LINEAR = 1, EPI_DGELU = 2 };

template <int CIN, int COUT>
struct ConvLayout {
  static_assert(CIN == 16 || CIN == 32, "input channels: 16 or 32");
  static_assert(COUT == 16 || COUT == 32, "output channels: 16 or 32");
  static constexpr int CHB = HX * 16;                    // bytes between channel chunks of a halo row
  static constexpr int ROWB = (CIN / 8) * CHB;           // bytes between halo rows (y)
  static constexpr int SLOTB = HY * ROWB;                // one halo plane
  static constexpr int WB = 27 * CIN * COUT * 2;         // packed BF16 weights
  static constexpr int HALO = WB;                        // halo slots after the weights
  static constexpr int BAR = HALO + NSLOT_NN * SLOTB;    // mbarrier, then the TMEM address
  static constexpr int BYTES = BAR + 16;
};

struct ConvArgs {
  int nx, ny, nz, zc;             // coarse interior, z planes per CTA
  const __nv_bfloat16 * in;       // [cell][CIN]
  const __nv_bfloat16 * w;        // packed [27][CIN/8][COUT][8]
  const float * bias;             // [COUT] (forward epilogues)
  const __nv_bfloat16 * zsave;    // [cell][COUT] pre-activations (EPI_DGELU)
  __nv_bfloat16 * out;            // [cell][COUT] (EPI_GELU, EPI_DGELU)
  __nv_bfloat16 * pre;            // [cell][COUT] pre-activations to keep (EPI_GELU, optional)
  float * outf;                   // [cell][nout] (EPI_LINEAR)
  int nout;
  unsigned * status;
};

__device__ __forceinline__ int wrapi(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

// 16-byte units of one halo plane (global plane kp) into a slot: coalesced
// over the channel chunks of consecutive cells, written to [y][chunk][x]
template <int CIN>
__device__ __forceinline__ void load_halo(char * slot, const __nv_bfloat16 * in, int nx, int ny, int x0, int y0,
                                          int kp) {
  constexpr int CC = CIN / 8;
  for (int u = threadIdx.x; u < HY * HX * CC; u += NN_THREADS) {
    const int cc = u % CC, xh = (u / CC) % HX, yh = u / (CC * HX);
    const int i = x0 - 1 + xh, j = wrapi(y0 - 1 + yh, ny);
    const bool valid = i >= 0 && i < nx;
    const __nv_bfloat16 * src = in + ((size_t)((size_t)kp * ny + j) * nx + (valid ? i : 0)) * CIN + cc * 8;
    cp16(slot + ((yh * CC + cc) * HX + xh) * 16, src, valid);
  }
}

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(NN_THREADS) conv3_kernel(ConvArgs A) {
  using L = ConvLayout<CIN, COUT>;
  extern __shared__ __align__(128) char smc[];
  char * wsm = smc;
  char * halo = smc + L::HALO;
  unsigned long long * bar = reinterpret_cast<unsigned long long *>(smc + L::BAR);
  unsigned * tslot = reinterpret_cast<unsigned *>(smc + L::BAR + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nbx = A.nx / TX;
  const int x0 = (blockIdx.x % nbx) * TX, y0 = (blockIdx.x / nbx) * TY;
  const int z0 = blockIdx.y * A.zc, z1 = min(z0 + A.zc, A.nz);

  if (warp == 0) tmem_alloc(tslot, 32);
  if (tid == 0) {
    nn_mbar_init(bar, 1);
    fence_barrier_init();
  }
  // weights (exact shared-memory image) and the first three halo planes
  for (int u = tid; u < L::WB / 16; u += NN_THREADS) cp16(wsm + u * 16, reinterpret_cast<const char *>(A.w) + u * 16, true);
  load_halo<CIN>(halo + 0 * L::SLOTB, A.in, A.nx, A.ny, x0, y0, wrapi(z0 - 1, A.nz));
  cp_commit();
  load_halo<CIN>(halo + 1 * L::SLOTB, A.in, A.nx, A.ny, x0, y0, z0);
  cp_commit();
  load_halo<CIN>(halo + 2 * L::SLOTB, A.in, A.nx, A.ny, x0, y0, wrapi(z0 + 1, A.nz));
  cp_commit();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tslot;
  constexpr uint32_t IDESC = instr_desc_bf16(128, COUT, 0, 0);
  const int m = warp * 32 + lane;                // accumulator row = TMEM lane of this thread
  const int xi = x0 + (m & 7), yj = y0 + (m >> 3);

  for (int z = z0, it = 0; z < z1; z++, it++) {
    const int r = z - z0 + 1;                    // plane z in slot r % 4
    if (z + 2 <= z1) load_halo<CIN>(halo + ((r + 2) % NSLOT_NN) * L::SLOTB, A.in, A.nx, A.ny, x0, y0,
                                       wrapi(z + 2, A.nz));
    cp_commit();
    cp_wait<1>();                                // planes up to z + 1 have landed
    fence_proxy_async();                         // make them visible to the tensor cores
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const unsigned hb = su32(halo), wb = su32(wsm);
#pragma unroll 1
      for (int t = 0; t < 27; t++) {
        const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
        const unsigned a0 = hb + ((r + dz) % NSLOT_NN) * L::SLOTB + (1 + dy) * L::ROWB + (1 + dx) * 16;
#pragma unroll
        for (int kk = 0; kk < CIN / 16; kk++) {
          const uint64_t ad = smem_desc(a0 + kk * 2 * L::CHB, L::CHB, L::ROWB);
          const uint64_t bd = smem_desc(wb + (t * (CIN / 8) + 2 * kk) * COUT * 16, COUT * 16, 128);
          mma_bf16(tmem, ad, bd, IDESC, t > 0 || kk > 0);
        }
      }
      mma_commit(bar);
    }
    const bool ok = nn_mbar_wait(bar, it & 1);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(A.status, ST_TIMEOUT);
      break;
    }
    tc_fence_after();
    const size_t cell = ((size_t)z * A.ny + yj) * A.nx + xi;
#pragma unroll
    for (int h = 0; h < COUT / 16; h++) {
      float v[16];
      tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + h * 16, v);
      if constexpr (EPI == EPI_LINEAR) {
#pragma unroll
        for (int q = 0; q < 16; q++)
          if (h * 16 + q < A.nout) A.outf[cell * A.nout + h * 16 + q] = v[q] + A.bias[h * 16 + q];
      } else {
        alignas(16) __nv_bfloat16 o[16];
        if constexpr (EPI == EPI_GELU) {
          alignas(16) __nv_bfloat16 zp[16];
#pragma unroll
          for (int q = 0; q < 16; q++) {
            const float zv = v[q] + A.bias[h * 16 + q];
            zp[q] = __float2bfloat16_rn(zv);
            o[q] = __float2bfloat16_rn(gelu(zv));
          }
          if (A.pre) {
            uint4 * dp = reinterpret_cast<uint4 *>(A.pre + cell * COUT + h * 16);
            dp[0] = reinterpret_cast<const uint4 *>(zp)[0];
            dp[1] = reinterpret_cast<const uint4 *>(zp)[1];
          }
        } else {
          alignas(16) __nv_bfloat16 zs[16];
          const uint4 * sp = reinterpret_cast<const uint4 *>(A.zsave + cell * COUT + h * 16);
          reinterpret_cast<uint4 *>(zs)[0] = sp[0];
          reinterpret_cast<uint4 *>(zs)[1] = sp[1];
#pragma unroll
          for (int q = 0; q < 16; q++) o[q] = __float2bfloat16_rn(v[q] * gelu_grad(__bfloat162float(zs[q])));
        }
        uint4 * op = reinterpret_cast<uint4 *>(A.out + cell * COUT + h * 16);
        op[0] = reinterpret_cast<const uint4 *>(o)[0];
        op[1] = reinterpret_cast<const uint4 *>(o)[1];
      }
    }
    tc_fence_before();
    __syncthreads();                             // TMEM and the oldest slot free for the next plane
  }
  cp_wait<0>();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_free(tmem, 32);
}

// ---- weights ---------------------------------------------------------------
// Master weights (FP32) w[t][co][ci], t = 9 (dz+1) + 3 (dy+1) + (dx+1), real
// channel counts cin x cout, into the BF16 shared-memory images of the forward
// convolution, [t][ci/8][co][ci%8] over padded counts CINP x COUTP, and of the
// input-gradient convolution (taps mirrored, channels swapped),
// [26-t][co/8][ci][co%8] over COUTP x CINP. Padding channels are zero.
__global__ void pack_weights_kernel(const float * __restrict__ w, int cin, int cout, int cinp, int coutp,
                                    __nv_bfloat16 * __restrict__ fwd, __nv_bfloat16 * __restrict__ bwd) {
  const int n = 27 * cinp * coutp;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int ci = q % cinp, co = (q / cinp) % coutp, t = q / (cinp * coutp);
    const float v = (ci < cin && co < cout) ? w[((size_t)t * cout + co) * cin + ci] : 0.f;
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    fwd[((size_t)(t * (cinp / 8) + ci / 8) * coutp + co) * 8 + ci % 8] = b;
    if (bwd) bwd[((size_t)((26 - t) * (coutp / 8) + co / 8) * cinp + ci) * 8 + co % 8] = b;
  }
}

template <int CIN, int COUT, int EPI>
int launch_conv3(const ConvArgs & a, cudaStream_t st) {
  using L = ConvLayout<CIN, COUT>;
  if (cudaFuncSetAttribute(conv3_kernel<CIN, COUT, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES) !=
      cudaSuccess)
    return 1;
  const dim3 grid((a.nx / TX) * (a.ny / TY), (a.nz + a.zc - 1) / a.zc);
  conv3_kernel<CIN, COUT, EPI><<<grid, NN_THREADS, L::BYTES, st>>>(a);
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

// z planes per CTA: about four CTAs' worth of work per SM pair
int conv_zchunk(int nx, int ny, int nz) {
  const long cols = (long)(nx / TX) * (ny / TY);
  long zc = cols * nz / (148L * 8);
  if (zc < 1) zc = 1;
  if (zc > nz) zc = nz;
  return (int)zc;
}

}  // namespace
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
  a.nx = nx; a.ny = ny; a.nz = nz; a.zc = conv_zchunk(nx, ny, nz);
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
