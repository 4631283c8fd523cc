// Dense 64x64 complex unitary on the six lowest qubits of a complex64 state, on the
// fifth-generation tensor cores.
//
// The state is viewed as columns of 64 contiguous amplitudes (512 bytes); a tile is 128
// columns.  Per tile, with X^T the tile as a 128 x 128 real matrix (row = column of the
// state, K = interleaved re/im of its 64 amplitudes, exactly the memory order) and W the
// 128 x 128 real form of U (row 2r+q = real/imaginary part of output r):
//     D = X^T W^T,  D[c][2r+q] = (U x_c)_r re/im,
// computed as X_hi W_hi + X_hi W_lo + X_lo W_hi with both operands split into BF16 high and
// low parts (about 16 significant bits each), FP32 accumulation in tensor memory.  Row c of D
// is the new column c in memory order, so each thread stores its column contiguously.
//
// Operands are in shared memory in the canonical K-major layout without swizzle: core
// matrices of 8 rows x 16 bytes, K-chunks 128 B apart, 8-row groups 2048 B apart.  One thread
// per warpgroup issues the MMAs (M=128, N=128, K=16, 8 K-steps x 3 products) and commits them
// to an mbarrier; the warpgroup waits (bounded), reads its accumulator rows with tcgen05.ld and
// stores.  Two warpgroups per block work on alternate tiles (own operand buffer, own TMEM
// columns, own named barrier); W is shared.  Waits are bounded by a time limit; on expiry the
// error word is set and the block frees its tensor memory and returns.
#include <complex>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "kernels.h"
#include "qsim.h"

namespace qsb {

namespace {

constexpr int kWG = 2;                       // warpgroups per block
constexpr int kThreadsTC = 128 * kWG;
constexpr uint32_t kOp = 128 * 128 * 2;      // one BF16 operand (128 rows x 128 K): 32 KiB
constexpr uint32_t kSmemTC = 2 * kOp + kWG * 2 * kOp;  // W hi/lo + per warpgroup X hi/lo = 192 KiB
constexpr uint32_t kTmemCols = 128 * kWG;

__device__ __forceinline__ uint64_t gtime_tc() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// byte offset of (row, K-chunk of 8 BF16) in the canonical K-major layout
__device__ __forceinline__ uint32_t canon(int row, int kchunk) {
  return (uint32_t)((row >> 3) * 2048 + kchunk * 128 + (row & 7) * 16);
}

// shared-memory matrix descriptor: start address, LBO = 128 B, SBO = 2048 B, version 1,
// no swizzle
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)(128u >> 4) << 16;
  d |= (uint64_t)(2048u >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: D FP32, A and B BF16, both K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint64_t limit_ns) {
  const uint64_t t0 = gtime_tc();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (gtime_tc() - t0 > limit_ns) return false;
  }
}

__device__ __forceinline__ void named_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// fp32 -> (bf16 high, bf16 low) pairs packed two per 32-bit word
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(hi) : "f"(b), "f"(a));
  const float ah = __uint_as_float(hi << 16), bh = __uint_as_float(hi & 0xFFFF0000u);
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(lo) : "f"(b - bh), "f"(a - ah));
}

#define TC_LD32(taddr, r)                                                                                    \
  asm volatile(                                                                                            \
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"    \
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                            \
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),     \
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),            \
        "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),          \
        "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),          \
        "=r"(r[29]), "=r"(r[30]), "=r"(r[31])                                                               \
      : "r"(taddr))

__global__ void __launch_bounds__(kThreadsTC, 1)
dense6_tc_kernel(float2* __restrict__ psi, uint64_t ncols, const uint4* __restrict__ wops, unsigned* err,
                 uint64_t limit_ns) {
  extern __shared__ __align__(1024) unsigned char smem_tc[];
  __shared__ __align__(8) uint64_t s_mbar[kWG];
  __shared__ uint32_t s_tmem;
  __shared__ int s_ok[kWG];
  const int t = threadIdx.x;
  const int wg = t >> 7, tl = t & 127, warp = (t >> 5) & 3;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem_tc);
  const uint32_t w_hi = sbase, w_lo = sbase + kOp;
  const uint32_t x_hi = sbase + 2 * kOp + wg * 2 * kOp, x_lo = x_hi + kOp;
  const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&s_mbar[wg]);

  // W (prepared on the host in the canonical layout) -> shared memory
  for (uint32_t i = t; i < 2 * kOp / 16; i += kThreadsTC) reinterpret_cast<uint4*>(smem_tc)[i] = wops[i];
  if (t == 0) {
    for (int g = 0; g < kWG; ++g) {
      const uint32_t mb = (uint32_t)__cvta_generic_to_shared(&s_mbar[g]);
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0 && wg == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(&s_tmem);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem + (uint32_t)(wg * 128);   // this warpgroup's 128 accumulator columns
  const uint64_t ntiles = ncols / 128;
  uint32_t phase = 0;

  for (uint64_t tile = (uint64_t)blockIdx.x * kWG + wg; tile < ntiles; tile += (uint64_t)gridDim.x * kWG) {
    const uint64_t col = tile * 128 + tl;
    float4* cp = reinterpret_cast<float4*>(psi + col * 64);
    // ---- operand X: this thread's column, split into BF16 high / low parts ----
#pragma unroll 4
    for (int j = 0; j < 16; ++j) {
      const float4 v0 = cp[2 * j], v1 = cp[2 * j + 1];
      uint4 h, l;
      split2(v0.x, v0.y, h.x, l.x);
      split2(v0.z, v0.w, h.y, l.y);
      split2(v1.x, v1.y, h.z, l.z);
      split2(v1.z, v1.w, h.w, l.w);
      const uint32_t off = canon(tl, j);
      asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(x_hi + off), "r"(h.x), "r"(h.y), "r"(h.z),
                   "r"(h.w) : "memory");
      asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(x_lo + off), "r"(l.x), "r"(l.y), "r"(l.z),
                   "r"(l.w) : "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    named_sync(1 + wg);
    if (tl == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t ko = (uint32_t)k * 256u;  // two K-chunks per K=16 step
        umma(tmem, sdesc(x_hi + ko), sdesc(w_hi + ko), k > 0 ? 1u : 0u);
        umma(tmem, sdesc(x_hi + ko), sdesc(w_lo + ko), 1u);
        umma(tmem, sdesc(x_lo + ko), sdesc(w_hi + ko), 1u);
      }
      umma_commit(mbar);
    }
    // one thread waits for the MMAs (bounded); the warpgroup follows its verdict
    if (tl == 0) {
      s_ok[wg] = mbar_wait(mbar, phase, limit_ns) ? 1 : 0;
      if (!s_ok[wg]) atomicExch(err, (unsigned)DERR_BARRIER_TIMEOUT);
    }
    phase ^= 1u;
    named_sync(1 + wg);
    if (!s_ok[wg]) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // ---- accumulator row tl (TMEM lane 32*warp + lane) = the new column ----
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t r[32];
      TC_LD32(lane_addr + (uint32_t)(q * 32), r);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int e = 0; e < 8; ++e)
        cp[8 * q + e] = make_float4(__uint_as_float(r[4 * e]), __uint_as_float(r[4 * e + 1]),
                                    __uint_as_float(r[4 * e + 2]), __uint_as_float(r[4 * e + 3]));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    named_sync(1 + wg);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0 && wg == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s_tmem), "r"(kTmemCols) : "memory");
  }
}

}  // namespace

size_t dense6_weight_bytes() { return 2 * kOp; }

// W = real form of U (64x64 complex, row-major), split into BF16 high/low parts, in the
// canonical K-major layout (hi operand then lo operand).
void dense6_prepare_weights(const std::complex<double>* U, uint8_t* out) {
  auto bf16 = [](float f) -> uint16_t {  // round to nearest even (finite inputs)
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
  };
  auto back = [](uint16_t h) -> float {
    const uint32_t u = (uint32_t)h << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  };
  std::memset(out, 0, 2 * kOp);
  for (int n = 0; n < 128; ++n)
    for (int k = 0; k < 128; ++k) {
      const int r = n >> 1, q = n & 1, s = k >> 1, p = k & 1;
      const std::complex<double> u = U[r * 64 + s];
      double w;
      if (q == 0) w = p == 0 ? u.real() : -u.imag();
      else w = p == 0 ? u.imag() : u.real();
      const float f = (float)w;
      const uint16_t hi = bf16(f);
      const uint16_t lo = bf16(f - back(hi));
      const uint32_t off = (uint32_t)((n >> 3) * 2048 + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2);
      std::memcpy(out + off, &hi, 2);
      std::memcpy(out + kOp + off, &lo, 2);
    }
}

cudaError_t launch_dense6_tc(void* psi, int n, const void* d_weights, unsigned* err, uint64_t limit_ns,
                             cudaStream_t s) {
  if (n < 13) return cudaErrorInvalidValue;  // at least one 128-column tile
  cudaError_t e = cudaFuncSetAttribute(dense6_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemTC);
  if (e != cudaSuccess) return e;
  const uint64_t ncols = 1ull << (n - 6);
  const uint64_t tiles = ncols / 128;
  uint64_t grid = (uint64_t)device_sm_count();
  const uint64_t need = (tiles + kWG - 1) / kWG;
  if (grid > need) grid = need;
  dense6_tc_kernel<<<(unsigned)grid, kThreadsTC, kSmemTC, s>>>(reinterpret_cast<float2*>(psi), ncols,
                                                                 reinterpret_cast<const uint4*>(d_weights), err,
                                                                 limit_ns);
  return cudaGetLastError();
}

}  // namespace qsb
