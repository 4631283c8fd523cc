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
// is the new column c in memory order: each thread moves its row into a staging buffer, then
// every warp stores whole 512-byte columns (coalesced).
//
// Operands are in shared memory in the canonical K-major layout without swizzle: core
// matrices of 8 rows x 16 bytes, K-chunks 128 B apart, 8-row groups 2048 B apart.  One thread
// per warpgroup issues the MMAs (M=128, N=128, K=16, 8 K-steps x 3 products) and commits them
// to an mbarrier; after a bounded wait the block reads its accumulator rows with tcgen05.ld.
// One warpgroup (128 threads) per block and SM: while a tile is converted, multiplied and
// written back, the next tile's columns are already on their way into a staging buffer
// (16-byte cp.async, a warp per column: coalesced).  Waits are bounded by a time limit; on
// expiry the error word is set and the block frees its tensor memory and returns.
#include <complex>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

#include "kernels.h"
#include "qsim.h"

namespace qsb {

namespace {

constexpr uint32_t kOp = 128 * 128 * 2;      // one BF16 operand (128 rows x 128 K): 32 KiB

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

// ---- one warpgroup per block; the next tile is staged while this one computes ----
// Shared memory: W hi/lo (64 KiB) | X hi/lo (64 KiB, reused as the output staging) | input
// staging (64 KiB).  Staging rows are 512 B (one state column); 16-byte chunk j of row c sits at
// chunk position j ^ (c & 7), so the per-row accesses of 8 consecutive threads hit distinct banks
// while the per-column copies of a warp stay contiguous (coalesced global loads and stores).
constexpr uint32_t kSmemPipe = 2 * kOp + 2 * kOp + 128 * 512;

__device__ __forceinline__ uint32_t stage_off(int row, int chunk) {
  return (uint32_t)(row * 512 + ((chunk ^ (row & 7)) << 4));
}

__device__ __forceinline__ void cp_async16_tc(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}

__global__ void __launch_bounds__(128, 1)
dense6_tc_pipe_kernel(float2* __restrict__ psi, uint64_t ncols, const uint4* __restrict__ wops, unsigned* err,
                      uint64_t limit_ns) {
  extern __shared__ __align__(1024) unsigned char smem_p[];
  __shared__ __align__(8) uint64_t s_mb;
  __shared__ uint32_t s_tm;
  __shared__ int s_okp;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem_p);
  const uint32_t w_hi = sbase, w_lo = sbase + kOp, x_hi = sbase + 2 * kOp, x_lo = x_hi + kOp;
  const uint32_t stg = sbase + 4 * kOp;
  const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&s_mb);
  const uint64_t ntiles = ncols / 128;
  const float4* src4 = reinterpret_cast<const float4*>(psi);
  float4* dst4 = reinterpret_cast<float4*>(psi);

  for (uint32_t i = t; i < 2 * kOp / 16; i += 128) reinterpret_cast<uint4*>(smem_p)[i] = wops[i];
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(&s_tm);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // stage the first tile: warp w copies columns 32w..32w+31, lane = 16-byte chunk
  auto stage = [&](uint64_t tile) {
    for (int k = 0; k < 32; ++k) {
      const int row = warp * 32 + k;
      cp_async16_tc(stg + stage_off(row, lane), src4 + (tile * 128 + row) * 32 + lane);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  uint64_t tile = blockIdx.x;
  if (tile < ntiles) stage(tile);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tm;
  uint32_t phase = 0;

  for (; tile < ntiles; tile += gridDim.x) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();  // the tile is staged (all threads' copies); D of the previous tile is read
    // ---- convert row t of the staging into the split operand ----
    const unsigned char* sp = smem_p + 4 * kOp;
#pragma unroll 4
    for (int j = 0; j < 16; ++j) {
      const float4 v0 = *reinterpret_cast<const float4*>(sp + stage_off(t, 2 * j));
      const float4 v1 = *reinterpret_cast<const float4*>(sp + stage_off(t, 2 * j + 1));
      uint4 h, l;
      split2(v0.x, v0.y, h.x, l.x);
      split2(v0.z, v0.w, h.y, l.y);
      split2(v1.x, v1.y, h.z, l.z);
      split2(v1.z, v1.w, h.w, l.w);
      const uint32_t off = canon(t, j);
      asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(x_hi + off), "r"(h.x), "r"(h.y), "r"(h.z),
                   "r"(h.w) : "memory");
      asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(x_lo + off), "r"(l.x), "r"(l.y), "r"(l.z),
                   "r"(l.w) : "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // operand complete, staging free
    const uint64_t next = tile + gridDim.x;
    if (next < ntiles) stage(next);
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t ko = (uint32_t)k * 256u;
        umma(tmem, sdesc(x_hi + ko), sdesc(w_hi + ko), k > 0 ? 1u : 0u);
        umma(tmem, sdesc(x_hi + ko), sdesc(w_lo + ko), 1u);
        umma(tmem, sdesc(x_lo + ko), sdesc(w_hi + ko), 1u);
      }
      umma_commit(mbar);
      s_okp = mbar_wait(mbar, phase, limit_ns) ? 1 : 0;
      if (!s_okp) atomicExch(err, (unsigned)DERR_BARRIER_TIMEOUT);
    }
    phase ^= 1u;
    __syncthreads();
    if (!s_okp) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // ---- accumulator row t -> the X buffer as FP32 output staging (same swizzled rows) ----
    unsigned char* op = smem_p + 2 * kOp;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t r[32];
      TC_LD32(lane_addr + (uint32_t)(q * 32), r);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int e = 0; e < 8; ++e)
        *reinterpret_cast<uint4*>(op + stage_off(t, 8 * q + e)) =
            make_uint4(r[4 * e], r[4 * e + 1], r[4 * e + 2], r[4 * e + 3]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // ---- coalesced stores: warp w writes columns 32w..32w+31, lane = 16-byte chunk ----
    for (int k = 0; k < 32; ++k) {
      const int row = warp * 32 + k;
      dst4[(tile * 128 + row) * 32 + lane] = *reinterpret_cast<const float4*>(op + stage_off(row, lane));
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
  }
}

// ---- six arbitrary positions B: a tile is 2^13 amplitudes over T = B + the 7 lowest other bits ----
// Local index l (13 bits over T ascending) -> row (its bits outside B, 0..127) and j (its bits in
// B, 0..63).  T holds physical bits 0..6 (every bit below 7 is in B or among the 7 lowest others),
// so 128 consecutive l are 1 KiB of contiguous memory: lane-consecutive 8-byte copies coalesce.
// Per amplitude, the global offset and the staging byte (row * 512 + swizzled 16-byte chunk of j)
// are XOR-linear in l, so each is tab_lo[l & 127] ^ tab_hi[l >> 7] (tables in the weights buffer).
struct GatherTabs {
  uint64_t src_lo[128];  // deposit(l, T) for l < 128
  uint64_t src_hi[64];   // deposit(l << 7, T)
  uint32_t dst_lo[128];  // staging byte of l < 128
  uint32_t dst_hi[64];   // staging byte of l << 7
  // pairs (physical bit 0 in B: amplitudes 2p and 2p + 1 are adjacent in memory and in a row):
  uint64_t psrc_lo[128];  // deposit(2 p, T) for p < 128
  uint64_t psrc_hi[32];   // deposit(p << 8, T)
  uint32_t pdst_lo[128];
  uint32_t pdst_hi[32];
  int32_t upos[64];      // physical bits outside T, ascending (the tile index's bits)
  int32_t nu;
  int32_t pairs;         // 1: physical bit 0 is in B (16-byte copies)
  int32_t pad[2];
};

__device__ __forceinline__ void cp_async8_tc(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}

template <bool kPairs>
__global__ void __launch_bounds__(128, 1)
dense6_tc_gather_kernel(float2* __restrict__ psi, uint64_t ntiles, const uint4* __restrict__ wops,
                        const GatherTabs* __restrict__ tabs, unsigned* err, uint64_t limit_ns) {
  extern __shared__ __align__(1024) unsigned char smem_g[];
  __shared__ __align__(8) uint64_t s_mb;
  __shared__ uint32_t s_tm;
  __shared__ int s_okg;
  __shared__ uint64_t s_hi[64];
  __shared__ uint32_t s_dhi[64];
  const int t = threadIdx.x, warp = t >> 5;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem_g);
  const uint32_t w_hi = sbase, w_lo = sbase + kOp, x_hi = sbase + 2 * kOp, x_lo = x_hi + kOp;
  const uint32_t stg = sbase + 4 * kOp;
  const uint32_t mbar = (uint32_t)__cvta_generic_to_shared(&s_mb);
  constexpr int kItems = kPairs ? 32 : 64;  // copies per thread per tile
  const uint64_t my_src = kPairs ? tabs->psrc_lo[t] : tabs->src_lo[t];
  const uint32_t my_dst = kPairs ? tabs->pdst_lo[t] : tabs->dst_lo[t];
  const int nu = tabs->nu;

  for (uint32_t i = t; i < 2 * kOp / 16; i += 128) reinterpret_cast<uint4*>(smem_g)[i] = wops[i];
  if (t < kItems) {
    s_hi[t] = kPairs ? tabs->psrc_hi[t] : tabs->src_hi[t];
    s_dhi[t] = kPairs ? tabs->pdst_hi[t] : tabs->dst_hi[t];
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(&s_tm);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(128)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  auto base_of = [&](uint64_t tile) {
    uint64_t b = 0;
    for (int k = 0; k < nu; ++k)
      if ((tile >> k) & 1ull) b |= 1ull << tabs->upos[k];
    return b;
  };
  // amplitude l = 128 i + t (pair 2 (128 i + t) with kPairs) of the tile: lanes take consecutive
  // l (coalesced)
  auto stage = [&](uint64_t tile) {
    const uint64_t b = base_of(tile) | my_src;
    for (int i = 0; i < kItems; ++i) {
      if constexpr (kPairs) cp_async16_tc(stg + (my_dst ^ s_dhi[i]), psi + (b | s_hi[i]));
      else cp_async8_tc(stg + (my_dst ^ s_dhi[i]), psi + (b | s_hi[i]));
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  uint64_t tile = blockIdx.x;
  if (tile < ntiles) stage(tile);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tm;
  uint32_t phase = 0;

  for (; tile < ntiles; tile += gridDim.x) {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const unsigned char* sp = smem_g + 4 * kOp;
#pragma unroll 4
    for (int j = 0; j < 16; ++j) {
      const float4 v0 = *reinterpret_cast<const float4*>(sp + stage_off(t, 2 * j));
      const float4 v1 = *reinterpret_cast<const float4*>(sp + stage_off(t, 2 * j + 1));
      uint4 h, l;
      split2(v0.x, v0.y, h.x, l.x);
      split2(v0.z, v0.w, h.y, l.y);
      split2(v1.x, v1.y, h.z, l.z);
      split2(v1.z, v1.w, h.w, l.w);
      const uint32_t off = canon(t, j);
      asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(x_hi + off), "r"(h.x), "r"(h.y), "r"(h.z),
                   "r"(h.w) : "memory");
      asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(x_lo + off), "r"(l.x), "r"(l.y), "r"(l.z),
                   "r"(l.w) : "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    const uint64_t next = tile + gridDim.x;
    const uint64_t cur_base = base_of(tile) | my_src;
    if (next < ntiles) stage(next);
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t ko = (uint32_t)k * 256u;
        umma(tmem, sdesc(x_hi + ko), sdesc(w_hi + ko), k > 0 ? 1u : 0u);
        umma(tmem, sdesc(x_hi + ko), sdesc(w_lo + ko), 1u);
        umma(tmem, sdesc(x_lo + ko), sdesc(w_hi + ko), 1u);
      }
      umma_commit(mbar);
      s_okg = mbar_wait(mbar, phase, limit_ns) ? 1 : 0;
      if (!s_okg) atomicExch(err, (unsigned)DERR_BARRIER_TIMEOUT);
    }
    phase ^= 1u;
    __syncthreads();
    if (!s_okg) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    unsigned char* op = smem_g + 2 * kOp;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t r[32];
      TC_LD32(lane_addr + (uint32_t)(q * 32), r);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int e = 0; e < 8; ++e)
        *reinterpret_cast<uint4*>(op + stage_off(t, 8 * q + e)) =
            make_uint4(r[4 * e], r[4 * e + 1], r[4 * e + 2], r[4 * e + 3]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // scattered 8- or 16-byte stores, lane-consecutive amplitudes (coalesced)
    for (int i = 0; i < kItems; ++i) {
      if constexpr (kPairs)
        *reinterpret_cast<float4*>(psi + (cur_base | s_hi[i])) = *reinterpret_cast<const float4*>(op + (my_dst ^ s_dhi[i]));
      else
        psi[cur_base | s_hi[i]] = *reinterpret_cast<const float2*>(op + (my_dst ^ s_dhi[i]));
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128) : "memory");
  }
}

}  // namespace

size_t dense6_gather_bytes() { return sizeof(GatherTabs); }

// Tables of the gather kernel for the six physical bits B (ascending).  Returns false when the
// state is too small (fewer than 13 bits).
bool dense6_gather_tables(int n, const int* B, uint8_t* out) {
  if (n < 13) return false;
  GatherTabs g;
  std::memset(&g, 0, sizeof(g));
  bool inB[64] = {};
  for (int q = 0; q < 6; ++q) inB[B[q]] = true;
  int T[13], nt = 0, other = 0;
  for (int p = 0; p < n; ++p) {
    if (inB[p]) T[nt++] = p;
    else if (other < 7) { T[nt++] = p; ++other; }
    else g.upos[g.nu++] = p;
  }
  // within T (ascending): which bits are B (j bits, in order) and which are row bits
  auto split = [&](uint32_t l, uint64_t* phys, uint32_t* byte) {
    uint64_t ph = 0;
    uint32_t row = 0, j = 0;
    int jr = 0, rr = 0;
    for (int b = 0; b < 13; ++b) {
      const uint32_t v = (l >> b) & 1u;
      if (v) ph |= 1ull << T[b];
      if (inB[T[b]]) j |= v << jr++;
      else row |= v << rr++;
    }
    *phys = ph;
    *byte = row * 512u + ((((j >> 1) ^ (row & 7u)) & 31u) << 4) + ((j & 1u) << 3);
  };
  for (uint32_t l = 0; l < 128; ++l) split(l, &g.src_lo[l], &g.dst_lo[l]);
  for (uint32_t i = 0; i < 64; ++i) split(i << 7, &g.src_hi[i], &g.dst_hi[i]);
  g.pairs = inB[0] ? 1 : 0;  // physical bit 0 is then T's and B's lowest: j bit 0
  for (uint32_t p = 0; p < 128; ++p) split(2 * p, &g.psrc_lo[p], &g.pdst_lo[p]);
  for (uint32_t i = 0; i < 32; ++i) split(i << 8, &g.psrc_hi[i], &g.pdst_hi[i]);
  std::memcpy(out, &g, sizeof(g));
  return true;
}

cudaError_t launch_dense6_tc_gather(void* psi, int n, const void* d_weights, const void* d_tabs, bool pairs,
                                    unsigned* err, uint64_t limit_ns, cudaStream_t s) {
  if (n < 13) return cudaErrorInvalidValue;
  auto kern = pairs ? dense6_tc_gather_kernel<true> : dense6_tc_gather_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemPipe);
  if (e != cudaSuccess) return e;
  const uint64_t tiles = 1ull << (n - 13);
  uint64_t grid = (uint64_t)device_sm_count();
  if (grid > tiles) grid = tiles;
  kern<<<(unsigned)grid, 128, kSmemPipe, s>>>(reinterpret_cast<float2*>(psi), tiles,
                                              reinterpret_cast<const uint4*>(d_weights),
                                              reinterpret_cast<const GatherTabs*>(d_tabs), err, limit_ns);
  return cudaGetLastError();
}

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
  if (n < 13) return cudaErrorInvalidValue;
  cudaError_t e =
      cudaFuncSetAttribute(dense6_tc_pipe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemPipe);
  if (e != cudaSuccess) return e;
  const uint64_t ncols = 1ull << (n - 6);
  const uint64_t tiles = ncols / 128;
  uint64_t grid = (uint64_t)device_sm_count();
  if (grid > tiles) grid = tiles;
  dense6_tc_pipe_kernel<<<(unsigned)grid, 128, kSmemPipe, s>>>(reinterpret_cast<float2*>(psi), ncols,
                                                               reinterpret_cast<const uint4*>(d_weights), err,
                                                               limit_ns);
  return cudaGetLastError();
}

}  // namespace qsb
