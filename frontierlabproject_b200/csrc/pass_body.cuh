// Device code of a pass (sweep), shared by the generic pass kernel (kern_pass.cu, nvcc)
// and the specialised kernels generated at plan time (jit.cpp, NVRTC).
//
// Per group (one value of the group bits) a team of 256 threads:
//   load   16-byte cp.async copies -> swizzled shared memory;
//   phases each thread reads its 2^LR amplitudes (the phase's register bits) from shared
//          memory, the Exec policy applies the phase's gates in registers, writes back;
//   store  shared memory -> 16-byte coalesced global stores, optionally through a bit
//          permutation of the local bits (in-place permutation passes).
// Two schedules:
//   pass_body        one team per block; either two group buffers (the next group's copies
//                    are in flight while the current group is processed) or one buffer and
//                    two resident blocks per SM.  Several passes in one launch (cooperative
//                    mode) are separated by a grid barrier whose wait is bounded.
//   pass_body_teams  two teams per block over three group buffers: slot s of the block's
//                    groups is processed by team s & 1 in buffer s % 3, and the team that
//                    finishes slot s copies slot s + 3 (the other team's) into the buffer it
//                    has just freed.  Copies are tracked by one mbarrier per buffer; every
//                    wait is bounded (error word set, the team returns).
#pragma once
#include "qsim.h"

namespace qsb {

template <typename Real> struct V2;
template <> struct V2<float> { using T = float2; };
template <> struct V2<double> { using T = double2; };

template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// a*x + b*y
template <typename C> __device__ __forceinline__ C cmac2(C a, C x, C b, C y) {
  C r;
  r.x = a.x * x.x - a.y * x.y + b.x * y.x - b.y * y.y;
  r.y = a.x * x.y + a.y * x.x + b.x * y.y + b.y * y.x;
  return r;
}

// Opaque to the optimiser: forces a value to be recomputed / a pointer to be re-read
// instead of keeping derived values live across the gate code.
__device__ __forceinline__ void opaque(uint32_t& x) { asm volatile("" : "+r"(x)); }
__device__ __forceinline__ void opaque(uint64_t& x) { asm volatile("" : "+l"(x)); }
template <typename T> __device__ __forceinline__ const T* opaque_ptr(const T* p) {
  asm volatile("" : "+l"(p));
  return p;
}

template <typename Real> __device__ __forceinline__ uint32_t swz(uint32_t l);
template <> __device__ __forceinline__ uint32_t swz<float>(uint32_t l) { return swz64(l); }
template <> __device__ __forceinline__ uint32_t swz<double>(uint32_t l) { return swz128(l); }

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bar[0] = arrivals, bar[1] = generation.  Returns false when the wait gave up (the
// error word is set; every block then leaves the kernel).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned* err, uint64_t limit_ns) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned* vgen = bar + 1;
    const unsigned gen = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const uint64_t t0 = global_ns();
      while (*vgen == gen) {
        if (*(volatile unsigned*)err != 0u) { ok = 0; break; }
        if (global_ns() - t0 > limit_ns) { atomicExch(err, (unsigned)DERR_BARRIER_TIMEOUT); ok = 0; break; }
        __nanosleep(100);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// physical offset of the local index l (deposit of l's bits onto the staged bits)
__device__ __forceinline__ uint64_t phys_of_local(uint32_t l, const int8_t* sbit, int m) {
  uint64_t q = 0;
  for (int j = 0; j < m; ++j) if ((l >> j) & 1u) q |= 1ull << sbit[j];
  return q;
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---- mbarriers (shared::cta) tracking cp.async copies ----
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// the barrier's pending count drops by one when all of this thread's earlier cp.async copies
// have completed (the barrier is initialised with one count per arriving thread)
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// non-blocking: true when the phase of the given parity has completed (acquire)
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for a phase: false (error word set unless another wait already set it) when
// the limit expired or another part of the grid reported an error.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned* err, uint64_t limit_ns) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try(bar, parity)) {
    if (err && *(volatile unsigned*)err != 0u) return false;
    if (global_ns() - t0 > limit_ns) {
      if (err) atomicCAS(err, 0u, (unsigned)DERR_LOAD_TIMEOUT);
      return false;
    }
  }
  return true;
}
__device__ __forceinline__ void named_barrier(unsigned id, unsigned nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

constexpr int kPassThreads = 256;
// load/store item rows per thread and group: 2^(r - 1) for complex64 (16-byte pairs), 2^r for
// complex128; r <= 6 (complex64) and r <= 4 (complex128) keep it within 32
constexpr int kMaxItems = 32;
static_assert(kMaxItems >= (1 << (kMaxR - 1)), "item tables too small for the register bits");

// Issue the asynchronous load of the group with physical base `gbase` into the shared buffer
// `buf` (16-byte copies, swizzled destinations).  Items: c64 -> two amplitudes (local bit 0
// inside the vector), c128 -> one amplitude.  `tbase` = physical offset of thread t's first
// item.  kUnroll = false: one copy's address at a time (few registers, for copies issued while
// a phase holds its amplitudes).
template <typename Real, bool kUnroll = true>
__device__ __forceinline__ void prefetch_group(typename V2<Real>::T* buf, const typename V2<Real>::T* psi,
                                               uint64_t gbase, uint64_t tbase, const uint64_t* pv, int T, int V,
                                               unsigned t) {
  constexpr int kItemBits = sizeof(Real) == 4 ? 1 : 0;
  if ((int)t >= T) return;
  const uint32_t lt = (uint32_t)t << kItemBits;
  const uint64_t base = gbase | tbase;
#pragma unroll(kUnroll ? kMaxItems : 1)
  for (int v = 0; v < kMaxItems; ++v) {
    if (v >= V) break;
    const uint32_t l = lt | (((uint32_t)v * (uint32_t)T) << kItemBits);
    cp_async16(buf + swz<Real>(l), psi + (base | pv[v]));
  }
}

// Group index -> physical base: five 7-bit levels of the deposit of g onto the group bits.
__device__ __forceinline__ uint64_t gbase_of(uint64_t g, const uint64_t* gtab) {
  return gtab[g & 127] | gtab[128 + ((g >> 7) & 127)] | gtab[256 + ((g >> 14) & 127)] |
         gtab[384 + ((g >> 21) & 127)] | gtab[512 + ((g >> 28) & 127)];
}

constexpr int kPhaseTab = 32;   // phases per pass whose thread bases are tabulated

// Loads (store = false) or stores the thread's 2^LR registers of a phase: register i at byte
// sb8 ^ (XOR of B8[j] over the set bits j of i).  JR >= 0 (complex64): register bit JR holds
// local bit 0, so registers i and i | 2^JR are adjacent and move as one 16-byte access (the
// phase's lanes then span distinct 16-byte slots: no bank conflicts); swap stores the two
// halves exchanged (local bit 0 left flipped by the phase).
template <typename C, int LR, int JR>
__device__ __forceinline__ void regs_io_j(C (&a)[1 << LR], unsigned char* sm, uint32_t sb8, const uint32_t (&B8)[LR],
                                          bool store, bool swap) {
#pragma unroll
  for (int i = 0; i < (1 << LR); ++i) {
    if (JR >= 0 && ((i >> JR) & 1)) continue;
    uint32_t s = sb8;
#pragma unroll
    for (int j = 0; j < LR; ++j)
      if (j != JR && ((i >> j) & 1)) s ^= B8[j];
    if constexpr (JR >= 0) {
      constexpr int i1 = 1 << (JR < 0 ? 0 : JR);
      float4* q = reinterpret_cast<float4*>(sm + s);
      if (store) {
        const C lo = swap ? a[i | i1] : a[i], hi = swap ? a[i] : a[i | i1];
        *q = make_float4(lo.x, lo.y, hi.x, hi.y);
      } else {
        const float4 v = *q;
        a[i].x = v.x; a[i].y = v.y;
        a[i | i1].x = v.z; a[i | i1].y = v.w;
      }
    } else {
      C* q = reinterpret_cast<C*>(sm + s);
      if (store) *q = a[i];
      else a[i] = *q;
    }
  }
}

// run-time choice of JR in [J, LR) (or -1)
template <typename C, int LR, int J>
__device__ __forceinline__ void regs_io(int jr, C (&a)[1 << LR], unsigned char* sm, uint32_t sb8,
                                        const uint32_t (&B8)[LR], bool store, bool swap) {
  if constexpr (J < LR && sizeof(C) == 8) {
    if (jr == J) { regs_io_j<C, LR, J>(a, sm, sb8, B8, store, swap); return; }
    regs_io<C, LR, J + 1>(jr, a, sm, sb8, B8, store, swap);
  } else {
    regs_io_j<C, LR, -1>(a, sm, sb8, B8, store, swap);
  }
}

// Packed registers (complex64, register bit 0 = local bit 0): R[q] holds the real parts and
// I[q] the imaginary parts of registers 2q and 2q + 1, so one packed FP32x2 instruction
// updates two amplitudes.  Shared memory then holds every 16-byte pair split,
// {re(2q), re(2q + 1), im(2q), im(2q + 1)}, except the group as copied from global memory
// (interleaved, read by a pass's first phase).  swap stores the two lanes exchanged (local
// bit 0 left flipped by the phase).
template <int LR>
__device__ __forceinline__ void packed_load(float2 (&R)[1 << (LR - 1)], float2 (&I)[1 << (LR - 1)],
                                            const unsigned char* sm, uint32_t sb8, const uint32_t (&B8)[LR],
                                            bool interleaved) {
#pragma unroll
  for (int q = 0; q < (1 << (LR - 1)); ++q) {
    uint32_t s = sb8;
#pragma unroll
    for (int j = 1; j < LR; ++j)
      if ((q >> (j - 1)) & 1) s ^= B8[j];
    const float4 v = *reinterpret_cast<const float4*>(sm + s);
    if (interleaved) {
      R[q] = make_float2(v.x, v.z);
      I[q] = make_float2(v.y, v.w);
    } else {
      R[q] = make_float2(v.x, v.y);
      I[q] = make_float2(v.z, v.w);
    }
  }
}
template <int LR>
__device__ __forceinline__ void packed_store(const float2 (&R)[1 << (LR - 1)], const float2 (&I)[1 << (LR - 1)],
                                             unsigned char* sm, uint32_t sb8, const uint32_t (&B8)[LR], bool swap) {
#pragma unroll
  for (int q = 0; q < (1 << (LR - 1)); ++q) {
    uint32_t s = sb8;
#pragma unroll
    for (int j = 1; j < LR; ++j)
      if ((q >> (j - 1)) & 1) s ^= B8[j];
    *reinterpret_cast<float4*>(sm + s) =
        swap ? make_float4(R[q].y, R[q].x, I[q].y, I[q].x) : make_float4(R[q].x, R[q].y, I[q].x, I[q].y);
  }
}

// Index deposits that do not change within a pass, tabulated in shared memory once per pass:
// group index -> physical base, thread index -> local / physical base per phase, per-thread
// load base and store-permutation source.
struct PassShared {
  uint64_t gtab[5 * 128];        // group index -> physical base (5 levels x 7 bits)
  uint64_t pt[kPhaseTab * 48];   // per phase: physical thread base, t bits 0-3 | 4-8
  uint64_t base[512];            // per thread: physical offset of its first item
  uint64_t pv[kMaxItems];        // physical offset of load/store item row v
  uint32_t lt[kPhaseTab * 48];   // per phase: local thread base
  uint32_t stt[512];             // per thread: store-permutation source of its first item
  uint32_t sv[kMaxItems];        // store-permutation source local offset of row v
  PassDesc pd;
};

// Fills the tables of pass p (all threads of the block; ends with a block barrier).
template <typename Real>
__device__ __forceinline__ void pass_setup(PassShared& sh, const uint8_t* __restrict__ prog, int p) {
  constexpr int kItemBits = sizeof(Real) == 4 ? 1 : 0;
  const int t = (int)threadIdx.x, nthr = (int)blockDim.x;
  const ProgramHeader* hdr = reinterpret_cast<const ProgramHeader*>(prog);
  if (t == 0) sh.pd = reinterpret_cast<const PassDesc*>(prog + hdr->off_pass)[p];
  __syncthreads();
  const PassDesc& pd = sh.pd;
  const int m = pd.m;
  const int T = 1 << (m - pd.r);                    // active threads of this pass (per team)
  const int V = 1 << (m - kItemBits) >> (m - pd.r);  // items per thread (<= kMaxItems)
  const int nt = m - pd.r;                           // thread-index bits
  for (int v = t; v < V; v += nthr) {
    const uint32_t lv = ((uint32_t)v * (uint32_t)T) << kItemBits;
    uint64_t q = 0;
    uint32_t s = 0;
    for (int j = 0; j < m; ++j)
      if ((lv >> j) & 1u) {
        q |= 1ull << pd.sbit[j];
        if (pd.store_perm) s |= 1u << pd.store_src[j];
      }
    sh.pv[v] = q;
    sh.sv[v] = s;
  }
  for (int e = t; e < 5 * 128; e += nthr) {
    const int level = e >> 7, idx = e & 127;
    uint64_t v = 0;
    for (int j = 0; j < 7; ++j) {
      const int gb = 7 * level + j;
      if (gb < pd.ngbits && ((idx >> j) & 1)) v |= 1ull << pd.gbit[gb];
    }
    sh.gtab[e] = v;
  }
  const int nph_tab = pd.nphase < kPhaseTab ? pd.nphase : kPhaseTab;
  for (int e = t; e < nph_tab * 48; e += nthr) {
    const int h = e / 48, k = e % 48;
    const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(prog + hdr->off_phase) + pd.phase0 + h;
    const int lo = k < 16 ? 0 : 4, val = k < 16 ? k : k - 16, nb = k < 16 ? 4 : 5;
    uint32_t lt = 0;
    uint64_t pt = 0;
    for (int b = 0; b < nb; ++b) {
      const int j = lo + b;
      if (j < nt && ((val >> b) & 1)) {
        lt |= 1u << ph->tbit[j];
        pt |= 1ull << pd.sbit[ph->tbit[j]];
      }
    }
    sh.lt[e] = lt;
    sh.pt[e] = pt;
  }
  for (int u = t; u < T; u += nthr) {
    const uint32_t l = (uint32_t)u << kItemBits;
    sh.base[u] = phys_of_local(l, pd.sbit, m);
    uint32_t st = 0;
    if (pd.store_perm)
      for (int j = 0; j < m; ++j) if ((l >> j) & 1u) st |= 1u << pd.store_src[j];
    sh.stt[u] = st;
  }
  __syncthreads();
}

// ex.run(prog, ph, pass, h, a, pb) applies the gates of phase h of pass `pass` to the
// thread's registers a[] (pb = physical index of the thread's register-0 amplitude) and
// returns the local bits left flipped in the registers (the write-back lands at the
// flipped addresses); ex.reg_offsets(ph, h, B8) gives the swizzled byte offset of each
// register bit of phase h.
//
// Phase h of one group in the buffer at byte `bsel` (buffers start one bit above every
// swizzled byte offset of a group, so addresses are XOR combinations indexing smem_raw
// directly).  t: thread index within the team (an active thread of the pass); *gbp: physical
// base of the group (shared).
template <typename Real, int LR, typename Exec>
__device__ __forceinline__ void group_phase(const Exec& ex, const uint8_t* __restrict__ prog, const PassShared& sh,
                                            int p, int h, uint32_t bsel, const uint64_t* gbp, unsigned t) {
  using C = typename V2<Real>::T;
  constexpr int NR = 1 << LR;
  constexpr bool kC64 = sizeof(Real) == 4;
  constexpr uint32_t kEsz = sizeof(C);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const ProgramHeader* hdr = reinterpret_cast<const ProgramHeader*>(prog);
  const PassDesc& pd = sh.pd;
  const int nt = pd.m - pd.r;
  const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(prog + hdr->off_phase) + pd.phase0 + h;
  uint32_t sb;
  uint64_t pb = *gbp;
  if (h < kPhaseTab) {
    const int e0 = h * 48 + (int)(t & 15u), e1 = h * 48 + 16 + (int)((t >> 4) & 31u);
    sb = swz<Real>(sh.lt[e0] | sh.lt[e1]);
    pb |= sh.pt[e0] | sh.pt[e1];
  } else {
    uint32_t lb = 0;
    for (int j = 0; j < nt; ++j)
      if ((t >> j) & 1u) { lb |= 1u << ph->tbit[j]; pb |= 1ull << pd.sbit[ph->tbit[j]]; }
    sb = swz<Real>(lb);
  }
  uint32_t sb8 = bsel ^ (sb * kEsz);
  uint32_t B8[LR];  // byte offset of register bit j (swizzled)
  ex.template reg_offsets<Real, LR>(ph, h, B8);
  if constexpr (Exec::kPacked) {
    float2 R[NR / 2], I[NR / 2];
    if (h == 0) packed_load<LR>(R, I, smem_raw, sb8, B8, true);
    else packed_load<LR>(R, I, smem_raw, sb8, B8, false);
    const uint32_t fl = ex.template run_packed<LR>(prog, h, R, I, pb);
    sb8 ^= swz<Real>(fl & ~1u) * kEsz;
    opaque(sb8);
#pragma unroll
    for (int j = 0; j < LR; ++j) opaque(B8[j]);
    if (fl & 1u) packed_store<LR>(R, I, smem_raw, sb8, B8, true);  // warp-uniform
    else packed_store<LR>(R, I, smem_raw, sb8, B8, false);
  } else {
    // register bit holding local bit 0 (complex64): its pairs are 16-byte accesses
    const int jr = kC64 ? ex.template pair_reg<LR>(ph, h) : -1;
    C a[NR];
    regs_io<C, LR, 0>(jr, a, smem_raw, sb8, B8, false, false);
    // fl: local bits whose values the phase left flipped in the registers
    const uint32_t fl = ex.template run<C, LR>(prog, ph, p, h, a, pb);
    // a flipped local bit 0 swaps the halves of each 16-byte pair instead
    const bool swap_pairs = jr >= 0 && (fl & 1u);
    sb8 ^= swz<Real>(jr >= 0 ? (fl & ~1u) : fl) * kEsz;
    opaque(sb8);
#pragma unroll
    for (int j = 0; j < LR; ++j) opaque(B8[j]);
    if (swap_pairs) regs_io<C, LR, 0>(jr, a, smem_raw, sb8, B8, true, true);  // warp-uniform
    else regs_io<C, LR, 0>(jr, a, smem_raw, sb8, B8, true, false);
  }
}

// All phases of one group; bar(): the team's barrier, after every phase.  NPH > 0: the pass's
// phase count, known when the kernel is compiled (the loop unrolls, and the phase index, its
// register offsets and its gate code become constants).
template <typename Real, int LR, typename Exec, int NPH, typename Bar>
__device__ __forceinline__ void group_phases(const Exec& ex, const uint8_t* __restrict__ prog, const PassShared& sh,
                                             int p, uint32_t bsel, const uint64_t* gbp, unsigned t, const Bar& bar) {
  const bool active = (int)t < (1 << (sh.pd.m - sh.pd.r));
  if constexpr (NPH > 0) {
#pragma unroll
    for (int h = 0; h < NPH; ++h) {
      if (active) group_phase<Real, LR>(ex, prog, sh, p, h, bsel, gbp, t);
      bar();
    }
  } else {
    for (int h = 0; h < sh.pd.nphase; ++h) {
      if (active) group_phase<Real, LR>(ex, prog, sh, p, h, bsel, gbp, t);
      bar();
    }
  }
}

// Coalesced global store of the group in the buffer at byte `bsel` (thread t of the team).
// kSplit: the buffer holds split 16-byte pairs (packed kernels; no store permutation).
template <typename Real, bool kSplit = false>
__device__ __forceinline__ void group_store(const PassShared& sh, typename V2<Real>::T* __restrict__ psi,
                                            uint32_t bsel, uint64_t gb, unsigned t) {
  using C = typename V2<Real>::T;
  constexpr bool kC64 = sizeof(Real) == 4;
  constexpr int kItemBits = kC64 ? 1 : 0;
  constexpr uint32_t kEsz = sizeof(C);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto at = [&](uint32_t byte) -> const C& { return *reinterpret_cast<const C*>(smem_raw + byte); };
  const PassDesc& pd = sh.pd;
  const int m = pd.m;
  const int T = 1 << (m - pd.r);
  const int V = 1 << (m - kItemBits) >> (m - pd.r);
  if ((int)t >= T) return;
  const uint32_t lt = (uint32_t)t << kItemBits;
  const uint64_t base = gb | sh.base[t];
  const uint32_t stt = sh.stt[t];
  if constexpr (kC64) {
#pragma unroll
    for (int v = 0; v < kMaxItems; ++v) {
      if (v >= V) break;
      float4 val;
      if (pd.store_perm) {
        const uint32_t s0 = stt | sh.sv[v];
        const uint32_t s1 = s0 ^ (1u << pd.store_src[0]);
        const C x0 = at(bsel ^ (swz<Real>(s0) * kEsz)), x1 = at(bsel ^ (swz<Real>(s1) * kEsz));
        val = make_float4(x0.x, x0.y, x1.x, x1.y);
      } else {
        const uint32_t l = lt | (((uint32_t)v * (uint32_t)T) << 1);
        val = *reinterpret_cast<const float4*>(smem_raw + (bsel ^ (swz<Real>(l) * kEsz)));
        if (kSplit) val = make_float4(val.x, val.z, val.y, val.w);
      }
      __stcg(reinterpret_cast<float4*>(psi + (base | sh.pv[v])), val);
    }
  } else {
#pragma unroll
    for (int v = 0; v < kMaxItems; ++v) {
      if (v >= V) break;
      const uint32_t l = lt | ((uint32_t)v * (uint32_t)T);
      const uint32_t src = pd.store_perm ? (stt | sh.sv[v]) : l;
      __stcg(psi + (base | sh.pv[v]), at(bsel ^ (swz<Real>(src) * kEsz)));
    }
  }
}

// One team per block.  kDouble: two group buffers per block (the next group's copies overlap
// this group's phases); otherwise one buffer and two resident blocks per SM overlap each
// other.
template <typename Real, int LR, typename Exec, bool kDouble = true, int NPH = 0>
__device__ __forceinline__ void pass_body(const Exec& ex, const uint8_t* __restrict__ prog,
                                          typename V2<Real>::T* __restrict__ psi,
                                          int pass_begin, int pass_end, unsigned* bar, unsigned* err,
                                          uint64_t barrier_limit_ns) {
  using C = typename V2<Real>::T;
  constexpr int kItemBits = sizeof(Real) == 4 ? 1 : 0;
  constexpr uint32_t kEsz = sizeof(C);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PassShared sh;
  __shared__ uint64_t s_gb[2];                 // physical base of the current group
  const unsigned t = threadIdx.x;
  auto block_bar = [] { __syncthreads(); };

  for (int p = pass_begin; p < pass_end; ++p) {
    if (p > pass_begin) {
      if (!grid_barrier(bar, err, barrier_limit_ns)) return;
    }
    pass_setup<Real>(sh, prog, p);
    const int m = sh.pd.m;
    const int T = 1 << (m - sh.pd.r);
    const int V = 1 << (m - kItemBits) >> (m - sh.pd.r);
    const uint64_t ngroups = 1ull << sh.pd.ngbits;
    const uint64_t tbase = (int)t < T ? sh.base[t] : 0ull;
    const uint32_t buf1 = kDouble ? (kEsz << m) : 0u;

    uint64_t g = blockIdx.x;
    if (kDouble) {
      if (g < ngroups)
        prefetch_group<Real>(reinterpret_cast<C*>(smem_raw), psi, gbase_of(g, sh.gtab), tbase, sh.pv, T, V, t);
      cp_async_commit();
    }
    for (int it = 0; g < ngroups; g += gridDim.x, ++it) {
      const uint32_t bsel = (it & 1) ? buf1 : 0u;  // byte offset of this group's buffer
      if (t == 0) s_gb[it & 1] = gbase_of(g, sh.gtab);  // read after the barrier below
      if (kDouble) {
        const uint64_t gn = g + gridDim.x;
        if (gn < ngroups)
          prefetch_group<Real>(reinterpret_cast<C*>(smem_raw + (bsel ^ buf1)), psi, gbase_of(gn, sh.gtab), tbase,
                               sh.pv, T, V, t);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        prefetch_group<Real>(reinterpret_cast<C*>(smem_raw), psi, gbase_of(g, sh.gtab), tbase, sh.pv, T, V, t);
        cp_async_commit();
        cp_async_wait<0>();
      }
      __syncthreads();
      group_phases<Real, LR, Exec, NPH>(ex, prog, sh, p, bsel, &s_gb[it & 1], t, block_bar);
      group_store<Real, Exec::kPacked>(sh, psi, bsel, s_gb[it & 1], t);
      __syncthreads();
    }
    cp_async_wait<0>();
    __syncthreads();
  }
}

// Last phase of a group (complex64, interleaved registers), stored from registers straight to
// global memory: once the phase's loads are done every thread of the block has read the
// buffer, so next() (the copies of the block's next group) is issued before the gates run, and
// the copies overlap the gate arithmetic and the stores.  Every thread of the block is an
// active thread of the pass (one block barrier inside).  ex.phys_offsets(h, P, L): physical
// offset (in amplitudes) of register bit j and the local bit it holds.  Register i, left
// holding the amplitude of register index i ^ (flipped bits), is written there.
template <typename Real, int LR, typename Exec, typename Bar, typename Next>
__device__ __forceinline__ void group_phase_direct(const Exec& ex, const uint8_t* __restrict__ prog,
                                                   const PassShared& sh, int p, int h, uint32_t bsel,
                                                   const uint64_t* gbp, unsigned t,
                                                   typename V2<Real>::T* __restrict__ psi, const Bar& bar,
                                                   const Next& next) {
  static_assert(sizeof(Real) == 4, "complex64 only");
  using C = float2;
  constexpr int NR = 1 << LR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const ProgramHeader* hdr = reinterpret_cast<const ProgramHeader*>(prog);
  const PassDesc& pd = sh.pd;
  const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(prog + hdr->off_phase) + pd.phase0 + h;
  uint32_t sb;
  uint64_t pb = *gbp;
  if (h < kPhaseTab) {
    const int e0 = h * 48 + (int)(t & 15u), e1 = h * 48 + 16 + (int)((t >> 4) & 31u);
    sb = swz64(sh.lt[e0] | sh.lt[e1]);
    pb |= sh.pt[e0] | sh.pt[e1];
  } else {
    uint32_t lb = 0;
    for (int j = 0; j < pd.m - pd.r; ++j)
      if ((t >> j) & 1u) { lb |= 1u << ph->tbit[j]; pb |= 1ull << pd.sbit[ph->tbit[j]]; }
    sb = swz64(lb);
  }
  uint32_t B8[LR];
  ex.template reg_offsets<Real, LR>(ph, h, B8);
  const int jr = ex.template pair_reg<LR>(ph, h);
  C a[NR];
  regs_io<C, LR, 0>(jr, a, smem_raw, bsel ^ (sb * 8u), B8, false, false);
  bar();  // the buffer is free
  next();
  const uint32_t fl = ex.template run<C, LR>(prog, ph, p, h, a, pb);
  uint64_t P[LR];
  uint32_t L[LR];
  ex.template phys_offsets<LR>(h, P, L);
  uint64_t base = pb;
#pragma unroll
  for (int j = 0; j < LR; ++j)
    if (j != jr && (fl & L[j])) base |= P[j];
  opaque(base);
  const bool swap = jr >= 0 && (fl & 1u);  // local bit 0 flipped: the halves of each pair swap
  if (jr >= 0) {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
      if ((i >> jr) & 1) continue;
      uint64_t off = 0;
#pragma unroll
      for (int j = 0; j < LR; ++j)
        if (j != jr && ((i >> j) & 1)) off |= P[j];
      const int i1 = i | (1 << jr);
      const C lo = swap ? a[i1] : a[i], hi = swap ? a[i] : a[i1];
      __stcg(reinterpret_cast<float4*>(psi + (base ^ off)), make_float4(lo.x, lo.y, hi.x, hi.y));
    }
  } else {
#pragma unroll
    for (int i = 0; i < NR; ++i) {
      uint64_t off = 0;
#pragma unroll
      for (int j = 0; j < LR; ++j)
        if ((i >> j) & 1) off |= P[j];
      __stcg(psi + (base ^ off), a[i]);
    }
  }
}

// One pass per launch, one group buffer per block (two resident blocks per SM), complex64 with
// interleaved registers, NPH phases known at compile time and every thread of the block active
// in the pass: the last phase stores to global memory itself (group_phase_direct), so each
// group's copies are issued during the previous group's last phase.
template <typename Real, int LR, typename Exec, int NPH>
__device__ __forceinline__ void pass_body_direct(const Exec& ex, const uint8_t* __restrict__ prog,
                                                 typename V2<Real>::T* __restrict__ psi, int p) {
  static_assert(NPH > 0, "phase count known at compile time");
  using C = typename V2<Real>::T;
  constexpr int kItemBits = sizeof(Real) == 4 ? 1 : 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PassShared sh;
  __shared__ uint64_t s_gb;  // physical base of the current group
  const unsigned t = threadIdx.x;
  pass_setup<Real>(sh, prog, p);
  // copies of group gg: row v of thread t is local index (t << 1) | lv_v, so (the deposit and
  // the swizzle being linear) its source is (group base | thread base) | P[v] and its swizzled
  // destination (swz(t << 1) * 8) ^ D[v], with P / D constants of the pass (ex.copy_offsets);
  // the thread's base is re-read from shared memory, so nothing stays live across the last phase
  constexpr int V = 1 << (LR - kItemBits);
  auto copy_group = [&](uint64_t gg) {
    if (gg < (1ull << sh.pd.ngbits)) {
      uint64_t P[V];
      uint32_t D[V];
      ex.template copy_offsets<V>(P, D);
      const uint64_t b = gbase_of(gg, sh.gtab) | sh.base[t];
      const uint32_t d = swz<Real>(t << kItemBits) * (uint32_t)sizeof(C);
#pragma unroll
      for (int v = 0; v < V; ++v) cp_async16(smem_raw + (d ^ D[v]), psi + (b | P[v]));
    }
    cp_async_commit();
  };
  const uint64_t ngroups = 1ull << sh.pd.ngbits;
  uint64_t g = blockIdx.x;
  copy_group(g);
  for (; g < ngroups; g += gridDim.x) {
    if (t == 0) s_gb = gbase_of(g, sh.gtab);  // the previous group's reads of s_gb are done
    cp_async_wait<0>();
    __syncthreads();
#pragma unroll
    for (int h = 0; h < NPH - 1; ++h) {
      group_phase<Real, LR>(ex, prog, sh, p, h, 0u, &s_gb, t);
      __syncthreads();
    }
    group_phase_direct<Real, LR>(ex, prog, sh, p, NPH - 1, 0u, &s_gb, t, psi, [] { __syncthreads(); },
                                 [&] { copy_group(g + gridDim.x); });
  }
  cp_async_wait<0>();
}

// Two teams of blockDim.x / 2 threads per block, three group buffers of 2^m amplitudes
// (complex64: 3 x 64 KiB).  One pass per launch.  The block's groups are its slots
// s = 0, 1, 2, ... (group blockIdx.x + s * gridDim.x): team s & 1 processes slot s in buffer
// s % 3; after finishing slot s a team copies slot s + 3 into buffer s % 3 for the other team.
// Team 0 then waits at slot 2k for team 1's slot 2k - 3, team 1 at slot 2k + 1 for team 0's
// slot 2k - 2: the teams alternate, and each group's copies run while both teams compute.
// kDirect (complex64, NPH > 0, every thread of a team active): the last phase stores from
// registers and issues the copies of slot s + 3 as soon as it has read buffer s % 3.
template <typename Real, int LR, typename Exec, int NPH = 0, bool kDirect = false>
__device__ __forceinline__ void pass_body_teams(const Exec& ex, const uint8_t* __restrict__ prog,
                                                typename V2<Real>::T* __restrict__ psi, int p, unsigned* err,
                                                uint64_t limit_ns) {
  using C = typename V2<Real>::T;
  constexpr int kItemBits = sizeof(Real) == 4 ? 1 : 0;
  constexpr uint32_t kEsz = sizeof(C);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PassShared sh;
  __shared__ uint64_t s_mbar[3];   // copies into buffer b complete
  __shared__ uint64_t s_gb[2];     // physical base of each team's current group
  __shared__ int s_ok[2];          // the team's leader saw its copies complete
  const unsigned tid = threadIdx.x, TS = blockDim.x >> 1;
  const unsigned team = tid >= TS ? 1u : 0u, t = tid - team * TS;
  if (tid == 0)
    for (int b = 0; b < 3; ++b) mbar_init(&s_mbar[b], TS);
  pass_setup<Real>(sh, prog, p);  // block barrier: the barriers are initialised
  const int m = sh.pd.m;
  const int T = 1 << (m - sh.pd.r);
  const int V = 1 << (m - kItemBits) >> (m - sh.pd.r);
  const uint64_t ngroups = 1ull << sh.pd.ngbits;
  const uint32_t bufb = kEsz << m;
  const uint64_t tbase = (int)t < T ? sh.base[t] : 0ull;
  auto group_of = [&](uint64_t s) { return (uint64_t)blockIdx.x + s * (uint64_t)gridDim.x; };
  // every thread of the loading team arrives once per load (inactive threads immediately)
  auto load_slot = [&](uint64_t s) {
    const uint32_t b = (uint32_t)(s % 3u);
    prefetch_group<Real>(reinterpret_cast<C*>(smem_raw + b * bufb), psi, gbase_of(group_of(s), sh.gtab), tbase,
                         sh.pv, T, V, t);
    cp_async_mbar_arrive(&s_mbar[b]);
  };
  // the same, issued inside a last phase: one copy address at a time, the thread's base re-read
  auto load_slot_rolled = [&](uint64_t s) {
    const uint32_t b = (uint32_t)(s % 3u);
    prefetch_group<Real, false>(reinterpret_cast<C*>(smem_raw + b * bufb), psi, gbase_of(group_of(s), sh.gtab),
                                sh.base[t], sh.pv, T, V, t);
    cp_async_mbar_arrive(&s_mbar[b]);
  };
  auto team_bar = [team, TS] { named_barrier(1u + team, TS); };
  if (team == 0) {
    if (group_of(0) < ngroups) load_slot(0);
    if (group_of(2) < ngroups) load_slot(2);
  } else if (group_of(1) < ngroups) {
    load_slot(1);
  }
  for (uint64_t s = team; group_of(s) < ngroups; s += 2) {
    const uint32_t b = (uint32_t)(s % 3u);
    const unsigned parity = (unsigned)((s / 3u) & 1u);
    if (t == 0) {
      s_ok[team] = mbar_wait_bounded(&s_mbar[b], parity, err, limit_ns) ? 1 : 0;
      s_gb[team] = gbase_of(group_of(s), sh.gtab);
    }
    team_bar();
    if (!s_ok[team]) {  // team-uniform: leave with no copy of this thread in flight
      cp_async_wait<0>();
      return;
    }
    (void)mbar_test(&s_mbar[b], parity);  // completed: acquires the copies for this thread
    const uint32_t bsel = b * bufb;
    if constexpr (kDirect) {
      static_assert(NPH > 0, "phase count known at compile time");
#pragma unroll
      for (int h = 0; h < NPH - 1; ++h) {
        group_phase<Real, LR>(ex, prog, sh, p, h, bsel, &s_gb[team], t);
        team_bar();
      }
      group_phase_direct<Real, LR>(ex, prog, sh, p, NPH - 1, bsel, &s_gb[team], t, psi, team_bar, [&] {
        if (group_of(s + 3) < ngroups) load_slot_rolled(s + 3);
      });
    } else {
      group_phases<Real, LR, Exec, NPH>(ex, prog, sh, p, bsel, &s_gb[team], t, team_bar);
      group_store<Real, Exec::kPacked>(sh, psi, bsel, s_gb[team], t);
      team_bar();  // buffer b is free
      if (group_of(s + 3) < ngroups) load_slot(s + 3);
    }
  }
}

}  // namespace qsb
