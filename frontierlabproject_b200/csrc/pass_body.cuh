// Device code of a pass (sweep), shared by the generic pass kernel (kern_pass.cu, nvcc)
// and the specialised kernels generated at plan time (jit.cpp, NVRTC).
//
// Per group (one value of the group bits) a block of 256 threads:
//   load   16-byte cp.async copies -> swizzled shared memory, double-buffered: the next
//          group's copies are in flight while the current group is processed;
//   phases each thread reads its 2^LR amplitudes (the phase's register bits) from shared
//          memory, the Exec policy applies the phase's gates in registers, writes back;
//   store  shared memory -> 16-byte coalesced global stores, optionally through a bit
//          permutation of the local bits (in-place permutation passes).
// Several passes in one launch (cooperative mode) are separated by a grid barrier whose
// wait is bounded (error word set, kernel returns).
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

constexpr int kPassThreads = 256;

// Issue the asynchronous load of the group with physical base `gbase` into the shared buffer
// `buf` (16-byte copies, swizzled destinations).  Items: c64 -> two amplitudes (local bit 0
// inside the vector), c128 -> one amplitude.  `tbase` = physical offset of this thread's
// first item.
template <typename Real>
__device__ __forceinline__ void prefetch_group(typename V2<Real>::T* buf, const typename V2<Real>::T* psi,
                                               uint64_t gbase, uint64_t tbase, const uint64_t* pv, int T, int V) {
  constexpr int kItemBits = sizeof(Real) == 4 ? 1 : 0;
  const unsigned t = threadIdx.x;
  if ((int)t >= T) return;
  const uint32_t lt = (uint32_t)t << kItemBits;
  const uint64_t base = gbase | tbase;
#pragma unroll
  for (int v = 0; v < 16; ++v) {
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

// ex.run(prog, ph, pass, h, a, pb) applies the gates of phase h of pass `pass` to the
// thread's registers a[] (pb = physical index of the thread's register-0 amplitude) and
// returns the local bits left flipped in the registers (the write-back lands at the
// flipped addresses); ex.reg_offsets(ph, h, B8) gives the swizzled byte offset of each
// register bit of phase h.
// kDouble: two group buffers per block (the next group's copies overlap this group's
// phases); otherwise one buffer and two resident blocks per SM overlap each other.
// Index deposits that do not change within a pass (group index -> physical base, thread
// index -> local/physical base per phase, per-thread load base) are tabulated in shared
// memory once per pass.
template <typename Real, int LR, typename Exec, bool kDouble = true>
__device__ __forceinline__ void pass_body(const Exec& ex, const uint8_t* __restrict__ prog,
                                          typename V2<Real>::T* __restrict__ psi,
                                          int pass_begin, int pass_end, unsigned* bar, unsigned* err,
                                          uint64_t barrier_limit_ns) {
  using C = typename V2<Real>::T;
  constexpr int NR = 1 << LR;
  constexpr bool kC64 = sizeof(Real) == 4;
  constexpr int kItemBits = kC64 ? 1 : 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PassDesc pd;
  __shared__ uint64_t pv[16];                  // physical offset of load/store item row v
  __shared__ uint32_t sv[16];                  // store-permutation source local offset of row v
  __shared__ uint64_t s_gtab[5 * 128];         // group index -> physical base (5 levels x 7 bits)
  __shared__ uint64_t s_pt[kPhaseTab * 48];    // per phase: physical thread base, t bits 0-3 | 4-8
  __shared__ uint32_t s_lt[kPhaseTab * 48];    // per phase: local thread base
  __shared__ uint64_t s_base[512];             // per thread: physical offset of its first item
  __shared__ uint32_t s_stt[512];              // per thread: store-permutation source of its first item
  __shared__ uint64_t s_gb[2];                 // physical base of the current group

  const unsigned t = threadIdx.x;
  const ProgramHeader* hdr = reinterpret_cast<const ProgramHeader*>(prog);

  for (int p = pass_begin; p < pass_end; ++p) {
    if (p > pass_begin) {
      if (!grid_barrier(bar, err, barrier_limit_ns)) return;
    }
    if (t == 0) pd = reinterpret_cast<const PassDesc*>(prog + hdr->off_pass)[p];
    __syncthreads();
    const int m = pd.m;
    const int T = 1 << (m - pd.r);                    // active threads of this pass
    const int V = 1 << (m - kItemBits) >> (m - pd.r);  // items per thread (16)
    const int nt = m - pd.r;                           // thread-index bits
    for (int v = (int)t; v < V; v += (int)blockDim.x) {
      const uint32_t lv = ((uint32_t)v * (uint32_t)T) << kItemBits;
      uint64_t q = 0;
      uint32_t s = 0;
      for (int j = 0; j < m; ++j)
        if ((lv >> j) & 1u) {
          q |= 1ull << pd.sbit[j];
          if (pd.store_perm) s |= 1u << pd.store_src[j];
        }
      pv[v] = q;
      sv[v] = s;
    }
    for (int e = (int)t; e < 5 * 128; e += (int)blockDim.x) {
      const int level = e >> 7, idx = e & 127;
      uint64_t v = 0;
      for (int j = 0; j < 7; ++j) {
        const int gb = 7 * level + j;
        if (gb < pd.ngbits && ((idx >> j) & 1)) v |= 1ull << pd.gbit[gb];
      }
      s_gtab[e] = v;
    }
    const int nph_tab = pd.nphase < kPhaseTab ? pd.nphase : kPhaseTab;
    for (int e = (int)t; e < nph_tab * 48; e += (int)blockDim.x) {
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
      s_lt[e] = lt;
      s_pt[e] = pt;
    }
    for (int u = (int)t; u < T; u += (int)blockDim.x) {
      const uint32_t l = (uint32_t)u << kItemBits;
      s_base[u] = phys_of_local(l, pd.sbit, m);
      uint32_t st = 0;
      if (pd.store_perm)
        for (int j = 0; j < m; ++j) if ((l >> j) & 1u) st |= 1u << pd.store_src[j];
      s_stt[u] = st;
    }
    __syncthreads();
    const uint64_t ngroups = 1ull << pd.ngbits;
    const bool active = (int)t < T;
    const uint64_t tbase = active ? s_base[t] : 0ull;
    // Group buffers: buffer 1 starts at byte (esz << m) of the dynamic shared memory, one bit
    // above every byte offset of a swizzled local index, so a buffer's addresses are XOR
    // combinations of byte offsets.  Accesses index smem_raw directly (shared-memory
    // loads/stores with the array base as the immediate offset).
    constexpr uint32_t kEsz = sizeof(C);
    const uint32_t buf1 = kDouble ? (kEsz << m) : 0u;
    auto at = [&](uint32_t byte) -> C& { return *reinterpret_cast<C*>(smem_raw + byte); };

    uint64_t g = blockIdx.x;
    if (kDouble) {
      if (g < ngroups)
        prefetch_group<Real>(reinterpret_cast<C*>(smem_raw), psi, gbase_of(g, s_gtab), tbase, pv, T, V);
      cp_async_commit();
    }
    for (int it = 0; g < ngroups; g += gridDim.x, ++it) {
      const uint32_t bsel = (it & 1) ? buf1 : 0u;  // byte offset of this group's buffer
      if (t == 0) s_gb[it & 1] = gbase_of(g, s_gtab);  // read after the barrier below
      if (kDouble) {
        const uint64_t gn = g + gridDim.x;
        if (gn < ngroups)
          prefetch_group<Real>(reinterpret_cast<C*>(smem_raw + (bsel ^ buf1)), psi, gbase_of(gn, s_gtab), tbase, pv,
                               T, V);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        prefetch_group<Real>(reinterpret_cast<C*>(smem_raw), psi, gbase_of(g, s_gtab), tbase, pv, T, V);
        cp_async_commit();
        cp_async_wait<0>();
      }
      __syncthreads();
      // ---- phases ----
      for (int h = 0; h < pd.nphase; ++h) {
        if (active) {
          const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(prog + hdr->off_phase) + pd.phase0 + h;
          uint32_t sb;
          uint64_t pb = s_gb[it & 1];
          if (h < kPhaseTab) {
            const int e0 = h * 48 + (int)(t & 15u), e1 = h * 48 + 16 + (int)((t >> 4) & 31u);
            sb = swz<Real>(s_lt[e0] | s_lt[e1]);
            pb |= s_pt[e0] | s_pt[e1];
          } else {
            uint32_t lb = 0;
            for (int j = 0; j < nt; ++j)
              if ((t >> j) & 1u) { lb |= 1u << ph->tbit[j]; pb |= 1ull << pd.sbit[ph->tbit[j]]; }
            sb = swz<Real>(lb);
          }
          uint32_t sb8 = bsel ^ (sb * kEsz);
          uint32_t B8[LR];  // byte offset of register bit j (swizzled)
          ex.template reg_offsets<Real, LR>(ph, h, B8);
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
        __syncthreads();
      }
      // ---- store ----
      if (active) {
        const uint32_t lt = (uint32_t)t << kItemBits;
        const uint64_t base = s_gb[it & 1] | s_base[t];
        const uint32_t stt = s_stt[t];
        if constexpr (kC64) {
#pragma unroll
          for (int v = 0; v < 16; ++v) {
            if (v >= V) break;
            float4 val;
            if (pd.store_perm) {
              const uint32_t s0 = stt | sv[v];
              const uint32_t s1 = s0 ^ (1u << pd.store_src[0]);
              const C x0 = at(bsel ^ (swz<Real>(s0) * kEsz)), x1 = at(bsel ^ (swz<Real>(s1) * kEsz));
              val = make_float4(x0.x, x0.y, x1.x, x1.y);
            } else {
              const uint32_t l = lt | (((uint32_t)v * (uint32_t)T) << 1);
              val = *reinterpret_cast<const float4*>(smem_raw + (bsel ^ (swz<Real>(l) * kEsz)));
            }
            __stcg(reinterpret_cast<float4*>(psi + (base | pv[v])), val);
          }
        } else {
#pragma unroll
          for (int v = 0; v < 16; ++v) {
            if (v >= V) break;
            const uint32_t l = lt | ((uint32_t)v * (uint32_t)T);
            const uint32_t src = pd.store_perm ? (stt | sv[v]) : l;
            __stcg(psi + (base | pv[v]), at(bsel ^ (swz<Real>(src) * kEsz)));
          }
        }
      }
      __syncthreads();
    }
    cp_async_wait<0>();
    __syncthreads();
  }
}

}  // namespace qsb
