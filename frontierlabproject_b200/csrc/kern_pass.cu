// Pass kernel: one sweep of the state per pass, every gate of the pass applied to each
// 2^m-amplitude group while it is on chip.
//
// Per group (one value of the group bits):
//   load   16-byte coalesced global loads -> swizzled shared memory (2^k contiguous
//          amplitudes per run, k >= 1 lowest physical bits always staged);
//   phases each thread reads its 2^R amplitudes (the phase's register bits) from shared
//          memory, applies the phase's gates in registers, writes them back;
//   store  shared memory -> 16-byte coalesced global stores, optionally through a bit
//          permutation of the local bits (in-place permutation passes).
// In cooperative mode one launch runs many passes, separated by a grid barrier whose
// wait is bounded (error word set, kernel returns) -- never an unbounded spin.
#include <cstdint>
#include <cuda_runtime.h>

#include "plan.h"
#include "qsim.h"
#include "kernels.h"

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

__device__ __forceinline__ void opaque(uint32_t& x) { asm volatile("" : "+r"(x)); }
__device__ __forceinline__ void opaque(uint64_t& x) { asm volatile("" : "+l"(x)); }
template <typename T> __device__ __forceinline__ const T* opaque_ptr(const T* p) {
  asm volatile("" : "+l"(p));
  return p;
}

template <typename Real>
__device__ __forceinline__ uint32_t swz(uint32_t l);
template <> __device__ __forceinline__ uint32_t swz<float>(uint32_t l) { return swz64(l); }
template <> __device__ __forceinline__ uint32_t swz<double>(uint32_t l) { return swz128(l); }

// ------------------------------------------------------------------------------------
// register-level gate bodies; J* are register-bit indices known at compile time
// ------------------------------------------------------------------------------------
template <typename C, int NR, int J>
__device__ __forceinline__ void g1_dense(C* a, const C* __restrict__ u) {
  const C u0 = u[0], u1 = u[1], u2 = u[2], u3 = u[3];
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << J)) continue;
    C x = a[i], y = a[i | (1 << J)];
    a[i] = cmac2(u0, x, u1, y);
    a[i | (1 << J)] = cmac2(u2, x, u3, y);
  }
}
template <typename C, int NR, int J>
__device__ __forceinline__ void g1_real(C* a, const C* __restrict__ u) {
  const auto u0 = u[0].x, u1 = u[1].x, u2 = u[2].x, u3 = u[3].x;
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << J)) continue;
    C x = a[i], y = a[i | (1 << J)], p, q;
    p.x = u0 * x.x + u1 * y.x; p.y = u0 * x.y + u1 * y.y;
    q.x = u2 * x.x + u3 * y.x; q.y = u2 * x.y + u3 * y.y;
    a[i] = p; a[i | (1 << J)] = q;
  }
}
// u00, u11 real; u01 = i*s1, u10 = i*s2
template <typename C, int NR, int J>
__device__ __forceinline__ void g1_reim(C* a, const C* __restrict__ u) {
  const auto c0 = u[0].x, s1 = u[1].y, s2 = u[2].y, c3 = u[3].x;
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << J)) continue;
    C x = a[i], y = a[i | (1 << J)], p, q;
    p.x = c0 * x.x - s1 * y.y; p.y = c0 * x.y + s1 * y.x;
    q.x = c3 * y.x - s2 * x.y; q.y = c3 * y.y + s2 * x.x;
    a[i] = p; a[i | (1 << J)] = q;
  }
}
template <typename C, int NR, int J>
__device__ __forceinline__ void g1_x(C* a) {
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << J)) continue;
    C t = a[i]; a[i] = a[i | (1 << J)]; a[i | (1 << J)] = t;
  }
}
template <typename C, int NR, int J>
__device__ __forceinline__ void g1_diag(C* a, const C* __restrict__ u) {
  const C d0 = u[0], d1 = u[1];
#pragma unroll
  for (int i = 0; i < NR; ++i) a[i] = cmul(a[i], (i & (1 << J)) ? d1 : d0);
}
template <typename C, int NR>
__device__ __forceinline__ void scale_all(C* a, C d) {
#pragma unroll
  for (int i = 0; i < NR; ++i) a[i] = cmul(a[i], d);
}
// 2q diagonal; JA/JB = -1 means the bit is fixed per thread (value va / vb)
template <typename C, int NR, int JA, int JB>
__device__ __forceinline__ void g2_diag(C* a, const C* __restrict__ u, int va, int vb) {
  const C d0 = u[0], d1 = u[1], d2 = u[2], d3 = u[3];
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    const int ba = JA >= 0 ? ((i >> (JA < 0 ? 0 : JA)) & 1) : va;
    const int bb = JB >= 0 ? ((i >> (JB < 0 ? 0 : JB)) & 1) : vb;
    const int idx = ba + 2 * bb;
    const C d = idx == 0 ? d0 : (idx == 1 ? d1 : (idx == 2 ? d2 : d3));
    a[i] = cmul(a[i], d);
  }
}
// controlled X: control JC (or fixed value vc when JC = -1), target JT
template <typename C, int NR, int JC, int JT>
__device__ __forceinline__ void g2_cx(C* a, int vc) {
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << JT)) continue;
    const int c = JC >= 0 ? ((i >> (JC < 0 ? 0 : JC)) & 1) : vc;
    if (JC >= 0 && !c) continue;
    if (JC < 0 && !vc) continue;
    C t = a[i]; a[i] = a[i | (1 << JT)]; a[i | (1 << JT)] = t;
  }
}
template <typename C, int NR, int JC, int JT>
__device__ __forceinline__ void g2_cu(C* a, const C* __restrict__ u, int vc) {
  if (JC < 0 && !vc) return;
  const C u0 = u[0], u1 = u[1], u2 = u[2], u3 = u[3];
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if (i & (1 << JT)) continue;
    if (JC >= 0 && !((i >> (JC < 0 ? 0 : JC)) & 1)) continue;
    C x = a[i], y = a[i | (1 << JT)];
    a[i] = cmac2(u0, x, u1, y);
    a[i | (1 << JT)] = cmac2(u2, x, u3, y);
  }
}
template <typename C, int NR, int JA, int JB>
__device__ __forceinline__ void g2_swap(C* a) {
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    // exchange amplitudes with (ba, bb) = (1, 0) and (0, 1)
    if (!((i >> JA) & 1) || ((i >> JB) & 1)) continue;
    const int j = (i & ~(1 << JA)) | (1 << JB);
    C t = a[i]; a[i] = a[j]; a[j] = t;
  }
}
template <typename C, int NR, int JA, int JB>
__device__ __forceinline__ void g2_dense(C* a, const C* __restrict__ u0) {
#pragma unroll
  for (int i = 0; i < NR; ++i) {
    if ((i >> JA) & 1 || (i >> JB) & 1) continue;
    // coefficients re-read per quadruple (L1-resident) instead of 32 live registers
    const C* u = opaque_ptr(u0);
    const int i1 = i | (1 << JA), i2 = i | (1 << JB), i3 = i1 | (1 << JB);
    const C x0 = a[i], x1 = a[i1], x2 = a[i2], x3 = a[i3];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      C s = cmac2(u[4 * r], x0, u[4 * r + 1], x1);
      C t = cmac2(u[4 * r + 2], x2, u[4 * r + 3], x3);
      s.x += t.x; s.y += t.y;
      a[r == 0 ? i : (r == 1 ? i1 : (r == 2 ? i2 : i3))] = s;
    }
  }
}

// ------------------------------------------------------------------------------------
// dispatch of one gate instruction
// ------------------------------------------------------------------------------------
template <typename C, int NR, int LR>
struct Dispatch {
  template <int J>
  __device__ __forceinline__ static void one(uint8_t kind, C* a, const C* u) {
    switch (kind) {
      case GK_1Q_DENSE: g1_dense<C, NR, J>(a, u); break;
      case GK_1Q_REAL: g1_real<C, NR, J>(a, u); break;
      case GK_1Q_REIM: g1_reim<C, NR, J>(a, u); break;
      case GK_1Q_X: g1_x<C, NR, J>(a); break;
      case GK_1Q_DIAG: g1_diag<C, NR, J>(a, u); break;
      default: break;
    }
  }
  // two register operands
  template <int JA, int JB>
  __device__ __forceinline__ static void two_rr(uint8_t kind, C* a, const C* u) {
    if constexpr (JA != JB) {
      switch (kind) {
        case GK_2Q_DENSE: g2_dense<C, NR, JA, JB>(a, u); break;
        case GK_2Q_DIAG: g2_diag<C, NR, JA, JB>(a, u, 0, 0); break;
        case GK_2Q_CX: g2_cx<C, NR, JA, JB>(a, 0); break;
        case GK_2Q_CU: g2_cu<C, NR, JA, JB>(a, u, 0); break;
        case GK_2Q_SWAP: g2_swap<C, NR, JA, JB>(a); break;
        default: break;
      }
    }
  }
  template <int JA>
  __device__ __forceinline__ static void two_r_any(uint8_t kind, int jb, C* a, const C* u) {
    switch (jb) {
      case 0: two_rr<JA, 0>(kind, a, u); break;
      case 1: two_rr<JA, 1>(kind, a, u); break;
      case 2: two_rr<JA, 2>(kind, a, u); break;
      case 3: two_rr<JA, 3>(kind, a, u); break;
      case 4: if constexpr (LR > 4) two_rr<JA, 4>(kind, a, u); break;
      default: break;
    }
  }
  // first operand fixed (value va), second a register bit
  template <int JB>
  __device__ __forceinline__ static void two_fr(uint8_t kind, int va, C* a, const C* u) {
    switch (kind) {
      case GK_2Q_DIAG: g2_diag<C, NR, -1, JB>(a, u, va, 0); break;
      case GK_2Q_CX: g2_cx<C, NR, -1, JB>(a, va); break;
      case GK_2Q_CU: g2_cu<C, NR, -1, JB>(a, u, va); break;
      default: break;
    }
  }
  template <int JA>
  __device__ __forceinline__ static void two_rf(uint8_t kind, int vb, C* a, const C* u) {
    if (kind == GK_2Q_DIAG) g2_diag<C, NR, JA, -1>(a, u, 0, vb);
  }
};

template <typename C, int LR>
__device__ __forceinline__ void apply_gate(const GateInstr g, C* a, const C* __restrict__ coef, uint64_t pbase) {
  constexpr int NR = 1 << LR;
  using D = Dispatch<C, NR, LR>;
  const C* u = coef + g.coef;
  const uint8_t kind = g.kind;
  if (kind < GK_2Q_DENSE) {
    if (g.a >= kFixed) {  // only diagonal gates may have a fixed operand
      const int v = (int)((pbase >> (g.a - kFixed)) & 1ull);
      scale_all<C, NR>(a, u[v]);
      return;
    }
    switch (g.a) {
      case 0: D::template one<0>(kind, a, u); break;
      case 1: D::template one<1>(kind, a, u); break;
      case 2: D::template one<2>(kind, a, u); break;
      case 3: D::template one<3>(kind, a, u); break;
      case 4: if constexpr (LR > 4) D::template one<4>(kind, a, u); break;
      default: break;
    }
    return;
  }
  const bool fa = g.a >= kFixed, fb = g.b >= kFixed;
  if (fa && fb) {  // diagonal with both bits fixed
    const int va = (int)((pbase >> (g.a - kFixed)) & 1ull), vb = (int)((pbase >> (g.b - kFixed)) & 1ull);
    scale_all<C, NR>(a, u[va + 2 * vb]);
    return;
  }
  if (fa) {
    const int va = (int)((pbase >> (g.a - kFixed)) & 1ull);
    switch (g.b) {
      case 0: D::template two_fr<0>(kind, va, a, u); break;
      case 1: D::template two_fr<1>(kind, va, a, u); break;
      case 2: D::template two_fr<2>(kind, va, a, u); break;
      case 3: D::template two_fr<3>(kind, va, a, u); break;
      case 4: if constexpr (LR > 4) D::template two_fr<4>(kind, va, a, u); break;
      default: break;
    }
    return;
  }
  if (fb) {
    const int vb = (int)((pbase >> (g.b - kFixed)) & 1ull);
    switch (g.a) {
      case 0: D::template two_rf<0>(kind, vb, a, u); break;
      case 1: D::template two_rf<1>(kind, vb, a, u); break;
      case 2: D::template two_rf<2>(kind, vb, a, u); break;
      case 3: D::template two_rf<3>(kind, vb, a, u); break;
      case 4: if constexpr (LR > 4) D::template two_rf<4>(kind, vb, a, u); break;
      default: break;
    }
    return;
  }
  switch (g.a) {
    case 0: D::template two_r_any<0>(kind, g.b, a, u); break;
    case 1: D::template two_r_any<1>(kind, g.b, a, u); break;
    case 2: D::template two_r_any<2>(kind, g.b, a, u); break;
    case 3: D::template two_r_any<3>(kind, g.b, a, u); break;
    case 4: if constexpr (LR > 4) D::template two_r_any<4>(kind, g.b, a, u); break;
    default: break;
  }
}

// ------------------------------------------------------------------------------------
// bounded grid barrier (cooperative launches only)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bar[0] = arrivals, bar[1] = generation.  Returns false when the wait gave up.
__device__ bool grid_barrier(unsigned* bar, unsigned* err, uint64_t limit_ns) {
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

// ------------------------------------------------------------------------------------
// the kernel
// ------------------------------------------------------------------------------------
// physical offset of the local index l (deposit of l's bits onto the staged bits)
__device__ __forceinline__ uint64_t phys_of_local(uint32_t l, const int8_t* sbit, int m) {
  uint64_t q = 0;
  for (int j = 0; j < m; ++j) if ((l >> j) & 1u) q |= 1ull << sbit[j];
  return q;
}
__device__ __forceinline__ uint64_t group_base(uint64_t g, const int8_t* gbit, int ng) {
  uint64_t b = 0;
  for (int j = 0; j < ng; ++j) if ((g >> j) & 1ull) b |= 1ull << gbit[j];
  return b;
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

// Issue the asynchronous load of group g into the shared buffer `buf` (16-byte copies,
// swizzled destinations).  Items: c64 -> two amplitudes (local bit 0 inside the vector),
// c128 -> one amplitude.
template <typename Real>
__device__ __forceinline__ void prefetch_group(typename V2<Real>::T* buf, const typename V2<Real>::T* psi,
                                               uint64_t g, const PassDesc& pd, const uint64_t* pv, int T, int V) {
  constexpr int kItemBits = sizeof(Real) == 4 ? 1 : 0;
  const unsigned t = threadIdx.x;
  if ((int)t >= T) return;
  const uint64_t gbase = group_base(g, pd.gbit, pd.ngbits);
  const uint32_t lt = (uint32_t)t << kItemBits;
  const uint64_t base = gbase | phys_of_local(lt, pd.sbit, pd.m);
#pragma unroll
  for (int v = 0; v < 16; ++v) {
    if (v >= V) break;
    const uint32_t l = lt | (((uint32_t)v * (uint32_t)T) << kItemBits);
    cp_async16(buf + swz<Real>(l), psi + (base | pv[v]));
  }
}

template <typename Real, int LR>
__global__ void __launch_bounds__(kPassThreads, 1)
pass_kernel(const uint8_t* __restrict__ prog, typename V2<Real>::T* __restrict__ psi, int pass_begin,
            int pass_end, unsigned* bar, unsigned* err, uint64_t barrier_limit_ns) {
  using C = typename V2<Real>::T;
  constexpr int NR = 1 << LR;
  constexpr bool kC64 = sizeof(Real) == 4;
  constexpr int kItemBits = kC64 ? 1 : 0;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ PassDesc pd;
  __shared__ uint64_t pv[16];     // physical offset of load/store item row v
  __shared__ uint32_t sv[16];     // store-permutation source local offset of row v

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
    __syncthreads();
    const uint64_t ngroups = 1ull << pd.ngbits;
    const bool active = (int)t < T;
    C* bufs[2] = {reinterpret_cast<C*>(smem_raw), reinterpret_cast<C*>(smem_raw) + (1u << m)};

    uint64_t g = blockIdx.x;
    if (g < ngroups) prefetch_group<Real>(bufs[0], psi, g, pd, pv, T, V);
    cp_async_commit();
    for (int it = 0; g < ngroups; g += gridDim.x, ++it) {
      C* sm = bufs[it & 1];
      const uint64_t gn = g + gridDim.x;
      if (gn < ngroups) prefetch_group<Real>(bufs[(it & 1) ^ 1], psi, gn, pd, pv, T, V);
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();
      // ---- phases ----
      for (int h = 0; h < pd.nphase; ++h) {
        if (active) {
          const PhaseDesc* ph = reinterpret_cast<const PhaseDesc*>(prog + hdr->off_phase) + pd.phase0 + h;
          uint32_t sb;
          uint64_t pb;
          {
            uint32_t lb = 0;
            pb = group_base(g, pd.gbit, pd.ngbits);
            const int nt = m - pd.r;
            for (int j = 0; j < nt; ++j)
              if ((t >> j) & 1u) { lb |= 1u << ph->tbit[j]; pb |= 1ull << pd.sbit[ph->tbit[j]]; }
            sb = swz<Real>(lb);
          }
          uint32_t B[LR];
#pragma unroll
          for (int j = 0; j < LR; ++j) B[j] = swz<Real>(1u << ph->rbit[j]);
          C a[NR];
#pragma unroll
          for (int i = 0; i < NR; ++i) {
            uint32_t s = sb;
#pragma unroll
            for (int j = 0; j < LR; ++j) if ((i >> j) & 1) s ^= B[j];
            a[i] = sm[s];
          }
          const GateInstr* gates = reinterpret_cast<const GateInstr*>(prog + hdr->off_gate) + ph->gate0;
          const C* coef = reinterpret_cast<const C*>(prog + hdr->off_coef);
          const int ng = ph->ngate;
          for (int gi = 0; gi < ng; ++gi) {
            const GateInstr gin = gates[gi];
            apply_gate<C, LR>(gin, a, coef, pb);
          }
          opaque(sb);
#pragma unroll
          for (int j = 0; j < LR; ++j) opaque(B[j]);
#pragma unroll
          for (int i = 0; i < NR; ++i) {
            uint32_t s = sb;
#pragma unroll
            for (int j = 0; j < LR; ++j) if ((i >> j) & 1) s ^= B[j];
            sm[s] = a[i];
          }
        }
        __syncthreads();
      }
      // ---- store ----
      if (active) {
        const uint64_t gbase = group_base(g, pd.gbit, pd.ngbits);
        const uint32_t lt = (uint32_t)t << kItemBits;
        const uint64_t base = gbase | phys_of_local(lt, pd.sbit, m);
        uint32_t stt = 0;
        if (pd.store_perm)
          for (int j = 0; j < m; ++j) if ((lt >> j) & 1u) stt |= 1u << pd.store_src[j];
        if constexpr (kC64) {
#pragma unroll
          for (int v = 0; v < 16; ++v) {
            if (v >= V) break;
            float4 val;
            if (pd.store_perm) {
              const uint32_t s0 = stt | sv[v];
              const uint32_t s1 = s0 ^ (1u << pd.store_src[0]);
              const C x0 = sm[swz<Real>(s0)], x1 = sm[swz<Real>(s1)];
              val = make_float4(x0.x, x0.y, x1.x, x1.y);
            } else {
              const uint32_t l = lt | (((uint32_t)v * (uint32_t)T) << 1);
              val = *reinterpret_cast<const float4*>(sm + swz<Real>(l));
            }
            __stcg(reinterpret_cast<float4*>(psi + (base | pv[v])), val);
          }
        } else {
#pragma unroll
          for (int v = 0; v < 16; ++v) {
            if (v >= V) break;
            const uint32_t l = lt | ((uint32_t)v * (uint32_t)T);
            const uint32_t src = pd.store_perm ? (stt | sv[v]) : l;
            __stcg(psi + (base | pv[v]), sm[swz<Real>(src)]);
          }
        }
      }
      __syncthreads();
    }
    cp_async_wait<0>();
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------
template <typename Real, int LR>
static cudaError_t launch_t(const uint8_t* d_prog, void* psi, int pass_begin, int pass_end, int threads,
                            size_t smem, int grid, bool cooperative, unsigned* bar, unsigned* err,
                            uint64_t limit_ns, cudaStream_t stream) {
  using C = typename V2<Real>::T;
  // the dynamic shared-memory limit was raised by pass_kernel_occupancy(), which the
  // executor always calls before launching or capturing
  auto kern = pass_kernel<Real, LR>;
  C* p = reinterpret_cast<C*>(psi);
  if (cooperative) {
    void* args[] = {(void*)&d_prog, (void*)&p, (void*)&pass_begin, (void*)&pass_end, (void*)&bar, (void*)&err,
                    (void*)&limit_ns};
    return cudaLaunchCooperativeKernel((void*)kern, dim3(grid), dim3(threads), args, smem, stream);
  }
  kern<<<grid, threads, smem, stream>>>(d_prog, p, pass_begin, pass_end, bar, err, limit_ns);
  return cudaGetLastError();
}

cudaError_t launch_pass_kernel(int dtype, const uint8_t* d_prog, void* psi, int pass_begin, int pass_end,
                               int threads, size_t smem, int grid, bool cooperative, unsigned* bar,
                               unsigned* err, uint64_t limit_ns, cudaStream_t stream) {
  if (dtype == 0)
    return launch_t<float, 5>(d_prog, psi, pass_begin, pass_end, threads, smem, grid, cooperative, bar, err,
                              limit_ns, stream);
  return launch_t<double, 4>(d_prog, psi, pass_begin, pass_end, threads, smem, grid, cooperative, bar, err,
                             limit_ns, stream);
}

cudaError_t pass_kernel_occupancy(int dtype, int threads, size_t smem, int* blocks_per_sm) {
  if (dtype == 0) {
    cudaFuncSetAttribute(pass_kernel<float, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pass_kernel<float, 5>, threads, smem);
  }
  cudaFuncSetAttribute(pass_kernel<double, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pass_kernel<double, 4>, threads, smem);
}

}  // namespace qsb
