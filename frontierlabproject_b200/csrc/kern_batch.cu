// Persistent kernel of the batched variational workload (layout and scheduling: batch.h).
//
// One launch processes every work item of a batch: blocks take items from a global counter,
// wait (bounded by a time limit; the error word is set when it runs out) for the items of
// the same instance's earlier stages, and run them:
//   SMALL  psi and lam in shared memory: forward sweep, lam = H psi, energy, reverse sweep;
//   FWD    for each group of the item: stage 2^m amplitudes of psi (16-byte cp.async), apply
//          the pass's gates in shared memory, store;
//   HAM    lam = H psi over amplitude chunks (L2 reads of the X-neighbours), energy;
//   BWD    stage psi and lam, for the pass's gates in reverse: Im <lam|G|psi> (FP64, one
//          atomic per warp and gate) and psi, lam <- U^dagger psi, lam; store both.
// Gradients and energies accumulate in FP64; the states are complex64.
#include <cstdint>
#include <cuda_runtime.h>

#include "batch.h"
#include "kernels.h"

namespace qsb {

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cmac(float2 a, float2 x, float2 b, float2 y) {
  return make_float2(a.x * x.x - a.y * x.y + b.x * y.x - b.y * y.y, a.x * x.y + a.y * x.x + b.x * y.y + b.y * y.x);
}

__device__ __forceinline__ uint64_t gtime() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// every thread of the block calls it (full warps); FP32 warp sum of per-thread FP32 terms,
// added in FP64
__device__ __forceinline__ void warp_addf(float v, double* dst) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0f) atomicAdd(dst, (double)v);
}

// every thread of the block calls it (full warps)
__device__ __forceinline__ void warp_add(double v, double* dst) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(dst, v);
}

__device__ __forceinline__ void cp16(void* smem_dst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_wait_all() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

struct Block {
  BatchItem it;
  BatchInst in;
  BatchPass ps;
  int key;                        // (instance, pass) of the tables below, -1: none
  int ok;
  int8_t loc[kBatchMaxQubits];    // local bit of qubit q in the current pass, -1: group bit
};

// Im(conj(l) v) in FP32 (per-pair gradient terms; each thread's sum is reduced in FP64)
__device__ __forceinline__ float im_cvf(float2 l, float2 v) { return l.x * v.y - l.y * v.x; }

// 2x2 matrix (m0 m1; m2 m3) on local bit j of A (and of L when kRev); kRev with GEN != 0:
// before the update, acc += Im <L| G |A> on the pair (GEN 1 X, 2 Y, 3 Z)
template <bool kRev, int GEN>
__device__ __forceinline__ void pairs2g(float2 m0, float2 m1, float2 m2, float2 m3, float2* A, float2* L, int m, int j,
                                        float& acc) {
  const uint32_t half = 1u << (m - 1), lo = (1u << j) - 1u;
  for (uint32_t k = threadIdx.x; k < half; k += blockDim.x) {
    const uint32_t i0 = ((k & ~lo) << 1) | (k & lo), i1 = i0 | (1u << j);
    const float2 p0 = A[i0], p1 = A[i1];
    A[i0] = cmac(m0, p0, m1, p1);
    A[i1] = cmac(m2, p0, m3, p1);
    if (kRev) {
      const float2 l0 = L[i0], l1 = L[i1];
      if (GEN == 1) acc += im_cvf(l0, p1) + im_cvf(l1, p0);
      if (GEN == 2) acc += im_cvf(l0, make_float2(p1.y, -p1.x)) + im_cvf(l1, make_float2(-p0.y, p0.x));
      if (GEN == 3) acc += im_cvf(l0, p0) - im_cvf(l1, p1);
      L[i0] = cmac(m0, l0, m1, l1);
      L[i1] = cmac(m2, l0, m3, l1);
    }
  }
}

template <bool kRev>
__device__ __forceinline__ void pairs2(float2 m0, float2 m1, float2 m2, float2 m3, int gen, float2* A, float2* L,
                                       int m, int j, float& acc) {
  if (!kRev || gen == 0) pairs2g<kRev, 0>(m0, m1, m2, m3, A, L, m, j, acc);
  else if (gen == 1) pairs2g<kRev, 1>(m0, m1, m2, m3, A, L, m, j, acc);
  else if (gen == 2) pairs2g<kRev, 2>(m0, m1, m2, m3, A, L, m, j, acc);
  else pairs2g<kRev, 3>(m0, m1, m2, m3, A, L, m, j, acc);
}

// Diagonal gate: entry d[b0 + 2 b1] per amplitude, the bits taken from the local index (jq >= 0)
// or fixed by the group (jq < 0: value fq).  kZ: acc += Im <L|Z_q0|A> before the update.
template <bool kRev, bool kZ>
__device__ __forceinline__ void diag_g(float2 d0, float2 d1, float2 d2, float2 d3, int j0, int f0, int j1, int f1,
                                       float2* A, float2* L, int m, float& acc) {
  for (uint32_t x = threadIdx.x; x < (1u << m); x += blockDim.x) {
    const int b0 = j0 >= 0 ? (int)((x >> j0) & 1u) : f0;
    const int b1 = j1 >= 0 ? (int)((x >> j1) & 1u) : f1;
    const float2 d = b1 ? (b0 ? d3 : d2) : (b0 ? d1 : d0);
    const float2 p = A[x];
    A[x] = cmul(d, p);
    if (kRev) {
      const float2 l = L[x];
      if (kZ) acc += b0 ? -im_cvf(l, p) : im_cvf(l, p);
      L[x] = cmul(d, l);
    }
  }
}

// One gate on the staged group (forward, or reverse with the gradient slot gslot).  The gate's
// fields are read once into registers (the loops touch only shared memory).
template <bool kRev>
__device__ void apply_gate(const BatchGate& gref, float2* A, float2* L, int m, uint64_t gb, const int8_t* loc,
                           double* gslot) {
  float acc = 0.0f;
  const int kind = gref.kind, q0 = gref.q0, q1 = gref.q1, gen = gref.gen;
  switch (kind) {
    case BG_1Q: {
      const float2 u0 = gref.u[0], u1 = gref.u[1], u2 = gref.u[2], u3 = gref.u[3];
      const int j = loc[q0];
      if (!kRev) pairs2<false>(u0, u1, u2, u3, 0, A, L, m, j, acc);
      else pairs2<true>(cconj(u0), cconj(u2), cconj(u1), cconj(u3), gen, A, L, m, j, acc);
      break;
    }
    case BG_DIAG1: case BG_DIAG2: {
      const bool two = kind == BG_DIAG2;
      float2 d[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float2 v = (two || e < 2) ? gref.u[two ? e : (e & 1)] : make_float2(0.f, 0.f);
        d[e] = kRev ? cconj(v) : v;
      }
      if (!two) { d[2] = d[0]; d[3] = d[1]; }
      const int j0 = loc[q0], f0 = (int)((gb >> q0) & 1ull);
      const int j1 = two ? loc[q1] : -1, f1 = two ? (int)((gb >> q1) & 1ull) : 0;
      if (kRev && gen == 3) diag_g<kRev, true>(d[0], d[1], d[2], d[3], j0, f0, j1, f1, A, L, m, acc);
      else diag_g<kRev, false>(d[0], d[1], d[2], d[3], j0, f0, j1, f1, A, L, m, acc);
      break;
    }
    case BG_2Q: {
      const int j0 = loc[q0], j1 = loc[q1];
      float2 u[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) u[e] = gref.u[e];
      auto M = [&](int r, int c) { return kRev ? cconj(u[4 * c + r]) : u[4 * r + c]; };
      if (j0 >= 0 && j1 >= 0) {
        const int lo = j0 < j1 ? j0 : j1, hi = j0 < j1 ? j1 : j0;
        const uint32_t quarter = 1u << (m - 2);
        for (uint32_t k = threadIdx.x; k < quarter; k += blockDim.x) {
          uint32_t base = k & ((1u << lo) - 1u);
          base |= (k & ((1u << (hi - 1)) - 1u) & ~((1u << lo) - 1u)) << 1;
          base |= (k & ~((1u << (hi - 1)) - 1u)) << 2;
          const uint32_t idx[4] = {base, base | (1u << j0), base | (1u << j1), base | (1u << j0) | (1u << j1)};
          float2 x[4], y[4];
#pragma unroll
          for (int c = 0; c < 4; ++c) { x[c] = A[idx[c]]; if (kRev) y[c] = L[idx[c]]; }
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            float2 s = make_float2(0.f, 0.f), t = make_float2(0.f, 0.f);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              const float2 mc = M(r, c);
              const float2 a = cmul(mc, x[c]);
              s.x += a.x; s.y += a.y;
              if (kRev) { const float2 b = cmul(mc, y[c]); t.x += b.x; t.y += b.y; }
            }
            A[idx[r]] = s;
            if (kRev) L[idx[r]] = t;
          }
        }
      } else if (j0 >= 0 || j1 >= 0) {
        // block-diagonal in the fixed qubit: the 2x2 block of its value on the staged one (entries
        // read from the gate at a run-time index, not from the register copy)
        auto G = [&](int r, int c) { return kRev ? cconj(gref.u[4 * c + r]) : gref.u[4 * r + c]; };
        if (j1 >= 0) {
          const int f = (int)((gb >> q0) & 1ull);
          pairs2<kRev>(G(f, f), G(f, f + 2), G(f + 2, f), G(f + 2, f + 2), 0, A, L, m, j1, acc);
        } else {
          const int f = (int)((gb >> q1) & 1ull);
          pairs2<kRev>(G(2 * f, 2 * f), G(2 * f, 2 * f + 1), G(2 * f + 1, 2 * f), G(2 * f + 1, 2 * f + 1), 0, A, L,
                       m, j0, acc);
        }
      }
      break;
    }
    default: break;
  }
  if (kRev && gen) warp_add((double)acc, gslot);
  __syncthreads();
}

// lam[x] = d(x) psi[x] + sum_i b_i psi[x ^ 2^i] for x in [x0, x1) (psi read through L2 when
// kGlobal); returns the thread's part of sum Re(conj(psi) lam)
// kSwz (shared memory only): the arrays are indexed through swz64 (register-phase layout)
template <bool kGlobal, bool kSwz = false>
__device__ __forceinline__ double hamiltonian(const float2* psi, float2* lam, int n, uint64_t x0, uint64_t x1,
                                              const double* a, const double* b) {
  auto ix = [](uint64_t x) -> uint64_t { return kSwz ? (uint64_t)swz64((uint32_t)x) : x; };
  double e = 0.0;
  for (uint64_t x = x0 + threadIdx.x; x < x1; x += blockDim.x) {
    double d = 0.0;
    for (int i = 0; i < n; ++i) {
      const int j = i + 1 == n ? 0 : i + 1;
      d += (((x >> i) ^ (x >> j)) & 1ull) ? -a[i] : a[i];
    }
    const float2 p = kGlobal ? __ldcg(psi + x) : psi[ix(x)];
    double re = d * p.x, im = d * p.y;
    for (int i = 0; i < n; ++i) {
      const float2 q = kGlobal ? __ldcg(psi + (x ^ (1ull << i))) : psi[ix(x ^ (1ull << i))];
      re += b[i] * q.x;
      im += b[i] * q.y;
    }
    const float2 out = make_float2((float)re, (float)im);
    if (kGlobal) __stcg(lam + x, out);
    else lam[ix(x)] = out;
    e += (double)p.x * re + (double)p.y * im;
  }
  return e;
}

// ---- register phases: 16 amplitudes per thread and state, gates in registers ----------------
constexpr int kRegs = 1 << kBatchRegBits;

// 2x2 on register bit J (pairs i, i | 2^J); kRev: gradient term of generator GEN first
template <int J, bool kRev, int GEN>
__device__ __forceinline__ void pairs_reg(float2 m0, float2 m1, float2 m2, float2 m3, float2 (&a)[kRegs],
                                          float2 (&l)[kRegs], float& acc) {
#pragma unroll
  for (int i = 0; i < kRegs; ++i) {
    if (i & (1 << J)) continue;
    const int i1 = i | (1 << J);
    const float2 p0 = a[i], p1 = a[i1];
    a[i] = cmac(m0, p0, m1, p1);
    a[i1] = cmac(m2, p0, m3, p1);
    if (kRev) {
      const float2 l0 = l[i], l1 = l[i1];
      if (GEN == 1) acc += im_cvf(l0, p1) + im_cvf(l1, p0);
      if (GEN == 2) acc += im_cvf(l0, make_float2(p1.y, -p1.x)) + im_cvf(l1, make_float2(-p0.y, p0.x));
      if (GEN == 3) acc += im_cvf(l0, p0) - im_cvf(l1, p1);
      l[i] = cmac(m0, l0, m1, l1);
      l[i1] = cmac(m2, l0, m3, l1);
    }
  }
}

// Real 2x2 (m0 m1; m2 m3) on register bit J: two multiply-adds per output component
template <int J, bool kRev, int GEN>
__device__ __forceinline__ void pairs_reg_real(float m0, float m1, float m2, float m3, float2 (&a)[kRegs],
                                               float2 (&l)[kRegs], float& acc) {
#pragma unroll
  for (int i = 0; i < kRegs; ++i) {
    if (i & (1 << J)) continue;
    const int i1 = i | (1 << J);
    const float2 p0 = a[i], p1 = a[i1];
    a[i] = make_float2(m0 * p0.x + m1 * p1.x, m0 * p0.y + m1 * p1.y);
    a[i1] = make_float2(m2 * p0.x + m3 * p1.x, m2 * p0.y + m3 * p1.y);
    if (kRev) {
      const float2 l0 = l[i], l1 = l[i1];
      if (GEN == 1) acc += im_cvf(l0, p1) + im_cvf(l1, p0);
      if (GEN == 2) acc += im_cvf(l0, make_float2(p1.y, -p1.x)) + im_cvf(l1, make_float2(-p0.y, p0.x));
      if (GEN == 3) acc += im_cvf(l0, p0) - im_cvf(l1, p1);
      l[i] = make_float2(m0 * l0.x + m1 * l1.x, m0 * l0.y + m1 * l1.y);
      l[i1] = make_float2(m2 * l0.x + m3 * l1.x, m2 * l0.y + m3 * l1.y);
    }
  }
}

template <int J, bool kRev>
__device__ __forceinline__ void pairs_reg_real_g(int gen, float m0, float m1, float m2, float m3, float2 (&a)[kRegs],
                                                 float2 (&l)[kRegs], float& acc) {
  if (!kRev || gen == 0) pairs_reg_real<J, kRev, 0>(m0, m1, m2, m3, a, l, acc);
  else if (gen == 1) pairs_reg_real<J, kRev, 1>(m0, m1, m2, m3, a, l, acc);
  else if (gen == 2) pairs_reg_real<J, kRev, 2>(m0, m1, m2, m3, a, l, acc);
  else pairs_reg_real<J, kRev, 3>(m0, m1, m2, m3, a, l, acc);
}

template <bool kRev>
__device__ __forceinline__ void pairs_reg_real_j(int j, int gen, float m0, float m1, float m2, float m3,
                                                 float2 (&a)[kRegs], float2 (&l)[kRegs], float& acc) {
  switch (j) {
    case 0: pairs_reg_real_g<0, kRev>(gen, m0, m1, m2, m3, a, l, acc); break;
    case 1: pairs_reg_real_g<1, kRev>(gen, m0, m1, m2, m3, a, l, acc); break;
    case 2: pairs_reg_real_g<2, kRev>(gen, m0, m1, m2, m3, a, l, acc); break;
    default: pairs_reg_real_g<3, kRev>(gen, m0, m1, m2, m3, a, l, acc); break;
  }
}

template <int J, bool kRev>
__device__ __forceinline__ void pairs_reg_g(int gen, float2 m0, float2 m1, float2 m2, float2 m3, float2 (&a)[kRegs],
                                            float2 (&l)[kRegs], float& acc) {
  if (!kRev || gen == 0) pairs_reg<J, kRev, 0>(m0, m1, m2, m3, a, l, acc);
  else if (gen == 1) pairs_reg<J, kRev, 1>(m0, m1, m2, m3, a, l, acc);
  else if (gen == 2) pairs_reg<J, kRev, 2>(m0, m1, m2, m3, a, l, acc);
  else pairs_reg<J, kRev, 3>(m0, m1, m2, m3, a, l, acc);
}

// Diagonal (e0 where register bit J is 0, e1 where it is 1); kZ: acc += Im <L|Z_J|A> first.
// The entry of each register is a compile-time choice (no per-amplitude selects); kUnit0: e0
// is exactly 1 (diagonal gates are stored divided by their first entry), its registers skip.
template <int J, bool kRev, bool kZ, bool kUnit0>
__device__ __forceinline__ void diag_reg1(float2 e0, float2 e1, float2 (&a)[kRegs], float2 (&l)[kRegs], float& acc) {
#pragma unroll
  for (int i = 0; i < kRegs; ++i) {
    const bool one = (i >> J) & 1;
    const float2 p = a[i];
    if (kRev && kZ) acc += one ? -im_cvf(l[i], p) : im_cvf(l[i], p);
    if (kUnit0 && !one) continue;
    a[i] = cmul(one ? e1 : e0, p);
    if (kRev) l[i] = cmul(one ? e1 : e0, l[i]);
  }
}

template <bool kRev, bool kZ>
__device__ __forceinline__ void diag_reg1_j(int j, float2 e0, float2 e1, float2 (&a)[kRegs], float2 (&l)[kRegs],
                                            float& acc) {
  const bool u0 = e0.x == 1.f && e0.y == 0.f;
  if (!kZ && u0 && e1.x == 1.f && e1.y == 0.f) return;  // identity here (a controlled phase off)
  if (u0) {
    switch (j) {
      case 0: diag_reg1<0, kRev, kZ, true>(e0, e1, a, l, acc); break;
      case 1: diag_reg1<1, kRev, kZ, true>(e0, e1, a, l, acc); break;
      case 2: diag_reg1<2, kRev, kZ, true>(e0, e1, a, l, acc); break;
      default: diag_reg1<3, kRev, kZ, true>(e0, e1, a, l, acc); break;
    }
  } else {
    switch (j) {
      case 0: diag_reg1<0, kRev, kZ, false>(e0, e1, a, l, acc); break;
      case 1: diag_reg1<1, kRev, kZ, false>(e0, e1, a, l, acc); break;
      case 2: diag_reg1<2, kRev, kZ, false>(e0, e1, a, l, acc); break;
      default: diag_reg1<3, kRev, kZ, false>(e0, e1, a, l, acc); break;
    }
  }
}

// Diagonal d[b_J0 + 2 b_J1] on two register bits; kUnit: mask of entries that are exactly 1
// (1: d0; 7: d0, d1 and d2, a controlled phase such as CZ), whose registers skip
template <int J0, int J1, bool kRev, int kUnit>
__device__ __forceinline__ void diag_reg2(float2 d0, float2 d1, float2 d2, float2 d3, float2 (&a)[kRegs],
                                          float2 (&l)[kRegs]) {
#pragma unroll
  for (int i = 0; i < kRegs; ++i) {
    const int v = ((i >> J0) & 1) | (((i >> J1) & 1) << 1);
    if ((kUnit >> v) & 1) continue;
    const float2 dd = v == 0 ? d0 : v == 1 ? d1 : v == 2 ? d2 : d3;
    a[i] = cmul(dd, a[i]);
    if (kRev) l[i] = cmul(dd, l[i]);
  }
}

template <int J0, bool kRev, int kUnit>
__device__ __forceinline__ void diag_reg2_j1(int j1, float2 d0, float2 d1, float2 d2, float2 d3, float2 (&a)[kRegs],
                                             float2 (&l)[kRegs]) {
  switch (j1) {
    case 0: if constexpr (J0 != 0) diag_reg2<J0, 0, kRev, kUnit>(d0, d1, d2, d3, a, l); break;
    case 1: if constexpr (J0 != 1) diag_reg2<J0, 1, kRev, kUnit>(d0, d1, d2, d3, a, l); break;
    case 2: if constexpr (J0 != 2) diag_reg2<J0, 2, kRev, kUnit>(d0, d1, d2, d3, a, l); break;
    default: if constexpr (J0 != 3) diag_reg2<J0, 3, kRev, kUnit>(d0, d1, d2, d3, a, l); break;
  }
}

template <bool kRev, int kUnit>
__device__ __forceinline__ void diag_reg2_u(int j0, int j1, float2 d0, float2 d1, float2 d2, float2 d3,
                                            float2 (&a)[kRegs], float2 (&l)[kRegs]) {
  switch (j0) {
    case 0: diag_reg2_j1<0, kRev, kUnit>(j1, d0, d1, d2, d3, a, l); break;
    case 1: diag_reg2_j1<1, kRev, kUnit>(j1, d0, d1, d2, d3, a, l); break;
    case 2: diag_reg2_j1<2, kRev, kUnit>(j1, d0, d1, d2, d3, a, l); break;
    default: diag_reg2_j1<3, kRev, kUnit>(j1, d0, d1, d2, d3, a, l); break;
  }
}

template <bool kRev>
__device__ __forceinline__ void diag_reg2_j(int j0, int j1, float2 d0, float2 d1, float2 d2, float2 d3,
                                            float2 (&a)[kRegs], float2 (&l)[kRegs]) {
  auto is1 = [](float2 v) { return v.x == 1.f && v.y == 0.f; };
  if (!is1(d0)) diag_reg2_u<kRev, 0>(j0, j1, d0, d1, d2, d3, a, l);
  else if (is1(d1) && is1(d2)) { if (!is1(d3)) diag_reg2_u<kRev, 7>(j0, j1, d0, d1, d2, d3, a, l); }
  else diag_reg2_u<kRev, 1>(j0, j1, d0, d1, d2, d3, a, l);
}

template <bool kRev>
__device__ __forceinline__ void pairs_reg_j(int j, int gen, float2 m0, float2 m1, float2 m2, float2 m3,
                                            float2 (&a)[kRegs], float2 (&l)[kRegs], float& acc) {
  switch (j) {
    case 0: pairs_reg_g<0, kRev>(gen, m0, m1, m2, m3, a, l, acc); break;
    case 1: pairs_reg_g<1, kRev>(gen, m0, m1, m2, m3, a, l, acc); break;
    case 2: pairs_reg_g<2, kRev>(gen, m0, m1, m2, m3, a, l, acc); break;
    default: pairs_reg_g<3, kRev>(gen, m0, m1, m2, m3, a, l, acc); break;
  }
}

// One gate of a register phase.  reg[q]: register bit of qubit q in this phase (-1: not in
// registers); fixed bits come from the slot's local base index or the group base.
// A gate of the current pass as the register phases read it, cached in shared memory when the
// pass changes (shared-memory latency instead of L1 for the per-gate fields); two-qubit dense
// matrices stay in global memory (gfull).
struct GateLite {
  uint8_t kind, q0, q1, gen;
  int32_t grad;
  int8_t r0, r1;   // register bit of q0 / q1 in the gate's phase, -1: not in registers
  int8_t l0, l1;   // local bit of q0 / q1 in the pass, -1: a group bit
  float2 u[4];
};
constexpr int kGateCache = 192;

// r0 / r1: register bits of the operands in this phase (-1: fixed), l0 / l1: their local bits
// (-1: group bits)
template <bool kRev, typename GT>
__device__ __forceinline__ void gate_reg(const GT& gref, const BatchGate* gfull, int r0, int r1, int l0, int l1,
                                         uint32_t base, uint64_t gb, float2 (&a)[kRegs], float2 (&l)[kRegs],
                                         double* gout) {
  float acc = 0.0f;
  const int kind = gref.kind, q0 = gref.q0, q1 = gref.q1, gen = gref.gen;
  auto fixedbit = [&](int q) -> int {
    const int L = q == q0 ? l0 : l1;
    return L >= 0 ? (int)((base >> L) & 1u) : (int)((gb >> q) & 1ull);
  };
  if (kind == BG_1Q) {
    const float2 u0 = gref.u[0], u1 = gref.u[1], u2 = gref.u[2], u3 = gref.u[3];
    if (u0.y == 0.f && u1.y == 0.f && u2.y == 0.f && u3.y == 0.f) {  // real (RY, H): gate-uniform branch
      if (!kRev) pairs_reg_real_j<false>(r0, 0, u0.x, u1.x, u2.x, u3.x, a, l, acc);
      else pairs_reg_real_j<true>(r0, gen, u0.x, u2.x, u1.x, u3.x, a, l, acc);
    } else if (!kRev) {
      pairs_reg_j<false>(r0, 0, u0, u1, u2, u3, a, l, acc);
    } else {
      pairs_reg_j<true>(r0, gen, cconj(u0), cconj(u2), cconj(u1), cconj(u3), a, l, acc);
    }
  } else if (kind == BG_DIAG1 || kind == BG_DIAG2) {
    // bits held in registers select the entry per register at compile time; fixed bits select
    // once per thread
    const bool two = kind == BG_DIAG2;
    auto ent = [&](int e) { const float2 v = gref.u[e]; return kRev ? cconj(v) : v; };
    const int j0 = r0;
    if (!two) {
      const float2 d0 = ent(0), d1 = ent(1);
      const bool z = kRev && gen == 3;
      if (j0 >= 0) {
        if (z) diag_reg1_j<kRev, true>(j0, d0, d1, a, l, acc);
        else diag_reg1_j<kRev, false>(j0, d0, d1, a, l, acc);
      } else {
        const int f0 = fixedbit(q0);
        const float2 dd = f0 ? d1 : d0;
        const bool unit = dd.x == 1.f && dd.y == 0.f;
#pragma unroll
        for (int i = 0; i < kRegs; ++i) {
          const float2 p = a[i];
          if (z) acc += im_cvf(l[i], p);
          if (!unit) {
            a[i] = cmul(dd, p);
            if (kRev) l[i] = cmul(dd, l[i]);
          }
        }
        if (z && f0) acc = -acc;
      }
    } else {
      const float2 d0 = ent(0), d1 = ent(1), d2 = ent(2), d3 = ent(3);
      const int j1 = r1;
      if (j0 >= 0 && j1 >= 0) {
        diag_reg2_j<kRev>(j0, j1, d0, d1, d2, d3, a, l);
      } else if (j0 >= 0) {
        const int f1 = fixedbit(q1);
        diag_reg1_j<kRev, false>(j0, f1 ? d2 : d0, f1 ? d3 : d1, a, l, acc);
      } else if (j1 >= 0) {
        const int f0 = fixedbit(q0);
        diag_reg1_j<kRev, false>(j1, f0 ? d1 : d0, f0 ? d3 : d2, a, l, acc);
      } else {
        const int v = fixedbit(q0) + 2 * fixedbit(q1);
        const float2 dd = v == 0 ? d0 : v == 1 ? d1 : v == 2 ? d2 : d3;
        if (dd.x != 1.f || dd.y != 0.f) {
#pragma unroll
          for (int i = 0; i < kRegs; ++i) {
            a[i] = cmul(dd, a[i]);
            if (kRev) l[i] = cmul(dd, l[i]);
          }
        }
      }
    }
  } else if (kind == BG_2Q) {
    // one operand in registers, the other fixed (block-diagonal in it): its 2x2 block
    auto M = [&](int r, int c) { return kRev ? cconj(gfull->u[4 * c + r]) : gfull->u[4 * r + c]; };
    if (r1 >= 0) {
      const int f = fixedbit(q0);
      pairs_reg_j<kRev>(r1, 0, M(f, f), M(f, f + 2), M(f + 2, f), M(f + 2, f + 2), a, l, acc);
    } else {
      const int f = fixedbit(q1);
      pairs_reg_j<kRev>(r0, 0, M(2 * f, 2 * f), M(2 * f, 2 * f + 1), M(2 * f + 1, 2 * f),
                        M(2 * f + 1, 2 * f + 1), a, l, acc);
    }
  }
  if (kRev && gen) warp_addf(acc, gout + gref.grad);
}

// All register phases of a pass on the staged group (kRev: phases and gates in reverse).
// Shared-memory layout: local index l at A[swz64(l)] (L likewise).
template <bool kRev>
__device__ void run_phases(const BatchGate* gates, const BatchPhase* phs, int nph, float2* A, float2* L, int m,
                           uint64_t gb, const int8_t* loc, int8_t* reg, double* gout, const GateLite* sg, int gfirst,
                           int ncached, int npass_gates) {
  // gates past the shared-memory cache look their register bits up in reg[] (rebuilt per phase)
  const bool all_cached = ncached >= npass_gates;
  for (int hh = 0; hh < nph; ++hh) {
    const BatchPhase& ph = phs[kRev ? nph - 1 - hh : hh];
    const int nr = ph.nr;
    if (!all_cached) {
      if ((int)threadIdx.x < kBatchMaxQubits) {
        const int q = threadIdx.x;
        int r = -1;
        for (int j = 0; j < nr; ++j)
          if (loc[q] >= 0 && ph.rbit[j] == loc[q]) r = j;
        reg[q] = (int8_t)r;
      }
      __syncthreads();
    }
    uint32_t RB[kBatchRegBits];
#pragma unroll
    for (int j = 0; j < kBatchRegBits; ++j) RB[j] = j < nr ? swz64(1u << ph.rbit[j]) : 0u;
    const int nt = m - nr;
    const int nslots = 1 << nt;
    for (int s0 = 0; s0 < nslots; s0 += blockDim.x) {
      const int slot = s0 + (int)threadIdx.x;
      const bool act = slot < nslots;
      uint32_t base = 0;
      for (int j = 0; j < nt; ++j)
        if ((slot >> j) & 1) base |= 1u << ph.tbit[j];
      const uint32_t sb = swz64(base);
      float2 a[kRegs], l[kRegs];
#pragma unroll
      for (int i = 0; i < kRegs; ++i) {
        uint32_t o = sb;
#pragma unroll
        for (int j = 0; j < kBatchRegBits; ++j) if ((i >> j) & 1) o ^= RB[j];
        // registers beyond 2^nr (small passes) and inactive slots hold zeros
        const bool use = act && (i >> nr) == 0;
        a[i] = use ? A[o] : make_float2(0.f, 0.f);
        l[i] = (kRev && use) ? L[o] : make_float2(0.f, 0.f);
      }
      for (int k = 0; k < ph.ngate; ++k) {
        const int gi = kRev ? ph.gate0 + ph.ngate - 1 - k : ph.gate0 + k;
        const int li = gi - gfirst;
        if (li >= 0 && li < ncached) {
          const GateLite& c = sg[li];
          gate_reg<kRev>(c, gates + gi, c.r0, c.r1, c.l0, c.l1, base, gb, a, l, gout);
        } else {
          const BatchGate& g = gates[gi];
          const int two = g.kind == BG_DIAG2 || g.kind == BG_2Q;
          gate_reg<kRev>(g, gates + gi, reg[g.q0], two ? reg[g.q1] : -1, loc[g.q0], two ? loc[g.q1] : -1, base, gb,
                         a, l, gout);
        }
      }
#pragma unroll
      for (int i = 0; i < kRegs; ++i) {
        uint32_t o = sb;
#pragma unroll
        for (int j = 0; j < kBatchRegBits; ++j) if ((i >> j) & 1) o ^= RB[j];
        if (act && (i >> nr) == 0) {
          A[o] = a[i];
          if (kRev) L[o] = l[i];
        }
      }
    }
    __syncthreads();
  }
}

template <int NT>
__global__ void __launch_bounds__(NT, 512 / NT) batch_kernel(const uint8_t* __restrict__ prog, float2* __restrict__ arena,
                                                   double* __restrict__ grads, double* __restrict__ energy,
                                                   unsigned* __restrict__ ctl, uint64_t limit_ns) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ Block B;
  __shared__ BatchPhase s_ph[kBatchMaxPhases];   // register phases of the current pass
  __shared__ int8_t s_reg[kBatchMaxQubits];      // register bit of each qubit in the current phase
  __shared__ uint64_t s_dep[128 + 64];     // local index -> global offset (bits 0-6 | 7-12)
  __shared__ uint64_t s_gdep[128 + 128];   // group index -> global offset (bits 0-6 | 7-13)
  __shared__ double s_coef[2 * kBatchMaxQubits];
  __shared__ GateLite s_gate[kGateCache];  // the current pass's gates (register phases)
  __shared__ int s_item;

  const BatchHeader* hdr = reinterpret_cast<const BatchHeader*>(prog);
  const BatchInst* insts = reinterpret_cast<const BatchInst*>(prog + hdr->off_inst);
  const BatchPass* passes = reinterpret_cast<const BatchPass*>(prog + hdr->off_pass);
  const BatchGate* gates = reinterpret_cast<const BatchGate*>(prog + hdr->off_gate);
  const BatchItem* items = reinterpret_cast<const BatchItem*>(prog + hdr->off_item);
  const double* coef = reinterpret_cast<const double*>(prog + hdr->off_coef);
  const BatchPhase* phases_g = reinterpret_cast<const BatchPhase*>(prog + hdr->off_phase);
  float2* A = reinterpret_cast<float2*>(smem_raw);
  float2* L = A + (1u << hdr->mbuf);
  const unsigned t = threadIdx.x;
  if (t == 0) B.key = -1;

  for (;;) {
    if (t == 0) s_item = (int)atomicAdd(ctl, 1u);
    __syncthreads();
    const int item = s_item;
    if (item >= hdr->nitem) break;
    // ---- wait for the instance's earlier stages ----
    if (t == 0) {
      B.it = items[item];
      int ok = *(volatile unsigned*)(ctl + 1) == 0u;
      if (ok && B.it.need > 0) {
        volatile unsigned* done = ctl + 2 + B.it.inst;
        const uint64_t t0 = gtime();
        while (*done < (unsigned)B.it.need) {
          if (*(volatile unsigned*)(ctl + 1)) { ok = 0; break; }
          if (gtime() - t0 > limit_ns) { atomicExch(ctl + 1, (unsigned)DERR_BARRIER_TIMEOUT); ok = 0; break; }
          __nanosleep(128);
        }
      }
      __threadfence();
      B.ok = ok;
      const int key = B.it.inst * 4096 + (B.it.kind == BI_HAM ? 4095 : B.it.pass);
      if (ok && key != B.key) {
        B.in = insts[B.it.inst];
        if (B.it.kind != BI_HAM) B.ps = passes[B.in.pass0 + B.it.pass];
      }
    }
    __syncthreads();
    if (!B.ok) break;
    const int n = B.in.n;
    const int key = B.it.inst * 4096 + (B.it.kind == BI_HAM ? 4095 : B.it.pass);
    if (key != B.key) {
      // per-pass tables
      if (B.it.kind != BI_HAM) {
        const int m = B.ps.m, ng = n - m;
        if ((int)t < kBatchMaxQubits) B.loc[t] = -1;
        __syncthreads();
        if ((int)t < m) B.loc[B.ps.sbit[t]] = (int8_t)t;
        if ((int)t < B.ps.nphase && (int)t < kBatchMaxPhases) s_ph[t] = phases_g[B.ps.phase0 + t];
        for (int e = (int)t; e < 128 + 64; e += NT) {
          const int lvl = e >= 128, v = lvl ? e - 128 : e;
          uint64_t q = 0;
          for (int j = 0; j < 7; ++j) {
            const int lj = 7 * lvl + j;
            if (lj < m && ((v >> j) & 1)) q |= 1ull << B.ps.sbit[lj];
          }
          s_dep[e] = q;
        }
        for (int e = (int)t; e < 256; e += NT) {
          const int lvl = e >= 128, v = lvl ? e - 128 : e;
          uint64_t q = 0;
          for (int j = 0; j < 7; ++j) {
            const int gj = 7 * lvl + j;
            if (gj < ng && ((v >> j) & 1)) q |= 1ull << B.ps.gbit[gj];
          }
          s_gdep[e] = q;
        }
      }
      if ((int)t < 2 * n) s_coef[t] = coef[B.in.coef0 + t];
      if (B.it.kind != BI_HAM && B.ps.nphase > 0)
        for (int e = (int)t; e < B.ps.ngate && e < kGateCache; e += NT) {
          const BatchGate& g = gates[B.ps.gate0 + e];
          GateLite c;
          c.kind = g.kind; c.q0 = g.q0; c.q1 = g.q1; c.gen = g.gen; c.grad = g.grad;
          // the gate's phase and its operands' local / register bits (from the pass descriptors)
          int h = 0;
          while (h + 1 < B.ps.nphase && phases_g[B.ps.phase0 + h + 1].gate0 <= B.ps.gate0 + e) ++h;
          const BatchPhase& gph = phases_g[B.ps.phase0 + h];
          auto local_of = [&](int q) {
            for (int j = 0; j < B.ps.m; ++j)
              if (B.ps.sbit[j] == q) return j;
            return -1;
          };
          auto reg_of = [&](int lb) {
            for (int j = 0; j < gph.nr && lb >= 0; ++j)
              if (gph.rbit[j] == lb) return j;
            return -1;
          };
          const bool two = g.kind == BG_DIAG2 || g.kind == BG_2Q;
          c.l0 = (int8_t)local_of(g.q0);
          c.l1 = (int8_t)(two ? local_of(g.q1) : -1);
          c.r0 = (int8_t)reg_of(c.l0);
          c.r1 = (int8_t)(two ? reg_of(c.l1) : -1);
#pragma unroll
          for (int k = 0; k < 4; ++k) c.u[k] = g.u[k];
          s_gate[e] = c;
        }
      __syncthreads();
      if (t == 0) B.key = key;
    }
    const BatchItem& it = B.it;
    double* gout = grads + B.in.grad0;

    const bool regs = it.kind != BI_HAM && B.ps.nphase > 0;
    if (it.kind == BI_SMALL) {
      const int dim = 1 << n;
      // |0...0>: index 0 is index 0 in the swizzled layout too
      for (int x = (int)t; x < dim; x += NT) A[x] = make_float2(x == 0 ? 1.f : 0.f, 0.f);
      __syncthreads();
      const BatchGate* gs = gates + B.ps.gate0;
      if (regs) {
        run_phases<false>(gates, s_ph, B.ps.nphase, A, L, n, 0, B.loc, s_reg, nullptr, s_gate, B.ps.gate0,
                          min(B.ps.ngate, kGateCache), B.ps.ngate);
        const double e = hamiltonian<false, true>(A, L, n, 0, (uint64_t)dim, s_coef, s_coef + n);
        warp_add(e, energy + it.inst);
        __syncthreads();
        run_phases<true>(gates, s_ph, B.ps.nphase, A, L, n, 0, B.loc, s_reg, gout, s_gate, B.ps.gate0,
                         min(B.ps.ngate, kGateCache), B.ps.ngate);
      } else {
        for (int k = 0; k < B.ps.ngate; ++k) apply_gate<false>(gs[k], A, L, n, 0, B.loc, nullptr);
        const double e = hamiltonian<false>(A, L, n, 0, (uint64_t)dim, s_coef, s_coef + n);
        warp_add(e, energy + it.inst);
        __syncthreads();
        for (int k = B.ps.ngate - 1; k >= 0; --k) apply_gate<true>(gs[k], A, L, n, 0, B.loc, gout + gs[k].grad);
      }
    } else if (it.kind == BI_HAM) {
      const float2* psi = arena + B.in.psi;
      float2* lam = arena + B.in.lam;
      const uint64_t chunk = 1ull << B.in.m;
      const double e = hamiltonian<true>(psi, lam, n, (uint64_t)it.first * chunk,
                                         (uint64_t)(it.first + it.count) * chunk, s_coef, s_coef + n);
      warp_add(e, energy + it.inst);
    } else {
      const bool rev = it.kind == BI_BWD;
      const int m = B.ps.m;
      float2* psi = arena + B.in.psi;
      float2* lam = arena + B.in.lam;
      const BatchGate* gs = gates + B.ps.gate0;
      const uint32_t pairs = 1u << (m - 1);
      for (int g = it.first; g < it.first + it.count; ++g) {
        const uint64_t gb = s_gdep[g & 127] | s_gdep[128 + (g >> 7)];
        // register phases keep the group at A[swz64(l)] (pairs of local bit 0 stay adjacent)
        auto sidx = [&](uint32_t l) -> uint32_t { return regs ? swz64(l) : l; };
        if (!rev && it.pass == 0) {
          for (uint32_t x = t; x < (1u << m); x += NT) A[x] = make_float2((gb == 0 && x == 0) ? 1.f : 0.f, 0.f);
        } else {
          for (uint32_t v = t; v < pairs; v += NT) {
            const uint32_t l = v << 1;
            const uint64_t off = gb | s_dep[l & 127] | s_dep[128 + (l >> 7)];
            cp16(A + sidx(l), psi + off);
            if (rev) cp16(L + sidx(l), lam + off);
          }
          cp_wait_all();
        }
        __syncthreads();
        if (regs) {
          if (!rev) run_phases<false>(gates, s_ph, B.ps.nphase, A, L, m, gb, B.loc, s_reg, nullptr, s_gate, B.ps.gate0,
                                      min(B.ps.ngate, kGateCache), B.ps.ngate);
          else run_phases<true>(gates, s_ph, B.ps.nphase, A, L, m, gb, B.loc, s_reg, gout, s_gate, B.ps.gate0,
                                    min(B.ps.ngate, kGateCache), B.ps.ngate);
        } else if (!rev) {
          for (int k = 0; k < B.ps.ngate; ++k) apply_gate<false>(gs[k], A, L, m, gb, B.loc, nullptr);
        } else {
          for (int k = B.ps.ngate - 1; k >= 0; --k) apply_gate<true>(gs[k], A, L, m, gb, B.loc, gout + gs[k].grad);
        }
        for (uint32_t v = t; v < pairs; v += NT) {
          const uint32_t l = v << 1;
          const uint64_t off = gb | s_dep[l & 127] | s_dep[128 + (l >> 7)];
          __stcg(reinterpret_cast<float4*>(psi + off), *reinterpret_cast<const float4*>(A + sidx(l)));
          if (rev) __stcg(reinterpret_cast<float4*>(lam + off), *reinterpret_cast<const float4*>(L + sidx(l)));
        }
        __syncthreads();
      }
    }
    // ---- publish completion ----
    __threadfence();
    __syncthreads();
    if (t == 0) atomicAdd(ctl + 2 + it.inst, 1u);
  }
}

template <int NT>
cudaError_t launch_t(const uint8_t* d_prog, void* arena, double* grads, double* energy, unsigned* ctl, int mbuf,
                     int blocks_per_sm_cap, uint64_t limit_ns, cudaStream_t s, int* grid_out) {
  const size_t smem = (size_t)2 * (sizeof(float2) << mbuf);
  auto kern = batch_kernel<NT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (blocks_per_sm_cap > 0 && per_sm > blocks_per_sm_cap) per_sm = blocks_per_sm_cap;
  const int grid = per_sm * device_sm_count();
  if (grid_out) *grid_out = grid;
  float2* ar = reinterpret_cast<float2*>(arena);
  void* args[] = {(void*)&d_prog, (void*)&ar, (void*)&grads, (void*)&energy, (void*)&ctl, (void*)&limit_ns};
  return cudaLaunchCooperativeKernel((void*)kern, dim3(grid), dim3(NT), args, smem, s);
}

}  // namespace

cudaError_t launch_batch(const uint8_t* d_prog, void* arena, double* grads, double* energy, unsigned* ctl,
                         int threads, int mbuf, int blocks_per_sm_cap, uint64_t limit_ns, cudaStream_t s,
                         int* grid_out) {
  if (mbuf < 1 || mbuf > kBatchMaxLocal) return cudaErrorInvalidValue;
  if (threads == 512)
    return launch_t<512>(d_prog, arena, grads, energy, ctl, mbuf, blocks_per_sm_cap, limit_ns, s, grid_out);
  if (threads == 256)
    return launch_t<256>(d_prog, arena, grads, energy, ctl, mbuf, blocks_per_sm_cap, limit_ns, s, grid_out);
  return cudaErrorInvalidValue;
}

}  // namespace qsb
