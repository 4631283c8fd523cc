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

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/qsim_b200.h"
#include "abi_ops.h"
#include "kernels.h"
#include "pass_body.cuh"
#include "plan.h"
#include "qsim.h"

namespace qsb {

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
// generic pass kernel: gate instructions interpreted from the program
// ------------------------------------------------------------------------------------
struct InterpExec {
  static constexpr bool kPacked = false;  // registers hold interleaved complex values
  template <typename Real, int LR>
  __device__ __forceinline__ static void reg_offsets(const PhaseDesc* ph, int, uint32_t (&B8)[LR]) {
#pragma unroll
    for (int j = 0; j < LR; ++j) B8[j] = swz<Real>(1u << ph->rbit[j]) * (uint32_t)sizeof(typename V2<Real>::T);
  }
  template <int LR>
  __device__ __forceinline__ static int pair_reg(const PhaseDesc* ph, int) {
#pragma unroll
    for (int j = 0; j < LR; ++j)
      if (ph->rbit[j] == 0) return j;
    return -1;
  }
  template <typename C, int LR>
  __device__ __forceinline__ static uint32_t run(const uint8_t* prog, const PhaseDesc* ph, int, int,
                                                 C (&a)[1 << LR], uint64_t pb) {
    const ProgramHeader* hdr = reinterpret_cast<const ProgramHeader*>(prog);
    const GateInstr* gates = reinterpret_cast<const GateInstr*>(prog + hdr->off_gate) + ph->gate0;
    const C* coef = reinterpret_cast<const C*>(prog + hdr->off_coef);
    const int ng = ph->ngate;
    for (int gi = 0; gi < ng; ++gi) {
      const GateInstr gin = gates[gi];
      apply_gate<C, LR>(gin, a, coef, pb);
    }
    return 0u;  // gates move data in the registers: nothing left flipped
  }
};

template <typename Real, int LR>
__global__ void __launch_bounds__(kPassThreads, 1)
pass_kernel(const uint8_t* __restrict__ prog, typename V2<Real>::T* __restrict__ psi, int pass_begin,
            int pass_end, unsigned* bar, unsigned* err, uint64_t barrier_limit_ns) {
  pass_body<Real, LR, InterpExec>(InterpExec{}, prog, psi, pass_begin, pass_end, bar, err, barrier_limit_ns);
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
    cudaFuncSetAttribute(pass_kernel<float, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pass_kernel<float, 5>, threads, smem);
  }
  cudaFuncSetAttribute(pass_kernel<double, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pass_kernel<double, 4>, threads, smem);
}

// ------------------------------------------------------------------------------------
// Allocation-free entry point.  The pass kernel's scratch (the encoded program and the
// grid-barrier / error words) lives in a fixed device array of this file instead of
// buffers allocated per state, for callers that cannot allocate device memory.
// ------------------------------------------------------------------------------------
constexpr size_t kWorkspaceBytes = size_t(1) << 20;  // 1 MiB: control words + program
constexpr size_t kWorkspaceCtl = 256;                // barrier (2 words) + error word, padded
static __device__ __align__(256) unsigned char g_workspace[kWorkspaceBytes];

// variant of the pass kernel whose program and control words sit in g_workspace
template <typename Real, int LR>
__global__ void __launch_bounds__(kPassThreads, 1)
pass_kernel_ws(const uint8_t* __restrict__ prog, typename V2<Real>::T* __restrict__ psi, int pass_begin,
               int pass_end, unsigned* bar, unsigned* err, uint64_t barrier_limit_ns) {
  pass_body<Real, LR, InterpExec>(InterpExec{}, prog, psi, pass_begin, pass_end, bar, err, barrier_limit_ns);
}

namespace {

// Device address of g_workspace for the current device, looked up once per device (the host
// symbol g_workspace is not a device address and must never be handed to a kernel).
cudaError_t workspace_address(unsigned char** out) {
  static std::mutex mu;
  static unsigned char* addr[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_workspace);
    if (e != cudaSuccess) return e;
    addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = addr[dev];
  return cudaSuccess;
}

template <typename Real, int LR>
cudaError_t launch_ws(const uint8_t* prog, void* psi, int npass, int threads, size_t smem, unsigned* bar,
                      unsigned* err, uint64_t limit_ns, cudaStream_t stream) {
  auto kern = pass_kernel_ws<Real, LR>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int grid = per_sm * device_sm_count();
  using C = typename V2<Real>::T;
  C* p = reinterpret_cast<C*>(psi);
  int b = 0;
  void* args[] = {(void*)&prog, (void*)&p, (void*)&b, (void*)&npass, (void*)&bar, (void*)&err, (void*)&limit_ns};
  return cudaLaunchCooperativeKernel((void*)kern, dim3(grid), dim3(threads), args, smem, stream);
}

}  // namespace

}  // namespace qsb

extern "C" QS_API int qs_apply_ops_noalloc(void* psi, int dtype, int num_qubits, const qs_op* ops, int nops,
                                          void* stream) {
  using namespace qsb;
  const char* kWho = "qs_apply_ops_noalloc";
  auto fail = [&](const std::string& m) {
    set_last_error(m);
    return QS_ERR_INVALID;
  };
  auto cuda_fail = [&](cudaError_t e) {
    set_last_error(std::string("CUDA error: ") + cudaGetErrorString(e));
    return QS_ERR_CUDA;
  };
  if (!psi || (nops > 0 && !ops)) return fail(std::string(kWho) + ": null argument");
  if (dtype != QS_C64 && dtype != QS_C128) return fail(std::string(kWho) + ": dtype must be QS_C64 or QS_C128");
  // the sweep kernel moves the state in 16-byte units
  if (reinterpret_cast<uintptr_t>(psi) & 15u)
    return fail(std::string(kWho) + ": psi must be 16-byte aligned");
  const int r = dtype == 0 ? 5 : 4;
  if (num_qubits < r + 1 || num_qubits > 36)
    return fail(std::string(kWho) + ": num_qubits must be in [" + std::to_string(r + 1) + ", 36]");
  if (nops < 0) return fail(std::string(kWho) + ": invalid op list");
  if (nops == 0) return 0;
  try {
    // psi must be device (or managed) memory that the current device can address
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e);
    cudaPointerAttributes attr{};
    e = cudaPointerGetAttributes(&attr, psi);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(std::string(kWho) + ": psi is not a device pointer");
    }
    if (!(attr.type == cudaMemoryTypeManaged || (attr.type == cudaMemoryTypeDevice && attr.device == dev)))
      return fail(std::string(kWho) + ": psi must be device memory of the current device");
    std::vector<QOp> q = convert_abi_ops(ops, nops, num_qubits, dtype, kWho, nullptr, false);
    std::vector<COp> cops;
    cops.reserve(q.size());
    for (const QOp& o : q) cops.push_back(classify(o));
    PlanConfig pc;
    pc.r = r;
    pc.m = std::max(r, std::min(dtype == 0 ? 13 : 12, num_qubits));
    const auto passes = plan_passes(cops, num_qubits, pc);
    const Program prog = build_program(q, passes, num_qubits, dtype, r);
    if (prog.bytes.size() > kWorkspaceBytes - kWorkspaceCtl)
      return fail(std::string(kWho) + ": the program of these ops needs " + std::to_string(prog.bytes.size()) +
                  " bytes; the static workspace holds " + std::to_string(kWorkspaceBytes - kWorkspaceCtl) +
                  " (split the ops into smaller calls)");
    unsigned char* ws = nullptr;
    if ((e = workspace_address(&ws)) != cudaSuccess) return cuda_fail(e);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned* ctl = reinterpret_cast<unsigned*>(ws);
    // the barrier and error words must start at zero for every call
    if ((e = cudaMemsetAsync(ctl, 0, kWorkspaceCtl, s)) != cudaSuccess) return cuda_fail(e);
    if ((e = cudaMemcpyAsync(ws + kWorkspaceCtl, prog.bytes.data(), prog.bytes.size(), cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
      return cuda_fail(e);
    e = dtype == 0 ? launch_ws<float, 5>(ws + kWorkspaceCtl, psi, prog.npass, prog.threads, prog.max_smem, ctl,
                                          ctl + 2, kDeviceWaitLimitNs, s)
                   : launch_ws<double, 4>(ws + kWorkspaceCtl, psi, prog.npass, prog.threads, prog.max_smem, ctl,
                                           ctl + 2, kDeviceWaitLimitNs, s);
    if (e != cudaSuccess) return cuda_fail(e);
    unsigned word = 0;
    if ((e = cudaMemcpyAsync(&word, ctl + 2, sizeof(word), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return cuda_fail(e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e);
    if (word != 0) {
      set_last_error(std::string(kWho) + ": device error: " + device_error_name(word) + " (error word " +
                     std::to_string(word) + ")");
      return QS_ERR_DEVICE;
    }
  } catch (const std::exception& ex) {
    return fail(ex.what());
  } catch (...) {
    return fail(std::string(kWho) + ": unexpected error");
  }
  return 0;
}
