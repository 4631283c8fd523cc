// State handle and C ABI of libqsim_b200 (see include/qsim_b200.h).
//
// Execution model
//  * permute() only relabels: pos2bit[p] is the physical bit that holds layout position p.
//  * Tile ops in cooperative/graphed mode are queued at physical bits and run when the
//    state is next observed (copy-out, synchronize, device pointer, reductions) or when a
//    sequential op arrives.  The queue is planned into passes (pass kernel); cooperative
//    mode runs all passes in one persistent launch with bounded grid barriers, graphed
//    mode replays a cached CUDA graph of one launch per pass.
//  * Observation first moves the data to the current layout with in-place permutation
//    passes (bit-exact), so pos2bit becomes the identity.
#include <algorithm>
#include <atomic>
#include <complex>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/qsim_b200.h"
#include "abi_ops.h"
#include "kernels.h"
#include "jit.h"
#include "plan.h"
#include "qsim.h"

using namespace qsb;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

struct CudaError {
  cudaError_t e;
};

#define CK(call)                                    \
  do {                                              \
    cudaError_t _e = (call);                        \
    if (_e != cudaSuccess) throw CudaError{_e};     \
  } while (0)

struct InvalidArg {
  std::string msg;
};

// a kernel reported an error word (QS_ERR_DEVICE); the state stays usable
struct DeviceFault {
  std::string msg;
};

// a status returned by one of this library's own entry points, passed on unchanged
struct Status {
  int code;
  std::string msg;
};

constexpr uint64_t kBarrierLimitNs = kDeviceWaitLimitNs;

int reg_bits(int dtype) { return dtype == 0 ? 5 : 4; }

}  // namespace

namespace qsb {
void set_last_error(const std::string& msg) { g_err = msg; }

// allocation fault injection: 0 = off, k > 0 = the k-th next allocation fails
static std::atomic<long long> g_fail_alloc{0};

static bool inject_alloc_failure() {
  long long c = g_fail_alloc.load();
  while (c > 0 && !g_fail_alloc.compare_exchange_weak(c, c - 1)) {
  }
  return c == 1;
}

cudaError_t dev_malloc(void** p, size_t bytes) {
  if (inject_alloc_failure()) return cudaErrorMemoryAllocation;
  return cudaMalloc(p, bytes);
}
cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t s) {
  if (inject_alloc_failure()) return cudaErrorMemoryAllocation;
  return cudaMallocAsync(p, bytes, s);
}
cudaError_t host_malloc(void** p, size_t bytes) {
  if (inject_alloc_failure()) return cudaErrorMemoryAllocation;
  return cudaMallocHost(p, bytes);
}
}  // namespace qsb


struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
  uint64_t key = 0;        // structure, state and program buffer, grid
  uint64_t values = 0;     // coefficient values baked into the launch parameters (specialised kernels)
  std::shared_ptr<JitKernels> kernels;
};

// FNV-1a of the program's coefficient table
uint64_t coef_values_hash(const Program& prog) {
  const ProgramHeader* hdr = (const ProgramHeader*)prog.bytes.data();
  uint64_t h = 1469598103934665603ull;
  for (size_t i = (size_t)hdr->off_coef; i < prog.bytes.size(); ++i) {
    h ^= prog.bytes[i];
    h *= 1099511628211ull;
  }
  return h;
}

struct qs_state {
  int n = 0;
  int dtype = 0;
  size_t esz = 8;
  uint64_t dim = 0;
  void* psi = nullptr;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  std::vector<int> pos2bit;
  std::vector<QOp> queue;
  int queue_mode = QS_MODE_COOPERATIVE;
  PlanConfig cfg;
  int grid_mult = 0;
  int jit_mode = 0;        // 0 auto (complex64, n >= 20, graphed), 1 always, -1 never
  int jit_lr = 5;          // register bits per thread of the specialised kernels
  int jit_packed = 0;      // FP32x2 arithmetic in the specialised kernels
  int jit_async = 0;       // generic kernels stand in while a structure's specialised kernels compile
  int jit_blocks = 2;      // resident blocks per SM of the specialised kernels (single-buffered
                           // blocks that overlap each other's group loads)
  uint64_t wait_limit_ns = kBarrierLimitNs;  // bounded device waits of the pass kernel's grid
                                             // barriers and the tensor-core kernel
  // device scratch: program buffer, control words (barrier x2, error), accumulators
  uint8_t* d_prog = nullptr;
  size_t prog_cap = 0;
  struct Slot {            // pinned staging of an encoded program
    uint8_t* host = nullptr;
    size_t cap = 0;
    cudaEvent_t done = nullptr;
  };
  static constexpr int kSlots = 4;
  Slot slots[kSlots];
  int next_slot = 0;
  unsigned* d_ctl = nullptr;
  double* d_acc = nullptr;
  double* h_acc = nullptr;    // pinned
  GraphEntry graph;
  std::vector<std::pair<uint64_t, std::pair<size_t, std::vector<PlannedPass>>>> plan_cache;
  qs_stats st{};
  void* d_dense = nullptr;    // tensor-core operand of the last dense 6-qubit unitary

  ~qs_state() {
    if (graph.exec) cudaGraphExecDestroy(graph.exec);
    if (d_dense) cudaFree(d_dense);
    if (psi) cudaFree(psi);
    if (d_prog) cudaFree(d_prog);
    for (Slot& s : slots) {
      if (s.host) cudaFreeHost(s.host);
      if (s.done) cudaEventDestroy(s.done);
    }
    if (h_acc) cudaFreeHost(h_acc);
    if (d_ctl) cudaFree(d_ctl);
    if (d_acc) cudaFree(d_acc);
    if (stream && own_stream) cudaStreamDestroy(stream);
  }

  bool identity_layout() const {
    for (int p = 0; p < n; ++p) if (pos2bit[p] != p) return false;
    return true;
  }

  void ensure_prog(size_t bytes) {
    if (bytes > prog_cap) {
      CK(cudaStreamSynchronize(stream));
      if (d_prog) CK(cudaFree(d_prog));
      d_prog = nullptr;
      prog_cap = 0;
      const size_t cap = std::max<size_t>(bytes * 2, 1 << 16);
      CK(dev_malloc((void**)&d_prog, cap));
      prog_cap = cap;
      if (graph.exec) { cudaGraphExecDestroy(graph.exec); graph.exec = nullptr; }
    }
  }

  // Copy the encoded program to the device, ordered on the stream.  The pinned staging
  // is a ring of slots so the host can prepare the next launches while earlier copies
  // are still queued behind running kernels.
  void upload(const Program& prog) {
    const size_t bytes = prog.bytes.size();
    ensure_prog(bytes);
    Slot& s = slots[next_slot];
    next_slot = (next_slot + 1) % kSlots;
    if (!s.done) CK(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
    CK(cudaEventSynchronize(s.done));  // the copy that last used this slot has run
    if (bytes > s.cap) {
      if (s.host) CK(cudaFreeHost(s.host));
      s.host = nullptr;
      s.cap = 0;
      const size_t cap = std::max<size_t>(bytes * 2, 1 << 16);
      CK(host_malloc((void**)&s.host, cap));
      s.cap = cap;
    }
    std::memcpy(s.host, prog.bytes.data(), bytes);
    CK(cudaMemcpyAsync(d_prog, s.host, bytes, cudaMemcpyHostToDevice, stream));
    CK(cudaEventRecord(s.done, stream));
  }

  int grid_for_program(const Program& prog) {
    int per_sm = 1;
    CK(pass_kernel_occupancy(dtype, prog.threads, prog.max_smem, &per_sm));
    if (per_sm < 1) throw InvalidArg{"pass kernel does not fit on an SM"};
    if (grid_mult > 0) per_sm = std::min(per_sm, grid_mult);
    return per_sm * device_sm_count();
  }

  // whether the next graphed flush of gates uses the specialised kernels
  bool want_jit() const {
    if (dtype != 0 || queue_mode != QS_MODE_GRAPHED) return false;
    if (jit_mode < 0 || (jit_mode == 0 && n < 20)) return false;
    std::string why;
    if (jit_available(&why)) return true;
    if (jit_mode > 0) throw InvalidArg{"jit requested but unavailable: " + why};
    return false;
  }

  void run_program(const Program& prog, int mode, bool use_jit = false) {
    if (prog.npass == 0) return;
    upload(prog);
    std::shared_ptr<JitKernels> jk;
    if (use_jit && mode != QS_MODE_COOPERATIVE) {
      JitConfig jc;
      jc.blocks = jit_blocks;
      jc.packed = jit_packed != 0;
      // while the specialised kernels of a new structure compile, the generic kernel runs the
      // same program (it takes the plan of 5 register bits with interleaved registers)
      const bool stand_in = jit_async != 0 && jit_lr == 5 && jit_packed == 0;
      jk = stand_in ? jit_try_get(prog, jc) : jit_get(prog, jc);
      if (jk) {
        st.jit_compile_ms += (unsigned long long)(jk->compile_seconds * 1e3 + 0.5);
        st.jit_modules += (unsigned long long)jk->chunks;
        st.jit_disk_hits += (unsigned long long)jk->disk_hits;
        jk->compile_seconds = 0.0;  // counted once
        jk->chunks = 0;
        jk->disk_hits = 0;
      } else {
        st.jit_pending_flushes += 1;
      }
      use_jit = jk != nullptr;
    }
    const int grid = use_jit ? 0 : grid_for_program(prog);
    if (mode == QS_MODE_COOPERATIVE) {
      CK(cudaMemsetAsync(d_ctl, 0, 2 * sizeof(unsigned), stream));
      CK(launch_pass_kernel(dtype, d_prog, psi, 0, prog.npass, prog.threads, prog.max_smem, grid, true, d_ctl,
                            d_ctl + 2, wait_limit_ns, stream));
      st.launches += 1;
    } else {
      // specialised kernels for large complex64 states (compiled once per structure): jk
      const uint64_t skey = jk ? jk->key : prog.structure_hash;
      const uint64_t key = skey ^ ((uint64_t)(uintptr_t)psi * 0x9E3779B97F4A7C15ull) ^
                           ((uint64_t)(uintptr_t)d_prog << 1) ^ (uint64_t)grid ^ (jk ? 0x5bd1e995ull : 0ull);
      // the specialised kernels take the coefficient values as launch parameters, which the
      // graph holds: same structure with other values updates the executable graph in place
      const uint64_t values = jk ? coef_values_hash(prog) : 0;
      const uint8_t* host_coef = prog.bytes.data() + ((const ProgramHeader*)prog.bytes.data())->off_coef;
      auto capture = [&]() {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int p = 0; p < prog.npass && e == cudaSuccess; ++p)
          e = jk ? jit_launch(*jk, p, d_prog, host_coef, psi, d_ctl + 2, prog.threads, prog.max_smem,
                              device_sm_count(), stream)
                 : launch_pass_kernel(dtype, d_prog, psi, p, p + 1, prog.threads, prog.max_smem, grid, false,
                                      d_ctl, d_ctl + 2, wait_limit_ns, stream);
        cudaError_t e2 = cudaStreamEndCapture(stream, &g);
        if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); throw CudaError{e}; }
        if (e2 != cudaSuccess) throw CudaError{e2};
        return g;
      };
      bool updated = false;
      if (graph.exec && graph.key == key && graph.values != values) {
        cudaGraph_t g = capture();
        cudaGraphExecUpdateResultInfo info;
        const cudaError_t eu = cudaGraphExecUpdate(graph.exec, g, &info);
        cudaGraphDestroy(g);
        if (eu == cudaSuccess) {
          graph.values = values;
          st.graph_builds += 1;
          updated = true;
        } else {
          cudaGetLastError();  // clear the update error; rebuild below
          CK(cudaGraphExecDestroy(graph.exec));
          graph.exec = nullptr;
        }
      }
      if (!graph.exec || graph.key != key) {
        if (graph.exec) { CK(cudaGraphExecDestroy(graph.exec)); graph.exec = nullptr; }
        graph.kernels = jk;  // keep the modules alive while the graph exists
        cudaGraph_t g = capture();
        cudaError_t e3 = cudaGraphInstantiate(&graph.exec, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) throw CudaError{e3};
        graph.key = key;
        graph.values = values;
        st.graph_builds += 1;
      } else if (!updated) {
        st.graph_replays += 1;
      }
      CK(cudaGraphLaunch(graph.exec, stream));
      st.launches += 1;
    }
    st.sweeps += prog.npass;
  }

  bool use_pass_kernel() const { return n >= reg_bits(dtype) + 1; }

  PlanConfig eff_cfg() const {
    PlanConfig c = cfg;
    c.r = reg_bits(dtype);
    c.m = std::max(c.r, std::min(c.m, n));
    return c;
  }

  void run_ops_sequential(const std::vector<QOp>& ops) {
    for (const QOp& o : ops) {
      if (o.arity == 1) CK(launch_gate1(dtype, psi, n, o.q0, o.U, stream));
      else CK(launch_gate2(dtype, psi, n, o.q0, o.q1, o.U, stream));
      st.launches += 1;
      st.gate_sweeps += 1;
    }
  }

  void flush() {
    if (queue.empty()) return;
    std::vector<QOp> ops;
    ops.swap(queue);
    st.flushes += 1;
    if (!use_pass_kernel() || queue_mode == QS_MODE_SEQUENTIAL) {
      run_ops_sequential(ops);
      return;
    }
    std::vector<COp> cops;
    cops.reserve(ops.size());
    for (const QOp& o : ops) cops.push_back(classify(o));
    const bool use_jit = want_jit();
    PlanConfig c = eff_cfg();
    if (use_jit) {
      c.r = jit_lr;
      c.m = std::max(c.r, std::min(cfg.m, n));
      c.pair_bit = jit_packed != 0;  // packed kernels: local bit 0 in every phase's registers
    }
    // The plan depends on the gate classes and bits only, not on the matrix values:
    // repeated circuits (parameter sweeps, benchmark steps) reuse it.
    uint64_t key = 1469598103934665603ull;
    auto mix = [&key](uint64_t v) { key = (key ^ v) * 1099511628211ull; };
    mix((uint64_t)n); mix((uint64_t)dtype); mix((uint64_t)c.m); mix((uint64_t)c.k); mix((uint64_t)c.hill_iters);
    mix((uint64_t)c.r);
    mix((uint64_t)c.pair_bit);
    for (const COp& o : cops) mix(((uint64_t)o.kind << 16) | ((uint64_t)(o.a & 0xff) << 8) | (uint64_t)(o.b & 0xff));
    const std::vector<PlannedPass>* passes = nullptr;
    for (auto& e : plan_cache)
      if (e.first == key && e.second.first == cops.size()) { passes = &e.second.second; break; }
    if (!passes) {
      if (plan_cache.size() >= 4) plan_cache.erase(plan_cache.begin());
      plan_cache.emplace_back(key, std::make_pair(cops.size(), plan_passes(cops, n, c)));
      passes = &plan_cache.back().second.second;
      st.plans += 1;
    }
    Program prog = build_program(ops, *passes, n, dtype, c.r);
    run_program(prog, queue_mode, use_jit);
  }

  // move data so that physical bit p holds layout position p
  void materialize() {
    flush();
    if (identity_layout()) return;
    std::vector<int> perm(n);
    for (int p = 0; p < n; ++p) perm[pos2bit[p]] = p;
    if (!use_pass_kernel()) {
      // tiny states: out-of-place scatter through a temporary buffer
      AsyncBuf tmp(stream);
      CK(tmp.alloc(dim * esz));
      CK(launch_permute_scatter(dtype, psi, tmp.p, n, perm.data(), stream));
      CK(cudaMemcpyAsync(psi, tmp.p, dim * esz, cudaMemcpyDeviceToDevice, stream));
      st.launches += 1;
    } else {
      PlanConfig c = eff_cfg();
      auto passes = plan_permutation(perm, n, c);
      std::vector<COp> none;
      Program prog = encode_program(passes, none, n, dtype);
      run_program(prog, QS_MODE_COOPERATIVE);
      st.perm_sweeps += prog.npass;
    }
    for (int p = 0; p < n; ++p) pos2bit[p] = p;
  }

  void check_device_error() {
    unsigned w[3] = {0, 0, 0};
    CK(cudaMemcpyAsync(w, d_ctl, sizeof(w), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    if (w[2] != 0) {
      CK(cudaMemsetAsync(d_ctl, 0, 3 * sizeof(unsigned), stream));
      CK(cudaStreamSynchronize(stream));
      throw DeviceFault{"device error: " + std::string(device_error_name(w[2])) + " (error word " +
                        std::to_string(w[2]) + ")"};
    }
  }

  void sync() {
    flush();
    CK(cudaStreamSynchronize(stream));
    check_device_error();
  }
};

// ------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------
namespace {

template <typename F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const InvalidArg& e) {
    return fail(QS_ERR_INVALID, e.msg);
  } catch (const DeviceFault& e) {
    return fail(QS_ERR_DEVICE, e.msg);
  } catch (const Status& e) {
    return fail(e.code, e.msg);
  } catch (const CudaError& e) {
    return fail(QS_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e.e));
  } catch (const std::exception& e) {
    return fail(QS_ERR_INVALID, e.what());
  }
}

void read_matrix(const qs_state* s, int dtype, const void* U, int u_on_device, int count, cplx* out) {
  const size_t esz = dtype == 0 ? 8 : 16;
  std::vector<uint8_t> buf(count * esz);
  const void* src = U;
  if (u_on_device) {
    CK(cudaMemcpy(buf.data(), U, count * esz, cudaMemcpyDeviceToHost));
    src = buf.data();
  }
  if (dtype == 0) {
    const float* f = (const float*)src;
    for (int i = 0; i < count; ++i) out[i] = cplx(f[2 * i], f[2 * i + 1]);
  } else {
    const double* f = (const double*)src;
    for (int i = 0; i < count; ++i) out[i] = cplx(f[2 * i], f[2 * i + 1]);
  }
  (void)s;
}

}  // namespace

namespace qsb {

std::vector<QOp> convert_abi_ops(const qs_op* ops, int nops, int n, int dtype, const char* who, const int* pos2bit,
                                 bool allow_device) {
  const std::string w(who);
  std::vector<QOp> out;
  out.reserve(nops > 0 ? nops : 0);
  for (int i = 0; i < nops; ++i) {
    const qs_op& o = ops[i];
    QOp q;
    int count = 0;
    if (o.kind == QS_OP_1Q) {
      if (o.q0 < 0 || o.q0 >= n) throw std::invalid_argument(w + ": invalid q0");
      q.arity = 1;
      q.q0 = pos2bit ? pos2bit[o.q0] : o.q0;
      count = 4;
    } else if (o.kind == QS_OP_2Q) {
      if (o.q0 < 0 || o.q0 >= n || o.q1 < 0 || o.q1 >= n) throw std::invalid_argument(w + ": invalid q0/q1");
      if (o.q0 == o.q1) throw std::invalid_argument(w + ": q0 == q1");
      q.arity = 2;
      q.q0 = pos2bit ? pos2bit[o.q0] : o.q0;
      q.q1 = pos2bit ? pos2bit[o.q1] : o.q1;
      count = 16;
    } else {
      throw std::invalid_argument(w + ": unknown op kind: " + std::to_string(o.kind));
    }
    if (!o.U) throw std::invalid_argument(w + ": null gate matrix");
    if (o.u_on_device && !allow_device) throw std::invalid_argument(w + ": gate matrices must be host memory");
    read_matrix(nullptr, dtype, o.U, o.u_on_device, count, q.U);
    out.push_back(q);
  }
  return out;
}

}  // namespace qsb

namespace {

// the tile API's op list (validated as apply_tile_dev), at physical bits when map_layout
std::vector<QOp> convert_ops(const qs_state* s, const qs_op* ops, int nops, int n, int dtype, bool map_layout) {
  return convert_abi_ops(ops, nops, n, dtype, "apply_tile_dev", map_layout ? s->pos2bit.data() : nullptr, true);
}

void enqueue(qs_state* s, std::vector<QOp>&& ops, int mode) {
  if (ops.empty()) return;
  s->st.gates += ops.size();
  if (mode == QS_MODE_SEQUENTIAL) {
    s->flush();
    s->run_ops_sequential(ops);
    return;
  }
  if (!s->queue.empty() && s->queue_mode != mode) s->flush();
  s->queue_mode = mode;
  for (auto& o : ops) s->queue.push_back(o);
  if (s->queue.size() > 200000) s->flush();
}

}  // namespace

// ------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------
extern "C" {

const char* qs_last_error(void) { return g_err.c_str(); }

int qs_jit_wait(void) {
  return guard([&] { jit_wait_all(); });
}

int qs_debug_fail_alloc(int k) {
  g_fail_alloc.store(k > 0 ? k : 0);
  return 0;
}
int qs_version(void) { return 100; }

int qs_device_count(int* out) {
  return guard([&] {
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) c = 0;
    *out = c;
  });
}

int qs_create(int num_qubits, int dtype, qs_state** out) {
  return guard([&] {
    if (!out) throw InvalidArg{"null output handle"};
    *out = nullptr;
    if (dtype != QS_C64 && dtype != QS_C128) throw InvalidArg{"dtype must be QS_C64 or QS_C128"};
    if (num_qubits < 1 || num_qubits > 36) throw InvalidArg{"num_qubits must be in [1, 36]"};
    std::unique_ptr<qs_state> s(new qs_state());
    s->n = num_qubits;
    s->dtype = dtype;
    s->esz = dtype == 0 ? 8 : 16;
    s->dim = 1ull << num_qubits;
    s->cfg.m = dtype == 0 ? 13 : 12;
    s->cfg.k = 3;
    s->pos2bit.resize(num_qubits);
    for (int p = 0; p < num_qubits; ++p) s->pos2bit[p] = p;
    CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    CK(dev_malloc(&s->psi, s->dim * s->esz));
    CK(dev_malloc((void**)&s->d_ctl, 4 * sizeof(unsigned)));
    CK(dev_malloc((void**)&s->d_acc, 8 * sizeof(double)));
    CK(host_malloc((void**)&s->h_acc, 8 * sizeof(double)));
    CK(cudaMemsetAsync(s->d_ctl, 0, 4 * sizeof(unsigned), s->stream));
    CK(launch_set_basis(dtype, s->psi, num_qubits, 0, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    *out = s.release();
  });
}

int qs_destroy(qs_state* s) {
  return guard([&] {
    if (!s) return;
    cudaStreamSynchronize(s->stream);
    delete s;
  });
}

int qs_num_qubits(const qs_state* s, int* out) {
  return guard([&] { if (!s) throw InvalidArg{"null state"}; *out = s->n; });
}
int qs_dim(const qs_state* s, unsigned long long* out) {
  return guard([&] { if (!s) throw InvalidArg{"null state"}; *out = s->dim; });
}
int qs_dtype(const qs_state* s, int* out) {
  return guard([&] { if (!s) throw InvalidArg{"null state"}; *out = s->dtype; });
}

int qs_reset(qs_state* s) {
  return guard([&] {
    if (!s) throw InvalidArg{"null state"};
    s->queue.clear();
    for (int p = 0; p < s->n; ++p) s->pos2bit[p] = p;
    CK(launch_set_basis(s->dtype, s->psi, s->n, 0, s->stream));
    s->st.launches += 1;
  });
}

int qs_synchronize(qs_state* s) {
  return guard([&] {
    if (!s) throw InvalidArg{"null state"};
    s->sync();
  });
}

int qs_copy_to_host(qs_state* s, void* dst, unsigned long long nbytes) {
  return guard([&] {
    if (!s || !dst) throw InvalidArg{"null argument"};
    if (nbytes != s->dim * s->esz) throw InvalidArg{"Output array must have size 2^num_qubits"};
    s->materialize();
    CK(cudaMemcpyAsync(dst, s->psi, nbytes, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->check_device_error();
  });
}

int qs_copy_from_host(qs_state* s, const void* src, unsigned long long nbytes) {
  return guard([&] {
    if (!s || !src) throw InvalidArg{"null argument"};
    if (nbytes != s->dim * s->esz) throw InvalidArg{"Input array must have size 2^num_qubits"};
    s->flush();
    for (int p = 0; p < s->n; ++p) s->pos2bit[p] = p;
    CK(cudaMemcpyAsync(s->psi, src, nbytes, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
  });
}

int qs_permute(qs_state* s, const int* layout_old, const int* layout_new, int n) {
  return guard([&] {
    if (!s) throw InvalidArg{"null state"};
    if (n != s->n || !layout_old || !layout_new)
      throw InvalidArg{"layout_old/layout_new must have length num_qubits"};
    std::vector<int> new_pos(n, -1), old_seen(n, 0), map(n, -1);
    for (int p = 0; p < n; ++p) {
      int gq = layout_new[p];
      if (gq < 0 || gq >= n) throw InvalidArg{"layout_new contains invalid qubit id"};
      if (new_pos[gq] != -1) throw InvalidArg{"layout_new is not a permutation"};
      new_pos[gq] = p;
    }
    for (int p = 0; p < n; ++p) {
      int gq = layout_old[p];
      if (gq < 0 || gq >= n) throw InvalidArg{"layout_old contains invalid qubit id"};
      if (old_seen[gq]++) throw InvalidArg{"layout_old is not a permutation"};
      map[p] = new_pos[gq];
    }
    // scatter semantics: data at position p moves to position map[p]
    std::vector<int> nb(n);
    for (int p = 0; p < n; ++p) nb[map[p]] = s->pos2bit[p];
    s->pos2bit.swap(nb);
    s->st.permutes += 1;
  });
}

int qs_apply_tile(qs_state* s, const qs_op* ops, int nops, int mode) {
  return guard([&] {
    if (!s) throw InvalidArg{"null state"};
    if (mode < 0 || mode > 2) throw InvalidArg{"unknown tile mode"};
    if (nops < 0 || (nops > 0 && !ops)) throw InvalidArg{"invalid op list"};
    enqueue(s, convert_ops(s, ops, nops, s->n, s->dtype, true), mode);
  });
}

int qs_apply_1q(qs_state* s, int target_qubit, const void* U, int u_on_device) {
  return guard([&] {
    if (!s) throw InvalidArg{"null state"};
    if (target_qubit < 0 || target_qubit >= s->n) throw InvalidArg{"Invalid target qubit"};
    if (!U) throw InvalidArg{"U must be a 2x2 matrix"};
    qs_op o{QS_OP_1Q, target_qubit, -1, u_on_device, U};
    enqueue(s, convert_ops(s, &o, 1, s->n, s->dtype, true), QS_MODE_SEQUENTIAL);
  });
}

int qs_apply_2q(qs_state* s, int q0, int q1, const void* U, int u_on_device) {
  return guard([&] {
    if (!s) throw InvalidArg{"null state"};
    if (q0 < 0 || q0 >= s->n || q1 < 0 || q1 >= s->n) throw InvalidArg{"Invalid qubit indices"};
    if (q0 == q1) throw InvalidArg{"q0 and q1 must be different"};
    if (!U) throw InvalidArg{"U must be a 4x4 matrix"};
    qs_op o{QS_OP_2Q, q0, q1, u_on_device, U};
    enqueue(s, convert_ops(s, &o, 1, s->n, s->dtype, true), QS_MODE_SEQUENTIAL);
  });
}

int qs_apply_diagonal_1q(qs_state* s, int target_qubit, const double* phase0, const double* phase1) {
  return guard([&] {
    if (!s) throw InvalidArg{"null state"};
    if (target_qubit < 0 || target_qubit >= s->n) throw InvalidArg{"Invalid target qubit"};
    s->flush();
    CK(launch_diag1(s->dtype, s->psi, s->n, s->pos2bit[target_qubit], cplx(phase0[0], phase0[1]),
                    cplx(phase1[0], phase1[1]), s->stream));
    s->st.gates += 1;
    s->st.launches += 1;
    s->st.gate_sweeps += 1;
  });
}

int qs_flush(qs_state* s) {
  return guard([&] { if (!s) throw InvalidArg{"null state"}; s->flush(); });
}

int qs_materialize(qs_state* s) {
  return guard([&] { if (!s) throw InvalidArg{"null state"}; s->materialize(); });
}

int qs_sample(qs_state* s, unsigned long long shots, unsigned long long seed, unsigned long long* out) {
  return guard([&] {
    if (!s || (!out && shots)) throw InvalidArg{"null argument"};
    if (shots == 0) return;
    if (shots > (1ull << 31)) throw InvalidArg{"sample: at most 2^31 shots per call"};
    s->materialize();  // indices are layout (logical) indices
    AsyncBuf scratch(s->stream), d_out(s->stream);
    CK(scratch.alloc(sample_scratch_bytes(s->n, shots)));
    CK(d_out.alloc(shots * sizeof(uint64_t)));
    CK(launch_sample(s->dtype, s->psi, s->n, shots, seed, scratch.p, (uint64_t*)d_out.p, s->stream));
    CK(cudaMemcpyAsync(out, d_out.p, shots * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->st.launches += 5;
  });
}

int qs_dense6_weights(const double* U, void* out) {
  return guard([&] {
    if (!U || !out) throw InvalidArg{"null argument"};
    std::vector<cplx> u(4096);
    for (int i = 0; i < 4096; ++i) u[i] = cplx(U[2 * i], U[2 * i + 1]);
    dense6_prepare_weights(u.data(), (uint8_t*)out);
  });
}

int qs_apply_dense6(qs_state* s, const double* U) {
  return guard([&] {
    if (!s || !U) throw InvalidArg{"null argument"};
    if (s->dtype != 0) throw InvalidArg{"apply_dense6: complex64 states only"};
    if (s->n < 13) throw InvalidArg{"apply_dense6: needs at least 13 qubits"};
    s->materialize();  // queued gates first; layout positions 0..5 become physical bits 0..5
    std::vector<cplx> u(4096);
    for (int i = 0; i < 4096; ++i) u[i] = cplx(U[2 * i], U[2 * i + 1]);
    std::vector<uint8_t> w(dense6_weight_bytes());
    dense6_prepare_weights(u.data(), w.data());
    if (!s->d_dense) CK(dev_malloc(&s->d_dense, dense6_weight_bytes() + dense6_gather_bytes()));
    // pageable source: staged before the call returns, copied in stream order
    CK(cudaMemcpyAsync(s->d_dense, w.data(), w.size(), cudaMemcpyHostToDevice, s->stream));
    CK(launch_dense6_tc(s->psi, s->n, s->d_dense, s->d_ctl + 2, s->wait_limit_ns, s->stream));
    s->st.launches += 1;
    s->st.gate_sweeps += 1;
  });
}

int qs_apply_dense(qs_state* s, int k, const int* qubits, const double* U) {
  return guard([&] {
    if (!s || !qubits || !U) throw InvalidArg{"null argument"};
    if (s->dtype != 0) throw InvalidArg{"apply_dense: complex64 states only"};
    if (s->n < 13) throw InvalidArg{"apply_dense: needs at least 13 qubits"};
    if (k < 1 || k > 6) throw InvalidArg{"apply_dense: 1 to 6 qubits"};
    std::vector<int> bphys(k);
    std::vector<char> used(s->n, 0);
    for (int j = 0; j < k; ++j) {
      if (qubits[j] < 0 || qubits[j] >= s->n) throw InvalidArg{"apply_dense: invalid qubit"};
      bphys[j] = s->pos2bit[qubits[j]];
      if (used[bphys[j]]++) throw InvalidArg{"apply_dense: qubits must be distinct"};
    }
    // the six physical bits of the kernel: the block's, then the lowest free ones (identity there)
    std::vector<int> b6 = bphys;
    for (int p = 0; (int)b6.size() < 6; ++p)
      if (!used[p]) { b6.push_back(p); used[p] = 1; }
    std::sort(b6.begin(), b6.end());
    int slot[6];  // kernel index bit of block qubit j
    for (int j = 0; j < k; ++j) slot[j] = (int)(std::find(b6.begin(), b6.end(), bphys[j]) - b6.begin());
    int fmask = 63;
    for (int j = 0; j < k; ++j) fmask &= ~(1 << slot[j]);
    const int d = 1 << k;
    std::vector<cplx> w(4096, cplx(0.0, 0.0));
    auto compress = [&](int r) {
      int v = 0;
      for (int j = 0; j < k; ++j) v |= ((r >> slot[j]) & 1) << j;
      return v;
    };
    for (int r = 0; r < 64; ++r)
      for (int c = 0; c < 64; ++c)
        if ((r & fmask) == (c & fmask)) {
          const int a = compress(r), b = compress(c);
          w[r * 64 + c] = cplx(U[2 * (a * d + b)], U[2 * (a * d + b) + 1]);
        }
    s->flush();  // queued gates run first (their bits are physical: no data movement needed)
    const size_t wbytes = dense6_weight_bytes(), tbytes = dense6_gather_bytes();
    std::vector<uint8_t> buf(wbytes + tbytes);
    dense6_prepare_weights(w.data(), buf.data());
    const bool low6 = b6 == std::vector<int>{0, 1, 2, 3, 4, 5};
    if (!low6 && !dense6_gather_tables(s->n, b6.data(), buf.data() + wbytes))
      throw InvalidArg{"apply_dense: needs at least 13 qubits"};
    if (!s->d_dense) CK(dev_malloc(&s->d_dense, wbytes + tbytes));
    CK(cudaMemcpyAsync(s->d_dense, buf.data(), buf.size(), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));  // the pageable source is read before it goes out of scope
    if (low6)
      CK(launch_dense6_tc(s->psi, s->n, s->d_dense, s->d_ctl + 2, s->wait_limit_ns, s->stream));
    else
      CK(launch_dense6_tc_gather(s->psi, s->n, s->d_dense, (const uint8_t*)s->d_dense + wbytes, b6[0] == 0,
                                 s->d_ctl + 2, s->wait_limit_ns, s->stream));
    s->st.launches += 1;
    s->st.gate_sweeps += 1;
  });
}

int qs_device_ptr(qs_state* s, void** out) {
  return guard([&] {
    if (!s || !out) throw InvalidArg{"null argument"};
    s->materialize();
    s->sync();
    *out = s->psi;
  });
}

int qs_set_stream(qs_state* s, void* stream) {
  return guard([&] {
    if (!s) throw InvalidArg{"null state"};
    s->flush();
    CK(cudaStreamSynchronize(s->stream));
    if (s->own_stream) CK(cudaStreamDestroy(s->stream));
    if (stream) {
      s->stream = (cudaStream_t)stream;
      s->own_stream = false;
    } else {
      CK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
      s->own_stream = true;
    }
    if (s->graph.exec) { cudaGraphExecDestroy(s->graph.exec); s->graph.exec = nullptr; }
  });
}

int qs_get_stream(qs_state* s, void** out) {
  return guard([&] { if (!s) throw InvalidArg{"null state"}; *out = (void*)s->stream; });
}

int qs_set_config(qs_state* s, const qs_config* c) {
  return guard([&] {
    if (!s || !c) throw InvalidArg{"null argument"};
    const int mmax = s->dtype == 0 ? 13 : 12;
    if (c->m < reg_bits(s->dtype) + 1 || c->m > mmax) throw InvalidArg{"config: m out of range"};
    if (c->k < 1 || c->k > c->m) throw InvalidArg{"config: k out of range"};
    if (c->hill_iters < 0) throw InvalidArg{"config: hill_iters must be >= 0"};
    if (c->jit_lr < 3 || c->jit_lr > 6 || c->m - c->jit_lr > 9) throw InvalidArg{"config: jit_lr out of range"};
    if (c->jit_blocks < 1 || c->jit_blocks > 4) throw InvalidArg{"config: jit_blocks must be 1, 2, 3 or 4"};
    if (c->jit_packed < 0 || c->jit_packed > 1) throw InvalidArg{"config: jit_packed must be 0 or 1"};
    if (c->jit_async < 0 || c->jit_async > 1) throw InvalidArg{"config: jit_async must be 0 or 1"};
    s->flush();
    s->cfg.m = c->m;
    s->cfg.k = c->k;
    s->cfg.hill_iters = c->hill_iters;
    s->grid_mult = c->grid_mult;
    s->jit_mode = c->jit;
    s->jit_lr = c->jit_lr;
    s->jit_blocks = c->jit_blocks;
    s->jit_packed = c->jit_packed;
    s->wait_limit_ns = c->wait_limit_ns ? c->wait_limit_ns : kBarrierLimitNs;
    s->jit_async = c->jit_async;
  });
}

int qs_get_config(qs_state* s, qs_config* c) {
  return guard([&] {
    if (!s || !c) throw InvalidArg{"null argument"};
    c->m = s->cfg.m; c->k = s->cfg.k; c->hill_iters = s->cfg.hill_iters; c->grid_mult = s->grid_mult;
    c->jit = s->jit_mode;
    c->jit_lr = s->jit_lr;
    c->jit_blocks = s->jit_blocks;
    c->jit_packed = s->jit_packed;
    c->wait_limit_ns = s->wait_limit_ns;
    c->jit_async = s->jit_async;
  });
}

int qs_get_stats(qs_state* s, qs_stats* out) {
  return guard([&] { if (!s || !out) throw InvalidArg{"null argument"}; *out = s->st; });
}
int qs_reset_stats(qs_state* s) {
  return guard([&] { if (!s) throw InvalidArg{"null state"}; s->st = qs_stats{}; });
}
int qs_get_pos2bit(qs_state* s, int* out, int n) {
  return guard([&] {
    if (!s || !out || n != s->n) throw InvalidArg{"bad arguments"};
    for (int p = 0; p < n; ++p) out[p] = s->pos2bit[p];
  });
}

int qs_norm_squared(qs_state* s, double* out) {
  return guard([&] {
    if (!s || !out) throw InvalidArg{"null argument"};
    s->flush();
    CK(cudaMemsetAsync(s->d_acc, 0, sizeof(double), s->stream));
    CK(launch_norm2(s->dtype, s->psi, s->n, s->d_acc, s->stream));
    CK(cudaMemcpyAsync(s->h_acc, s->d_acc, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    s->check_device_error();
    *out = s->h_acc[0];
  });
}

int qs_inner_product(qs_state* a, qs_state* b, double* re, double* im) {
  return guard([&] {
    if (!a || !b || !re || !im) throw InvalidArg{"null argument"};
    if (a->n != b->n) throw InvalidArg{"states differ in size"};
    a->materialize();
    b->materialize();
    CK(cudaStreamSynchronize(b->stream));
    CK(cudaMemsetAsync(a->d_acc, 0, 2 * sizeof(double), a->stream));
    CK(launch_inner_mixed(a->dtype, a->psi, b->dtype, b->psi, a->n, a->d_acc, a->stream));
    CK(cudaMemcpyAsync(a->h_acc, a->d_acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, a->stream));
    CK(cudaStreamSynchronize(a->stream));
    a->check_device_error();
    *re = a->h_acc[0];
    *im = a->h_acc[1];
  });
}

int qs_expect_zz_x(qs_state* psi, qs_state* lam, const double* a, const double* b, double* energy) {
  return guard([&] {
    if (!psi || !lam || !a || !b || !energy) throw InvalidArg{"null argument"};
    if (psi->n != lam->n || psi->dtype != lam->dtype) throw InvalidArg{"states differ in size or dtype"};
    if (psi == lam) throw InvalidArg{"psi and lam must be different states"};
    psi->materialize();
    lam->flush();
    CK(cudaStreamSynchronize(lam->stream));
    lam->queue.clear();
    for (int p = 0; p < lam->n; ++p) lam->pos2bit[p] = p;
    CK(cudaMemsetAsync(psi->d_acc, 0, sizeof(double), psi->stream));
    CK(launch_zz_x(psi->dtype, psi->psi, lam->psi, psi->n, a, b, psi->d_acc, psi->stream));
    CK(cudaMemcpyAsync(psi->h_acc, psi->d_acc, sizeof(double), cudaMemcpyDeviceToHost, psi->stream));
    CK(cudaStreamSynchronize(psi->stream));
    *energy = psi->h_acc[0];
    psi->st.launches += 1;
  });
}

int qs_adjoint_sweep(qs_state* psi, qs_state* lam, const qs_adj_op* ops, int nops, double* grads, int ngrads) {
  return guard([&] {
    if (!psi || !lam || (nops > 0 && !ops) || (ngrads > 0 && !grads)) throw InvalidArg{"null argument"};
    if (psi->n != lam->n || psi->dtype != lam->dtype) throw InvalidArg{"states differ in size or dtype"};
    if (psi == lam) throw InvalidArg{"psi and lam must be different states"};
    const int n = psi->n;
    for (int i = 0; i < nops; ++i) {
      const qs_adj_op& o = ops[i];
      if (!o.U) throw InvalidArg{"adjoint: null gate matrix"};
      if (o.kind == QS_OP_1Q) {
        if (o.q0 < 0 || o.q0 >= n) throw InvalidArg{"adjoint: invalid q0"};
        if (o.gen < 0 || o.gen > 3) throw InvalidArg{"adjoint: generator must be 0..3"};
        if (o.gen && (o.grad_index < 0 || o.grad_index >= ngrads)) throw InvalidArg{"adjoint: grad_index out of range"};
      } else if (o.kind == QS_OP_2Q) {
        if (o.q0 < 0 || o.q0 >= n || o.q1 < 0 || o.q1 >= n || o.q0 == o.q1)
          throw InvalidArg{"adjoint: invalid q0/q1"};
        if (o.gen != 0) throw InvalidArg{"adjoint: two-qubit gates carry no parameter"};
      } else {
        throw InvalidArg{"adjoint: unknown op kind: " + std::to_string(o.kind)};
      }
    }
    psi->materialize();
    lam->materialize();
    CK(cudaStreamSynchronize(lam->stream));
    AsyncBuf grad_buf(psi->stream);
    CK(grad_buf.alloc(std::max(1, ngrads) * sizeof(double)));
    double* d_grad = (double*)grad_buf.p;
    CK(cudaMemsetAsync(d_grad, 0, std::max(1, ngrads) * sizeof(double), psi->stream));
    for (int i = nops - 1; i >= 0; --i) {
      const qs_adj_op& o = ops[i];
      if (o.kind == QS_OP_1Q) {
        cplx Ud[4];
        for (int r = 0; r < 2; ++r)
          for (int c = 0; c < 2; ++c) Ud[2 * r + c] = std::conj(cplx(o.U[2 * (2 * c + r)], o.U[2 * (2 * c + r) + 1]));
        CK(launch_adjoint_gate1(psi->dtype, psi->psi, lam->psi, n, o.q0, Ud, o.gen,
                                o.gen ? d_grad + o.grad_index : d_grad, psi->stream));
      } else {
        cplx Ud[16];
        for (int r = 0; r < 4; ++r)
          for (int c = 0; c < 4; ++c) Ud[4 * r + c] = std::conj(cplx(o.U[2 * (4 * c + r)], o.U[2 * (4 * c + r) + 1]));
        CK(launch_adjoint_gate2(psi->dtype, psi->psi, lam->psi, n, o.q0, o.q1, Ud, psi->stream));
      }
      psi->st.launches += 1;
      psi->st.gate_sweeps += 2;
    }
    if (ngrads > 0) CK(cudaMemcpyAsync(grads, d_grad, ngrads * sizeof(double), cudaMemcpyDeviceToHost, psi->stream));
    CK(cudaStreamSynchronize(psi->stream));
  });
}

}  // extern "C"

// ------------------------------------------------------------------------------------
// Adjoint gradient with the specialised kernels: forward tile, stacked observable, one
// reverse program over Phi = psi (+) H psi
// ------------------------------------------------------------------------------------
namespace {

std::vector<GradOp> read_grad_ops(const qs_adj_op* ops, int nops, int n, int nparams) {
  if (nops < 0 || (nops > 0 && !ops)) throw InvalidArg{"gradient: null ops"};
  std::vector<GradOp> out(nops);
  for (int i = 0; i < nops; ++i) {
    const qs_adj_op& o = ops[i];
    GradOp& g = out[i];
    if (!o.U) throw InvalidArg{"gradient: null gate matrix"};
    if (o.kind == QS_OP_1Q) {
      if (o.q0 < 0 || o.q0 >= n) throw InvalidArg{"gradient: invalid q0"};
      if (o.gen < 0 || o.gen > 3) throw InvalidArg{"gradient: generator must be 0..3"};
      if (o.gen && (o.grad_index < 0 || o.grad_index >= nparams)) throw InvalidArg{"gradient: grad_index out of range"};
      g.op.arity = 1;
      g.op.q0 = o.q0;
      for (int e = 0; e < 4; ++e) g.op.U[e] = cplx(o.U[2 * e], o.U[2 * e + 1]);
      g.gen = o.gen;
      g.slot = o.gen ? o.grad_index : -1;
    } else if (o.kind == QS_OP_2Q) {
      if (o.q0 < 0 || o.q0 >= n || o.q1 < 0 || o.q1 >= n || o.q0 == o.q1) throw InvalidArg{"gradient: invalid q0/q1"};
      if (o.gen != 0) throw InvalidArg{"gradient: two-qubit gates carry no parameter"};
      g.op.arity = 2;
      g.op.q0 = o.q0;
      g.op.q1 = o.q1;
      for (int e = 0; e < 16; ++e) g.op.U[e] = cplx(o.U[2 * e], o.U[2 * e + 1]);
    } else {
      throw InvalidArg{"gradient: unknown op kind: " + std::to_string(o.kind)};
    }
  }
  return out;
}

bool same_grad_structure(const std::vector<GradOp>& a, const std::vector<GradOp>& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (a[i].op.arity != b[i].op.arity || a[i].op.q0 != b[i].op.q0 || a[i].op.q1 != b[i].op.q1 ||
        a[i].gen != b[i].gen || a[i].slot != b[i].slot)
      return false;
  return true;
}

PlanConfig grad_plan_cfg(int n, const qs_config* c) {
  PlanConfig p;
  p.r = c && (c->jit_lr == 5 || c->jit_lr == 6) ? c->jit_lr : 5;
  p.m = c && c->m > 0 ? c->m : 13;
  p.k = c && c->k > 0 ? c->k : 3;
  p.hill_iters = c ? c->hill_iters : 16;
  p.m = std::max(p.r, std::min(p.m, n + 1));
  return p;
}

}  // namespace

struct qs_grad {
  int n = 0, nparams = 0;
  std::vector<GradOp> structure;
  qs_state* fwd = nullptr;        // the forward state (n qubits), specialised kernels
  PlanConfig pc;
  std::vector<PlannedPass> rplan;  // reverse program (n + 1 qubits)
  void* phi = nullptr;             // stacked state, 2^(n+1) complex64
  uint8_t* d_prog = nullptr;
  size_t prog_cap = 0;
  uint8_t* h_prog = nullptr;       // pinned staging of the reverse program
  cudaEvent_t copied = nullptr;    // the last copy out of h_prog has run
  size_t hprog_cap = 0;
  double* d_out = nullptr;         // energy, then the terms
  double* h_out = nullptr;         // pinned
  size_t out_cap = 0;
  GraphEntry graph;
  int rev_phases = 0, nterm = 0, fwd_sweeps = 0;

  ~qs_grad() {
    if (fwd) cudaStreamSynchronize(fwd->stream);
    if (graph.exec) cudaGraphExecDestroy(graph.exec);
    if (phi) cudaFree(phi);
    if (d_prog) cudaFree(d_prog);
    if (h_prog) cudaFreeHost(h_prog);
    if (copied) cudaEventDestroy(copied);
    if (d_out) cudaFree(d_out);
    if (h_out) cudaFreeHost(h_out);
    delete fwd;
  }

  void run(const std::vector<GradOp>& f, const double* a, const double* b, double* energy, double* grads) {
    qs_state* s = fwd;
    cudaStream_t st = s->stream;
    // forward: psi = U|0>, one graphed tile of the specialised kernels
    s->queue.clear();
    for (int p = 0; p < n; ++p) s->pos2bit[p] = p;
    CK(launch_set_basis(0, s->psi, n, 0, st));
    std::vector<QOp> q;
    q.reserve(f.size());
    for (const GradOp& g : f) q.push_back(g.op);
    const unsigned long long sw0 = s->st.sweeps;
    enqueue(s, std::move(q), QS_MODE_GRAPHED);
    s->flush();
    fwd_sweeps = (int)(s->st.sweeps - sw0);
    if (!grads) {  // energy only
      CK(cudaMemsetAsync(s->d_acc, 0, sizeof(double), st));
      CK(launch_zz_x_stack(s->psi, phi, n, a, b, s->d_acc, st));
      s->st.launches += 1;
      CK(cudaMemcpyAsync(s->h_acc, s->d_acc, sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      s->check_device_error();
      *energy = s->h_acc[0];
      return;
    }
    // reverse program (host): scalar extraction for these values, encoding, term weights; a
    // gate whose class changed with its values (a diagonal became dense) takes a new plan
    if (!grad_plan_fits(f, rplan)) {
      rplan = plan_grad_passes(f, n, pc, nullptr);
      rev_phases = 0;
      for (const PlannedPass& ps : rplan) rev_phases += (int)ps.phases.size();
    }
    GradProgram gp = build_grad_program(f, n, rplan, pc.r);
    nterm = gp.prog.nterm;
    const size_t outb = (size_t)(1 + nterm) * sizeof(double);
    if (outb > out_cap) {
      CK(cudaStreamSynchronize(st));
      if (d_out) CK(cudaFree(d_out));
      if (h_out) CK(cudaFreeHost(h_out));
      d_out = nullptr;
      h_out = nullptr;
      out_cap = 0;
      CK(dev_malloc((void**)&d_out, outb));
      CK(host_malloc((void**)&h_out, outb));
      out_cap = outb;
      if (graph.exec) { cudaGraphExecDestroy(graph.exec); graph.exec = nullptr; }
    }
    const size_t pb = gp.prog.bytes.size();
    if (pb > prog_cap || pb > hprog_cap) {
      CK(cudaStreamSynchronize(st));
      if (d_prog) CK(cudaFree(d_prog));
      if (h_prog) CK(cudaFreeHost(h_prog));
      d_prog = nullptr;
      h_prog = nullptr;
      prog_cap = hprog_cap = 0;
      CK(dev_malloc((void**)&d_prog, pb * 2));
      CK(host_malloc((void**)&h_prog, pb * 2));
      prog_cap = hprog_cap = pb * 2;
      if (graph.exec) { cudaGraphExecDestroy(graph.exec); graph.exec = nullptr; }
    }
    // the staging is rewritten only after its previous copy ran (a run that failed midway may
    // have left one queued)
    if (!copied) CK(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
    CK(cudaEventSynchronize(copied));
    std::memcpy(h_prog, gp.prog.bytes.data(), pb);
    CK(cudaMemcpyAsync(d_prog, h_prog, pb, cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(copied, st));
    CK(cudaMemsetAsync(d_out, 0, outb, st));
    // Phi = psi (+) H psi and the energy
    CK(launch_zz_x_stack(s->psi, phi, n, a, b, d_out, st));
    s->st.launches += 1;
    if (gp.prog.npass > 0) {  // (a circuit without gates has no reverse sweep: every term is zero)
      // the reverse program: one launch per pass, captured as a graph (parameter values only
      // update it)
      JitConfig jc;
      jc.blocks = 2;
      jc.packed = false;
      std::shared_ptr<JitKernels> jk = jit_get(gp.prog, jc);
      s->st.jit_compile_ms += (unsigned long long)(jk->compile_seconds * 1e3 + 0.5);
      s->st.jit_modules += (unsigned long long)jk->chunks;
      s->st.jit_disk_hits += (unsigned long long)jk->disk_hits;
      jk->compile_seconds = 0.0;
      jk->chunks = 0;
      jk->disk_hits = 0;
      const uint64_t key = jk->key ^ ((uint64_t)(uintptr_t)phi * 0x9E3779B97F4A7C15ull) ^
                           ((uint64_t)(uintptr_t)d_prog << 1) ^ ((uint64_t)(uintptr_t)d_out << 3);
      const uint64_t values = coef_values_hash(gp.prog);
      const uint8_t* host_coef = gp.prog.bytes.data() + ((const ProgramHeader*)gp.prog.bytes.data())->off_coef;
      auto capture = [&]() {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (int p = 0; p < gp.prog.npass && e == cudaSuccess; ++p)
          e = jit_launch(*jk, p, d_prog, host_coef, phi, s->d_ctl + 2, gp.prog.threads, gp.prog.max_smem,
                         device_sm_count(), st, d_out + 1);
        cudaError_t e2 = cudaStreamEndCapture(st, &g);
        if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); throw CudaError{e}; }
        if (e2 != cudaSuccess) throw CudaError{e2};
        return g;
      };
      bool updated = false;
      if (graph.exec && graph.key == key && graph.values != values) {
        cudaGraph_t g = capture();
        cudaGraphExecUpdateResultInfo info;
        const cudaError_t eu = cudaGraphExecUpdate(graph.exec, g, &info);
        cudaGraphDestroy(g);
        if (eu == cudaSuccess) {
          graph.values = values;
          updated = true;
        } else {
          cudaGetLastError();
          CK(cudaGraphExecDestroy(graph.exec));
          graph.exec = nullptr;
        }
      }
      if (!graph.exec || graph.key != key) {
        if (graph.exec) { CK(cudaGraphExecDestroy(graph.exec)); graph.exec = nullptr; }
        graph.kernels = jk;
        cudaGraph_t g = capture();
        cudaError_t e3 = cudaGraphInstantiate(&graph.exec, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) throw CudaError{e3};
        graph.key = key;
        graph.values = values;
        s->st.graph_builds += 1;
      } else if (updated) {
        s->st.graph_builds += 1;
      } else {
        s->st.graph_replays += 1;
      }
      CK(cudaGraphLaunch(graph.exec, st));
      s->st.launches += 1;
      s->st.sweeps += gp.prog.npass;
    }
    CK(cudaMemcpyAsync(h_out, d_out, outb, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    s->check_device_error();
    *energy = h_out[0];
    for (int k = 0; k < nparams; ++k) grads[k] = 0.0;
    for (int t = 0; t < nterm; ++t) grads[gp.term_slot[t]] += gp.term_w[t] * h_out[1 + t];
  }
};

extern "C" {

int qs_grad_create(int num_qubits, const qs_adj_op* ops, int nops, int nparams, const qs_config* cfg,
                   qs_grad** out) {
  return guard([&] {
    if (!out) throw InvalidArg{"null output handle"};
    *out = nullptr;
    if (num_qubits < 10 || num_qubits > 33) throw InvalidArg{"gradient: num_qubits must be in [10, 33]"};
    if (nparams < 0) throw InvalidArg{"gradient: nparams < 0"};
    std::string why;
    if (!jit_available(&why)) throw InvalidArg{"gradient: specialised kernels unavailable: " + why};
    std::unique_ptr<qs_grad> g(new qs_grad());
    g->n = num_qubits;
    g->nparams = nparams;
    g->structure = read_grad_ops(ops, nops, num_qubits, nparams);
    g->pc = grad_plan_cfg(num_qubits, cfg);
    g->rplan = plan_grad_passes(g->structure, num_qubits, g->pc, nullptr);
    for (const PlannedPass& ps : g->rplan) g->rev_phases += (int)ps.phases.size();
    qs_state* s = nullptr;
    const int rc = qs_create(num_qubits, QS_C64, &s);
    if (rc != 0) throw Status{rc, std::string(qs_last_error())};
    g->fwd = s;
    s->jit_mode = 1;
    if (cfg) {
      if (cfg->m > 0) s->cfg.m = std::min(cfg->m, 13);
      if (cfg->k > 0) s->cfg.k = cfg->k;
      s->cfg.hill_iters = cfg->hill_iters;
      if (cfg->jit_lr == 5 || cfg->jit_lr == 6) s->jit_lr = cfg->jit_lr;
    }
    CK(dev_malloc(&g->phi, (sizeof(float) * 2) << (num_qubits + 1)));
    *out = g.release();
  });
}

int qs_grad_run(qs_grad* g, const qs_adj_op* ops, int nops, const double* a, const double* b, double* energy,
                double* grads) {
  return guard([&] {
    if (!g || !a || !b || !energy) throw InvalidArg{"null argument"};
    std::vector<GradOp> f = read_grad_ops(ops, nops, g->n, g->nparams);
    if (!same_grad_structure(f, g->structure))
      throw InvalidArg{"gradient: the circuit's structure differs from the one the handle was created for"};
    g->run(f, a, b, energy, grads);
  });
}

int qs_grad_info(const qs_grad* g, int* fwd_sweeps, int* rev_sweeps, int* rev_phases, int* terms) {
  return guard([&] {
    if (!g) throw InvalidArg{"null handle"};
    if (fwd_sweeps) *fwd_sweeps = g->fwd_sweeps;
    if (rev_sweeps) *rev_sweeps = (int)g->rplan.size();
    if (rev_phases) *rev_phases = g->rev_phases;
    if (terms) *terms = g->nterm;
  });
}

int qs_grad_stats(qs_grad* g, qs_stats* out) {
  return guard([&] {
    if (!g || !out) throw InvalidArg{"null argument"};
    *out = g->fwd->st;
  });
}

int qs_grad_destroy(qs_grad* g) {
  return guard([&] { delete g; });
}

int qs_grad_jit_check(int num_qubits, const qs_adj_op* ops, int nops, int nparams, const qs_config* cfg,
                      int* sweeps, char* logbuf, int logcap) {
  return guard([&] {
    if (num_qubits < 10 || num_qubits > 33) throw InvalidArg{"gradient: num_qubits must be in [10, 33]"};
    std::vector<GradOp> f = read_grad_ops(ops, nops, num_qubits, nparams);
    const PlanConfig pc = grad_plan_cfg(num_qubits, cfg);
    std::vector<PlannedPass> passes = plan_grad_passes(f, num_qubits, pc, nullptr);
    GradProgram gp = build_grad_program(f, num_qubits, passes, pc.r);
    JitConfig jc;
    jc.blocks = 2;
    jc.packed = false;
    std::string log;
    const bool ok = jit_compile_check(gp.prog, &log, jc);
    if (logbuf && logcap > 0) {
      const size_t k = std::min<size_t>(log.size(), (size_t)logcap - 1);
      std::memcpy(logbuf, log.data(), k);
      logbuf[k] = '\0';
    }
    if (!ok) throw InvalidArg{"jit compile failed:\n" + log.substr(0, 4000)};
    if (sweeps) *sweeps = gp.prog.npass;
  });
}

int qs_grad_emulate(int num_qubits, const qs_adj_op* ops, int nops, int nparams, const qs_config* cfg,
                    const void* psi, const void* lam, double* grads) {
  return guard([&] {
    if (!psi || !lam || (nparams > 0 && !grads)) throw InvalidArg{"null argument"};
    if (num_qubits < 10 || num_qubits > 22) throw InvalidArg{"gradient emulation: num_qubits must be in [10, 22]"};
    std::vector<GradOp> f = read_grad_ops(ops, nops, num_qubits, nparams);
    const PlanConfig pc = grad_plan_cfg(num_qubits, cfg);
    std::vector<PlannedPass> passes = plan_grad_passes(f, num_qubits, pc, nullptr);
    if (!grad_plan_fits(f, passes)) throw InvalidArg{"gradient emulation: plan does not hold the gates"};
    GradProgram gp = build_grad_program(f, num_qubits, passes, pc.r);
    const uint64_t dim = 1ull << num_qubits;
    std::vector<std::complex<float>> phi(2 * dim);
    const std::complex<float>* ps = (const std::complex<float>*)psi;
    const std::complex<float>* ls = (const std::complex<float>*)lam;
    for (uint64_t x = 0; x < dim; ++x) { phi[2 * x] = ps[x]; phi[2 * x + 1] = ls[x]; }
    std::vector<double> terms(std::max(1, gp.prog.nterm), 0.0);
    emulate_grad_program(gp, phi.data(), terms.data());
    for (int k = 0; k < nparams; ++k) grads[k] = 0.0;
    for (int t = 0; t < gp.prog.nterm; ++t) grads[gp.term_slot[t]] += gp.term_w[t] * terms[t];
  });
}

int qs_apply_1q_gate(void* psi, int dtype, const void* U, int target_qubit, int num_qubits, void* stream) {
  return guard([&] {
    if (!psi || !U) throw InvalidArg{"null argument"};
    if (dtype != 0 && dtype != 1) throw InvalidArg{"dtype must be QS_C64 or QS_C128"};
    if (num_qubits < 1 || num_qubits > 36) throw InvalidArg{"num_qubits must be in [1, 36]"};
    if (target_qubit < 0 || target_qubit >= num_qubits) throw InvalidArg{"Invalid target qubit"};
    cplx m[4];
    read_matrix(nullptr, dtype, U, 0, 4, m);
    CK(launch_gate1(dtype, psi, num_qubits, target_qubit, m, (cudaStream_t)stream));
  });
}

int qs_apply_2q_gate(void* psi, int dtype, const void* U, int q0, int q1, int num_qubits, void* stream) {
  return guard([&] {
    if (!psi || !U) throw InvalidArg{"null argument"};
    if (dtype != 0 && dtype != 1) throw InvalidArg{"dtype must be QS_C64 or QS_C128"};
    if (num_qubits < 2 || num_qubits > 36) throw InvalidArg{"num_qubits must be in [2, 36]"};
    if (q0 < 0 || q0 >= num_qubits || q1 < 0 || q1 >= num_qubits) throw InvalidArg{"Invalid qubit indices"};
    if (q0 == q1) throw InvalidArg{"q0 and q1 must be different"};
    cplx m[16];
    read_matrix(nullptr, dtype, U, 0, 16, m);
    CK(launch_gate2(dtype, psi, num_qubits, q0, q1, m, (cudaStream_t)stream));
  });
}

int qs_permute_scatter(const void* in, void* out, int dtype, int num_qubits, const int* map, void* stream) {
  return guard([&] {
    if (!in || !out || !map) throw InvalidArg{"null argument"};
    if (num_qubits < 1 || num_qubits > 36) throw InvalidArg{"num_qubits must be in [1, 36]"};
    std::vector<int> seen(num_qubits, 0);
    for (int p = 0; p < num_qubits; ++p) {
      if (map[p] < 0 || map[p] >= num_qubits || seen[map[p]]++) throw InvalidArg{"map is not a permutation"};
    }
    CK(launch_permute_scatter(dtype, in, out, num_qubits, map, (cudaStream_t)stream));
  });
}

// ---- host-only planner inspection -----------------------------------------------------
static PlanConfig cfg_from(int dtype, int n, const qs_config* c) {
  PlanConfig p;
  p.r = reg_bits(dtype);
  p.m = c ? c->m : (dtype == 0 ? 13 : 12);
  p.k = c ? c->k : 3;
  p.hill_iters = c ? c->hill_iters : 16;
  p.m = std::max(p.r, std::min(p.m, n));
  return p;
}

int qs_plan_info(int num_qubits, int dtype, const qs_op* ops, int nops, const qs_config* cfg, int* sweeps,
                 int* phases) {
  return guard([&] {
    if (num_qubits < reg_bits(dtype) + 1 || num_qubits > 36) throw InvalidArg{"num_qubits out of range"};
    auto q = convert_ops(nullptr, ops, nops, num_qubits, dtype, false);
    std::vector<COp> c;
    for (auto& o : q) c.push_back(classify(o));
    PlanConfig pc = cfg_from(dtype, num_qubits, cfg);
    // complex64 with an explicit register-bit count: plan as the specialised kernels would
    if (dtype == 0 && cfg && cfg->jit_lr >= 3 && cfg->jit_lr <= 6) pc.r = cfg->jit_lr;
    pc.pair_bit = dtype == 0 && cfg && cfg->jit_packed == 1;
    auto passes = plan_passes(c, num_qubits, pc);
    int ph = 0;
    for (auto& p : passes) ph += (int)p.phases.size();
    if (sweeps) *sweeps = (int)passes.size();
    if (phases) *phases = ph;
  });
}

int qs_plan_emulate(int num_qubits, int dtype, const qs_op* ops, int nops, const qs_config* cfg, void* psi) {
  return guard([&] {
    if (num_qubits < reg_bits(dtype) + 1 || num_qubits > 24) throw InvalidArg{"num_qubits out of range"};
    auto q = convert_ops(nullptr, ops, nops, num_qubits, dtype, false);
    std::vector<COp> c;
    for (auto& o : q) c.push_back(classify(o));
    PlanConfig pc = cfg_from(dtype, num_qubits, cfg);
    // complex64 with an explicit register-bit count: the program the specialised kernels run
    if (dtype == 0 && cfg && cfg->jit_lr >= 3 && cfg->jit_lr <= 6) pc.r = cfg->jit_lr;
    auto passes = plan_passes(c, num_qubits, pc);
    Program prog = build_program(q, passes, num_qubits, dtype, pc.r);
    emulate_program(prog.bytes.data(), psi, num_qubits, dtype);
  });
}

int qs_jit_check(int num_qubits, const qs_op* ops, int nops, const qs_config* cfg, int* sweeps, char* logbuf,
                 int logcap) {
  return guard([&] {
    if (num_qubits < reg_bits(0) + 1 || num_qubits > 36) throw InvalidArg{"num_qubits out of range"};
    auto q = convert_ops(nullptr, ops, nops, num_qubits, 0, false);
    std::vector<COp> c;
    for (auto& o : q) c.push_back(classify(o));
    PlanConfig pc = cfg_from(0, num_qubits, cfg);
    pc.r = (cfg && cfg->jit_lr >= 3 && cfg->jit_lr <= 6) ? cfg->jit_lr : 5;
    pc.pair_bit = cfg && cfg->jit_packed == 1;
    auto passes = plan_passes(c, num_qubits, pc);
    Program prog = build_program(q, passes, num_qubits, 0, pc.r);
    std::string log;
    JitConfig jc;
    if (cfg && cfg->jit_blocks >= 1 && cfg->jit_blocks <= 4) jc.blocks = cfg->jit_blocks;
    jc.packed = cfg && cfg->jit_packed == 1;
    const bool ok = jit_compile_check(prog, &log, jc);
    if (logbuf && logcap > 0) {
      const size_t k = std::min<size_t>(log.size(), (size_t)logcap - 1);
      std::memcpy(logbuf, log.data(), k);
      logbuf[k] = '\0';
    }
    if (!ok) throw InvalidArg{"jit compile failed:\n" + log.substr(0, 4000)};
    if (sweeps) *sweeps = prog.npass;
  });
}

int qs_perm_emulate(int num_qubits, int dtype, const int* perm, const qs_config* cfg, void* psi, int* sweeps) {
  return guard([&] {
    if (num_qubits < reg_bits(dtype) + 1 || num_qubits > 24) throw InvalidArg{"num_qubits out of range"};
    std::vector<int> p(perm, perm + num_qubits), seen(num_qubits, 0);
    for (int b = 0; b < num_qubits; ++b)
      if (p[b] < 0 || p[b] >= num_qubits || seen[p[b]]++) throw InvalidArg{"perm is not a permutation"};
    auto passes = plan_permutation(p, num_qubits, cfg_from(dtype, num_qubits, cfg));
    std::vector<COp> none;
    Program prog = encode_program(passes, none, num_qubits, dtype);
    emulate_program(prog.bytes.data(), psi, num_qubits, dtype);
    if (sweeps) *sweeps = prog.npass;
  });
}

}  // extern "C"
