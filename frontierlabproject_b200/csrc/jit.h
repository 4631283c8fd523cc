// Pass kernels specialised at plan time: each pass's register phases become straight-line
// CUDA (no per-gate dispatch; permutation gates are register renames; zero, +-1, real and
// imaginary matrix entries skip their multiplies), compiled for sm_100a with NVRTC and
// loaded as cubins.  Coefficient values are not compiled in: each pass kernel receives its
// range of the coefficient table as a by-value launch parameter (constant bank, read by the
// arithmetic instructions as operands), so a circuit whose parameters change reuses the
// compiled kernels (the cache key is the program structure plus the zero/one/real/imaginary
// class of every matrix entry).
#pragma once
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "plan.h"

namespace qsb {

// Geometry of the specialised kernels.  The register bits per thread (lr) are fixed when
// the program is planned (2^(m - lr) threads per team); blocks = 1 double-buffers the
// group loads inside a block, blocks = 2 gives each of two resident blocks one buffer,
// blocks = 3 runs one block per SM of two teams over three buffers (pass_body_teams), blocks = 4
// two double-buffered blocks per SM.
struct JitConfig {
  int blocks = 1;
  bool packed = true;   // FP32x2 registers for passes whose phases all hold local bit 0
};

struct JitKernels {
  std::vector<void*> functions;  // CUfunction per pass
  std::vector<void*> modules;    // CUmodule per compiled chunk
  std::vector<int> cbase, ccount;  // per pass: coefficient-table range passed as its parameter
  std::vector<std::vector<uint32_t>> splats;  // per pass: splatted entries after the range
                                              // (table entry * 4 + component: x, y, -x, -y)
  uint64_t key = 0;
  int blocks = 1;
  bool grad = false;    // gradient program: the kernels take the term array (jit_launch gterm)
  double compile_seconds = 0.0;
  int chunks = 0;       // compiled modules
  int disk_hits = 0;    // of which read from the on-disk cache
  ~JitKernels();
};

// True when NVRTC and the driver entry points are available (message otherwise).
bool jit_available(std::string* why);

// Cache key of a complex64 program (structure + entry classes + geometry).
uint64_t jit_key(const Program& prog, const JitConfig& cfg);

// CUDA source of the specialised kernels for passes [pass_begin, pass_end).
// splats (optional): per pass, the splatted coefficients its parameter block carries.
std::string jit_source(const Program& prog, int pass_begin, int pass_end, uint64_t key, const JitConfig& cfg,
                       std::vector<std::vector<uint32_t>>* splats = nullptr);

// Compile (cached) the kernels of every pass of a complex64 program.  Compiled modules are
// also kept on disk across processes ($QSIM_JIT_CACHE, default ~/.cache/qsim_b200/jit; "off"
// disables it), keyed by their source, the device headers, the options and NVRTC's version.
std::shared_ptr<JitKernels> jit_get(const Program& prog, const JitConfig& cfg);

// Non-blocking form of jit_get: the kernels when they are compiled (in memory), else nullptr
// after starting (once per program structure) their compile on a background thread; a
// later call returns them once that compile has finished (or throws its error).
std::shared_ptr<JitKernels> jit_try_get(const Program& prog, const JitConfig& cfg);
// Waits for every compile started by jit_try_get.
void jit_wait_all();

// Launch the specialised kernel of pass p (one launch per pass, no grid barrier).
// host_coef = the program's coefficient table in host memory: the pass's range of it is
// copied into the launch's parameter block.  smem_double = bytes of two group buffers
// (Program::max_smem); threads = the program's team size; err = device error word (bounded
// waits of the two-team kernels); gterm = the FP64 term array of a gradient program (its
// kernels add their terms there; ignored otherwise).
cudaError_t jit_launch(const JitKernels& k, int p, const uint8_t* d_prog, const void* host_coef, void* psi,
                       unsigned* err, int threads, size_t smem_double, int sms, cudaStream_t stream,
                       double* gterm = nullptr);

// Dynamic shared memory of a specialised kernel: group buffers for the geometry.
inline size_t jit_smem_bytes(int blocks, size_t smem_double) {
  return blocks == 2 ? smem_double / 2 : blocks == 3 ? smem_double / 2 * 3 : smem_double;
}

// Compile a program's source on the host only (tests; returns the NVRTC log on failure).
bool jit_compile_check(const Program& prog, std::string* log, const JitConfig& cfg = JitConfig());

}  // namespace qsb
