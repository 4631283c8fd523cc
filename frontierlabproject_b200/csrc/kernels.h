// Kernel launchers of libqsim_b200 (all on the caller's stream).
#pragma once
#include <complex>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

namespace qsb {

// pass kernel (kern_pass.cu)
cudaError_t launch_pass_kernel(int dtype, const uint8_t* d_prog, void* psi, int pass_begin, int pass_end,
                               int threads, size_t smem, int grid, bool cooperative, unsigned* bar,
                               unsigned* err, uint64_t limit_ns, cudaStream_t stream);
cudaError_t pass_kernel_occupancy(int dtype, int threads, size_t smem, int* blocks_per_sm);

// per-gate kernels: one full sweep per gate (kern_gate.cu)
cudaError_t launch_gate1(int dtype, void* psi, int n, int q, const std::complex<double>* U, cudaStream_t s);
cudaError_t launch_gate2(int dtype, void* psi, int n, int q0, int q1, const std::complex<double>* U,
                         cudaStream_t s);
cudaError_t launch_diag1(int dtype, void* psi, int n, int q, std::complex<double> d0, std::complex<double> d1,
                         cudaStream_t s);
// out[j] = in[i], j = sum_p bit_p(i) << map[p]   (out-of-place)
cudaError_t launch_permute_scatter(int dtype, const void* in, void* out, int n, const int* map, cudaStream_t s);

// reductions into double accumulators (kern_gate.cu); acc must be zeroed by the caller
cudaError_t launch_norm2(int dtype, const void* psi, int n, double* acc, cudaStream_t s);
cudaError_t launch_inner(int dtype, const void* a, const void* b, int n, double* acc2, cudaStream_t s);
cudaError_t launch_inner_mixed(int dtype_a, const void* a, int dtype_b, const void* b, int n, double* acc2,
                               cudaStream_t s);
cudaError_t launch_set_basis(int dtype, void* psi, int n, uint64_t index, cudaStream_t s);

// adjoint differentiation (kern_adjoint.cu)
cudaError_t launch_zz_x(int dtype, const void* psi, void* lam, int n, const double* a, const double* b,
                        double* energy, cudaStream_t s);
// Stacked state of the gradient sweep (complex64): phi[2x] = psi[x], phi[2x + 1] = (H psi)[x]
// (2^(n+1) amplitudes), energy += <psi|H psi> (FP64).
cudaError_t launch_zz_x_stack(const void* psi, void* phi, int n, const double* a, const double* b, double* energy,
                              cudaStream_t s);
cudaError_t launch_adjoint_gate1(int dtype, void* psi, void* lam, int n, int q, const std::complex<double>* Ud,
                                 int gen, double* acc, cudaStream_t s);
cudaError_t launch_adjoint_gate2(int dtype, void* psi, void* lam, int n, int q0, int q1,
                                 const std::complex<double>* Ud, cudaStream_t s);

// batched variational workload (kern_batch.cu): one cooperative persistent launch
cudaError_t launch_batch(const uint8_t* d_prog, void* arena, double* grads, double* energy, unsigned* ctl,
                         int threads, int mbuf, int blocks_per_sm_cap, uint64_t limit_ns, cudaStream_t s,
                         int* grid_out);

// dense 64x64 unitary on the six lowest qubits on the tensor cores (kern_dense_tc.cu):
// weights = dense6_weight_bytes() bytes prepared by dense6_prepare_weights (device copy)
size_t dense6_weight_bytes();
void dense6_prepare_weights(const std::complex<double>* U, uint8_t* out);
cudaError_t launch_dense6_tc(void* psi, int n, const void* d_weights, unsigned* err, uint64_t limit_ns,
                             cudaStream_t s);
// the same on six arbitrary physical bits B (ascending): tables of dense6_gather_bytes() bytes
// from dense6_gather_tables (false: fewer than 13 qubits), device copy d_tabs; pairs: physical
// bit 0 is in B (B[0] == 0), so the copies move 16-byte amplitude pairs
size_t dense6_gather_bytes();
bool dense6_gather_tables(int n, const int* B, uint8_t* out);
cudaError_t launch_dense6_tc_gather(void* psi, int n, const void* d_weights, const void* d_tabs, bool pairs,
                                    unsigned* err, uint64_t limit_ns, cudaStream_t s);

// measurement sampling (kern_sample.cu): `shots` indices drawn from |psi|^2, ascending, into
// out (device); scratch: sample_scratch_bytes(n, shots) bytes of device memory
size_t sample_scratch_bytes(int n, uint64_t shots);
cudaError_t launch_sample(int dtype, const void* psi, int n, uint64_t shots, uint64_t seed, void* scratch,
                          uint64_t* out, cudaStream_t s);

int device_sm_count();

// Every device / pinned-host allocation of the library goes through these.  After
// qs_debug_fail_alloc(k), the k-th next one fails with cudaErrorMemoryAllocation and
// allocates nothing, so tests can check that each error path releases what it holds.
cudaError_t dev_malloc(void** p, size_t bytes);
cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t s);
cudaError_t host_malloc(void** p, size_t bytes);

// Device buffer from the stream-ordered allocator, freed in stream order when it goes out of
// scope (also when an exception leaves the scope).
struct AsyncBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  explicit AsyncBuf(cudaStream_t st) : s(st) {}
  AsyncBuf(const AsyncBuf&) = delete;
  AsyncBuf& operator=(const AsyncBuf&) = delete;
  cudaError_t alloc(size_t bytes) { return dev_malloc_async(&p, bytes, s); }
  ~AsyncBuf() {
    if (p) cudaFreeAsync(p, s);
  }
};

// message returned by qs_last_error() on the calling thread (state.cu)
void set_last_error(const std::string& msg);

}  // namespace qsb
