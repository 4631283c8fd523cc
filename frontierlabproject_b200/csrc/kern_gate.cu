// Per-gate kernels (one full sweep of the state per gate -- the "plain method"), the
// out-of-place scatter permutation with the reference's semantics, and FP64 reductions.
//
// Gate matrices travel as kernel parameters, so no device copy of the matrix exists
// whose lifetime could end before the kernel reads it.
#include <complex>
#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace qsb {

template <typename Real> struct Cx;
template <> struct Cx<float> { using T = float2; };
template <> struct Cx<double> { using T = double2; };

template <typename C> struct M2 { C u[4]; };
template <typename C> struct M4 { C u[16]; };
struct Map { int p[40]; };

template <typename C> __device__ __forceinline__ C mac2(C a, C x, C b, C y) {
  C r;
  r.x = a.x * x.x - a.y * x.y + b.x * y.x - b.y * y.y;
  r.y = a.x * x.y + a.y * x.x + b.x * y.y + b.y * y.x;
  return r;
}

static int grid_for(uint64_t work, int threads) {
  static int sms = 0;
  if (!sms) sms = device_sm_count();
  uint64_t blocks = (work + threads - 1) / threads;
  uint64_t cap = (uint64_t)sms * 16;
  return (int)(blocks < cap ? (blocks ? blocks : 1) : cap);
}

int device_sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

// 1q: pair (i0, i0 + 2^q); consecutive threads take consecutive i0 (coalesced).
template <typename C>
__global__ void gate1_kernel(C* __restrict__ psi, int n, int q, M2<C> U) {
  const uint64_t half = 1ull << (n - 1);
  const uint64_t lo = (1ull << q) - 1;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < half;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = ((k & ~lo) << 1) | (k & lo);
    const uint64_t i1 = i0 | (1ull << q);
    const C x = psi[i0], y = psi[i1];
    psi[i0] = mac2(U.u[0], x, U.u[1], y);
    psi[i1] = mac2(U.u[2], x, U.u[3], y);
  }
}

// 2q: matrix index b_q0 + 2 b_q1
template <typename C>
__global__ void gate2_kernel(C* __restrict__ psi, int n, int q0, int q1, M4<C> U) {
  const int lo = q0 < q1 ? q0 : q1, hi = q0 < q1 ? q1 : q0;
  const uint64_t quarter = 1ull << (n - 2);
  const uint64_t mlo = (1ull << lo) - 1, mmid = (1ull << (hi - 1)) - 1;
  const uint64_t b0 = 1ull << q0, b1 = 1ull << q1;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < quarter;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t base = k & mlo;
    base |= ((k & mmid & ~mlo) << 1);
    base |= (k & ~mmid) << 2;
    const uint64_t idx[4] = {base, base | b0, base | b1, base | b0 | b1};
    C x[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) x[c] = psi[idx[c]];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      C s = mac2(U.u[4 * r], x[0], U.u[4 * r + 1], x[1]);
      C t = mac2(U.u[4 * r + 2], x[2], U.u[4 * r + 3], x[3]);
      s.x += t.x; s.y += t.y;
      psi[idx[r]] = s;
    }
  }
}

template <typename C>
__global__ void diag1_kernel(C* __restrict__ psi, int n, int q, C d0, C d1) {
  const uint64_t dim = 1ull << n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
    const C d = (i >> q) & 1ull ? d1 : d0;
    const C x = psi[i];
    C r;
    r.x = x.x * d.x - x.y * d.y;
    r.y = x.x * d.y + x.y * d.x;
    psi[i] = r;
  }
}

template <typename C>
__global__ void permute_scatter_kernel(const C* __restrict__ in, C* __restrict__ out, int n, Map map) {
  const uint64_t dim = 1ull << n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t j = 0;
    for (int p = 0; p < n; ++p) j |= ((i >> p) & 1ull) << map.p[p];
    out[j] = in[i];
  }
}

template <typename C>
__global__ void set_basis_kernel(C* __restrict__ psi, int n, uint64_t index) {
  const uint64_t dim = 1ull << n;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
    C z;
    z.x = i == index ? 1 : 0;
    z.y = 0;
    psi[i] = z;
  }
}

// block-level FP64 reduction then one atomic per block
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename C>
__global__ void norm2_kernel(const C* __restrict__ psi, int n, double* acc) {
  __shared__ double part[32];
  const uint64_t dim = 1ull << n;
  double s = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
    const C x = psi[i];
    s += (double)x.x * x.x + (double)x.y * x.y;
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) atomicAdd(acc, v);
  }
}

// <a|b> = sum conj(a) b (a and b may differ in precision: complex64 against complex128)
template <typename CA, typename CB>
__global__ void inner_kernel(const CA* __restrict__ a, const CB* __restrict__ b, int n, double* acc) {
  __shared__ double pr[32], pi[32];
  const uint64_t dim = 1ull << n;
  double sr = 0.0, si = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
    const CA x = a[i];
    const CB y = b[i];
    sr += (double)x.x * y.x + (double)x.y * y.y;
    si += (double)x.x * y.y - (double)x.y * y.x;
  }
  sr = warp_sum(sr);
  si = warp_sum(si);
  if ((threadIdx.x & 31) == 0) { pr[threadIdx.x >> 5] = sr; pi[threadIdx.x >> 5] = si; }
  __syncthreads();
  if (threadIdx.x < 32) {
    const bool ok = threadIdx.x < (blockDim.x >> 5);
    double vr = ok ? pr[threadIdx.x] : 0.0, vi = ok ? pi[threadIdx.x] : 0.0;
    vr = warp_sum(vr);
    vi = warp_sum(vi);
    if (threadIdx.x == 0) { atomicAdd(acc, vr); atomicAdd(acc + 1, vi); }
  }
}

// ------------------------------------------------------------------------------------
template <typename Real>
static typename Cx<Real>::T cv(std::complex<double> z) {
  typename Cx<Real>::T r;
  r.x = (Real)z.real();
  r.y = (Real)z.imag();
  return r;
}

cudaError_t launch_gate1(int dtype, void* psi, int n, int q, const std::complex<double>* U, cudaStream_t s) {
  const int th = 256;
  const int grid = grid_for(1ull << (n - 1), th);
  if (dtype == 0) {
    M2<float2> m;
    for (int i = 0; i < 4; ++i) m.u[i] = cv<float>(U[i]);
    gate1_kernel<float2><<<grid, th, 0, s>>>((float2*)psi, n, q, m);
  } else {
    M2<double2> m;
    for (int i = 0; i < 4; ++i) m.u[i] = cv<double>(U[i]);
    gate1_kernel<double2><<<grid, th, 0, s>>>((double2*)psi, n, q, m);
  }
  return cudaGetLastError();
}

cudaError_t launch_gate2(int dtype, void* psi, int n, int q0, int q1, const std::complex<double>* U,
                         cudaStream_t s) {
  const int th = 256;
  const int grid = grid_for(1ull << (n - 2), th);
  if (dtype == 0) {
    M4<float2> m;
    for (int i = 0; i < 16; ++i) m.u[i] = cv<float>(U[i]);
    gate2_kernel<float2><<<grid, th, 0, s>>>((float2*)psi, n, q0, q1, m);
  } else {
    M4<double2> m;
    for (int i = 0; i < 16; ++i) m.u[i] = cv<double>(U[i]);
    gate2_kernel<double2><<<grid, th, 0, s>>>((double2*)psi, n, q0, q1, m);
  }
  return cudaGetLastError();
}

cudaError_t launch_diag1(int dtype, void* psi, int n, int q, std::complex<double> d0, std::complex<double> d1,
                         cudaStream_t s) {
  const int th = 256;
  const int grid = grid_for(1ull << n, th);
  if (dtype == 0) diag1_kernel<float2><<<grid, th, 0, s>>>((float2*)psi, n, q, cv<float>(d0), cv<float>(d1));
  else diag1_kernel<double2><<<grid, th, 0, s>>>((double2*)psi, n, q, cv<double>(d0), cv<double>(d1));
  return cudaGetLastError();
}

cudaError_t launch_permute_scatter(int dtype, const void* in, void* out, int n, const int* map, cudaStream_t s) {
  Map mp;
  for (int p = 0; p < 40; ++p) mp.p[p] = p < n ? map[p] : 0;
  const int th = 256;
  const int grid = grid_for(1ull << n, th);
  if (dtype == 0) permute_scatter_kernel<float2><<<grid, th, 0, s>>>((const float2*)in, (float2*)out, n, mp);
  else permute_scatter_kernel<double2><<<grid, th, 0, s>>>((const double2*)in, (double2*)out, n, mp);
  return cudaGetLastError();
}

cudaError_t launch_norm2(int dtype, const void* psi, int n, double* acc, cudaStream_t s) {
  const int th = 512;
  const int grid = grid_for(1ull << n, th);
  if (dtype == 0) norm2_kernel<float2><<<grid, th, 0, s>>>((const float2*)psi, n, acc);
  else norm2_kernel<double2><<<grid, th, 0, s>>>((const double2*)psi, n, acc);
  return cudaGetLastError();
}

cudaError_t launch_inner(int dtype, const void* a, const void* b, int n, double* acc2, cudaStream_t s) {
  return launch_inner_mixed(dtype, a, dtype, b, n, acc2, s);
}

cudaError_t launch_inner_mixed(int dtype_a, const void* a, int dtype_b, const void* b, int n, double* acc2,
                               cudaStream_t s) {
  const int th = 512;
  const int grid = grid_for(1ull << n, th);
  if (dtype_a == 0 && dtype_b == 0)
    inner_kernel<float2, float2><<<grid, th, 0, s>>>((const float2*)a, (const float2*)b, n, acc2);
  else if (dtype_a == 0)
    inner_kernel<float2, double2><<<grid, th, 0, s>>>((const float2*)a, (const double2*)b, n, acc2);
  else if (dtype_b == 0)
    inner_kernel<double2, float2><<<grid, th, 0, s>>>((const double2*)a, (const float2*)b, n, acc2);
  else
    inner_kernel<double2, double2><<<grid, th, 0, s>>>((const double2*)a, (const double2*)b, n, acc2);
  return cudaGetLastError();
}

cudaError_t launch_set_basis(int dtype, void* psi, int n, uint64_t index, cudaStream_t s) {
  const int th = 256;
  const int grid = grid_for(1ull << n, th);
  if (dtype == 0) set_basis_kernel<float2><<<grid, th, 0, s>>>((float2*)psi, n, index);
  else set_basis_kernel<double2><<<grid, th, 0, s>>>((double2*)psi, n, index);
  return cudaGetLastError();
}

}  // namespace qsb
