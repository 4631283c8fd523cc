// Adjoint differentiation kernels.
//
//  * zz_x_kernel: lam = H psi for H = sum_i a_i Z_i Z_{i+1} + b_i X_i (periodic), and the
//    FP64 partial sums of <psi|lam> (the energy).
//  * adjoint_gate1_kernel: one gate of the reverse sweep: with psi_k, lam_k the states after
//    gate k, accumulates Im <lam_k| G |psi_k> in FP64 (dE/dtheta of R(theta) = exp(-i theta G/2))
//    and uncomputes both states by U^dagger, in a single read+write of the two states.
//  * adjoint_gate2_kernel: a two-qubit gate of the reverse sweep (no parameter).
// Inner products accumulate per thread in FP64, reduce per block, one atomic per block.
#include <complex>
#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace qsb {

namespace {

template <typename Real> struct CxA;
template <> struct CxA<float> { using T = float2; };
template <> struct CxA<double> { using T = double2; };

struct Coef { double a[40], b[40]; };

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void block_add(double v, double* acc) {
  __shared__ double part[32];
  v = warp_sum_d(v);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
    w = warp_sum_d(w);
    if (threadIdx.x == 0) atomicAdd(acc, w);
  }
  __syncthreads();
}

// kStack (complex64): lam receives the stacked state of the gradient sweep instead,
// lam[2x] = psi[x] and lam[2x + 1] = (H psi)[x] (one 16-byte store).
template <typename C, bool kStack = false>
__global__ void zz_x_kernel(const C* __restrict__ psi, C* __restrict__ lam, int n, Coef cf, double* energy) {
  // sum_i a_i Z_i Z_{i+1} = A - 2 sum_{i: y_i = 1} a_i with y = x XOR (x rotated right by one bit)
  // (bit i of y: bits i and i+1 mod n differ); the partial sums of a over each 8-bit chunk of y
  // are tabulated per block
  __shared__ double s_tab[5][256];
  __shared__ double s_atot;
  for (int e = threadIdx.x; e < 5 * 256; e += blockDim.x) {
    const int c = e >> 8, v = e & 255;
    double t = 0.0;
    for (int j = 0; j < 8; ++j)
      if (((v >> j) & 1) && 8 * c + j < n) t += cf.a[8 * c + j];
    s_tab[c][v] = t;
  }
  if (threadIdx.x == 0) {
    double A = 0.0;
    for (int i = 0; i < n; ++i) A += cf.a[i];
    s_atot = A;
  }
  __syncthreads();
  const uint64_t dim = 1ull << n;
  const int nchunk = (n + 7) / 8;
  double e = 0.0;
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < dim; x += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t y = x ^ (((x >> 1) | ((x & 1ull) << (n - 1))) & (dim - 1));
    double ssum = 0.0;
    for (int c = 0; c < nchunk; ++c) ssum += s_tab[c][(y >> (8 * c)) & 255u];
    const double d = s_atot - 2.0 * ssum;
    const C p = psi[x];
    double re = d * p.x, im = d * p.y;
    for (int i = 0; i < n; ++i) {
      const C q = psi[x ^ (1ull << i)];
      re += cf.b[i] * q.x;
      im += cf.b[i] * q.y;
    }
    if constexpr (kStack) {
      reinterpret_cast<float4*>(lam)[x] = make_float4(p.x, p.y, (float)re, (float)im);
    } else {
      C out;
      out.x = re;
      out.y = im;
      lam[x] = out;
    }
    e += (double)p.x * re + (double)p.y * im;
  }
  block_add(e, energy);
}

template <typename C>
__device__ __forceinline__ C mulc(const C& u, const C& x) {
  C r;
  r.x = u.x * x.x - u.y * x.y;
  r.y = u.x * x.y + u.y * x.x;
  return r;
}
template <typename C>
__device__ __forceinline__ C addc(const C& a, const C& b) {
  C r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}

template <typename C> struct U2 { C u[4]; };
template <typename C> struct U4 { C u[16]; };

// generator: 0 none, 1 X, 2 Y, 3 Z
template <typename C>
__global__ void adjoint_gate1_kernel(C* __restrict__ psi, C* __restrict__ lam, int n, int q, U2<C> Ud, int gen,
                                     double* acc) {
  const uint64_t half = 1ull << (n - 1);
  const uint64_t lo = (1ull << q) - 1;
  double g = 0.0;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < half; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = ((k & ~lo) << 1) | (k & lo);
    const uint64_t i1 = i0 | (1ull << q);
    const C p0 = psi[i0], p1 = psi[i1], l0 = lam[i0], l1 = lam[i1];
    if (gen) {
      // (G psi) on the pair, then Im( conj(l0) g0 + conj(l1) g1 )
      double g0r, g0i, g1r, g1i;
      if (gen == 1) { g0r = p1.x; g0i = p1.y; g1r = p0.x; g1i = p0.y; }          // X
      else if (gen == 2) { g0r = p1.y; g0i = -p1.x; g1r = -p0.y; g1i = p0.x; }   // Y: (-i p1, i p0)
      else { g0r = p0.x; g0i = p0.y; g1r = -p1.x; g1i = -p1.y; }                 // Z
      g += (double)l0.x * g0i - (double)l0.y * g0r + (double)l1.x * g1i - (double)l1.y * g1r;
    }
    psi[i0] = addc(mulc(Ud.u[0], p0), mulc(Ud.u[1], p1));
    psi[i1] = addc(mulc(Ud.u[2], p0), mulc(Ud.u[3], p1));
    lam[i0] = addc(mulc(Ud.u[0], l0), mulc(Ud.u[1], l1));
    lam[i1] = addc(mulc(Ud.u[2], l0), mulc(Ud.u[3], l1));
  }
  if (gen) block_add(g, acc);
}

template <typename C>
__global__ void adjoint_gate2_kernel(C* __restrict__ psi, C* __restrict__ lam, int n, int q0, int q1, U4<C> Ud) {
  const int lo = q0 < q1 ? q0 : q1, hi = q0 < q1 ? q1 : q0;
  const uint64_t quarter = 1ull << (n - 2);
  const uint64_t mlo = (1ull << lo) - 1, mmid = (1ull << (hi - 1)) - 1;
  const uint64_t b0 = 1ull << q0, b1 = 1ull << q1;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < quarter; k += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t base = k & mlo;
    base |= ((k & mmid & ~mlo) << 1);
    base |= (k & ~mmid) << 2;
    const uint64_t idx[4] = {base, base | b0, base | b1, base | b0 | b1};
    C x[4], y[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) { x[c] = psi[idx[c]]; y[c] = lam[idx[c]]; }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      C s = mulc(Ud.u[4 * r], x[0]), t = mulc(Ud.u[4 * r], y[0]);
#pragma unroll
      for (int c = 1; c < 4; ++c) { s = addc(s, mulc(Ud.u[4 * r + c], x[c])); t = addc(t, mulc(Ud.u[4 * r + c], y[c])); }
      psi[idx[r]] = s;
      lam[idx[r]] = t;
    }
  }
}

int grid_of(uint64_t work, int threads) {
  static int sms = 0;
  if (!sms) sms = device_sm_count();
  uint64_t blocks = (work + threads - 1) / threads;
  const uint64_t cap = (uint64_t)sms * 8;
  return (int)(blocks < cap ? (blocks ? blocks : 1) : cap);
}

template <typename Real>
typename CxA<Real>::T cvt(std::complex<double> z) {
  typename CxA<Real>::T r;
  r.x = (Real)z.real();
  r.y = (Real)z.imag();
  return r;
}

}  // namespace

cudaError_t launch_zz_x(int dtype, const void* psi, void* lam, int n, const double* a, const double* b,
                        double* energy, cudaStream_t s) {
  Coef cf;
  for (int i = 0; i < 40; ++i) { cf.a[i] = i < n ? a[i] : 0.0; cf.b[i] = i < n ? b[i] : 0.0; }
  const int th = 256;
  const int grid = grid_of(1ull << n, th);
  if (dtype == 0) zz_x_kernel<float2><<<grid, th, 0, s>>>((const float2*)psi, (float2*)lam, n, cf, energy);
  else zz_x_kernel<double2><<<grid, th, 0, s>>>((const double2*)psi, (double2*)lam, n, cf, energy);
  return cudaGetLastError();
}

cudaError_t launch_zz_x_stack(const void* psi, void* phi, int n, const double* a, const double* b, double* energy,
                              cudaStream_t s) {
  Coef cf;
  for (int i = 0; i < 40; ++i) { cf.a[i] = i < n ? a[i] : 0.0; cf.b[i] = i < n ? b[i] : 0.0; }
  const int th = 256;
  const int grid = grid_of(1ull << n, th);
  zz_x_kernel<float2, true><<<grid, th, 0, s>>>((const float2*)psi, (float2*)phi, n, cf, energy);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_gate1(int dtype, void* psi, void* lam, int n, int q, const std::complex<double>* Ud,
                                 int gen, double* acc, cudaStream_t s) {
  const int th = 256;
  const int grid = grid_of(1ull << (n - 1), th);
  if (dtype == 0) {
    U2<float2> m;
    for (int i = 0; i < 4; ++i) m.u[i] = cvt<float>(Ud[i]);
    adjoint_gate1_kernel<float2><<<grid, th, 0, s>>>((float2*)psi, (float2*)lam, n, q, m, gen, acc);
  } else {
    U2<double2> m;
    for (int i = 0; i < 4; ++i) m.u[i] = cvt<double>(Ud[i]);
    adjoint_gate1_kernel<double2><<<grid, th, 0, s>>>((double2*)psi, (double2*)lam, n, q, m, gen, acc);
  }
  return cudaGetLastError();
}

cudaError_t launch_adjoint_gate2(int dtype, void* psi, void* lam, int n, int q0, int q1,
                                 const std::complex<double>* Ud, cudaStream_t s) {
  const int th = 256;
  const int grid = grid_of(1ull << (n - 2), th);
  if (dtype == 0) {
    U4<float2> m;
    for (int i = 0; i < 16; ++i) m.u[i] = cvt<float>(Ud[i]);
    adjoint_gate2_kernel<float2><<<grid, th, 0, s>>>((float2*)psi, (float2*)lam, n, q0, q1, m);
  } else {
    U4<double2> m;
    for (int i = 0; i < 16; ++i) m.u[i] = cvt<double>(Ud[i]);
    adjoint_gate2_kernel<double2><<<grid, th, 0, s>>>((double2*)psi, (double2*)lam, n, q0, q1, m);
  }
  return cudaGetLastError();
}

}  // namespace qsb
