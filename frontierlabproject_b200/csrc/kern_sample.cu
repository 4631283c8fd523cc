// Measurement sampling: `shots` basis indices drawn from |psi|^2 (multinomial), on the device.
//
//   1. block sums of |psi(x)|^2 over blocks of kSampleBlock amplitudes (FP64);
//   2. exclusive prefix of the block sums (FP64: tiles of 4096 scanned per block, the tile totals
//      scanned, then added back);
//   3. sorted uniforms: u_(k) = C_k / C_{shots+1}, k = 1..shots, with C the prefix sums of
//      shots + 1 i.i.d. Exp(1) draws (the order statistics of `shots` uniforms), scaled by
//      the total probability;
//   4. one warp per probability block: the shots whose uniforms fall in the block's range
//      are located by binary search, the block is walked in 32-amplitude chunks with warp
//      prefix sums, and each shot takes the first amplitude whose cumulative sum exceeds it.
// Work O(2^n + shots); the result is the shots' indices in ascending order.
#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace qsb {

namespace {

constexpr int kSampleBlock = 1 << 12;  // amplitudes per probability block

template <typename C>
__global__ void block_prob_kernel(const C* __restrict__ psi, uint64_t dim, double* __restrict__ bsum) {
  __shared__ double part[32];
  const uint64_t b = blockIdx.x;
  const uint64_t x0 = b * kSampleBlock;
  double s = 0.0;
  for (uint64_t x = x0 + threadIdx.x; x < x0 + kSampleBlock && x < dim; x += blockDim.x) {
    const C v = psi[x];
    s += (double)v.x * v.x + (double)v.y * v.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) bsum[b] = w;
  }
}

constexpr int kScanThreads = 256, kScanItems = 16, kScanTile = kScanThreads * kScanItems;  // 4096 per tile

// Exclusive prefix of each kScanTile-element tile of v[0..n) in place (coalesced through shared
// memory: each thread scans 16 consecutive elements, the block scans the thread totals with warp
// shuffles); the tile's total goes to sums[tile].
__global__ void __launch_bounds__(kScanThreads) tile_scan_kernel(double* __restrict__ v, uint64_t n,
                                                                 double* __restrict__ sums) {
  __shared__ double sh[kScanTile];
  __shared__ double wsum[kScanThreads / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int j = 0; j < kScanItems; ++j) {
    const uint64_t i = base + t + j * kScanThreads;
    sh[t + j * kScanThreads] = i < n ? v[i] : 0.0;
  }
  __syncthreads();
  double loc[kScanItems];
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    loc[j] = s;
    s += sh[t * kScanItems + j];
  }
  double incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const double w = lane < kScanThreads / 32 ? wsum[lane] : 0.0;
    double wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < kScanThreads / 32) wsum[lane] = wi - w;  // exclusive over warps
  }
  __syncthreads();
  const double off = wsum[warp] + (incl - s);
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) sh[t * kScanItems + j] = loc[j] + off;
  if (t == kScanThreads - 1) sums[blockIdx.x] = off + s;
  __syncthreads();
  for (int j = 0; j < kScanItems; ++j) {
    const uint64_t i = base + t + j * kScanThreads;
    if (i < n) v[i] = sh[t + j * kScanThreads];
  }
}

// v[i] += pre[i / kScanTile] for i < n, and v[n] = pre[ntiles] (the total)
__global__ void add_tile_offsets_kernel(double* __restrict__ v, uint64_t n, const double* __restrict__ pre,
                                        uint64_t ntiles) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v[i] += pre[i / kScanTile];
  if (blockIdx.x == 0 && threadIdx.x == 0) v[n] = pre[ntiles];
}

// In-place exclusive prefix of v[0..n) with one block of 1024 threads; v[n] = total (for the
// tile totals, a few thousand entries).
__global__ void __launch_bounds__(1024) scan_kernel(double* __restrict__ v, uint64_t n) {
  __shared__ double part[1024];
  const uint64_t per = (n + 1023) / 1024;
  const uint64_t i0 = threadIdx.x * per, i1 = i0 + per < n ? i0 + per : n;
  double s = 0.0;
  for (uint64_t i = i0; i < i1; ++i) s += v[i];
  part[threadIdx.x] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan of the 1024 partial sums
  for (int off = 1; off < 1024; off <<= 1) {
    const double add = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0.0;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  double run = threadIdx.x ? part[threadIdx.x - 1] : 0.0;
  for (uint64_t i = i0; i < i1; ++i) {
    const double x = v[i];
    v[i] = run;
    run += x;
  }
  if (threadIdx.x == 1023) v[n] = part[1023];
}

// counter-based generator (SplitMix64 finaliser) -> uniform in (0, 1]
__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t k) {
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * (k + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return ((double)(z >> 11) + 1.0) * (1.0 / 9007199254740992.0);
}

__global__ void exp_draw_kernel(double* __restrict__ e, uint64_t n, uint64_t seed) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x)
    e[k] = -log(uniform01(seed, k));
}

// first index k in [lo, hi) with a[k] >= x (hi if none)
__device__ __forceinline__ uint64_t lower_bound(const double* a, uint64_t lo, uint64_t hi, double x) {
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// e: exclusive prefix of shots + 1 exponential draws, e[shots + 1] = their total: shot k's
// uniform is e[k+1] / e[shots+1], scaled here by the probability total bpre[nblocks]
template <typename C>
__global__ void assign_kernel(const C* __restrict__ psi, uint64_t dim, const double* __restrict__ bpre,
                              uint64_t nblocks, const double* __restrict__ e, uint64_t shots,
                              uint64_t* __restrict__ out) {
  const unsigned lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const double scale = bpre[nblocks] / e[shots + 1];
  for (uint64_t b = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); b < nblocks; b += warps) {
    const double lo = bpre[b], hi = bpre[b + 1];
    if (hi <= lo) continue;
    // shots with lo <= u < hi (u_k = e[k+1] * scale, nondecreasing in k); the last block
    // also takes any shot at or above its end (rounding of the totals)
    uint64_t k0 = lower_bound(e + 1, 0, shots, lo / scale);
    const uint64_t k1 = b + 1 == nblocks ? shots : lower_bound(e + 1, 0, shots, hi / scale);
    if (k0 >= k1) continue;
    double run = lo;
    const uint64_t x0 = b * kSampleBlock;
    for (uint64_t c = x0; c < x0 + kSampleBlock && c < dim && k0 < k1; c += 32) {
      const uint64_t x = c + lane;
      double p = 0.0;
      if (x < dim) { const C v = psi[x]; p = (double)v.x * v.x + (double)v.y * v.y; }
      double incl = p;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)lane >= o) incl += t;
      }
      const double chunk_end = run + __shfl_sync(0xffffffffu, incl, 31);
      const double my_end = run + incl;
      const bool last_chunk = c + 32 >= x0 + kSampleBlock || c + 32 >= dim;
      while (k0 < k1) {
        const double u = e[k0 + 1] * scale;
        if (u >= chunk_end && !last_chunk) break;
        // first lane whose cumulative end exceeds u (a shot past the end goes to the last lane)
        const unsigned m = __ballot_sync(0xffffffffu, my_end > u && p > 0.0);
        unsigned sel;
        if (m) sel = __ffs(m) - 1;
        else sel = 31 - __clz(__ballot_sync(0xffffffffu, p > 0.0) | 1u);
        if (lane == 0) out[k0] = c + sel;
        ++k0;
      }
      run = chunk_end;
    }
  }
}

uint64_t scan_tiles(uint64_t n) { return (n + kScanTile - 1) / kScanTile; }

// exclusive prefix of v[0..n) in place, v[n] = total; sums: scan_tiles(n) + 1 doubles
void device_scan(double* v, uint64_t n, double* sums, cudaStream_t s) {
  const uint64_t nt = scan_tiles(n);
  tile_scan_kernel<<<(unsigned)nt, kScanThreads, 0, s>>>(v, n, sums);
  scan_kernel<<<1, 1024, 0, s>>>(sums, nt);
  const uint64_t g = (n + 255) / 256;
  add_tile_offsets_kernel<<<(unsigned)(g < 4096 ? (g ? g : 1) : 4096), 256, 0, s>>>(v, n, sums, nt);
}

}  // namespace

size_t sample_scratch_bytes(int n, uint64_t shots) {
  const uint64_t nb = ((1ull << n) + kSampleBlock - 1) / kSampleBlock;
  return (nb + 1 + shots + 2 + scan_tiles(nb) + 1 + scan_tiles(shots + 1) + 1) * sizeof(double);
}

cudaError_t launch_sample(int dtype, const void* psi, int n, uint64_t shots, uint64_t seed, void* scratch,
                          uint64_t* out, cudaStream_t s) {
  const uint64_t dim = 1ull << n;
  const uint64_t nb = (dim + kSampleBlock - 1) / kSampleBlock;
  double* bsum = reinterpret_cast<double*>(scratch);   // nb + 1
  double* e = bsum + nb + 1;                           // shots + 2
  double* sums_b = e + shots + 2;                      // scan_tiles(nb) + 1
  double* sums_e = sums_b + scan_tiles(nb) + 1;        // scan_tiles(shots + 1) + 1
  if (dtype == 0) block_prob_kernel<float2><<<(unsigned)nb, 256, 0, s>>>((const float2*)psi, dim, bsum);
  else block_prob_kernel<double2><<<(unsigned)nb, 256, 0, s>>>((const double2*)psi, dim, bsum);
  device_scan(bsum, nb, sums_b, s);
  // shots + 1 draws into e[0..shots]; the exclusive scan leaves e[k+1] = sum of the first k+1
  // draws and e[shots+1] = the total
  const uint64_t g = (shots + 1 + 255) / 256;
  exp_draw_kernel<<<(unsigned)(g < 4096 ? g : 4096), 256, 0, s>>>(e, shots + 1, seed);
  device_scan(e, shots + 1, sums_e, s);
  const unsigned warps_per_block = 8;
  uint64_t grid = (nb + warps_per_block - 1) / warps_per_block;
  if (grid > 65535) grid = 65535;
  if (dtype == 0)
    assign_kernel<float2><<<(unsigned)grid, 32 * warps_per_block, 0, s>>>((const float2*)psi, dim, bsum, nb, e,
                                                                          shots, out);
  else
    assign_kernel<double2><<<(unsigned)grid, 32 * warps_per_block, 0, s>>>((const double2*)psi, dim, bsum, nb, e,
                                                                           shots, out);
  return cudaGetLastError();
}

}  // namespace qsb
