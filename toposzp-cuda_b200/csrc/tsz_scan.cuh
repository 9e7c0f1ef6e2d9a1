// Device-wide scan of u32 arrays (reduce, scan of the tile partials, apply),
// with addition or maximum as the operator.  Used where a scan runs over
// millions of items (rank fallback), so that no stage is a single CTA walking
// the whole array.
#pragma once
#include <cuda_runtime.h>

namespace tsz {

constexpr int kScanThreads = 256;
constexpr int kScanPer = 16;
constexpr int kScanTile = kScanThreads * kScanPer;

struct OpAdd {
  __device__ __forceinline__ unsigned operator()(unsigned a, unsigned b) const { return a + b; }
};
struct OpMax {
  __device__ __forceinline__ unsigned operator()(unsigned a, unsigned b) const { return a > b ? a : b; }
};

template <class Op>
__device__ __forceinline__ unsigned warp_incl_scan(unsigned v, Op op) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = op(v, u);
  }
  return v;
}

// CTA-wide exclusive scan (identity 0) of one value per thread; total in *tot
template <class Op>
__device__ __forceinline__ unsigned cta_excl_scan_u32(unsigned v, Op op, unsigned *s_w, unsigned *tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned inc = warp_incl_scan(v, op);
  const unsigned ex_w = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  unsigned pre = 0, all = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
    if (w < warp) pre = op(pre, s_w[w]);
    all = op(all, s_w[w]);
  }
  __syncthreads();
  *tot = all;
  return op(pre, lane ? ex_w : 0u);
}

template <class Op>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const unsigned *__restrict__ in,
                                                                   unsigned long long n, unsigned *__restrict__ part) {
  __shared__ unsigned s_w[kScanThreads / 32];
  Op op;
  const unsigned long long t0 = (unsigned long long)blockIdx.x * kScanTile;
  unsigned v = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    const unsigned long long i = t0 + (unsigned long long)k * kScanThreads + threadIdx.x;
    if (i < n) v = op(v, in[i]);
  }
  unsigned tot;
  cta_excl_scan_u32(v, op, s_w, &tot);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// exclusive scan of the tile partials in place (one CTA, chunks of blockDim)
template <class Op>
__global__ void __launch_bounds__(1024) scan_partials_kernel(unsigned *__restrict__ part, unsigned ntiles) {
  __shared__ unsigned s_w[32];
  __shared__ unsigned s_carry;
  Op op;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (unsigned c = 0; c < ntiles; c += blockDim.x) {
    const unsigned i = c + threadIdx.x;
    const unsigned v = i < ntiles ? part[i] : 0u;
    unsigned tot;
    const unsigned ex = cta_excl_scan_u32(v, op, s_w, &tot);
    const unsigned carry = s_carry;
    if (i < ntiles) part[i] = op(carry, ex);
    __syncthreads();
    if (threadIdx.x == 0) s_carry = op(carry, tot);
    __syncthreads();
  }
}

// out[i] = carry-in of the tile (op) the scan of in over the tile, exclusive or inclusive
template <class Op>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const unsigned *__restrict__ in,
                                                                  unsigned long long n,
                                                                  const unsigned *__restrict__ part,
                                                                  unsigned *__restrict__ out, int inclusive) {
  __shared__ unsigned s_w[kScanThreads / 32];
  Op op;
  const unsigned long long t0 = (unsigned long long)blockIdx.x * kScanTile;
  // thread t owns items t0 + t*kScanPer .. +kScanPer-1 (consecutive)
  const unsigned long long b = t0 + (unsigned long long)threadIdx.x * kScanPer;
  unsigned v[kScanPer];
  unsigned s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    v[k] = (b + k < n) ? in[b + k] : 0u;
    s = op(s, v[k]);
  }
  unsigned tot;
  unsigned run = op(part[blockIdx.x], cta_excl_scan_u32(s, op, s_w, &tot));
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    if (b + k < n) {
      const unsigned nx = op(run, v[k]);
      out[b + k] = inclusive ? nx : run;
      run = nx;
    }
  }
}

// Scan of n items (in -> out, may alias); part: ceil(n / kScanTile) words of scratch.
template <class Op>
inline cudaError_t device_scan_u32(const unsigned *in, unsigned *out, unsigned long long n, unsigned *part,
                                   bool inclusive, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const unsigned ntiles = (unsigned)((n + kScanTile - 1) / kScanTile);
  scan_reduce_kernel<Op><<<ntiles, kScanThreads, 0, s>>>(in, n, part);
  scan_partials_kernel<Op><<<1, 1024, 0, s>>>(part, ntiles);
  scan_apply_kernel<Op><<<ntiles, kScanThreads, 0, s>>>(in, n, part, out, inclusive ? 1 : 0);
  return cudaGetLastError();
}

inline unsigned long long scan_parts(unsigned long long n) { return (n + kScanTile - 1) / kScanTile + 1; }

}  // namespace tsz
