// Device-wide scan of unsigned arrays (reduce, scan of the tile partials,
// apply), with addition or maximum as the operator, over 32- or 64-bit words.
// Used where a scan runs over millions of items (rank fallback, block offsets
// of the plain codec), so that no stage is a single CTA walking the whole
// array.
#pragma once
#include <cuda_runtime.h>

namespace tsz {

constexpr int kScanThreads = 256;
constexpr int kScanPer = 16;
constexpr int kScanTile = kScanThreads * kScanPer;

struct OpAdd {
  template <class V>
  __device__ __forceinline__ V operator()(V a, V b) const { return a + b; }
};
struct OpMax {
  template <class V>
  __device__ __forceinline__ V operator()(V a, V b) const { return a > b ? a : b; }
};

template <class V, class Op>
__device__ __forceinline__ V warp_incl_scan(V v, Op op) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const V u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v = op(v, u);
  }
  return v;
}

// CTA-wide exclusive scan (identity 0) of one value per thread; total in *tot
template <class V, class Op>
__device__ __forceinline__ V cta_excl_scan(V v, Op op, V *s_w, V *tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const V inc = warp_incl_scan(v, op);
  const V ex_w = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 31) s_w[warp] = inc;
  __syncthreads();
  V pre = 0, all = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
    if (w < warp) pre = op(pre, s_w[w]);
    all = op(all, s_w[w]);
  }
  __syncthreads();
  *tot = all;
  return op(pre, lane ? ex_w : V(0));
}

template <class V, class Op>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const V *__restrict__ in, unsigned long long n,
                                                                   V *__restrict__ part) {
  __shared__ V s_w[kScanThreads / 32];
  Op op;
  const unsigned long long t0 = (unsigned long long)blockIdx.x * kScanTile;
  V v = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    const unsigned long long i = t0 + (unsigned long long)k * kScanThreads + threadIdx.x;
    if (i < n) v = op(v, in[i]);
  }
  V tot;
  cta_excl_scan(v, op, s_w, &tot);
  if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

// exclusive scan of the tile partials in place (one CTA, chunks of blockDim)
template <class V, class Op>
__global__ void __launch_bounds__(1024) scan_partials_kernel(V *__restrict__ part, unsigned ntiles) {
  __shared__ V s_w[32];
  __shared__ V s_carry;
  Op op;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (unsigned c = 0; c < ntiles; c += blockDim.x) {
    const unsigned i = c + threadIdx.x;
    const V v = i < ntiles ? part[i] : V(0);
    V tot;
    const V ex = cta_excl_scan(v, op, s_w, &tot);
    const V carry = s_carry;
    if (i < ntiles) part[i] = op(carry, ex);
    __syncthreads();
    if (threadIdx.x == 0) s_carry = op(carry, tot);
    __syncthreads();
  }
}

// out[i] = carry-in of the tile (op) the scan of in over the tile, exclusive or inclusive
template <class V, class Op>
__global__ void __launch_bounds__(kScanThreads) scan_apply_kernel(const V *__restrict__ in, unsigned long long n,
                                                                  const V *__restrict__ part, V *__restrict__ out,
                                                                  int inclusive) {
  __shared__ V s_w[kScanThreads / 32];
  Op op;
  const unsigned long long t0 = (unsigned long long)blockIdx.x * kScanTile;
  // thread t owns items t0 + t*kScanPer .. +kScanPer-1 (consecutive)
  const unsigned long long b = t0 + (unsigned long long)threadIdx.x * kScanPer;
  V v[kScanPer];
  V s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    v[k] = (b + k < n) ? in[b + k] : V(0);
    s = op(s, v[k]);
  }
  V tot;
  V run = op(part[blockIdx.x], cta_excl_scan(s, op, s_w, &tot));
#pragma unroll
  for (int k = 0; k < kScanPer; k++) {
    if (b + k < n) {
      const V nx = op(run, v[k]);
      out[b + k] = inclusive ? nx : run;
      run = nx;
    }
  }
}

// Scan of n items (in -> out, may alias); part: scan_parts(n) words of scratch.
template <class V, class Op>
inline cudaError_t device_scan(const V *in, V *out, unsigned long long n, V *part, bool inclusive, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const unsigned ntiles = (unsigned)((n + kScanTile - 1) / kScanTile);
  scan_reduce_kernel<V, Op><<<ntiles, kScanThreads, 0, s>>>(in, n, part);
  scan_partials_kernel<V, Op><<<1, 1024, 0, s>>>(part, ntiles);
  scan_apply_kernel<V, Op><<<ntiles, kScanThreads, 0, s>>>(in, n, part, out, inclusive ? 1 : 0);
  return cudaGetLastError();
}

template <class Op>
inline cudaError_t device_scan_u32(const unsigned *in, unsigned *out, unsigned long long n, unsigned *part,
                                   bool inclusive, cudaStream_t s) {
  return device_scan<unsigned, Op>(in, out, n, part, inclusive, s);
}

inline unsigned long long scan_parts(unsigned long long n) { return (n + kScanTile - 1) / kScanTile + 1; }

}  // namespace tsz
