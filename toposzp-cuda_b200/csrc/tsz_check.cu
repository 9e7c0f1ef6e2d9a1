// Topology report of a decompressed field against its original: critical
// points preserved / lost / changed / new, the pointwise error against the
// bound, and the local order of adjacent points.  The counts follow the
// reference drivers' verification steps (example/test_cuda_topology.cu:540-602
// preservation and new points, :636-660 error bound, :800-868 local order of
// adjacent interior pairs; example/test_cuda_topology_3d.cu:636-730 for 3D,
// whose driver checks preservation and the bound only: the order check is
// extended here to the three axes).  Acceptance in the reference:
// max error <= 2 eb and more than 90 % of the critical points preserved
// (example/test_cuda_topology.cu:1052, example/test_cuda_topology_3d.cu:829).
//
// One pass over the field: CTAs take rows (fixed x, y; all z) from a grid-
// stride loop, classify each interior point in both fields, and reduce their
// counters per CTA before one atomic per counter.
#include <cfloat>
#include <cstring>

#include "tsz_ops.h"

namespace tsz {

// counter slots of the report (device words)
enum : int {
  kRepOrig = 0,        // 0..3: original critical points, [0] total, [t] by type t
  kRepDec = 4,         // 4..7: decompressed critical points
  kRepPreserved = 8,
  kRepLost = 9,
  kRepChanged = 10,
  kRepNew = 11,
  kRepLostType = 12,   // 12..15: lost by original type
  kRepPairs = 16,      // 16..19: adjacent pairs with a strict original order: all, >= 1 CP, both CPs, >= 1 extremum
  kRepViol = 20,       // 20..23: the same pairs whose order changed
  kRepOver1 = 24,      // error > 1.01 eb
  kRepOver2 = 25,      // error > 2 eb
  kRepMaxErr = 26,     // bits of the largest error (double, non-negative)
  kRepWords = 27,
};

__device__ __forceinline__ int cls_at(const float *__restrict__ f, long long q, const Geom &g) {
  if (g.nd == 2) return classify4(f[q], f[q - g.d3], f[q + g.d3], f[q - 1], f[q + 1]);
  return classify6(f[q], f[q - g.plane], f[q + g.plane], f[q - g.d3], f[q + g.d3], f[q - 1], f[q + 1]);
}

__device__ __forceinline__ int order_of(float a, float b) { return (a < b) ? -1 : ((a > b) ? 1 : 0); }

__global__ void __launch_bounds__(256) topo_report_kernel(const float *__restrict__ orig,
                                                          const float *__restrict__ dec, Geom g, float eb,
                                                          unsigned long long *__restrict__ out) {
  __shared__ unsigned long long s_cnt[kRepWords];
  for (int i = threadIdx.x; i < kRepWords; i += blockDim.x) s_cnt[i] = 0ull;
  __syncthreads();
  unsigned c[kRepMaxErr];
#pragma unroll
  for (int i = 0; i < kRepMaxErr; i++) c[i] = 0u;
  double maxerr = 0.0;
  const long long rows = g.d1 * g.d2;
  const double lim1 = (double)eb * 1.01, lim2 = (double)eb * 2.0;
  for (long long row = blockIdx.x; row < rows; row += gridDim.x) {
    const long long x = (g.nd == 2) ? 0 : row / g.d2;
    const long long y = (g.nd == 2) ? row : row - x * g.d2;
    const long long base = row * g.d3;
    const bool row_in = y >= 1 && y <= g.d2 - 2 && (g.nd == 2 || (x >= 1 && x <= g.d1 - 2));
    for (long long z = threadIdx.x; z < g.d3; z += blockDim.x) {
      const long long q = base + z;
      const double e = fabs((double)orig[q] - (double)dec[q]);
      if (e > maxerr) maxerr = e;   // a NaN difference never compares greater, as in the reference
      if (e > lim1) c[kRepOver1]++;
      if (e > lim2) c[kRepOver2]++;
      if (!row_in || z < 1 || z > g.d3 - 2) continue;
      const int to = cls_at(orig, q, g), td = cls_at(dec, q, g);
      // (counters indexed by compile-time constants only: they stay in registers)
      const bool lost = to && td == 0;
      c[kRepOrig] += to != 0;
      c[kRepDec] += td != 0;
#pragma unroll
      for (int t = 1; t <= 3; t++) {
        c[kRepOrig + t] += to == t;
        c[kRepDec + t] += td == t;
        c[kRepLostType + t] += lost && to == t;
      }
      c[kRepPreserved] += to && td == to;
      c[kRepLost] += lost;
      c[kRepChanged] += to && td && td != to;
      c[kRepNew] += td && !to;
      // pairs with the next interior point along each axis
      const float oa = orig[q], da = dec[q];
#pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        long long stride;
        bool ok;
        if (ax == 0) { stride = 1; ok = z + 1 <= g.d3 - 2; }
        else if (ax == 1) { stride = g.d3; ok = y + 1 <= g.d2 - 2; }
        else { stride = g.plane; ok = g.nd == 3 && x + 1 <= g.d1 - 2; }
        if (!ok) continue;
        const long long b = q + stride;
        const int oo = order_of(oa, orig[b]);
        if (oo == 0) continue;
        const bool viol = order_of(da, dec[b]) != oo;
        const int tb = cls_at(orig, b, g);
        c[kRepPairs]++;
        if (viol) c[kRepViol]++;
        if (to || tb) { c[kRepPairs + 1]++; if (viol) c[kRepViol + 1]++; }
        if (to && tb) { c[kRepPairs + 2]++; if (viol) c[kRepViol + 2]++; }
        if (to == 1 || to == 2 || tb == 1 || tb == 2) { c[kRepPairs + 3]++; if (viol) c[kRepViol + 3]++; }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kRepMaxErr; i++) {
    const unsigned v = __reduce_add_sync(0xffffffffu, c[i]);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&s_cnt[i], (unsigned long long)v);
  }
  // non-negative doubles order like their bit patterns
  unsigned long long mb = (unsigned long long)__double_as_longlong(maxerr);
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long u = __shfl_xor_sync(0xffffffffu, mb, o);
    mb = u > mb ? u : mb;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(&s_cnt[kRepMaxErr], mb);
  __syncthreads();
  for (int i = threadIdx.x; i < kRepWords; i += blockDim.x) {
    const unsigned long long v = s_cnt[i];
    if (i == kRepMaxErr) atomicMax(&out[i], v);
    else if (v) atomicAdd(&out[i], v);
  }
}

}  // namespace tsz

using namespace tsz;

extern "C" SZP_B200_API int szp_b200_topo_check(szp_b200_ctx *ctx, const float *d_orig, const float *d_dec,
                                                szp_b200_geom geom, float absErrBound,
                                                szp_b200_topo_report *report) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !d_orig || !d_dec || !report) { set_error("szp_b200_topo_check: null argument"); return -1; }
  unsigned long long n;
  Geom g;
  if (!geom_elements(geom, &n, &g)) { set_error("szp_b200_topo_check: invalid geometry"); return -1; }
  if (!ctx->scratch.reserve(kRepWords * 8 + 256)) return -1;
  unsigned long long *w = ctx->scratch.take<unsigned long long>(kRepWords);
  cudaStream_t s = ctx->stream;
  if (cuda_fail(cudaMemsetAsync(w, 0, kRepWords * 8, s), "memset")) return -1;
  const long long rows = g.d1 * g.d2;
  const long long grid = rows < (long long)ctx->sm_count * 16 ? rows : (long long)ctx->sm_count * 16;
  topo_report_kernel<<<(unsigned)(grid > 0 ? grid : 1), 256, 0, s>>>(d_orig, d_dec, g, absErrBound, w);
  if (cuda_fail(cudaGetLastError(), "topology report launch")) return -1;
  ctx->launches += 1;
  unsigned long long h[kRepWords];
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words, w, kRepWords * 8, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "topology report"))
    return -1;
  for (int i = 0; i < kRepWords; i++) h[i] = ctx->h_words[i];
  for (int i = 0; i < 4; i++) {
    report->orig_cps[i] = h[kRepOrig + i];
    report->dec_cps[i] = h[kRepDec + i];
    report->lost_by_type[i] = h[kRepLostType + i];
    report->pairs[i] = h[kRepPairs + i];
    report->violations[i] = h[kRepViol + i];
  }
  report->preserved = h[kRepPreserved];
  report->lost = h[kRepLost];
  report->changed = h[kRepChanged];
  report->new_cps = h[kRepNew];
  report->over_1eb = h[kRepOver1];
  report->over_2eb = h[kRepOver2];
  std::memcpy(&report->max_err, &h[kRepMaxErr], 8);
  return 0;
}
