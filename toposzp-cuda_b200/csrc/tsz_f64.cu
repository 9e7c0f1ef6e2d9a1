// fp64 3D topology compression: the reference's double-precision path
// (SZp/src/szp_cuda_topology_3d.cu:1066-1188, API
// SZp/include/szp_cuda_topology_3d.cuh:34-38).
//
//   1. types from the caller's critical-point list (x, y, z in range, type 1..3)
//   2. q = (int)(x * (1/eb)) in double (:641-646)
//   3. three saddle-repair passes in q-space (:736-826, driven at :1125-1145):
//      each pass reads a snapshot of q and rewrites the interior saddles
//      (type 3) whose saddle shape the quantization broke with the first of
//      c, c - 1, c + 1 that is high along one axis, low along another and
//      keeps every neighbouring maximum above / minimum below it
//   4. the topology block layout over the repaired ints with 2-bit tags
//      (:836-958): [u64 0][blocks], the same stream format as the fp32 path.
//
// Layout of the work on the device.  The reference snapshots the whole q
// array before each pass (a 4N device copy) and runs one thread per interior
// voxel.  Only saddles change, and a pass reads nothing but the saddles and
// their six neighbours, so here:
//   * one streaming kernel quantizes the field (8 elements per thread, 16-byte
//     loads and stores) and, for every interior saddle it meets, evaluates
//     pass 1 on the spot from the doubles of the six neighbours (pass 1's
//     snapshot is the plain quantization, so q of a neighbour is its own
//     quantized double) and writes the repaired value; the saddle's index goes
//     to a compact list (warp-aggregated append)
//   * passes 2 and 3 run over that list only: an evaluation kernel reads q and
//     writes the pass's new saddle values to a side array (the snapshot), an
//     apply kernel scatters them back
//   * the octet encoder (int values with tags) writes the stream.
// HBM traffic per element: 8 B read + 1 B types read + 4 B write (quantize),
// 4 B + 1 B read and the stream written (encode); saddle passes touch only
// the saddles' neighbourhoods.
#include <cstdlib>
#include <cstring>

#include "tsz_ops.h"

namespace tsz {

constexpr int kF64Threads = 256;

// (int)(x * inv): the reference kernel's C conversion (see quantize)
__device__ __forceinline__ int quantize_f64(double x, double inv) { return (int)__dmul_rn(x, inv); }

// Interior voxel of a 3D grid with all extents >= 3, whose +x neighbour is an
// element of the field (i + plane < n).
__device__ __forceinline__ bool interior3(long long i, const Geom &g, unsigned long long n) {
  if (g.d1 < 3 || g.d2 < 3 || g.d3 < 3) return false;
  long long r, z;
  const long long x = fdivmod(i, g.plane, g.m_plane, r);
  const long long y = fdivmod(r, g.d3, g.m_d3, z);
  return x >= 1 && x <= g.d1 - 2 && y >= 1 && y <= g.d2 - 2 && z >= 1 && z <= g.d3 - 2 &&
         (unsigned long long)(i + g.plane) < n;
}

// The repair of one saddle from its value c, its six neighbours v (x-, x+,
// y-, y+, z-, z+) and their types; returns c when the saddle shape holds or
// no candidate qualifies.  Integer arithmetic wraps (c - 1 at INT_MIN).
__device__ __forceinline__ int repair_saddle(int c, const int v[6], const unsigned t[6]) {
  int hi[3], lo[3], nh = 0, nl = 0;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    hi[a] = max(v[2 * a], v[2 * a + 1]);
    lo[a] = min(v[2 * a], v[2 * a + 1]);
    nh += c > hi[a];
    nl += c < lo[a];
  }
  if (nh >= 1 && nl >= 1) return c;
  // c itself fails the shape test above, so the candidates that remain are
  // c - 1 and then c + 1
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const int tv = (int)((unsigned)c + (k == 0 ? 0xffffffffu : 1u));
    int th = 0, tl = 0;
#pragma unroll
    for (int a = 0; a < 3; a++) { th += tv > hi[a]; tl += tv < lo[a]; }
    if (th < 1 || tl < 1) continue;
    bool ok = true;
#pragma unroll
    for (int j = 0; j < 6; j++) {
      if (t[j] == 1 && v[j] <= tv) ok = false;
      if (t[j] == 2 && v[j] >= tv) ok = false;
    }
    if (ok) return tv;
  }
  return c;
}

__device__ __forceinline__ void neighbour_offsets(const Geom &g, long long o[6]) {
  o[0] = -g.plane; o[1] = g.plane; o[2] = -g.d3; o[3] = g.d3; o[4] = -1; o[5] = 1;
}

// Quantize + pass 1 + saddle list.  Threads own 8 consecutive elements; a
// CTA sweeps tiles of kF64Threads * 8 elements in a grid-stride loop whose
// trip count is uniform over the CTA (for the warp-aggregated append).
__global__ void __launch_bounds__(kF64Threads) f64_quantize_kernel(const double *__restrict__ d, int *__restrict__ q,
                                                                   unsigned long long n, double inv,
                                                                   const unsigned char *__restrict__ ty, Geom g,
                                                                   unsigned long long *__restrict__ list,
                                                                   unsigned long long cap,
                                                                   unsigned long long *__restrict__ count,
                                                                   int repair, int *__restrict__ err) {
  const bool vec = ((reinterpret_cast<uintptr_t>(d) | reinterpret_cast<uintptr_t>(q)) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(ty) & 7) == 0;
  const unsigned long long octs = (n + 7) / 8;
  const int lane = threadIdx.x & 31;
  long long off[6];
  neighbour_offsets(g, off);
  for (unsigned long long o0 = (unsigned long long)blockIdx.x * kF64Threads; o0 < octs;
       o0 += (unsigned long long)gridDim.x * kF64Threads) {
    const unsigned long long oct = o0 + threadIdx.x;
    const long long i0 = (long long)oct * 8;
    int qv[8];
    unsigned tyw[8];
    int nv = 0;
    if (oct < octs) {
      nv = (int)((n - (unsigned long long)i0) < 8 ? (n - (unsigned long long)i0) : 8);
      if (vec && nv == 8) {
        const double2 *p = reinterpret_cast<const double2 *>(d + i0);
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const double2 u = __ldcs(p + k);
          qv[2 * k] = quantize_f64(u.x, inv);
          qv[2 * k + 1] = quantize_f64(u.y, inv);
        }
        const unsigned long long w = __ldg(reinterpret_cast<const unsigned long long *>(ty + i0));
#pragma unroll
        for (int t = 0; t < 8; t++) tyw[t] = (unsigned)(w >> (8 * t)) & 0xffu;
      } else {
#pragma unroll
        for (int t = 0; t < 8; t++) {
          qv[t] = t < nv ? quantize_f64(d[i0 + t], inv) : 0;
          tyw[t] = t < nv ? (unsigned)ty[i0 + t] : 0u;
        }
      }
    }
    // saddles: pass 1 against the plain quantization of the neighbours
    unsigned smask = 0;
#pragma unroll
    for (int t = 0; t < 8; t++) {
      if (t < nv && tyw[t] == 3u && interior3(i0 + t, g, n)) {
        smask |= 1u << t;
        if (!repair) continue;
        int v[6];
        unsigned tt[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {
          const long long b = i0 + t + off[j];
          v[j] = quantize_f64(__ldg(d + b), inv);
          tt[j] = __ldg(ty + b);
        }
        qv[t] = repair_saddle(qv[t], v, tt);
      }
    }
    if (nv == 8 && vec) {
      int4 *p = reinterpret_cast<int4 *>(q + i0);
      __stcs(p, make_int4(qv[0], qv[1], qv[2], qv[3]));
      __stcs(p + 1, make_int4(qv[4], qv[5], qv[6], qv[7]));
    } else {
#pragma unroll
      for (int t = 0; t < 8; t++) if (t < nv) q[i0 + t] = qv[t];
    }
    // warp-aggregated append of the saddle indices
    const unsigned c = __popc(smask);
    unsigned inc = c;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      const unsigned u = __shfl_up_sync(0xffffffffu, inc, s);
      if (lane >= s) inc += u;
    }
    const unsigned tot = __shfl_sync(0xffffffffu, inc, 31);
    unsigned long long base = 0;
    if (lane == 31 && tot) base = atomicAdd(count, (unsigned long long)tot);
    base = __shfl_sync(0xffffffffu, base, 31);
    unsigned long long pos = base + (inc - c);
    for (unsigned m = smask; m; m &= m - 1) {
      const int t = __ffs(m) - 1;
      if (pos < cap) list[pos] = (unsigned long long)(i0 + t);
      else atomicOr(err, 1);
      pos++;
    }
  }
}

// One repair pass over the saddle list: the new value of every listed saddle
// from q (the pass's snapshot) into nv.
__global__ void __launch_bounds__(kF64Threads) f64_repair_eval_kernel(const int *__restrict__ q,
                                                                      const unsigned char *__restrict__ ty, Geom g,
                                                                      const unsigned long long *__restrict__ list,
                                                                      const unsigned long long *__restrict__ count,
                                                                      unsigned long long cap, int *__restrict__ nv) {
  const unsigned long long k = *count < cap ? *count : cap;
  long long off[6];
  neighbour_offsets(g, off);
  for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < k;
       j += (unsigned long long)gridDim.x * blockDim.x) {
    const long long p = (long long)list[j];
    int v[6];
    unsigned tt[6];
#pragma unroll
    for (int a = 0; a < 6; a++) {
      v[a] = __ldg(q + p + off[a]);
      tt[a] = __ldg(ty + p + off[a]);
    }
    nv[j] = repair_saddle(__ldg(q + p), v, tt);
  }
}

__global__ void __launch_bounds__(kF64Threads) f64_repair_apply_kernel(int *__restrict__ q,
                                                                       const unsigned long long *__restrict__ list,
                                                                       const unsigned long long *__restrict__ count,
                                                                       unsigned long long cap,
                                                                       const int *__restrict__ nv) {
  const unsigned long long k = *count < cap ? *count : cap;
  for (unsigned long long j = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; j < k;
       j += (unsigned long long)gridDim.x * blockDim.x)
    q[list[j]] = nv[j];
}

// Device scratch of one fp64 compression of n elements with at most `cps`
// critical points (types, q, saddle list and side values, tile descriptors).
static size_t f64_scratch_bytes(unsigned long long n, unsigned long long cps, int B) {
  const unsigned long long nb = (n + B - 1) / B;
  const unsigned long long cap = cps < n ? cps : n;
  return a256(n) + a256(n * 4) + a256(cap * 8 + 8) + a256(cap * 4 + 4) +
         a256((nb / enc_tile_blocks(B) + 2) * sizeof(TileDesc)) + 4096;
}

// Steps 1-4 on ctx->stream.  d_cps: `count` CriticalPoint3D records on the
// device (may be null when count is 0).  Writes the stream ([u64 0][blocks])
// to d_out and its length to *out_len.  Scratch must hold f64_scratch_bytes.
static int f64_compress_impl(szp_b200_ctx *ctx, const double *d_data, unsigned long long n, const Geom &g,
                             double eb, int B, const int *d_cps, long long count, int passes,
                             unsigned char *d_out, unsigned long long out_cap, unsigned long long *out_len,
                             int *d_q_out) {
  cudaStream_t s = ctx->stream;
  const unsigned long long cap = (unsigned long long)count < n ? (unsigned long long)count : n;
  unsigned char *d_types = ctx->scratch.take<unsigned char>(n);
  int *d_q = d_q_out ? d_q_out : ctx->scratch.take<int>(n);
  unsigned long long *d_list = ctx->scratch.take<unsigned long long>(cap + 1);
  int *d_nv = ctx->scratch.take<int>(cap + 1);
  if (!d_types || !d_q || !d_list || !d_nv) { set_error("scratch arena too small"); return -1; }
  unsigned long long *w = ctx->d_words;  // [5] saddle count, [6] status
  int *w_err = reinterpret_cast<int *>(w + 6);
  if (cuda_fail(cudaMemsetAsync(d_types, 0, n, s), "memset types") ||
      cuda_fail(cudaMemsetAsync(w + 5, 0, 16, s), "memset words"))
    return -1;
  if (count > 0) {
    if (cuda_fail(launch_mark_types(d_cps, 6, count, g, n, d_types, s), "mark types")) return -1;
    ctx->launches += 1;
  }
  const unsigned long long octs = (n + 7) / 8;
  const unsigned long long qg = (octs + kF64Threads - 1) / kF64Threads;
  const unsigned qgrid = (unsigned)(qg < (unsigned long long)ctx->sm_count * 8 ? qg : (unsigned long long)ctx->sm_count * 8);
  const double inv = 1.0 / eb;
  f64_quantize_kernel<<<qgrid ? qgrid : 1, kF64Threads, 0, s>>>(d_data, d_q, n, inv, d_types, g, d_list, cap, w + 5,
                                                                 passes > 0 ? 1 : 0, w_err);
  if (cuda_fail(cudaGetLastError(), "fp64 quantize launch")) return -1;
  ctx->launches += 1;
  if (cap > 0) {
    const unsigned long long lg = (cap + kF64Threads - 1) / kF64Threads;
    const unsigned grid = (unsigned)(lg < (unsigned long long)ctx->sm_count * 8 ? lg : (unsigned long long)ctx->sm_count * 8);
    for (int p = 1; p < passes; p++) {
      f64_repair_eval_kernel<<<grid, kF64Threads, 0, s>>>(d_q, d_types, g, d_list, w + 5, cap, d_nv);
      f64_repair_apply_kernel<<<grid, kF64Threads, 0, s>>>(d_q, d_list, w + 5, cap, d_nv);
      if (cuda_fail(cudaGetLastError(), "saddle repair launch")) return -1;
      ctx->launches += 2;
    }
  }
  // the encoder clears words 0..7 when it starts: read the status first
  int st = 0;
  if (cuda_fail(cudaMemcpyAsync(&ctx->h_words[6], w + 6, 8, cudaMemcpyDeviceToHost, s), "D2H status") ||
      cuda_fail(cudaStreamSynchronize(s), "saddle repair"))
    return -1;
  st = (int)(ctx->h_words[6] & 0xffffffffu);
  if (st) { set_error("saddle list overflow (status %d)", st); return -1; }
  unsigned long long tot[3];
  if (encode_pass(ctx, kEncIntTypes, nullptr, d_q, d_types, n, B, 1.0f, g, d_out, out_cap, nullptr, kCpNone,
                  nullptr, 0, tot))
    return -1;
  *out_len = 8 + tot[0];
  return 0;
}

}  // namespace tsz

using namespace tsz;

extern "C" {

SZP_B200_API size_t szp_b200_f64_topo_scratch_bytes(size_t n, size_t critical_count, int blockSize) {
  if (n == 0 || blockSize <= 0) return 0;
  return f64_scratch_bytes(n, critical_count, blockSize);
}

SZP_B200_API int szp_b200_double_compress_topology_3d_dev(szp_b200_ctx *ctx, const double *d_data,
                                                          szp_b200_geom geom, double absErrBound, int blockSize,
                                                          const CriticalPoint3D *d_cps, size_t critical_count,
                                                          int passes, unsigned char *d_out, size_t out_cap,
                                                          size_t *out_len, int *d_q) {
  clear_error();
  DeviceGuard dg(ctx);
  if (!ctx || !d_data || !d_out || !out_len) { set_error("szp_b200_double_compress_topology_3d_dev: null argument"); return -1; }
  *out_len = 0;
  unsigned long long n;
  Geom g;
  if (geom.nd != 3 || !geom_elements(geom, &n, &g)) {
    set_error("szp_b200_double_compress_topology_3d_dev: invalid 3D geometry");
    return -1;
  }
  if (!(absErrBound > 0.0)) { set_error("szp_b200_double_compress_topology_3d_dev: error bound must be > 0"); return -1; }
  if (!valid_block_size(blockSize, "szp_b200_double_compress_topology_3d_dev")) return -1;
  if (critical_count > 0 && !d_cps) { set_error("szp_b200_double_compress_topology_3d_dev: null critical points"); return -1; }
  if (critical_count > (size_t)0x7fffffffffffll) { set_error("szp_b200_double_compress_topology_3d_dev: too many critical points"); return -1; }
  if (passes < 0 || passes > 64) { set_error("szp_b200_double_compress_topology_3d_dev: passes must be in [0, 64]"); return -1; }
  if (out_cap < topo_stream_bound(n, blockSize)) {
    set_error("szp_b200_double_compress_topology_3d_dev: output capacity %zu below the bound %zu", out_cap,
              topo_stream_bound(n, blockSize));
    return -1;
  }
  if (!ctx->scratch.reserve(f64_scratch_bytes(n, critical_count, blockSize))) return -1;
  unsigned long long len = 0;
  if (f64_compress_impl(ctx, d_data, n, g, absErrBound, blockSize, reinterpret_cast<const int *>(d_cps),
                        (long long)critical_count, passes, d_out, out_cap, &len, d_q))
    return -1;
  *out_len = len;
  return 0;
}

unsigned char *szp_cuda_double_compress_topology_3d(double *oriData, size_t *outSize, double absErrBound,
                                                    size_t nbEle, int blockSize, CriticalPoint3D *critical_points,
                                                    int critical_count, int d1, int d2, int d3) {
  clear_error();
  if (!outSize) { set_error("szp_cuda_double_compress_topology_3d: null outSize"); return nullptr; }
  *outSize = 0;
  if (absErrBound <= 0.0 || !oriData || nbEle == 0) return nullptr;
  if (!valid_block_size(blockSize, "szp_cuda_double_compress_topology_3d")) return nullptr;
  if (d1 <= 0 || d2 <= 0 || d3 <= 0) {
    set_error("szp_cuda_double_compress_topology_3d: invalid dimensions %d x %d x %d", d1, d2, d3);
    return nullptr;
  }
  if (nbEle >= kMaxElements) { set_error("szp_cuda_double_compress_topology_3d: too many elements"); return nullptr; }
  szp_b200_ctx *ctx = default_ctx();
  if (!ctx) return nullptr;
  const unsigned long long n = nbEle;
  const long long count = (critical_points && critical_count > 0) ? critical_count : 0;
  const size_t cap = topo_stream_bound(n, blockSize);
  const size_t need = a256(n * 8) + a256((size_t)count * sizeof(CriticalPoint3D) + 8) + a256(cap) +
                      f64_scratch_bytes(n, (unsigned long long)count, blockSize);
  if (!ctx->scratch.reserve(need)) return nullptr;
  double *d_data = ctx->scratch.take<double>(n);
  int *d_cps = count ? ctx->scratch.take<int>((size_t)count * 6) : nullptr;
  unsigned char *d_stream = ctx->scratch.take<unsigned char>(cap);
  cudaStream_t s = ctx->stream;
  if (cuda_fail(cudaMemcpyAsync(d_data, oriData, n * 8, cudaMemcpyHostToDevice, s), "H2D data")) return nullptr;
  if (count && cuda_fail(cudaMemcpyAsync(d_cps, critical_points, (size_t)count * sizeof(CriticalPoint3D),
                                         cudaMemcpyHostToDevice, s), "H2D critical points"))
    return nullptr;
  const Geom g = make_geom(3, d1, d2, d3);
  unsigned long long len = 0;
  if (f64_compress_impl(ctx, d_data, n, g, absErrBound, blockSize, d_cps, count, 3, d_stream, cap, &len, nullptr))
    return nullptr;
  unsigned char *out = (unsigned char *)malloc(len);
  if (!out) { set_error("szp_cuda_double_compress_topology_3d: host allocation failed"); return nullptr; }
  if (cuda_fail(cudaMemcpyAsync(out, d_stream, len, cudaMemcpyDeviceToHost, s), "D2H stream") ||
      cuda_fail(cudaStreamSynchronize(s), "sync")) {
    free(out);
    return nullptr;
  }
  *outSize = len;
  return out;
}

}  // extern "C"
