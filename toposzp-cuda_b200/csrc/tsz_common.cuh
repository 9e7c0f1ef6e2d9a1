// Shared definitions for the TopoSZp B200 library.
//
// Compressed block layout (identical to the reference CUDA path,
// SZp/src/szp_cuda_topology.cu:577-680 and SZp/src/szp_cuda_decompress.cu:673-741):
//   int32 anchor (little-endian)
//   if n > 1: u8 bit count bc; if bc > 0: ceil((n-1)/8) sign bytes (MSB first),
//             then (bc/8)*(n-1) full magnitude bytes (little-endian per value),
//             then ceil((bc%8)*(n-1)/8) bytes of the low bc%8 bits, MSB first
//   [topology stream only] ceil(2n/8) bytes of 2-bit type tags, MSB first
#pragma once

#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

namespace tsz {

constexpr int kMaxBlockSize = 257;   // reference limit (SZP_CUDA_TOPO_MAX_BLOCK + 1)
constexpr int kWarps = 8;            // warps per CTA in the codec kernels
constexpr int kThreads = kWarps * 32;
constexpr uint32_t kNoExtremum = 0xFFFFFFFFu;

// error codes written by kernels into a device status word
enum : int {
  kOk = 0,
  kErrLookbackTimeout = 1,
  kErrOutputOverflow = 2,
  kErrMalformed = 3,
  kErrCapacity = 4,
  kErrWaitTimeout = 5,
};

__host__ __device__ __forceinline__ uint32_t mag_bytes(uint32_t cnt, uint32_t bc) {
  uint32_t fb = bc >> 3, rem = bc & 7u;
  uint32_t len = fb * cnt;
  if (rem) len += (rem * cnt - 1u) / 8u + 1u;
  return len;
}

// bytes of one block of n elements with bit count bc (CUDA layout)
__host__ __device__ __forceinline__ uint32_t block_bytes(uint32_t n, uint32_t bc, bool tags) {
  uint32_t s = 4;
  if (n > 1) {
    s += 1;
    if (bc) s += (n - 2u) / 8u + 1u + mag_bytes(n - 1u, bc);
  }
  if (tags) s += (2u * n + 7u) / 8u;
  return s;
}

__host__ __device__ __forceinline__ uint32_t max_block_bytes(uint32_t B, bool tags) {
  return block_bytes(B, 33, tags);
}

// Geometry of a field: 2D fields use (rows, cols) = (d2, d3) with nd = 2.
struct Geom {
  int nd;
  long long d1, d2, d3;     // 3D: x, y, z extents; 2D: d1 = 1, d2 = rows, d3 = cols
  long long plane;          // d2 * d3
  unsigned long long m_d3, m_plane;  // ceil(2^64 / d) for the coordinate split (0 when d == 1)
};

// ceil(2^64 / d) for d >= 2 (0 marks d == 1)
inline unsigned long long magic_u64(unsigned long long d) {
  if (d <= 1) return 0ull;
  return (unsigned long long)((((unsigned __int128)1 << 64) + d - 1) / d);
}

// (q, r) = divmod(i, d) with q = hi64(i * ceil(2^64 / d)): exact whenever
// i * d < 2^64, which holds for every flat index of a field that fits in memory
__device__ __forceinline__ long long fdivmod(long long i, long long d, unsigned long long m, long long &r) {
  const long long q = m ? (long long)__umul64hi((unsigned long long)i, m) : i;
  r = i - q * d;
  return q;
}

// order-preserving 32-bit code of a float (-0 folded onto +0)
__host__ __device__ __forceinline__ uint32_t float_code(float v) {
  uint32_t b;
#ifdef __CUDA_ARCH__
  b = __float_as_uint(v);
#else
  __builtin_memcpy(&b, &v, 4);
#endif
  if (b == 0x80000000u) b = 0;
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__host__ __device__ __forceinline__ float code_float(uint32_t c) {
  uint32_t b = (c & 0x80000000u) ? (c & 0x7FFFFFFFu) : ~c;
  float v;
#ifdef __CUDA_ARCH__
  v = __uint_as_float(b);
#else
  __builtin_memcpy(&v, &b, 4);
#endif
  return v;
}

// (int)((double)x * inv): the C conversion of the reference's kernels
// (truncation toward zero; on sm_100a values beyond the int range saturate and
// NaN converts to INT_MIN)
__device__ __forceinline__ int quantize(float x, double inv) {
  return (int)__dmul_rn((double)x, inv);
}

// quantization bin of a critical point: float add first, then the double multiply
// (SZp/src/szp_cuda_topology.cu:67)
__device__ __forceinline__ int quant_bin(float c, float eb, double inv) {
  return (int)__dmul_rn((double)__fadd_rn(c, eb), inv);
}

// bit count of a block: floor(log2f((float)max)) + 1 (SZp/src/szp_cuda_topology.cu:558)
__device__ __forceinline__ uint32_t bitcount(uint32_t m) {
  return m ? (uint32_t)floorf(log2f((float)m)) + 1u : 0u;
}

// 4-neighbour classification (SZp/src/szp_cuda_topology.cu:57-64)
__device__ __forceinline__ int classify4(float c, float up, float dn, float lf, float rt) {
  if (c > up && c > dn && c > lf && c > rt) return 1;
  if (c < up && c < dn && c < lf && c < rt) return 2;
  if ((c < up && c < dn && c > lf && c > rt) || (c > up && c > dn && c < lf && c < rt)) return 3;
  return 0;
}

// 6-neighbour classification (SZp/src/szp_cuda_topology_3d.cu:134-160)
__device__ __forceinline__ int classify6(float c, float xm, float xp, float ym, float yp,
                                         float zm, float zp) {
  if (c > xm && c > xp && c > ym && c > yp && c > zm && c > zp) return 1;
  if (c < xm && c < xp && c < ym && c < yp && c < zm && c < zp) return 2;
  int hi = (c > xm && c > xp) + (c > ym && c > yp) + (c > zm && c > zp);
  int lo = (c < xm && c < xp) + (c < ym && c < yp) + (c < zm && c < zp);
  return (hi >= 1 && lo >= 1) ? 3 : 0;
}

// classify element i of a field (0 on the boundary)
__device__ __forceinline__ int classify_at(const float *__restrict__ d, long long i, const Geom &g) {
  long long r;
  if (g.nd == 2) {
    long long row = fdivmod(i, g.d3, g.m_d3, r);
    if (row < 1 || row > g.d2 - 2 || r < 1 || r > g.d3 - 2) return 0;
    return classify4(__ldg(d + i), __ldg(d + i - g.d3), __ldg(d + i + g.d3), __ldg(d + i - 1),
                     __ldg(d + i + 1));
  }
  long long x = fdivmod(i, g.plane, g.m_plane, r);
  long long z;
  long long y = fdivmod(r, g.d3, g.m_d3, z);
  if (x < 1 || x > g.d1 - 2 || y < 1 || y > g.d2 - 2 || z < 1 || z > g.d3 - 2) return 0;
  return classify6(__ldg(d + i), __ldg(d + i - g.plane), __ldg(d + i + g.plane), __ldg(d + i - g.d3),
                   __ldg(d + i + g.d3), __ldg(d + i - 1), __ldg(d + i + 1));
}

// Decoupled look-back tile descriptor: a status/bytes word plus two count
// words (aggregate and inclusive), each count word written before its status.
struct TileDesc {
  unsigned long long status;   // bits 63..62: 0 none, 1 aggregate, 2 inclusive; 61..0 bytes
  unsigned long long agg_cnt;  // (cps << 32) | extrema, this tile only
  unsigned long long inc_cnt;  // inclusive counts up to and including this tile
  unsigned long long pad;
};

constexpr unsigned long long kStatShift = 62;
constexpr unsigned long long kByteMask = (1ull << 62) - 1ull;

}  // namespace tsz
