// Fused topology encoder for blockSize 64, the block size of the reference's
// benchmark configurations: classification of every point (4 neighbours in
// 2D, 6 in 3D), quantization, deltas, bit packing with the 2-bit type tags,
// the critical-point pairs for the rank stage, and the decoupled look-back
// that places every tile in the stream -- one pass over the field.
//
// Same stream bytes as the general octet encoder (tsz_codec2.cuh) and the
// reference (SZp/src/szp_cuda_topology_3d.cu:832-1059,
// SZp/src/szp_cuda_topology.cu:532-772); it differs in how the work maps onto
// the machine:
//   * thread t of a CTA owns elements 8t .. 8t+7 of a 2048-element tile, so a
//     warp reads 1 KB of the field with two 16-byte loads per lane and eight
//     lanes form one codec block;
//   * the +-1 neighbours come from the adjacent lanes (shuffles), and each
//     edge along the row is compared once for both of its points;
//   * the two other axes are folded into max / min masks one axis at a time,
//     so that only one neighbour octet pair is live;
//   * index arithmetic is per octet (one coordinate split), never per point;
//   * the CTA keeps two tile images and runs one tile behind (its look-back
//     waits while the next tile's front half is already published).
#include "tsz_codec2.cuh"
#include "tsz_enc64.h"
#include "tsz_ops.h"
#include "tsz_runtime.h"

namespace tsz {

constexpr int kE64Threads = 256;
constexpr int kE64Tile = 8 * kE64Threads;        // elements per tile
constexpr int kE64Blocks = kE64Tile / 64;        // codec blocks per tile
constexpr unsigned kE64BlockMax = 289;           // block_bytes(64, 33, tags): a safe bound
constexpr unsigned kE64Img = (kE64Blocks * kE64BlockMax + 64u + 15u) & ~15u;
constexpr unsigned kE64Stage = kE64Tile * 8u;    // staged critical-point pairs (one per element at most)
constexpr unsigned kE64Part = kE64Img + kE64Stage;

struct E64Sh {
  unsigned long long w64[kE64Threads / 32];
  unsigned long long gbyte, gcnt;
  unsigned tile_bytes, tile_cps, tile_ext;
  unsigned boff[kE64Blocks];
};

// hi / lo masks of one axis: bit t set when c[t] is above (below) both of its
// neighbours at -off and +off.  c > max.NaN(m, p) is exactly (c > m && c > p),
// NaN operands included.
__device__ __forceinline__ void e64_axis(const float *__restrict__ d, long long i0, long long off, unsigned inter,
                                         bool vec, const float (&c)[8], unsigned &hi, unsigned &lo) {
  float m[8], p[8];
  if (vec) {
    const float4 *pm = reinterpret_cast<const float4 *>(d + i0 - off);
    const float4 *pp = reinterpret_cast<const float4 *>(d + i0 + off);
    const float4 a0 = __ldg(pm), a1 = __ldg(pm + 1), b0 = __ldg(pp), b1 = __ldg(pp + 1);
    m[0] = a0.x; m[1] = a0.y; m[2] = a0.z; m[3] = a0.w; m[4] = a1.x; m[5] = a1.y; m[6] = a1.z; m[7] = a1.w;
    p[0] = b0.x; p[1] = b0.y; p[2] = b0.z; p[3] = b0.w; p[4] = b1.x; p[5] = b1.y; p[6] = b1.z; p[7] = b1.w;
  } else {
#pragma unroll
    for (int t = 0; t < 8; t++) {
      const bool in = (inter >> t) & 1u;
      m[t] = in ? __ldg(d + i0 + t - off) : 0.f;
      p[t] = in ? __ldg(d + i0 + t + off) : 0.f;
    }
  }
  unsigned h = 0, w = 0;
#pragma unroll
  for (int t = 0; t < 8; t++) {
    h |= (c[t] > fmax_nan(m[t], p[t]) ? 1u : 0u) << t;
    w |= (c[t] < fmin_nan(m[t], p[t]) ? 1u : 0u) << t;
  }
  hi = h;
  lo = w;
}

// Front half of a tile: load, classify, quantize, pack into img, stage the
// critical-point pairs, publish the tile's aggregate.  All threads call it.
template <bool D3>
__device__ __forceinline__ void e64_front(const Enc64Args &a, long long tile, unsigned char *img, uint2 *stage,
                                          E64Sh &sh) {
  const int tid = threadIdx.x, lane = tid & 31;
  const int l = lane & 7, bi = tid >> 3;
  const long long n = (long long)a.n;
  const long long i0 = tile * kE64Tile + 8 * tid;   // local index of the octet
  const long long g0 = (long long)a.base + i0;       // its global index
  const long long bstart = tile * kE64Tile + 64 * bi;
  const int len = bstart >= n ? 0 : (n - bstart >= 64 ? 64 : (int)(n - bstart));
  const int e0 = 8 * l;
  const int nv = len - e0 < 0 ? 0 : (len - e0 > 8 ? 8 : len - e0);

  // ---- values of the octet ----
  float x[8];
  if (nv == 8) {
    const float4 *px = reinterpret_cast<const float4 *>(a.data + g0);
    const float4 u = __ldg(px), v = __ldg(px + 1);
    x[0] = u.x; x[1] = u.y; x[2] = u.z; x[3] = u.w; x[4] = v.x; x[5] = v.y; x[6] = v.z; x[7] = v.w;
  } else {
#pragma unroll
    for (int t = 0; t < 8; t++) x[t] = t < nv ? __ldg(a.data + g0 + t) : 0.f;
  }

  // ---- interior mask: one coordinate split per octet ----
  unsigned inter = 0;
  bool wrap = false;
  if (nv > 0) {
    long long r, z0, y, xx = 0;
    if (D3) {
      xx = fdivmod(g0, a.g.plane, a.g.m_plane, r);
      y = fdivmod(r, a.g.d3, a.g.m_d3, z0);
    } else {
      y = fdivmod(g0, a.g.d3, a.g.m_d3, z0);
    }
    if (z0 + 7 < a.g.d3) {
      const bool row_in = y >= 1 && y <= a.g.d2 - 2 && (!D3 || (xx >= 1 && xx <= a.g.d1 - 2));
      if (row_in) {
        const long long lo = 1 - z0, hi = a.g.d3 - 2 - z0;
        const int ulo = lo > 0 ? (int)lo : 0, uhi = hi < 7 ? (int)hi : 7;
        if (ulo <= uhi) inter = ((2u << uhi) - 1u) & ~((1u << ulo) - 1u);
      }
      inter &= (nv >= 8) ? 0xffu : ((1u << nv) - 1u);
    } else {
      wrap = true;   // the octet crosses a row: elements of several rows
      inter = octet_interior(g0, nv, a.g);
    }
  }

  // ---- classification ----
  // +-1 along the row: the adjacent lanes' values (the warp covers 256
  // consecutive elements); the warp's end lanes load their outer neighbour
  float prev = __shfl_up_sync(0xffffffffu, x[7], 1);
  float next = __shfl_down_sync(0xffffffffu, x[0], 1);
  if (lane == 0 && (inter & 1u)) prev = __ldg(a.data + g0 - 1);
  if (lane == 31 && (inter & 0x80u)) next = __ldg(a.data + g0 + 8);
  unsigned types = 0, cpm = 0, exm = 0;
  if (__any_sync(0xffffffffu, inter != 0u)) {
    // edge j (0..8) joins element j-1 and j (element -1 = prev, 8 = next)
    unsigned gt = 0, lt = 0;
    float cl = prev;
#pragma unroll
    for (int t = 0; t < 8; t++) {
      gt |= (cl > x[t] ? 1u : 0u) << t;
      lt |= (cl < x[t] ? 1u : 0u) << t;
      cl = x[t];
    }
    gt |= (cl > next ? 1u : 0u) << 8;
    lt |= (cl < next ? 1u : 0u) << 8;
    const unsigned hz = lt & (gt >> 1), lz = gt & (lt >> 1);
    unsigned ha = 0, la = 0, hb = 0, lb = 0;
    if (inter) {
      // vector loads when the octet lies in one row and the offset keeps the
      // 16-byte alignment; per-element loads otherwise
      const long long oa = D3 ? a.g.plane : a.g.d3;
      e64_axis(a.data, g0, oa, inter, !wrap && (oa & 3) == 0, x, ha, la);
      if (D3) e64_axis(a.data, g0, a.g.d3, inter, !wrap && (a.g.d3 & 3) == 0, x, hb, lb);
    }
    unsigned mx, mn, sd;
    if (D3) {
      mx = ha & hb & hz;
      mn = la & lb & lz & ~mx;
      sd = (ha | hb | hz) & (la | lb | lz) & ~mx & ~mn;
    } else {
      // rows are the vertical axis, the row direction the horizontal one
      mx = ha & hz;
      mn = la & lz & ~mx;
      sd = ((la & hz) | (ha & lz)) & ~mx & ~mn;
    }
    mx &= inter;
    mn &= inter;
    sd &= inter;
    cpm = mx | mn | sd;
    exm = mx | mn;
    // 2-bit types: maximum 01, minimum 10, saddle 11 (element t at bits 2t)
    types = spread2(mx | sd) | (spread2(mn | sd) << 1);
  }

  // ---- quantization and deltas ----
  int q[8];
#pragma unroll
  for (int t = 0; t < 8; t++) q[t] = t < nv ? quantize(x[t], a.inv) : 0;
  int qn = __shfl_down_sync(0xffffffffu, q[0], 1, 8);
  if (l == 7) qn = 0;
  const int cnt = len > 0 ? len - 1 : 0;
  unsigned negm = 0, maxm = 0, mags[8];
#pragma unroll
  for (int t = 0; t < 8; t++) {
    mags[t] = 0;
    if (e0 + t < cnt) {
      const int nx = (t < 7) ? q[t + 1] : qn;
      const unsigned ud = (unsigned)nx - (unsigned)q[t];
      const bool ng = (int)ud < 0;
      mags[t] = ng ? 0u - ud : ud;
      negm |= (ng ? 1u : 0u) << t;
      maxm = mags[t] > maxm ? mags[t] : maxm;
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    const unsigned u = __shfl_xor_sync(0xffffffffu, maxm, o, 8);
    maxm = u > maxm ? u : maxm;
  }
  const unsigned bc = bitcount(maxm);
  const unsigned bbytes = len ? block_bytes((unsigned)len, bc, true) : 0u;

  // ---- tile scan: block bytes (bits 0..23), CPs (24..43), extrema (44..63) ----
  unsigned boff, cpo, exo;
  {
    const unsigned long long v = (unsigned long long)(l == 0 ? bbytes : 0u) |
                                 ((unsigned long long)__popc(cpm) << 24) |
                                 ((unsigned long long)__popc(exm) << 44);
    unsigned long long tot;
    const unsigned long long ex = cta_excl_scan64<kE64Threads / 32>(v, sh.w64, &tot);
    // lane 0 of the group added this block's bytes before the other lanes
    boff = (unsigned)(ex & 0xffffffull) - (l == 0 ? 0u : bbytes);
    cpo = (unsigned)((ex >> 24) & 0xfffffull);
    exo = (unsigned)(ex >> 44);
    if (tid == 0) {
      sh.tile_bytes = (unsigned)(tot & 0xffffffull);
      sh.tile_cps = (unsigned)((tot >> 24) & 0xfffffull);
      sh.tile_ext = (unsigned)(tot >> 44);
      publish_aggregate(a.desc, tile, tot & 0xffffffull,
                        (((tot >> 24) & 0xfffffull) << 32) | (tot >> 44));
    }
  }
  if (l == 0) sh.boff[bi] = boff;

  // ---- critical-point pairs, staged in raster order ----
  if (cpm) {
    unsigned ci = cpo, ei = exo;
#pragma unroll
    for (int t = 0; t < 8; t++) {
      if ((cpm >> t) & 1u) {
        const bool ext = (exm >> t) & 1u;
        stage[ci++] = make_uint2(float_code(x[t]), ext ? ei : kNoExtremum);
        ei += ext ? 1u : 0u;
      }
    }
  }

  // ---- pack the octet into the tile image ----
  if (nv > 0) {
    unsigned p = boff;
    if (l == 0) {
      const unsigned an = (unsigned)q[0];
      img[p] = (unsigned char)an;
      img[p + 1] = (unsigned char)(an >> 8);
      img[p + 2] = (unsigned char)(an >> 16);
      img[p + 3] = (unsigned char)(an >> 24);
      if (len > 1) img[p + 4] = (unsigned char)bc;
    }
    p += 4;
    if (len > 1) {
      p += 1;
      if (bc) {
        const unsigned sbytes = (unsigned)(cnt + 7) / 8u;
        const bool has_d = e0 < cnt;
        if (has_d) img[p + l] = (unsigned char)(__brev(negm) >> 24);   // delta e0 + t at bit 7 - t
        p += sbytes;
        const unsigned fb = bc >> 3, rem = bc & 7u;
        if (has_d) {
          if (fb == 1) {
#pragma unroll
            for (int t = 0; t < 8; t++)
              if (e0 + t < cnt) img[p + (unsigned)(e0 + t)] = (unsigned char)(mags[t] >> rem);
          } else if (fb >= 2) {
#pragma unroll
            for (int t = 0; t < 8; t++) {
              if (e0 + t < cnt) {
                unsigned v = mags[t] >> rem;
                const unsigned o = p + (unsigned)(e0 + t) * fb;
                for (unsigned u = 0; u < fb; u++) { img[o + u] = (unsigned char)v; v >>= 8; }
              }
            }
          }
        }
        p += fb * (unsigned)cnt;
        if (rem) {
          const unsigned rbytes = (rem * (unsigned)cnt - 1u) / 8u + 1u;
          if (has_d) {
            const unsigned mask = (1u << rem) - 1u;
            unsigned long long acc = 0;
#pragma unroll
            for (int t = 0; t < 8; t++) acc = (acc << rem) | (unsigned long long)(mags[t] & mask);
            // the octet's 8 rem bits are exactly rem bytes at byte l * rem
            const unsigned ob = (unsigned)l * rem;
#pragma unroll
            for (unsigned u = 0; u < 7; u++)
              if (u < rem && ob + u < rbytes) img[p + ob + u] = (unsigned char)(acc >> (8 * (rem - 1u - u)));
          }
          p += rbytes;
        }
      }
    }
    // tag byte j: elements 4j .. 4j+3, element 4j in the top two bits
    const unsigned tb = ((unsigned)len + 3u) / 4u;
    const unsigned t0 = ((types & 3u) << 6) | (((types >> 2) & 3u) << 4) | (((types >> 4) & 3u) << 2) |
                        ((types >> 6) & 3u);
    const unsigned t1 = (((types >> 8) & 3u) << 6) | (((types >> 10) & 3u) << 4) | (((types >> 12) & 3u) << 2) |
                        ((types >> 14) & 3u);
    if (2u * l < tb) img[p + 2 * l] = (unsigned char)t0;
    if (2u * l + 1u < tb) img[p + 2 * l + 1] = (unsigned char)t1;
  }
}

// Back half of a tile: look-back for the tile's stream and CP offsets, block
// index, write-out of the image and copy-out of the staged pairs.  Ends with
// a CTA barrier.
__device__ __forceinline__ void e64_back(const Enc64Args &a, long long tile, const unsigned char *img,
                                         const uint2 *stage, E64Sh &sh) {
  const int tid = threadIdx.x;
  const long long n = (long long)a.n;
  const long long nblocks = (n + 63) / 64;
  const long long ntiles = (n + kE64Tile - 1) / kE64Tile;
  const unsigned tile_bytes = sh.tile_bytes;
  {
    const Prefix pf = lookback_cta<kE64Threads / 32>(a.desc, tile, tile_bytes,
                                                      ((unsigned long long)sh.tile_cps << 32) | sh.tile_ext, a.err,
                                                      a.spin_limit);
    if (tid == 0) {
      sh.gbyte = pf.bytes;
      sh.gcnt = pf.cnt;
      if (tile == ntiles - 1 && a.total) {
        a.total[0] = pf.bytes + tile_bytes;
        a.total[1] = (pf.cnt >> 32) + sh.tile_cps;
        a.total[2] = (pf.cnt & 0xffffffffull) + sh.tile_ext;
      }
    }
  }
  __syncthreads();
  const unsigned long long G0 = sh.gbyte;
  const bool fits = (G0 + tile_bytes) <= a.out_cap;
  if (!fits && tid == 0) atomicExch(a.err, kErrOutputOverflow);
  if (a.blk_off && tid < kE64Blocks) {
    const long long b = tile * kE64Blocks + tid;
    if (b < nblocks) a.blk_off[b] = G0 + sh.boff[tid];
  }
  // write-out: aligned 16-byte stores in the middle
  if (fits && tile_bytes) {
    const uint32_t *imgw = reinterpret_cast<const uint32_t *>(img);
    unsigned char *dst = a.out + G0;
    unsigned head = (unsigned)((16u - (unsigned)(reinterpret_cast<uintptr_t>(dst) & 15u)) & 15u);
    if (head > tile_bytes) head = tile_bytes;
    if ((unsigned)tid < head) dst[tid] = img[tid];
    const unsigned nq = (tile_bytes - head) >> 4;
    const unsigned shb = 8u * (head & 3u);
    const unsigned w0 = head >> 2;
    uint4 *dq = reinterpret_cast<uint4 *>(dst + head);
    for (unsigned qd = tid; qd < nq; qd += kE64Threads) {
      const unsigned wi = w0 + 4u * qd;
      uint4 v;
      if (shb) {
        v.x = __funnelshift_r(imgw[wi], imgw[wi + 1], shb);
        v.y = __funnelshift_r(imgw[wi + 1], imgw[wi + 2], shb);
        v.z = __funnelshift_r(imgw[wi + 2], imgw[wi + 3], shb);
        v.w = __funnelshift_r(imgw[wi + 3], imgw[wi + 4], shb);
      } else {
        v.x = imgw[wi]; v.y = imgw[wi + 1]; v.z = imgw[wi + 2]; v.w = imgw[wi + 3];
      }
      dq[qd] = v;
    }
    const unsigned t0b = head + 16u * nq;
    if (t0b + tid < tile_bytes) dst[t0b + tid] = img[t0b + tid];
  }
  // critical-point pairs in raster order
  {
    const unsigned long long cb = sh.gcnt >> 32;
    const uint32_t eb0 = (uint32_t)(sh.gcnt & 0xffffffffull);
    const unsigned ntc = sh.tile_cps;
    uint2 *cp = a.cp_out;
    for (unsigned k = tid; k < ntc; k += kE64Threads) {
      if (cb + k < a.cp_cap) {
        uint2 pr = stage[k];
        if (pr.y != kNoExtremum) pr.y += eb0;
        cp[cb + k] = pr;
      }
    }
    if (tid == 0 && cb + ntc > a.cp_cap) atomicExch(a.err, kErrCapacity);
  }
  __syncthreads();
}

// Persistent CTAs claim tiles in order; each keeps two images and runs one
// tile behind (tile k's aggregate is published before tile k-1 looks back),
// so a look-back only ever waits for tiles held by running CTAs.
template <bool D3>
__global__ void __launch_bounds__(kE64Threads, 4) enc64_kernel(Enc64Args a) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ E64Sh sh[2];
  __shared__ long long s_claim;
  const long long ntiles = ((long long)a.n + kE64Tile - 1) / kE64Tile;
  const long long tend = a.tile_hi ? (long long)a.tile_hi : ntiles;
  long long prev = -1;
  int cur = 0;
  while (true) {
    if (threadIdx.x == 0) s_claim = (long long)a.tile_lo + (long long)atomicAdd(a.tile_ctr, 1u);
    __syncthreads();
    const long long tile = s_claim;
    const bool more = tile < tend;
    unsigned char *part = smem_dyn + (size_t)cur * kE64Part;
    if (more) e64_front<D3>(a, tile, part, reinterpret_cast<uint2 *>(part + kE64Img), sh[cur]);
    __syncthreads();
    if (prev >= 0) {
      const unsigned char *pp = smem_dyn + (size_t)(cur ^ 1) * kE64Part;
      e64_back(a, prev, pp, reinterpret_cast<const uint2 *>(pp + kE64Img), sh[cur ^ 1]);
    }
    if (!more) break;
    prev = tile;
    cur ^= 1;
  }
}

unsigned long long enc64_tiles(unsigned long long n) { return (n + kE64Tile - 1) / kE64Tile; }

size_t enc64_smem_bytes() { return 2 * (size_t)kE64Part; }

static cudaError_t launch_enc64(const Enc64Args &a, cudaStream_t s, int sm_count) {
  const size_t smem = enc64_smem_bytes();
  auto k = a.g.nd == 3 ? enc64_kernel<true> : enc64_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kE64Threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  const unsigned long long ntiles = enc64_tiles(a.n);
  const unsigned long long hi = a.tile_hi ? a.tile_hi : ntiles;
  const unsigned long long span = hi > a.tile_lo ? hi - a.tile_lo : 0;
  unsigned long long grid = (unsigned long long)sm_count * per_sm;
  if (grid > span) grid = span;
  if (grid < 1) grid = 1;
  k<<<(unsigned)grid, kE64Threads, smem, s>>>(a);
  return cudaGetLastError();
}

// Bounded-wait check of the look-back: a two-tile field encoded from tile 1
// on, so tile 0 never publishes and tile 1's look-back must give up after
// spin_limit polls, report kErrLookbackTimeout and finish its write-out (at
// offset 0 of the output, inside its capacity).
int selftest_lookback(int spin_limit, int *status, float *ms) {
  const unsigned long long n = 2 * kE64Tile;
  const size_t cap = 2 * kE64Img;
  unsigned char *buf = nullptr;
  const size_t bytes = n * 4 + cap + 2 * sizeof(TileDesc) + kE64Tile * sizeof(uint2) + 256;
  if (cuda_fail(cudaMalloc(&buf, bytes), "cudaMalloc")) return -1;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = -1;
  if (!cuda_fail(cudaMemset(buf, 0, bytes), "memset") && !cuda_fail(cudaEventCreate(&e0), "event") &&
      !cuda_fail(cudaEventCreate(&e1), "event")) {
    Enc64Args a{};
    a.data = reinterpret_cast<const float *>(buf);
    a.n = n;
    a.inv = 1.0e3;
    a.g = make_geom(2, 64, (long long)n / 64, 1);
    a.out = buf + n * 4;
    a.out_cap = cap;
    a.desc = reinterpret_cast<TileDesc *>(buf + n * 4 + cap);
    a.cp_out = reinterpret_cast<uint2 *>(buf + n * 4 + cap + 2 * sizeof(TileDesc));
    a.cp_cap = kE64Tile;
    unsigned long long *w = reinterpret_cast<unsigned long long *>(buf + bytes - 64);
    a.tile_ctr = reinterpret_cast<unsigned *>(w);
    a.err = reinterpret_cast<int *>(w + 1);
    a.total = w + 2;
    a.tile_lo = 1;
    a.tile_hi = 2;
    a.spin_limit = spin_limit;
    cudaEventRecord(e0, 0);
    const cudaError_t le = launch_enc64(a, 0, 1);
    cudaEventRecord(e1, 0);
    int h = 0;
    if (!cuda_fail(le, "probe launch") && !cuda_fail(cudaMemcpy(&h, a.err, 4, cudaMemcpyDeviceToHost), "D2H")) {
      cudaEventElapsedTime(ms, e0, e1);
      *status = h;
      rc = 0;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(buf);
  return rc;
}

bool enc64_applies(const EncArgs &a, int mode) {
  return mode == kEncClassify && a.B == 64 && a.cp_mode == kCpPairs && a.out != nullptr &&
         (reinterpret_cast<uintptr_t>(a.data) & 15) == 0 && enc_tile_blocks(64) == kE64Blocks;
}

cudaError_t launch_enc64_args(const Enc64Args &a, cudaStream_t s, int sm_count) { return launch_enc64(a, s, sm_count); }

cudaError_t launch_enc64_from(const EncArgs &e, cudaStream_t s, int sm_count) {
  Enc64Args a{};
  a.data = e.data;
  a.n = e.n;
  a.inv = e.inv;
  a.g = e.g;
  a.out = e.out;
  a.out_cap = e.out_cap;
  a.blk_off = e.blk_off;
  a.desc = e.desc;
  a.tile_ctr = e.tile_ctr;
  a.tile_lo = e.tile_lo;
  a.tile_hi = e.tile_hi;
  a.err = e.err;
  a.total = e.total;
  a.cp_out = reinterpret_cast<uint2 *>(e.cp_out);
  a.cp_cap = e.cp_cap;
  a.spin_limit = 0;
  return launch_enc64(a, s, sm_count);
}

}  // namespace tsz

using namespace tsz;

extern "C" SZP_B200_API int szp_b200_selftest_bounded_wait(int which, int spin_limit, int *status, float *ms) {
  clear_error();
  if (!status || !ms) { set_error("szp_b200_selftest_bounded_wait: null argument"); return -1; }
  if (spin_limit < 1 || spin_limit > (1 << 20)) {
    set_error("szp_b200_selftest_bounded_wait: spin_limit must lie in [1, 2^20]");
    return -1;
  }
  *status = 0;
  *ms = 0.f;
  if (which == 0) return selftest_lookback(spin_limit, status, ms);
  if (which == 1) return selftest_grid_barrier(spin_limit, status, ms);
  set_error("szp_b200_selftest_bounded_wait: which must be 0 (look-back) or 1 (grid barrier)");
  return -1;
}
