// Octet codec kernels (blockSize <= 256).
//
// Each lane owns 8 consecutive elements of a codec block ("octet" l covers
// elements 8l..8l+7 and deltas 8l..8l+7); a group of G = next_pow2(ceil(B/8))
// lanes serves one block, a warp serves 32/G blocks.  With this mapping every
// section of the block layout is byte-aligned per lane: the 8 sign bits of an
// octet are one byte, its 8 remainder fields are exactly `rem` bytes, its 8
// tags are two bytes and its full magnitude bytes are contiguous.  Packing and
// unpacking therefore need no cross-lane bit merging; the decoder's prefix
// sum is an in-lane serial sum plus a log2(G) group scan.
#pragma once
#include "tsz_codec.h"
#include "tsz_lookback.cuh"

namespace tsz {

// Dynamic shared memory of an encoder CTA: the tile image (tb blocks at their
// largest size) followed, in classification mode, by the staging area of the
// tile's critical-point pairs (one uint2 per point of the tile).
__host__ __device__ __forceinline__ unsigned enc2_img_bytes(int B, bool tags, int tb) {
  return ((unsigned)tb * max_block_bytes((uint32_t)B, tags) + 64u + 15u) & ~15u;
}
__host__ __device__ __forceinline__ unsigned enc2_total_smem(int B, bool tags, bool classify, int warps, int tb) {
  return enc2_img_bytes(B, tags, tb) + (classify ? (unsigned)warps * 256u * 8u : 0u);
}

// loads 8 floats at p[i..i+7]: one 32-byte vector load when aligned and fully
// in range, otherwise scalar loads for the elements selected by need
__device__ __forceinline__ void load_oct(const float *__restrict__ p, long long i, long long n,
                                         unsigned need, float (&v)[8]) {
  if (need == 0) return;
  if (i >= 0 && i + 8 <= n && ((reinterpret_cast<uintptr_t>(p + i) & 15) == 0)) {
    const float4 a = __ldg(reinterpret_cast<const float4 *>(p + i));
    const float4 b = __ldg(reinterpret_cast<const float4 *>(p + i) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  } else {
#pragma unroll
    for (int t = 0; t < 8; t++)
      if (need & (1u << t)) v[t] = __ldg(p + i + t);
  }
}

// NaN-propagating max / min (PTX max.NaN / min.NaN): NaN when either is NaN
__device__ __forceinline__ float fmax_nan(float x, float y) {
  float r;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ float fmin_nan(float x, float y) {
  float r;
  asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(x), "f"(y));
  return r;
}

// bit t of an 8-bit mask -> bit 2t
__device__ __forceinline__ unsigned spread2(unsigned x) {
  x = (x | (x << 4)) & 0x0F0Fu;
  x = (x | (x << 2)) & 0x3333u;
  x = (x | (x << 1)) & 0x5555u;
  return x;
}
// bit 2t -> bit t (the inverse of spread2 on the even bits)
__device__ __forceinline__ unsigned compact2(unsigned x) {
  x &= 0x5555u;
  x = (x | (x >> 1)) & 0x3333u;
  x = (x | (x >> 2)) & 0x0F0Fu;
  x = (x | (x >> 4)) & 0x00FFu;
  return x;
}

// 2-bit types of an octet (element t in bits 2t..2t+1); c[] holds the values
// of the octet, nv of them valid, i0 the flat index of element 0
// interior mask of an octet (bit t: element i0 + t is interior), nv valid
__device__ __forceinline__ unsigned octet_interior(long long i0, int nv, const Geom &g) {
  // coordinates of element 0, then incremented with wrap-around
  long long r, x, y, z;
  if (g.nd == 2) { x = 0; y = fdivmod(i0, g.d3, g.m_d3, r); z = r; }
  else { x = fdivmod(i0, g.plane, g.m_plane, r); y = fdivmod(r, g.d3, g.m_d3, z); }
  unsigned inter = 0;
  if (z + 7 < g.d3) {
    // the octet lies in one row: interior columns 1 .. d3-2
    const bool row_in = y >= 1 && y <= g.d2 - 2 && (g.nd == 2 || (x >= 1 && x <= g.d1 - 2));
    if (row_in) {
      const long long lo = 1 - z, hi = g.d3 - 2 - z;
      const int ulo = lo > 0 ? (int)lo : 0, uhi = hi < 7 ? (int)hi : 7;
      if (ulo <= uhi) inter = ((2u << uhi) - 1u) & ~((1u << ulo) - 1u);
    }
    inter &= (nv >= 8) ? 0xffu : ((1u << nv) - 1u);
  } else {
#pragma unroll
    for (int t = 0; t < 8; t++) {
      const bool in = t < nv;
      bool ok = in && y >= 1 && y <= g.d2 - 2 && z >= 1 && z <= g.d3 - 2;
      if (g.nd == 3) ok = ok && x >= 1 && x <= g.d1 - 2;
      if (ok) inter |= 1u << t;
      z++;
      while (z >= g.d3) { z -= g.d3; y++; if (y >= g.d2) { y -= g.d2; x++; } }
    }
  }
  return inter;
}

// first classification axis of an octet: planes (3D) or rows (2D)
__device__ __forceinline__ long long octet_axis_a(const Geom &g) { return (g.nd == 2) ? g.d3 : g.plane; }

// 2-bit types of an octet (element t in bits 2t..2t+1): c[] holds its values,
// nv of them valid, i0 the flat index of element 0, inter its interior mask;
// ma / pa hold the neighbours at -/+ octet_axis_a (loaded by the caller for
// the interior elements, ahead of the octet's own values: the longest wait)
__device__ __forceinline__ unsigned classify_octet(const float *__restrict__ d, long long n, long long i0,
                                                   int nv, const float (&c)[8], const Geom &g, unsigned inter,
                                                   const float (&ma)[8], const float (&pa)[8],
                                                   const float (&mb)[8], const float (&pb)[8]) {
  if (inter == 0) return 0u;
  // +-1 neighbours: inside the octet, plus one scalar load at each end
  const float prev = (inter & 1u) ? __ldg(d + i0 - 1) : 0.f;
  float next = 0.f;
#pragma unroll
  for (int t = 0; t < 8; t++)
    if (t == nv - 1 && (inter & (1u << t))) next = __ldg(d + i0 + nv);
  // Per axis, hi: c above both neighbours, lo: c below both.  c > max(m, p)
  // with a NaN-propagating max is exactly (c > m && c > p), NaNs included
  // (any NaN makes both false), and likewise for lo with min.
  unsigned hi_a = 0, lo_a = 0, hi_b = 0, lo_b = 0, hi_c = 0, lo_c = 0;
#pragma unroll
  for (int t = 0; t < 8; t++) {
    if (!(inter & (1u << t))) continue;
    if (c[t] > fmax_nan(ma[t], pa[t])) hi_a |= 1u << t;
    if (c[t] < fmin_nan(ma[t], pa[t])) lo_a |= 1u << t;
  }
  if (g.nd == 3) {
#pragma unroll
    for (int t = 0; t < 8; t++) {
      if (!(inter & (1u << t))) continue;
      if (c[t] > fmax_nan(mb[t], pb[t])) hi_b |= 1u << t;
      if (c[t] < fmin_nan(mb[t], pb[t])) lo_b |= 1u << t;
    }
  }
#pragma unroll
  for (int t = 0; t < 8; t++) {
    if (!(inter & (1u << t))) continue;
    const float lf = (t == 0) ? prev : c[t - 1 < 0 ? 0 : t - 1];
    const float rt = (t == nv - 1) ? next : c[t + 1 > 7 ? 7 : t + 1];
    if (c[t] > fmax_nan(lf, rt)) hi_c |= 1u << t;
    if (c[t] < fmin_nan(lf, rt)) lo_c |= 1u << t;
  }
  unsigned mx, mn, sd;
  if (g.nd == 2) {
    // vertical axis (rows) is a, horizontal (columns) is c
    mx = hi_a & hi_c;
    mn = lo_a & lo_c & ~mx;
    sd = ((lo_a & hi_c) | (hi_a & lo_c)) & ~mx & ~mn;
  } else {
    mx = hi_a & hi_b & hi_c;
    mn = lo_a & lo_b & lo_c & ~mx;
    sd = (hi_a | hi_b | hi_c) & (lo_a | lo_b | lo_c) & ~mx & ~mn;
  }
  // 2-bit types from the disjoint masks: maximum 01, minimum 10, saddle 11
  return spread2(mx | sd) | (spread2(mn | sd) << 1);
}

// CTA-wide exclusive scan of one 64-bit value per thread (packed fields that
// never carry into each other); returns the exclusive prefix, total in *total
template <int WARPS>
__device__ __forceinline__ unsigned long long cta_excl_scan64(unsigned long long v, unsigned long long *s_warp,
                                                              unsigned long long *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  unsigned long long wpre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < WARPS; w++) {
    const unsigned long long sw = s_warp[w];
    if (w < warp) wpre += sw;
    tot += sw;
  }
  *total = tot;
  return wpre + inc - v;
}

// Shared state of one encoder CTA (WARPS warps, codec blocks of at most 8G
// elements, 32/G blocks per warp).
template <int G, int WARPS>
struct EncShared {
  static constexpr int TB = WARPS * (32 / G);
  uint32_t bytes[TB];
  unsigned long long w64[WARPS];
  long long tile;
  int field;
  unsigned long long gbyte, gcnt;
  unsigned tile_bytes, tile_cps, tile_ext;
};

// 2-bit tags of nv (1..8) consecutive elements from a byte-per-element
// type array, element t in bits 2t..2t+1.
__device__ __forceinline__ unsigned load_type_octet(const unsigned char *__restrict__ ty, long long i0, int nv) {
  unsigned types = 0;
  if (nv == 8 && ((reinterpret_cast<uintptr_t>(ty + i0) & 7) == 0)) {
    const unsigned long long w = __ldg(reinterpret_cast<const unsigned long long *>(ty + i0));
#pragma unroll
    for (int t = 0; t < 8; t++) types |= (unsigned)((w >> (8 * t)) & 3u) << (2 * t);
  } else {
#pragma unroll
    for (int t = 0; t < 8; t++)
      if (t < nv) types |= (unsigned)(ty[i0 + t] & 3u) << (2 * t);
  }
  return types;
}

// Per-thread values of a tile that the record mode of phase 6 reads after
// the look-back (only the unpipelined path keeps them).
struct EncRegs {
  unsigned types, cpm, cpo, exo;
  long long i0;
};

// Front half of a tile (phases 1-3): quantize, classify, pack the tile image
// into img, stage the critical-point pairs behind it and publish the tile's
// aggregate.  All threads of the CTA call it.  The look-back and write-out
// (encode2_back) may follow at once or after the next tile's front half, on
// a different image and EncShared.
template <int MODE, int G, int WARPS>
__device__ __forceinline__ void encode2_front(const EncArgs &a, const long long tile, unsigned char *img,
                                              EncShared<G, WARPS> &sh, EncRegs &rg) {
  constexpr int BPW = 32 / G;
  constexpr int TB = WARPS * BPW;
  uint32_t *s_bytes = sh.bytes;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int gi = lane / G, l = lane % G;
  const bool tags = mode_tags(MODE);
  const long long n = (long long)a.n;
  const int B = a.B;
  const long long nblocks = (n + B - 1) / B;
  {
    const int bi = warp * BPW + gi;
    const long long blk = tile * TB + bi;
    const long long base = blk * B;
    const int len = (blk < nblocks) ? (int)((n - base) < B ? (n - base) : B) : 0;
    const int e0 = 8 * l;
    const int nv = len - e0 < 0 ? 0 : (len - e0 > 8 ? 8 : len - e0);
    const long long i0 = base + e0;

    // ---- phase 1: load, quantize, classify ----
    float x[8];
    int q[8];
    unsigned types = 0;
#pragma unroll
    for (int t = 0; t < 8; t++) { x[t] = 0.f; q[t] = 0; }
    if (MODE == kEncInts || MODE == kEncIntTypes) {
      if (nv == 8 && ((reinterpret_cast<uintptr_t>(a.ints + i0) & 15) == 0)) {
        const int4 u = __ldg(reinterpret_cast<const int4 *>(a.ints + i0));
        const int4 w = __ldg(reinterpret_cast<const int4 *>(a.ints + i0) + 1);
        q[0] = u.x; q[1] = u.y; q[2] = u.z; q[3] = u.w; q[4] = w.x; q[5] = w.y; q[6] = w.z; q[7] = w.w;
      } else {
#pragma unroll
        for (int t = 0; t < 8; t++) if (t < nv) q[t] = __ldg(a.ints + i0 + t);
      }
      if (MODE == kEncIntTypes && nv > 0) types = load_type_octet(a.types, i0, nv);
    } else {
      unsigned inter = 0;
      float ma[8], pa[8], mb[8], pb[8];
      if (MODE == kEncClassify && nv > 0) {
        inter = octet_interior(i0, nv, a.g);
        const long long oa = octet_axis_a(a.g);
        load_oct(a.data, i0 - oa, n, inter, ma);
        load_oct(a.data, i0 + oa, n, inter, pa);
        if (a.g.nd == 3) {
          load_oct(a.data, i0 - a.g.d3, n, inter, mb);
          load_oct(a.data, i0 + a.g.d3, n, inter, pb);
        }
      }
      load_oct(a.data, i0, n, nv >= 8 ? 0xffu : ((1u << nv) - 1u), x);
#pragma unroll
      for (int t = 0; t < 8; t++) if (t < nv) q[t] = quantize(x[t], a.inv);
      if (MODE == kEncClassify) {
        if (nv > 0) types = classify_octet(a.data, n, i0, nv, x, a.g, inter, ma, pa, mb, pb);
      } else if (MODE == kEncTypes && nv > 0) {
        types = load_type_octet(a.types, i0, nv);
      }
    }
    // deltas d = e0 + t use q[t + 1] - q[t]; q[8] is the next lane's q[0]
    int qn = __shfl_down_sync(0xffffffffu, q[0], 1, G);
    if (l == G - 1) qn = 0;  // blocks of at most 8G elements: no element 8G
    const int cnt = len > 0 ? len - 1 : 0;
    unsigned negm = 0, maxm = 0;
#pragma unroll
    for (int t = 0; t < 8; t++) {
      if (e0 + t < cnt) {
        const int nx = (t < 7) ? q[t + 1] : qn;
        const unsigned ud = (unsigned)nx - (unsigned)q[t];
        const bool ng = (int)ud < 0;
        const unsigned m = ng ? 0u - ud : ud;
        if (ng) negm |= 1u << t;
        maxm = m > maxm ? m : maxm;
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      const unsigned u = __shfl_xor_sync(0xffffffffu, maxm, o);
      maxm = u > maxm ? u : maxm;
    }
    const unsigned bc = bitcount(maxm);
    if (l == 0) s_bytes[bi] = len ? block_bytes((unsigned)len, bc, tags) : 0u;
    unsigned cpm = 0, exm = 0;
    if (MODE == kEncClassify) {
      // type 01 / 10: extremum, 11: saddle
      const unsigned lo2 = types & 0x5555u, hi2 = (types >> 1) & 0x5555u;
      cpm = compact2(lo2 | hi2);
      exm = compact2(lo2 ^ hi2);
    }
    __syncthreads();

    // ---- phase 2: tile scans (block bytes; per-thread CP / extremum counts) ----
    // one scan of the three counts packed into 64 bits: block bytes in bits
    // 0..23 (a tile holds at most TB blocks of max_block_bytes, far below
    // 2^24), CPs in 24..43 and extrema in 44..63 (at most 8 per thread)
    unsigned tbytes, tcps, text;
    unsigned boff, cpo, exo;
    {
      const unsigned bv = (threadIdx.x < TB) ? s_bytes[threadIdx.x] : 0u;
      const unsigned long long v = (unsigned long long)bv | ((unsigned long long)__popc(cpm) << 24) |
                                   ((unsigned long long)__popc(exm) << 44);
      unsigned long long tot;
      const unsigned long long ex = cta_excl_scan64<WARPS>(v, sh.w64, &tot);
      boff = (unsigned)(ex & 0xffffffull);
      cpo = (unsigned)((ex >> 24) & 0xfffffull);
      exo = (unsigned)(ex >> 44);
      tbytes = (unsigned)(tot & 0xffffffull);
      tcps = (unsigned)((tot >> 24) & 0xfffffull);
      text = (unsigned)(tot >> 44);
    }
    // each thread overwrites only the entry it read before the scan
    if (threadIdx.x < TB) s_bytes[threadIdx.x] = boff;
    if (threadIdx.x == 0) {
      sh.tile_bytes = tbytes;
      sh.tile_cps = tcps;
      sh.tile_ext = text;
      publish_aggregate(a.desc, tile, tbytes, ((unsigned long long)tcps << 32) | text);
    }
    __syncthreads();
    // critical-point pairs of the tile, staged in thread (= raster) order;
    // extremum indices tile-local until the look-back gives the base
    uint2 *cp_stage = reinterpret_cast<uint2 *>(img + enc2_img_bytes(B, tags, TB));
    if (MODE == kEncClassify && a.cp_mode == kCpPairs && cpm) {
      unsigned ci = cpo, ei = exo;
#pragma unroll
      for (int t = 0; t < 8; t++) {
        if (!(cpm & (1u << t))) continue;
        const unsigned ty = (types >> (2 * t)) & 3u;
        const bool ext = (ty == 1u || ty == 2u);
        cp_stage[ci++] = make_uint2(float_code(__ldg(a.data + i0 + t)), ext ? ei++ : kNoExtremum);
      }
    }

    // ---- phase 3: pack the octet into the tile image ----
    if (a.out != nullptr && nv > 0) {
      unsigned p = s_bytes[bi];
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
          unsigned mags[8];
#pragma unroll
          for (int t = 0; t < 8; t++) {
            mags[t] = 0;
            if (e0 + t < cnt) {
              const int nx = (t < 7) ? q[t + 1] : qn;
              const unsigned ud = (unsigned)nx - (unsigned)q[t];
              mags[t] = ((int)ud < 0) ? 0u - ud : ud;
            }
          }
          const unsigned sbytes = (unsigned)(cnt + 7) / 8u;
          const bool has_d = e0 < cnt;
          if (has_d) {
            // sign byte: delta e0 + t at bit 7 - t
            img[p + l] = (unsigned char)(__brev(negm) >> 24);
          }
          p += sbytes;
          const unsigned fb = bc >> 3, rem = bc & 7u;
          // Predicated fixed-count stores rather than loops over fb / rem:
          // the blocks of a warp have their own bit counts, and loops with
          // per-block trip counts would run one after the other.
          if (has_d) {
            // full magnitude bytes: one byte per delta when fb == 1
#pragma unroll
            for (int t = 0; t < 8; t++)
              if (fb == 1 && e0 + t < cnt) img[p + (unsigned)(e0 + t)] = (unsigned char)(mags[t] >> rem);
            if (fb >= 2) {
#pragma unroll
              for (int t = 0; t < 8; t++) {
                if (e0 + t < cnt) {
                  unsigned v = mags[t] >> rem;
                  const unsigned o = (unsigned)(e0 + t) * fb;
                  for (unsigned u = 0; u < fb; u++) { img[p + o + u] = (unsigned char)v; v >>= 8; }
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
              // the octet's 8*rem bits are exactly rem bytes at byte l*rem
              const unsigned ob = (unsigned)l * rem;
#pragma unroll
              for (unsigned u = 0; u < 7; u++)
                if (u < rem && ob + u < rbytes) img[p + ob + u] = (unsigned char)(acc >> (8 * (rem - 1u - u)));
            }
            p += rbytes;
          }
        }
      }
      if (tags) {
        const unsigned tb = ((unsigned)len + 3u) / 4u;
        // tag byte for elements 4j..4j+3: element 4j in the top two bits
        const unsigned t0 = ((types & 3u) << 6) | (((types >> 2) & 3u) << 4) | (((types >> 4) & 3u) << 2) |
                            ((types >> 6) & 3u);
        const unsigned t1 = (((types >> 8) & 3u) << 6) | (((types >> 10) & 3u) << 4) |
                            (((types >> 12) & 3u) << 2) | ((types >> 14) & 3u);
        if (2u * l < tb) img[p + 2 * l] = (unsigned char)t0;
        if (2u * l + 1u < tb) img[p + 2 * l + 1] = (unsigned char)t1;
      }
    }

    rg.types = types;
    rg.cpm = cpm;
    rg.cpo = cpo;
    rg.exo = exo;
    rg.i0 = i0;
  }
}

// Back half of a tile (phases 4-6): decoupled look-back for the tile's stream
// and CP offsets, block index, write-out of the image staged by
// encode2_front, copy-out of the staged pairs.  rg: the front half's
// per-thread values, required for the record CP mode (nullptr otherwise).
// All threads of the CTA call it; it ends with a CTA barrier.
template <int MODE, int G, int WARPS>
__device__ __forceinline__ void encode2_back(const EncArgs &a, const long long tile, unsigned char *img,
                                             EncShared<G, WARPS> &sh, const EncRegs *rg) {
  constexpr int BPW = 32 / G;
  constexpr int TB = WARPS * BPW;
  uint32_t *s_bytes = sh.bytes;
  const bool tags = mode_tags(MODE);
  uint32_t *imgw = reinterpret_cast<uint32_t *>(img);
  const long long n = (long long)a.n;
  const int B = a.B;
  const long long nblocks = (n + B - 1) / B;
  const long long ntiles = (nblocks + TB - 1) / TB;
  const unsigned tile_bytes = sh.tile_bytes;
  const uint2 *cp_stage = reinterpret_cast<const uint2 *>(img + enc2_img_bytes(B, tags, TB));
  {
    // ---- phase 4: look-back (whole CTA) ----
    {
      const Prefix pf = lookback_cta<WARPS>(a.desc, tile, tile_bytes,
                                            ((unsigned long long)sh.tile_cps << 32) | sh.tile_ext, a.err);
      if (threadIdx.x == 0) {
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
    const bool fits = a.out != nullptr && (G0 + tile_bytes) <= a.out_cap;
    if (a.out != nullptr && !fits && threadIdx.x == 0) atomicExch(a.err, kErrOutputOverflow);
    if (a.blk_off && threadIdx.x < TB) {
      const long long b2 = tile * TB + threadIdx.x;
      if (b2 < nblocks) a.blk_off[b2] = G0 + s_bytes[threadIdx.x];
    }

    // ---- phase 5: write the tile image (aligned 16-byte stores in the middle) ----
    if (fits && tile_bytes) {
      unsigned char *dst = a.out + G0;
      unsigned head = (unsigned)((16u - (unsigned)(reinterpret_cast<uintptr_t>(dst) & 15u)) & 15u);
      if (head > tile_bytes) head = tile_bytes;
      if (threadIdx.x < head) dst[threadIdx.x] = img[threadIdx.x];
      const unsigned nq = (tile_bytes - head) >> 4;
      const unsigned sh = 8u * (head & 3u);
      const unsigned w0 = head >> 2;
      uint4 *dq = reinterpret_cast<uint4 *>(dst + head);
      for (unsigned qd = threadIdx.x; qd < nq; qd += WARPS * 32) {
        const unsigned wi = w0 + 4u * qd;
        uint4 v;
        if (sh) {
          v.x = __funnelshift_r(imgw[wi], imgw[wi + 1], sh);
          v.y = __funnelshift_r(imgw[wi + 1], imgw[wi + 2], sh);
          v.z = __funnelshift_r(imgw[wi + 2], imgw[wi + 3], sh);
          v.w = __funnelshift_r(imgw[wi + 3], imgw[wi + 4], sh);
        } else {
          v.x = imgw[wi]; v.y = imgw[wi + 1]; v.z = imgw[wi + 2]; v.w = imgw[wi + 3];
        }
        dq[qd] = v;
      }
      const unsigned t0b = head + 16u * nq;
      if (t0b + threadIdx.x < tile_bytes) dst[t0b + threadIdx.x] = img[t0b + threadIdx.x];
    }

    // ---- phase 6: critical points in raster order (thread order == raster order) ----
    if (MODE == kEncClassify && a.cp_mode == kCpPairs) {
      const unsigned long long cb = sh.gcnt >> 32;
      const uint32_t eb0 = (uint32_t)(sh.gcnt & 0xffffffffull);
      const unsigned ntc = sh.tile_cps;
      for (unsigned k = threadIdx.x; k < ntc; k += WARPS * 32) {
        if (cb + k < a.cp_cap) {
          uint2 pr = cp_stage[k];
          if (pr.y != kNoExtremum) pr.y += eb0;
          reinterpret_cast<uint2 *>(a.cp_out)[cb + k] = pr;
        }
      }
    } else if (MODE == kEncClassify && a.cp_mode == kCpRecords && rg && rg->cpm) {
      const unsigned types = rg->types, cpm = rg->cpm;
      const long long i0 = rg->i0;
      unsigned long long ci = (sh.gcnt >> 32) + rg->cpo;
      unsigned long long ei = (sh.gcnt & 0xffffffffull) + rg->exo;
#pragma unroll
      for (int t = 0; t < 8; t++) {
        if (!(cpm & (1u << t))) continue;
        const unsigned ty = (types >> (2 * t)) & 3u;
        const bool ext = (ty == 1u || ty == 2u);
        const long long idx = i0 + t;
        if (ci < a.cp_cap) {
          const float xv = __ldg(a.data + idx);
          if (a.cp_mode == kCpPairs) {
            reinterpret_cast<uint2 *>(a.cp_out)[ci] = make_uint2(float_code(xv), ext ? (uint32_t)ei : kNoExtremum);
          } else {
            long long r;
            const int bin = quant_bin(xv, a.eb, a.inv);
            if (a.g.nd == 2) {
              const long long row = fdivmod(idx, a.g.d3, a.g.m_d3, r);
              int *rec = reinterpret_cast<int *>(a.cp_out) + 5 * ci;
              rec[0] = (int)row; rec[1] = (int)r; rec[2] = (int)ty; rec[3] = bin; rec[4] = 0;
            } else {
              long long z;
              const long long x3 = fdivmod(idx, a.g.plane, a.g.m_plane, r);
              const long long y3 = fdivmod(r, a.g.d3, a.g.m_d3, z);
              int *rec = reinterpret_cast<int *>(a.cp_out) + 6 * ci;
              rec[0] = (int)x3; rec[1] = (int)y3; rec[2] = (int)z; rec[3] = (int)ty; rec[4] = bin; rec[5] = 0;
            }
          }
        }
        ci++;
        if (ext) ei++;
      }
    }
    __syncthreads();
  }
}

// Encodes tile `tile` (TB codec blocks) of the field described by `a`: all
// threads of the CTA call it; it ends with a CTA barrier.
template <int MODE, int G, int WARPS>
__device__ __forceinline__ void encode2_tile(const EncArgs &a, const long long tile, unsigned char *img,
                                             EncShared<G, WARPS> &sh) {
  EncRegs rg;
  encode2_front<MODE, G, WARPS>(a, tile, img, sh, rg);
  encode2_back<MODE, G, WARPS>(a, tile, img, sh, &rg);
}

// One field: persistent CTAs claim tiles from a.tile_ctr in order (within
// [a.tile_lo, a.tile_hi) when a.tile_hi is set: a launch per part of the
// field).  With a.img_stride set the CTA keeps two tile images and runs one
// tile behind: it publishes tile k's aggregate (front half) before it looks
// back for tile k-1 and writes that one out, so the look-back's wait overlaps
// a tile of work.  A CTA waits only after publishing the aggregates of every
// tile it holds, and tiles are claimed in order, so every tile a look-back
// waits for belongs to a running CTA that is not waiting.  The record CP mode
// (per-thread values needed after the look-back) takes the unpipelined loop.
template <int MODE, int G>
__global__ void __launch_bounds__(kThreads, (MODE == kEncClassify ? 3 : 4))
encode2_kernel(EncArgs a) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ EncShared<G, kWarps> sh[2];
  __shared__ long long s_claim;
  const long long nblocks = ((long long)a.n + a.B - 1) / a.B;
  const long long ntiles = (nblocks + EncShared<G, kWarps>::TB - 1) / EncShared<G, kWarps>::TB;
  const long long tend = a.tile_hi ? (long long)a.tile_hi : ntiles;
  if (a.img_stride == 0 || (MODE == kEncClassify && a.cp_mode == kCpRecords)) {
    while (true) {
      if (threadIdx.x == 0) s_claim = (long long)a.tile_lo + (long long)atomicAdd(a.tile_ctr, 1u);
      __syncthreads();
      const long long tile = s_claim;
      if (tile >= tend) break;
      encode2_tile<MODE, G, kWarps>(a, tile, smem_dyn, sh[0]);
    }
    return;
  }
  long long prev = -1;
  int cur = 0;
  while (true) {
    if (threadIdx.x == 0) s_claim = (long long)a.tile_lo + (long long)atomicAdd(a.tile_ctr, 1u);
    __syncthreads();
    const long long tile = s_claim;
    const bool more = tile < tend;
    if (more) {
      EncRegs rg;
      encode2_front<MODE, G, kWarps>(a, tile, smem_dyn + (size_t)cur * a.img_stride, sh[cur], rg);
    }
    if (prev >= 0)
      encode2_back<MODE, G, kWarps>(a, prev, smem_dyn + (size_t)(cur ^ 1) * a.img_stride, sh[cur ^ 1], nullptr);
    if (!more) break;
    prev = tile;
    cur ^= 1;
  }
}

template <int MODE, int G, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, (MODE == kEncClassify ? 24 : 32) / WARPS)
encode2_batch_kernel(const EncArgs *__restrict__ fields, const unsigned long long *__restrict__ tile_start,
                     const unsigned *__restrict__ nfields_dev, unsigned *queue) {
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ EncShared<G, WARPS> sh;
  __shared__ EncArgs s_a;
  const int nf = (int)*nfields_dev;
  const unsigned long long total = tile_start[nf];
  int have = -1;
  while (true) {
    if (threadIdx.x == 0) {
      const unsigned long long t = atomicAdd(queue, 1u);
      if (t >= total) {
        sh.tile = -1;
      } else {
        int lo = 0, hi = nf - 1;   // last field with tile_start <= t
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (tile_start[mid] <= t) lo = mid; else hi = mid - 1;
        }
        sh.field = lo;
        sh.tile = (long long)(t - tile_start[lo]);
      }
    }
    __syncthreads();
    if (sh.tile < 0) break;
    if (sh.field != have) {
      have = sh.field;
      const unsigned long long *src = reinterpret_cast<const unsigned long long *>(fields + have);
      unsigned long long *dst = reinterpret_cast<unsigned long long *>(&s_a);
      for (int w = threadIdx.x; w < (int)(sizeof(EncArgs) / 8); w += WARPS * 32) dst[w] = src[w];
      __syncthreads();
    }
    encode2_tile<MODE, G, WARPS>(s_a, sh.tile, smem_dyn, sh);
  }
}

// reads 8 bytes starting at an arbitrary shared-memory byte position
__device__ __forceinline__ unsigned long long ld_bytes8(const unsigned char *img, unsigned p) {
  const uint32_t *w = reinterpret_cast<const uint32_t *>(img);
  const unsigned wi = p >> 2, sh = 8u * (p & 3u);
  const uint32_t a = w[wi], b = w[wi + 1], c = w[wi + 2];
  const uint32_t lo = sh ? __funnelshift_r(a, b, sh) : a;
  const uint32_t hi = sh ? __funnelshift_r(b, c, sh) : b;
  return ((unsigned long long)hi << 32) | lo;
}

// eight CTAs per SM (32 registers, full occupancy)
template <bool TAGS, int G>
__global__ void __launch_bounds__(kThreads, 8)
decode2_kernel(DecArgs a) {
  constexpr int BPW = 32 / G;
  constexpr int TB = kWarps * BPW;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ unsigned long long s_off[TB + 1];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int gi = lane / G, l = lane % G;
  unsigned char *img = smem_dyn;

  const long long n = (long long)a.n;
  const int B = a.B;
  const long long nblocks = (n + B - 1) / B;
  const long long b0 = (long long)blockIdx.x * TB;
  if (b0 >= nblocks) return;
  const int nb = (int)((nblocks - b0) < TB ? (nblocks - b0) : TB);
  for (int t = threadIdx.x; t <= nb; t += kThreads) {
    unsigned long long o;
    if (t < nb) o = a.blk_off[b0 + t];
    else o = (b0 + nb < nblocks) ? a.blk_off[b0 + nb] : a.payload_len;
    s_off[t] = o;
  }
  __syncthreads();
  // the image holds the payload bytes from the 16-byte boundary at or below
  // payload + lo: img[ib + k] is payload[lo + k]
  const unsigned long long lo = s_off[0];
  unsigned long long hi = s_off[nb];
  if (hi > a.payload_len) hi = a.payload_len;
  if (lo > hi || hi - lo > a.img_cap) {
    if (threadIdx.x == 0) atomicExch(a.err, kErrMalformed);
    return;
  }
  const unsigned ib = (unsigned)(reinterpret_cast<uintptr_t>(a.payload + lo) & 15u);
  {
    // addresses as integers: the aligned start may precede the payload
    const uintptr_t pb = reinterpret_cast<uintptr_t>(a.payload), pe = pb + a.payload_len;
    const uintptr_t g16 = pb + lo - ib;   // 16-byte aligned
    const unsigned nq = (ib + (unsigned)(hi - lo) + 15u) >> 4;
    uint4 *imgq = reinterpret_cast<uint4 *>(img);
    // a chunk wholly inside [payload, payload + payload_len) is one vector load;
    // the first and last chunks may reach outside and go byte by byte
    for (uint32_t q = threadIdx.x; q < nq; q += kThreads) {
      const uintptr_t src = g16 + 16u * q;
      uint4 v;
      if (src >= pb && src + 16 <= pe) {
        v = __ldg(reinterpret_cast<const uint4 *>(src));
      } else {
        uint32_t w4[4] = {0u, 0u, 0u, 0u};
        for (int t = 0; t < 16; t++)
          if (src + t >= pb && src + t < pe)
            w4[t >> 2] |= (uint32_t)(*reinterpret_cast<const unsigned char *>(src + t)) << (8 * (t & 3));
        v = make_uint4(w4[0], w4[1], w4[2], w4[3]);
      }
      imgq[q] = v;
    }
    if (threadIdx.x == 0) imgq[nq] = make_uint4(0u, 0u, 0u, 0u);  // padding for 8-byte window reads
  }
  __syncthreads();

  const int bi = warp * BPW + gi;
  const bool have = bi < nb;
  const long long blk = b0 + bi;
  const long long base = blk * B;
  const int len = have ? (int)((n - base) < B ? (n - base) : B) : 0;
  const int e0 = 8 * l;
  const int nv = len - e0 < 0 ? 0 : (len - e0 > 8 ? 8 : len - e0);
  bool ok = have;
  unsigned start = 0, bend = 0;
  if (ok) {
    if (s_off[bi] < s_off[0] || s_off[bi] + 4 > hi || s_off[bi + 1] < s_off[bi] || s_off[bi + 1] > s_off[nb])
      ok = false;
    start = (unsigned)(s_off[bi] - lo) + ib;
    bend = (unsigned)((s_off[bi + 1] < hi ? s_off[bi + 1] : hi) - lo) + ib;
  }
  unsigned bc = 0;
  int anchor = 0;
  const int cnt = len > 0 ? len - 1 : 0;
  if (ok) {
    anchor = (int)((unsigned)img[start] | ((unsigned)img[start + 1] << 8) | ((unsigned)img[start + 2] << 16) |
                   ((unsigned)img[start + 3] << 24));
    if (len > 1) bc = (start + 4 < bend) ? img[start + 4] : 0u;
    if (bc > 32u || start + block_bytes_layout((unsigned)len, bc, TAGS, a.cpu_layout != 0) > bend) ok = false;
  }
  if (have && !ok && l == 0) atomicExch(a.err, kErrMalformed);
  // deltas e0 .. e0+7
  unsigned dl[8];
  unsigned tsum = 0;
#pragma unroll
  for (int t = 0; t < 8; t++) dl[t] = 0;
  unsigned p = start + 4 + (len > 1 ? 1u : 0u);
  if (ok && bc && e0 < cnt) {
    const unsigned sbytes = (unsigned)(cnt + 7) / 8u;
    const unsigned negb = img[p + l];
    const unsigned mag = p + sbytes;
    const unsigned fb = bc >> 3, rem = bc & 7u;
    // Branch-free for the common widths (fb <= 1), so that the blocks of a
    // warp, which have their own bit counts, do not serialise: the remainder
    // window is read even when rem == 0 (its address then is the end of the
    // magnitude section, inside the image) and masked to nothing.
    const unsigned rsec = mag + fb * (unsigned)cnt;
    // this octet's remainder fields: rem bytes at byte l*rem, MSB first;
    // bytes in stream order -> big-endian integer: byte-swap the 8-byte
    // window and keep its top rem bytes
    const unsigned long long w = ld_bytes8(img, rsec + (unsigned)l * rem);
    const unsigned long long sw =
        ((unsigned long long)__byte_perm((unsigned)w, 0u, 0x0123) << 32) | __byte_perm((unsigned)(w >> 32), 0u, 0x0123);
    const unsigned long long rbits = rem ? (sw >> (64u - 8u * rem)) : 0ull;
    const unsigned long long fw = (fb == 1) ? ld_bytes8(img, mag + (unsigned)e0) : 0ull;
    const unsigned rmask = (1u << rem) - 1u;
#pragma unroll
    for (int t = 0; t < 8; t++) {
      unsigned v = ((unsigned)(rbits >> (rem * (7u - t))) & rmask) | (((unsigned)(fw >> (8 * t)) & 0xffu) << rem);
      if (fb >= 2 && e0 + t < cnt) {
        unsigned full = 0;
        const unsigned o = mag + (unsigned)(e0 + t) * fb;
        for (unsigned u = 0; u < fb; u++) full |= (unsigned)img[o + u] << (8 * u);
        v |= full << rem;
      }
      const unsigned neg = (negb >> (7 - t)) & 1u;
      dl[t] = (e0 + t < cnt) ? ((v ^ (0u - neg)) + neg) : 0u;
      tsum += dl[t];
    }
  }
  // exclusive scan of the octet sums inside the group
  unsigned inc = tsum;
#pragma unroll
  for (int o = 1; o < G; o <<= 1) {
    const unsigned u = __shfl_up_sync(0xffffffffu, inc, o, G);
    if (l >= o) inc += u;
  }
  unsigned v = (unsigned)anchor + inc - tsum;
  unsigned n_ext = 0;
  if (ok && nv > 0) {
    int qv[8];
#pragma unroll
    for (int t = 0; t < 8; t++) { qv[t] = (int)v; v += dl[t]; }
    const long long i0 = base + e0;
    if (a.out_f) {
      float f[8];
#pragma unroll
      for (int t = 0; t < 8; t++) f[t] = __fmul_rn((float)qv[t], a.eb);
      if (nv == 8 && ((reinterpret_cast<uintptr_t>(a.out_f + i0) & 15) == 0)) {
        reinterpret_cast<float4 *>(a.out_f + i0)[0] = make_float4(f[0], f[1], f[2], f[3]);
        reinterpret_cast<float4 *>(a.out_f + i0)[1] = make_float4(f[4], f[5], f[6], f[7]);
      } else {
#pragma unroll
        for (int t = 0; t < 8; t++) if (t < nv) a.out_f[i0 + t] = f[t];
      }
    }
    if (a.out_i) {
      if (nv == 8 && ((reinterpret_cast<uintptr_t>(a.out_i + i0) & 15) == 0)) {
        reinterpret_cast<int4 *>(a.out_i + i0)[0] = make_int4(qv[0], qv[1], qv[2], qv[3]);
        reinterpret_cast<int4 *>(a.out_i + i0)[1] = make_int4(qv[4], qv[5], qv[6], qv[7]);
      } else {
#pragma unroll
        for (int t = 0; t < 8; t++) if (t < nv) a.out_i[i0 + t] = qv[t];
      }
    }
    if (TAGS) {
      const unsigned tsec =
          start + block_bytes_layout((unsigned)len, bc, true, a.cpu_layout != 0) - ((unsigned)len + 3u) / 4u;
      const unsigned tb = ((unsigned)len + 3u) / 4u;
      const unsigned b0t = (2u * l < tb) ? img[tsec + 2 * l] : 0u;
      const unsigned b1t = (2u * l + 1u < tb) ? img[tsec + 2 * l + 1] : 0u;
      unsigned ty[8];
      ty[0] = (b0t >> 6) & 3u; ty[1] = (b0t >> 4) & 3u; ty[2] = (b0t >> 2) & 3u; ty[3] = b0t & 3u;
      ty[4] = (b1t >> 6) & 3u; ty[5] = (b1t >> 4) & 3u; ty[6] = (b1t >> 2) & 3u; ty[7] = b1t & 3u;
      unsigned ne = 0;
#pragma unroll
      for (int t = 0; t < 8; t++) if (t < nv && (ty[t] == 1u || ty[t] == 2u)) ne++;
      if (a.fn_u8) {
        if (nv == 8 && ((reinterpret_cast<uintptr_t>(a.fn_u8 + i0) & 7) == 0)) {
          unsigned long long w = 0;
#pragma unroll
          for (int t = 0; t < 8; t++) w |= (unsigned long long)ty[t] << (8 * t);
          *reinterpret_cast<unsigned long long *>(a.fn_u8 + i0) = w;
        } else {
#pragma unroll
          for (int t = 0; t < 8; t++) if (t < nv) a.fn_u8[i0 + t] = (unsigned char)ty[t];
        }
      }
      if (a.fn_i) {
#pragma unroll
        for (int t = 0; t < 8; t++) if (t < nv) a.fn_i[i0 + t] = (int)ty[t];
      }
      n_ext = ne;
    }
  }
  if (TAGS && a.ext_count) {
    // one atomic per CTA: every CTA adds to the same word, so per-warp
    // atomics would queue at its L2 slice
    __shared__ unsigned s_ext[kWarps];
    n_ext = __reduce_add_sync(0xffffffffu, n_ext);
    if (lane == 0) s_ext[warp] = n_ext;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned tot = 0;
#pragma unroll
      for (int w = 0; w < kWarps; w++) tot += s_ext[w];
      if (tot) atomicAdd(a.ext_count, (unsigned long long)tot);
    }
  }
}

}  // namespace tsz
