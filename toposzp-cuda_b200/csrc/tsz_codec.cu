// Block codec kernels: fused quantize + classify + pack (single pass with a
// decoupled look-back for the output offsets), and the tile decoder.
//
// Encoder data flow per CTA tile (kWarps * BPW codec blocks):
//   1. each warp owns BPW blocks; lanes hold elements j = lane + 32k.  They
//      quantize, classify (or read types), form deltas and reduce the block's
//      max magnitude -> bit count -> byte size.
//   2. the CTA scans the block sizes (and CP counts) inside the tile.
//   3. the warps pack their blocks into a shared-memory byte image of the
//      tile; every byte is written exactly once with a plain byte store
//      (signs via ballots, tags via shuffles, remainder bits gathered from a
//      per-warp magnitude scratch), so no zeroing and no atomics are needed.
//   4. warp 0 runs the look-back to get the tile's global byte offset and
//      its CP / extremum offsets; the tile image is then written out with
//      aligned 32-bit stores (edge bytes stored individually).
#include "tsz_codec.h"
#include "tsz_codec2.cuh"
#include "tsz_lookback.cuh"

namespace tsz {

// ----------------------------------------------------------------------------
// encoder
// ----------------------------------------------------------------------------

template <int MODE, int KMAX, int BPW>
__global__ void __launch_bounds__(kThreads)
encode_kernel(EncArgs a) {
  constexpr int TB = kWarps * BPW;  // codec blocks per tile
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ uint32_t s_bytes[TB + 1];
  __shared__ uint32_t s_cps[TB + 1];
  __shared__ uint32_t s_ext[TB + 1];
  __shared__ long long s_tile;
  __shared__ unsigned long long s_gbyte, s_gcnt;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned FULL = 0xffffffffu;
  const bool tags = mode_tags(MODE);

  uint32_t *scratch = reinterpret_cast<uint32_t *>(smem_dyn);            // kWarps * KMAX * 32
  unsigned char *img = smem_dyn + kWarps * KMAX * 32 * 4;                 // tile byte image
  uint32_t *imgw = reinterpret_cast<uint32_t *>(img);
  uint32_t *mymags = scratch + warp * KMAX * 32;

  const long long n = (long long)a.n;
  const int B = a.B;
  const long long nblocks = (n + B - 1) / B;
  const long long ntiles = (nblocks + TB - 1) / TB;

  while (true) {
    if (threadIdx.x == 0) s_tile = (long long)atomicAdd(a.tile_ctr, 1u);
    __syncthreads();
    const long long tile = s_tile;
    if (tile >= ntiles) break;

    // ---- phase 1: load, quantize, classify, size ----
    int q[BPW][KMAX];
    uint32_t tg[BPW][KMAX];
    uint32_t bcs[BPW];
    int lens[BPW];
#pragma unroll
    for (int i = 0; i < BPW; i++) {
      const int bi = warp + kWarps * i;
      const long long blk = tile * TB + bi;
      const long long base = blk * B;
      const int len = (blk < nblocks) ? (int)((n - base) < B ? (n - base) : B) : 0;
      lens[i] = len;
      uint32_t maxm = 0, cps = 0, ext = 0;
      int prev_last = 0;
#pragma unroll
      for (int k = 0; k < KMAX; k++) {
        const int j = lane + 32 * k;
        const bool in = j < len;
        int qv = 0;
        uint32_t tv = 0;
        if (in) {
          if (MODE == kEncInts || MODE == kEncIntTypes) {
            qv = a.ints[base + j];
            if (MODE == kEncIntTypes) tv = (uint32_t)(a.types[base + j] & 3u);
          } else {
            const float x = a.data[base + j];
            qv = quantize(x, a.inv);
            if (MODE == kEncClassify) tv = (uint32_t)classify_at(a.data, base + j, a.g);
            else if (MODE == kEncTypes) tv = (uint32_t)(a.types[base + j] & 3u);
          }
        }
        q[i][k] = qv;
        tg[i][k] = tv;
        int prv = __shfl_up_sync(FULL, qv, 1);
        if (lane == 0) prv = (k == 0) ? qv : prev_last;
        prev_last = __shfl_sync(FULL, qv, 31);
        if (in && j >= 1) {
          uint32_t ud = (uint32_t)qv - (uint32_t)prv;
          uint32_t m = ((int)ud < 0) ? (0u - ud) : ud;
          maxm = m > maxm ? m : maxm;
        }
        if (MODE == kEncClassify) {
          cps += __popc(__ballot_sync(FULL, tv != 0));
          ext += __popc(__ballot_sync(FULL, tv == 1 || tv == 2));
        }
      }
      maxm = __reduce_max_sync(FULL, maxm);
      const uint32_t bc = bitcount(maxm);
      bcs[i] = bc;
      if (lane == 0) {
        s_bytes[bi] = len ? block_bytes((uint32_t)len, bc, tags) : 0u;
        s_cps[bi] = cps;
        s_ext[bi] = ext;
      }
    }
    __syncthreads();

    // ---- phase 2: tile-local exclusive scan (warp 0) ----
    if (warp == 0) {
      uint32_t vb = lane < TB ? s_bytes[lane] : 0u;
      uint32_t vc = lane < TB ? s_cps[lane] : 0u;
      uint32_t ve = lane < TB ? s_ext[lane] : 0u;
      uint32_t ib = vb, ic = vc, ie = ve;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t tb_ = __shfl_up_sync(FULL, ib, o), tc = __shfl_up_sync(FULL, ic, o),
                 te = __shfl_up_sync(FULL, ie, o);
        if (lane >= o) { ib += tb_; ic += tc; ie += te; }
      }
      if (lane < TB) { s_bytes[lane] = ib - vb; s_cps[lane] = ic - vc; s_ext[lane] = ie - ve; }
      if (lane == TB - 1) {
        s_bytes[TB] = ib; s_cps[TB] = ic; s_ext[TB] = ie;
        // publish this tile's aggregate before packing so successors can resolve early
        publish_aggregate(a.desc, tile, ib, ((unsigned long long)ic << 32) | (unsigned long long)ie);
      }
    }
    __syncthreads();
    const uint32_t tile_bytes = s_bytes[TB];

    // ---- phase 3: pack each block into the tile image ----
#pragma unroll
    for (int i = 0; i < BPW; i++) {
      const int bi = warp + kWarps * i;
      const int len = lens[i];
      if (len == 0 || a.out == nullptr) continue;
      const uint32_t bc = bcs[i];
      uint32_t p = s_bytes[bi];
      if (lane == 0) {
        const uint32_t an = (uint32_t)q[i][0];
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
          const uint32_t cnt = (uint32_t)len - 1u;
          const uint32_t sbytes = (cnt + 7u) / 8u;
          // magnitudes (by delta index) into the per-warp scratch, sign masks by chunk
          uint32_t negm[KMAX];
          int prev_last = 0;
#pragma unroll
          for (int k = 0; k < KMAX; k++) {
            const int j = lane + 32 * k;
            const int qv = q[i][k];
            int prv = __shfl_up_sync(FULL, qv, 1);
            if (lane == 0) prv = (k == 0) ? qv : prev_last;
            prev_last = __shfl_sync(FULL, qv, 31);
            bool neg = false;
            if (j >= 1 && j < len) {
              uint32_t ud = (uint32_t)qv - (uint32_t)prv;
              neg = (int)ud < 0;
              mymags[j - 1] = neg ? (0u - ud) : ud;
            }
            negm[k] = __ballot_sync(FULL, neg);
          }
          // sign bytes: delta d <-> element d + 1; 32 deltas per chunk k
#pragma unroll
          for (int k = 0; k < KMAX; k++) {
            if (lane == k) {
              uint32_t dk = negm[k] >> 1;
              if (k + 1 < KMAX) dk |= negm[k + 1] << 31;
              const uint32_t r = __brev(dk);
#pragma unroll
              for (int u = 0; u < 4; u++) {
                const uint32_t m = 4u * k + u;
                if (m < sbytes) img[p + m] = (unsigned char)(r >> (24 - 8 * u));
              }
            }
          }
          p += sbytes;
          __syncwarp();
          const uint32_t fb = bc >> 3, rem = bc & 7u;
          if (fb) {
#pragma unroll
            for (int k = 0; k < KMAX; k++) {
              const int d = lane + 32 * k;
              if (d < (int)cnt) {
                uint32_t v = mymags[d] >> rem;
                for (uint32_t t = 0; t < fb; t++) { img[p + d * fb + t] = (unsigned char)v; v >>= 8; }
              }
            }
            p += fb * cnt;
          }
          if (rem) {
            const uint32_t rbytes = (rem * cnt - 1u) / 8u + 1u;
            const uint32_t mask = (1u << rem) - 1u;
            for (uint32_t m = lane; m < rbytes; m += 32) {
              // output byte m holds bits [8m, 8m + 8) of the remainder bit stream
              const uint32_t b0 = 8u * m, b1 = b0 + 8u;
              uint32_t d0 = b0 / rem, d1 = (b1 - 1u) / rem;
              if (d1 >= cnt) d1 = cnt - 1u;
              uint32_t acc = 0;
              for (uint32_t d = d0; d <= d1; d++) {
                const uint32_t v = mymags[d] & mask;
                // value bits occupy [d*rem, d*rem + rem); place relative to b0 (MSB first)
                const int sh = (int)(b0 + 8u) - (int)(d * rem + rem);  // left shift into byte
                acc |= (sh >= 0) ? (v << sh) : (v >> (-sh));
              }
              img[p + m] = (unsigned char)acc;
            }
            p += rbytes;
          }
          __syncwarp();
        }
      }
      if (tags) {
#pragma unroll
        for (int k = 0; k < KMAX; k++) {
          const int j = lane + 32 * k;
          uint32_t v = (j < len) ? (tg[i][k] << (6 - 2 * (j & 3))) : 0u;
          v |= __shfl_xor_sync(FULL, v, 1);
          v |= __shfl_xor_sync(FULL, v, 2);
          if (j < len && (j & 3) == 0) img[p + (j >> 2)] = (unsigned char)v;
        }
      }
    }

    // ---- phase 4: look-back for the tile's global offsets ----
    if (warp == 0) {
      const unsigned long long agg_cnt =
          ((unsigned long long)s_cps[TB] << 32) | (unsigned long long)s_ext[TB];
      Prefix pf = lookback(a.desc, tile, tile_bytes, agg_cnt, a.err, true);
      if (lane == 0) {
        s_gbyte = pf.bytes;
        s_gcnt = pf.cnt;
        if (tile == ntiles - 1 && a.total) {
          a.total[0] = pf.bytes + tile_bytes;
          a.total[1] = (pf.cnt >> 32) + s_cps[TB];
          a.total[2] = (pf.cnt & 0xffffffffull) + s_ext[TB];
        }
      }
    }
    __syncthreads();
    const unsigned long long G = s_gbyte;
    const bool fits = a.out != nullptr && (G + tile_bytes) <= a.out_cap;
    if (a.out != nullptr && !fits && threadIdx.x == 0) atomicExch(a.err, kErrOutputOverflow);

    if (a.blk_off && threadIdx.x < TB) {
      const long long blk = tile * TB + threadIdx.x;
      if (blk < nblocks) a.blk_off[blk] = G + s_bytes[threadIdx.x];
    }

    // ---- phase 5: write the tile image ----
    if (fits && tile_bytes) {
      unsigned char *dst = a.out + G;
      uint32_t head = (uint32_t)((4u - (uint32_t)(G & 3ull)) & 3u);
      if (head > tile_bytes) head = tile_bytes;
      if (threadIdx.x < head) dst[threadIdx.x] = img[threadIdx.x];
      const uint32_t nw = (tile_bytes - head) >> 2;
      uint32_t *dstw = reinterpret_cast<uint32_t *>(dst + head);
      const uint32_t sh = 8u * (head & 3u);
      for (uint32_t w = threadIdx.x; w < nw; w += kThreads) {
        const uint32_t p0 = head + 4u * w;
        const uint32_t lo = imgw[p0 >> 2];
        const uint32_t v = sh ? __funnelshift_r(lo, imgw[(p0 >> 2) + 1], sh) : lo;
        dstw[w] = v;
      }
      const uint32_t tail0 = head + 4u * nw;
      if (tail0 + threadIdx.x < tile_bytes) dst[tail0 + threadIdx.x] = img[tail0 + threadIdx.x];
    }

    // ---- phase 6: critical-point emission (raster order) ----
    if (MODE == kEncClassify && a.cp_mode != kCpNone) {
      const unsigned long long cp_base = s_gcnt >> 32;
      const unsigned long long ex_base = s_gcnt & 0xffffffffull;
#pragma unroll
      for (int i = 0; i < BPW; i++) {
        const int bi = warp + kWarps * i;
        const int len = lens[i];
        if (len == 0) continue;
        const long long base = (tile * TB + bi) * (long long)B;
        unsigned long long cpo = cp_base + s_cps[bi];
        unsigned long long exo = ex_base + s_ext[bi];
#pragma unroll
        for (int k = 0; k < KMAX; k++) {
          const int j = lane + 32 * k;
          const uint32_t tv = tg[i][k];
          const unsigned cm = __ballot_sync(FULL, tv != 0);
          const unsigned em = __ballot_sync(FULL, tv == 1 || tv == 2);
          const unsigned lt = (1u << lane) - 1u;
          if (tv != 0 && j < len) {
            const unsigned long long ci = cpo + __popc(cm & lt);
            const unsigned long long ei = exo + __popc(em & lt);
            const long long idx = base + j;
            const float x = a.data[idx];
            if (a.cp_mode == kCpPairs) {
              if (ci < a.cp_cap) {
                uint2 pr;
                pr.x = float_code(x);
                pr.y = (tv == 1 || tv == 2) ? (uint32_t)ei : kNoExtremum;
                reinterpret_cast<uint2 *>(a.cp_out)[ci] = pr;
              }
            } else if (ci < a.cp_cap) {
              long long r;
              const int bin = quant_bin(x, a.eb, a.inv);
              if (a.g.nd == 2) {
                const long long row = fdivmod(idx, a.g.d3, a.g.m_d3, r);
                int *rec = reinterpret_cast<int *>(a.cp_out) + 5 * ci;
                rec[0] = (int)row; rec[1] = (int)r; rec[2] = (int)tv; rec[3] = bin; rec[4] = 0;
              } else {
                long long z;
                const long long x3 = fdivmod(idx, a.g.plane, a.g.m_plane, r);
                const long long y3 = fdivmod(r, a.g.d3, a.g.m_d3, z);
                int *rec = reinterpret_cast<int *>(a.cp_out) + 6 * ci;
                rec[0] = (int)x3; rec[1] = (int)y3; rec[2] = (int)z; rec[3] = (int)tv;
                rec[4] = bin; rec[5] = 0;
              }
            }
          }
          cpo += __popc(cm);
          exo += __popc(em);
        }
      }
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------------------
// decoder
// ----------------------------------------------------------------------------

template <bool TAGS, int KMAX, int BPW>
__global__ void __launch_bounds__(kThreads)
decode_kernel(DecArgs a) {
  constexpr int TB = kWarps * BPW;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  __shared__ unsigned long long s_off[TB + 1];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const unsigned FULL = 0xffffffffu;
  unsigned char *img = smem_dyn;

  const long long n = (long long)a.n;
  const int B = a.B;
  const long long nblocks = (n + B - 1) / B;
  const long long tile = blockIdx.x;
  const long long b0 = tile * TB;
  if (b0 >= nblocks) return;
  const int nb = (int)((nblocks - b0) < TB ? (nblocks - b0) : TB);

  if (threadIdx.x <= TB) {
    const long long blk = b0 + threadIdx.x;
    unsigned long long o;
    if (threadIdx.x < nb) o = a.blk_off[blk];
    else o = (b0 + nb < nblocks) ? a.blk_off[b0 + nb] : a.payload_len;
    if (threadIdx.x == nb) s_off[nb] = o;
    else if (threadIdx.x < nb) s_off[threadIdx.x] = o;
  }
  __syncthreads();
  // stage [lo, hi) of the payload, lo rounded down to 4 bytes
  const unsigned long long lo = s_off[0] & ~3ull;
  unsigned long long hi = s_off[nb];
  if (hi > a.payload_len) hi = a.payload_len;
  if (s_off[0] > hi) {
    if (threadIdx.x == 0) atomicExch(a.err, kErrMalformed);
    return;
  }
  const unsigned long long span = hi - lo;
  if (span > a.img_cap) {
    if (threadIdx.x == 0) atomicExch(a.err, kErrMalformed);
    return;
  }
  {
    const unsigned long long full_words = (a.payload_len & ~3ull);
    const uint32_t nw = (uint32_t)((span + 3) >> 2);
    const uint32_t *srcw = reinterpret_cast<const uint32_t *>(a.payload + lo);
    uint32_t *imgw = reinterpret_cast<uint32_t *>(img);
    for (uint32_t w = threadIdx.x; w < nw; w += kThreads) {
      const unsigned long long gpos = lo + 4ull * w;
      uint32_t v;
      if (gpos + 4 <= full_words) {
        v = __ldg(srcw + w);
      } else {
        v = 0;
        for (int t = 0; t < 4; t++)
          if (gpos + t < a.payload_len) v |= (uint32_t)a.payload[gpos + t] << (8 * t);
      }
      imgw[w] = v;
    }
    if (threadIdx.x < 2) imgw[nw + threadIdx.x] = 0;  // padding for 2-byte reads
  }
  __syncthreads();

#pragma unroll
  for (int i = 0; i < BPW; i++) {
    const int bi = warp + kWarps * i;
    if (bi >= nb) continue;
    const long long blk = b0 + bi;
    const long long base = blk * B;
    const int len = (int)((n - base) < B ? (n - base) : B);
    // offsets must be monotone and inside the staged span; otherwise the
    // stream is malformed and the block is skipped (no out-of-range reads)
    if (s_off[bi] < s_off[0] || s_off[bi] + 4 > hi || s_off[bi + 1] < s_off[bi] ||
        s_off[bi + 1] > s_off[nb]) {
      if (lane == 0) atomicExch(a.err, kErrMalformed);
      continue;
    }
    uint32_t p = (uint32_t)(s_off[bi] - lo);
    const uint32_t bend = (uint32_t)((s_off[bi + 1] < hi ? s_off[bi + 1] : hi) - lo);
    const int anchor = (int)((uint32_t)img[p] | ((uint32_t)img[p + 1] << 8) |
                             ((uint32_t)img[p + 2] << 16) | ((uint32_t)img[p + 3] << 24));
    p += 4;
    uint32_t bc = 0;
    uint32_t sig = 0, mag = 0, rsec = 0, fb = 0, rem = 0, cnt = 0;
    if (len > 1) {
      bc = (p < bend) ? img[p] : 0u;
      p += 1;
      cnt = (uint32_t)len - 1u;
      if (bc > 32u) {
        if (lane == 0) atomicExch(a.err, kErrMalformed);
        continue;
      }
    }
    // the block must fit inside its own byte range
    if (p - (uint32_t)(s_off[bi] - lo) + 0u > bend - (uint32_t)(s_off[bi] - lo) ||
        (uint32_t)(s_off[bi] - lo) + block_bytes((uint32_t)len, bc, TAGS) > bend) {
      if (lane == 0) atomicExch(a.err, kErrMalformed);
      continue;
    }
    if (len > 1 && bc) {
      sig = p;
      mag = p + (cnt + 7u) / 8u;
      fb = bc >> 3;
      rem = bc & 7u;
      rsec = mag + fb * cnt;
      p = mag + mag_bytes(cnt, bc);
    }
    int carry = anchor;
    unsigned next = 0;
#pragma unroll
    for (int k = 0; k < KMAX; k++) {
      const int j = lane + 32 * k;
      uint32_t delta = 0;
      if (bc && j >= 1 && j < len) {
        const uint32_t d = (uint32_t)j - 1u;
        const uint32_t neg = (img[sig + (d >> 3)] >> (7u - (d & 7u))) & 1u;
        uint32_t v = 0;
        if (rem) {
          const uint32_t bit = d * rem;
          const uint32_t w16 = ((uint32_t)img[rsec + (bit >> 3)] << 8) | img[rsec + (bit >> 3) + 1];
          v = (w16 >> (16u - (bit & 7u) - rem)) & ((1u << rem) - 1u);
        }
        if (fb) {
          uint32_t full = 0;
          for (uint32_t t = 0; t < fb; t++) full |= (uint32_t)img[mag + d * fb + t] << (8 * t);
          v |= full << rem;
        }
        delta = neg ? (0u - v) : v;
      }
      // inclusive warp scan of the deltas
      uint32_t s = delta;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, s, o);
        if (lane >= o) s += t;
      }
      const int qv = (int)((uint32_t)carry + s);
      carry = __shfl_sync(FULL, qv, 31);
      if (j < len) {
        if (a.out_f) a.out_f[base + j] = __fmul_rn((float)qv, a.eb);
        if (a.out_i) a.out_i[base + j] = qv;
        if (TAGS) {
          const uint32_t t = (img[p + (j >> 2)] >> (6 - 2 * (j & 3))) & 3u;
          if (a.fn_i) a.fn_i[base + j] = (int)t;
          if (a.fn_u8) a.fn_u8[base + j] = (unsigned char)t;
          next += (t == 1u || t == 2u);
        }
      }
    }
    if (TAGS && a.ext_count) {
      next = __reduce_add_sync(FULL, next);
      if (lane == 0 && next) atomicAdd(a.ext_count, (unsigned long long)next);
    }
  }
}

// ----------------------------------------------------------------------------
// host launchers
// ----------------------------------------------------------------------------

int kmax_for(int B) { return B <= 32 ? 1 : B <= 64 ? 2 : B <= 128 ? 4 : 9; }
int bpw_for(int kmax) { return kmax <= 2 ? 4 : kmax <= 4 ? 2 : 1; }
int tile_blocks_for(int B) { return kWarps * bpw_for(kmax_for(B)); }

size_t enc_smem_bytes(int B, bool tags) {
  const int km = kmax_for(B);
  const int tb = tile_blocks_for(B);
  size_t img = (size_t)tb * max_block_bytes((uint32_t)B, tags) + 16;
  return (size_t)kWarps * km * 32 * 4 + ((img + 15) & ~(size_t)15);
}

size_t dec_smem_bytes(int B, bool tags) {
  const int tb = tile_blocks_for(B);
  size_t img = (size_t)tb * max_block_bytes((uint32_t)B, tags) + 32;
  return (img + 15) & ~(size_t)15;
}

template <int MODE, int KMAX, int BPW>
static cudaError_t launch_enc(const EncArgs &a, cudaStream_t s, int grid) {
  auto k = encode_kernel<MODE, KMAX, BPW>;
  const size_t sm = enc_smem_bytes(a.B, mode_tags(MODE));
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k<<<grid, kThreads, sm, s>>>(a);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_enc_mode(const EncArgs &a, cudaStream_t s, int grid) {
  switch (kmax_for(a.B)) {
    case 1: return launch_enc<MODE, 1, 4>(a, s, grid);
    case 2: return launch_enc<MODE, 2, 4>(a, s, grid);
    case 4: return launch_enc<MODE, 4, 2>(a, s, grid);
    default: return launch_enc<MODE, 9, 1>(a, s, grid);
  }
}

// ---- octet kernels (blockSize <= 256) ----
int octet_group(int B) {
  const int o = (B + 7) / 8;
  int g = 1;
  while (g < o) g <<= 1;
  return g;
}

size_t enc2_smem_bytes(int B, bool tags, bool classify) {
  const int tb = kWarps * (32 / octet_group(B));
  return enc2_total_smem(B, tags, classify, kWarps, tb);
}

template <int MODE, int G>
static cudaError_t launch_enc2(const EncArgs &a0, cudaStream_t s, int grid) {
  auto k = encode2_kernel<MODE, G>;
  EncArgs a = a0;
  const size_t one = enc2_smem_bytes(a.B, mode_tags(MODE), MODE == kEncClassify);
  // two tile images (pipelined look-back) unless the record CP mode is on
  const bool two = !(MODE == kEncClassify && a.cp_mode == kCpRecords);
  a.img_stride = two ? (unsigned)one : 0u;
  const size_t sm = two ? 2 * one : one;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k<<<grid, kThreads, sm, s>>>(a);
  return cudaGetLastError();
}

template <int MODE>
static cudaError_t launch_enc2_mode(const EncArgs &a, cudaStream_t s, int grid) {
  switch (octet_group(a.B)) {
    case 1: return launch_enc2<MODE, 1>(a, s, grid);
    case 2: return launch_enc2<MODE, 2>(a, s, grid);
    case 4: return launch_enc2<MODE, 4>(a, s, grid);
    case 8: return launch_enc2<MODE, 8>(a, s, grid);
    case 16: return launch_enc2<MODE, 16>(a, s, grid);
    default: return launch_enc2<MODE, 32>(a, s, grid);
  }
}

int enc_tile_blocks(int B) { return B <= 256 ? kWarps * (32 / octet_group(B)) : tile_blocks_for(B); }

cudaError_t launch_encode(int mode, const EncArgs &a, cudaStream_t s, int grid) {
  if (a.B <= 256) {
    if (mode == kEncClassify) return launch_enc2_mode<kEncClassify>(a, s, grid);
    if (mode == kEncTypes) return launch_enc2_mode<kEncTypes>(a, s, grid);
    if (mode == kEncIntTypes) return launch_enc2_mode<kEncIntTypes>(a, s, grid);
    if (mode == kEncQuant) return launch_enc2_mode<kEncQuant>(a, s, grid);
    return launch_enc2_mode<kEncInts>(a, s, grid);
  }
  if (mode == kEncClassify) return launch_enc_mode<kEncClassify>(a, s, grid);
  if (mode == kEncTypes) return launch_enc_mode<kEncTypes>(a, s, grid);
  if (mode == kEncIntTypes) return launch_enc_mode<kEncIntTypes>(a, s, grid);
  if (mode == kEncQuant) return launch_enc_mode<kEncQuant>(a, s, grid);
  return launch_enc_mode<kEncInts>(a, s, grid);
}

template <bool TAGS, int KMAX, int BPW>
static cudaError_t launch_dec(const DecArgs &a, cudaStream_t s) {
  auto k = decode_kernel<TAGS, KMAX, BPW>;
  const size_t sm = dec_smem_bytes(a.B, TAGS);
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const long long nblocks = ((long long)a.n + a.B - 1) / a.B;
  const long long tiles = (nblocks + kWarps * BPW - 1) / (kWarps * BPW);
  if (tiles <= 0) return cudaSuccess;
  k<<<(unsigned)tiles, kThreads, sm, s>>>(a);
  return cudaGetLastError();
}

template <bool TAGS>
static cudaError_t launch_dec_tags(const DecArgs &a, cudaStream_t s) {
  switch (kmax_for(a.B)) {
    case 1: return launch_dec<TAGS, 1, 4>(a, s);
    case 2: return launch_dec<TAGS, 2, 4>(a, s);
    case 4: return launch_dec<TAGS, 4, 2>(a, s);
    default: return launch_dec<TAGS, 9, 1>(a, s);
  }
}

template <bool TAGS, int G>
static cudaError_t launch_dec2(DecArgs a, cudaStream_t s) {
  auto k = decode2_kernel<TAGS, G>;
  const int tb = kWarps * (32 / G);
  const size_t sm = (((size_t)tb * max_block_bytes((uint32_t)a.B, TAGS) + 64) + 15) & ~(size_t)15;
  a.img_cap = sm - 48;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const long long nblocks = ((long long)a.n + a.B - 1) / a.B;
  const long long tiles = (nblocks + tb - 1) / tb;
  if (tiles <= 0) return cudaSuccess;
  k<<<(unsigned)tiles, kThreads, sm, s>>>(a);
  return cudaGetLastError();
}

template <bool TAGS>
static cudaError_t launch_dec2_tags(DecArgs a, cudaStream_t s) {
  switch (octet_group(a.B)) {
    case 1: return launch_dec2<TAGS, 1>(a, s);
    case 2: return launch_dec2<TAGS, 2>(a, s);
    case 4: return launch_dec2<TAGS, 4>(a, s);
    case 8: return launch_dec2<TAGS, 8>(a, s);
    case 16: return launch_dec2<TAGS, 16>(a, s);
    default: return launch_dec2<TAGS, 32>(a, s);
  }
}

cudaError_t launch_decode(bool tags, DecArgs a, cudaStream_t s) {
  if (a.B <= 256) return tags ? launch_dec2_tags<true>(a, s) : launch_dec2_tags<false>(a, s);
  // the generic decoder stages the payload in 4-byte words: the stream must
  // start on a 4-byte boundary (the octet decoder takes any alignment)
  if (reinterpret_cast<uintptr_t>(a.payload) & 3u) return cudaErrorMisalignedAddress;
  a.img_cap = dec_smem_bytes(a.B, tags) - 16;
  return tags ? launch_dec_tags<true>(a, s) : launch_dec_tags<false>(a, s);
}

}  // namespace tsz
