// Single-pass decoupled look-back over tiles (one warp per CTA calls it).
//
// Each tile publishes its aggregate (byte count + packed (cps, extrema) counts),
// then walks its predecessors 32 at a time until it meets an inclusive prefix.
// Every wait is bounded: after kSpinLimit polls the tile records
// kErrLookbackTimeout in *err and proceeds with what it has, so a stalled
// predecessor can never hang the kernel.
#pragma once
#include "tsz_common.cuh"

namespace tsz {

constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

struct Prefix {
  unsigned long long bytes;
  unsigned long long cnt;  // (cps << 32) | extrema
};

// Publishes tile t's aggregate as early as possible (one thread).  Tile 0's
// aggregate is its inclusive prefix.
__device__ __forceinline__ void publish_aggregate(TileDesc *desc, long long t, unsigned long long agg_bytes,
                                                  unsigned long long agg_cnt) {
  if (t == 0) {
    st_relaxed_u64(&desc[0].inc_cnt, agg_cnt);
    st_release_u64(&desc[0].status, (2ull << kStatShift) | agg_bytes);
  } else {
    st_relaxed_u64(&desc[t].agg_cnt, agg_cnt);
    st_release_u64(&desc[t].status, (1ull << kStatShift) | agg_bytes);
  }
}

// Called by all 32 lanes of one warp.  Returns the exclusive prefix of tile t.
// With published == false the aggregate is published first.
__device__ inline Prefix lookback(TileDesc *desc, long long t, unsigned long long agg_bytes,
                                  unsigned long long agg_cnt, int *err, bool published = false) {
  const int lane = threadIdx.x & 31;
  Prefix ex{0ull, 0ull};
  if (!published && lane == 0) publish_aggregate(desc, t, agg_bytes, agg_cnt);
  if (t == 0) {
    __syncwarp();
    return ex;
  }
  long long base = t - 1;
  bool timed_out = false;
  while (true) {
    long long idx = base - lane;
    unsigned long long st = (2ull << kStatShift);
    if (idx >= 0) {
      st = ld_acquire_u64(&desc[idx].status);
      int spins = 0;
      while ((st >> kStatShift) == 0ull) {
        if (++spins > kSpinLimit) { timed_out = true; break; }
        __nanosleep(spins < 64 ? 32 : 256);
        st = ld_acquire_u64(&desc[idx].status);
      }
    }
    unsigned long long flag = st >> kStatShift;
    if (flag == 0ull) flag = 2ull;  // timed out: treat as an empty inclusive value
    unsigned inc_mask = __ballot_sync(0xffffffffu, flag == 2ull);
    int first = inc_mask ? (__ffs(inc_mask) - 1) : 32;
    unsigned long long b = 0, c = 0;
    if (lane <= first && idx >= 0 && (st >> kStatShift) != 0ull) {
      b = st & kByteMask;
      c = (flag == 2ull) ? ld_relaxed_u64(&desc[idx].inc_cnt) : ld_relaxed_u64(&desc[idx].agg_cnt);
    }
    for (int o = 16; o > 0; o >>= 1) {
      b += __shfl_xor_sync(0xffffffffu, b, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    ex.bytes += b;
    ex.cnt += c;
    if (first < 32) break;
    base -= 32;
  }
  if (__any_sync(0xffffffffu, timed_out) && lane == 0) atomicExch(err, kErrLookbackTimeout);
  if (lane == 0) {
    st_relaxed_u64(&desc[t].inc_cnt, ex.cnt + agg_cnt);
    st_release_u64(&desc[t].status, (2ull << kStatShift) | ((ex.bytes + agg_bytes) & kByteMask));
  }
  __syncwarp();
  return ex;
}

}  // namespace tsz

namespace tsz {

// CTA-wide look-back: all WARPS * 32 threads of the CTA call it after the
// tile's aggregate has been published.  Each round inspects one predecessor
// per thread, so a walk back over P in-flight tiles takes about P / (WARPS *
// 32) rounds instead of P / 32.  One CTA barrier per round: every warp sums
// its own predecessors up to its nearest inclusive one and posts (nearest
// inclusive, sums) to a double-buffered slot; after the barrier every thread
// adds the posts of the warps up to the first warp holding an inclusive
// prefix (round r writes buffer r & 1, which round r + 2 may overwrite only
// after every thread has passed round r + 1's barrier).
// spin_limit: polls of one predecessor before the wait gives up (0: kSpinLimit)
template <int WARPS = kWarps>
__device__ inline Prefix lookback_cta(TileDesc *desc, long long t, unsigned long long agg_bytes,
                                      unsigned long long agg_cnt, int *err, int spin_limit = 0) {
  const int limit = spin_limit > 0 ? spin_limit : kSpinLimit;
  __shared__ unsigned s_first[2][WARPS];
  __shared__ unsigned long long s_b[2][WARPS], s_c[2][WARPS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  Prefix ex{0ull, 0ull};
  if (t == 0) return ex;
  long long base = t - 1;
  bool timed_out = false;
  for (int r = 0;; r ^= 1) {
    const long long idx = base - (long long)threadIdx.x;
    unsigned long long st = (2ull << kStatShift);
    if (idx >= 0) {
      st = ld_acquire_u64(&desc[idx].status);
      int spins = 0;
      while ((st >> kStatShift) == 0ull) {
        if (++spins > limit) { timed_out = true; break; }
        __nanosleep(spins < 64 ? 32 : 256);
        st = ld_acquire_u64(&desc[idx].status);
      }
    }
    unsigned long long flag = st >> kStatShift;
    if (flag == 0ull) flag = 2ull;   // timed out: an empty inclusive value
    // this warp's nearest inclusive predecessor (smallest lane)
    const unsigned wm = __ballot_sync(0xffffffffu, flag == 2ull);
    const int wfirst = wm ? (__ffs(wm) - 1) : 32;
    unsigned long long b = 0, c = 0;
    if (lane <= wfirst && idx >= 0 && (st >> kStatShift) != 0ull) {
      b = st & kByteMask;
      c = (flag == 2ull) ? ld_relaxed_u64(&desc[idx].inc_cnt) : ld_relaxed_u64(&desc[idx].agg_cnt);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      b += __shfl_xor_sync(0xffffffffu, b, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
      s_first[r][warp] = wm ? 1u : 0u;
      s_b[r][warp] = b;
      s_c[r][warp] = c;
    }
    __syncthreads();
    bool found = false;
#pragma unroll
    for (int w = 0; w < WARPS; w++) {
      if (!found) {
        ex.bytes += s_b[r][w];
        ex.cnt += s_c[r][w];
        found = s_first[r][w] != 0u;
      }
    }
    if (found) break;
    base -= WARPS * 32;
  }
  if (timed_out) atomicExch(err, kErrLookbackTimeout);
  if (threadIdx.x == 0) {
    st_relaxed_u64(&desc[t].inc_cnt, ex.cnt + agg_cnt);
    st_release_u64(&desc[t].status, (2ull << kStatShift) | ((ex.bytes + agg_bytes) & kByteMask));
  }
  return ex;
}

}  // namespace tsz
