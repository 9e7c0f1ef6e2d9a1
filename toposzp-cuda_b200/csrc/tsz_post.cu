// Post-processing of a decoded field with the exact serial-raster semantics of
// the reference drivers (example/test_cuda_topology.cu:117-326, :493-531 and
// example/test_cuda_topology_3d.cu:75-434, :600-631).
//
// Each reference pass visits points in raster order and updates them in
// place, so a point sees the FINAL values of earlier points and the
// PRE-PASS values of later points.  Only a pass's candidates change (extrema
// for the stencil and enforcement passes, lost saddles for RBF, saddles for
// the axis-pattern stencil), so the passes run over compact candidate lists
// and update F in place as well:
//   * a candidate's result goes to F[e] and, with the pass's generation, to
//     S[e] = (generation << 32) | float bits: one 64-bit word that a reader
//     takes whole (relaxed), so value and readiness never need ordering;
//   * a candidate is computed once every EARLIER candidate it reads has its
//     result for this pass (read from S); otherwise it is retried (stencil
//     and enforcement: a few times, a CTA barrier apart; RBF and axis
//     pattern: bounded polls of the missing words) and then deferred to the
//     next round;
//   * every LATER point a candidate reads lists that candidate among its own
//     earlier reads, so it cannot have been updated yet: F still holds its
//     pre-pass value, exactly as in the serial pass.
// Rounds repeat over the deferred items until none is left (their number is
// the longest chain of adjacent candidates in raster order).  When the
// stencil pass runs, enforcement is fused into it for every candidate with no
// candidate face neighbour, and the enforcement pass proper runs only over the
// rest (face_item_run, enforce_sparse_kernel).  The raw decoded value each
// point is clamped against is the item's own F value before its write when
// the field is the decoded field itself, else gathered per list entry when
// the lists are built.  Floating-point expressions use explicit round-to-nearest
// intrinsics so that no multiply-add is contracted (the reference host code is
// compiled without contraction).
#include <cfloat>

#include "tsz_lookback.cuh"
#include <algorithm>
#include <mutex>
#include <vector>

#include "tsz_ops.h"

namespace tsz {

enum { kPassStencil = 0, kPassEnforce = 1, kPassRbf = 2, kPassAxis = 3 };

// CTA-wide exclusive scan of one value per thread (kPostThreads threads)
__device__ __forceinline__ unsigned cta_excl_scan_post(unsigned v, unsigned *s_warp, unsigned *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  unsigned wpre = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < 256 / 32; w++) {
    const unsigned sw = s_warp[w];
    if (w < warp) wpre += sw;
    tot += sw;
  }
  *total = tot;
  return wpre + inc - v;
}
constexpr int kPostThreads = 256;
constexpr int kPostPer = 8;
constexpr int kPostTile = kPostThreads * kPostPer;

__constant__ double c_w2[9];
__constant__ double c_w3[27];

struct PostArgs {
  float *F;                     // the field, updated in place
  // raw decoded value of each entry of the pass's list; null: the field is
  // the decoded field itself, so an item's raw value is its own F value
  // before its first write in the pass (F[e] changes only by e's own item)
  const float *OL;
  float *RAW;                   // fused stencil with OL null: raw values of the items left for enforcement
  unsigned char *T;             // types in bits 0..1
  const int *sp;
  unsigned long long n_sp;
  Geom g;
  long long n;
  float eb;
  float eps;
  unsigned gen;                 // generation of the current pass
  unsigned long long *S;        // (generation << 32) | result bits, per point
  const unsigned *R;            // RBF candidates (lost saddles) bitmap
  const unsigned *X;            // interior-extremum bitmap (the stencil / enforcement candidates)
  const unsigned *XP;           // per bitmap word: list position of its first extremum (X entries before it)
  int *err;
  unsigned *restored;
  int spin_limit;               // grid-barrier polls before giving up (0: default)
  // stencil pass fused with enforcement (null: plain stencil pass): bitmap
  // over list positions of the items that still need the enforcement pass
  unsigned *NI;
};

// No "memory" clobber: a result word is read whole and carries its own
// readiness, so these loads need no order with the other loads of an item, and
// the compiler may issue them together (a clobber would serialise every load
// after it behind the one before).  A retry re-reads after a barrier.
__device__ __forceinline__ unsigned long long ld_rlx(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void st_rlx(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ int ty(const PostArgs &a, long long q) { return a.T[q] & 3; }

// coordinates of flat index e
struct C3 { long long x, y, z; };
__device__ __forceinline__ C3 coords(const Geom &g, long long e) {
  C3 c;
  long long r;
  if (g.nd == 2) { c.x = 0; c.y = fdivmod(e, g.d3, g.m_d3, r); c.z = r; }
  else { c.x = fdivmod(e, g.plane, g.m_plane, r); c.y = fdivmod(r, g.d3, g.m_d3, c.z); }
  return c;
}

// 4/6-neighbour classification on F (stable during a pass)
__device__ __forceinline__ int classify_F(const PostArgs &a, long long q) {
  const float *F = a.F;
  if (a.g.nd == 2)
    return classify4(F[q], F[q - a.g.d3], F[q + a.g.d3], F[q - 1], F[q + 1]);
  return classify6(F[q], F[q - a.g.plane], F[q + a.g.plane], F[q - a.g.d3], F[q + a.g.d3], F[q - 1],
                   F[q + 1]);
}

__device__ __forceinline__ bool bit_at(const unsigned *b, long long q) { return (b[q >> 5] >> (q & 31)) & 1u; }

// q is a candidate of pass PASS (q_interior: q lies in the interior)
template <int PASS>
__device__ __forceinline__ bool is_cand_known(const PostArgs &a, long long q, bool q_interior) {
  if (!q_interior) return false;
  if (PASS == kPassRbf) return bit_at(a.R, q);
  const int t = ty(a, q);
  if (PASS == kPassStencil || PASS == kPassEnforce) return t == 1 || t == 2;
  return t == 3;
}

__device__ __forceinline__ bool interior_off(const PostArgs &a, const C3 &c, int dx, int dy, int dz) {
  bool qi = c.y + dy >= 1 && c.y + dy <= a.g.d2 - 2 && c.z + dz >= 1 && c.z + dz <= a.g.d3 - 2;
  if (a.g.nd == 3) qi = qi && c.x + dx >= 1 && c.x + dx <= a.g.d1 - 2;
  return qi;
}

// neighbour of e at offset (dx, dy, dz) (dx = 0 in 2D) as the serial pass
// sees it; earlier candidates are resolved before e is computed
template <int PASS>
__device__ __forceinline__ float valo(const PostArgs &a, long long e, const C3 &c, int dx, int dy, int dz) {
  const long long q = e + (long long)dx * a.g.plane + (long long)dy * a.g.d3 + dz;
  if (q > e) return a.F[q];
  if (is_cand_known<PASS>(a, q, interior_off(a, c, dx, dy, dz)))
    return __uint_as_float((unsigned)ld_rlx(&a.S[q]));
  return a.F[q];
}

// value of the earlier point e + (dx, dy, dz) as the serial pass sees it,
// with its loads issued whether or not the caller uses it (exists: the point
// lies in the field; 0 otherwise)
template <int PASS>
__device__ __forceinline__ float far_back(const PostArgs &a, long long e, const C3 &c, int dx, int dy, int dz,
                                          bool exists) {
  if (!exists) return 0.f;
  const long long q = e + (long long)dx * a.g.plane + (long long)dy * a.g.d3 + dz;
  const bool cand = is_cand_known<PASS>(a, q, interior_off(a, c, dx, dy, dz));
  const float fv = a.F[q];
  return cand ? __uint_as_float((unsigned)ld_rlx(&a.S[q])) : fv;
}

// every earlier candidate that an RBF / axis-pattern item may read has its
// result for this pass: the earlier points of the 3x3(x3) box and the points
// two steps back along each axis.  The candidate tests of all of them are
// issued first, then the result words of the candidates, so an item waits
// for two loads in a row, not one per point.  polls > 0: while a result is
// missing, poll the missing words up to polls times (a bounded wait for
// items of the same launch that are computing them); the item is deferred
// when one is still missing.
constexpr int kDepPolls = 256;

template <int PASS, int ND>
__device__ bool deps_ready(const PostArgs &a, long long e, const C3 &c, int polls = 0) {
  constexpr int NB = ND == 3 ? 13 : 4;   // earlier box points
  long long q[NB + 3];
  bool cand[NB + 3];
  int k = 0;
#pragma unroll
  for (int dx = (ND == 3 ? -1 : 0); dx <= 0; dx++)
#pragma unroll
    for (int dy = -1; dy <= 1; dy++)
#pragma unroll
      for (int dz = -1; dz <= 1; dz++) {
        if (dx == 0 && (dy > 0 || (dy == 0 && dz >= 0))) continue;
        q[k] = e + (long long)dx * a.g.plane + (long long)dy * a.g.d3 + dz;
        cand[k] = is_cand_known<PASS>(a, q[k], interior_off(a, c, dx, dy, dz));
        k++;
      }
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int dx = j == 0 ? -2 : 0, dy = j == 1 ? -2 : 0, dz = j == 2 ? -2 : 0;
    const bool in = (ND == 3 || j > 0) && c.x + dx >= 0 && c.y + dy >= 0 && c.z + dz >= 0;
    q[NB + j] = e + (long long)dx * a.g.plane + (long long)dy * a.g.d3 + dz;
    cand[NB + j] = in && is_cand_known<PASS>(a, q[NB + j], interior_off(a, c, dx, dy, dz));
  }
  unsigned pend = 0;
#pragma unroll
  for (int i = 0; i < NB + 3; i++)
    if (cand[i] && (unsigned)(ld_rlx(&a.S[q[i]]) >> 32) != a.gen) pend |= 1u << i;
  for (int p = 0; pend && p < polls; p++) {
    __nanosleep(256);
#pragma unroll
    for (int i = 0; i < NB + 3; i++)
      if (((pend >> i) & 1u) && (unsigned)(ld_rlx(&a.S[q[i]]) >> 32) == a.gen) pend &= ~(1u << i);
  }
  return pend == 0;
}

// ----------------------------------------------------------------------------
// per-point updates
// ----------------------------------------------------------------------------
__device__ __forceinline__ float clampf(float v, float lo, float hi) {
  if (v > hi) v = hi;
  if (v < lo) v = lo;
  return v;
}

// Face neighbours of a stencil / enforcement item as the serial pass sees
// them: xm, ym, zm (earlier points: results of earlier candidates, else F)
// and xp, yp, zp (later points: F).  In 2D the x pair is unused.
struct Face { float xm, xp, ym, yp, zm, zp; };

// 2D stencil (example/test_cuda_topology.cu:118-165)
__device__ __forceinline__ float stencil2(const PostArgs &a, const Face &f, float cur, int t, int s, float o) {
  const float hi = __fadd_rn(o, a.eb), lo = __fsub_rn(o, a.eb);
  float m = cur;
  const float nb[4] = {f.ym, f.yp, f.zm, f.zp};   // rows -1, +1, then columns -1, +1
#pragma unroll
  for (int k = 0; k < 4; k++)
    if (t == 1 ? (nb[k] > m) : (nb[k] < m)) m = nb[k];
  float target;
  if (t == 1) target = __fmul_rn(m, __fadd_rn(1.0f, __fmul_rn((float)s, FLT_EPSILON)));
  else if (s == 0) target = __fmul_rn(m, __fsub_rn(1.0f, FLT_EPSILON));
  else target = __fmul_rn(m, __fsub_rn(1.0f, __fmul_rn(__fdiv_rn(1.0f, (float)s), FLT_EPSILON)));
  return clampf(target, lo, hi);
}

// 3D stencil (example/test_cuda_topology_3d.cu:77-128)
__device__ __forceinline__ float stencil3(const PostArgs &a, const Face &f, int t, int s, float o) {
  const float d = __fmul_rn(a.eb, 0.999f);
  const float hi = __fadd_rn(o, d), lo = __fsub_rn(o, d);
  float target;
  if (t == 1) {
    const float m = fmaxf(fmaxf(f.xm, f.xp), fmaxf(fmaxf(f.ym, f.yp), fmaxf(f.zm, f.zp)));
    target = __fmul_rn(m, __fadd_rn(1.0f, __fmul_rn((float)s, FLT_EPSILON)));
  } else {
    const float m = fminf(fminf(f.xm, f.xp), fminf(fminf(f.ym, f.yp), fminf(f.zm, f.zp)));
    target = (s == 0) ? __fmul_rn(m, __fsub_rn(1.0f, FLT_EPSILON))
                      : __fmul_rn(m, __fsub_rn(1.0f, __fmul_rn(__fdiv_rn(1.0f, (float)s), FLT_EPSILON)));
  }
  return clampf(target, lo, hi);
}

// enforcement (example/test_cuda_topology.cu:168-198, _3d.cu:131-167)
template <int ND>
__device__ __forceinline__ float enforce(const PostArgs &a, const Face &f, float cur, int t, float o) {
  const float d = __fmul_rn(a.eb, 0.999f);
  const float hi = __fadd_rn(o, d), lo = __fsub_rn(o, d);
  const float soft = __fmul_rn(0.25f, a.eps);
  float m;
  if (ND == 2) {
    // north, south, west, east
    m = (t == 1) ? fmaxf(fmaxf(f.ym, f.yp), fmaxf(f.zm, f.zp)) : fminf(fminf(f.ym, f.yp), fminf(f.zm, f.zp));
  } else {
    m = (t == 1) ? fmaxf(fmaxf(f.xm, f.xp), fmaxf(fmaxf(f.ym, f.yp), fmaxf(f.zm, f.zp)))
                 : fminf(fminf(f.xm, f.xp), fminf(fminf(f.ym, f.yp), fminf(f.zm, f.zp)));
  }
  if (t == 1) {
    float tg = __fadd_rn(m, soft);
    if (tg > hi) tg = hi;
    if (tg < lo) tg = lo;
    return (cur < tg) ? tg : cur;
  }
  float tg = __fsub_rn(m, soft);
  if (tg < lo) tg = lo;
  if (tg > hi) tg = hi;
  return (cur > tg) ? tg : cur;
}

// An item of the stencil or enforcement pass, held in registers across the
// local retries.  Its face neighbours as the serial pass sees them: the
// earlier ones (x-1 in 3D, y-1, z-1) are results of this pass where they are
// candidates (bits of X; the result word sits at the list position XP of the
// bitmap word plus the extrema before it in the word), F otherwise; the
// later ones are F.  Everything but the missing result words is loaded once;
// a retry reloads only those.
struct FaceItem {
  long long e;
  float cur, o;          // F at e before the item writes, and its raw value
  int t, s;              // type, sort position (stencil)
  Face f;
  unsigned wait;         // bit k: earlier candidate neighbour k not read yet
  unsigned pos[3];       // their list positions
  bool iso;              // no face neighbour is a candidate (fused stencil)
};

template <int PASS, int ND>
__device__ __forceinline__ void face_item_load(const PostArgs &a, const unsigned *__restrict__ list, unsigned idx,
                                               FaceItem &it) {
  const long long e = (long long)list[idx];
  const long long pl = a.g.plane, d3 = a.g.d3;
  it.e = e;
  it.t = ty(a, e);
  it.s = (PASS == kPassStencil && idx < a.n_sp) ? a.sp[idx] : 0;
  it.cur = a.F[e];
  it.o = a.OL ? a.OL[idx] : it.cur;
  // e is interior: every face neighbour lies in the field
  it.f.xm = ND == 3 ? a.F[e - pl] : 0.f;
  it.f.xp = ND == 3 ? a.F[e + pl] : 0.f;
  it.f.ym = a.F[e - d3];
  it.f.yp = a.F[e + d3];
  it.f.zm = a.F[e - 1];
  it.f.zp = a.F[e + 1];
  unsigned wait = 0;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    it.pos[k] = 0;
    if (ND == 2 && k == 0) continue;
    const long long q = e - (k == 0 ? pl : (k == 1 ? d3 : 1ll));
    const long long wi = q >> 5;
    const unsigned bw = a.X[wi], b = (unsigned)(q & 31);
    wait |= ((bw >> b) & 1u) << k;
    it.pos[k] = a.XP[wi] + (unsigned)__popc(bw & ((1u << b) - 1u));
  }
  it.wait = wait;
  it.iso = false;
  if (PASS == kPassStencil && a.NI) {
    unsigned later = 0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      if (ND == 2 && k == 0) continue;
      const long long q = e + (k == 0 ? pl : (k == 1 ? d3 : 1ll));
      later |= (a.X[q >> 5] >> (unsigned)(q & 31)) & 1u;
    }
    it.iso = (wait | later) == 0u;
  }
}

// Reads the result words still missing; false while one is not final.
__device__ __forceinline__ bool face_item_ready(const PostArgs &a, FaceItem &it) {
  unsigned long long w[3];
#pragma unroll
  for (int k = 0; k < 3; k++) w[k] = ((it.wait >> k) & 1u) ? ld_rlx(&a.S[it.pos[k]]) : 0ull;
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (((it.wait >> k) & 1u) && (unsigned)(w[k] >> 32) == a.gen) {
      const float v = __uint_as_float((unsigned)w[k]);
      if (k == 0) it.f.xm = v;
      else if (k == 1) it.f.ym = v;
      else it.f.zm = v;
      it.wait &= ~(1u << k);
    }
  }
  return it.wait == 0u;
}

// bits [b, b + 32) of a bitmap of nbits bits (zeros outside)
__device__ __forceinline__ unsigned get32(const unsigned *__restrict__ bm, long long b, long long nbits) {
  const long long w = b >> 5;  // arithmetic shift: floor for negative b
  const unsigned sh = (unsigned)(b & 31);
  const long long nw = (nbits + 31) >> 5;
  const unsigned lo = (w >= 0 && w < nw) ? bm[w] : 0u;
  const unsigned hi = (w + 1 >= 0 && w + 1 < nw) ? bm[w + 1] : 0u;
  return sh ? __funnelshift_r(lo, hi, sh) : lo;
}

// Locks of the RBF box around e (example/test_cuda_topology.cu:229-242,
// example/test_cuda_topology_3d.cu:325-341): box point q is locked when it is
// interior and an interior extremum (a bit of the extremum bitmap a.X) lies
// within Chebyshev distance 1 of it.  Read from the 5x5(x5) window of a.X
// around e, one 5-bit row segment per row (z - 2 .. z + 2).  A segment that
// runs past a row end reads points of the neighbouring row's boundary
// columns, and a row outside the field reads boundary rows or nothing; none
// of them holds an interior extremum, so the window needs no clipping.
// Bit (dx + 1) * 9 + (dy + 1) * 3 + (dz + 1) (dx = 0 in 2D: bit (dy + 1) * 3 + dz + 1).
template <int ND>
__device__ __forceinline__ unsigned box_locks(const PostArgs &a, long long e, const C3 &c) {
  constexpr int NX = ND == 3 ? 5 : 1;
  unsigned seg[NX][5];
#pragma unroll
  for (int i = 0; i < NX; i++)
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const long long b = e + (ND == 3 ? (long long)(i - 2) * a.g.plane : 0ll) + (long long)(j - 2) * a.g.d3 - 2;
      seg[i][j] = get32(a.X, b, a.n) & 31u;
    }
  unsigned m = 0;
#pragma unroll
  for (int dx = (ND == 3 ? -1 : 0); dx <= (ND == 3 ? 1 : 0); dx++)
#pragma unroll
    for (int dy = -1; dy <= 1; dy++) {
      unsigned acc = 0;
#pragma unroll
      for (int ox = (ND == 3 ? -1 : 0); ox <= (ND == 3 ? 1 : 0); ox++)
#pragma unroll
        for (int oy = -1; oy <= 1; oy++) acc |= seg[(ND == 3 ? dx + ox + 2 : 0)][dy + oy + 2];
#pragma unroll
      for (int dz = -1; dz <= 1; dz++) {
        // window bits dz + 1 .. dz + 3 are the columns dz - 1 .. dz + 1
        if (((acc >> (dz + 1)) & 7u) && interior_off(a, c, dx, dy, dz))
          m |= 1u << ((ND == 3 ? (dx + 1) * 9 : 0) + (dy + 1) * 3 + (dz + 1));
      }
    }
  return m;
}

__device__ __forceinline__ int cls4_eps(float c, float n, float s, float w, float e, float eps) {
  const float np = __fadd_rn(n, eps), sp = __fadd_rn(s, eps), wp = __fadd_rn(w, eps), ep = __fadd_rn(e, eps);
  const float nm = __fsub_rn(n, eps), sm = __fsub_rn(s, eps), wm = __fsub_rn(w, eps), em = __fsub_rn(e, eps);
  if (c > np && c > sp && c > wp && c > ep) return 1;
  if (c < nm && c < sm && c < wm && c < em) return 2;
  const int vh = (c > np) && (c > sp), vl = (c < nm) && (c < sm);
  const int hh = (c > wp) && (c > ep), hl = (c < wm) && (c < em);
  return ((vh && hl) || (vl && hh)) ? 3 : 0;
}

// 2D RBF saddle restoration of candidate e (example/test_cuda_topology.cu:227-326)
__device__ float rbf2(const PostArgs &a, long long e, const C3 &c, float o, bool &ok) {
  const long long cols = a.g.d3;
  const long long rows = a.g.d2;
  ok = false;
  // 3x3 neighbourhood values as seen by the serial pass
  float v[3][3];
  for (int da = -1; da <= 1; da++)
    for (int db = -1; db <= 1; db++)
      v[da + 1][db + 1] = (da == 0 && db == 0) ? a.F[e] : valo<kPassRbf>(a, e, c, 0, da, db);
  const unsigned lk = box_locks<2>(a, e, c);
  double num = 0.0, den = 0.0;
  for (int da = -1; da <= 1; da++)
    for (int db = -1; db <= 1; db++) {
      double ww = c_w2[(da + 1) * 3 + (db + 1)];
      if ((lk >> ((da + 1) * 3 + (db + 1))) & 1u) ww = __dmul_rn(ww, 0.4);
      num = __dadd_rn(num, __dmul_rn(ww, (double)v[da + 1][db + 1]));
      den = __dadd_rn(den, ww);
    }
  const float old = a.F[e];
  if (!(den > 0.0)) return old;
  const float d = __fmul_rn(a.eb, 0.999f);
  const float lo = __fsub_rn(o, d), hi = __fadd_rn(o, d);
  const float n = v[0][1], s = v[2][1], w = v[1][0], ea = v[1][2];
  float cand = __double2float_rn(__ddiv_rn(num, den));
  {
    const float q = __fmul_rn(0.25f, a.eps);
    float clo = __fsub_rn(fminf(fmaxf(n, s), fmaxf(w, ea)), q);
    float chi = __fadd_rn(fmaxf(fminf(n, s), fminf(w, ea)), q);
    if (clo > chi) {
      const float mid = __fmul_rn(0.5f, __fadd_rn(clo, chi));
      clo = __fsub_rn(mid, q);
      chi = __fadd_rn(mid, q);
    }
    if (cand < clo) cand = clo;
    if (cand > chi) cand = chi;
  }
  if (cand < lo) cand = lo;
  if (cand > hi) cand = hi;
  // outer ring values needed by the neighbour validations
  const bool vu = (c.y - 1 >= 1) && ty(a, e - cols) == 0;
  const bool vd = (c.y + 1 < rows - 1) && ty(a, e + cols) == 0;
  const bool vl = (c.z - 1 >= 1) && ty(a, e - 1) == 0;
  const bool vr = (c.z + 1 < cols - 1) && ty(a, e + 1) == 0;
  // loaded wherever the points exist, so that the loads overlap
  const float gu = far_back<kPassRbf>(a, e, c, 0, -2, 0, c.y >= 2);
  const float gl = far_back<kPassRbf>(a, e, c, 0, 0, -2, c.z >= 2);
  const float gd = c.y + 2 < rows ? a.F[e + 2 * cols] : 0.f;
  const float gr = c.z + 2 < cols ? a.F[e + 2] : 0.f;
  const float u2 = vu ? gu : 0.f, d2 = vd ? gd : 0.f, l2 = vl ? gl : 0.f, r2 = vr ? gr : 0.f;
  const float step = __fsub_rn(cand, old);
  float alpha = 1.0f;
  for (int it = 0; it < 10; it++) {
    float trial = __fadd_rn(old, __fmul_rn(alpha, step));
    if (trial < lo) trial = lo;
    if (trial > hi) trial = hi;
    const float eps = a.eps;
    bool bad = false;
    // neighbour (i-1, j): its neighbours are (i-2, j), (i, j) = trial, (i-1, j-1), (i-1, j+1)
    if (vu && cls4_eps(n, u2, trial, v[0][0], v[0][2], eps) != 0) bad = true;
    if (!bad && vd && cls4_eps(s, trial, d2, v[2][0], v[2][2], eps) != 0) bad = true;
    if (!bad && vl && cls4_eps(w, v[0][0], v[2][0], l2, trial, eps) != 0) bad = true;
    if (!bad && vr && cls4_eps(ea, v[0][2], v[2][2], trial, r2, eps) != 0) bad = true;
    if (!bad && cls4_eps(trial, n, s, w, ea, eps) != 3) bad = true;
    if (!bad) { ok = true; return trial; }
    alpha = __fmul_rn(alpha, 0.5f);
  }
  return old;
}

// values around e in 3D: index (dx+2, dy+2, dz+2) over a 5x5x5 window, filled lazily
struct Win3 {
  float v[5][5][5];
  unsigned char have[5][5][5];
  C3 c;  // coordinates of the center
};

template <int PASS>
__device__ __forceinline__ float w3getp(const PostArgs &a, long long e, Win3 &W, int dx, int dy, int dz,
                                        float center) {
  if (dx == 0 && dy == 0 && dz == 0) return center;
  unsigned char &h = W.have[dx + 2][dy + 2][dz + 2];
  if (!h) {
    W.v[dx + 2][dy + 2][dz + 2] = valo<PASS>(a, e, W.c, dx, dy, dz);
    h = 1;
  }
  return W.v[dx + 2][dy + 2][dz + 2];
}

template <int PASS>
__device__ __forceinline__ int cls6_at(const PostArgs &a, long long e, Win3 &W, int dx, int dy, int dz,
                                       float center) {
  return classify6(w3getp<PASS>(a, e, W, dx, dy, dz, center), w3getp<PASS>(a, e, W, dx - 1, dy, dz, center),
                   w3getp<PASS>(a, e, W, dx + 1, dy, dz, center), w3getp<PASS>(a, e, W, dx, dy - 1, dz, center),
                   w3getp<PASS>(a, e, W, dx, dy + 1, dz, center), w3getp<PASS>(a, e, W, dx, dy, dz - 1, center),
                   w3getp<PASS>(a, e, W, dx, dy, dz + 1, center));
}

// the center is a saddle and every regular neighbour stays regular
template <int PASS>
__device__ bool valid3(const PostArgs &a, long long e, const C3 &c, Win3 &W, float trial) {
  if (cls6_at<PASS>(a, e, W, 0, 0, 0, trial) != 3) return false;
  const long long pl = a.g.plane, d3 = a.g.d3;
  if (c.x - 1 >= 1 && ty(a, e - pl) == 0 && cls6_at<PASS>(a, e, W, -1, 0, 0, trial) != 0) return false;
  if (c.x + 1 < a.g.d1 - 1 && ty(a, e + pl) == 0 && cls6_at<PASS>(a, e, W, 1, 0, 0, trial) != 0) return false;
  if (c.y - 1 >= 1 && ty(a, e - d3) == 0 && cls6_at<PASS>(a, e, W, 0, -1, 0, trial) != 0) return false;
  if (c.y + 1 < a.g.d2 - 1 && ty(a, e + d3) == 0 && cls6_at<PASS>(a, e, W, 0, 1, 0, trial) != 0) return false;
  if (c.z - 1 >= 1 && ty(a, e - 1) == 0 && cls6_at<PASS>(a, e, W, 0, 0, -1, trial) != 0) return false;
  if (c.z + 1 < a.g.d3 - 1 && ty(a, e + 1) == 0 && cls6_at<PASS>(a, e, W, 0, 0, 1, trial) != 0) return false;
  return true;
}

// 3D RBF (example/test_cuda_topology_3d.cu:317-434).  Every value the
// validation can read is loaded once into registers (compile-time indices):
// the 3x3x3 box around e and the points two steps out along each axis, the
// latter loaded wherever they exist and used only where the serial code reads
// them (the neighbour on that side is interior and regular).  The candidate
// tests come first and every value load after them, so an item waits for a
// few loads in a row, not one per point.  A trial changes only the centre
// value.
__device__ float rbf3(const PostArgs &a, long long e, const C3 &c, float o, bool &ok) {
  ok = false;
  const float old = a.F[e];
  float v[27];   // box value at (dx, dy, dz): v[(dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)]
  // which earlier box points (i < 13) are candidates, then every value: the
  // result of an earlier candidate, else F (loads issued together)
  bool cb[13];
#pragma unroll
  for (int i = 0; i < 13; i++) {
    const int dx = i / 9 - 1, dy = (i / 3) % 3 - 1, dz = i % 3 - 1;
    cb[i] = is_cand_known<kPassRbf>(a, e + dx * a.g.plane + dy * a.g.d3 + dz, interior_off(a, c, dx, dy, dz));
  }
#pragma unroll
  for (int i = 0; i < 27; i++) {
    const int dx = i / 9 - 1, dy = (i / 3) % 3 - 1, dz = i % 3 - 1;
    const long long q = e + dx * a.g.plane + dy * a.g.d3 + dz;
    v[i] = (i == 13) ? old : (i < 13 && cb[i]) ? __uint_as_float((unsigned)ld_rlx(&a.S[q])) : a.F[q];
  }
  // neighbours whose classification the validation checks, and their far sides
  const long long pl = a.g.plane, d3 = a.g.d3;
  const bool cxm = c.x - 1 >= 1 && ty(a, e - pl) == 0, cxp = c.x + 1 < a.g.d1 - 1 && ty(a, e + pl) == 0;
  const bool cym = c.y - 1 >= 1 && ty(a, e - d3) == 0, cyp = c.y + 1 < a.g.d2 - 1 && ty(a, e + d3) == 0;
  const bool czm = c.z - 1 >= 1 && ty(a, e - 1) == 0, czp = c.z + 1 < a.g.d3 - 1 && ty(a, e + 1) == 0;
  // the far sides, loaded wherever they exist (not only after the type
  // tests) so that their loads overlap; used as the serial pass reads them
  const float gxm = far_back<kPassRbf>(a, e, c, -2, 0, 0, c.x >= 2);
  const float gym = far_back<kPassRbf>(a, e, c, 0, -2, 0, c.y >= 2);
  const float gzm = far_back<kPassRbf>(a, e, c, 0, 0, -2, c.z >= 2);
  const float gxp = c.x + 2 < a.g.d1 ? a.F[e + 2 * pl] : 0.f;
  const float gyp = c.y + 2 < a.g.d2 ? a.F[e + 2 * d3] : 0.f;
  const float gzp = c.z + 2 < a.g.d3 ? a.F[e + 2] : 0.f;
  const float fxm = cxm ? gxm : 0.f, fym = cym ? gym : 0.f, fzm = czm ? gzm : 0.f;
  const float fxp = cxp ? gxp : 0.f, fyp = cyp ? gyp : 0.f, fzp = czp ? gzp : 0.f;
  const unsigned lk = box_locks<3>(a, e, c);
  double num = 0.0, den = 0.0;
#pragma unroll
  for (int i = 0; i < 27; i++) {
    double ww = c_w3[i];
    if ((lk >> i) & 1u) ww = __dmul_rn(ww, 0.4);
    num = __dadd_rn(num, __dmul_rn(ww, (double)v[i]));
    den = __dadd_rn(den, ww);
  }
  if (!(den > 0.0)) return old;
  const float d = __fmul_rn(a.eb, 0.999f);
  const float lo = __fsub_rn(o, d), hi = __fadd_rn(o, d);
  float cand = __double2float_rn(__ddiv_rn(num, den));
  if (cand < lo) cand = lo;
  if (cand > hi) cand = hi;
#define V3(dx, dy, dz) v[((dx) + 1) * 9 + ((dy) + 1) * 3 + ((dz) + 1)]
  const float step = __fsub_rn(cand, old);
  float alpha = 1.0f;
  for (int it = 0; it < 10; it++) {
    float tr = __fadd_rn(old, __fmul_rn(alpha, step));
    if (tr < lo) tr = lo;
    if (tr > hi) tr = hi;
    // classify6(centre, x-, x+, y-, y+, z-, z+) of the centre and of each checked neighbour
    bool good = classify6(tr, V3(-1, 0, 0), V3(1, 0, 0), V3(0, -1, 0), V3(0, 1, 0), V3(0, 0, -1), V3(0, 0, 1)) == 3;
    if (good && cxm)
      good = classify6(V3(-1, 0, 0), fxm, tr, V3(-1, -1, 0), V3(-1, 1, 0), V3(-1, 0, -1), V3(-1, 0, 1)) == 0;
    if (good && cxp)
      good = classify6(V3(1, 0, 0), tr, fxp, V3(1, -1, 0), V3(1, 1, 0), V3(1, 0, -1), V3(1, 0, 1)) == 0;
    if (good && cym)
      good = classify6(V3(0, -1, 0), V3(-1, -1, 0), V3(1, -1, 0), fym, tr, V3(0, -1, -1), V3(0, -1, 1)) == 0;
    if (good && cyp)
      good = classify6(V3(0, 1, 0), V3(-1, 1, 0), V3(1, 1, 0), tr, fyp, V3(0, 1, -1), V3(0, 1, 1)) == 0;
    if (good && czm)
      good = classify6(V3(0, 0, -1), V3(-1, 0, -1), V3(1, 0, -1), V3(0, -1, -1), V3(0, 1, -1), fzm, tr) == 0;
    if (good && czp)
      good = classify6(V3(0, 0, 1), V3(-1, 0, 1), V3(1, 0, 1), V3(0, -1, 1), V3(0, 1, 1), tr, fzp) == 0;
    if (good) { ok = true; return tr; }
    alpha = __fmul_rn(alpha, 0.5f);
  }
#undef V3
  return old;
}

// 3D axis-pattern saddle stencil (example/test_cuda_topology_3d.cu:187-314)
__device__ float axis3(const PostArgs &a, long long e, const C3 &c, float o, bool &ok) {
  ok = false;
  Win3 W;
  W.c = c;
  for (int i = 0; i < 125; i++) (&W.have[0][0][0])[i] = 0;
  const float old = a.F[e];
  if (cls6_at<kPassAxis>(a, e, W, 0, 0, 0, old) == 3) return old;
  const float d = __fmul_rn(a.eb, 0.999f);
  const float lo = __fsub_rn(o, d), hi = __fadd_rn(o, d);
  const float nb[6] = {w3getp<kPassAxis>(a, e, W, -1, 0, 0, old), w3getp<kPassAxis>(a, e, W, 1, 0, 0, old),
                       w3getp<kPassAxis>(a, e, W, 0, -1, 0, old), w3getp<kPassAxis>(a, e, W, 0, 1, 0, old),
                       w3getp<kPassAxis>(a, e, W, 0, 0, -1, old), w3getp<kPassAxis>(a, e, W, 0, 0, 1, old)};
  for (int pat = 1; pat <= 6; pat++) {
    float hthr = -1e30f, lthr = 1e30f;
    for (int ax = 0; ax < 3; ax++) {
      const float pmax = fmaxf(nb[2 * ax], nb[2 * ax + 1]);
      const float pmin = fminf(nb[2 * ax], nb[2 * ax + 1]);
      if ((pat >> ax) & 1) { if (pmax > hthr) hthr = pmax; }
      else { if (pmin < lthr) lthr = pmin; }
    }
    if (hthr >= lthr) continue;
    float target = __fmul_rn(0.5f, __fadd_rn(hthr, lthr));
    float nudge = __fmul_rn(__fsub_rn(lthr, hthr), 0.01f);
    if (nudge < FLT_EPSILON) nudge = FLT_EPSILON;
    if (target <= hthr) target = __fadd_rn(hthr, nudge);
    if (target >= lthr) target = __fsub_rn(lthr, nudge);
    if (target <= hthr || target >= lthr) continue;
    if (target > hi || target < lo) continue;
    if (valid3<kPassAxis>(a, e, c, W, target)) { ok = true; return target; }
  }
  return old;
}

// ----------------------------------------------------------------------------
// candidate lists
// ----------------------------------------------------------------------------

// Interior extrema (X) and interior saddles (Z) in raster order plus the
// interior-extremum bitmap Eb, in one pass over the types: persistent
// CTAs take tiles of kListTile points in order (32 consecutive points per
// thread), publish their counts and find their list offsets by decoupled
// look-back (extrema in the byte word, saddles in the count word), then write
// their entries through shared memory so each tile's slice of X and Z is
// stored contiguously (X staged from the front of one buffer, Z from its back:
// a point is in at most one list).  The last tile writes the totals to
// tot[0] = (extrema << 32) | saddles.  The raw decoded value of every list
// entry (Ox / Oz at its point) goes to OX / OZ beside it, for each list whose
// source is given (none is needed when the passes read raw values from the
// field itself).
constexpr int kListPer = 32;
constexpr int kListTile = kPostThreads * kListPer;

__global__ void __launch_bounds__(kPostThreads)
list_build_kernel(const unsigned char *__restrict__ T, Geom g, long long n, TileDesc *desc, unsigned *tile_ctr,
                  int *err, unsigned *X, unsigned *Z, unsigned char *Eb,
                  unsigned long long *tot, const float *__restrict__ Ox, const float *__restrict__ Oz,
                  float *OX, float *OZ, unsigned *XP) {
  __shared__ unsigned s_w1[kWarps], s_w2[kWarps];
  __shared__ unsigned s_buf[kListTile];
  __shared__ long long s_tile;
  __shared__ unsigned long long s_xb, s_zb;
  const long long ntiles = (n + kListTile - 1) / kListTile;
  while (true) {
    if (threadIdx.x == 0) s_tile = (long long)atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const long long tile = s_tile;
    if (tile >= ntiles) break;
    const long long i0 = tile * kListTile + (long long)threadIdx.x * kListPer;
    unsigned em = 0, sm = 0, im = 0;
    if (i0 < n) {
      long long r, x, y, z;
      if (g.nd == 2) { x = 0; y = fdivmod(i0, g.d3, g.m_d3, r); z = r; }
      else { x = fdivmod(i0, g.plane, g.m_plane, r); y = fdivmod(r, g.d3, g.m_d3, z); }
      if (z + kListPer - 1 < g.d3 && i0 + kListPer <= n) {
        // the 32 points share one row: interior columns 1 .. d3-2
        const bool row_in = y >= 1 && y <= g.d2 - 2 && (g.nd == 2 || (x >= 1 && x <= g.d1 - 2));
        if (row_in) {
          const long long lo = 1 - z, hi = g.d3 - 2 - z;   // interior offsets u in [lo, hi]
          const int ulo = lo > 0 ? (int)lo : 0, uhi = hi < kListPer - 1 ? (int)hi : kListPer - 1;
          if (ulo <= uhi) im = (uhi == 31 ? 0xffffffffu : ((2u << uhi) - 1u)) & ~((1u << ulo) - 1u);
        }
      } else {
        for (int u = 0; u < kListPer && i0 + u < n; u++) {
          bool in = y >= 1 && y <= g.d2 - 2 && z >= 1 && z <= g.d3 - 2;
          if (g.nd == 3) in = in && x >= 1 && x <= g.d1 - 2;
          if (in) im |= 1u << u;
          z++;
          while (z >= g.d3) { z -= g.d3; y++; if (y >= g.d2) { y -= g.d2; x++; } }
        }
      }
      if (im) {
        const bool vec = i0 + kListPer <= n && ((reinterpret_cast<uintptr_t>(T + i0) & 15) == 0);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          unsigned long long w0 = 0, w1 = 0;
          if (vec) {
            const uint4 v = __ldg(reinterpret_cast<const uint4 *>(T + i0) + h);
            w0 = ((unsigned long long)v.y << 32) | v.x;
            w1 = ((unsigned long long)v.w << 32) | v.z;
          } else {
            for (int u = 0; u < 8; u++) {
              if (i0 + 16 * h + u < n) w0 |= (unsigned long long)T[i0 + 16 * h + u] << (8 * u);
              if (i0 + 16 * h + 8 + u < n) w1 |= (unsigned long long)T[i0 + 16 * h + 8 + u] << (8 * u);
            }
          }
#pragma unroll
          for (int u = 0; u < 16; u++) {
            const unsigned t = (unsigned)((u < 8 ? w0 : w1) >> (8 * (u & 7))) & 3u;
            const unsigned bit = 1u << (16 * h + u);
            if (im & bit) {
              if (t == 1u || t == 2u) em |= bit;
              if (t == 3u) sm |= bit;
            }
          }
        }
      }
      // 4 bitmap bytes of this thread's 32 points (i0 is a multiple of 32)
      if (i0 + kListPer <= n) {
        reinterpret_cast<unsigned *>(Eb)[i0 >> 5] = em;
      } else {
        for (int k = 0; k < 4 && i0 + 8 * k < n; k++) Eb[(i0 >> 3) + k] = (unsigned char)(em >> (8 * k));
      }
    }
    unsigned te, ts;
    const unsigned eo = cta_excl_scan_post((unsigned)__popc(em), s_w1, &te);
    const unsigned so = cta_excl_scan_post((unsigned)__popc(sm), s_w2, &ts);
    if (threadIdx.x == 0) publish_aggregate(desc, tile, te, ts);
    {
      unsigned xe = eo, xs = so;
      unsigned mm = em;
      while (mm) { const int u = __ffs(mm) - 1; mm &= mm - 1; s_buf[xe++] = (unsigned)(i0 + u); }
      mm = sm;
      while (mm) { const int u = __ffs(mm) - 1; mm &= mm - 1; s_buf[kListTile - 1 - xs++] = (unsigned)(i0 + u); }
    }
    const Prefix pf = lookback_cta<kWarps>(desc, tile, te, ts, err);
    if (threadIdx.x == 0) {
      s_xb = pf.bytes;
      s_zb = pf.cnt;
      if (tile == ntiles - 1) *tot = ((pf.bytes + te) << 32) | (pf.cnt + ts);
    }
    __syncthreads();
    const unsigned long long xb = s_xb, zb = s_zb;
    // list position of the first extremum of this thread's bitmap word
    if (i0 < n) XP[i0 >> 5] = (unsigned)(xb + eo);
    // entries four at a time per thread: the raw-value gathers of a batch
    // are in flight together
    for (unsigned k0 = threadIdx.x; k0 < te; k0 += 4 * kPostThreads) {
      unsigned q[4];
      float v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const unsigned k = k0 + u * kPostThreads;
        q[u] = k < te ? s_buf[k] : 0u;
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (Ox && k0 + u * kPostThreads < te) v[u] = Ox[q[u]];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const unsigned k = k0 + u * kPostThreads;
        if (k < te) {
          // a list position past n means corrupt tile offsets: recorded, not written
          if (xb + k < (unsigned long long)n) {
            X[xb + k] = q[u];
            if (Ox) OX[xb + k] = v[u];
          } else {
            atomicExch(err, kErrMalformed);
          }
        }
      }
    }
    for (unsigned k0 = threadIdx.x; k0 < ts; k0 += 4 * kPostThreads) {
      unsigned q[4];
      float v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const unsigned k = k0 + u * kPostThreads;
        q[u] = k < ts ? s_buf[kListTile - 1 - k] : 0u;
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (Oz && k0 + u * kPostThreads < ts) v[u] = Oz[q[u]];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const unsigned k = k0 + u * kPostThreads;
        if (k < ts) {
          if (zb + k < (unsigned long long)n) {
            Z[zb + k] = q[u];
            if (Oz) OZ[zb + k] = v[u];
          } else {
            atomicExch(err, kErrMalformed);
          }
        }
      }
    }
    __syncthreads();
  }
}

// lost saddles (RBF candidates): saddles of the original field that F no
// longer classifies as saddles (example/test_cuda_topology.cu:244-254)
__global__ void fn_detect_kernel(PostArgs a, const unsigned *__restrict__ Z, unsigned long long nz,
                                 unsigned *__restrict__ R, unsigned *__restrict__ Y, unsigned *y_count) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool lost = false;
  long long q = 0;
  if (i < nz) {
    q = (long long)Z[i];
    lost = classify_F(a, q) != 3;
  }
  const unsigned m = __ballot_sync(0xffffffffu, lost);
  unsigned base = 0;
  const int lane = threadIdx.x & 31;
  if (lane == 0 && m) base = atomicAdd(y_count, (unsigned)__popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (lost) {
    Y[base + __popc(m & ((1u << lane) - 1u))] = (unsigned)i;
    atomicOr(&R[q >> 5], 1u << (q & 31));
  }
}

// Outcome of one item of a pass.
enum { kItemDone = 0, kItemDeferred = 1, kItemNeedsEnforce = 2 };

__device__ __forceinline__ float stencil_nd(const PostArgs &a, const Face &f, float cur, int t, int s, float o,
                                            int nd) {
  return nd == 2 ? stencil2(a, f, cur, t, s, o) : stencil3(a, f, t, s, o);
}

// The stencil pass fused with enforcement (a.NI set), item idx at point e.
// The candidates split into the connected components of face adjacency, and
// each pass reads, besides unchanged points, only the candidates of the
// item's own component.  So a candidate with no candidate neighbour (three in
// four on smooth fields) runs its enforcement right after its stencil, on the
// same neighbour values, and stores only the final value (nothing reads its
// result words).  The items of larger components run the stencil as usual
// (result words, deferral) and report kItemNeedsEnforce; the enforcement pass
// runs over them alone.
template <int PASS, int ND>
__device__ __forceinline__ int face_item_run(const PostArgs &a, unsigned idx, FaceItem &it) {
  if (!face_item_ready(a, it)) return kItemDeferred;
  const long long e = it.e;
  float r;
  int st = kItemDone;
  if (PASS == kPassStencil) {
    r = stencil_nd(a, it.f, it.cur, it.t, it.s, it.o, ND);
    if (a.NI) {
      if (it.iso) {
        a.F[e] = enforce<ND>(a, it.f, r, it.t, it.o);
        return kItemDone;
      }
      if (a.RAW) a.RAW[idx] = it.o;   // F[e] holds the stencil result from here on
      st = kItemNeedsEnforce;
    }
  } else {
    r = enforce<ND>(a, it.f, it.cur, it.t, it.o);
  }
  // in place: every reader of e's pre-pass value has finished (they are the
  // earlier candidates e waited for); later readers take e's result from S
  // at e's list position (dense, one coalesced word per item)
  a.F[e] = r;
  st_rlx(&a.S[idx], ((unsigned long long)a.gen << 32) | __float_as_uint(r));
  return st;
}

// One item of the RBF or axis-pattern pass (list index idx): its result goes
// to F and to S at its point, or it is deferred while an earlier candidate it
// reads is not final.
template <int PASS, int ND>
__device__ __forceinline__ int pass_item(const PostArgs &a, const unsigned *__restrict__ list, unsigned idx,
                                         int polls) {
  const long long e = (long long)list[idx];
  bool ok = false;
  const C3 c = coords(a.g, e);
  if (!deps_ready<PASS, ND>(a, e, c, polls)) return kItemDeferred;
  const float o = a.OL ? a.OL[idx] : a.F[e];
  const float r = PASS == kPassRbf ? ((ND == 2) ? rbf2(a, e, c, o, ok) : rbf3(a, e, c, o, ok)) : axis3(a, e, c, o, ok);
  if (ok) atomicAdd(a.restored, 1u);
  // in place: every reader of e's pre-pass value has finished (they are the
  // earlier candidates e waited for); later readers take e's result from S
  a.F[e] = r;
  st_rlx(&a.S[e], ((unsigned long long)a.gen << 32) | __float_as_uint(r));
  return kItemDone;
}

// An item whose earlier candidate is handled by the same CTA at the same
// time (the previous point of a row, or of the previous row) would be
// deferred to the next round; the CTA instead retries its pending items a
// few times, a block barrier apart, so that chains inside the CTA resolve in
// this round.  Every thread of the CTA must call it.  Returns true while the
// item is still pending.  In the fused stencil pass, the items left for the
// enforcement pass are marked in the a.NI bitmap here (one atomic per warp
// when the warp's items share a bitmap word, as in a round over the whole
// list).
constexpr int kLocalRetries = 5;

template <int PASS, int ND>
__device__ __forceinline__ bool pass_item_local(const PostArgs &a, const unsigned *__restrict__ list, unsigned idx,
                                                bool valid, int polls = 0) {
  // RBF and axis-pattern items are long and uneven: a block barrier would make
  // every thread wait for the slowest, so they wait for missing results on
  // their own (bounded, polls) or retry in rounds
  if (PASS != kPassStencil && PASS != kPassEnforce)
    return valid && pass_item<PASS, ND>(a, list, idx, polls) == kItemDeferred;
  bool pending = valid, need = false;
  FaceItem item;
  if (valid) face_item_load<PASS, ND>(a, list, idx, item);
  for (int it = 0; it < kLocalRetries; it++) {
    if (pending) {
      const int st = face_item_run<PASS, ND>(a, idx, item);
      pending = st == kItemDeferred;
      need = need || st == kItemNeedsEnforce;
    }
    if (!__syncthreads_or(pending)) break;
  }
  if (PASS == kPassStencil && a.NI) {
    const unsigned m = __ballot_sync(0xffffffffu, need);
    if (m) {
      const int lane = threadIdx.x & 31;
      const int first = __ffs(m) - 1;
      const unsigned wi = idx >> 5;
      const unsigned w_first = __shfl_sync(0xffffffffu, wi, first);
      const unsigned bit = need ? 1u << (idx & 31) : 0u;
      if (__all_sync(0xffffffffu, !need || wi == w_first)) {
        const unsigned bits = __reduce_or_sync(0xffffffffu, bit);
        if (lane == first) atomicOr(&a.NI[w_first], bits);
      } else if (need) {
        atomicOr(&a.NI[wi], bit);
      }
    }
  }
  return pending;
}

// One round of a pass over a worklist of list indices (identity when W is
// null).  Items whose earlier candidates are not final yet go to Wn.
// eight CTAs per SM (32 registers): the round is latency-bound, more warps
// hide more of it
template <int PASS, int ND>
__global__ void __launch_bounds__(kPostThreads, 8)
pass_round_kernel(PostArgs a, const unsigned *__restrict__ list, const unsigned *__restrict__ W,
                  unsigned nw, unsigned *__restrict__ Wn, unsigned *wn_count) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned idx = 0;
  if (i < nw) idx = W ? W[i] : i;
  const bool defer = pass_item_local<PASS, ND>(a, list, idx, i < nw);
  const unsigned m = __ballot_sync(0xffffffffu, defer);
  const int lane = threadIdx.x & 31;
  unsigned base = 0;
  if (lane == 0 && m) base = atomicAdd(wn_count, (unsigned)__popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (defer) Wn[base + __popc(m & ((1u << lane) - 1u))] = idx;
}


// Round 0 of the enforcement pass that follows the fused stencil pass: the
// items are the set bits of the bitmap NI over list positions.  Each CTA
// takes kSparseWords bitmap words (a window of the list in raster order),
// gathers their set positions in shared memory in order and runs them as a
// round does, so that neighbouring items still meet in one CTA and resolve
// by its local retries.  Deferred items go to Wn.
constexpr int kSparseWords = 24;
static_assert(kSparseWords * 32 % kPostThreads == 0 && kSparseWords <= 32, "window of whole thread strides");

template <int ND>
__global__ void __launch_bounds__(kPostThreads, 8)
enforce_sparse_kernel(PostArgs a, const unsigned *__restrict__ list, const unsigned *__restrict__ NI,
                      unsigned nwords, unsigned *__restrict__ Wn, unsigned *wn_count) {
  __shared__ unsigned s_idx[kSparseWords * 32];
  __shared__ unsigned s_word[kSparseWords], s_off[kSparseWords];
  __shared__ unsigned s_total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned w0 = blockIdx.x * kSparseWords;
  if (warp == 0) {
    const unsigned wi = w0 + lane;
    const unsigned bits = (lane < kSparseWords && wi < nwords) ? NI[wi] : 0u;
    const unsigned c = __popc(bits);
    unsigned incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane < kSparseWords) {
      s_word[lane] = bits;
      s_off[lane] = incl - c;
    }
    if (lane == 31) s_total = incl;
  }
  __syncthreads();
  // every thread expands bit positions threadIdx.x + 256 j of the window, in
  // order: position p goes to the slot of its word plus the set bits before it
#pragma unroll
  for (int j = 0; j < kSparseWords * 32 / kPostThreads; j++) {
    const unsigned pbit = (unsigned)threadIdx.x + (unsigned)(j * kPostThreads);
    const unsigned wd = s_word[pbit >> 5], b = pbit & 31u;
    if ((wd >> b) & 1u) s_idx[s_off[pbit >> 5] + (unsigned)__popc(wd & ((1u << b) - 1u))] = w0 * 32u + pbit;
  }
  __syncthreads();
  const unsigned total = s_total;
  for (unsigned base = 0; base < total; base += kPostThreads) {
    const unsigned i = base + threadIdx.x;
    const bool valid = i < total;
    const unsigned idx = valid ? s_idx[i] : 0u;
    const bool defer = pass_item_local<kPassEnforce, ND>(a, list, idx, valid);
    const unsigned m = __ballot_sync(0xffffffffu, defer);
    unsigned wb = 0;
    if (lane == 0 && m) wb = atomicAdd(wn_count, (unsigned)__popc(m));
    wb = __shfl_sync(0xffffffffu, wb, 0);
    if (defer) Wn[wb + __popc(m & ((1u << lane) - 1u))] = idx;
  }
}

// A round over a worklist whose length is on the device (*nw_dev), in a
// grid-stride loop over a grid of any size (no barrier inside).
template <int PASS, int ND>
__global__ void __launch_bounds__(kPostThreads)
pass_round_dev_kernel(PostArgs a, const unsigned *__restrict__ list, const unsigned *__restrict__ W,
                      const unsigned *nw_dev, unsigned *__restrict__ Wn, unsigned *wn_count) {
  const unsigned nw = *nw_dev;
  const int lane = threadIdx.x & 31;
  const unsigned stride = gridDim.x * blockDim.x;
  // every item of the round in flight at once: an item may wait for the
  // earlier ones it reads, which are being computed beside it
  const int polls = nw <= stride ? kDepPolls : 0;
  for (unsigned base = blockIdx.x * blockDim.x; base < nw; base += stride) {
    const unsigned i = base + threadIdx.x;
    unsigned idx = 0;
    if (i < nw) idx = W[i];
    const bool defer = pass_item_local<PASS, ND>(a, list, idx, i < nw, polls);
    const unsigned m = __ballot_sync(0xffffffffu, defer);
    unsigned wb = 0;
    if (lane == 0 && m) wb = atomicAdd(wn_count, (unsigned)__popc(m));
    wb = __shfl_sync(0xffffffffu, wb, 0);
    if (defer) Wn[wb + __popc(m & ((1u << lane) - 1u))] = idx;
  }
}

// Grid-wide barrier of a cooperative launch (every CTA resident): one
// arrival counter and a generation word.  The last CTA to arrive resets the
// counter and advances the generation; the others wait for the generation to
// change.  The wait is bounded: after kBarSpinLimit polls the CTA records
// kErrWaitTimeout and leaves the barrier (the pass then reports an error).
constexpr int kBarSpinLimit = 1 << 22;

__device__ __forceinline__ unsigned ld_acq_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_rel_u32(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err, int spin_limit = 0) {
  const int limit = spin_limit > 0 ? spin_limit : kBarSpinLimit;
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    const unsigned g = ld_acq_u32(bar + 1);
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      st_rel_u32(bar + 1, g + 1);
    } else {
      // exponential back-off keeps the pollers of all CTAs from crowding the
      // generation word's L2 line while the last arrivals are still counting
      int spins = 0;
      unsigned nap = 64;
      while (ld_acq_u32(bar + 1) == g) {
        if (++spins > limit) {
          ok = 0;
          atomicExch(err, kErrWaitTimeout);
          break;
        }
        __nanosleep(nap);
        if (nap < 1024) nap <<= 1;
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// The rounds of a pass after round 1 (or all of them) in one cooperative
// launch: rounds are separated by grid barriers instead of host round trips.  The worklist starts as W_start with
// *nstart_dev items (the deferred items of a round-0 launch) or, when W_start
// is null, as sel (list indices; null = the whole list) with the pass's total
// item count.  The total is *total_dev when that is not null, else total.
// Worklists and counters written during the launch are read through L2
// (__ldcg), since other SMs wrote them.  Every CTA takes the same branch at
// every barrier: the counts it reads are final after the barrier.
// status: 0 done, 1 round limit, 2 no progress.
constexpr int kCoopRoundLimit = 100000;

// At least two CTAs per SM (128 registers): the long RBF items need the
// resident threads more than registers.
template <int PASS, int ND>
__global__ void __launch_bounds__(kPostThreads, 2)
pass_coop_kernel(PostArgs a, const unsigned *__restrict__ list, const unsigned *sel, unsigned total,
                 const unsigned *total_dev, const unsigned *W_start, const unsigned *nstart_dev, unsigned *Wx,
                 unsigned *Wy, unsigned *cnts, unsigned *bar, unsigned long long *status) {
  const unsigned tot = total_dev ? __ldcg(total_dev) : total;
  const unsigned *W = W_start ? W_start : sel;
  unsigned nw = W_start ? __ldcg(nstart_dev) : tot;
  const bool after_round0 = W_start != nullptr;
  int b = 0;
  const unsigned stride = gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (int round = 0; nw > 0; round++) {
    if (round >= kCoopRoundLimit) {
      if (blockIdx.x == 0 && threadIdx.x == 0) status[0] = 1;
      return;
    }
    unsigned *Wn = b ? Wy : Wx;
    // three counters in rotation: round r counts into cnts[r % 3].  The one
    // the next round uses was last read before the barrier that ended round
    // r - 1, which every CTA has passed once any CTA is in round r, so
    // clearing it now cannot hide a count from a slower CTA.
    unsigned *cnt = cnts + (round % 3);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(cnts + ((round + 1) % 3), 0u);
    for (unsigned base = blockIdx.x * blockDim.x; base < nw; base += stride) {
      const unsigned i = base + threadIdx.x;
      unsigned idx = 0;
      if (i < nw) idx = W ? __ldcg(W + i) : i;
      const bool defer = pass_item_local<PASS, ND>(a, list, idx, i < nw, nw <= stride ? kDepPolls : 0);
      const unsigned m = __ballot_sync(0xffffffffu, defer);
      unsigned wb = 0;
      if (lane == 0 && m) wb = atomicAdd(cnt, (unsigned)__popc(m));
      wb = __shfl_sync(0xffffffffu, wb, 0);
      if (defer) Wn[wb + __popc(m & ((1u << lane) - 1u))] = idx;
    }
    if (!grid_barrier(bar, a.err, a.spin_limit)) return;
    const unsigned next = __ldcg(cnt);
    if ((round > 0 || after_round0) && next >= nw) {
      if (blockIdx.x == 0 && threadIdx.x == 0) status[0] = 2;
      return;
    }
    W = Wn;
    nw = next;
    b ^= 1;
  }
  (void)tot;
}

__global__ void types_from_int_kernel(const int *__restrict__ fn, unsigned char *__restrict__ T, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) T[i] = (unsigned char)(fn[i] & 3);
}

static bool g_weights_ready[64];
static std::mutex g_weights_mu;

// once per device; contexts on several host threads may get here together
static cudaError_t upload_weights(int dev) {
  std::lock_guard<std::mutex> lk(g_weights_mu);
  if (dev >= 0 && dev < 64 && g_weights_ready[dev]) return cudaSuccess;
  // Gaussian weights in double with the reference formula
  // (example/test_cuda_topology.cu:259-265, example/test_cuda_topology_3d.cu:360-367)
  double s2 = 0.8 * 0.8;
  double w2[9], w3[27];
  for (int a = -1; a <= 1; a++)
    for (int b = -1; b <= 1; b++) w2[(a + 1) * 3 + (b + 1)] = exp(-((double)a * a + b * b) / (2.0 * s2));
  for (int a = -1; a <= 1; a++)
    for (int b = -1; b <= 1; b++)
      for (int c = -1; c <= 1; c++)
        w3[(a + 1) * 9 + (b + 1) * 3 + (c + 1)] = exp(-(double)(a * a + b * b + c * c) / (2.0 * s2));
  cudaError_t e = cudaMemcpyToSymbol(c_w2, w2, sizeof(w2));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_w3, w3, sizeof(w3));
  if (e == cudaSuccess && dev >= 0 && dev < 64) g_weights_ready[dev] = true;
  return e;
}

size_t post_scratch_bytes(unsigned long long n) {
  const unsigned long long ntiles = (n + kPostTile - 1) / kPostTile;
  const unsigned long long words = (n + 31) / 32;
  // T, descriptors, RBF + extrema bitmaps + extremum word positions, lists X
  // and Z, worklists (2), Y, raw values of X and Z
  return a256(n) + a256((ntiles + 1) * sizeof(TileDesc)) + 3 * a256(words * 4 + 4) + 7 * a256(n * 4) + 8192;
}


// generation counter of the result words (never reused while the buffer lives)
static unsigned next_gen(szp_b200_ctx *ctx) { return ++ctx->post_gen; }

// persistent result-word buffer of the workspace, zeroed when (re)allocated
unsigned long long *post_words(szp_b200_ctx *ctx, unsigned long long n) {
  if (ctx->post_S && ctx->post_S_cap >= n) return ctx->post_S;
  if (ctx->post_S) cudaFree(ctx->post_S);
  ctx->post_S = nullptr;
  ctx->post_S_cap = 0;
  if (cudaMalloc(&ctx->post_S, n * 8) != cudaSuccess) {
    cudaGetLastError();
    ctx->post_S = nullptr;
    set_error("device allocation of %llu result words failed", n);
    return nullptr;
  }
  if (cudaMemsetAsync(ctx->post_S, 0, n * 8, ctx->stream) != cudaSuccess) return nullptr;
  ctx->post_S_cap = n;
  ctx->post_gen = 0;
  return ctx->post_S;
}

// Grid of the cooperative tail of pass PASS on this workspace's device (all
// CTAs resident), or 0 when the workspace runs its tails as ordinary
// launches: no cooperative launch on the device, or a workspace whose stream
// shares the GPU with others (server workers), where a cooperative launch
// can only start once all of its CTAs fit beside the other streams' kernels.
template <int PASS, int ND>
static int coop_grid(szp_b200_ctx *ctx) {
  static int grid_for_dev[64];
  const int dev = ctx->device;
  if (ctx->coop_off || dev < 0 || dev >= 64) return 0;
  if (grid_for_dev[dev] == 0) {
    int coop = 0, nb = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pass_coop_kernel<PASS, ND>, kPostThreads, 0) !=
            cudaSuccess ||
        nb <= 0) {
      cudaGetLastError();
      grid_for_dev[dev] = -1;
    } else {
      grid_for_dev[dev] = nb * ctx->sm_count;
    }
  }
  return grid_for_dev[dev] > 0 ? grid_for_dev[dev] : 0;
}

// Rounds over deferred items as ordinary launches, kBurstRounds of them
// between host checks of the remaining count: W holds the items on entry
// (their count in word 7), W and Wo alternate.  Every round completes at
// least the earliest pending item, so a burst that completes none reports an
// error.
constexpr int kBurstRounds = 4;
constexpr int kRoundLimit = 100000;

template <int PASS, int ND>
static int finish_rounds(szp_b200_ctx *ctx, PostArgs &a, const unsigned *list, unsigned *W, unsigned *Wo) {
  cudaStream_t s = ctx->stream;
  unsigned *c[3] = {reinterpret_cast<unsigned *>(ctx->d_words + 7), reinterpret_cast<unsigned *>(ctx->d_words + 11),
                    reinterpret_cast<unsigned *>(ctx->d_words + 12)};
  unsigned *h_left = reinterpret_cast<unsigned *>(ctx->h_words + 15);
  int ci = 0;
  unsigned prev = 0xffffffffu;
  for (int r = 0; r < kRoundLimit; r += kBurstRounds) {
    for (int k = 0; k < kBurstRounds; k++) {
      unsigned *cn = c[(ci + 1) % 3];
      if (cuda_fail(cudaMemsetAsync(cn, 0, 4, s), "memset")) return -1;
      pass_round_dev_kernel<PASS, ND><<<ctx->sm_count * 4, kPostThreads, 0, s>>>(a, list, W, c[ci], Wo, cn);
      std::swap(W, Wo);
      ci = (ci + 1) % 3;
    }
    ctx->launches += kBurstRounds;
    if (cuda_fail(cudaGetLastError(), "pass round") ||
        cuda_fail(cudaMemcpyAsync(h_left, c[ci], 4, cudaMemcpyDeviceToHost, s), "D2H") ||
        cuda_fail(cudaStreamSynchronize(s), "pass round"))
      return -1;
    const unsigned left = *h_left;
    if (left == 0) return 0;
    if (left >= prev) { set_error("post-processing pass made no progress"); return -1; }
    prev = left;
  }
  set_error("post-processing pass did not converge");
  return -1;
}

// Runs one pass: round 0 as one launch over all of its items -- list
// positions 0 .. count-1, or sel[0 .. *count_dev) (count known only on the
// device), or the set bits of the bitmap ni_bits of ni_words words (the
// enforcement after the fused stencil) -- then the rounds over the deferred
// items: in one cooperative launch that reads its counts on the device (after
// one more ordinary round when round 0 ran over a list), or as bursts of
// ordinary launches (finish_rounds).
template <int PASS, int ND>
static int run_pass(szp_b200_ctx *ctx, PostArgs &a, const unsigned *list, const unsigned *sel, unsigned count,
                    const unsigned *count_dev, unsigned *W0, unsigned *W1, const unsigned *ni_bits = nullptr,
                    unsigned ni_words = 0) {
  if (ni_bits ? ni_words == 0 : (!count_dev && count == 0)) return 0;
  const int grid = coop_grid<PASS, ND>(ctx);
  cudaStream_t s = ctx->stream;
  // words 7 (round-0 count) and 10..13: three round counters, the barrier
  // counter and generation, the length of the round-1 worklist
  unsigned *n0 = reinterpret_cast<unsigned *>(ctx->d_words + 7);
  unsigned *cnts = reinterpret_cast<unsigned *>(ctx->d_words + 10);
  unsigned *bar = cnts + 3;
  unsigned *n1 = cnts + 6;
  unsigned long long *status = ctx->d_words + 9;
  if (cuda_fail(cudaMemsetAsync(n0, 0, 4, s), "memset")) return -1;
  if (ni_bits)
    enforce_sparse_kernel<ND><<<(ni_words + kSparseWords - 1) / kSparseWords, kPostThreads, 0, s>>>(
        a, list, ni_bits, ni_words, W0, n0);
  else if (count_dev)
    pass_round_dev_kernel<PASS, ND><<<ctx->sm_count * 2, kPostThreads, 0, s>>>(a, list, sel, count_dev, W0, n0);
  else
    pass_round_kernel<PASS, ND><<<(count + kPostThreads - 1) / kPostThreads, kPostThreads, 0, s>>>(
        a, list, sel, count, W0, n0);
  ctx->launches += 1;
  if (cuda_fail(cudaGetLastError(), "pass round")) return -1;
  if (!grid) return finish_rounds<PASS, ND>(ctx, a, list, W0, W1);
  if (cuda_fail(cudaMemsetAsync(cnts, 0, 32, s), "memset")) return -1;
  const unsigned *W_start = W0, *nstart = n0;
  unsigned *Wx = W1, *Wy = W0;
  if (!count_dev) {
    // one more ordinary round (the round-0 remainder can still be large)
    pass_round_dev_kernel<PASS, ND><<<ctx->sm_count * 8, kPostThreads, 0, s>>>(a, list, W0, n0, W1, n1);
    ctx->launches += 1;
    if (cuda_fail(cudaGetLastError(), "pass round")) return -1;
    W_start = W1;
    nstart = n1;
    Wx = W0;
    Wy = W1;
  }
  const unsigned zero = 0;
  const unsigned *no_total = nullptr;
  void *args[] = {(void *)&a,       (void *)&list,   (void *)&sel, (void *)&zero, (void *)&no_total,
                  (void *)&W_start, (void *)&nstart, (void *)&Wx,  (void *)&Wy,   (void *)&cnts,
                  (void *)&bar,     (void *)&status};
  if (cuda_fail(cudaLaunchCooperativeKernel((const void *)pass_coop_kernel<PASS, ND>, dim3(grid), dim3(kPostThreads),
                                            args, 0, s),
                "cooperative pass launch"))
    return -1;
  ctx->launches += 1;
  return 0;
}

template <int ND>
static int run_all_passes(szp_b200_ctx *ctx, PostArgs &a, unsigned *X, unsigned nx, unsigned *Z, unsigned nz,
                          unsigned *Y, unsigned *W0, unsigned *W1, unsigned *R,
                          const unsigned *Eb, float *OX, const float *OZ,
                          int axis_stencil, bool raw_in_F) {
  cudaStream_t s = ctx->stream;
  const long long n = a.n;
  // raw_in_F: OX / OZ were not gathered; OX keeps the raw values of the
  // items the fused stencil leaves for enforcement
  a.OL = raw_in_F ? nullptr : OX;
  a.RAW = nullptr;
  a.X = Eb;
  if (a.sp && a.n_sp > 0) {
    // stencil fused with enforcement; the items next to another candidate
    // are marked in a bitmap over list positions (in R, unused until the
    // lost-saddle detection) and only they run the enforcement pass
    const unsigned ni_words = (nx + 31) / 32;
    unsigned *NIb = R;
    if (cuda_fail(cudaMemsetAsync(NIb, 0, (size_t)ni_words * 4, s), "memset")) return -1;
    a.gen = next_gen(ctx);
    a.NI = NIb;
    a.RAW = raw_in_F ? OX : nullptr;
    if (run_pass<kPassStencil, ND>(ctx, a, X, nullptr, nx, nullptr, W0, W1)) return -1;
    a.NI = nullptr;
    a.RAW = nullptr;
    a.OL = OX;   // raw values of the remaining items (gathered, or stashed by the stencil)
    tl_mark(ctx, "post_stencil");
    a.gen = next_gen(ctx);
    if (run_pass<kPassEnforce, ND>(ctx, a, X, nullptr, 0, nullptr, W0, W1, NIb, ni_words)) return -1;
  } else {
    a.gen = next_gen(ctx);
    if (run_pass<kPassEnforce, ND>(ctx, a, X, nullptr, nx, nullptr, W0, W1)) return -1;
  }
  tl_mark(ctx, "post_enforce");
  // the lost saddles (from F after enforcement); RBF reads the locks from the
  // extremum bitmap (box_locks)
  const long long words = (n + 31) / 32;
  if (cuda_fail(cudaMemsetAsync(R, 0, words * 4, s), "memset")) return -1;
  unsigned *ycnt = reinterpret_cast<unsigned *>(ctx->d_words + 8);
  if (cuda_fail(cudaMemsetAsync(ycnt, 0, 4, s), "memset")) return -1;
  a.R = R;
  if (nz) fn_detect_kernel<<<(nz + 255) / 256, 256, 0, s>>>(a, Z, nz, R, Y, ycnt);
  ctx->launches += nz ? 1 : 0;
  if (cuda_fail(cudaGetLastError(), "fn detect")) return -1;
  tl_mark(ctx, "post_fn_locks");
  // RBF runs over Z restricted to the lost saddles (Y holds indices into Z);
  // their number stays on the device.  Saddles keep their raw values until
  // RBF itself writes them.
  a.OL = raw_in_F ? nullptr : OZ;
  a.gen = next_gen(ctx);
  if (nz && run_pass<kPassRbf, ND>(ctx, a, Z, Y, 0, ycnt, W0, W1)) return -1;
  tl_mark(ctx, "post_rbf");
  if (axis_stencil && ND == 3 && nz) {
    a.OL = OZ;   // gathered in every mode: RBF has changed some saddles
    a.gen = next_gen(ctx);
    if (run_pass<kPassAxis, ND>(ctx, a, Z, nullptr, nz, nullptr, W0, W1)) return -1;
    tl_mark(ctx, "post_axis");
  }
  return 0;
}

int postprocess_with(szp_b200_ctx *ctx, float *d_data, const float *d_orig, unsigned char *d_T,
                     unsigned long long *d_S, TileDesc *desc, const int *d_sp,
                     unsigned long long n_sp, const Geom &g, float eb, int axis_stencil, int *restored_out) {
  const long long n = g.d1 * g.d2 * g.d3;
  if (g.d2 < 3 || g.d3 < 3 || (g.nd == 3 && g.d1 < 3)) { if (restored_out) *restored_out = 0; return 0; }
  if (n >= (1ll << 32)) { set_error("post-processing supports fields of fewer than 2^32 points"); return -1; }
  int dev = 0;
  cudaGetDevice(&dev);
  if (cuda_fail(upload_weights(dev), "weights")) return -1;
  cudaStream_t s = ctx->stream;
  Arena &A = ctx->scratch;
  unsigned *X = A.take<unsigned>(n), *Z = A.take<unsigned>(n), *Y = A.take<unsigned>(n);
  unsigned *W0 = A.take<unsigned>(n), *W1 = A.take<unsigned>(n);
  unsigned *R = A.take<unsigned>((n + 31) / 32);
  unsigned *Eb = A.take<unsigned>((n + 31) / 32 + 1);
  unsigned *XP = A.take<unsigned>((n + 31) / 32 + 1);
  float *OX = A.take<float>(n), *OZ = A.take<float>(n);
  if (!X || !Z || !Y || !W0 || !W1 || !R || !Eb || !XP || !OX || !OZ) {
    set_error("scratch arena too small for post-processing");
    return -1;
  }
  unsigned long long *w = ctx->d_words;  // [9] pass status, [10] round counters
  if (cuda_fail(cudaMemsetAsync(w, 0, 96, s), "memset")) return -1;
  {
    // the words past the last written byte of the bitmap must read as zero
    const long long words = (n + 31) / 32;
    if (cuda_fail(cudaMemsetAsync(Eb + words - 1, 0, 8, s), "memset")) return -1;
  }
  unsigned *tile_ctr = reinterpret_cast<unsigned *>(w + 3);
  unsigned long long *d_tot = w + 2;
  const long long ltiles = (n + kListTile - 1) / kListTile;
  if (cuda_fail(cudaMemsetAsync(desc, 0, (ltiles + 1) * sizeof(TileDesc), s), "memset")) return -1;
  // post-processing of the decoded field itself: each item reads its raw
  // value from F before it writes (no gathered raw lists), except the
  // axis-pattern pass, which runs after RBF has changed saddles
  const bool raw_in_F = d_orig == d_data;
  const bool axis_raw = axis_stencil && g.nd == 3;
  {
    const unsigned grid = (unsigned)std::min<long long>(ltiles, (long long)ctx->sm_count * 6);
    list_build_kernel<<<grid, kPostThreads, 0, s>>>(d_T, g, n, desc, tile_ctr, reinterpret_cast<int *>(w + 4), X,
                                                    Z, reinterpret_cast<unsigned char *>(Eb), d_tot,
                                                    raw_in_F ? nullptr : d_orig,
                                                    raw_in_F && !axis_raw ? nullptr : d_orig, OX, OZ, XP);
  }
  ctx->launches += 1;
  unsigned long long tot = 0;
  if (cuda_fail(cudaGetLastError(), "lists") ||
      cuda_fail(cudaMemcpyAsync(&tot, d_tot, 8, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "lists"))
    return -1;
  const unsigned nx = (unsigned)(tot >> 32), nz = (unsigned)(tot & 0xffffffffull);
  tl_mark(ctx, "post_lists");
  PostArgs a{};
  a.F = d_data;
  a.T = d_T;
  a.sp = d_sp;
  a.n_sp = d_sp ? n_sp : 0;
  a.g = g;
  a.n = n;
  a.eb = eb;
  a.eps = fmaxf(1e-6f, 0.1f * eb);
  a.S = d_S;
  a.XP = XP;
  a.err = reinterpret_cast<int *>(w + 4);
  a.restored = reinterpret_cast<unsigned *>(w + 5);
  const int rc = (g.nd == 2)
                     ? run_all_passes<2>(ctx, a, X, nx, Z, nz, Y, W0, W1, R, Eb, OX, OZ, axis_stencil,
                                         raw_in_F)
                     : run_all_passes<3>(ctx, a, X, nx, Z, nz, Y, W0, W1, R, Eb, OX, OZ, axis_stencil,
                                         raw_in_F);
  if (rc) return -1;
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words, w, 96, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "postprocess"))
    return -1;
  const int err = (int)(ctx->h_words[4] & 0xffffffffu);
  if (err) { set_error("post-processing status %d", err); return -1; }
  if (ctx->h_words[9] == 1) { set_error("post-processing pass did not converge"); return -1; }
  if (ctx->h_words[9] == 2) { set_error("post-processing pass made no progress"); return -1; }
  if (restored_out) *restored_out = (int)(ctx->h_words[5] & 0xffffffffu);
  return 0;
}

// Bounded-wait check of the grid barrier: the last CTA of the launch leaves
// without arriving, so the others must give up after spin_limit polls and
// report kErrWaitTimeout (no CTA waits on anything that can hang).
__global__ void barrier_timeout_probe_kernel(unsigned *bar, int *err, int spin_limit) {
  if (blockIdx.x == gridDim.x - 1) return;
  grid_barrier(bar, err, spin_limit);
}

int selftest_grid_barrier(int spin_limit, int *status, float *ms) {
  unsigned *d = nullptr;
  if (cuda_fail(cudaMalloc(&d, 64), "cudaMalloc")) return -1;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = -1;
  if (!cuda_fail(cudaMemset(d, 0, 64), "memset") && !cuda_fail(cudaEventCreate(&e0), "event") &&
      !cuda_fail(cudaEventCreate(&e1), "event")) {
    cudaEventRecord(e0, 0);
    barrier_timeout_probe_kernel<<<2, 64>>>(d, reinterpret_cast<int *>(d + 4), spin_limit);
    cudaEventRecord(e1, 0);
    int h = 0;
    if (!cuda_fail(cudaGetLastError(), "probe launch") &&
        !cuda_fail(cudaMemcpy(&h, d + 4, 4, cudaMemcpyDeviceToHost), "D2H")) {
      cudaEventElapsedTime(ms, e0, e1);
      *status = h;
      rc = 0;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d);
  return rc;
}

int postprocess(szp_b200_ctx *ctx, float *d_data, const float *d_orig,
                const unsigned char *d_types_u8, const int *d_types_i, const int *d_sp,
                unsigned long long n_sp, const Geom &g, float eb, int axis_stencil,
                int *restored_out) {
  const long long n = g.d1 * g.d2 * g.d3;
  Arena &A = ctx->scratch;
  unsigned long long *S = post_words(ctx, (unsigned long long)n);
  unsigned char *T = A.take<unsigned char>(n);
  const unsigned long long ntiles = (n + kPostTile - 1) / kPostTile;
  TileDesc *desc = A.take<TileDesc>(ntiles + 1);
  if (!S || !T || !desc) { set_error("scratch arena too small for post-processing"); return -1; }
  cudaStream_t s = ctx->stream;
  if (d_types_i) {
    types_from_int_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_types_i, T, n);
    ctx->launches += 1;
  } else if (cuda_fail(cudaMemcpyAsync(T, d_types_u8, n, cudaMemcpyDeviceToDevice, s), "copy types")) {
    return -1;
  }
  return postprocess_with(ctx, d_data, d_orig, T, S, desc, d_sp, n_sp, g, eb, axis_stencil, restored_out);
}

}  // namespace tsz
