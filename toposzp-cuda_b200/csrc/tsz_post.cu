// Post-processing of a decoded field with the exact serial-raster semantics of
// the reference drivers (example/test_cuda_topology.cu:117-326, :493-531 and
// example/test_cuda_topology_3d.cu:75-434, :600-631).
//
// Each reference pass visits points in raster order and updates them in
// place, so a point sees the FINAL values of earlier points and the
// PRE-PASS values of later points.  Here one kernel per pass reproduces that:
//   * F holds the field before the pass and is not written during the pass;
//   * a candidate's result goes to S[e] = (generation << 32) | float bits;
//   * reading neighbour q: if q is an earlier candidate of this pass, wait for
//     S[q] to carry this pass's generation and use it; otherwise read F[q];
//   * tiles of 2048 points are claimed in raster order through an atomic
//     counter, so every awaited point belongs to a CTA that is already
//     running, and waits are bounded (kErrWaitTimeout).
// A scatter kernel then copies the pass results into F.  Floating-point
// expressions use explicit round-to-nearest intrinsics so that no multiply-add
// is contracted (the reference host code is compiled without contraction).
#include <cfloat>

#include "tsz_lookback.cuh"
#include <algorithm>
#include <vector>

#include "tsz_ops.h"

namespace tsz {

enum { kPassStencil = 0, kPassEnforce = 1, kPassRbf = 2, kPassAxis = 3 };
constexpr int kPostThreads = 256;
constexpr int kPostPer = 8;
constexpr int kPostTile = kPostThreads * kPostPer;
constexpr unsigned char kCandFlag = 0x80;

__constant__ double c_w2[9];
__constant__ double c_w3[27];

struct PostArgs {
  float *F;
  const float *O;
  unsigned char *T;             // types in bits 0..1, candidate flag in bit 7
  const int *sp;
  unsigned long long n_sp;
  Geom g;
  long long n;
  float eb;
  float eps;
  unsigned gen;
  unsigned long long *S;
  TileDesc *desc;
  unsigned *tile_ctr;
  int *err;
  unsigned *restored;
};

__device__ __forceinline__ unsigned long long ld_rlx(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
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
__device__ __forceinline__ bool interior(const Geom &g, const C3 &c) {
  if (c.y < 1 || c.y > g.d2 - 2 || c.z < 1 || c.z > g.d3 - 2) return false;
  if (g.nd == 3 && (c.x < 1 || c.x > g.d1 - 2)) return false;
  return true;
}
__device__ __forceinline__ bool interior_at(const Geom &g, long long q) { return interior(g, coords(g, q)); }

__device__ __forceinline__ float wait_result(const PostArgs &a, long long q) {
  unsigned long long v = ld_rlx(&a.S[q]);
  int spins = 0;
  while ((unsigned)(v >> 32) != a.gen) {
    if (++spins > kSpinLimit) { atomicExch(a.err, kErrWaitTimeout); return a.F[q]; }
    __nanosleep(spins < 32 ? 20 : 200);
    v = ld_rlx(&a.S[q]);
  }
  return __uint_as_float((unsigned)v);
}

// ----------------------------------------------------------------------------
// candidate predicates (evaluated on F, which is stable during a pass)
// ----------------------------------------------------------------------------
__device__ __forceinline__ int classify_F(const PostArgs &a, long long q) {
  const float *F = a.F;
  if (a.g.nd == 2)
    return classify4(F[q], F[q - a.g.d3], F[q + a.g.d3], F[q - 1], F[q + 1]);
  return classify6(F[q], F[q - a.g.plane], F[q + a.g.plane], F[q - a.g.d3], F[q + a.g.d3], F[q - 1],
                   F[q + 1]);
}

template <int PASS>
__device__ __forceinline__ bool is_cand(const PostArgs &a, long long q) {
  const int t = ty(a, q);
  if (PASS == kPassStencil || PASS == kPassEnforce) {
    if (t != 1 && t != 2) return false;
    return interior_at(a.g, q);
  }
  if (t != 3) return false;
  if (!interior_at(a.g, q)) return false;
  // the axis-pattern pass re-tests every saddle against the current values
  // inside the update itself (example/test_cuda_topology_3d.cu:203-206)
  if (PASS == kPassAxis) return true;
  return classify_F(a, q) != 3;
}

// value of neighbour q as the serial pass would see it from point e (q != e)
template <int PASS>
__device__ __forceinline__ float val(const PostArgs &a, long long e, long long q) {
  if (q < e && is_cand<PASS>(a, q)) return wait_result(a, q);
  return a.F[q];
}

// ----------------------------------------------------------------------------
// per-point updates
// ----------------------------------------------------------------------------
__device__ __forceinline__ float clampf(float v, float lo, float hi) {
  if (v > hi) v = hi;
  if (v < lo) v = lo;
  return v;
}

// 2D stencil (example/test_cuda_topology.cu:118-165)
__device__ float stencil2(const PostArgs &a, long long e, int t, int s) {
  const long long cols = a.g.d3;
  const float o = a.O[e];
  const float hi = __fadd_rn(o, a.eb), lo = __fsub_rn(o, a.eb);
  float m = a.F[e];
  const long long nb[4] = {e - cols, e + cols, e - 1, e + 1};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const float v = val<kPassStencil>(a, e, nb[k]);
    if (t == 1 ? (v > m) : (v < m)) m = v;
  }
  float target;
  if (t == 1) target = __fmul_rn(m, __fadd_rn(1.0f, __fmul_rn((float)s, FLT_EPSILON)));
  else if (s == 0) target = __fmul_rn(m, __fsub_rn(1.0f, FLT_EPSILON));
  else target = __fmul_rn(m, __fsub_rn(1.0f, __fmul_rn(__fdiv_rn(1.0f, (float)s), FLT_EPSILON)));
  return clampf(target, lo, hi);
}

// 3D stencil (example/test_cuda_topology_3d.cu:77-128)
__device__ float stencil3(const PostArgs &a, long long e, int t, int s) {
  const float o = a.O[e];
  const float d = __fmul_rn(a.eb, 0.999f);
  const float hi = __fadd_rn(o, d), lo = __fsub_rn(o, d);
  const long long pl = a.g.plane, d3 = a.g.d3;
  const float xm = val<kPassStencil>(a, e, e - pl), xp = a.F[e + pl];
  const float ym = val<kPassStencil>(a, e, e - d3), yp = a.F[e + d3];
  const float zm = val<kPassStencil>(a, e, e - 1), zp = a.F[e + 1];
  // later neighbours read through val too (candidates later than e use F)
  float target;
  if (t == 1) {
    const float m = fmaxf(fmaxf(xm, xp), fmaxf(fmaxf(ym, yp), fmaxf(zm, zp)));
    target = __fmul_rn(m, __fadd_rn(1.0f, __fmul_rn((float)s, FLT_EPSILON)));
  } else {
    const float m = fminf(fminf(xm, xp), fminf(fminf(ym, yp), fminf(zm, zp)));
    target = (s == 0) ? __fmul_rn(m, __fsub_rn(1.0f, FLT_EPSILON))
                      : __fmul_rn(m, __fsub_rn(1.0f, __fmul_rn(__fdiv_rn(1.0f, (float)s), FLT_EPSILON)));
  }
  return clampf(target, lo, hi);
}

// enforcement (example/test_cuda_topology.cu:168-198, _3d.cu:131-167)
template <int ND>
__device__ float enforce(const PostArgs &a, long long e, int t) {
  const float o = a.O[e];
  const float d = __fmul_rn(a.eb, 0.999f);
  const float hi = __fadd_rn(o, d), lo = __fsub_rn(o, d);
  const float soft = __fmul_rn(0.25f, a.eps);
  const float cur = a.F[e];
  float m;
  if (ND == 2) {
    const long long cols = a.g.d3;
    const float n = val<kPassEnforce>(a, e, e - cols), s = a.F[e + cols];
    const float w = val<kPassEnforce>(a, e, e - 1), ea = a.F[e + 1];
    m = (t == 1) ? fmaxf(fmaxf(n, s), fmaxf(w, ea)) : fminf(fminf(n, s), fminf(w, ea));
  } else {
    const long long pl = a.g.plane, d3 = a.g.d3;
    const float xm = val<kPassEnforce>(a, e, e - pl), xp = a.F[e + pl];
    const float ym = val<kPassEnforce>(a, e, e - d3), yp = a.F[e + d3];
    const float zm = val<kPassEnforce>(a, e, e - 1), zp = a.F[e + 1];
    m = (t == 1) ? fmaxf(fmaxf(xm, xp), fmaxf(fmaxf(ym, yp), fmaxf(zm, zp)))
                 : fminf(fminf(xm, xp), fminf(fminf(ym, yp), fminf(zm, zp)));
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

// lock: point q (interior) has an interior extremum within Chebyshev distance 1
__device__ bool locked2(const PostArgs &a, long long q) {
  const C3 c = coords(a.g, q);
  if (c.y < 1 || c.y > a.g.d2 - 2 || c.z < 1 || c.z > a.g.d3 - 2) return false;
  for (int da = -1; da <= 1; da++)
    for (int db = -1; db <= 1; db++) {
      const long long ii = c.y + da, jj = c.z + db;
      if (ii < 1 || ii > a.g.d2 - 2 || jj < 1 || jj > a.g.d3 - 2) continue;
      const int t = ty(a, ii * a.g.d3 + jj);
      if (t == 1 || t == 2) return true;
    }
  return false;
}

__device__ bool locked3(const PostArgs &a, long long q) {
  const C3 c = coords(a.g, q);
  if (!interior(a.g, c)) return false;
  for (int da = -1; da <= 1; da++)
    for (int db = -1; db <= 1; db++)
      for (int dc = -1; dc <= 1; dc++) {
        const long long xx = c.x + da, yy = c.y + db, zz = c.z + dc;
        if (xx < 1 || xx > a.g.d1 - 2 || yy < 1 || yy > a.g.d2 - 2 || zz < 1 || zz > a.g.d3 - 2)
          continue;
        const int t = ty(a, xx * a.g.plane + yy * a.g.d3 + zz);
        if (t == 1 || t == 2) return true;
      }
  return false;
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
__device__ float rbf2(const PostArgs &a, long long e, const C3 &c, bool &ok) {
  const long long cols = a.g.d3;
  const long long rows = a.g.d2;
  ok = false;
  // 3x3 neighbourhood values as seen by the serial pass
  float v[3][3];
  for (int da = -1; da <= 1; da++)
    for (int db = -1; db <= 1; db++)
      v[da + 1][db + 1] = (da == 0 && db == 0) ? a.F[e] : val<kPassRbf>(a, e, e + da * cols + db);
  double num = 0.0, den = 0.0;
  for (int da = -1; da <= 1; da++)
    for (int db = -1; db <= 1; db++) {
      double ww = c_w2[(da + 1) * 3 + (db + 1)];
      if (locked2(a, e + da * cols + db)) ww = __dmul_rn(ww, 0.4);
      num = __dadd_rn(num, __dmul_rn(ww, (double)v[da + 1][db + 1]));
      den = __dadd_rn(den, ww);
    }
  const float old = a.F[e];
  if (!(den > 0.0)) return old;
  const float o = a.O[e];
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
  const float u2 = vu ? val<kPassRbf>(a, e, e - 2 * cols) : 0.f;
  const float d2 = vd ? val<kPassRbf>(a, e, e + 2 * cols) : 0.f;
  const float l2 = vl ? val<kPassRbf>(a, e, e - 2) : 0.f;
  const float r2 = vr ? val<kPassRbf>(a, e, e + 2) : 0.f;
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
};

__device__ __forceinline__ float w3get(const PostArgs &a, long long e, Win3 &W, int dx, int dy, int dz,
                                       float center) {
  if (dx == 0 && dy == 0 && dz == 0) return center;
  unsigned char &h = W.have[dx + 2][dy + 2][dz + 2];
  if (!h) {
    W.v[dx + 2][dy + 2][dz + 2] = val<kPassRbf>(a, e, e + dx * a.g.plane + dy * a.g.d3 + dz);
    h = 1;
  }
  return W.v[dx + 2][dy + 2][dz + 2];
}

template <int PASS>
__device__ __forceinline__ float w3getp(const PostArgs &a, long long e, Win3 &W, int dx, int dy, int dz,
                                        float center) {
  if (dx == 0 && dy == 0 && dz == 0) return center;
  unsigned char &h = W.have[dx + 2][dy + 2][dz + 2];
  if (!h) {
    W.v[dx + 2][dy + 2][dz + 2] = val<PASS>(a, e, e + dx * a.g.plane + dy * a.g.d3 + dz);
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

// 3D RBF (example/test_cuda_topology_3d.cu:317-434)
__device__ float rbf3(const PostArgs &a, long long e, const C3 &c, bool &ok) {
  ok = false;
  Win3 W;
  for (int i = 0; i < 125; i++) (&W.have[0][0][0])[i] = 0;
  const float old = a.F[e];
  double num = 0.0, den = 0.0;
  for (int da = -1; da <= 1; da++)
    for (int db = -1; db <= 1; db++)
      for (int dc = -1; dc <= 1; dc++) {
        double ww = c_w3[(da + 1) * 9 + (db + 1) * 3 + (dc + 1)];
        if (locked3(a, e + da * a.g.plane + db * a.g.d3 + dc)) ww = __dmul_rn(ww, 0.4);
        const float v = w3getp<kPassRbf>(a, e, W, da, db, dc, old);
        num = __dadd_rn(num, __dmul_rn(ww, (double)v));
        den = __dadd_rn(den, ww);
      }
  if (!(den > 0.0)) return old;
  const float o = a.O[e];
  const float d = __fmul_rn(a.eb, 0.999f);
  const float lo = __fsub_rn(o, d), hi = __fadd_rn(o, d);
  float cand = __double2float_rn(__ddiv_rn(num, den));
  if (cand < lo) cand = lo;
  if (cand > hi) cand = hi;
  const float step = __fsub_rn(cand, old);
  float alpha = 1.0f;
  for (int it = 0; it < 10; it++) {
    float trial = __fadd_rn(old, __fmul_rn(alpha, step));
    if (trial < lo) trial = lo;
    if (trial > hi) trial = hi;
    if (valid3<kPassRbf>(a, e, c, W, trial)) { ok = true; return trial; }
    alpha = __fmul_rn(alpha, 0.5f);
  }
  return old;
}

// 3D axis-pattern saddle stencil (example/test_cuda_topology_3d.cu:187-314)
__device__ float axis3(const PostArgs &a, long long e, const C3 &c, bool &ok) {
  ok = false;
  Win3 W;
  for (int i = 0; i < 125; i++) (&W.have[0][0][0])[i] = 0;
  const float old = a.F[e];
  if (cls6_at<kPassAxis>(a, e, W, 0, 0, 0, old) == 3) return old;
  const float o = a.O[e];
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
// pass kernel
// ----------------------------------------------------------------------------
template <int PASS, int ND>
__global__ void __launch_bounds__(kPostThreads)
post_pass_kernel(PostArgs a) {
  __shared__ long long s_tile;
  __shared__ unsigned s_w[kPostThreads / 32];
  __shared__ unsigned long long s_base;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long ntiles = (a.n + kPostTile - 1) / kPostTile;
  while (true) {
    if (threadIdx.x == 0) s_tile = (long long)atomicAdd(a.tile_ctr, 1u);
    __syncthreads();
    const long long tile = s_tile;
    if (tile >= ntiles) break;
    const long long t0 = tile * kPostTile;
    // candidates of this thread: elements t0 + threadIdx.x*8 + u (contiguous per thread)
    unsigned cmask = 0;
    for (int u = 0; u < kPostPer; u++) {
      const long long e = t0 + (long long)threadIdx.x * kPostPer + u;
      if (e < a.n && is_cand<PASS>(a, e)) cmask |= 1u << u;
    }
    unsigned long long rank0 = 0;
    if (PASS == kPassStencil) {
      const unsigned c = __popc(cmask);
      unsigned incl = c;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      if (lane == 31) s_w[warp] = incl;
      __syncthreads();
      unsigned wpre = 0, ttot = 0;
      for (int w = 0; w < kPostThreads / 32; w++) { if (w < warp) wpre += s_w[w]; ttot += s_w[w]; }
      if (warp == 0) {
        Prefix pf = lookback(a.desc, tile, 0, ttot, a.err);
        if (lane == 0) s_base = pf.cnt;
      }
      __syncthreads();
      rank0 = s_base + wpre + incl - c;
    }
    for (int u = 0; u < kPostPer; u++) {
      if (!(cmask & (1u << u))) continue;
      const long long e = t0 + (long long)threadIdx.x * kPostPer + u;
      const int t = ty(a, e);
      float r;
      bool ok = false;
      if (PASS == kPassStencil) {
        const int s = (rank0 < a.n_sp) ? a.sp[rank0] : 0;
        rank0++;
        r = (ND == 2) ? stencil2(a, e, t, s) : stencil3(a, e, t, s);
      } else if (PASS == kPassEnforce) {
        r = enforce<ND>(a, e, t);
      } else if (PASS == kPassRbf) {
        const C3 c = coords(a.g, e);
        r = (ND == 2) ? rbf2(a, e, c, ok) : rbf3(a, e, c, ok);
      } else {
        const C3 c = coords(a.g, e);
        r = axis3(a, e, c, ok);
      }
      if (ok) atomicAdd(a.restored, 1u);
      a.T[e] |= kCandFlag;
      st_rlx(&a.S[e], ((unsigned long long)a.gen << 32) | __float_as_uint(r));
    }
    __syncthreads();
  }
}

// copy pass results into F and clear the candidate flags
__global__ void post_scatter_kernel(float *__restrict__ F, unsigned char *__restrict__ T,
                                    const unsigned long long *__restrict__ S, long long n) {
  const long long i0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (i0 >= n) return;
  if (i0 + 4 <= n && ((reinterpret_cast<uintptr_t>(T + i0) & 3) == 0)) {
    uint32_t w = *reinterpret_cast<const uint32_t *>(T + i0);
    if (!(w & 0x80808080u)) return;
    for (int u = 0; u < 4; u++) {
      if ((w >> (8 * u)) & 0x80u) {
        F[i0 + u] = __uint_as_float((unsigned)S[i0 + u]);
        T[i0 + u] &= 0x7f;
      }
    }
    return;
  }
  for (long long i = i0; i < i0 + 4 && i < n; i++)
    if (T[i] & 0x80) { F[i] = __uint_as_float((unsigned)S[i]); T[i] &= 0x7f; }
}

__global__ void types_from_int_kernel(const int *__restrict__ fn, unsigned char *__restrict__ T, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) T[i] = (unsigned char)(fn[i] & 3);
}

template <int PASS, int ND>
static cudaError_t run_pass(szp_b200_ctx *ctx, PostArgs a, TileDesc *desc, long long ntiles) {
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  if ((e = cudaMemsetAsync(a.tile_ctr, 0, 4, s)) != cudaSuccess) return e;
  if (PASS == kPassStencil &&
      (e = cudaMemsetAsync(desc, 0, (ntiles + 1) * sizeof(TileDesc), s)) != cudaSuccess)
    return e;
  const int grid = (int)std::min<long long>(ntiles, (long long)ctx->sm_count * 8);
  post_pass_kernel<PASS, ND><<<grid, kPostThreads, 0, s>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const long long sg = (a.n + 4 * 256 - 1) / (4 * 256);
  post_scatter_kernel<<<(unsigned)sg, 256, 0, s>>>(a.F, a.T, a.S, a.n);
  ctx->launches += 2;
  return cudaGetLastError();
}

static bool g_weights_ready[64];

static cudaError_t upload_weights(int dev) {
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
  return a256(n) + a256((ntiles + 1) * sizeof(TileDesc)) + 4096;
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

int postprocess_with(szp_b200_ctx *ctx, float *d_data, const float *d_orig, unsigned char *d_T,
                     unsigned long long *d_S, TileDesc *desc, const int *d_sp,
                     unsigned long long n_sp, const Geom &g, float eb, int axis_stencil,
                     int *restored_out) {
  const long long n = g.d1 * g.d2 * g.d3;
  if (g.d2 < 3 || g.d3 < 3 || (g.nd == 3 && g.d1 < 3)) { if (restored_out) *restored_out = 0; return 0; }
  int dev = 0;
  cudaGetDevice(&dev);
  if (cuda_fail(upload_weights(dev), "weights")) return -1;
  cudaStream_t s = ctx->stream;
  unsigned long long *w = ctx->d_words;
  if (cuda_fail(cudaMemsetAsync(w, 0, 64, s), "memset")) return -1;
  PostArgs a{};
  a.F = d_data;
  a.O = d_orig;
  a.T = d_T;
  a.sp = d_sp;
  a.n_sp = d_sp ? n_sp : 0;
  a.g = g;
  a.n = n;
  a.eb = eb;
  a.eps = fmaxf(1e-6f, 0.1f * eb);
  a.S = d_S;
  a.desc = desc;
  a.tile_ctr = reinterpret_cast<unsigned *>(w + 3);
  a.err = reinterpret_cast<int *>(w + 4);
  a.restored = reinterpret_cast<unsigned *>(w + 5);
  const long long ntiles = (n + kPostTile - 1) / kPostTile;
  cudaError_t e = cudaSuccess;
  if (d_sp && n_sp > 0) {
    a.gen = next_gen(ctx);
    e = (g.nd == 2) ? run_pass<kPassStencil, 2>(ctx, a, desc, ntiles) : run_pass<kPassStencil, 3>(ctx, a, desc, ntiles);
    if (cuda_fail(e, "stencil pass")) return -1;
    tl_mark(ctx, "post_stencil");
  }
  a.gen = next_gen(ctx);
  e = (g.nd == 2) ? run_pass<kPassEnforce, 2>(ctx, a, desc, ntiles) : run_pass<kPassEnforce, 3>(ctx, a, desc, ntiles);
  if (cuda_fail(e, "enforcement pass")) return -1;
  tl_mark(ctx, "post_enforce");
  a.gen = next_gen(ctx);
  e = (g.nd == 2) ? run_pass<kPassRbf, 2>(ctx, a, desc, ntiles) : run_pass<kPassRbf, 3>(ctx, a, desc, ntiles);
  if (cuda_fail(e, "rbf pass")) return -1;
  tl_mark(ctx, "post_rbf");
  if (axis_stencil && g.nd == 3) {
    a.gen = next_gen(ctx);
    e = run_pass<kPassAxis, 3>(ctx, a, desc, ntiles);
    if (cuda_fail(e, "axis pass")) return -1;
    tl_mark(ctx, "post_axis");
  }
  if (cuda_fail(cudaMemcpyAsync(ctx->h_words, w, 64, cudaMemcpyDeviceToHost, s), "D2H") ||
      cuda_fail(cudaStreamSynchronize(s), "postprocess"))
    return -1;
  const int err = (int)(ctx->h_words[4] & 0xffffffffu);
  if (err) { set_error("post-processing status %d", err); return -1; }
  if (restored_out) *restored_out = (int)(ctx->h_words[5] & 0xffffffffu);
  return 0;
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
