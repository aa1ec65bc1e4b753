// CPU oracle for the restricted-Voronoi / tangent-plane CVT Lloyd step.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: the tests, the smoke
// check and the CPU-baseline leg of the benchmark call it.  The product
// library (gpu_cvt_b200/csrc) never links, loads or calls it.
//
// It restates, sequentially on the CPU, the algorithm of the reference's GPU
// stage kernels (Harper-Yan/GPU_CVT):
//   vertex normals ........ site_normals.cuh:19-41
//   tangent frame ......... site_normals.cuh:69-110 (uv_from_nearest_vertex_normal)
//   site KNN .............. bitonic-hubs-grid.cuh:862-995 (exact K+1 incl. self,
//                            ascending squared distance), site_knn.cuh:79-103
//                            (drop self, pad with last)
//   vertex KNN ............ near_project.cuh:54-92 (insertion top-K, ties keep the
//                            lower index, EXCLUDE_SELF quirk, frozen skip)
//   clip + centroid ....... 2dClip.cuh:11-135 (Sutherland-Hodgman, eps 1e-12,
//                            64-vertex cap, shoelace centroid, |A|<1e-18 -> mean,
//                            n<3 -> NaN)
//   closest point / project near_project.cuh:12-53, 149-189
//   freeze test ........... freezetest.cuh:155-212, 270-327, 451-466, 50-54
//   tiers ................. main.cu:18-150
//   Lloyd loop ............ main.cu:669-881
//   BVH + Hausdorff ....... evaluate.cuh:15-357
//   quality ............... evaluate.cuh:388-462
//   face extraction ....... near_project.cuh:201-352, buildmesh.cuh:11-21,97-109,
//                            170-201,225-241, main.cu:928-974
//
// Floating point.  Every FP32 expression is written with its rounding pinned:
// products and sums are separately rounded unless an explicit fmaf() appears
// (compile with -ffp-contract=off), divisions and square roots are IEEE.  The
// reference's rsqrtf() is restated as 1/sqrtf() (a <=1-ulp difference).  With
// that, a GPU kernel that follows the same operation sequence produces the
// same bits.  Profiles:
//   0 REF   FP32 everywhere, the reference's operation order.
//   1 MIXED FP32 state; the clip half-plane predicates / intersections and the
//           point-triangle barycentrics in FP64; Neumaier-compensated centroid
//           sums; a NaN centroid keeps the old site (scripts/testfreeze.py:410-417).
//   2 FP64  FP64 state and arithmetic throughout (the FP64 oracle).
//
// KNN ordering: lists are sorted by (squared distance, index), so exact
// distance ties are broken by the lower index (the reference's bitonic sort
// leaves tie order unspecified, bitonic-shared.cuh:12-81).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum { P_REF = 0, P_MIXED = 1, P_FP64 = 2 };

template <class T> struct V3 { T x, y, z; };
template <class T> struct V2 { T x, y; };

template <class T> inline T fmaT(T a, T b, T c) { return std::fma(a, b, c); }

template <class T> inline T dot3(V3<T> a, V3<T> b) {
  return fmaT(a.z, b.z, fmaT(a.y, b.y, a.x * b.x));
}
template <class T> inline V3<T> sub3(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> cross3(V3<T> a, V3<T> b) {
  return {fmaT(a.y, b.z, -(a.z * b.y)), fmaT(a.z, b.x, -(a.x * b.z)), fmaT(a.x, b.y, -(a.y * b.x))};
}
template <class T> inline V3<T> ld3(const T* p, long i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
template <class T> inline void st3(T* p, long i, V3<T> v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }
template <class T, class S> inline V3<T> cvt3(V3<S> a) { return {(T)a.x, (T)a.y, (T)a.z}; }

// squared distance in the order (x, y, z): fma(z,z, fma(y,y, x*x))
template <class T> inline T dist2(V3<T> p, V3<T> q) {
  T dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
  return fmaT(dz, dz, fmaT(dy, dy, dx * dx));
}

inline bool finite3f(float x, float y) { return std::isfinite(x) && std::isfinite(y); }

// ---------------------------------------------------------------------------
// KNN (exact, (d2, index) order)
// ---------------------------------------------------------------------------
template <class T> struct Cand { T d; uint32_t i; };
template <class T> inline bool cand_less(const Cand<T>& a, const Cand<T>& b) {
  return a.d < b.d || (a.d == b.d && a.i < b.i);
}

// bounded sorted list of the best kk candidates
template <class T> struct TopK {
  int kk, n = 0;
  Cand<T> c[64];
  explicit TopK(int k) : kk(k) {}
  inline bool full() const { return n == kk; }
  inline T worst() const { return n == kk ? c[kk - 1].d : std::numeric_limits<T>::infinity(); }
  inline void push(T d, uint32_t i) {
    Cand<T> x{d, i};
    if (n == kk && !cand_less(x, c[kk - 1])) return;
    int p = (n < kk) ? n++ : kk - 1;
    while (p > 0 && cand_less(x, c[p - 1])) { c[p] = c[p - 1]; --p; }
    c[p] = x;
  }
};

// Uniform grid over a point set, used to answer exact KNN queries quickly.
// The answer is identical to brute force (the search stops only once the
// k-th candidate is provably closer than every unvisited cell).
template <class T> struct PGrid {
  T lo[3], h;
  int dim[3];
  std::vector<int> start;
  std::vector<uint32_t> ids;
  const T* P = nullptr;
  long n = 0;
  void build(const T* pts, long np, double target_per_cell) {
    P = pts; n = np;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    long valid = 0;
    for (long i = 0; i < n; ++i) {
      double x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
      if (!(std::isfinite(x) && std::isfinite(y) && std::isfinite(z))) continue;
      ++valid;
      mn[0] = std::min(mn[0], x); mn[1] = std::min(mn[1], y); mn[2] = std::min(mn[2], z);
      mx[0] = std::max(mx[0], x); mx[1] = std::max(mx[1], y); mx[2] = std::max(mx[2], z);
    }
    if (valid == 0) { for (int a = 0; a < 3; ++a) { mn[a] = 0; mx[a] = 1; } }
    double ext = std::max({mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2], 1e-12});
    // cells ~ valid/target on a 2-manifold -> cell size from the bbox area
    double area = 2.0 * ((mx[0] - mn[0]) * (mx[1] - mn[1]) + (mx[1] - mn[1]) * (mx[2] - mn[2]) +
                         (mx[0] - mn[0]) * (mx[2] - mn[2])) + 1e-30;
    double hh = std::sqrt(area * target_per_cell / std::max<long>(valid, 1));
    hh = std::max(hh, ext / 1024.0);
    h = (T)hh;
    long total = 1;
    for (int a = 0; a < 3; ++a) {
      lo[a] = (T)(mn[a] - 1e-6 * ext);
      dim[a] = std::max(1, (int)std::ceil((mx[a] - mn[a] + 2e-6 * ext) / hh));
      total *= dim[a];
    }
    start.assign(total + 2, 0);
    std::vector<long> cell(n);
    for (long i = 0; i < n; ++i) { cell[i] = cell_of(pts + 3 * i); start[cell[i] + 1]++; }
    for (long c = 0; c <= total; ++c) start[c + 1] += start[c];
    ids.assign(n, 0);
    std::vector<int> cur(start.begin(), start.end());
    for (long i = 0; i < n; ++i) ids[cur[cell[i]]++] = (uint32_t)i;
  }
  long ncell() const { return (long)dim[0] * dim[1] * dim[2]; }
  int coord(T v, int a) const {
    double f = std::floor(((double)v - (double)lo[a]) / (double)h);
    if (!(f >= 0)) f = 0;  // also catches NaN
    if (f > dim[a] - 1) f = dim[a] - 1;
    return (int)f;
  }
  long cell_of(const T* p) const {
    if (!(std::isfinite((double)p[0]) && std::isfinite((double)p[1]) && std::isfinite((double)p[2])))
      return ncell();  // NaN bucket: never searched
    return ((long)coord(p[2], 2) * dim[1] + coord(p[1], 1)) * dim[0] + coord(p[0], 0);
  }
  // visit every point of the cells at Chebyshev ring r around (cx,cy,cz)
  template <class F> void ring(int cx, int cy, int cz, int r, F&& f) const {
    for (int z = cz - r; z <= cz + r; ++z) {
      if (z < 0 || z >= dim[2]) continue;
      for (int y = cy - r; y <= cy + r; ++y) {
        if (y < 0 || y >= dim[1]) continue;
        bool face = (std::abs(z - cz) == r) || (std::abs(y - cy) == r);
        for (int x = cx - r; x <= cx + r; x += (face || r == 0) ? 1 : 2 * r) {
          if (x < 0 || x >= dim[0]) continue;
          long c = ((long)z * dim[1] + y) * dim[0] + x;
          for (int k = start[c]; k < start[c + 1]; ++k) f(ids[k]);
        }
      }
    }
  }
  // lower bound on the distance from q to any cell outside ring r
  double margin(const T* q, int c[3], int r) const {
    double m = std::numeric_limits<double>::infinity();
    for (int a = 0; a < 3; ++a) {
      if (c[a] - r > 0) m = std::min(m, (double)q[a] - ((double)lo[a] + (double)(c[a] - r) * (double)h));
      if (c[a] + r < dim[a] - 1) m = std::min(m, ((double)lo[a] + (double)(c[a] + r + 1) * (double)h) - (double)q[a]);
    }
    return m;
  }
  template <class Accept>
  void knn(const T* q, TopK<T>& top, Accept&& accept) const {
    V3<T> qq{q[0], q[1], q[2]};
    if (!(std::isfinite((double)q[0]) && std::isfinite((double)q[1]) && std::isfinite((double)q[2]))) return;
    int c[3] = {coord(q[0], 0), coord(q[1], 1), coord(q[2], 2)};
    int rmax = std::max({dim[0], dim[1], dim[2]});
    for (int r = 0; r <= rmax; ++r) {
      ring(c[0], c[1], c[2], r, [&](uint32_t j) {
        if (!accept(j)) return;
        top.push(dist2(ld3(P, j), qq), j);
      });
      double m = margin(q, c, r) - 1e-3 * (double)h;
      if (m == std::numeric_limits<double>::infinity()) break;
      if (top.full() && m > 0 && (double)top.worst() < m * m) break;
    }
  }
};

}  // namespace

// ===========================================================================
// exported C ABI (all arrays are caller-owned host memory)
// ===========================================================================
extern "C" {

int oracle_version(void) { return 1; }

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// VF CSR in face order (main.cu:259-285).
void oracle_build_vf(int nV, int nF, const int* F, int* vf_off, int* vf_faces) {
  for (int v = 0; v <= nV; ++v) vf_off[v] = 0;
  for (int f = 0; f < nF; ++f)
    for (int k = 0; k < 3; ++k) vf_off[F[3 * f + k] + 1]++;
  for (int v = 0; v < nV; ++v) vf_off[v + 1] += vf_off[v];
  std::vector<int> cur(vf_off, vf_off + nV + 1);
  for (int f = 0; f < nF; ++f)
    for (int k = 0; k < 3; ++k) vf_faces[cur[F[3 * f + k]]++] = f;
}

// Area-weighted vertex normals (site_normals.cuh:19-41).  Face normals are
// summed per vertex in increasing face order; normalisation by 1/sqrtf.
void oracle_vertex_normals(const float* V, int nV, const int* F, int nF, float* N) {
  std::vector<int> off(nV + 1), fcs(3 * (size_t)nF);
  oracle_build_vf(nV, nF, F, off.data(), fcs.data());
  for (int v = 0; v < nV; ++v) {
    V3<float> acc{0.f, 0.f, 0.f};
    for (int k = off[v]; k < off[v + 1]; ++k) {
      int f = fcs[k];
      V3<float> a = ld3(V, F[3 * f]), b = ld3(V, F[3 * f + 1]), c = ld3(V, F[3 * f + 2]);
      V3<float> fn = cross3(sub3(b, a), sub3(c, a));
      acc = {acc.x + fn.x, acc.y + fn.y, acc.z + fn.z};
    }
    float l2 = dot3(acc, acc);
    if (l2 > 0.f) {
      float inv = 1.0f / std::sqrt(l2);
      acc = {acc.x * inv, acc.y * inv, acc.z * inv};
    }
    st3(N, v, acc);
  }
}

// Exact K nearest points (self included) for every point, brute force.
// Rows of frozen points are left untouched (bitonic-hubs-grid.cuh:891).
// Missing entries (n < kk) get index 0xFFFFFFFF and distance +inf.
void oracle_knn_points_bf(const float* P, int n, int kk, const unsigned char* frozen,
                          uint32_t* knn, float* dist) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    if (frozen && frozen[i]) continue;
    TopK<float> top(kk);
    V3<float> q = ld3(P, i);
    if (std::isfinite(q.x) && std::isfinite(q.y) && std::isfinite(q.z))
      for (int j = 0; j < n; ++j) {
        V3<float> p = ld3(P, j);
        float d = dist2(p, q);
        if (std::isnan(d)) continue;
        top.push(d, (uint32_t)j);
      }
    for (int t = 0; t < kk; ++t) {
      knn[(size_t)i * kk + t] = t < top.n ? top.c[t].i : 0xFFFFFFFFu;
      if (dist) dist[(size_t)i * kk + t] = t < top.n ? top.c[t].d : std::numeric_limits<float>::infinity();
    }
  }
}

// Same answer as oracle_knn_points_bf, through a uniform grid (for large n).
void oracle_knn_points_grid(const float* P, int n, int kk, const unsigned char* frozen,
                            uint32_t* knn, float* dist) {
  PGrid<float> g;
  g.build(P, n, 2.0 * kk);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    if (frozen && frozen[i]) continue;
    TopK<float> top(kk);
    g.knn(P + 3 * (size_t)i, top, [](uint32_t) { return true; });
    for (int t = 0; t < kk; ++t) {
      knn[(size_t)i * kk + t] = t < top.n ? top.c[t].i : 0xFFFFFFFFu;
      if (dist) dist[(size_t)i * kk + t] = t < top.n ? top.c[t].d : std::numeric_limits<float>::infinity();
    }
  }
}

// knn_drop_self_kernel (site_knn.cuh:79-103): keep the first K entries that are
// not i; none -> all i; fewer than K -> repeat the last kept entry.
void oracle_drop_self(const uint32_t* in, int n, int kin, int kout, const unsigned char* frozen,
                      uint32_t* out) {
  for (int i = 0; i < n; ++i) {
    if (frozen && frozen[i]) continue;
    int w = 0;
    const uint32_t* s = in + (size_t)i * kin;
    uint32_t* d = out + (size_t)i * kout;
    for (int t = 0; t < kin && w < kout; ++t) {
      if ((int)s[t] == i) continue;
      d[w++] = s[t];
    }
    if (w == 0) {
      for (int k = 0; k < kout; ++k) d[k] = (uint32_t)i;
    } else {
      uint32_t fill = d[w - 1];
      for (; w < kout; ++w) d[w] = fill;
    }
  }
}

// knn_vertices_bruteforce_k (near_project.cuh:54-92): the k nearest mesh
// vertices of each query; ties keep the lower vertex index; with
// exclude_self, vertex index == query index is skipped; frozen rows untouched.
void oracle_knn_vertices_bf(const float* V, int nV, const float* Q, int nQ, int k,
                            int exclude_self, const unsigned char* frozen, int* out) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int qi = 0; qi < nQ; ++qi) {
    if (frozen && frozen[qi]) continue;
    TopK<float> top(k);
    V3<float> q = ld3(Q, qi);
    for (int vi = 0; vi < nV; ++vi) {
      if (exclude_self && vi == qi) continue;
      float d = dist2(ld3(V, vi), q);
      if (std::isnan(d)) continue;
      top.push(d, (uint32_t)vi);
    }
    for (int t = 0; t < k; ++t) out[(size_t)qi * k + t] = t < top.n ? (int)top.c[t].i : -1;
  }
}

}  // extern "C"

// ===========================================================================
// geometry per profile
// ===========================================================================
namespace {

template <class T> struct Frame { V3<T> u, v; };

// uv_from_nearest_vertex_normal (site_normals.cuh:69-110)
template <class T> Frame<T> frame_from_normal(V3<T> n) {
  const T tiny = (T)1e-30;
  T inv = T(1) / std::sqrt(dot3(n, n) + tiny);
  n = {n.x * inv, n.y * inv, n.z * inv};
  V3<T> h = (std::fabs(n.z) > (T)0.9) ? V3<T>{1, 0, 0} : V3<T>{0, 0, 1};
  V3<T> u = cross3(h, n);
  T iu = T(1) / std::sqrt(dot3(u, u) + tiny);
  u = {u.x * iu, u.y * iu, u.z * iu};
  V3<T> v = cross3(n, u);
  T iv = T(1) / std::sqrt(dot3(v, v) + tiny);
  v = {v.x * iv, v.y * iv, v.z * iv};
  return {u, v};
}

constexpr int kMaxPoly = 64;

// Sutherland-Hodgman clip by a*x + b*y - c <= eps (2dClip.cuh:11-53).
// P: polygon coordinate type; Q: predicate / intersection arithmetic type.
template <class P, class Q>
int clip_halfplane(const V2<P>* in, int n, V2<P>* out, Q a, Q b, Q c, Q eps) {
  if (n <= 0) return 0;
  auto f = [&](V2<P> p) { return fmaT(a, (Q)p.x, fmaT(b, (Q)p.y, -c)); };
  auto isect = [&](V2<P> s, V2<P> e, Q fs, Q fe) {
    Q t = fs / ((fs - fe) + (Q)1e-30);
    return V2<P>{(P)fmaT(t, (Q)e.x - (Q)s.x, (Q)s.x), (P)fmaT(t, (Q)e.y - (Q)s.y, (Q)s.y)};
  };
  V2<P> s = in[n - 1];
  Q fs = f(s);
  bool ins_s = fs <= eps;
  int m = 0;
  for (int i = 0; i < n; ++i) {
    V2<P> e = in[i];
    Q fe = f(e);
    bool ins_e = fe <= eps;
    if (ins_e) {
      if (!ins_s) out[m++] = isect(s, e, fs, fe);
      out[m++] = e;
    } else if (ins_s) {
      out[m++] = isect(s, e, fs, fe);
    }
    s = e; fs = fe; ins_s = ins_e;
    if (m >= kMaxPoly) { m = kMaxPoly; break; }
  }
  return m;
}

// Neumaier compensated accumulation
template <class T> struct CSum {
  T s = 0, c = 0;
  void add(T x) {
    T t = s + x;
    if (std::fabs(s) >= std::fabs(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
  }
  T get() const { return s + c; }
};

// poly_centroid_2d (2dClip.cuh:55-80)
template <class P> V2<P> poly_centroid(const V2<P>* poly, int n, bool compensated) {
  const P nanv = std::numeric_limits<P>::quiet_NaN();
  if (n < 3) return {nanv, nanv};
  P A2, Cx, Cy;
  if (!compensated) {
    A2 = 0; Cx = 0; Cy = 0;
    for (int i = 0; i < n; ++i) {
      V2<P> p = poly[i], q = poly[(i + 1) % n];
      P cr = fmaT(p.x, q.y, -(q.x * p.y));
      A2 = A2 + cr;
      Cx = fmaT(p.x + q.x, cr, Cx);
      Cy = fmaT(p.y + q.y, cr, Cy);
    }
  } else {
    CSum<P> a, x, y;
    for (int i = 0; i < n; ++i) {
      V2<P> p = poly[i], q = poly[(i + 1) % n];
      P cr = fmaT(p.x, q.y, -(q.x * p.y));
      a.add(cr);
      x.add((p.x + q.x) * cr);
      y.add((p.y + q.y) * cr);
    }
    A2 = a.get(); Cx = x.get(); Cy = y.get();
  }
  P A = (P)0.5 * A2;
  if (std::fabs(A) < (P)1e-18) {
    P mx = 0, my = 0;
    for (int i = 0; i < n; ++i) { mx = mx + poly[i].x; my = my + poly[i].y; }
    return {mx / (P)n, my / (P)n};
  }
  P inv6A = (P)1 / ((P)6 * A);
  return {Cx * inv6A, Cy * inv6A};
}

// clip the square [-R,R]^2 by the bisectors of the K neighbours, in list order,
// and return the 3-D centroid (centroids_tangent_voronoi, 2dClip.cuh:82-135).
template <class T>
V3<T> cell_centroid(const T* S, long ns, long i, const uint32_t* nb, int K, Frame<T> fr, T R,
                    int profile, int* nverts_out) {
  V2<T> A[kMaxPoly + 2], B[kMaxPoly + 2];
  A[0] = {-R, -R}; A[1] = {R, -R}; A[2] = {R, R}; A[3] = {-R, R};
  int n = 4;
  V2<T>* cur = A;
  V2<T>* nxt = B;
  V3<T> si = ld3(S, i);
  for (int t = 0; t < K; ++t) {
    uint32_t j = nb[t];
    if (j >= (uint32_t)ns) continue;
    V3<T> sj = ld3(S, j);
    if (profile == P_MIXED) {
      double dx = (double)sj.x - (double)si.x, dy = (double)sj.y - (double)si.y, dz = (double)sj.z - (double)si.z;
      V3<double> d{dx, dy, dz}, u = cvt3<double>(fr.u), v = cvt3<double>(fr.v);
      double a = dot3(d, u), b = dot3(d, v), c = 0.5 * dot3(d, d);
      n = clip_halfplane<T, double>(cur, n, nxt, a, b, c, 1e-12);
    } else {
      V3<T> d = sub3(sj, si);
      T a = dot3(d, fr.u), b = dot3(d, fr.v), c = (T)0.5 * dot3(d, d);
      n = clip_halfplane<T, T>(cur, n, nxt, a, b, c, (T)1e-12);
    }
    std::swap(cur, nxt);
    if (n == 0) break;
  }
  if (nverts_out) *nverts_out = n;
  V2<T> c2 = poly_centroid(cur, n, profile == P_MIXED);
  const T nanv = std::numeric_limits<T>::quiet_NaN();
  if (!(std::isfinite(c2.x) && std::isfinite(c2.y))) return {nanv, nanv, nanv};
  return {si.x + fmaT(fr.u.x, c2.x, fr.v.x * c2.y), si.y + fmaT(fr.u.y, c2.x, fr.v.y * c2.y),
          si.z + fmaT(fr.u.z, c2.x, fr.v.z * c2.y)};
}

// closest_point_tri (near_project.cuh:12-53), Ericson's region test
template <class T> V3<T> closest_point_tri(V3<T> P, V3<T> A, V3<T> B, V3<T> C) {
  const T e = (T)1e-30;
  V3<T> AB = sub3(B, A), AC = sub3(C, A), AP = sub3(P, A);
  T d1 = dot3(AB, AP), d2 = dot3(AC, AP);
  if (d1 <= 0 && d2 <= 0) return A;
  V3<T> BP = sub3(P, B);
  T d3 = dot3(AB, BP), d4 = dot3(AC, BP);
  if (d3 >= 0 && d4 <= d3) return B;
  T vc = fmaT(d1, d4, -(d3 * d2));
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    T v = d1 / ((d1 - d3) + e);
    return {fmaT(AB.x, v, A.x), fmaT(AB.y, v, A.y), fmaT(AB.z, v, A.z)};
  }
  V3<T> CP = sub3(P, C);
  T d5 = dot3(AB, CP), d6 = dot3(AC, CP);
  if (d6 >= 0 && d5 <= d6) return C;
  T vb = fmaT(d5, d2, -(d1 * d6));
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    T w = d2 / ((d2 - d6) + e);
    return {fmaT(AC.x, w, A.x), fmaT(AC.y, w, A.y), fmaT(AC.z, w, A.z)};
  }
  T va = fmaT(d3, d6, -(d5 * d4));
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    T w = (d4 - d3) / (((d4 - d3) + (d5 - d6)) + e);
    V3<T> BC = sub3(C, B);
    return {fmaT(BC.x, w, B.x), fmaT(BC.y, w, B.y), fmaT(BC.z, w, B.z)};
  }
  T denom = (T)1 / (((va + vb) + vc) + e);
  T v = vb * denom, w = vc * denom;
  return {A.x + fmaT(AB.x, v, AC.x * w), A.y + fmaT(AB.y, v, AC.y * w), A.z + fmaT(AB.z, v, AC.z * w)};
}

// project_centroids_to_mesh (near_project.cuh:149-189): the closest point over
// the one-rings of the KPROJ nearest vertices, strict '<' keeps the first hit.
template <class T>
V3<T> project_point(V3<T> c, const float* V, int nV, const int* F, int nF, const int* off,
                    const int* fcs, const int* knnv, int kproj, int profile) {
  V3<T> bestP = c;
  if (profile == P_MIXED) {
    V3<double> cd = cvt3<double>(c), bp = cd;
    double best = 1e30;
    for (int t = 0; t < kproj; ++t) {
      int v = knnv[t];
      if ((unsigned)v >= (unsigned)nV) continue;
      for (int ii = off[v]; ii < off[v + 1]; ++ii) {
        int fi = fcs[ii];
        if ((unsigned)fi >= (unsigned)nF) continue;
        V3<double> A = cvt3<double>(ld3(V, F[3 * fi])), B = cvt3<double>(ld3(V, F[3 * fi + 1])),
                   C = cvt3<double>(ld3(V, F[3 * fi + 2]));
        V3<double> p = closest_point_tri(cd, A, B, C);
        V3<double> dd = sub3(p, cd);
        double d2 = dot3(dd, dd);
        if (d2 < best) { best = d2; bp = p; }
      }
    }
    return cvt3<T>(bp);
  }
  T best = (T)1e30;
  for (int t = 0; t < kproj; ++t) {
    int v = knnv[t];
    if ((unsigned)v >= (unsigned)nV) continue;
    for (int ii = off[v]; ii < off[v + 1]; ++ii) {
      int fi = fcs[ii];
      if ((unsigned)fi >= (unsigned)nF) continue;
      V3<T> A = cvt3<T>(ld3(V, F[3 * fi])), B = cvt3<T>(ld3(V, F[3 * fi + 1])), C = cvt3<T>(ld3(V, F[3 * fi + 2]));
      V3<T> p = closest_point_tri(c, A, B, C);
      V3<T> dd = sub3(p, c);
      T d2 = dot3(dd, dd);
      if (d2 < best) { best = d2; bestP = p; }
    }
  }
  return bestP;
}

// exact k nearest mesh vertices of q ((d2, index) order); skip == -1 for none
template <class T>
void vertex_knn(const PGrid<float>* g, const float* V, int nV, V3<T> q, int k, int skip, int* out) {
  TopK<T> top(k);
  if (std::isfinite((double)q.x) && std::isfinite((double)q.y) && std::isfinite((double)q.z)) {
    if (g) {
      // grid search in float coordinates (exact for T=float; for T=double the
      // grid only orders the visit, distances are recomputed in T)
      float qf[3] = {(float)q.x, (float)q.y, (float)q.z};
      int c[3] = {g->coord(qf[0], 0), g->coord(qf[1], 1), g->coord(qf[2], 2)};
      int rmax = std::max({g->dim[0], g->dim[1], g->dim[2]});
      for (int r = 0; r <= rmax; ++r) {
        g->ring(c[0], c[1], c[2], r, [&](uint32_t j) {
          if ((int)j == skip) return;
          top.push(dist2(cvt3<T>(ld3(V, j)), q), j);
        });
        double m = g->margin(qf, c, r) - 1e-3 * (double)g->h - 1e-6 * std::fabs((double)g->h);
        if (m == std::numeric_limits<double>::infinity()) break;
        if (top.full() && m > 0 && (double)top.worst() < m * m * (1.0 - 1e-6)) break;
      }
    } else {
      for (int j = 0; j < nV; ++j) {
        if (j == skip) continue;
        top.push(dist2(cvt3<T>(ld3(V, j)), q), (uint32_t)j);
      }
    }
  }
  for (int t = 0; t < k; ++t) out[t] = t < top.n ? (int)top.c[t].i : -1;
}

// ---------------------------------------------------------------------------
// tiers (main.cu:18-150)
// ---------------------------------------------------------------------------
void sym3_eigenvalues(const double C[9], double lam[3]) {
  double v[3] = {1.0, 0.0, 0.0};
  for (int it = 0; it < 20; ++it) {
    double w[3] = {C[0] * v[0] + C[1] * v[1] + C[2] * v[2], C[3] * v[0] + C[4] * v[1] + C[5] * v[2],
                   C[6] * v[0] + C[7] * v[1] + C[8] * v[2]};
    double n = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    if (n < 1e-30) break;
    v[0] = w[0] / n; v[1] = w[1] / n; v[2] = w[2] / n;
  }
  lam[0] = v[0] * (C[0] * v[0] + C[1] * v[1] + C[2] * v[2]) + v[1] * (C[3] * v[0] + C[4] * v[1] + C[5] * v[2]) +
           v[2] * (C[6] * v[0] + C[7] * v[1] + C[8] * v[2]);
  double C2[9];
  for (int i = 0; i < 9; ++i) C2[i] = C[i];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) C2[3 * r + c] -= lam[0] * v[r] * v[c];
  double v2[3] = {0.0, 1.0, 0.0};
  for (int it = 0; it < 20; ++it) {
    double w[3] = {C2[0] * v2[0] + C2[1] * v2[1] + C2[2] * v2[2], C2[3] * v2[0] + C2[4] * v2[1] + C2[5] * v2[2],
                   C2[6] * v2[0] + C2[7] * v2[1] + C2[8] * v2[2]};
    double n = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    if (n < 1e-30) break;
    v2[0] = w[0] / n; v2[1] = w[1] / n; v2[2] = w[2] / n;
  }
  lam[1] = v2[0] * (C2[0] * v2[0] + C2[1] * v2[1] + C2[2] * v2[2]) + v2[1] * (C2[3] * v2[0] + C2[4] * v2[1] + C2[5] * v2[2]) +
           v2[2] * (C2[6] * v2[0] + C2[7] * v2[1] + C2[8] * v2[2]);
  lam[2] = C[0] + C[4] + C[8] - lam[0] - lam[1];
}

}  // namespace

extern "C" {

void oracle_frames(const float* N, const int* nearest, int n, float* U, float* Vv) {
  for (int i = 0; i < n; ++i) {
    int nn = nearest[i];
    if (nn < 0) { st3(U, i, V3<float>{1, 0, 0}); st3(Vv, i, V3<float>{0, 1, 0}); continue; }
    Frame<float> fr = frame_from_normal(ld3(N, nn));
    st3(U, i, fr.u); st3(Vv, i, fr.v);
  }
}

// centroids_tangent_voronoi for all sites (profile 0 or 1); optional per-site
// final polygon vertex count.
void oracle_clip_centroids(const float* S, int n, const float* U, const float* Vv, const uint32_t* knn,
                           int K, float R, int profile, float* cent, int* nverts) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    Frame<float> fr{ld3(U, i), ld3(Vv, i)};
    V3<float> c = cell_centroid<float>(S, n, i, knn + (size_t)i * K, K, fr, R, profile,
                                       nverts ? nverts + i : nullptr);
    st3(cent, i, c);
  }
}

void oracle_closest_point_tri(const float* P, const float* A, const float* B, const float* C, float* out) {
  V3<float> r = closest_point_tri(ld3(P, 0), ld3(A, 0), ld3(B, 0), ld3(C, 0));
  st3(out, 0, r);
}

void oracle_project(const float* cent, int n, const float* V, int nV, const int* F, int nF,
                    const int* off, const int* fcs, const int* knnv, int kproj, int profile,
                    const float* Sold, float* Snew) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    V3<float> c = ld3(cent, i);
    if (profile == P_MIXED && !(std::isfinite(c.x) && std::isfinite(c.y) && std::isfinite(c.z))) {
      st3(Snew, i, ld3(Sold, i));
      continue;
    }
    st3(Snew, i, project_point<float>(c, V, nV, F, nF, off, fcs, knnv + (size_t)i * kproj, kproj, profile));
  }
}

// freeze_test_kernel_streak / _tiered + freeze_apply_cand_kernel.  need_per_tier
// holds streak[t]-1 clamped to >= 1 (freezetest.cuh:298-299).  counts[4] +=
// {same, low, both, newly frozen}.
void oracle_freeze(const float* S, const float* Snew, int n, const uint32_t* knn, const uint32_t* prev,
                   int K, int has_prev, const unsigned char* tier, const float* thr2_tier,
                   const int* need_tier, unsigned char* streak, unsigned char* cand,
                   unsigned char* frozen, int* counts) {
  for (int i = 0; i < n; ++i) {
    if (!has_prev) { streak[i] = 0; cand[i] = 0; continue; }
    int t = tier ? tier[i] : 0;
    if (t > 5) t = 5;
    bool same = true;
    for (int j = 0; j < K; ++j)
      if (knn[(size_t)i * K + j] != prev[(size_t)i * K + j]) { same = false; break; }
    V3<float> a = ld3(S, i), b = ld3(Snew, i);
    bool low = dist2(b, a) <= thr2_tier[t];
    bool both = same && low;
    counts[0] += same; counts[1] += low; counts[2] += both;
    unsigned char s = streak[i];
    s = both ? (unsigned char)(s < 255 ? s + 1 : s) : 0;
    streak[i] = s;
    cand[i] = (s >= need_tier[t]) ? 1 : 0;
  }
  for (int i = 0; i < n; ++i)
    if (cand[i] && !frozen[i]) { frozen[i] = 1; counts[3]++; }
}

// tier ids (main.cu:24-31 / 41-59 / 97-149): mode 1 = 5 tiers by normal
// variation, mode 2 = 6 tiers with the covariance-L split of tier 4.
// site_normal[i] is the unit normal used for site i.
void oracle_tiers(int mode, int n, int K, const float* site_normal, const uint32_t* knn,
                  unsigned char* tier, double* nv_out, double* L_out) {
  static const double TH[4] = {0.15, 0.35, 0.55, 0.80};
  for (int i = 0; i < n; ++i) {
    double sum = 0.0;
    int cnt = 0;
    for (int j = 0; j < K; ++j) {
      int jj = (int)knn[(size_t)i * K + j];
      if (jj < 0 || jj >= n) continue;
      double c = (double)site_normal[3 * i] * (double)site_normal[3 * jj] +
                 (double)site_normal[3 * i + 1] * (double)site_normal[3 * jj + 1] +
                 (double)site_normal[3 * i + 2] * (double)site_normal[3 * jj + 2];
      if (c > 1.0) c = 1.0;
      if (c < -1.0) c = -1.0;
      sum += c;
      cnt++;
    }
    double nv = cnt > 0 ? (1.0 - sum / (double)cnt) : 0.0;
    double L = 0.0;
    if (mode == 2) {
      double mean[3] = {0, 0, 0};
      int c2 = 0;
      for (int j = 0; j < K; ++j) {
        int jj = (int)knn[(size_t)i * K + j];
        if (jj < 0 || jj >= n) continue;
        for (int a = 0; a < 3; ++a) mean[a] += (double)site_normal[3 * jj + a];
        c2++;
      }
      if (c2 >= 2) {
        for (int a = 0; a < 3; ++a) mean[a] /= c2;
        double C[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < K; ++j) {
          int jj = (int)knn[(size_t)i * K + j];
          if (jj < 0 || jj >= n) continue;
          double d[3] = {(double)site_normal[3 * jj] - mean[0], (double)site_normal[3 * jj + 1] - mean[1],
                         (double)site_normal[3 * jj + 2] - mean[2]};
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) C[3 * r + c] += d[r] * d[c];
        }
        double lam[3];
        sym3_eigenvalues(C, lam);
        if (lam[0] > lam[1]) std::swap(lam[0], lam[1]);
        if (lam[1] > lam[2]) std::swap(lam[1], lam[2]);
        if (lam[0] > lam[1]) std::swap(lam[0], lam[1]);
        if (lam[2] > 1e-30) L = (lam[2] - lam[1]) / lam[2];
      }
    }
    int t = 0;
    while (t < 4 && nv >= TH[t]) t++;
    if (mode == 2 && t == 4 && L > 0.80) t = 5;
    tier[i] = (unsigned char)t;
    if (nv_out) nv_out[i] = nv;
    if (L_out) L_out[i] = L;
  }
}

}  // extern "C"

// ===========================================================================
// BVH (evaluate.cuh:106-201), used by the Hausdorff evaluation and by the
// BVH projection option
// ===========================================================================
// point->AABB squared distance (evaluate.cuh:44-51)
static inline float aabb_d2(V3<float> p, const float* bmin, const float* bmax) {
  float d = 0.f;
  float q[3] = {p.x, p.y, p.z};
  for (int a = 0; a < 3; ++a) {
    if (q[a] < bmin[a]) { float t = bmin[a] - q[a]; d = std::fma(t, t, d); }
    else if (q[a] > bmax[a]) { float t = q[a] - bmax[a]; d = std::fma(t, t, d); }
  }
  return d;
}

// BVH node layout as in evaluate.cuh:15-22 (40 bytes)
struct OBVHNode { float bmin[3], bmax[3]; int left, right, triStart, triCount; };

static int obvh_rec(std::vector<OBVHNode>& nodes, std::vector<int>& tri, const std::vector<float>& info,
                    std::vector<int>& tids, int leaf) {
  // info per triangle: bmin(3) bmax(3) ctr(3)
  OBVHNode nd{};
  for (int a = 0; a < 3; ++a) { nd.bmin[a] = 1e30f; nd.bmax[a] = -1e30f; }
  for (int t : tids)
    for (int a = 0; a < 3; ++a) {
      nd.bmin[a] = std::fmin(nd.bmin[a], info[9 * t + a]);
      nd.bmax[a] = std::fmax(nd.bmax[a], info[9 * t + 3 + a]);
    }
  nd.left = nd.right = -1; nd.triStart = -1; nd.triCount = 0;
  int me = (int)nodes.size();
  nodes.push_back(nd);
  if ((int)tids.size() <= leaf) {
    nodes[me].triStart = (int)tri.size();
    nodes[me].triCount = (int)tids.size();
    tri.insert(tri.end(), tids.begin(), tids.end());
    return me;
  }
  float cmin[3] = {1e30f, 1e30f, 1e30f}, cmax[3] = {-1e30f, -1e30f, -1e30f};
  for (int t : tids)
    for (int a = 0; a < 3; ++a) {
      cmin[a] = std::fmin(cmin[a], info[9 * t + 6 + a]);
      cmax[a] = std::fmax(cmax[a], info[9 * t + 6 + a]);
    }
  float ex = cmax[0] - cmin[0], ey = cmax[1] - cmin[1], ez = cmax[2] - cmin[2];
  int axis = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
  std::stable_sort(tids.begin(), tids.end(),
                   [&](int a, int b) { return info[9 * a + 6 + axis] < info[9 * b + 6 + axis]; });
  int mid = (int)tids.size() / 2;
  std::vector<int> L(tids.begin(), tids.begin() + mid), R(tids.begin() + mid, tids.end());
  int l = obvh_rec(nodes, tri, info, L, leaf);
  int r = obvh_rec(nodes, tri, info, R, leaf);
  nodes[me].left = l;
  nodes[me].right = r;
  return me;
}

static void obvh_build(const float* V, const int* F, int nF, int leaf, std::vector<OBVHNode>& nodes,
                       std::vector<int>& tri) {
  std::vector<float> info((size_t)9 * nF);
  for (int i = 0; i < nF; ++i) {
    V3<float> a = ld3(V, F[3 * i]), b = ld3(V, F[3 * i + 1]), c = ld3(V, F[3 * i + 2]);
    float* o = &info[(size_t)9 * i];
    o[0] = std::fmin(a.x, std::fmin(b.x, c.x)); o[1] = std::fmin(a.y, std::fmin(b.y, c.y)); o[2] = std::fmin(a.z, std::fmin(b.z, c.z));
    o[3] = std::fmax(a.x, std::fmax(b.x, c.x)); o[4] = std::fmax(a.y, std::fmax(b.y, c.y)); o[5] = std::fmax(a.z, std::fmax(b.z, c.z));
    const float third = 1.0f / 3.0f;
    o[6] = (a.x + (b.x + c.x)) * third; o[7] = (a.y + (b.y + c.y)) * third; o[8] = (a.z + (b.z + c.z)) * third;
  }
  nodes.clear(); tri.clear();
  std::vector<int> tids(nF);
  for (int i = 0; i < nF; ++i) tids[i] = i;
  if (nF > 0) obvh_rec(nodes, tri, info, tids, leaf);
}

// ===========================================================================
// options beyond the reference: PCA frames and the BVH projection.  Each
// restates the device routine of the same name in gpu_cvt_b200/csrc/
// cvt_math.cuh operation for operation, so the results agree bit for bit.
// ===========================================================================
namespace {

constexpr int kPcaSteps = 8;

// normal of the neighbourhood: eigenvector of the smallest eigenvalue of the
// covariance of the listed neighbours' offsets, by power iteration on the
// adjugate of C from n0, oriented like n0; n0 itself when fewer than 3
// neighbours, zero spread or a non-finite result
template <class T>
V3<T> pca_normal(const T* S, long ns, const uint32_t* row, int K, V3<T> si, V3<T> n0) {
  T sx = 0, sy = 0, sz = 0, xx = 0, xy = 0, xz = 0, yy = 0, yz = 0, zz = 0;
  int m = 0;
  for (int t = 0; t < K; ++t) {
    const uint32_t j = row[t];
    if (j >= (uint32_t)ns) continue;
    const V3<T> d = sub3(ld3(S, (long)j), si);
    sx = sx + d.x; sy = sy + d.y; sz = sz + d.z;
    xx = fmaT(d.x, d.x, xx); xy = fmaT(d.x, d.y, xy); xz = fmaT(d.x, d.z, xz);
    yy = fmaT(d.y, d.y, yy); yz = fmaT(d.y, d.z, yz); zz = fmaT(d.z, d.z, zz);
    ++m;
  }
  if (m < 3) return n0;
  const T im = (T)1 / (T)m;
  const T mx = sx * im, my = sy * im, mz = sz * im;
  const T cxx = fmaT(-sx, mx, xx), cxy = fmaT(-sx, my, xy), cxz = fmaT(-sx, mz, xz);
  const T cyy = fmaT(-sy, my, yy), cyz = fmaT(-sy, mz, yz), czz = fmaT(-sz, mz, zz);
  const T tr = (cxx + cyy) + czz;
  if (!(tr > (T)1e-30)) return n0;
  // adjugate of C: eigenvalues l2 l3, l1 l3, l1 l2 for C's l1 <= l2 <= l3,
  // so the normal's (l1) direction dominates by the factor l2 / l1
  const T axx = fmaT(cyy, czz, -(cyz * cyz)), axy = fmaT(cxz, cyz, -(cxy * czz)), axz = fmaT(cxy, cyz, -(cxz * cyy));
  const T ayy = fmaT(cxx, czz, -(cxz * cxz)), ayz = fmaT(cxy, cxz, -(cxx * cyz)), azz = fmaT(cxx, cyy, -(cxy * cxy));
  V3<T> v = n0;
  for (int it = 0; it < kPcaSteps; ++it) {
    const V3<T> w{fmaT(axz, v.z, fmaT(axy, v.y, axx * v.x)), fmaT(ayz, v.z, fmaT(ayy, v.y, axy * v.x)),
                  fmaT(azz, v.z, fmaT(ayz, v.y, axz * v.x))};
    const T nw = std::sqrt(dot3(w, w));
    if (!(nw > (T)1e-30)) return n0;
    const T inv = (T)1 / nw;
    v = {w.x * inv, w.y * inv, w.z * inv};
  }
  if (!(std::isfinite((double)v.x) && std::isfinite((double)v.y) && std::isfinite((double)v.z))) return n0;
  if (dot3(v, n0) < (T)0) v = {-v.x, -v.y, -v.z};
  return v;
}

// (|c - s| (1 + 1e-4) + 1e-5 max|s|)^2 in double: an upper bound of the
// squared distance from c to the mesh when s lies on it
template <class T> double bvh_bound2(V3<T> c, V3<T> s) {
  const double dx = (double)c.x - (double)s.x, dy = (double)c.y - (double)s.y, dz = (double)c.z - (double)s.z;
  const double m = std::fmax(std::fmax(std::fabs((double)s.x), std::fabs((double)s.y)), std::fabs((double)s.z));
  const double d = std::sqrt(std::fma(dz, dz, std::fma(dy, dy, dx * dx))) * 1.0001 + 1e-5 * m;
  return std::isfinite(d) ? d * d : 1e30;
}

// closest point on the mesh through the BVH: near-first traversal, boxes
// entered while their FP32 squared distance is below the best so far, strict
// '<' per face (first face in traversal order wins ties); best starts at
// bound2 and the search reruns unbounded if nothing beats it
template <class T, class Q>
V3<T> project_bvh(V3<T> c, const std::vector<OBVHNode>& nodes, const std::vector<int>& tri, const float* V,
                  const int* F, Q bound2) {
  if (!(std::isfinite((double)c.x) && std::isfinite((double)c.y) && std::isfinite((double)c.z))) return c;
  const V3<Q> cq = cvt3<Q>(c);
  const V3<float> cf = cvt3<float>(c);
  V3<Q> bp = cq;
  if (nodes.empty()) return c;
  std::vector<int> stack;
  for (int pass = 0; pass < 2; ++pass) {
    Q best = pass == 0 ? bound2 : (Q)1e30;
    bool found = false;
    stack.clear();
    stack.push_back(0);
    while (!stack.empty()) {
      const OBVHNode nd = nodes[stack.back()];
      stack.pop_back();
      if ((Q)aabb_d2(cf, nd.bmin, nd.bmax) >= best) continue;
      if (nd.triCount > 0) {
        for (int k = 0; k < nd.triCount; ++k) {
          const int t = tri[nd.triStart + k];
          const V3<Q> A = cvt3<Q>(ld3(V, F[3 * t])), B = cvt3<Q>(ld3(V, F[3 * t + 1])), C = cvt3<Q>(ld3(V, F[3 * t + 2]));
          const V3<Q> p = closest_point_tri(cq, A, B, C);
          const V3<Q> dd = sub3(p, cq);
          const Q d2 = dot3(dd, dd);
          if (d2 < best) { best = d2; bp = p; found = true; }
        }
      } else {
        const OBVHNode& L = nodes[nd.left];
        const OBVHNode& R = nodes[nd.right];
        const Q dl = (Q)aabb_d2(cf, L.bmin, L.bmax), dr = (Q)aabb_d2(cf, R.bmin, R.bmax);
        if (dl < dr) {
          if (dr < best) stack.push_back(nd.right);
          if (dl < best) stack.push_back(nd.left);
        } else {
          if (dl < best) stack.push_back(nd.left);
          if (dr < best) stack.push_back(nd.right);
        }
      }
    }
    if (found) break;
  }
  return cvt3<T>(bp);
}

}  // namespace

// ===========================================================================
// Lloyd loop (main.cu:640-881), generalised to nSites != nV
// ===========================================================================
namespace {

struct RunParams {
  int K;          // neighbours after dropping self (K_NEIGH)
  int mode;       // 0 freezing off, 1 five tiers, 2 six tiers
  int profile;    // P_REF / P_MIXED / P_FP64
  int iters;
  int kproj;      // nearest mesh vertices for the projection one-rings (5)
  int ex_quirk;   // mode 0: skip vertex index == site index in centroid->mesh KNN
  float R;        // clip square half size (input mesh max bbox edge)
  int proj_mode;  // 0: one-ring of the kproj nearest vertices; 1: closest point through the BVH
  int frame_mode; // 0: nearest vertex normal; 1: PCA normal of the neighbour list
};

const int kStreak1[6] = {5, 10, 15, 20, 25, 25};
const int kStreak2[6] = {5, 10, 15, 20, 25, 10};

template <class T>
void lloyd_run(const float* V, int nV, const int* F, int nF, const float* N, T* S, int n,
               const RunParams& p, int* counts, double* maxdisp, unsigned char* frozen_out,
               unsigned char* tier_out, uint32_t* knn_out, int* knnv_out, float* cent_out) {
  const int K = p.K, KK = p.K + 1, KP = p.kproj;
  std::vector<int> off(nV + 1), fcs(3 * (size_t)nF);
  oracle_build_vf(nV, nF, F, off.data(), fcs.data());
  PGrid<float> vg;
  vg.build(V, nV, 4.0);
  std::vector<uint32_t> raw((size_t)n * KK), knn((size_t)n * K, 0u), prev((size_t)n * K, 0u);
  std::vector<int> knnv((size_t)n * KP, -1);
  std::vector<int> nnv(n, -1);  // frame vertex of each site's last active iteration
  std::vector<OBVHNode> bvh_nodes;
  std::vector<int> bvh_tri;
  if (p.proj_mode == 1) obvh_build(V, F, nF, 8, bvh_nodes, bvh_tri);
  std::vector<unsigned char> frozen(n, 0), streak(n, 0), cand(n, 0), tier(n, 0);
  std::vector<T> Snew((size_t)3 * n);
  float thr2 = ((0.01f * p.R) * 0.01f) * p.R;
  float thr2_tier[6];
  int need[6];
  for (int t = 0; t < 6; ++t) {
    thr2_tier[t] = thr2;
    int s = p.mode == 0 ? 5 : (p.mode == 1 ? kStreak1[t] : kStreak2[t]);
    need[t] = std::max(1, s - 1);
  }
  auto site_knn = [&](const unsigned char* fr) {
    PGrid<T> g;
    g.build(S, n, 2.0 * KK);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
      if (fr && fr[i]) continue;
      TopK<T> top(KK);
      g.knn(S + 3 * (size_t)i, top, [](uint32_t) { return true; });
      uint32_t* r = raw.data() + (size_t)i * KK;
      for (int t = 0; t < KK; ++t) r[t] = t < top.n ? top.c[t].i : 0xFFFFFFFFu;
      // drop self (site_knn.cuh:79-103)
      uint32_t* d = knn.data() + (size_t)i * K;
      int w = 0;
      for (int t = 0; t < KK && w < K; ++t) {
        if ((int)r[t] == i) continue;
        d[w++] = r[t];
      }
      if (w == 0) for (int k = 0; k < K; ++k) d[k] = (uint32_t)i;
      else { uint32_t fill = d[w - 1]; for (; w < K; ++w) d[w] = fill; }
    }
  };
  auto nearest_vertex = [&](V3<T> q) { int o; vertex_knn<T>(&vg, V, nV, q, 1, -1, &o); return o; };

  if (p.mode != 0) {
    // tier pre-pass (main.cu:640-667): KNN of the initial sites, site normal =
    // normal of the site's nearest mesh vertex (= vertex i when sites are the
    // vertices, as in the reference).
    site_knn(nullptr);
    std::vector<float> sn((size_t)3 * n);
    for (int i = 0; i < n; ++i) {
      int v = nearest_vertex(ld3(S, i));
      V3<float> nn = v >= 0 ? ld3(N, v) : V3<float>{0, 0, 0};
      st3(sn.data(), i, nn);
    }
    oracle_tiers(p.mode, n, K, sn.data(), knn.data(), tier.data(), nullptr, nullptr);
  }

  for (int it = 0; it < p.iters; ++it) {
    site_knn(frozen.data());
    for (int i = 0; i < n; ++i)
      if (frozen[i]) std::memcpy(&knn[(size_t)i * K], &prev[(size_t)i * K], sizeof(uint32_t) * K);
    const int skip_mode0 = (p.mode == 0 && p.ex_quirk);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
      V3<T> si = ld3(S, i);
      if (!frozen[i]) nnv[i] = nearest_vertex(si);
      // frozen sites: the first entry of their kept vertex list; with the BVH
      // projection (no vertex list) their kept frame vertex
      int nn = (frozen[i] && p.proj_mode == 0) ? knnv[(size_t)i * KP] : nnv[i];
      Frame<T> fr;
      if (nn < 0) {
        fr = {{1, 0, 0}, {0, 1, 0}};
      } else {
        V3<T> n0 = cvt3<T>(ld3(N, nn));
        if (p.frame_mode == 1) n0 = pca_normal<T>(S, n, &knn[(size_t)i * K], K, si, n0);
        fr = frame_from_normal(n0);
      }
      V3<T> c = cell_centroid<T>(S, n, i, &knn[(size_t)i * K], K, fr, (T)p.R, p.profile, nullptr);
      if (cent_out) st3(cent_out, i, cvt3<float>(c));
      bool finite = std::isfinite((double)c.x) && std::isfinite((double)c.y) && std::isfinite((double)c.z);
      V3<T> sn;
      if (p.profile != P_REF && !finite) {
        sn = si;
      } else if (p.proj_mode == 1) {
        if (p.profile == P_MIXED) sn = project_bvh<T, double>(c, bvh_nodes, bvh_tri, V, F, bvh_bound2(c, si));
        else sn = project_bvh<T, T>(c, bvh_nodes, bvh_tri, V, F, (T)bvh_bound2(c, si));
      } else {
        if (!frozen[i]) vertex_knn<T>(&vg, V, nV, c, KP, skip_mode0 ? i : -1, &knnv[(size_t)i * KP]);
        sn = project_point<T>(c, V, nV, F, nF, off.data(), fcs.data(), &knnv[(size_t)i * KP], KP,
                              p.profile == P_MIXED ? P_MIXED : P_REF);
      }
      st3(Snew.data(), i, sn);
    }
    int cnt[4] = {0, 0, 0, 0};
    double md = 0.0;
    for (int i = 0; i < n; ++i) {
      double dd = (double)dist2(ld3(Snew.data(), i), ld3(S, i));
      if (dd > md) md = dd;
    }
    if (it == 0) {
      for (int i = 0; i < n; ++i) { streak[i] = 0; cand[i] = 0; }
    } else {
      for (int i = 0; i < n; ++i) {
        int t = std::min<int>(tier[i], 5);
        bool same = std::memcmp(&knn[(size_t)i * K], &prev[(size_t)i * K], sizeof(uint32_t) * K) == 0;
        T d2 = dist2(ld3(Snew.data(), i), ld3(S, i));
        bool low = d2 <= (T)thr2_tier[t];
        bool both = same && low;
        cnt[0] += same; cnt[1] += low; cnt[2] += both;
        unsigned char s = streak[i];
        s = both ? (unsigned char)(s < 255 ? s + 1 : s) : 0;
        streak[i] = s;
        cand[i] = (s >= need[t]) ? 1 : 0;
      }
      for (int i = 0; i < n; ++i)
        if (cand[i] && !frozen[i]) { frozen[i] = 1; cnt[3]++; }
    }
    if (p.mode == 0) {
      std::fill(frozen.begin(), frozen.end(), 0);
      std::fill(streak.begin(), streak.end(), 0);
    }
    if (counts) for (int a = 0; a < 4; ++a) counts[4 * it + a] = cnt[a];
    if (maxdisp) maxdisp[it] = std::sqrt(md);
    prev = knn;
    std::memcpy(S, Snew.data(), sizeof(T) * 3 * (size_t)n);
  }
  if (frozen_out) std::memcpy(frozen_out, frozen.data(), n);
  if (tier_out) std::memcpy(tier_out, tier.data(), n);
  if (knn_out) std::memcpy(knn_out, knn.data(), sizeof(uint32_t) * (size_t)n * K);
  if (knnv_out) std::memcpy(knnv_out, knnv.data(), sizeof(int) * (size_t)n * KP);
}

}  // namespace

extern "C" {

// One full remesh run.  S (n*3) is updated in place.  counts: iters*4 ints
// {same, low, both, newly}; maxdisp: iters doubles (max site motion).  The
// optional outputs give the final frozen mask, tiers, site KNN (n*K) and
// vertex KNN (n*kproj).  cent_out (n*3 floats) receives the centroids of the
// last iteration.  profile 0/1: float state.
void oracle_lloyd_run(const float* V, int nV, const int* F, int nF, const float* N, float* S, int n, int K,
                      int mode, int profile, int iters, int kproj, int ex_quirk, float R, int* counts,
                      double* maxdisp, unsigned char* frozen_out, unsigned char* tier_out, uint32_t* knn_out,
                      int* knnv_out, float* cent_out, int proj_mode, int frame_mode) {
  RunParams p{K, mode, profile == P_FP64 ? P_REF : profile, iters, kproj, ex_quirk, R, proj_mode, frame_mode};
  lloyd_run<float>(V, nV, F, nF, N, S, n, p, counts, maxdisp, frozen_out, tier_out, knn_out, knnv_out, cent_out);
}

// The FP64 oracle: the same loop with double state and arithmetic.
void oracle_lloyd_run_f64(const float* V, int nV, const int* F, int nF, const float* N, double* S, int n, int K,
                          int mode, int iters, int kproj, int ex_quirk, float R, int* counts, double* maxdisp,
                          unsigned char* frozen_out, unsigned char* tier_out, uint32_t* knn_out, int* knnv_out,
                          int proj_mode, int frame_mode) {
  RunParams p{K, mode, P_REF, iters, kproj, ex_quirk, R, proj_mode, frame_mode};
  lloyd_run<double>(V, nV, F, nF, N, S, n, p, counts, maxdisp, frozen_out, tier_out, knn_out, knnv_out, nullptr);
}

// frames from the PCA normal of each site's listed neighbours, started from
// the normal of vertex nearest[i] (cvt_frames_pca)
void oracle_pca_frames(const float* S, int n, const uint32_t* knn, int K, const float* N, const int* nearest,
                       float* U, float* Vv) {
  for (int i = 0; i < n; ++i) {
    int nn = nearest[i];
    if (nn < 0) { st3(U, i, V3<float>{1, 0, 0}); st3(Vv, i, V3<float>{0, 1, 0}); continue; }
    V3<float> nrm = pca_normal<float>(S, n, knn + (size_t)i * K, K, ld3(S, i), ld3(N, nn));
    Frame<float> fr = frame_from_normal(nrm);
    st3(U, i, fr.u); st3(Vv, i, fr.v);
  }
}

// closest point on the mesh through its BVH for every centroid
// (cvt_project_bvh); Sold may be NULL except in MIXED
void oracle_project_bvh(const float* cent, int n, const float* V, int nV, const int* F, int nF, int profile,
                        const float* Sold, float* Snew) {
  (void)nV;
  std::vector<OBVHNode> nodes;
  std::vector<int> tri;
  obvh_build(V, F, nF, 8, nodes, tri);
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    V3<float> c = ld3(cent, i);
    bool finite = std::isfinite(c.x) && std::isfinite(c.y) && std::isfinite(c.z);
    if (profile == P_MIXED && !finite) { st3(Snew, i, ld3(Sold, i)); continue; }
    double b2 = Sold ? bvh_bound2(c, ld3(Sold, i)) : 1e30;
    V3<float> r = profile == P_MIXED ? project_bvh<float, double>(c, nodes, tri, V, F, b2)
                                     : project_bvh<float, float>(c, nodes, tri, V, F, (float)b2);
    st3(Snew, i, r);
  }
}

// ===========================================================================
// evaluation: BVH (evaluate.cuh:106-201), Hausdorff (evaluate.cuh:203-383),
// quality (evaluate.cuh:388-462)
// ===========================================================================

// point->triangle squared distance (evaluate.cuh:54-104)
float oracle_point_tri_d2(const float* P, const float* A, const float* B, const float* C) {
  V3<float> p = ld3(P, 0), a = ld3(A, 0), b = ld3(B, 0), c = ld3(C, 0);
  V3<float> ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
  float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.f && d2 <= 0.f) return dot3(ap, ap);
  V3<float> bp = sub3(p, b);
  float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.f && d4 <= d3) return dot3(bp, bp);
  float vc = std::fma(d1, d4, -(d3 * d2));
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
    float v = d1 / (d1 - d3);
    V3<float> pr{std::fma(ab.x, v, a.x), std::fma(ab.y, v, a.y), std::fma(ab.z, v, a.z)};
    V3<float> d = sub3(p, pr);
    return dot3(d, d);
  }
  V3<float> cp = sub3(p, c);
  float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.f && d5 <= d6) return dot3(cp, cp);
  float vb = std::fma(d5, d2, -(d1 * d6));
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
    float w = d2 / (d2 - d6);
    V3<float> pr{std::fma(ac.x, w, a.x), std::fma(ac.y, w, a.y), std::fma(ac.z, w, a.z)};
    V3<float> d = sub3(p, pr);
    return dot3(d, d);
  }
  float va = std::fma(d3, d6, -(d5 * d4));
  if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
    float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    V3<float> bc = sub3(c, b);
    V3<float> pr{std::fma(bc.x, w, b.x), std::fma(bc.y, w, b.y), std::fma(bc.z, w, b.z)};
    V3<float> d = sub3(p, pr);
    return dot3(d, d);
  }
  float denom = 1.f / ((va + vb) + vc);
  float v = vb * denom, w = vc * denom;
  V3<float> pr{a.x + std::fma(ab.x, v, ac.x * w), a.y + std::fma(ab.y, v, ac.y * w), a.z + std::fma(ab.z, v, ac.z * w)};
  V3<float> d = sub3(p, pr);
  return dot3(d, d);
}

int oracle_bvh_node_count(const float* V, const int* F, int nF, int leaf) {
  std::vector<OBVHNode> nodes;
  std::vector<int> tri;
  obvh_build(V, F, nF, leaf, nodes, tri);
  return (int)nodes.size();
}

// nodes_out: nNodes * 10 words (bmin, bmax as float bits; left, right, start, count)
void oracle_bvh_build(const float* V, const int* F, int nF, int leaf, void* nodes_out, int* tri_out) {
  std::vector<OBVHNode> nodes;
  std::vector<int> tri;
  obvh_build(V, F, nF, leaf, nodes, tri);
  std::memcpy(nodes_out, nodes.data(), nodes.size() * sizeof(OBVHNode));
  std::memcpy(tri_out, tri.data(), tri.size() * sizeof(int));
}

static float obvh_closest(const std::vector<OBVHNode>& nodes, const std::vector<int>& tri, const float* V,
                          const int* F, V3<float> p) {
  float best = 1e30f;
  if (nodes.empty()) return best;
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const OBVHNode& nd = nodes[stack[--sp]];
    if (aabb_d2(p, nd.bmin, nd.bmax) >= best) continue;
    if (nd.triCount > 0) {
      for (int k = 0; k < nd.triCount; ++k) {
        int t = tri[nd.triStart + k];
        float pp[3] = {p.x, p.y, p.z};
        float d2 = oracle_point_tri_d2(pp, V + 3 * F[3 * t], V + 3 * F[3 * t + 1], V + 3 * F[3 * t + 2]);
        if (d2 < best) best = d2;
      }
    } else {
      if (nd.left >= 0) stack[sp++] = nd.left;
      if (nd.right >= 0) stack[sp++] = nd.right;
    }
  }
  return best;
}

// probe points (evaluate.cuh:253-283): vertices, then per face the centroid
// and the three edge midpoints.
static void probe_points(const float* V, int nV, const int* F, int nF, std::vector<float>& P) {
  P.resize((size_t)3 * (nV + 4 * (size_t)nF));
  std::memcpy(P.data(), V, sizeof(float) * 3 * nV);
  const float third = 1.0f / 3.0f;
  for (int f = 0; f < nF; ++f) {
    V3<float> a = ld3(V, F[3 * f]), b = ld3(V, F[3 * f + 1]), c = ld3(V, F[3 * f + 2]);
    long base = nV + 4L * f;
    st3(P.data(), base + 0, V3<float>{(a.x + (b.x + c.x)) * third, (a.y + (b.y + c.y)) * third, (a.z + (b.z + c.z)) * third});
    st3(P.data(), base + 1, V3<float>{(a.x + b.x) * 0.5f, (a.y + b.y) * 0.5f, (a.z + b.z) * 0.5f});
    st3(P.data(), base + 2, V3<float>{(b.x + c.x) * 0.5f, (b.y + c.y) * 0.5f, (b.z + c.z) * 0.5f});
    st3(P.data(), base + 3, V3<float>{(c.x + a.x) * 0.5f, (c.y + a.y) * 0.5f, (c.z + a.z) * 0.5f});
  }
}

// One-sided Hausdorff distance: max over the probes of (V1,F1) of the distance
// to the surface (V2,F2) (hausdorff_bvh_gpu, evaluate.cuh:291-357).  use_bvh=0
// scans every triangle (the brute-force check of the BVH traversal).
float oracle_hausdorff_one_sided(const float* V1, int nV1, const int* F1, int nF1, const float* V2, int nV2,
                                 const int* F2, int nF2, int use_bvh) {
  (void)nV2;
  std::vector<float> P;
  probe_points(V1, nV1, F1, nF1, P);
  long nP = (long)P.size() / 3;
  std::vector<OBVHNode> nodes;
  std::vector<int> tri;
  if (use_bvh) obvh_build(V2, F2, nF2, 8, nodes, tri);
  float mx = 0.f;
#pragma omp parallel for schedule(dynamic, 256) reduction(max : mx)
  for (long i = 0; i < nP; ++i) {
    V3<float> p = ld3(P.data(), i);
    float best;
    if (use_bvh) best = obvh_closest(nodes, tri, V2, F2, p);
    else {
      best = 1e30f;
      for (int t = 0; t < nF2; ++t) {
        float d2 = oracle_point_tri_d2(&P[3 * i], V2 + 3 * F2[3 * t], V2 + 3 * F2[3 * t + 1], V2 + 3 * F2[3 * t + 2]);
        if (d2 < best) best = d2;
      }
    }
    if (best > mx) mx = best;
  }
  return std::sqrt(mx);
}

// eval_quality_angles_cpu (evaluate.cuh:388-462); out[6] = Qmin, Qavg,
// theta_min, theta_min_avg, theta_lt_30_pct, theta_gt_90_pct
void oracle_quality(const float* V, const int* F, int nF, float* out) {
  auto angle_deg = [](V3<float> u, V3<float> v) {
    float du = std::sqrt(dot3(u, u)), dv = std::sqrt(dot3(v, v));
    float denom = std::fmax(du * dv, 1e-30f);
    float cs = dot3(u, v) / denom;
    cs = std::fmin(1.f, std::fmax(-1.f, cs));
    return std::acos(cs) * (180.0f / 3.14159265358979323846f);
  };
  float Qmin = 1e30f, tmin_all = 1e30f;
  double Qsum = 0, thsum = 0, lt30 = 0, gt90 = 0, cnt = 0;
  for (int f = 0; f < nF; ++f) {
    V3<float> a = ld3(V, F[3 * f]), b = ld3(V, F[3 * f + 1]), c = ld3(V, F[3 * f + 2]);
    V3<float> ab = sub3(b, a), ac = sub3(c, a), ba = sub3(a, b), bc = sub3(c, b), ca = sub3(a, c), cb = sub3(b, c);
    float A = angle_deg(ab, ac), B = angle_deg(ba, bc), C = angle_deg(ca, cb);
    float tmin = std::fmin(A, std::fmin(B, C));
    tmin_all = std::fmin(tmin_all, tmin);
    thsum += tmin;
    lt30 += (A < 30.f) + (B < 30.f) + (C < 30.f);
    gt90 += (A > 90.f) + (B > 90.f) + (C > 90.f);
    cnt += 3.0;
    float l0 = std::sqrt(dot3(ab, ab)), l1 = std::sqrt(dot3(bc, bc)), l2 = std::sqrt(dot3(ca, ca));
    V3<float> cr = cross3(ab, ac);
    float area = 0.5f * std::sqrt(dot3(cr, cr));
    float s = 0.5f * ((l0 + l1) + l2);
    float e = std::fmax(l0, std::fmax(l1, l2));
    float denom = std::fmax(s * e, 1e-30f);
    float q = (6.0f / std::sqrt(3.0f)) * (area / denom);
    Qmin = std::fmin(Qmin, q);
    Qsum += q;
  }
  out[0] = Qmin;
  out[1] = nF > 0 ? (float)(Qsum / nF) : 0.f;
  out[2] = tmin_all;
  out[3] = nF > 0 ? (float)(thsum / nF) : 0.f;
  out[4] = cnt > 0 ? (float)(lt30 * 100.0 / cnt) : 0.f;
  out[5] = cnt > 0 ? (float)(gt90 * 100.0 / cnt) : 0.f;
}

// ===========================================================================
// dual-triangle extraction (near_project.cuh:201-352, buildmesh.cuh,
// main.cu:928-974).  Returns the number of faces written to F_out (sorted,
// unique, degenerate ones removed); F_out must hold n*256 triangles.
// ===========================================================================
int oracle_extract_faces(const float* S, int n, const float* U, const float* Vv, const uint32_t* knn, int K,
                         float R2, float eps_clip, float tol_active, float degenerate_eps, int* F_out) {
  const int MAXP = 256;
  std::vector<uint64_t> keys;
  keys.reserve((size_t)n * 8);
#pragma omp parallel
  {
    std::vector<uint64_t> local;
    std::vector<V2<float>> A(MAXP), B(MAXP);
    std::vector<int> LA(MAXP), LB(MAXP);
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
      V3<float> si = ld3(S, i), ui = ld3(U, i), vi = ld3(Vv, i);
      int na = 4;
      A[0] = {-R2, -R2}; A[1] = {R2, -R2}; A[2] = {R2, R2}; A[3] = {-R2, R2};
      LA[0] = LA[1] = LA[2] = LA[3] = -1;
      const uint32_t* nb = knn + (size_t)i * K;
      auto abc = [&](int j, float& a, float& b, float& c) {
        V3<float> d = sub3(ld3(S, j), si);
        a = dot3(d, ui); b = dot3(d, vi); c = 0.5f * dot3(d, d);
      };
      for (int t = 0; t < K; ++t) {
        int j = (int)nb[t];
        if ((unsigned)j >= (unsigned)n || j == i) continue;
        float a, b, c;
        abc(j, a, b, c);
        auto f = [&](V2<float> p) { return std::fma(a, p.x, std::fma(b, p.y, -c)); };
        int nb2 = 0;
        if (na > 0) {
          V2<float> s = A[na - 1];
          int ls = LA[na - 1];
          float fs = f(s);
          (void)ls;
          for (int k = 0; k < na; ++k) {
            V2<float> e = A[k];
            int le = LA[k];
            float fe = f(e);
            bool ins_e = fe <= eps_clip, ins_s = fs <= eps_clip;
            auto isect = [&]() {
              float tt = fs / ((fs - fe) + 1e-30f);
              return V2<float>{std::fma(tt, e.x - s.x, s.x), std::fma(tt, e.y - s.y, s.y)};
            };
            if (ins_e) {
              if (!ins_s && nb2 < MAXP) { B[nb2] = isect(); LB[nb2] = j; nb2++; }
              if (nb2 < MAXP) { B[nb2] = e; LB[nb2] = le; nb2++; }
            } else if (ins_s) {
              if (nb2 < MAXP) { B[nb2] = isect(); LB[nb2] = j; nb2++; }
            }
            s = e; fs = fe;
          }
        }
        na = nb2;
        std::swap(A, B);
        std::swap(LA, LB);
        if (na == 0) break;
      }
      if (na < 3) continue;
      for (int k = 0; k < na; ++k) {
        V2<float> p = A[k];
        float b1 = 1e30f, b2 = 1e30f;
        int j1 = -1, j2 = -1;
        for (int t = 0; t < K; ++t) {
          int j = (int)nb[t];
          if ((unsigned)j >= (unsigned)n || j == i) continue;
          float a, b, c;
          abc(j, a, b, c);
          float s = std::fabs(std::fma(a, p.x, std::fma(b, p.y, -c)));
          if (s < b1) { b2 = b1; j2 = j1; b1 = s; j1 = j; }
          else if (s < b2) { b2 = s; j2 = j; }
        }
        if (!(j1 >= 0 && j2 >= 0 && j1 != j2 && b1 <= tol_active && b2 <= tol_active)) continue;
        int a = i, b = j1, c = j2;
        if (a > b) std::swap(a, b);
        if (b > c) std::swap(b, c);
        if (a > b) std::swap(a, b);
        local.push_back((uint64_t)(uint32_t)a | ((uint64_t)(uint32_t)b << 21) | ((uint64_t)(uint32_t)c << 42));
      }
    }
#pragma omp critical
    keys.insert(keys.end(), local.begin(), local.end());
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  int nf = 0;
  for (uint64_t k : keys) {
    int a = (int)(k & 0x1FFFFF), b = (int)((k >> 21) & 0x1FFFFF), c = (int)((k >> 42) & 0x1FFFFF);
    bool deg = (a == b || b == c || a == c) || a >= n || b >= n || c >= n;
    if (!deg) {
      V3<float> A = ld3(S, a), B = ld3(S, b), C = ld3(S, c);
      V3<float> e0 = sub3(B, A), e1 = sub3(C, B), e2 = sub3(A, C);
      float l0 = std::sqrt(dot3(e0, e0)), l1 = std::sqrt(dot3(e1, e1)), l2 = std::sqrt(dot3(e2, e2));
      V3<float> cr = cross3(sub3(B, A), sub3(C, A));
      float ar = std::sqrt(dot3(cr, cr));
      deg = !(l0 > degenerate_eps && l1 > degenerate_eps && l2 > degenerate_eps && ar > degenerate_eps);
    }
    if (deg) continue;
    F_out[3 * nf] = a; F_out[3 * nf + 1] = b; F_out[3 * nf + 2] = c;
    nf++;
  }
  return nf;
}

}  // extern "C"
