// Device geometry for the tangent-plane CVT Lloyd step.
//
// Rounding is pinned: the library is compiled with -fmad=false, so a*b+c is
// two rounded operations unless an explicit fmaT() is written, and every
// division / square root is the IEEE-rounded intrinsic.  The operation order
// of each routine follows the reference kernels it replaces (cited below);
// the reference's rsqrtf() becomes 1/sqrt (IEEE), a <=1-ulp difference.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cvt {

enum Profile { PROF_REF = 0, PROF_MIXED = 1, PROF_FP64 = 2 };

template <class T> struct V3 { T x, y, z; };
template <class T> struct V2 { T x, y; };

__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float divT(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double divT(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float sqrtT(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double sqrtT(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ float absT(float a) { return fabsf(a); }
__device__ __forceinline__ double absT(double a) { return fabs(a); }
template <class T> __device__ __forceinline__ bool finiteT(T a) { return isfinite(a); }

template <class T> __device__ __forceinline__ V3<T> sub3(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> __device__ __forceinline__ T dot3(V3<T> a, V3<T> b) {
  return fmaT(a.z, b.z, fmaT(a.y, b.y, a.x * b.x));
}
template <class T> __device__ __forceinline__ V3<T> cross3(V3<T> a, V3<T> b) {
  return {fmaT(a.y, b.z, -(a.z * b.y)), fmaT(a.z, b.x, -(a.x * b.z)), fmaT(a.x, b.y, -(a.y * b.x))};
}
template <class T> __device__ __forceinline__ T dist2(V3<T> p, V3<T> q) {
  T dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
  return fmaT(dz, dz, fmaT(dy, dy, dx * dx));
}
template <class T, class S> __device__ __forceinline__ V3<T> cvt3(V3<S> a) { return {(T)a.x, (T)a.y, (T)a.z}; }
template <class T> __device__ __forceinline__ V3<T> ld3(const T* __restrict__ p, long i) {
  return {p[3 * i], p[3 * i + 1], p[3 * i + 2]};
}
template <class T> __device__ __forceinline__ void st3(T* __restrict__ p, long i, V3<T> v) {
  p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z;
}
template <class T> __device__ __forceinline__ bool finite3(V3<T> a) {
  return finiteT(a.x) && finiteT(a.y) && finiteT(a.z);
}

// --------------------------------------------------------------------------
// tangent frame from a vertex normal (site_normals.cuh:69-110)
// --------------------------------------------------------------------------
template <class T> struct Frame { V3<T> u, v; };

template <class T> __device__ __forceinline__ Frame<T> frame_from_normal(V3<T> n) {
  const T tiny = (T)1e-30;
  T inv = divT((T)1, sqrtT(dot3(n, n) + tiny));
  n = {n.x * inv, n.y * inv, n.z * inv};
  V3<T> h = (absT(n.z) > (T)0.9) ? V3<T>{1, 0, 0} : V3<T>{0, 0, 1};
  V3<T> u = cross3(h, n);
  T iu = divT((T)1, sqrtT(dot3(u, u) + tiny));
  u = {u.x * iu, u.y * iu, u.z * iu};
  V3<T> v = cross3(n, u);
  T iv = divT((T)1, sqrtT(dot3(v, v) + tiny));
  v = {v.x * iv, v.y * iv, v.z * iv};
  return {u, v};
}

// --------------------------------------------------------------------------
// PCA normal of a site's neighbourhood (frame option; the reference builds
// every frame from the nearest vertex normal, site_normals.cuh:69-110).
// The eigenvector of the smallest eigenvalue of the covariance C of the
// listed neighbours' offsets, found by power iteration on the adjugate of C,
// which has the same eigenvectors with the order reversed (error shrinks by
// l1 / l2 per step: fast wherever the neighbourhood is a surface patch, even
// a narrow one).  The iteration starts from the reference normal n0 and runs
// a fixed kPcaSteps steps; its sign is then chosen to agree with n0.  Fewer
// than 3 neighbours, a zero spread, or a non-finite result give n0 back.
// Only IEEE-rounded arithmetic with an explicit operation order, so a CPU
// restatement reproduces the bits.
// --------------------------------------------------------------------------
constexpr int kPcaSteps = 8;

template <class T>
__device__ __forceinline__ V3<T> pca_normal(const T* __restrict__ S, long site_base, int n_sites,
                                            const uint32_t* __restrict__ row, int K, V3<T> si, V3<T> n0) {
  T sx = 0, sy = 0, sz = 0, xx = 0, xy = 0, xz = 0, yy = 0, yz = 0, zz = 0;
  int m = 0;
  for (int t = 0; t < K; ++t) {
    const uint32_t j = __ldg(row + t);
    if (j >= (uint32_t)n_sites) continue;
    const V3<T> d = sub3(ld3(S, site_base + (long)j), si);
    sx = sx + d.x; sy = sy + d.y; sz = sz + d.z;
    xx = fmaT(d.x, d.x, xx); xy = fmaT(d.x, d.y, xy); xz = fmaT(d.x, d.z, xz);
    yy = fmaT(d.y, d.y, yy); yz = fmaT(d.y, d.z, yz); zz = fmaT(d.z, d.z, zz);
    ++m;
  }
  if (m < 3) return n0;
  const T im = divT((T)1, (T)m);
  const T mx = sx * im, my = sy * im, mz = sz * im;
  // C = sum d d^T - m mean mean^T = sum d d^T - s mean^T
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
    const T nw = sqrtT(dot3(w, w));
    if (!(nw > (T)1e-30)) return n0;
    const T inv = divT((T)1, nw);
    v = {w.x * inv, w.y * inv, w.z * inv};
  }
  if (!finite3(v)) return n0;
  if (dot3(v, n0) < (T)0) v = {-v.x, -v.y, -v.z};
  return v;
}

// --------------------------------------------------------------------------
// centroid of the clipped polygon (2dClip.cuh:55-80); Neumaier compensation
// in the MIXED profile.
// --------------------------------------------------------------------------
template <class T> struct CSum {
  T s, c;
  __device__ __forceinline__ CSum() : s(0), c(0) {}
  __device__ __forceinline__ void add(T x) {
    T t = s + x;
    if (absT(s) >= absT(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ T get() const { return s + c; }
};

// Polygon accessor: vertex k of the polygon currently held in a buffer.
template <class P, class Buf>
__device__ __forceinline__ V2<P> poly_centroid(const Buf& poly, int n, bool compensated) {
  const P nanv = (P)NAN;
  if (n < 3) return {nanv, nanv};
  P A2, Cx, Cy;
  if (!compensated) {
    A2 = 0; Cx = 0; Cy = 0;
    V2<P> p = poly.get(0);
    for (int i = 0; i < n; ++i) {
      V2<P> q = poly.get(i + 1 == n ? 0 : i + 1);
      P cr = fmaT(p.x, q.y, -(q.x * p.y));
      A2 = A2 + cr;
      Cx = fmaT(p.x + q.x, cr, Cx);
      Cy = fmaT(p.y + q.y, cr, Cy);
      p = q;
    }
  } else {
    CSum<P> a, x, y;
    V2<P> p = poly.get(0);
    for (int i = 0; i < n; ++i) {
      V2<P> q = poly.get(i + 1 == n ? 0 : i + 1);
      P cr = fmaT(p.x, q.y, -(q.x * p.y));
      a.add(cr);
      x.add((p.x + q.x) * cr);
      y.add((p.y + q.y) * cr);
      p = q;
    }
    A2 = a.get(); Cx = x.get(); Cy = y.get();
  }
  P A = (P)0.5 * A2;
  if (absT(A) < (P)1e-18) {
    P mx = 0, my = 0;
    for (int i = 0; i < n; ++i) { V2<P> q = poly.get(i); mx = mx + q.x; my = my + q.y; }
    return {divT(mx, (P)n), divT(my, (P)n)};
  }
  P inv6A = divT((P)1, (P)6 * A);
  return {Cx * inv6A, Cy * inv6A};
}

// --------------------------------------------------------------------------
// closest point on a triangle (near_project.cuh:12-53)
// --------------------------------------------------------------------------
template <class T> __device__ __forceinline__ V3<T> closest_point_tri(V3<T> P, V3<T> A, V3<T> B, V3<T> C) {
  const T e = (T)1e-30;
  V3<T> AB = sub3(B, A), AC = sub3(C, A), AP = sub3(P, A);
  T d1 = dot3(AB, AP), d2 = dot3(AC, AP);
  if (d1 <= 0 && d2 <= 0) return A;
  V3<T> BP = sub3(P, B);
  T d3 = dot3(AB, BP), d4 = dot3(AC, BP);
  if (d3 >= 0 && d4 <= d3) return B;
  T vc = fmaT(d1, d4, -(d3 * d2));
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    T v = divT(d1, (d1 - d3) + e);
    return {fmaT(AB.x, v, A.x), fmaT(AB.y, v, A.y), fmaT(AB.z, v, A.z)};
  }
  V3<T> CP = sub3(P, C);
  T d5 = dot3(AB, CP), d6 = dot3(AC, CP);
  if (d6 >= 0 && d5 <= d6) return C;
  T vb = fmaT(d5, d2, -(d1 * d6));
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    T w = divT(d2, (d2 - d6) + e);
    return {fmaT(AC.x, w, A.x), fmaT(AC.y, w, A.y), fmaT(AC.z, w, A.z)};
  }
  T va = fmaT(d3, d6, -(d5 * d4));
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    T w = divT(d4 - d3, ((d4 - d3) + (d5 - d6)) + e);
    V3<T> BC = sub3(C, B);
    return {fmaT(BC.x, w, B.x), fmaT(BC.y, w, B.y), fmaT(BC.z, w, B.z)};
  }
  T denom = divT((T)1, ((va + vb) + vc) + e);
  T v = vb * denom, w = vc * denom;
  return {A.x + fmaT(AB.x, v, AC.x * w), A.y + fmaT(AB.y, v, AC.y * w), A.z + fmaT(AB.z, v, AC.z * w)};
}

// closest point over the one-rings of the kproj nearest vertices
// (project_centroids_to_mesh, near_project.cuh:149-189).  Q is the
// arithmetic type (double for the MIXED barycentrics).  A face that contains
// an earlier listed vertex was already tested in that vertex's one-ring with
// the same inputs; a repeat can never pass the strict '<', so it is skipped.
template <class T, class Q>
__device__ __forceinline__ V3<T> project_onering(V3<T> c, const float* __restrict__ V, int nV,
                                                 const int* __restrict__ F, int nF,
                                                 const int* __restrict__ off, const int* __restrict__ fcs,
                                                 const int* knnv, int kproj) {
  V3<Q> cq = cvt3<Q>(c), bp = cq;
  Q best = (Q)1e30;
  for (int t = 0; t < kproj; ++t) {
    int v = knnv[t];
    if ((unsigned)v >= (unsigned)nV) continue;
    int beg = __ldg(off + v), end = __ldg(off + v + 1);
    for (int ii = beg; ii < end; ++ii) {
      int fi = __ldg(fcs + ii);
      if ((unsigned)fi >= (unsigned)nF) continue;
      int ia = __ldg(F + 3 * fi), ib = __ldg(F + 3 * fi + 1), ic = __ldg(F + 3 * fi + 2);
      bool seen = false;
      for (int s = 0; s < t; ++s) {
        const int w = knnv[s];
        seen = seen || w == ia || w == ib || w == ic;
      }
      if (seen) continue;
      V3<Q> A = {(Q)__ldg(V + 3 * ia), (Q)__ldg(V + 3 * ia + 1), (Q)__ldg(V + 3 * ia + 2)};
      V3<Q> B = {(Q)__ldg(V + 3 * ib), (Q)__ldg(V + 3 * ib + 1), (Q)__ldg(V + 3 * ib + 2)};
      V3<Q> C = {(Q)__ldg(V + 3 * ic), (Q)__ldg(V + 3 * ic + 1), (Q)__ldg(V + 3 * ic + 2)};
      V3<Q> p = closest_point_tri(cq, A, B, C);
      V3<Q> dd = sub3(p, cq);
      Q d2 = dot3(dd, dd);
      if (d2 < best) { best = d2; bp = p; }
    }
  }
  return cvt3<T>(bp);
}

// One-ring records: for every vertex->face CSR entry (same order as the CSR),
// the face's three corner positions and vertex ids and a bounding sphere in
// four 16-byte words,
//   r0 = {A.x, A.y, A.z, B.x}, r1 = {B.y, B.z, C.x, C.y}, r2 = {C.z, ia, ib, ic},
//   r3 = {centre.x, centre.y, centre.z, radius}
// (ids as int bits), so a projection reads one offset and then independent
// 16-byte loads instead of the chain CSR entry -> face -> corners: r2 and r3
// for every entry, r0 and r1 only for the faces that the shared-vertex and
// sphere tests keep (2 % faster than loading all four up front).  The
// sphere is centred on the float-rounded centroid; its radius is the largest
// corner distance, computed in double and rounded up, so it holds the whole
// triangle.  radius < 0 marks a face the projection never skips: an invalid
// entry, or a triangle with a corner angle below ~5.7 degrees
// (sin^2 < kPruneSin2), whose face-region formula is ill-conditioned.
constexpr int kRingWords = 4;
constexpr double kPruneSin2 = 0.01;

__global__ void k_build_ring_records(const float* __restrict__ V, const int* __restrict__ F, int nF,
                                     const int* __restrict__ fcs, long n_entries, float4* __restrict__ rec) {
  const long ii = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (ii >= n_entries) return;
  const int fi = fcs[ii];
  int ia = -1, ib = -1, ic = -1;
  float a[3] = {0.f, 0.f, 0.f}, b[3] = {0.f, 0.f, 0.f}, c[3] = {0.f, 0.f, 0.f};
  float4 sph = make_float4(0.f, 0.f, 0.f, -1.f);
  if ((unsigned)fi < (unsigned)nF) {
    ia = F[3 * fi]; ib = F[3 * fi + 1]; ic = F[3 * fi + 2];
    for (int k = 0; k < 3; ++k) { a[k] = V[3 * ia + k]; b[k] = V[3 * ib + k]; c[k] = V[3 * ic + k]; }
    float m[3];
    double r2 = 0.0;
    for (int k = 0; k < 3; ++k) m[k] = (float)(((double)a[k] + (double)b[k] + (double)c[k]) / 3.0);
    const float* P[3] = {a, b, c};
    bool ok = true;
    for (int j = 0; j < 3; ++j) {
      double d2 = 0.0, u[3], v[3];
      for (int k = 0; k < 3; ++k) {
        const double d = (double)P[j][k] - (double)m[k];
        d2 += d * d;
        u[k] = (double)P[(j + 1) % 3][k] - (double)P[j][k];
        v[k] = (double)P[(j + 2) % 3][k] - (double)P[j][k];
      }
      r2 = fmax(r2, d2);
      const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
      const double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2], vv = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      ok = ok && (cx * cx + cy * cy + cz * cz) >= kPruneSin2 * (uu * vv);  // false for NaN / zero-length edges
    }
    const float rad = __double2float_ru(sqrt(r2) * (1.0 + 1e-9));
    if (ok && isfinite(rad)) sph = make_float4(m[0], m[1], m[2], rad);
  }
  rec[kRingWords * ii] = make_float4(a[0], a[1], a[2], b[0]);
  rec[kRingWords * ii + 1] = make_float4(b[1], b[2], c[0], c[1]);
  rec[kRingWords * ii + 2] = make_float4(c[2], __int_as_float(ia), __int_as_float(ib), __int_as_float(ic));
  rec[kRingWords * ii + 3] = sph;
}

// project_onering over the one-ring records: the same faces in the same
// order, the same arithmetic, so the same result bit for bit.
//
// A face whose bounding sphere lies so far from c that its computed d2 must
// be >= the best so far cannot pass the strict '<' and is skipped, which
// leaves the result unchanged.  The lower bound on the distance from c to
// any point the closest-point code can return for the face,
//   lb = |c - centre| - radius - 0.05 (|c - centre| + radius)
//        - 1e-4 max|coordinate| - 1e-4 |c - centre|^2 / radius,
// subtracts margins far above the rounding involved: the vertex and edge
// results lie on the triangle up to the rounding of one fma per coordinate
// (edge parameters are in [0, 1] under correct rounding); the face-region
// result errs by about kappa u |AP|^2 / |edge| for kappa = 1/sin^2 <= 100
// (the corner-angle flag), unit roundoff u <= 2^-24 and |AP| <= |c - centre|
// + radius; |c - centre| is computed in FP32 from coordinates of magnitude
// <= max|coordinate|; and the computed d2 is >= (1 - 5u) |p - c|^2.  A face is
// skipped when lb > 0 and lb^2 > 1.001 best.
template <class T, class Q>
__device__ __forceinline__ V3<T> project_onering_rec(V3<T> c, const float4* __restrict__ rec, int nV,
                                                     const int* __restrict__ off, const int* knnv, int kproj) {
  V3<Q> cq = cvt3<Q>(c), bp = cq;
  Q best = (Q)1e30;
  const float qx = (float)c.x, qy = (float)c.y, qz = (float)c.z;
  const float qm = fmaxf(fabsf(qx), fmaxf(fabsf(qy), fabsf(qz)));
  for (int t = 0; t < kproj; ++t) {
    int v = knnv[t];
    if ((unsigned)v >= (unsigned)nV) continue;
    int beg = __ldg(off + v), end = __ldg(off + v + 1);
    for (int ii = beg; ii < end; ++ii) {
      const float4* r = rec + kRingWords * (long)ii;
      // ids and sphere first; the corner words only for faces that are tested
      const float4 r2 = __ldg(r + 2), r3 = __ldg(r + 3);
      const int ia = __float_as_int(r2.y), ib = __float_as_int(r2.z), ic = __float_as_int(r2.w);
      if (ia < 0) continue;
      bool seen = false;
      for (int s = 0; s < t; ++s) {
        const int w = knnv[s];
        seen = seen || w == ia || w == ib || w == ic;
      }
      if (seen) continue;
      if (r3.w >= 0.f) {
        const float dx = qx - r3.x, dy = qy - r3.y, dz = qz - r3.z;
        const float dc = __fsqrt_rn(fmaT(dz, dz, fmaT(dy, dy, dx * dx)));
        const float mc = fmaxf(qm, fmaxf(fabsf(r3.x), fmaxf(fabsf(r3.y), fabsf(r3.z))));
        const float lb = dc - r3.w - 0.05f * (dc + r3.w) - 1e-4f * mc - 1e-4f * divT(dc * dc, r3.w);
        if (lb > 0.f && (double)lb * (double)lb > 1.001 * (double)best) continue;
      }
      const float4 r0 = __ldg(r), r1 = __ldg(r + 1);
      V3<Q> A = {(Q)r0.x, (Q)r0.y, (Q)r0.z};
      V3<Q> B = {(Q)r0.w, (Q)r1.x, (Q)r1.y};
      V3<Q> C = {(Q)r1.z, (Q)r1.w, (Q)r2.x};
      V3<Q> p = closest_point_tri(cq, A, B, C);
      V3<Q> dd = sub3(p, cq);
      Q d2 = dot3(dd, dd);
      if (d2 < best) { best = d2; bp = p; }
    }
  }
  return cvt3<T>(bp);
}

// --------------------------------------------------------------------------
// evaluation primitives (evaluate.cuh:44-104)
// --------------------------------------------------------------------------
// 40-byte BVH node, layout of evaluate.cuh:15-22
struct BVHNode {
  float bmin[3], bmax[3];
  int left, right, triStart, triCount;
};

__device__ __forceinline__ float aabb_d2(V3<float> p, const float* bmin, const float* bmax) {
  float d = 0.f;
  float q[3] = {p.x, p.y, p.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (q[a] < bmin[a]) { float t = bmin[a] - q[a]; d = fmaT(t, t, d); }
    else if (q[a] > bmax[a]) { float t = q[a] - bmax[a]; d = fmaT(t, t, d); }
  }
  return d;
}

__device__ __forceinline__ float point_tri_d2(V3<float> p, V3<float> a, V3<float> b, V3<float> c) {
  V3<float> ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
  float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.f && d2 <= 0.f) return dot3(ap, ap);
  V3<float> bp = sub3(p, b);
  float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.f && d4 <= d3) return dot3(bp, bp);
  float vc = fmaT(d1, d4, -(d3 * d2));
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
    float v = divT(d1, d1 - d3);
    V3<float> pr{fmaT(ab.x, v, a.x), fmaT(ab.y, v, a.y), fmaT(ab.z, v, a.z)};
    V3<float> d = sub3(p, pr);
    return dot3(d, d);
  }
  V3<float> cp = sub3(p, c);
  float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.f && d5 <= d6) return dot3(cp, cp);
  float vb = fmaT(d5, d2, -(d1 * d6));
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
    float w = divT(d2, d2 - d6);
    V3<float> pr{fmaT(ac.x, w, a.x), fmaT(ac.y, w, a.y), fmaT(ac.z, w, a.z)};
    V3<float> d = sub3(p, pr);
    return dot3(d, d);
  }
  float va = fmaT(d3, d6, -(d5 * d4));
  if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
    float w = divT(d4 - d3, (d4 - d3) + (d5 - d6));
    V3<float> bc = sub3(c, b);
    V3<float> pr{fmaT(bc.x, w, b.x), fmaT(bc.y, w, b.y), fmaT(bc.z, w, b.z)};
    V3<float> d = sub3(p, pr);
    return dot3(d, d);
  }
  float denom = divT(1.f, (va + vb) + vc);
  float v = vb * denom, w = vc * denom;
  V3<float> pr{a.x + fmaT(ab.x, v, ac.x * w), a.y + fmaT(ab.y, v, ac.y * w), a.z + fmaT(ab.z, v, ac.z * w)};
  V3<float> d = sub3(p, pr);
  return dot3(d, d);
}

// Traversal stack: at most one pending sibling per level; the median-split
// tree is at most 2 log2(nF) deep.
constexpr int kBvhStack = 96;

// Closest point on the whole mesh through the BVH (projection option; the
// reference projects onto the one-rings of the KPROJ nearest vertices,
// near_project.cuh:149-189).  Near-first traversal; a box is entered only
// when its FP32 squared distance to c is below the best squared distance so
// far, and a face replaces the best only with a strictly smaller squared
// distance, so ties keep the first face met in traversal order.  `best`
// starts at bound2, an upper bound of the answer (the caller's distance to a
// point on the mesh, with margin); if no face beats it the search is rerun
// without the bound.  Q is the barycentric arithmetic type.  The traversal
// order and every comparison are fixed, so a CPU restatement that walks the
// same tree returns the same bits.  A non-finite c is returned unchanged.
template <class T, class Q>
__device__ __forceinline__ V3<T> project_bvh(V3<T> c, const BVHNode* __restrict__ nodes, const int* __restrict__ tri,
                                             const float* __restrict__ V, const int* __restrict__ F, Q bound2,
                                             int* overflow) {
  if (!finite3(c)) return c;
  const V3<Q> cq = cvt3<Q>(c);
  const V3<float> cf = cvt3<float>(c);
  V3<Q> bp = cq;
  int stack[kBvhStack];
  for (int pass = 0; pass < 2; ++pass) {
    Q best = pass == 0 ? bound2 : (Q)1e30;
    bool found = false;
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const BVHNode nd = nodes[stack[--sp]];
      if ((Q)aabb_d2(cf, nd.bmin, nd.bmax) >= best) continue;
      if (nd.triCount > 0) {
        for (int k = 0; k < nd.triCount; ++k) {
          const int t = __ldg(tri + nd.triStart + k);
          const int ia = __ldg(F + 3 * t), ib = __ldg(F + 3 * t + 1), ic = __ldg(F + 3 * t + 2);
          const V3<Q> A = {(Q)__ldg(V + 3 * ia), (Q)__ldg(V + 3 * ia + 1), (Q)__ldg(V + 3 * ia + 2)};
          const V3<Q> B = {(Q)__ldg(V + 3 * ib), (Q)__ldg(V + 3 * ib + 1), (Q)__ldg(V + 3 * ib + 2)};
          const V3<Q> C = {(Q)__ldg(V + 3 * ic), (Q)__ldg(V + 3 * ic + 1), (Q)__ldg(V + 3 * ic + 2)};
          const V3<Q> p = closest_point_tri(cq, A, B, C);
          const V3<Q> dd = sub3(p, cq);
          const Q d2 = dot3(dd, dd);
          if (d2 < best) { best = d2; bp = p; found = true; }
        }
      } else {
        const BVHNode L = nodes[nd.left], R = nodes[nd.right];
        const Q dl = (Q)aabb_d2(cf, L.bmin, L.bmax), dr = (Q)aabb_d2(cf, R.bmin, R.bmax);
        if (sp + 2 > kBvhStack) { atomicAdd(overflow, 1); continue; }
        if (dl < dr) {
          if (dr < best) stack[sp++] = nd.right;
          if (dl < best) stack[sp++] = nd.left;
        } else {
          if (dl < best) stack[sp++] = nd.left;
          if (dr < best) stack[sp++] = nd.right;
        }
      }
    }
    if (found) break;
  }
  return cvt3<T>(bp);
}

// Upper bound of the squared distance from c to the mesh, given a point s on
// the mesh (up to rounding): (|c - s| (1 + 1e-4) + 1e-5 max|coordinate|)^2.
template <class T>
__device__ __forceinline__ double bvh_bound2(V3<T> c, V3<T> s) {
  const double dx = (double)c.x - (double)s.x, dy = (double)c.y - (double)s.y, dz = (double)c.z - (double)s.z;
  const double m = fmax(fmax(fabs((double)s.x), fabs((double)s.y)), fabs((double)s.z));
  const double d = __dsqrt_rn(__fma_rn(dz, dz, __fma_rn(dy, dy, dx * dx))) * 1.0001 + 1e-5 * m;
  return isfinite(d) ? d * d : 1e30;
}

}  // namespace cvt
