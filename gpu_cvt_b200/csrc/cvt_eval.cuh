// Evaluation: BVH traversal over the reference surface and the one-sided Hausdorff
// distance of a candidate mesh (evaluate.cuh:15-383), plus the dual-triangle
// extraction that produces the candidate mesh from the sites
// (near_project.cuh:201-352, buildmesh.cuh:11-241, main.cu:928-974).
#pragma once
#include <algorithm>
#include <vector>
#include "cvt_engine.cuh"

namespace cvt {

// The tree is the reference's (bounds from the triangle boxes, leaf <= 8
// triangles, otherwise the centroid-sorted list split at its middle, nodes in
// pre-order, evaluate.cuh:114-201); it is built on the device, cvt_ingest.cuh.

// Per-probe closest squared distance to the BVH surface.  Near-first
// traversal: of two children the nearer box is visited first, which only
// changes the order, not the minimum (stack: kBvhStack, cvt_math.cuh).

__device__ __forceinline__ float bvh_closest_d2(V3<float> p, const BVHNode* __restrict__ nodes,
                                                const int* __restrict__ tri, const float* __restrict__ V,
                                                const int* __restrict__ F, int* overflow) {
  float best = 1e30f;
  int stack[kBvhStack];
  int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const BVHNode nd = nodes[stack[--sp]];
    if (aabb_d2(p, nd.bmin, nd.bmax) >= best) continue;
    if (nd.triCount > 0) {
      for (int k = 0; k < nd.triCount; ++k) {
        int t = __ldg(tri + nd.triStart + k);
        V3<float> a = ld3(V, __ldg(F + 3 * t)), b = ld3(V, __ldg(F + 3 * t + 1)), c = ld3(V, __ldg(F + 3 * t + 2));
        float d2 = point_tri_d2(p, a, b, c);
        if (d2 < best) best = d2;
      }
    } else {
      const BVHNode L = nodes[nd.left], R = nodes[nd.right];
      float dl = aabb_d2(p, L.bmin, L.bmax), dr = aabb_d2(p, R.bmin, R.bmax);
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
  return best;
}

// probe k of the candidate mesh: vertices, then per face the centroid and
// the three edge midpoints (evaluate.cuh:253-283)
__device__ __forceinline__ V3<float> probe_point(const float* __restrict__ V, int nV, const int* __restrict__ F, long k) {
  if (k < nV) return ld3(V, k);
  long f = (k - nV) >> 2;
  int w = (int)((k - nV) & 3);
  V3<float> a = ld3(V, F[3 * f]), b = ld3(V, F[3 * f + 1]), c = ld3(V, F[3 * f + 2]);
  const float third = 1.0f / 3.0f;
  if (w == 0) return {(a.x + (b.x + c.x)) * third, (a.y + (b.y + c.y)) * third, (a.z + (b.z + c.z)) * third};
  if (w == 1) return {(a.x + b.x) * 0.5f, (a.y + b.y) * 0.5f, (a.z + b.z) * 0.5f};
  if (w == 2) return {(b.x + c.x) * 0.5f, (b.y + c.y) * 0.5f, (b.z + c.z) * 0.5f};
  return {(c.x + a.x) * 0.5f, (c.y + a.y) * 0.5f, (c.z + a.z) * 0.5f};
}

// max over probes of the closest squared distance, reduced in-kernel:
// warp max, then one atomicMax on the float bits (non-negative floats
// order as unsigned ints) -- replaces the CUB max of evaluate.cuh:335-343.
__global__ void __launch_bounds__(128) k_hausdorff(const float* __restrict__ Vc, int nVc, const int* __restrict__ Fc,
                                                   long nP, const BVHNode* __restrict__ nodes, const int* __restrict__ tri,
                                                   const float* __restrict__ Vr, const int* __restrict__ Fr,
                                                   unsigned* out_bits, int* overflow) {
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  float d = 0.f;
  if (k < nP) d = bvh_closest_d2(probe_point(Vc, nVc, Fc, k), nodes, tri, Vr, Fr, overflow);
  unsigned b = __float_as_uint(d);
  b = __reduce_max_sync(0xffffffffu, b);
  if ((threadIdx.x & 31) == 0) atomicMax(out_bits, b);
}

// ---------------------------------------------------------------------------
// dual-triangle extraction
// ---------------------------------------------------------------------------
constexpr int kFaceMaxPoly = 256;   // MAX_POLY (main.cu:393)

// Labelled clip (near_project.cuh:201-244) + active-bisector pairs
// (near_project.cuh:318-351) + key emission (buildmesh.cuh:170-201) per site.
// Buffers: per thread 2 x kFaceMaxPoly float2 + labels in local memory.
__global__ void __launch_bounds__(64) k_face_keys(const float* __restrict__ S, const float* __restrict__ U,
                                                  const float* __restrict__ Vv, const uint32_t* __restrict__ knn,
                                                  int n, int K, float R2, float eps_clip, float tol_active,
                                                  unsigned long long* keys, int* key_count, int max_keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float2 bufA[kFaceMaxPoly], bufB[kFaceMaxPoly];
  int labA[kFaceMaxPoly], labB[kFaceMaxPoly];
  float2* cp = bufA; float2* np = bufB;
  int* cl = labA; int* nl = labB;
  int na = 4;
  cp[0] = make_float2(-R2, -R2); cp[1] = make_float2(R2, -R2); cp[2] = make_float2(R2, R2); cp[3] = make_float2(-R2, R2);
  cl[0] = cl[1] = cl[2] = cl[3] = -1;
  const V3<float> si = ld3(S, i), ui = ld3(U, i), vi = ld3(Vv, i);
  const uint32_t* nb = knn + (size_t)i * K;
  for (int t = 0; t < K; ++t) {
    int j = (int)nb[t];
    if ((unsigned)j >= (unsigned)n || j == i) continue;
    V3<float> d = sub3(ld3(S, j), si);
    float a = dot3(d, ui), b = dot3(d, vi), c = 0.5f * dot3(d, d);
    int m = 0;
    if (na > 0) {
      float2 s = cp[na - 1];
      float fs = fmaT(a, s.x, fmaT(b, s.y, -c));
      for (int k = 0; k < na; ++k) {
        float2 e = cp[k];
        int le = cl[k];
        float fe = fmaT(a, e.x, fmaT(b, e.y, -c));
        bool ins_e = fe <= eps_clip, ins_s = fs <= eps_clip;
        if (ins_e) {
          if (!ins_s && m < kFaceMaxPoly) {
            float tt = divT(fs, (fs - fe) + 1e-30f);
            np[m] = make_float2(fmaT(tt, e.x - s.x, s.x), fmaT(tt, e.y - s.y, s.y)); nl[m] = j; m++;
          }
          if (m < kFaceMaxPoly) { np[m] = e; nl[m] = le; m++; }
        } else if (ins_s && m < kFaceMaxPoly) {
          float tt = divT(fs, (fs - fe) + 1e-30f);
          np[m] = make_float2(fmaT(tt, e.x - s.x, s.x), fmaT(tt, e.y - s.y, s.y)); nl[m] = j; m++;
        }
        s = e; fs = fe;
      }
    }
    na = m;
    float2* tp = cp; cp = np; np = tp;
    int* tl = cl; cl = nl; nl = tl;
    if (na == 0) break;
  }
  if (na < 3) return;
  for (int k = 0; k < na; ++k) {
    float2 p = cp[k];
    float b1 = 1e30f, b2 = 1e30f;
    int j1 = -1, j2 = -1;
    for (int t = 0; t < K; ++t) {
      int j = (int)nb[t];
      if ((unsigned)j >= (unsigned)n || j == i) continue;
      V3<float> d = sub3(ld3(S, j), si);
      float a = dot3(d, ui), b = dot3(d, vi), c = 0.5f * dot3(d, d);
      float s = fabsf(fmaT(a, p.x, fmaT(b, p.y, -c)));
      if (s < b1) { b2 = b1; j2 = j1; b1 = s; j1 = j; }
      else if (s < b2) { b2 = s; j2 = j; }
    }
    if (!(j1 >= 0 && j2 >= 0 && j1 != j2 && b1 <= tol_active && b2 <= tol_active)) continue;
    int x = i, y = j1, z = j2, tmp;
    if (x > y) { tmp = x; x = y; y = tmp; }
    if (y > z) { tmp = y; y = z; z = tmp; }
    if (x > y) { tmp = x; x = y; y = tmp; }
    int pos = atomicAdd(key_count, 1);
    if (pos < max_keys)
      keys[pos] = (unsigned long long)(uint32_t)x | ((unsigned long long)(uint32_t)y << 21) |
                  ((unsigned long long)(uint32_t)z << 42);
  }
}

}  // namespace cvt

namespace cvt {

// decode the sorted unique keys (buildmesh.cuh:99-109) and drop degenerate
// triangles (buildmesh.cuh:225-241, eps 1e-6); flags[k] = keep
__global__ void k_face_decode(const unsigned long long* __restrict__ keys, int nk, const float* __restrict__ S, int n,
                              float eps, int* __restrict__ tri, int* __restrict__ keep) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk) return;
  unsigned long long key = keys[k];
  int a = (int)(key & 0x1FFFFFull), b = (int)((key >> 21) & 0x1FFFFFull), c = (int)((key >> 42) & 0x1FFFFFull);
  bool deg = (a == b || b == c || a == c) || a >= n || b >= n || c >= n;
  if (!deg) {
    V3<float> A = ld3(S, a), B = ld3(S, b), C = ld3(S, c);
    V3<float> e0 = sub3(B, A), e1 = sub3(C, B), e2 = sub3(A, C);
    float l0 = sqrtT(dot3(e0, e0)), l1 = sqrtT(dot3(e1, e1)), l2 = sqrtT(dot3(e2, e2));
    V3<float> cr = cross3(sub3(B, A), sub3(C, A));
    float ar = sqrtT(dot3(cr, cr));
    deg = !(l0 > eps && l1 > eps && l2 > eps && ar > eps);
  }
  tri[3 * k] = a; tri[3 * k + 1] = b; tri[3 * k + 2] = c;
  keep[k] = deg ? 0 : 1;
}

__global__ void k_face_compact(const int* __restrict__ tri, const int* __restrict__ keep, const int* __restrict__ pos,
                               int nk, int* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nk || !keep[k]) return;
  int p = pos[k];
  out[3 * p] = tri[3 * k]; out[3 * p + 1] = tri[3 * k + 1]; out[3 * p + 2] = tri[3 * k + 2];
}

// quality metrics (evaluate.cuh:388-462) as a device reduction: acc[0] Qsum,
// acc[1] min-angle sum, acc[2] #angles < 30, acc[3] #angles > 90 (doubles);
// mins[0] Qmin bits, mins[1] theta_min bits (non-negative floats as uint)
__global__ void k_quality(const float* __restrict__ V, const int* __restrict__ F, int nF, double* acc, unsigned* mins) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  double q = 0.0, th = 0.0, lt = 0.0, gt = 0.0;
  float qmin = 3.0e38f, tmin = 3.0e38f;
  if (f < nF) {
    V3<float> a = ld3(V, F[3 * f]), b = ld3(V, F[3 * f + 1]), c = ld3(V, F[3 * f + 2]);
    V3<float> ab = sub3(b, a), ac = sub3(c, a), ba = sub3(a, b), bc = sub3(c, b), ca = sub3(a, c), cb = sub3(b, c);
    auto ang = [](V3<float> u, V3<float> v) {
      float du = sqrtT(dot3(u, u)), dv = sqrtT(dot3(v, v));
      float den = fmaxf(du * dv, 1e-30f);
      float cs = divT(dot3(u, v), den);
      cs = fminf(1.f, fmaxf(-1.f, cs));
      return acosf(cs) * (180.0f / 3.14159265358979323846f);
    };
    float A = ang(ab, ac), B = ang(ba, bc), Cc = ang(ca, cb);
    tmin = fminf(A, fminf(B, Cc));
    th = tmin;
    lt = (A < 30.f) + (B < 30.f) + (Cc < 30.f);
    gt = (A > 90.f) + (B > 90.f) + (Cc > 90.f);
    float l0 = sqrtT(dot3(ab, ab)), l1 = sqrtT(dot3(bc, bc)), l2 = sqrtT(dot3(ca, ca));
    V3<float> cr = cross3(ab, ac);
    float area = 0.5f * sqrtT(dot3(cr, cr));
    float s = 0.5f * ((l0 + l1) + l2);
    float e = fmaxf(l0, fmaxf(l1, l2));
    float den = fmaxf(s * e, 1e-30f);
    float qq = divT(6.0f, sqrtT(3.0f)) * divT(area, den);
    qmin = qq;
    q = qq;
  }
  for (int o = 16; o; o >>= 1) {
    q += __shfl_xor_sync(0xffffffffu, q, o);
    th += __shfl_xor_sync(0xffffffffu, th, o);
    lt += __shfl_xor_sync(0xffffffffu, lt, o);
    gt += __shfl_xor_sync(0xffffffffu, gt, o);
    qmin = fminf(qmin, __shfl_xor_sync(0xffffffffu, qmin, o));
    tmin = fminf(tmin, __shfl_xor_sync(0xffffffffu, tmin, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc + 0, q); atomicAdd(acc + 1, th); atomicAdd(acc + 2, lt); atomicAdd(acc + 3, gt);
    atomicMin(mins + 0, __float_as_uint(qmin));
    atomicMin(mins + 1, __float_as_uint(tmin));
  }
}

}  // namespace cvt
