// Stage-API kernels: one kernel (family) per reference stage, operating on
// caller-owned device buffers in the reference's layouts.  They share the
// device routines of the fused engine.
#pragma once
#include "cvt_engine.cuh"

namespace cvt {

// ---------------------------------------------------------------------------
// grid over an arbitrary device point set (geometry chosen on the device)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int f2ord(float v) {
  int b = __float_as_int(v);
  return b >= 0 ? b : b ^ 0x7fffffff;
}
__device__ __forceinline__ float ord2f(int o) {
  int b = o >= 0 ? o : o ^ 0x7fffffff;
  return __int_as_float(b);
}

__global__ void k_bbox_init(int* bb) {
  if (threadIdx.x < 3) { bb[threadIdx.x] = 0x7fffffff; bb[3 + threadIdx.x] = (int)0x80000000; }
}

__global__ void k_bbox(int n, const float* __restrict__ P, int* bb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float v[3] = {INFINITY, INFINITY, INFINITY};
  float w[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (i < n) {
    float x = P[3 * i], y = P[3 * i + 1], z = P[3 * i + 2];
    if (isfinite(x) && isfinite(y) && isfinite(z)) { v[0] = w[0] = x; v[1] = w[1] = y; v[2] = w[2] = z; }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float mn = v[a], mx = w[a];
    for (int o = 16; o; o >>= 1) {
      mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0 && isfinite(mn)) {
      atomicMin(bb + a, f2ord(mn));
      atomicMax(bb + 3 + a, f2ord(mx));
    }
  }
}

// Geometry for ~`per_cell` points per occupied cell on a surface, at most
// max_cells spatial cells.
__global__ void k_grid_geom(const int* bb, int n, float per_cell, int max_cells, GridGeom* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  float lo[3], hi[3];
  bool any = bb[0] != 0x7fffffff;
  for (int a = 0; a < 3; ++a) {
    lo[a] = any ? ord2f(bb[a]) : 0.f;
    hi[a] = any ? ord2f(bb[3 + a]) : 1.f;
  }
  float ext[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  float emax = fmaxf(fmaxf(ext[0], ext[1]), fmaxf(ext[2], 1e-20f));
  double area = 2.0 * ((double)ext[0] * ext[1] + (double)ext[1] * ext[2] + (double)ext[0] * ext[2]) + 1e-30;
  double h = sqrt(area * per_cell / (double)max(n, 1));
  h = fmax(h, (double)emax / 1024.0);
  GridGeom g;
  for (int it = 0; it < 64; ++it) {
    long long prod = 1;
    for (int a = 0; a < 3; ++a) {
      g.dim[a] = max(1, (int)ceil(((double)ext[a] + 2e-6 * emax) / h));
      prod *= g.dim[a];
    }
    if (prod <= max_cells) break;
    h *= 1.0 + fmax(0.05, cbrt((double)prod / (double)max_cells) - 1.0);
  }
  for (int a = 0; a < 3; ++a) g.lo[a] = lo[a] - 1e-6f * emax;
  g.h = (float)h;
  g.inv_h = (float)(1.0 / h);
  g.cell_base = 0;
  g.ncell = g.dim[0] * g.dim[1] * g.dim[2];
  *out = g;
}

// ---------------------------------------------------------------------------
// stage KNN kernels
// ---------------------------------------------------------------------------
template <int KK>
__global__ void __launch_bounds__(128) k_stage_knn_points(const GridGeom* geom, const int* __restrict__ cell_start,
                                                          const Pt4<float>* __restrict__ sorted, int total_cells,
                                                          const uint8_t* frozen, int kk, uint32_t* knn, float* dist) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n_grid = __ldg(cell_start + total_cells);
  if (t >= n_grid) return;
  const Pt4<float> me = sorted[t];
  const int g = (int)me.id;
  if (frozen && frozen[g]) return;
  TopK<float, KK> top;
  const GridGeom G = *geom;
  grid_knn<float, float, KK>(G, cell_start, sorted, V3<float>{me.x, me.y, me.z}, top, [](uint32_t) { return true; });
#pragma unroll
  for (int k = 0; k < KK; ++k) {
    if (k >= kk) break;
    knn[(size_t)g * kk + k] = KeyOps<float>::idx(top.k[k]);
    if (dist) dist[(size_t)g * kk + k] = KeyOps<float>::dist(top.k[k]);
  }
}

// queries are separate points; out_int != 0 writes int (-1 for missing)
template <int KK>
__global__ void __launch_bounds__(128) k_stage_knn_query(const GridGeom* geom, const int* __restrict__ cell_start,
                                                         const Pt4<float>* __restrict__ sorted, const float* __restrict__ Q,
                                                         int nQ, const uint8_t* frozen, int kk, int exclude_self,
                                                         uint32_t* knn, float* dist) {
  const int qi = blockIdx.x * blockDim.x + threadIdx.x;
  if (qi >= nQ) return;
  if (frozen && frozen[qi]) return;
  TopK<float, KK> top;
  const GridGeom G = *geom;
  const int skip = exclude_self ? qi : -1;
  grid_knn<float, float, KK>(G, cell_start, sorted, ld3(Q, qi), top, [skip](uint32_t id) { return (int)id != skip; });
#pragma unroll
  for (int k = 0; k < KK; ++k) {
    if (k >= kk) break;
    knn[(size_t)qi * kk + k] = KeyOps<float>::idx(top.k[k]);
    if (dist) dist[(size_t)qi * kk + k] = KeyOps<float>::dist(top.k[k]);
  }
}

__global__ void k_stage_drop_self(const uint32_t* __restrict__ in, int n, int kin, int kout, uint32_t* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* s = in + (size_t)i * kin;
  uint32_t* d = out + (size_t)i * kout;
  int w = 0;
  for (int t = 0; t < kin && w < kout; ++t) {
    uint32_t j = s[t];
    if ((int)j == i) continue;
    d[w++] = j;
  }
  if (w == 0) {
    for (int k = 0; k < kout; ++k) d[k] = (uint32_t)i;
  } else {
    uint32_t fill = d[w - 1];
    for (; w < kout; ++w) d[w] = fill;
  }
}

__global__ void k_stage_restore_rows(const uint8_t* __restrict__ frozen, const uint32_t* __restrict__ prev,
                                     uint32_t* __restrict__ cur, int n, int k) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !frozen[i]) return;
  for (int a = 0; a < k; ++a) cur[(size_t)i * k + a] = prev[(size_t)i * k + a];
}

// area-weighted vertex normals, summed in face order per vertex
__global__ void k_stage_normals(const float* __restrict__ V, int nV, const int* __restrict__ F,
                                const int* __restrict__ off, const int* __restrict__ fcs, float* __restrict__ N) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nV) return;
  V3<float> acc{0.f, 0.f, 0.f};
  for (int k = off[v]; k < off[v + 1]; ++k) {
    int f = fcs[k];
    V3<float> a = ld3(V, F[3 * f]), b = ld3(V, F[3 * f + 1]), c = ld3(V, F[3 * f + 2]);
    V3<float> fn = cross3(sub3(b, a), sub3(c, a));
    acc = {acc.x + fn.x, acc.y + fn.y, acc.z + fn.z};
  }
  float l2 = dot3(acc, acc);
  if (l2 > 0.f) {
    float inv = divT(1.0f, sqrtT(l2));
    acc = {acc.x * inv, acc.y * inv, acc.z * inv};
  }
  st3(N, v, acc);
}

__global__ void k_stage_frames(const float* __restrict__ N0, const int* __restrict__ knnV, int kproj, int n,
                               float* __restrict__ U, float* __restrict__ Vv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int nn = knnV[(size_t)i * kproj];
  if (nn < 0) { st3(U, i, V3<float>{1, 0, 0}); st3(Vv, i, V3<float>{0, 1, 0}); return; }
  Frame<float> fr = frame_from_normal(ld3(N0, nn));
  st3(U, i, fr.u);
  st3(Vv, i, fr.v);
}

// frames from the PCA normal of each site's listed neighbours (pca_normal),
// started from the normal of the vertex knnV[i * kproj] -- the frame option
// of the engine (frame_mode 1)
__global__ void k_stage_frames_pca(const float* __restrict__ S, int n, const uint32_t* __restrict__ knn, int K,
                                   const float* __restrict__ N0, const int* __restrict__ knnV, int kproj,
                                   float* __restrict__ U, float* __restrict__ Vv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int nn = knnV[(size_t)i * kproj];
  if (nn < 0) { st3(U, i, V3<float>{1, 0, 0}); st3(Vv, i, V3<float>{0, 1, 0}); return; }
  const V3<float> nrm = pca_normal<float>(S, 0, n, knn + (size_t)i * K, K, ld3(S, i), ld3(N0, nn));
  Frame<float> fr = frame_from_normal(nrm);
  st3(U, i, fr.u);
  st3(Vv, i, fr.v);
}

// clip + centroid for every site; overflowing polygons go to the fallback
template <int PROF, int BLOCK, int CAP>
__global__ void __launch_bounds__(BLOCK) k_stage_clip(const float* __restrict__ S, const float* __restrict__ U,
                                                      const float* __restrict__ Vv, const uint32_t* __restrict__ knn,
                                                      int n, int K, float R, float* __restrict__ cent, int* nverts,
                                                      int* ovf) {
  using PP = typename PT<PROF>::PP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V2<PP>* sm = reinterpret_cast<V2<PP>*>(smem_raw);
  PolyRef<PP> A{sm + threadIdx.x, BLOCK}, B{sm + CAP * BLOCK + threadIdx.x, BLOCK};
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n) return;
  V3<float> si = ld3(S, i);
  Frame<float> fr{ld3(U, i), ld3(Vv, i)};
  PolyRef<PP> cur = A, nxt = B;
  int np = clip_cell<PROF>(S, 0, n, si, knn + (size_t)i * K, K, fr, R, cur, nxt, CAP, false);
  if (np < 0) {
    int k = atomicAdd(ovf, 1);
    ovf[1 + k] = i;
    return;
  }
  V2<PP> c2 = poly_centroid<PP>(cur, np, PROF == PROF_MIXED);
  V3<float> c;
  if (!(finiteT(c2.x) && finiteT(c2.y))) c = {NAN, NAN, NAN};
  else {
    float cx = (float)c2.x, cy = (float)c2.y;
    c = {si.x + fmaT(fr.u.x, cx, fr.v.x * cy), si.y + fmaT(fr.u.y, cx, fr.v.y * cy), si.z + fmaT(fr.u.z, cx, fr.v.z * cy)};
  }
  st3(cent, i, c);
  if (nverts) nverts[i] = np;
}

template <int PROF>
__global__ void __launch_bounds__(64) k_stage_clip_fallback(const float* __restrict__ S, const float* __restrict__ U,
                                                            const float* __restrict__ Vv, const uint32_t* __restrict__ knn,
                                                            int n, int K, float R, float* __restrict__ cent, int* nverts,
                                                            const int* ovf) {
  using PP = typename PT<PROF>::PP;
  V2<PP> buf[2][kFallbackCap];
  const int cnt = *ovf;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    const int i = ovf[1 + k];
    V3<float> si = ld3(S, i);
    Frame<float> fr{ld3(U, i), ld3(Vv, i)};
    PolyRef<PP> cur{buf[0], 1}, nxt{buf[1], 1};
    int np = clip_cell<PROF>(S, 0, n, si, knn + (size_t)i * K, K, fr, R, cur, nxt, kFallbackCap, false);
    V2<PP> c2 = poly_centroid<PP>(cur, np, PROF == PROF_MIXED);
    V3<float> c;
    if (!(finiteT(c2.x) && finiteT(c2.y))) c = {NAN, NAN, NAN};
    else {
      float cx = (float)c2.x, cy = (float)c2.y;
      c = {si.x + fmaT(fr.u.x, cx, fr.v.x * cy), si.y + fmaT(fr.u.y, cx, fr.v.y * cy), si.z + fmaT(fr.u.z, cx, fr.v.z * cy)};
    }
    st3(cent, i, c);
    if (nverts) nverts[i] = np;
  }
}

template <int PROF>
__global__ void k_stage_project(const float* __restrict__ cent, const float* __restrict__ V, const int* __restrict__ F,
                                const int* __restrict__ off, const int* __restrict__ fcs, const int* __restrict__ knnV,
                                int kproj, int nV, int nF, int nQ, const float* __restrict__ Sold, float* __restrict__ Snew) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nQ) return;
  V3<float> c = ld3(cent, i);
  if (PROF == PROF_MIXED && !finite3(c)) { st3(Snew, i, ld3(Sold, i)); return; }
  int kv[16];
  for (int t = 0; t < kproj && t < 16; ++t) kv[t] = knnV[(size_t)i * kproj + t];
  V3<float> r = (PROF == PROF_REF) ? project_onering<float, float>(c, V, nV, F, nF, off, fcs, kv, min(kproj, 16))
                                   : project_onering<float, double>(c, V, nV, F, nF, off, fcs, kv, min(kproj, 16));
  st3(Snew, i, r);
}

// exact closest point on the mesh through its BVH (project_bvh), the
// projection option of the engine (proj_mode 1); Sold (may be NULL) bounds
// the search and, in MIXED, replaces a non-finite centroid
template <int PROF>
__global__ void k_stage_project_bvh(const float* __restrict__ cent, int nQ, const BVHNode* __restrict__ nodes,
                                    const int* __restrict__ tri, const float* __restrict__ V, const int* __restrict__ F,
                                    const float* __restrict__ Sold, float* __restrict__ Snew, int* ovf) {
  using Q = typename PT<PROF>::Q;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nQ) return;
  V3<float> c = ld3(cent, i);
  if (PROF == PROF_MIXED && !finite3(c)) { st3(Snew, i, ld3(Sold, i)); return; }
  const Q bound2 = Sold ? (Q)bvh_bound2(c, ld3(Sold, i)) : (Q)1e30;
  st3(Snew, i, project_bvh<float, Q>(c, nodes, tri, V, F, bound2, ovf));
}

struct FreezeTable { float thr2[6]; int need[6]; };

__global__ void k_stage_freeze(const float* __restrict__ S, const float* __restrict__ Snew,
                               const uint32_t* __restrict__ knn, const uint32_t* __restrict__ prev, int n, int K,
                               int has_prev, const uint8_t* __restrict__ tier, FreezeTable tab, uint8_t* streak,
                               uint8_t* cand, uint8_t* frozen, int* counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int same = 0, low = 0, both = 0, newly = 0;
  if (i < n) {
    if (!has_prev) {
      streak[i] = 0;
      cand[i] = 0;
    } else {
      int t = tier ? min((int)tier[i], 5) : 0;
      bool sm = true;
      for (int j = 0; j < K; ++j)
        if (knn[(size_t)i * K + j] != prev[(size_t)i * K + j]) { sm = false; break; }
      bool lw = dist2(ld3(Snew, i), ld3(S, i)) <= tab.thr2[t];
      bool bt = sm && lw;
      int s = streak[i];
      s = bt ? (s < 255 ? s + 1 : s) : 0;
      streak[i] = (uint8_t)s;
      uint8_t c = (s >= tab.need[t]) ? 1 : 0;
      cand[i] = c;
      same = sm; low = lw; both = bt;
      if (c && !frozen[i]) { frozen[i] = 1; newly = 1; }
    }
  }
  const unsigned full = 0xffffffffu;
  int a = __popc(__ballot_sync(full, same)), b = __popc(__ballot_sync(full, low));
  int c = __popc(__ballot_sync(full, both)), d = __popc(__ballot_sync(full, newly));
  if ((threadIdx.x & 31) == 0) {
    if (a) atomicAdd(counts + 0, a);
    if (b) atomicAdd(counts + 1, b);
    if (c) atomicAdd(counts + 2, c);
    if (d) atomicAdd(counts + 3, d);
  }
}

__global__ void k_stage_count_frozen(const uint8_t* __restrict__ frozen, int n, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int v = (i < n && frozen[i]) ? 1 : 0;
  int c = __popc(__ballot_sync(0xffffffffu, v));
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void k_stage_tiers(int mode, int n, int K, const float* __restrict__ sn, const uint32_t* __restrict__ knn,
                              uint8_t* __restrict__ tier) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  auto normal = [&](int j, float out[3]) { out[0] = sn[3 * j]; out[1] = sn[3 * j + 1]; out[2] = sn[3 * j + 2]; };
  tier[i] = (uint8_t)tier_of(mode, i, n, K, knn + (size_t)i * K, normal);
}

}  // namespace cvt
