// Fused Lloyd-iteration kernels over many (mesh, site set) segments.
//
// One iteration (main.cu:669-881 per segment) is:
//   grid build over the sites of active segments (count -> scan -> scatter)
//   k_active_list  the non-frozen sites
//   k_frame_vertex the mesh vertex nearest to each of them (its normal
//                gives the frame, main.cu:685-700), on a second stream
//                while the site KNN runs
//   k_knn_verify per active site (one warp): the K-list from the site's
//                candidate list where its motion bound proves it exact
//   k_knn_search the other active sites (one warp each): exact (K+1)-NN in
//                the segment, drop self (site_knn.cuh:79), by one radius
//                query where a bound is known, else ring by ring; frozen
//                sites keep the previous list (main.cu:678)
//   k_site_clip  per site (one thread): frame (site_normals.cuh:69; or,
//                as an option, from the PCA normal of the neighbours),
//                tangent-plane clip and centroid (2dClip.cuh:82)
//   k_clip_overflow  the same for the rare cells whose polygon outgrows
//                the shared-memory buffer (exact 64-vertex cap)
//   k_site_vsearch per site (one thread): centroid -> 5 nearest vertices
//                (main.cu:719-735, frozen sites keep theirs)
//   k_site_proj  per site (one thread): one-ring projection over those
//                vertices (near_project.cuh:149; or, as an
//                option, the exact closest point through the BVH), freeze test
//                and apply (freezetest.cuh:155-212, 270-327, 451-466),
//                tier assignment on the segment's first iteration
//                (main.cu:640-667)
//   k_site_far   the sites whose centroid lies so far off the surface that
//                the vertex grid search gave up: exact brute-force 5-NN by
//                a block, then the rest of the step
//   (bookkeeping) per-segment iteration counters / statistics slots, run by
//                the last block of k_site_far
// All sizes come from device memory, so the whole iteration is captured once
// in a CUDA graph and relaunched while segments come and go.
#pragma once
#include "cvt_grid.cuh"

namespace cvt {

constexpr int kStatsRing = 256;   // iterations of per-segment statistics kept
constexpr int kStatsWords = 8;    // same, low, both, newly, maxdisp2 bits, iter, KNN lists reused, searched
constexpr int kKProj = 5;         // KPROJ (main.cu:394)
// Largest box (in vertex-grid cells) a bounded vertex query visits before it
// leaves the site to the ring search: ring 1's 27 cells.
constexpr int kVertexBoxCells = 27;
constexpr int kFallbackCap = 66;  // 64-vertex reference cap + room for the overshoot
// threads per SM that k_site_clip's launch bounds ask to keep resident: it
// caps registers near 80 (6 blocks of 128 with 32 KB of polygon buffers each
// for FP32 polygons, 6 of 64 for FP64 ones) whatever the block size
constexpr int kClipThreadsF = 768;
constexpr int kClipThreadsD = 384;

struct MeshDev {
  const float* V;
  const int* F;
  const int* vf_off;
  const int* vf_faces;
  const float* N;
  const int* vcell_start;
  const Pt4<float>* vsorted;
  const float4* ring;  // one-ring records, kRingWords per CSR entry (k_build_ring_records)
  const BVHNode* bvh;  // BVH over the faces (built before a segment that projects through it is placed)
  const int* bvh_tri;
  GridGeom vg;
  int nV, nF;
  float R;     // clip square half-size: longest input bbox edge (main.cu:421)
  float thr2;  // freeze displacement threshold, squared (main.cu:431)
};

struct SegDev {
  int mesh;       // index into the mesh table
  int site_base;  // first global site index
  int n_sites;
  int mode;       // 0 / 1 / 2
  int ex_quirk;
  int iter;       // iterations completed (device-side count)
  float kth_est;  // first-iteration estimate of the K-th neighbour's squared distance
  float stop_motion2;  // stop once an iteration's max squared motion <= this (< 0: never)
  int stop_iters;      // stop after this many iterations (0: never)
  float thr2_tier[6];
  int need_tier[6];
  float step_motion;   // largest site motion of the segment's last iteration
};

template <int PROF> struct PT;
template <> struct PT<PROF_REF> { using T = float; using Q = float; using PP = float; };
template <> struct PT<PROF_MIXED> { using T = float; using Q = double; using PP = float; };
template <> struct PT<PROF_FP64> { using T = double; using Q = double; using PP = double; };

template <class T> struct EngineArgs {
  const SegDev* segs;
  const GridGeom* geom;
  const int* active;      // 0 free, 1 iterating, 2 stopped by its stop rule
  const MeshDev* meshes;
  const int* site_seg;
  T* S[2];
  uint32_t* knn;      // K neighbours per site (local indices), the current list
  uint8_t* same;      // list unchanged vs the previous iteration (site KNN kernel)
  float* kth;         // last K-th neighbour's squared distance per site, < 0 unknown
  int* act;           // sorted positions of the sites whose list is recomputed
  int* act_count;
  int* knnv;
  int* nnv;
  uint8_t* frozen;
  uint8_t* streak;
  uint8_t* tier;
  const int* cell_start;
  const Pt4<T>* sorted;
  int total_cells;
  int* stats;
  int* ovf;  // [0] = count, [1 + k] = overflowed site
  int* far;  // [0] = count, [1 + k] = site whose vertex search was deferred
  T* cent;   // centroid per site (3 values), k_site_clip -> k_site_proj
  int K;
  int proj_mode;  // 0: one-ring of the KPROJ nearest vertices; 1: closest point through the BVH
  int* bvh_ovf;   // BVH traversal stack overflows (never expected: the tree depth is bounded)
  uint32_t* cand;    // candidate list per site (global ids), MM entries (k_knn_verify / k_knn_search)
  float* cand_rho;   // its MM-th distance when it was built, rounded down (< 0: no list; inf: every other site)
  float* cand_D;     // motion bound accumulated since it was built (k_knn_verify)
  int* srch;         // per verify warp: srch_cap slots of sorted positions left for a full search
  float* srch_thr;   // per slot: squared distance that the site's MM nearest lie within (< 0: unknown)
  int* srch_n;       // per verify warp: slots used
  int srch_cap;
  unsigned long long* blockmax;  // per coarse block (cell slots of the segment): iteration << 32 | max motion bits
};

__device__ __forceinline__ float f32_ru(float x) { return x; }
__device__ __forceinline__ float f32_ru(double x) { return __double2float_ru(x); }
__device__ __forceinline__ float f32_rd(float x) { return x; }
__device__ __forceinline__ float f32_rd(double x) { return __double2float_rd(x); }

// Coarse motion blocks of a segment: kBlockCells^3 grid cells, stored in the
// first cells of the segment's cell range (there are fewer blocks than
// cells).  Positions outside the grid fall in the edge blocks, like cells.
// Larger blocks make the step condition looser but take the maximum motion
// over more sites (measured: 4 cells kept more lists than 3 cells of a grid
// sized for the candidate list's length).
constexpr int kBlockCells = 4;
__device__ __forceinline__ int block_dim(const GridGeom& g, int a) { return (g.dim[a] + kBlockCells - 1) / kBlockCells; }

template <class T>
__device__ __forceinline__ int motion_block(const GridGeom& g, V3<T> p, int& bx, int& by, int& bz) {
  bx = grid_coord(g, p.x, 0) / kBlockCells; by = grid_coord(g, p.y, 1) / kBlockCells;
  bz = grid_coord(g, p.z, 2) / kBlockCells;
  return g.cell_base + (bz * block_dim(g, 1) + by) * block_dim(g, 0) + bx;
}

// polygon storage: vertex k at p[k * stride] (shared memory: thread-
// interleaved; local memory: stride 1)
template <class PP> struct PolyRef {
  V2<PP>* p;
  int stride;
  __device__ __forceinline__ V2<PP> get(int k) const { return p[k * stride]; }
  __device__ __forceinline__ void set(int k, V2<PP> v) const { p[k * stride] = v; }
};

// Sutherland-Hodgman clip by a*x + b*y - c <= eps (2dClip.cuh:11-53).  Stops
// with ovf = true before writing vertex `cap` (buffer full); keeps the
// reference's 64-vertex cap (2dClip.cuh:47-50) for larger buffers.  r2 returns
// the largest squared vertex radius of the output (NaN if any vertex is NaN).
template <class PP, class Q>
__device__ __forceinline__ int clip_poly(const PolyRef<PP>& in, int n, const PolyRef<PP>& out, Q a, Q b, Q c,
                                         Q eps, int cap, bool& ovf, Q& r2) {
  r2 = (Q)0;
  if (n <= 0) return 0;
  auto f = [&](V2<PP> p) -> Q { return fmaT(a, (Q)p.x, fmaT(b, (Q)p.y, -c)); };
  auto isect = [&](V2<PP> s, V2<PP> e, Q fs, Q fe) -> V2<PP> {
    Q t = divT(fs, (fs - fe) + (Q)1e-30);
    return {(PP)fmaT(t, (Q)e.x - (Q)s.x, (Q)s.x), (PP)fmaT(t, (Q)e.y - (Q)s.y, (Q)s.y)};
  };
  auto put = [&](int k, V2<PP> v) {
    out.set(k, v);
    const Q q = fmaT((Q)v.y, (Q)v.y, (Q)v.x * (Q)v.x);
    r2 = (q > r2 || q != q) ? q : r2;
  };
  V2<PP> s = in.get(n - 1);
  Q fs = f(s);
  bool ins_s = fs <= eps;
  int m = 0;
  for (int i = 0; i < n; ++i) {
    V2<PP> e = in.get(i);
    Q fe = f(e);
    bool ins_e = fe <= eps;
    if (ins_e) {
      if (!ins_s) {
        if (m >= cap) { ovf = true; return m; }
        put(m++, isect(s, e, fs, fe));
      }
      if (m >= cap) { ovf = true; return m; }
      put(m++, e);
    } else if (ins_s) {
      if (m >= cap) { ovf = true; return m; }
      put(m++, isect(s, e, fs, fe));
    }
    s = e; fs = fe; ins_s = ins_e;
    if (m >= 64) { m = 64; break; }
  }
  return m;
}

// True when the half-plane a*x + b*y <= c holds, as the clip's predicate
// computes it, at every point within sqrt(r2) of the origin: then clipping
// by it returns the polygon unchanged (same vertices, same order) and can be
// skipped.  By Cauchy-Schwarz a*x + b*y <= sqrt((a^2+b^2) r2); the 1e-4
// relative margin covers the rounding of this test (a few ulp) and of the
// predicate fma(a, x, fma(b, y, -c)) (< 2 ulp of c), so the skip is exact.
// c > 1e-18 keeps the products away from underflow.  NaN fails the test.
template <class Q>
__device__ __forceinline__ bool halfplane_contains_disk(Q a, Q b, Q c, Q r2) {
  return c > (Q)1e-18 && fmaT(a, a, b * b) * r2 * (Q)1.0001 < c * c;
}

// Clip the square [-R,R]^2 by the bisectors of the listed neighbours; returns
// the vertex count (polygon in `cur` on return) or -1 on buffer overflow.
//
// Security radius: a bisector whose half-plane contains the disk around the
// site that holds the current polygon cannot cut it and is skipped
// (halfplane_contains_disk).  When the row is this iteration's K-nearest list
// of the same positions (ascending distance), every later neighbour j has
// |d_j| >= |d_t|; the tangent-plane normal of its bisector is at most |d_j|
// long and its offset is |d_j|^2/2, so once |d_t|^2 > 4 r2 (with a 1e-3
// margin for the distance keys' rounding) none of the remaining bisectors can
// cut the polygon and the loop ends.  Both shortcuts only leave out clips
// that would return their input unchanged: the result is the same bit for
// bit as clipping by all K bisectors.
template <int PROF>
__device__ __forceinline__ int clip_cell(const typename PT<PROF>::T* __restrict__ S, int site_base, int n_sites,
                                         V3<typename PT<PROF>::T> si, const uint32_t* __restrict__ row, int K,
                                         const Frame<typename PT<PROF>::T>& fr, float R,
                                         PolyRef<typename PT<PROF>::PP>& cur, PolyRef<typename PT<PROF>::PP>& nxt,
                                         int cap, bool row_sorted) {
  using T = typename PT<PROF>::T;
  using Q = typename PT<PROF>::Q;
  using PP = typename PT<PROF>::PP;
  const PP r = (PP)R;
  cur.set(0, {-r, -r}); cur.set(1, {r, -r}); cur.set(2, {r, r}); cur.set(3, {-r, r});
  int n = 4;
  Q r2 = (Q)2 * (Q)r * (Q)r * (Q)1.0001;
  bool ovf = false;
  // the next neighbour's position is loaded while the current one clips
  uint32_t jn = __ldg(row);
  V3<T> sn = jn < (uint32_t)n_sites ? ld3(S, (long)site_base + jn) : si;
  // Every lane runs all K trips; a finished lane only skips their bodies.  A
  // data-dependent `break` lets lanes leave at different trips, and the warp
  // then runs the rest of the site's work in fragments (measured 2x slower).
  bool done = false;
  for (int t = 0; t < K; ++t) {
    if (done) continue;
    const uint32_t j = jn;
    const V3<T> sj = sn;
    if (t + 1 < K) {
      jn = __ldg(row + t + 1);
      if (jn < (uint32_t)n_sites) sn = ld3(S, (long)site_base + jn);
    }
    if (j >= (uint32_t)n_sites) continue;
    Q a, b, c;
    if (PROF == PROF_MIXED) {
      V3<double> d{(double)sj.x - (double)si.x, (double)sj.y - (double)si.y, (double)sj.z - (double)si.z};
      V3<double> u = cvt3<double>(fr.u), v = cvt3<double>(fr.v);
      a = (Q)dot3(d, u); b = (Q)dot3(d, v); c = (Q)(0.5 * dot3(d, d));
    } else {
      V3<T> d = sub3(sj, si);
      a = (Q)dot3(d, fr.u); b = (Q)dot3(d, fr.v); c = (Q)((T)0.5 * dot3(d, d));
    }
    if (halfplane_contains_disk(a, b, c, r2)) {
      done = row_sorted && c > (Q)1e-18 && (Q)2.002 * r2 < c;
      continue;
    }
    n = clip_poly<PP, Q>(cur, n, nxt, a, b, c, (Q)1e-12, cap, ovf, r2);
    if (ovf) { n = -1; done = true; continue; }
    PolyRef<PP> tmp = cur; cur = nxt; nxt = tmp;
    if (n == 0) done = true;
  }
  return n;
}

// ---------------------------------------------------------------------------
// tiers (main.cu:18-150) in FP64, identical operation order to the host code
// ---------------------------------------------------------------------------
__device__ inline void sym3_eigenvalues_d(const double C[9], double lam[3]) {
  double v[3] = {1.0, 0.0, 0.0};
  for (int it = 0; it < 20; ++it) {
    double w[3] = {C[0] * v[0] + C[1] * v[1] + C[2] * v[2], C[3] * v[0] + C[4] * v[1] + C[5] * v[2],
                   C[6] * v[0] + C[7] * v[1] + C[8] * v[2]};
    double n = __dsqrt_rn(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    if (n < 1e-30) break;
    v[0] = __ddiv_rn(w[0], n); v[1] = __ddiv_rn(w[1], n); v[2] = __ddiv_rn(w[2], n);
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
    double n = __dsqrt_rn(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    if (n < 1e-30) break;
    v2[0] = __ddiv_rn(w[0], n); v2[1] = __ddiv_rn(w[1], n); v2[2] = __ddiv_rn(w[2], n);
  }
  lam[1] = v2[0] * (C2[0] * v2[0] + C2[1] * v2[1] + C2[2] * v2[2]) + v2[1] * (C2[3] * v2[0] + C2[4] * v2[1] + C2[5] * v2[2]) +
           v2[2] * (C2[6] * v2[0] + C2[7] * v2[1] + C2[8] * v2[2]);
  lam[2] = C[0] + C[4] + C[8] - lam[0] - lam[1];
}

// normal(i) gives the unit normal of local site i as float[3]
template <class NormalOf>
__device__ inline int tier_of(int mode, int i, int n, int K, const uint32_t* row, NormalOf normal) {
  const double TH[4] = {0.15, 0.35, 0.55, 0.80};
  float ni[3];
  normal(i, ni);
  double sum = 0.0;
  int cnt = 0;
  for (int j = 0; j < K; ++j) {
    int jj = (int)row[j];
    if (jj < 0 || jj >= n) continue;
    float nj[3];
    normal(jj, nj);
    double c = (double)ni[0] * (double)nj[0] + (double)ni[1] * (double)nj[1] + (double)ni[2] * (double)nj[2];
    if (c > 1.0) c = 1.0;
    if (c < -1.0) c = -1.0;
    sum += c;
    cnt++;
  }
  double nv = cnt > 0 ? (1.0 - __ddiv_rn(sum, (double)cnt)) : 0.0;
  double L = 0.0;
  if (mode == 2) {
    double mean[3] = {0, 0, 0};
    int c2 = 0;
    for (int j = 0; j < K; ++j) {
      int jj = (int)row[j];
      if (jj < 0 || jj >= n) continue;
      float nj[3];
      normal(jj, nj);
      for (int a = 0; a < 3; ++a) mean[a] += (double)nj[a];
      c2++;
    }
    if (c2 >= 2) {
      for (int a = 0; a < 3; ++a) mean[a] = __ddiv_rn(mean[a], (double)c2);
      double C[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int j = 0; j < K; ++j) {
        int jj = (int)row[j];
        if (jj < 0 || jj >= n) continue;
        float nj[3];
        normal(jj, nj);
        double d[3] = {(double)nj[0] - mean[0], (double)nj[1] - mean[1], (double)nj[2] - mean[2]};
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) C[3 * r + c] += d[r] * d[c];
      }
      double lam[3];
      sym3_eigenvalues_d(C, lam);
      double tmp;
      if (lam[0] > lam[1]) { tmp = lam[0]; lam[0] = lam[1]; lam[1] = tmp; }
      if (lam[1] > lam[2]) { tmp = lam[1]; lam[1] = lam[2]; lam[2] = tmp; }
      if (lam[0] > lam[1]) { tmp = lam[0]; lam[0] = lam[1]; lam[1] = tmp; }
      if (lam[2] > 1e-30) L = __ddiv_rn(lam[2] - lam[1], lam[2]);
    }
  }
  int t = 0;
  while (t < 4 && nv >= TH[t]) t++;
  if (mode == 2 && t == 4 && L > 0.80) t = 5;
  return t;
}

// ---------------------------------------------------------------------------
// k_active_list: sorted positions of the sites whose neighbour list is
// recomputed this iteration (frozen sites keep theirs, main.cu:678).  The
// append is aggregated per block (one atomic per block, not per warp: the
// per-warp atomics on one counter serialised the kernel), which keeps each
// block's active sites together and in sorted order.
// ---------------------------------------------------------------------------
constexpr int kActiveListThreads = 256;

template <class T>
__global__ void __launch_bounds__(kActiveListThreads) k_active_list(EngineArgs<T> a) {
  __shared__ int warp_base[kActiveListThreads / 32];
  __shared__ int block_base;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n_grid = __ldg(a.cell_start + a.total_cells);
  bool act = false;
  if (t < n_grid) {
    const int g = (int)a.sorted[t].id;
    const SegDev& sd = a.segs[__ldg(a.site_seg + g)];
    act = !(sd.mode != 0 && a.frozen[g]);
  }
  const unsigned m = __ballot_sync(0xffffffffu, act);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) warp_base[wid] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    int sum = 0;
    for (int w = 0; w < kActiveListThreads / 32; ++w) {
      const int c = warp_base[w];
      warp_base[w] = sum;
      sum += c;
    }
    block_base = sum ? atomicAdd(a.act_count, sum) : 0;
  }
  __syncthreads();
  if (act) a.act[block_base + warp_base[wid] + __popc(m & ((1u << lane) - 1u))] = t;
}

// ---------------------------------------------------------------------------
// k_frame_vertex: each listed site's nearest mesh vertex (the frame vertex,
// main.cu:685-700), one thread per site, in the same key order as any other
// search, so the same vertex.  The site's vertex of the last iteration is
// at the squared distance thr from its new position, so the nearest vertex
// lies in the box of cells within sqrt(thr): a few cells, against the 27 of
// the ring search, which runs when there is no such vertex or the box is
// larger.  Runs on a second stream while the site KNN runs; k_site_clip is
// the first kernel to read a.nnv.
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_frame_vertex(EngineArgs<T> a) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= __ldg(a.act_count)) return;
  const Pt4<T> me = a.sorted[a.act[w]];
  const int g = (int)me.id;
  const MeshDev& md = a.meshes[a.segs[__ldg(a.site_seg + g)].mesh];
  const V3<T> q{me.x, me.y, me.z};
  auto all = [](uint32_t) { return true; };
  TopK<T, 1> nv;
  const int old = a.nnv[g];
  bool done = false;
  if ((unsigned)old < (unsigned)md.nV) {
    const V3<T> pv{(T)__ldg(md.V + 3 * old), (T)__ldg(md.V + 3 * old + 1), (T)__ldg(md.V + 3 * old + 2)};
    const T thr = dist2(pv, q);
    const float qm = fmaxf(fabsf((float)q.x), fmaxf(fabsf((float)q.y), fabsf((float)q.z)));
    const float rad = __fsqrt_ru(f32_ru(thr)) * 1.0001f + 1e-3f * md.vg.h + 4e-7f * qm;
    done = grid_knn_box<T, float, 1>(md.vg, md.vcell_start, md.vsorted, q, thr, rad, nv, all, kVertexBoxCells);
    if (!done) nv = TopK<T, 1>();
  }
  if (!done) grid_knn<T, float, 1>(md.vg, md.vcell_start, md.vsorted, q, nv, all);
  a.nnv[g] = (int)KeyOps<T>::idx(nv.k[0]);
}

// ---------------------------------------------------------------------------
// Site KNN (k_knn_verify + k_knn_search): exact K nearest other sites
// within the site's segment (the reference's K+1 nearest with self dropped,
// site_knn.cuh:79-103), one warp per site; lane j holds the j-th neighbour,
// so the list row is read (for the freeze test's equality) and written
// coalesced.  Sets same[g] (new list == stored list) and kth[g].
// ---------------------------------------------------------------------------
// Candidate lists (MM > 0): besides its K neighbours, a site keeps the MM
// nearest other sites of its last full search (ids and the MM-th squared
// distance r2b = rho^2) and a bound D on how much closer any other site can
// have come since.  Every iteration adds to D the site's own last motion and
// the largest last motion of any site in the 8 coarse blocks (kBlockCells^3
// cells each, edge B = kBlockCells h) nearest the site's old position, which
// reach at least B/2 beyond it on every side.  A site j outside the list
// started at distance >= rho; while it starts a step within B/2 of site i
// its step is among those counted, and from farther it cannot end the step
// within rho as long as (largest motion of the step in the segment) + (i's
// motion) < B/2 - rho, which every iteration checks.  So when the K-th nearest
// of the re-keyed list is closer than rho - D, no site outside the list is
// closer: the list's first K are exactly the K nearest of all, the keys a
// full search returns, at a fraction of its work.  Otherwise (and in a
// segment's first iteration) the full search runs for MM neighbours and
// refreshes the list.  Margins of 1e-4 cover the rounding of the distances
// and of the accumulated motion; a NaN motion fails every test.
// The K-list of site g: lane j holds entry j (its key); writes the list
// (local indices; only entries that changed), the K-th squared distance
// (the next search's bound) and the `same` flag (list unchanged).
template <class T, int KK>
__device__ __forceinline__ void knn_store(const EngineArgs<T>& a, int g, const SegDev& sd,
                                          typename KeyOps<T>::Key key, int lane) {
  using O = KeyOps<T>;
  const auto kth = shfl_key(key, KK - 1);
  if (lane == 0) a.kth[g] = O::is_empty(kth) ? -1.f : (float)O::dist(kth);
  const uint32_t gid = O::idx(key);
  const uint32_t out = gid == 0xffffffffu ? 0xffffffffu : gid - (uint32_t)sd.site_base;
  uint32_t* row = a.knn + (size_t)g * KK;
  bool diff = false;
  if (lane < KK) {
    diff = row[lane] != out;
    if (diff) row[lane] = out;
  }
  const unsigned changed = __ballot_sync(0xffffffffu, diff);
  if (lane == 0) a.same[g] = changed ? 0 : 1;
}

// Full search of the site at sorted position t (one warp): the K nearest
// (MM = 0), or the MM nearest, which refresh its candidate list and whose
// first K are the K-list.  seg receives the site's segment.  With candidate
// lists the search is first tried as one radius query (warp_radius_knn,
// scratch buf of 64 keys): within bound tb when the check left one (the
// largest re-keyed distance of the site's complete old list, so at least MM
// sites lie within it), else within a squared distance expected to hold
// about (MM + 64) / 2 sites; when the count falls outside [MM, 64] the ring
// search runs instead.  Both return the MM smallest (distance, index) keys.
template <class T, int KK, int MM>
__device__ __forceinline__ void knn_search_site(const EngineArgs<T>& a, int t, float tb, int lane, int& seg,
                                                typename KeyOps<T>::Key* buf) {
  using O = KeyOps<T>;
  using Key = typename O::Key;
  const Pt4<T> me = a.sorted[t];
  const int g = (int)me.id;
  const int s = __ldg(a.site_seg + g);
  seg = s;
  const SegDev& sd = a.segs[s];
  // The K nearest other sites: the reference's K+1 nearest with self dropped
  // (site_knn.cuh:79-103) are exactly these, also when duplicates of the site
  // with smaller indices push self out of the K+1 (then the first K are kept,
  // the same K points), and the K-th distance equals the (K+1)-th with self.
  const V3<T> q{me.x, me.y, me.z};
  const float kp = a.kth[g];
  const uint32_t self = (uint32_t)g;
  auto not_self = [self](uint32_t id) { return id != self; };
  Key key;
  if constexpr (MM > 0) {
    static_assert(MM <= 64, "at most 64 candidates");
    Key mk[2];
    const float rho = a.cand_rho[g];
    const GridGeom G = a.geom[s];
    // kth holds the site's last K-th squared distance (K sites within it);
    // kth_est, from the segment's density, is expected to hold 2 (K + 1)
    constexpr double kTarget = (MM + 64) / 2.0;
    const T thr_r = tb >= 0.f ? (T)tb
                    : kp >= 0.f ? (T)kp * (T)(kTarget / KK) : (T)sd.kth_est * (T)(kTarget / (2.0 * (KK + 1)));
    const float qm = fmaxf(fabsf((float)q.x), fmaxf(fabsf((float)q.y), fabsf((float)q.z)));
    const float rad = __fsqrt_ru(f32_ru(thr_r)) * 1.0001f + 1e-3f * G.h + 4e-7f * qm;
    if (!warp_radius_knn<T, T, MM>(G, a.cell_start, a.sorted, q, thr_r, rad, lane, not_self, buf, mk)) {
      const T thrM = tb >= 0.f ? (T)tb
                     : rho >= 0.f && !isinf(rho) ? (T)rho * (T)rho * (T)1.2
                     : (kp >= 0.f ? (T)kp * (T)(1.1 * (MM + 1) / (KK + 1)) : (T)sd.kth_est * (T)((MM + 1.0) / (KK + 1)));
      if constexpr (MM > 32) {
        warp_knn<T, T, MM>(G, a.cell_start, a.sorted, q, thrM, lane, not_self, mk);
      } else {
        Key one[1];
        warp_knn<T, T, MM>(G, a.cell_start, a.sorted, q, thrM, lane, not_self, one);
        mk[0] = one[0];
        mk[1] = O::empty();
      }
    }
#pragma unroll
    for (int r = 0; r < 2; ++r)
      if (32 * r + lane < MM) a.cand[(size_t)g * MM + 32 * r + lane] = O::idx(mk[r]);
    const Key mth = shfl_key(mk[(MM - 1) / 32], (MM - 1) % 32);
    if (lane == 0) {
      a.cand_rho[g] = O::is_empty(mth) ? __int_as_float(0x7f800000) : __fsqrt_rd(f32_rd(O::dist(mth)));
      a.cand_D[g] = 0.f;
    }
    key = mk[0];
  } else {
    (void)tb; (void)buf;
    // candidates beyond 1.1x the last K-th squared distance are skipped; sites
    // move little between iterations, and a bound that proves too tight
    // restarts the search without it (swept 1.02-1.5: 1.05-1.1 fastest)
    const T thr0 = kp >= 0.f ? (T)kp * (T)1.1 : (T)sd.kth_est;
    Key kl[1];
    warp_knn<T, T, KK>(a.geom[s], a.cell_start, a.sorted, q, thr0, lane, not_self, kl);
    key = kl[0];
  }
  knn_store<T, KK>(a, g, sd, key, lane);
}

// Candidate-list check of active site w by a half warp (16 lanes, one site
// each half, three list entries per lane: element e = 3 hl + r), so a warp
// checks two sites at once.  The motion bound D grows by the largest last
// motion M in the 8 coarse blocks nearest the site's old position (lanes
// hl < 8 read one block each), which hold every site that started the step
// within B/2 of it, plus the site's own motion; the step condition asks
// that the segment's largest motion plus the site's own stay below
// B/2 - rho (B/2 shrunk by 1e-3 for the rounding of cell coordinates), so a
// site that started the step outside those blocks ends it beyond rho.  The list is re-keyed at the current positions and its
// KK smallest selected in order (half_select3); it is accepted when the
// KK-th is closer than rho - D.  `valid`: this half has a site.  Every lane
// runs every warp-wide step; true when the half's K-list came from the list
// (and is stored: row entries that changed, kth, same, the list's new
// order, D).  bound: for a site whose complete list was re-keyed, the
// largest re-keyed squared distance rounded up (its MM list sites are MM
// other sites, so the MM nearest lie within it); else -1.
template <class T, int KK, int MM>
__device__ __forceinline__ bool knn_verify_half(const EngineArgs<T>& a, int parity, int w, bool valid, int lane,
                                                int& seg, float& bound) {
  static_assert(KK <= 32 && MM > KK && MM <= 48, "candidate list of KK < MM <= 48 entries");
  using O = KeyOps<T>;
  using Key = typename O::Key;
  const int hl = lane & 15, half = lane >> 4;
  const unsigned hmask = 0xffffu << (16 * half);
  int g = -1, s = -1;
  float rho = -1.f;
  V3<T> q{0, 0, 0};
  if (valid) {
    const Pt4<T> me = a.sorted[a.act[w]];
    g = (int)me.id;
    s = __ldg(a.site_seg + g);
    rho = a.cand_rho[g];
    q = {me.x, me.y, me.z};
  }
  seg = s;
  const bool have = valid && rho >= 0.f;
  bool ok = have;
  // motion bound: lanes hl and hl + 16 < 27 read blocks
  unsigned mbits = 0u;
  float D = 0.f, lim = 0.f;
  if (ok) {
    const SegDev& sd = a.segs[s];
    const GridGeom G = a.geom[s];
    // the 2 x 2 x 2 blocks nearest the old position: per axis the block of
    // its cell and the neighbour on the side of the nearer block face, which
    // reach at least kBlockCells / 2 cells beyond the cell on either side
    const V3<T> po = ld3(a.S[parity ^ 1], g);
    const int c0[3] = {grid_coord(G, po.x, 0), grid_coord(G, po.y, 1), grid_coord(G, po.z, 2)};
    int b0[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) b0[ax] = c0[ax] / kBlockCells - (c0[ax] % kBlockCells < kBlockCells / 2 ? 1 : 0);
    const int dx = block_dim(G, 0), dy = block_dim(G, 1), dz = block_dim(G, 2);
    if (hl < 8) {
      const int x = b0[0] + (hl & 1), y = b0[1] + ((hl >> 1) & 1), z = b0[2] + (hl >> 2);
      if (x >= 0 && x < dx && y >= 0 && y < dy && z >= 0 && z < dz) {
        const unsigned long long v = a.blockmax[G.cell_base + (z * dy + y) * dx + x];
        if ((unsigned)(v >> 32) == (unsigned)(sd.iter - 1)) mbits = (unsigned)v;
      }
    }
    mbits = __reduce_max_sync(hmask, mbits);
    // this site's own motion (also inside M, but usually far below it)
    const float mu = __fsqrt_rn(f32_ru(dist2(q, ld3(a.S[parity ^ 1], g)))) * 1.000001f;
    D = __fadd_ru(a.cand_D[g], __fadd_ru(__uint_as_float(mbits), mu));
    const bool step_ok = __fadd_ru(sd.step_motion, mu) * 1.0001f < (0.4995f * (float)kBlockCells * G.h - rho) * 0.9999f;
    lim = rho * 0.9999f - D * 1.0001f;
    ok = isinf(rho) || (step_ok && lim > 0.f);
  }
  // re-key and select (both halves take part in every pass)
  Key k[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    const int e = 3 * hl + r;
    k[r] = O::empty();
    if (have && e < MM) {
      const uint32_t id = __ldg(a.cand + (size_t)g * MM + e);
      if (id != 0xffffffffu) k[r] = O::make(dist2(ld3(a.S[parity], (long)id), q), id);
    }
  }
  bool moved;
  half_select3<T, KK>(k, hl, half, moved);
  constexpr int KL = (KK - 1) / 3, KR = (KK - 1) % 3;
  const Key kth = shfl16_key(k[KR], KL);
  {
    T dm = (T)0;
    int nv = 0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
      if (!O::is_empty(k[r])) { const T d = O::dist(k[r]); dm = d > dm ? d : dm; ++nv; }
#pragma unroll
    for (int o = 8; o >= 1; o >>= 1) {
      const T od = __shfl_xor_sync(0xffffffffu, dm, o, 16);
      dm = od > dm ? od : dm;
      nv += __shfl_xor_sync(0xffffffffu, nv, o, 16);
    }
    bound = have && nv == MM ? f32_ru(dm) : -1.f;
  }
  ok = ok && !O::is_empty(kth) && (isinf(rho) || f32_ru(O::dist(kth)) * 1.0003f < lim * lim);
  // store (per half: entries e < KK of this lane, the flags by lane hl 0)
  bool diff = false;
  if (ok) {
    const uint32_t base = (uint32_t)a.segs[s].site_base;
    uint32_t* row = a.knn + (size_t)g * KK;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const int e = 3 * hl + r;
      if (moved && e < MM) a.cand[(size_t)g * MM + e] = O::idx(k[r]);
      if (e < KK) {
        const uint32_t gid = O::idx(k[r]);
        const uint32_t out = gid == 0xffffffffu ? 0xffffffffu : gid - base;
        if (row[e] != out) { row[e] = out; diff = true; }
      }
    }
    if (hl == 0) { a.cand_D[g] = D; a.kth[g] = (float)O::dist(kth); }
  }
  const unsigned changed = __ballot_sync(0xffffffffu, diff) & hmask;
  if (ok && hl == 0) a.same[g] = changed ? 0 : 1;
  return ok;
}

// Per-warp running count of one statistics word for the segment it is on:
// added to the segment's slot when the segment changes and at the end.
template <class T>
struct SegCounter {
  int cur = -1, n = 0;
  // `lane` 0 adds for the whole warp (or half warp: pass its lane within the half)
  __device__ __forceinline__ void add(const EngineArgs<T>& a, int seg, int word, int lane) {
    if (seg != cur) { flush(a, word, lane); cur = seg; n = 0; }
    ++n;
  }
  __device__ __forceinline__ void flush(const EngineArgs<T>& a, int word, int lane) {
    if (lane == 0 && cur >= 0 && n)
      atomicAdd(a.stats + ((size_t)cur * kStatsRing + (a.segs[cur].iter % kStatsRing)) * kStatsWords + word, n);
  }
};

// Site KNN, two persistent kernels, each launched with the warps its launch
// bounds keep resident on every SM (so no block waits for a second wave):
// k_knn_verify's warp i takes active positions i, i + nw, i + 2 nw, ...,
// takes each site's K-list from its candidate list where the motion bound
// proves it exact, and appends the other sites to its own part of a.srch
// (no atomics: every verify warp owns a.srch_cap slots); k_knn_search's warp
// j searches, in full, the sites of verify warps j, j + nws, ...  Without
// candidate lists (MM = 0) only k_knn_search runs, over every active site.
// The reused lists and the full searches are added to the segments'
// statistics (words 6 and 7 of the iteration's slot).
constexpr int kKnnVerifyWarpsPerSM = 48;
constexpr int kKnnSearchWarpsPerSM = 32;

template <class T, int KK, int MM, int BS>
__global__ void __launch_bounds__(BS, kKnnVerifyWarpsPerSM * 32 / BS) k_knn_verify(EngineArgs<T> a, int parity) {
  const int lane = threadIdx.x & 31;
  const int wi = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
  const int n = __ldg(a.act_count);
  int* mine = a.srch + (size_t)wi * a.srch_cap;
  float* mine_thr = a.srch_thr + (size_t)wi * a.srch_cap;
  int cnt = 0;
  SegCounter<T> reused;  // per half, kept by lanes 0 and 16
  const int hl = lane & 15, half = lane >> 4;
  // two sites per warp: the halves take positions 2i + half, 2i + half + 2 nw, ...
  for (int w0 = 2 * wi; w0 < n; w0 += 2 * nw) {
    const int w = w0 + half;
    int seg;
    float bound;
    const bool ok = knn_verify_half<T, KK, MM>(a, parity, w, w < n, lane, seg, bound);
    const bool need = w < n && !ok;
    if (ok) reused.add(a, seg, 6, hl);
    // the warp's list: half 0's site first, then half 1's
    const unsigned b = __ballot_sync(0xffffffffu, need && hl == 0);
    if (need && hl == 0) {
      const int slot = cnt + (half ? (int)(b & 1u) : 0);
      mine[slot] = a.act[w];
      mine_thr[slot] = bound;
    }
    cnt += __popc(b);
  }
  reused.flush(a, 6, hl);
  if (lane == 0) a.srch_n[wi] = cnt;
}

template <class T, int KK, int MM, int BS>
__global__ void __launch_bounds__(BS, kKnnSearchWarpsPerSM * 32 / BS) k_knn_search(EngineArgs<T> a, int parity,
                                                                                   int n_lists) {
  (void)parity;
  const int lane = threadIdx.x & 31;
  const int wi = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
  SegCounter<T> searched;
  if constexpr (MM > 0) {
    __shared__ typename KeyOps<T>::Key buf[BS / 32][64];  // per warp: the radius query's keys
    auto* mybuf = buf[threadIdx.x >> 5];
    for (int l = wi; l < n_lists; l += nw) {
      const int* list = a.srch + (size_t)l * a.srch_cap;
      const float* thr = a.srch_thr + (size_t)l * a.srch_cap;
      const int n = a.srch_n[l];
      for (int k = 0; k < n; ++k) {
        int seg;
        knn_search_site<T, KK, MM>(a, list[k], thr[k], lane, seg, mybuf);
        searched.add(a, seg, 7, lane);
      }
    }
  } else {
    const int n = __ldg(a.act_count);
    for (int w = wi; w < n; w += nw) {
      int seg;
      knn_search_site<T, KK, MM>(a, a.act[w], -1.f, lane, seg, nullptr);
      searched.add(a, seg, 7, lane);
    }
  }
  searched.flush(a, 7, lane);
}

// ---------------------------------------------------------------------------
// per-site step after the KNN
// ---------------------------------------------------------------------------
struct SiteOut {
  int seg;
  int same, low, both, newly;
  float disp2;
};

// Frame, clip and centroid of site g into a.cent; false when the polygon
// outgrew the buffers (the site is then redone by k_clip_overflow).
template <int PROF, int FRAME>
__device__ __forceinline__ bool site_clip(const EngineArgs<typename PT<PROF>::T>& a, int parity, int g,
                                          PolyRef<typename PT<PROF>::PP> A, PolyRef<typename PT<PROF>::PP> B,
                                          int cap) {
  using T = typename PT<PROF>::T;
  using PP = typename PT<PROF>::PP;
  const int s = __ldg(a.site_seg + g);
  const SegDev& sd = a.segs[s];
  const MeshDev& md = a.meshes[sd.mesh];
  const T* __restrict__ S = a.S[parity];
  const bool fz = sd.mode != 0 && a.frozen[g];
  const V3<T> si = ld3(S, g);
  // frame from the nearest vertex normal (frozen sites: their kept vertex
  // list; with the BVH projection, which keeps no vertex list, their kept
  // frame vertex); FRAME 1: from the PCA normal of the neighbour list,
  // started from that vertex normal
  const int nn = (fz && a.proj_mode == 0) ? a.knnv[(size_t)g * kKProj] : a.nnv[g];
  Frame<T> fr;
  if (nn < 0) {
    fr = {{(T)1, (T)0, (T)0}, {(T)0, (T)1, (T)0}};
  } else {
    V3<T> n0{(T)__ldg(md.N + 3 * nn), (T)__ldg(md.N + 3 * nn + 1), (T)__ldg(md.N + 3 * nn + 2)};
    if (FRAME == 1) n0 = pca_normal(S, sd.site_base, sd.n_sites, a.knn + (size_t)g * a.K, a.K, si, n0);
    fr = frame_from_normal(n0);
  }
  PolyRef<PP> cur = A, nxt = B;
  const int np = clip_cell<PROF>(S, sd.site_base, sd.n_sites, si, a.knn + (size_t)g * a.K, a.K, fr, md.R, cur, nxt,
                                 cap, !fz);
  if (np < 0) return false;
  const V2<PP> c2 = poly_centroid<PP>(cur, np, PROF == PROF_MIXED);
  V3<T> cent;
  if (!(finiteT(c2.x) && finiteT(c2.y))) {
    cent = {(T)NAN, (T)NAN, (T)NAN};
  } else {
    const T cx = (T)c2.x, cy = (T)c2.y;
    cent = {si.x + fmaT(fr.u.x, cx, fr.v.x * cy), si.y + fmaT(fr.u.y, cx, fr.v.y * cy),
            si.z + fmaT(fr.u.z, cx, fr.v.z * cy)};
  }
  st3(a.cent, g, cent);
  return true;
}

template <int PROF, int BLOCK, int CAP, int FRAME>
__global__ void __launch_bounds__(BLOCK, (sizeof(typename PT<PROF>::PP) == 8 ? kClipThreadsD : kClipThreadsF) / BLOCK)
    k_site_clip(EngineArgs<typename PT<PROF>::T> a, int parity) {
  using PP = typename PT<PROF>::PP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V2<PP>* sm = reinterpret_cast<V2<PP>*>(smem_raw);
  PolyRef<PP> A{sm + threadIdx.x, BLOCK}, B{sm + CAP * BLOCK + threadIdx.x, BLOCK};
  const int t = blockIdx.x * BLOCK + threadIdx.x;
  const int n_grid = __ldg(a.cell_start + a.total_cells);
  if (t < n_grid) {
    const int g = (int)a.sorted[t].id;
    if (!site_clip<PROF, FRAME>(a, parity, g, A, B, CAP)) {
      const int k = atomicAdd(a.ovf, 1);
      a.ovf[1 + k] = g;
    }
  }
}

template <int PROF, int FRAME>
__global__ void __launch_bounds__(64) k_clip_overflow(EngineArgs<typename PT<PROF>::T> a, int parity) {
  using PP = typename PT<PROF>::PP;
  V2<PP> buf[2][kFallbackCap];
  const int n = *(volatile int*)a.ovf;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    site_clip<PROF, FRAME>(a, parity, a.ovf[1 + k], PolyRef<PP>{buf[0], 1}, PolyRef<PP>{buf[1], 1}, kFallbackCap);
}

// Projection, tiers and the freeze test of site g, given the centroid in
// a.cent and (PROJ 0) its 5 nearest vertices knnv; PROJ 1 projects through
// the mesh's BVH and ignores knnv.
template <int PROF, int PROJ>
__device__ __forceinline__ void site_finish(const EngineArgs<typename PT<PROF>::T>& a, int parity, int g,
                                            const int (&knnv)[kKProj], SiteOut& o) {
  using T = typename PT<PROF>::T;
  const int s = __ldg(a.site_seg + g);
  const SegDev& sd = a.segs[s];
  const MeshDev& md = a.meshes[sd.mesh];
  const int K = a.K;
  const uint32_t* row = a.knn + (size_t)g * K;
  const int i = g - sd.site_base;
  const bool fz = sd.mode != 0 && a.frozen[g];
  const V3<T> si = ld3(a.S[parity], g);
  const V3<T> cent = ld3((const T*)a.cent, g);

  // projection
  V3<T> sn;
  if (PROF == PROF_MIXED && !finite3(cent)) {
    sn = si;
  } else if (PROJ == 1) {
    using Q = typename PT<PROF>::Q;
    sn = project_bvh<T, Q>(cent, md.bvh, md.bvh_tri, md.V, md.F, (Q)bvh_bound2(cent, si), a.bvh_ovf);
  } else if (PROF == PROF_REF) {
    sn = project_onering_rec<T, float>(cent, md.ring, md.nV, md.vf_off, knnv, kKProj);
  } else {
    sn = project_onering_rec<T, double>(cent, md.ring, md.nV, md.vf_off, knnv, kKProj);
  }
  st3(a.S[parity ^ 1], g, sn);

  // tiers on the segment's first iteration (modes 1/2)
  const int it = sd.iter;
  if (it == 0 && sd.mode != 0) {
    const int base = sd.site_base;
    auto normal = [&](int j, float out[3]) {
      int v = a.nnv[base + j];
      if (v < 0) { out[0] = out[1] = out[2] = 0.f; return; }
      out[0] = __ldg(md.N + 3 * v); out[1] = __ldg(md.N + 3 * v + 1); out[2] = __ldg(md.N + 3 * v + 2);
    };
    a.tier[g] = (uint8_t)tier_of(sd.mode, i, sd.n_sites, K, row, normal);
  }

  // freeze test + apply
  o.seg = s;
  o.same = o.low = o.both = o.newly = 0;
  const T d2 = dist2(sn, si);
  o.disp2 = (float)d2;
  if (it == 0) {
    a.streak[g] = 0;
  } else {
    const int tt = min((int)a.tier[g], 5);
    // a frozen site's list is the previous one by construction
    const bool same = fz || a.same[g] != 0;
    const bool low = d2 <= (T)sd.thr2_tier[tt];
    const bool both = same && low;
    int st = a.streak[g];
    st = both ? (st < 255 ? st + 1 : st) : 0;
    const bool cand = st >= sd.need_tier[tt];
    o.same = same; o.low = low; o.both = both;
    if (sd.mode == 0) {
      a.streak[g] = 0;   // mode 0 clears streak and frozen every iteration (main.cu:837-846)
    } else {
      a.streak[g] = (uint8_t)st;
      if (cand && !a.frozen[g]) { a.frozen[g] = 1; o.newly = 1; }
    }
  }
}

// Rings the per-thread centroid -> vertex search may visit before the site
// is handed to k_site_far (a centroid far off the surface, e.g. of a cell
// that the neighbours leave almost unbounded in the first iteration).
constexpr int kVertexRingLimit = 4;

// Centroid -> its kKProj nearest mesh vertices, for every gridded site that
// is not frozen (one thread per site), into a.knnv.  A site whose search
// would pass kVertexRingLimit rings is listed in a.far and its list marked
// kVertexDeferred; k_site_far finishes it.  A kernel of its own: the search
// needs a fraction of the projection's registers, so it runs at twice the
// projection's resident warps (FP32 positions: 48 per SM, measured 3 %
// faster for the projection group than the compiler's 56 registers and no
// faster at 64; FP64 positions keep the compiler's choice, which spills
// less).
constexpr int kVertexDeferred = -2;

template <int PROF, int BS>
__global__ void __launch_bounds__(BS, PROF == PROF_FP64 ? 1 : 1536 / BS) k_site_vsearch(EngineArgs<typename PT<PROF>::T> a, int parity) {
  using T = typename PT<PROF>::T;
  (void)parity;
  const int t = blockIdx.x * BS + threadIdx.x;
  const int n_grid = __ldg(a.cell_start + a.total_cells);
  if (t >= n_grid) return;
  const int g = (int)a.sorted[t].id;
  const int s = __ldg(a.site_seg + g);
  const SegDev& sd = a.segs[s];
  if (sd.mode != 0 && a.frozen[g]) return;  // frozen sites keep their vertices
  const MeshDev& md = a.meshes[sd.mesh];
  int* kv = a.knnv + (size_t)g * kKProj;
  const int skip = (sd.mode == 0 && sd.ex_quirk) ? g - sd.site_base : -1;
  auto accept = [skip](uint32_t id) { return (int)id != skip; };
  const V3<T> c = ld3((const T*)a.cent, g);
  TopK<T, kKProj> top;
  // the site's 5 vertices of the last iteration lie within the largest of
  // their squared distances to the new centroid, so the 5 nearest do: one
  // box query of the cells within it (exact when it finds 5 vertices)
  bool done = false;
  {
    T thr = (T)0;
    bool ok = true;
#pragma unroll
    for (int k = 0; k < kKProj; ++k) {
      const int v = kv[k];
      ok = ok && (unsigned)v < (unsigned)md.nV && v != skip;
      if (ok) {
        const V3<T> pv{(T)__ldg(md.V + 3 * v), (T)__ldg(md.V + 3 * v + 1), (T)__ldg(md.V + 3 * v + 2)};
        const T d = dist2(pv, c);
        thr = d > thr ? d : thr;
      }
    }
    if (ok) {
      const float qm = fmaxf(fabsf((float)c.x), fmaxf(fabsf((float)c.y), fabsf((float)c.z)));
      const float rad = __fsqrt_ru(f32_ru(thr)) * 1.0001f + 1e-3f * md.vg.h + 4e-7f * qm;
      done = grid_knn_box<T, float, kKProj>(md.vg, md.vcell_start, md.vsorted, c, thr, rad, top, accept,
                                            kVertexBoxCells);
      if (!done) top = TopK<T, kKProj>();
    }
  }
  if (!done && !grid_knn<T, float, kKProj>(md.vg, md.vcell_start, md.vsorted, c, top, accept, kVertexRingLimit)) {
    const int k = atomicAdd(a.far, 1);
    a.far[1 + k] = g;
    kv[0] = kVertexDeferred;
    return;
  }
#pragma unroll
  for (int k = 0; k < kKProj; ++k) kv[k] = (int)KeyOps<T>::idx(top.k[k]);
}

// Everything after the centroid and (PROJ 0) the vertex search of
// k_site_vsearch; false when that search was deferred (the site is then
// listed in a.far and finished by k_site_far).
template <int PROF, int PROJ>
__device__ __forceinline__ bool site_proj(const EngineArgs<typename PT<PROF>::T>& a, int parity, int g, SiteOut& o) {
  if (PROJ == 1) {
    const int none[kKProj] = {-1, -1, -1, -1, -1};
    site_finish<PROF, 1>(a, parity, g, none, o);
    return true;
  }
  const int* kv = a.knnv + (size_t)g * kKProj;
  int knnv[kKProj];
#pragma unroll
  for (int k = 0; k < kKProj; ++k) knnv[k] = kv[k];
  if (knnv[0] == kVertexDeferred) return false;
  site_finish<PROF, 0>(a, parity, g, knnv, o);
  return true;
}

__device__ __forceinline__ void stats_atomic(int* stats, const SegDev* segs, const SiteOut& o) {
  int* sl = stats + ((size_t)o.seg * kStatsRing + (segs[o.seg].iter % kStatsRing)) * kStatsWords;
  if (o.same) atomicAdd(sl + 0, 1);
  if (o.low) atomicAdd(sl + 1, 1);
  if (o.both) atomicAdd(sl + 2, 1);
  if (o.newly) atomicAdd(sl + 3, 1);
  atomicMax(reinterpret_cast<unsigned*>(sl + 4), __float_as_uint(o.disp2));
}

// Per-block staging of the per-segment counters: the first segment a warp
// of the block reports claims the slot; counts of other segments go to
// global memory directly.  (One set of global atomics per block instead of
// per warp: thousands of warps adding to the same few words serialised in
// L2.)  Sums and a max of float bits, so the totals do not depend on order.
struct StatsStage {
  int seg;
  unsigned v[5];  // same, low, both, newly, max squared displacement (float bits)
};

__device__ __forceinline__ void stats_stage_init(StatsStage& s) {
  if (threadIdx.x < 5) s.v[threadIdx.x] = 0u;
  if (threadIdx.x == 0) s.seg = -1;
}

__device__ __forceinline__ void stats_flush(int* stats, const SegDev* segs, const SiteOut& o, StatsStage& stage) {
  // warp-aggregated per-segment counters; every lane of the warp takes part
  const unsigned full = 0xffffffffu;
  const int key = o.seg;
  const unsigned peers = __match_any_sync(full, key);
  const int leader = __ffs(peers) - 1;
  const int lane = threadIdx.x & 31;
  const int same = __popc(__ballot_sync(full, o.same) & peers);
  const int low = __popc(__ballot_sync(full, o.low) & peers);
  const int both = __popc(__ballot_sync(full, o.both) & peers);
  const int newly = __popc(__ballot_sync(full, o.newly) & peers);
  const unsigned dbits = __reduce_max_sync(peers, __float_as_uint(o.seg >= 0 ? o.disp2 : 0.f));
  if (lane == leader && key >= 0) {
    const int owner = atomicCAS(&stage.seg, -1, key);
    if (owner == -1 || owner == key) {
      if (same) atomicAdd(&stage.v[0], (unsigned)same);
      if (low) atomicAdd(&stage.v[1], (unsigned)low);
      if (both) atomicAdd(&stage.v[2], (unsigned)both);
      if (newly) atomicAdd(&stage.v[3], (unsigned)newly);
      atomicMax(&stage.v[4], dbits);
    } else {
      int* sl = stats + ((size_t)key * kStatsRing + (segs[key].iter % kStatsRing)) * kStatsWords;
      if (same) atomicAdd(sl + 0, same);
      if (low) atomicAdd(sl + 1, low);
      if (both) atomicAdd(sl + 2, both);
      if (newly) atomicAdd(sl + 3, newly);
      atomicMax(reinterpret_cast<unsigned*>(sl + 4), dbits);
    }
  }
}

// after a __syncthreads that follows every warp's stats_flush
__device__ __forceinline__ void stats_stage_flush(int* stats, const SegDev* segs, const StatsStage& stage) {
  if (threadIdx.x != 0 || stage.seg < 0) return;
  int* sl = stats + ((size_t)stage.seg * kStatsRing + (segs[stage.seg].iter % kStatsRing)) * kStatsWords;
  for (int w = 0; w < 4; ++w)
    if (stage.v[w]) atomicAdd(sl + w, (int)stage.v[w]);
  atomicMax(reinterpret_cast<unsigned*>(sl + 4), stage.v[4]);
}

// This step's motion of site g (o from site_finish; o.seg < 0: none) into
// its coarse block at its old position, for the next iteration's KNN:
// warp-collective, one atomic per distinct block of the warp.  The stamp is
// the segment's iteration, so an entry from an earlier iteration reads as
// no motion.
template <class T>
__device__ __forceinline__ void motion_to_block(const EngineArgs<T>& a, int parity, int g, const SiteOut& o) {
  int blk = -1;
  unsigned bits = 0u, stamp = 0u;
  if (g >= 0 && o.seg >= 0) {
    int bx, by, bz;
    blk = motion_block(a.geom[o.seg], ld3(a.S[parity], g), bx, by, bz);
    bits = __float_as_uint(sqrtf(o.disp2));
    stamp = (unsigned)a.segs[o.seg].iter;
  }
  const unsigned peers = __match_any_sync(0xffffffffu, blk);
  const unsigned mb = __reduce_max_sync(peers, bits);
  if (blk >= 0 && (int)(threadIdx.x & 31) == __ffs(peers) - 1)
    atomicMax(a.blockmax + blk, ((unsigned long long)stamp << 32) | mb);
}

// One-ring projection: 24 resident warps per SM (80 registers), the
// fastest budget of a register sweep (64 or 51: spills; 96 or 128: too few
// warps).  The BVH projection keeps the compiler's choice.
template <int PROF, int BS, int PROJ>
__global__ void __launch_bounds__(BS, PROJ == 0 ? 768 / BS : 1) k_site_proj(EngineArgs<typename PT<PROF>::T> a, int parity) {
  __shared__ StatsStage stage;
  stats_stage_init(stage);
  __syncthreads();
  const int t = blockIdx.x * BS + threadIdx.x;
  const int n_grid = __ldg(a.cell_start + a.total_cells);
  SiteOut o{-1, 0, 0, 0, 0, 0.f};
  int g = -1;
  if (t < n_grid) {
    g = (int)a.sorted[t].id;
    site_proj<PROF, PROJ>(a, parity, g, o);
  }
  if (a.blockmax) motion_to_block(a, parity, g, o);
  stats_flush(a.stats, a.segs, o, stage);
  __syncthreads();
  stats_stage_flush(a.stats, a.segs, stage);
}

// Iteration bookkeeping, run by one block: advance active segments, clear
// their next stats slot, apply each segment's stop rule (a stopped segment is
// no longer gridded or iterated: active = 2), reset the overflow, deferred
// and active-site counts for the next iteration.
__device__ __forceinline__ void seg_advance(SegDev* segs, int* active, int nseg, int* stats, int* ovf, int* far,
                                            int* act_count) {
  for (int s = threadIdx.x; s < nseg; s += blockDim.x) {
    if (active[s] != 1) continue;
    int it = segs[s].iter;
    int* cur = stats + ((size_t)s * kStatsRing + (it % kStatsRing)) * kStatsWords;
    cur[5] = it;
    const float d2 = __uint_as_float((unsigned)cur[4]);
    int nx = it + 1;
    int* sl = stats + ((size_t)s * kStatsRing + (nx % kStatsRing)) * kStatsWords;
    for (int w = 0; w < kStatsWords; ++w) sl[w] = 0;
    segs[s].iter = nx;
    // the step bound of the candidate lists (NaN fails every test)
    segs[s].step_motion = sqrtf(d2);
    const float lim = segs[s].stop_motion2;
    const int cap = segs[s].stop_iters;
    if ((lim >= 0.f && d2 <= lim) || (cap > 0 && nx >= cap)) active[s] = 2;
  }
  if (threadIdx.x == 0) { ovf[0] = 0; far[0] = 0; *act_count = 0; }
}

// Deferred sites (a.far): one block per site finds the 5 nearest mesh
// vertices of the centroid by scanning all of them (each thread every 128th
// vertex, then a merge of the 128 lists by thread 0; exact, the keys are
// unique), then thread 0 finishes the site.
// The last block to finish then runs the iteration's bookkeeping
// (seg_advance), counted by `ticket`, which it leaves at zero.
template <int PROF>
__global__ void __launch_bounds__(128) k_site_far(EngineArgs<typename PT<PROF>::T> a, int parity, SegDev* segs,
                                                   int* active, int nseg, unsigned* ticket) {
  using T = typename PT<PROF>::T;
  using Key = typename KeyOps<T>::Key;
  __shared__ Key keys[128 * kKProj];
  __shared__ bool last;
  const int n = *(volatile int*)a.far;
  for (int k = blockIdx.x; k < n; k += gridDim.x) {
    const int g = a.far[1 + k];
    const int s = __ldg(a.site_seg + g);
    const SegDev& sd = a.segs[s];
    const MeshDev& md = a.meshes[sd.mesh];
    const int skip = (sd.mode == 0 && sd.ex_quirk) ? g - sd.site_base : -1;
    const V3<T> q = ld3((const T*)a.cent, g);
    TopK<T, kKProj> top;
    for (int v = threadIdx.x; v < md.nV; v += 128) {
      if (v == skip) continue;
      const V3<T> p{(T)__ldg(md.V + 3 * v), (T)__ldg(md.V + 3 * v + 1), (T)__ldg(md.V + 3 * v + 2)};
      const T d = dist2(p, q);
      if (d <= top.worst_d()) top.insert(KeyOps<T>::make(d, (uint32_t)v));
    }
#pragma unroll
    for (int j = 0; j < kKProj; ++j) keys[threadIdx.x * kKProj + j] = top.k[j];
    __syncthreads();
    if (threadIdx.x == 0) {
      TopK<T, kKProj> all;
      for (int j = 0; j < 128 * kKProj; ++j) all.insert(keys[j]);
      int knnv[kKProj];
      int* kv = a.knnv + (size_t)g * kKProj;
#pragma unroll
      for (int j = 0; j < kKProj; ++j) { knnv[j] = (int)KeyOps<T>::idx(all.k[j]); kv[j] = knnv[j]; }
      SiteOut o{-1, 0, 0, 0, 0, 0.f};
      site_finish<PROF, 0>(a, parity, g, knnv, o);
      stats_atomic(a.stats, a.segs, o);
      if (a.blockmax) {
        int bx, by, bz;
        const int blk = motion_block(a.geom[o.seg], ld3(a.S[parity], g), bx, by, bz);
        atomicMax(a.blockmax + blk, ((unsigned long long)(unsigned)a.segs[o.seg].iter << 32) |
                                        __float_as_uint(sqrtf(o.disp2)));
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  seg_advance(segs, active, nseg, a.stats, a.ovf, a.far, a.act_count);
  if (threadIdx.x == 0) *ticket = 0u;
}

}  // namespace cvt
