// Mesh ingest on the device: validation, vertex compaction (main.cu:230-257),
// vertex->face CSR in face order (main.cu:259-285), surface area, the
// sampler's face-area prefix sums and the evaluation BVH (evaluate.cuh:114-201).
//
// The BVH is built level by level.  Every node of the reference's recursive
// builder splits its triangles, stably sorted along the longest axis of
// their centroid extent, at the middle.  The tree's shape therefore depends
// on the triangle count only, so the host plans every level (segments of the
// id array, pre-order node numbers) and the device does the data work: per
// segment bounds and centroid extent (warp-aggregated atomics), then one
// stable radix sort of (segment rank, centroid key) pairs over the whole id
// array.  A stable LSD radix sort orders equal keys by their current
// position, exactly as std::stable_sort does, so nodes and triangle order are
// identical to the recursive build.
#pragma once
#include "cvt_eval.cuh"

namespace cvt {

// float -> int whose signed order is the float order (-0 below +0)
__device__ __forceinline__ int ing_f2ord(float v) {
  int b = __float_as_int(v);
  return b >= 0 ? b : b ^ 0x7fffffff;
}
__device__ __forceinline__ float ing_ord2f(int o) { return __int_as_float(o >= 0 ? o : o ^ 0x7fffffff); }

// Face corners: range check (bad |= 1) and referenced-vertex marks.
__global__ void k_ingest_mark(const int* __restrict__ F, long n3, int nV, int* __restrict__ used, int* bad) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n3) return;
  const int v = F[k];
  if ((unsigned)v >= (unsigned)nV) { atomicOr(bad, 1); return; }
  used[v] = 1;
}

// Bounds of every input vertex (R, main.cu:169-227) and of the referenced ones
// (bbox of the compacted mesh); a referenced vertex with a non-finite
// coordinate sets bad |= 2.  bb: all lo[3] hi[3], used lo[3] hi[3] (ord ints).
__global__ void k_ingest_bounds(const float* __restrict__ V, int nV, const int* __restrict__ used, int* bb,
                                int* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float p[3] = {0.f, 0.f, 0.f};
  bool fin = false, u = false;
  if (i < nV) {
    p[0] = V[3 * i]; p[1] = V[3 * i + 1]; p[2] = V[3 * i + 2];
    fin = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]);
    u = used[i] != 0;
    if (u && !fin) atomicOr(bad, 2);
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    int mn_all = fin ? ing_f2ord(p[a]) : INT_MAX, mx_all = fin ? ing_f2ord(p[a]) : INT_MIN;
    int mn_u = (fin && u) ? mn_all : INT_MAX, mx_u = (fin && u) ? mx_all : INT_MIN;
    mn_all = __reduce_min_sync(0xffffffffu, mn_all);
    mx_all = __reduce_max_sync(0xffffffffu, mx_all);
    mn_u = __reduce_min_sync(0xffffffffu, mn_u);
    mx_u = __reduce_max_sync(0xffffffffu, mx_u);
    if ((threadIdx.x & 31) == 0) {
      if (mn_all != INT_MAX) { atomicMin(bb + a, mn_all); atomicMax(bb + 3 + a, mx_all); }
      if (mn_u != INT_MAX) { atomicMin(bb + 6 + a, mn_u); atomicMax(bb + 9 + a, mx_u); }
    }
  }
}

__global__ void k_ingest_bounds_init(int* bb) {
  if (threadIdx.x < 12) bb[threadIdx.x] = (threadIdx.x % 6) < 3 ? INT_MAX : INT_MIN;
}

// Area of each face in FP64, the arithmetic of the host loop (main.cu area
// for the grid density; sampler CDF).
__global__ void k_face_area(const float* __restrict__ V, const int* __restrict__ F, int nF, double* __restrict__ out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nF) return;
  const float* a = V + 3 * (size_t)F[3 * f];
  const float* b = V + 3 * (size_t)F[3 * f + 1];
  const float* c = V + 3 * (size_t)F[3 * f + 2];
  const double e1x = (double)b[0] - a[0], e1y = (double)b[1] - a[1], e1z = (double)b[2] - a[2];
  const double e2x = (double)c[0] - a[0], e2y = (double)c[1] - a[1], e2z = (double)c[2] - a[2];
  const double cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
  out[f] = 0.5 * __dsqrt_rn(cx * cx + cy * cy + cz * cz);
}

// used vertex i -> dV[remap[i]]; unused -> dunref[i - remap[i]] (input order)
__global__ void k_ingest_compact(const float* __restrict__ V, int nV, const int* __restrict__ used,
                                 const int* __restrict__ remap, float* __restrict__ dV, float* __restrict__ dunref) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nV) return;
  float* o = used[i] ? dV + 3 * (size_t)remap[i] : dunref + 3 * (size_t)(i - remap[i]);
  o[0] = V[3 * i]; o[1] = V[3 * i + 1]; o[2] = V[3 * i + 2];
}

// faces through the remap; CSR sort keys (vertex << 32 | face) and counts
__global__ void k_ingest_faces(const int* __restrict__ F, long n3, const int* __restrict__ remap, int* __restrict__ dF,
                               unsigned long long* __restrict__ keys, int* __restrict__ count) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n3) return;
  const int v = remap[F[k]];
  dF[k] = v;
  keys[k] = ((unsigned long long)(unsigned)v << 32) | (unsigned long long)(k / 3);
  atomicAdd(count + v, 1);
}

__global__ void k_iota(int* __restrict__ out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = i;
}

__global__ void k_keys_low32(const unsigned long long* __restrict__ keys, long n, int* __restrict__ out) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = (int)(unsigned)(keys[k] & 0xffffffffull);
}

// ---------------------------------------------------------------------------
// BVH, level by level
// ---------------------------------------------------------------------------
// Per triangle: bmin(3) bmax(3) centroid(3), the host builder's expressions.
__global__ void k_tri_info(const float* __restrict__ V, const int* __restrict__ F, int nF, float* __restrict__ info) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nF) return;
  const float* a = V + 3 * (size_t)F[3 * t];
  const float* b = V + 3 * (size_t)F[3 * t + 1];
  const float* c = V + 3 * (size_t)F[3 * t + 2];
  float* o = info + 9 * (size_t)t;
  const float third = 1.0f / 3.0f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    o[k] = fminf(a[k], fminf(b[k], c[k]));
    o[3 + k] = fmaxf(a[k], fmaxf(b[k], c[k]));
    o[6 + k] = (a[k] + (b[k] + c[k])) * third;
  }
}

// One frontier segment of the id array.  node < 0: a leaf finished on an
// earlier level (carried so that the sort keeps its triangles in place).
struct BvhSeg {
  int start, count, node, left, right;
};

__device__ __forceinline__ int seg_of(const BvhSeg* __restrict__ segs, int nseg, int p) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].start <= p) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// acc per segment: bmin3 bmax3 cmin3 cmax3 as ord ints (initialised by k_seg_acc_init)
__global__ void k_seg_acc_init(int nseg, int* acc) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
#pragma unroll
  for (int k = 0; k < 12; ++k) acc[12 * s + k] = (k % 6) < 3 ? INT_MAX : INT_MIN;
}

__global__ void k_seg_reduce(const int* __restrict__ tids, int n, const BvhSeg* __restrict__ segs, int nseg,
                             const float* __restrict__ info, int* __restrict__ acc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = p < n;
  int s = -1;
  if (in) {
    s = seg_of(segs, nseg, p);
    if (segs[s].node < 0) s = -1;   // finished leaf: nothing to emit
  }
  const unsigned peers = __match_any_sync(0xffffffffu, s);
  const int leader = __ffs(peers) - 1;
  const float* o = info + 9 * (size_t)(s >= 0 ? tids[p] : 0);
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    // bmin <- tri bmin, bmax <- tri bmax, cmin/cmax <- centroid
    const int src = k < 9 ? k : k - 3;
    const bool is_min = (k % 6) < 3;
    int v = is_min ? INT_MAX : INT_MIN;
    if (s >= 0) v = ing_f2ord(o[src]);
    v = is_min ? __reduce_min_sync(peers, v) : __reduce_max_sync(peers, v);
    if ((int)(threadIdx.x & 31) == leader && s >= 0) {
      if (is_min) atomicMin(acc + 12 * s + k, v); else atomicMax(acc + 12 * s + k, v);
    }
  }
}

// Nodes of this level (pre-order slots), split axis per segment (-1: leaf).
__global__ void k_seg_emit(const BvhSeg* __restrict__ segs, int nseg, const int* __restrict__ acc, int leaf,
                           BVHNode* __restrict__ nodes, int* __restrict__ axis) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const BvhSeg g = segs[s];
  if (g.node < 0) { axis[s] = -1; return; }
  BVHNode nd;
#pragma unroll
  for (int a = 0; a < 3; ++a) { nd.bmin[a] = ing_ord2f(acc[12 * s + a]); nd.bmax[a] = ing_ord2f(acc[12 * s + 3 + a]); }
  if (g.count <= leaf) {
    nd.left = nd.right = -1;
    nd.triStart = g.start;
    nd.triCount = g.count;
    axis[s] = -1;
  } else {
    const float ex = ing_ord2f(acc[12 * s + 9]) - ing_ord2f(acc[12 * s + 6]);
    const float ey = ing_ord2f(acc[12 * s + 10]) - ing_ord2f(acc[12 * s + 7]);
    const float ez = ing_ord2f(acc[12 * s + 11]) - ing_ord2f(acc[12 * s + 8]);
    axis[s] = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
    nd.left = g.left;
    nd.right = g.right;
    nd.triStart = -1;
    nd.triCount = 0;
  }
  nodes[g.node] = nd;
}

// sort keys: segment rank in the high word; within a segment that splits the
// centroid coordinate on its axis (-0 folded into +0, monotone unsigned map),
// else 0 so that the stable sort leaves the segment as it is
__global__ void k_seg_keys(const int* __restrict__ tids, int n, const BvhSeg* __restrict__ segs, int nseg,
                           const int* __restrict__ axis, const float* __restrict__ info,
                           unsigned long long* __restrict__ keys) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int s = seg_of(segs, nseg, p);
  const int ax = axis[s];
  unsigned lo = 0;
  if (ax >= 0) {
    const unsigned u = __float_as_uint(info[9 * (size_t)tids[p] + 6 + ax] + 0.0f);
    lo = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
  }
  keys[p] = ((unsigned long long)(unsigned)s << 32) | lo;
}

}  // namespace cvt
