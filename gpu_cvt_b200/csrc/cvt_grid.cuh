// Uniform-grid spatial hash and exact K-nearest-neighbour search.
//
// Replaces the reference's random-hub index (bitonic-hubs-grid.cuh:1142-1656,
// rebuilt with ~20 cudaMalloc per call, host shuffles and H x H bound
// matrices) with a per-segment uniform grid rebuilt by a counting sort every
// iteration.  The answer is the exact K nearest points in (squared distance,
// index) order; the search widens ring by ring until the K-th candidate is
// provably closer than every unvisited cell, so the result does not depend
// on the cell size (only the time does).
#pragma once
#include "cvt_math.cuh"

namespace cvt {

// Grid over one segment's points.  Cells [cell_base, cell_base + ncell) are
// spatial (x fastest); cell_base + ncell is the bucket of non-finite points,
// which is never searched.
struct GridGeom {
  float lo[3];
  float h, inv_h;
  int dim[3];
  int cell_base;
  int ncell;
};

// Cell-ordered copy of a point: coordinates plus the point's global index.
template <class T> struct alignas(16) Pt4 { T x, y, z; uint32_t id; };

template <class T>
__device__ __forceinline__ int grid_coord(const GridGeom& g, T v, int a) {
  float f = floorf(((float)v - g.lo[a]) * g.inv_h);
  int c = (f >= 0.f) ? (f < (float)g.dim[a] ? (int)f : g.dim[a] - 1) : 0;
  return c;
}

template <class T>
__device__ __forceinline__ int grid_cell(const GridGeom& g, V3<T> p) {
  if (!finite3(p)) return g.cell_base + g.ncell;
  int cx = grid_coord(g, p.x, 0), cy = grid_coord(g, p.y, 1), cz = grid_coord(g, p.z, 2);
  return g.cell_base + (cz * g.dim[1] + cy) * g.dim[0] + cx;
}

// ---------------------------------------------------------------------------
// top-K with (distance, index) keys
// ---------------------------------------------------------------------------
template <class T> struct KeyOps;

// float: the key is (float bits << 32 | index); non-negative floats order as
// their bit patterns, so one 64-bit compare orders by distance then index.
template <> struct KeyOps<float> {
  using Key = unsigned long long;
  static __device__ __forceinline__ Key make(float d, uint32_t i) {
    return ((Key)__float_as_uint(d) << 32) | (Key)i;
  }
  static __device__ __forceinline__ Key empty() { return ~0ull; }
  static __device__ __forceinline__ bool less(Key a, Key b) { return a < b; }
  static __device__ __forceinline__ Key kmin(Key a, Key b) { return a < b ? a : b; }
  static __device__ __forceinline__ Key kmax(Key a, Key b) { return a < b ? b : a; }
  static __device__ __forceinline__ uint32_t idx(Key k) { return (uint32_t)(k & 0xffffffffull); }
  static __device__ __forceinline__ float dist(Key k) {
    return k == ~0ull ? __int_as_float(0x7f800000) : __uint_as_float((uint32_t)(k >> 32));
  }
  static __device__ __forceinline__ bool is_empty(Key k) { return k == ~0ull; }
};

struct DKey { double d; uint32_t i; };
template <> struct KeyOps<double> {
  using Key = DKey;
  static __device__ __forceinline__ Key make(double d, uint32_t i) { return {d, i}; }
  static __device__ __forceinline__ Key empty() { return {__longlong_as_double(0x7ff0000000000000ll), 0xffffffffu}; }
  static __device__ __forceinline__ bool less(Key a, Key b) { return a.d < b.d || (a.d == b.d && a.i < b.i); }
  static __device__ __forceinline__ Key kmin(Key a, Key b) { return less(a, b) ? a : b; }
  static __device__ __forceinline__ Key kmax(Key a, Key b) { return less(a, b) ? b : a; }
  static __device__ __forceinline__ uint32_t idx(Key k) { return k.i; }
  static __device__ __forceinline__ double dist(Key k) { return k.d; }
  static __device__ __forceinline__ bool is_empty(Key k) { return k.i == 0xffffffffu && isinf(k.d); }
};

// Sorted register list; insertion keeps the KK smallest keys.  Branch-free
// update new[j] = max(old[j-1], min(old[j], x)) keeps the list in registers.
template <class T, int KK> struct TopK {
  using O = KeyOps<T>;
  typename O::Key k[KK];
  __device__ __forceinline__ TopK() {
#pragma unroll
    for (int j = 0; j < KK; ++j) k[j] = O::empty();
  }
  __device__ __forceinline__ T worst_d() const { return O::dist(k[KK - 1]); }
  __device__ __forceinline__ bool full() const { return !O::is_empty(k[KK - 1]); }
  __device__ __forceinline__ void insert(typename O::Key x) {
    if (!O::less(x, k[KK - 1])) return;
#pragma unroll
    for (int j = KK - 1; j > 0; --j) k[j] = O::kmax(k[j - 1], O::kmin(k[j], x));
    k[0] = O::kmin(k[0], x);
  }
};

// Exact KK-nearest search of q among the points of one grid.  accept(id)
// filters candidates (used for the vertex-index exclusion quirk).
// With rlim > 0 the search gives up (returns false, top incomplete) when it
// has not finished after rlim rings: a query far from every point would
// otherwise visit the whole grid, one cell at a time.
template <class T, class PT, int KK, class Accept>
__device__ __forceinline__ bool grid_knn(const GridGeom& g, const int* __restrict__ cell_start,
                                         const Pt4<PT>* __restrict__ pts, V3<T> q, TopK<T, KK>& top,
                                         Accept accept, int rlim = 0) {
  if (!finite3(q)) return true;
  const int cx = grid_coord(g, q.x, 0), cy = grid_coord(g, q.y, 1), cz = grid_coord(g, q.z, 2);
  const int rmax = max(g.dim[0], max(g.dim[1], g.dim[2]));
  const float slack = 1e-3f * g.h;
  const float qf[3] = {(float)q.x, (float)q.y, (float)q.z};
  const int c[3] = {cx, cy, cz};
  auto scan_range = [&](int b, int e) {
    for (int k = b; k < e; ++k) {
      Pt4<PT> p = pts[k];
      if (!accept(p.id)) continue;
      T d = dist2(V3<T>{(T)p.x, (T)p.y, (T)p.z}, q);
      if (d <= top.worst_d()) top.insert(KeyOps<T>::make(d, p.id));
    }
  };
  for (int r = 1; r <= rmax; ++r) {
    const int z0 = max(cz - r, 0), z1 = min(cz + r, g.dim[2] - 1);
    const int y0 = max(cy - r, 0), y1 = min(cy + r, g.dim[1] - 1);
    const int x0 = max(cx - r, 0), x1 = min(cx + r, g.dim[0] - 1);
    for (int z = z0; z <= z1; ++z) {
      for (int y = y0; y <= y1; ++y) {
        const int row = g.cell_base + (z * g.dim[1] + y) * g.dim[0];
        const bool full_row = (r == 1) || abs(z - cz) == r || abs(y - cy) == r;
        if (full_row) {
          scan_range(__ldg(cell_start + row + x0), __ldg(cell_start + row + x1 + 1));
        } else {
          if (cx - r >= 0) scan_range(__ldg(cell_start + row + cx - r), __ldg(cell_start + row + cx - r + 1));
          if (cx + r < g.dim[0]) scan_range(__ldg(cell_start + row + cx + r), __ldg(cell_start + row + cx + r + 1));
        }
      }
    }
    // lower bound on the distance to any point outside the visited block
    float m = __int_as_float(0x7f800000);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (c[a] - r > 0) m = fminf(m, qf[a] - (g.lo[a] + (float)(c[a] - r) * g.h));
      if (c[a] + r < g.dim[a] - 1) m = fminf(m, (g.lo[a] + (float)(c[a] + r + 1) * g.h) - qf[a]);
    }
    if (isinf(m)) break;
    m -= slack;
    if (top.full() && m > 0.f && (double)top.worst_d() < (double)m * (double)m) break;
    if (r == rlim) return false;
  }
  return true;
}

// The KK nearest points of q from one box query (one thread): every
// accepted point of the cells in q +- rad with squared distance <= thr is
// offered to top.  When top fills, it holds the KK nearest in (squared
// distance, index) order, the keys grid_knn returns: a point left out is
// farther than thr, so farther than every key kept.  rad must cover
// sqrt(thr) with margin (cell coordinates are monotone in the position).
// Returns false, top partly filled, when fewer than KK points pass or the
// box spans more than max_cells cells; the caller then resets top and runs
// grid_knn.
template <class T, class PT, int KK, class Accept>
__device__ __forceinline__ bool grid_knn_box(const GridGeom& g, const int* __restrict__ cell_start,
                                             const Pt4<PT>* __restrict__ pts, V3<T> q, T thr, float rad,
                                             TopK<T, KK>& top, Accept accept, int max_cells) {
  if (!finite3(q) || !(rad < INFINITY) || !(thr >= (T)0)) return false;
  const float qf[3] = {(float)q.x, (float)q.y, (float)q.z};
  int lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = grid_coord(g, __fsub_rd(qf[a], rad), a);
    hi[a] = grid_coord(g, __fadd_ru(qf[a], rad), a);
  }
  if ((hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1) > max_cells) return false;
  for (int z = lo[2]; z <= hi[2]; ++z) {
    for (int y = lo[1]; y <= hi[1]; ++y) {
      const int row = g.cell_base + (z * g.dim[1] + y) * g.dim[0];
      const int e = __ldg(cell_start + row + hi[0] + 1);
      for (int k = __ldg(cell_start + row + lo[0]); k < e; ++k) {
        const Pt4<PT> p = pts[k];
        if (!accept(p.id)) continue;
        const T d = dist2(V3<T>{(T)p.x, (T)p.y, (T)p.z}, q);
        if (d <= thr && d <= top.worst_d()) top.insert(KeyOps<T>::make(d, p.id));
      }
    }
  }
  return top.full();
}

// ---------------------------------------------------------------------------
// warp-cooperative search: one warp per query point
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long shfl_key(unsigned long long k, int src) {
  return __shfl_sync(0xffffffffu, k, src);
}
__device__ __forceinline__ DKey shfl_key(DKey k, int src) {
  return {__shfl_sync(0xffffffffu, k.d, src), __shfl_sync(0xffffffffu, k.i, src)};
}
__device__ __forceinline__ unsigned long long shfl_up_key(unsigned long long k) {
  return __shfl_up_sync(0xffffffffu, k, 1);
}
__device__ __forceinline__ DKey shfl_up_key(DKey k) {
  return {__shfl_up_sync(0xffffffffu, k.d, 1), __shfl_up_sync(0xffffffffu, k.i, 1)};
}
__device__ __forceinline__ unsigned long long min_key(unsigned long long) { return 0ull; }
__device__ __forceinline__ DKey min_key(DKey) { return {-INFINITY, 0u}; }

// Visit the candidates of Chebyshev ring r around (cx,cy,cz) in chunks of 32:
// every lane calls visit(pos) the same number of times, pos = a sorted
// position or -1.  The ring's cell ranges (two slots per (z,y) row: the whole
// x-range for rows on the shell's faces, else the two end cells) are spread
// over the lanes, their lengths warp-scanned, and each lane finds the range of
// its candidate by a shuffle binary search over the prefix sums.
template <class Visit>
__device__ __forceinline__ void warp_ring(const GridGeom& g, const int* __restrict__ cell_start, int cx, int cy,
                                          int cz, int r, int lane, Visit&& visit) {
  const int z0 = max(cz - r, 0), z1 = min(cz + r, g.dim[2] - 1);
  const int y0 = max(cy - r, 0), y1 = min(cy + r, g.dim[1] - 1);
  const int x0 = max(cx - r, 0), x1 = min(cx + r, g.dim[0] - 1);
  const int ny = y1 - y0 + 1;
  const int nslots = 2 * (z1 - z0 + 1) * ny;
  for (int base = 0; base < nslots; base += 32) {
    const int slot = base + lane;
    int b = 0, e = 0;
    if (slot < nslots) {
      const int rowi = slot >> 1, which = slot & 1;
      const int z = z0 + rowi / ny, y = y0 + rowi % ny;
      const int row = g.cell_base + (z * g.dim[1] + y) * g.dim[0];
      const bool full_row = (r == 1) || abs(z - cz) == r || abs(y - cy) == r;
      if (full_row) {
        if (which == 0) { b = __ldg(cell_start + row + x0); e = __ldg(cell_start + row + x1 + 1); }
      } else {
        const int x = which == 0 ? cx - r : cx + r;
        if (x >= 0 && x < g.dim[0]) { b = __ldg(cell_start + row + x); e = __ldg(cell_start + row + x + 1); }
      }
    }
    const int len = e - b;
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int excl = incl - len;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    for (int c = 0; c < total; c += 32) {
      const int i = c + lane;
      int lo = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const int probe = lo + step;
        const int ex = __shfl_sync(0xffffffffu, excl, probe & 31);
        if (probe < 32 && ex <= i) lo = probe;
      }
      const int rb = __shfl_sync(0xffffffffu, b, lo);
      const int rex = __shfl_sync(0xffffffffu, excl, lo);
      visit(i < total ? rb + (i - rex) : -1);
    }
  }
}

// lower bound on the distance from q to any cell outside ring r (+inf when
// the visited block covers the grid)
__device__ __forceinline__ float ring_margin(const GridGeom& g, const float qf[3], const int c[3], int r) {
  float m = __int_as_float(0x7f800000);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (c[a] - r > 0) m = fminf(m, qf[a] - (g.lo[a] + (float)(c[a] - r) * g.h));
    if (c[a] + r < g.dim[a] - 1) m = fminf(m, (g.lo[a] + (float)(c[a] + r + 1) * g.h) - qf[a]);
  }
  return m;
}

// Exact KK nearest points of q (uniform across the warp), KK <= 64.  The
// sorted list spans R = ceil(KK/32) registers per lane: list[r] at lane j is
// entry 32*r + j.  Candidates beyond the estimate thr0 (the caller's guess of
// the KK-th squared distance) are skipped, and thr tightens to the current
// KK-th distance once the list is full.  The result is exact whatever the
// estimate: a skipped candidate lies above a threshold that is >= the final
// KK-th distance, and an estimate that proves too tight (the list is not full
// although every point within it was visited) restarts the search with
// thr = +inf.
template <class T, class PT, int KK, class Accept>
__device__ __forceinline__ void warp_knn(const GridGeom& g, const int* __restrict__ cell_start,
                                         const Pt4<PT>* __restrict__ pts, V3<T> q, T thr0, int lane, Accept accept,
                                         typename KeyOps<T>::Key (&list)[(KK + 31) / 32]) {
  constexpr int R = (KK + 31) / 32;
  static_assert(KK <= 64, "at most two keys per lane");
  using O = KeyOps<T>;
  using Key = typename O::Key;
#pragma unroll
  for (int r = 0; r < R; ++r) list[r] = O::empty();
  if (!finite3(q)) return;
  const int c[3] = {grid_coord(g, q.x, 0), grid_coord(g, q.y, 1), grid_coord(g, q.z, 2)};
  const float qf[3] = {(float)q.x, (float)q.y, (float)q.z};
  const int rmax = max(g.dim[0], max(g.dim[1], g.dim[2]));
  const float slack = 1e-3f * g.h;
  const T INF = (T)INFINITY;
  constexpr int KR = (KK - 1) / 32, KL = (KK - 1) % 32;  // the K-th entry
  T thr = thr0 > (T)0 ? thr0 : INF;
  Key kth = O::empty();
  for (int ring = 1; ring <= rmax; ++ring) {
    warp_ring(g, cell_start, c[0], c[1], c[2], ring, lane, [&](int pos) {
      Key key = O::empty();
      bool pass = false;
      if (pos >= 0) {
        const Pt4<PT> p = pts[pos];
        if (accept(p.id)) {
          const T d = dist2(V3<T>{(T)p.x, (T)p.y, (T)p.z}, q);
          key = O::make(d, p.id);
          pass = d <= thr && O::less(key, kth);
        }
      }
      unsigned mask = __ballot_sync(0xffffffffu, pass);
      if (mask) {
        while (mask) {
          const int src = __ffs(mask) - 1;
          mask &= mask - 1;
          const Key x = shfl_key(key, src);
          // new[j] = max(old[j-1], min(old[j], x)) over the whole list.  A key
          // that is no longer below the K-th entry leaves entries < KK
          // unchanged, so the K-th entry is refreshed once per chunk; lanes
          // past the list's end hold overflow entries that are never read.
          Key carry = min_key(x);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            Key prev = shfl_up_key(list[r]);
            if (lane == 0) prev = carry;
            if (r + 1 < R) carry = shfl_key(list[r], 31);
            list[r] = O::kmax(prev, O::kmin(list[r], x));
          }
        }
        kth = shfl_key(list[KR], KL);
      }
    });
    const bool full = !O::is_empty(kth);
    if (full) thr = fmin(thr, O::dist(kth));
    float m = ring_margin(g, qf, c, ring);
    const bool all_seen = isinf(m);
    m -= slack;
    if (full) {
      if (all_seen || (m > 0.f && (double)O::dist(kth) < (double)m * (double)m)) break;
    } else if (thr < INF && (all_seen || (m > 0.f && (double)thr < (double)m * (double)m))) {
      thr = INF;
#pragma unroll
      for (int r = 0; r < R; ++r) list[r] = O::empty();
      kth = O::empty();
      ring = 0;
    } else if (all_seen) {
      break;
    }
  }
}

// ---------------------------------------------------------------------------
// Radius query + sort: one warp per query point
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long shfl_xor_key(unsigned long long k, int m) {
  return __shfl_xor_sync(0xffffffffu, k, m);
}
__device__ __forceinline__ DKey shfl_xor_key(DKey k, int m) {
  return {__shfl_xor_sync(0xffffffffu, k.d, m), __shfl_xor_sync(0xffffffffu, k.i, m)};
}

// Bitonic sort of 64 keys held two per lane (element 32 r + lane in k[r]),
// ascending: 21 compare-exchange steps, all but one across lanes.
template <class T>
__device__ __forceinline__ void warp_bitonic64(typename KeyOps<T>::Key (&k)[2], int lane) {
  using O = KeyOps<T>;
#pragma unroll
  for (int kk = 2; kk <= 64; kk <<= 1) {
#pragma unroll
    for (int j = kk >> 1; j > 0; j >>= 1) {
      if (j == 32) {  // kk == 64: the partner is the lane's other register, ascending
        const auto lo = O::kmin(k[0], k[1]), hi = O::kmax(k[0], k[1]);
        k[0] = lo; k[1] = hi;
      } else {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const bool up = ((32 * r + lane) & kk) == 0;
          const auto o = shfl_xor_key(k[r], j);
          k[r] = (((lane & j) == 0) == up) ? O::kmin(k[r], o) : O::kmax(k[r], o);
        }
      }
    }
  }
}

// Exact MM nearest points of q (uniform across the warp) from one radius
// query: every accepted point whose squared distance is <= thr is gathered
// into buf (the warp's CAP = 64 keys of shared memory) and the gathered
// keys are sorted.  When at least MM and at most 64 points pass, the first
// MM of list (element 32 r + lane in list[r], the layout of warp_knn) are
// the MM nearest in (squared distance, index) order: every point left out
// is farther than thr, so farther than the MM-th gathered one.  The cells
// visited are those of the box q +- rad, which the caller sizes so that it
// holds every point within sqrt(thr) (rad rounded up with margin; cell
// coordinates are monotone in the position).  Returns false when the count
// is outside [MM, 64] (the caller then runs warp_knn); it stops scanning as
// soon as more than 64 points have passed.
template <class T, class PT, int MM, class Accept>
__device__ __forceinline__ bool warp_radius_knn(const GridGeom& g, const int* __restrict__ cell_start,
                                                const Pt4<PT>* __restrict__ pts, V3<T> q, T thr, float rad,
                                                int lane, Accept accept, typename KeyOps<T>::Key* buf,
                                                typename KeyOps<T>::Key (&list)[2]) {
  static_assert(MM >= 1 && MM <= 64, "at most 64 neighbours");
  constexpr int CAP = 64;
  using O = KeyOps<T>;
  using Key = typename O::Key;
  if (!finite3(q) || !(rad < INFINITY) || !(thr >= (T)0)) return false;
  const float qf[3] = {(float)q.x, (float)q.y, (float)q.z};
  int lo[3], hi[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    lo[ax] = grid_coord(g, __fsub_rd(qf[ax], rad), ax);
    hi[ax] = grid_coord(g, __fadd_ru(qf[ax], rad), ax);
  }
  const int ny = hi[1] - lo[1] + 1;
  const int nrows = ny * (hi[2] - lo[2] + 1);
  const unsigned below = (1u << lane) - 1u;
  int cnt = 0;
  for (int base = 0; base < nrows; base += 32) {
    // one (z, y) row of the box per lane: a contiguous range of sorted points
    const int rowi = base + lane;
    int b = 0, e = 0;
    if (rowi < nrows) {
      const int z = lo[2] + rowi / ny, y = lo[1] + rowi % ny;
      const int row = g.cell_base + (z * g.dim[1] + y) * g.dim[0];
      b = __ldg(cell_start + row + lo[0]);
      e = __ldg(cell_start + row + hi[0] + 1);
    }
    const int len = e - b;
    int incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int excl = incl - len;
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    for (int c = 0; c < total; c += 32) {
      const int i = c + lane;
      int src = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const int probe = src + step;
        const int ex = __shfl_sync(0xffffffffu, excl, probe & 31);
        if (probe < 32 && ex <= i) src = probe;
      }
      const int rb = __shfl_sync(0xffffffffu, b, src);
      const int rex = __shfl_sync(0xffffffffu, excl, src);
      bool pass = false;
      Key key = O::empty();
      if (i < total) {
        const Pt4<PT> p = pts[rb + (i - rex)];
        if (accept(p.id)) {
          const T d = dist2(V3<T>{(T)p.x, (T)p.y, (T)p.z}, q);
          key = O::make(d, p.id);
          pass = d <= thr;
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, pass);
      const int slot = cnt + __popc(m & below);
      if (pass && slot < CAP) buf[slot] = key;
      cnt += __popc(m);
      if (cnt > CAP) return false;
    }
  }
  if (cnt < MM) return false;
  __syncwarp();
  list[0] = lane < cnt ? buf[lane] : O::empty();
  list[1] = lane + 32 < cnt ? buf[lane + 32] : O::empty();
  __syncwarp();  // every lane has read buf before the next query writes it
  warp_bitonic64<T>(list, lane);
  return true;
}

// ---------------------------------------------------------------------------
// Warp-wide selection of the KK smallest keys of short lists, in order,
// one list per half warp (16 lanes) with three keys per lane (element
// e = 3 hl + r, hl = lane within the half): odd-even transposition passes
// until the first KK elements are in order and every later one is above the
// KK-th (the order among the later ones does not matter).  A list that is
// already nearly in order (a site's candidate list from an earlier
// iteration, re-keyed at the sites' new positions) needs a pass or two; 64
// passes order any list.  Every pass is an odd-even transposition of the
// half's 48 elements; both
// halves run the same passes (the shuffles are warp-wide), a half that is
// in order only repeats no-op exchanges.  `moved` tells whether this half's
// keys moved.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long shfl16_key(unsigned long long k, int src) {
  return __shfl_sync(0xffffffffu, k, src, 16);
}
__device__ __forceinline__ DKey shfl16_key(DKey k, int src) {
  return {__shfl_sync(0xffffffffu, k.d, src, 16), __shfl_sync(0xffffffffu, k.i, src, 16)};
}
__device__ __forceinline__ unsigned long long shfl16_down_key(unsigned long long k) {
  return __shfl_down_sync(0xffffffffu, k, 1, 16);
}
__device__ __forceinline__ DKey shfl16_down_key(DKey k) {
  return {__shfl_down_sync(0xffffffffu, k.d, 1, 16), __shfl_down_sync(0xffffffffu, k.i, 1, 16)};
}
__device__ __forceinline__ unsigned long long shfl16_up_key(unsigned long long k) {
  return __shfl_up_sync(0xffffffffu, k, 1, 16);
}
__device__ __forceinline__ DKey shfl16_up_key(DKey k) {
  return {__shfl_up_sync(0xffffffffu, k.d, 1, 16), __shfl_up_sync(0xffffffffu, k.i, 1, 16)};
}

template <class T, int KK>
__device__ __forceinline__ void half_select3(typename KeyOps<T>::Key (&k)[3], int hl, int half, bool& moved) {
  using O = KeyOps<T>;
  constexpr int KL = (KK - 1) / 3, KR = (KK - 1) % 3;  // lane and register of element KK-1
  const int e0 = 3 * hl;
  moved = false;
  for (int pass = 0; pass < 64; ++pass) {
    const auto nx0 = shfl16_down_key(k[0]);
    const auto kth = shfl16_key(k[KR], KL);
    const bool kth_empty = O::is_empty(kth);
    bool ok = true;
    if (e0 + 1 <= KK - 1) ok = ok && O::less(k[0], k[1]);
    if (e0 + 2 <= KK - 1) ok = ok && O::less(k[1], k[2]);
    if (e0 + 3 <= KK - 1 && hl < 15) ok = ok && O::less(k[2], nx0);
#pragma unroll
    for (int r = 0; r < 3; ++r)
      if (e0 + r >= KK) ok = ok && (kth_empty || O::less(kth, k[r]));
    const unsigned b = __ballot_sync(0xffffffffu, ok);
    if (b == 0xffffffffu) break;
    if (((b >> (16 * half)) & 0xffffu) != 0xffffu) moved = true;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const auto n0 = shfl16_down_key(k[0]);
      const auto p2 = shfl16_up_key(k[2]);
      if ((hl & 1) == p) {
        const auto lo = O::kmin(k[0], k[1]), hi = O::kmax(k[0], k[1]);
        k[0] = lo; k[1] = hi;
        if (hl < 15) k[2] = O::kmin(k[2], n0);
      } else {
        const auto lo = O::kmin(k[1], k[2]), hi = O::kmax(k[1], k[2]);
        k[1] = lo; k[2] = hi;
        if (hl > 0) k[0] = O::kmax(k[0], p2);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// grid build: count -> exclusive scan -> scatter
// ---------------------------------------------------------------------------
struct SegGrid {           // the minimal per-point view the build needs
  const GridGeom* geom;    // one geometry per segment
  const int* seg_of;       // segment of each point (nullptr: all segment 0)
  const int* active;       // per-segment state, 1 = iterating (nullptr: all)
};

template <class T>
__global__ void k_grid_count(int n, const T* __restrict__ P, SegGrid sg, int* __restrict__ cell_count,
                             int2* __restrict__ cellrank) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  int s = sg.seg_of ? sg.seg_of[g] : 0;
  if (s < 0 || (sg.active && sg.active[s] != 1)) { cellrank[g] = make_int2(-1, 0); return; }
  GridGeom G = sg.geom[s];
  int cell = grid_cell(G, ld3(P, g));
  int rank = atomicAdd(cell_count + cell, 1);
  cellrank[g] = make_int2(cell, rank);
}

template <class T>
__global__ void k_grid_scatter(int n, const T* __restrict__ P, const int2* __restrict__ cellrank,
                               const int* __restrict__ cell_start, Pt4<T>* __restrict__ sorted) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  int2 cr = cellrank[g];
  if (cr.x < 0) return;
  V3<T> p = ld3(P, g);
  Pt4<T> o;
  o.x = p.x; o.y = p.y; o.z = p.z; o.id = (uint32_t)g;
  sorted[cell_start[cr.x] + cr.y] = o;
}

// Exclusive scan of n ints: block sums, scan of the block sums, then a
// block-local rescan with the block offset.  out[n] = total.
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* smem_warp, int& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem_warp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = (lane < (blockDim.x >> 5)) ? smem_warp[lane] : 0;
    int ws = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, ws, o);
      if (lane >= o) ws += y;
    }
    smem_warp[lane] = ws - w;
    if (lane == 31) smem_warp[32] = ws;
  }
  __syncthreads();
  total = smem_warp[32];
  int r = smem_warp[wid] + x - v;
  __syncthreads();
  return r;
}

// one block scans the block sums tile by tile, carrying the running total
__device__ __forceinline__ void scan_partials_block(int nb, int* __restrict__ part, int* sw) {
  int carry = 0;
  for (int tile = 0; tile < nb; tile += kScanTile) {
    int base = tile + threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) { v[k] = (base + k < nb) ? part[base + k] : 0; s += v[k]; }
    int total;
    int off = block_exclusive_scan(s, sw, total) + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (base + k < nb) part[base + k] = off;
      off += v[k];
    }
    carry += total;
  }
  if (threadIdx.x == 0) part[nb] = carry;
}

// Block sums of the input.  With a ticket (a zeroed counter), the last block
// to finish also scans the block sums (the partials step), so the scan takes
// two launches; it leaves the ticket at zero again.
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(int n, const int* __restrict__ in, int* __restrict__ part,
                                                              unsigned* ticket) {
  __shared__ int sw[33];
  __shared__ bool last;
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) s += (base + k < n) ? in[base + k] : 0;
  int total;
  block_exclusive_scan(s, sw, total);
  if (threadIdx.x == 0) part[blockIdx.x] = total;
  if (ticket == nullptr) return;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  scan_partials_block(gridDim.x, part, sw);
  if (threadIdx.x == 0) *ticket = 0u;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_partials(int nb, int* __restrict__ part) {
  __shared__ int sw[33];
  scan_partials_block(nb, part, sw);
}

// clear_in: the input is zeroed once read (the engine's cell counts are then
// ready for the next iteration's counting without a memset)
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(int n, int* __restrict__ in, const int* __restrict__ part,
                                                             int* __restrict__ out, int clear_in) {
  __shared__ int sw[33];
  int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) { v[k] = (base + k < n) ? in[base + k] : 0; s += v[k]; }
  if (clear_in) {
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
      if (base + k < n) in[base + k] = 0;
  }
  int total;
  int off = block_exclusive_scan(s, sw, total) + part[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = off;
    off += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = part[gridDim.x];
}

inline int scan_blocks(int n) { return (n + kScanTile - 1) / kScanTile; }

// part must hold scan_blocks(n) + 1 ints
// Exclusive scan of n ints, out[n] = total.  With a ticket (a zeroed
// counter owned by the caller) two launches, else three; returns the number
// of launches.
inline int launch_exclusive_scan(int n, int* in, int* part, int* out, cudaStream_t st, bool clear_in = false,
                                 unsigned* ticket = nullptr) {
  int nb = scan_blocks(n);
  if (nb < 1) nb = 1;
  k_scan_reduce<<<nb, kScanThreads, 0, st>>>(n, in, part, ticket);
  if (ticket == nullptr) k_scan_partials<<<1, kScanThreads, 0, st>>>(nb, part);
  k_scan_apply<<<nb, kScanThreads, 0, st>>>(n, in, part, out, clear_in ? 1 : 0);
  return ticket == nullptr ? 3 : 2;
}

}  // namespace cvt
