// libgpucvt: C ABI (include/gpu_cvt.h) over the sm_100a kernels.
// Unity translation unit: the device code lives in the included headers.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include "../../include/gpu_cvt.h"
#include "cvt_eval.cuh"
#include "cvt_ingest.cuh"
#include "cvt_stage.cuh"

using namespace cvt;

// ---------------------------------------------------------------------------
// errors, launch accounting
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};

static cvt_status_t fail(cvt_status_t s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      return fail(e_ == cudaErrorMemoryAllocation ? CVT_ERR_OOM : CVT_ERR_CUDA,                  \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                           \
    }                                                                                            \
  } while (0)

#define LAUNCHED(n) g_launches.fetch_add((n), std::memory_order_relaxed)
#define CKLAUNCH()                                                                               \
  do {                                                                                           \
    LAUNCHED(1);                                                                                 \
    cudaError_t e_ = cudaGetLastError();                                                         \
    if (e_ != cudaSuccess) return fail(CVT_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
  } while (0)

static inline cudaStream_t S_(void* s) { return reinterpret_cast<cudaStream_t>(s); }
static inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

extern "C" const char* cvt_status_string(cvt_status_t s) {
  switch (s) {
    case CVT_OK: return "ok";
    case CVT_ERR_INVALID: return "invalid argument";
    case CVT_ERR_CUDA: return "CUDA error";
    case CVT_ERR_OOM: return "out of device memory";
    case CVT_ERR_UNSUPPORTED: return "unsupported";
    case CVT_ERR_CAPACITY: return "capacity exceeded";
  }
  return "unknown";
}
extern "C" const char* cvt_last_error(void) { return g_last_error.c_str(); }
extern "C" int cvt_version(void) { return 1; }
extern "C" unsigned long long cvt_launch_count(void) { return g_launches.load(); }

// Device memory: one stream-ordered pool per device, owned by the library,
// that keeps what is freed for the next allocation instead of handing it back
// to the driver (release threshold = unlimited).  Meshes, engines and call
// temporaries come and go without allocator calls into the driver once the
// pool has grown to the working set; cvt_release_cached_memory trims it.
static std::mutex g_pool_mu;
static std::vector<cudaMemPool_t> g_pools;

static cudaError_t lib_pool(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if ((int)g_pools.size() <= dev) g_pools.resize(dev + 1, nullptr);
  if (!g_pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
    uint64_t keep = ~0ull;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return e;
    }
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return cudaSuccess;
}

static cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st) {
  cudaMemPool_t pool;
  cudaError_t e = lib_pool(&pool);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(p, std::max<size_t>(bytes, 16), pool, st);
}

// long-lived objects: allocated and freed on the legacy stream, then waited for
static cudaError_t dev_alloc_sync(void** p, size_t bytes) {
  cudaError_t e = dev_alloc(p, bytes, 0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  return e;
}
static void dev_free_sync(void* p) {
  if (p) { cudaFreeAsync(p, 0); cudaStreamSynchronize(0); }
}

static void graph_cache_clear();

extern "C" cvt_status_t cvt_release_cached_memory(void) {
  graph_cache_clear();
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (cudaMemPool_t pool : g_pools)
    if (pool) {
      cudaError_t e = cudaMemPoolTrimTo(pool, 0);
      if (e != cudaSuccess) return fail(CVT_ERR_CUDA, std::string("cvt_release_cached_memory: ") + cudaGetErrorString(e));
    }
  return CVT_OK;
}

// streaming multiprocessors of the current device (grid size of the
// grid-stride fallback kernels: one block per SM)
static int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 148;
  return n > 0 ? n : 148;
}

// Streams a host thread runs engine iterations on besides the caller's: the
// second branch of an eagerly launched iteration, and the origin and second
// branch of a graph capture.  One set per thread and device, because a
// capture in cudaStreamCaptureModeThreadLocal must not share a stream with
// another thread's work; created on first use, destroyed at thread exit.
// (Creating and destroying streams per engine cost ~0.3 ms per one-call
// remesh.)
struct ThreadStreams {
  cudaStream_t side = nullptr, cap = nullptr, cap_side = nullptr;
};
struct ThreadStreamSet {
  std::vector<ThreadStreams> dev;
  ~ThreadStreamSet() {
    for (ThreadStreams& t : dev)
      for (cudaStream_t s : {t.side, t.cap, t.cap_side})
        if (s) cudaStreamDestroy(s);
  }
};
static cudaError_t thread_streams(ThreadStreams** out) {
  static thread_local ThreadStreamSet set;
  int d = 0;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess) return e;
  if ((int)set.dev.size() <= d) set.dev.resize(d + 1);
  ThreadStreams& t = set.dev[d];
  for (cudaStream_t* s : {&t.side, &t.cap, &t.cap_side})
    if (!*s && (e = cudaStreamCreateWithFlags(s, cudaStreamNonBlocking)) != cudaSuccess) return e;
  *out = &t;
  return cudaSuccess;
}

// stream-ordered scratch
struct Scratch {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit Scratch(cudaStream_t s) : st(s) {}
  template <class X> cudaError_t get(X** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = dev_alloc(&q, count * sizeof(X), st);
    if (e == cudaSuccess) { ptrs.push_back(q); *p = reinterpret_cast<X*>(q); }
    return e;
  }
  ~Scratch() { for (void* q : ptrs) cudaFreeAsync(q, st); }
};

// ---------------------------------------------------------------------------
// grid build over one device point set (stage API + mesh vertex grid)
// ---------------------------------------------------------------------------
struct PointGrid {
  GridGeom* geom = nullptr;
  int* cell_count = nullptr;
  int* cell_start = nullptr;
  int* part = nullptr;
  int2* cellrank = nullptr;
  Pt4<float>* sorted = nullptr;
  int total_cells = 0;  // scan length (spatial capacity + NaN bucket)
};

// geometry supplied by the host (hgeom != nullptr) or derived on the device
// from the bbox with ~per_cell points per cell
static cvt_status_t build_point_grid(Scratch& sc, const float* P, int n, float per_cell, const GridGeom* hgeom,
                                     PointGrid& pg) {
  cudaStream_t st = sc.st;
  int cap = hgeom ? hgeom->ncell : std::max(64, 2 * n);
  pg.total_cells = cap + 1;
  CK(sc.get(&pg.geom, 1));
  CK(sc.get(&pg.cell_count, (size_t)pg.total_cells));
  CK(sc.get(&pg.cell_start, (size_t)pg.total_cells + 1));
  CK(sc.get(&pg.part, (size_t)scan_blocks(pg.total_cells) + 2));
  CK(sc.get(&pg.cellrank, (size_t)std::max(n, 1)));
  CK(sc.get(&pg.sorted, (size_t)std::max(n, 1)));
  if (hgeom) {
    CK(cudaMemcpyAsync(pg.geom, hgeom, sizeof(GridGeom), cudaMemcpyHostToDevice, st));
  } else {
    int* bb;
    CK(sc.get(&bb, 6));
    k_bbox_init<<<1, 32, 0, st>>>(bb);
    CKLAUNCH();
    if (n > 0) { k_bbox<<<cdiv(n, 256), 256, 0, st>>>(n, P, bb); CKLAUNCH(); }
    k_grid_geom<<<1, 32, 0, st>>>(bb, n, per_cell, cap, pg.geom);
    CKLAUNCH();
  }
  CK(cudaMemsetAsync(pg.cell_count, 0, sizeof(int) * pg.total_cells, st));
  if (n > 0) {
    k_grid_count<float><<<cdiv(n, 256), 256, 0, st>>>(n, P, SegGrid{pg.geom, nullptr, nullptr}, pg.cell_count, pg.cellrank);
    CKLAUNCH();
  }
  launch_exclusive_scan(pg.total_cells, pg.cell_count, pg.part, pg.cell_start, st);
  LAUNCHED(3);
  CK(cudaGetLastError());
  if (n > 0) {
    k_grid_scatter<float><<<cdiv(n, 256), 256, 0, st>>>(n, P, pg.cellrank, pg.cell_start, pg.sorted);
    CKLAUNCH();
  }
  return CVT_OK;
}

// ---------------------------------------------------------------------------
// stage API
// ---------------------------------------------------------------------------
template <int KK>
static void launch_knn_points(const PointGrid& pg, int n, const uint8_t* frozen, int kk, uint32_t* knn, float* dist,
                              cudaStream_t st) {
  k_stage_knn_points<KK><<<cdiv(n, 128), 128, 0, st>>>(pg.geom, pg.cell_start, pg.sorted, pg.total_cells, frozen, kk,
                                                       knn, dist);
}
template <int KK>
static void launch_knn_query(const PointGrid& pg, const float* Q, int nQ, const uint8_t* frozen, int kk, int ex,
                             uint32_t* knn, float* dist, cudaStream_t st) {
  k_stage_knn_query<KK><<<cdiv(nQ, 128), 128, 0, st>>>(pg.geom, pg.cell_start, pg.sorted, Q, nQ, frozen, kk, ex, knn,
                                                       dist);
}

#define KK_DISPATCH(kk, FN, ...)                                 \
  do {                                                           \
    if ((kk) <= 1) FN<1>(__VA_ARGS__);                           \
    else if ((kk) <= 5) FN<5>(__VA_ARGS__);                      \
    else if ((kk) <= 9) FN<9>(__VA_ARGS__);                      \
    else if ((kk) <= 17) FN<17>(__VA_ARGS__);                    \
    else if ((kk) <= 21) FN<21>(__VA_ARGS__);                    \
    else if ((kk) <= 25) FN<25>(__VA_ARGS__);                    \
    else if ((kk) <= 33) FN<33>(__VA_ARGS__);                    \
    else FN<64>(__VA_ARGS__);                                    \
  } while (0)

extern "C" cvt_status_t cvt_knn_sites(const float* pts, int n, int kk, const uint8_t* frozen, uint32_t* knn,
                                      float* dist, void* stream) {
  if (n < 0 || kk < 1 || kk > 64 || (n > 0 && (!pts || !knn))) return fail(CVT_ERR_INVALID, "cvt_knn_sites: bad arguments");
  if (n == 0) return CVT_OK;
  cudaStream_t st = S_(stream);
  Scratch sc(st);
  PointGrid pg;
  cvt_status_t s = build_point_grid(sc, pts, n, 0.2f * kk, nullptr, pg);
  if (s != CVT_OK) return s;
  KK_DISPATCH(kk, launch_knn_points, pg, n, frozen, kk, knn, dist, st);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_knn_query_to_points(const float* cand, int n_cand, const float* query, int n_query, int kk,
                                                const uint8_t* frozen, uint32_t* knn, float* dist, void* stream) {
  if (n_cand < 0 || n_query < 0 || kk < 1 || kk > 64 || (n_query > 0 && (!query || !knn)) || (n_cand > 0 && !cand))
    return fail(CVT_ERR_INVALID, "cvt_knn_query_to_points: bad arguments");
  if (n_query == 0) return CVT_OK;
  cudaStream_t st = S_(stream);
  Scratch sc(st);
  PointGrid pg;
  cvt_status_t s = build_point_grid(sc, cand, n_cand, 0.2f * kk + 1.f, nullptr, pg);
  if (s != CVT_OK) return s;
  KK_DISPATCH(kk, launch_knn_query, pg, query, n_query, frozen, kk, 0, knn, dist, st);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_knn_vertices(const float* V, int nV, const float* Q, int nQ, int k, int exclude_self,
                                         const uint8_t* frozen, int* out, void* stream) {
  if (nV < 0 || nQ < 0 || k < 1 || k > 64 || (nQ > 0 && (!Q || !out)) || (nV > 0 && !V))
    return fail(CVT_ERR_INVALID, "cvt_knn_vertices: bad arguments");
  if (nQ == 0) return CVT_OK;
  cudaStream_t st = S_(stream);
  Scratch sc(st);
  PointGrid pg;
  cvt_status_t s = build_point_grid(sc, V, nV, 0.2f * k + 1.f, nullptr, pg);
  if (s != CVT_OK) return s;
  // int output: the uint32 sentinel 0xFFFFFFFF reads as -1
  KK_DISPATCH(k, launch_knn_query, pg, Q, nQ, frozen, k, exclude_self ? 1 : 0, reinterpret_cast<uint32_t*>(out),
              (float*)nullptr, st);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_knn_drop_self(const uint32_t* in, int n, int kin, int kout, uint32_t* out, void* stream) {
  if (n < 0 || kin < 1 || kout < 1 || (n > 0 && (!in || !out))) return fail(CVT_ERR_INVALID, "cvt_knn_drop_self: bad arguments");
  if (n == 0) return CVT_OK;
  k_stage_drop_self<<<cdiv(n, 256), 256, 0, S_(stream)>>>(in, n, kin, kout, out);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_restore_frozen_rows(const uint8_t* frozen, const uint32_t* prev, uint32_t* cur, int n, int k,
                                                void* stream) {
  if (n < 0 || k < 1 || (n > 0 && (!frozen || !prev || !cur))) return fail(CVT_ERR_INVALID, "cvt_restore_frozen_rows: bad arguments");
  if (n == 0) return CVT_OK;
  k_stage_restore_rows<<<cdiv(n, 256), 256, 0, S_(stream)>>>(frozen, prev, cur, n, k);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_vertex_normals(const float* V, int nV, const int* F, int nF, const int* vf_off,
                                           const int* vf_faces, float* N, void* stream) {
  if (nV < 0 || nF < 0 || (nV > 0 && (!V || !vf_off || !N)) || (nF > 0 && (!F || !vf_faces)))
    return fail(CVT_ERR_INVALID, "cvt_vertex_normals: bad arguments");
  if (nV == 0) return CVT_OK;
  k_stage_normals<<<cdiv(nV, 256), 256, 0, S_(stream)>>>(V, nV, F, vf_off, vf_faces, N);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_frames(const float* N0, const int* knnV, int kproj, int n, float* U, float* V, void* stream) {
  if (n < 0 || kproj < 1 || (n > 0 && (!N0 || !knnV || !U || !V))) return fail(CVT_ERR_INVALID, "cvt_frames: bad arguments");
  if (n == 0) return CVT_OK;
  k_stage_frames<<<cdiv(n, 256), 256, 0, S_(stream)>>>(N0, knnV, kproj, n, U, V);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_frames_pca(const float* S, int n, const uint32_t* knn, int K, const float* N0,
                                       const int* knnV, int kproj, float* U, float* V, void* stream) {
  if (n < 0 || K < 1 || kproj < 1 || (n > 0 && (!S || !knn || !N0 || !knnV || !U || !V)))
    return fail(CVT_ERR_INVALID, "cvt_frames_pca: bad arguments");
  if (n == 0) return CVT_OK;
  k_stage_frames_pca<<<cdiv(n, 128), 128, 0, S_(stream)>>>(S, n, knn, K, N0, knnV, kproj, U, V);
  CKLAUNCH();
  return CVT_OK;
}

constexpr int kClipBlock = 128;
constexpr int kClipCap = 32;

template <int PROF>
static cvt_status_t clip_dispatch(const float* S, const float* U, const float* V, const uint32_t* knn, int n, int K, float R,
                                  float* cent, int* nverts, cudaStream_t st) {
  Scratch sc(st);
  int* ovf;
  CK(sc.get(&ovf, (size_t)n + 1));
  CK(cudaMemsetAsync(ovf, 0, sizeof(int), st));
  const size_t smem = 2 * kClipCap * kClipBlock * sizeof(V2<float>);
  static bool attr = false;
  if (!attr) {
    CK(cudaFuncSetAttribute(k_stage_clip<PROF, kClipBlock, kClipCap>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  k_stage_clip<PROF, kClipBlock, kClipCap><<<cdiv(n, kClipBlock), kClipBlock, smem, st>>>(S, U, V, knn, n, K, R, cent, nverts, ovf);
  CKLAUNCH();
  k_stage_clip_fallback<PROF><<<sm_count(), 64, 0, st>>>(S, U, V, knn, n, K, R, cent, nverts, ovf);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_clip_centroids(const float* S, const float* U, const float* V, const uint32_t* knn, int n,
                                           int K, float R, int profile, float* cent, int* nverts, void* stream) {
  if (n < 0 || K < 1 || (n > 0 && (!S || !U || !V || !knn || !cent))) return fail(CVT_ERR_INVALID, "cvt_clip_centroids: bad arguments");
  if (profile != CVT_PROFILE_REF && profile != CVT_PROFILE_MIXED)
    return fail(CVT_ERR_UNSUPPORTED, "cvt_clip_centroids: profile must be REF or MIXED (FP64 runs in the engine)");
  if (n == 0) return CVT_OK;
  if (profile == CVT_PROFILE_REF) return clip_dispatch<PROF_REF>(S, U, V, knn, n, K, R, cent, nverts, S_(stream));
  return clip_dispatch<PROF_MIXED>(S, U, V, knn, n, K, R, cent, nverts, S_(stream));
}

extern "C" cvt_status_t cvt_project(const float* cent, const float* V, const int* F, const int* vf_off, const int* vf_faces,
                                    const int* knnV, int kproj, int nV, int nF, int nQ, int profile, const float* Sold,
                                    float* Snew, void* stream) {
  if (nQ < 0 || kproj < 1 || kproj > 16 || (nQ > 0 && (!cent || !V || !F || !vf_off || !vf_faces || !knnV || !Snew)))
    return fail(CVT_ERR_INVALID, "cvt_project: bad arguments");
  if (profile == CVT_PROFILE_MIXED && nQ > 0 && !Sold) return fail(CVT_ERR_INVALID, "cvt_project: MIXED needs Sold");
  if (profile != CVT_PROFILE_REF && profile != CVT_PROFILE_MIXED) return fail(CVT_ERR_UNSUPPORTED, "cvt_project: profile");
  if (nQ == 0) return CVT_OK;
  if (profile == CVT_PROFILE_REF)
    k_stage_project<PROF_REF><<<cdiv(nQ, 128), 128, 0, S_(stream)>>>(cent, V, F, vf_off, vf_faces, knnV, kproj, nV, nF, nQ, Sold, Snew);
  else
    k_stage_project<PROF_MIXED><<<cdiv(nQ, 128), 128, 0, S_(stream)>>>(cent, V, F, vf_off, vf_faces, knnV, kproj, nV, nF, nQ, Sold, Snew);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_freeze(const float* S, const float* Snew, const uint32_t* knn, const uint32_t* prev_knn, int n,
                                   int K, int has_prev, const uint8_t* tier, const float* thr2_tier, const int* need_tier,
                                   uint8_t* streak, uint8_t* cand, uint8_t* frozen, int* counts, void* stream) {
  if (n < 0 || K < 1 || !thr2_tier || !need_tier ||
      (n > 0 && (!S || !Snew || !knn || !prev_knn || !streak || !cand || !frozen || !counts)))
    return fail(CVT_ERR_INVALID, "cvt_freeze: bad arguments");
  if (n == 0) return CVT_OK;
  FreezeTable tab;
  for (int t = 0; t < 6; ++t) { tab.thr2[t] = thr2_tier[t]; tab.need[t] = need_tier[t]; }
  k_stage_freeze<<<cdiv(n, 256), 256, 0, S_(stream)>>>(S, Snew, knn, prev_knn, n, K, has_prev, tier, tab, streak, cand, frozen, counts);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_count_frozen(const uint8_t* frozen, int n, int* out_sum, void* stream) {
  if (n < 0 || !out_sum || (n > 0 && !frozen)) return fail(CVT_ERR_INVALID, "cvt_count_frozen: bad arguments");
  if (n == 0) return CVT_OK;
  k_stage_count_frozen<<<cdiv(n, 256), 256, 0, S_(stream)>>>(frozen, n, out_sum);
  CKLAUNCH();
  return CVT_OK;
}

extern "C" cvt_status_t cvt_tiers(int mode, int n, int K, const float* site_normal, const uint32_t* knn, uint8_t* tier,
                                  void* stream) {
  if ((mode != 1 && mode != 2) || n < 0 || K < 1 || (n > 0 && (!site_normal || !knn || !tier)))
    return fail(CVT_ERR_INVALID, "cvt_tiers: bad arguments");
  if (n == 0) return CVT_OK;
  k_stage_tiers<<<cdiv(n, 128), 128, 0, S_(stream)>>>(mode, n, K, site_normal, knn, tier);
  CKLAUNCH();
  return CVT_OK;
}

// ---------------------------------------------------------------------------
// resident meshes
// ---------------------------------------------------------------------------
struct cvt_mesh {
  int nV = 0, nF = 0;
  float R = 0.f, area = 0.f, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, diag = 0.f;
  float* dV = nullptr;
  int* dF = nullptr;
  int* doff = nullptr;
  int* dfcs = nullptr;
  float* dN = nullptr;
  double* dcdf = nullptr;  // face-area prefix sums (site sampler)
  GridGeom vg{};
  int* dvcell_start = nullptr;
  Pt4<float>* dvsorted = nullptr;
  float4* dring = nullptr;    // one-ring records (kRingWords per CSR entry)
  float* dunref = nullptr;    // input vertices no face uses (Hausdorff probes only)
  int n_unref = 0;
  BVHNode* dnodes = nullptr;  // built on first use (Hausdorff)
  int* dtri = nullptr;
  int nnodes = 0;
  void* arena = nullptr;      // V, F, CSR, normals, ring records, unreferenced vertices
  void* arena_grid = nullptr; // vertex grid (sized once the area is known)
  size_t bytes = 0;
  std::mutex lazy_mu;         // guards the first-use builds (BVH, area CDF)
  MeshDev dev() const {
    MeshDev m;
    m.V = dV; m.F = dF; m.vf_off = doff; m.vf_faces = dfcs; m.N = dN;
    m.vcell_start = dvcell_start; m.vsorted = dvsorted; m.ring = dring; m.vg = vg;
    m.bvh = dnodes; m.bvh_tri = dtri;
    m.nV = nV; m.nF = nF; m.R = R;
    m.thr2 = ((0.01f * R) * 0.01f) * R;
    return m;
  }
};

// Many device arrays carved out of one cudaMalloc (256-byte aligned slices):
// one allocator call and one free per object instead of one per array.
struct Arena {
  std::vector<std::pair<void**, size_t>> slots;
  size_t size = 0;
  template <class X> void add(X** p, size_t count) {
    slots.push_back({reinterpret_cast<void**>(p), size});
    size += (std::max<size_t>(count * sizeof(X), 16) + 255) & ~size_t(255);
  }
  cudaError_t commit(void** base) {
    cudaError_t e = dev_alloc_sync(base, std::max<size_t>(size, 256));
    if (e != cudaSuccess) { *base = nullptr; return e; }
    for (auto& s : slots) *s.first = static_cast<char*>(*base) + s.second;
    return cudaSuccess;
  }
};

static void mesh_free(cvt_mesh* m) {
  if (!m) return;
  dev_free_sync(m->arena); dev_free_sync(m->arena_grid); dev_free_sync(m->dcdf); dev_free_sync(m->dnodes);
  dev_free_sync(m->dtri);
  delete m;
}

// Subtree node count of the median-split BVH for n triangles (shape only).
static int bvh_subtree_nodes(int n, int leaf, std::vector<std::pair<int, int>>& memo) {
  if (n <= leaf) return 1;
  for (auto& kv : memo) if (kv.first == n) return kv.second;
  const int c = 1 + bvh_subtree_nodes(n / 2, leaf, memo) + bvh_subtree_nodes(n - n / 2, leaf, memo);
  memo.push_back({n, c});
  return c;
}

// BVH of the mesh (evaluate.cuh:114-201, leaf 8), built on the device level
// by level (cvt_ingest.cuh) the first time a Hausdorff distance needs it.
static cvt_status_t mesh_ensure_bvh(cvt_mesh* m) {
  std::lock_guard<std::mutex> lk(m->lazy_mu);
  if (m->dnodes) return CVT_OK;
  constexpr int leaf = 8;
  const int nF = m->nF;
  cudaStream_t st = 0;
  std::vector<std::pair<int, int>> memo;
  const int n_nodes = bvh_subtree_nodes(nF, leaf, memo);
  BVHNode* dn = nullptr;
  int* dt = nullptr;
  cudaError_t e = dev_alloc_sync(reinterpret_cast<void**>(&dn), sizeof(BVHNode) * (size_t)n_nodes);
  if (e == cudaSuccess) e = dev_alloc_sync(reinterpret_cast<void**>(&dt), sizeof(int) * (size_t)nF);
  auto bail = [&](cudaError_t err) {
    dev_free_sync(dn); dev_free_sync(dt);
    return fail(err == cudaErrorMemoryAllocation ? CVT_ERR_OOM : CVT_ERR_CUDA,
                std::string("mesh BVH: ") + cudaGetErrorString(err));
  };
  if (e != cudaSuccess) return bail(e);
  {
    Scratch sc(st);
    float* tinfo;
    int *ids2, *acc, *axis;
    unsigned long long *keys, *keys2;
    BvhSeg* dseg;
    // a split segment has more than `leaf` triangles, so both halves hold at
    // least leaf/2: the frontier never has more than nF/(leaf/2) + 1 segments
    const size_t max_seg = (size_t)nF / (leaf / 2) + 2;
    if ((e = sc.get(&tinfo, 9 * (size_t)nF)) != cudaSuccess || (e = sc.get(&ids2, (size_t)nF)) != cudaSuccess ||
        (e = sc.get(&keys, (size_t)nF)) != cudaSuccess || (e = sc.get(&keys2, (size_t)nF)) != cudaSuccess ||
        (e = sc.get(&acc, 12 * max_seg)) != cudaSuccess || (e = sc.get(&axis, max_seg)) != cudaSuccess ||
        (e = sc.get(&dseg, max_seg)) != cudaSuccess)
      return bail(e);
    k_tri_info<<<cdiv(nF, 256), 256, 0, st>>>(m->dV, m->dF, nF, tinfo);
    k_iota<<<cdiv(nF, 256), 256, 0, st>>>(dt, nF);
    LAUNCHED(2);
    size_t tb = 0;
    if ((e = cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, dt, ids2, nF, 0, 64, st)) != cudaSuccess)
      return bail(e);
    void* tmp;
    if ((e = sc.get(reinterpret_cast<char**>(&tmp), tb)) != cudaSuccess) return bail(e);
    std::vector<BvhSeg> segs{{0, nF, 0, -1, -1}};
    int* cur = dt;
    int* alt = ids2;
    while (true) {
      bool split = false;
      for (auto& g : segs)
        if (g.node >= 0 && g.count > leaf) {
          g.left = g.node + 1;
          g.right = g.node + 1 + bvh_subtree_nodes(g.count / 2, leaf, memo);
          split = true;
        }
      const int nseg = (int)segs.size();
      if ((e = cudaMemcpyAsync(dseg, segs.data(), sizeof(BvhSeg) * nseg, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return bail(e);
      k_seg_acc_init<<<cdiv(nseg, 256), 256, 0, st>>>(nseg, acc);
      k_seg_reduce<<<cdiv(nF, 256), 256, 0, st>>>(cur, nF, dseg, nseg, tinfo, acc);
      k_seg_emit<<<cdiv(nseg, 256), 256, 0, st>>>(dseg, nseg, acc, leaf, dn, axis);
      LAUNCHED(3);
      if (!split) break;
      k_seg_keys<<<cdiv(nF, 256), 256, 0, st>>>(cur, nF, dseg, nseg, axis, tinfo, keys);
      LAUNCHED(1);
      int sbits = 1;
      while (sbits < 31 && (1LL << sbits) < (long long)nseg) ++sbits;
      if ((e = cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, cur, alt, nF, 0, 32 + sbits, st)) != cudaSuccess)
        return bail(e);
      std::swap(cur, alt);
      std::vector<BvhSeg> next;
      next.reserve(2 * segs.size());
      for (const auto& g : segs) {
        if (g.node >= 0 && g.count > leaf) {
          next.push_back({g.start, g.count / 2, g.left, -1, -1});
          next.push_back({g.start + g.count / 2, g.count - g.count / 2, g.right, -1, -1});
        } else {
          next.push_back({g.start, g.count, -1, -1, -1});
        }
      }
      // (a pageable upload has left the host buffer when cudaMemcpyAsync
      // returns; the device copy is reused in stream order)
      segs.swap(next);
    }
    if (cur != dt && (e = cudaMemcpyAsync(dt, cur, sizeof(int) * (size_t)nF, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
      return bail(e);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(st)) != cudaSuccess) return bail(e);
  }
  m->nnodes = n_nodes;
  m->dtri = dt;
  m->bytes += sizeof(BVHNode) * (size_t)n_nodes + sizeof(int) * (size_t)nF;
  m->dnodes = dn;
  return CVT_OK;
}

// Face-area prefix sums (FP64) for the site sampler, built on first use.
static cvt_status_t mesh_ensure_cdf(cvt_mesh* m) {
  std::lock_guard<std::mutex> lk(m->lazy_mu);
  if (m->dcdf) return CVT_OK;
  const int nF = m->nF;
  cudaStream_t st = 0;
  double* d = nullptr;
  cudaError_t e = dev_alloc_sync(reinterpret_cast<void**>(&d), sizeof(double) * std::max(nF, 1));
  if (e == cudaSuccess) {
    Scratch sc(st);
    double* fa;
    size_t tb = 0;
    void* tmp;
    if ((e = sc.get(&fa, (size_t)nF)) == cudaSuccess &&
        (e = cub::DeviceScan::InclusiveSum(nullptr, tb, fa, d, nF, st)) == cudaSuccess &&
        (e = sc.get(reinterpret_cast<char**>(&tmp), tb)) == cudaSuccess) {
      k_face_area<<<cdiv(nF, 256), 256, 0, st>>>(m->dV, m->dF, nF, fa);
      LAUNCHED(1);
      if ((e = cudaGetLastError()) == cudaSuccess) e = cub::DeviceScan::InclusiveSum(tmp, tb, fa, d, nF, st);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    dev_free_sync(d);
    return fail(e == cudaErrorMemoryAllocation ? CVT_ERR_OOM : CVT_ERR_CUDA,
                std::string("mesh area CDF: ") + cudaGetErrorString(e));
  }
  m->bytes += sizeof(double) * nF;
  m->dcdf = d;
  return CVT_OK;
}

// Uniform grid for surface points: cell edge = factor * radius expected to
// hold k points at the surface density n/area; at most max_cells cells.
static GridGeom surface_grid(const float lo[3], const float hi[3], double area, long n, double k, double factor,
                             long max_cells) {
  GridGeom g{};
  double ext[3] = {(double)hi[0] - lo[0], (double)hi[1] - lo[1], (double)hi[2] - lo[2]};
  double emax = std::max({ext[0], ext[1], ext[2], 1e-20});
  double dens = (double)std::max<long>(n, 1) / std::max(area, 1e-30);
  double h = factor * std::sqrt(k / (M_PI * dens));
  h = std::max(h, emax / 2048.0);
  if (!(h > 0) || !std::isfinite(h)) h = emax;
  double pad = 1e-4 * emax;
  for (int it = 0; it < 200; ++it) {
    long prod = 1;
    for (int a = 0; a < 3; ++a) {
      g.dim[a] = std::max(1, (int)std::ceil((ext[a] + 2 * pad) / h));
      prod *= g.dim[a];
    }
    if (prod <= max_cells) break;
    h *= 1.05;
  }
  for (int a = 0; a < 3; ++a) g.lo[a] = (float)(lo[a] - pad);
  g.h = (float)h;
  g.inv_h = (float)(1.0 / h);
  g.cell_base = 0;
  g.ncell = g.dim[0] * g.dim[1] * g.dim[2];
  return g;
}

static float g_vcell_factor = 1.25f;   // swept 0.8-2.0 on the torus and rounded-box workloads

extern "C" void cvt_set_vertex_cell_factor(float f) { if (f > 0.f) g_vcell_factor = f; }

// The device does the ingest (cvt_ingest.cuh): upload, validation, bounds,
// compaction, areas and the face CSR; the host reads back five scalars to
// size the resident arrays and the vertex grid.
// Mesh ingest on stream st (the public call uses the legacy stream;
// cvt_remesh_batch ingests many meshes at once, one non-blocking stream per
// host thread).  Long-lived arrays come from the library pool on the legacy
// stream and are waited for before st uses them.
static cvt_status_t mesh_create_on(const float* V, int nV, const int* F, int nF, cvt_mesh_t* out, cudaStream_t st) {
  if (!out || !V || !F || nV <= 0 || nF <= 0) return fail(CVT_ERR_INVALID, "cvt_mesh_create: empty mesh or null pointer");
  cvt_mesh* m = new cvt_mesh();
  cudaError_t e = cudaSuccess;
#define MCK(x)                                                                              \
  do {                                                                                      \
    e = (x);                                                                                \
    if (e != cudaSuccess) {                                                                 \
      mesh_free(m);                                                                         \
      return fail(e == cudaErrorMemoryAllocation ? CVT_ERR_OOM : CVT_ERR_CUDA,              \
                  std::string("cvt_mesh_create: ") + cudaGetErrorString(e));                \
    }                                                                                       \
  } while (0)
  const long n3 = 3L * nF;
  Scratch sc(st);
  float* rV;
  int *rF, *used, *remap, *info;   // info: bad, bounds[12]
  double *farea, *area_sum;
  MCK(sc.get(&rV, 3 * (size_t)nV));
  MCK(sc.get(&rF, (size_t)n3));
  MCK(sc.get(&used, (size_t)nV));
  MCK(sc.get(&remap, (size_t)nV));
  MCK(sc.get(&info, 13));
  MCK(sc.get(&farea, (size_t)nF));
  MCK(sc.get(&area_sum, 1));
  MCK(cudaMemcpyAsync(rV, V, sizeof(float) * 3 * (size_t)nV, cudaMemcpyHostToDevice, st));
  MCK(cudaMemcpyAsync(rF, F, sizeof(int) * (size_t)n3, cudaMemcpyHostToDevice, st));
  MCK(cudaMemsetAsync(used, 0, sizeof(int) * (size_t)nV, st));
  MCK(cudaMemsetAsync(info, 0, sizeof(int), st));
  k_ingest_bounds_init<<<1, 32, 0, st>>>(info + 1);
  k_ingest_mark<<<cdiv(n3, 256), 256, 0, st>>>(rF, n3, nV, used, info);
  k_ingest_bounds<<<cdiv(nV, 256), 256, 0, st>>>(rV, nV, used, info + 1, info);
  LAUNCHED(3);
  MCK(cudaGetLastError());
  {
    size_t tb = 0;
    MCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, used, remap, nV, st));
    void* tmp;
    MCK(sc.get(reinterpret_cast<char**>(&tmp), tb));
    MCK(cub::DeviceScan::ExclusiveSum(tmp, tb, used, remap, nV, st));
  }
  int h[15];
  MCK(cudaMemcpyAsync(h, info, sizeof(int) * 13, cudaMemcpyDeviceToHost, st));
  MCK(cudaMemcpyAsync(h + 13, remap + nV - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaMemcpyAsync(h + 14, used + nV - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  if (h[0] & 1) { mesh_free(m); return fail(CVT_ERR_INVALID, "cvt_mesh_create: face index out of range"); }
  if (h[0] & 2) { mesh_free(m); return fail(CVT_ERR_INVALID, "cvt_mesh_create: non-finite coordinate in a face's vertex"); }
  auto ord2f = [](int o) { int b = o >= 0 ? o : o ^ 0x7fffffff; float f; std::memcpy(&f, &b, 4); return f; };
  // R over every input vertex (main.cu:169-227)
  float bmin[3], bmax[3];
  for (int a = 0; a < 3; ++a) {
    bmin[a] = ord2f(h[1 + a]); bmax[a] = ord2f(h[4 + a]);
    m->lo[a] = ord2f(h[7 + a]); m->hi[a] = ord2f(h[10 + a]);
  }
  m->R = std::fmax(bmax[0] - bmin[0], std::fmax(bmax[1] - bmin[1], bmax[2] - bmin[2]));
  const int nn = h[13] + h[14];
  m->nV = nn;
  m->nF = nF;
  m->n_unref = nV - nn;
  double dx = (double)m->hi[0] - m->lo[0], dy = (double)m->hi[1] - m->lo[1], dz = (double)m->hi[2] - m->lo[2];
  m->diag = (float)std::sqrt(dx * dx + dy * dy + dz * dz);
  Arena ar;
  ar.add(&m->dV, 3 * (size_t)nn);
  ar.add(&m->dF, (size_t)n3);
  ar.add(&m->doff, (size_t)nn + 1);
  ar.add(&m->dfcs, (size_t)n3);
  ar.add(&m->dN, 3 * (size_t)nn);
  ar.add(&m->dring, (size_t)kRingWords * 3 * nF);
  ar.add(&m->dunref, 3 * (size_t)m->n_unref);
  // the vertex grid's cell array is sized after the area is known
  MCK(ar.commit(&m->arena));
  m->bytes = ar.size;
  unsigned long long *keys, *keys2;
  int* vcount;
  MCK(sc.get(&keys, (size_t)n3));
  MCK(sc.get(&keys2, (size_t)n3));
  MCK(sc.get(&vcount, (size_t)nn + 1));
  MCK(cudaMemsetAsync(vcount, 0, sizeof(int) * ((size_t)nn + 1), st));
  k_ingest_compact<<<cdiv(nV, 256), 256, 0, st>>>(rV, nV, used, remap, m->dV, m->dunref);
  k_ingest_faces<<<cdiv(n3, 256), 256, 0, st>>>(rF, n3, remap, m->dF, keys, vcount);
  k_face_area<<<cdiv(nF, 256), 256, 0, st>>>(m->dV, m->dF, nF, farea);
  LAUNCHED(3);
  MCK(cudaGetLastError());
  {
    // vertex -> face CSR in face order (main.cu:259-285): sort (vertex, face)
    int vbits = 1;
    while (vbits < 32 && (1LL << vbits) <= (long long)nn) ++vbits;
    size_t tb_sort = 0, tb_scan = 0, tb_sum = 0;
    MCK(cub::DeviceRadixSort::SortKeys(nullptr, tb_sort, keys, keys2, (int)n3, 0, 32 + vbits, st));
    MCK(cub::DeviceScan::ExclusiveSum(nullptr, tb_scan, vcount, m->doff, nn + 1, st));
    MCK(cub::DeviceReduce::Sum(nullptr, tb_sum, farea, area_sum, nF, st));
    void* tmp;
    MCK(sc.get(reinterpret_cast<char**>(&tmp), std::max(tb_sort, std::max(tb_scan, tb_sum))));
    MCK(cub::DeviceRadixSort::SortKeys(tmp, tb_sort, keys, keys2, (int)n3, 0, 32 + vbits, st));
    k_keys_low32<<<cdiv(n3, 256), 256, 0, st>>>(keys2, n3, m->dfcs);
    LAUNCHED(1);
    MCK(cub::DeviceScan::ExclusiveSum(tmp, tb_scan, vcount, m->doff, nn + 1, st));
    MCK(cub::DeviceReduce::Sum(tmp, tb_sum, farea, area_sum, nF, st));
  }
  double area = 0.0;
  MCK(cudaMemcpyAsync(&area, area_sum, sizeof(double), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  m->area = (float)area;
  m->vg = surface_grid(m->lo, m->hi, area, nn, 6.0, g_vcell_factor, 4L * nn + 64);
  {
    Arena ag;
    ag.add(&m->dvcell_start, (size_t)m->vg.ncell + 2);
    ag.add(&m->dvsorted, (size_t)nn);
    MCK(ag.commit(&m->arena_grid));
    m->bytes += ag.size;
  }
  k_stage_normals<<<cdiv(nn, 256), 256, 0, st>>>(m->dV, nn, m->dF, m->doff, m->dfcs, m->dN);
  LAUNCHED(1);
  MCK(cudaGetLastError());
  k_build_ring_records<<<cdiv(n3, 256), 256, 0, st>>>(m->dV, m->dF, nF, m->dfcs, n3, m->dring);
  LAUNCHED(1);
  MCK(cudaGetLastError());
  {
    Scratch sg(st);
    PointGrid pg;
    cvt_status_t s = build_point_grid(sg, m->dV, nn, 0.f, &m->vg, pg);
    if (s != CVT_OK) { mesh_free(m); return s; }
    MCK(cudaMemcpyAsync(m->dvcell_start, pg.cell_start, sizeof(int) * (m->vg.ncell + 2), cudaMemcpyDeviceToDevice, st));
    MCK(cudaMemcpyAsync(m->dvsorted, pg.sorted, sizeof(Pt4<float>) * nn, cudaMemcpyDeviceToDevice, st));
  }
  MCK(cudaStreamSynchronize(st));
#undef MCK
  *out = m;
  return CVT_OK;
}

extern "C" cvt_status_t cvt_mesh_create(const float* V, int nV, const int* F, int nF, cvt_mesh_t* out) {
  return mesh_create_on(V, nV, F, nF, out, 0);
}

extern "C" cvt_status_t cvt_mesh_info(cvt_mesh_t m, cvt_mesh_info_t* info) {
  if (!m || !info) return fail(CVT_ERR_INVALID, "cvt_mesh_info: null");
  info->nV = m->nV; info->nF = m->nF; info->R = m->R; info->area = m->area;
  for (int a = 0; a < 3; ++a) { info->bbox_lo[a] = m->lo[a]; info->bbox_hi[a] = m->hi[a]; }
  info->diag = m->diag;
  info->device_bytes = m->bytes;
  return CVT_OK;
}

extern "C" cvt_status_t cvt_mesh_device_arrays(cvt_mesh_t m, const float** V, const int** F, const float** N,
                                               const int** vf_off, const int** vf_faces) {
  if (!m) return fail(CVT_ERR_INVALID, "cvt_mesh_device_arrays: null");
  if (V) *V = m->dV;
  if (F) *F = m->dF;
  if (N) *N = m->dN;
  if (vf_off) *vf_off = m->doff;
  if (vf_faces) *vf_faces = m->dfcs;
  return CVT_OK;
}

extern "C" cvt_status_t cvt_mesh_destroy(cvt_mesh_t m) {
  if (!m) return CVT_OK;
  cudaDeviceSynchronize();
  mesh_free(m);
  return CVT_OK;
}

extern "C" cvt_status_t cvt_hausdorff_to_mesh(cvt_mesh_t ref, const float* Vc, int nVc, const int* Fc, int nFc, float* out,
                                              void* stream) {
  if (!ref || !out || nVc < 0 || nFc < 0 || (nVc > 0 && !Vc) || (nFc > 0 && !Fc))
    return fail(CVT_ERR_INVALID, "cvt_hausdorff_to_mesh: bad arguments");
  cudaStream_t st = S_(stream);
  long nP = (long)nVc + 4L * nFc;
  if (nP == 0) { *out = 0.f; return CVT_OK; }
  cvt_status_t ls = mesh_ensure_bvh(ref);
  if (ls != CVT_OK) return ls;
  Scratch sc(st);
  unsigned* bits;
  int* ovf;
  CK(sc.get(&bits, 1));
  CK(sc.get(&ovf, 1));
  CK(cudaMemsetAsync(bits, 0, sizeof(unsigned), st));
  CK(cudaMemsetAsync(ovf, 0, sizeof(int), st));
  k_hausdorff<<<cdiv(nP, 128), 128, 0, st>>>(Vc, nVc, Fc, nP, ref->dnodes, ref->dtri, ref->dV, ref->dF, bits, ovf);
  CKLAUNCH();
  unsigned hb = 0;
  int ho = 0;
  CK(cudaMemcpyAsync(&hb, bits, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&ho, ovf, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (ho) return fail(CVT_ERR_CAPACITY, "cvt_hausdorff_to_mesh: BVH deeper than the traversal stack");
  float d2;
  std::memcpy(&d2, &hb, sizeof(float));
  *out = std::sqrt(d2);
  return CVT_OK;
}

extern "C" cvt_status_t cvt_mesh_get_bvh(cvt_mesh_t m, void* nodes, int nodes_cap, int* tri, int tri_cap, int* n_nodes) {
  if (!m || !n_nodes) return fail(CVT_ERR_INVALID, "cvt_mesh_get_bvh: null");
  cvt_status_t ls = mesh_ensure_bvh(m);
  if (ls != CVT_OK) return ls;
  *n_nodes = m->nnodes;
  if (nodes) {
    if (nodes_cap < m->nnodes) return fail(CVT_ERR_CAPACITY, "cvt_mesh_get_bvh: node buffer too small");
    CK(cudaMemcpy(nodes, m->dnodes, sizeof(BVHNode) * (size_t)m->nnodes, cudaMemcpyDeviceToHost));
  }
  if (tri) {
    if (tri_cap < m->nF) return fail(CVT_ERR_CAPACITY, "cvt_mesh_get_bvh: triangle buffer too small");
    CK(cudaMemcpy(tri, m->dtri, sizeof(int) * (size_t)m->nF, cudaMemcpyDeviceToHost));
  }
  return CVT_OK;
}

extern "C" cvt_status_t cvt_project_bvh(cvt_mesh_t m, const float* cent, int n, int profile, const float* Sold,
                                        float* Snew, void* stream) {
  if (!m || n < 0 || (n > 0 && (!cent || !Snew))) return fail(CVT_ERR_INVALID, "cvt_project_bvh: bad arguments");
  if (profile == CVT_PROFILE_MIXED && n > 0 && !Sold) return fail(CVT_ERR_INVALID, "cvt_project_bvh: MIXED needs Sold");
  if (profile != CVT_PROFILE_REF && profile != CVT_PROFILE_MIXED)
    return fail(CVT_ERR_UNSUPPORTED, "cvt_project_bvh: profile must be REF or MIXED (FP64 runs in the engine)");
  if (n == 0) return CVT_OK;
  cvt_status_t ls = mesh_ensure_bvh(m);
  if (ls != CVT_OK) return ls;
  cudaStream_t st = S_(stream);
  Scratch sc(st);
  int* ovf;
  CK(sc.get(&ovf, 1));
  CK(cudaMemsetAsync(ovf, 0, sizeof(int), st));
  if (profile == CVT_PROFILE_REF)
    k_stage_project_bvh<PROF_REF><<<cdiv(n, 128), 128, 0, st>>>(cent, n, m->dnodes, m->dtri, m->dV, m->dF, Sold, Snew, ovf);
  else
    k_stage_project_bvh<PROF_MIXED><<<cdiv(n, 128), 128, 0, st>>>(cent, n, m->dnodes, m->dtri, m->dV, m->dF, Sold, Snew, ovf);
  CKLAUNCH();
  int h_ovf = 0;
  CK(cudaMemcpyAsync(&h_ovf, ovf, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (h_ovf) return fail(CVT_ERR_CAPACITY, "cvt_project_bvh: BVH traversal stack overflow");
  return CVT_OK;
}

extern "C" cvt_status_t cvt_hausdorff_meshes(cvt_mesh_t a, cvt_mesh_t b, float* out, float* a_to_b, float* b_to_a,
                                             void* stream) {
  if (!a || !b || !out) return fail(CVT_ERR_INVALID, "cvt_hausdorff_meshes: bad arguments");
  cvt_status_t ls = mesh_ensure_bvh(a);
  if (ls == CVT_OK) ls = mesh_ensure_bvh(b);
  if (ls != CVT_OK) return ls;
  cudaStream_t st = S_(stream);
  Scratch sc(st);
  unsigned* bits;
  int* ovf;
  CK(sc.get(&bits, 2));
  CK(sc.get(&ovf, 1));
  CK(cudaMemsetAsync(bits, 0, 2 * sizeof(unsigned), st));
  CK(cudaMemsetAsync(ovf, 0, sizeof(int), st));
  // probes of `from` (every input vertex, then per face the centroid and the
  // three edge midpoints) against the BVH of `to`, max into *dst
  auto side = [&](const cvt_mesh* from, const cvt_mesh* to, unsigned* dst) -> cudaError_t {
    const long nP = (long)from->nV + 4L * from->nF;
    k_hausdorff<<<cdiv(nP, 128), 128, 0, st>>>(from->dV, from->nV, from->dF, nP, to->dnodes, to->dtri, to->dV,
                                               to->dF, dst, ovf);
    LAUNCHED(1);
    if (from->n_unref) {
      k_hausdorff<<<cdiv(from->n_unref, 128), 128, 0, st>>>(from->dunref, from->n_unref, nullptr, from->n_unref,
                                                             to->dnodes, to->dtri, to->dV, to->dF, dst, ovf);
      LAUNCHED(1);
    }
    return cudaGetLastError();
  };
  CK(side(a, b, bits));
  CK(side(b, a, bits + 1));
  unsigned hb[2] = {0, 0};
  int ho = 0;
  CK(cudaMemcpyAsync(hb, bits, sizeof(hb), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&ho, ovf, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (ho) return fail(CVT_ERR_CAPACITY, "cvt_hausdorff_meshes: BVH deeper than the traversal stack");
  float d2[2];
  std::memcpy(d2, hb, sizeof(d2));
  if (a_to_b) *a_to_b = std::sqrt(d2[0]);
  if (b_to_a) *b_to_a = std::sqrt(d2[1]);
  *out = std::sqrt(std::max(d2[0], d2[1]));
  return CVT_OK;
}

// ---------------------------------------------------------------------------
// engine
// ---------------------------------------------------------------------------
extern "C" void cvt_params_default(cvt_params_t* p) {
  if (!p) return;
  p->k = 24;
  p->mode = 0;
  p->profile = CVT_PROFILE_REF;
  p->kproj = 5;
  p->ex_quirk = 1;
  p->cell_factor = 1.1f;
  p->use_graph = 1;
  p->knn_block = p->clip_block = p->proj_block = 0;
  p->proj_mode = CVT_PROJ_ONERING;
  p->frame_mode = CVT_FRAME_VERTEX_NORMAL;
  p->knn_reuse = 1;
}

// launch shapes the tiles may take (cvt_params_t knn_block / clip_block /
// proj_block); 0 in the params selects the first
static const int kKnnBlocks[] = {128, 64, 256};
static const int kClipBlocksF[] = {128, 64};
static const int kClipBlocksD[] = {64, 32};
static const int kProjBlocks[] = {128, 64, 256};

static bool in_set(int v, const int* set, int n) {
  for (int i = 0; i < n; ++i) if (set[i] == v) return true;
  return false;
}
// fill 0 fields with the defaults; false if a field holds an unsupported shape
static bool resolve_tiles(cvt_params_t* p) {
  const bool f64 = p->profile == CVT_PROFILE_FP64;
  const int* clip = f64 ? kClipBlocksD : kClipBlocksF;
  if (p->knn_block == 0) p->knn_block = kKnnBlocks[0];
  if (p->clip_block == 0) p->clip_block = clip[0];
  if (p->proj_block == 0) p->proj_block = kProjBlocks[0];
  return in_set(p->knn_block, kKnnBlocks, 3) && in_set(p->clip_block, clip, 2) && in_set(p->proj_block, kProjBlocks, 3);
}

// first-fit interval allocator over [0, cap)
struct RangeAlloc {
  std::vector<std::pair<int, int>> free_;  // (start, len), sorted by start
  void init(int cap) { free_.assign(1, {0, cap}); }
  int take(int len) {
    if (len <= 0) return -1;
    for (size_t k = 0; k < free_.size(); ++k)
      if (free_[k].second >= len) {
        int s = free_[k].first;
        free_[k].first += len;
        free_[k].second -= len;
        if (free_[k].second == 0) free_.erase(free_.begin() + k);
        return s;
      }
    return -1;
  }
  void give(int s, int len) {
    if (len <= 0) return;
    free_.push_back({s, len});
    std::sort(free_.begin(), free_.end());
    std::vector<std::pair<int, int>> m;
    for (auto& r : free_) {
      if (!m.empty() && m.back().first + m.back().second == r.first) m.back().second += r.second;
      else m.push_back(r);
    }
    free_.swap(m);
  }
};

__global__ void k_fill_int(int* p, int n, int v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}
__global__ void k_f32_to_f64(const float* a, double* b, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}
__global__ void k_f64_to_f32(const double* a, float* b, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

struct cvt_engine {
  cvt_params_t p{};
  int K = 24, max_seg = 0, max_sites = 0, max_cells = 0;
  int dev = 0;  // device the engine lives on
  bool f64 = false;
  // host mirrors
  std::vector<SegDev> segs;
  std::vector<GridGeom> geom;
  std::vector<int> active;
  std::vector<cvt_mesh_t> seg_mesh;
  std::vector<int> seg_cells;  // cells reserved (spatial + NaN bucket)
  std::vector<int> host_iters;
  std::vector<int> seg_p0;  // global parity when the segment was placed
  RangeAlloc site_alloc, cell_alloc;
  int parity = 0;
  // device: every array below is a slice of one allocation
  void* arena = nullptr;
  size_t bytes = 0;
  SegDev* d_segs = nullptr;
  GridGeom* d_geom = nullptr;
  int* d_active = nullptr;
  MeshDev* d_meshes = nullptr;
  int* d_site_seg = nullptr;
  void* d_S[2] = {nullptr, nullptr};
  uint32_t* d_knn = nullptr;
  uint8_t* d_same = nullptr;
  float* d_kth = nullptr;
  int* d_act = nullptr;
  int* d_act_count = nullptr;
  int* d_knnv = nullptr;
  int* d_nnv = nullptr;
  uint8_t* d_frozen = nullptr;
  uint8_t* d_streak = nullptr;
  uint8_t* d_tier = nullptr;
  int2* d_cellrank = nullptr;
  void* d_sorted = nullptr;
  int* d_cell_count = nullptr;
  int* d_cell_start = nullptr;
  int* d_part = nullptr;
  int* d_stats = nullptr;
  int* d_ovf = nullptr;
  int* d_far = nullptr;
  unsigned* d_tickets = nullptr;  // [0] grid scan, [1] far sites + bookkeeping (zero between launches),
                                  // [2] BVH stack overflows of the projection (never expected)
  int num_sms = 148;
  void* d_cent = nullptr;
  uint32_t* d_cand = nullptr;   // candidate lists (knn_reuse): cand_len(K) global ids per site
  float* d_cand_rho = nullptr;
  float* d_cand_D = nullptr;
  int* d_srch = nullptr;          // sites left for a full KNN search, srch_cap slots per verify warp
  float* d_srch_thr = nullptr;    // per slot: the check's bound on the site's MM-th distance
  int* d_srch_n = nullptr;
  int srch_cap = 0;
  unsigned long long* d_blockmax = nullptr;  // per cell slot: coarse-block motion of the last step
  // graphs
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  // fork / join of the frame-vertex search, which runs on a second stream
  // while the site KNN runs: for eager iterations and for graph captures
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_cfork = nullptr, ev_cjoin = nullptr;
  int graph_nodes = 0;
  long long last_launches = 0;
};

// Instantiated iteration graphs of destroyed engines, kept for reuse: an
// engine whose iteration has the same shape (device, precision profile, K,
// launch shapes: the same kernels in the same order) loads its own kernel
// parameters into a kept graph with cudaGraphExecUpdate instead of
// instantiating a new one, and a destroyed engine hands its graphs back
// instead of destroying them (destroying two cost ~0.3 ms per one-call
// remesh).  At most kGraphCacheMax are kept; cvt_release_cached_memory
// destroys them.
struct GraphKey {
  int dev, profile, k, knn_block, clip_block, proj_block, proj_mode, frame_mode;
  bool knn_reuse;
  bool operator==(const GraphKey& o) const {
    return dev == o.dev && profile == o.profile && k == o.k && knn_block == o.knn_block &&
           clip_block == o.clip_block && proj_block == o.proj_block && proj_mode == o.proj_mode &&
           frame_mode == o.frame_mode && knn_reuse == o.knn_reuse;
  }
};
constexpr size_t kGraphCacheMax = 16;
static std::mutex g_graph_mu;
static std::vector<std::pair<GraphKey, cudaGraphExec_t>> g_graph_cache;

static GraphKey graph_key(const cvt_engine* e) {
  return {e->dev, e->p.profile, e->K, e->p.knn_block, e->p.clip_block, e->p.proj_block, e->p.proj_mode,
          e->p.frame_mode, e->p.knn_reuse != 0};
}

static cudaGraphExec_t graph_cache_take(const GraphKey& k) {
  std::lock_guard<std::mutex> lk(g_graph_mu);
  for (size_t i = 0; i < g_graph_cache.size(); ++i)
    if (g_graph_cache[i].first == k) {
      cudaGraphExec_t x = g_graph_cache[i].second;
      g_graph_cache.erase(g_graph_cache.begin() + i);
      return x;
    }
  return nullptr;
}

static void graph_cache_put(const GraphKey& k, cudaGraphExec_t x) {
  {
    std::lock_guard<std::mutex> lk(g_graph_mu);
    if (g_graph_cache.size() < kGraphCacheMax) { g_graph_cache.emplace_back(k, x); return; }
  }
  cudaGraphExecDestroy(x);
}

static void graph_cache_clear() {
  std::lock_guard<std::mutex> lk(g_graph_mu);
  for (auto& kv : g_graph_cache) cudaGraphExecDestroy(kv.second);
  g_graph_cache.clear();
}

// the graph of this iteration: a kept graph of the same shape updated with
// gr's parameters, else a new instantiation
static cudaError_t graph_exec_for(const GraphKey& k, cudaGraph_t gr, cudaGraphExec_t* out) {
  if (cudaGraphExec_t x = graph_cache_take(k)) {
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(x, gr, &info) == cudaSuccess) { *out = x; return cudaSuccess; }
    cudaGetLastError();  // a rejected update leaves no sticky error
    cudaGraphExecDestroy(x);
  }
  return cudaGraphInstantiate(out, gr, 0);
}

static void engine_free(cvt_engine* e) {
  if (!e) return;
  for (int k = 0; k < 2; ++k)
    if (e->gexec[k]) graph_cache_put(graph_key(e), e->gexec[k]);
  for (cudaEvent_t ev : {e->ev_fork, e->ev_join, e->ev_cfork, e->ev_cjoin})
    if (ev) cudaEventDestroy(ev);
  dev_free_sync(e->arena);
  delete e;
}

// candidate list length for the site KNN's list reuse: K + 16, even, <= 64
// (the longer the list, the longer it survives the sites' motion, and the
// more a refresh costs)
static constexpr int cand_len(int k) { return k + 16 > 64 ? 64 : k + 16; }

// Neighbours a site-grid cell is sized for (times cell_factor): K+1.  (Cells
// sized for the candidate list's length made its full searches cheaper but
// the coarse motion blocks coarser, which kept fewer lists: slower overall.)
static double grid_neighbours(const cvt_params_t& p) { return (double)(p.k + 1); }

static bool k_supported(int k) { return k == 8 || k == 12 || k == 16 || k == 20 || k == 24 || k == 32; }

extern "C" cvt_status_t cvt_engine_create(const cvt_params_t* p, int max_segments, int max_sites, int max_cells,
                                          cvt_engine_t* out) {
  if (!p || !out || max_segments < 1 || max_sites < 1 || max_cells < 2)
    return fail(CVT_ERR_INVALID, "cvt_engine_create: bad arguments");
  if (!k_supported(p->k)) return fail(CVT_ERR_UNSUPPORTED, "cvt_engine_create: k must be one of 8,12,16,20,24,32");
  if (p->kproj != kKProj) return fail(CVT_ERR_UNSUPPORTED, "cvt_engine_create: kproj must be 5");
  if (p->mode < 0 || p->mode > 2) return fail(CVT_ERR_INVALID, "cvt_engine_create: mode must be 0, 1 or 2");
  if (p->profile < 0 || p->profile > 2) return fail(CVT_ERR_INVALID, "cvt_engine_create: profile");
  if (p->proj_mode < 0 || p->proj_mode > 1) return fail(CVT_ERR_INVALID, "cvt_engine_create: proj_mode must be 0 or 1");
  if (p->frame_mode < 0 || p->frame_mode > 1) return fail(CVT_ERR_INVALID, "cvt_engine_create: frame_mode must be 0 or 1");
  cvt_params_t q = *p;
  if (!resolve_tiles(&q))
    return fail(CVT_ERR_UNSUPPORTED, "cvt_engine_create: knn_block / proj_block must be 64, 128 or 256, clip_block "
                                     "64 or 128 (FP64 profile: 32 or 64)");
  cvt_engine* e = new cvt_engine();
  e->p = q;
  e->num_sms = sm_count();
  cudaGetDevice(&e->dev);
  e->K = p->k;
  e->f64 = p->profile == CVT_PROFILE_FP64;
  e->max_seg = max_segments;
  e->max_sites = max_sites;
  e->max_cells = max_cells;
  e->segs.assign(max_segments, SegDev{});
  e->geom.assign(max_segments, GridGeom{});
  e->active.assign(max_segments, 0);
  e->seg_mesh.assign(max_segments, nullptr);
  e->seg_cells.assign(max_segments, 0);
  e->host_iters.assign(max_segments, 0);
  e->seg_p0.assign(max_segments, 0);
  e->site_alloc.init(max_sites);
  e->cell_alloc.init(max_cells);
  const size_t tsz = e->f64 ? sizeof(double) : sizeof(float);
  const size_t psz = e->f64 ? sizeof(Pt4<double>) : sizeof(Pt4<float>);
  cudaError_t err = cudaSuccess;
#define ECK(x)                                                                               \
  do {                                                                                       \
    err = (x);                                                                               \
    if (err != cudaSuccess) {                                                                \
      engine_free(e);                                                                        \
      return fail(err == cudaErrorMemoryAllocation ? CVT_ERR_OOM : CVT_ERR_CUDA,             \
                  std::string("cvt_engine_create: ") + cudaGetErrorString(err));             \
    }                                                                                        \
  } while (0)
  const size_t ns = (size_t)max_sites;
  Arena ar;
  ar.add(&e->d_segs, max_segments);
  ar.add(&e->d_geom, max_segments);
  ar.add(&e->d_active, max_segments);
  ar.add(&e->d_meshes, max_segments);
  ar.add(&e->d_site_seg, ns);
  for (int k = 0; k < 2; ++k) ar.add(reinterpret_cast<char**>(&e->d_S[k]), tsz * 3 * ns);
  ar.add(&e->d_knn, (size_t)e->K * ns);
  ar.add(&e->d_same, ns);
  ar.add(&e->d_kth, ns);
  ar.add(&e->d_act, ns);
  ar.add(&e->d_act_count, 1);
  ar.add(&e->d_knnv, (size_t)kKProj * ns);
  ar.add(&e->d_nnv, ns);
  ar.add(&e->d_frozen, ns);
  ar.add(&e->d_streak, ns);
  ar.add(&e->d_tier, ns);
  ar.add(&e->d_cellrank, ns);
  ar.add(reinterpret_cast<char**>(&e->d_sorted), psz * ns);
  ar.add(&e->d_cell_count, (size_t)max_cells);
  ar.add(&e->d_cell_start, (size_t)max_cells + 1);
  ar.add(&e->d_part, (size_t)scan_blocks(max_cells) + 2);
  ar.add(&e->d_stats, (size_t)max_segments * kStatsRing * kStatsWords);
  ar.add(&e->d_ovf, ns + 1);
  ar.add(&e->d_far, ns + 1);
  ar.add(&e->d_tickets, 3);  // scan ticket, bookkeeping ticket, BVH stack overflows
  ar.add(reinterpret_cast<char**>(&e->d_cent), tsz * 3 * ns);
  if (q.knn_reuse) {
    ar.add(&e->d_cand, (size_t)cand_len(e->K) * ns);
    ar.add(&e->d_cand_rho, ns);
    ar.add(&e->d_cand_D, ns);
    e->srch_cap = (int)cdiv((long)ns, (long)e->num_sms * kKnnVerifyWarpsPerSM) + 2;  // two sites per warp step
    ar.add(&e->d_srch, (size_t)e->srch_cap * e->num_sms * kKnnVerifyWarpsPerSM);
    ar.add(&e->d_srch_thr, (size_t)e->srch_cap * e->num_sms * kKnnVerifyWarpsPerSM);
    ar.add(&e->d_srch_n, (size_t)e->num_sms * kKnnVerifyWarpsPerSM);
    ar.add(&e->d_blockmax, (size_t)max_cells);
  }
  ECK(ar.commit(&e->arena));
  e->bytes = ar.size;
  ECK(cudaMemset(e->arena, 0, ar.size));
  k_fill_int<<<cdiv((long)ns, 256), 256>>>(e->d_site_seg, (int)ns, -1);
  LAUNCHED(1);
  ECK(cudaGetLastError());
  for (cudaEvent_t* ev : {&e->ev_fork, &e->ev_join, &e->ev_cfork, &e->ev_cjoin})
    ECK(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  ECK(cudaDeviceSynchronize());
#undef ECK
  *out = e;
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_destroy(cvt_engine_t e) {
  if (!e) return CVT_OK;
  cudaDeviceSynchronize();
  engine_free(e);
  return CVT_OK;
}

// defer_tables: leave the segment's entries of the device tables (segment,
// grid geometry, mesh view, active flag) and the final wait to the caller,
// which uploads the tables of many segments at once (each small copy from
// pageable host memory waits for the stream); the sites buffer must then
// stay valid until the stream has passed this segment's copy.
static cvt_status_t add_segment_impl(cvt_engine* e, cvt_mesh_t mesh, const float* sites, int n, int sites_on_device,
                                     int* seg_id, cudaStream_t st, bool defer_tables) {
  if (!e || !mesh || !sites || n < 1 || !seg_id) return fail(CVT_ERR_INVALID, "cvt_engine_add_segment: bad arguments");
  int s = -1;
  for (int k = 0; k < e->max_seg; ++k) if (!e->active[k] && !e->seg_mesh[k]) { s = k; break; }
  if (s < 0) return fail(CVT_ERR_CAPACITY, "cvt_engine_add_segment: no free segment slot");
  if (e->p.proj_mode == CVT_PROJ_BVH) {
    cvt_status_t bs = mesh_ensure_bvh(mesh);  // the projection walks it
    if (bs != CVT_OK) return bs;
  }
  GridGeom g = surface_grid(mesh->lo, mesh->hi, mesh->area, n, grid_neighbours(e->p), e->p.cell_factor, 4L * n + 64);
  int cells = g.ncell + 1;
  int base = e->site_alloc.take(n);
  if (base < 0) return fail(CVT_ERR_CAPACITY, "cvt_engine_add_segment: site capacity exhausted");
  int cbase = e->cell_alloc.take(cells);
  if (cbase < 0) { e->site_alloc.give(base, n); return fail(CVT_ERR_CAPACITY, "cvt_engine_add_segment: cell capacity exhausted"); }
  g.cell_base = cbase;
  SegDev sd{};
  sd.mesh = s;
  sd.site_base = base;
  sd.n_sites = n;
  sd.mode = e->p.mode;
  sd.ex_quirk = e->p.ex_quirk;
  sd.iter = 0;
  // twice the (K+1)-th squared distance of a uniform planar density n/area
  sd.kth_est = (float)(2.0 * (e->K + 1) * (double)mesh->area / (M_PI * (double)n));
  sd.stop_motion2 = -1.f;
  sd.stop_iters = 0;
  MeshDev md = mesh->dev();
  static const int kStreak1[6] = {5, 10, 15, 20, 25, 25};  // main.cu:22, 543-553
  static const int kStreak2[6] = {5, 10, 15, 20, 25, 10};  // main.cu:39, 554-563
  for (int t = 0; t < 6; ++t) {
    sd.thr2_tier[t] = md.thr2;
    int stv = e->p.mode == 0 ? 5 : (e->p.mode == 1 ? kStreak1[t] : kStreak2[t]);
    sd.need_tier[t] = std::max(1, stv - 1);
  }
  e->segs[s] = sd;
  e->geom[s] = g;
  e->active[s] = 1;
  e->seg_mesh[s] = mesh;
  e->seg_cells[s] = cells;
  e->host_iters[s] = 0;
  e->seg_p0[s] = e->parity;
  const size_t tsz = e->f64 ? sizeof(double) : sizeof(float);
  if (!defer_tables) {
    CK(cudaMemcpyAsync(e->d_segs + s, &e->segs[s], sizeof(SegDev), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(e->d_geom + s, &e->geom[s], sizeof(GridGeom), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(e->d_meshes + s, &md, sizeof(MeshDev), cudaMemcpyHostToDevice, st));
  }
  char* Sdst = (char*)e->d_S[e->parity] + tsz * 3 * (size_t)base;
  if (!e->f64) {
    CK(cudaMemcpyAsync(Sdst, sites, sizeof(float) * 3 * (size_t)n,
                       sites_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  } else {
    const float* src = sites;
    Scratch sc(st);
    if (!sites_on_device) {
      float* tmp;
      CK(sc.get(&tmp, 3 * (size_t)n));
      CK(cudaMemcpyAsync(tmp, sites, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, st));
      src = tmp;
    }
    k_f32_to_f64<<<cdiv(3L * n, 256), 256, 0, st>>>(src, (double*)Sdst, 3L * n);
    CKLAUNCH();
  }
  k_fill_int<<<cdiv(n, 256), 256, 0, st>>>(e->d_site_seg + base, n, s);
  CKLAUNCH();
  k_fill_int<<<cdiv(5L * n, 256), 256, 0, st>>>(e->d_knnv + 5L * base, 5 * n, -1);
  CKLAUNCH();
  CK(cudaMemsetAsync(e->d_frozen + base, 0, n, st));
  CK(cudaMemsetAsync(e->d_streak + base, 0, n, st));
  CK(cudaMemsetAsync(e->d_tier + base, 0, n, st));
  CK(cudaMemsetAsync(e->d_knn + (size_t)e->K * base, 0, sizeof(uint32_t) * e->K * (size_t)n, st));
  CK(cudaMemsetAsync(e->d_same + base, 0, n, st));
  k_fill_int<<<cdiv(n, 256), 256, 0, st>>>(reinterpret_cast<int*>(e->d_kth) + base, n, (int)0xbf800000);  // -1.0f
  CKLAUNCH();
  if (e->d_cand_rho) {  // no candidate lists yet; no motion recorded in the segment's blocks
    k_fill_int<<<cdiv(n, 256), 256, 0, st>>>(reinterpret_cast<int*>(e->d_cand_rho) + base, n, (int)0xbf800000);
    CKLAUNCH();
    CK(cudaMemsetAsync(e->d_blockmax + cbase, 0, sizeof(unsigned long long) * (size_t)cells, st));
  }
  CK(cudaMemsetAsync(e->d_stats + (size_t)s * kStatsRing * kStatsWords, 0, sizeof(int) * kStatsRing * kStatsWords, st));
  *seg_id = s;
  if (defer_tables) return CVT_OK;
  CK(cudaMemcpyAsync(e->d_active + s, &e->active[s], sizeof(int), cudaMemcpyHostToDevice, st));
  // the host mirrors above are read by the async copies; keep them stable
  CK(cudaStreamSynchronize(st));
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_add_segment(cvt_engine_t e, cvt_mesh_t mesh, const float* sites, int n,
                                               int sites_on_device, int* seg_id, void* stream) {
  return add_segment_impl(e, mesh, sites, n, sites_on_device, seg_id, S_(stream), false);
}

// The device tables of every segment slot from the host mirrors, in four
// copies, then a wait (after add_segment_impl with defer_tables).
static cvt_status_t upload_segment_tables(cvt_engine* e, cudaStream_t st) {
  std::vector<MeshDev> md(e->max_seg);
  for (int k = 0; k < e->max_seg; ++k)
    if (e->seg_mesh[k]) md[k] = e->seg_mesh[k]->dev();
  CK(cudaMemcpyAsync(e->d_segs, e->segs.data(), sizeof(SegDev) * e->max_seg, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(e->d_geom, e->geom.data(), sizeof(GridGeom) * e->max_seg, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(e->d_meshes, md.data(), sizeof(MeshDev) * e->max_seg, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(e->d_active, e->active.data(), sizeof(int) * e->max_seg, cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_remove_segment(cvt_engine_t e, int s) {
  if (!e || s < 0 || s >= e->max_seg || !e->seg_mesh[s]) return fail(CVT_ERR_INVALID, "cvt_engine_remove_segment: bad segment");
  CK(cudaDeviceSynchronize());
  e->active[s] = 0;
  CK(cudaMemcpy(e->d_active + s, &e->active[s], sizeof(int), cudaMemcpyHostToDevice));
  k_fill_int<<<cdiv(e->segs[s].n_sites, 256), 256>>>(e->d_site_seg + e->segs[s].site_base, e->segs[s].n_sites, -1);
  CKLAUNCH();
  CK(cudaDeviceSynchronize());
  e->site_alloc.give(e->segs[s].site_base, e->segs[s].n_sites);
  e->cell_alloc.give(e->geom[s].cell_base, e->seg_cells[s]);
  e->seg_mesh[s] = nullptr;
  return CVT_OK;
}

constexpr int kCellCap = 16;

template <class T> static EngineArgs<T> engine_args(cvt_engine* e) {
  EngineArgs<T> a;
  a.segs = e->d_segs; a.geom = e->d_geom; a.active = e->d_active; a.meshes = e->d_meshes; a.site_seg = e->d_site_seg;
  a.S[0] = (T*)e->d_S[0]; a.S[1] = (T*)e->d_S[1];
  a.knn = e->d_knn; a.same = e->d_same; a.kth = e->d_kth; a.act = e->d_act; a.act_count = e->d_act_count;
  a.knnv = e->d_knnv; a.nnv = e->d_nnv;
  a.frozen = e->d_frozen; a.streak = e->d_streak; a.tier = e->d_tier;
  a.cell_start = e->d_cell_start; a.sorted = (const Pt4<T>*)e->d_sorted; a.total_cells = e->max_cells;
  a.stats = e->d_stats; a.ovf = e->d_ovf; a.far = e->d_far; a.cent = (T*)e->d_cent; a.K = e->K;
  a.proj_mode = e->p.proj_mode; a.bvh_ovf = reinterpret_cast<int*>(e->d_tickets + 2);
  a.cand = e->d_cand; a.cand_rho = e->d_cand_rho; a.cand_D = e->d_cand_D; a.srch = e->d_srch; a.srch_thr = e->d_srch_thr; a.srch_n = e->d_srch_n; a.srch_cap = e->srch_cap; a.blockmax = e->d_blockmax;
  return a;
}

// the site KNN: with candidate lists, the check (one warp per active site)
// and then the full searches of the sites it left (a grid-stride kernel);
// without, the full searches of every active site.  Returns the launches.
template <class T, int KK, int MM, int BS>
static int launch_site_knn_b(const EngineArgs<T>& a, int parity, int nsites, int nsm, cudaStream_t st) {
  (void)nsites;
  const int vgrid = nsm * (kKnnVerifyWarpsPerSM * 32 / BS);  // the shape a.srch_cap is sized for
  int L = 0;
  if constexpr (MM > 0) {
    k_knn_verify<T, KK, MM, BS><<<vgrid, BS, 0, st>>>(a, parity);
    L++;
  }
  k_knn_search<T, KK, MM, BS><<<nsm * (kKnnSearchWarpsPerSM * 32 / BS), BS, 0, st>>>(a, parity,
                                                                                    nsm * kKnnVerifyWarpsPerSM);
  return L + 1;
}

template <class T, int KK, int MM>
static int launch_site_knn_m(const EngineArgs<T>& a, int parity, int nsites, int bs, int nsm, cudaStream_t st) {
  if (bs == 64) return launch_site_knn_b<T, KK, MM, 64>(a, parity, nsites, nsm, st);
  if (bs == 256) return launch_site_knn_b<T, KK, MM, 256>(a, parity, nsites, nsm, st);
  return launch_site_knn_b<T, KK, MM, 128>(a, parity, nsites, nsm, st);
}

template <class T, int KK>
static int launch_site_knn(const EngineArgs<T>& a, int parity, int nsites, int bs, bool reuse, int nsm,
                           cudaStream_t st) {
  if (reuse) return launch_site_knn_m<T, KK, cand_len(KK)>(a, parity, nsites, bs, nsm, st);
  return launch_site_knn_m<T, KK, 0>(a, parity, nsites, bs, nsm, st);
}

template <int PROF, int FRAME>
static void launch_site_clip_f(const EngineArgs<typename PT<PROF>::T>& a, int parity, int ns, int bs, int nsm,
                               cudaStream_t st) {
  using PP = typename PT<PROF>::PP;
  const size_t smem = 2 * kCellCap * (size_t)bs * sizeof(V2<PP>);
  if (sizeof(PP) == 8) {
    if (bs == 32) k_site_clip<PROF, 32, kCellCap, FRAME><<<cdiv(ns, 32), 32, smem, st>>>(a, parity);
    else k_site_clip<PROF, 64, kCellCap, FRAME><<<cdiv(ns, 64), 64, smem, st>>>(a, parity);
  } else {
    if (bs == 64) k_site_clip<PROF, 64, kCellCap, FRAME><<<cdiv(ns, 64), 64, smem, st>>>(a, parity);
    else k_site_clip<PROF, 128, kCellCap, FRAME><<<cdiv(ns, 128), 128, smem, st>>>(a, parity);
  }
  k_clip_overflow<PROF, FRAME><<<nsm, 64, 0, st>>>(a, parity);
}

// the clip kernel and its overflow fallback (two launches)
template <int PROF>
static void launch_site_clip(const EngineArgs<typename PT<PROF>::T>& a, int parity, int ns, int bs, int frame_mode,
                             int nsm, cudaStream_t st) {
  if (frame_mode == 1) launch_site_clip_f<PROF, 1>(a, parity, ns, bs, nsm, st);
  else launch_site_clip_f<PROF, 0>(a, parity, ns, bs, nsm, st);
}

template <int PROF, int PROJ>
static void launch_site_proj_p(const EngineArgs<typename PT<PROF>::T>& a, int parity, int ns, int bs, cudaStream_t st) {
  if (bs == 64) k_site_proj<PROF, 64, PROJ><<<cdiv(ns, 64), 64, 0, st>>>(a, parity);
  else if (bs == 256) k_site_proj<PROF, 256, PROJ><<<cdiv(ns, 256), 256, 0, st>>>(a, parity);
  else k_site_proj<PROF, 128, PROJ><<<cdiv(ns, 128), 128, 0, st>>>(a, parity);
}

template <int PROF>
static void launch_site_proj(const EngineArgs<typename PT<PROF>::T>& a, int parity, int ns, int bs, int proj_mode,
                             cudaStream_t st) {
  if (proj_mode == 1) launch_site_proj_p<PROF, 1>(a, parity, ns, bs, st);
  else launch_site_proj_p<PROF, 0>(a, parity, ns, bs, st);
}


// the second branch of an iteration: its stream and the fork / join events
struct Branch {
  cudaStream_t side;
  cudaEvent_t fork, join;
};

// ev (optional, 6 events): recorded before the grid build, after it, after
// the KNN kernel, after the clip kernels, after the projection kernels and
// after the bookkeeping kernel
template <int PROF>
static cvt_status_t enqueue_iteration_t(cvt_engine* e, int parity, cudaStream_t st, const Branch& br, int* nlaunch,
                                        cudaEvent_t* ev) {
  using T = typename PT<PROF>::T;
  using PP = typename PT<PROF>::PP;
  EngineArgs<T> a = engine_args<T>(e);
  const int ns = e->max_sites;
  int L = 0;
  if (ev) CK(cudaEventRecord(ev[0], st));
  // d_cell_count is all zero here: set at creation, cleared by the scan
  k_grid_count<T><<<cdiv(ns, 256), 256, 0, st>>>(ns, (const T*)e->d_S[parity], SegGrid{e->d_geom, e->d_site_seg, e->d_active},
                                                 e->d_cell_count, e->d_cellrank);
  L++;
  L += launch_exclusive_scan(e->max_cells, e->d_cell_count, e->d_part, e->d_cell_start, st, true, e->d_tickets);
  k_grid_scatter<T><<<cdiv(ns, 256), 256, 0, st>>>(ns, (const T*)e->d_S[parity], e->d_cellrank, e->d_cell_start,
                                                   (Pt4<T>*)e->d_sorted);
  L++;
  // cell_start[max_cells] is the number of gridded sites (read on the device)
  a.total_cells = e->max_cells;
  // d_act_count is zero here: set at creation, reset by the bookkeeping
  k_active_list<T><<<cdiv(ns, kActiveListThreads), kActiveListThreads, 0, st>>>(a);
  L++;
  // the frame vertices are first read by the clip: search them on the side
  // stream while the site KNN runs
  CK(cudaEventRecord(br.fork, st));
  CK(cudaStreamWaitEvent(br.side, br.fork, 0));
  k_frame_vertex<T><<<cdiv(ns, 128), 128, 0, br.side>>>(a);
  CK(cudaEventRecord(br.join, br.side));
  L++;
  if (ev) CK(cudaEventRecord(ev[1], st));
  const bool reuse = e->p.knn_reuse != 0;
  const int nsm = e->num_sms;
  switch (e->K) {
    case 8: L += launch_site_knn<T, 8>(a, parity, ns, e->p.knn_block, reuse, nsm, st); break;
    case 12: L += launch_site_knn<T, 12>(a, parity, ns, e->p.knn_block, reuse, nsm, st); break;
    case 16: L += launch_site_knn<T, 16>(a, parity, ns, e->p.knn_block, reuse, nsm, st); break;
    case 20: L += launch_site_knn<T, 20>(a, parity, ns, e->p.knn_block, reuse, nsm, st); break;
    case 24: L += launch_site_knn<T, 24>(a, parity, ns, e->p.knn_block, reuse, nsm, st); break;
    default: L += launch_site_knn<T, 32>(a, parity, ns, e->p.knn_block, reuse, nsm, st); break;
  }
  if (ev) CK(cudaEventRecord(ev[2], st));
  CK(cudaStreamWaitEvent(st, br.join, 0));
  launch_site_clip<PROF>(a, parity, ns, e->p.clip_block, e->p.frame_mode, e->num_sms, st);
  L += 2;
  if (ev) CK(cudaEventRecord(ev[3], st));
  if (e->p.proj_mode == CVT_PROJ_ONERING) {
    k_site_vsearch<PROF, 128><<<cdiv(ns, 128), 128, 0, st>>>(a, parity);
    L++;
  }
  launch_site_proj<PROF>(a, parity, ns, e->p.proj_block, e->p.proj_mode, st);
  k_site_far<PROF><<<e->num_sms, 128, 0, st>>>(a, parity, e->d_segs, e->d_active, e->max_seg, e->d_tickets + 1);
  L += 2;
  if (ev) CK(cudaEventRecord(ev[4], st));
  if (ev) CK(cudaEventRecord(ev[5], st));
  CK(cudaGetLastError());
  *nlaunch = L;
  return CVT_OK;
}

static cvt_status_t enqueue_iteration(cvt_engine* e, int parity, cudaStream_t st, const Branch& br, int* nlaunch,
                                      cudaEvent_t* ev = nullptr) {
  switch (e->p.profile) {
    case CVT_PROFILE_REF: return enqueue_iteration_t<PROF_REF>(e, parity, st, br, nlaunch, ev);
    case CVT_PROFILE_MIXED: return enqueue_iteration_t<PROF_MIXED>(e, parity, st, br, nlaunch, ev);
    default: return enqueue_iteration_t<PROF_FP64>(e, parity, st, br, nlaunch, ev);
  }
}

// k_site_clip's dynamic shared memory (two 16-vertex polygon buffers per
// thread) is at most 32 KB per block for every launch shape, within the
// default 48 KB limit, so no function attribute is needed.
static_assert(2 * kCellCap * 128 * sizeof(V2<float>) <= 48 * 1024 && 2 * kCellCap * 64 * sizeof(V2<double>) <= 48 * 1024,
              "clip buffers exceed the default dynamic shared memory limit");

extern "C" cvt_status_t cvt_engine_run(cvt_engine_t e, int iters, void* stream) {
  if (!e || iters < 0) return fail(CVT_ERR_INVALID, "cvt_engine_run: bad arguments");
  cudaStream_t st = S_(stream);
  cvt_status_t s = CVT_OK;
  long long launches = 0;
  ThreadStreams* ts = nullptr;
  if (iters > 0) CK(thread_streams(&ts));
  const Branch eager{ts ? ts->side : nullptr, e->ev_fork, e->ev_join};
  e->last_launches = 0;
  for (int it = 0; it < iters; ++it) {
    const int par = e->parity;
    const bool capture = e->p.use_graph && !e->gexec[par];
    int nl = 0;
    if (e->p.use_graph && !capture) {
      CK(cudaGraphLaunch(e->gexec[par], st));
      nl = e->graph_nodes;
    } else {
      // an iteration without a graph yet runs eagerly; its graph is then
      // captured and instantiated while the GPU runs it
      s = enqueue_iteration(e, par, st, eager, &nl);
      if (s != CVT_OK) return s;
    }
    LAUNCHED(nl);
    // the iteration is enqueued: account for it before anything can fail
    launches += nl;
    e->last_launches = launches;
    e->parity ^= 1;
    for (int k = 0; k < e->max_seg; ++k) if (e->active[k] == 1) e->host_iters[k]++;
    if (capture) {
      int ng = 0;
      CK(cudaStreamBeginCapture(ts->cap, cudaStreamCaptureModeThreadLocal));
      cvt_status_t q = enqueue_iteration(e, par, ts->cap, Branch{ts->cap_side, e->ev_cfork, e->ev_cjoin}, &ng);
      cudaGraph_t gr = nullptr;
      cudaError_t ce = cudaStreamEndCapture(ts->cap, &gr);
      if (q != CVT_OK) { if (gr) cudaGraphDestroy(gr); return q; }
      if (ce != cudaSuccess) return fail(CVT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      ce = graph_exec_for(graph_key(e), gr, &e->gexec[par]);
      cudaGraphDestroy(gr);
      if (ce != cudaSuccess) return fail(CVT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
      e->graph_nodes = ng;
    }
  }
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_profile(cvt_engine_t e, int iters, float* ms, void* stream) {
  if (!e || !ms || iters < 1) return fail(CVT_ERR_INVALID, "cvt_engine_profile: bad arguments");
  cudaStream_t st = S_(stream);
  cvt_status_t s = CVT_OK;
  ThreadStreams* ts = nullptr;
  CK(thread_streams(&ts));
  cudaEvent_t ev[6];
  for (int k = 0; k < 6; ++k) CK(cudaEventCreate(&ev[k]));
  double acc[5] = {0, 0, 0, 0, 0};
  for (int it = 0; it < iters; ++it) {
    int nl = 0;
    s = enqueue_iteration(e, e->parity, st, Branch{ts->side, e->ev_fork, e->ev_join}, &nl, ev);
    if (s != CVT_OK) break;
    LAUNCHED(nl);
    e->parity ^= 1;
    for (int k = 0; k < e->max_seg; ++k) if (e->active[k] == 1) e->host_iters[k]++;
    CK(cudaEventSynchronize(ev[5]));
    for (int k = 0; k < 5; ++k) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
      acc[k] += t;
    }
  }
  for (int k = 0; k < 6; ++k) cudaEventDestroy(ev[k]);
  for (int k = 0; k < 5; ++k) ms[k] = (float)(acc[k] / iters);
  return s;
}

// Ping-pong buffer holding a segment's current sites.  A segment stopped by
// its stop rule keeps its sites where its last iteration wrote them, so the
// buffer follows from the parity at placement and the iterations done, read
// from the device.  Synchronous.
static cvt_status_t seg_sites_buffer(cvt_engine* e, int s, cudaStream_t st, int* par) {
  int it = 0;
  CK(cudaMemcpyAsync(&it, reinterpret_cast<char*>(e->d_segs + s) + offsetof(SegDev, iter), sizeof(int),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  e->host_iters[s] = it;
  *par = (e->seg_p0[s] + it) & 1;
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_get_sites(cvt_engine_t e, int s, float* out, int out_on_device, void* stream) {
  if (!e || !out || s < 0 || s >= e->max_seg || !e->seg_mesh[s]) return fail(CVT_ERR_INVALID, "cvt_engine_get_sites: bad arguments");
  cudaStream_t st = S_(stream);
  const SegDev& sd = e->segs[s];
  size_t cnt = 3 * (size_t)sd.n_sites;
  int par = 0;
  cvt_status_t ps = seg_sites_buffer(e, s, st, &par);
  if (ps != CVT_OK) return ps;
  if (!e->f64) {
    const float* src = (const float*)e->d_S[par] + 3 * (size_t)sd.site_base;
    CK(cudaMemcpyAsync(out, src, sizeof(float) * cnt, out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  } else {
    const double* src = (const double*)e->d_S[par] + 3 * (size_t)sd.site_base;
    Scratch sc(st);
    float* tmp = out;
    if (!out_on_device) CK(sc.get(&tmp, cnt));
    k_f64_to_f32<<<cdiv((long)cnt, 256), 256, 0, st>>>(src, tmp, (long)cnt);
    CKLAUNCH();
    if (!out_on_device) CK(cudaMemcpyAsync(out, tmp, sizeof(float) * cnt, cudaMemcpyDeviceToHost, st));
  }
  if (!out_on_device) CK(cudaStreamSynchronize(st));
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_get_sites_f64(cvt_engine_t e, int s, double* out, void* stream) {
  if (!e || !out || s < 0 || s >= e->max_seg || !e->seg_mesh[s] || !e->f64)
    return fail(CVT_ERR_INVALID, "cvt_engine_get_sites_f64: bad arguments (FP64 engines only)");
  cudaStream_t st = S_(stream);
  const SegDev& sd = e->segs[s];
  int par = 0;
  cvt_status_t ps = seg_sites_buffer(e, s, st, &par);
  if (ps != CVT_OK) return ps;
  const double* src = (const double*)e->d_S[par] + 3 * (size_t)sd.site_base;
  CK(cudaMemcpyAsync(out, src, sizeof(double) * 3 * (size_t)sd.n_sites, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_get_state(cvt_engine_t e, int s, uint32_t* knn, int* knnv, uint8_t* frozen,
                                             uint8_t* tier, void* stream) {
  if (!e || s < 0 || s >= e->max_seg || !e->seg_mesh[s]) return fail(CVT_ERR_INVALID, "cvt_engine_get_state: bad segment");
  cudaStream_t st = S_(stream);
  const SegDev& sd = e->segs[s];
  const size_t n = sd.n_sites, b = sd.site_base;
  // the list of the last completed iteration sits in the buffer it wrote
  const uint32_t* kl = e->d_knn;
  if (knn) CK(cudaMemcpyAsync(knn, kl + (size_t)e->K * b, sizeof(uint32_t) * e->K * n, cudaMemcpyDeviceToHost, st));
  if (knnv) CK(cudaMemcpyAsync(knnv, e->d_knnv + 5 * b, sizeof(int) * 5 * n, cudaMemcpyDeviceToHost, st));
  if (frozen) CK(cudaMemcpyAsync(frozen, e->d_frozen + b, n, cudaMemcpyDeviceToHost, st));
  if (tier) CK(cudaMemcpyAsync(tier, e->d_tier + b, n, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_get_stats(cvt_engine_t e, int s, int iter, cvt_iter_stats_t* out, void* stream) {
  if (!e || !out || s < 0 || s >= e->max_seg || !e->seg_mesh[s]) return fail(CVT_ERR_INVALID, "cvt_engine_get_stats: bad segment");
  if (iter < 0 || iter >= e->host_iters[s] || iter < e->host_iters[s] - kStatsRing)
    return fail(CVT_ERR_INVALID, "cvt_engine_get_stats: iteration not held");
  cudaStream_t st = S_(stream);
  int w[kStatsWords];
  CK(cudaMemcpyAsync(w, e->d_stats + ((size_t)s * kStatsRing + (iter % kStatsRing)) * kStatsWords, sizeof(w),
                     cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  out->same = w[0]; out->low = w[1]; out->both = w[2]; out->newly_frozen = w[3];
  float d2;
  std::memcpy(&d2, &w[4], sizeof(float));
  out->max_motion = std::sqrt(d2);
  out->iter = w[5];
  out->knn_reused = w[6];
  out->knn_searched = w[7];
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_segment_iters(cvt_engine_t e, int s, int* iters) {
  if (!e || !iters || s < 0 || s >= e->max_seg || !e->seg_mesh[s]) return fail(CVT_ERR_INVALID, "cvt_engine_segment_iters: bad segment");
  *iters = e->host_iters[s];
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_last_launches(cvt_engine_t e, long long* n) {
  if (!e || !n) return fail(CVT_ERR_INVALID, "cvt_engine_last_launches: null");
  *n = e->last_launches;
  return CVT_OK;
}

// capacity for one mesh + site set
static void engine_caps(const cvt_mesh* m, int n, const cvt_params_t* p, int* cells) {
  GridGeom g = surface_grid(m->lo, m->hi, m->area, n, grid_neighbours(*p), p->cell_factor, 4L * n + 64);
  *cells = g.ncell + 1;
}

extern "C" cvt_status_t cvt_segment_cells(cvt_mesh_t mesh, int n_sites, const cvt_params_t* p, int* cells) {
  if (!mesh || n_sites < 0 || !p || !cells) return fail(CVT_ERR_INVALID, "cvt_segment_cells: bad arguments");
  engine_caps(mesh, n_sites, p, cells);
  return CVT_OK;
}

// Three timed passes over the same fresh copy of the sites: pass r runs
// knn/proj candidate r and clip candidate min(r, 1) (candidate 0 = default).
// The kernels are timed separately by cvt_engine_profile, so one pass
// measures one candidate of each; results do not depend on the shapes.
extern "C" cvt_status_t cvt_autotune(cvt_mesh_t mesh, const float* sites, int n_sites, int iters, cvt_params_t* p,
                                     float* ms_out) {
  if (!mesh || !sites || n_sites < 1 || iters < 2 || !p) return fail(CVT_ERR_INVALID, "cvt_autotune: bad arguments");
  cvt_params_t q = *p;
  if (!resolve_tiles(&q)) return fail(CVT_ERR_UNSUPPORTED, "cvt_autotune: unsupported launch shape in params");
  const int* clip = q.profile == CVT_PROFILE_FP64 ? kClipBlocksD : kClipBlocksF;
  int cells = 0;
  engine_caps(mesh, n_sites, &q, &cells);
  cvt_engine_t e = nullptr;
  cvt_status_t s = cvt_engine_create(&q, 1, n_sites, cells, &e);
  if (s != CVT_OK) return s;
  // pass 0 runs the default shapes; another shape replaces a default only
  // when it is more than 3 % faster (closer calls are within the noise of a
  // few iterations and the default is the one measured over whole runs)
  float best[3] = {1e30f, 1e30f, 1e30f};
  int pick[3] = {q.knn_block, q.clip_block, q.proj_block};
  auto better = [](float t, float cur, bool first) { return first ? true : t < 0.97f * cur; };
  for (int r = 0; r < 3 && s == CVT_OK; ++r) {
    e->p.knn_block = kKnnBlocks[r];
    e->p.clip_block = clip[r < 2 ? r : 1];
    e->p.proj_block = kProjBlocks[r];
    int seg = -1;
    s = cvt_engine_add_segment(e, mesh, sites, n_sites, 0, &seg, nullptr);
    float ms[5], warm[5];
    if (s == CVT_OK) s = cvt_engine_profile(e, 1, warm, nullptr);   // first launches of these shapes
    if (s == CVT_OK) s = cvt_engine_profile(e, iters, ms, nullptr);
    if (s == CVT_OK) s = cvt_engine_remove_segment(e, seg);
    if (s != CVT_OK) break;
    if (better(ms[1], best[0], r == 0)) { best[0] = ms[1]; pick[0] = e->p.knn_block; }
    if (r < 2 && better(ms[2], best[1], r == 0)) { best[1] = ms[2]; pick[1] = e->p.clip_block; }
    if (better(ms[3], best[2], r == 0)) { best[2] = ms[3]; pick[2] = e->p.proj_block; }
  }
  cvt_engine_destroy(e);
  if (s != CVT_OK) return s;
  p->knn_block = pick[0];
  p->clip_block = pick[1];
  p->proj_block = pick[2];
  if (ms_out) for (int k = 0; k < 3; ++k) ms_out[k] = best[k];
  return CVT_OK;
}

extern "C" cvt_status_t cvt_remesh(const float* V, int nV, const int* F, int nF, const float* sites_in, int n_sites,
                                   const cvt_params_t* p, int iters, float* sites_out, int* counts) {
  if (!V || !F || !sites_in || !sites_out || !p || n_sites < 1 || iters < 0)
    return fail(CVT_ERR_INVALID, "cvt_remesh: bad arguments");
  cvt_mesh_t m = nullptr;
  cvt_status_t s = cvt_mesh_create(V, nV, F, nF, &m);
  if (s != CVT_OK) return s;
  int cells = 0;
  engine_caps(m, n_sites, p, &cells);
  cvt_engine_t e = nullptr;
  s = cvt_engine_create(p, 1, n_sites, cells, &e);
  if (s != CVT_OK) { cvt_mesh_destroy(m); return s; }
  int seg = -1;
  s = cvt_engine_add_segment(e, m, sites_in, n_sites, 0, &seg, nullptr);
  if (s == CVT_OK) s = cvt_engine_run(e, iters, nullptr);
  if (s == CVT_OK) s = cvt_engine_get_sites(e, seg, sites_out, 0, nullptr);
  if (s == CVT_OK && counts) {
    // the segment's whole statistics ring in one copy
    std::vector<int> ring((size_t)kStatsRing * kStatsWords);
    cudaError_t ce = cudaMemcpy(ring.data(), e->d_stats + (size_t)seg * kStatsRing * kStatsWords,
                                sizeof(int) * ring.size(), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) s = fail(CVT_ERR_CUDA, std::string("cvt_remesh: ") + cudaGetErrorString(ce));
    const int lo = std::max(0, iters - kStatsRing);
    for (int it = 0; it < iters && s == CVT_OK; ++it)
      for (int a = 0; a < 4; ++a)
        counts[4 * it + a] = it < lo ? -1 : ring[(size_t)(it % kStatsRing) * kStatsWords + a];
  }
  cvt_engine_destroy(e);
  cvt_mesh_destroy(m);
  return s;
}

// Many meshes in one call: every mesh becomes a segment of one engine, so
// each Lloyd iteration of all of them is one pass of the iteration's kernels.
// Host threads that ingest the meshes of one cvt_remesh_batch call.
constexpr int kIngestThreads = 8;

// Every segment's sites into its host array with one read of the segment
// table and one wait at the end (cvt_engine_get_sites waits twice per
// segment).
static cvt_status_t engine_get_sites_all(cvt_engine* e, const int* seg, int n, float* const* out) {
  cudaStream_t st = S_(nullptr);
  std::vector<SegDev> hs(e->max_seg);
  CK(cudaMemcpyAsync(hs.data(), e->d_segs, sizeof(SegDev) * e->max_seg, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int i = 0; i < n; ++i) {
    const int s = seg[i];
    const SegDev& sd = e->segs[s];
    e->host_iters[s] = hs[s].iter;
    const int par = (e->seg_p0[s] + hs[s].iter) & 1;
    const size_t cnt = 3 * (size_t)sd.n_sites;
    if (!e->f64) {
      const float* src = (const float*)e->d_S[par] + 3 * (size_t)sd.site_base;
      CK(cudaMemcpyAsync(out[i], src, sizeof(float) * cnt, cudaMemcpyDeviceToHost, st));
    } else {
      const double* src = (const double*)e->d_S[par] + 3 * (size_t)sd.site_base;
      Scratch sc(st);  // freed in stream order, after the copy
      float* tmp;
      CK(sc.get(&tmp, cnt));
      k_f64_to_f32<<<cdiv((long)cnt, 256), 256, 0, st>>>(src, tmp, (long)cnt);
      CKLAUNCH();
      CK(cudaMemcpyAsync(out[i], tmp, sizeof(float) * cnt, cudaMemcpyDeviceToHost, st));
    }
  }
  CK(cudaStreamSynchronize(st));
  return CVT_OK;
}

extern "C" cvt_status_t cvt_remesh_batch(int n_meshes, const float* const* V, const int* nV, const int* const* F,
                                         const int* nF, const float* const* sites_in, const int* n_sites,
                                         const cvt_params_t* p, int iters, float* const* sites_out) {
  if (n_meshes < 1 || !V || !nV || !F || !nF || !sites_in || !n_sites || !p || !sites_out || iters < 0)
    return fail(CVT_ERR_INVALID, "cvt_remesh_batch: bad arguments");
  for (int i = 0; i < n_meshes; ++i)
    if (!V[i] || !F[i] || !sites_in[i] || !sites_out[i] || n_sites[i] < 1)
      return fail(CVT_ERR_INVALID, "cvt_remesh_batch: bad arguments for mesh " + std::to_string(i));
  std::vector<cvt_mesh_t> meshes(n_meshes, nullptr);
  cvt_status_t s = CVT_OK;
  // Mesh ingest, many meshes at once: each host thread takes meshes off a
  // shared counter and ingests them on its own non-blocking stream (one
  // mesh's ingest is a chain of small kernels and host reads that leaves the
  // GPU idle most of the time; 256 meshes took 83 ms one after another).
  {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(CVT_ERR_CUDA, "cvt_remesh_batch: no device");
    std::vector<cvt_status_t> ms(n_meshes, CVT_OK);
    std::vector<std::string> merr(n_meshes);
    std::atomic<int> next{0};
    auto ingest = [&]() {
      cudaStream_t st = nullptr;
      if (cudaSetDevice(dev) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        for (int i; (i = next++) < n_meshes;) { ms[i] = CVT_ERR_CUDA; merr[i] = "cvt_remesh_batch: stream creation failed"; }
        return;
      }
      for (int i; (i = next++) < n_meshes;) {
        ms[i] = mesh_create_on(V[i], nV[i], F[i], nF[i], &meshes[i], st);
        if (ms[i] != CVT_OK) merr[i] = g_last_error;
      }
      cudaStreamDestroy(st);
    };
    const int nth = std::min(n_meshes, kIngestThreads);
    std::vector<std::thread> pool;
    for (int t = 1; t < nth; ++t) pool.emplace_back(ingest);
    ingest();
    for (std::thread& t : pool) t.join();
    for (int i = 0; i < n_meshes && s == CVT_OK; ++i)
      if (ms[i] != CVT_OK) s = fail(ms[i], merr[i]);
  }
  long total_sites = 0, total_cells = 0;
  for (int i = 0; i < n_meshes && s == CVT_OK; ++i) {
    int cells = 0;
    engine_caps(meshes[i], n_sites[i], p, &cells);
    total_sites += n_sites[i];
    total_cells += cells;
  }
  if (s == CVT_OK && (total_sites > INT_MAX || total_cells > INT_MAX))
    s = fail(CVT_ERR_CAPACITY, "cvt_remesh_batch: more than 2^31 sites or grid cells in one call");
  cvt_engine_t e = nullptr;
  if (s == CVT_OK) s = cvt_engine_create(p, n_meshes, (int)total_sites, (int)total_cells, &e);
  std::vector<int> seg(n_meshes, -1);
  // segments added with their tables uploaded once for all
  for (int i = 0; i < n_meshes && s == CVT_OK; ++i)
    s = add_segment_impl(e, meshes[i], sites_in[i], n_sites[i], 0, &seg[i], S_(nullptr), true);
  if (e) {
    const cvt_status_t u = upload_segment_tables(e, S_(nullptr));
    if (s == CVT_OK) s = u;
  }
  if (s == CVT_OK) s = cvt_engine_run(e, iters, nullptr);
  if (s == CVT_OK) s = engine_get_sites_all(e, seg.data(), n_meshes, sites_out);
  if (e) cvt_engine_destroy(e);
  for (cvt_mesh_t m : meshes)
    if (m) cvt_mesh_destroy(m);
  return s;
}

// ---------------------------------------------------------------------------
// evaluation: dual triangles, quality, Hausdorff (evaluate stage)
// ---------------------------------------------------------------------------
extern "C" cvt_status_t cvt_extract_faces(const float* S, const float* U, const float* V, const uint32_t* knn, int n, int K,
                                          float R2, int* F_out, int max_faces, int* n_faces, void* stream) {
  if (n < 0 || K < 1 || !n_faces || (n > 0 && (!S || !U || !V || !knn)) || (max_faces > 0 && !F_out))
    return fail(CVT_ERR_INVALID, "cvt_extract_faces: bad arguments");
  *n_faces = 0;
  if (n == 0) return CVT_OK;
  cudaStream_t st = S_(stream);
  Scratch sc(st);
  int* cnt;
  CK(sc.get(&cnt, 1));
  int cap = std::max(16 * n, 1024);
  unsigned long long* keys = nullptr;
  int nk = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    Scratch ks(st);
    CK(ks.get(&keys, (size_t)cap));
    CK(cudaMemsetAsync(cnt, 0, sizeof(int), st));
    k_face_keys<<<cdiv(n, 64), 64, 0, st>>>(S, U, V, knn, n, K, R2, 1e-8f, 1e-7f, keys, cnt, cap);
    CKLAUNCH();
    CK(cudaMemcpyAsync(&nk, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (nk <= cap) {
      // sort + unique on the device (the reference sorts on the host, main.cu:952-954)
      unsigned long long *sorted, *uniq;
      int* nu_d;
      CK(sc.get(&sorted, (size_t)std::max(nk, 1)));
      CK(sc.get(&uniq, (size_t)std::max(nk, 1)));
      CK(sc.get(&nu_d, 1));
      size_t tb = 0, tb2 = 0;
      CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys, sorted, nk, 0, 63, st));
      CK(cub::DeviceSelect::Unique(nullptr, tb2, sorted, uniq, nu_d, nk, st));
      void* tmp;
      CK(sc.get((char**)&tmp, std::max(tb, tb2)));
      size_t tbs = std::max(tb, tb2);
      CK(cub::DeviceRadixSort::SortKeys(tmp, tbs, keys, sorted, nk, 0, 63, st));
      tbs = std::max(tb, tb2);
      CK(cub::DeviceSelect::Unique(tmp, tbs, sorted, uniq, nu_d, nk, st));
      LAUNCHED(2);
      int nu = 0;
      CK(cudaMemcpyAsync(&nu, nu_d, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (nu == 0) return CVT_OK;
      int *tri, *keep, *pos, *part;
      CK(sc.get(&tri, 3 * (size_t)nu));
      CK(sc.get(&keep, (size_t)nu));
      CK(sc.get(&pos, (size_t)nu + 1));
      CK(sc.get(&part, (size_t)scan_blocks(nu) + 2));
      k_face_decode<<<cdiv(nu, 256), 256, 0, st>>>(uniq, nu, S, n, 1e-6f, tri, keep);
      CKLAUNCH();
      launch_exclusive_scan(nu, keep, part, pos, st);
      LAUNCHED(3);
      int nf = 0;
      CK(cudaMemcpyAsync(&nf, pos + nu, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      *n_faces = nf;
      if (nf > max_faces) return fail(CVT_ERR_CAPACITY, "cvt_extract_faces: more faces than max_faces (needed count in *n_faces)");
      k_face_compact<<<cdiv(nu, 256), 256, 0, st>>>(tri, keep, pos, nu, F_out);
      CKLAUNCH();
      return CVT_OK;
    }
    cap = nk;  // retry with the exact key count
  }
  return fail(CVT_ERR_CUDA, "cvt_extract_faces: key count changed between passes");
}

extern "C" cvt_status_t cvt_quality(const float* V, const int* F, int nF, float* out, void* stream) {
  if (nF < 0 || !out || (nF > 0 && (!V || !F))) return fail(CVT_ERR_INVALID, "cvt_quality: bad arguments");
  for (int k = 0; k < 6; ++k) out[k] = 0.f;
  if (nF == 0) { out[0] = 1e30f; out[2] = 1e30f; return CVT_OK; }
  cudaStream_t st = S_(stream);
  Scratch sc(st);
  double* acc;
  unsigned* mins;
  CK(sc.get(&acc, 4));
  CK(sc.get(&mins, 2));
  CK(cudaMemsetAsync(acc, 0, 4 * sizeof(double), st));
  CK(cudaMemsetAsync(mins, 0x7f, 2 * sizeof(unsigned), st));
  k_quality<<<cdiv(nF, 256), 256, 0, st>>>(V, F, nF, acc, mins);
  CKLAUNCH();
  double h[4];
  unsigned m[2];
  CK(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(m, mins, sizeof(m), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  float qmin, tmin;
  std::memcpy(&qmin, &m[0], 4);
  std::memcpy(&tmin, &m[1], 4);
  out[0] = qmin;
  out[1] = (float)(h[0] / nF);
  out[2] = tmin;
  out[3] = (float)(h[1] / nF);
  out[4] = (float)(h[2] * 100.0 / (3.0 * nF));
  out[5] = (float)(h[3] * 100.0 / (3.0 * nF));
  return CVT_OK;
}

// frames of the current sites (frozen sites keep their vertex list; the rest
// take their nearest mesh vertex): main.cu:883-897
template <class T>
__global__ void k_eval_frames(const T* __restrict__ S, int base, int n, const uint8_t* __restrict__ frozen,
                              const int* __restrict__ knnv, int mode, MeshDev md, float* __restrict__ Sf,
                              float* __restrict__ U, float* __restrict__ Vv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = base + i;
  V3<T> p = ld3(S, g);
  st3(Sf, i, cvt3<float>(p));
  int nn;
  if (mode != 0 && frozen[g]) {
    nn = knnv[(size_t)g * kKProj];
  } else {
    TopK<T, 1> v1;
    grid_knn<T, float, 1>(md.vg, md.vcell_start, md.vsorted, p, v1, [](uint32_t) { return true; });
    nn = (int)KeyOps<T>::idx(v1.k[0]);
  }
  if (nn < 0) { st3(U, i, V3<float>{1, 0, 0}); st3(Vv, i, V3<float>{0, 1, 0}); return; }
  Frame<float> fr = frame_from_normal(ld3(md.N, nn));
  st3(U, i, fr.u);
  st3(Vv, i, fr.v);
}

static cvt_status_t engine_eval_impl(cvt_engine_t e, int s, cvt_eval_t* out, int* faces_host, int max_faces_host,
                                     int* n_faces_host, void* stream);

extern "C" cvt_status_t cvt_engine_evaluate(cvt_engine_t e, int s, cvt_eval_t* out, void* stream) {
  return engine_eval_impl(e, s, out, nullptr, 0, nullptr, stream);
}

extern "C" cvt_status_t cvt_engine_faces(cvt_engine_t e, int s, int* faces, int max_faces, int* n_faces, cvt_eval_t* out,
                                         void* stream) {
  if (!n_faces || max_faces < 0 || (max_faces > 0 && !faces)) return fail(CVT_ERR_INVALID, "cvt_engine_faces: bad arguments");
  cvt_eval_t tmp;
  return engine_eval_impl(e, s, out ? out : &tmp, faces, max_faces, n_faces, stream);
}

static cvt_status_t engine_eval_impl(cvt_engine_t e, int s, cvt_eval_t* out, int* faces_host, int max_faces_host,
                                     int* n_faces_host, void* stream) {
  if (!e || !out || s < 0 || s >= e->max_seg || !e->seg_mesh[s]) return fail(CVT_ERR_INVALID, "cvt_engine_evaluate: bad segment");
  cudaStream_t st = S_(stream);
  const SegDev& sd = e->segs[s];
  const int n = sd.n_sites;
  const cvt_mesh* m = e->seg_mesh[s];
  int par = 0;
  cvt_status_t ps = seg_sites_buffer(e, s, st, &par);
  if (ps != CVT_OK) return ps;
  Scratch sc(st);
  float *Sf, *U, *V;
  CK(sc.get(&Sf, 3 * (size_t)n));
  CK(sc.get(&U, 3 * (size_t)n));
  CK(sc.get(&V, 3 * (size_t)n));
  if (e->f64)
    k_eval_frames<double><<<cdiv(n, 128), 128, 0, st>>>((const double*)e->d_S[par], sd.site_base, n, e->d_frozen,
                                                         e->d_knnv, sd.mode, m->dev(), Sf, U, V);
  else
    k_eval_frames<float><<<cdiv(n, 128), 128, 0, st>>>((const float*)e->d_S[par], sd.site_base, n, e->d_frozen,
                                                        e->d_knnv, sd.mode, m->dev(), Sf, U, V);
  CKLAUNCH();
  // R2 = longest bbox edge of the current sites (main.cu:899-909)
  int* bb;
  CK(sc.get(&bb, 6));
  k_bbox_init<<<1, 32, 0, st>>>(bb);
  CKLAUNCH();
  k_bbox<<<cdiv(n, 256), 256, 0, st>>>(n, Sf, bb);
  CKLAUNCH();
  int hb[6];
  CK(cudaMemcpyAsync(hb, bb, sizeof(hb), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  float lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    int o = hb[a] >= 0 ? hb[a] : hb[a] ^ 0x7fffffff;
    int q = hb[3 + a] >= 0 ? hb[3 + a] : hb[3 + a] ^ 0x7fffffff;
    std::memcpy(&lo[a], &o, 4);
    std::memcpy(&hi[a], &q, 4);
  }
  float R2 = 2.0f * 0.5f * std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
  const uint32_t* knn = e->d_knn + (size_t)e->K * sd.site_base;
  int max_faces = 4 * n + 64;
  int* Fc;
  CK(sc.get(&Fc, 3 * (size_t)max_faces));
  int nf = 0;
  cvt_status_t r = cvt_extract_faces(Sf, U, V, knn, n, e->K, R2, Fc, max_faces, &nf, stream);
  if (r == CVT_ERR_CAPACITY) {
    max_faces = nf;
    CK(sc.get(&Fc, 3 * (size_t)max_faces));
    r = cvt_extract_faces(Sf, U, V, knn, n, e->K, R2, Fc, max_faces, &nf, stream);
  }
  if (r != CVT_OK) return r;
  float q[6];
  r = cvt_quality(Sf, Fc, nf, q, stream);
  if (r != CVT_OK) return r;
  float dH = 0.f;
  r = cvt_hausdorff_to_mesh(const_cast<cvt_mesh*>(m), Sf, n, Fc, nf, &dH, stream);
  if (r != CVT_OK) return r;
  if (n_faces_host) {
    *n_faces_host = nf;
    if (nf > max_faces_host) return fail(CVT_ERR_CAPACITY, "cvt_engine_faces: more faces than max_faces (count in *n_faces)");
    if (nf > 0) {
      CK(cudaMemcpyAsync(faces_host, Fc, sizeof(int) * 3 * (size_t)nf, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    }
  }
  out->dH = dH;
  out->Qmin = q[0]; out->Qavg = q[1]; out->theta_min = q[2]; out->theta_min_avg = q[3];
  out->theta_lt_30_pct = q[4]; out->theta_gt_90_pct = q[5];
  out->n_faces = nf;
  out->diag = m->diag;
  return CVT_OK;
}

// ---------------------------------------------------------------------------
// allocation-free site KNN (scratch in a fixed device array)
// ---------------------------------------------------------------------------
#include "cvt_noalloc.cu"

// ---------------------------------------------------------------------------
// stop rules, progress polling, device site sampler
// ---------------------------------------------------------------------------
extern "C" cvt_status_t cvt_engine_set_stop(cvt_engine_t e, int s, float max_motion, int max_iters) {
  if (!e || s < 0 || s >= e->max_seg || !e->seg_mesh[s] || max_iters < 0)
    return fail(CVT_ERR_INVALID, "cvt_engine_set_stop: bad arguments");
  const float m2 = max_motion >= 0.f ? max_motion * max_motion : -1.f;
  e->segs[s].stop_motion2 = m2;
  e->segs[s].stop_iters = max_iters;
  char* base = reinterpret_cast<char*>(e->d_segs + s);
  CK(cudaMemcpy(base + offsetof(SegDev, stop_motion2), &m2, sizeof(float), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(base + offsetof(SegDev, stop_iters), &max_iters, sizeof(int), cudaMemcpyHostToDevice));
  return CVT_OK;
}

extern "C" cvt_status_t cvt_engine_poll(cvt_engine_t e, int* iters, int* state, int cap, void* stream) {
  if (!e || cap < 0 || (cap > 0 && (!iters || !state))) return fail(CVT_ERR_INVALID, "cvt_engine_poll: bad arguments");
  cudaStream_t st = S_(stream);
  std::vector<SegDev> sd(e->max_seg);
  std::vector<int> act(e->max_seg);
  CK(cudaMemcpyAsync(sd.data(), e->d_segs, sizeof(SegDev) * e->max_seg, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(act.data(), e->d_active, sizeof(int) * e->max_seg, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int k = 0; k < e->max_seg; ++k) {
    if (!e->seg_mesh[k]) continue;
    e->active[k] = act[k];
    e->host_iters[k] = sd[k].iter;
  }
  for (int k = 0; k < cap && k < e->max_seg; ++k) {
    iters[k] = e->seg_mesh[k] ? e->host_iters[k] : 0;
    state[k] = e->seg_mesh[k] ? e->active[k] : 0;
  }
  return CVT_OK;
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double unit53(unsigned long long h) { return (double)(h >> 11) * 0x1.0p-53; }

// area-uniform points: face by the area CDF, then the square-root
// barycentric map; a counter-based hash of (seed, i) gives the three uniforms
__global__ void k_sample_sites(const double* __restrict__ cdf, int nF, const float* __restrict__ V,
                               const int* __restrict__ F, int n, unsigned long long seed, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long h0 = mix64(seed * 0x100000001b3ull + (unsigned long long)i * 3ull);
  unsigned long long h1 = mix64(h0 + 1ull), h2 = mix64(h0 + 2ull);
  const double total = cdf[nF - 1];
  const double u = unit53(h0) * total;
  int lo = 0, hi = nF - 1;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (cdf[mid] > u) hi = mid; else lo = mid + 1;
  }
  const double r1 = __dsqrt_rn(unit53(h1)), r2 = unit53(h2);
  const int ia = F[3 * lo], ib = F[3 * lo + 1], ic = F[3 * lo + 2];
  for (int a = 0; a < 3; ++a) {
    const double pa = V[3 * ia + a], pb = V[3 * ib + a], pc = V[3 * ic + a];
    out[3 * (size_t)i + a] = (float)((1.0 - r1) * pa + r1 * (1.0 - r2) * pb + r1 * r2 * pc);
  }
}

extern "C" cvt_status_t cvt_mesh_sample_sites(cvt_mesh_t m, int n, unsigned long long seed, float* out, void* stream) {
  if (!m || n < 0 || (n > 0 && !out)) return fail(CVT_ERR_INVALID, "cvt_mesh_sample_sites: bad arguments");
  if (n == 0) return CVT_OK;
  cvt_status_t ls = mesh_ensure_cdf(m);
  if (ls != CVT_OK) return ls;
  k_sample_sites<<<cdiv(n, 256), 256, 0, S_(stream)>>>(m->dcdf, m->nF, m->dV, m->dF, n, seed, out);
  CKLAUNCH();
  return CVT_OK;
}
