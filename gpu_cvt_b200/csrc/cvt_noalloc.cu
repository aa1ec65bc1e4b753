// cvt_knn_sites_noalloc: the site KNN of cvt_knn_sites without any device
// allocation.  (Included at the end of cvt_capi.cu, whose kernels it reuses,
// so the scratch array, its address look-up and the launches share one
// translation unit.)
//
// Why it exists: some callers cannot allocate device memory at call time --
// a serving process that admitted its work against a fixed HBM budget and
// reserved that memory up front, or a host application whose own allocator
// owns the device heap -- and for them a library call that may grow the heap
// (or fail with out-of-memory halfway through) is not acceptable.  This
// variant keeps every temporary of the search (bounding box, grid geometry,
// cell counts and starts, scan partials, per-point cell ranks, the
// cell-ordered point copy) in one fixed array compiled into the library.
//
// Limits and rules:
//   * at most CVT_NOALLOC_MAX_POINTS points per call (larger calls return
//     CVT_ERR_CAPACITY and do nothing);
//   * the array (~5 MB) is held by every GPU that loads the library, until
//     the process exits;
//   * all calls share that one array: calls whose work overlaps on the GPU
//     (different streams, or different host threads without ordering) race
//     and corrupt each other's results -- order them on one stream;
//   * the first call on a device looks the array's device address up
//     (cudaGetSymbolAddress); make that first call before any stream capture;
//   * the address is cached per device ordinal for the life of the process:
//     cudaDeviceReset (or any other teardown of the device's primary
//     context) leaves it stale, so a program that resets a device must not
//     call this entry point afterwards.

#include <mutex>

namespace noalloc {

constexpr int kMaxPoints = CVT_NOALLOC_MAX_POINTS;
constexpr int kCap = 2 * kMaxPoints;  // spatial cells: the allocating path's max(64, 2n)
constexpr size_t up256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kScanParts = (size_t)(kCap + 1 + kScanTile - 1) / kScanTile + 2;
constexpr size_t kOffBbox = 0;
constexpr size_t kOffGeom = up256(kOffBbox + 6 * sizeof(int));
constexpr size_t kOffCount = up256(kOffGeom + sizeof(GridGeom));
constexpr size_t kOffStart = up256(kOffCount + (size_t)(kCap + 1) * sizeof(int));
constexpr size_t kOffPart = up256(kOffStart + (size_t)(kCap + 2) * sizeof(int));
constexpr size_t kOffRank = up256(kOffPart + kScanParts * sizeof(int));
constexpr size_t kOffSorted = up256(kOffRank + (size_t)kMaxPoints * sizeof(int2));
constexpr size_t kBytes = up256(kOffSorted + (size_t)kMaxPoints * sizeof(Pt4<float>));

}  // namespace noalloc

// In host code this name is only a stand-in for the device array, never a
// device address: kernels are given the address looked up below.
static __device__ __align__(256) unsigned char g_knn_scratch[noalloc::kBytes];

static std::mutex g_knn_scratch_mu;
static void* g_knn_scratch_addr[256];  // per device ordinal

// device address of the scratch array on the current device (looked up once
// per device, with that device current)
static cvt_status_t knn_scratch_address(void** out) {
  int dev = -1;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) return fail(CVT_ERR_UNSUPPORTED, "cvt_knn_sites_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_knn_scratch_mu);
  if (!g_knn_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_knn_scratch);
    if (e != cudaSuccess || !p)
      return fail(CVT_ERR_CUDA, std::string("cvt_knn_sites_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_knn_scratch_addr[dev] = p;
  }
  *out = g_knn_scratch_addr[dev];
  return CVT_OK;
}

extern "C" cvt_status_t cvt_knn_sites_noalloc(const float* pts, int n, int kk, const uint8_t* frozen, uint32_t* knn,
                                              float* dist, void* stream) {
  if (n < 0 || kk < 1 || kk > 64 || (n > 0 && (!pts || !knn)))
    return fail(CVT_ERR_INVALID, "cvt_knn_sites_noalloc: bad arguments");
  if (n > noalloc::kMaxPoints)
    return fail(CVT_ERR_CAPACITY, "cvt_knn_sites_noalloc: more than CVT_NOALLOC_MAX_POINTS (" +
                                      std::to_string(noalloc::kMaxPoints) + ") points; use cvt_knn_sites");
  if (n == 0) return CVT_OK;
  void* base = nullptr;
  cvt_status_t s = knn_scratch_address(&base);
  if (s != CVT_OK) return s;
  cudaStream_t st = S_(stream);
  unsigned char* b = static_cast<unsigned char*>(base);
  int* bb = reinterpret_cast<int*>(b + noalloc::kOffBbox);
  PointGrid pg;
  pg.geom = reinterpret_cast<GridGeom*>(b + noalloc::kOffGeom);
  pg.cell_count = reinterpret_cast<int*>(b + noalloc::kOffCount);
  pg.cell_start = reinterpret_cast<int*>(b + noalloc::kOffStart);
  pg.part = reinterpret_cast<int*>(b + noalloc::kOffPart);
  pg.cellrank = reinterpret_cast<int2*>(b + noalloc::kOffRank);
  pg.sorted = reinterpret_cast<Pt4<float>*>(b + noalloc::kOffSorted);
  const int cap = std::max(64, 2 * n);
  pg.total_cells = cap + 1;
  // the array keeps the previous call's contents: the bounding box and the
  // cell counts must start from their initial values
  k_bbox_init<<<1, 32, 0, st>>>(bb);
  CKLAUNCH();
  k_bbox<<<cdiv(n, 256), 256, 0, st>>>(n, pts, bb);
  CKLAUNCH();
  k_grid_geom<<<1, 32, 0, st>>>(bb, n, 0.2f * kk, cap, pg.geom);
  CKLAUNCH();
  CK(cudaMemsetAsync(pg.cell_count, 0, sizeof(int) * pg.total_cells, st));
  k_grid_count<float><<<cdiv(n, 256), 256, 0, st>>>(n, pts, SegGrid{pg.geom, nullptr, nullptr}, pg.cell_count, pg.cellrank);
  CKLAUNCH();
  launch_exclusive_scan(pg.total_cells, pg.cell_count, pg.part, pg.cell_start, st);
  LAUNCHED(3);
  CK(cudaGetLastError());
  k_grid_scatter<float><<<cdiv(n, 256), 256, 0, st>>>(n, pts, pg.cellrank, pg.cell_start, pg.sorted);
  CKLAUNCH();
  KK_DISPATCH(kk, launch_knn_points, pg, n, frozen, kk, knn, dist, st);
  CKLAUNCH();
  return CVT_OK;
}
