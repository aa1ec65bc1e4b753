/*
 * gpu_cvt.h -- C ABI of the B200 tangent-plane CVT remesher (libgpucvt.so).
 *
 * Drop-in for the stage functions of Harper-Yan/GPU_CVT (header-only CUDA
 * kernels driven by main.cu) plus a resident multi-mesh engine.  Plain
 * pointers and sizes only: positions are float[3] records (the reference's
 * float3 AoS), faces int[3], neighbour indices uint32 (the reference's idx_t)
 * unless stated, masks uint8.  `stream` is a cudaStream_t (NULL = legacy
 * default stream).  Stage functions are asynchronous on `stream`; they take
 * caller-owned DEVICE pointers and take their temporaries stream-ordered
 * from the library's memory pool (see cvt_release_cached_memory), freeing
 * them in stream order before return.
 *
 * Every function returns cvt_status_t; CVT_OK is 0.  cvt_last_error() gives
 * the message of the last failure on the calling thread.  (The reference
 * reports nothing and exits the process on CUDA errors, cuda_util.cuh:3-11.)
 *
 * Numerical profiles (cvt_params_t.profile / `profile` arguments):
 *   0 CVT_PROFILE_REF   FP32, the reference kernels' operation order
 *   1 CVT_PROFILE_MIXED FP32 state; FP64 clip predicates/intersections and
 *                       projection barycentrics; compensated centroid sums;
 *                       a NaN centroid keeps the old site
 *   2 CVT_PROFILE_FP64  FP64 state and arithmetic (engine only)
 */
#ifndef GPU_CVT_H_
#define GPU_CVT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CVT_OK = 0,
  CVT_ERR_INVALID = 1,   /* bad argument (sizes, null pointers, unsupported K) */
  CVT_ERR_CUDA = 2,      /* a CUDA runtime call failed */
  CVT_ERR_OOM = 3,       /* device allocation failed */
  CVT_ERR_UNSUPPORTED = 4,
  CVT_ERR_CAPACITY = 5   /* request does not fit the configured capacity */
} cvt_status_t;

enum { CVT_PROFILE_REF = 0, CVT_PROFILE_MIXED = 1, CVT_PROFILE_FP64 = 2 };

const char* cvt_status_string(cvt_status_t s);
const char* cvt_last_error(void);
int cvt_version(void);
/* Number of kernel launches this library has issued in this process. */
unsigned long long cvt_launch_count(void);

/* ======================================================================
 * Stage API -- one function per reference stage, caller-owned device memory
 * ==================================================================== */

/* Replaces run_knn_bitonic_hubs (site_knn.cuh:20-52, C_and_Q
 * bitonic-hubs-grid.cuh:1142): exact kk nearest points of every point (self
 * included), ascending squared distance, ties by lower index.  knn: n*kk
 * uint32, dist: n*kk float (squared distances; may be NULL).  Rows of points
 * with frozen[i] != 0 are left untouched (frozen may be NULL).  Entries
 * beyond the number of points are 0xFFFFFFFF / +inf.  kk in 1..64. */
cvt_status_t cvt_knn_sites(const float* pts, int n, int kk, const uint8_t* frozen,
                           uint32_t* knn, float* dist, void* stream);

/* No counterpart in the reference.  The same answer as cvt_knn_sites, for
 * callers that cannot allocate device memory while they run (a serving
 * process that reserved a fixed HBM budget up front, or a host whose own
 * allocator owns the device heap): the search's temporaries live in one
 * fixed array compiled into the library (about 5 MB, held on every GPU that
 * loads the library until the process exits), so the call allocates and
 * frees nothing.  At most CVT_NOALLOC_MAX_POINTS points (larger n returns
 * CVT_ERR_CAPACITY).  All calls share the array: calls that overlap on the
 * GPU race; keep them ordered on one stream.  The first call on a device
 * looks up the array's address; make it before any stream capture.  The
 * address is kept for the life of the process: after cudaDeviceReset (or
 * anything else that destroys the device's primary context) it is stale, so
 * a program that resets a device must not call this entry point again. */
#define CVT_NOALLOC_MAX_POINTS 131072
cvt_status_t cvt_knn_sites_noalloc(const float* pts, int n, int kk, const uint8_t* frozen,
                                   uint32_t* knn, float* dist, void* stream);

/* Replaces run_knn_bitonic_query_to_mesh (site_knn.cuh:57-77): the kk nearest
 * of the n_cand candidate points for each of n_query query points. */
cvt_status_t cvt_knn_query_to_points(const float* cand, int n_cand, const float* query, int n_query,
                                     int kk, const uint8_t* frozen, uint32_t* knn, float* dist,
                                     void* stream);

/* Replaces knn_vertices_bruteforce_k<KPROJ,EXCLUDE_SELF> (near_project.cuh:54-92):
 * int output (n_query*k), -1 when fewer than k vertices; exclude_self != 0
 * skips vertex index == query index (the reference's mode-0 quirk). */
cvt_status_t cvt_knn_vertices(const float* V, int nV, const float* Q, int nQ, int k,
                              int exclude_self, const uint8_t* frozen, int* out, void* stream);

/* Replaces knn_drop_self_kernel<KIN,KOUT> (site_knn.cuh:79-103). */
cvt_status_t cvt_knn_drop_self(const uint32_t* in, int n, int kin, int kout, uint32_t* out,
                               void* stream);

/* Replaces restore_prev_knn_for_frozen_kernel (main.cu:301-312) and
 * restore_prev_knn_vertices_kernel (near_project.cuh:95-104): rows of frozen
 * entries are copied from prev to cur (k 32-bit words per row). */
cvt_status_t cvt_restore_frozen_rows(const uint8_t* frozen, const uint32_t* prev, uint32_t* cur,
                                     int n, int k, void* stream);

/* Replaces zero_normals + accumulate_face_normals_atomic + normalize_normals
 * (site_normals.cuh:14-41): area-weighted vertex normals, summed per vertex
 * in face order through the vertex->face CSR (deterministic). */
cvt_status_t cvt_vertex_normals(const float* V, int nV, const int* F, int nF, const int* vf_off,
                                const int* vf_faces, float* N, void* stream);

/* Replaces uv_from_nearest_vertex_normal<KPROJ> (site_normals.cuh:69-110):
 * frame of site i from the normal of vertex knnV[i*kproj]. */
cvt_status_t cvt_frames(const float* N0, const int* knnV, int kproj, int n, float* U, float* V,
                        void* stream);
/* Option beside uv_from_nearest_vertex_normal (site_normals.cuh:69-110):
 * frame of site i from the PCA normal of its K listed neighbours (knn: n*K
 * local indices into S) -- the eigenvector of the smallest eigenvalue of
 * their covariance, by a fixed power iteration started from the normal of
 * vertex knnV[i*kproj] and oriented like it; fewer than 3 neighbours keep
 * that vertex normal.  The engine's frame_mode CVT_FRAME_PCA. */
cvt_status_t cvt_frames_pca(const float* S, int n, const uint32_t* knn, int K, const float* N0, const int* knnV,
                            int kproj, float* U, float* V, void* stream);

/* Replaces centroids_tangent_voronoi (2dClip.cuh:82-135): clip [-R,R]^2 by the
 * bisectors of the K listed neighbours (list order), area centroid mapped back
 * to 3-D.  nverts (may be NULL): final polygon vertex count per site. */
cvt_status_t cvt_clip_centroids(const float* S, const float* U, const float* V, const uint32_t* knn,
                                int n, int K, float R, int profile, float* cent, int* nverts,
                                void* stream);

/* Replaces project_centroids_to_mesh<KPROJ> (near_project.cuh:149-189):
 * closest point over the one-rings of the kproj listed vertices.  Sold is
 * read only by the MIXED profile (NaN centroid keeps the old site). */
cvt_status_t cvt_project(const float* cent, const float* V, const int* F, const int* vf_off,
                         const int* vf_faces, const int* knnV, int kproj, int nV, int nF, int nQ,
                         int profile, const float* Sold, float* Snew, void* stream);

/* Replaces freeze_test_kernel_streak (freezetest.cuh:155-212, tier == NULL:
 * thr2_tier[0] / need_tier[0] for every site) and
 * freeze_test_kernel_streak_tiered (freezetest.cuh:270-327) followed by
 * freeze_apply_cand_kernel (freezetest.cuh:451-466).  need_tier[t] = the
 * number of consecutive passing transitions required (the reference's
 * streak[t]-1, at least 1).  thr2_tier/need_tier: 6 entries, host memory.
 * counts (device, 4 ints) accumulates {same, low, both, newly frozen}. */
cvt_status_t cvt_freeze(const float* S, const float* Snew, const uint32_t* knn, const uint32_t* prev_knn,
                        int n, int K, int has_prev, const uint8_t* tier, const float* thr2_tier,
                        const int* need_tier, uint8_t* streak, uint8_t* cand, uint8_t* frozen,
                        int* counts, void* stream);

/* Replaces count_frozen_kernel (freezetest.cuh:50-54): *out_sum += #frozen. */
cvt_status_t cvt_count_frozen(const uint8_t* frozen, int n, int* out_sum, void* stream);

/* Replaces the host tier assignment (main.cu:18-150, called at 640-667):
 * mode 1 = five tiers by normal variation, mode 2 = six tiers with the
 * covariance split.  site_normal: n*3 floats (unit normals). */
cvt_status_t cvt_tiers(int mode, int n, int K, const float* site_normal, const uint32_t* knn,
                       uint8_t* tier, void* stream);

/* Replaces hausdorff_cand_to_ref_gpu (evaluate.cuh:291-383): one-sided
 * Hausdorff distance from the probe set of (Vc,Fc) (vertices, face
 * centroids, edge midpoints) to the surface of `ref_mesh`.  Synchronous;
 * result in *out (host). */
typedef struct cvt_mesh* cvt_mesh_t;
cvt_status_t cvt_hausdorff_to_mesh(cvt_mesh_t ref_mesh, const float* Vc, int nVc, const int* Fc, int nFc,
                                   float* out, void* stream);

/* Replaces the in-repo surface extraction (cell_poly2d_kernel
 * near_project.cuh:246-352, emit_faces_from_labels_kernel buildmesh.cuh:170-201,
 * host sort/unique/decode/degenerate filter main.cu:928-974): dual triangles
 * (i, j1, j2) of the sites' restricted Voronoi cells, sorted by their packed
 * key, unique, degenerate ones (edge or area <= 1e-6) removed.  F_out: device,
 * max_faces*3 ints; *n_faces (host) gets the count (also on CVT_ERR_CAPACITY,
 * then nothing is written).  Synchronous. */
cvt_status_t cvt_extract_faces(const float* S, const float* U, const float* V, const uint32_t* knn, int n, int K,
                               float R2, int* F_out, int max_faces, int* n_faces, void* stream);

/* Replaces eval_quality_angles_cpu (evaluate.cuh:388-462) as a device
 * reduction.  out[6] (host) = Qmin, Qavg, theta_min, theta_min_avg,
 * theta_lt_30_pct, theta_gt_90_pct.  Synchronous. */
cvt_status_t cvt_quality(const float* V, const int* F, int nF, float* out, void* stream);

/* Device memory of meshes, engines and call temporaries comes from one
 * stream-ordered pool per device that keeps freed memory for reuse, so calls
 * after the first allocate nothing from the driver; destroyed engines also
 * leave their instantiated iteration graphs (at most 16) for the next engine
 * of the same shape.  This hands the cached, unused memory back and destroys
 * the kept graphs (e.g. before another library needs the HBM). */
cvt_status_t cvt_release_cached_memory(void);

/* ======================================================================
 * Resident meshes (main.cu:421-542: load, compact, normals, VF CSR, BVH)
 * ==================================================================== */
typedef struct {
  int nV, nF;          /* after dropping unreferenced vertices */
  float R;             /* longest bbox edge of the input vertices */
  float area;
  float bbox_lo[3], bbox_hi[3];
  float diag;          /* bbox diagonal */
  size_t device_bytes; /* HBM held by the mesh (grows when the BVH or the
                          sampler's area table is first built) */
} cvt_mesh_info_t;

/* Host arrays in; the mesh is compacted, uploaded and preprocessed (vertex
 * normals, vertex->face CSR, vertex grid) and stays resident.  The BVH is
 * built on the first Hausdorff distance against the mesh, the area table on
 * the first cvt_mesh_sample_sites; both are then kept (first use is
 * thread-safe). */
cvt_status_t cvt_mesh_create(const float* V, int nV, const int* F, int nF, cvt_mesh_t* out);
/* Cell edge of the vertex grid of meshes created afterwards, in units of the
 * radius expected to hold 6 vertices (default 1.25; a tuning knob only). */
void cvt_set_vertex_cell_factor(float f);
cvt_status_t cvt_mesh_info(cvt_mesh_t m, cvt_mesh_info_t* info);
/* Device views of the compacted mesh (valid until cvt_mesh_destroy). */
cvt_status_t cvt_mesh_device_arrays(cvt_mesh_t m, const float** V, const int** F, const float** N,
                                    const int** vf_off, const int** vf_faces);
cvt_status_t cvt_mesh_destroy(cvt_mesh_t m);
/* The evaluation BVH (built on first use): n_nodes 40-byte nodes {float
 * bmin[3], bmax[3]; int left, right, triStart, triCount} in pre-order and the
 * nF face ids the leaves index (evaluate.cuh:15-22,114-201).  nodes / tri
 * may be NULL (count only); otherwise host buffers of nodes_cap / tri_cap
 * entries.  Synchronous. */
cvt_status_t cvt_mesh_get_bvh(cvt_mesh_t m, void* nodes, int nodes_cap, int* tri, int tri_cap, int* n_nodes);
/* Symmetric Hausdorff distance between two meshes (scripts/evaluate.py:
 * 271-290, hausdorff_bvh): each mesh's probes -- every input vertex (also
 * those no face uses), every face centroid and edge midpoint -- against the
 * other's BVH, FP32 as the GPU evaluator (evaluate.cuh:291-357).  *out =
 * max of the two sides; a_to_b / b_to_a (may be NULL) are the one-sided
 * distances.  Synchronous. */
cvt_status_t cvt_hausdorff_meshes(cvt_mesh_t a, cvt_mesh_t b, float* out, float* a_to_b, float* b_to_a, void* stream);
/* Option beside project_centroids_to_mesh (near_project.cuh:149-189): the
 * exact closest point on the whole mesh to each of the n centroids (device
 * arrays, n*3 floats), through the mesh's BVH (built on first use): the
 * face with the smallest squared distance, first met in the BVH's near-first
 * order on ties.  Sold (the sites before the step; may be NULL except in
 * MIXED) bounds the search; in MIXED a non-finite centroid keeps its old
 * site.  profile REF or MIXED (FP64 barycentrics).  The engine's proj_mode
 * CVT_PROJ_BVH.  Synchronous (checks the traversal stack). */
cvt_status_t cvt_project_bvh(cvt_mesh_t m, const float* cent, int n, int profile, const float* Sold, float* Snew,
                             void* stream);
/* n area-uniform points on the mesh (device out, n*3 floats): a face drawn by
 * area, then the square-root barycentric map, three uniforms per point from
 * a counter hash of (seed, i).  New (the reference starts from the vertices,
 * main.cu:493). */
cvt_status_t cvt_mesh_sample_sites(cvt_mesh_t m, int n, unsigned long long seed, float* out, void* stream);

/* ======================================================================
 * Engine: many (mesh, site set) segments iterated together; each Lloyd
 * iteration is one pass of fused kernels over all active segments, captured
 * in a CUDA graph.  Follows main.cu:669-881 per segment.
 * ==================================================================== */
typedef struct {
  int k;              /* neighbours per site after dropping self: 8,12,16,20,24,32 */
  int mode;           /* 0 freezing off, 1 five tiers, 2 six tiers */
  int profile;        /* CVT_PROFILE_* */
  int kproj;          /* nearest vertices for the projection (5) */
  int ex_quirk;       /* mode 0: centroid->vertex KNN skips vertex index == site index */
  float cell_factor;  /* site-grid cell edge / expected (K+1)-th neighbour radius */
  int use_graph;      /* capture iterations in a CUDA graph */
  /* launch shapes (threads per block); results do not depend on them:
   * knn_block 64|128|256 (one warp per site), clip_block 64|128 (FP64
   * profile: 32|64), proj_block 64|128|256; 0 = default. */
  int knn_block, clip_block, proj_block;
  /* options beyond the reference (defaults reproduce it):
   * proj_mode  CVT_PROJ_ONERING (0): the closest point over the one-rings of
   *            the kproj nearest vertices (near_project.cuh:149-189);
   *            CVT_PROJ_BVH (1): the exact closest point on the whole mesh
   *            through its BVH (built when the first segment is placed).
   *            Frozen sites then keep the frame vertex of the last iteration
   *            they were active (no vertex list is kept).
   * frame_mode CVT_FRAME_VERTEX_NORMAL (0): the frame from the normal of the
   *            site's nearest vertex (site_normals.cuh:69-110);
   *            CVT_FRAME_PCA (1): from the PCA normal of the site's K
   *            neighbours (the smallest-eigenvalue eigenvector of their
   *            covariance, oriented like the vertex normal). */
  int proj_mode, frame_mode;
  /* knn_reuse 1 (default): each site also keeps the K+16 nearest sites of
   * its last full KNN search, and while the sites' accumulated motion proves
   * that no other site can have come closer than its K-th neighbour, the
   * K-list is taken from those candidates (same lists as a full search);
   * 0: a full search every iteration. */
  int knn_reuse;
} cvt_params_t;
#define CVT_PROJ_ONERING 0
#define CVT_PROJ_BVH 1
#define CVT_FRAME_VERTEX_NORMAL 0
#define CVT_FRAME_PCA 1

void cvt_params_default(cvt_params_t* p);
/* Launch-shape autotuner: times every candidate block size of the site KNN,
 * clip and projection kernels over `iters` Lloyd iterations (iters >= 2) of
 * the given sites on the mesh, in a scratch engine, and writes the fastest
 * into p->knn_block / clip_block / proj_block (the other fields are used as
 * given); a shape replaces the default only when it is > 3 % faster.  ms (may be NULL) receives the per-iteration ms of the chosen
 * shapes {knn, clip, proj}.  Synchronous; allocates a scratch engine. */
cvt_status_t cvt_autotune(cvt_mesh_t mesh, const float* sites, int n_sites, int iters, cvt_params_t* p, float* ms);

typedef struct cvt_engine* cvt_engine_t;

/* Per-segment statistics of one iteration (freezetest.cuh counts +
 * motion).  max_motion is the largest site displacement (not squared).
 * knn_reused / knn_searched: site KNN lists taken from the kept candidate
 * lists / found by a full search (knn_reuse). */
typedef struct {
  int same, low, both, newly_frozen;
  float max_motion;
  int iter;
  int knn_reused, knn_searched;
} cvt_iter_stats_t;

/* Grid cells a segment of n_sites sites on `mesh` reserves with params p
 * (its cell_factor and k); sum them over the segments for max_cells. */
cvt_status_t cvt_segment_cells(cvt_mesh_t mesh, int n_sites, const cvt_params_t* p, int* cells);
/* Capacity-based engine: up to max_segments segments holding up to
 * max_sites sites and max_cells grid cells in total. */
cvt_status_t cvt_engine_create(const cvt_params_t* p, int max_segments, int max_sites, int max_cells,
                               cvt_engine_t* out);
cvt_status_t cvt_engine_destroy(cvt_engine_t e);
/* Place a segment: `sites` (n*3 floats, host or device per sites_on_device)
 * on `mesh`.  Returns the segment id.  The segment starts at iteration 0. */
cvt_status_t cvt_engine_add_segment(cvt_engine_t e, cvt_mesh_t mesh, const float* sites, int n,
                                    int sites_on_device, int* seg_id, void* stream);
/* Free a segment's slot (its sites stop being iterated at once). */
cvt_status_t cvt_engine_remove_segment(cvt_engine_t e, int seg_id);
/* Run `iters` Lloyd iterations of every active segment (asynchronous).  With
 * use_graph, each iteration replays one of two CUDA graphs (one per buffer
 * parity); an iteration whose graph does not exist yet is launched directly,
 * and its graph is captured while the GPU runs it.  Each iteration forks a
 * second stream owned by the calling host thread.  One engine must not run
 * from two threads at once. */
cvt_status_t cvt_engine_run(cvt_engine_t e, int iters, void* stream);
/* Copy a segment's current sites out (n*3 floats; FP64 engines convert).
 * Synchronous (it reads the segment's iteration count from the device). */
cvt_status_t cvt_engine_get_sites(cvt_engine_t e, int seg_id, float* out, int out_on_device, void* stream);
/* FP64 engines: the double-precision sites (n*3 doubles, host). */
cvt_status_t cvt_engine_get_sites_f64(cvt_engine_t e, int seg_id, double* out, void* stream);
/* Host copies of per-site state: knn (n*k uint32, local indices), knnv
 * (n*kproj int), frozen / tier (n uint8).  Any pointer may be NULL.  Sync. */
cvt_status_t cvt_engine_get_state(cvt_engine_t e, int seg_id, uint32_t* knn, int* knnv, uint8_t* frozen,
                                  uint8_t* tier, void* stream);
/* Statistics of the segment's iteration `iter` (must be one of the last
 * 256 it ran).  Sync. */
cvt_status_t cvt_engine_get_stats(cvt_engine_t e, int seg_id, int iter, cvt_iter_stats_t* out, void* stream);
/* Iterations the segment has completed (host-side count). */
cvt_status_t cvt_engine_segment_iters(cvt_engine_t e, int seg_id, int* iters);
/* Run `iters` iterations without a graph, timing each kernel group with CUDA
 * events on `stream`; ms[5] = average ms per iteration of {grid build, site
 * KNN kernel, clip kernel (+ overflow fallback), projection kernel (+ far
 * fallback and the iteration's bookkeeping, which runs in its last block),
 * 0 (kept for layout)}.  Synchronous. */
cvt_status_t cvt_engine_profile(cvt_engine_t e, int iters, float* ms, void* stream);
/* The evaluation of main.cu:883-1040 for one segment: frames of the current
 * sites, dual triangles with the last iteration's neighbour lists, quality,
 * and the one-sided Hausdorff distance to the segment's mesh.  Synchronous. */
typedef struct {
  float dH;
  float Qmin, Qavg, theta_min, theta_min_avg, theta_lt_30_pct, theta_gt_90_pct;
  int n_faces;
  float diag;  /* bbox diagonal of the segment's mesh */
} cvt_eval_t;
cvt_status_t cvt_engine_evaluate(cvt_engine_t e, int seg_id, cvt_eval_t* out, void* stream);
/* The same evaluation, also copying the dual triangles (host, max_faces*3
 * ints; *n_faces gets the count, also on CVT_ERR_CAPACITY) -- the mesh that
 * main.cu:982 writes as iter_%03d.obj.  `out` may be NULL. */
cvt_status_t cvt_engine_faces(cvt_engine_t e, int seg_id, int* faces, int max_faces, int* n_faces, cvt_eval_t* out,
                              void* stream);
/* Stop rule of a segment, applied on the device after every iteration: the
 * segment stops iterating once an iteration moves no site by more than
 * max_motion (absolute; < 0: no motion rule) or after max_iters iterations
 * (0: no cap).  The serving loop's "until max site motion < 1e-4 of the bbox
 * diagonal, capped at 150 iterations". */
cvt_status_t cvt_engine_set_stop(cvt_engine_t e, int seg_id, float max_motion, int max_iters);
/* Progress of the first `cap` segment slots, read from the device
 * (synchronous): iters[s] = iterations done, state[s] = 0 free, 1 iterating,
 * 2 stopped by its stop rule. */
cvt_status_t cvt_engine_poll(cvt_engine_t e, int* iters, int* state, int cap, void* stream);
/* Kernel launches issued by the last cvt_engine_run (graph nodes included). */
cvt_status_t cvt_engine_last_launches(cvt_engine_t e, long long* n);

/* One-call remesh with HOST buffers (the main.cu driver without I/O):
 * upload, `iters` Lloyd iterations, download.  counts (iters*4 ints, may be
 * NULL) receives {same, low, both, newly frozen} per iteration. */
cvt_status_t cvt_remesh(const float* V, int nV, const int* F, int nF, const float* sites_in, int n_sites,
                        const cvt_params_t* p, int iters, float* sites_out, int* counts);
/* Many meshes in one call, HOST buffers (the main.cu driver run once per
 * mesh, main.cu:369-1073, replaced by one batched run): mesh i is V[i]
 * (nV[i]*3 floats), F[i] (nF[i]*3 ints) with sites_in[i] (n_sites[i]*3
 * floats); every mesh is a segment of one engine, so each Lloyd iteration
 * of all meshes is one pass of the iteration's kernels.  sites_out[i]
 * receives mesh i's sites after `iters` iterations -- the same values
 * cvt_remesh returns for that mesh alone.  The meshes are ingested by up to
 * 8 host threads, each on its own non-blocking stream (the call creates and
 * joins them); a mesh that fails ingest fails the call with its error.
 * Synchronous. */
cvt_status_t cvt_remesh_batch(int n_meshes, const float* const* V, const int* nV, const int* const* F, const int* nF,
                              const float* const* sites_in, const int* n_sites, const cvt_params_t* p, int iters,
                              float* const* sites_out);

#ifdef __cplusplus
}
#endif
#endif /* GPU_CVT_H_ */
