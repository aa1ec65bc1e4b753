// Reference-kernel harness (TEST INFRASTRUCTURE ONLY).
//
// Drives the reference's own CUDA stage kernels -- the unmodified
// Harper-Yan/GPU_CVT headers, included from the reference checkout at build
// time (oracle/Makefile `ref` target) -- through the Lloyd loop of
// main.cu:640-974 with three generalisations the reference's driver lacks:
//   * sites are an input array (nSites != nV; main.cu:493 copies the vertices),
//   * K (neighbours after dropping self) is 20, 24 or 32 (main.cu:398 fixes 32),
//   * the candidate mesh for the final Hausdorff figure comes from the in-repo
//     face extraction (main.cu:928-974) instead of the Geogram subprocess.
// For modes 1/2 the tier pass uses, as the site normal, the normal of the
// site's nearest mesh vertex (main.cu:650-664 reads hN[i], i.e. vertex i,
// which is the same thing when the sites are the vertices).
// The untimed duplicate KNN work of main.cu:883-909 does not change the
// state and is skipped.
//
// knn_mode 0 uses the reference's hub KNN (run_knn_bitonic_hubs /
// run_knn_bitonic_query_to_mesh).  knn_mode 1 replaces it by an exact
// brute-force search (harness kernel below for site->site; the reference's
// knn_vertices_bruteforce_k for site/centroid->vertex in modes 1/2), keeping
// every other stage kernel of the reference: built for sm_100a with nvcc
// 12.9 the hub KNN returns corrupted neighbour ids on B200 (most rows zero),
// which makes knn_mode 0 unusable as a parity reference there.
//
// Usage: ref_harness <in.bin> <out.bin>
//   in : int32 nV, nF, nS, K, mode, iters, knn_mode, ndump, dump_iters[ndump];
//        float32 V[nV*3]; int32 F[nF*3]; float32 S[nS*3]
//   out: int32 iters, ndump; float32 S_dump[ndump][nS*3]; int32 counts[iters*4];
//        uint32 knn_it0[nS*K]; int32 knnv_it0[nS*5]; float32 cent_it0[nS*3];
//        uint8 frozen[nS]; uint8 tier[nS]; float32 stage_ms[iters*6];
//        float32 quality[6]; float32 dH; int32 nFaces; float32 wall_ms
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include "site_normals.cuh"
#include "site_knn.cuh"
#include "2dClip.cuh"
#include "near_project.cuh"
#include "freezetest.cuh"
#include "buildmesh.cuh"
#include "evaluate.cuh"

namespace harness {

constexpr int KPROJ = 5;
constexpr int MAX_POLY = 256;

// exact kk nearest sites (self included), ascending (distance, index);
// frozen rows untouched (the contract of bitonic-hubs-grid.cuh:862-995)
template <int KK>
__global__ void bf_knn_sites(const float3* __restrict__ P, int n, const unsigned char* __restrict__ frozen,
                             idx_t* __restrict__ knn, float* __restrict__ dist) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || frozen[i]) return;
  float bd[KK];
  idx_t bi[KK];
  for (int t = 0; t < KK; ++t) { bd[t] = 3.0e38f; bi[t] = 0xffffffffu; }
  float3 q = P[i];
  for (int j = 0; j < n; ++j) {
    float3 p = P[j];
    float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
    float d = dx * dx + dy * dy + dz * dz;
    if (d > bd[KK - 1] || (d == bd[KK - 1] && (idx_t)j > bi[KK - 1])) continue;
    int pos = KK - 1;
    bd[pos] = d; bi[pos] = (idx_t)j;
    while (pos > 0 && (bd[pos] < bd[pos - 1] || (bd[pos] == bd[pos - 1] && bi[pos] < bi[pos - 1]))) {
      float td = bd[pos - 1]; bd[pos - 1] = bd[pos]; bd[pos] = td;
      idx_t ti = bi[pos - 1]; bi[pos - 1] = bi[pos]; bi[pos] = ti;
      --pos;
    }
  }
  for (int t = 0; t < KK; ++t) { knn[(size_t)i * KK + t] = bi[t]; dist[(size_t)i * KK + t] = bd[t]; }
}

template <int K>
__global__ void restore_rows(const unsigned char* frozen, const idx_t* prev, idx_t* cur, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !frozen[i]) return;
  for (int a = 0; a < K; ++a) cur[(size_t)i * K + a] = prev[(size_t)i * K + a];
}

// host tier rules (main.cu:18-150), restated
static void tiers(int mode, int n, int K, const std::vector<float>& sn, const std::vector<idx_t>& knn,
                  std::vector<unsigned char>& tier) {
  static const double TH[4] = {0.15, 0.35, 0.55, 0.80};
  tier.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    double sum = 0.0;
    int cnt = 0;
    for (int j = 0; j < K; ++j) {
      int jj = (int)knn[(size_t)i * K + j];
      if (jj < 0 || jj >= n) continue;
      double c = (double)sn[3 * i] * sn[3 * jj] + (double)sn[3 * i + 1] * sn[3 * jj + 1] +
                 (double)sn[3 * i + 2] * sn[3 * jj + 2];
      c = std::min(1.0, std::max(-1.0, c));
      sum += c;
      cnt++;
    }
    double nv = cnt > 0 ? 1.0 - sum / cnt : 0.0;
    double L = 0.0;
    if (mode == 2) {
      double mean[3] = {0, 0, 0};
      int c2 = 0;
      for (int j = 0; j < K; ++j) {
        int jj = (int)knn[(size_t)i * K + j];
        if (jj < 0 || jj >= n) continue;
        for (int a = 0; a < 3; ++a) mean[a] += sn[3 * jj + a];
        c2++;
      }
      if (c2 >= 2) {
        for (int a = 0; a < 3; ++a) mean[a] /= c2;
        double C[9] = {0};
        for (int j = 0; j < K; ++j) {
          int jj = (int)knn[(size_t)i * K + j];
          if (jj < 0 || jj >= n) continue;
          double d[3] = {sn[3 * jj] - mean[0], sn[3 * jj + 1] - mean[1], sn[3 * jj + 2] - mean[2]};
          for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) C[3 * r + c] += d[r] * d[c];
        }
        // power iteration for the two largest eigenvalues
        double v[3] = {1, 0, 0}, lam[3];
        for (int it = 0; it < 20; ++it) {
          double w[3] = {C[0] * v[0] + C[1] * v[1] + C[2] * v[2], C[3] * v[0] + C[4] * v[1] + C[5] * v[2],
                         C[6] * v[0] + C[7] * v[1] + C[8] * v[2]};
          double nn = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
          if (nn < 1e-30) break;
          for (int a = 0; a < 3; ++a) v[a] = w[a] / nn;
        }
        lam[0] = v[0] * (C[0] * v[0] + C[1] * v[1] + C[2] * v[2]) + v[1] * (C[3] * v[0] + C[4] * v[1] + C[5] * v[2]) +
                 v[2] * (C[6] * v[0] + C[7] * v[1] + C[8] * v[2]);
        double C2[9];
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) C2[3 * r + c] = C[3 * r + c] - lam[0] * v[r] * v[c];
        double v2[3] = {0, 1, 0};
        for (int it = 0; it < 20; ++it) {
          double w[3] = {C2[0] * v2[0] + C2[1] * v2[1] + C2[2] * v2[2], C2[3] * v2[0] + C2[4] * v2[1] + C2[5] * v2[2],
                         C2[6] * v2[0] + C2[7] * v2[1] + C2[8] * v2[2]};
          double nn = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
          if (nn < 1e-30) break;
          for (int a = 0; a < 3; ++a) v2[a] = w[a] / nn;
        }
        lam[1] = v2[0] * (C2[0] * v2[0] + C2[1] * v2[1] + C2[2] * v2[2]) +
                 v2[1] * (C2[3] * v2[0] + C2[4] * v2[1] + C2[5] * v2[2]) +
                 v2[2] * (C2[6] * v2[0] + C2[7] * v2[1] + C2[8] * v2[2]);
        lam[2] = C[0] + C[4] + C[8] - lam[0] - lam[1];
        std::sort(lam, lam + 3);
        if (lam[2] > 1e-30) L = (lam[2] - lam[1]) / lam[2];
      }
    }
    int t = 0;
    while (t < 4 && nv >= TH[t]) t++;
    if (mode == 2 && t == 4 && L > 0.80) t = 5;
    tier[i] = (unsigned char)t;
  }
}

struct In {
  int nV, nF, nS, K, mode, iters, knn_mode;
  std::vector<int> dump;
  std::vector<float> V, S;
  std::vector<int> F;
};

template <int K_NEIGH>
int run(const In& in, FILE* fo) {
  constexpr int K_SITE = K_NEIGH + 1;
  const int nV = in.nV, nF = in.nF, nS = in.nS, mode = in.mode, iters = in.iters;
  auto wall0 = std::chrono::steady_clock::now();
  // R over the input vertices (main.cu:169-227)
  float3 bmin = make_float3(1e30f, 1e30f, 1e30f), bmax = make_float3(-1e30f, -1e30f, -1e30f);
  std::vector<float3> hV(nV);
  std::vector<int3i> hF(nF);
  for (int i = 0; i < nV; ++i) {
    hV[i] = make_float3(in.V[3 * i], in.V[3 * i + 1], in.V[3 * i + 2]);
    bmin.x = fminf(bmin.x, hV[i].x); bmin.y = fminf(bmin.y, hV[i].y); bmin.z = fminf(bmin.z, hV[i].z);
    bmax.x = fmaxf(bmax.x, hV[i].x); bmax.y = fmaxf(bmax.y, hV[i].y); bmax.z = fmaxf(bmax.z, hV[i].z);
  }
  for (int f = 0; f < nF; ++f) hF[f] = {in.F[3 * f], in.F[3 * f + 1], in.F[3 * f + 2]};
  float R = fmaxf(bmax.x - bmin.x, fmaxf(bmax.y - bmin.y, bmax.z - bmin.z));
  float freeze_disp = 0.01f * R * 0.01f * R;

  float3 *dV, *dN, *dS, *dSnew, *du, *dv, *dCent;
  int3i* dF;
  cudaMalloc(&dV, nV * sizeof(float3));
  cudaMalloc(&dN, nV * sizeof(float3));
  cudaMalloc(&dF, nF * sizeof(int3i));
  cudaMemcpy(dV, hV.data(), nV * sizeof(float3), cudaMemcpyHostToDevice);
  cudaMemcpy(dF, hF.data(), nF * sizeof(int3i), cudaMemcpyHostToDevice);
  const int T = 1024;
  zero_normals<<<(nV + T - 1) / T, T>>>(dN, nV);
  accumulate_face_normals_atomic<<<(nF + T - 1) / T, T>>>(dV, dF, dN, nF);
  normalize_normals<<<(nV + T - 1) / T, T>>>(dN, nV);

  cudaMalloc(&dS, nS * sizeof(float3));
  cudaMalloc(&dSnew, nS * sizeof(float3));
  cudaMalloc(&du, nS * sizeof(float3));
  cudaMalloc(&dv, nS * sizeof(float3));
  cudaMalloc(&dCent, nS * sizeof(float3));
  cudaMemcpy(dS, in.S.data(), nS * sizeof(float3), cudaMemcpyHostToDevice);
  idx_t *dRaw, *dKNN, *dPrev;
  float *dDist, *dKnnVdist;
  cudaMalloc(&dRaw, (size_t)nS * K_SITE * sizeof(idx_t));
  cudaMalloc(&dDist, (size_t)nS * K_SITE * sizeof(float));
  cudaMalloc(&dKNN, (size_t)nS * K_NEIGH * sizeof(idx_t));
  cudaMalloc(&dPrev, (size_t)nS * K_NEIGH * sizeof(idx_t));
  cudaMemset(dPrev, 0, (size_t)nS * K_NEIGH * sizeof(idx_t));
  int *dKnnV, *dPrevKnnV;
  cudaMalloc(&dKnnV, (size_t)nS * KPROJ * sizeof(int));
  cudaMalloc(&dPrevKnnV, (size_t)nS * KPROJ * sizeof(int));
  cudaMalloc(&dKnnVdist, (size_t)nS * KPROJ * sizeof(float));
  unsigned char *dFrozen, *dCand, *dStreak, *dTier = nullptr;
  cudaMalloc(&dFrozen, nS);
  cudaMalloc(&dCand, nS);
  cudaMalloc(&dStreak, nS);
  cudaMemset(dFrozen, 0, nS);
  cudaMemset(dCand, 0, nS);
  cudaMemset(dStreak, 0, nS);
  float* dThr;
  int* dStreakTier;
  int* dCounts;
  cudaMalloc(&dThr, 6 * sizeof(float));
  cudaMalloc(&dStreakTier, 6 * sizeof(int));
  cudaMalloc(&dCounts, 4 * sizeof(int));
  // vertex -> face CSR (main.cu:259-285)
  std::vector<int> off(nV + 1, 0), fcs(3 * (size_t)nF);
  for (int f = 0; f < nF; ++f) { off[hF[f].x + 1]++; off[hF[f].y + 1]++; off[hF[f].z + 1]++; }
  for (int v = 0; v < nV; ++v) off[v + 1] += off[v];
  {
    std::vector<int> cur(off);
    for (int f = 0; f < nF; ++f) { fcs[cur[hF[f].x]++] = f; fcs[cur[hF[f].y]++] = f; fcs[cur[hF[f].z]++] = f; }
  }
  int *dOff, *dFcs;
  cudaMalloc(&dOff, (nV + 1) * sizeof(int));
  cudaMalloc(&dFcs, fcs.size() * sizeof(int));
  cudaMemcpy(dOff, off.data(), (nV + 1) * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(dFcs, fcs.data(), fcs.size() * sizeof(int), cudaMemcpyHostToDevice);

  dim3 blk(256), grd((nS + 255) / 256);
  cudaEvent_t k0, k1;
  cudaEventCreate(&k0);
  cudaEventCreate(&k1);
  auto site_knn = [&](const float3* pts) -> float {
    if (in.knn_mode == 0) return run_knn_bitonic_hubs(nS, K_SITE, dFrozen, pts, dRaw, dDist);
    cudaEventRecord(k0);
    bf_knn_sites<K_SITE><<<grd, blk>>>(pts, nS, dFrozen, dRaw, dDist);
    cudaEventRecord(k1);
    cudaEventSynchronize(k1);
    float t = 0;
    cudaEventElapsedTime(&t, k0, k1);
    return t;
  };
  // site/centroid -> 5 nearest vertices for modes 1/2 (frozen rows untouched)
  auto vertex_knn = [&](const float3* q, const char* name) -> float {
    if (in.knn_mode == 0)
      return run_knn_bitonic_query_to_mesh(nV, dV, q, nS, KPROJ, dFrozen, (idx_t*)dKnnV, dKnnVdist, name);
    cudaEventRecord(k0);
    knn_vertices_bruteforce_k<KPROJ, false><<<grd, blk>>>(dV, nV, q, nS, dFrozen, dKnnV);
    cudaEventRecord(k1);
    cudaEventSynchronize(k1);
    float t = 0;
    cudaEventElapsedTime(&t, k0, k1);
    return t;
  };
  std::vector<unsigned char> hTier(nS, 0);
  if (mode != 0) {
    static const int S1[6] = {5, 10, 15, 20, 25, 25};
    static const int S2[6] = {5, 10, 15, 20, 25, 10};
    float thr[6];
    for (int t = 0; t < 6; ++t) thr[t] = freeze_disp;
    cudaMemcpy(dThr, thr, sizeof(thr), cudaMemcpyHostToDevice);
    cudaMemcpy(dStreakTier, mode == 1 ? S1 : S2, 6 * sizeof(int), cudaMemcpyHostToDevice);
    site_knn(dS);
    knn_drop_self_kernel<K_SITE, K_NEIGH, idx_t><<<grd, blk>>>(dRaw, dKNN, nS);
    knn_vertices_bruteforce_k<KPROJ, false><<<grd, blk>>>(dV, nV, dS, nS, dFrozen, dKnnV);
    cudaDeviceSynchronize();
    std::vector<idx_t> hk((size_t)nS * K_NEIGH);
    std::vector<int> hkv((size_t)nS * KPROJ);
    std::vector<float> hN((size_t)nV * 3), sn((size_t)nS * 3);
    cudaMemcpy(hk.data(), dKNN, hk.size() * sizeof(idx_t), cudaMemcpyDeviceToHost);
    cudaMemcpy(hkv.data(), dKnnV, hkv.size() * sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(hN.data(), dN, hN.size() * sizeof(float), cudaMemcpyDeviceToHost);
    for (int i = 0; i < nS; ++i) {
      int v = hkv[(size_t)i * KPROJ];
      for (int a = 0; a < 3; ++a) sn[3 * i + a] = v >= 0 ? hN[3 * v + a] : 0.f;
    }
    tiers(mode, nS, K_NEIGH, sn, hk, hTier);
    cudaMalloc(&dTier, nS);
    cudaMemcpy(dTier, hTier.data(), nS, cudaMemcpyHostToDevice);
  }

  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto ms = [&]() { float t = 0; cudaEventSynchronize(e1); cudaEventElapsedTime(&t, e0, e1); return t; };
  std::vector<float> stage((size_t)iters * 6, 0.f);
  std::vector<int> counts((size_t)iters * 4, 0);
  std::vector<std::vector<float>> dumps;
  std::vector<idx_t> knn0((size_t)nS * K_NEIGH);
  std::vector<int> knnv0((size_t)nS * KPROJ);
  std::vector<float> cent0((size_t)nS * 3);
  size_t next_dump = 0;

  for (int it = 0; it < iters; ++it) {
    float* st = &stage[(size_t)it * 6];
    st[0] = site_knn(dS);
    knn_drop_self_kernel<K_SITE, K_NEIGH, idx_t><<<grd, blk>>>(dRaw, dKNN, nS);
    if (mode != 0) restore_rows<K_NEIGH><<<grd, blk>>>(dFrozen, dPrev, dKNN, nS);
    if (mode != 0) {
      cudaMemcpy(dPrevKnnV, dKnnV, (size_t)nS * KPROJ * sizeof(int), cudaMemcpyDeviceToDevice);
      st[1] = vertex_knn(dS, "site_to_mesh");
      restore_prev_knn_vertices_kernel<KPROJ><<<grd, blk>>>(dFrozen, dPrevKnnV, dKnnV, nS);
    } else {
      cudaEventRecord(e0);
      knn_vertices_bruteforce_k<KPROJ, false><<<grd, blk>>>(dV, nV, dS, nS, dFrozen, dKnnV);
      cudaEventRecord(e1);
      st[1] = ms();
    }
    cudaEventRecord(e0);
    uv_from_nearest_vertex_normal<KPROJ><<<grd, blk>>>(dN, dKnnV, du, dv, nS);
    cudaEventRecord(e1);
    st[2] = ms();
    cudaEventRecord(e0);
    centroids_tangent_voronoi<<<grd, blk>>>(dS, du, dv, dKNN, nS, K_NEIGH, R, dFrozen, dCent);
    cudaEventRecord(e1);
    st[3] = ms();
    if (mode != 0) {
      cudaMemcpy(dPrevKnnV, dKnnV, (size_t)nS * KPROJ * sizeof(int), cudaMemcpyDeviceToDevice);
      st[4] = vertex_knn(dCent, "centroid_to_mesh");
      restore_prev_knn_vertices_kernel<KPROJ><<<grd, blk>>>(dFrozen, dPrevKnnV, dKnnV, nS);
    } else {
      cudaEventRecord(e0);
      knn_vertices_bruteforce_k<KPROJ, true><<<grd, blk>>>(dV, nV, dCent, nS, dFrozen, dKnnV);
      cudaEventRecord(e1);
      st[4] = ms();
    }
    cudaEventRecord(e0);
    project_centroids_to_mesh<KPROJ><<<grd, blk>>>(dCent, dV, (const int3*)dF, dOff, dFcs, dKnnV, nV, nF, nS, dFrozen,
                                                   dS, dSnew);
    cudaEventRecord(e1);
    st[5] = ms();
    if (it == 0) {
      cudaMemcpy(knn0.data(), dKNN, knn0.size() * sizeof(idx_t), cudaMemcpyDeviceToHost);
      cudaMemcpy(knnv0.data(), dKnnV, knnv0.size() * sizeof(int), cudaMemcpyDeviceToHost);
      cudaMemcpy(cent0.data(), dCent, cent0.size() * sizeof(float), cudaMemcpyDeviceToHost);
    }
    int has_prev = it > 0 ? 1 : 0;
    cudaMemset(dCounts, 0, 4 * sizeof(int));
    cudaMemset(dCand, 0, nS);
    if (mode == 0)
      freeze_test_kernel_streak<K_NEIGH, idx_t><<<grd, blk>>>(dS, dSnew, dKNN, dPrev, dCand, dStreak, freeze_disp, nS,
                                                              has_prev, 5, dCounts);
    else
      freeze_test_kernel_streak_tiered<K_NEIGH, idx_t><<<grd, blk>>>(dS, dSnew, dKNN, dPrev, dCand, dStreak, dTier,
                                                                     dThr, dStreakTier, nS, has_prev, dCounts);
    freeze_apply_cand_kernel<<<grd, blk>>>(dCand, dFrozen, nS, dCounts);
    cudaMemcpy(&counts[(size_t)it * 4], dCounts, 4 * sizeof(int), cudaMemcpyDeviceToHost);
    if (mode == 0) {
      cudaMemset(dFrozen, 0, nS);
      cudaMemset(dStreak, 0, nS);
    }
    cudaMemcpy(dPrev, dKNN, (size_t)nS * K_NEIGH * sizeof(idx_t), cudaMemcpyDeviceToDevice);
    std::swap(dS, dSnew);
    if (next_dump < in.dump.size() && in.dump[next_dump] == it + 1) {
      std::vector<float> s((size_t)nS * 3);
      cudaMemcpy(s.data(), dS, s.size() * sizeof(float), cudaMemcpyDeviceToHost);
      dumps.push_back(std::move(s));
      next_dump++;
    }
  }
  cudaDeviceSynchronize();
  float wall_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - wall0).count();

  // final evaluation: candidate mesh by face extraction (main.cu:883-974) and
  // quality + one-sided Hausdorff (main.cu:1009-1035)
  std::vector<float3> hS(nS);
  cudaMemcpy(hS.data(), dS, nS * sizeof(float3), cudaMemcpyDeviceToHost);
  if (mode != 0) {
    cudaMemcpy(dPrevKnnV, dKnnV, (size_t)nS * KPROJ * sizeof(int), cudaMemcpyDeviceToDevice);
    vertex_knn(dS, "site_to_mesh");
    restore_prev_knn_vertices_kernel<KPROJ><<<grd, blk>>>(dFrozen, dPrevKnnV, dKnnV, nS);
  } else {
    knn_vertices_bruteforce_k<KPROJ, false><<<grd, blk>>>(dV, nV, dS, nS, dFrozen, dKnnV);
  }
  uv_from_nearest_vertex_normal<KPROJ><<<grd, blk>>>(dN, dKnnV, du, dv, nS);
  float3 mn = make_float3(1e30f, 1e30f, 1e30f), mx = make_float3(-1e30f, -1e30f, -1e30f);
  for (int i = 0; i < nS; ++i) {
    mn.x = std::min(mn.x, hS[i].x); mn.y = std::min(mn.y, hS[i].y); mn.z = std::min(mn.z, hS[i].z);
    mx.x = std::max(mx.x, hS[i].x); mx.y = std::max(mx.y, hS[i].y); mx.z = std::max(mx.z, hS[i].z);
  }
  float R2 = 2.0f * 0.5f * std::max(mx.x - mn.x, std::max(mx.y - mn.y, mx.z - mn.z));
  float2* dPoly;
  int *dPolyN, *dKeyCount;
  int2* dLab;
  uint64_t* dKeys;
  size_t maxCand = (size_t)nS * MAX_POLY;
  cudaMalloc(&dPoly, maxCand * sizeof(float2));
  cudaMalloc(&dLab, maxCand * sizeof(int2));
  cudaMalloc(&dPolyN, nS * sizeof(int));
  cudaMalloc(&dKeys, maxCand * sizeof(uint64_t));
  cudaMalloc(&dKeyCount, sizeof(int));
  cudaMemset(dPolyN, 0, nS * sizeof(int));
  cell_poly2d_kernel<K_NEIGH, MAX_POLY, idx_t><<<grd, blk>>>(dS, du, dv, dKNN, nS, R2, 1e-8f, 1e-7f, dPoly, dPolyN, dLab);
  cudaMemset(dKeyCount, 0, sizeof(int));
  emit_faces_from_labels_kernel<MAX_POLY><<<grd, blk>>>(dPolyN, dLab, nS, dKeys, dKeyCount, (int)maxCand);
  int hCount = 0;
  cudaMemcpy(&hCount, dKeyCount, sizeof(int), cudaMemcpyDeviceToHost);
  hCount = std::max(0, std::min(hCount, (int)maxCand));
  std::vector<uint64_t> hKeys(hCount);
  cudaMemcpy(hKeys.data(), dKeys, hCount * sizeof(uint64_t), cudaMemcpyDeviceToHost);
  std::sort(hKeys.begin(), hKeys.end());
  hKeys.erase(std::unique(hKeys.begin(), hKeys.end()), hKeys.end());
  std::vector<Tri> faces, kept;
  decode_keys_to_faces(hKeys, faces);
  for (const Tri& t : faces)
    if (!is_degenerate_tri(hS, t.a, t.b, t.c, 1e-6f)) kept.push_back(t);
  std::vector<int3i> hFc;
  for (const Tri& t : kept) hFc.push_back({t.a, t.b, t.c});
  float q[6] = {0, 0, 0, 0, 0, 0};
  eval_quality_angles_cpu(hS, hFc, q[0], q[1], q[2], q[3], q[4], q[5]);
  std::vector<BVHNode> nodes;
  std::vector<int> triIdx;
  build_bvh(hV, hF, 8, nodes, triIdx);
  BVHNode* dNodes;
  int* dTri;
  float3* dVc;
  int3i* dFc;
  cudaMalloc(&dNodes, nodes.size() * sizeof(BVHNode));
  cudaMalloc(&dTri, triIdx.size() * sizeof(int));
  cudaMalloc(&dVc, nS * sizeof(float3));
  cudaMalloc(&dFc, std::max<size_t>(hFc.size(), 1) * sizeof(int3i));
  cudaMemcpy(dNodes, nodes.data(), nodes.size() * sizeof(BVHNode), cudaMemcpyHostToDevice);
  cudaMemcpy(dTri, triIdx.data(), triIdx.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(dVc, hS.data(), nS * sizeof(float3), cudaMemcpyHostToDevice);
  cudaMemcpy(dFc, hFc.data(), hFc.size() * sizeof(int3i), cudaMemcpyHostToDevice);
  float dH = hausdorff_cand_to_ref_gpu(dV, nV, dF, nF, dNodes, (int)nodes.size(), dTri, dVc, nS, dFc, (int)hFc.size());

  std::vector<unsigned char> frozen(nS);
  cudaMemcpy(frozen.data(), dFrozen, nS, cudaMemcpyDeviceToHost);
  cudaError_t err = cudaDeviceSynchronize();
  if (err == cudaSuccess) err = cudaGetLastError();
  if (err != cudaSuccess) {
    fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err));
    return 3;
  }
  int nd = (int)dumps.size(), nFc = (int)hFc.size();
  fwrite(&iters, 4, 1, fo);
  fwrite(&nd, 4, 1, fo);
  for (auto& d : dumps) fwrite(d.data(), 4, d.size(), fo);
  fwrite(counts.data(), 4, counts.size(), fo);
  fwrite(knn0.data(), 4, knn0.size(), fo);
  fwrite(knnv0.data(), 4, knnv0.size(), fo);
  fwrite(cent0.data(), 4, cent0.size(), fo);
  fwrite(frozen.data(), 1, frozen.size(), fo);
  fwrite(hTier.data(), 1, hTier.size(), fo);
  fwrite(stage.data(), 4, stage.size(), fo);
  fwrite(q, 4, 6, fo);
  fwrite(&dH, 4, 1, fo);
  fwrite(&nFc, 4, 1, fo);
  fwrite(&wall_ms, 4, 1, fo);
  return 0;
}

}  // namespace harness

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
    return 2;
  }
  FILE* fi = fopen(argv[1], "rb");
  if (!fi) return 2;
  harness::In in;
  int hdr[8];
  if (fread(hdr, 4, 8, fi) != 8) return 2;
  in.nV = hdr[0]; in.nF = hdr[1]; in.nS = hdr[2]; in.K = hdr[3]; in.mode = hdr[4]; in.iters = hdr[5];
  in.knn_mode = hdr[6];
  in.dump.resize(hdr[7]);
  if (hdr[7] && fread(in.dump.data(), 4, hdr[7], fi) != (size_t)hdr[7]) return 2;
  in.V.resize((size_t)in.nV * 3);
  in.F.resize((size_t)in.nF * 3);
  in.S.resize((size_t)in.nS * 3);
  if (fread(in.V.data(), 4, in.V.size(), fi) != in.V.size()) return 2;
  if (fread(in.F.data(), 4, in.F.size(), fi) != in.F.size()) return 2;
  if (fread(in.S.data(), 4, in.S.size(), fi) != in.S.size()) return 2;
  fclose(fi);
  // the hub index needs >= 1024 points per cell (bitonic-hubs-grid.cuh:1313-1318)
  if (in.knn_mode == 0 && (in.nS < 1024 || in.nV < 1024)) {
    fprintf(stderr, "the reference KNN needs at least 1024 sites and vertices\n");
    return 4;
  }
  FILE* fo = fopen(argv[2], "wb");
  if (!fo) return 2;
  int rc;
  switch (in.K) {
    case 20: rc = harness::run<20>(in, fo); break;
    case 24: rc = harness::run<24>(in, fo); break;
    case 32: rc = harness::run<32>(in, fo); break;
    default: fprintf(stderr, "K must be 20, 24 or 32\n"); rc = 2;
  }
  fclose(fo);
  return rc;
}
