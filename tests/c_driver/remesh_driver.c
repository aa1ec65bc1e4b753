/* A plain C driver of libgpucvt, the way the reference's main.cu would call
 * it: mesh in, sites = the mesh vertices (main.cu:493), 30 Lloyd iterations
 * of the resident engine with five-tier freezing, evaluation, then the same
 * run through the one-call cvt_remesh.  Built and run by
 * tests/test_host.py (link) and tests/test_gpu_engine.py (run).
 * Prints "faces F dH H Qavg Q frozen_iter29 N same S". */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gpu_cvt.h"

#define CHECK(x)                                                                   \
  do {                                                                             \
    cvt_status_t s_ = (x);                                                         \
    if (s_ != CVT_OK) {                                                            \
      fprintf(stderr, "%s failed: %s (%s)\n", #x, cvt_status_string(s_), cvt_last_error()); \
      return 1;                                                                    \
    }                                                                              \
  } while (0)

/* UV sphere: nu x nv quads split into triangles, poles shared */
static void uv_sphere(int nu, int nv, float** V, int* nV, int** F, int* nF) {
  const double pi = 3.14159265358979323846;
  *nV = nu * (nv - 1) + 2;
  *nF = 2 * nu * (nv - 1);
  *V = (float*)malloc(sizeof(float) * 3 * (size_t)*nV);
  *F = (int*)malloc(sizeof(int) * 3 * (size_t)*nF);
  float* v = *V;
  int* f = *F;
  int k = 0;
  v[k++] = 0.f; v[k++] = 0.f; v[k++] = 1.f;
  for (int j = 1; j < nv; ++j) {
    double th = pi * j / nv;
    for (int i = 0; i < nu; ++i) {
      double ph = 2.0 * pi * i / nu;
      v[k++] = (float)(sin(th) * cos(ph)); v[k++] = (float)(sin(th) * sin(ph)); v[k++] = (float)cos(th);
    }
  }
  v[k++] = 0.f; v[k++] = 0.f; v[k++] = -1.f;
  int t = 0;
  const int south = *nV - 1;
  for (int i = 0; i < nu; ++i) {
    int a = 1 + i, b = 1 + (i + 1) % nu;
    f[t++] = 0; f[t++] = a; f[t++] = b;
  }
  for (int j = 1; j < nv - 1; ++j)
    for (int i = 0; i < nu; ++i) {
      int a = 1 + (j - 1) * nu + i, b = 1 + (j - 1) * nu + (i + 1) % nu;
      int c = a + nu, d = b + nu;
      f[t++] = a; f[t++] = c; f[t++] = b;
      f[t++] = b; f[t++] = c; f[t++] = d;
    }
  for (int i = 0; i < nu; ++i) {
    int a = 1 + (nv - 2) * nu + i, b = 1 + (nv - 2) * nu + (i + 1) % nu;
    f[t++] = a; f[t++] = south; f[t++] = b;
  }
}

int main(void) {
  float* V;
  int* F;
  int nV, nF;
  uv_sphere(96, 48, &V, &nV, &F, &nF);
  const int iters = 30;

  cvt_params_t p;
  cvt_params_default(&p);
  p.k = 24;
  p.mode = 1;
  p.profile = CVT_PROFILE_MIXED;

  cvt_mesh_t mesh;
  CHECK(cvt_mesh_create(V, nV, F, nF, &mesh));
  int cells = 0;
  CHECK(cvt_segment_cells(mesh, nV, &p, &cells));
  cvt_engine_t e;
  CHECK(cvt_engine_create(&p, 1, nV, cells, &e));
  int seg = -1;
  CHECK(cvt_engine_add_segment(e, mesh, V, nV, 0, &seg, NULL));
  CHECK(cvt_engine_run(e, iters, NULL));
  cvt_eval_t ev;
  CHECK(cvt_engine_evaluate(e, seg, &ev, NULL));
  cvt_iter_stats_t st;
  CHECK(cvt_engine_get_stats(e, seg, iters - 1, &st, NULL));
  float* S1 = (float*)malloc(sizeof(float) * 3 * (size_t)nV);
  float* S2 = (float*)malloc(sizeof(float) * 3 * (size_t)nV);
  CHECK(cvt_engine_get_sites(e, seg, S1, 0, NULL));
  uint8_t* frozen = (uint8_t*)malloc((size_t)nV);
  CHECK(cvt_engine_get_state(e, seg, NULL, NULL, frozen, NULL, NULL));
  int nfrozen = 0;
  for (int i = 0; i < nV; ++i) nfrozen += frozen[i];
  CHECK(cvt_engine_destroy(e));
  CHECK(cvt_mesh_destroy(mesh));

  CHECK(cvt_remesh(V, nV, F, nF, V, nV, &p, iters, S2, NULL));
  const int same = memcmp(S1, S2, sizeof(float) * 3 * (size_t)nV) == 0;
  printf("faces %d dH %.6g Qavg %.6g frozen %d same %d\n", ev.n_faces, ev.dH / ev.diag, ev.Qavg, nfrozen, same);
  free(V); free(F); free(S1); free(S2); free(frozen);
  return same ? 0 : 2;
}
