// swm_batch.cu -- batched ensembles of independent problems.
// First form: one handle per problem, stepped in sequence on the device, each
// with its own dt.  (The persistent multi-problem kernels replace this path.)
#include <cstdlib>
#include <vector>

#include "../../include/swm.h"

struct swm_batch {
  std::vector<swm_handle> h;
  std::vector<long long> cells;
};

extern "C" {

int swm_batch_create(int n, const swm_params* p, swm_batch_handle* out) {
  if (!out || !p || n < 1) return SWM_ERR_PARAM;
  *out = nullptr;
  swm_batch* b = new swm_batch();
  for (int i = 0; i < n; ++i) {
    swm_handle h = nullptr;
    int rc = swm_create(&p[i], &h);
    if (rc) {
      swm_batch_destroy(b);
      return rc;
    }
    b->h.push_back(h);
    b->cells.push_back((long long)p[i].nx * p[i].ny);
  }
  *out = b;
  return SWM_OK;
}

int swm_batch_destroy(swm_batch_handle b) {
  if (!b) return SWM_OK;
  for (auto h : b->h) swm_destroy(h);
  delete b;
  return SWM_OK;
}

int swm_batch_set_planes(swm_batch_handle b, int i, const double* planes) {
  if (!b || i < 0 || i >= (int)b->h.size()) return SWM_ERR_PARAM;
  return swm_set_planes(b->h[i], planes);
}

int swm_batch_get_planes(swm_batch_handle b, int i, double* planes) {
  if (!b || i < 0 || i >= (int)b->h.size()) return SWM_ERR_PARAM;
  return swm_get_planes(b->h[i], planes);
}

int swm_batch_step(swm_batch_handle b, double* dt_out) {
  if (!b) return SWM_ERR_PARAM;
  int warn = 0;
  for (size_t i = 0; i < b->h.size(); ++i) {
    double dt;
    int rc = swm_timestep(b->h[i], &dt);
    if (rc < 0) return rc;
    rc = swm_step(b->h[i], 0.0, dt);
    if (rc < 0) return rc;
    if (rc > 0) warn = rc;
    if (dt_out) dt_out[i] = dt;
  }
  return warn;
}

int swm_batch_cells(swm_batch_handle b, long long* cells) {
  if (!b || !cells) return SWM_ERR_PARAM;
  long long s = 0;
  for (auto c : b->cells) s += c;
  *cells = s;
  return SWM_OK;
}

}  // extern "C"
