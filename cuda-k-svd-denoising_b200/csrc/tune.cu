// Autotuner: picks the update sweep's slice size (entries per CTA before
// another CTA joins an atom) for a workload by timing one sweep with each
// candidate on the caller's data.  Fewer, larger slices cut the per-step
// all-reduce (every CTA of an atom reads every other CTA's partial); more,
// smaller slices spread the residual-row traffic over more SMs.
#include <cuda_runtime.h>

#include <cstring>

#include "capi_common.cuh"
#include "ksvd_internal.cuh"

using namespace ksvd::api;

extern "C" ksvd_status ksvd_autotune(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict,
                                     ksvd_tune_result* out) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_dict || N < 1) return fail(c, KSVD_ERR_INVALID, "bad argument");
  const int64_t n64 = int64_t(c->p.patch_width_dim) * c->p.patch_height_dim;
  if (n64 < 1 || n64 > 512) return fail(c, KSVD_ERR_INVALID, "patch size out of range");
  const int n = int(n64), K = c->p.atoms, L = c->p.omp_iter;
  static const int kSlices[] = {32, 48, 64, 96, 128, 192, 256};
  constexpr int kNum = int(sizeof(kSlices) / sizeof(kSlices[0]));
  static_assert(kNum <= KSVD_TUNE_MAX, "too many candidates");
  float *dict = nullptr, *coef0 = nullptr, *coef = nullptr;
  int32_t* idx = nullptr;
  KSVD_TRY(wsT(c, "tune_dict", size_t(K) * n, &dict));
  KSVD_TRY(wsT(c, "tune_idx", size_t(N) * L, &idx));
  KSVD_TRY(wsT(c, "tune_coef0", size_t(N) * L, &coef0));
  KSVD_TRY(wsT(c, "tune_coef", size_t(N) * L, &coef));
  // the codes of the first iteration (the context's own OMP form)
  KSVD_TRY(omp_form(c, d_patches, N, d_dict, idx, coef0, c->p.precision == KSVD_PREC_BF16_LEARNED
                                                             ? KSVD_PREC_BF16_RESCORE
                                                             : c->p.precision));
  const int saved = c->upd_slice;
  cudaEvent_t e0 = get_event(c), e1 = get_event(c);
  double best = 1e300;
  int best_slice = saved;
  ksvd_tune_result r;
  std::memset(&r, 0, sizeof(r));
  ksvd_status st = KSVD_OK;
  for (int i = 0; i < kNum && st == KSVD_OK; ++i) {
    c->upd_slice = kSlices[i];
    float ms = 0.0f;
    for (int rep = 0; rep < 2 && st == KSVD_OK; ++rep) {  // the first sweep warms up
      cudaMemcpyAsync(dict, d_dict, size_t(K) * n * 4, cudaMemcpyDeviceToDevice, c->stream);
      cudaMemcpyAsync(coef, coef0, size_t(N) * L * 4, cudaMemcpyDeviceToDevice, c->stream);
      cudaEventRecord(e0, c->stream);
      st = update_form(c, d_patches, N, dict, idx, coef);
      cudaEventRecord(e1, c->stream);
      if (st == KSVD_OK) st = check_dev_flags(c, "autotune");
      if (st == KSVD_OK) cudaEventElapsedTime(&ms, e0, e1);
    }
    r.slice[i] = kSlices[i];
    r.update_ms[i] = ms;
    if (st == KSVD_OK && ms < best) {
      best = ms;
      best_slice = kSlices[i];
    }
  }
  c->event_pool.push_back(e0);
  c->event_pool.push_back(e1);
  if (st != KSVD_OK) {
    c->upd_slice = saved;
    return st;
  }
  c->upd_slice = best_slice;
  r.update_slice = best_slice;
  r.candidates = kNum;
  if (out) *out = r;
  return KSVD_OK;
}

extern "C" ksvd_status ksvd_set_update_slice(ksvd_ctx* c, int slice) {
  if (!c) return KSVD_ERR_INVALID;
  if (slice < 0 || slice > 4096) return fail(c, KSVD_ERR_INVALID, "slice must be in [0, 4096]");
  c->upd_slice = slice;
  return KSVD_OK;
}
