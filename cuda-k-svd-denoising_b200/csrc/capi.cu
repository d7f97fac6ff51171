// C ABI of ksvd_sm100 (declared in include/ksvd_sm100.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "capi_common.cuh"
#include "ksvd_internal.cuh"

using ksvd::PatchGeom;

namespace {

using namespace ksvd::api;

bool geom_of(const ksvd_params& p, int W, int H, PatchGeom* g) {
  return ksvd::make_geom(W, H, p.patch_width_dim, p.patch_height_dim, p.sliding_width, p.sliding_height, g);
}

ksvd_status validate_params(const ksvd_params* p, std::string* why) {
  auto bad = [&](const char* m) {
    *why = m;
    return KSVD_ERR_INVALID;
  };
  if (p->patch_width_dim < 1 || p->patch_height_dim < 1) return bad("patch dimensions must be >= 1");
  if (p->sliding_width < 1 || p->sliding_height < 1) return bad("sliding steps must be >= 1");
  if (p->atoms < 1) return bad("atoms must be >= 1");
  if (p->omp_iter < 1 || p->omp_iter > 32) return bad("ompIter must be in [1, 32]");
  if (p->ksvd_iter < 0) return bad("ksvdIter must be >= 0");
  if (p->type < KSVD_CUDA_K_GESVD || p->type > KSVD_CUDA_K_SM100A) return bad("unknown type");
  if (p->precision != KSVD_PREC_FP32 && p->precision != KSVD_PREC_BF16_RESCORE &&
      p->precision != KSVD_PREC_FP16_RESCORE && p->precision != KSVD_PREC_BF16_LEARNED)
    return bad("unknown precision");
  if (p->sub_image_width_dim < 0 || p->sub_image_height_dim < 0) return bad("sub-image dimensions must be >= 0");
  return KSVD_OK;
}

ksvd_status check_kernel_support(ksvd_ctx* c) {
  // the patch area is bounded before it is formed as an int
  const int64_t n64 = int64_t(c->p.patch_width_dim) * c->p.patch_height_dim;
  if (n64 < 1 || n64 > 512) return fail(c, KSVD_ERR_INVALID, "patch size pw x ph must be in [1, 512]");
  const int n = int(n64), K = c->p.atoms, L = c->p.omp_iter;
  if (!ksvd::omp_tc_supported(n, K, L) && !ksvd::omp_fp32_supported(n, K, L) && !ksvd::omp_stream_supported(n, K, L))
    return fail(c, KSVD_ERR_INVALID, "patch size x atoms x ompIter beyond every OMP kernel (atoms <= 1024)");
  if (!ksvd::update_res_supported(n))
    return fail(c, KSVD_ERR_INVALID, "patch size > 512 not supported by the update kernel");
  return KSVD_OK;
}

}  // namespace

extern "C" {

int ksvd_abi_version(void) { return KSVD_ABI_VERSION; }

void ksvd_params_default(ksvd_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->patch_width_dim = 8;
  p->patch_height_dim = 8;
  p->sliding_width = 2;
  p->sliding_height = 2;
  p->atoms = 256;
  p->ksvd_iter = 10;
  p->omp_iter = 5;
  p->bw = 1;
  p->speckle = 0;
  p->type = KSVD_CUDA_K_SM100A;
  p->min_omp_iter_batch = 0;
  p->sub_image_width_dim = 0;
  p->sub_image_height_dim = 0;
  p->precision = KSVD_PREC_FP32;
  p->compat = KSVD_COMPAT_REFERENCE;
  p->device = 0;
}

static const char* kTypeNames[] = {"CUDA_K_GESVD", "CUDA_K_GESVDJ", "CUDA_K_GESVDA", "CUDA_K_SM100A"};

int ksvd_type_from_string(const char* name, int* known) {
  if (known) *known = 0;
  if (!name) return KSVD_CUDA_K_GESVD;
  for (int i = 0; i < 4; ++i)
    if (std::strcmp(name, kTypeNames[i]) == 0) {
      if (known) *known = 1;
      return i;
    }
  return KSVD_CUDA_K_GESVD;
}

const char* ksvd_type_name(int type) {
  if (type < 0 || type > 3) return "UNKNOWN";
  return kTypeNames[type];
}

const char* ksvd_status_string(int st) {
  switch (st) {
    case KSVD_OK: return "ok";
    case KSVD_ERR_LOAD: return "image loading failed";
    case KSVD_ERR_DENOISE: return "denoising failed";
    case KSVD_ERR_SAVE: return "image saving failed";
    case KSVD_ERR_INVALID: return "invalid argument";
    case KSVD_ERR_CUDA: return "CUDA error";
    case KSVD_ERR_NO_MEMORY: return "out of device memory";
    case KSVD_ERR_TIMEOUT: return "device wait timed out";
    case KSVD_ERR_NUMERIC: return "numerical failure";
    case KSVD_ERR_NO_DEVICE: return "no CUDA device";
    case KSVD_ERR_TOO_LARGE: return "size beyond the fixed maximum";
    default: return "unknown status";
  }
}

int64_t ksvd_num_patches(const ksvd_params* p, int width, int height) {
  if (!p) return -1;
  PatchGeom g;
  if (!geom_of(*p, width, height, &g)) return -1;
  return g.N;
}

ksvd_status ksvd_create(const ksvd_params* p, ksvd_ctx** out) {
  if (!p || !out) return KSVD_ERR_INVALID;
  *out = nullptr;
  std::string why;
  if (validate_params(p, &why) != KSVD_OK) return KSVD_ERR_INVALID;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return KSVD_ERR_NO_DEVICE;
  }
  if (p->device < 0 || p->device >= ndev) return KSVD_ERR_INVALID;
  ksvd_ctx* c = new (std::nothrow) ksvd_ctx();
  if (!c) return KSVD_ERR_NO_MEMORY;
  c->p = *p;
  c->device = p->device;
  if (cudaSetDevice(c->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->d_flags, sizeof(ksvd::GridBarrier)) != cudaSuccess ||
      cudaMalloc(&c->d_stats, sizeof(ksvd::DevStats)) != cudaSuccess ||
      cudaMalloc(&c->d_phase, sizeof(ksvd::DevStats)) != cudaSuccess ||
      cudaMemset(c->d_phase, 0, sizeof(ksvd::DevStats)) != cudaSuccess ||
      cudaMemset(c->d_flags, 0, sizeof(ksvd::GridBarrier)) != cudaSuccess ||
      cudaMemset(c->d_stats, 0, sizeof(ksvd::DevStats)) != cudaSuccess) {
    cudaGetLastError();
    ksvd_destroy(c);
    return KSVD_ERR_CUDA;
  }
  c->stream = c->own_stream;
  *out = c;
  return KSVD_OK;
}

void ksvd_destroy(ksvd_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& kv : c->bufs)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  for (auto& kv : c->families)
    for (auto& pr : kv.second.pending) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  for (auto e : c->event_pool) cudaEventDestroy(e);
  if (c->d_flags) cudaFree(c->d_flags);
  if (c->d_stats) cudaFree(c->d_stats);
  if (c->d_phase) cudaFree(c->d_phase);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

const char* ksvd_last_error(const ksvd_ctx* c) { return c ? c->err.c_str() : "null context"; }

ksvd_status ksvd_set_stream(ksvd_ctx* c, void* stream) {
  if (!c) return KSVD_ERR_INVALID;
  c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
  return KSVD_OK;
}

void* ksvd_get_stream(const ksvd_ctx* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

ksvd_status ksvd_profile_enable(ksvd_ctx* c, int enable) {
  if (!c) return KSVD_ERR_INVALID;
  c->profiling = enable < 0 ? 0 : (enable > 2 ? 2 : enable);
  return KSVD_OK;
}

ksvd_status ksvd_profile_reset(ksvd_ctx* c) {
  if (!c) return KSVD_ERR_INVALID;
  cudaStreamSynchronize(c->stream);
  cudaMemset(c->d_phase, 0, sizeof(ksvd::DevStats));
  for (auto& kv : c->families) {
    for (auto& pr : kv.second.pending) {
      c->event_pool.push_back(pr.first);
      c->event_pool.push_back(pr.second);
    }
    kv.second.pending.clear();
    kv.second.total_ms = 0.0;
    kv.second.launches = 0;
  }
  return KSVD_OK;
}

ksvd_status ksvd_profile_read(ksvd_ctx* c, const char* family, double* total_ms, int64_t* launches) {
  if (!c || !family) return KSVD_ERR_INVALID;
  KSVD_TRY(check_ctx(c));
  KSVD_CU(c, cudaStreamSynchronize(c->stream), "profile sync");
  auto it = c->families.find(family);
  if (it == c->families.end()) {
    if (total_ms) *total_ms = 0.0;
    if (launches) *launches = 0;
    return KSVD_OK;
  }
  auto& f = it->second;
  for (auto& pr : f.pending) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, pr.first, pr.second);
    f.total_ms += ms;
    c->event_pool.push_back(pr.first);
    c->event_pool.push_back(pr.second);
  }
  f.pending.clear();
  if (total_ms) *total_ms = f.total_ms;
  if (launches) *launches = f.launches;
  return KSVD_OK;
}

int64_t ksvd_launch_count(const ksvd_ctx* c) { return c ? c->launch_count : 0; }

ksvd_status ksvd_profile_counters(ksvd_ctx* c, int64_t* out, int count) {
  if (!c || !out || count < 1) return KSVD_ERR_INVALID;
  KSVD_TRY(check_ctx(c));
  ksvd::DevStats h{};
  KSVD_CU(c, cudaStreamSynchronize(c->stream), "profile sync");
  KSVD_CU(c, cudaMemcpy(&h, c->d_phase, sizeof(h), cudaMemcpyDeviceToHost), "counters");
  const int64_t v[4] = {int64_t(h.power_iters), int64_t(h.atoms_updated), int64_t(h.omp_rescore_misses),
                        int64_t(h.pad)};
  for (int i = 0; i < count; ++i) out[i] = i < 4 ? v[i] : 0;
  return KSVD_OK;
}

ksvd_status ksvd_profile_phases(ksvd_ctx* c, double* ms_out, int count) {
  if (!c || !ms_out || count < 1) return KSVD_ERR_INVALID;
  KSVD_TRY(check_ctx(c));
  ksvd::DevStats h{};
  KSVD_CU(c, cudaStreamSynchronize(c->stream), "profile sync");
  KSVD_CU(c, cudaMemcpy(&h, c->d_phase, sizeof(h), cudaMemcpyDeviceToHost), "phase timers");
  for (int i = 0; i < count; ++i) ms_out[i] = (i < 16) ? double(h.phase_ns[i]) * 1e-6 : 0.0;
  return KSVD_OK;
}

// ---------------------------------------------------------------------------
// Stage entry points
// ---------------------------------------------------------------------------

ksvd_status ksvd_extract_patches(ksvd_ctx* c, const float* d_img, int width, int height, float* d_patches) {
  KSVD_TRY(check_ctx(c));
  if (!d_img || !d_patches) return fail(c, KSVD_ERR_INVALID, "null pointer");
  PatchGeom g;
  if (!geom_of(c->p, width, height, &g)) return fail(c, KSVD_ERR_INVALID, "patch geometry does not fit the image");
  Prof pr(c, "im2col", 1);
  KSVD_CU(c, ksvd::launch_im2col(d_img, g, d_patches, c->stream), "im2col");
  return KSVD_OK;
}

ksvd_status ksvd_init_dictionary(ksvd_ctx* c, const float* d_patches, int64_t N, float* d_dict) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_dict) return fail(c, KSVD_ERR_INVALID, "null pointer");
  const int64_t n64 = int64_t(c->p.patch_width_dim) * c->p.patch_height_dim;
  if (n64 < 1 || n64 > (int64_t(1) << 20)) return fail(c, KSVD_ERR_INVALID, "patch area out of range");
  const int n = int(n64), K = c->p.atoms;
  if (N < 1 || N / 2 + K > N) return fail(c, KSVD_ERR_INVALID, "fewer patches than N/2 + atoms");
  {
    Prof pr(c, "init_dict", 1);
    KSVD_CU(c,
            ksvd::launch_init_dict(d_patches, N, n, K, (c->p.compat & KSVD_COMPAT_INT_NORM) ? 1 : 0, d_dict,
                                   c->d_flags, c->stream),
            "init_dict");
  }
  return check_dev_flags(c, "initDictionary");
}

}  // extern "C"

namespace ksvd {
namespace api {

ksvd_status omp_form(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict, int32_t* d_idx,
                     float* d_coef, int precision, bool for_update) {
  const int n = c->p.patch_width_dim * c->p.patch_height_dim, K = c->p.atoms, L = c->p.omp_iter;
  c->resid_fused = false;
  double* gram = nullptr;
  KSVD_TRY(wsT(c, "gram", size_t(K) * K, &gram));
  {
    Prof pr(c, "gram", 1);
    KSVD_CU(c, ksvd::launch_gram_f64(d_dict, K, n, gram, c->stream), "gram");
  }
  if (precision == KSVD_PREC_BF16_LEARNED) return omp_learned_impl(c, d_patches, N, d_dict, gram, d_idx, d_coef);
  Prof pr(c, "omp", 1);
  ksvd::DevStats* ph = c->profiling >= 2 ? c->d_phase : nullptr;
  // The tensor-core forms need the 16-bit dictionary in shared memory (atoms
  // <= 256); beyond that, and for the FP32 form, the FP32 kernels run: the
  // resident-dictionary one when it fits, else the streamed one.
  // Before an update sweep the 16-bit kernels also write the sweep's residual
  // rows (the same buffers and arithmetic as launch_residual); patches that
  // took fewer than L atoms are listed and formed after them.
  float* resid = nullptr;
  int* last = nullptr;
  int64_t* fix = nullptr;
  unsigned long long* nfix = nullptr;
  auto fused_buffers = [&]() -> ksvd_status {
    KSVD_TRY(wsT(c, "upd_resid", size_t(N) * n, &resid));
    KSVD_TRY(wsT(c, "upd_last", size_t(N), &last));
    KSVD_TRY(wsT(c, "omp_fix_list", size_t(N), &fix));
    KSVD_TRY(wsT(c, "omp_fix_count", 1, &nfix));
    KSVD_CU(c, cudaMemsetAsync(nfix, 0, sizeof(unsigned long long), c->stream), "fix count");
    return KSVD_OK;
  };
  auto listed_rows = [&]() -> ksvd_status {  // timed with the OMP, which formed the other rows
    KSVD_CU(c,
            ksvd::launch_residual_list(d_patches, N, n, d_dict, K, L, d_idx, d_coef, resid, last, fix, nfix,
                                       c->num_sms, c->stream),
            "residual (listed patches)");
    c->resid_fused = true;
    return KSVD_OK;
  };
  if (precision != KSVD_PREC_FP32 && ksvd::omp_tc_supported(n, K, L)) {
    if (for_update) KSVD_TRY(fused_buffers());
    KSVD_CU(c,
            ksvd::launch_omp_tc(d_patches, N, n, d_dict, gram, K, L, d_idx, d_coef, c->num_sms,
                                precision == KSVD_PREC_FP16_RESCORE ? 1 : 0, c->d_flags, ph, c->stream, resid, last,
                                fix, nfix),
            "omp (tensor cores)");
    if (for_update) KSVD_TRY(listed_rows());
  } else if (precision != KSVD_PREC_FP32 && ksvd::omp_tcb_supported(n, K, L)) {
    void* scratch = nullptr;
    KSVD_TRY(ws(c, "tcb_scratch", ksvd::omp_tcb_scratch_bytes(n, K), &scratch));
    if (for_update) KSVD_TRY(fused_buffers());
    KSVD_CU(c,
            ksvd::launch_omp_tcb(d_patches, N, n, d_dict, gram, K, L, d_idx, d_coef, c->num_sms,
                                 precision == KSVD_PREC_FP16_RESCORE ? 1 : 0, scratch, c->d_flags, ph, c->stream,
                                 resid, last, fix, nfix),
            "omp (tensor cores, streamed dictionary)");
    if (for_update) KSVD_TRY(listed_rows());
  } else if (ksvd::omp_fp32_supported(n, K, L)) {
    float* resid = nullptr;
    int* last = nullptr;
    if (for_update) {  // the sweep's residual rows from the kernel's own residual tile
      KSVD_TRY(wsT(c, "upd_resid", size_t(N) * n, &resid));
      KSVD_TRY(wsT(c, "upd_last", size_t(N), &last));
    }
    KSVD_CU(c,
            ksvd::launch_omp_fp32(d_patches, N, n, d_dict, gram, K, L, d_idx, d_coef, c->num_sms, ph, c->stream,
                                  resid, last),
            "omp");
    c->resid_fused = for_update;
  } else {
    KSVD_CU(c,
            ksvd::launch_omp_stream(d_patches, N, n, d_dict, gram, K, L, d_idx, d_coef, c->num_sms, ph, c->stream),
            "omp (streamed dictionary)");
  }
  return KSVD_OK;
}

}  // namespace api
}  // namespace ksvd

static ksvd_status omp_impl(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict, int32_t* d_idx,
                            float* d_coef) {
  return omp_form(c, d_patches, N, d_dict, d_idx, d_coef, c->p.precision);
}

// The OMP of a K-SVD iteration: an update sweep on the same codes follows.
static ksvd_status omp_iter_impl(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict, int32_t* d_idx,
                                 float* d_coef) {
  return omp_form(c, d_patches, N, d_dict, d_idx, d_coef, c->p.precision, true);
}

extern "C" {

ksvd_status ksvd_omp(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict, int32_t* d_idx,
                     float* d_coef) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_dict || !d_idx || !d_coef || N < 1) return fail(c, KSVD_ERR_INVALID, "bad argument");
  KSVD_TRY(check_kernel_support(c));
  KSVD_TRY(omp_impl(c, d_patches, N, d_dict, d_idx, d_coef));
  return check_dev_flags(c, "omp");
}

}  // extern "C"

namespace ksvd {
namespace api {

ksvd_status update_prepare(ksvd_ctx* c, const float* d_patches, int64_t N, float* d_dict, const int32_t* d_idx,
                           float* d_coef, int ctas, ksvd::UpdGroup* g) {
  const int n = c->p.patch_width_dim * c->p.patch_height_dim, K = c->p.atoms, L = c->p.omp_iter;
  ksvd::CsrWork w;
  w.nchunks = ksvd::csr_num_chunks(N);
  KSVD_TRY(wsT(c, "csr_counts", size_t(w.nchunks) * K, &w.chunk_counts));
  KSVD_TRY(wsT(c, "csr_atom_ptr", size_t(2) * K + 1, &w.atom_ptr));
  KSVD_TRY(wsT(c, "csr_entries", size_t(N) * L, &w.entries));
  w.records = nullptr;  // the residual-based sweep needs only the entries
  float *resid = nullptr, *gw = nullptr;
  unsigned* sync = nullptr;
  KSVD_TRY(wsT(c, "upd_resid", size_t(N) * n, &resid));
  KSVD_TRY(wsT(c, "upd_partials", ksvd::update_res_partial_floats(n, ctas), &gw));
  KSVD_TRY(wsT(c, "upd_sync", size_t(2) * K, &sync));
  int* last = nullptr;
  KSVD_TRY(wsT(c, "upd_last", size_t(N), &last));
  {
    Prof pr(c, "csr", 4);
    KSVD_CU(c, ksvd::launch_csr_build(d_idx, d_coef, N, L, K, w, c->stream), "csr build");
  }
  if (!c->resid_fused) {
    Prof pr(c, "residual", 1);
    KSVD_CU(c,
            ksvd::launch_residual(d_patches, N, n, d_dict, K, L, d_idx, d_coef, resid, last, c->num_sms, c->stream),
            "residual");
  }
  c->resid_fused = false;
  std::memset(g, 0, sizeof(*g));
  g->R = resid;
  g->D = d_dict;
  g->coef = d_coef;
  g->atom_ptr = w.atom_ptr;
  g->entries = w.entries;
  g->last = last;
  g->gw = gw;
  g->sync = sync;
  g->n = n;
  g->K = K;
  g->L = L;
  g->q1_cap = (c->p.compat & KSVD_COMPAT_Q1_CAP) ? 1 : 0;
  g->cap = ksvd::update_res_capacity(n);
  g->ctas = ctas;
  g->slice_target = c->upd_slice;
  return KSVD_OK;
}

ksvd_status update_form(ksvd_ctx* c, const float* d_patches, int64_t N, float* d_dict, const int32_t* d_idx,
                        float* d_coef) {
  const int n = c->p.patch_width_dim * c->p.patch_height_dim;
  const int grid = ksvd::update_res_grid_size(n, c->num_sms);
  if (grid < 1) return fail(c, KSVD_ERR_CUDA, "update kernel cannot be made co-resident");
  ksvd::UpdBatch b;
  std::memset(&b, 0, sizeof(b));
  b.ngroups = 1;
  KSVD_TRY(update_prepare(c, d_patches, N, d_dict, d_idx, d_coef, grid, &b.g[0]));
  KSVD_CU(c, cudaMemsetAsync(c->d_stats, 0, sizeof(ksvd::DevStats), c->stream), "stats reset");
  Prof pr(c, "update", 1);
  KSVD_CU(c, ksvd::launch_update_batch(b, c->d_flags, c->d_stats, c->profiling >= 2 ? 1 : 0, grid, c->stream),
          "update");
  if (c->profiling) {
    // fold this sweep's phase timers into the profiling accumulator
    KSVD_CU(c, ksvd::launch_accumulate_phases(c->d_stats, c->d_phase, c->stream), "phase timers");
  }
  return KSVD_OK;
}

}  // namespace api
}  // namespace ksvd

static ksvd_status update_impl(ksvd_ctx* c, const float* d_patches, int64_t N, float* d_dict, const int32_t* d_idx,
                               float* d_coef) {
  return update_form(c, d_patches, N, d_dict, d_idx, d_coef);
}

extern "C" {

ksvd_status ksvd_update_dictionary(ksvd_ctx* c, const float* d_patches, int64_t N, float* d_dict,
                                   const int32_t* d_idx, float* d_coef) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_dict || !d_idx || !d_coef || N < 1) return fail(c, KSVD_ERR_INVALID, "bad argument");
  KSVD_TRY(check_kernel_support(c));
  KSVD_TRY(update_impl(c, d_patches, N, d_dict, d_idx, d_coef));
  return check_dev_flags(c, "updateDictionary");
}

ksvd_status ksvd_iterate(ksvd_ctx* c, const float* d_patches, int64_t N, float* d_dict, int32_t* d_idx,
                         float* d_coef, int iters) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_dict || !d_idx || !d_coef || N < 1 || iters < 0)
    return fail(c, KSVD_ERR_INVALID, "bad argument");
  KSVD_TRY(check_kernel_support(c));
  for (int i = 0; i < iters; ++i) {
    KSVD_TRY(omp_iter_impl(c, d_patches, N, d_dict, d_idx, d_coef));
    KSVD_TRY(update_impl(c, d_patches, N, d_dict, d_idx, d_coef));
  }
  return check_dev_flags(c, "kSvd");
}

ksvd_status ksvd_build_image(ksvd_ctx* c, const float* d_noisy, int width, int height, float sigma2,
                             const float* d_dict, const int32_t* d_idx, const float* d_coef, int64_t N,
                             float* d_out, double* lambda_out) {
  KSVD_TRY(check_ctx(c));
  if (!d_noisy || !d_dict || !d_idx || !d_coef || !d_out) return fail(c, KSVD_ERR_INVALID, "null pointer");
  if (!(sigma2 > 0.0f)) return fail(c, KSVD_ERR_INVALID, "sigma2 must be > 0");
  PatchGeom g;
  if (!geom_of(c->p, width, height, &g)) return fail(c, KSVD_ERR_INVALID, "patch geometry does not fit the image");
  if (N != g.N) return fail(c, KSVD_ERR_INVALID, "num_patches does not match the image geometry");
  float* acc = nullptr;
  double* partials = nullptr;
  double* lam = nullptr;
  KSVD_TRY(wsT(c, "img_acc", size_t(width) * height, &acc));
  KSVD_TRY(wsT(c, "img_partials", size_t(ksvd::col2im_num_tiles(g)), &partials));
  KSVD_TRY(wsT(c, "img_lambda", 1, &lam));
  int np = 0;
  {
    Prof pr(c, "col2im", 1);
    KSVD_CU(c,
            ksvd::launch_col2im(d_noisy, g, d_dict, c->p.atoms, c->p.omp_iter, d_idx, d_coef, acc, partials, &np,
                                c->stream),
            "col2im");
  }
  {
    Prof pr(c, "blend", 2);
    KSVD_CU(c, ksvd::launch_blend(d_noisy, g, acc, partials, np, double(sigma2), c->p.speckle, d_out, lam, c->stream),
            "blend");
  }
  if (lambda_out) {
    KSVD_CU(c, cudaMemcpyAsync(lambda_out, lam, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "lambda");
    KSVD_CU(c, cudaStreamSynchronize(c->stream), "lambda sync");
  }
  return KSVD_OK;
}

ksvd_status ksvd_codes_to_dense(ksvd_ctx* c, const int32_t* d_idx, const float* d_coef, int64_t N, float* d_dense) {
  KSVD_TRY(check_ctx(c));
  if (!d_idx || !d_coef || !d_dense || N < 1) return fail(c, KSVD_ERR_INVALID, "bad argument");
  Prof pr(c, "codes_to_dense", 1);
  KSVD_CU(c, ksvd::launch_codes_to_dense(d_idx, d_coef, N, c->p.omp_iter, c->p.atoms, d_dense, c->stream),
          "codes_to_dense");
  return KSVD_OK;
}

// ---------------------------------------------------------------------------
// Whole denoise (host buffers)
// ---------------------------------------------------------------------------
// The K-SVD pipeline on one device image y (log2 domain for speckle): patch
// gather, initial dictionary, ksvd_iter x (OMP + update), final OMP and the
// rebuild into d_out (exp2 applied for speckle).  ev[0..5] (may be null)
// bracket gather, set-up, iterations, final OMP and rebuild.
static ksvd_status denoise_image(ksvd_ctx* c, const float* y, int width, int height, float sigma2, float* d_out,
                                 double* lam, int64_t* npatch, cudaEvent_t* ev) {
  PatchGeom g;
  if (!geom_of(c->p, width, height, &g)) return fail(c, KSVD_ERR_INVALID, "patch geometry does not fit the image");
  const int n = g.n, K = c->p.atoms, L = c->p.omp_iter;
  if (g.N / 2 + K > g.N) return fail(c, KSVD_ERR_INVALID, "fewer patches than N/2 + atoms");
  float *d_patches = nullptr, *d_dict = nullptr, *d_coef = nullptr;
  int32_t* d_idx = nullptr;
  KSVD_TRY(wsT(c, "den_patches", size_t(g.N) * n, &d_patches));
  KSVD_TRY(wsT(c, "den_dict", size_t(K) * n, &d_dict));
  KSVD_TRY(wsT(c, "den_idx", size_t(g.N) * L, &d_idx));
  KSVD_TRY(wsT(c, "den_coef", size_t(g.N) * L, &d_coef));
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ev[i], c->stream);
  };
  mark(0);
  ksvd_status st = ksvd_extract_patches(c, y, width, height, d_patches);
  mark(1);
  if (st == KSVD_OK) st = ksvd_init_dictionary(c, d_patches, g.N, d_dict);
  mark(2);
  for (int i = 0; st == KSVD_OK && i < c->p.ksvd_iter; ++i) {
    st = omp_iter_impl(c, d_patches, g.N, d_dict, d_idx, d_coef);
    if (st == KSVD_OK) st = update_impl(c, d_patches, g.N, d_dict, d_idx, d_coef);
  }
  mark(3);
  if (st == KSVD_OK) st = omp_impl(c, d_patches, g.N, d_dict, d_idx, d_coef);
  mark(4);
  if (st == KSVD_OK) st = ksvd_build_image(c, y, width, height, sigma2, d_dict, d_idx, d_coef, g.N, d_out, lam);
  mark(5);
  *npatch = g.N;
  return st;
}

ksvd_status ksvd_denoise(ksvd_ctx* c, const float* img, int width, int height, float sigma2, float* out,
                         ksvd_stats* stats) {
  using clk = std::chrono::steady_clock;
  KSVD_TRY(check_ctx(c));
  if (!img || !out) return fail(c, KSVD_ERR_INVALID, "null image pointer");
  if (width < 1 || height < 1) return fail(c, KSVD_ERR_INVALID, "empty image");
  if (!(sigma2 > 0.0f)) return fail(c, KSVD_ERR_INVALID, "sigma2 must be > 0");
  KSVD_TRY(check_kernel_support(c));
  c->prop.sigma2 = sigma2;  // the learned OMP's fallback threshold
  const int tw = c->p.sub_image_width_dim, th = c->p.sub_image_height_dim;
  const bool tiled = tw != 0 || th != 0;
  if (tiled && (tw < 1 || th < 1 || th > width || tw > height))
    return fail(c, KSVD_ERR_INVALID, "sub-image dimensions do not fit the image");
  const size_t P = size_t(width) * height;
  float *d_img = nullptr, *d_y = nullptr, *d_out = nullptr;
  KSVD_TRY(wsT(c, "den_img", P, &d_img));
  KSVD_TRY(wsT(c, "den_y", P, &d_y));
  KSVD_TRY(wsT(c, "den_out", P, &d_out));
  cudaEvent_t ev[6];
  for (auto& e : ev) e = get_event(c);
  auto release = [&]() {
    for (auto e : ev) c->event_pool.push_back(e);
  };
  const auto t0 = clk::now();
  KSVD_CU(c, cudaMemcpyAsync(d_img, img, P * sizeof(float), cudaMemcpyHostToDevice, c->stream), "H2D image");
  const float* y = d_img;
  if (c->p.speckle) {
    Prof pr(c, "log2", 1);
    KSVD_CU(c, ksvd::launch_log2_image(d_img, d_y, int64_t(P), c->stream), "log2");
    y = d_y;
  }
  const auto t1 = clk::now();
  ksvd_status st = KSVD_OK;
  double lam = 0.0;
  int64_t npatch = 0;
  if (!tiled) {
    st = denoise_image(c, y, width, height, sigma2, d_out, &lam, &npatch, ev);
  } else {
    // Sub-image mode (cuda_svd_denoiser.cu:130-188, 503-528): the image is cut
    // into non-overlapping sub-images of subImageHeightDim (along x) by
    // subImageWidthDim (along y), the patch convention, at a step of their own
    // size; each is denoised on its own (own dictionary) and written back in
    // place.  Pixels outside the complete sub-images are returned as input.
    KSVD_CU(c, cudaMemcpyAsync(d_out, d_img, P * sizeof(float), cudaMemcpyDeviceToDevice, c->stream), "copy");
    float *d_tin = nullptr, *d_tout = nullptr;
    KSVD_TRY(wsT(c, "den_tile_in", size_t(tw) * th, &d_tin));
    KSVD_TRY(wsT(c, "den_tile_out", size_t(tw) * th, &d_tout));
    const int nx = (width - th) / th + 1, ny = (height - tw) / tw + 1;
    for (int i : {0, 1, 2}) cudaEventRecord(ev[i], c->stream);
    double lsum = 0.0;
    for (int ix = 0; st == KSVD_OK && ix < nx; ++ix) {
      for (int iy = 0; st == KSVD_OK && iy < ny; ++iy) {
        const size_t off = size_t(iy) * tw * width + size_t(ix) * th;
        KSVD_CU(c,
                cudaMemcpy2DAsync(d_tin, size_t(th) * 4, y + off, size_t(width) * 4, size_t(th) * 4, tw,
                                  cudaMemcpyDeviceToDevice, c->stream),
                "sub-image gather");
        double lt = 0.0;
        int64_t nt = 0;
        st = denoise_image(c, d_tin, th, tw, sigma2, d_tout, &lt, &nt, nullptr);
        if (st != KSVD_OK) break;
        KSVD_CU(c,
                cudaMemcpy2DAsync(d_out + off, size_t(width) * 4, d_tout, size_t(th) * 4, size_t(th) * 4, tw,
                                  cudaMemcpyDeviceToDevice, c->stream),
                "sub-image scatter");
        lsum += lt;
        npatch += nt;
      }
    }
    lam = lsum / double(nx * ny);
    for (int i : {3, 4, 5}) cudaEventRecord(ev[i], c->stream);
  }
  if (st == KSVD_OK) st = check_dev_flags(c, "denoise");
  const auto t2 = clk::now();
  if (st == KSVD_OK) {
    cudaError_t e = cudaMemcpyAsync(out, d_out, P * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) st = cuda_fail(c, e, "D2H image");
  }
  const auto t3 = clk::now();
  if (st == KSVD_OK && stats) {
    auto ms = [](clk::time_point a, clk::time_point b) {
      return int64_t(std::chrono::duration_cast<std::chrono::milliseconds>(b - a).count());
    };
    std::memset(stats, 0, sizeof(*stats));
    stats->init_ms = ms(t0, t1);
    stats->working_ms = ms(t1, t2);
    stats->finalize_ms = ms(t2, t3);
    stats->num_patches = npatch;
    stats->lambda = lam;
    float f = 0.0f;
    cudaEventElapsedTime(&f, ev[0], ev[1]);
    stats->extract_ms = f;
    // sub-image mode: the whole sub-image loop counts as iterations
    cudaEventElapsedTime(&f, ev[2], ev[3]);
    stats->iter_ms = f;
    cudaEventElapsedTime(&f, ev[3], ev[4]);
    stats->final_omp_ms = f;
    cudaEventElapsedTime(&f, ev[4], ev[5]);
    stats->build_ms = f;
    ksvd::DevStats ds{};
    if (cudaMemcpy(&ds, c->d_stats, sizeof(ds), cudaMemcpyDeviceToHost) == cudaSuccess) {
      stats->power_iters = int64_t(ds.power_iters);
      stats->atoms_updated = int64_t(ds.atoms_updated);
    }
  }
  release();
  return st;
}

}  // extern "C"
