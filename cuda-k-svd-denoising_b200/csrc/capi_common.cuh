// Context helpers shared by the C ABI translation units: status mapping,
// the named device workspace, per-family event timing, device error flags.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "ksvd_internal.cuh"

namespace ksvd {
namespace api {

inline ksvd_status fail(ksvd_ctx* c, ksvd_status st, const std::string& msg) {
  if (c) c->err = msg;
  return st;
}

inline ksvd_status cuda_fail(ksvd_ctx* c, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  if (e == cudaErrorMemoryAllocation) return fail(c, KSVD_ERR_NO_MEMORY, m);
  return fail(c, KSVD_ERR_CUDA, m);
}

#define KSVD_CU(ctx, expr, what)                      \
  do {                                                \
    cudaError_t e_ = (expr);                          \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
  } while (0)

#define KSVD_TRY(expr)                 \
  do {                                 \
    ksvd_status s_ = (expr);           \
    if (s_ != KSVD_OK) return s_;      \
  } while (0)

// Named device buffer that only grows.
inline ksvd_status ws(ksvd_ctx* c, const char* name, size_t bytes, void** out) {
  auto& b = c->bufs[name];
  if (bytes == 0) bytes = 16;
  if (b.bytes < bytes) {
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.ptr, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return cuda_fail(c, e, (std::string("allocating ") + name).c_str());
    }
    b.bytes = bytes;
  }
  *out = b.ptr;
  return KSVD_OK;
}

template <typename T>
inline ksvd_status wsT(ksvd_ctx* c, const char* name, size_t count, T** out) {
  void* p = nullptr;
  KSVD_TRY(ws(c, name, count * sizeof(T), &p));
  *out = static_cast<T*>(p);
  return KSVD_OK;
}

inline cudaEvent_t get_event(ksvd_ctx* c) {
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Records CUDA events around the launches of one kernel family when
// profiling is on; always counts launches.
struct Prof {
  ksvd_ctx* c;
  ksvd_ctx::Family* f = nullptr;
  cudaEvent_t e0 = nullptr;
  int kernels;
  Prof(ksvd_ctx* ctx, const char* fam, int nkernels) : c(ctx), kernels(nkernels) {
    if (c->profiling) {
      f = &c->families[fam];
      e0 = get_event(c);
      cudaEventRecord(e0, c->stream);
    }
  }
  ~Prof() {
    c->launch_count += kernels;
    if (f) {
      cudaEvent_t e1 = get_event(c);
      cudaEventRecord(e1, c->stream);
      f->pending.emplace_back(e0, e1);
      f->launches += 1;
    }
  }
};

inline ksvd_status check_ctx(ksvd_ctx* c) {
  if (!c) return KSVD_ERR_INVALID;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
  return KSVD_OK;
}

// Reads and clears the device error word (synchronises the stream).
inline ksvd_status check_dev_flags(ksvd_ctx* c, const char* where) {
  ksvd::GridBarrier h{};
  KSVD_CU(c, cudaMemcpyAsync(&h, c->d_flags, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "reading flags");
  KSVD_CU(c, cudaStreamSynchronize(c->stream), where);
  if (h.err != ksvd::DEVERR_NONE) {
    cudaMemsetAsync(c->d_flags, 0, sizeof(ksvd::GridBarrier), c->stream);
    cudaStreamSynchronize(c->stream);
    switch (h.err) {
      case ksvd::DEVERR_TIMEOUT:
        return fail(c, KSVD_ERR_TIMEOUT, std::string(where) + ": a bounded grid-barrier wait timed out");
      case ksvd::DEVERR_ZERO_ATOM:
        return fail(c, KSVD_ERR_NUMERIC, std::string(where) + ": an initial atom has zero norm");
      default:
        return fail(c, KSVD_ERR_CUDA, std::string(where) + ": device error flag set");
    }
  }
  return KSVD_OK;
}

// OMP of the given precision form and one update sweep (capi.cu), the
// learned proposal's candidates and OMP (proposal.cu).  With for_update, an
// update sweep on the same codes follows directly: the tensor-core OMP then
// also writes the sweep's residual rows (c->resid_fused).
ksvd_status omp_form(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict, int32_t* d_idx,
                     float* d_coef, int precision, bool for_update = false);
ksvd_status update_form(ksvd_ctx* c, const float* d_patches, int64_t N, float* d_dict, const int32_t* d_idx,
                        float* d_coef);
// The CSR and residual of one sweep (on the context's stream) and its group
// descriptor for launch_update_batch with `ctas` CTAs (cta_begin left 0).
// The residual is not formed again when the OMP before it wrote it
// (c->resid_fused, cleared here).
ksvd_status update_prepare(ksvd_ctx* c, const float* d_patches, int64_t N, float* d_dict, const int32_t* d_idx,
                           float* d_coef, int ctas, ksvd::UpdGroup* g);
ksvd_status proposal_candidates_impl(ksvd_ctx* c, const float* d_patches, int64_t N, int32_t* d_cand);
ksvd_status omp_learned_impl(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict, const double* gram,
                             int32_t* d_idx, float* d_coef);

}  // namespace api
}  // namespace ksvd
