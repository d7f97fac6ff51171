// Learned support proposal: parameters, training loop, inference and the
// learned OMP (restricted pursuit + full-OMP fallback), behind the C ABI
// declared in include/ksvd_sm100.h.  The reference has no counterpart; the
// pursuit it narrows is CuBlasMatrixOmp::work (cublas_matrix_omp.cu:193-233).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "capi_common.cuh"
#include "ksvd_internal.cuh"

using namespace ksvd::api;

namespace {

constexpr int kH = KSVD_PROPOSAL_HIDDEN;
constexpr int kC = KSVD_PROPOSAL_CANDIDATES;

int r16(int x) { return (x + 15) / 16 * 16; }

// Offsets of the parameter blocks in the flat FP32 vector.
struct Offs {
  int64_t W1, b1, W2, b2, W3, b3, total;
};
Offs offs_of(int n, int K) {
  Offs o;
  o.W1 = 0;
  o.b1 = o.W1 + int64_t(kH) * n;
  o.W2 = o.b1 + kH;
  o.b2 = o.W2 + int64_t(kH) * kH;
  o.W3 = o.b2 + kH;
  o.b3 = o.W3 + int64_t(K) * kH;
  o.total = o.b3 + K;
  return o;
}

ksvd_status prop_shape(ksvd_ctx* c) {
  const int64_t n64 = int64_t(c->p.patch_width_dim) * c->p.patch_height_dim;
  if (n64 < 1 || n64 > 512) return fail(c, KSVD_ERR_INVALID, "proposal: patch size must be in [1, 512]");
  const int n = int(n64), K = c->p.atoms;
  if (K < kC || K > 256) return fail(c, KSVD_ERR_INVALID, "proposal: atoms must be in [16, 256]");
  auto& P = c->prop;
  P.n = n;
  P.n16 = r16(n);
  P.K = K;
  P.K16 = r16(K);
  P.H = kH;
  P.nparams = offs_of(n, K).total;
  return KSVD_OK;
}

struct Bufs {
  float *w, *m1, *m2, *g, *b3p;
  __nv_bfloat16 *w1b, *w2b, *w3b;
};

ksvd_status prop_bufs(ksvd_ctx* c, Bufs* b) {
  const auto& P = c->prop;
  KSVD_TRY(wsT(c, "prop_w", size_t(P.nparams), &b->w));
  KSVD_TRY(wsT(c, "prop_m1", size_t(P.nparams), &b->m1));
  KSVD_TRY(wsT(c, "prop_m2", size_t(P.nparams), &b->m2));
  KSVD_TRY(wsT(c, "prop_g", size_t(P.nparams), &b->g));
  KSVD_TRY(wsT(c, "prop_b3p", size_t(P.K16), &b->b3p));
  KSVD_TRY(wsT(c, "prop_w1b", size_t(kH) * P.n16, &b->w1b));
  KSVD_TRY(wsT(c, "prop_w2b", size_t(kH) * kH, &b->w2b));
  KSVD_TRY(wsT(c, "prop_w3b", size_t(P.K16) * kH, &b->w3b));
  return KSVD_OK;
}

// BF16 copies of the weights (zero-padded) and the padded last bias.
ksvd_status refresh_copies(ksvd_ctx* c, const Bufs& b) {
  const auto& P = c->prop;
  const Offs o = offs_of(P.n, P.K);
  KSVD_CU(c, ksvd::launch_mlp_to_bf16(b.w + o.W1, kH, P.n, kH, P.n16, b.w1b, c->stream), "proposal weights");
  KSVD_CU(c, ksvd::launch_mlp_to_bf16(b.w + o.W2, kH, kH, kH, kH, b.w2b, c->stream), "proposal weights");
  KSVD_CU(c, ksvd::launch_mlp_to_bf16(b.w + o.W3, P.K, kH, P.K16, kH, b.w3b, c->stream), "proposal weights");
  KSVD_CU(c, cudaMemsetAsync(b.b3p, 0, size_t(P.K16) * 4, c->stream), "proposal bias");
  KSVD_CU(c, cudaMemcpyAsync(b.b3p, b.w + o.b3, size_t(P.K) * 4, cudaMemcpyDeviceToDevice, c->stream),
          "proposal bias");
  c->launch_count += 4;
  return KSVD_OK;
}

ksvd_status reset_optimizer(ksvd_ctx* c, const Bufs& b) {
  KSVD_CU(c, cudaMemsetAsync(b.m1, 0, size_t(c->prop.nparams) * 4, c->stream), "adam state");
  KSVD_CU(c, cudaMemsetAsync(b.m2, 0, size_t(c->prop.nparams) * 4, c->stream), "adam state");
  c->prop.steps = 0;
  return KSVD_OK;
}

// Activations of one batch of B rows.
struct Acts {
  __nv_bfloat16 *X, *H1, *H2, *dZ3, *dZ2, *dZ1;
  float *Z1, *Z2, *Z3, *tmp;
};

ksvd_status acts_of(ksvd_ctx* c, int64_t B, bool train, Acts* a) {
  const auto& P = c->prop;
  std::memset(a, 0, sizeof(*a));
  KSVD_TRY(wsT(c, train ? "prop_tX" : "prop_X", size_t(B) * P.n16, &a->X));
  KSVD_TRY(wsT(c, train ? "prop_tH1" : "prop_H1", size_t(B) * kH, &a->H1));
  KSVD_TRY(wsT(c, train ? "prop_tH2" : "prop_H2", size_t(B) * kH, &a->H2));
  if (train) {
    KSVD_TRY(wsT(c, "prop_tZ1", size_t(B) * kH, &a->Z1));
    KSVD_TRY(wsT(c, "prop_tZ2", size_t(B) * kH, &a->Z2));
    KSVD_TRY(wsT(c, "prop_tZ3", size_t(B) * P.K16, &a->Z3));
    KSVD_TRY(wsT(c, "prop_tdZ3", size_t(B) * P.K16, &a->dZ3));
    KSVD_TRY(wsT(c, "prop_tdZ2", size_t(B) * kH, &a->dZ2));
    KSVD_TRY(wsT(c, "prop_tdZ1", size_t(B) * kH, &a->dZ1));
    KSVD_TRY(wsT(c, "prop_tmp", size_t(std::max(kH * P.n16, P.K16 * kH)), &a->tmp));
  }
  return KSVD_OK;
}

ksvd::GemmArgs gemm0(ksvd_ctx* c) {
  ksvd::GemmArgs g;
  std::memset(&g, 0, sizeof(g));
  g.flags = c->d_flags;
  return g;
}

// Forward pass of B rows of a.X.  train: keep the pre-activations and the
// logits (a.Z3); otherwise the top candidates go to cand (B x kC).
ksvd_status forward(ksvd_ctx* c, const Bufs& b, const Acts& a, int64_t B, bool train, int32_t* cand) {
  const auto& P = c->prop;
  const Offs o = offs_of(P.n, P.K);
  ksvd::GemmArgs g = gemm0(c);
  g.A = a.X;
  g.lda = P.n16;
  g.B = b.w1b;
  g.ldb = P.n16;
  g.M = int(B);
  g.N = kH;
  g.K = P.n16;
  g.bias = b.w + o.b1;
  g.c_f32 = train ? a.Z1 : nullptr;
  g.ldc_f32 = kH;
  g.c_bf16 = a.H1;
  g.ldc_bf16 = kH;
  KSVD_CU(c, ksvd::launch_gemm(g, true, true, ksvd::kEpiBiasGelu, c->stream), "proposal layer 1");
  g.A = a.H1;
  g.lda = kH;
  g.B = b.w2b;
  g.ldb = kH;
  g.K = kH;
  g.bias = b.w + o.b2;
  g.c_f32 = train ? a.Z2 : nullptr;
  g.c_bf16 = a.H2;
  KSVD_CU(c, ksvd::launch_gemm(g, true, true, ksvd::kEpiBiasGelu, c->stream), "proposal layer 2");
  g.A = a.H2;
  g.B = b.w3b;
  g.N = P.K16;
  g.bias = b.b3p;
  g.c_bf16 = nullptr;
  if (train) {
    g.c_f32 = a.Z3;
    g.ldc_f32 = P.K16;
    KSVD_CU(c, ksvd::launch_gemm(g, true, true, ksvd::kEpiBiasF32, c->stream), "proposal layer 3");
  } else {
    g.c_f32 = nullptr;
    g.topk = cand;
    g.ktop = kC;
    g.n_valid = P.K;
    KSVD_CU(c, ksvd::launch_gemm(g, true, true, ksvd::kEpiTopK, c->stream), "proposal layer 3");
  }
  c->launch_count += 3;
  return KSVD_OK;
}

// Loss gradient and backward pass into b.g (parameter order of Offs).
// sup/rows: the supports of the batch rows (see launch_mlp_bce).
ksvd_status backward(ksvd_ctx* c, const Bufs& b, const Acts& a, int64_t B, const int32_t* sup,
                     const int64_t* rows, double* loss_dev) {
  const auto& P = c->prop;
  const Offs o = offs_of(P.n, P.K);
  const int L = c->p.omp_iter;
  KSVD_CU(c, ksvd::launch_mlp_bce(a.Z3, B, P.K, P.K16, sup, L, rows, a.dZ3, loss_dev, c->stream), "proposal loss");
  // dW3 = dZ3^T H2 (K16 x H; rows >= K are zero)
  ksvd::GemmArgs g = gemm0(c);
  g.A = a.dZ3;
  g.lda = P.K16;
  g.B = a.H2;
  g.ldb = kH;
  g.M = P.K16;
  g.N = kH;
  g.K = int(B);
  g.c_f32 = (P.K == P.K16) ? b.g + o.W3 : a.tmp;
  g.ldc_f32 = kH;
  KSVD_CU(c, ksvd::launch_gemm(g, false, false, ksvd::kEpiF32, c->stream), "proposal dW3");
  if (P.K != P.K16)
    KSVD_CU(c, cudaMemcpyAsync(b.g + o.W3, a.tmp, size_t(P.K) * kH * 4, cudaMemcpyDeviceToDevice, c->stream),
            "proposal dW3");
  KSVD_CU(c, ksvd::launch_mlp_colsum(a.dZ3, B, P.K, P.K16, b.g + o.b3, c->stream), "proposal db3");
  // dZ2 = (dZ3 W3) * GELU'(Z2)
  g = gemm0(c);
  g.A = a.dZ3;
  g.lda = P.K16;
  g.B = b.w3b;
  g.ldb = kH;
  g.M = int(B);
  g.N = kH;
  g.K = P.K16;
  g.aux = a.Z2;
  g.ld_aux = kH;
  g.c_bf16 = a.dZ2;
  g.ldc_bf16 = kH;
  KSVD_CU(c, ksvd::launch_gemm(g, true, false, ksvd::kEpiGeluBack, c->stream), "proposal dZ2");
  // dW2 = dZ2^T H1
  g = gemm0(c);
  g.A = a.dZ2;
  g.lda = kH;
  g.B = a.H1;
  g.ldb = kH;
  g.M = kH;
  g.N = kH;
  g.K = int(B);
  g.c_f32 = b.g + o.W2;
  g.ldc_f32 = kH;
  KSVD_CU(c, ksvd::launch_gemm(g, false, false, ksvd::kEpiF32, c->stream), "proposal dW2");
  KSVD_CU(c, ksvd::launch_mlp_colsum(a.dZ2, B, kH, kH, b.g + o.b2, c->stream), "proposal db2");
  // dZ1 = (dZ2 W2) * GELU'(Z1)
  g = gemm0(c);
  g.A = a.dZ2;
  g.lda = kH;
  g.B = b.w2b;
  g.ldb = kH;
  g.M = int(B);
  g.N = kH;
  g.K = kH;
  g.aux = a.Z1;
  g.ld_aux = kH;
  g.c_bf16 = a.dZ1;
  g.ldc_bf16 = kH;
  KSVD_CU(c, ksvd::launch_gemm(g, true, false, ksvd::kEpiGeluBack, c->stream), "proposal dZ1");
  // dW1 = dZ1^T X (H x n16; columns >= n are dropped)
  g = gemm0(c);
  g.A = a.dZ1;
  g.lda = kH;
  g.B = a.X;
  g.ldb = P.n16;
  g.M = kH;
  g.N = P.n16;
  g.K = int(B);
  g.c_f32 = (P.n == P.n16) ? b.g + o.W1 : a.tmp;
  g.ldc_f32 = P.n16;
  KSVD_CU(c, ksvd::launch_gemm(g, false, false, ksvd::kEpiF32, c->stream), "proposal dW1");
  if (P.n != P.n16) KSVD_CU(c, ksvd::launch_mlp_unpad(a.tmp, kH, P.n, P.n16, b.g + o.W1, c->stream), "proposal dW1");
  KSVD_CU(c, ksvd::launch_mlp_colsum(a.dZ1, B, kH, kH, b.g + o.b1, c->stream), "proposal db1");
  c->launch_count += 11;
  return KSVD_OK;
}

ksvd_status init_weights(ksvd_ctx* c, uint64_t seed) {
  KSVD_TRY(prop_shape(c));
  Bufs b;
  KSVD_TRY(prop_bufs(c, &b));
  const auto& P = c->prop;
  const Offs o = offs_of(P.n, P.K);
  std::vector<float> h(static_cast<size_t>(P.nparams), 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int64_t off, int rows, int fan_in) {
    std::uniform_real_distribution<float> u(-1.0f / std::sqrt(float(fan_in)), 1.0f / std::sqrt(float(fan_in)));
    for (int64_t i = 0; i < int64_t(rows) * fan_in; ++i) h[size_t(off + i)] = u(rng);
  };
  fill(o.W1, kH, P.n);
  fill(o.W2, kH, kH);
  fill(o.W3, P.K, kH);
  KSVD_CU(c, cudaMemcpyAsync(b.w, h.data(), h.size() * 4, cudaMemcpyHostToDevice, c->stream), "proposal init");
  KSVD_TRY(refresh_copies(c, b));
  KSVD_TRY(reset_optimizer(c, b));
  KSVD_CU(c, cudaStreamSynchronize(c->stream), "proposal init");
  c->prop.ready = true;
  return KSVD_OK;
}

ksvd_status train_impl(ksvd_ctx* c, const float* d_patches, int64_t N, const int32_t* d_sup, int T, int epochs,
                       int batch, float lr, uint64_t seed, ksvd_proposal_stats* st) {
  if (!c->prop.ready) KSVD_TRY(init_weights(c, seed));
  Bufs b;
  KSVD_TRY(prop_bufs(c, &b));
  const int64_t P = int64_t(T) * N;
  const int64_t per_epoch = P / batch;
  if (per_epoch < 1) return fail(c, KSVD_ERR_INVALID, "proposal: fewer pairs than one batch");
  Acts a;
  KSVD_TRY(acts_of(c, batch, true, &a));
  int64_t* perm = nullptr;
  double* losses = nullptr;
  const int64_t nsteps = per_epoch * epochs;
  KSVD_TRY(wsT(c, "prop_perm", size_t(P), &perm));
  KSVD_TRY(wsT(c, "prop_losses", size_t(nsteps), &losses));
  KSVD_CU(c, cudaMemsetAsync(losses, 0, size_t(nsteps) * 8, c->stream), "proposal losses");
  std::vector<int64_t> order(static_cast<size_t>(P));
  std::mt19937_64 rng(seed ^ 0x9E3779B97F4A7C15ull);
  cudaEvent_t e0 = get_event(c), e1 = get_event(c);
  cudaEventRecord(e0, c->stream);
  const Offs o = offs_of(c->prop.n, c->prop.K);
  (void)o;
  int64_t step = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    std::iota(order.begin(), order.end(), int64_t(0));
    std::shuffle(order.begin(), order.end(), rng);
    KSVD_CU(c, cudaMemcpyAsync(perm, order.data(), order.size() * 8, cudaMemcpyHostToDevice, c->stream),
            "proposal order");
    KSVD_CU(c, cudaStreamSynchronize(c->stream), "proposal order");  // the host order is reused next epoch
    for (int64_t s = 0; s < per_epoch; ++s, ++step) {
      const int64_t* rows = perm + s * batch;
      KSVD_CU(c, ksvd::launch_mlp_input(d_patches, batch, c->prop.n, c->prop.n16, rows, N, a.X, c->stream),
              "proposal input");
      KSVD_TRY(forward(c, b, a, batch, true, nullptr));
      KSVD_TRY(backward(c, b, a, batch, d_sup, rows, losses + step));
      c->prop.steps += 1;
      KSVD_CU(c, ksvd::launch_mlp_adam(b.w, b.g, b.m1, b.m2, c->prop.nparams, lr, int(c->prop.steps), c->stream),
              "proposal adam");
      KSVD_TRY(refresh_copies(c, b));
      c->launch_count += 2;
    }
  }
  cudaEventRecord(e1, c->stream);
  KSVD_TRY(check_dev_flags(c, "proposal training"));
  std::vector<double> hl(static_cast<size_t>(nsteps));
  KSVD_CU(c, cudaMemcpy(hl.data(), losses, hl.size() * 8, cudaMemcpyDeviceToHost), "proposal losses");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  c->event_pool.push_back(e0);
  c->event_pool.push_back(e1);
  if (st) {
    const int64_t w = std::max<int64_t>(1, nsteps / 100);
    st->pairs = per_epoch * batch;
    st->steps = nsteps;
    st->first_loss = std::accumulate(hl.begin(), hl.begin() + w, 0.0) / double(w);
    st->final_loss = std::accumulate(hl.end() - w, hl.end(), 0.0) / double(w);
    st->train_ms = ms;
  }
  return KSVD_OK;
}

}  // namespace

namespace ksvd {
namespace api {

// Top candidates of N patches (d_cand: N x kC).
ksvd_status proposal_candidates_impl(ksvd_ctx* c, const float* d_patches, int64_t N, int32_t* d_cand) {
  if (!c->prop.ready) return fail(c, KSVD_ERR_INVALID, "proposal has no weights (init, set, train or fit it)");
  Bufs b;
  KSVD_TRY(prop_bufs(c, &b));
  Acts a;
  KSVD_TRY(acts_of(c, N, false, &a));
  KSVD_CU(c, ksvd::launch_mlp_input(d_patches, N, c->prop.n, c->prop.n16, nullptr, 0, a.X, c->stream),
          "proposal input");
  c->launch_count += 1;
  return forward(c, b, a, N, false, d_cand);
}

// The learned OMP: candidates, restricted pursuit, full-OMP fallback (the
// BF16 + exact re-score form) of the patches left above the threshold.
ksvd_status omp_learned_impl(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict, const double* gram,
                             int32_t* d_idx, float* d_coef) {
  const int n = c->p.patch_width_dim * c->p.patch_height_dim, K = c->p.atoms, L = c->p.omp_iter;
  if (!(c->prop.sigma2 > 0.0))
    return fail(c, KSVD_ERR_INVALID, "learned OMP: noise variance not set (ksvd_set_noise_variance)");
  int32_t* cand = nullptr;
  int64_t* fb_list = nullptr;
  unsigned long long* fb_count = nullptr;
  KSVD_TRY(wsT(c, "prop_cand", size_t(N) * kC, &cand));
  KSVD_TRY(wsT(c, "prop_fb_list", size_t(N), &fb_list));
  KSVD_TRY(wsT(c, "prop_fb_count", 1, &fb_count));
  {
    Prof pr(c, "proposal", 0);
    KSVD_TRY(proposal_candidates_impl(c, d_patches, N, cand));
  }
  const double thr = KSVD_PROPOSAL_FALLBACK * std::sqrt(c->prop.sigma2 * double(n));
  {
    Prof pr(c, "omp_restricted", 2);
    KSVD_CU(c, cudaMemsetAsync(fb_count, 0, 8, c->stream), "fallback count");
    KSVD_CU(c,
            ksvd::launch_omp_restricted(d_patches, N, n, d_dict, gram, K, L, cand, kC, thr * thr, d_idx, d_coef,
                                        fb_list, fb_count, c->num_sms, c->stream),
            "restricted omp");
  }
  unsigned long long nfb = 0;
  KSVD_CU(c, cudaMemcpyAsync(&nfb, fb_count, 8, cudaMemcpyDeviceToHost, c->stream), "fallback count");
  KSVD_CU(c, cudaStreamSynchronize(c->stream), "fallback count");
  c->prop.last_fallbacks = int64_t(nfb);
  c->prop.total_fallbacks += int64_t(nfb);
  c->prop.last_patches = N;
  if (nfb == 0) return KSVD_OK;
  const int64_t m = int64_t(nfb);
  float* fy = nullptr;
  int32_t* fi = nullptr;
  float* fc = nullptr;
  KSVD_TRY(wsT(c, "prop_fb_y", size_t(m) * n, &fy));
  KSVD_TRY(wsT(c, "prop_fb_idx", size_t(m) * L, &fi));
  KSVD_TRY(wsT(c, "prop_fb_coef", size_t(m) * L, &fc));
  Prof pr(c, "omp_fallback", 3);
  KSVD_CU(c, ksvd::launch_gather_rows(d_patches, n, fb_list, m, fy, c->stream), "fallback gather");
  if (ksvd::omp_tc_supported(n, K, L)) {
    KSVD_CU(c,
            ksvd::launch_omp_tc(fy, m, n, d_dict, gram, K, L, fi, fc, c->num_sms, 0, c->d_flags, nullptr, c->stream),
            "fallback omp");
  } else {
    KSVD_CU(c, ksvd::launch_omp_fp32(fy, m, n, d_dict, gram, K, L, fi, fc, c->num_sms, nullptr, c->stream),
            "fallback omp");
  }
  KSVD_CU(c, ksvd::launch_scatter_codes(fi, fc, L, fb_list, m, d_idx, d_coef, c->stream), "fallback scatter");
  return KSVD_OK;
}

}  // namespace api
}  // namespace ksvd

extern "C" {

int64_t ksvd_proposal_num_params(const ksvd_params* p) {
  if (!p) return -1;
  const int64_t n = int64_t(p->patch_width_dim) * p->patch_height_dim;
  if (n < 1 || n > 512 || p->atoms < 1) return -1;
  return offs_of(int(n), p->atoms).total;
}

ksvd_status ksvd_proposal_init(ksvd_ctx* c, uint64_t seed) {
  KSVD_TRY(check_ctx(c));
  return init_weights(c, seed);
}

ksvd_status ksvd_proposal_set_params(ksvd_ctx* c, const float* params, int64_t count) {
  KSVD_TRY(check_ctx(c));
  if (!params) return fail(c, KSVD_ERR_INVALID, "null parameters");
  KSVD_TRY(prop_shape(c));
  if (count != c->prop.nparams) return fail(c, KSVD_ERR_INVALID, "proposal: wrong parameter count");
  Bufs b;
  KSVD_TRY(prop_bufs(c, &b));
  KSVD_CU(c, cudaMemcpyAsync(b.w, params, size_t(count) * 4, cudaMemcpyHostToDevice, c->stream), "proposal params");
  KSVD_TRY(refresh_copies(c, b));
  KSVD_TRY(reset_optimizer(c, b));
  KSVD_CU(c, cudaStreamSynchronize(c->stream), "proposal params");
  c->prop.ready = true;
  return KSVD_OK;
}

ksvd_status ksvd_proposal_get_params(ksvd_ctx* c, float* params, int64_t count) {
  KSVD_TRY(check_ctx(c));
  if (!params) return fail(c, KSVD_ERR_INVALID, "null parameters");
  if (!c->prop.ready) return fail(c, KSVD_ERR_INVALID, "proposal has no weights");
  if (count != c->prop.nparams) return fail(c, KSVD_ERR_INVALID, "proposal: wrong parameter count");
  Bufs b;
  KSVD_TRY(prop_bufs(c, &b));
  KSVD_CU(c, cudaMemcpyAsync(params, b.w, size_t(count) * 4, cudaMemcpyDeviceToHost, c->stream), "proposal params");
  KSVD_CU(c, cudaStreamSynchronize(c->stream), "proposal params");
  return KSVD_OK;
}

ksvd_status ksvd_proposal_loss_grad(ksvd_ctx* c, const float* d_patches, int64_t B, const int32_t* d_sup,
                                    double* loss, float* d_grad) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_sup || !d_grad || B < 16 || (B % 16) != 0 || B > (int64_t(1) << 30))
    return fail(c, KSVD_ERR_INVALID, "proposal: bad batch (B a multiple of 16)");
  if (!c->prop.ready) return fail(c, KSVD_ERR_INVALID, "proposal has no weights");
  Bufs b;
  KSVD_TRY(prop_bufs(c, &b));
  Acts a;
  KSVD_TRY(acts_of(c, B, true, &a));
  double* ld = nullptr;
  KSVD_TRY(wsT(c, "prop_loss1", 1, &ld));
  KSVD_CU(c, cudaMemsetAsync(ld, 0, 8, c->stream), "proposal loss");
  KSVD_CU(c, ksvd::launch_mlp_input(d_patches, B, c->prop.n, c->prop.n16, nullptr, 0, a.X, c->stream),
          "proposal input");
  KSVD_TRY(forward(c, b, a, B, true, nullptr));
  KSVD_TRY(backward(c, b, a, B, d_sup, nullptr, ld));
  KSVD_CU(c, cudaMemcpyAsync(d_grad, b.g, size_t(c->prop.nparams) * 4, cudaMemcpyDeviceToDevice, c->stream),
          "proposal grad");
  double h = 0.0;
  KSVD_CU(c, cudaMemcpyAsync(&h, ld, 8, cudaMemcpyDeviceToHost, c->stream), "proposal loss");
  KSVD_TRY(check_dev_flags(c, "proposal gradient"));
  if (loss) *loss = h;
  return KSVD_OK;
}

ksvd_status ksvd_proposal_train(ksvd_ctx* c, const float* d_patches, int64_t N, const int32_t* d_sup, int T,
                                int epochs, int batch, float lr, uint64_t seed, ksvd_proposal_stats* st) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_sup || N < 1 || T < 1 || epochs < 1 || batch < 16 || (batch % 16) != 0 || !(lr > 0.0f))
    return fail(c, KSVD_ERR_INVALID, "proposal: bad training arguments");
  KSVD_TRY(prop_shape(c));
  if (st) std::memset(st, 0, sizeof(*st));
  return train_impl(c, d_patches, N, d_sup, T, epochs, batch, lr, seed, st);
}

ksvd_status ksvd_proposal_fit(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict, int iters,
                              int epochs, uint64_t seed, ksvd_proposal_stats* st) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_dict || N < 1 || iters < 1 || epochs < 1)
    return fail(c, KSVD_ERR_INVALID, "proposal: bad fit arguments");
  KSVD_TRY(prop_shape(c));
  if (st) std::memset(st, 0, sizeof(*st));
  const int n = c->prop.n, K = c->prop.K, L = c->p.omp_iter;
  // the plain FP32 method from a copy of the dictionary; the supports of
  // each iteration's OMP are the training targets
  float *dict = nullptr, *coef = nullptr;
  int32_t* sup = nullptr;
  KSVD_TRY(wsT(c, "prop_fit_dict", size_t(K) * n, &dict));
  KSVD_TRY(wsT(c, "prop_fit_coef", size_t(N) * L, &coef));
  KSVD_TRY(wsT(c, "prop_fit_sup", size_t(iters) * N * L, &sup));
  KSVD_CU(c, cudaMemcpyAsync(dict, d_dict, size_t(K) * n * 4, cudaMemcpyDeviceToDevice, c->stream), "fit dictionary");
  cudaEvent_t e0 = get_event(c), e1 = get_event(c);
  cudaEventRecord(e0, c->stream);
  for (int t = 0; t < iters; ++t) {
    int32_t* idx = sup + size_t(t) * N * L;
    KSVD_TRY(omp_form(c, d_patches, N, dict, idx, coef, KSVD_PREC_FP32));
    if (t + 1 < iters) KSVD_TRY(update_form(c, d_patches, N, dict, idx, coef));
  }
  cudaEventRecord(e1, c->stream);
  KSVD_TRY(check_dev_flags(c, "proposal pairs"));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  c->event_pool.push_back(e0);
  c->event_pool.push_back(e1);
  c->prop.ready = false;  // fresh weights
  KSVD_TRY(init_weights(c, seed));
  // minibatches of 4096 pairs, Adam at 1e-3
  KSVD_TRY(train_impl(c, d_patches, N, sup, iters, epochs, 4096, 1e-3f, seed, st));
  if (st) st->collect_ms = ms;
  return KSVD_OK;
}

ksvd_status ksvd_proposal_candidates(ksvd_ctx* c, const float* d_patches, int64_t N, int32_t* d_cand) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_cand || N < 1) return fail(c, KSVD_ERR_INVALID, "bad argument");
  KSVD_TRY(proposal_candidates_impl(c, d_patches, N, d_cand));
  return check_dev_flags(c, "proposal candidates");
}

ksvd_status ksvd_omp_restricted(ksvd_ctx* c, const float* d_patches, int64_t N, const float* d_dict,
                                const int32_t* d_cand, int C, int32_t* d_idx, float* d_coef, int64_t* above) {
  KSVD_TRY(check_ctx(c));
  if (!d_patches || !d_dict || !d_cand || !d_idx || !d_coef || N < 1 || C < 1 || C > kC)
    return fail(c, KSVD_ERR_INVALID, "bad argument");
  const int64_t n64 = int64_t(c->p.patch_width_dim) * c->p.patch_height_dim;
  const int K = c->p.atoms, L = c->p.omp_iter;
  if (n64 < 1 || n64 > 512 || !ksvd::omp_restricted_supported(int(n64), L, C))
    return fail(c, KSVD_ERR_INVALID, "restricted OMP: patch size or ompIter out of range");
  const int n = int(n64);
  double* gram = nullptr;
  int64_t* fb_list = nullptr;
  unsigned long long* fb_count = nullptr;
  KSVD_TRY(wsT(c, "gram", size_t(K) * K, &gram));
  KSVD_TRY(wsT(c, "prop_fb_list", size_t(N), &fb_list));
  KSVD_TRY(wsT(c, "prop_fb_count", 1, &fb_count));
  KSVD_CU(c, ksvd::launch_gram_f64(d_dict, K, n, gram, c->stream), "gram");
  const double thr = c->prop.sigma2 > 0.0 ? KSVD_PROPOSAL_FALLBACK * std::sqrt(c->prop.sigma2 * double(n)) : 0.0;
  const double thr2 = c->prop.sigma2 > 0.0 ? thr * thr : INFINITY;
  KSVD_CU(c, cudaMemsetAsync(fb_count, 0, 8, c->stream), "fallback count");
  KSVD_CU(c,
          ksvd::launch_omp_restricted(d_patches, N, n, d_dict, gram, K, L, d_cand, C, thr2, d_idx, d_coef, fb_list,
                                      fb_count, c->num_sms, c->stream),
          "restricted omp");
  c->launch_count += 2;
  unsigned long long h = 0;
  KSVD_CU(c, cudaMemcpyAsync(&h, fb_count, 8, cudaMemcpyDeviceToHost, c->stream), "fallback count");
  KSVD_TRY(check_dev_flags(c, "restricted omp"));
  if (above) *above = int64_t(h);
  return KSVD_OK;
}

ksvd_status ksvd_set_noise_variance(ksvd_ctx* c, float sigma2) {
  if (!c) return KSVD_ERR_INVALID;
  if (!(sigma2 > 0.0f)) return fail(c, KSVD_ERR_INVALID, "sigma2 must be > 0");
  c->prop.sigma2 = sigma2;
  return KSVD_OK;
}

ksvd_status ksvd_proposal_fallbacks(const ksvd_ctx* c, int64_t* last, int64_t* total, int64_t* patches) {
  if (!c) return KSVD_ERR_INVALID;
  if (last) *last = c->prop.last_fallbacks;
  if (total) *total = c->prop.total_fallbacks;
  if (patches) *patches = c->prop.last_patches;
  return KSVD_OK;
}

}  // extern "C"
