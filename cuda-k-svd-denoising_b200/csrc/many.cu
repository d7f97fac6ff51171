// Many images of uneven size and patch shape through one pipeline
// (ksvd_denoise_many).  The reference denoises a config's files one after the
// other (batch_denoiser.cpp:36-118, main.cpp:56-112), each with its own
// kSvd (cuda_svd_denoiser.cu:368-408).  Here every image keeps its own
// context (dictionary, codes, workspace) and stream; per K-SVD iteration the
// images' OMP, atom lists and residuals run concurrently on a pool of
// streams, then ONE persistent cooperative launch sweeps every image's atoms
// at once, the SMs split between the images in proportion to their sweep
// work (one CTA group per image, groups never wait on one another).  From
// the second iteration on, the whole batch iteration (fork, per-image work,
// the shared sweep, join) is captured once as a CUDA graph and replayed.
// With tuning on, the split of the SMs is chosen by timing one sweep for
// each candidate weighting on the first iteration's codes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "capi_common.cuh"
#include "ksvd_internal.cuh"

using namespace ksvd::api;

namespace {

struct Job {
  ksvd_ctx* c = nullptr;
  int64_t N = 0;
  int n = 0;
  float *d_img = nullptr, *d_y = nullptr, *d_patches = nullptr, *d_dict = nullptr, *d_coef = nullptr;
  float* d_out = nullptr;
  int32_t* d_idx = nullptr;
};

// CTAs per job: weights w_i^alpha with w_i the bytes one sweep moves
// (N L (4n + 8)), at least one CTA each, largest remainders, summing to G.
std::vector<int> split_ctas(const std::vector<double>& w, double alpha, int G) {
  const int m = int(w.size());
  std::vector<double> v(m);
  double tot = 0.0;
  for (int i = 0; i < m; ++i) tot += (v[i] = std::pow(w[i], alpha));
  std::vector<int> c(m, 1);
  int left = G - m;
  std::vector<std::pair<double, int>> rem;
  int used = 0;
  for (int i = 0; i < m; ++i) {
    const double share = double(left) * v[i] / tot;
    const int f = int(share);
    c[i] += f;
    used += f;
    rem.emplace_back(share - f, i);
  }
  std::sort(rem.begin(), rem.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
  for (int k = 0; k < left - used; ++k) c[rem[size_t(k) % rem.size()].second] += 1;
  return c;
}

}  // namespace

extern "C" ksvd_status ksvd_denoise_many(const ksvd_image_job* jobs, int count, int device, int tune,
                                         ksvd_many_stats* stats) {
  if (!jobs || count < 1 || count > ksvd::kUpdMaxGroups) return KSVD_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return KSVD_ERR_NO_DEVICE;
  }
  int num_sms = 0;
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
  if (count > num_sms) return KSVD_ERR_INVALID;
  const int T = jobs[0].params.ksvd_iter;
  for (int i = 0; i < count; ++i) {
    const ksvd_image_job& j = jobs[i];
    if (!j.img || !j.out || j.width < 1 || j.height < 1 || !(j.sigma2 > 0.0f)) return KSVD_ERR_INVALID;
    if (j.params.ksvd_iter != T || j.params.device != device) return KSVD_ERR_INVALID;
    if (j.params.sub_image_width_dim != 0 || j.params.sub_image_height_dim != 0) return KSVD_ERR_INVALID;
    if (j.params.precision == KSVD_PREC_BF16_LEARNED) return KSVD_ERR_INVALID;  // needs a host sync per OMP
  }
  std::vector<Job> J(static_cast<size_t>(count));
  const int S = std::min(count, 16);
  std::vector<cudaStream_t> pool(static_cast<size_t>(S), nullptr);
  cudaStream_t main_s = nullptr;
  std::vector<cudaEvent_t> evs;
  auto new_event = [&]() {
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    evs.push_back(e);
    return e;
  };
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  ksvd_status st = KSVD_OK;
  auto cleanup = [&]() {
    if (main_s) cudaStreamSynchronize(main_s);
    for (auto s : pool)
      if (s) cudaStreamSynchronize(s);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    for (auto e : evs) cudaEventDestroy(e);
    for (auto& j : J)
      if (j.c) ksvd_destroy(j.c);
    for (auto s : pool)
      if (s) cudaStreamDestroy(s);
    if (main_s) cudaStreamDestroy(main_s);
  };
#define MANY_TRY(expr)          \
  do {                          \
    st = (expr);                \
    if (st != KSVD_OK) {        \
      cleanup();                \
      return st;                \
    }                           \
  } while (0)
#define MANY_CU(expr)                      \
  do {                                     \
    if ((expr) != cudaSuccess) {           \
      cudaGetLastError();                  \
      cleanup();                           \
      return KSVD_ERR_CUDA;                \
    }                                      \
  } while (0)

  MANY_CU(cudaStreamCreateWithFlags(&main_s, cudaStreamNonBlocking));
  for (auto& s : pool) MANY_CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  cudaEvent_t t0 = nullptr, t1 = nullptr, t2 = nullptr, t3 = nullptr, ts = nullptr, ti = nullptr;
  for (cudaEvent_t* e : {&t0, &t1, &t2, &t3, &ts, &ti}) {
    MANY_CU(cudaEventCreate(e));
    evs.push_back(*e);
  }
  MANY_CU(cudaEventRecord(t0, main_s));
  cudaEvent_t fork0 = new_event();
  MANY_CU(cudaEventRecord(fork0, main_s));

  // ---- per image: context, upload, patches, initial dictionary -------------
  int64_t total_patches = 0;
  for (int i = 0; i < count; ++i) {
    Job& j = J[size_t(i)];
    const ksvd_image_job& jb = jobs[i];
    MANY_TRY(ksvd_create(&jb.params, &j.c));
    ksvd_ctx* c = j.c;
    c->stream = pool[size_t(i % S)];
    c->prop.sigma2 = jb.sigma2;
    MANY_CU(cudaStreamWaitEvent(c->stream, fork0, 0));
    const int64_t P = int64_t(jb.width) * jb.height;
    const int64_t N = ksvd_num_patches(&jb.params, jb.width, jb.height);
    const int64_t n64 = int64_t(jb.params.patch_width_dim) * jb.params.patch_height_dim;
    if (N < 1 || n64 < 1 || n64 > 512 || N / 2 + jb.params.atoms > N) {
      cleanup();
      return KSVD_ERR_INVALID;
    }
    j.N = N;
    j.n = int(n64);
    total_patches += N;
    const int K = jb.params.atoms, L = jb.params.omp_iter;
    MANY_TRY(wsT(c, "many_img", size_t(P), &j.d_img));
    MANY_TRY(wsT(c, "many_y", size_t(P), &j.d_y));
    MANY_TRY(wsT(c, "many_out", size_t(P), &j.d_out));
    MANY_TRY(wsT(c, "many_patches", size_t(N) * j.n, &j.d_patches));
    MANY_TRY(wsT(c, "many_dict", size_t(K) * j.n, &j.d_dict));
    MANY_TRY(wsT(c, "many_idx", size_t(N) * L, &j.d_idx));
    MANY_TRY(wsT(c, "many_coef", size_t(N) * L, &j.d_coef));
    MANY_CU(cudaMemcpyAsync(j.d_img, jb.img, size_t(P) * 4, cudaMemcpyHostToDevice, c->stream));
    const float* y = j.d_img;
    if (jb.params.speckle) {
      MANY_CU(ksvd::launch_log2_image(j.d_img, j.d_y, P, c->stream));
      y = j.d_y;
    }
    MANY_TRY(ksvd_extract_patches(c, y, jb.width, jb.height, j.d_patches));
  }
  for (int i = 0; i < count; ++i) {
    Job& j = J[size_t(i)];
    MANY_TRY(ksvd_init_dictionary(j.c, j.d_patches, j.N, j.d_dict));  // synchronises the image's stream
  }

  // ---- the SM split of the shared sweep --------------------------------------
  std::vector<double> w(static_cast<size_t>(count));
  for (int i = 0; i < count; ++i)
    w[size_t(i)] = double(J[size_t(i)].N) * jobs[i].params.omp_iter * (4.0 * J[size_t(i)].n + 8.0);
  double alpha = 1.0;
  std::vector<int> ctas = split_ctas(w, alpha, num_sms);

  ksvd::UpdBatch batch;
  std::memset(&batch, 0, sizeof(batch));
  batch.ngroups = count;
  ksvd_ctx* c0 = J[0].c;

  // one batch iteration: fork, per image OMP + atom lists + residual, one
  // shared sweep on the main stream, join
  auto iteration = [&](bool omp) -> ksvd_status {
    cudaEvent_t fk = new_event();
    if (cudaEventRecord(fk, main_s) != cudaSuccess) return KSVD_ERR_CUDA;
    for (auto s : pool)
      if (cudaStreamWaitEvent(s, fk, 0) != cudaSuccess) return KSVD_ERR_CUDA;
    int begin = 0;
    for (int i = 0; i < count; ++i) {
      Job& j = J[size_t(i)];
      if (omp) KSVD_TRY(omp_form(j.c, j.d_patches, j.N, j.d_dict, j.d_idx, j.d_coef, j.c->p.precision));
      KSVD_TRY(update_prepare(j.c, j.d_patches, j.N, j.d_dict, j.d_idx, j.d_coef, ctas[size_t(i)], &batch.g[i]));
      batch.g[i].cta_begin = begin;
      begin += ctas[size_t(i)];
    }
    for (auto s : pool) {
      cudaEvent_t jn = new_event();
      if (cudaEventRecord(jn, s) != cudaSuccess || cudaStreamWaitEvent(main_s, jn, 0) != cudaSuccess)
        return KSVD_ERR_CUDA;
    }
    if (ksvd::launch_update_batch(batch, c0->d_flags, c0->d_stats, 0, num_sms, main_s) != cudaSuccess) {
      cudaGetLastError();
      return KSVD_ERR_CUDA;
    }
    // the pool streams are joined into the main stream here; whatever runs
    // on them next starts with a fork from the main stream
    return KSVD_OK;
  };

  MANY_CU(cudaEventRecord(ts, main_s));  // set-up done (the init calls synchronised every image's stream)
  MANY_CU(cudaEventRecord(t1, main_s));
  int used_graph = 0;
  if (T > 0) {
    if (tune) {
      // codes of the first iteration, then one timed sweep per weighting,
      // each from saved copies of the dictionaries and coefficients
      std::vector<float*> dsave(static_cast<size_t>(count)), csave(static_cast<size_t>(count));
      for (int i = 0; i < count; ++i) {
        Job& j = J[size_t(i)];
        const size_t kd = size_t(j.c->p.atoms) * j.n, kc = size_t(j.N) * j.c->p.omp_iter;
        MANY_TRY(wsT(j.c, "many_dsave", kd, &dsave[size_t(i)]));
        MANY_TRY(wsT(j.c, "many_csave", kc, &csave[size_t(i)]));
        MANY_TRY(omp_form(j.c, j.d_patches, j.N, j.d_dict, j.d_idx, j.d_coef, j.c->p.precision));
        MANY_CU(cudaMemcpyAsync(dsave[size_t(i)], j.d_dict, kd * 4, cudaMemcpyDeviceToDevice, j.c->stream));
        MANY_CU(cudaMemcpyAsync(csave[size_t(i)], j.d_coef, kc * 4, cudaMemcpyDeviceToDevice, j.c->stream));
      }
      double best = 1e300;
      double best_alpha = 1.0;
      for (double a : {0.5, 0.75, 1.0}) {
        ctas = split_ctas(w, a, num_sms);
        for (int rep = 0; rep < 2; ++rep) {
          for (int i = 0; i < count; ++i) {
            Job& j = J[size_t(i)];
            const size_t kd = size_t(j.c->p.atoms) * j.n, kc = size_t(j.N) * j.c->p.omp_iter;
            MANY_CU(cudaMemcpyAsync(j.d_dict, dsave[size_t(i)], kd * 4, cudaMemcpyDeviceToDevice, j.c->stream));
            MANY_CU(cudaMemcpyAsync(j.d_coef, csave[size_t(i)], kc * 4, cudaMemcpyDeviceToDevice, j.c->stream));
          }
          MANY_CU(cudaEventRecord(t2, main_s));
          MANY_TRY(iteration(false));
          MANY_CU(cudaEventRecord(t3, main_s));
          MANY_CU(cudaStreamSynchronize(main_s));
          MANY_TRY(check_dev_flags(c0, "batch sweep"));
          float ms = 0.0f;
          cudaEventElapsedTime(&ms, t2, t3);
          if (rep == 1 && ms < best) {
            best = ms;
            best_alpha = a;
          }
        }
      }
      alpha = best_alpha;
      ctas = split_ctas(w, alpha, num_sms);
      // the first iteration's sweep from the saved state with the chosen split
      for (int i = 0; i < count; ++i) {
        Job& j = J[size_t(i)];
        const size_t kd = size_t(j.c->p.atoms) * j.n, kc = size_t(j.N) * j.c->p.omp_iter;
        MANY_CU(cudaMemcpyAsync(j.d_dict, dsave[size_t(i)], kd * 4, cudaMemcpyDeviceToDevice, j.c->stream));
        MANY_CU(cudaMemcpyAsync(j.d_coef, csave[size_t(i)], kc * 4, cudaMemcpyDeviceToDevice, j.c->stream));
      }
      MANY_CU(cudaEventRecord(t1, main_s));  // the timed iterations start here
      MANY_TRY(iteration(true));
    } else {
      MANY_TRY(iteration(true));  // allocates every workspace buffer
    }
    if (T > 1) {
      // capture one batch iteration and replay it; if the capture is refused,
      // the iterations run as plain launches
      bool captured = false;
      if (cudaStreamBeginCapture(main_s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const ksvd_status cs = iteration(true);
        const cudaError_t ce = cudaStreamEndCapture(main_s, &graph);
        if (cs == KSVD_OK && ce == cudaSuccess && graph &&
            cudaGraphInstantiate(&gexec, graph, 0) == cudaSuccess)
          captured = true;
        cudaGetLastError();
      } else {
        cudaGetLastError();
      }
      if (captured) {
        used_graph = 1;
        for (int t = 1; t < T; ++t) MANY_CU(cudaGraphLaunch(gexec, main_s));
      } else {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr;
        graph = nullptr;
        for (int t = 1; t < T; ++t) MANY_TRY(iteration(true));
      }
    }
  }
  MANY_CU(cudaEventRecord(t2, main_s));
  MANY_CU(cudaEventRecord(ti, main_s));
  // ---- final OMP and the rebuild, per image ----------------------------------
  cudaEvent_t fk = new_event();
  MANY_CU(cudaEventRecord(fk, main_s));
  for (auto s : pool) MANY_CU(cudaStreamWaitEvent(s, fk, 0));
  for (int i = 0; i < count; ++i) {
    Job& j = J[size_t(i)];
    const ksvd_image_job& jb = jobs[i];
    MANY_TRY(omp_form(j.c, j.d_patches, j.N, j.d_dict, j.d_idx, j.d_coef, j.c->p.precision));
    const float* y = jb.params.speckle ? j.d_y : j.d_img;
    MANY_TRY(ksvd_build_image(j.c, y, jb.width, jb.height, jb.sigma2, j.d_dict, j.d_idx, j.d_coef, j.N, j.d_out,
                              nullptr));
    MANY_CU(cudaMemcpyAsync(jb.out, j.d_out, size_t(jb.width) * jb.height * 4, cudaMemcpyDeviceToHost,
                            j.c->stream));
  }
  for (auto s : pool) {
    cudaEvent_t jn = new_event();
    MANY_CU(cudaEventRecord(jn, s));
    MANY_CU(cudaStreamWaitEvent(main_s, jn, 0));
  }
  MANY_CU(cudaEventRecord(t3, main_s));
  MANY_CU(cudaStreamSynchronize(main_s));
  for (int i = 0; i < count; ++i) MANY_TRY(check_dev_flags(J[size_t(i)].c, "batch denoise"));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    float a = 0.0f, b = 0.0f;
    cudaEventElapsedTime(&a, t1, t2);
    cudaEventElapsedTime(&b, t0, t3);
    stats->num_patches = total_patches;
    stats->iter_ms = a;
    stats->total_ms = b;
    cudaEventElapsedTime(&a, t0, ts);
    stats->setup_ms = a;
    cudaEventElapsedTime(&a, ts, t1);
    stats->tune_ms = a;
    cudaEventElapsedTime(&a, ti, t3);
    stats->final_ms = a;
    stats->graph = used_graph;
    stats->streams = S;
    stats->split_alpha = alpha;
    for (int i = 0; i < count; ++i) stats->update_ctas[i] = ctas[size_t(i)];
  }
  cleanup();
  return KSVD_OK;
#undef MANY_TRY
#undef MANY_CU
}
