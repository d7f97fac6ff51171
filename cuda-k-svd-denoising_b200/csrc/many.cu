// Many images of uneven size and patch shape through one pipeline
// (ksvd_denoise_many).  The reference denoises a config's files one after the
// other (batch_denoiser.cpp:36-118, main.cpp:56-112), each with its own
// kSvd (cuda_svd_denoiser.cu:368-408).  Here every image keeps its own
// context (dictionary, codes, workspace) and stream; per K-SVD iteration the
// images' OMP, atom lists and residuals run concurrently on a pool of
// streams, then ONE persistent cooperative launch sweeps every image's atoms.
// The launch's CTAs form lanes: a lane runs its images' sweeps one after the
// other, lanes run side by side.  The plan comes from a model of one image's
// sweep time on w CTAs (a latency floor per atom plus the local work spread
// over the CTAs, dearer when the columns overflow shared memory): small
// images, bound by the floor, share narrow lanes, while the images whose
// columns need many CTAs take a wide lane in turn.  From the second
// iteration on, the whole batch iteration (fork, per-image work, the shared
// sweep, join) is captured once as a CUDA graph and replayed.  With tuning
// on, the three best modelled plans are timed on the first iteration's
// codes and the fastest is kept.
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

// One image as the sweep planner sees it: patches, features, atoms, atoms per
// patch and the update kernel's resident columns per CTA.
struct LaneShape {
  double N;
  int n, K, L, cap;
};

// CTA lanes of the shared sweep: lane l owns CTAs [begin, begin + width) and
// runs its images one after the other; ms: its modelled time.
struct LanePlan {
  std::vector<int> begin, width;
  std::vector<std::vector<int>> imgs;
  std::vector<double> ms;
  double total_ms = 0.0;
};

// Sweep time of one image on w CTAs (ms), a model measured on B200 with the
// update kernel (one image at a time on every SM, 64 images of 8 x 8 to
// 22 x 22 patches): per atom a latency floor of 11 + 0.025 n us (the
// all-reduces and the hand-over between atoms), plus the local passes over
// the atom's columns, 8.6e-4 us per column and feature spread over the w
// CTAs, five times dearer for columns beyond a CTA's shared-memory capacity
// (streamed from memory on every power step).
double sweep_model_ms(const LaneShape& s, int w) {
  const double E = s.N * s.L / double(s.K);  // entries per atom
  const double floor_us = 11.0 + 0.025 * s.n;
  const double work_us = 8.6e-4 * s.n * s.N * s.L / double(w);
  const double streamed = std::max(0.0, 1.0 - double(s.cap) * w / E);
  return (s.K * floor_us + work_us * (1.0 + 4.0 * streamed)) * 1e-3;
}

// Longest-processing-time-first assignment of `imgs` to lanes of the given
// widths starting at CTA `begin0`; appended to `plan`, returns the longest
// lane's modelled time.
double lpt_lanes(const std::vector<LaneShape>& sh, std::vector<int> imgs, const std::vector<int>& widths, int begin0,
                 LanePlan& plan) {
  const int wmax = *std::max_element(widths.begin(), widths.end());
  std::sort(imgs.begin(), imgs.end(), [&](int x, int y) {
    const double tx = sweep_model_ms(sh[size_t(x)], wmax), ty = sweep_model_ms(sh[size_t(y)], wmax);
    return tx > ty || (tx == ty && x < y);
  });
  const size_t l0 = plan.width.size();
  int b = begin0;
  for (int w : widths) {
    plan.begin.push_back(b);
    plan.width.push_back(w);
    plan.imgs.emplace_back();
    plan.ms.push_back(0.0);
    b += w;
  }
  for (int i : imgs) {
    size_t best = l0;
    double fin = 1e300;
    for (size_t l = l0; l < plan.width.size(); ++l) {
      const double f = plan.ms[l] + sweep_model_ms(sh[size_t(i)], plan.width[l]);
      if (f < fin) {
        fin = f;
        best = l;
      }
    }
    plan.ms[best] = fin;
    plan.imgs[best].push_back(i);
  }
  double mx = 0.0;
  for (size_t l = l0; l < plan.width.size(); ++l) mx = std::max(mx, plan.ms[l]);
  return mx;
}

std::vector<int> even_widths(int total, int k) {
  std::vector<int> w(size_t(k), total / k);
  for (int r = 0; r < total % k; ++r) w[size_t(r)] += 1;
  return w;
}

// A lane that got no image hands its CTAs to the lane before it (or after
// it, for the first), so that every CTA sweeps; the lanes' times are then
// modelled again.
void absorb_empty_lanes(const std::vector<LaneShape>& sh, LanePlan& p) {
  size_t l = 0;
  while (l < p.width.size() && p.width.size() > 1) {
    if (!p.imgs[l].empty()) {
      ++l;
      continue;
    }
    if (l > 0) {
      p.width[l - 1] += p.width[l];
    } else {
      p.width[1] += p.width[0];
      p.begin[1] = p.begin[0];
    }
    p.begin.erase(p.begin.begin() + long(l));
    p.width.erase(p.width.begin() + long(l));
    p.imgs.erase(p.imgs.begin() + long(l));
    p.ms.erase(p.ms.begin() + long(l));
  }
  p.total_ms = 0.0;
  for (size_t k = 0; k < p.width.size(); ++k) {
    double t = 0.0;
    for (int i : p.imgs[k]) t += sweep_model_ms(sh[size_t(i)], p.width[k]);
    p.ms[k] = t;
    p.total_ms = std::max(p.total_ms, t);
  }
}

// Candidate lane plans for the shared sweep, best modelled first:
//  * k equal lanes, images assigned longest first;
//  * one wide lane of W CTAs running the nb images that take longest there,
//    one after the other, and k equal lanes on the remaining CTAs for the rest.
std::vector<LanePlan> lane_plans(const std::vector<LaneShape>& sh, int G) {
  const int m = int(sh.size());
  std::vector<LanePlan> out;
  std::vector<int> all(static_cast<size_t>(m));
  for (int i = 0; i < m; ++i) all[size_t(i)] = i;
  for (int k : {1, 2, 3, 4, 6, 8, 12, 16, 24, 32}) {
    if (k > m || k > G) continue;
    LanePlan p;
    p.total_ms = lpt_lanes(sh, all, even_widths(G, k), 0, p);
    out.push_back(std::move(p));
  }
  for (int W : {G / 2, (2 * G) / 3, (3 * G) / 4, (5 * G) / 6}) {
    if (W < 1 || W >= G) continue;
    std::vector<int> by_t = all;
    std::sort(by_t.begin(), by_t.end(), [&](int x, int y) {
      const double tx = sweep_model_ms(sh[size_t(x)], W), ty = sweep_model_ms(sh[size_t(y)], W);
      return tx > ty || (tx == ty && x < y);
    });
    for (int nb = 1; nb < m; ++nb) {
      for (int k : {1, 2, 4, 8, 16}) {
        if (k > G - W || k > m - nb) continue;
        LanePlan p;
        const std::vector<int> big(by_t.begin(), by_t.begin() + nb), rest(by_t.begin() + nb, by_t.end());
        const double tb = lpt_lanes(sh, big, {W}, 0, p);
        const double tr = lpt_lanes(sh, rest, even_widths(G - W, k), W, p);
        p.total_ms = std::max(tb, tr);
        out.push_back(std::move(p));
      }
    }
  }
  for (LanePlan& p : out) absorb_empty_lanes(sh, p);
  std::stable_sort(out.begin(), out.end(), [](const LanePlan& x, const LanePlan& y) { return x.total_ms < y.total_ms; });
  return out;
}

// A plan as per-image CTA ranges and the group order of the sweep (lane by
// lane, images of a lane in sequence).
void plan_ranges(const LanePlan& p, int m, std::vector<int>& begin, std::vector<int>& ctas, std::vector<int>& order) {
  begin.assign(size_t(m), 0);
  ctas.assign(size_t(m), 0);
  order.clear();
  for (size_t l = 0; l < p.width.size(); ++l)
    for (int i : p.imgs[l]) {
      begin[size_t(i)] = p.begin[l];
      ctas[size_t(i)] = p.width[l];
      order.push_back(i);
    }
}

}  // namespace

extern "C" ksvd_status ksvd_many_plan(const ksvd_image_job* jobs, int count, int num_sms, int* cta_begin, int* ctas,
                                      int* order, double* model_ms) {
  if (!jobs || count < 1 || count > ksvd::kUpdMaxGroups || num_sms < 1 || !cta_begin || !ctas || !order)
    return KSVD_ERR_INVALID;
  std::vector<LaneShape> shapes(static_cast<size_t>(count));
  for (int i = 0; i < count; ++i) {
    const ksvd_params& p = jobs[i].params;
    const int64_t N = ksvd_num_patches(&p, jobs[i].width, jobs[i].height);
    const int n = p.patch_width_dim * p.patch_height_dim;
    if (N < 1 || n < 1 || p.atoms < 1 || p.omp_iter < 1) return KSVD_ERR_INVALID;
    const int cap = ksvd::update_res_capacity(n);
    if (cap < 16) return KSVD_ERR_INVALID;
    shapes[size_t(i)] = LaneShape{double(N), n, p.atoms, p.omp_iter, cap};
  }
  const std::vector<LanePlan> plans = lane_plans(shapes, num_sms);
  std::vector<int> b, c, o;
  plan_ranges(plans[0], count, b, c, o);
  for (int i = 0; i < count; ++i) {
    cta_begin[i] = b[size_t(i)];
    ctas[i] = c[size_t(i)];
    order[i] = o[size_t(i)];
  }
  if (model_ms) *model_ms = plans[0].total_ms;
  return KSVD_OK;
}

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
  cudaEvent_t t0 = nullptr, t1 = nullptr, t2 = nullptr, t3 = nullptr, ts = nullptr, ti = nullptr, tm = nullptr,
              tw = nullptr;
  for (cudaEvent_t* e : {&t0, &t1, &t2, &t3, &ts, &ti, &tm, &tw}) {
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

  // ---- the lane plan of the shared sweep ------------------------------------
  std::vector<LaneShape> shapes(static_cast<size_t>(count));
  for (int i = 0; i < count; ++i) {
    const Job& j = J[size_t(i)];
    shapes[size_t(i)] = LaneShape{double(j.N), j.n, jobs[i].params.atoms, jobs[i].params.omp_iter,
                                  ksvd::update_res_capacity(j.n)};
  }
  const std::vector<LanePlan> plans = lane_plans(shapes, num_sms);
  size_t chosen = 0;
  std::vector<int> cbeg, ctas, order;
  plan_ranges(plans[0], count, cbeg, ctas, order);
  std::vector<ksvd::UpdGroup> groups(static_cast<size_t>(count));

  ksvd::UpdBatch batch;
  std::memset(&batch, 0, sizeof(batch));
  batch.ngroups = count;
  ksvd_ctx* c0 = J[0].c;

  // one batch iteration: fork, per image OMP + atom lists + residual, one
  // shared sweep on the main stream, join; `mid` (optional) is recorded
  // between the two
  auto iteration = [&](bool omp, cudaEvent_t mid) -> ksvd_status {
    cudaEvent_t fk = new_event();
    if (cudaEventRecord(fk, main_s) != cudaSuccess) return KSVD_ERR_CUDA;
    for (auto s : pool)
      if (cudaStreamWaitEvent(s, fk, 0) != cudaSuccess) return KSVD_ERR_CUDA;
    for (int i = 0; i < count; ++i) {
      Job& j = J[size_t(i)];
      if (omp) KSVD_TRY(omp_form(j.c, j.d_patches, j.N, j.d_dict, j.d_idx, j.d_coef, j.c->p.precision, true));
      KSVD_TRY(update_prepare(j.c, j.d_patches, j.N, j.d_dict, j.d_idx, j.d_coef, ctas[size_t(i)], &groups[size_t(i)]));
      groups[size_t(i)].cta_begin = cbeg[size_t(i)];
    }
    for (int k = 0; k < count; ++k) batch.g[k] = groups[size_t(order[size_t(k)])];  // the sweep's group order
    for (auto s : pool) {
      cudaEvent_t jn = new_event();
      if (cudaEventRecord(jn, s) != cudaSuccess || cudaStreamWaitEvent(main_s, jn, 0) != cudaSuccess)
        return KSVD_ERR_CUDA;
    }
    if (mid && cudaEventRecord(mid, main_s) != cudaSuccess) return KSVD_ERR_CUDA;
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
      // codes of the first iteration, then one timed sweep per lane plan,
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
      const size_t ntry = std::min<size_t>(plans.size(), 3);
      for (size_t pi = 0; pi < ntry; ++pi) {
        plan_ranges(plans[pi], count, cbeg, ctas, order);
        for (int rep = 0; rep < 2; ++rep) {
          for (int i = 0; i < count; ++i) {
            Job& j = J[size_t(i)];
            const size_t kd = size_t(j.c->p.atoms) * j.n, kc = size_t(j.N) * j.c->p.omp_iter;
            MANY_CU(cudaMemcpyAsync(j.d_dict, dsave[size_t(i)], kd * 4, cudaMemcpyDeviceToDevice, j.c->stream));
            MANY_CU(cudaMemcpyAsync(j.d_coef, csave[size_t(i)], kc * 4, cudaMemcpyDeviceToDevice, j.c->stream));
          }
          MANY_CU(cudaEventRecord(t2, main_s));
          MANY_TRY(iteration(false, nullptr));
          MANY_CU(cudaEventRecord(t3, main_s));
          MANY_CU(cudaStreamSynchronize(main_s));
          MANY_TRY(check_dev_flags(c0, "batch sweep"));
          float ms = 0.0f;
          cudaEventElapsedTime(&ms, t2, t3);
          if (rep == 1 && ms < best) {
            best = ms;
            chosen = pi;
          }
        }
      }
      plan_ranges(plans[chosen], count, cbeg, ctas, order);
      // the first iteration's sweep from the saved state with the chosen split
      for (int i = 0; i < count; ++i) {
        Job& j = J[size_t(i)];
        const size_t kd = size_t(j.c->p.atoms) * j.n, kc = size_t(j.N) * j.c->p.omp_iter;
        MANY_CU(cudaMemcpyAsync(j.d_dict, dsave[size_t(i)], kd * 4, cudaMemcpyDeviceToDevice, j.c->stream));
        MANY_CU(cudaMemcpyAsync(j.d_coef, csave[size_t(i)], kc * 4, cudaMemcpyDeviceToDevice, j.c->stream));
      }
      MANY_CU(cudaEventRecord(t1, main_s));  // the timed iterations start here
      MANY_TRY(iteration(true, tm));
    } else {
      MANY_TRY(iteration(true, tm));  // allocates every workspace buffer
    }
    MANY_CU(cudaEventRecord(tw, main_s));
    if (T > 1) {
      // capture one batch iteration and replay it; if the capture is refused,
      // the iterations run as plain launches
      bool captured = false;
      if (cudaStreamBeginCapture(main_s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const ksvd_status cs = iteration(true, nullptr);
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
        for (int t = 1; t < T; ++t) MANY_TRY(iteration(true, nullptr));
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
    if (T > 0) {
      cudaEventElapsedTime(&a, t1, tm);
      stats->codes_ms = a;
      cudaEventElapsedTime(&a, tm, tw);
      stats->sweep_ms = a;
    }
    stats->graph = used_graph;
    stats->streams = S;
    stats->plan_ms = plans[chosen].total_ms;
    stats->lanes = int(plans[chosen].width.size());
    for (int i = 0; i < count; ++i) {
      stats->update_ctas[i] = ctas[size_t(i)];
      stats->update_cta_begin[i] = cbeg[size_t(i)];
    }
  }
  cleanup();
  return KSVD_OK;
#undef MANY_TRY
#undef MANY_CU
}
