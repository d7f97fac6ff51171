// Internal declarations shared by the CUDA translation units of ksvd_sm100.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "ksvd_sm100.h"

namespace ksvd {

// ---------------------------------------------------------------------------
// Device-side error codes written to the context's flag word.
// ---------------------------------------------------------------------------
enum DevErr : int {
  DEVERR_NONE = 0,
  DEVERR_TIMEOUT = 1,    // a bounded grid-barrier wait gave up
  DEVERR_ZERO_ATOM = 2,  // an initial atom had zero norm
  DEVERR_BAD_INDEX = 3,  // a code index outside [0, K)
};

// State of the software grid barrier used by the persistent cooperative
// kernels.  Reset by the host before every launch.
struct GridBarrier {
  unsigned int count;
  unsigned int gen;
  int err;
  int pad;
};

// Counters the kernels report back (device memory, reset per call).
struct DevStats {
  unsigned long long power_iters;
  unsigned long long atoms_updated;
  unsigned long long omp_rescore_misses;  // tensor-core OMP: error windows wider than the candidate list
  unsigned long long pad;                 // tensor-core OMP: exact re-scores
  // Wall time (ns) CTA 0 spends in each phase of the persistent kernels:
  // update: [7] slice set-up, [0] wait for the previous atom, [1] column
  // load, [2] local power pass, [3] wait for the other CTAs' partials,
  // [4] partial all-reduce + normalisation, [5] coefficients + residual;
  // omp: [8] correlation + argmax, [9] least squares + residual, [10] tile
  // load/store, [11] exact re-scores.
  unsigned long long phase_ns[16];
};

// ---------------------------------------------------------------------------
// Kernel launchers (each returns the launch's cudaError_t).
// ---------------------------------------------------------------------------
struct PatchGeom {
  int W, H;     // image width (x) and height (y)
  int pw, ph;   // patchWidthDim (extent along y), patchHeightDim (along x)
  int sw, sh;   // slidingWidth (step along y), slidingHeight (step along x)
  int nx, ny;   // patch positions along x (outer) and y (inner)
  int64_t N;    // nx * ny
  int n;        // pw * ph
};

bool make_geom(int W, int H, int pw, int ph, int sw, int sh, PatchGeom* g);

cudaError_t launch_im2col(const float* img, const PatchGeom& g, float* patches, cudaStream_t s);
cudaError_t launch_log2_image(const float* in, float* out, int64_t count, cudaStream_t s);
cudaError_t launch_init_dict(const float* patches, int64_t N, int n, int K, int int_norm, float* dict,
                             GridBarrier* flags, cudaStream_t s);
cudaError_t launch_gram_f64(const float* dict, int K, int n, double* gram, cudaStream_t s);
cudaError_t launch_codes_to_dense(const int32_t* idx, const float* coef, int64_t N, int L, int K,
                                  float* dense, cudaStream_t s);

// OMP (FP32 SIMT correlation).  gram: K x K doubles from launch_gram_f64.
// resid_out / last_out (optional, together): every patch's residual row with
// its final coefficients and its highest support atom with a nonzero
// coefficient, as launch_residual forms them.
size_t omp_fp32_smem_bytes(int n, int K, int L);
bool omp_fp32_supported(int n, int K, int L);
cudaError_t launch_omp_fp32(const float* patches, int64_t N, int n, const float* dict, const double* gram,
                            int K, int L, int32_t* idx, float* coef, int num_sms, DevStats* stats,
                            cudaStream_t s, float* resid_out = nullptr, int* last_out = nullptr);

// OMP (FP32 SIMT) with the dictionary streamed through shared memory in
// feature chunks: any K <= 1024 and n as long as one 4-feature chunk fits.
bool omp_stream_supported(int n, int K, int L);
cudaError_t launch_omp_stream(const float* patches, int64_t N, int n, const float* dict, const double* gram, int K,
                              int L, int32_t* idx, float* coef, int num_sms, DevStats* stats, cudaStream_t s);

// OMP with the BF16 tensor-core correlation and exact FP32/FP64 re-scoring.
size_t omp_tc_smem_bytes(int n, int K, int L);
bool omp_tc_supported(int n, int K, int L);
// resid_out (optional, N x n): the residual row y - D_S g of every patch that
// took L atoms, with its final coefficients, as launch_residual forms it;
// the others are appended to fix_list (count in *fix_count, zeroed by the
// caller) for launch_residual's list form.  last_out (with resid_out, N): the
// highest support atom with a nonzero coefficient (-1 if none).
cudaError_t launch_omp_tc(const float* patches, int64_t N, int n, const float* dict, const double* gram, int K,
                          int L, int32_t* idx, float* coef, int num_sms, int fp16, GridBarrier* flags,
                          DevStats* stats, cudaStream_t s, float* resid_out = nullptr, int* last_out = nullptr,
                          int64_t* fix_list = nullptr, unsigned long long* fix_count = nullptr);

// OMP with the 16-bit tensor-core correlation for dictionaries beyond the
// resident kernel (atoms <= 512, n <= 256): the 16-bit dictionary streams
// from `scratch` (omp_tcb_scratch_bytes, written by the launch).
bool omp_tcb_supported(int n, int K, int L);
size_t omp_tcb_scratch_bytes(int n, int K);
// resid_out, last_out, fix_list, fix_count (optional): as for launch_omp_tc.
cudaError_t launch_omp_tcb(const float* patches, int64_t N, int n, const float* dict, const double* gram, int K,
                           int L, int32_t* idx, float* coef, int num_sms, int fp16, void* scratch,
                           GridBarrier* flags, DevStats* stats, cudaStream_t s, float* resid_out = nullptr,
                           int* last_out = nullptr, int64_t* fix_list = nullptr,
                           unsigned long long* fix_count = nullptr);

// Dictionary update.
struct CsrWork {
  int* chunk_counts;   // nchunks x K
  int* atom_ptr;       // 2K + 1 (atom_ptr[0..K], then scratch)
  int* entries;        // N * L (patch * L + slot), grouped by atom, ascending patch
  int* records;        // optional (nullptr: not written): N * L records of
                       // csr_record_ints(L) ints, same order:
                       // {patch, slot, atom of slot 0..L-1 (-1 if unused), pad}
  int64_t nchunks;
};
inline int csr_record_ints(int L) { return (L + 2 + 3) / 4 * 4; }
int64_t csr_num_chunks(int64_t N);
cudaError_t launch_csr_build(const int32_t* idx, const float* coef, int64_t N, int L, int K, CsrWork w,
                             cudaStream_t s);
cudaError_t launch_accumulate_phases(const DevStats* src, DevStats* dst, cudaStream_t s);

// Dictionary update on a maintained residual (kernels_update_res.cu).
bool update_res_supported(int n);
int update_res_grid_size(int n, int num_sms);
size_t update_res_partial_floats(int n, int grid);
// last (optional, N ints): the highest atom of each patch's support, -1 if none.
cudaError_t launch_residual(const float* Y, int64_t N, int n, const float* D, int K, int L, const int32_t* idx,
                            const float* coef, float* R, int* last, int num_sms, cudaStream_t s);
// The same for the patches list[0 .. *count) only (count read on the device,
// at most N).
cudaError_t launch_residual_list(const float* Y, int64_t N, int n, const float* D, int K, int L, const int32_t* idx,
                                 const float* coef, float* R, int* last, const int64_t* list,
                                 const unsigned long long* count, int num_sms, cudaStream_t s);
// sync: 2K unsigned words (zeroed by the launch); gw: update_res_partial_floats.
// stats receives the counters always, the phase times when timers != 0.
// One problem of a (multi-problem) update sweep: its buffers (as for
// launch_update_res; gw: 2 x ctas x round4(n) floats, sync: 2K words, zeroed
// by the launch), sizes, the resident-column capacity (update_res_capacity(n)
// or less) and its CTAs [cta_begin, cta_begin + ctas) of the launch.
struct UpdGroup {
  float* R;
  float* D;
  float* coef;
  const int* atom_ptr;
  const int* entries;
  const int* last;
  float* gw;
  unsigned* sync;
  int n, K, L, q1_cap, cap, cta_begin, ctas, slice_target;
};
constexpr int kUpdMaxGroups = 64;
struct UpdBatch {
  int ngroups;
  UpdGroup g[kUpdMaxGroups];
};
int update_res_capacity(int n);
// One cooperative launch of `grid` CTAs (one per SM at most) over all groups;
// each group's CTA range lies in [0, grid); groups whose ranges share CTAs run
// one after the other on them, in table order.
cudaError_t launch_update_batch(const UpdBatch& batch, GridBarrier* flags, DevStats* stats, int timers, int grid,
                                cudaStream_t s);
// last (optional): from launch_residual; a residual row is not stored back by
// the patch's last atom.  slice_target: entries per CTA before another CTA
// joins an atom (<= 0: the default, 64).
cudaError_t launch_update_res(float* R, int n, float* D, int K, int L, float* coef, const int* atom_ptr,
                              const int* entries, int q1_cap, float* gw, unsigned* sync, GridBarrier* flags,
                              DevStats* stats, int timers, const int* last, int slice_target, int grid,
                              cudaStream_t s);

// ---------------------------------------------------------------------------
// Learned support proposal (kernels_mlp.cu, kernels_omp_restricted.cu).
// ---------------------------------------------------------------------------
enum GemmEpi : int {
  kEpiF32 = 0,       // C -> c_f32
  kEpiBiasF32 = 1,   // C + bias -> c_f32
  kEpiBiasGelu = 2,  // z = C + bias -> c_f32 (optional), GELU(z) -> c_bf16
  kEpiGeluBack = 3,  // C * GELU'(aux) -> c_bf16
  kEpiTopK = 4,      // C + bias: the ktop largest of the first n_valid columns -> topk
};
constexpr int kMaxTopK = 16;

// C[M x N] = A[M x K] . B[N x K]^T, BF16 operands, FP32 accumulation.  With a
// K-contiguous operand element (r, k) is at P[r * ld + k], otherwise at
// P[k * ld + r].  N and K multiples of 16; N <= 256 or a multiple of 256.
struct GemmArgs {
  const __nv_bfloat16* A;
  long long lda;
  const __nv_bfloat16* B;
  long long ldb;
  int M, N, K;
  const float* bias;
  float* c_f32;
  long long ldc_f32;
  __nv_bfloat16* c_bf16;
  long long ldc_bf16;
  const float* aux;
  long long ld_aux;
  int32_t* topk;
  int ktop, n_valid;
  GridBarrier* flags;
};
bool gemm_shape_ok(const GemmArgs& g, bool a_kcontig, bool b_kcontig);
cudaError_t launch_gemm(const GemmArgs& g, bool a_kcontig, bool b_kcontig, int epi, cudaStream_t s);
cudaError_t launch_mlp_input(const float* Y, int64_t B, int n, int np16, const int64_t* rows, int64_t mod,
                             __nv_bfloat16* X, cudaStream_t s);
cudaError_t launch_mlp_bce(const float* Z, int64_t B, int K, int K16, const int32_t* sup, int L, const int64_t* rows,
                           __nv_bfloat16* dZ, double* loss_sum, cudaStream_t s);
cudaError_t launch_mlp_colsum(const __nv_bfloat16* G, int64_t B, int C, int ld, float* out, cudaStream_t s);
cudaError_t launch_mlp_adam(float* w, const float* grad, float* m1, float* m2, int64_t count, float lr, int step,
                            cudaStream_t s);
cudaError_t launch_mlp_to_bf16(const float* w, int rows, int cols, int rows_pad, int ld, __nv_bfloat16* out,
                               cudaStream_t s);
cudaError_t launch_mlp_unpad(const float* src, int rows, int cols, int ld, float* dst, cudaStream_t s);

// OMP restricted to C candidate atoms per patch (exact FP64 correlations of
// the candidates); patches whose residual norm ends above sqrt(thr2) are
// appended to fb_list (fb_count counts them).
cudaError_t launch_omp_restricted(const float* patches, int64_t N, int n, const float* dict, const double* gram,
                                  int K, int L, const int32_t* cand, int C, double thr2, int32_t* idx, float* coef,
                                  int64_t* fb_list, unsigned long long* fb_count, int num_sms, cudaStream_t s);
bool omp_restricted_supported(int n, int L, int C);
// Gather rows list[0..count) of src (row width w floats) into dst; scatter the
// codes of the gathered rows back into the N x L idx / coef.
cudaError_t launch_gather_rows(const float* src, int w, const int64_t* list, int64_t count, float* dst,
                               cudaStream_t s);
cudaError_t launch_scatter_codes(const int32_t* sidx, const float* scoef, int L, const int64_t* list, int64_t count,
                                 int32_t* idx, float* coef, cudaStream_t s);

// Image rebuild.
cudaError_t launch_col2im(const float* noisy, const PatchGeom& g, const float* dict, int K, int L,
                          const int32_t* idx, const float* coef, float* acc, double* partials,
                          int* num_partials, cudaStream_t s);
int col2im_num_tiles(const PatchGeom& g);
cudaError_t launch_blend(const float* noisy, const PatchGeom& g, const float* acc, const double* partials,
                         int num_partials, double sigma2, int speckle, float* out, double* lambda_dev,
                         cudaStream_t s);

}  // namespace ksvd

// ---------------------------------------------------------------------------
// The context behind the opaque ksvd_ctx handle.
// ---------------------------------------------------------------------------
struct ksvd_ctx {
  ksvd_params p{};
  int device = 0;
  int num_sms = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;

  // Named device buffers, grown on demand and kept until ksvd_destroy.
  struct Buf {
    void* ptr = nullptr;
    size_t bytes = 0;
  };
  std::map<std::string, Buf> bufs;

  // Per-kernel-family device timing.
  struct Family {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
    double total_ms = 0.0;
    int64_t launches = 0;
  };
  int profiling = 0;  // 0 off, 1 per-family event timing, 2 + in-kernel phase timers
  std::map<std::string, Family> families;
  std::vector<cudaEvent_t> event_pool;
  int64_t launch_count = 0;
  int upd_slice = 0;  // entries per CTA of the update sweep (0: the kernel's default; ksvd_autotune)
  // the last OMP (of a K-SVD iteration) already wrote the update's residual
  // rows and last-atom table; the next update_prepare skips launch_residual
  bool resid_fused = false;

  // Learned support proposal (proposal.cu): shapes, state and the noise
  // variance behind the fallback threshold; its device buffers are named
  // workspace buffers ("prop_*").
  struct Proposal {
    bool ready = false;  // weights present (initialised, set or trained)
    int n = 0, n16 = 0, K = 0, K16 = 0, H = 0;
    int64_t nparams = 0;
    int64_t steps = 0;    // Adam steps taken
    double sigma2 = 0.0;  // noise variance (<= 0: not set)
    int64_t last_fallbacks = 0, total_fallbacks = 0, last_patches = 0;
  } prop;

  ksvd::GridBarrier* d_flags = nullptr;  // error flag word + barrier
  ksvd::DevStats* d_stats = nullptr;      // per-call counters
  ksvd::DevStats* d_phase = nullptr;      // phase timers, accumulated while profiling
};
