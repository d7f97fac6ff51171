/*
 * ksvd_sm100 — C ABI of the B200 (sm_100a) K-SVD denoiser.
 *
 * Drop-in boundary for the hot path of newfla/CUDA-K-SVD-Denoising's
 * denoisingLib: patch extraction, dictionary initialisation, the K-SVD
 * iteration (OMP sparse coding + sequential per-atom dictionary update) and
 * the image rebuild.  Every entry point takes plain pointers and sizes.
 *
 * Layouts (the reference's column-major matrices, src/lib/baseUtilityLib/
 * baseUtilityLib.h:16-36, stored as contiguous rows here):
 *   image    : height x width floats, row-major (pixel (x, y) at y*width + x)
 *   patches  : N x n floats, one contiguous patch per row (the reference's
 *              n x N column-major "noisePatches"), n = patchWidthDim *
 *              patchHeightDim; element r*patchWidthDim + c of patch (ix, iy)
 *              is pixel (x = ix*slidingHeight + r, y = iy*slidingWidth + c),
 *              patch index ix*ny + iy (cuda_svd_denoiser.cu:221-256)
 *   dict     : K x n floats, one unit-norm atom per row (the reference's n x K
 *              "dictionary")
 *   codes    : compact sparse code, idx N x L int32 (atom, or -1 for an unused
 *              slot) and coef N x L floats; the reference keeps the same values
 *              in a dense K x N matrix (cublas_matrix_omp.cu:79);
 *              ksvd_codes_to_dense() produces that layout.
 *
 * Pointers named d_* are device pointers on the context's device; all work
 * is ordered on the context's stream (ksvd_set_stream).  Functions without
 * d_* arguments take host memory.
 *
 * Status values 0, -1, -2, -3 keep the meaning of the reference's
 * CudaKSvdDenoiser::denoising() result (cuda_svd_denoiser.cu:86-102).
 */
#ifndef KSVD_SM100_H
#define KSVD_SM100_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KSVD_ABI_VERSION 1

/* Replaces denoising::DenoiserType (src/lib/denoisingLib/denoisingLib.h:21).
 * The three cuSOLVER-backed values are accepted and run the sm_100a path
 * (they only chose the SVD engine used in the dictionary update,
 * cuda_svd_denoiser.cu:72-84); KSVD_CUDA_K_SM100A names it explicitly. */
typedef enum ksvd_type {
  KSVD_CUDA_K_GESVD = 0,
  KSVD_CUDA_K_GESVDJ = 1,
  KSVD_CUDA_K_GESVDA = 2,
  KSVD_CUDA_K_SM100A = 3
} ksvd_type;

typedef enum ksvd_status {
  KSVD_OK = 0,
  KSVD_ERR_LOAD = -1,     /* image could not be loaded        (denoising() -1) */
  KSVD_ERR_DENOISE = -2,  /* denoising failed                 (denoising() -2) */
  KSVD_ERR_SAVE = -3,     /* image could not be saved         (denoising() -3) */
  KSVD_ERR_INVALID = -10, /* bad argument or parameter combination             */
  KSVD_ERR_CUDA = -11,    /* a CUDA call failed (see ksvd_last_error)          */
  KSVD_ERR_NO_MEMORY = -12,
  KSVD_ERR_TIMEOUT = -13, /* a bounded device wait gave up                     */
  KSVD_ERR_NUMERIC = -14, /* zero-norm initial atom or non-finite data         */
  KSVD_ERR_NO_DEVICE = -15,
  KSVD_ERR_TOO_LARGE = -16 /* beyond the fixed maximum of ksvd_omp_noalloc      */
} ksvd_status;

/* Arithmetic of the OMP correlation D^T R.  The tensor-core forms re-score
 * exactly (FP64 from the FP32 data) every atom whose tensor-core correlation
 * lies within the operand-rounding error bound of the best one, so the
 * selected atom is the exact argmax either way; FP16 (11-bit significand,
 * exact power-of-two scaling per patch) gives an 8x narrower bound than BF16
 * and therefore far fewer re-scores.
 * The tensor-core forms apply for atoms <= 256 when the tile of 128 patches
 * and the 16-bit dictionary fit in shared memory; beyond that the FP32
 * kernels run (dictionary resident in shared memory when it fits, streamed
 * through it otherwise: atoms <= 1024). */
typedef enum ksvd_precision {
  KSVD_PREC_FP32 = 0,         /* plain FP32 FMA                              */
  KSVD_PREC_BF16_RESCORE = 1, /* BF16 tensor cores + exact re-score         */
  KSVD_PREC_FP16_RESCORE = 2, /* FP16 tensor cores + exact re-score         */
  KSVD_PREC_BF16_LEARNED = 3  /* learned top-16 proposal (BF16 MLP on the
                                 tensor cores) + OMP restricted to it, exact
                                 FP64 scores; patches whose residual stays
                                 above the threshold are re-coded by the
                                 BF16 + re-score OMP (see ksvd_proposal_*)  */
} ksvd_precision;

/* Reference behaviours reproduced on request (bit flags for ksvd_params.compat). */
#define KSVD_COMPAT_INT_NORM 0x1u /* initDictionary sums squares into an int
                                     accumulator (cuda_svd_denoiser.cu:59)   */
#define KSVD_COMPAT_Q1_CAP 0x2u   /* only the first 1024 patches of an atom's
                                     support enter its update
                                     (cuda_svd_denoiser.cu:295-296,315,324)   */
#define KSVD_COMPAT_REFERENCE (KSVD_COMPAT_INT_NORM | KSVD_COMPAT_Q1_CAP)

/* Mirrors denoising::Denoiser's parameters (denoisingLib.h:44-56) and the
 * config.json globalParams keys (batch_denoiser.cpp:60-73). */
typedef struct ksvd_params {
  int patch_width_dim;      /* "patchWidthDim"     default 8  */
  int patch_height_dim;     /* "patchHeightDim"    default 8  */
  int sliding_width;        /* "slidingWidth"      default 2  */
  int sliding_height;       /* "slidingHeight"     default 2  */
  int atoms;                /* "atoms"             default 256 */
  int ksvd_iter;            /* "ksvdIter"          default 10 */
  int omp_iter;             /* "ompIter"           default 5  */
  int bw;                   /* "B&W"               default 1  */
  int speckle;              /* "speckle"           default 0  */
  int type;                 /* "type" (ksvd_type)  default KSVD_CUDA_K_SM100A */
  int min_omp_iter_batch;   /* "minOmpIterBatch"   accepted, no effect here */
  int sub_image_width_dim;  /* "subImageWidthDim"  default 0  */
  int sub_image_height_dim; /* "subImageHeightDim" default 0  */
  int precision;            /* ksvd_precision      default KSVD_PREC_FP32 */
  unsigned compat;          /* KSVD_COMPAT_*       default KSVD_COMPAT_REFERENCE */
  int device;               /* CUDA device ordinal default 0 */
} ksvd_params;

/* Timings in ms (TimeElapsed, baseUtilityLib.h:38-44) and a few counters. */
typedef struct ksvd_stats {
  int64_t init_ms;
  int64_t working_ms;
  int64_t finalize_ms;
  int64_t num_patches;
  double lambda;         /* blend weight of createImage */
  double iter_ms;        /* device time of the K-SVD iterations (OMP + update) */
  double final_omp_ms;   /* device time of the final OMP */
  double extract_ms;     /* device time of the patch gather */
  double build_ms;       /* device time of the image rebuild */
  int64_t power_iters;   /* power iterations spent in the last update sweep */
  int64_t atoms_updated; /* atoms with a non-empty support in the last sweep */
} ksvd_stats;

typedef struct ksvd_ctx ksvd_ctx;

/* Defaults of denoisingLib.h:44-56 (type/precision/compat as documented). */
void ksvd_params_default(ksvd_params* p);

/* "CUDA_K_GESVD" / "CUDA_K_GESVDJ" / "CUDA_K_GESVDA" / "CUDA_K_SM100A" ->
 * ksvd_type.  Replaces DenoiserTypeMap (denoisingLib.h:23-31); like the
 * reference's std::map::operator[], an unknown name yields 0 (CUDA_K_GESVD).
 * *known is set to 1 for a listed name, 0 otherwise (may be NULL). */
int ksvd_type_from_string(const char* name, int* known);
const char* ksvd_type_name(int type);

/* Replaces Denoiser::factory (denoiser.cpp:108-127) + the parameter copy of
 * BatchDenoiser::factory (batch_denoiser.cpp:36-118).  Validates p, selects
 * the device and creates the context's stream.  Device memory is allocated
 * on first use and kept for the life of the context. */
ksvd_status ksvd_create(const ksvd_params* p, ksvd_ctx** out);
void ksvd_destroy(ksvd_ctx* ctx);
const char* ksvd_last_error(const ksvd_ctx* ctx);
const char* ksvd_status_string(int status);
int ksvd_abi_version(void);

/* Work is ordered on this stream (cudaStream_t passed as void*; NULL means
 * the context's own stream). */
ksvd_status ksvd_set_stream(ksvd_ctx* ctx, void* stream);
void* ksvd_get_stream(const ksvd_ctx* ctx);

/* Number of patches the parameters give for a width x height image. */
int64_t ksvd_num_patches(const ksvd_params* p, int width, int height);

/* CudaKSvdDenoiser::denoising() minus file I/O (cuda_svd_denoiser.cu:90-102,
 * 126-216): host image in, host image out.  sigma2 is the noise variance (the
 * reference's Denoiser::sigma, denoiser.cpp:56).  For speckle the input is the
 * linear image; the log2/exp2 transform (denoisingLib.h:124-143) is applied
 * inside.  Sub-image tiling (subImage*Dim != 0) is honoured. */
ksvd_status ksvd_denoise(ksvd_ctx* ctx, const float* img, int width, int height, float sigma2,
                         float* out, ksvd_stats* stats);

/* ---- stage entry points (device pointers) -------------------------------- */

/* createPatches (cuda_svd_denoiser.cu:221-256). d_patches: N x n. */
ksvd_status ksvd_extract_patches(ksvd_ctx* ctx, const float* d_img, int width, int height,
                                 float* d_patches);

/* initDictionary + normalizeDictKernel (cuda_svd_denoiser.cu:52-63,261-280):
 * atoms = patches N/2 .. N/2+K-1 divided by their norm. */
ksvd_status ksvd_init_dictionary(ksvd_ctx* ctx, const float* d_patches, int64_t num_patches,
                                 float* d_dict);

/* CuBlasMatrixOmp::work (cublas_matrix_omp.cu:107-402): L = omp_iter atoms per
 * patch, argmax |D^T r| with lowest-index ties, least squares on the support,
 * stop when ||r|| < 1e-3. */
ksvd_status ksvd_omp(ksvd_ctx* ctx, const float* d_patches, int64_t num_patches, const float* d_dict,
                     int32_t* d_idx, float* d_coef);

/* updateDictionary (cuda_svd_denoiser.cu:285-362): one sequential sweep over
 * the atoms; d_dict and d_coef are updated in place. */
ksvd_status ksvd_update_dictionary(ksvd_ctx* ctx, const float* d_patches, int64_t num_patches,
                                   float* d_dict, const int32_t* d_idx, float* d_coef);

/* kSvd's loop (cuda_svd_denoiser.cu:374-397): iters x (OMP + update), without
 * the final OMP. */
ksvd_status ksvd_iterate(ksvd_ctx* ctx, const float* d_patches, int64_t num_patches, float* d_dict,
                         int32_t* d_idx, float* d_coef, int iters);

/* createImage (cuda_svd_denoiser.cu:413-498) on device: d_noisy is the
 * (log-domain for speckle) noisy image, d_out the blended image (exp2 applied
 * for speckle).  *lambda_out (host, may be NULL) receives the blend weight. */
ksvd_status ksvd_build_image(ksvd_ctx* ctx, const float* d_noisy, int width, int height, float sigma2,
                             const float* d_dict, const int32_t* d_idx, const float* d_coef,
                             int64_t num_patches, float* d_out, double* lambda_out);

/* Compact codes -> the reference's dense K x N column-major code matrix
 * (element (k, p) at p*K + k).  d_dense must hold K*N floats. */
ksvd_status ksvd_codes_to_dense(ksvd_ctx* ctx, const int32_t* d_idx, const float* d_coef,
                                int64_t num_patches, float* d_dense);

/* Profiling level.  1: every kernel family records CUDA events around its
 * launches on the context's stream, and the update's counters accumulate.
 * 2: in addition the persistent kernels time their phases on the device and
 * the tensor-core OMP counts its exact re-scores (slightly slower).  0: off. */
ksvd_status ksvd_profile_enable(ksvd_ctx* ctx, int enable);
/* Sum of launch durations (ms) and launch count of a kernel family since the
 * last reset ("im2col", "init_dict", "gram", "omp", "csr", "update", "col2im",
 * ...).  Synchronises the stream. */
ksvd_status ksvd_profile_read(ksvd_ctx* ctx, const char* family, double* total_ms, int64_t* launches);
ksvd_status ksvd_profile_reset(ksvd_ctx* ctx);
/* Total number of kernels this context launched since creation. */
int64_t ksvd_launch_count(const ksvd_ctx* ctx);
/* Wall time (ms) the first CTA of the persistent kernels spent per phase
 * while profiling at level 2 (since the last reset): update [7] slice set-up,
 * [0] wait for the previous atom, [1] column load, [2] local power pass,
 * [3] wait for the other CTAs' partials, [4] partial all-reduce and
 * normalisation, [5] coefficients and residual store; OMP [8] correlation +
 * argmax, [9] residual update (least squares included for the FP32 kernels),
 * [10] tile load/store, [11] exact re-scores, [12] Cholesky append and solve
 * (tensor-core kernel).  Synchronises the stream. */
ksvd_status ksvd_profile_phases(ksvd_ctx* ctx, double* ms_out, int count);
/* Counters accumulated while profiling: [0] power iterations, [1] atoms
 * updated (level >= 1), [2] tensor-core OMP error windows wider than its
 * candidate list, [3] tensor-core OMP exact re-scores (level 2).
 * Synchronises the stream. */
ksvd_status ksvd_profile_counters(ksvd_ctx* ctx, int64_t* out, int count);

/* OMP sparse coding (the same FP32 kernels and results as ksvd_omp) for
 * callers that cannot allocate device memory: code inside a CUDA graph being
 * captured or replayed, plugins whose host framework owns every device
 * allocation, real-time loops that must not allocate once running.  It needs
 * no context and allocates nothing: the caller passes p (patch size, atoms,
 * omp_iter are used), the patches (num_patches x n), the dictionary (atoms x
 * n) and the outputs idx / coef (num_patches x omp_iter), all on the current
 * device, and the stream (NULL = legacy default stream).  The dictionary Gram
 * lives in a 2 MiB array compiled into the library, so atoms is limited to
 * 512 (KSVD_ERR_TOO_LARGE beyond) for every patch size that ksvd_omp accepts
 * (the dictionary is streamed through shared memory when it does not fit
 * there).  Every call on a device shares that array: calls whose work
 * overlaps on the GPU (e.g. on two streams) race; serialise them.  The first
 * call on each device looks the array's address up and caches it; make it
 * before starting any stream capture.  The cached address belongs to the
 * device's primary context: do not call this again after cudaDeviceReset().
 * It has no counterpart in the reference (whose OMP allocates on every call,
 * cublas_matrix_omp.cu:79,125-165,254-255). */
ksvd_status ksvd_omp_noalloc(const ksvd_params* p, const float* d_patches, int64_t num_patches,
                             const float* d_dict, int32_t* d_idx, float* d_coef, void* stream);

/* ---- many images in one pipeline -------------------------------------------
 * ksvd_denoise_many denoises up to 64 images of any size and patch shape
 * (each with its own parameters, noise variance and dictionary) together: per
 * K-SVD iteration the images' OMP, atom lists and residuals run concurrently
 * on a pool of streams and one persistent launch sweeps the atoms of every
 * image: its CTAs form lanes that run side by side, each lane sweeping its
 * images one after the other (the plan of ksvd_many_plan).  The second and
 * later iterations replay a CUDA graph of the whole batch iteration.  With
 * tune != 0 the three best modelled lane plans are timed on the first
 * iteration's codes and the fastest is kept.  The per-image results
 * equal ksvd_denoise's for the same parameters.  Every job must have the same
 * ksvd_iter and device, no sub-images and not the learned form.  Replaces the
 * reference's file-by-file loop (batch_denoiser.cpp:36-118, main.cpp:56-112). */
typedef struct ksvd_image_job {
  ksvd_params params; /* this image's parameters */
  const float* img;   /* host, height x width (linear for speckle) */
  float* out;         /* host, height x width */
  int width, height;
  float sigma2; /* noise variance */
} ksvd_image_job;

typedef struct ksvd_many_stats {
  int64_t num_patches; /* all images */
  double iter_ms;      /* device time of the K-SVD iterations of all images */
  double total_ms;     /* device time of the whole call (uploads to downloads) */
  int graph;           /* 1: iterations 2..T replayed from a CUDA graph */
  int streams;         /* streams in the pool */
  double plan_ms;      /* modelled time of the shared sweep's lane plan */
  int update_ctas[64]; /* CTAs of each image's lane in the shared sweep */
  double setup_ms;     /* uploads, patch gathers, initial dictionaries */
  double tune_ms;      /* choosing the lane plan (0 without tuning) */
  double final_ms;     /* final OMP, rebuild and downloads */
  double codes_ms;     /* first timed iteration: every image's OMP, atom lists and residual */
  double sweep_ms;     /* first timed iteration: the shared update sweep */
  int lanes;           /* CTA lanes of the shared sweep (a lane sweeps its images in turn) */
  int update_cta_begin[64]; /* first CTA of each image's lane */
} ksvd_many_stats;

ksvd_status ksvd_denoise_many(const ksvd_image_job* jobs, int count, int device, int tune, ksvd_many_stats* stats);

/* The lane plan of ksvd_denoise_many's shared sweep without tuning, for a GPU
 * of num_sms SMs (host only, no GPU needed): per image its first CTA and CTA
 * count (images sharing a range sweep one after the other), the sweep order
 * of the images (count entries) and the plan's modelled time in ms. */
ksvd_status ksvd_many_plan(const ksvd_image_job* jobs, int count, int num_sms, int* cta_begin, int* ctas, int* order,
                           double* model_ms);

/* ---- autotuning -------------------------------------------------------------
 * The update sweep splits each atom's patches over CTAs of about `slice`
 * entries each; the best slice depends on the workload (patch size, support
 * sizes).  ksvd_autotune times one sweep with each candidate slice on the
 * caller's patches and dictionary (codes from one OMP call of the context's
 * form), keeps the fastest in the context and reports them all.  Results
 * differ between slices only in the summation order of the partial sums. */
#define KSVD_TUNE_MAX 8
typedef struct ksvd_tune_result {
  int update_slice;                /* the slice chosen */
  int candidates;                  /* number of slices timed */
  int slice[KSVD_TUNE_MAX];        /* the slices */
  double update_ms[KSVD_TUNE_MAX]; /* device time of one sweep with each */
} ksvd_tune_result;
ksvd_status ksvd_autotune(ksvd_ctx* ctx, const float* d_patches, int64_t num_patches, const float* d_dict,
                          ksvd_tune_result* out);
/* Sets the slice directly (0 = the default, 64). */
ksvd_status ksvd_set_update_slice(ksvd_ctx* ctx, int slice);

/* ---- learned support proposal --------------------------------------------
 * A small network proposes, for each patch, the KSVD_PROPOSAL_CANDIDATES atoms
 * most likely to be in its OMP support; the OMP of precision
 * KSVD_PREC_BF16_LEARNED then picks its atoms among those candidates only
 * (argmax over the candidates of the exact correlations, the reference's
 * least squares and stopping rule), and every patch whose final residual
 * norm exceeds KSVD_PROPOSAL_FALLBACK * sqrt(sigma2 * n) is re-coded by the
 * full OMP.  The reference has no counterpart: its OMP scores every atom
 * (cublas_matrix_omp.cu:193-233).
 *
 * Network: x = (y - mean) sqrt(n) / |y - mean|  ->  512 (GELU)  ->  512 (GELU)  ->  atoms
 * (sigmoid scores); BF16 weights and activations, FP32 accumulation, FP32
 * master weights trained with Adam on the binary cross-entropy between the
 * scores and the support mask.  Parameters, in this order, row-major:
 * W1 [512 x n], b1 [512], W2 [512 x 512], b2 [512], W3 [atoms x 512],
 * b3 [atoms].  The atoms' identities are those of the dictionary the
 * supports came from: a proposal is trained for one image's dictionary
 * trajectory (ksvd_proposal_fit) and used on that image. */
#define KSVD_PROPOSAL_HIDDEN 512
#define KSVD_PROPOSAL_CANDIDATES 16
#define KSVD_PROPOSAL_FALLBACK 1.15

typedef struct ksvd_proposal_stats {
  int64_t pairs;     /* (patch, support) pairs trained on per epoch */
  int64_t steps;     /* optimiser steps taken */
  double first_loss; /* mean loss of the first 1% of the steps */
  double final_loss; /* mean loss of the last 1% of the steps */
  double collect_ms; /* device time generating the pairs (fit only) */
  double train_ms;   /* device time of the training steps */
} ksvd_proposal_stats;

/* Number of network parameters for these patch and dictionary sizes. */
int64_t ksvd_proposal_num_params(const ksvd_params* p);
/* Random initial weights (uniform +-1/sqrt(fan_in), zero biases) from seed. */
ksvd_status ksvd_proposal_init(ksvd_ctx* ctx, uint64_t seed);
/* Host FP32 parameter vector in / out (count = ksvd_proposal_num_params). */
ksvd_status ksvd_proposal_set_params(ksvd_ctx* ctx, const float* params, int64_t count);
ksvd_status ksvd_proposal_get_params(ksvd_ctx* ctx, float* params, int64_t count);
/* Mean loss and its gradient (FP32, parameter order above, device buffer
 * d_grad of num_params floats) for the batch d_patches [B x n] with supports
 * d_supports [B x omp_iter] (-1 = unused slot); B a multiple of 16. */
ksvd_status ksvd_proposal_loss_grad(ksvd_ctx* ctx, const float* d_patches, int64_t B, const int32_t* d_supports,
                                    double* loss, float* d_grad);
/* Trains on the T x N pairs (patch p, supports row t * N + p of d_supports
 * [T x N x omp_iter]) for `epochs` passes in seeded random order, minibatches
 * of `batch` pairs (a multiple of 16), Adam with learning rate lr. */
ksvd_status ksvd_proposal_train(ksvd_ctx* ctx, const float* d_patches, int64_t N, const int32_t* d_supports, int T,
                                int epochs, int batch, float lr, uint64_t seed, ksvd_proposal_stats* stats);
/* Generates the pairs with the plain FP32 method, collect_iters K-SVD
 * iterations from d_dict (left unchanged), the supports of each iteration's
 * OMP, and trains on them (fresh weights from seed, epochs passes). */
ksvd_status ksvd_proposal_fit(ksvd_ctx* ctx, const float* d_patches, int64_t N, const float* d_dict,
                              int collect_iters, int epochs, uint64_t seed, ksvd_proposal_stats* stats);
/* The network's top KSVD_PROPOSAL_CANDIDATES atoms per patch, best first
 * (d_cand: N x KSVD_PROPOSAL_CANDIDATES). */
ksvd_status ksvd_proposal_candidates(ksvd_ctx* ctx, const float* d_patches, int64_t N, int32_t* d_cand);
/* OMP restricted to C candidates per patch (d_cand: N x C, C <= 16), no
 * fallback; *above (may be NULL) receives the number of patches whose
 * residual norm ends above the fallback threshold (needs the noise variance). */
ksvd_status ksvd_omp_restricted(ksvd_ctx* ctx, const float* d_patches, int64_t N, const float* d_dict,
                                const int32_t* d_cand, int C, int32_t* d_idx, float* d_coef, int64_t* above);
/* Noise variance behind the fallback threshold of the learned OMP
 * (ksvd_denoise sets it from its sigma2 argument). */
ksvd_status ksvd_set_noise_variance(ksvd_ctx* ctx, float sigma2);
/* Patches re-coded by the full OMP: in the last learned OMP call, and in all
 * calls since the context was created; *patches: patches of the last call. */
ksvd_status ksvd_proposal_fallbacks(const ksvd_ctx* ctx, int64_t* last, int64_t* total, int64_t* patches);

/* ---- config.json (batch_denoiser.cpp:36-118) ------------------------------
 * The reference's keys: inputFolder, outputFolder, files[] {name, ref, and
 * per-file overrides}, globalParams {patchWidthDim, patchHeightDim,
 * slidingWidth, slidingHeight, atoms, ksvdIter, ompIter, B&W, speckle, type,
 * minOmpIterBatch, subImageWidthDim, subImageHeightDim}; additional optional
 * keys noiseVariance, precision ("FP32" | "BF16" | "FP16") and compat. */

/* Number of files in a config.json, -1 if it cannot be read. */
int ksvd_batch_count(const char* json_path);
/* Parameters and paths of file `index` (output name <out>/<pw>_<ph>_<name>
 * as in batch_denoiser.cpp:96).  Strings are truncated to cap bytes; a
 * noise variance <= 0 means "estimate from the image". */
ksvd_status ksvd_batch_entry(const char* json_path, int index, ksvd_params* p, char* input_path,
                             char* output_path, char* ref_path, size_t cap, double* noise_variance);
/* testBatchDenoiser (src/main.cpp:56-112): denoises every file of the config
 * (PGM/PPM in, 8-bit PGM out) and, if verbose, prints the per-image report.
 * Returns the number of failed images, -1 for an unreadable config. */
int ksvd_run_batch(const char* json_path, int verbose);

#ifdef __cplusplus
}
#endif
#endif /* KSVD_SM100_H */
