// Patch-side kernels: im2col gather, speckle log transform, dictionary
// initialisation, the FP64 dictionary Gram, codes -> dense adapter.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "ksvd_internal.cuh"

namespace ksvd {

bool make_geom(int W, int H, int pw, int ph, int sw, int sh, PatchGeom* g) {
  if (W <= 0 || H <= 0 || pw <= 0 || ph <= 0 || sw <= 0 || sh <= 0) return false;
  if (ph > W || pw > H) return false;
  if (int64_t(pw) * ph > (int64_t(1) << 20)) return false;  // the patch area must fit an int comfortably
  g->W = W;
  g->H = H;
  g->pw = pw;
  g->ph = ph;
  g->sw = sw;
  g->sh = sh;
  g->nx = (W - ph) / sh + 1;
  g->ny = (H - pw) / sw + 1;
  g->N = int64_t(g->nx) * g->ny;
  g->n = pw * ph;
  return true;
}

// ---------------------------------------------------------------------------
// im2col (createPatches, cuda_svd_denoiser.cu:221-256).
// One CTA per (ix, run of kIm2colRun patches along y).  The CTA stages the
// image band x in [x0, x0+ph) x y in [y_begin, y_end) transposed in shared
// memory (band[r][y]), so that each patch column (fixed r, consecutive c) is
// a contiguous run; the run's patches are one contiguous output range that
// is written with coalesced 16-byte stores.
// ---------------------------------------------------------------------------
constexpr int kIm2colRun = 64;

__global__ void __launch_bounds__(256) im2col_kernel(const float* __restrict__ img, PatchGeom g,
                                                     float* __restrict__ out) {
  extern __shared__ float band[];
  const int ix = blockIdx.y;
  const int iy0 = blockIdx.x * kIm2colRun;
  const int iy1 = min(g.ny, iy0 + kIm2colRun);
  const int y_begin = iy0 * g.sw;
  const int rows = (iy1 - 1) * g.sw + g.pw - y_begin;
  const int x0 = ix * g.sh;
  for (int t = threadIdx.x; t < rows * g.ph; t += blockDim.x) {
    int y = t / g.ph, r = t - y * g.ph;
    band[r * rows + y] = __ldg(img + size_t(y_begin + y) * g.W + (x0 + r));
  }
  __syncthreads();
  const size_t base = (size_t(ix) * g.ny + iy0) * g.n;
  const int total = (iy1 - iy0) * g.n;
  if ((g.n & 3) == 0) {
    float4* out4 = reinterpret_cast<float4*>(out + base);
    for (int t4 = threadIdx.x; t4 < (total >> 2); t4 += blockDim.x) {
      float v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        int t = t4 * 4 + u;
        int q = t / g.n, e = t - q * g.n;
        int r = e / g.pw, c = e - r * g.pw;
        v[u] = band[r * rows + q * g.sw + c];
      }
      out4[t4] = make_float4(v[0], v[1], v[2], v[3]);
    }
  } else {
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
      int q = t / g.n, e = t - q * g.n;
      int r = e / g.pw, c = e - r * g.pw;
      out[base + t] = band[r * rows + q * g.sw + c];
    }
  }
}

cudaError_t launch_im2col(const float* img, const PatchGeom& g, float* patches, cudaStream_t s) {
  int rows = (kIm2colRun - 1) * g.sw + g.pw;
  size_t smem = size_t(rows) * g.ph * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(im2col_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
  }
  dim3 grid((g.ny + kIm2colRun - 1) / kIm2colRun, g.nx);
  im2col_kernel<<<grid, 256, smem, s>>>(img, g, patches);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// myLog (denoisingLib.h:124-133) applied to the image for speckle mode.
// ---------------------------------------------------------------------------
__global__ void log2_kernel(const float* __restrict__ in, float* __restrict__ out, int64_t count) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x) {
    float x = in[i];
    out[i] = (x == 0.0f) ? 0.0f : log2f(x);
  }
}

cudaError_t launch_log2_image(const float* in, float* out, int64_t count, cudaStream_t s) {
  int blocks = int(std::min<int64_t>((count + 255) / 256, 148 * 16));
  log2_kernel<<<blocks, 256, 0, s>>>(in, out, count);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// initDictionary + normalizeDictKernel (cuda_svd_denoiser.cu:52-63, 261-280).
// Atom k = patch N/2 + k divided by its norm.  With int_norm the squared norm
// is summed the way the reference's transform_reduce with the int init value
// 0 sums it: each partial sum (float add of the int accumulator and x*x) is
// truncated back to int.  Explicit _rn intrinsics keep the product and the
// sum as two separately rounded float operations, as on the host.
// One warp per atom; lane 0 runs the sequential sum.
// ---------------------------------------------------------------------------
__global__ void init_dict_kernel(const float* __restrict__ patches, int64_t N, int n, int K, int int_norm,
                                 float* __restrict__ dict, GridBarrier* flags) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= K) return;
  const float* src = patches + (N / 2 + warp) * int64_t(n);
  float norm = 0.0f;
  if (lane == 0) {
    if (int_norm) {
      int acc = 0;
      for (int i = 0; i < n; ++i) {
        float x = src[i];
        float sq = __fmul_rn(x, x);
        acc = __float2int_rz(__fadd_rn(__int2float_rn(acc), sq));
      }
      norm = __fsqrt_rn(__int2float_rn(acc));
    } else {
      float acc = 0.0f;
      for (int i = 0; i < n; ++i) acc = __fadd_rn(acc, __fmul_rn(src[i], src[i]));
      norm = __fsqrt_rn(acc);
    }
  }
  norm = __shfl_sync(0xffffffffu, norm, 0);
  if (!(norm > 0.0f) && lane == 0) atomicCAS(&flags->err, DEVERR_NONE, DEVERR_ZERO_ATOM);
  for (int i = lane; i < n; i += 32) dict[int64_t(warp) * n + i] = __fdiv_rn(src[i], norm);
}

cudaError_t launch_init_dict(const float* patches, int64_t N, int n, int K, int int_norm, float* dict,
                             GridBarrier* flags, cudaStream_t s) {
  int threads = 128;
  int blocks = (K * 32 + threads - 1) / threads;
  init_dict_kernel<<<blocks, threads, 0, s>>>(patches, N, n, K, int_norm, dict, flags);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Dictionary Gram D D^T in FP64 from the FP32 atoms (products exact in
// double).  The OMP least-squares step reads its support block from it, so
// near-collinear supports keep an accurate Cholesky pivot.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) gram_f64_kernel(const float* __restrict__ dict, int K, int n,
                                                       double* __restrict__ gram) {
  __shared__ float A[16][65];
  __shared__ float B[16][65];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int a0 = blockIdx.y * 16, b0 = blockIdx.x * 16;
  double acc = 0.0;
  for (int k0 = 0; k0 < n; k0 += 64) {
    for (int t = threadIdx.x; t < 16 * 64; t += 256) {
      int r = t >> 6, c = t & 63;
      int k = k0 + c;
      A[r][c] = (a0 + r < K && k < n) ? dict[int64_t(a0 + r) * n + k] : 0.0f;
      B[r][c] = (b0 + r < K && k < n) ? dict[int64_t(b0 + r) * n + k] : 0.0f;
    }
    __syncthreads();
#pragma unroll 8
    for (int c = 0; c < 64; ++c) acc = fma(double(A[ty][c]), double(B[tx][c]), acc);
    __syncthreads();
  }
  if (a0 + ty < K && b0 + tx < K) gram[int64_t(a0 + ty) * K + (b0 + tx)] = acc;
}

cudaError_t launch_gram_f64(const float* dict, int K, int n, double* gram, cudaStream_t s) {
  dim3 grid((K + 15) / 16, (K + 15) / 16);
  gram_f64_kernel<<<grid, 256, 0, s>>>(dict, K, n, gram);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Compact codes -> the reference's dense K x N code matrix (copyData3Kernel,
// cublas_matrix_omp.cu:37-47, writes the same positions).
// ---------------------------------------------------------------------------
__global__ void codes_to_dense_kernel(const int32_t* __restrict__ idx, const float* __restrict__ coef,
                                      int64_t N, int L, int K, float* __restrict__ dense) {
  for (int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; p < N; p += int64_t(gridDim.x) * blockDim.x) {
    for (int s = 0; s < L; ++s) {
      int a = idx[p * L + s];
      if (a >= 0 && a < K) dense[p * K + a] = coef[p * L + s];
    }
  }
}

cudaError_t launch_codes_to_dense(const int32_t* idx, const float* coef, int64_t N, int L, int K, float* dense,
                                  cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(dense, 0, size_t(N) * K * sizeof(float), s);
  if (e != cudaSuccess) return e;
  int blocks = int(std::min<int64_t>((N + 255) / 256, 148 * 8));
  codes_to_dense_kernel<<<blocks, 256, 0, s>>>(idx, coef, N, L, K, dense);
  return cudaGetLastError();
}

}  // namespace ksvd
