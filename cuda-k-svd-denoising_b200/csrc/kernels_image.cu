// Image rebuild (createImage, cuda_svd_denoiser.cu:413-498).
//
// The reference forms all denoised patches D X with one SGEMM, copies them to
// the host and overlap-adds them in a single host thread.  Here:
//   col2im_kernel  one CTA per TS x TS pixel tile (TS = 32, 16 or 8; large
//                  patches use col2im_direct_kernel, one thread per pixel,
//                  with the same sums): the denoised patches that
//                  cover the tile (x_hat_p = sum_s x_s d_s from the compact
//                  codes) are formed in shared memory, then each pixel sums
//                  the covering patches in patch order (ix, then iy, the
//                  reference's order) and the tile's share of
//                  sum (img/w - y)^2 is reduced in FP64;
//   lambda_kernel  fixed-order sum of the tile partials ->
//                  lambda = |sqrt(sum / (sigma2 * P)) - 1|;
//   blend_kernel   out = (lambda y + img) / (lambda + w), exp2 for speckle.
// Pixels no patch covers (w = 0) are excluded from the lambda sum and come
// back as y (the reference would divide 0/0 there).
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "ksvd_internal.cuh"

namespace ksvd {

constexpr size_t kCol2imSmemLimit = 100 * 1024;

static int tile_patches_1d(int TS, int ext, int stride) { return (TS + ext - 1) / stride + 1; }

// Tile side of the shared-memory gather: the largest of 32, 16, 8 whose
// covering patches fit the budget; 0 when none does (large patches), in
// which case the direct gather runs.
static int pick_tile(const PatchGeom& g) {
  const int cands[] = {32, 16, 8};
  for (int TS : cands) {
    size_t np = size_t(tile_patches_1d(TS, g.ph, g.sh)) * tile_patches_1d(TS, g.pw, g.sw);
    if (np * g.n * sizeof(float) <= kCol2imSmemLimit) return TS;
  }
  return 0;
}

constexpr int kDirectThreads = 256;

int col2im_num_tiles(const PatchGeom& g) {
  const int TS = pick_tile(g);
  if (TS == 0) return int((int64_t(g.W) * g.H + kDirectThreads - 1) / kDirectThreads);
  return ((g.W + TS - 1) / TS) * ((g.H + TS - 1) / TS);
}

// ix range covering x: ix*sh <= x < ix*sh + ph, 0 <= ix < nx
__device__ __forceinline__ int cover_lo(int x, int ext, int stride) {
  int t = x - ext + 1;
  return t <= 0 ? 0 : (t + stride - 1) / stride;
}
__device__ __forceinline__ int cover_hi(int x, int stride, int npos) { return min(npos - 1, x / stride); }

__global__ void __launch_bounds__(256) col2im_kernel(const float* __restrict__ noisy, PatchGeom g, int TS,
                                                     const float* __restrict__ D, int K, int L,
                                                     const int32_t* __restrict__ idx, const float* __restrict__ coef,
                                                     float* __restrict__ acc_out, double* __restrict__ partials) {
  extern __shared__ float xs[];
  __shared__ double red[32];
  const int tx0 = blockIdx.x * TS, ty0 = blockIdx.y * TS;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int tx1 = min(g.W, tx0 + TS) - 1, ty1 = min(g.H, ty0 + TS) - 1;
  const int ixl = cover_lo(tx0, g.ph, g.sh), ixh = cover_hi(tx1, g.sh, g.nx);
  const int iyl = cover_lo(ty0, g.pw, g.sw), iyh = cover_hi(ty1, g.sw, g.ny);
  const int npx = max(0, ixh - ixl + 1), npy = max(0, iyh - iyl + 1);
  for (int q = warp; q < npx * npy; q += nwarps) {
    const int ix = ixl + q / npy, iy = iyl + q % npy;
    const int64_t p = int64_t(ix) * g.ny + iy;
    // the patch's code, one (atom, coefficient) pair per lane, broadcast below
    int a_l = -1;
    float x_l = 0.0f;
    if (lane < L) {
      a_l = __ldg(idx + p * L + lane);
      x_l = __ldg(coef + p * L + lane);
      if (a_l < 0 || a_l >= K) a_l = -1;
    }
    // features lane, lane + 32, ... in groups of kCF; per group the rows of
    // kCS atoms are loaded before their FMAs (sum over s ascending, as in a
    // plain loop)
    constexpr int kCF = 5, kCS = 4;
    for (int i0 = 0; i0 < g.n; i0 += 32 * kCF) {
      float v[kCF];
#pragma unroll
      for (int f = 0; f < kCF; ++f) v[f] = 0.0f;
      for (int s0 = 0; s0 < L; s0 += kCS) {  // L <= 32, the same trip count in every lane
        float dv[kCS][kCF];
        float xv[kCS];
        bool uv[kCS];
#pragma unroll
        for (int u = 0; u < kCS; ++u) {
          const int s = s0 + u;
          const int a = __shfl_sync(0xffffffffu, a_l, s & 31);
          const float x = __shfl_sync(0xffffffffu, x_l, s & 31);
          const bool use = s < L && a >= 0;
          uv[u] = use;
          xv[u] = x;
#pragma unroll
          for (int f = 0; f < kCF; ++f) {
            const int i = i0 + 32 * f + lane;
            dv[u][f] = (use && i < g.n) ? __ldg(D + int64_t(a) * g.n + i) : 0.0f;
          }
        }
#pragma unroll
        for (int u = 0; u < kCS; ++u) {
          if (uv[u])
#pragma unroll
            for (int f = 0; f < kCF; ++f) v[f] = fmaf(xv[u], dv[u][f], v[f]);
        }
      }
#pragma unroll
      for (int f = 0; f < kCF; ++f) {
        const int i = i0 + 32 * f + lane;
        if (i < g.n) xs[q * g.n + i] = v[f];
      }
    }
  }
  __syncthreads();
  double part = 0.0;
  for (int t = threadIdx.x; t < TS * TS; t += blockDim.x) {
    const int x = tx0 + t % TS, y = ty0 + t / TS;
    if (x >= g.W || y >= g.H) continue;
    const int ia = max(ixl, cover_lo(x, g.ph, g.sh)), ib = min(ixh, cover_hi(x, g.sh, g.nx));
    const int ja = max(iyl, cover_lo(y, g.pw, g.sw)), jb = min(iyh, cover_hi(y, g.sw, g.ny));
    float acc = 0.0f;
    int w = 0;
    for (int ix = ia; ix <= ib; ++ix)
      for (int iy = ja; iy <= jb; ++iy) {
        const int q = (ix - ixl) * npy + (iy - iyl);
        acc += xs[q * g.n + (x - ix * g.sh) * g.pw + (y - iy * g.sw)];
        ++w;
      }
    acc_out[size_t(y) * g.W + x] = acc;
    if (w > 0) {
      const double d = double(acc) / double(w) - double(noisy[size_t(y) * g.W + x]);
      part += d * d;
    }
  }
  part = block_sum(part, red);
  if (threadIdx.x == 0) partials[blockIdx.y * gridDim.x + blockIdx.x] = part;
}

// The same sums without shared memory, for patches too large for a tile's
// covering patches to fit it: one thread per pixel forms the element of each
// covering patch it needs (x_hat_p[r] = sum_s x_s d_s[r], the same FMA order
// as col2im_kernel) and adds them in the same patch order, so the result is
// identical; each block reduces its share of the lambda sum.
__global__ void __launch_bounds__(kDirectThreads) col2im_direct_kernel(
    const float* __restrict__ noisy, PatchGeom g, const float* __restrict__ D, int K, int L,
    const int32_t* __restrict__ idx, const float* __restrict__ coef, float* __restrict__ acc_out,
    double* __restrict__ partials) {
  __shared__ double red[32];
  const int64_t P = int64_t(g.W) * g.H;
  const int64_t q = int64_t(blockIdx.x) * kDirectThreads + threadIdx.x;
  double part = 0.0;
  if (q < P) {
    const int y = int(q / g.W), x = int(q - int64_t(y) * g.W);
    const int ia = cover_lo(x, g.ph, g.sh), ib = cover_hi(x, g.sh, g.nx);
    const int ja = cover_lo(y, g.pw, g.sw), jb = cover_hi(y, g.sw, g.ny);
    float acc = 0.0f;
    int w = 0;
    for (int ix = ia; ix <= ib; ++ix)
      for (int iy = ja; iy <= jb; ++iy) {
        const int64_t p = int64_t(ix) * g.ny + iy;
        const int off = (x - ix * g.sh) * g.pw + (y - iy * g.sw);
        float v = 0.0f;
        for (int s = 0; s < L; ++s) {
          const int a = __ldg(idx + p * L + s);
          if (a < 0 || a >= K) continue;
          v = fmaf(__ldg(coef + p * L + s), __ldg(D + int64_t(a) * g.n + off), v);
        }
        acc += v;
        ++w;
      }
    acc_out[q] = acc;
    if (w > 0) {
      const double d = double(acc) / double(w) - double(noisy[q]);
      part = d * d;
    }
  }
  part = block_sum(part, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = part;
}

__global__ void __launch_bounds__(1024) lambda_kernel(const double* __restrict__ partials, int np, double sigma2,
                                                      double pixels, double* __restrict__ lambda_dev) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
  s = block_sum(s, red);
  if (threadIdx.x == 0) lambda_dev[0] = fabs(sqrt(s / (sigma2 * pixels)) - 1.0);
}

__global__ void blend_kernel(const float* __restrict__ noisy, PatchGeom g, const float* __restrict__ acc,
                             const double* __restrict__ lambda_dev, int speckle, float* __restrict__ out) {
  const double lam = lambda_dev[0];
  const float lamf = float(lam);
  const int64_t P = int64_t(g.W) * g.H;
  for (int64_t q = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; q < P; q += int64_t(gridDim.x) * blockDim.x) {
    const int y = int(q / g.W), x = int(q - int64_t(y) * g.W);
    const int cx = max(0, min(g.nx - 1, x / g.sh) - cover_lo(x, g.ph, g.sh) + 1);
    const int cy = max(0, min(g.ny - 1, y / g.sw) - cover_lo(y, g.pw, g.sw) + 1);
    const float w = float(cx * cy);
    const float yv = noisy[q];
    float v = (w > 0.0f) ? (lamf * yv + acc[q]) / (lamf + w) : yv;
    if (speckle) v = exp2f(v);
    out[q] = v;
  }
}

cudaError_t launch_col2im(const float* noisy, const PatchGeom& g, const float* dict, int K, int L,
                          const int32_t* idx, const float* coef, float* acc, double* partials, int* num_partials,
                          cudaStream_t s) {
  const int TS = pick_tile(g);
  if (TS == 0) {
    const int64_t blocks = (int64_t(g.W) * g.H + kDirectThreads - 1) / kDirectThreads;
    col2im_direct_kernel<<<unsigned(blocks), kDirectThreads, 0, s>>>(noisy, g, dict, K, L, idx, coef, acc, partials);
    *num_partials = int(blocks);
    return cudaGetLastError();
  }
  const size_t np = size_t(tile_patches_1d(TS, g.ph, g.sh)) * tile_patches_1d(TS, g.pw, g.sw);
  const size_t smem = np * g.n * sizeof(float);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(col2im_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
  }
  dim3 grid((g.W + TS - 1) / TS, (g.H + TS - 1) / TS);
  col2im_kernel<<<grid, 256, smem, s>>>(noisy, g, TS, dict, K, L, idx, coef, acc, partials);
  *num_partials = int(grid.x * grid.y);
  return cudaGetLastError();
}

cudaError_t launch_blend(const float* noisy, const PatchGeom& g, const float* acc, const double* partials,
                         int num_partials, double sigma2, int speckle, float* out, double* lambda_dev,
                         cudaStream_t s) {
  lambda_kernel<<<1, 1024, 0, s>>>(partials, num_partials, sigma2, double(g.W) * double(g.H), lambda_dev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int64_t P = int64_t(g.W) * g.H;
  const int blocks = int(std::min<int64_t>((P + 255) / 256, 148 * 16));
  blend_kernel<<<blocks, 256, 0, s>>>(noisy, g, acc, lambda_dev, speckle, out);
  return cudaGetLastError();
}

}  // namespace ksvd
