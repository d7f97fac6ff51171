// OMP restricted to a per-patch candidate set (the learned proposal's top
// candidates), with the fallback bookkeeping.  It is the same pursuit as
// CuBlasMatrixOmp::work (cublas_matrix_omp.cu:186-393: argmax |D^T r| with
// lowest atom index on ties, least squares of the patch on the support, stop
// when |r| < 1e-3, re-selected or dependent atom ends the pursuit) with the
// argmax taken over the candidates only.
//
// One warp per patch.  Lane pair (2c, 2c + 1) owns candidate c: it forms
// b_c = d_c . y exactly (FP64 from the FP32 data; the two lanes sum
// alternate groups of four features, two FP64 chains each) and keeps the candidate's correlation with the
// residual in the Batch-OMP form
//     alpha_c = b_c - sum_s g_s G[c][s]          (FP64, FP64 Gram)
// so no residual vector is ever formed.  Each candidate's Gram entries with
// the support sit in shared memory: per step all candidate lanes load their
// one new entry at once, and the winner's row is the Cholesky append's
// G[new][S].  Lane 0 extends the Cholesky factor
// of the support Gram by one row per step, keeps the forward solution
// z = L^-1 b of the support, solves for the coefficients g and tracks
// |r|^2 = |y|^2 - |z|^2.  A patch whose final residual norm is above the
// threshold is appended to the fallback list; the caller re-codes those
// patches with the full OMP.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "ksvd_internal.cuh"

namespace ksvd {

constexpr int kRWarps = 8;
constexpr int kRLMax = 16;
constexpr int kRMaxN = 512;

__global__ void __launch_bounds__(kRWarps * 32)
    omp_restricted_kernel(const float* __restrict__ Y, int64_t N, int n, const float* __restrict__ D,
                          const double* __restrict__ Gram, int K, int L, const int32_t* __restrict__ cand, int C,
                          double thr2, int32_t* __restrict__ idx_out, float* __restrict__ coef_out,
                          int64_t* __restrict__ fb_list, unsigned long long* __restrict__ fb_count, int vec4) {
  __shared__ __align__(16) float ys[kRWarps][kRMaxN];
  __shared__ double lf[kRWarps][kRLMax * (kRLMax + 1) / 2];  // Cholesky rows, diagonal as 1 / L_ii
  __shared__ double zf[kRWarps][kRLMax];                     // forward solution L^-1 b
  __shared__ double gm[kRWarps][kRLMax];                     // coefficients
  __shared__ int sup[kRWarps][kRLMax];
  __shared__ double gcs[kRWarps][16][kRLMax + 1];  // per candidate: G[candidate][support atom s] (padded: no bank conflicts)
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = lane >> 1, h = lane & 1;
  double* Lp = lf[w];
  auto Lat = [&](int i, int j) -> double& { return Lp[i * (i + 1) / 2 + j]; };
  const int64_t warps = int64_t(gridDim.x) * kRWarps;
  for (int64_t p = int64_t(blockIdx.x) * kRWarps + w; p < N; p += warps) {
    const float* y = Y + p * n;
    double yy = 0.0;
    for (int k = lane; k < n; k += 32) {
      const float v = y[k];
      ys[w][k] = v;
      yy = fma(double(v), double(v), yy);
    }
    yy = warp_sum(yy);
    __syncwarp();
    // candidate of this lane pair (-1: none)
    int a = -1;
    if (c < C) {
      a = cand[p * C + c];
      if (a < 0 || a >= K) a = -1;
    }
    // b_c = d_c . y in FP64: the lane pair splits the features, several
    // independent loads in flight per lane
    double b = 0.0;
    if (a >= 0) {
      const float* d = D + int64_t(a) * n;
      double b0 = 0.0, b1 = 0.0;
      if (vec4) {
        const float4* d4 = reinterpret_cast<const float4*>(d);
        const float4* y4 = reinterpret_cast<const float4*>(ys[w]);
        const int n4 = n >> 2;
        for (int f0 = h; f0 < n4; f0 += 8) {
          float4 dv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) dv[u] = (f0 + 2 * u < n4) ? __ldg(d4 + f0 + 2 * u) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (f0 + 2 * u < n4) {
              const float4 yv = y4[f0 + 2 * u];
              b0 = fma(double(dv[u].x), double(yv.x), b0);
              b1 = fma(double(dv[u].y), double(yv.y), b1);
              b0 = fma(double(dv[u].z), double(yv.z), b0);
              b1 = fma(double(dv[u].w), double(yv.w), b1);
            }
          }
        }
      } else {
        for (int k = h; k < n; k += 2) b0 = fma(double(__ldg(d + k)), double(ys[w][k]), b0);
      }
      b = b0 + b1;
    }
    b += __shfl_xor_sync(0xffffffffu, b, 1);
    double alpha = b;
    int cnt = 0;
    double rr = yy;
    // a zero patch: every correlation is 0 and the full pursuit takes atom 0
    // with coefficient 0 (lowest index), then stops
    if (yy == 0.0) {
      if (lane == 0) {
        sup[w][0] = 0;
        gm[w][0] = 0.0;
      }
      cnt = 1;
    } else {
      for (int step = 0; step < L; ++step) {
        if (step > 0 && sqrt(fmax(rr, 0.0)) < 1e-3) break;  // :218, the norm of the previous step
        // argmax |alpha| over the candidates, lowest atom index on ties
        double key = (a >= 0 && h == 0) ? fabs(alpha) : -1.0;
        int ka = (a >= 0 && h == 0) ? a : 0x7fffffff;
        int kc = c;  // the winner's candidate slot
        double kb = b;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double k2 = __shfl_xor_sync(0xffffffffu, key, o);
          const int a2 = __shfl_xor_sync(0xffffffffu, ka, o);
          const int c2 = __shfl_xor_sync(0xffffffffu, kc, o);
          const double b2 = __shfl_xor_sync(0xffffffffu, kb, o);
          if (k2 > key || (k2 == key && a2 < ka)) {
            key = k2;
            ka = a2;
            kc = c2;
            kb = b2;
          }
        }
        if (key < 0.0) break;  // no candidate at all
        const int k = cnt;
        // each candidate's Gram entry with the new atom, loaded in parallel:
        // the support atoms are candidates, so the winner's row of the cache
        // holds G[new][S_i] for the Cholesky append
        if (a >= 0 && h == 0) gcs[w][c][k] = Gram[int64_t(a) * K + ka];
        __syncwarp();
        int stop = 0;
        if (lane == 0) {
          for (int s2 = 0; s2 < k; ++s2)
            if (sup[w][s2] == ka) stop = 1;  // re-selected atom: the pursuit ends
          if (!stop) {
            const double* gw = gcs[w][kc];
            double ww = 0.0;
            for (int i = 0; i < k; ++i) {
              double s3 = gw[i];
              for (int j = 0; j < i; ++j) s3 -= Lat(i, j) * Lat(k, j);
              const double wi = s3 * Lat(i, i);
              Lat(k, i) = wi;
              ww += wi * wi;
            }
            const double piv2 = gw[k] - ww;
            if (!(piv2 > 0.0)) {
              stop = 1;  // the new atom depends linearly on the support
            } else {
              Lat(k, k) = 1.0 / sqrt(piv2);
              sup[w][k] = ka;
              double zk = kb;
              for (int j = 0; j < k; ++j) zk -= Lat(k, j) * zf[w][j];
              zk *= Lat(k, k);
              zf[w][k] = zk;
              for (int i = k; i >= 0; --i) {
                double s3 = zf[w][i];
                for (int j = i + 1; j <= k; ++j) s3 -= Lat(j, i) * gm[w][j];
                gm[w][i] = s3 * Lat(i, i);
              }
            }
          }
        }
        stop = __shfl_sync(0xffffffffu, stop, 0);
        __syncwarp();
        if (stop) break;
        cnt += 1;
        // |r|^2 = |y|^2 - |z|^2 and the candidates' new correlations
        double zz = 0.0;
        for (int i = 0; i < cnt; ++i) zz = fma(zf[w][i], zf[w][i], zz);
        rr = yy - zz;
        if (a >= 0 && h == 0) {
          double s3 = b;
          for (int i = 0; i < cnt; ++i) s3 = fma(-gm[w][i], gcs[w][c][i], s3);
          alpha = s3;
        }
      }
    }
    __syncwarp();
    if (lane < L) {
      const bool used = lane < cnt;
      idx_out[p * L + lane] = used ? sup[w][lane] : -1;
      coef_out[p * L + lane] = used ? float(gm[w][lane]) : 0.0f;
    }
    if (lane == 0 && rr > thr2) {
      const unsigned long long pos = atomicAdd(fb_count, 1ull);
      fb_list[pos] = p;
    }
    __syncwarp();
  }
}

__global__ void gather_rows_kernel(const float* __restrict__ src, int w, const int64_t* __restrict__ list,
                                   int64_t count, float* __restrict__ dst) {
  const int64_t total = count * w;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = i / w;
    dst[i] = src[list[r] * w + (i - r * w)];
  }
}

__global__ void scatter_codes_kernel(const int32_t* __restrict__ sidx, const float* __restrict__ scoef, int L,
                                     const int64_t* __restrict__ list, int64_t count, int32_t* __restrict__ idx,
                                     float* __restrict__ coef) {
  const int64_t total = count * L;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = i / L;
    const int64_t q = list[r] * L + (i - r * L);
    idx[q] = sidx[i];
    coef[q] = scoef[i];
  }
}

bool omp_restricted_supported(int n, int L, int C) { return n >= 1 && n <= kRMaxN && L >= 1 && L <= kRLMax && C >= 1 && C <= 16; }

cudaError_t launch_omp_restricted(const float* patches, int64_t N, int n, const float* dict, const double* gram, int K,
                                  int L, const int32_t* cand, int C, double thr2, int32_t* idx, float* coef,
                                  int64_t* fb_list, unsigned long long* fb_count, int num_sms, cudaStream_t s) {
  if (!omp_restricted_supported(n, L, C)) return cudaErrorInvalidValue;
  const int64_t want = (N + kRWarps - 1) / kRWarps;
  const int64_t cap = int64_t(num_sms) * 8;
  const int blocks = int(want < cap ? want : cap);
  const int vec4 = ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(dict) & 15) == 0) ? 1 : 0;
  omp_restricted_kernel<<<blocks > 0 ? blocks : 1, kRWarps * 32, 0, s>>>(patches, N, n, dict, gram, K, L, cand, C,
                                                                          thr2, idx, coef, fb_list, fb_count, vec4);
  return cudaGetLastError();
}

static int rows_blocks(int64_t total) {
  const int64_t b = (total + 255) / 256;
  return int(b < 8192 ? (b > 0 ? b : 1) : 8192);
}

cudaError_t launch_gather_rows(const float* src, int w, const int64_t* list, int64_t count, float* dst,
                               cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  gather_rows_kernel<<<rows_blocks(count * w), 256, 0, s>>>(src, w, list, count, dst);
  return cudaGetLastError();
}

cudaError_t launch_scatter_codes(const int32_t* sidx, const float* scoef, int L, const int64_t* list, int64_t count,
                                 int32_t* idx, float* coef, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  scatter_codes_kernel<<<rows_blocks(count * L), 256, 0, s>>>(sidx, scoef, L, list, count, idx, coef);
  return cudaGetLastError();
}

}  // namespace ksvd
