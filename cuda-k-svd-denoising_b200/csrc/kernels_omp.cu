// Batched OMP sparse coding, plain FP32 form (CuBlasMatrixOmp::work,
// cublas_matrix_omp.cu:107-402).
//
// The reference runs each OMP step as one cuBLAS SGEMM (D^T R) followed by
// about 4 N per-patch cuBLAS calls issued from host loops (Isamax, gesvda
// pseudo-inverse, two Sgemv, Snrm2).  Here one persistent kernel does every
// step of every patch on chip:
//   * the CTA keeps the whole dictionary in shared memory, k-major, and walks
//     tiles of kTP patches (grid = one CTA per SM);
//   * per step, the K x kTP correlation D^T R is a register-tiled FP32 SIMT
//     product (8 atoms x 4 patches per thread, 16-byte shared loads);
//   * argmax |.| per patch with the lowest atom index winning ties, as
//     cublasIsamax does (:216-233);
//   * the least-squares coefficients on the support (the reference's
//     pseudo-inverse, :269-339) come from a Cholesky factor of the support
//     Gram grown by one row per step, in FP64 from the FP64 dictionary Gram
//     (diagonal kept inverted; the forward solution z = L^-1 b grows by one
//     element per step, only the back substitution runs over the support);
//   * the residual y - D_S g (:352-380) and its norm (:382-393) are formed
//     per patch by one warp; a patch whose residual norm is below 1e-3 stops
//     (:218).  Before an update sweep the tile's final residual rows go to
//     the sweep's residual buffer (the arithmetic of launch_residual).
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "ksvd_internal.cuh"

namespace ksvd {

constexpr int kTP = 32;         // patches per tile
constexpr int kOmpThreads = 256;
constexpr int kAtomBlock = 256;  // atoms per register-tiled pass (32 groups x 8)
constexpr int kLMax = 32;        // omp_iter limit (support list fits a warp)

struct OmpLayout {
  int Kpad, dks, rks, ysn;
  size_t off_dk, off_rk, off_ys, off_lc, off_bv, off_s, off_gam, off_sel, off_cnt, off_done, off_redv, off_redi,
      off_gs, off_bs, off_np, total;
};

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline OmpLayout omp_layout(int n, int K, int L) {
  OmpLayout o;
  o.Kpad = (K + kAtomBlock - 1) / kAtomBlock * kAtomBlock;
  o.dks = o.Kpad + 4;
  o.rks = kTP + 4;
  o.ysn = n + 1;  // odd row stride: lanes over patches hit distinct banks
  size_t off = 0;
  o.off_dk = off;
  off = al16(off + size_t(n) * o.dks * 4);
  o.off_rk = off;
  off = al16(off + size_t(n) * o.rks * 4);
  o.off_ys = off;
  off = al16(off + size_t(kTP) * o.ysn * 4);
  o.off_lc = off;
  off = al16(off + size_t(kTP) * L * L * 8);
  o.off_bv = off;
  off = al16(off + size_t(kTP) * L * 8);
  o.off_s = off;
  off = al16(off + size_t(kTP) * L * 4);
  o.off_gam = off;
  off = al16(off + size_t(kTP) * L * 4);
  o.off_sel = off;
  off = al16(off + kTP * 4);
  o.off_cnt = off;
  off = al16(off + kTP * 4);
  o.off_done = off;
  off = al16(off + kTP * 4);
  o.off_redv = off;
  off = al16(off + 8 * kTP * 4);
  o.off_redi = off;
  off = al16(off + 8 * kTP * 4);
  o.off_gs = off;
  off = al16(off + size_t(kTP) * (L + 1) * 8);
  o.off_bs = off;
  off = al16(off + kTP * 8);
  o.off_np = off;
  off = al16(off + 8 * kTP * 4);
  o.total = off;
  return o;
}

__device__ __forceinline__ bool better(float v1, int i1, float v2, int i2) {
  return v1 > v2 || (v1 == v2 && i1 < i2);
}

__global__ void __launch_bounds__(kOmpThreads, 1)
    omp_fp32_kernel(const float* __restrict__ Y, int64_t N, int n, const float* __restrict__ D,
                    const double* __restrict__ Gram, int K, int L, int32_t* __restrict__ idx_out,
                    float* __restrict__ coef_out, int64_t ntiles, float* __restrict__ R_out,
                    int* __restrict__ last_out, DevStats* stats) {
  extern __shared__ __align__(16) unsigned char smem[];
  const OmpLayout lo = omp_layout(n, K, L);
  float* Dk = reinterpret_cast<float*>(smem + lo.off_dk);
  float* Rk = reinterpret_cast<float*>(smem + lo.off_rk);
  float* Ys = reinterpret_cast<float*>(smem + lo.off_ys);
  double* Lc = reinterpret_cast<double*>(smem + lo.off_lc);
  double* bvec = reinterpret_cast<double*>(smem + lo.off_bv);
  int* S = reinterpret_cast<int*>(smem + lo.off_s);
  float* gam = reinterpret_cast<float*>(smem + lo.off_gam);
  int* sel = reinterpret_cast<int*>(smem + lo.off_sel);
  int* cnt = reinterpret_cast<int*>(smem + lo.off_cnt);
  int* done = reinterpret_cast<int*>(smem + lo.off_done);
  float* redv = reinterpret_cast<float*>(smem + lo.off_redv);
  int* redi = reinterpret_cast<int*>(smem + lo.off_redi);
  double* gS = reinterpret_cast<double*>(smem + lo.off_gs);
  double* bS = reinterpret_cast<double*>(smem + lo.off_bs);
  float* npart = reinterpret_cast<float*>(smem + lo.off_np);
  const int ysn = lo.ysn;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int dks = lo.dks, rks = lo.rks, Kpad = lo.Kpad;

  // Dictionary, k-major, padded atoms zero.
  for (int t = tid; t < K * n; t += kOmpThreads) {
    int a = t / n, k = t - a * n;
    Dk[k * dks + a] = __ldg(D + t);
  }
  if (Kpad > K) {
    const int padw = Kpad - K;
    for (int t = tid; t < n * padw; t += kOmpThreads) {
      int k = t / padw, a = K + (t - k * padw);
      Dk[k * dks + a] = 0.0f;
    }
  }
  __syncthreads();

  const int ag = tid >> 3, pg = tid & 7;  // atom group (32), patch group (8)
  const bool timer = (blockIdx.x == 0 && tid == 0 && stats != nullptr);
  // phase times (slots 8..11) gather in shared memory, flushed once at the end
  __shared__ unsigned long long s_ph[4];
  if (timer)
    for (int k = 0; k < 4; ++k) s_ph[k] = 0ull;
  unsigned long long tmark = timer ? globaltimer_ns() : 0ull;
  auto lap = [&](int slot) {
    if (timer) {
      const unsigned long long t = globaltimer_ns();
      s_ph[slot - 8] += t - tmark;
      tmark = t;
    }
  };

  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t p0 = tile * kTP;
    const int np = (N - p0 < kTP) ? int(N - p0) : kTP;
    const float* Yt = Y + p0 * n;
    for (int t = tid; t < kTP * n; t += kOmpThreads) {
      int p = t / n, k = t - p * n;
      float v = (p < np) ? __ldg(Yt + t) : 0.0f;
      Ys[p * ysn + k] = v;
      Rk[k * rks + p] = v;
    }
    if (tid < kTP) {
      cnt[tid] = 0;
      done[tid] = (tid >= np);
    }
    __syncthreads();
    lap(10);

    for (int step = 0; step < L; ++step) {
      const int active = (tid < kTP) ? !done[tid] : 0;
      if (!__syncthreads_or(active)) break;

      // ---- correlation D^T R and per-thread argmax ------------------------
      float bv[4];
      int bi[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        bv[j] = -1.0f;
        bi[j] = 0x7fffffff;
      }
      for (int ab = 0; ab < Kpad; ab += kAtomBlock) {
        float acc[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;
        const float* dcol = Dk + ab + ag * 8;
        const float* rcol = Rk + pg * 4;
#pragma unroll 4
        for (int k = 0; k < n; ++k) {
          const float4 d0 = *reinterpret_cast<const float4*>(dcol + k * dks);
          const float4 d1 = *reinterpret_cast<const float4*>(dcol + k * dks + 4);
          const float4 r = *reinterpret_cast<const float4*>(rcol + k * rks);
          const float dv[8] = {d0.x, d0.y, d0.z, d0.w, d1.x, d1.y, d1.z, d1.w};
          const float rv[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
          for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(dv[i], rv[j], acc[i][j]);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int a = ab + ag * 8 + i;
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const float v = fabsf(acc[i][j]);
            if (a < K && v > bv[j]) {
              bv[j] = v;
              bi[j] = a;
            }
          }
        }
      }
      // reduce over the 4 atom groups of the warp (lanes 8 and 16 apart)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int off = 8; off <= 16; off <<= 1) {
          float ov = __shfl_xor_sync(0xffffffffu, bv[j], off);
          int oi = __shfl_xor_sync(0xffffffffu, bi[j], off);
          if (better(ov, oi, bv[j], bi[j])) {
            bv[j] = ov;
            bi[j] = oi;
          }
        }
      }
      if (lane < 8) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          redv[warp * kTP + pg * 4 + j] = bv[j];
          redi[warp * kTP + pg * 4 + j] = bi[j];
        }
      }
      __syncthreads();
      if (tid < kTP) {
        float v = redv[tid];
        int i = redi[tid];
        for (int w = 1; w < 8; ++w) {
          float ov = redv[w * kTP + tid];
          int oi = redi[w * kTP + tid];
          if (better(ov, oi, v, i)) {
            v = ov;
            i = oi;
          }
        }
        sel[tid] = (i < K) ? i : 0;
      }
      __syncthreads();
      lap(8);

      // ---- least squares on the grown support, residual, norm -------------
      // (1) dependence test and support-Gram column, all patches at once:
      //     gS[p][i] = G[S_i][a] (i < k), gS[p][k] = G[a][a]
      for (int t = tid; t < kTP * (L + 1); t += kOmpThreads) {
        const int p = t / (L + 1), i = t - p * (L + 1);
        if (done[p]) continue;
        const int k = cnt[p], a = sel[p];
        if (i < k) {
          const int si = S[p * L + i];
          if (si == a) done[p] = 2;  // re-selected atom: the pursuit of p ends
          gS[p * (L + 1) + i] = Gram[int64_t(si) * K + a];
        } else if (i == k) {
          gS[p * (L + 1) + i] = Gram[int64_t(a) * K + a];
        }
      }
      // (2) b_p = d_a . y_p in FP64, four patches per warp
      for (int q = 0; q < kTP / 8; ++q) {
        const int p = warp * (kTP / 8) + q;
        const int a = sel[p];
        double bp = 0.0;
        for (int k = lane; k < n; k += 32) bp = fma(double(Dk[k * dks + a]), double(Ys[p * ysn + k]), bp);
        bp = warp_sum(bp);
        if (lane == 0) bS[p] = bp;
      }
      __syncthreads();
      // (3) Cholesky row append and solve, one thread per patch
      if (tid < kTP) {
        const int p = tid;
        if (done[p] == 2) done[p] = 1;
        if (!done[p]) {
          const int k = cnt[p], a = sel[p];
          double* Lp = Lc + p * L * L;
          const double* g = gS + p * (L + 1);
          double ww = 0.0;
          for (int i = 0; i < k; ++i) {
            double s = g[i];
            for (int j2 = 0; j2 < i; ++j2) s -= Lp[i * L + j2] * Lp[k * L + j2];
            const double wi = s * Lp[i * L + i];  // the diagonal is kept as 1 / L_ii
            Lp[k * L + i] = wi;
            ww += wi * wi;
          }
          const double piv2 = g[k] - ww;
          if (!(piv2 > 0.0)) {
            done[p] = 1;  // the new atom depends linearly on the support
          } else {
            const double il = 1.0 / sqrt(piv2);
            Lp[k * L + k] = il;
            S[p * L + k] = a;
            // bvec holds the forward solution z = L^-1 b of the support so
            // far; only its new element is computed
            double zk = bS[p];
            for (int j2 = 0; j2 < k; ++j2) zk -= Lp[k * L + j2] * bvec[p * L + j2];
            bvec[p * L + k] = zk * il;
            cnt[p] = k + 1;
            double yv[kLMax];
            for (int i = k; i >= 0; --i) {
              double s = bvec[p * L + i];
              for (int j2 = i + 1; j2 <= k; ++j2) s -= Lp[j2 * L + i] * yv[j2];
              yv[i] = s * Lp[i * L + i];
            }
            for (int i = 0; i <= k; ++i) gam[p * L + i] = float(yv[i]);
          }
        }
      }
      __syncthreads();
      // (4) residual r = y - D_S g (lanes over patches, warps over row chunks)
      {
        const int p = lane;
        const int rows = (n + 7) / 8;
        const int k0 = warp * rows, k1 = min(n, k0 + rows);
        float nrm = 0.0f;
        if (!done[p]) {
          const int kk = cnt[p];
          for (int k = k0; k < k1; ++k) {
            float r = Ys[p * ysn + k];
            for (int s2 = 0; s2 < kk; ++s2) r = fmaf(-gam[p * L + s2], Dk[k * dks + S[p * L + s2]], r);
            Rk[k * rks + p] = r;
            nrm = fmaf(r, r, nrm);
          }
        }
        npart[warp * kTP + p] = nrm;
      }
      __syncthreads();
      if (tid < kTP && !done[tid]) {
        float nrm = 0.0f;
        for (int w = 0; w < 8; ++w) nrm += npart[w * kTP + tid];
        if (sqrtf(nrm) < 1e-3f) done[tid] = 1;
      }
      __syncthreads();
      lap(9);
    }

    // ---- compact codes ------------------------------------------------------
    for (int t = tid; t < np * L; t += kOmpThreads) {
      const int p = t / L, s = t - p * L;
      const bool used = s < cnt[p];
      idx_out[(p0 + p) * L + s] = used ? S[p * L + s] : -1;
      coef_out[(p0 + p) * L + s] = used ? gam[p * L + s] : 0.0f;
    }
    // before an update sweep: the residual rows (Rk holds each patch's
    // residual with its final coefficients: a patch that stopped kept the
    // last one formed) and the highest support atom with a nonzero
    // coefficient
    if (R_out) {
      for (int t = tid; t < np * n; t += kOmpThreads) {
        const int p = t / n, k = t - p * n;
        __stcg(R_out + (p0 + p) * n + k, Rk[k * rks + p]);
      }
      if (tid < np) {
        int top = -1;
        for (int s = 0; s < cnt[tid]; ++s)
          if (gam[tid * L + s] != 0.0f) top = max(top, S[tid * L + s]);
        last_out[p0 + tid] = top;
      }
    }
    __syncthreads();
    lap(10);
  }
  if (timer)
    for (int k = 0; k < 4; ++k) atomicAdd(&stats->phase_ns[8 + k], s_ph[k]);
}

size_t omp_fp32_smem_bytes(int n, int K, int L) { return omp_layout(n, K, L).total; }

bool omp_fp32_supported(int n, int K, int L) {
  return L >= 1 && L <= kLMax && n >= 1 && K >= 1 && omp_fp32_smem_bytes(n, K, L) <= 227 * 1024;
}

cudaError_t launch_omp_fp32(const float* patches, int64_t N, int n, const float* dict, const double* gram, int K,
                            int L, int32_t* idx, float* coef, int num_sms, DevStats* stats, cudaStream_t s,
                            float* resid_out, int* last_out) {
  size_t smem = omp_fp32_smem_bytes(n, K, L);
  cudaError_t e = cudaFuncSetAttribute(omp_fp32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  int64_t ntiles = (N + kTP - 1) / kTP;
  int grid = int(std::min<int64_t>(ntiles, num_sms));
  if (resid_out && !last_out) return cudaErrorInvalidValue;
  omp_fp32_kernel<<<grid, kOmpThreads, smem, s>>>(patches, N, n, dict, gram, K, L, idx, coef, ntiles, resid_out,
                                                  last_out, stats);
  return cudaGetLastError();
}

}  // namespace ksvd
