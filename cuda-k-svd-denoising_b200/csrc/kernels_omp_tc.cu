// Batched OMP with the correlation D^T R on the 5th-generation tensor cores
// (CuBlasMatrixOmp::work, cublas_matrix_omp.cu:107-402, BF16 form).
//
// Per CTA (persistent over tiles of 128 patches, one CTA per SM):
//   * the dictionary lives in shared memory as the BF16 B operand (atoms x n,
//     K-major, no swizzle: 8-row x 16-byte core matrices);
//   * each OMP step, one thread issues n/16 tcgen05.mma (M = 128 patches,
//     N = atoms, K = 16, BF16 inputs, FP32 accumulation in tensor memory) and
//     commits them to an mbarrier;
//   * the four threads of patch m own TMEM lane m and a quarter of its
//     columns each: they stream the correlations out of tensor memory
//     (tcgen05.ld), keep the atoms inside the 16-bit error window, and the
//     CTA re-scores every windowed candidate exactly,
//         c_a = d_a . y - sum_s g_s <d_a, d_s>   (FP64, FP32 inputs)
//     taking the largest, lowest atom index on ties (cublasIsamax,
//     :216-233);
//   * thread (m, 0) extends the Cholesky factor of the support Gram (FP64, from the FP64
//     dictionary Gram), solves for the coefficients (the reference's
//     pseudo-inverse, :269-339), forms the FP32 residual y - D_S g and its
//     norm (:352-393; stop when below 1e-3, :218) and writes the residual as
//     BF16 into the A operand of the next step.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "ksvd_internal.cuh"
#include "tcgen05_util.cuh"

namespace ksvd {

constexpr int kTcTile = 128;     // patches per tile = UMMA M = TMEM lanes
constexpr int kTcQ = 4;          // threads per patch (column quarters)
constexpr int kTcThreads = kTcTile * kTcQ;
// |c_tc - c| / (|r| |d|): both operands rounded to p-bit significands (2 x
// 2^-p) plus FP32 accumulation and subnormal slack.
constexpr float kErrBf16 = 2.0f / 256.0f + 4.0e-4f;
constexpr float kErrF16 = 2.0f / 2048.0f + 1.0e-4f;

// 16-bit operand element: BF16 (8-bit significand) or FP16 (11-bit).
template <bool F16>
struct Op16;
template <>
struct Op16<false> {
  static __device__ __forceinline__ unsigned short cvt(float x) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
  }
  static constexpr unsigned fmt = 1u;  // instruction-descriptor format code
  static constexpr float err = kErrBf16;
};
template <>
struct Op16<true> {
  static __device__ __forceinline__ unsigned short cvt(float x) { return __half_as_ushort(__float2half_rn(x)); }
  static constexpr unsigned fmt = 0u;
  static constexpr float err = kErrF16;
};

__device__ __forceinline__ void store8(unsigned char* dst, const unsigned short (&h)[8]) {
  uint4 v;
  v.x = unsigned(h[0]) | (unsigned(h[1]) << 16);
  v.y = unsigned(h[2]) | (unsigned(h[3]) << 16);
  v.z = unsigned(h[4]) | (unsigned(h[5]) << 16);
  v.w = unsigned(h[6]) | (unsigned(h[7]) << 16);
  *reinterpret_cast<uint4*>(dst) = v;
}

// Power of two 2^e with max_abs * 2^-e in [2^13, 2^14) (1 for max_abs == 0):
// scaling the A operand by 2^-e is exact and keeps FP16 far from overflow and
// from its subnormal range.
__device__ __forceinline__ float pow2_scale(float max_abs) {
  if (!(max_abs > 0.0f)) return 1.0f;
  int e;
  frexpf(max_abs, &e);  // max_abs = f * 2^e, f in [0.5, 1)
  return ldexpf(1.0f, e - 14);
}
constexpr int kTcLMax = 16;
constexpr unsigned long long kMmaWaitNs = 2000000000ull;

struct TcLayout {
  int Kp, np16, ysn, tri, qw;
  size_t off_b, off_a, off_y, off_lc, off_bv, off_s, off_gam, off_sum, off_pp, off_xq, off_bar, off_tmem, total;
  unsigned tmem_cols;
};

// Per-patch scalars shared by the patch's four threads.
struct TcPatch {
  int cnt, done;
  float rmean, rscale, rnorm, ysum;
  double yy;
};

// Exchange between the four threads of a patch.
struct TcX {
  float qmax[kTcQ];                 // largest tensor-core |c| per column quarter
  unsigned long long qmask[kTcQ];   // columns of each quarter inside the error window
  float2 part[kTcQ];                // residual partial norms (all, centred)
  double best, best_b;              // exact best |c| and its d_a . y
  int best_a, ncand;                // its atom; number of candidates this step
  int noff, pad;                    // offset of the candidates in the tile's list
};

__host__ __device__ inline size_t tc_al(size_t x, size_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline TcLayout tc_layout(int n, int K, int L) {
  TcLayout o;
  o.Kp = int(tc_al(K, 16));
  o.np16 = int(tc_al(n, 16));
  o.ysn = n + 1;
  o.tri = L * (L + 1) / 2;
  size_t off = 0;
  o.off_b = off;
  off = tc_al(off + size_t(o.Kp) * o.np16 * 2, 128);
  o.off_a = off;
  off = tc_al(off + size_t(kTcTile) * o.np16 * 2, 128);
  o.off_y = off;
  off = tc_al(off + size_t(kTcTile) * o.ysn * 4, 16);
  o.off_lc = off;
  off = tc_al(off + size_t(kTcTile) * o.tri * 8, 16);
  o.off_bv = off;
  off = tc_al(off + size_t(kTcTile) * L * 8, 16);
  o.off_s = off;
  off = tc_al(off + size_t(kTcTile) * L * 4, 16);
  o.off_gam = off;
  off = tc_al(off + size_t(kTcTile) * L * 4, 16);
  o.off_sum = off;
  off = tc_al(off + size_t(o.Kp) * 4, 16);
  o.off_pp = off;
  off = tc_al(off + size_t(kTcTile) * sizeof(TcPatch), 16);
  o.off_xq = off;
  off = tc_al(off + size_t(kTcTile) * sizeof(TcX), 16);
  o.off_bar = off;
  off = tc_al(off + 16, 16);
  o.off_tmem = off;
  off = tc_al(off + 16, 16);
  o.total = off;
  unsigned cols = 32;
  while (cols < unsigned(o.Kp)) cols <<= 1;
  o.tmem_cols = cols;
  o.qw = int(tc_al((o.Kp + kTcQ - 1) / kTcQ, 16));  // columns per quarter, 16-column loads
  return o;
}

template <bool F16>
__global__ void __launch_bounds__(kTcThreads, 1)
    omp_tc_kernel(const float* __restrict__ Y, int64_t N, int n, const float* __restrict__ D,
                  const double* __restrict__ Gram, int K, int L, int32_t* __restrict__ idx_out,
                  float* __restrict__ coef_out, int64_t ntiles, int d_vec4, float* __restrict__ R_out,
                  int* __restrict__ last_out, int64_t* __restrict__ fix_list,
                  unsigned long long* __restrict__ fix_count, int r_vec4, GridBarrier* flags, DevStats* stats) {
  extern __shared__ __align__(128) unsigned char smem[];
  const TcLayout lo = tc_layout(n, K, L);
  unsigned char* Bt = smem + lo.off_b;
  unsigned char* At = smem + lo.off_a;
  float* Ys = reinterpret_cast<float*>(smem + lo.off_y);
  double* Lc = reinterpret_cast<double*>(smem + lo.off_lc);
  double* bv = reinterpret_cast<double*>(smem + lo.off_bv);
  int* Ss = reinterpret_cast<int*>(smem + lo.off_s);
  float* gam = reinterpret_cast<float*>(smem + lo.off_gam);
  float* asum = reinterpret_cast<float*>(smem + lo.off_sum);  // sum_k d_a[k] per atom
  TcPatch* pp = reinterpret_cast<TcPatch*>(smem + lo.off_pp);
  TcX* xq = reinterpret_cast<TcX*>(smem + lo.off_xq);
  unsigned long long* mbar = reinterpret_cast<unsigned long long*>(smem + lo.off_bar);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(smem + lo.off_tmem);
  // candidate list of the re-score, in the A operand's buffer: |c| and d . y
  // (FP64), then the packed (patch << 24 | atom) entries
  const int capl = int((size_t(kTcTile) * lo.np16 * 2) / 20);
  double* lcs = reinterpret_cast<double*>(At);
  double* lbs = lcs + capl;
  int* lpk = reinterpret_cast<int*>(lbs + capl);
  __shared__ int s_wtot[4];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Kp = lo.Kp, np16 = lo.np16, ysn = lo.ysn, tri = lo.tri, qw = lo.qw;
  const int nkc = np16 / 8;

  // ---- set-up: TMEM, mbarrier, 16-bit dictionary operand, atom sums --------
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(lo.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(mbar, 1);
    fence_mbar_init();
  }
  for (int t = tid; t < Kp * nkc; t += kTcThreads) {
    const int a = t / nkc, kc = t - a * nkc;
    unsigned short h[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int k = kc * 8 + e;
      h[e] = Op16<F16>::cvt((a < K && k < n) ? __ldg(D + int64_t(a) * n + k) : 0.0f);
    }
    store8(Bt + canon_off(a, kc * 8, Kp), h);
  }
  for (int a = tid; a < Kp; a += kTcThreads) {
    float sa = 0.0f;
    if (a < K)
      for (int k = 0; k < n; ++k) sa += __ldg(D + int64_t(a) * n + k);
    asum[a] = sa;
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;
  const unsigned idesc = umma_idesc_16(kTcTile, Kp, Op16<F16>::fmt);
  const unsigned a_base = smem_u32(At), b_base = smem_u32(Bt);
  unsigned phase = 0;
  bool failed = false;

  // thread roles: patch m = 32 g + lane (TMEM lane), quarter q of the columns
  // and of the residual chunks
  const int g = warp & 3, q = warp >> 2;
  const int m = g * 32 + lane;
  const unsigned lane_addr = tmem + (unsigned(g * 32) << 16);
  const int c_lo = q * qw, c_hi = min(Kp, c_lo + qw);
  const int kc_lo = (nkc * q) / kTcQ, kc_hi = (nkc * (q + 1)) / kTcQ;
  TcPatch& P = pp[m];
  TcX& X = xq[m];
  const float* yr = Ys + m * ysn;
  double* Lp = Lc + m * tri;
  auto Lat = [&](int i, int j) -> double& { return Lp[i * (i + 1) / 2 + j]; };

  const bool timer = (blockIdx.x == 0 && tid == 0 && stats != nullptr);
  // phase times (slots 8..12) gather in shared memory, flushed once at the end
  __shared__ unsigned long long s_ph[5];
  if (timer)
    for (int k = 0; k < 5; ++k) s_ph[k] = 0ull;
  unsigned long long tmark = timer ? globaltimer_ns() : 0ull;
  auto lap = [&](int slot) {
    if (timer) {
      const unsigned long long t = globaltimer_ns();
      s_ph[slot - 8] += t - tmark;
      tmark = t;
    }
  };
  int nscored = 0;
  int64_t p0 = 0;  // first patch of the current tile
  // chunk kc of patch m's residual row into R_out
  auto store_row_chunk = [&](int kc, const float (&r)[8]) {
    float* dst = R_out + (p0 + m) * int64_t(n) + kc * 8;
    if (r_vec4 && kc * 8 + 8 <= n) {
      __stcg(reinterpret_cast<float4*>(dst), make_float4(r[0], r[1], r[2], r[3]));
      __stcg(reinterpret_cast<float4*>(dst) + 1, make_float4(r[4], r[5], r[6], r[7]));
    } else {
#pragma unroll
      for (int e = 0; e < 8; ++e)
        if (kc * 8 + e < n) __stcg(dst + e, r[e]);
    }
  };

  for (int64_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    p0 = tile * kTcTile;
    const int np = (N - p0 < kTcTile) ? int(N - p0) : kTcTile;
    for (int t = tid; t < kTcTile * n; t += kTcThreads) {
      const int p = t / n, k = t - p * n;
      Ys[p * ysn + k] = (p < np) ? __ldg(Y + p0 * n + t) : 0.0f;
    }
    if (tid == 0 && tile + gridDim.x < ntiles) {
      // this CTA's next tile of patches into L2 while this one is worked on
      const int64_t pn = p0 + int64_t(gridDim.x) * kTcTile;
      const int64_t np_next = (N - pn < kTcTile) ? N - pn : kTcTile;
      const float* src = Y + pn * n;
      const unsigned bytes = unsigned(np_next * n * 4) & ~15u;
      if ((reinterpret_cast<uintptr_t>(src) & 15) == 0 && bytes > 0) bulk_prefetch_l2(src, bytes);
    }
    __syncthreads();
    // per-patch sums, a quarter of the features per thread (combined in a
    // fixed order), then the first A operand row
    {
      float ys = 0.0f;
      double yy = 0.0;
      for (int k = q; k < n; k += kTcQ) {
        ys += yr[k];
        yy = fma(double(yr[k]), double(yr[k]), yy);
      }
      X.part[q].x = ys;
      X.qmask[q] = static_cast<unsigned long long>(__double_as_longlong(yy));
    }
    __syncthreads();
    {
      const float ys = (X.part[0].x + X.part[1].x) + (X.part[2].x + X.part[3].x);
      const float mean = ys / float(n);
      float mx = 0.0f, cc = 0.0f;
      for (int k = q; k < n; k += kTcQ) {
        const float c = yr[k] - mean;
        mx = fmaxf(mx, fabsf(c));
        cc = fmaf(c, c, cc);
      }
      __syncthreads();  // every quarter has read the sums
      X.part[q] = make_float2(mx, cc);
      __syncthreads();
      if (q == 0) {
        double yy = 0.0;
#pragma unroll
        for (int j = 0; j < kTcQ; ++j) yy += __longlong_as_double(static_cast<long long>(X.qmask[j]));
        P.cnt = 0;
        P.done = m >= np;
        P.ysum = ys;
        P.yy = yy;
        P.rmean = mean;
        P.rscale = pow2_scale(fmaxf(fmaxf(X.part[0].x, X.part[1].x), fmaxf(X.part[2].x, X.part[3].x)));
        P.rnorm = sqrtf((X.part[0].y + X.part[1].y) + (X.part[2].y + X.part[3].y));
      }
    }
    __syncthreads();
    {
      const float mean = P.rmean, inv = 1.0f / P.rscale;
      for (int kc = kc_lo; kc < kc_hi; ++kc) {
        unsigned short h[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int k = kc * 8 + e;
          h[e] = Op16<F16>::cvt(k < n ? (yr[k] - mean) * inv : 0.0f);
        }
        store8(At + canon_off(m, kc * 8, kTcTile), h);
      }
    }
    lap(10);
    for (int step = 0; step < L; ++step) {
      fence_proxy_async_smem();
      tc_fence_before();
      if (!__syncthreads_or(!P.done)) break;
      lap(9);
      // ---- correlation on the tensor cores ---------------------------------
      if (tid == 0) {
        tc_fence_after();
        for (int kk = 0; kk < np16 / 16; ++kk) {
          const unsigned long long ad = umma_desc(a_base + kk * 2 * kTcTile * 16, kTcTile * 16, 128);
          const unsigned long long bd = umma_desc(b_base + kk * 2 * Kp * 16, Kp * 16, 128);
          tc_mma(tmem, ad, bd, idesc, kk > 0 ? 1u : 0u);
        }
        tc_commit(mbar);
      }
      const bool ok = mbar_wait(mbar, phase, kMmaWaitNs);
      phase ^= 1u;
      if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicCAS(&flags->err, DEVERR_NONE, DEVERR_TIMEOUT);
        failed = true;
        phase ^= 1u;  // the drain waits for the phase that did not complete
        break;
      }
      tc_fence_after();
      lap(8);
      // ---- this quarter's correlations (tensor part + exact mean part) -----
      const bool done = P.done != 0;
      const float rmean = P.rmean, rscale = P.rscale;
      float cv[64];  // up to 64 columns per quarter (Kp <= 256)
      float qmax = -1.0f;
      if (c_lo < Kp) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (c_lo + 16 * j < c_hi) {
            float v[16];
            tc_ld16(lane_addr + unsigned(c_lo + 16 * j), v);
            tc_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int a = c_lo + 16 * j + i;
              const float c = (a < K) ? fabsf(fmaf(rmean, asum[a], v[i] * rscale)) : -1.0f;
              cv[16 * j + i] = c;
              qmax = fmaxf(qmax, c);
            }
          }
        }
      }
      X.qmax[q] = qmax;
      __syncthreads();
      // ---- candidates: atoms inside the error window -----------------------
      // |c_tc - c| <= err |r - rmean 1| |d|, so the exact argmax is among the
      // atoms with c_tc >= max c_tc - 2 err |r - rmean 1|.
      {
        unsigned long long mask = 0ull;
        if (!done && c_lo < Kp) {
          float gmax = X.qmax[0];
#pragma unroll
          for (int j = 1; j < kTcQ; ++j) gmax = fmaxf(gmax, X.qmax[j]);
          const float thr = gmax - 2.0f * Op16<F16>::err * P.rnorm;
#pragma unroll
          for (int i = 0; i < 64; ++i) {
            const int a = c_lo + i;
            if (a < c_hi && a < K && cv[i] >= thr) mask |= 1ull << i;
          }
        }
        X.qmask[q] = mask;
      }
      __syncthreads();
      // ---- exact re-score of every candidate of the tile ------------------
      // The tile's (patch, atom) candidates form one list, kept in the A
      // operand's buffer (free between the MMA and the residual update), and
      // four consecutive lanes score each entry:
      //   b_a = d_a . y (FP64 from FP32 data),  c_a = b_a - sum_s g_s G[a][s];
      // each patch then takes its largest |c_a|, lowest atom index on ties.
      {
        if (q == 0) {  // candidate counts and list offsets (warps 0..3)
          int cntm = 0;
          if (!done)
#pragma unroll
            for (int qq = 0; qq < kTcQ; ++qq) cntm += __popcll(X.qmask[qq]);
          int incl = cntm;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
          }
          if (lane == 31) s_wtot[g] = incl;
          X.ncand = cntm;
          X.noff = incl - cntm;
          X.best = -1.0;
          X.best_a = 0x7fffffff;
          X.best_b = 0.0;
        }
        __syncthreads();
        const int total = s_wtot[0] + s_wtot[1] + s_wtot[2] + s_wtot[3];
        if (q == 0)
          for (int w = 0; w < g; ++w) X.noff += s_wtot[w];
        const int grp = tid >> 2, js = tid & 3;
        const unsigned gmask = 0xFu << (lane & ~3);
        for (int rb = 0; rb < total; rb += capl) {
          const int rh = min(total, rb + capl);
          if (q == 0 && X.ncand > 0 && X.noff < rh && X.noff + X.ncand > rb) {
            int li = X.noff;  // ascending atom order
            for (int qq = 0; qq < kTcQ && li < rh; ++qq) {
              unsigned long long mk = X.qmask[qq];
              while (mk && li < rh) {
                const int a = qq * qw + (__ffsll((long long)mk) - 1);
                mk &= mk - 1ull;
                if (li >= rb) lpk[li - rb] = (m << 24) | a;
                ++li;
              }
            }
          }
          __syncthreads();
          for (int t = grp; t < rh - rb; t += kTcThreads / 4) {
            const int v = lpk[t];
            const int ps = v >> 24, a = v & 0xFFFFFF;
            const float* yrs = Ys + ps * ysn;
            const int cnt = pp[ps].cnt;
            double gs = 0.0;  // support part, lanes js, js + 4, ...
            for (int s2 = js; s2 < cnt; s2 += 4)
              gs = fma(double(gam[ps * L + s2]), Gram[int64_t(a) * K + Ss[ps * L + s2]], gs);
            double b0 = 0.0, b1 = 0.0;
            if (d_vec4) {
              const float4* dr = reinterpret_cast<const float4*>(D + int64_t(a) * n);
              const int n4 = n / 4;
              for (int k0 = js; k0 < n4; k0 += 16) {
                float4 dv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                  const int k4 = k0 + 4 * u;
                  dv[u] = (k4 < n4) ? __ldg(dr + k4) : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                  const int k4 = k0 + 4 * u;
                  if (k4 < n4) {
                    const float* yv = yrs + 4 * k4;
                    b0 = fma(double(dv[u].x), double(yv[0]), b0);
                    b1 = fma(double(dv[u].y), double(yv[1]), b1);
                    b0 = fma(double(dv[u].z), double(yv[2]), b0);
                    b1 = fma(double(dv[u].w), double(yv[3]), b1);
                  }
                }
              }
            } else {
              for (int k = js; k < n; k += 4) b0 = fma(double(__ldg(D + int64_t(a) * n + k)), double(yrs[k]), b0);
            }
            double ba = b0 + b1;
            ba += __shfl_xor_sync(gmask, ba, 1);
            ba += __shfl_xor_sync(gmask, ba, 2);
            gs += __shfl_xor_sync(gmask, gs, 1);
            gs += __shfl_xor_sync(gmask, gs, 2);
            if (js == 0) {
              lcs[t] = fabs(ba - gs);
              lbs[t] = ba;
              ++nscored;
            }
          }
          __syncthreads();
          if (q == 0 && X.ncand > 0) {
            const int lo = max(X.noff, rb), hi = min(X.noff + X.ncand, rh);
            for (int t = lo; t < hi; ++t) {
              const double aca = lcs[t - rb];
              const int a = lpk[t - rb] & 0xFFFFFF;
              if (aca > X.best || (aca == X.best && a < X.best_a)) {
                X.best = aca;
                X.best_a = a;
                X.best_b = lbs[t - rb];
              }
            }
          }
          __syncthreads();
        }
      }
      __syncthreads();
      lap(11);
      // ---- quarter 0: selection, Cholesky append, solve, residual scale ----
      if (q == 0 && !done) {
        const double bbb = X.best_b;
        const int ba = X.best_a;
        const int a = (ba >= 0 && ba < K) ? ba : 0;
        const int k = P.cnt;
        bool stop = false;
        for (int s2 = 0; s2 < k; ++s2)
          if (Ss[m * L + s2] == a) stop = true;  // re-selected atom: the pursuit ends
        if (!stop) {
          double ww = 0.0;
          for (int i = 0; i < k; ++i) {
            double s3 = Gram[int64_t(Ss[m * L + i]) * K + a];
            for (int j = 0; j < i; ++j) s3 -= Lat(i, j) * Lat(k, j);
            const double wi = s3 * Lat(i, i);  // the diagonal is kept as 1 / L_ii
            Lat(k, i) = wi;
            ww += wi * wi;
          }
          const double piv2 = Gram[int64_t(a) * K + a] - ww;
          if (!(piv2 > 0.0)) {
            stop = true;  // the new atom depends linearly on the support
          } else {
            Lat(k, k) = 1.0 / sqrt(piv2);
            Ss[m * L + k] = a;
            // bv holds the forward solution z = L^-1 b of the support so far;
            // only its new element is computed
            double zk = bbb;
            for (int j = 0; j < k; ++j) zk -= Lat(k, j) * bv[m * L + j];
            zk *= Lat(k, k);
            bv[m * L + k] = zk;
            double yv[kTcLMax];
            for (int i = k; i >= 0; --i) {
              double s3 = bv[m * L + i];
              for (int j = i + 1; j <= k; ++j) s3 -= Lat(j, i) * yv[j];
              yv[i] = s3 * Lat(i, i);
            }
            for (int i = 0; i <= k; ++i) gam[m * L + i] = float(yv[i]);
            const int kk = k + 1;
            P.cnt = kk;
            // |r|^2 = |y|^2 - |L^-1 b|^2 (least squares) bounds |r - rmean|;
            // mean of r from the patch sum and the atom sums
            double rr = P.yy;
            float rs = P.ysum;
            for (int i = 0; i < kk; ++i) {
              rr -= bv[m * L + i] * bv[m * L + i];
              rs = fmaf(-gam[m * L + i], asum[Ss[m * L + i]], rs);
            }
            P.rmean = rs / float(n);
            P.rscale = pow2_scale(float(sqrt(fmax(rr, 0.0))) * 1.01f + 1e-30f);
          }
        }
        if (stop) P.done = 1;
      }
      __syncthreads();
      lap(12);
      // ---- residual quarter (FP32), partial norms, next A operand -----------
      // (with the patch's final coefficients, the row also goes to R_out)
      const bool live = !done && !P.done;
      float nrm = 0.0f, cn = 0.0f;
      if (live) {
        const int cnt = P.cnt;
        const bool fin = R_out != nullptr && cnt == L;
        const float mean = P.rmean, inv = 1.0f / P.rscale;
        for (int kc = kc_lo; kc < kc_hi; ++kc) {
          float r[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const int kk = kc * 8 + e;
            r[e] = (kk < n) ? yr[kk] : 0.0f;
          }
          if (d_vec4 && kc * 8 + 8 <= n) {
            // the chunk of every support atom is loaded before it is used
            constexpr int kSB = 2;
            for (int s0 = 0; s0 < cnt; s0 += kSB) {
              float4 da[kSB], db[kSB];
              float gg[kSB];
#pragma unroll
              for (int u = 0; u < kSB; ++u) {
                const int s2 = s0 + u;
                if (s2 < cnt) {
                  const float4* dr = reinterpret_cast<const float4*>(D + int64_t(Ss[m * L + s2]) * n + kc * 8);
                  gg[u] = gam[m * L + s2];
                  da[u] = __ldg(dr);
                  db[u] = __ldg(dr + 1);
                }
              }
#pragma unroll
              for (int u = 0; u < kSB; ++u) {
                if (s0 + u < cnt) {
                  r[0] = fmaf(-gg[u], da[u].x, r[0]);
                  r[1] = fmaf(-gg[u], da[u].y, r[1]);
                  r[2] = fmaf(-gg[u], da[u].z, r[2]);
                  r[3] = fmaf(-gg[u], da[u].w, r[3]);
                  r[4] = fmaf(-gg[u], db[u].x, r[4]);
                  r[5] = fmaf(-gg[u], db[u].y, r[5]);
                  r[6] = fmaf(-gg[u], db[u].z, r[6]);
                  r[7] = fmaf(-gg[u], db[u].w, r[7]);
                }
              }
            }
          } else {
            for (int s2 = 0; s2 < cnt; ++s2) {
              const float gg = gam[m * L + s2];
              const float* dr = D + int64_t(Ss[m * L + s2]) * n + kc * 8;
#pragma unroll
              for (int e = 0; e < 8; ++e)
                if (kc * 8 + e < n) r[e] = fmaf(-gg, __ldg(dr + e), r[e]);
            }
          }
          if (fin) store_row_chunk(kc, r);
          unsigned short h[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const bool in = kc * 8 + e < n;
            nrm = fmaf(r[e], r[e], nrm);
            const float c = in ? r[e] - mean : 0.0f;
            cn = fmaf(c, c, cn);
            h[e] = Op16<F16>::cvt(c * inv);
          }
          store8(At + canon_off(m, kc * 8, kTcTile), h);
        }
      }
      float2* part = X.part;
      part[q] = make_float2(nrm, cn);
      __syncthreads();
      if (q == 0 && live) {
        float tn = 0.0f, tc = 0.0f;
        for (int j = 0; j < kTcQ; ++j) {
          tn += part[j].x;
          tc += part[j].y;
        }
        P.rnorm = sqrtf(tc);
        if (sqrtf(tn) < 1e-3f) P.done = 1;
      }
      lap(9);
    }
    // ---- compact codes ------------------------------------------------------
    __syncthreads();
    if (q == 0 && m < np) {
      const int cnt = P.cnt;
      int top = -1;  // highest support atom with a nonzero coefficient
      for (int s2 = 0; s2 < L; ++s2) {
        const bool used = s2 < cnt;
        idx_out[(p0 + m) * L + s2] = used ? Ss[m * L + s2] : -1;
        coef_out[(p0 + m) * L + s2] = used ? gam[m * L + s2] : 0.0f;
        if (used && gam[m * L + s2] != 0.0f) top = max(top, Ss[m * L + s2]);
      }
      if (last_out) last_out[p0 + m] = top;
    }
    // patches that stopped before L atoms: their last residual pass ran with
    // earlier coefficients (or the pursuit ended in the Cholesky step), so
    // their rows are left to launch_residual over the list
    if (R_out && q == 0 && m < np && P.cnt < L) fix_list[atomicAdd(fix_count, 1ull)] = p0 + m;
    __syncthreads();
  }
  if (stats && nscored) atomicAdd(&stats->pad, (unsigned long long)nscored);
  if (timer)
    for (int k = 0; k < 5; ++k) atomicAdd(&stats->phase_ns[8 + k], s_ph[k]);
  // ---- teardown --------------------------------------------------------------
  if (failed && tid == 0) mbar_wait(mbar, phase, kMmaWaitNs);  // bounded drain of MMAs in flight
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(lo.tmem_cols) : "memory");
  }
}

size_t omp_tc_smem_bytes(int n, int K, int L) { return tc_layout(n, K, L).total; }

template __global__ void omp_tc_kernel<false>(const float*, int64_t, int, const float*, const double*, int, int,
                                              int32_t*, float*, int64_t, int, float*, int*, int64_t*,
                                              unsigned long long*, int, GridBarrier*, DevStats*);
template __global__ void omp_tc_kernel<true>(const float*, int64_t, int, const float*, const double*, int, int,
                                             int32_t*, float*, int64_t, int, float*, int*, int64_t*,
                                             unsigned long long*, int, GridBarrier*, DevStats*);

bool omp_tc_supported(int n, int K, int L) {
  return L >= 1 && L <= kTcLMax && n >= 1 && K >= 1 && tc_al(K, 16) <= 256 &&
         omp_tc_smem_bytes(n, K, L) <= 232448 - 256;
}

cudaError_t launch_omp_tc(const float* patches, int64_t N, int n, const float* dict, const double* gram, int K, int L,
                          int32_t* idx, float* coef, int num_sms, int fp16, GridBarrier* flags, DevStats* stats,
                          cudaStream_t s, float* resid_out, int* last_out, int64_t* fix_list,
                          unsigned long long* fix_count) {
  const size_t smem = omp_tc_smem_bytes(n, K, L);
  auto kern = fp16 ? omp_tc_kernel<true> : omp_tc_kernel<false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const int64_t ntiles = (N + kTcTile - 1) / kTcTile;
  const int grid = int(std::min<int64_t>(ntiles, num_sms));
  const int d_vec4 = ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(dict) & 15) == 0) ? 1 : 0;
  const int r_vec4 = ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(resid_out) & 15) == 0) ? 1 : 0;
  if (resid_out && (!last_out || !fix_list || !fix_count)) return cudaErrorInvalidValue;
  kern<<<grid, kTcThreads, smem, s>>>(patches, N, n, dict, gram, K, L, idx, coef, ntiles, d_vec4, resid_out, last_out,
                                      fix_list, fix_count, r_vec4, flags, stats);
  return cudaGetLastError();
}

}  // namespace ksvd
