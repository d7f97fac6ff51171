// Batched OMP with the 16-bit tensor-core correlation for dictionaries too
// large for the resident-dictionary kernel (kernels_omp_tc.cu): up to 512
// atoms and patches of up to 256 values (CuBlasMatrixOmp::work,
// cublas_matrix_omp.cu:107-402, with the correlation of :193-206 on the
// tensor cores).
//
// Same pursuit and exact re-score as the resident kernel; what changes:
//   * the 16-bit dictionary (B operand, atoms x n) is built once per call in
//     global memory in the no-swizzle K-major canonical layout, so that the
//     16 features of one MMA K-slice are one contiguous block of 32 Kp bytes;
//     each OMP step streams those blocks through a ring of shared-memory
//     slots with 1-D bulk copies (thread 0 issues both the copies and the
//     MMAs; a slot is refilled once the MMA that read it has committed);
//   * the accumulator takes up to 512 TMEM columns (M = 128 patches, N = Kp,
//     as up to two MMAs per K-slice: UMMA N is at most 256 with M = 128;
//     atoms 256.. go to TMEM columns 256..);
//     the epilogue reads each thread's quarter of the columns twice (largest
//     |c| first, then the candidates inside the error window) instead of
//     holding it in registers;
//   * the FP32 patches stay in global memory (L2) instead of shared memory:
//     the exact re-scores and the residual read them there.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "ksvd_internal.cuh"
#include "tcgen05_util.cuh"

namespace ksvd {

constexpr int kTbTile = 128;  // patches per tile = UMMA M = TMEM lanes
constexpr int kTbQ = 4;       // threads per patch (column quarters)
constexpr int kTbThreads = kTbTile * kTbQ;
constexpr int kTbSlots = 4;   // ring of K-slices
constexpr int kTbLMax = 16;
constexpr int kTbMaxK = 512;
constexpr int kTbMaxN = 512;
constexpr unsigned long long kTbWaitNs = 2000000000ull;
constexpr float kTbErrBf16 = 2.0f / 256.0f + 4.0e-4f;
constexpr float kTbErrF16 = 2.0f / 2048.0f + 1.0e-4f;

template <bool F16>
struct TbOp;
template <>
struct TbOp<false> {
  static __device__ __forceinline__ unsigned short cvt(float x) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(x));
  }
  static constexpr unsigned fmt = 1u;
  static constexpr float err = kTbErrBf16;
};
template <>
struct TbOp<true> {
  static __device__ __forceinline__ unsigned short cvt(float x) { return __half_as_ushort(__float2half_rn(x)); }
  static constexpr unsigned fmt = 0u;
  static constexpr float err = kTbErrF16;
};

__device__ __forceinline__ void tb_store8(unsigned char* dst, const unsigned short (&h)[8]) {
  uint4 v;
  v.x = unsigned(h[0]) | (unsigned(h[1]) << 16);
  v.y = unsigned(h[2]) | (unsigned(h[3]) << 16);
  v.z = unsigned(h[4]) | (unsigned(h[5]) << 16);
  v.w = unsigned(h[6]) | (unsigned(h[7]) << 16);
  *reinterpret_cast<uint4*>(dst) = v;
}

__device__ __forceinline__ float tb_pow2_scale(float max_abs) {
  if (!(max_abs > 0.0f)) return 1.0f;
  int e;
  frexpf(max_abs, &e);
  return ldexpf(1.0f, e - 14);
}

struct TbPatch {
  int cnt, done;
  float rmean, rscale, rnorm, ysum;
  double yy;
};

struct TbX {
  float qmax[kTbQ];
  unsigned long long qmask[kTbQ][2];  // candidate columns of each quarter (128 columns)
  float2 part[kTbQ];
  double best, best_b;
  int best_a, ncand;
  int noff, pad;
};

__host__ __device__ inline size_t tb_al(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct TbLayout {
  int Kp, np16, tri, qw;
  size_t slot_bytes;
  size_t off_ring, off_a, off_lc, off_bv, off_s, off_gam, off_sum, off_pp, off_xq, off_bar, off_tmem, total;
  unsigned tmem_cols;
};

__host__ __device__ inline TbLayout tb_layout(int n, int K, int L) {
  TbLayout o;
  o.Kp = int(tb_al(K, 16));
  o.np16 = int(tb_al(n, 16));
  o.tri = L * (L + 1) / 2;
  o.slot_bytes = size_t(o.Kp) * 16 * 2;  // one K-slice of 16 features
  size_t off = 0;
  o.off_ring = off;
  off = tb_al(off + size_t(kTbSlots) * o.slot_bytes, 128);
  o.off_a = off;
  off = tb_al(off + size_t(kTbTile) * o.np16 * 2, 128);
  o.off_lc = off;
  off = tb_al(off + size_t(kTbTile) * o.tri * 8, 16);
  o.off_bv = off;
  off = tb_al(off + size_t(kTbTile) * L * 8, 16);
  o.off_s = off;
  off = tb_al(off + size_t(kTbTile) * L * 4, 16);
  o.off_gam = off;
  off = tb_al(off + size_t(kTbTile) * L * 4, 16);
  o.off_sum = off;
  off = tb_al(off + size_t(o.Kp) * 4, 16);
  o.off_pp = off;
  off = tb_al(off + size_t(kTbTile) * sizeof(TbPatch), 16);
  o.off_xq = off;
  off = tb_al(off + size_t(kTbTile) * sizeof(TbX), 16);
  o.off_bar = off;
  off = tb_al(off + 8 * (2 * kTbSlots + 1), 16);
  o.off_tmem = off;
  off = tb_al(off + 16, 16);
  o.total = off;
  unsigned cols = 32;
  while (cols < unsigned(o.Kp)) cols <<= 1;
  o.tmem_cols = cols;
  o.qw = int(tb_al((o.Kp + kTbQ - 1) / kTbQ, 16));  // <= 128
  return o;
}

// The 16-bit dictionary (Kp x np16, canonical K-major layout, zero padding)
// and the atom sums in global memory.
template <bool F16>
__global__ void tb_prep_kernel(const float* __restrict__ D, int K, int n, int Kp, int np16,
                               unsigned char* __restrict__ Bg, float* __restrict__ asum) {
  const int nkc = np16 / 8;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < Kp * nkc; t += gridDim.x * blockDim.x) {
    const int a = t / nkc, kc = t - a * nkc;
    unsigned short h[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int k = kc * 8 + e;
      h[e] = TbOp<F16>::cvt((a < K && k < n) ? __ldg(D + int64_t(a) * n + k) : 0.0f);
    }
    tb_store8(Bg + canon_off(a, kc * 8, Kp), h);
  }
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < Kp; a += gridDim.x * blockDim.x) {
    float sa = 0.0f;
    if (a < K)
      for (int k = 0; k < n; ++k) sa += __ldg(D + int64_t(a) * n + k);
    asum[a] = sa;
  }
}

template <bool F16>
__global__ void __launch_bounds__(kTbThreads, 1)
    omp_tcb_kernel(const float* __restrict__ Y, int64_t N, int n, const float* __restrict__ D,
                   const unsigned char* __restrict__ Bg, const float* __restrict__ asum_g,
                   const double* __restrict__ Gram, int K, int L, int32_t* __restrict__ idx_out,
                   float* __restrict__ coef_out, int64_t ntiles, int d_vec4, float* __restrict__ R_out,
                   int* __restrict__ last_out, int64_t* __restrict__ fix_list,
                   unsigned long long* __restrict__ fix_count, int r_vec4, GridBarrier* flags, DevStats* stats) {
  extern __shared__ __align__(128) unsigned char smem[];
  const TbLayout lo = tb_layout(n, K, L);
  unsigned char* ring = smem + lo.off_ring;
  unsigned char* At = smem + lo.off_a;
  double* Lc = reinterpret_cast<double*>(smem + lo.off_lc);
  double* bv = reinterpret_cast<double*>(smem + lo.off_bv);
  int* Ss = reinterpret_cast<int*>(smem + lo.off_s);
  float* gam = reinterpret_cast<float*>(smem + lo.off_gam);
  float* asum = reinterpret_cast<float*>(smem + lo.off_sum);
  TbPatch* pp = reinterpret_cast<TbPatch*>(smem + lo.off_pp);
  TbX* xq = reinterpret_cast<TbX*>(smem + lo.off_xq);
  unsigned long long* full = reinterpret_cast<unsigned long long*>(smem + lo.off_bar);
  unsigned long long* empty = full + kTbSlots;
  unsigned long long* done_bar = empty + kTbSlots;
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(smem + lo.off_tmem);
  const int capl = int((size_t(kTbTile) * lo.np16 * 2) / 20);
  double* lcs = reinterpret_cast<double*>(At);
  double* lbs = lcs + capl;
  int* lpk = reinterpret_cast<int*>(lbs + capl);
  __shared__ int s_wtot[4];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Kp = lo.Kp, np16 = lo.np16, tri = lo.tri, qw = lo.qw;
  const int nkc = np16 / 8, nks = np16 / 16;

  if (warp == 0) tc_alloc(tmem_slot, lo.tmem_cols);
  if (tid == 0) {
    for (int s = 0; s < kTbSlots; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(done_bar, 1);
    fence_mbar_init();
  }
  for (int a = tid; a < Kp; a += kTbThreads) asum[a] = asum_g[a];
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tmem_slot;
  // atoms [0, n0) and [256, 256 + n1): one MMA each per K-slice (N <= 256)
  const int n0 = Kp < 256 ? Kp : 256, n1 = Kp - n0;
  const unsigned idesc0 = umma_idesc_16(kTbTile, n0, TbOp<F16>::fmt);
  const unsigned idesc1 = umma_idesc_16(kTbTile, n1 > 0 ? n1 : 16, TbOp<F16>::fmt);
  const unsigned a_base = smem_u32(At);
  // ring bookkeeping (thread 0 only): slices issued / consumed over the
  // kernel's life; slice i uses slot i % kTbSlots
  unsigned long long issued = 0, consumed = 0;
  unsigned full_par = 0, empty_par = 0, done_par = 0;  // per-slot parity bits / done barrier parity
  unsigned empty_pending = 0;                           // slots whose MMA commit is not yet waited for
  bool failed = false;

  const int g = warp & 3, q = warp >> 2;
  const int m = g * 32 + lane;
  const unsigned lane_addr = tmem + (unsigned(g * 32) << 16);
  const int c_lo = q * qw, c_hi = min(Kp, c_lo + qw);
  const int kc_lo = (nkc * q) / kTbQ, kc_hi = (nkc * (q + 1)) / kTbQ;
  TbPatch& P = pp[m];
  TbX& X = xq[m];
  double* Lp = Lc + m * tri;
  auto Lat = [&](int i, int j) -> double& { return Lp[i * (i + 1) / 2 + j]; };
  int nscored = 0;

  // thread 0: one step of MMAs over all K-slices, streaming the slices
  auto mma_step = [&]() -> bool {
    const unsigned long long first = consumed;
    auto issue = [&](unsigned long long i) -> bool {
      const int s = int(i % kTbSlots);
      if (empty_pending & (1u << s)) {  // the slot's previous MMA must have read it
        if (!mbar_wait(empty + s, (empty_par >> s) & 1u, kTbWaitNs)) return false;
        empty_par ^= 1u << s;
        empty_pending &= ~(1u << s);
      }
      const int kk = int((i - first) % unsigned(nks));
      mbar_arrive_expect_tx(full + s, unsigned(lo.slot_bytes));
      bulk_g2s(ring + size_t(s) * lo.slot_bytes, Bg + size_t(kk) * lo.slot_bytes, unsigned(lo.slot_bytes), full + s);
      return true;
    };
    // prologue: fill the ring
    while (issued < first + kTbSlots && issued < first + nks) {
      if (!issue(issued)) return false;
      ++issued;
    }
    for (int kk = 0; kk < nks; ++kk) {
      const unsigned long long i = first + kk;
      const int s = int(i % kTbSlots);
      if (!mbar_wait(full + s, (full_par >> s) & 1u, kTbWaitNs)) return false;
      full_par ^= 1u << s;
      tc_fence_after();
      const unsigned long long ad = umma_desc(a_base + kk * 2 * kTbTile * 16, kTbTile * 16, 128);
      const unsigned slot = smem_u32(ring + size_t(s) * lo.slot_bytes);
      // rows 256.. of the slice start 256 / 8 core matrices (of 128 bytes) in
      tc_mma(tmem, ad, umma_desc(slot, Kp * 16, 128), idesc0, kk > 0 ? 1u : 0u);
      if (n1 > 0) tc_mma(tmem + 256u, ad, umma_desc(slot + (256 / 8) * 128, Kp * 16, 128), idesc1, kk > 0 ? 1u : 0u);
      tc_commit(empty + s);
      empty_pending |= 1u << s;
      ++consumed;
      if (issued < first + nks) {
        if (!issue(issued)) return false;
        ++issued;
      }
    }
    tc_commit(done_bar);
    if (!mbar_wait(done_bar, done_par, kTbWaitNs)) return false;
    done_par ^= 1u;
    return true;
  };

  for (int64_t tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    const int64_t p0 = tile * kTbTile;
    const int np = (N - p0 < kTbTile) ? int(N - p0) : kTbTile;
    const float* yg = Y + (p0 + (m < np ? m : 0)) * n;  // this patch's values (global)
    // per-patch sums over a quarter of the features
    {
      float ys = 0.0f;
      double yy = 0.0;
      if (m < np)
        for (int k = q; k < n; k += kTbQ) {
          const float v = __ldg(yg + k);
          ys += v;
          yy = fma(double(v), double(v), yy);
        }
      X.part[q].x = ys;
      X.qmask[q][0] = static_cast<unsigned long long>(__double_as_longlong(yy));
    }
    __syncthreads();
    {
      const float ys = (X.part[0].x + X.part[1].x) + (X.part[2].x + X.part[3].x);
      const float mean = ys / float(n);
      float mx = 0.0f, cc = 0.0f;
      if (m < np)
        for (int k = q; k < n; k += kTbQ) {
          const float c = __ldg(yg + k) - mean;
          mx = fmaxf(mx, fabsf(c));
          cc = fmaf(c, c, cc);
        }
      __syncthreads();
      X.part[q] = make_float2(mx, cc);
      __syncthreads();
      if (q == 0) {
        double yy = 0.0;
#pragma unroll
        for (int j = 0; j < kTbQ; ++j) yy += __longlong_as_double(static_cast<long long>(X.qmask[j][0]));
        P.cnt = 0;
        P.done = m >= np;
        P.ysum = ys;
        P.yy = yy;
        P.rmean = mean;
        P.rscale = tb_pow2_scale(fmaxf(fmaxf(X.part[0].x, X.part[1].x), fmaxf(X.part[2].x, X.part[3].x)));
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
          h[e] = TbOp<F16>::cvt((k < n && m < np) ? (__ldg(yg + k) - mean) * inv : 0.0f);
        }
        tb_store8(At + canon_off(m, kc * 8, kTbTile), h);
      }
    }
    for (int step = 0; step < L; ++step) {
      fence_proxy_async_smem();
      tc_fence_before();
      if (!__syncthreads_or(!P.done)) break;
      // ---- correlation on the tensor cores (dictionary streamed) -----------
      int ok = 1;
      if (tid == 0) {
        tc_fence_after();
        ok = mma_step() ? 1 : 0;
      }
      if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicCAS(&flags->err, DEVERR_NONE, DEVERR_TIMEOUT);
        failed = true;
        break;
      }
      tc_fence_after();
      // ---- pass 1: this quarter's largest |c| -------------------------------
      const bool done = P.done != 0;
      const float rmean = P.rmean, rscale = P.rscale;
      float qmax = -1.0f;
      for (int c0 = c_lo; c0 < c_hi; c0 += 16) {
        float v[16];
        tc_ld16(lane_addr + unsigned(c0), v);
        tc_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int a = c0 + i;
          if (a < K) qmax = fmaxf(qmax, fabsf(fmaf(rmean, asum[a], v[i] * rscale)));
        }
      }
      X.qmax[q] = qmax;
      __syncthreads();
      // ---- pass 2: candidates inside the error window -----------------------
      {
        unsigned long long mk0 = 0ull, mk1 = 0ull;
        float gmax = X.qmax[0];
#pragma unroll
        for (int j = 1; j < kTbQ; ++j) gmax = fmaxf(gmax, X.qmax[j]);
        const float thr = gmax - 2.0f * TbOp<F16>::err * P.rnorm;
        for (int c0 = c_lo; c0 < c_hi; c0 += 16) {
          float v[16];
          tc_ld16(lane_addr + unsigned(c0), v);
          tc_wait_ld();
          if (!done) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
              const int a = c0 + i;
              const int bit = a - c_lo;
              if (a < K && fabsf(fmaf(rmean, asum[a], v[i] * rscale)) >= thr) {
                if (bit < 64)
                  mk0 |= 1ull << bit;
                else
                  mk1 |= 1ull << (bit - 64);
              }
            }
          }
        }
        X.qmask[q][0] = mk0;
        X.qmask[q][1] = mk1;
      }
      __syncthreads();
      // ---- exact re-score of every candidate of the tile ------------------
      {
        if (q == 0) {
          int cntm = 0;
          if (!done)
#pragma unroll
            for (int qq = 0; qq < kTbQ; ++qq) cntm += __popcll(X.qmask[qq][0]) + __popcll(X.qmask[qq][1]);
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
            for (int qq = 0; qq < kTbQ && li < rh; ++qq)
              for (int w2 = 0; w2 < 2 && li < rh; ++w2) {
                unsigned long long mk = X.qmask[qq][w2];
                while (mk && li < rh) {
                  const int a = qq * qw + w2 * 64 + (__ffsll((long long)mk) - 1);
                  mk &= mk - 1ull;
                  if (li >= rb) lpk[li - rb] = (m << 24) | a;
                  ++li;
                }
              }
          }
          __syncthreads();
          for (int t = grp; t < rh - rb; t += kTbThreads / 4) {
            const int v = lpk[t];
            const int ps = v >> 24, a = v & 0xFFFFFF;
            const float* yrs = Y + (p0 + ps) * n;
            const int cnt = pp[ps].cnt;
            double gs = 0.0;
            for (int s2 = js; s2 < cnt; s2 += 4)
              gs = fma(double(gam[ps * L + s2]), Gram[int64_t(a) * K + Ss[ps * L + s2]], gs);
            double b0 = 0.0, b1 = 0.0;
            if (d_vec4) {
              const float4* dr = reinterpret_cast<const float4*>(D + int64_t(a) * n);
              const float4* yv4 = reinterpret_cast<const float4*>(yrs);
              const int n4 = n / 4;
              for (int k4 = js; k4 < n4; k4 += 4) {
                const float4 dv = __ldg(dr + k4), yv = __ldg(yv4 + k4);
                b0 = fma(double(dv.x), double(yv.x), b0);
                b1 = fma(double(dv.y), double(yv.y), b1);
                b0 = fma(double(dv.z), double(yv.z), b0);
                b1 = fma(double(dv.w), double(yv.w), b1);
              }
            } else {
              for (int k = js; k < n; k += 4) b0 = fma(double(__ldg(D + int64_t(a) * n + k)), double(__ldg(yrs + k)), b0);
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
            const int lo2 = max(X.noff, rb), hi2 = min(X.noff + X.ncand, rh);
            for (int t = lo2; t < hi2; ++t) {
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
      // ---- quarter 0: selection, Cholesky append, solve, residual scale ----
      if (q == 0 && !done) {
        const double bbb = X.best_b;
        const int ba = X.best_a;
        const int a = (ba >= 0 && ba < K) ? ba : 0;
        const int k = P.cnt;
        bool stop = false;
        for (int s2 = 0; s2 < k; ++s2)
          if (Ss[m * L + s2] == a) stop = true;
        if (!stop) {
          double ww = 0.0;
          for (int i = 0; i < k; ++i) {
            double s3 = Gram[int64_t(Ss[m * L + i]) * K + a];
            for (int j = 0; j < i; ++j) s3 -= Lat(i, j) * Lat(k, j);
            const double wi = s3 * Lat(i, i);
            Lat(k, i) = wi;
            ww += wi * wi;
          }
          const double piv2 = Gram[int64_t(a) * K + a] - ww;
          if (!(piv2 > 0.0)) {
            stop = true;
          } else {
            Lat(k, k) = 1.0 / sqrt(piv2);
            Ss[m * L + k] = a;
            double zk = bbb;
            for (int j = 0; j < k; ++j) zk -= Lat(k, j) * bv[m * L + j];
            zk *= Lat(k, k);
            bv[m * L + k] = zk;
            double yv[kTbLMax];
            for (int i = k; i >= 0; --i) {
              double s3 = bv[m * L + i];
              for (int j = i + 1; j <= k; ++j) s3 -= Lat(j, i) * yv[j];
              yv[i] = s3 * Lat(i, i);
            }
            for (int i = 0; i <= k; ++i) gam[m * L + i] = float(yv[i]);
            const int kk = k + 1;
            P.cnt = kk;
            double rr = P.yy;
            float rs = P.ysum;
            for (int i = 0; i < kk; ++i) {
              rr -= bv[m * L + i] * bv[m * L + i];
              rs = fmaf(-gam[m * L + i], asum[Ss[m * L + i]], rs);
            }
            P.rmean = rs / float(n);
            P.rscale = tb_pow2_scale(float(sqrt(fmax(rr, 0.0))) * 1.01f + 1e-30f);
          }
        }
        if (stop) P.done = 1;
      }
      __syncthreads();
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
          if (d_vec4 && kc * 8 + 8 <= n) {
            const float4 y0 = __ldg(reinterpret_cast<const float4*>(yg + kc * 8));
            const float4 y1 = __ldg(reinterpret_cast<const float4*>(yg + kc * 8) + 1);
            r[0] = y0.x, r[1] = y0.y, r[2] = y0.z, r[3] = y0.w;
            r[4] = y1.x, r[5] = y1.y, r[6] = y1.z, r[7] = y1.w;
            for (int s2 = 0; s2 < cnt; ++s2) {
              const float4* dr = reinterpret_cast<const float4*>(D + int64_t(Ss[m * L + s2]) * n + kc * 8);
              const float gg = gam[m * L + s2];
              const float4 da = __ldg(dr), db = __ldg(dr + 1);
              r[0] = fmaf(-gg, da.x, r[0]);
              r[1] = fmaf(-gg, da.y, r[1]);
              r[2] = fmaf(-gg, da.z, r[2]);
              r[3] = fmaf(-gg, da.w, r[3]);
              r[4] = fmaf(-gg, db.x, r[4]);
              r[5] = fmaf(-gg, db.y, r[5]);
              r[6] = fmaf(-gg, db.z, r[6]);
              r[7] = fmaf(-gg, db.w, r[7]);
            }
          } else {
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              const int kk = kc * 8 + e;
              r[e] = (kk < n) ? __ldg(yg + kk) : 0.0f;
            }
            for (int s2 = 0; s2 < cnt; ++s2) {
              const float gg = gam[m * L + s2];
              const float* dr = D + int64_t(Ss[m * L + s2]) * n + kc * 8;
#pragma unroll
              for (int e = 0; e < 8; ++e)
                if (kc * 8 + e < n) r[e] = fmaf(-gg, __ldg(dr + e), r[e]);
            }
          }
          if (fin) {
            float* dst = R_out + (p0 + m) * int64_t(n) + kc * 8;
            if (r_vec4 && kc * 8 + 8 <= n) {
              __stcg(reinterpret_cast<float4*>(dst), make_float4(r[0], r[1], r[2], r[3]));
              __stcg(reinterpret_cast<float4*>(dst) + 1, make_float4(r[4], r[5], r[6], r[7]));
            } else {
#pragma unroll
              for (int e = 0; e < 8; ++e)
                if (kc * 8 + e < n) __stcg(dst + e, r[e]);
            }
          }
          unsigned short h[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const bool in = kc * 8 + e < n;
            nrm = fmaf(r[e], r[e], nrm);
            const float c = in ? r[e] - mean : 0.0f;
            cn = fmaf(c, c, cn);
            h[e] = TbOp<F16>::cvt(c * inv);
          }
          tb_store8(At + canon_off(m, kc * 8, kTbTile), h);
        }
      }
      X.part[q] = make_float2(nrm, cn);
      __syncthreads();
      if (q == 0 && live) {
        float tn = 0.0f, tc = 0.0f;
        for (int j = 0; j < kTbQ; ++j) {
          tn += X.part[j].x;
          tc += X.part[j].y;
        }
        P.rnorm = sqrtf(tc);
        if (sqrtf(tn) < 1e-3f) P.done = 1;
      }
    }
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
      // a patch that stopped before L atoms: its rows are left to
      // launch_residual over the list
      if (R_out && cnt < L) fix_list[atomicAdd(fix_count, 1ull)] = p0 + m;
    }
    __syncthreads();
  }
  if (stats && nscored) atomicAdd(&stats->pad, (unsigned long long)nscored);
  // ---- teardown: drain what is in flight (bounded), free the TMEM ------------
  if (tid == 0) {
    for (int s = 0; s < kTbSlots; ++s)
      if (empty_pending & (1u << s)) mbar_wait(empty + s, (empty_par >> s) & 1u, kTbWaitNs);
    // bulk copies issued but not consumed (only after a failure)
    for (unsigned long long i = consumed; i < issued; ++i) {
      const int s = int(i % kTbSlots);
      mbar_wait(full + s, (full_par >> s) & 1u, kTbWaitNs);
      full_par ^= 1u << s;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tc_dealloc(tmem, lo.tmem_cols);
  }
}

size_t omp_tcb_smem_bytes(int n, int K, int L) { return tb_layout(n, K, L).total; }

bool omp_tcb_supported(int n, int K, int L) {
  return L >= 1 && L <= kTbLMax && n >= 1 && n <= kTbMaxN && K >= 1 && K <= kTbMaxK &&
         omp_tcb_smem_bytes(n, K, L) <= 232448 - 1024;
}

size_t omp_tcb_scratch_bytes(int n, int K) {
  const TbLayout o = tb_layout(n, K, 1);
  return size_t(o.Kp) * o.np16 * 2 + size_t(o.Kp) * 4;
}

cudaError_t launch_omp_tcb(const float* patches, int64_t N, int n, const float* dict, const double* gram, int K,
                           int L, int32_t* idx, float* coef, int num_sms, int fp16, void* scratch,
                           GridBarrier* flags, DevStats* stats, cudaStream_t s, float* resid_out, int* last_out,
                           int64_t* fix_list, unsigned long long* fix_count) {
  if (!omp_tcb_supported(n, K, L)) return cudaErrorInvalidValue;
  if (resid_out && (!last_out || !fix_list || !fix_count)) return cudaErrorInvalidValue;
  const TbLayout o = tb_layout(n, K, L);
  unsigned char* Bg = static_cast<unsigned char*>(scratch);
  float* asum = reinterpret_cast<float*>(Bg + size_t(o.Kp) * o.np16 * 2);
  if (fp16)
    tb_prep_kernel<true><<<num_sms, 256, 0, s>>>(dict, K, n, o.Kp, o.np16, Bg, asum);
  else
    tb_prep_kernel<false><<<num_sms, 256, 0, s>>>(dict, K, n, o.Kp, o.np16, Bg, asum);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t smem = o.total;
  auto kern = fp16 ? omp_tcb_kernel<true> : omp_tcb_kernel<false>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  const int64_t ntiles = (N + kTbTile - 1) / kTbTile;
  const int grid = int(std::min<int64_t>(ntiles, num_sms));
  const int d_vec4 = ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(dict) & 15) == 0 &&
                      (reinterpret_cast<uintptr_t>(patches) & 15) == 0)
                         ? 1
                         : 0;
  const int r_vec4 = ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(resid_out) & 15) == 0) ? 1 : 0;
  kern<<<grid, kTbThreads, smem, s>>>(patches, N, n, dict, Bg, asum, gram, K, L, idx, coef, ntiles, d_vec4,
                                      resid_out, last_out, fix_list, fix_count, r_vec4, flags, stats);
  return cudaGetLastError();
}

}  // namespace ksvd
