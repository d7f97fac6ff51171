// Sequential K-SVD dictionary update (updateDictionary,
// cuda_svd_denoiser.cu:285-362) on a maintained residual.
//
// The residual R = Y - X D (one n-vector per patch) is formed once before the
// sweep.  For atom j with support Omega_j (c entries, only the first 1024
// with the Q1 cap) the columns of the reference's error matrix are then
//     e_p = r_p + x_{j,p} d_j            (p in Omega_j)
// which equals y_p - sum_{s != j} x_{s,p} d_s with every earlier atom of the
// sweep already updated (the reference's Gauss-Seidel order, :309-361).  The
// top left singular vector u of E = [e_p] (gesvdj's U[:,0], :328-346) is
// found by power iteration on E itself, w = E (E^T u), warm-started from the
// old atom; u is signed so that u . d_j(old) >= 0; then
//     d_j <- u,  x_{j,p} <- u . e_p (= sigma v_p, :349-358),
//     r_p <- e_p - x_{j,p} u,
// with x_{j,p} = 0 (and r_p <- e_p) for entries beyond the cap.
//
// One persistent cooperative kernel walks the atoms.  An atom's entries are
// split over `active` CTAs (about slice_target entries each); each keeps its
// columns in shared memory (those beyond the capacity are re-read from the
// residual on every pass).  A power step is one pass over the local columns
// producing a partial w, then an all-reduce: each CTA writes its partial,
// arrives on the atom's counter and, once all active CTAs have arrived, sums
// all partials in the same fixed order, so every CTA holds the same u and
// takes the same convergence decision.  An atom's CTAs wait for the previous
// atom's CTAs to finish their residual stores before reading the residual;
// since those in turn waited for the atom before, every earlier atom of the
// sweep is complete by then.  CTAs with no entries in an atom skip it.  All
// waits are bounded.
#include <cuda_runtime.h>

#include <cstring>

#include "device_util.cuh"
#include "ksvd_internal.cuh"

namespace ksvd {

constexpr int kUrThreads = 512;
constexpr int kUrWarps = kUrThreads / 32;
constexpr int kUrDefaultSlice = 64;   // entries per CTA before another CTA joins an atom (default)
constexpr int kUrMaxIters = 200;
constexpr float kUrTol = 2.0e-7f;     // max |u_new - u_old| to stop
constexpr size_t kUrSmemMax = 232448 - 256;  // opt-in shared memory per block, less the static part

__host__ __device__ inline int ur_n4(int n) { return (n + 3) & ~3; }

// Row stride of the resident columns (floats): a multiple of 4 whose float4
// count is odd, so that the 8 rows a quarter-warp reads with 16-byte loads
// sit in distinct banks.
__host__ __device__ inline int ur_es(int n) { return 4 * ((ur_n4(n) / 4) | 1); }
constexpr int kUrRows = 32;  // reduction rows: 16 column groups + 16 streaming warps

// Shared memory: [cap x es] columns | ent[2][cap] | xold[2][cap] | keep[2][cap] |
// u[n4] | dold[n4] | dnext[n4] | wred[kUrRows x n4]
__host__ __device__ inline size_t ur_fixed_bytes(int n) {
  const int n4 = ur_n4(n);
  return size_t(n4) * 4 * 3 + size_t(kUrRows) * n4 * 4;
}

int update_res_capacity(int n) {
  const size_t per = size_t(ur_es(n)) * 4 + 24;
  const size_t fixed = ur_fixed_bytes(n);
  if (fixed + per * 16 > kUrSmemMax) return 0;
  // a multiple of 4 keeps u, dold, dnext and wred (read as float4) 16-byte aligned
  return int((kUrSmemMax - fixed) / per) & ~3;
}

size_t update_res_smem_bytes(int n, int cap) { return size_t(cap) * (size_t(ur_es(n)) * 4 + 24) + ur_fixed_bytes(n); }

// Bounded spin of thread 0 until *ctr >= target.  False on timeout or when an
// error is already flagged.
KSVD_DEV bool ur_wait_count(const unsigned* ctr, unsigned target, GridBarrier* flags) {
  if (ld_acquire_u32(ctr) >= target) return true;
  const unsigned long long t0 = globaltimer_ns();
  while (ld_acquire_u32(ctr) < target) {
    if (ld_relaxed_i32(&flags->err) != DEVERR_NONE) return false;
    if (globaltimer_ns() - t0 > kBarrierTimeoutNs) {
      atomicCAS(&flags->err, DEVERR_NONE, DEVERR_TIMEOUT);
      return false;
    }
    __nanosleep(20);
  }
  return true;
}

__host__ __device__ inline int ur_active(int c, int G, int target) {
  const int a = (c + target - 1) / target;
  return a < G ? a : G;
}

// residual_kernel: R = Y - X D, one warp per patch (every patch, or those of
// a device-side list).  The patch's atoms and
// coefficients sit in lanes 0..L-1 and are broadcast by shuffles; each lane
// forms 16-byte pieces of the row with the support atoms' loads in flight
// together (same FMA order as r = y - sum_s x_s d_s, s ascending).  last[p]
// (optional) receives the highest atom of the patch's support (-1 if none):
// the sweep visits atoms in ascending order, so no atom after that one reads
// the patch's residual row again in the sweep.
__global__ void __launch_bounds__(256) residual_kernel(const float* __restrict__ Y, int64_t N, int n,
                                                       const float* __restrict__ D, int K, int L,
                                                       const int32_t* __restrict__ idx,
                                                       const float* __restrict__ coef, float* __restrict__ R,
                                                       int* __restrict__ last, int vec4,
                                                       const int64_t* __restrict__ list,
                                                       const unsigned long long* __restrict__ count) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  int64_t total = N;  // every patch, or list[0 .. *count)
  if (list) {
    const unsigned long long c = *count;
    total = c < static_cast<unsigned long long>(N) ? int64_t(c) : N;
  }
  for (int64_t w = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w < total; w += warps) {
    const int64_t p = list ? list[w] : w;
    int a = -1;
    float x = 0.0f;
    if (lane < L) {
      a = __ldg(idx + p * L + lane);
      x = __ldg(coef + p * L + lane);
      if (a < 0 || a >= K || x == 0.0f) a = -1;
    }
    if (last) {
      int top = a;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) top = max(top, __shfl_xor_sync(0xffffffffu, top, o));
      if (lane == 0) last[p] = top;
    }
    if (vec4) {
      const int F = n >> 2;
      const float4* y4 = reinterpret_cast<const float4*>(Y + p * n);
      float4* r4 = reinterpret_cast<float4*>(R + p * n);
      for (int f0 = 0; f0 < F; f0 += 32) {
        const int f = f0 + lane;
        const bool in = f < F;
        float4 r = in ? __ldg(y4 + f) : make_float4(0.f, 0.f, 0.f, 0.f);
        for (int s0 = 0; s0 < L; s0 += 8) {
          float4 dv[8];
          float xs[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int as = __shfl_sync(0xffffffffu, a, (s0 + u) & 31);
            xs[u] = __shfl_sync(0xffffffffu, x, (s0 + u) & 31);
            const bool use = in && s0 + u < L && as >= 0;
            dv[u] = use ? __ldg(reinterpret_cast<const float4*>(D + int64_t(as) * n) + f)
                        : make_float4(0.f, 0.f, 0.f, 0.f);
            if (!use) xs[u] = 0.0f;
          }
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            if (xs[u] != 0.0f) {
              r.x = fmaf(-xs[u], dv[u].x, r.x);
              r.y = fmaf(-xs[u], dv[u].y, r.y);
              r.z = fmaf(-xs[u], dv[u].z, r.z);
              r.w = fmaf(-xs[u], dv[u].w, r.w);
            }
          }
        }
        if (in) r4[f] = r;
      }
    } else {
      for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        const bool in = i < n;
        float r = in ? Y[p * n + i] : 0.0f;
        for (int s = 0; s < L; ++s) {
          const int as = __shfl_sync(0xffffffffu, a, s & 31);
          const float xs = __shfl_sync(0xffffffffu, x, s & 31);
          if (in && as >= 0) r = fmaf(-xs, __ldg(D + int64_t(as) * n + i), r);
        }
        if (in) R[p * n + i] = r;
      }
    }
  }
}

// Arrive on a counter with release semantics: after a __syncthreads(), the
// writes of every thread of the CTA are visible to whoever acquires the count.
KSVD_DEV void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// One launch sweeps one or several problems (images): group g owns the CTAs
// [cta_begin, cta_begin + ctas) and walks its own atoms with its own buffers,
// counters and partials.  Groups whose ranges share CTAs run one after the
// other on those CTAs, in the order of the table; a group only waits for its
// own CTAs, and every CTA takes its groups in the same (table) order, so the
// lowest unfinished group always has all its CTAs and the launch cannot
// deadlock.
template <int NW>
__global__ void __launch_bounds__(kUrThreads, 1)
    update_res_kernel(const UpdBatch batch, GridBarrier* flags, DevStats* stats, int timers) {
  extern __shared__ __align__(16) unsigned char ursm[];
  __shared__ int s_ok;
  __shared__ int s_stop;
  __shared__ __align__(8) unsigned long long s_mbar;  // completion of the residual-row bulk copies
  __shared__ unsigned long long s_ph[8];  // phase times of this CTA (slots 0..7)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned mpar = 0;  // parity of the next phase of s_mbar
  if (tid == 0) {
    mbar_init(&s_mbar, 1);
    fence_mbar_init();
  }
  __syncthreads();

  // phase times gather in shared memory and are flushed once at the end
  const bool timer = (timers != 0 && blockIdx.x == 0 && tid == 0);
  if (timer)
    for (int k = 0; k < 8; ++k) s_ph[k] = 0ull;
  unsigned long long tmark = timer ? globaltimer_ns() : 0ull;
  auto lap = [&](int slot) {
    if (timer) {
      const unsigned long long t = globaltimer_ns();
      s_ph[slot] += t - tmark;
      tmark = t;
    }
  };
  // thread 0 waits, the block learns the outcome
  auto block_wait = [&](const unsigned* ctr, unsigned target) -> bool {
    if (tid == 0) s_ok = ur_wait_count(ctr, target, flags) ? 1 : 0;
    __syncthreads();
    const bool ok = s_ok != 0;
    __syncthreads();
    return ok;
  };

  // every group whose CTA range holds this CTA, in the order of the table
  for (int gi = 0; gi < batch.ngroups; ++gi) {
    const UpdGroup& grp = batch.g[gi];
    if (int(blockIdx.x) < grp.cta_begin || int(blockIdx.x) >= grp.cta_begin + grp.ctas) continue;
    __syncthreads();  // the previous group's shared memory is no longer read
    float* const R = grp.R;
    float* const D = grp.D;
    float* const coef = grp.coef;
    const int* __restrict__ const atom_ptr = grp.atom_ptr;
    const int* __restrict__ const entries = grp.entries;
    const int* __restrict__ const last = grp.last;
    float* const gw = grp.gw;
    unsigned* const sync = grp.sync;
    const int n = grp.n, K = grp.K, L = grp.L, q1_cap = grp.q1_cap, cap = grp.cap;
    const int slice_target = grp.slice_target > 0 ? grp.slice_target : kUrDefaultSlice;
    const int n4 = ur_n4(n), es = ur_es(n);
    const int F = n4 / 4, es4 = es / 4;  // float4 per row of u / w, per resident column
    float* Es = reinterpret_cast<float*>(ursm);
    const float4* Es4 = reinterpret_cast<const float4*>(ursm);
    int* ent_b = reinterpret_cast<int*>(ursm + size_t(cap) * es * 4);  // [2][cap]
    float* xold_b = reinterpret_cast<float*>(ent_b + 2 * cap);           // [2][cap]
    int* keep_b = reinterpret_cast<int*>(xold_b + 2 * cap);  // [2][cap]: residual row stored back
    float* u = reinterpret_cast<float*>(keep_b + 2 * cap);
    float* dold = u + n4;
    float* dnext = dold + n4;
    float* wred = dnext + n4;  // [kUrRows][n4]
    float4* u4 = reinterpret_cast<float4*>(u);
    const float4* dold4 = reinterpret_cast<const float4*>(dold);
    float4* wred4 = reinterpret_cast<float4*>(wred);

    const int G = grp.ctas, b = int(blockIdx.x) - grp.cta_begin;
    unsigned* iter_cnt = sync;
    unsigned* done_cnt = sync + K;
    int Gr = kUrThreads / F;  // column groups of the w pass, partial groups of the all-reduce
    if (Gr > 16) Gr = 16;
    if (Gr < 1) Gr = 1;
    // bulk copies need 16-byte aligned rows of a multiple of 16 bytes
    const bool tma = (n & 3) == 0 && (reinterpret_cast<uintptr_t>(R) & 15) == 0;

    // this CTA's slice [sb, se) of atom a's c entries starting at beg
    auto slice_of = [&](int a, int& beg, int& c, int& active, int& sb, int& se) {
      beg = atom_ptr[a];
      c = atom_ptr[a + 1] - beg;
      active = ur_active(c, G, slice_target);
      sb = int(int64_t(c) * b / active);
      se = int(int64_t(c) * (b + 1) / active);
    };
    // entries, old coefficients and store-back flags of [sb, sb + cnt) into
    // meta buffer `slot` and atom a into dst (all threads; several loads in
    // flight per thread).  A residual row is stored back unless a is the last
    // atom of the patch's support.
    auto load_meta = [&](int beg, int sb, int cnt, int slot, int a, float* dst) {
      int* ent = ent_b + slot * cap;
      float* xo = xold_b + slot * cap;
      int* kp = keep_b + slot * cap;
      constexpr int kB = 4;
      for (int t0 = tid; t0 < cnt; t0 += kUrThreads * kB) {
        int e[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) {
          const int t = t0 + k * kUrThreads;
          e[k] = (t < cnt) ? __ldg(entries + beg + sb + t) : 0;
        }
        float x[kB];
        int lt[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) {
          const bool in = t0 + k * kUrThreads < cnt;
          x[k] = in ? __ldcg(coef + e[k]) : 0.0f;
          lt[k] = (in && last != nullptr) ? __ldg(last + e[k] / L) : -1;
        }
#pragma unroll
        for (int k = 0; k < kB; ++k) {
          const int t = t0 + k * kUrThreads;
          if (t < cnt) {
            ent[t] = e[k];
            xo[t] = x[k];
            kp[t] = (lt[k] != a) ? 1 : 0;
          }
        }
      }
      for (int i = tid; i < n4; i += kUrThreads) dst[i] = (i < n) ? __ldcg(D + int64_t(a) * n + i) : 0.0f;
    };
    // u . e_q for a resident column (one thread, 16-byte loads, 4 chains)
    auto dot_u = [&](int q) -> float {
      const float4* er = Es4 + size_t(q) * es4;
      float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll 6
      for (int f = 0; f < F; ++f) {
        const float4 e = er[f], w = u4[f];
        a0 = fmaf(e.x, w.x, a0);
        a1 = fmaf(e.y, w.y, a1);
        a2 = fmaf(e.z, w.z, a2);
        a3 = fmaf(e.w, w.w, a3);
      }
      return (a0 + a1) + (a2 + a3);
    };

    int jprev = -1, aprev = 0;
    int slot = 0;        // meta buffer of the current atom
    int meta_atom = -1;  // atom whose meta was prefetched into buffer `slot`
    for (int j = 0; j < K; ++j) {
      int beg, c, active, sb, se;
      slice_of(j, beg, c, active, sb, se);
      if (c == 0) continue;
      const int jp = jprev, ap = aprev;
      jprev = j;
      aprev = active;
      if (b >= active) continue;
      const int c_eff = (q1_cap && c > 1024) ? 1024 : c;
      const int m = se - sb;
      const int mres = m < cap ? m : cap;
      // columns [0, mc) of the slice enter the power iteration
      int mc = c_eff - sb;
      mc = mc < 0 ? 0 : (mc > m ? m : mc);
      const int mcr = mc < cap ? mc : cap;  // of which resident
      const bool streamed = mc > cap;        // some enter from the residual
      const int* ent_s = ent_b + slot * cap;
      const float* xold_s = xold_b + slot * cap;
      float* v_s = xold_b + slot * cap;  // per-column scalars once the columns are built
      const int* keep_s = keep_b + slot * cap;

      // ---- entries, old coefficients and the old atom: never written by other
      // atoms, so read before the wait (or prefetched during the previous atom)
      if (meta_atom == j) {
        for (int i = tid; i < n4; i += kUrThreads) dold[i] = dnext[i];
      } else {
        load_meta(beg, sb, mres, slot, j, dold);
      }
      lap(7);
      __syncthreads();
      if (jp >= 0 && !block_wait(done_cnt + jp, unsigned(ap))) return;
      lap(0);

      // the next non-empty atom; if this CTA works on it, its meta is fetched
      // while this CTA waits for the first partials
      int jn = j + 1;
      while (jn < K && atom_ptr[jn + 1] == atom_ptr[jn]) ++jn;
      int nbeg = 0, nc = 0, nact = 0, nsb = 0, nse = 0;
      bool prefetch = false;
      if (jn < K) {
        slice_of(jn, nbeg, nc, nact, nsb, nse);
        prefetch = b < nact;
      }

      // ---- resident columns e_q = r_q + x_q d_old ---------------------------
      if (tma) {
        // residual rows by bulk copies (the residual was written by other CTAs
        // through the generic proxy: acquire above, proxy fence here), then
        // e = r + x d in place
        if (tid == 0) mbar_arrive_expect_tx(&s_mbar, unsigned(mres) * unsigned(n) * 4u);
        __syncthreads();
        asm volatile("fence.proxy.async.global;" ::: "memory");
        for (int q = tid; q < mres; q += kUrThreads)
          bulk_g2s(Es + size_t(q) * es, R + int64_t(ent_s[q] / L) * n, unsigned(n) * 4u, &s_mbar);
        const bool ok = mbar_wait(&s_mbar, mpar, kBarrierTimeoutNs);
        mpar ^= 1u;
        if (__syncthreads_or(!ok)) {
          if (tid == 0) atomicCAS(&flags->err, DEVERR_NONE, DEVERR_TIMEOUT);
          return;
        }
        for (int t = tid; t < mres * F; t += kUrThreads) {
          const int q = t / F, f = t - q * F;
          const float x = xold_s[q];
          const float4 d = dold4[f];
          float4* ep = reinterpret_cast<float4*>(Es) + size_t(q) * es4 + f;
          float4 e = *ep;
          e.x = fmaf(x, d.x, e.x);
          e.y = fmaf(x, d.y, e.y);
          e.z = fmaf(x, d.z, e.z);
          e.w = fmaf(x, d.w, e.w);
          *ep = e;
        }
      } else {
        for (int t = tid; t < mres * n4; t += kUrThreads) {
          const int q = t / n4, i = t - q * n4;
          float e = 0.0f;
          if (i < n) e = fmaf(xold_s[q], dold[i], __ldcg(R + int64_t(ent_s[q] / L) * n + i));
          Es[size_t(q) * es + i] = e;
        }
      }
      for (int i = tid; i < n4; i += kUrThreads) u[i] = dold[i];
      __syncthreads();
      lap(1);

      // Two streamed columns (q0, q1 = q0 + kUrWarps, both >= cap) from the
      // residual; a column index >= lim gives zeros.
      auto stream_cols = [&](int q0, int lim, float (&e0)[NW], float (&e1)[NW], int& ea, int& eb) {
        const int q1 = q0 + kUrWarps;
        ea = (q0 < lim) ? __ldg(entries + beg + sb + q0) : -1;
        eb = (q1 < lim) ? __ldg(entries + beg + sb + q1) : -1;
        const float xa = (ea >= 0) ? __ldcg(coef + ea) : 0.0f;
        const float xb = (eb >= 0) ? __ldcg(coef + eb) : 0.0f;
        const float* ra = R + int64_t(ea >= 0 ? ea / L : 0) * n;
        const float* rb = R + int64_t(eb >= 0 ? eb / L : 0) * n;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const int i = lane + 32 * k;
          e0[k] = (i < n && ea >= 0) ? fmaf(xa, dold[i], __ldcg(ra + i)) : 0.0f;
          e1[k] = (i < n && eb >= 0) ? fmaf(xb, dold[i], __ldcg(rb + i)) : 0.0f;
        }
      };

      // ---- power iteration ---------------------------------------------------
      int iters = 0;
      float dprev = 0.0f;  // warp 0: the previous step's change
      for (int it = 0; it < kUrMaxIters; ++it) {
        // v_q = u . e_q, one thread per resident column
        for (int q = tid; q < mcr; q += kUrThreads) v_s[q] = dot_u(q);
        if (streamed) {  // columns beyond the capacity: a warp per two columns
          float ur[NW], wacc[NW];
#pragma unroll
          for (int k = 0; k < NW; ++k) {
            const int i = lane + 32 * k;
            ur[k] = (i < n) ? u[i] : 0.0f;
            wacc[k] = 0.0f;
          }
          for (int q = cap + warp; q < mc; q += 2 * kUrWarps) {
            float e0[NW], e1[NW];
            int ea, eb;
            stream_cols(q, mc, e0, e1, ea, eb);
            float d0 = 0.0f, d1 = 0.0f;
#pragma unroll
            for (int k = 0; k < NW; ++k) {
              d0 = fmaf(ur[k], e0[k], d0);
              d1 = fmaf(ur[k], e1[k], d1);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              d0 += __shfl_xor_sync(0xffffffffu, d0, o);
              d1 += __shfl_xor_sync(0xffffffffu, d1, o);
            }
#pragma unroll
            for (int k = 0; k < NW; ++k) wacc[k] = fmaf(d1, e1[k], fmaf(d0, e0[k], wacc[k]));
          }
#pragma unroll
          for (int k = 0; k < NW; ++k) {
            const int i = lane + 32 * k;
            if (i < n4) wred[(16 + warp) * n4 + i] = wacc[k];
          }
        }
        __syncthreads();
        // w = sum_q v_q e_q: column group g (q = g mod Gr) of float4 column f
        {
          const int f = tid % F, g = tid / F;
          if (g < Gr) {
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll 4
            for (int q = g; q < mcr; q += Gr) {
              const float v = v_s[q];
              const float4 e = Es4[size_t(q) * es4 + f];
              acc.x = fmaf(v, e.x, acc.x);
              acc.y = fmaf(v, e.y, acc.y);
              acc.z = fmaf(v, e.z, acc.z);
              acc.w = fmaf(v, e.w, acc.w);
            }
            wred4[g * F + f] = acc;
          }
        }
        __syncthreads();
        float4* gwp = reinterpret_cast<float4*>(gw + (size_t(it & 1) * G + b) * n4);
        for (int f = tid; f < F; f += kUrThreads) {
          float4 acc = wred4[f];
#pragma unroll 4
          for (int g = 1; g < Gr; ++g) {
            const float4 v = wred4[g * F + f];
            acc.x += v.x;
            acc.y += v.y;
            acc.z += v.z;
            acc.w += v.w;
          }
          if (streamed)
#pragma unroll
            for (int w = 0; w < kUrWarps; ++w) {
              const float4 v = wred4[(16 + w) * F + f];
              acc.x += v.x;
              acc.y += v.y;
              acc.z += v.z;
              acc.w += v.w;
            }
          __stcg(gwp + f, acc);
        }
        __syncthreads();
        lap(2);
        if (tid == 0) red_release_add(iter_cnt + j, 1u);
        if (it == 0 && prefetch)  // overlaps the wait below
          load_meta(nbeg, nsb, min(nse - nsb, cap), slot ^ 1, jn, dnext);
        if (!block_wait(iter_cnt + j, unsigned(it + 1) * unsigned(active))) return;
        lap(3);
        // all-reduce: group g sums partials g, g + Gr, ... of float4 column f in
        // ascending order (loads batched)
        {
          const int f = tid % F, g = tid / F;
          if (g < Gr) {
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
            const float4* base = reinterpret_cast<const float4*>(gw + size_t(it & 1) * G * n4) + f;
            constexpr int kB = 12;  // one round of loads for up to 12 Gr partials per thread
            for (int bb0 = g; bb0 < active; bb0 += Gr * kB) {
              float4 v[kB];
#pragma unroll
              for (int k = 0; k < kB; ++k) {
                const int bb = bb0 + k * Gr;
                v[k] = (bb < active) ? __ldcg(base + size_t(bb) * F) : make_float4(0.f, 0.f, 0.f, 0.f);
              }
#pragma unroll
              for (int k = 0; k < kB; ++k) {
                acc.x += v[k].x;
                acc.y += v[k].y;
                acc.z += v[k].z;
                acc.w += v[k].w;
              }
            }
            wred4[g * F + f] = acc;
          }
        }
        __syncthreads();
        iters = it + 1;
        // warp 0 finishes the step: w, its norm, the new u, the change, the
        // stop decision and, when stopping, the sign (u . d_old >= 0)
        if (warp == 0) {
          constexpr int kF = 4;  // float4 per lane (F <= 128)
          float4 wv[kF];
          float s2 = 0.0f;
#pragma unroll
          for (int k = 0; k < kF; ++k) {
            const int f = lane + 32 * k;
            float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
            if (f < F)
#pragma unroll 4
              for (int g = 0; g < Gr; ++g) {
                const float4 v = wred4[g * F + f];
                acc.x += v.x;
                acc.y += v.y;
                acc.z += v.z;
                acc.w += v.w;
              }
            wv[k] = acc;
            s2 = fmaf(acc.x, acc.x, fmaf(acc.y, acc.y, fmaf(acc.z, acc.z, fmaf(acc.w, acc.w, s2))));
          }
          const float nrm2 = warp_sum(s2);
          bool stop;
          if (!(nrm2 > 0.0f)) {
            stop = true;  // E == 0: keep the old atom direction
          } else {
            const float inv = 1.0f / sqrtf(nrm2);
            float dm = 0.0f;
#pragma unroll
            for (int k = 0; k < kF; ++k) {
              const int f = lane + 32 * k;
              if (f < F) {
                const float4 o = u4[f];
                float4 un;
                un.x = wv[k].x * inv;
                un.y = wv[k].y * inv;
                un.z = wv[k].z * inv;
                un.w = wv[k].w * inv;
                dm = fmaxf(dm, fmaxf(fmaxf(fabsf(un.x - o.x), fabsf(un.y - o.y)),
                                     fmaxf(fabsf(un.z - o.z), fabsf(un.w - o.w))));
                u4[f] = un;
              }
            }
            dm = warp_max(dm);
            // stop when the change is below the tolerance, or when the observed
            // contraction rho = dm / dprev puts the remaining distance to the
            // limit, about dm rho / (1 - rho), below it
            const float rho = (it > 0 && dprev > 0.0f) ? dm / dprev : 1.0f;
            stop = dm < kUrTol || (rho < 0.5f && dm < 1e-3f && dm * rho < kUrTol * (1.0f - rho));
            dprev = dm;
          }
          if (stop) {
            float sd = 0.0f;
#pragma unroll
            for (int k = 0; k < kF; ++k) {
              const int f = lane + 32 * k;
              if (f < F) {
                const float4 a = u4[f], d = dold4[f];
                sd = fmaf(a.x, d.x, fmaf(a.y, d.y, fmaf(a.z, d.z, fmaf(a.w, d.w, sd))));
              }
            }
            sd = warp_sum(sd);
            if (sd < 0.0f)
#pragma unroll
              for (int k = 0; k < kF; ++k) {
                const int f = lane + 32 * k;
                if (f < F) {
                  float4 a = u4[f];
                  a.x = -a.x;
                  a.y = -a.y;
                  a.z = -a.z;
                  a.w = -a.w;
                  u4[f] = a;
                }
              }
          }
          if (lane == 0) s_stop = stop ? 1 : 0;
        }
        __syncthreads();
        lap(4);
        if (s_stop) break;
      }
      if (b == 0) {
        for (int i = tid; i < n; i += kUrThreads) __stcg(D + int64_t(j) * n + i, u[i]);
        if (tid == 0) {
          atomicAdd(&stats->power_iters, (unsigned long long)iters);
          atomicAdd(&stats->atoms_updated, 1ull);
        }
      }

      // ---- coefficients x = u . e (0 beyond the cap) and residual e - x u ----
      for (int q = tid; q < mres; q += kUrThreads) {
        const float x = (q < mc) ? dot_u(q) : 0.0f;
        v_s[q] = x;
        __stcg(coef + ent_s[q], x);
      }
      if (m > cap) {  // streamed columns: a warp per two columns
        float ur[NW];
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const int i = lane + 32 * k;
          ur[k] = (i < n) ? u[i] : 0.0f;
        }
        for (int q = cap + warp; q < m; q += 2 * kUrWarps) {
          float e0[NW], e1[NW];
          int ea, eb;
          stream_cols(q, m, e0, e1, ea, eb);
          float x0 = 0.0f, x1 = 0.0f;
#pragma unroll
          for (int k = 0; k < NW; ++k) {
            x0 = fmaf(ur[k], e0[k], x0);
            x1 = fmaf(ur[k], e1[k], x1);
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            x0 += __shfl_xor_sync(0xffffffffu, x0, o);
            x1 += __shfl_xor_sync(0xffffffffu, x1, o);
          }
          if (q >= mc) x0 = 0.0f;
          if (q + kUrWarps >= mc) x1 = 0.0f;
          float* ra = R + int64_t(ea / L) * n;
          if (last == nullptr || __ldg(last + ea / L) != j) {
#pragma unroll
            for (int k = 0; k < NW; ++k) {
              const int i = lane + 32 * k;
              if (i < n) __stcg(ra + i, fmaf(-x0, ur[k], e0[k]));
            }
          }
          if (lane == 0) __stcg(coef + ea, x0);
          if (eb >= 0) {
            float* rb = R + int64_t(eb / L) * n;
            if (last == nullptr || __ldg(last + eb / L) != j) {
#pragma unroll
              for (int k = 0; k < NW; ++k) {
                const int i = lane + 32 * k;
                if (i < n) __stcg(rb + i, fmaf(-x1, ur[k], e1[k]));
              }
            }
            if (lane == 0) __stcg(coef + eb, x1);
          }
        }
      }
      __syncthreads();
      if (tma) {  // rows of 16-byte aligned float4
        for (int t = tid; t < mres * F; t += kUrThreads) {
          const int q = t / F, f = t - q * F;
          if (!keep_s[q]) continue;
          const float x = v_s[q];
          const float4 e = Es4[size_t(q) * es4 + f], w = u4[f];
          float4 r;
          r.x = fmaf(-x, w.x, e.x);
          r.y = fmaf(-x, w.y, e.y);
          r.z = fmaf(-x, w.z, e.z);
          r.w = fmaf(-x, w.w, e.w);
          __stcg(reinterpret_cast<float4*>(R + int64_t(ent_s[q] / L) * n) + f, r);
        }
      } else {
        for (int t = tid; t < mres * n; t += kUrThreads) {
          const int q = t / n, i = t - q * n;
          if (keep_s[q]) __stcg(R + int64_t(ent_s[q] / L) * n + i, fmaf(-v_s[q], u[i], Es[size_t(q) * es + i]));
        }
      }
      fence_proxy_async_smem();  // generic accesses of Es before the next bulk copies into it
      __syncthreads();
      if (tid == 0) red_release_add(done_cnt + j, 1u);
      lap(5);
      if (prefetch) {
        slot ^= 1;
        meta_atom = jn;
      } else {
        meta_atom = -1;
      }
    }
  }
  if (timer)
    for (int k = 0; k < 8; ++k) atomicAdd(&stats->phase_ns[k], s_ph[k]);
}

template <int NW>
static void* ur_fn() {
  return reinterpret_cast<void*>(update_res_kernel<NW>);
}

static void* pick_update_res(int n) {
  switch ((n + 31) / 32) {
    case 1: return ur_fn<1>();
    case 2: return ur_fn<2>();
    case 3: return ur_fn<3>();
    case 4: return ur_fn<4>();
    case 5: return ur_fn<5>();
    case 6: return ur_fn<6>();
    case 7: return ur_fn<7>();
    case 8: return ur_fn<8>();
    case 9: return ur_fn<9>();
    case 10: return ur_fn<10>();
    case 11: return ur_fn<11>();
    case 12: return ur_fn<12>();
    case 13: return ur_fn<13>();
    case 14: return ur_fn<14>();
    case 15: return ur_fn<15>();
    case 16: return ur_fn<16>();
    default: return nullptr;
  }
}

bool update_res_supported(int n) { return n >= 1 && n <= 512 && update_res_capacity(n) >= 16; }

int update_res_grid_size(int n, int num_sms) {
  void* fn = pick_update_res(n);
  const int cap = update_res_capacity(n);
  if (!fn || cap < 16) return 0;
  const size_t smem = update_res_smem_bytes(n, cap);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kUrThreads, smem) != cudaSuccess) return 0;
  if (per_sm < 1) return 0;
  return num_sms;  // one CTA per SM: co-resident by construction
}

size_t update_res_partial_floats(int n, int grid) { return size_t(2) * grid * ur_n4(n); }

cudaError_t launch_residual(const float* Y, int64_t N, int n, const float* D, int K, int L, const int32_t* idx,
                            const float* coef, float* R, int* last, int num_sms, cudaStream_t s) {
  const int64_t want = (N + 7) / 8;
  const int blocks = int(want < int64_t(num_sms) * 16 ? want : int64_t(num_sms) * 16);
  const int vec4 = ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(Y) & 15) == 0 &&
                    (reinterpret_cast<uintptr_t>(D) & 15) == 0 && (reinterpret_cast<uintptr_t>(R) & 15) == 0)
                       ? 1
                       : 0;
  residual_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(Y, N, n, D, K, L, idx, coef, R, last, vec4, nullptr,
                                                          nullptr);
  return cudaGetLastError();
}

cudaError_t launch_residual_list(const float* Y, int64_t N, int n, const float* D, int K, int L, const int32_t* idx,
                                 const float* coef, float* R, int* last, const int64_t* list,
                                 const unsigned long long* count, int num_sms, cudaStream_t s) {
  if (!list || !count) return cudaErrorInvalidValue;
  const int vec4 = ((n & 3) == 0 && (reinterpret_cast<uintptr_t>(Y) & 15) == 0 &&
                    (reinterpret_cast<uintptr_t>(D) & 15) == 0 && (reinterpret_cast<uintptr_t>(R) & 15) == 0)
                       ? 1
                       : 0;
  residual_kernel<<<num_sms * 2, 256, 0, s>>>(Y, N, n, D, K, L, idx, coef, R, last, vec4, list, count);
  return cudaGetLastError();
}

cudaError_t launch_update_batch(const UpdBatch& batch, GridBarrier* flags, DevStats* stats, int timers, int grid,
                                cudaStream_t s) {
  if (batch.ngroups < 1 || batch.ngroups > kUpdMaxGroups || grid < 1) return cudaErrorInvalidValue;
  int nmax = 0;
  for (int i = 0; i < batch.ngroups; ++i) {
    const UpdGroup& g = batch.g[i];
    if (g.ctas < 1 || g.cta_begin < 0 || g.cta_begin + g.ctas > grid) return cudaErrorInvalidValue;
    if (g.cap < 16 || g.cap > update_res_capacity(g.n)) return cudaErrorInvalidValue;
    nmax = g.n > nmax ? g.n : nmax;
  }
  void* fn = pick_update_res(nmax);
  if (!fn) return cudaErrorInvalidValue;
  size_t smem = 0;
  for (int i = 0; i < batch.ngroups; ++i) {
    const size_t b = update_res_smem_bytes(batch.g[i].n, batch.g[i].cap);
    smem = b > smem ? b : smem;
  }
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  for (int i = 0; i < batch.ngroups; ++i) {
    e = cudaMemsetAsync(batch.g[i].sync, 0, size_t(2) * batch.g[i].K * sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
  }
  UpdBatch b = batch;
  void* args[] = {(void*)&b, (void*)&flags, (void*)&stats, (void*)&timers};
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kUrThreads), args, smem, s);
}

cudaError_t launch_update_res(float* R, int n, float* D, int K, int L, float* coef, const int* atom_ptr,
                              const int* entries, int q1_cap, float* gw, unsigned* sync, GridBarrier* flags,
                              DevStats* stats, int timers, const int* last, int slice_target, int grid,
                              cudaStream_t s) {
  const int cap = update_res_capacity(n);
  if (cap < 16 || grid < 1) return cudaErrorInvalidValue;
  UpdBatch b;
  std::memset(&b, 0, sizeof(b));
  b.ngroups = 1;
  UpdGroup& g = b.g[0];
  g.R = R;
  g.D = D;
  g.coef = coef;
  g.atom_ptr = atom_ptr;
  g.entries = entries;
  g.last = last;
  g.gw = gw;
  g.sync = sync;
  g.n = n;
  g.K = K;
  g.L = L;
  g.q1_cap = q1_cap;
  g.cap = cap;
  g.cta_begin = 0;
  g.ctas = grid;
  g.slice_target = slice_target;
  return launch_update_batch(b, flags, stats, timers, grid, s);
}

}  // namespace ksvd
