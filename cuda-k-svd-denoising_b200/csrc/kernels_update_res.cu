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
// split over `active` CTAs (about kUrTargetSlice entries each); each keeps its
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

#include "device_util.cuh"
#include "ksvd_internal.cuh"

namespace ksvd {

constexpr int kUrThreads = 512;
constexpr int kUrWarps = kUrThreads / 32;
constexpr int kUrTargetSlice = 96;    // entries per CTA before another CTA joins an atom
constexpr int kUrMaxIters = 200;
constexpr float kUrTol = 2.0e-7f;     // max |u_new - u_old| to stop
constexpr size_t kUrSmemMax = 232448 - 256;  // opt-in shared memory per block, less the static part

__host__ __device__ inline int ur_n4(int n) { return (n + 3) & ~3; }

// Shared memory: [cap x n4] columns | ent[2][cap] | xold[2][cap] | u[n4] |
// dold[n4] | dnext[n4] | wred[kUrWarps x n4]
__host__ __device__ inline size_t ur_fixed_bytes(int n) {
  const int n4 = ur_n4(n);
  return size_t(n4) * 4 * 3 + size_t(kUrWarps) * n4 * 4;
}

int update_res_capacity(int n) {
  const size_t per = size_t(ur_n4(n)) * 4 + 16;
  const size_t fixed = ur_fixed_bytes(n);
  if (fixed + per * 16 > kUrSmemMax) return 0;
  // a multiple of 4 keeps u, dold, dnext and wred (read as float4) 16-byte aligned
  return int((kUrSmemMax - fixed) / per) & ~3;
}

size_t update_res_smem_bytes(int n, int cap) { return size_t(cap) * (size_t(ur_n4(n)) * 4 + 16) + ur_fixed_bytes(n); }

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

__host__ __device__ inline int ur_active(int c, int G) {
  const int a = (c + kUrTargetSlice - 1) / kUrTargetSlice;
  return a < G ? a : G;
}

// residual_kernel: R = Y - X D, one warp per patch (the code slots are read
// by every lane of the warp: uniform, cached loads).
__global__ void __launch_bounds__(256) residual_kernel(const float* __restrict__ Y, int64_t N, int n,
                                                       const float* __restrict__ D, int K, int L,
                                                       const int32_t* __restrict__ idx,
                                                       const float* __restrict__ coef, float* __restrict__ R) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t p = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); p < N; p += warps) {
    for (int i = lane; i < n; i += 32) {
      float r = Y[p * n + i];
      for (int s = 0; s < L; ++s) {
        const int a = __ldg(idx + p * L + s);
        const float x = __ldg(coef + p * L + s);
        if (a >= 0 && a < K && x != 0.0f) r = fmaf(-x, __ldg(D + int64_t(a) * n + i), r);
      }
      R[p * n + i] = r;
    }
  }
}

// Arrive on a counter with release semantics: after a __syncthreads(), the
// writes of every thread of the CTA are visible to whoever acquires the count.
KSVD_DEV void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <int NW>
__global__ void __launch_bounds__(kUrThreads, 1)
    update_res_kernel(float* R, int n, float* D, int K, int L, float* coef, const int* __restrict__ atom_ptr,
                      const int* __restrict__ entries, int q1_cap, int cap, float* gw, unsigned* sync,
                      GridBarrier* flags, DevStats* stats, int timers) {
  extern __shared__ __align__(16) unsigned char ursm[];
  const int n4 = ur_n4(n);
  float* Es = reinterpret_cast<float*>(ursm);
  int* ent_b = reinterpret_cast<int*>(ursm + size_t(cap) * n4 * 4);  // [2][cap]
  float* xold_b = reinterpret_cast<float*>(ent_b + 2 * cap);           // [2][cap]
  float* u = xold_b + 2 * cap;
  float* dold = u + n4;
  float* dnext = dold + n4;
  float* wred = dnext + n4;
  __shared__ int s_ok;
  __shared__ int s_stop;
  __shared__ unsigned long long s_ph[8];  // phase times of this CTA (slots 0..7)

  const int G = int(gridDim.x), b = int(blockIdx.x);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned* iter_cnt = sync;
  unsigned* done_cnt = sync + K;
  const int F = n4 / 4;                       // float4 per partial row
  int Gr = kUrThreads / F;                    // reduction groups
  if (Gr > kUrWarps) Gr = kUrWarps;
  if (Gr < 1) Gr = 1;

  // phase times gather in shared memory and are flushed once at the end
  const bool timer = (timers != 0 && b == 0 && tid == 0);
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
  // this CTA's slice [sb, se) of atom a's c entries starting at beg
  auto slice_of = [&](int a, int& beg, int& c, int& active, int& sb, int& se) {
    beg = atom_ptr[a];
    c = atom_ptr[a + 1] - beg;
    active = ur_active(c, G);
    sb = int(int64_t(c) * b / active);
    se = int(int64_t(c) * (b + 1) / active);
  };
  // entries and old coefficients of [sb, sb + cnt) into meta buffer `slot`
  // and atom a into dst (all threads; several loads in flight per thread)
  auto load_meta = [&](int beg, int sb, int cnt, int slot, int a, float* dst) {
    int* ent = ent_b + slot * cap;
    float* xo = xold_b + slot * cap;
    constexpr int kB = 4;
    for (int t0 = tid; t0 < cnt; t0 += kUrThreads * kB) {
      int e[kB];
#pragma unroll
      for (int k = 0; k < kB; ++k) {
        const int t = t0 + k * kUrThreads;
        e[k] = (t < cnt) ? __ldg(entries + beg + sb + t) : 0;
      }
      float x[kB];
#pragma unroll
      for (int k = 0; k < kB; ++k) x[k] = (t0 + k * kUrThreads < cnt) ? __ldcg(coef + e[k]) : 0.0f;
#pragma unroll
      for (int k = 0; k < kB; ++k) {
        const int t = t0 + k * kUrThreads;
        if (t < cnt) {
          ent[t] = e[k];
          xo[t] = x[k];
        }
      }
    }
    for (int i = tid; i < n4; i += kUrThreads) dst[i] = (i < n) ? __ldcg(D + int64_t(a) * n + i) : 0.0f;
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
    const int* ent_s = ent_b + slot * cap;
    const float* xold_s = xold_b + slot * cap;

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

    // ---- resident columns e_q = r_q + x_q d_old (loads batched) -----------
    if ((n & 3) == 0) {
      constexpr int kB = 8;
      const int total = mres * F;
      for (int f0 = tid; f0 < total; f0 += kUrThreads * kB) {
        float4 r[kB];
#pragma unroll
        for (int k = 0; k < kB; ++k) {
          const int f = f0 + k * kUrThreads;
          if (f < total) {
            const int q = f / F, i4 = f - q * F;
            r[k] = __ldcg(reinterpret_cast<const float4*>(R + int64_t(ent_s[q] / L) * n) + i4);
          }
        }
#pragma unroll
        for (int k = 0; k < kB; ++k) {
          const int f = f0 + k * kUrThreads;
          if (f < total) {
            const int q = f / F, i4 = f - q * F;
            const float x = xold_s[q];
            const float4 d = reinterpret_cast<const float4*>(dold)[i4];
            float4 e;
            e.x = fmaf(x, d.x, r[k].x);
            e.y = fmaf(x, d.y, r[k].y);
            e.z = fmaf(x, d.z, r[k].z);
            e.w = fmaf(x, d.w, r[k].w);
            reinterpret_cast<float4*>(Es + size_t(q) * n4)[i4] = e;
          }
        }
      }
    } else {
      for (int f = tid; f < mres * n4; f += kUrThreads) {
        const int q = f / n4, i = f - q * n4;
        float e = 0.0f;
        if (i < n) e = fmaf(xold_s[q], dold[i], __ldcg(R + int64_t(ent_s[q] / L) * n + i));
        Es[size_t(q) * n4 + i] = e;
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
    const int mcr = mc < cap ? mc : cap;
    for (int it = 0; it < kUrMaxIters; ++it) {
      float ur[NW], wacc[NW];
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const int i = lane + 32 * k;
        ur[k] = (i < n) ? u[i] : 0.0f;
        wacc[k] = 0.0f;
      }
      for (int q = warp; q < mcr; q += kUrWarps) {  // resident columns
        const float* er = Es + size_t(q) * n4;
        float ev[NW];
        float dp = 0.0f;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const int i = lane + 32 * k;
          ev[k] = (i < n) ? er[i] : 0.0f;
          dp = fmaf(ur[k], ev[k], dp);
        }
        dp = warp_sum(dp);
#pragma unroll
        for (int k = 0; k < NW; ++k) wacc[k] = fmaf(dp, ev[k], wacc[k]);
      }
      for (int q = cap + warp; q < mc; q += 2 * kUrWarps) {  // streamed columns
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
        if (i < n4) wred[warp * n4 + i] = wacc[k];
      }
      __syncthreads();
      float* gwp = gw + (size_t(it & 1) * G + b) * n4;
      for (int i = tid; i < n4; i += kUrThreads) {
        float s = 0.0f;
#pragma unroll
        for (int w = 0; w < kUrWarps; ++w) s += wred[w * n4 + i];
        __stcg(gwp + i, s);
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
          constexpr int kB = 8;
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
          reinterpret_cast<float4*>(wred + g * n4)[f] = acc;
        }
      }
      __syncthreads();
      iters = it + 1;
      // warp 0 finishes the step: w, its norm, the new u, the change, the
      // stop decision and, when stopping, the sign (u . d_old >= 0)
      if (warp == 0) {
        float wv[NW];
        float s2 = 0.0f;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const int i = lane + 32 * k;
          float wi = 0.0f;
          if (i < n)
            for (int g = 0; g < Gr; ++g) wi += wred[g * n4 + i];
          wv[k] = wi;
          s2 = fmaf(wi, wi, s2);
        }
        const float nrm2 = warp_sum(s2);
        bool stop;
        if (!(nrm2 > 0.0f)) {
          stop = true;  // E == 0: keep the old atom direction
        } else {
          const float inv = 1.0f / sqrtf(nrm2);
          float dm = 0.0f;
#pragma unroll
          for (int k = 0; k < NW; ++k) {
            const int i = lane + 32 * k;
            if (i < n) {
              const float un = wv[k] * inv;
              dm = fmaxf(dm, fabsf(un - u[i]));
              u[i] = un;
            }
          }
          dm = warp_max(dm);
          // stop when the change is below the tolerance, or when the
          // observed contraction rho = dm / dprev puts the remaining distance
          // to the limit, about dm * rho / (1 - rho), below it
          const float rho = (it > 0 && dprev > 0.0f) ? dm / dprev : 1.0f;
          stop = dm < kUrTol || (rho < 0.5f && dm < 1e-3f && dm * rho < 0.5f * kUrTol * (1.0f - rho) * 2.0f);
          dprev = dm;
        }
        if (stop) {
          float sd = 0.0f;
#pragma unroll
          for (int k = 0; k < NW; ++k) {
            const int i = lane + 32 * k;
            if (i < n) sd = fmaf(u[i], dold[i], sd);
          }
          sd = warp_sum(sd);
          if (sd < 0.0f)
#pragma unroll
            for (int k = 0; k < NW; ++k) {
              const int i = lane + 32 * k;
              if (i < n) u[i] = -u[i];
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
    {
      float ur[NW];
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        const int i = lane + 32 * k;
        ur[k] = (i < n) ? u[i] : 0.0f;
      }
      for (int q = warp; q < mres; q += kUrWarps) {  // resident columns
        const float* er = Es + size_t(q) * n4;
        float ev[NW];
        float x = 0.0f;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const int i = lane + 32 * k;
          ev[k] = (i < n) ? er[i] : 0.0f;
          x = fmaf(ur[k], ev[k], x);
        }
        x = warp_sum(x);
        if (q >= mc) x = 0.0f;
        const int e = ent_s[q];
        float* rr = R + int64_t(e / L) * n;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const int i = lane + 32 * k;
          if (i < n) __stcg(rr + i, fmaf(-x, ur[k], ev[k]));
        }
        if (lane == 0) __stcg(coef + e, x);
      }
      for (int q = cap + warp; q < m; q += 2 * kUrWarps) {  // streamed columns
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
#pragma unroll
        for (int k = 0; k < NW; ++k) {
          const int i = lane + 32 * k;
          if (i < n) __stcg(ra + i, fmaf(-x0, ur[k], e0[k]));
        }
        if (lane == 0) __stcg(coef + ea, x0);
        if (eb >= 0) {
          float* rb = R + int64_t(eb / L) * n;
#pragma unroll
          for (int k = 0; k < NW; ++k) {
            const int i = lane + 32 * k;
            if (i < n) __stcg(rb + i, fmaf(-x1, ur[k], e1[k]));
          }
          if (lane == 0) __stcg(coef + eb, x1);
        }
      }
    }
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
                            const float* coef, float* R, int num_sms, cudaStream_t s) {
  const int64_t want = (N + 7) / 8;
  const int blocks = int(want < int64_t(num_sms) * 16 ? want : int64_t(num_sms) * 16);
  residual_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(Y, N, n, D, K, L, idx, coef, R);
  return cudaGetLastError();
}

cudaError_t launch_update_res(float* R, int n, float* D, int K, int L, float* coef, const int* atom_ptr,
                              const int* entries, int q1_cap, float* gw, unsigned* sync, GridBarrier* flags,
                              DevStats* stats, int timers, int grid, cudaStream_t s) {
  void* fn = pick_update_res(n);
  const int cap = update_res_capacity(n);
  if (!fn || cap < 16 || grid < 1) return cudaErrorInvalidValue;
  const size_t smem = update_res_smem_bytes(n, cap);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(sync, 0, size_t(2) * K * sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  int capv = cap;
  void* args[] = {(void*)&R,       (void*)&n,       (void*)&D,      (void*)&K,    (void*)&L,
                  (void*)&coef,    (void*)&atom_ptr, (void*)&entries, (void*)&q1_cap, (void*)&capv,
                  (void*)&gw,      (void*)&sync,    (void*)&flags,  (void*)&stats,   (void*)&timers};
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kUrThreads), args, smem, s);
}

}  // namespace ksvd
