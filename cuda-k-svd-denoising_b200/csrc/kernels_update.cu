// Sequential K-SVD dictionary update (updateDictionary,
// cuda_svd_denoiser.cu:285-362).
//
// 1. CSR of atom -> (patch, slot) entries, patches ascending, built from the
//    compact codes, nonzero coefficients only.  Replaces
//    findRelevantIndicesKernel (:36-50), which scans the dense K x N code
//    matrix with one thread per atom.
// 2. One persistent cooperative kernel walks the atoms in order (the
//    reference's Gauss-Seidel sweep, :309-361).  For atom j with support
//    Omega_j (c entries; only the first 1024 with the Q1 cap):
//      A  every CTA forms its slice of the residual columns
//           e_p = y_p - sum_{s != j} x_{s,p} d_s
//         in shared memory and accumulates the partial Gram sum e_p e_p^T;
//      B  the partial Grams are summed in a fixed order, each CTA owning a
//         slice of the n x n entries;
//      C  every CTA loads the summed Gram and runs the same power iteration,
//         starting from the old atom, to its top eigenvector u (the top left
//         singular vector of E, which is what gesvdj's U[:,0] is used for,
//         :328-346); u is signed so that u . d_j(old) >= 0; then
//           d_j <- u,  x_{j,p} <- u . e_p  (= sigma v_p, :349-358)
//         with x_{j,p} = 0 for entries beyond the cap.
//    Phases are separated by a bounded software grid barrier.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "ksvd_internal.cuh"

namespace ksvd {

// ---------------------------------------------------------------------------
// CSR build
// ---------------------------------------------------------------------------
constexpr int kCsrChunk = 256;  // patches per CTA (8 warps x 32)

int64_t csr_num_chunks(int64_t N) { return (N + kCsrChunk - 1) / kCsrChunk; }

__device__ __forceinline__ bool entry_valid(const int32_t* idx, const float* coef, int64_t e, int K) {
  int a = idx[e];
  return a >= 0 && a < K && coef[e] != 0.0f;
}

// counts[a * nchunks + c] = entries of atom a in chunk c
__global__ void __launch_bounds__(kCsrChunk) csr_count_kernel(const int32_t* __restrict__ idx,
                                                              const float* __restrict__ coef, int64_t N, int L,
                                                              int K, int64_t nchunks, int* __restrict__ counts) {
  extern __shared__ int hist[];
  for (int a = threadIdx.x; a < K; a += blockDim.x) hist[a] = 0;
  __syncthreads();
  const int64_t p = int64_t(blockIdx.x) * kCsrChunk + threadIdx.x;
  if (p < N)
    for (int s = 0; s < L; ++s)
      if (entry_valid(idx, coef, p * L + s, K)) atomicAdd(&hist[idx[p * L + s]], 1);
  __syncthreads();
  for (int a = threadIdx.x; a < K; a += blockDim.x) counts[int64_t(a) * nchunks + blockIdx.x] = hist[a];
}

// One CTA per atom: exclusive scan of its chunk counts in place, total out.
__global__ void __launch_bounds__(256) csr_scan_chunks_kernel(int* __restrict__ counts, int64_t nchunks,
                                                              int* __restrict__ atom_tot) {
  __shared__ int warp_tot[8];
  __shared__ int carry_s;
  int* col = counts + int64_t(blockIdx.x) * nchunks;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (int64_t base = 0; base < nchunks; base += 256) {
    const int64_t c = base + threadIdx.x;
    const int v = (c < nchunks) ? col[c] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    int wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += warp_tot[w];
    const int carry = carry_s;
    if (c < nchunks) col[c] = carry + wbase + x - v;
    __syncthreads();
    if (threadIdx.x == 255) carry_s = carry + wbase + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) atom_tot[blockIdx.x] = carry_s;
}

// atom_ptr = exclusive scan of atom totals (single CTA).
__global__ void csr_scan_atoms_kernel(const int* __restrict__ atom_tot, int K, int* __restrict__ atom_ptr) {
  if (threadIdx.x == 0) {
    int run = 0;
    for (int a = 0; a < K; ++a) {
      atom_ptr[a] = run;
      run += atom_tot[a];
    }
    atom_ptr[K] = run;
  }
}

// Entries in patch order: a warp owns 32 consecutive patches; an entry's
// position is atom_ptr + chunk offset + earlier warps' count + the number of
// entries of the same atom in lower lanes of its warp.
__global__ void __launch_bounds__(kCsrChunk) csr_fill_kernel(const int32_t* __restrict__ idx,
                                                             const float* __restrict__ coef, int64_t N, int L,
                                                             int K, int64_t nchunks, const int* __restrict__ counts,
                                                             const int* __restrict__ atom_ptr,
                                                             int* __restrict__ entries) {
  extern __shared__ int csr_sm[];
  int* wcnt = csr_sm;              // 8 x K
  int* watoms = csr_sm + 8 * K;    // 8 x 32 x L
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = threadIdx.x; t < 8 * K; t += blockDim.x) wcnt[t] = 0;
  const int64_t p = int64_t(blockIdx.x) * kCsrChunk + threadIdx.x;
  int* mine = watoms + (warp * 32 + lane) * L;
  for (int s = 0; s < L; ++s) {
    int a = -1;
    if (p < N && entry_valid(idx, coef, p * L + s, K)) a = idx[p * L + s];
    mine[s] = a;
  }
  __syncthreads();
  for (int s = 0; s < L; ++s)
    if (mine[s] >= 0) atomicAdd(&wcnt[warp * K + mine[s]], 1);
  __syncthreads();
  for (int a = threadIdx.x; a < K; a += blockDim.x) {
    int run = atom_ptr[a] + counts[int64_t(a) * nchunks + blockIdx.x];
    for (int w = 0; w < 8; ++w) {
      int t = wcnt[w * K + a];
      wcnt[w * K + a] = run;
      run += t;
    }
  }
  __syncthreads();
  const int* wa = watoms + warp * 32 * L;
  for (int s = 0; s < L; ++s) {
    const int a = mine[s];
    if (a < 0) continue;
    int rank = 0;
    for (int l2 = 0; l2 < lane; ++l2)
      for (int s2 = 0; s2 < L; ++s2) rank += (wa[l2 * L + s2] == a);
    entries[wcnt[warp * K + a] + rank] = int(p * L + s);
  }
}

cudaError_t launch_csr_build(const int32_t* idx, const float* coef, int64_t N, int L, int K, CsrWork w,
                             cudaStream_t s) {
  const int64_t nch = w.nchunks;
  csr_count_kernel<<<unsigned(nch), kCsrChunk, K * sizeof(int), s>>>(idx, coef, N, L, K, nch, w.chunk_counts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // atom totals are parked in atom_ptr[0..K) temporarily? no: separate area
  int* atom_tot = w.atom_ptr + (K + 1);
  csr_scan_chunks_kernel<<<K, 256, 0, s>>>(w.chunk_counts, nch, atom_tot);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  csr_scan_atoms_kernel<<<1, 32, 0, s>>>(atom_tot, K, w.atom_ptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  size_t smem = (size_t(8) * K + size_t(8) * 32 * L) * sizeof(int);
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(csr_fill_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
  }
  csr_fill_kernel<<<unsigned(nch), kCsrChunk, smem, s>>>(idx, coef, N, L, K, nch, w.chunk_counts, w.atom_ptr,
                                                         w.entries);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Persistent update kernel
//
// Shared memory: the dictionary (K x n FP32, when it fits; the atoms are
// updated in place by every CTA, so it never has to be re-read), one chunk of
// kEChunk residual columns, their metadata (patch, slot, the other atoms and
// coefficients of the patch), u, the old atom and reduction scratch.
// The n x n Gram is held in registers in the 16 x 16 thread layout of the
// phase-A accumulators (TN x TN per thread) and the power iteration runs on
// it there: v = G u is a per-thread TN x TN block product plus a reduction
// over the 16 lanes that share a row block.
// ---------------------------------------------------------------------------
constexpr int kUpdThreads = 256;
constexpr int kEChunk = 32;              // residual columns staged per pass
constexpr int kMinEntriesPerCta = 16;    // phase A uses ceil(c / 16) CTAs at most
constexpr int kMaxPowerIters = 1000;
constexpr float kPowerTol = 2.0e-7f;     // max |u_new - u_old| to stop

struct UpdLayout {
  size_t off_ds, off_e, off_mp, off_ms, off_ma, off_mc, off_u, off_dold, off_red, total;
};

__host__ __device__ inline size_t upd_al16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline UpdLayout upd_layout(int n, int K, int L, bool dsmem) {
  const int npad = (n + 15) / 16 * 16;
  UpdLayout o;
  size_t off = 0;
  o.off_ds = off;
  off = upd_al16(off + (dsmem ? size_t(K) * n * 4 : 0));
  o.off_e = off;
  off = upd_al16(off + size_t(kEChunk) * n * 4);
  o.off_mp = off;
  off = upd_al16(off + kEChunk * 4);
  o.off_ms = off;
  off = upd_al16(off + kEChunk * 4);
  o.off_ma = off;
  off = upd_al16(off + size_t(kEChunk) * L * 4);
  o.off_mc = off;
  off = upd_al16(off + size_t(kEChunk) * L * 4);
  o.off_u = off;
  off = upd_al16(off + size_t(npad) * 4);
  o.off_dold = off;
  off = upd_al16(off + size_t(npad) * 4);
  o.off_red = off;
  off = upd_al16(off + 64 * 4);
  o.total = off;
  return o;
}

template <int TN, bool DSMEM>
__global__ void __launch_bounds__(kUpdThreads, 1)
    update_kernel(const float* __restrict__ Y, int64_t N, int n, float* D, int K, int L,
                  const int32_t* __restrict__ idx, float* coef, const int* __restrict__ atom_ptr,
                  const int* __restrict__ entries, int q1_cap, float* gpart, float* gsum, GridBarrier* bar,
                  DevStats* stats) {
  extern __shared__ __align__(16) unsigned char usm[];
  const UpdLayout lo = upd_layout(n, K, L, DSMEM);
  float* Ds = reinterpret_cast<float*>(usm + lo.off_ds);
  float* E = reinterpret_cast<float*>(usm + lo.off_e);
  int* mp = reinterpret_cast<int*>(usm + lo.off_mp);
  int* ms = reinterpret_cast<int*>(usm + lo.off_ms);
  int* ma = reinterpret_cast<int*>(usm + lo.off_ma);
  float* mc = reinterpret_cast<float*>(usm + lo.off_mc);
  float* u = reinterpret_cast<float*>(usm + lo.off_u);
  float* dold = reinterpret_cast<float*>(usm + lo.off_dold);
  float* red = reinterpret_cast<float*>(usm + lo.off_red);
  (void)N;

  const unsigned G = gridDim.x;
  const int b = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ti = tid >> 4, tj = tid & 15;
  const int nn = n * n;
  const int npad = 16 * TN;

  if (DSMEM) {
    for (int t = tid; t < K * n; t += kUpdThreads) Ds[t] = __ldcg(D + t);
    __syncthreads();
  }
  auto datom = [&](int a, int i) -> float { return DSMEM ? Ds[a * n + i] : __ldcg(D + int64_t(a) * n + i); };

  // Stages metadata of entries [t0, t0 + m) and builds their residual
  // columns e_p = y_p - sum_{s != slot} x_s d_s into E.
  auto build_chunk = [&](int beg, int t0, int m) {
    for (int t = tid; t < kEChunk * L; t += kUpdThreads) {
      const int q = t / L, s = t - q * L;
      if (q < m) {
        const int es = __ldg(entries + beg + t0 + q);
        const int p = es / L, sl = es - p * L;
        if (s == 0) {
          mp[q] = p;
          ms[q] = sl;
        }
        const int a = __ldg(idx + int64_t(p) * L + s);
        const bool ok = (s != sl) && a >= 0 && a < K;
        ma[q * L + s] = ok ? a : -1;
        mc[q * L + s] = ok ? __ldcg(coef + int64_t(p) * L + s) : 0.0f;
      }
    }
    __syncthreads();
    for (int q = warp; q < kEChunk; q += kUpdThreads / 32) {
      float* er = E + q * n;
      if (q < m) {
        const int64_t p = mp[q];
        for (int i = lane; i < n; i += 32) {
          float e = __ldg(Y + p * n + i);
          for (int s = 0; s < L; ++s) {
            const int a = ma[q * L + s];
            if (a >= 0) e = fmaf(-mc[q * L + s], datom(a, i), e);
          }
          er[i] = e;
        }
      } else {
        for (int i = lane; i < n; i += 32) er[i] = 0.0f;
      }
    }
    __syncthreads();
  };

  float blk[TN][TN];
  const bool timer = (b == 0 && tid == 0);
  unsigned long long tmark = timer ? globaltimer_ns() : 0ull;
  auto lap = [&](int slot) {
    if (timer) {
      const unsigned long long t = globaltimer_ns();
      stats->phase_ns[slot] += t - tmark;
      tmark = t;
    }
  };

  for (int j = 0; j < K; ++j) {
    const int beg = atom_ptr[j];
    const int c = atom_ptr[j + 1] - beg;
    if (c == 0) continue;
    const int c_eff = (q1_cap && c > 1024) ? 1024 : c;
    const int active = min(int(G), (c_eff + kMinEntriesPerCta - 1) / kMinEntriesPerCta);
    for (int i = tid; i < npad; i += kUpdThreads) dold[i] = (i < n) ? datom(j, i) : 0.0f;

    // ---- phase A: partial Gram of this CTA's residual columns -------------
    const int sb = int(int64_t(c_eff) * b / active), se = int(int64_t(c_eff) * (b + 1) / active);
    const bool in_a = b < active;
    if (in_a) {
#pragma unroll
      for (int r = 0; r < TN; ++r)
#pragma unroll
        for (int s = 0; s < TN; ++s) blk[r][s] = 0.0f;
      for (int t0 = sb; t0 < se; t0 += kEChunk) {
        const int m = min(kEChunk, se - t0);
        build_chunk(beg, t0, m);
        for (int q = 0; q < m; ++q) {
          const float* er = E + q * n;
          float ra[TN], rb[TN];
#pragma unroll
          for (int r = 0; r < TN; ++r) {
            const int i = ti + 16 * r;
            ra[r] = (i < n) ? er[i] : 0.0f;
          }
#pragma unroll
          for (int s = 0; s < TN; ++s) {
            const int k = tj + 16 * s;
            rb[s] = (k < n) ? er[k] : 0.0f;
          }
#pragma unroll
          for (int r = 0; r < TN; ++r)
#pragma unroll
            for (int s = 0; s < TN; ++s) blk[r][s] = fmaf(ra[r], rb[s], blk[r][s]);
        }
        if (t0 + kEChunk < se) __syncthreads();  // E is rebuilt by the next chunk
      }
      float* gp = gpart + size_t(b) * nn;
#pragma unroll
      for (int r = 0; r < TN; ++r)
#pragma unroll
        for (int s = 0; s < TN; ++s) {
          const int i = ti + 16 * r, k = tj + 16 * s;
          if (i < n && k < n) gp[i * n + k] = blk[r][s];
        }
    }
    __syncthreads();
    lap(0);
    if (!grid_sync(bar, G)) return;
    lap(1);

    // ---- phase B: fixed-order sum of the active partial Grams --------------
    {
      const int qb = int(int64_t(nn) * b / G), qe = int(int64_t(nn) * (b + 1) / G);
      for (int q = qb + tid; q < qe; q += kUpdThreads) {
        float s = 0.0f;
        for (int bb = 0; bb < active; ++bb) s += __ldcg(gpart + size_t(bb) * nn + q);
        gsum[q] = s;
      }
    }
    __syncthreads();
    lap(2);
    if (!grid_sync(bar, G)) return;
    lap(3);

    // ---- phase C: power iteration on the register-resident Gram ------------
#pragma unroll
    for (int r = 0; r < TN; ++r)
#pragma unroll
      for (int s = 0; s < TN; ++s) {
        const int i = ti + 16 * r, k = tj + 16 * s;
        blk[r][s] = (i < n && k < n) ? __ldcg(gsum + i * n + k) : 0.0f;
      }
    for (int i = tid; i < npad; i += kUpdThreads) u[i] = dold[i];
    __syncthreads();
    int iters = 0;
    for (int it = 0; it < kMaxPowerIters; ++it) {
      float ub[TN], v[TN];
#pragma unroll
      for (int s = 0; s < TN; ++s) ub[s] = u[tj + 16 * s];
#pragma unroll
      for (int r = 0; r < TN; ++r) {
        float acc = 0.0f;
#pragma unroll
        for (int s = 0; s < TN; ++s) acc = fmaf(blk[r][s], ub[s], acc);
        v[r] = acc;
      }
#pragma unroll
      for (int r = 0; r < TN; ++r) {
#pragma unroll
        for (int o = 1; o < 16; o <<= 1) v[r] += __shfl_xor_sync(0xffffffffu, v[r], o);
      }
      float part = 0.0f;
      if (tj == 0) {
#pragma unroll
        for (int r = 0; r < TN; ++r) part = fmaf(v[r], v[r], part);
      }
      const float nrm2 = block_sum(part, red);
      iters = it + 1;
      if (!(nrm2 > 0.0f)) break;  // E == 0: keep the old atom direction
      const float inv = 1.0f / sqrtf(nrm2);
      float d = 0.0f;
      if (tj == 0) {
#pragma unroll
        for (int r = 0; r < TN; ++r) {
          const float vn = v[r] * inv;
          d = fmaxf(d, fabsf(vn - u[ti + 16 * r]));
          u[ti + 16 * r] = vn;
        }
      }
      const float dmax = block_max(d, red);
      if (dmax < kPowerTol) break;
    }
    lap(4);
    const float sd = block_sum((tid < n) ? u[tid] * dold[tid] : 0.0f, red);
    if (sd < 0.0f && tid < n) u[tid] = -u[tid];
    __syncthreads();
    if (DSMEM)
      for (int i = tid; i < n; i += kUpdThreads) Ds[j * n + i] = u[i];
    if (b == 0) {
      for (int i = tid; i < n; i += kUpdThreads) D[int64_t(j) * n + i] = u[i];
      if (tid == 0) {
        atomicAdd(&stats->power_iters, (unsigned long long)iters);
        atomicAdd(&stats->atoms_updated, 1ull);
      }
    }

    // ---- coefficients x_{j,p} = u . e_p ------------------------------------
    if (in_a) {
      const bool resident = (se - sb) <= kEChunk;  // E still holds this CTA's columns
      for (int t0 = sb; t0 < se; t0 += kEChunk) {
        const int m = min(kEChunk, se - t0);
        if (!resident) {
          __syncthreads();
          build_chunk(beg, t0, m);
        }
        for (int q = warp; q < m; q += kUpdThreads / 32) {
          const float* er = E + q * n;
          float dp = 0.0f;
          for (int i = lane; i < n; i += 32) dp = fmaf(u[i], er[i], dp);
          dp = warp_sum(dp);
          if (lane == 0) coef[int64_t(mp[q]) * L + ms[q]] = dp;
        }
      }
    }
    if (c > c_eff) {  // Q1 cap: coefficients beyond the first 1024 entries become 0
      const int zb = c_eff + int(int64_t(c - c_eff) * b / G), ze = c_eff + int(int64_t(c - c_eff) * (b + 1) / G);
      for (int t = zb + tid; t < ze; t += kUpdThreads) coef[__ldg(entries + beg + t)] = 0.0f;
    }
    __syncthreads();
    lap(5);
    if (!grid_sync(bar, G)) return;
    lap(6);
  }
}

__global__ void accumulate_phases_kernel(const DevStats* __restrict__ src, DevStats* __restrict__ dst) {
  const int t = threadIdx.x;
  if (t < 16) dst->phase_ns[t] += src->phase_ns[t];
}

cudaError_t launch_accumulate_phases(const DevStats* src, DevStats* dst, cudaStream_t s) {
  accumulate_phases_kernel<<<1, 32, 0, s>>>(src, dst);
  return cudaGetLastError();
}

bool update_supported(int n) { return n >= 1 && n <= 160; }

static bool dict_in_smem(int n, int K, int L) { return upd_layout(n, K, L, true).total <= 220 * 1024; }

size_t update_smem_bytes(int n, int K, int L) { return upd_layout(n, K, L, dict_in_smem(n, K, L)).total; }

template <int TN>
static void* update_fn(bool dsmem) {
  return dsmem ? reinterpret_cast<void*>(update_kernel<TN, true>) : reinterpret_cast<void*>(update_kernel<TN, false>);
}

static void* pick_update(int n, bool dsmem) {
  switch ((n + 15) / 16) {
    case 1: return update_fn<1>(dsmem);
    case 2: return update_fn<2>(dsmem);
    case 3: return update_fn<3>(dsmem);
    case 4: return update_fn<4>(dsmem);
    case 5: return update_fn<5>(dsmem);
    case 6: return update_fn<6>(dsmem);
    case 7: return update_fn<7>(dsmem);
    case 8: return update_fn<8>(dsmem);
    case 9: return update_fn<9>(dsmem);
    case 10: return update_fn<10>(dsmem);
    default: return nullptr;
  }
}

int update_grid_size(int n, int K, int L, int num_sms) {
  const bool dsmem = dict_in_smem(n, K, L);
  void* fn = pick_update(n, dsmem);
  if (!fn) return 0;
  const size_t smem = update_smem_bytes(n, K, L);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kUpdThreads, smem) != cudaSuccess) return 0;
  if (per_sm < 1) return 0;
  return num_sms;  // one CTA per SM: co-resident by construction
}

cudaError_t launch_update(const float* patches, int64_t N, int n, float* dict, int K, int L, const int32_t* idx,
                          float* coef, CsrWork w, int q1_cap, float* gpart, float* gsum, GridBarrier* bar,
                          DevStats* stats, int grid, cudaStream_t s) {
  const bool dsmem = dict_in_smem(n, K, L);
  void* fn = pick_update(n, dsmem);
  if (!fn || grid < 1) return cudaErrorInvalidValue;
  const size_t smem = update_smem_bytes(n, K, L);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(bar, 0, sizeof(GridBarrier), s);
  if (e != cudaSuccess) return e;
  const int* atom_ptr = w.atom_ptr;
  const int* entries = w.entries;
  void* args[] = {(void*)&patches, (void*)&N,       (void*)&n,       (void*)&dict,     (void*)&K,
                  (void*)&L,       (void*)&idx,     (void*)&coef,    (void*)&atom_ptr, (void*)&entries,
                  (void*)&q1_cap,  (void*)&gpart,   (void*)&gsum,    (void*)&bar,      (void*)&stats};
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kUpdThreads), args, smem, s);
}

}  // namespace ksvd
