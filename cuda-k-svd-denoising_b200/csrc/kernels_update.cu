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
// ---------------------------------------------------------------------------
constexpr int kUpdThreads = 256;
constexpr int kEChunk = 32;              // residual columns staged per pass
constexpr int kMaxPowerIters = 1000;
constexpr float kPowerTol = 2.0e-7f;     // max |u_new - u_old| to stop

__host__ __device__ inline size_t update_floats(int n) {
  size_t a = size_t(kEChunk) * n, b = size_t(n) * (n + 1);
  return (a > b ? a : b) + 3 * size_t(n) + 64;
}

// e_p (lane-strided element i) for entry (p, slot): y_p - sum_{s != slot} x_s d_s.
__device__ __forceinline__ float residual_elem(const float* __restrict__ Y, const float* D, const int32_t* idx,
                                               const float* coef, int64_t p, int slot, int L, int n, int K, int i) {
  float e = __ldg(Y + p * n + i);
  for (int s = 0; s < L; ++s) {
    if (s == slot) continue;
    const int a = __ldg(idx + p * L + s);
    if (a < 0 || a >= K) continue;
    e = fmaf(-__ldcg(coef + p * L + s), __ldcg(D + int64_t(a) * n + i), e);
  }
  return e;
}

template <int TN>
__global__ void __launch_bounds__(kUpdThreads, 1)
    update_kernel(const float* __restrict__ Y, int64_t N, int n, float* D, int K, int L,
                  const int32_t* __restrict__ idx, float* coef, const int* __restrict__ atom_ptr,
                  const int* __restrict__ entries, int q1_cap, float* gpart, float* gsum, GridBarrier* bar,
                  DevStats* stats) {
  extern __shared__ __align__(16) float sm[];
  const size_t big = (size_t(kEChunk) * n > size_t(n) * (n + 1)) ? size_t(kEChunk) * n : size_t(n) * (n + 1);
  float* E = sm;
  float* Gs = sm;
  float* u = sm + big;
  float* dold = u + n;
  float* spare = dold + n;
  float* red = spare + n;  // 64 floats
  (void)N;
  (void)spare;

  const unsigned G = gridDim.x;
  const int b = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ti = tid >> 4, tj = tid & 15;
  const int nn = n * n;

  for (int j = 0; j < K; ++j) {
    const int beg = atom_ptr[j];
    const int c = atom_ptr[j + 1] - beg;
    if (c == 0) continue;
    const int c_eff = (q1_cap && c > 1024) ? 1024 : c;
    for (int i = tid; i < n; i += kUpdThreads) dold[i] = __ldcg(D + int64_t(j) * n + i);

    // ---- phase A: partial Gram of this CTA's residual columns -------------
    float acc[TN][TN];
#pragma unroll
    for (int r = 0; r < TN; ++r)
#pragma unroll
      for (int s = 0; s < TN; ++s) acc[r][s] = 0.0f;
    const int sb = int(int64_t(c_eff) * b / G), se = int(int64_t(c_eff) * (b + 1) / G);
    for (int t0 = sb; t0 < se; t0 += kEChunk) {
      const int m = min(kEChunk, se - t0);
      for (int q = warp; q < kEChunk; q += kUpdThreads / 32) {
        float* er = E + q * n;
        if (q < m) {
          const int es = __ldg(entries + beg + t0 + q);
          const int64_t p = es / L;
          const int slot = es - int(p) * L;
          for (int i = lane; i < n; i += 32) er[i] = residual_elem(Y, D, idx, coef, p, slot, L, n, K, i);
        } else {
          for (int i = lane; i < n; i += 32) er[i] = 0.0f;
        }
      }
      __syncthreads();
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
          for (int s = 0; s < TN; ++s) acc[r][s] = fmaf(ra[r], rb[s], acc[r][s]);
      }
      __syncthreads();
    }
    float* gp = gpart + size_t(b) * nn;
#pragma unroll
    for (int r = 0; r < TN; ++r)
#pragma unroll
      for (int s = 0; s < TN; ++s) {
        const int i = ti + 16 * r, k = tj + 16 * s;
        if (i < n && k < n) gp[i * n + k] = acc[r][s];
      }
    if (!grid_sync(bar, G)) return;

    // ---- phase B: fixed-order sum of the partial Grams ---------------------
    {
      const int qb = int(int64_t(nn) * b / G), qe = int(int64_t(nn) * (b + 1) / G);
      for (int q = qb + tid; q < qe; q += kUpdThreads) {
        float s = 0.0f;
        for (unsigned bb = 0; bb < G; ++bb) s += __ldcg(gpart + size_t(bb) * nn + q);
        gsum[q] = s;
      }
    }
    if (!grid_sync(bar, G)) return;

    // ---- phase C: top eigenvector by power iteration (same in every CTA) ---
    for (int q = tid; q < nn; q += kUpdThreads) {
      const int i = q / n, k = q - i * n;
      Gs[i * (n + 1) + k] = __ldcg(gsum + q);
    }
    for (int i = tid; i < n; i += kUpdThreads) u[i] = dold[i];
    __syncthreads();
    int iters = 0;
    for (int it = 0; it < kMaxPowerIters; ++it) {
      float vi = 0.0f;
      if (tid < n) {
        const float* row = Gs + tid * (n + 1);
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
        int k = 0;
        for (; k + 3 < n; k += 4) {
          s0 = fmaf(row[k], u[k], s0);
          s1 = fmaf(row[k + 1], u[k + 1], s1);
          s2 = fmaf(row[k + 2], u[k + 2], s2);
          s3 = fmaf(row[k + 3], u[k + 3], s3);
        }
        for (; k < n; ++k) s0 = fmaf(row[k], u[k], s0);
        vi = (s0 + s1) + (s2 + s3);
      }
      const float nrm2 = block_sum(vi * vi, red);
      iters = it + 1;
      if (!(nrm2 > 0.0f)) break;  // E == 0: keep the old atom direction
      const float vn = vi / sqrtf(nrm2);
      const float diff = (tid < n) ? fabsf(vn - u[tid]) : 0.0f;
      const float dmax = block_max(diff, red);
      if (tid < n) u[tid] = vn;
      __syncthreads();
      if (dmax < kPowerTol) break;
    }
    const float sd = block_sum((tid < n) ? u[tid] * dold[tid] : 0.0f, red);
    const float sgn = (sd < 0.0f) ? -1.0f : 1.0f;
    if (tid < n) u[tid] *= sgn;
    __syncthreads();
    if (b == 0) {
      for (int i = tid; i < n; i += kUpdThreads) D[int64_t(j) * n + i] = u[i];
      if (tid == 0) {
        atomicAdd(&stats->power_iters, (unsigned long long)iters);
        atomicAdd(&stats->atoms_updated, 1ull);
      }
    }
    // coefficients of this CTA's slice of all c entries
    {
      const int cb = int(int64_t(c) * b / G), ce = int(int64_t(c) * (b + 1) / G);
      for (int t = cb + warp; t < ce; t += kUpdThreads / 32) {
        const int es = __ldg(entries + beg + t);
        if (t >= c_eff) {
          if (lane == 0) coef[es] = 0.0f;
          continue;
        }
        const int64_t p = es / L;
        const int slot = es - int(p) * L;
        float dp = 0.0f;
        for (int i = lane; i < n; i += 32) dp = fmaf(u[i], residual_elem(Y, D, idx, coef, p, slot, L, n, K, i), dp);
        dp = warp_sum(dp);
        if (lane == 0) coef[es] = dp;
      }
    }
    if (!grid_sync(bar, G)) return;
  }
}

bool update_supported(int n) { return n >= 1 && n <= 160; }

size_t update_smem_bytes(int n) { return update_floats(n) * sizeof(float); }

template <int TN>
static void* update_fn() {
  return reinterpret_cast<void*>(update_kernel<TN>);
}

static void* pick_update(int n) {
  switch ((n + 15) / 16) {
    case 1: return update_fn<1>();
    case 2: return update_fn<2>();
    case 3: return update_fn<3>();
    case 4: return update_fn<4>();
    case 5: return update_fn<5>();
    case 6: return update_fn<6>();
    case 7: return update_fn<7>();
    case 8: return update_fn<8>();
    case 9: return update_fn<9>();
    case 10: return update_fn<10>();
    default: return nullptr;
  }
}

int update_grid_size(int n, int num_sms) {
  void* fn = pick_update(n);
  if (!fn) return 0;
  size_t smem = update_smem_bytes(n);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kUpdThreads, smem) != cudaSuccess) return 0;
  if (per_sm < 1) return 0;
  return num_sms;  // one CTA per SM: co-resident by construction
}

cudaError_t launch_update(const float* patches, int64_t N, int n, float* dict, int K, int L, const int32_t* idx,
                          float* coef, CsrWork w, int q1_cap, float* gpart, float* gsum, GridBarrier* bar,
                          DevStats* stats, int grid, cudaStream_t s) {
  void* fn = pick_update(n);
  if (!fn || grid < 1) return cudaErrorInvalidValue;
  size_t smem = update_smem_bytes(n);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(bar, 0, sizeof(GridBarrier), s);
  if (e != cudaSuccess) return e;
  const int* atom_ptr = w.atom_ptr;
  const int* entries = w.entries;
  void* args[] = {(void*)&patches, (void*)&N,       (void*)&n,       (void*)&dict,  (void*)&K,
                  (void*)&L,       (void*)&idx,     (void*)&coef,    (void*)&atom_ptr, (void*)&entries,
                  (void*)&q1_cap,  (void*)&gpart,   (void*)&gsum,    (void*)&bar,   (void*)&stats};
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kUpdThreads), args, smem, s);
}

}  // namespace ksvd
