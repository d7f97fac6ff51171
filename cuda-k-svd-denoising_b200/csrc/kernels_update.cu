// Support lists of the dictionary update (updateDictionary,
// cuda_svd_denoiser.cu:285-362): the CSR of atom -> (patch, slot) entries,
// patches ascending, built from the compact codes, nonzero coefficients only.
// Replaces findRelevantIndicesKernel (:36-50), which scans the dense K x N
// code matrix with one thread per atom.  The sweep itself is in
// kernels_update_res.cu.
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
                                                             int* __restrict__ entries, int* __restrict__ records) {
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
    const int pos = wcnt[warp * K + a] + rank;
    entries[pos] = int(p * L + s);
    if (!records) continue;
    const int R = (L + 2 + 3) / 4 * 4;
    int* rec = records + int64_t(pos) * R;
    rec[0] = int(p);
    rec[1] = s;
    for (int s2 = 0; s2 < L; ++s2) rec[2 + s2] = mine[s2];
    for (int r2 = L + 2; r2 < R; ++r2) rec[r2] = -1;
  }
}

cudaError_t launch_csr_build(const int32_t* idx, const float* coef, int64_t N, int L, int K, CsrWork w,
                             cudaStream_t s) {
  const int64_t nch = w.nchunks;
  csr_count_kernel<<<unsigned(nch), kCsrChunk, K * sizeof(int), s>>>(idx, coef, N, L, K, nch, w.chunk_counts);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // atom totals sit after atom_ptr[0..K]
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
                                                         w.entries, w.records);
  return cudaGetLastError();
}

__global__ void accumulate_phases_kernel(const DevStats* __restrict__ src, DevStats* __restrict__ dst) {
  const int t = threadIdx.x;
  if (t < 16) dst->phase_ns[t] += src->phase_ns[t];
  if (t == 16) dst->power_iters += src->power_iters;
  if (t == 17) dst->atoms_updated += src->atoms_updated;
}

cudaError_t launch_accumulate_phases(const DevStats* src, DevStats* dst, cudaStream_t s) {
  accumulate_phases_kernel<<<1, 32, 0, s>>>(src, dst);
  return cudaGetLastError();
}

}  // namespace ksvd
