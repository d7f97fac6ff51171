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
                                                         w.entries, w.records);
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
constexpr int kEChunk = 32;              // residual columns per pipeline stage
constexpr int kMinEntriesPerCta = 16;    // phase A uses ceil(c / 16) CTAs at most
constexpr int kMaxPowerIters = 1000;
constexpr float kPowerTol = 2.0e-7f;     // max |u_new - u_old| to stop
constexpr unsigned long long kCopyWaitNs = 2000000000ull;  // bound of one bulk-copy wait

struct UpdLayout {
  size_t off_ds, off_e, off_rec, off_cf, off_u, off_dold, off_red, off_bar, total;
};

__host__ __device__ inline size_t upd_al16(size_t x) { return (x + 15) & ~size_t(15); }

// Three residual-column buffers (the third lets the next atom's first chunk
// be fetched while the current atom still uses its buffers), three record
// buffers, one gathered-coefficient buffer per column buffer, the mbarriers
// (3 for records, 3 for columns).
__host__ __device__ inline UpdLayout upd_layout(int n, int K, int L, bool dsmem) {
  const int npad = (n + 15) / 16 * 16;
  const int R = (L + 2 + 3) / 4 * 4;
  UpdLayout o;
  size_t off = 0;
  o.off_ds = off;
  off = upd_al16(off + (dsmem ? size_t(K) * n * 4 : 0));
  o.off_e = off;
  off = upd_al16(off + size_t(3) * kEChunk * n * 4);
  o.off_rec = off;
  off = upd_al16(off + size_t(3) * kEChunk * R * 4);
  o.off_cf = off;
  off = upd_al16(off + size_t(3) * kEChunk * L * 4);
  o.off_u = off;
  off = upd_al16(off + size_t(npad) * 4);
  o.off_dold = off;
  off = upd_al16(off + size_t(npad) * 4);
  o.off_red = off;
  off = upd_al16(off + 64 * 4);
  o.off_bar = off;
  off = upd_al16(off + 6 * 8);
  o.total = off;
  return o;
}

KSVD_DEV void bulk_s2g(void* gdst, const void* ssrc, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(ssrc)),
               "r"(bytes)
               : "memory");
}
KSVD_DEV void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
KSVD_DEV void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
KSVD_DEV void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

template <int TN, bool DSMEM>
__global__ void __launch_bounds__(kUpdThreads, 1)
    update_kernel(const float* __restrict__ Y, int64_t N, int n, float* D, int K, int L,
                  const int32_t* __restrict__ idx, float* coef, const int* __restrict__ atom_ptr,
                  const int* __restrict__ entries, const int* __restrict__ records, int q1_cap, int tma,
                  float* gpart, float* gsum, float* escr, int64_t escr_cap, GridBarrier* bar, DevStats* stats) {
  extern __shared__ __align__(16) unsigned char usm[];
  const UpdLayout lo = upd_layout(n, K, L, DSMEM);
  const int R = (L + 2 + 3) / 4 * 4;
  float* Ds = reinterpret_cast<float*>(usm + lo.off_ds);
  float* Ebase = reinterpret_cast<float*>(usm + lo.off_e);
  int* recb = reinterpret_cast<int*>(usm + lo.off_rec);
  float* cfb = reinterpret_cast<float*>(usm + lo.off_cf);
  float* u = reinterpret_cast<float*>(usm + lo.off_u);
  float* dold = reinterpret_cast<float*>(usm + lo.off_dold);
  float* red = reinterpret_cast<float*>(usm + lo.off_red);
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(usm + lo.off_bar);  // [0..2] rec, [3..5] col
  (void)N;

  const unsigned G = gridDim.x;
  const int b = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ti = tid >> 4, tj = tid & 15;
  const int nn = n * n;
  const int npad = 16 * TN;
  float* my_escr = escr + size_t(b) * size_t(escr_cap) * n;

  if (tid == 0) {
    for (int k = 0; k < 6; ++k) mbar_init(&bars[k], 1);
    fence_mbar_init();
  }
  if (DSMEM)
    for (int t = tid; t < K * n; t += kUpdThreads) Ds[t] = __ldcg(D + t);
  __syncthreads();
  // parity bit of the next phase of each mbarrier; only thread 0 waits on
  // record barriers, every thread waits on column barriers.
  unsigned parity = 0;
  bool failed = false;  // thread 0: a bulk-copy wait timed out

  auto datom = [&](int a, int i) -> float { return DSMEM ? Ds[a * n + i] : __ldcg(D + int64_t(a) * n + i); };
  auto wait_bar = [&](int k) -> bool {
    const bool ok = mbar_wait(&bars[k], (parity >> k) & 1u, kCopyWaitNs);
    parity ^= (1u << k);
    return ok;
  };

  // ---- pipeline stages (thread 0 issues every bulk copy) -------------------
  // records of chunk [t0, t0+m) of atom entries starting at beg -> ring slot r3
  auto issue_records = [&](int beg, int t0, int m, int r3) {
    if (tid == 0 && !failed) {
      mbar_arrive_expect_tx(&bars[r3], unsigned(m * R * 4));
      bulk_g2s(recb + r3 * kEChunk * R, records + int64_t(beg + t0) * R, unsigned(m * R * 4), &bars[r3]);
    }
  };
  // patches of the chunk whose records sit in ring slot r3 -> column buffer buf
  auto issue_patches = [&](int m, int r3, int buf, bool rec_waited) {
    if (tid == 0 && !failed) {
      if (!rec_waited && !wait_bar(r3)) {
        failed = true;
        return;
      }
      const int* rc = recb + r3 * kEChunk * R;
      float* Eb = Ebase + size_t(buf) * kEChunk * n;
      bulk_wait_read0();  // scratch stores out of this buffer have read it
      if (tma) {
        mbar_arrive_expect_tx(&bars[3 + buf], unsigned(m) * unsigned(n) * 4u);
        for (int q = 0; q < m; ++q) bulk_g2s(Eb + q * n, Y + int64_t(rc[q * R]) * n, unsigned(n) * 4u, &bars[3 + buf]);
      }
    }
  };
  // Other-slot coefficients of the chunk whose records sit in ring slot r3:
  // each thread loads up to kCfRegs of them into registers (prefetch) and
  // later stores them into cf buffer `buf`.
  constexpr int kCfRegs = 4;
  auto gather_load = [&](int m, int r3, float (&vals)[kCfRegs]) {
    const int* rc = recb + r3 * kEChunk * R;
#pragma unroll
    for (int g = 0; g < kCfRegs; ++g) {
      const int t = tid + g * kUpdThreads;
      float v = 0.0f;
      if (t < m * L) {
        const int q = t / L, s2 = t - q * L;
        const int a = rc[q * R + 2 + s2];
        if (s2 != rc[q * R + 1] && a >= 0) v = __ldcg(coef + int64_t(rc[q * R]) * L + s2);
      }
      vals[g] = v;
    }
  };
  auto gather_store = [&](int m, int buf, const float (&vals)[kCfRegs]) {
    float* cf = cfb + buf * kEChunk * L;
#pragma unroll
    for (int g = 0; g < kCfRegs; ++g) {
      const int t = tid + g * kUpdThreads;
      if (t < m * L) cf[t] = vals[g];
    }
  };
  // Waits for the columns of buffer buf (records in r3, coefficients already
  // in cf buffer buf), subtracts the other atoms in place and (store=true)
  // copies the finished columns to this CTA's scratch at column offset soff.
  auto finish = [&](int m, int r3, int buf, bool store, int soff) -> bool {
    const int* rc = recb + r3 * kEChunk * R;
    float* Eb = Ebase + size_t(buf) * kEChunk * n;
    const float* cf = cfb + buf * kEChunk * L;
    bool ok = true;
    if (tma) ok = wait_bar(3 + buf);
    if (__syncthreads_or(!ok || (tid == 0 && failed))) {
      if (tid == 0) atomicCAS(&bar->err, DEVERR_NONE, DEVERR_TIMEOUT);
      return false;
    }
    if (!tma) {  // generic loads when rows are not 16-byte aligned
      for (int q = warp; q < m; q += kUpdThreads / 32)
        for (int i = lane; i < n; i += 32) Eb[q * n + i] = __ldg(Y + int64_t(rc[q * R]) * n + i);
      __syncthreads();
    }
    for (int q = warp; q < m; q += kUpdThreads / 32) {
      const int* rq = rc + q * R;
      for (int i = lane; i < n; i += 32) {
        float e = Eb[q * n + i];
        for (int s2 = 0; s2 < L; ++s2) {
          const float cv = cf[q * L + s2];
          if (cv != 0.0f) e = fmaf(-cv, datom(rq[2 + s2], i), e);
        }
        Eb[q * n + i] = e;
      }
    }
    fence_proxy_async_smem();  // generic writes of Eb before later bulk accesses
    __syncthreads();
    if (store && tid == 0) {
      bulk_s2g(my_escr + size_t(soff) * n, Eb, unsigned(m) * unsigned(n) * 4u);
      bulk_commit();
    }
    return true;
  };
  // Waits (thread 0) for the records in ring slot r3 and makes them visible.
  auto records_ready = [&](int r3) -> bool {
    if (tid == 0 && !failed && !wait_bar(r3)) failed = true;
    if (__syncthreads_or(tid == 0 && failed)) {
      if (tid == 0) atomicCAS(&bar->err, DEVERR_NONE, DEVERR_TIMEOUT);
      return false;
    }
    return true;
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

  // Column buffers of the k-th processed atom: chunk 0 in buffer P = k & 1
  // (fetched ahead during the previous atom), later chunks alternate between
  // buffer 2 and buffer 1 - P; the coefficient pass streams through P and 2,
  // so buffer 1 - P is free for the next atom's first chunk.
  int kproc = 0;
  bool prefetched = false;  // records of chunks 0/1 and patches of chunk 0 in flight
  for (int j = 0; j < K; ++j) {
    const int beg = atom_ptr[j];
    const int c = atom_ptr[j + 1] - beg;
    if (c == 0) continue;
    const int P = kproc & 1;
    ++kproc;
    auto colbuf = [&](int ch) { return ch == 0 ? P : ((ch & 1) ? 2 : 1 - P); };
    const int c_eff = (q1_cap && c > 1024) ? 1024 : c;
    const int active = min(int(G), (c_eff + kMinEntriesPerCta - 1) / kMinEntriesPerCta);
    for (int i = tid; i < npad; i += kUpdThreads) dold[i] = (i < n) ? datom(j, i) : 0.0f;
    // the next atom with a non-empty support and this CTA's first chunk of it
    int jn = j + 1;
    while (jn < K && atom_ptr[jn + 1] == atom_ptr[jn]) ++jn;
    int nbeg = 0, nsb = 0, nse = 0;
    bool n_in = false;
    if (jn < K) {
      nbeg = atom_ptr[jn];
      const int cn = atom_ptr[jn + 1] - nbeg;
      const int cne = (q1_cap && cn > 1024) ? 1024 : cn;
      const int nact = min(int(G), (cne + kMinEntriesPerCta - 1) / kMinEntriesPerCta);
      nsb = int(int64_t(cne) * b / nact);
      nse = int(int64_t(cne) * (b + 1) / nact);
      n_in = b < nact;
    }

    // ---- phase A: partial Gram of this CTA's residual columns -------------
    const int sb = int(int64_t(c_eff) * b / active), se = int(int64_t(c_eff) * (b + 1) / active);
    const bool in_a = b < active;
    const int nch = in_a ? (se - sb + kEChunk - 1) / kEChunk : 0;
    const bool resident = nch == 1;
    if (in_a) {
#pragma unroll
      for (int r = 0; r < TN; ++r)
#pragma unroll
        for (int s2 = 0; s2 < TN; ++s2) blk[r][s2] = 0.0f;
      lap(0);
      float cfv[kCfRegs];
      if (!prefetched) {
        issue_records(beg, sb, min(kEChunk, se - sb), 0);
        if (nch > 1) issue_records(beg, sb + kEChunk, min(kEChunk, se - sb - kEChunk), 1);
        if (!records_ready(0)) return;
        issue_patches(min(kEChunk, se - sb), 0, colbuf(0), true);
      }
      // coefficients change with every atom: gathered only now
      gather_load(min(kEChunk, se - sb), 0, cfv);
      gather_store(min(kEChunk, se - sb), colbuf(0), cfv);
      lap(11);
      for (int ch = 0; ch < nch; ++ch) {
        const int buf = colbuf(ch), r3 = ch % 3;
        const int t0 = sb + ch * kEChunk;
        const int m = min(kEChunk, se - t0);
        const int m1 = min(kEChunk, se - t0 - kEChunk);  // next chunk (if any)
        if (ch + 1 < nch) issue_patches(m1, (ch + 1) % 3, colbuf(ch + 1), false);
        if (ch + 2 < nch) issue_records(beg, t0 + 2 * kEChunk, min(kEChunk, se - t0 - 2 * kEChunk), (ch + 2) % 3);
        lap(11);
        if (!finish(m, r3, buf, !resident && tma, t0 - sb)) return;
        lap(12);
        // the next chunk's records are visible now (waited above, synced in
        // finish): prefetch its coefficients while this chunk accumulates
        if (ch + 1 < nch) gather_load(m1, (ch + 1) % 3, cfv);
        const float* Eb = Ebase + size_t(buf) * kEChunk * n;
        for (int q = 0; q < m; ++q) {
          const float* er = Eb + q * n;
          float ra[TN], rb[TN];
#pragma unroll
          for (int r = 0; r < TN; ++r) {
            const int i = ti + 16 * r;
            ra[r] = (i < n) ? er[i] : 0.0f;
          }
#pragma unroll
          for (int s2 = 0; s2 < TN; ++s2) {
            const int k = tj + 16 * s2;
            rb[s2] = (k < n) ? er[k] : 0.0f;
          }
#pragma unroll
          for (int r = 0; r < TN; ++r)
#pragma unroll
            for (int s2 = 0; s2 < TN; ++s2) blk[r][s2] = fmaf(ra[r], rb[s2], blk[r][s2]);
        }
        if (ch + 1 < nch) gather_store(m1, colbuf(ch + 1), cfv);
        fence_proxy_async_smem();
        __syncthreads();
        lap(13);
      }
      float* gp = gpart + size_t(b) * nn;
#pragma unroll
      for (int r = 0; r < TN; ++r)
#pragma unroll
        for (int s2 = 0; s2 < TN; ++s2) {
          const int i = ti + 16 * r, k = tj + 16 * s2;
          if (i <= k && k < n) gp[i * n + k] = blk[r][s2];
        }
    }
    __syncthreads();
    // records of the next atom's first chunks (immutable during the sweep)
    prefetched = false;
    if (n_in && tma) {
      issue_records(nbeg, nsb, min(kEChunk, nse - nsb), 0);
      if (nse - nsb > kEChunk) issue_records(nbeg, nsb + kEChunk, min(kEChunk, nse - nsb - kEChunk), 1);
      prefetched = true;
    }
    lap(0);
    if (!grid_sync(bar, G)) return;
    lap(1);

    // ---- phase B: fixed-order sum of the active partial Grams --------------
    if (prefetched) issue_patches(min(kEChunk, nse - nsb), 0, 1 - P, false);
    {
      const int qb = int(int64_t(nn) * b / G), qe = int(int64_t(nn) * (b + 1) / G);
      for (int q = qb + tid; q < qe; q += kUpdThreads) {
        const int i = q / n, k = q - i * n;
        if (i > k) continue;
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
        int bb = 0;
        for (; bb + 3 < active; bb += 4) {
          s0 += __ldcg(gpart + size_t(bb) * nn + q);
          s1 += __ldcg(gpart + size_t(bb + 1) * nn + q);
          s2 += __ldcg(gpart + size_t(bb + 2) * nn + q);
          s3 += __ldcg(gpart + size_t(bb + 3) * nn + q);
        }
        for (; bb < active; ++bb) s0 += __ldcg(gpart + size_t(bb) * nn + q);
        const float v = (s0 + s1) + (s2 + s3);
        gsum[q] = v;
        gsum[k * n + i] = v;  // both triangles: phase C reads rows contiguously
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
      for (int s2 = 0; s2 < TN; ++s2) {
        const int i = ti + 16 * r, k = tj + 16 * s2;
        blk[r][s2] = (i < n && k < n) ? __ldcg(gsum + i * n + k) : 0.0f;
      }
    for (int i = tid; i < npad; i += kUpdThreads) u[i] = dold[i];
    __syncthreads();
    lap(14);
    int iters = 0;
    for (int it = 0; it < kMaxPowerIters; ++it) {
      float ub[TN], v[TN];
#pragma unroll
      for (int s2 = 0; s2 < TN; ++s2) ub[s2] = u[tj + 16 * s2];
#pragma unroll
      for (int r = 0; r < TN; ++r) {
        float acc = 0.0f;
#pragma unroll
        for (int s2 = 0; s2 < TN; ++s2) acc = fmaf(blk[r][s2], ub[s2], acc);
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
      auto dots = [&](int buf, int t0, int m) {
        const float* Eb = Ebase + size_t(buf) * kEChunk * n;
        for (int q = warp; q < m; q += kUpdThreads / 32) {
          const float* er = Eb + q * n;
          float dp = 0.0f;
          for (int i = lane; i < n; i += 32) dp = fmaf(u[i], er[i], dp);
          dp = warp_sum(dp);
          if (lane == 0) coef[__ldg(entries + beg + t0 + q)] = dp;
        }
      };
      if (resident) {
        dots(P, sb, se - sb);  // buffer P still holds this CTA's columns
        fence_proxy_async_smem();
      } else if (!tma) {
        // rows not 16-byte aligned: rebuild the columns (generic loads)
        issue_records(beg, sb, min(kEChunk, se - sb), 0);
        for (int ch = 0; ch < nch; ++ch) {
          const int buf = ch & 1, r3 = ch % 3;
          const int t0 = sb + ch * kEChunk;
          const int m = min(kEChunk, se - t0);
          if (ch + 1 < nch) issue_records(beg, t0 + kEChunk, min(kEChunk, se - t0 - kEChunk), (ch + 1) % 3);
          if (!records_ready(r3)) return;
          float cfv[kCfRegs];
          gather_load(m, r3, cfv);
          gather_store(m, buf, cfv);
          if (!finish(m, r3, buf, false, 0)) return;
          dots(buf, t0, m);
          __syncthreads();
        }
      } else {
        // stream the columns back from the scratch
        if (tid == 0) bulk_wait0();  // this CTA's scratch stores are complete
        auto sbuf = [&](int ch) { return (ch & 1) ? 2 : P; };
        auto issue_cols = [&](int ch) {
          if (tid == 0 && !failed) {
            const int t0 = sb + ch * kEChunk, m = min(kEChunk, se - t0), buf = sbuf(ch);
            mbar_arrive_expect_tx(&bars[3 + buf], unsigned(m) * unsigned(n) * 4u);
            bulk_g2s(Ebase + size_t(buf) * kEChunk * n, my_escr + size_t(t0 - sb) * n, unsigned(m) * unsigned(n) * 4u,
                     &bars[3 + buf]);
          }
        };
        __syncthreads();  // the scratch is complete before it is read back
        issue_cols(0);
        for (int ch = 0; ch < nch; ++ch) {
          const int buf = sbuf(ch);
          const int t0 = sb + ch * kEChunk;
          const int m = min(kEChunk, se - t0);
          if (ch + 1 < nch) issue_cols(ch + 1);
          const bool ok = wait_bar(3 + buf);
          if (__syncthreads_or(!ok || (tid == 0 && failed))) {
            if (tid == 0) atomicCAS(&bar->err, DEVERR_NONE, DEVERR_TIMEOUT);
            return;
          }
          dots(buf, t0, m);
          fence_proxy_async_smem();
          __syncthreads();
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
  if (tid == 0) bulk_wait0();
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

int64_t update_scratch_cap(int64_t N, int grid) {
  int64_t per = (N + grid - 1) / grid + 1;
  return per > kMinEntriesPerCta ? per : kMinEntriesPerCta;
}

cudaError_t launch_update(const float* patches, int64_t N, int n, float* dict, int K, int L, const int32_t* idx,
                          float* coef, CsrWork w, int q1_cap, float* gpart, float* gsum, float* escr,
                          int64_t escr_cap, GridBarrier* bar, DevStats* stats, int grid, cudaStream_t s) {
  // bulk copies need 16-byte aligned rows
  int tma = ((n * 4) % 16 == 0 && (reinterpret_cast<uintptr_t>(patches) & 15) == 0) ? 1 : 0;
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
  const int* records = w.records;
  void* args[] = {(void*)&patches, (void*)&N,     (void*)&n,       (void*)&dict,     (void*)&K,
                  (void*)&L,       (void*)&idx,   (void*)&coef,    (void*)&atom_ptr, (void*)&entries,
                  (void*)&records, (void*)&q1_cap, (void*)&tma,    (void*)&gpart,    (void*)&gsum,
                  (void*)&escr,    (void*)&escr_cap, (void*)&bar,  (void*)&stats};
  return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kUpdThreads), args, smem, s);
}

}  // namespace ksvd
