// Learned support proposal: a BF16 MLP n -> 512 -> 512 -> K (GELU, sigmoid
// scores) whose forward and backward passes run on the 5th-generation tensor
// cores, plus the small kernels of its training step (input scaling, loss
// gradient, bias gradients, Adam).
//
// One GEMM kernel serves every layer: C[M x N] = A[M x K] . B[N x K]^T with
// BF16 operands and FP32 accumulation in tensor memory.  A CTA owns a tile of
// 128 rows (UMMA M, one TMEM lane per row) by up to 256 columns (UMMA N); the
// K dimension streams through shared memory in chunks of 64 with two stages:
// while the tensor cores work on one chunk, the CTA's threads fill the other.
// Operands are written into the no-swizzle K-major canonical layout (core
// matrices of 8 rows x 16 bytes): with cp.async 16-byte copies when the
// operand is contiguous along K in global memory (activations x weights), or
// with 8 strided 2-byte loads packed into one 16-byte store when it is
// contiguous along M/N (the transposed operands of the backward pass).  One
// thread issues the MMAs and commits them to a per-stage mbarrier; the
// epilogue reads the accumulator with tcgen05.ld and fuses bias, GELU, the
// GELU derivative or the top-k candidate selection.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>

#include "device_util.cuh"
#include "ksvd_internal.cuh"
#include "tcgen05_util.cuh"

namespace ksvd {

constexpr int kGM = 128;      // rows per tile
constexpr int kGKC = 64;      // K per stage
constexpr int kGStages = 2;
constexpr int kGThreads = 256;
constexpr unsigned long long kGemmWaitNs = 2000000000ull;

__host__ __device__ inline int g_ntile(int N) { return N < 256 ? N : 256; }

__host__ __device__ inline size_t gemm_smem_bytes(int nt) {
  // stages x (A 128 x 64 + B nt x 64) BF16, then 2 mbarriers and the TMEM slot
  return size_t(kGStages) * (size_t(kGM) + size_t(nt)) * kGKC * 2 + 64;
}
// Dynamic shared memory requested per CTA: at least 80 KB, so that at most two
// CTAs share an SM and their TMEM allocations (up to 256 columns each) fit
// in its 512 columns without waiting.
__host__ __device__ inline size_t gemm_smem_request(int nt) {
  const size_t b = gemm_smem_bytes(nt);
  return b > 81920 ? b : 81920;
}

KSVD_DEV void cp_async16(unsigned dst, const void* src, unsigned src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
KSVD_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
KSVD_DEV void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
KSVD_DEV void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

KSVD_DEV float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
KSVD_DEV float gelu_grad_f(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// One operand tile (R rows x 64 K) of chunk k0 into the canonical layout at
// smem byte address `base`.  KC: the operand is contiguous along K (element
// (r, k) at P[r * ld + k]); otherwise along the rows (P[k * ld + r]).  Rows
// >= rows and columns >= K are zero.
template <bool KC>
KSVD_DEV void load_tile(unsigned base, const __nv_bfloat16* P, long long ld, int r0, int rows, int R, int k0, int K,
                        int tid) {
  if (KC) {
    // 16-byte pieces: piece t -> row t / 8, k-group t % 8
    for (int t = tid; t < R * 8; t += kGThreads) {
      const int r = t >> 3, g = t & 7;
      const int k = k0 + g * 8;
      const bool in = (r0 + r < rows) && (k < K);
      const __nv_bfloat16* src = in ? P + (long long)(r0 + r) * ld + k : P;
      cp_async16(base + canon_off(r, g * 8, R), src, in ? 16u : 0u);
    }
  } else {
    // consecutive threads take consecutive rows (coalesced 2-byte loads)
    for (int t = tid; t < R * 8; t += kGThreads) {
      const int r = t % R, g = t / R;
      const int k = k0 + g * 8;
      unsigned short h[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const bool in = (r0 + r < rows) && (k + e < K);
        h[e] = in ? __bfloat16_as_ushort(P[(long long)(k + e) * ld + (r0 + r)]) : (unsigned short)0;
      }
      uint4 v;
      v.x = unsigned(h[0]) | (unsigned(h[1]) << 16);
      v.y = unsigned(h[2]) | (unsigned(h[3]) << 16);
      v.z = unsigned(h[4]) | (unsigned(h[5]) << 16);
      v.w = unsigned(h[6]) | (unsigned(h[7]) << 16);
      asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(base + canon_off(r, g * 8, R)), "r"(v.x),
                   "r"(v.y), "r"(v.z), "r"(v.w)
                   : "memory");
    }
  }
}

template <bool AK, bool BK, int EPI>
__global__ void __launch_bounds__(kGThreads) gemm_bf16_kernel(GemmArgs g) {
  extern __shared__ __align__(128) unsigned char gsm[];
  const int nt = g_ntile(g.N);
  const size_t a_bytes = size_t(kGM) * kGKC * 2, b_bytes = size_t(nt) * kGKC * 2;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(gsm + kGStages * (a_bytes + b_bytes));
  unsigned* tslot = reinterpret_cast<unsigned*>(bars + kGStages);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kGM, n0 = blockIdx.y * nt;
  unsigned tcols = 32;
  while (tcols < unsigned(nt)) tcols <<= 1;

  if (warp == 0) tc_alloc(tslot, tcols);
  if (tid == 0) {
    for (int s = 0; s < kGStages; ++s) mbar_init(bars + s, 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tslot;
  const unsigned idesc = umma_idesc_16(kGM, nt, 1u);  // BF16 x BF16 -> FP32
  const unsigned sbase = smem_u32(gsm);
  auto a_addr = [&](int s) { return sbase + unsigned(s * (a_bytes + b_bytes)); };
  auto b_addr = [&](int s) { return sbase + unsigned(s * (a_bytes + b_bytes) + a_bytes); };
  const int nk = (g.K + kGKC - 1) / kGKC;
  unsigned phase_bits = 0;  // parity of the next completion of each stage's barrier
  unsigned pending = 0;     // stages with a commit not yet waited for (thread 0)
  bool failed = false;

  auto load_chunk = [&](int c) {
    const int s = c % kGStages;
    load_tile<AK>(a_addr(s), g.A, g.lda, m0, g.M, kGM, c * kGKC, g.K, tid);
    load_tile<BK>(b_addr(s), g.B, g.ldb, n0, g.N, nt, c * kGKC, g.K, tid);
  };
  load_chunk(0);
  cp_async_commit();
  for (int c = 0; c < nk; ++c) {
    const int s = c % kGStages;
    // the other stage is free once the MMAs of chunk c - 1 are complete
    if (c >= 1) {
      const int sp = (c - 1) % kGStages;
      bool ok = true;
      if (tid == 0) ok = mbar_wait(bars + sp, (phase_bits >> sp) & 1u, kGemmWaitNs);
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      phase_bits ^= 1u << sp;
      pending &= ~(1u << sp);
    }
    if (c + 1 < nk) load_chunk(c + 1);
    cp_async_commit();
    cp_async_wait1();  // chunk c has landed
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kk = 0; kk < kGKC / 16; ++kk) {
        const unsigned long long ad = umma_desc(a_addr(s) + kk * 2 * kGM * 16, kGM * 16, 128);
        const unsigned long long bd = umma_desc(b_addr(s) + kk * 2 * nt * 16, nt * 16, 128);
        tc_mma(tmem, ad, bd, idesc, (c > 0 || kk > 0) ? 1u : 0u);
      }
      tc_commit(bars + s);
      pending |= 1u << s;
    }
  }
  cp_async_wait0();
  // the last chunk's MMAs (and so every MMA) complete
  if (!failed) {
    const int sl = (nk - 1) % kGStages;
    bool ok = true;
    if (tid == 0) ok = mbar_wait(bars + sl, (phase_bits >> sl) & 1u, kGemmWaitNs);
    if (__syncthreads_or(!ok)) {
      failed = true;
    } else {
      phase_bits ^= 1u << sl;
      pending &= ~(1u << sl);
    }
  }
  if (failed) {
    if (tid == 0 && g.flags) atomicCAS(&g.flags->err, DEVERR_NONE, DEVERR_TIMEOUT);
  } else {
    tc_fence_after();
    // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 ------------------
    const int lg = warp & 3;
    const int m = m0 + lg * 32 + lane;
    const unsigned lane_addr = tmem + (unsigned(lg * 32) << 16);
    if (EPI == kEpiTopK) {
      // the row's top-k columns (descending score, lower column first on
      // ties) among the first g.n_valid columns.  The two warps of a TMEM
      // lane quadrant take one half of the columns each and keep a sorted
      // list of the 16 best: a new score's place is the number of kept
      // scores >= it (the columns come in ascending order, so a kept tie is
      // always the lower column), and the list shifts by predicated moves
      // without a serial chain.  The halves' lists then meet in shared memory
      // (the operand stages, free once every MMA has completed) and the
      // first warp group merges them.
      const int half = warp >> 2;
      const int cw = nt / 2;  // a multiple of 8
      const int ml = lg * 32 + lane;  // row within the tile
      float bv[kMaxTopK];
      int bi[kMaxTopK];
#pragma unroll
      for (int i = 0; i < kMaxTopK; ++i) {
        bv[i] = -INFINITY;
        bi[i] = 0x7fffffff;
      }
      for (int c0 = half * cw; c0 < (half + 1) * cw; c0 += 8) {
        float v[8];
        tc_ld8(lane_addr + unsigned(c0), v);
        tc_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int col = n0 + c0 + i;
          if (col >= g.n_valid) continue;
          const float z = v[i] + g.bias[col];
          if (z > bv[kMaxTopK - 1] || (z == bv[kMaxTopK - 1] && col < bi[kMaxTopK - 1])) {
            int pos = 0;
#pragma unroll
            for (int j = 0; j < kMaxTopK; ++j) pos += (bv[j] >= z) ? 1 : 0;
#pragma unroll
            for (int j = kMaxTopK - 1; j >= 0; --j) {
              if (j > pos) {
                bv[j] = bv[j - 1 >= 0 ? j - 1 : 0];
                bi[j] = bi[j - 1 >= 0 ? j - 1 : 0];
              } else if (j == pos) {
                bv[j] = z;
                bi[j] = col;
              }
            }
          }
        }
      }
      float* zs = reinterpret_cast<float*>(gsm);                 // [2 x 128][16]
      int* cs = reinterpret_cast<int*>(zs + 2 * kGM * kMaxTopK);  // [2 x 128][16]
      const int slot = (half * kGM + ml) * kMaxTopK;
#pragma unroll
      for (int j = 0; j < kMaxTopK; ++j) {
        zs[slot + j] = bv[j];
        cs[slot + j] = bi[j];
      }
      __syncthreads();
      if (half == 0 && m < g.M) {
        // merge: the first half's columns are the lower ones, so it wins ties
        const float* za = zs + ml * kMaxTopK;
        const int* ca = cs + ml * kMaxTopK;
        const float* zb = zs + (kGM + ml) * kMaxTopK;
        const int* cb = cs + (kGM + ml) * kMaxTopK;
        int ia = 0, ib = 0;
        const int kt = g.ktop;
        for (int j = 0; j < kt; ++j) {
          const bool take_a = ib >= kMaxTopK || (ia < kMaxTopK && za[ia] >= zb[ib]);
          g.topk[(long long)m * kt + j] = take_a ? ca[ia] : cb[ib];
          if (take_a)
            ++ia;
          else
            ++ib;
        }
      }
    } else {
      const int half = warp >> 2;  // column half of this warp
      const int cw = nt / 2;       // a multiple of 8
      for (int c0 = half * cw; c0 < (half + 1) * cw; c0 += 8) {
        float v[8];
        tc_ld8(lane_addr + unsigned(c0), v);
        tc_wait_ld();
        if (m >= g.M) continue;
        const int col = n0 + c0;
        if (EPI == kEpiF32) {
          float* dst = g.c_f32 + (long long)m * g.ldc_f32 + col;
#pragma unroll
          for (int i = 0; i < 8; ++i) dst[i] = v[i];
        } else if (EPI == kEpiBiasF32) {
          float* dst = g.c_f32 + (long long)m * g.ldc_f32 + col;
#pragma unroll
          for (int i = 0; i < 8; ++i) dst[i] = v[i] + g.bias[col + i];
        } else if (EPI == kEpiBiasGelu) {
          unsigned short h[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const float z = v[i] + g.bias[col + i];
            v[i] = z;
            h[i] = __bfloat16_as_ushort(__float2bfloat16_rn(gelu_f(z)));
          }
          if (g.c_f32) {
            float* dst = g.c_f32 + (long long)m * g.ldc_f32 + col;
#pragma unroll
            for (int i = 0; i < 8; ++i) dst[i] = v[i];
          }
          uint4 pk;
          pk.x = unsigned(h[0]) | (unsigned(h[1]) << 16);
          pk.y = unsigned(h[2]) | (unsigned(h[3]) << 16);
          pk.z = unsigned(h[4]) | (unsigned(h[5]) << 16);
          pk.w = unsigned(h[6]) | (unsigned(h[7]) << 16);
          *reinterpret_cast<uint4*>(g.c_bf16 + (long long)m * g.ldc_bf16 + col) = pk;
        } else {  // kEpiGeluBack: dZ = acc * GELU'(z) with z the saved pre-activation
          unsigned short h[8];
          const float* zr = g.aux + (long long)m * g.ld_aux + col;
#pragma unroll
          for (int i = 0; i < 8; ++i) h[i] = __bfloat16_as_ushort(__float2bfloat16_rn(v[i] * gelu_grad_f(zr[i])));
          uint4 pk;
          pk.x = unsigned(h[0]) | (unsigned(h[1]) << 16);
          pk.y = unsigned(h[2]) | (unsigned(h[3]) << 16);
          pk.z = unsigned(h[4]) | (unsigned(h[5]) << 16);
          pk.w = unsigned(h[6]) | (unsigned(h[7]) << 16);
          *reinterpret_cast<uint4*>(g.c_bf16 + (long long)m * g.ldc_bf16 + col) = pk;
        }
      }
    }
  }
  // ---- teardown -------------------------------------------------------------
  if (failed && tid == 0) {
    // bounded drain of the MMAs still in flight before the TMEM is released
    for (int s = 0; s < kGStages; ++s)
      if (pending & (1u << s)) mbar_wait(bars + s, (phase_bits >> s) & 1u, kGemmWaitNs);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tc_dealloc(tmem, tcols);
  }
}

template <bool AK, bool BK, int EPI>
static cudaError_t launch_gemm_t(const GemmArgs& g, cudaStream_t s) {
  const int nt = g_ntile(g.N);
  const size_t smem = gemm_smem_request(nt);
  auto kern = gemm_bf16_kernel<AK, BK, EPI>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  dim3 grid((g.M + kGM - 1) / kGM, (g.N + nt - 1) / nt);
  kern<<<grid, kGThreads, smem, s>>>(g);
  return cudaGetLastError();
}

bool gemm_shape_ok(const GemmArgs& g, bool a_kcontig, bool b_kcontig) {
  if (g.M < 1 || g.N < 16 || g.K < 16 || (g.N % 16) != 0 || (g.K % 16) != 0) return false;
  if (g.N > 256 && (g.N % 256) != 0) return false;
  auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  if (a_kcontig && (!al16(g.A) || (g.lda % 8) != 0)) return false;
  if (b_kcontig && (!al16(g.B) || (g.ldb % 8) != 0)) return false;
  return true;
}

cudaError_t launch_gemm(const GemmArgs& g, bool a_kcontig, bool b_kcontig, int epi, cudaStream_t s) {
  if (!gemm_shape_ok(g, a_kcontig, b_kcontig)) return cudaErrorInvalidValue;
  if (epi == kEpiTopK && (g.ktop < 1 || g.ktop > kMaxTopK || g.N > 256)) return cudaErrorInvalidValue;
  // the combinations the MLP uses
  if (a_kcontig && b_kcontig) {
    switch (epi) {
      case kEpiBiasGelu: return launch_gemm_t<true, true, kEpiBiasGelu>(g, s);
      case kEpiBiasF32: return launch_gemm_t<true, true, kEpiBiasF32>(g, s);
      case kEpiTopK: return launch_gemm_t<true, true, kEpiTopK>(g, s);
      case kEpiF32: return launch_gemm_t<true, true, kEpiF32>(g, s);
      default: return cudaErrorInvalidValue;
    }
  }
  if (a_kcontig && !b_kcontig) {
    switch (epi) {
      case kEpiGeluBack: return launch_gemm_t<true, false, kEpiGeluBack>(g, s);
      case kEpiF32: return launch_gemm_t<true, false, kEpiF32>(g, s);
      default: return cudaErrorInvalidValue;
    }
  }
  if (!a_kcontig && !b_kcontig && epi == kEpiF32) return launch_gemm_t<false, false, kEpiF32>(g, s);
  return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// Elementwise kernels of the proposal
// ---------------------------------------------------------------------------

// Network input: the patch with its mean removed, scaled to norm sqrt(n),
// x = (y - mean) sqrt(n) / |y - mean| (0 for a flat patch), as BF16, padded
// with zeros to np16 columns.  rows (optional) selects the patches: patch
// rows[b] mod `mod` (mod 0: rows[b]).
__global__ void mlp_input_kernel(const float* __restrict__ Y, int64_t B, int n, int np16,
                                 const int64_t* __restrict__ rows, int64_t mod, __nv_bfloat16* __restrict__ X) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t b = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); b < B; b += warps) {
    const int64_t p = rows ? (mod > 0 ? rows[b] % mod : rows[b]) : b;
    const float* y = Y + p * n;
    float sm = 0.0f;
    for (int k = lane; k < n; k += 32) sm += y[k];
    const float mean = warp_sum(sm) / float(n);
    float ss = 0.0f;
    for (int k = lane; k < n; k += 32) ss = fmaf(y[k] - mean, y[k] - mean, ss);
    ss = warp_sum(ss);
    const float sc = ss > 0.0f ? sqrtf(float(n) / ss) : 0.0f;
    for (int k = lane; k < np16; k += 32)
      X[b * np16 + k] = __float2bfloat16_rn(k < n ? (y[k] - mean) * sc : 0.0f);
  }
}

// Loss of the sigmoid scores against the support mask (binary cross-entropy
// with logits, mean over the B x K entries) and its gradient dZ (BF16, rows
// of K16 columns, zero beyond K).  The targets of row b are the atoms
// sup[r * L .. r * L + L - 1] (-1 for an unused slot) with r = rows[b] (or b).
__global__ void mlp_bce_kernel(const float* __restrict__ Z, int64_t B, int K, int K16, const int32_t* __restrict__ sup,
                               int L, const int64_t* __restrict__ rows, __nv_bfloat16* __restrict__ dZ,
                               double* __restrict__ loss_sum) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  const float inv = 1.0f / (float(B) * float(K));
  double acc = 0.0;
  for (int64_t b = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); b < B; b += warps) {
    const int64_t r = rows ? rows[b] : b;
    const int t = (lane < L) ? sup[r * L + lane] : -1;
    for (int j0 = 0; j0 < K16; j0 += 32) {  // warp-uniform trip count
      const int j = j0 + lane;
      bool pos = false;
      for (int s2 = 0; s2 < L; ++s2) pos |= (__shfl_sync(0xffffffffu, t, s2) == j);
      if (j >= K16) continue;
      float g = 0.0f;
      if (j < K) {
        const float z = Z[b * K16 + j];
        const float sg = 1.0f / (1.0f + expf(-z));
        g = (sg - (pos ? 1.0f : 0.0f)) * inv;
        // log(1 + e^z) - t z, computed stably
        const float sp = fmaxf(z, 0.0f) + log1pf(expf(-fabsf(z)));
        acc += double(sp - (pos ? z : 0.0f));
      }
      dZ[b * K16 + j] = __float2bfloat16_rn(g);
    }
  }
  acc = warp_sum(acc);
  if (lane == 0 && acc != 0.0) atomicAdd(loss_sum, acc / (double(B) * double(K)));
}

// Column sums of the first C columns of a B-row BF16 matrix with row stride
// ld (the bias gradients): FP32 per column.
__global__ void mlp_colsum_kernel(const __nv_bfloat16* __restrict__ G, int64_t B, int C, int ld,
                                  float* __restrict__ out) {
  __shared__ float part[8][33];
  const int c = blockIdx.x * 32 + (threadIdx.x & 31);
  const int ry = threadIdx.x >> 5;  // 8 row groups
  float s = 0.0f;
  if (c < C)
    for (int64_t b = ry; b < B; b += 8) s += __bfloat162float(G[b * ld + c]);
  part[ry][threadIdx.x & 31] = s;
  __syncthreads();
  if (ry == 0 && c < C) {
    float t = 0.0f;
    for (int i = 0; i < 8; ++i) t += part[i][threadIdx.x & 31];
    out[c] = t;
  }
}

// Adam (bias-corrected) on the FP32 master parameters.
__global__ void mlp_adam_kernel(float* __restrict__ w, const float* __restrict__ grad, float* __restrict__ m1,
                                float* __restrict__ m2, int64_t count, float lr, float b1, float b2, float eps,
                                float c1, float c2) {
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += int64_t(gridDim.x) * blockDim.x) {
    const float gi = grad[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    w[i] -= lr * (a * c1) / (sqrtf(v * c2) + eps);
  }
}

// BF16 copy of a rows x cols FP32 block into a rows x ld BF16 matrix (columns
// cols..ld-1 are zero), rows_pad - rows zero rows after it.
__global__ void mlp_to_bf16_kernel(const float* __restrict__ w, int rows, int cols, int rows_pad, int ld,
                                   __nv_bfloat16* __restrict__ out) {
  const int64_t total = int64_t(rows_pad) * ld;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int r = int(i / ld), c = int(i - int64_t(r) * ld);
    out[i] = __float2bfloat16_rn((r < rows && c < cols) ? w[int64_t(r) * cols + c] : 0.0f);
  }
}

// FP32 rows x cols block from a rows x ld FP32 matrix (drops the padding).
__global__ void mlp_unpad_kernel(const float* __restrict__ src, int rows, int cols, int ld, float* __restrict__ dst) {
  const int64_t total = int64_t(rows) * cols;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += int64_t(gridDim.x) * blockDim.x) {
    const int r = int(i / cols), c = int(i - int64_t(r) * cols);
    dst[i] = src[int64_t(r) * ld + c];
  }
}

static int ew_blocks(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return int(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

cudaError_t launch_mlp_input(const float* Y, int64_t B, int n, int np16, const int64_t* rows, int64_t mod,
                             __nv_bfloat16* X, cudaStream_t s) {
  mlp_input_kernel<<<ew_blocks(B * 32), 256, 0, s>>>(Y, B, n, np16, rows, mod, X);
  return cudaGetLastError();
}

cudaError_t launch_mlp_bce(const float* Z, int64_t B, int K, int K16, const int32_t* sup, int L, const int64_t* rows,
                           __nv_bfloat16* dZ, double* loss_sum, cudaStream_t s) {
  if (L > 32) return cudaErrorInvalidValue;
  mlp_bce_kernel<<<ew_blocks(B * 32), 256, 0, s>>>(Z, B, K, K16, sup, L, rows, dZ, loss_sum);
  return cudaGetLastError();
}

cudaError_t launch_mlp_colsum(const __nv_bfloat16* G, int64_t B, int C, int ld, float* out, cudaStream_t s) {
  mlp_colsum_kernel<<<(C + 31) / 32, 256, 0, s>>>(G, B, C, ld, out);
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float* w, const float* grad, float* m1, float* m2, int64_t count, float lr, int step,
                            cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = float(1.0 / (1.0 - std::pow(double(b1), double(step))));
  const float c2 = float(1.0 / (1.0 - std::pow(double(b2), double(step))));
  mlp_adam_kernel<<<ew_blocks(count), 256, 0, s>>>(w, grad, m1, m2, count, lr, b1, b2, 1e-8f, c1, c2);
  return cudaGetLastError();
}

cudaError_t launch_mlp_to_bf16(const float* w, int rows, int cols, int rows_pad, int ld, __nv_bfloat16* out,
                               cudaStream_t s) {
  mlp_to_bf16_kernel<<<ew_blocks(int64_t(rows_pad) * ld), 256, 0, s>>>(w, rows, cols, rows_pad, ld, out);
  return cudaGetLastError();
}

cudaError_t launch_mlp_unpad(const float* src, int rows, int cols, int ld, float* dst, cudaStream_t s) {
  mlp_unpad_kernel<<<ew_blocks(int64_t(rows) * cols), 256, 0, s>>>(src, rows, cols, ld, dst);
  return cudaGetLastError();
}

}  // namespace ksvd
