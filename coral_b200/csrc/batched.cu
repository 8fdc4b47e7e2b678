// Grouped (batched, uneven) SGEMM and batched STRSV.
//
// No reference counterpart: each instance has exactly the semantics of
// coral_sgemm (sgemm.rs:106-130, epilogue f32_edge.rs:37-58) or coral_strsv
// (strsv.rs:60-74); the batch is described by an array of descriptors in
// DEVICE memory, so a call enqueues a fixed number of kernels with no host
// work per instance and can be captured in a CUDA graph (size the handle's
// scratch with one uncaptured call first).
//
// Grouped GEMM on the tensor cores (bf16 inputs, or fp32 inputs in
// split-BF16x3 mode): grouped_tc.cu.  The FP32 FMA form below serves fp32
// inputs in the NATIVE and SPLIT_BF16X6 modes.
//
// Grouped GEMM (FMA form): k_tile_prefix (one CTA) turns the descriptors into an
// exclusive prefix sum of 64 x 64 output tiles; k_gemm_grouped (persistent,
// 4 CTAs per SM) walks the global tile index space with a grid stride, finds
// each tile's instance by binary search over the prefix array and computes
// the tile on the FP32 FMA pipes: 256 threads, 4 x 4 outputs per thread,
// 16-deep K slabs double-buffered through shared memory.  The bf16-input
// variant reads bf16 operands and accumulates in fp32.
//
// Batched TRSV: one CTA per instance, blocked right-looking substitution over
// 64-row diagonal blocks: one warp solves the block (substitution, the
// divide by the diagonal as strlsv.rs:66-140 does), then all warps subtract
// the block's panel times the new solution from the remaining right-hand side
// (coalesced column streaming).  Transposed operators are walked backwards.
#include "common.cuh"

#include <cuda_bf16.h>

namespace coral {
namespace {

struct GemmProblem {
  int32_t op_a, op_b, m, n, k;
  float alpha, beta;
  int32_t reserved;
  const void* a;
  const void* b;
  float* c;
  int64_t lda, ldb, ldc;
};
static_assert(sizeof(GemmProblem) == sizeof(coral_sgemm_problem_t), "descriptor layout");

struct TrsvProblem {
  int32_t uplo, trans, diag, n;
  const float* a;
  float* x;
  int64_t lda, incx;
};
static_assert(sizeof(TrsvProblem) == sizeof(coral_strsv_problem_t), "descriptor layout");

constexpr int kGT = 64;       // output tile edge
constexpr int kGK = 16;       // K slab
constexpr int kGThreads = 256;

__global__ void k_tile_prefix(const GemmProblem* __restrict__ probs, int count, int* __restrict__ prefix) {
  __shared__ int warp_tot[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < count; base += blockDim.x) {
    const int i = base + threadIdx.x;
    int t = 0;
    if (i < count) {
      const GemmProblem p = probs[i];
      t = (p.m > 0 && p.n > 0) ? ((p.m + kGT - 1) / kGT) * ((p.n + kGT - 1) / kGT) : 0;
    }
    // block-wide exclusive scan
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int v = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    if (lane == 31) warp_tot[w] = v;
    __syncthreads();
    if (w == 0) {
      int s = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int u = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += u;
      }
      warp_tot[lane] = s;  // inclusive warp totals
    }
    __syncthreads();
    const int excl = carry + (w ? warp_tot[w - 1] : 0) + v - t;
    if (i < count) prefix[i] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + t;
    __syncthreads();
  }
  if (threadIdx.x == 0) prefix[count] = carry;
}

template <typename TIn>
__device__ __forceinline__ float ld_in(const TIn* p);
template <> __device__ __forceinline__ float ld_in<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld_in<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __bfloat162float(*p);
}

template <typename TIn>
__global__ void __launch_bounds__(kGThreads)
k_gemm_grouped(const GemmProblem* __restrict__ probs, int count, const int* __restrict__ prefix) {
  __shared__ __align__(16) float As[2][kGK][kGT + 4];
  __shared__ __align__(16) float Bs[2][kGK][kGT + 4];
  const int total = prefix[count];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    // instance holding tile t: last i with prefix[i] <= t
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const GemmProblem p = probs[lo];
    const int local = t - prefix[lo];
    const int mt = (p.m + kGT - 1) / kGT;
    const int m0 = (local % mt) * kGT, n0 = (local / mt) * kGT;
    const TIn* A = static_cast<const TIn*>(p.a);
    const TIn* B = static_cast<const TIn*>(p.b);
    const bool a_km = p.op_a != CORAL_NO_TRANSPOSE, b_km = p.op_b == CORAL_NO_TRANSPOSE;

    float ra[4], rb[4];
    auto load = [&](int k0) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int idx = threadIdx.x + e * kGThreads;
        int r, kk;
        if (a_km) { kk = idx % kGK; r = idx / kGK; } else { r = idx % kGT; kk = idx / kGT; }
        const int gr = m0 + r, gk = k0 + kk;
        ra[e] = (gr < p.m && gk < p.k) ? ld_in<TIn>(a_km ? A + gk + (size_t)gr * p.lda : A + gr + (size_t)gk * p.lda) : 0.f;
        int c;
        if (b_km) { kk = idx % kGK; c = idx / kGK; } else { c = idx % kGT; kk = idx / kGT; }
        const int gc = n0 + c, gk2 = k0 + kk;
        rb[e] = (gc < p.n && gk2 < p.k) ? ld_in<TIn>(b_km ? B + gk2 + (size_t)gc * p.ldb : B + gc + (size_t)gk2 * p.ldb) : 0.f;
      }
    };
    auto store = [&](int buf) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int idx = threadIdx.x + e * kGThreads;
        int r, kk;
        if (a_km) { kk = idx % kGK; r = idx / kGK; } else { r = idx % kGT; kk = idx / kGT; }
        As[buf][kk][r] = ra[e];
        int c;
        if (b_km) { kk = idx % kGK; c = idx / kGK; } else { c = idx % kGT; kk = idx / kGT; }
        Bs[buf][kk][c] = rb[e];
      }
    };
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    const int ks = (p.k + kGK - 1) / kGK;
    __syncthreads();  // previous tile's readers are done with the buffers
    if (ks > 0) {
      load(0);
      store(0);
    }
    __syncthreads();
    for (int s = 0; s < ks; ++s) {
      const int cur = s & 1;
      if (s + 1 < ks) load((s + 1) * kGK);
#pragma unroll
      for (int kk = 0; kk < kGK; ++kk) {
        const float4 a4 = *reinterpret_cast<const float4*>(&As[cur][kk][ty * 4]);
        const float4 b4 = *reinterpret_cast<const float4*>(&Bs[cur][kk][tx * 4]);
        const float a[4] = {a4.x, a4.y, a4.z, a4.w}, b[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
      }
      if (s + 1 < ks) store(cur ^ 1);
      __syncthreads();
    }
    const bool beta0 = p.beta == 0.f, beta1 = p.beta == 1.f;
    const bool scale_only = p.alpha == 0.f || p.k == 0;  // sgemm_nn.rs:29-45
    // the four C loads of a column before its stores (no round trip per element)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gc = n0 + tx * 4 + j;
      if (gc >= p.n) continue;
      if (scale_only && beta1) continue;
      float cv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int gr = m0 + ty * 4 + i;
        cv[i] = (!beta0 && gr < p.m) ? p.c[gr + (size_t)gc * p.ldc] : 0.f;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int gr = m0 + ty * 4 + i;
        if (gr >= p.m) continue;
        float* cp = p.c + gr + (size_t)gc * p.ldc;
        if (scale_only) {
          *cp = beta0 ? 0.f : cv[i] * p.beta;
        } else {
          const float v = p.alpha * acc[i][j];
          *cp = beta0 ? v : beta1 ? cv[i] + v : p.beta * cv[i] + v;
        }
      }
    }
  }
}

// ---- batched TRSV --------------------------------------------------------------
constexpr int kBT = 64;
constexpr int kBTThreads = 256;

__global__ void __launch_bounds__(kBTThreads, 4)
k_trsv_batched(const TrsvProblem* __restrict__ probs, int count) {
  __shared__ float D[kBT][kBT + 1];  // D[r][c] = op(A)(b0 + r, b0 + c)
  __shared__ float xb[kBT];
  const int pi = blockIdx.x;
  if (pi >= count) return;
  const TrsvProblem p = probs[pi];
  const int n = p.n;
  if (n <= 0) return;
  const bool t = p.trans != CORAL_NO_TRANSPOSE;
  const bool lower_eff = (p.uplo == CORAL_LOWER) != t;
  const bool unit = p.diag == CORAL_UNIT;
  const float* A = p.a;
  float* x = p.x;
  const size_t lda = p.lda, incx = p.incx;
  auto opA = [&](int r, int c) -> float {  // op(A)(r, c)
    return t ? A[c + (size_t)r * lda] : A[r + (size_t)c * lda];
  };
  const int nblk = (n + kBT - 1) / kBT;
  for (int bi = 0; bi < nblk; ++bi) {
    const int blk = lower_eff ? bi : nblk - 1 - bi;
    const int b0 = blk * kBT, bn = min(kBT, n - b0);
    // stage the diagonal block of op(A): loads in groups of 8 before their
    // stores, so the block costs two memory round trips
#pragma unroll
    for (int q0 = 0; q0 < kBT * kBT / kBTThreads; q0 += 8) {
      float dv[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int e = threadIdx.x + (q0 + q) * kBTThreads;
        const int r = e % kBT, c = e / kBT;
        dv[q] = (r < bn && c < bn) ? (t ? A[(b0 + c) + (size_t)(b0 + r) * lda] : A[(b0 + r) + (size_t)(b0 + c) * lda])
                                   : 0.f;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int e = threadIdx.x + (q0 + q) * kBTThreads;
        D[e % kBT][e / kBT] = dv[q];
      }
    }
    if (threadIdx.x < kBT) xb[threadIdx.x] = threadIdx.x < bn ? x[(size_t)(b0 + threadIdx.x) * incx] : 0.f;
    __syncthreads();
    // warp 0: substitution on the diagonal block (lane owns rows lane, lane+32)
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      float r0 = xb[lane], r1 = xb[lane + 32];
      for (int s = 0; s < bn; ++s) {
        const int j = lower_eff ? s : bn - 1 - s;
        const int owner = j & 31;
        float xj = (j < 32) ? r0 : r1;
        xj = __shfl_sync(0xffffffffu, xj, owner);
        if (!unit) xj = xj / D[j][j];
        if (lane == owner) {
          if (j < 32) r0 = xj; else r1 = xj;
        }
        // eliminate column j from the rows still to be solved
        const int i0 = lane, i1 = lane + 32;
        if (lower_eff) {
          if (i0 > j && i0 < bn) r0 = fmaf(-D[i0][j], xj, r0);
          if (i1 > j && i1 < bn) r1 = fmaf(-D[i1][j], xj, r1);
        } else {
          if (i0 < j) r0 = fmaf(-D[i0][j], xj, r0);
          if (i1 < j) r1 = fmaf(-D[i1][j], xj, r1);
        }
      }
      xb[lane] = r0;
      xb[lane + 32] = r1;
    }
    __syncthreads();
    if (threadIdx.x < bn) x[(size_t)(b0 + threadIdx.x) * incx] = xb[threadIdx.x];
    // update the rows still to be solved: rhs_i -= sum_c op(A)(i, b0 + c) xb[c]
    const int r_lo = lower_eff ? b0 + bn : 0, r_hi = lower_eff ? n : b0;
    // Two rows at a time, their loads 16 per row before the sums (a single
    // CTA solves the largest instances, so its memory parallelism sets the
    // batch's tail)
    for (int i = r_lo + threadIdx.x; i < r_hi; i += 2 * kBTThreads) {
      const int i2 = i + kBTThreads;
      const bool two = i2 < r_hi;
      float s4[4] = {0.f, 0.f, 0.f, 0.f}, u4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 1
      for (int c0 = 0; c0 < kBT; c0 += 16) {
        float a[16], b[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          a[c] = c0 + c < bn ? opA(i, b0 + c0 + c) : 0.f;
          b[c] = two && c0 + c < bn ? opA(i2, b0 + c0 + c) : 0.f;
        }
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          s4[c & 3] = fmaf(a[c], xb[c0 + c], s4[c & 3]);
          u4[c & 3] = fmaf(b[c], xb[c0 + c], u4[c & 3]);
        }
      }
      x[(size_t)i * incx] -= (s4[0] + s4[1]) + (s4[2] + s4[3]);
      if (two) x[(size_t)i2 * incx] -= (u4[0] + u4[1]) + (u4[2] + u4[3]);
    }
    __syncthreads();
  }
}

}  // namespace
}  // namespace coral

using namespace coral;

extern "C" {

coral_status_t coral_sgemm_grouped(coral_handle_t hh, int input_type, size_t count,
                                   const coral_sgemm_problem_t* problems) {
  CORAL_HANDLE(hh);
  if (input_type != CORAL_INPUT_F32 && input_type != CORAL_INPUT_BF16) return bad_arg(H, 1);
  if (count == 0) return CORAL_OK;
  if (!problems) return bad_arg(H, 3);
  if (count > (size_t)INT32_MAX / 2) return CORAL_ERR_NOT_SUPPORTED;
  // Tensor cores for bf16 inputs and for fp32 inputs in split-BF16x3 mode;
  // exact FP32 FMA tiles otherwise (NATIVE, and SPLIT_BF16X6, whose error
  // bound the two-piece split does not meet).
  if (input_type == CORAL_INPUT_BF16 || H->gemm_mode == CORAL_GEMM_SPLIT_BF16X3)
    return enqueue_grouped_tc(H, input_type == CORAL_INPUT_BF16, count, problems);
  int* prefix = static_cast<int*>(scratch(H, (count + 1) * sizeof(int)));
  if (!prefix) return CORAL_ERR_ALLOC;
  const GemmProblem* pr = reinterpret_cast<const GemmProblem*>(problems);
  k_tile_prefix<<<1, 1024, 0, H->stream>>>(pr, (int)count, prefix);
  coral_status_t s = launch_status(H);
  if (s != CORAL_OK) return s;
  const unsigned grid = (unsigned)H->sm_count * 4;
  timed_begin(H);
  if (input_type == CORAL_INPUT_F32)
    k_gemm_grouped<float><<<grid, kGThreads, 0, H->stream>>>(pr, (int)count, prefix);
  else
    k_gemm_grouped<__nv_bfloat16><<<grid, kGThreads, 0, H->stream>>>(pr, (int)count, prefix);
  s = launch_status(H);
  timed_end(H);
  return s;
}

coral_status_t coral_set_grouped_config(coral_handle_t hh, const int tile_n[4]) {
  CORAL_HANDLE(hh);
  if (!tile_n) {
    H->grouped_policy = GroupedPolicy{{64, 128, 128, 256}};
    return CORAL_OK;
  }
  for (int i = 0; i < 4; ++i)
    if (tile_n[i] != 64 && tile_n[i] != 128 && tile_n[i] != 256) return bad_arg(H, 1);
  for (int i = 0; i < 4; ++i) H->grouped_policy.bn[i] = tile_n[i];
  return CORAL_OK;
}

coral_status_t coral_get_grouped_config(coral_handle_t hh, int tile_n[4]) {
  CORAL_HANDLE(hh);
  if (!tile_n) return bad_arg(H, 1);
  for (int i = 0; i < 4; ++i) tile_n[i] = H->grouped_policy.bn[i];
  return CORAL_OK;
}

coral_status_t coral_strsv_batched(coral_handle_t hh, size_t count,
                                   const coral_strsv_problem_t* problems) {
  CORAL_HANDLE(hh);
  if (count == 0) return CORAL_OK;
  if (!problems) return bad_arg(H, 2);
  if (count > (size_t)INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  timed_begin(H);
  k_trsv_batched<<<(unsigned)count, kBTThreads, 0, H->stream>>>(
      reinterpret_cast<const TrsvProblem*>(problems), (int)count);
  coral_status_t s = launch_status(H);
  timed_end(H);
  return s;
}

}  // extern "C"
