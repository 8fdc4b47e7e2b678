// Split-BF16 SGEMM / CGEMM on the 5th-generation tensor cores (tcgen05 + TMEM).
//
// An fp32 value a is split into bf16 pieces a = a0 + a1 (+ a2) + r, each piece
// the round-to-nearest bf16 of what the previous ones left (exact fp32
// subtractions).  With two pieces, |r| <= 2^-18 |a|; with three, 2^-27 |a|.
//   SPLIT_BF16X3: op(A) op(B) ~ A0 B0 + A0 B1 + A1 B0          (3 products)
//   SPLIT_BF16X6: ... + A1 B1 + A0 B2 + A2 B0                  (6 products)
// Every product is exact in the tensor core and accumulates in fp32 in TMEM.
//
// Pipeline per call:
//   1. split pre-pass: op(A) -> pieces [m][kp] and op(B)^T -> pieces [n][kp],
//      bf16, K contiguous (kp = k rounded up to 8 so rows are 16-byte
//      multiples).  Transposes through shared memory when the stored matrix
//      is contiguous along M/N.  Complex operands use the 4M mapping folded
//      into one real GEMM: A'' = [Re A | Im A] (k' = 2k) and rows
//      2j, 2j+1 of B'' = [Re B_j | -Im B_j], [Im B_j | Re B_j], so that
//      columns 2j, 2j+1 of A'' B''^T are Re and Im of C_j.
//   2. GEMM kernel: one CTA per 128 x BN tile of C.  Warp 0 lane 0 issues
//      TMA loads of all pieces of a 32-deep K slab into a 4-stage ring
//      (64-byte swizzle, full/empty mbarriers); warp 1 lane 0 issues the
//      tcgen05.mma products (M=128, N=BN, K=16 per instruction) into one
//      fp32 TMEM accumulator of BN columns and commits each stage back to
//      the producer; then all 4 warps read the accumulator row by row
//      (tcgen05.ld 32x32b, thread = row) and apply the reference's epilogue
//      (beta == 0: C = alpha*acc without reading C; beta == 1: C += alpha*acc;
//      else beta*C + alpha*acc; f32_edge.rs:37-58) with coalesced column
//      stores.
// All waits are bounded: a wait that gives up sets the handle's status word
// (reported as CORAL_ERR_TIMEOUT by coral_sync) and the CTA drains and exits.
#include "common.cuh"
#include "tc_common.cuh"

#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

namespace coral {

int gemm_bad_arg(int op_a, int op_b, size_t m, size_t n, size_t k, const void* a, size_t lda,
                 const void* b, size_t ldb, const void* c, size_t ldc, bool complex_ops);

// ---- tensor-map encoding (driver entry point, no libcuda link) -------------
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

bool encode_kmajor_map(CUtensorMap* map, const void* base, int elem_bytes, uint64_t inner,
                       uint64_t outer, uint64_t row_stride_bytes, uint32_t box_inner,
                       uint32_t box_outer, int swizzle_bytes) {
  auto fn = tmap_encode_fn();
  if (!fn) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_stride_bytes & 15)) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {row_stride_bytes};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUtensorMapDataType dt = elem_bytes == 8   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                           : elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                           : elem_bytes == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                             : CU_TENSOR_MAP_DATA_TYPE_UINT8;
  CUresult r = fn(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE,
                  swizzle_bytes == 0    ? CU_TENSOR_MAP_SWIZZLE_NONE
                  : swizzle_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                        : CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

namespace {

constexpr int kBM = 128;
constexpr int kBK = 32;   // bf16 elements per 64-byte swizzled row of a K slab
constexpr int kStages = 4;
constexpr int kSwizzle = kBK * 2;   // bytes: the TMA swizzle span of a slab row
// K slabs of kBK per 64-deep unit of the handle's chunk setting
constexpr int kSlabsPer64 = 64 / kBK;

__device__ __forceinline__ uint64_t slab_desc(uint32_t saddr) {
  return kSwizzle == 128 ? tc::desc_k_sw128(saddr) : tc::desc_k_sw64(saddr);
}

template <int P> struct SplitPlan;
// Products A_a(q) * B_b(q), small terms first, with the products that share an
// A piece adjacent so the tensor core keeps that piece in its A collector
// buffer (collect(q): fill, use, last use) instead of reading it again.
template <> struct SplitPlan<3> {
  static constexpr int kPieces = 2, kProducts = 3;
  // A1 B0, A0 B1 (fill A0), A0 B0 (last use of A0)
  __host__ __device__ static constexpr int a(int q) { return q == 0 ? 1 : 0; }
  __host__ __device__ static constexpr int b(int q) { return q == 1 ? 1 : 0; }
  __host__ __device__ static constexpr int collect(int q) {
    return q == 1 ? tc::kCollectFill : q == 2 ? tc::kCollectLastUse : tc::kCollectNone;
  }
};
template <> struct SplitPlan<6> {
  static constexpr int kPieces = 3, kProducts = 6;
  // A2 B0, A1 B1 (fill A1), A1 B0 (last use), A0 B2 (fill A0), A0 B1, A0 B0 (last use)
  __host__ __device__ static constexpr int a(int q) { return q == 0 ? 2 : q <= 2 ? 1 : 0; }
  __host__ __device__ static constexpr int b(int q) { return q == 3 ? 2 : (q == 1 || q == 4) ? 1 : 0; }
  __host__ __device__ static constexpr int collect(int q) {
    return (q == 1 || q == 3) ? tc::kCollectFill
           : q == 4           ? tc::kCollectUse
           : (q == 2 || q == 5) ? tc::kCollectLastUse
                              : tc::kCollectNone;
  }
};

// Issues product q of a split plan with its collector usage.
template <typename Plan>
__device__ __forceinline__ void mma_plan(int q, uint32_t acc, uint64_t ad, uint64_t bd, uint32_t idesc,
                                         uint32_t accumulate) {
  switch (Plan::collect(q)) {
    case tc::kCollectFill: tc::mma_f16_ca<tc::kCollectFill>(acc, ad, bd, idesc, accumulate); break;
    case tc::kCollectUse: tc::mma_f16_ca<tc::kCollectUse>(acc, ad, bd, idesc, accumulate); break;
    case tc::kCollectLastUse: tc::mma_f16_ca<tc::kCollectLastUse>(acc, ad, bd, idesc, accumulate); break;
    default: tc::mma_f16(acc, ad, bd, idesc, accumulate); break;
  }
}

struct SplitMaps {
  CUtensorMap a[3];
  CUtensorMap b[3];
};

// ---- 1. split pre-pass -------------------------------------------------------
// NPC = number of bf16 pieces (2 or 3).
template <int NPC>
__device__ __forceinline__ void split_value(float v, __nv_bfloat16 (&p)[3]) {
  static_assert(NPC == 2 || NPC == 3, "2 or 3 pieces");
  p[0] = __float2bfloat16_rn(v);
  float r = v - __bfloat162float(p[0]);
  p[1] = __float2bfloat16_rn(r);
  p[2] = __float2bfloat16_rn(0.f);
  if (NPC == 3) {
    r = r - __bfloat162float(p[1]);
    p[2] = __float2bfloat16_rn(r);
  }
}

// Real operand: dst[p][r][l] = piece p of src(r, l), where src(r, l) is
// X[l + r*ld] (K-major storage) or X[r + l*ld] (storage contiguous along r).
// 32 x 32 tiles, 32 x 8 threads; the contiguous-along-r case transposes
// through shared memory so both the loads and the stores are coalesced.
template <int NPC, bool kKMajorSrc>
__global__ void __launch_bounds__(256)
k_split_real(const float* __restrict__ X, size_t ld, int R, int Kd, __nv_bfloat16* __restrict__ dst,
             size_t kp, size_t piece_stride) {
  __shared__ float tile[32][33];
  const int r0 = blockIdx.y * 32, l0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  if (kKMajorSrc) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int r = r0 + ty + 8 * q, l = l0 + tx;
      tile[ty + 8 * q][tx] = (r < R && l < Kd) ? __ldg(X + l + (size_t)r * ld) : 0.f;
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int l = l0 + ty + 8 * q, r = r0 + tx;
      tile[tx][ty + 8 * q] = (r < R && l < Kd) ? __ldg(X + r + (size_t)l * ld) : 0.f;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int r = r0 + ty + 8 * q, l = l0 + tx;
    if (r < R && l < (int)kp) {
      __nv_bfloat16 p[3];
      split_value<NPC>(tile[ty + 8 * q][tx], p);
      size_t o = (size_t)r * kp + l;
#pragma unroll
      for (int i = 0; i < NPC; ++i) dst[i * piece_stride + o] = p[i];
    }
  }
}

// Eight consecutive K values of one row split into NPC pieces, each piece's
// eight bf16 stored with one 16-byte store at dst + i * piece_stride + o.
template <int NPC>
__device__ __forceinline__ void split_store8(const float (&v)[8], __nv_bfloat16* __restrict__ dst,
                                             size_t piece_stride, size_t o) {
  __align__(16) __nv_bfloat16 q[3][8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    __nv_bfloat16 p[3];
    split_value<NPC>(v[j], p);
#pragma unroll
    for (int i = 0; i < NPC; ++i) q[i][j] = p[i];
  }
#pragma unroll
  for (int i = 0; i < NPC; ++i)
    __stcs(reinterpret_cast<uint4*>(dst + i * piece_stride + o), *reinterpret_cast<const uint4*>(q[i]));
}

// Vector forms of k_split_real, for a 16-byte-aligned X with ld % 4 == 0
// (dst rows are 16-byte multiples: kp % 8 == 0).
// K-major storage (src(r, l) = X[l + r*ld]): a thread converts 8 consecutive
// K values of a row -- two 16-byte loads, one 16-byte store per piece; a
// block covers 2048 K values of one row, rows strided over grid.y.
template <int NPC>
__global__ void __launch_bounds__(256)
k_split_rows(const float* __restrict__ X, size_t ld, int R, int Kd, __nv_bfloat16* __restrict__ dst, size_t kp,
             size_t piece_stride) {
  const size_t l = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 8;
  if (l >= kp) return;
  for (int r = blockIdx.y; r < R; r += gridDim.y) {
    const float* src = X + (size_t)r * ld + l;
    float v[8];
    if (l + 8 <= (size_t)Kd) {
      const float4 a = __ldcs(reinterpret_cast<const float4*>(src));
      const float4 b = __ldcs(reinterpret_cast<const float4*>(src) + 1);
      v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
      v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else {
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = l + j < (size_t)Kd ? src[j] : 0.f;
    }
    split_store8<NPC>(v, dst, piece_stride, (size_t)r * kp + l);
  }
}

// Storage contiguous along r (src(r, l) = X[r + l*ld]): 64 x 64 tiles read
// as 16-byte column segments, transposed through shared memory (pitch 65:
// at most 2-way bank conflicts on the column reads), written as 16-byte
// row segments of 8 K values; a warp writes 4 rows x 128 contiguous bytes
// per piece.  Tiles along r are strided over grid.y.
template <int NPC>
__global__ void __launch_bounds__(256)
k_split_cols(const float* __restrict__ X, size_t ld, int R, int Kd, __nv_bfloat16* __restrict__ dst, size_t kp,
             size_t piece_stride) {
  __shared__ float tile[64][65];   // [l][r]
  const int t = threadIdx.x;
  const int l0 = blockIdx.x * 64;
  for (int r0 = blockIdx.y * 64; r0 < R; r0 += gridDim.y * 64) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int ll = t / 16 + 16 * q, r4 = t % 16;
      const int l = l0 + ll, r = r0 + 4 * r4;
      float e[4] = {0.f, 0.f, 0.f, 0.f};
      if (l < Kd) {
        const float* src = X + r + (size_t)l * ld;
        if (r + 3 < R) {
          const float4 a = __ldcs(reinterpret_cast<const float4*>(src));
          e[0] = a.x; e[1] = a.y; e[2] = a.z; e[3] = a.w;
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j) e[j] = r + j < R ? src[j] : 0.f;
        }
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) tile[ll][4 * r4 + j] = e[j];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int task = t + 256 * q, c = task % 8, rl = task / 8;
      const int r = r0 + rl;
      const size_t l = (size_t)l0 + 8 * c;
      if (r < R && l < kp) {
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = tile[8 * c + j][rl];
        split_store8<NPC>(v, dst, piece_stride, (size_t)r * kp + l);
      }
    }
    __syncthreads();
  }
}

// Splits op(X)'s R x Kd block into NPC pieces [R][kp]: the vector kernels
// when X is 16-byte aligned with ld % 4 == 0, else k_split_real.
template <int NPC>
void launch_split_real(cudaStream_t st, const float* X, size_t ld, int R, int Kd, bool kmajor,
                       __nv_bfloat16* dst, size_t kp, size_t piece_stride) {
  const bool vec = aligned16(X) && ld % 4 == 0;
  if (vec && kmajor) {
    const dim3 g((unsigned)((kp / 8 + 255) / 256), (unsigned)(R < 65535 ? R : 65535));
    k_split_rows<NPC><<<g, 256, 0, st>>>(X, ld, R, Kd, dst, kp, piece_stride);
  } else if (vec) {
    const int rt = (R + 63) / 64;
    const dim3 g((unsigned)((kp + 63) / 64), (unsigned)(rt < 65535 ? rt : 65535));
    k_split_cols<NPC><<<g, 256, 0, st>>>(X, ld, R, Kd, dst, kp, piece_stride);
  } else {
    const dim3 g((unsigned)((kp + 31) / 32), (unsigned)((R + 31) / 32));
    if (kmajor) k_split_real<NPC, true><<<g, 256, 0, st>>>(X, ld, R, Kd, dst, kp, piece_stride);
    else k_split_real<NPC, false><<<g, 256, 0, st>>>(X, ld, R, Kd, dst, kp, piece_stride);
  }
}

// Complex operand, 4M layout.  src(r, l) is the complex element of op(X)
// (conjugated when `conj`), storage K-major (X[l + r*ld]) or not (X[r + l*ld]).
//   kIsB == false: dst row r = [Re src(r, :) | Im src(r, :)]          (k' = 2k)
//   kIsB == true : dst row 2r = [Re | -Im], row 2r+1 = [Im | Re]       (k' = 2k)
template <int NPC, bool kKMajorSrc, bool kIsB>
__global__ void __launch_bounds__(256)
k_split_cplx(const float2* __restrict__ X, size_t ld, int R, int Kd, bool conj,
             __nv_bfloat16* __restrict__ dst, size_t kp, size_t piece_stride) {
  __shared__ float2 tile[32][33];
  const int r0 = blockIdx.y * 32, l0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  if (kKMajorSrc) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int r = r0 + ty + 8 * q, l = l0 + tx;
      tile[ty + 8 * q][tx] = (r < R && l < Kd) ? __ldg(X + l + (size_t)r * ld) : make_float2(0.f, 0.f);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int l = l0 + ty + 8 * q, r = r0 + tx;
      tile[tx][ty + 8 * q] = (r < R && l < Kd) ? __ldg(X + r + (size_t)l * ld) : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int r = r0 + ty + 8 * q, l = l0 + tx;
    if (r >= R || l >= Kd) continue;
    float2 v = tile[ty + 8 * q][tx];
    if (conj) v.y = -v.y;
    __nv_bfloat16 pr[3], pi[3], pn[3];
    split_value<NPC>(v.x, pr);
    split_value<NPC>(v.y, pi);
    split_value<NPC>(-v.y, pn);
    if (!kIsB) {
      size_t o = (size_t)r * kp;
#pragma unroll
      for (int i = 0; i < NPC; ++i) {
        dst[i * piece_stride + o + l] = pr[i];
        dst[i * piece_stride + o + Kd + l] = pi[i];
      }
    } else {
      size_t o0 = (size_t)(2 * r) * kp, o1 = o0 + kp;
#pragma unroll
      for (int i = 0; i < NPC; ++i) {
        dst[i * piece_stride + o0 + l] = pr[i];
        dst[i * piece_stride + o0 + Kd + l] = pn[i];
        dst[i * piece_stride + o1 + l] = pi[i];
        dst[i * piece_stride + o1 + Kd + l] = pr[i];
      }
    }
  }
}

// Complex operand, 3M layout: three real matrices of op(X) (conjugated when
// `conj`), each [R][kp] with NPC pieces: part 0 Re, part 1 Im, part 2 Re + Im
// (the sum rounded in fp32 before it is split).  K past Kd is written as zero.
template <int NPC, bool kKMajorSrc>
__global__ void __launch_bounds__(256)
k_split_cplx3(const float2* __restrict__ X, size_t ld, int R, int Kd, bool conj,
              __nv_bfloat16* __restrict__ dst, size_t kp, size_t piece_stride, size_t part_stride) {
  __shared__ float2 tile[32][33];
  const int r0 = blockIdx.y * 32, l0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  if (kKMajorSrc) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int r = r0 + ty + 8 * q, l = l0 + tx;
      tile[ty + 8 * q][tx] = (r < R && l < Kd) ? __ldg(X + l + (size_t)r * ld) : make_float2(0.f, 0.f);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int l = l0 + ty + 8 * q, r = r0 + tx;
      tile[tx][ty + 8 * q] = (r < R && l < Kd) ? __ldg(X + r + (size_t)l * ld) : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int r = r0 + ty + 8 * q, l = l0 + tx;
    if (r >= R || l >= (int)kp) continue;
    float2 v = tile[ty + 8 * q][tx];  // zero past Kd
    if (conj) v.y = -v.y;
    const float vals[3] = {v.x, v.y, v.x + v.y};
    const size_t o = (size_t)r * kp + l;
#pragma unroll
    for (int part = 0; part < 3; ++part) {
      __nv_bfloat16 p[3];
      split_value<NPC>(vals[part], p);
#pragma unroll
      for (int i = 0; i < NPC; ++i) dst[part * part_stride + i * piece_stride + o] = p[i];
    }
  }
}

// 3M combine: with T1 = Re A Re B, T2 = Im A Im B, T3 = (Re A + Im A)(Re B + Im B)
// (m x n, column-major, ld m), C = alpha (T1 - T2 + i (T3 - T1 - T2)) + beta C.
__global__ void k_combine_3m(const float* __restrict__ t1, const float* __restrict__ t2,
                             const float* __restrict__ t3, int m, int n, float2 alpha, float2 beta,
                             float2* __restrict__ C, size_t ldc) {
  const size_t total = (size_t)m * n;
  const bool beta0 = beta.x == 0.f && beta.y == 0.f;
  const bool beta1 = beta.x == 1.f && beta.y == 0.f;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const float a = t1[t], b = t2[t], c3 = t3[t];
    const float re = a - b, im = c3 - a - b;
    float2 v = make_float2(alpha.x * re - alpha.y * im, alpha.x * im + alpha.y * re);
    float2* cp = C + t % m + (t / m) * ldc;
    if (!beta0) {
      const float2 cv = *cp;
      if (beta1) { v.x += cv.x; v.y += cv.y; }
      else {
        v.x += beta.x * cv.x - beta.y * cv.y;
        v.y += beta.x * cv.y + beta.y * cv.x;
      }
    }
    *cp = v;
  }
}

// ---- 2. tcgen05 GEMM ---------------------------------------------------------
struct EpiParams {
  float* C;          // real: float column-major; complex: float2 column-major
  size_t ldc;
  int m, n;          // logical C extent (complex: n complex columns)
  float alpha_re, alpha_im, beta_re, beta_im;
  int complex_out;   // 1: accumulator columns (2j, 2j+1) are (Re, Im) of C column j
};

// Tile order: groups of 16 M-tiles sweep all N-tiles, so CTAs resident at
// the same time share A and B slabs through L2.
__device__ __forceinline__ void tile_coords(int tile, int m_tiles, int n_tiles, int& mt, int& nt) {
  const int group = 16;
  const int per_group = group * n_tiles;
  const int g = tile / per_group;
  const int gm0 = g * group;
  const int gsz = min(group, m_tiles - gm0);
  const int within = tile - g * per_group;
  mt = gm0 + within % gsz;
  nt = within / gsz;
}

// Persistent kernel, 2 + 8 warps:
//   warp 0 lane 0: TMA producer over a 4-stage ring of K slabs (all pieces);
//   warp 1 lane 0: tcgen05.mma issuer.  The K loop of a tile is cut into
//     chunks of `chunk_kb` slabs; chunk c accumulates (from zero) into TMEM
//     buffer c % 2 and is committed to chunk_full[c % 2];
//   warps 2-9: drain each finished chunk into fp32 registers with
//     round-to-nearest adds (thread = one row of the tile, half of the
//     columns), release the buffer (chunk_empty), and after the tile's last
//     chunk apply the epilogue and store C.
// Draining per chunk bounds how many tensor-core accumulation steps any
// partial sum goes through; the register adds round to nearest.
constexpr int kEpiWarps = 8;
constexpr int kSplitThreads = 64 + 32 * kEpiWarps;
constexpr int kCGroup = 8;  // C columns loaded together by the epilogue

template <int NP, int BN>
__global__ void __launch_bounds__(kSplitThreads, 1)
k_gemm_split(const __grid_constant__ SplitMaps maps, int kdim, int m_tiles, int n_tiles,
             int chunk_kb, int splits, float* ws, int ws_cols, EpiParams ep, unsigned* status,
             uint64_t limit_ns) {
  using Plan = SplitPlan<NP>;
  constexpr int kPieces = Plan::kPieces;
  constexpr uint32_t kATile = kBM * kBK * 2;  // bytes per A piece tile
  constexpr uint32_t kBTile = BN * kBK * 2;
  constexpr uint32_t kStageBytes = kPieces * (kATile + kBTile);
  constexpr uint32_t kIdesc = tc::idesc_bf16_f32(kBM, BN);
  constexpr int kCols = BN / 2;  // accumulator columns per epilogue thread

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = tc::align1024_shared(smem_raw);
  __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages];
  __shared__ __align__(8) uint64_t chunk_full[2], chunk_empty[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (kdim + kBK - 1) / kBK;
  // Work item = (output tile, K part); with splits > 1 each part covers
  // ceil(nk / splits) slabs and its raw sums go to the workspace.
  const int total_items = m_tiles * n_tiles * splits;
  const int sk = (nk + splits - 1) / splits;
  auto slab_range = [&](int item, int& lo, int& hi) {
    const int part = item % splits;
    lo = min(nk, part * sk);
    hi = min(nk, lo + sk);
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      tc::mbar_init(&full_bar[s], 1);
      tc::mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&chunk_full[b], 1);
      tc::mbar_init(&chunk_empty[b], kEpiWarps);
    }
    abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(&tmem_slot, 2 * BN);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer ----
      for (int p = 0; p < kPieces; ++p) {
        tc::prefetch_tmap(&maps.a[p]);
        tc::prefetch_tmap(&maps.b[p]);
      }
      int it = 0;  // k-slab counter across tiles
      for (int item = blockIdx.x; item < total_items && !abort_flag; item += gridDim.x) {
        int mt, nt, kb_lo, kb_hi;
        tile_coords(item / splits, m_tiles, n_tiles, mt, nt);
        slab_range(item, kb_lo, kb_hi);
        // K-serpentine: items of odd waves walk their slabs downwards, so a
        // wave starts on the slabs the previous wave read last, which are
        // the ones still in L2.  The MMA side consumes stages in order and
        // does not depend on the direction.
        const bool down = ((item / (int)gridDim.x) & 1) != 0;
        for (int j = 0; j < kb_hi - kb_lo; ++j, ++it) {
          const int kb = down ? kb_hi - 1 - j : kb_lo + j;
          const int s = it % kStages;
          if (it >= kStages && !tc::mbar_wait(&empty_bar[s], ((it / kStages) - 1) & 1, limit_ns)) {
            atomicOr(status, kStatusTimeout);
            atomicExch(&abort_flag, 1);
            break;
          }
          if (*(volatile int*)&abort_flag) break;
          uint8_t* st = smem + (size_t)s * kStageBytes;
          tc::mbar_expect_tx(&full_bar[s], kStageBytes);
          for (int p = 0; p < kPieces; ++p) {
            tc::tma_load_2d(st + p * kATile, &maps.a[p], &full_bar[s], kb * kBK, mt * kBM);
            tc::tma_load_2d(st + kPieces * kATile + p * kBTile, &maps.b[p], &full_bar[s], kb * kBK, nt * BN);
          }
        }
      }
      // Drain: every issued load lands before the CTA may exit.
      for (int j = (it > kStages ? it - kStages : 0); j < it; ++j)
        tc::mbar_wait(&full_bar[j % kStages], (j / kStages) & 1, limit_ns);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer ----
      int it = 0, gc = 0;  // k-slab and chunk counters across tiles
      bool stop = false;
      for (int item = blockIdx.x; item < total_items && !stop; item += gridDim.x) {
        int kb_lo, kb_hi;
        slab_range(item, kb_lo, kb_hi);
        const int chunks = (kb_hi - kb_lo + chunk_kb - 1) / chunk_kb;
        for (int c = 0; c < chunks && !stop; ++c, ++gc) {
          const int b = gc & 1;
          if (gc >= 2 && !tc::mbar_wait(&chunk_empty[b], ((gc >> 1) - 1) & 1, limit_ns)) {
            atomicOr(status, kStatusTimeout);
            atomicExch(&abort_flag, 1);
            stop = true;
            break;
          }
          tc::tc_fence_after();
          const uint32_t acc = tmem + b * BN;
          const int kb0 = kb_lo + c * chunk_kb, kb1 = min(kb_hi, kb0 + chunk_kb);
          for (int kb = kb0; kb < kb1; ++kb, ++it) {
            const int s = it % kStages;
            if (!tc::mbar_wait(&full_bar[s], (it / kStages) & 1, limit_ns)) {
              atomicOr(status, kStatusTimeout);
              atomicExch(&abort_flag, 1);
              stop = true;
              break;
            }
            tc::tc_fence_after();
            const uint32_t sa = tc::smem_u32(smem + (size_t)s * kStageBytes);
            const uint32_t sb = sa + kPieces * kATile;
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk) {
#pragma unroll
              for (int q = 0; q < Plan::kProducts; ++q) {
                const uint64_t ad = slab_desc(sa + Plan::a(q) * kATile + kk * 32);
                const uint64_t bd = slab_desc(sb + Plan::b(q) * kBTile + kk * 32);
                mma_plan<Plan>(q, acc, ad, bd, kIdesc, ((kb - kb0) | kk | q) != 0);
              }
            }
            tc::mma_commit(&empty_bar[s]);
          }
          tc::mma_commit(&chunk_full[b]);
        }
      }
    }
  } else {
    // ---- epilogue warps ----
    const int ew = warp - 2;
    const int quad = warp & 3;           // TMEM lane quadrant this warp may access
    const int half = ew >> 2;            // column half of the tile
    const uint32_t lane_base = (uint32_t)(quad * 32) << 16;
    const bool beta0 = ep.beta_re == 0.f && ep.beta_im == 0.f;
    const bool beta1 = ep.beta_re == 1.f && ep.beta_im == 0.f;
    int gc = 0;
    bool stop = false;
    for (int item = blockIdx.x; item < total_items && !stop; item += gridDim.x) {
      int mt, nt, kb_lo, kb_hi;
      tile_coords(item / splits, m_tiles, n_tiles, mt, nt);
      slab_range(item, kb_lo, kb_hi);
      const int chunks = (kb_hi - kb_lo + chunk_kb - 1) / chunk_kb;
      float sum[kCols];
#pragma unroll
      for (int j = 0; j < kCols; ++j) sum[j] = 0.f;
      for (int c = 0; c < chunks; ++c, ++gc) {
        const int b = gc & 1;
        if (!tc::mbar_wait(&chunk_full[b], (gc >> 1) & 1, limit_ns)) {
          atomicOr(status, kStatusTimeout);
          stop = true;
          break;
        }
        tc::tc_fence_after();
        const uint32_t acc = tmem + b * BN + half * kCols + lane_base;
#pragma unroll
        for (int c0 = 0; c0 < kCols; c0 += 32) {
          uint32_t r[32];
          tc::tmem_ld32(acc + c0, r);
          tc::tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 32; ++j) sum[c0 + j] += __uint_as_float(r[j]);
        }
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&chunk_empty[b]);
      }
      if (stop || *(volatile int*)&abort_flag) break;
      const int row = mt * kBM + quad * 32 + lane;
      if (row >= ep.m) continue;
      const int col0 = nt * BN + half * kCols;  // first accumulator column of this thread
      if (splits > 1) {  // raw partial sums; k_split_reduce applies the epilogue
        float* wp = ws + ((size_t)(item % splits) * ws_cols) * ep.m + row;
#pragma unroll
        for (int j = 0; j < kCols; ++j)
          if (col0 + j < ws_cols) wp[(size_t)(col0 + j) * ep.m] = sum[j];
      } else if (!ep.complex_out) {
        // C is read in groups of kCGroup columns, all loads of a group before
        // any store: a store followed by a load the compiler cannot prove
        // disjoint would otherwise cost a memory round trip per column.
        float* crow = ep.C + row;
#pragma unroll
        for (int g = 0; g < kCols; g += kCGroup) {
          float cv[kCGroup];
#pragma unroll
          for (int j = 0; j < kCGroup; ++j)
            cv[j] = (!beta0 && col0 + g + j < ep.n) ? crow[(size_t)(col0 + g + j) * ep.ldc] : 0.f;
#pragma unroll
          for (int j = 0; j < kCGroup; ++j) {
            const int col = col0 + g + j;
            if (col < ep.n) {
              const float v = ep.alpha_re * sum[g + j];
              crow[(size_t)col * ep.ldc] = beta0 ? v : beta1 ? cv[j] + v : ep.beta_re * cv[j] + v;
            }
          }
        }
      } else {
        float2* crow = reinterpret_cast<float2*>(ep.C) + row;
#pragma unroll
        for (int g = 0; g < kCols / 2; g += kCGroup / 2) {
          float2 cvs[kCGroup / 2];
#pragma unroll
          for (int j = 0; j < kCGroup / 2; ++j)
            cvs[j] = (!beta0 && col0 / 2 + g + j < ep.n) ? crow[(size_t)(col0 / 2 + g + j) * ep.ldc]
                                                          : make_float2(0.f, 0.f);
#pragma unroll
          for (int j = 0; j < kCGroup / 2; ++j) {
            const int col = col0 / 2 + g + j;
            if (col < ep.n) {
              const float ar = sum[2 * (g + j)], ai = sum[2 * (g + j) + 1];
              float2 v = make_float2(ep.alpha_re * ar - ep.alpha_im * ai, ep.alpha_re * ai + ep.alpha_im * ar);
              if (!beta0) {
                const float2 cv = cvs[j];
                if (beta1) { v.x += cv.x; v.y += cv.y; }
                else {
                  v.x += ep.beta_re * cv.x - ep.beta_im * cv.y;
                  v.y += ep.beta_re * cv.y + ep.beta_im * cv.x;
                }
              }
              crow[(size_t)col * ep.ldc] = v;
            }
          }
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) tc::tmem_dealloc(tmem, 2 * BN);
}

// ---- 2b. CTA-pair tcgen05 GEMM (cta_group::2) ---------------------------------
// A 256 x 256 tile of C per cluster of two CTAs on two SMs.  For each 32-deep
// K slab, CTA r (r = 0, 1) stages rows [128 r, 128 r + 128) of the tile's A
// pieces and of its B pieces; the even CTA issues tcgen05.mma.cta_group::2
// (M = 256, N = 256, K = 16), which reads A and B from both CTAs' shared
// memory and accumulates rows [128 r, 128 r + 128) x 256 columns into CTA r's
// TMEM.  Per SM an instruction reads 128 rows of B where the single-CTA
// 128 x 256 tile reads 256, so the B operand's shared-memory traffic per flop
// halves, and each CTA's ring slot is 32 KB instead of 48 KB (6 stages).
// Barriers:
//   full_bar[s]   even CTA only: armed by its producer with both CTAs' bytes;
//                 both CTAs' TMA loads count on it (.cta_group::2 loads);
//   empty_bar[s]  both CTAs: the MMA commit multicast to the pair;
//   chunk_full[b] both CTAs: likewise, after a chunk's last MMA;
//   chunk_empty[b] even CTA only: 2 x kEpiWarps arrivals, the odd CTA's
//                 epilogue warps arriving through the cluster window.
// Epilogue, split-K and the K-serpentine order follow k_gemm_split.  Every
// wait is bounded; a CTA that gives up sets the status word, and its partner's
// waits then run out too, so both CTAs reach the closing cluster barrier.
constexpr int kPairHalf = 128;  // rows of A and of B staged per CTA
constexpr int kPairTile = 256;  // tile edge in M and N

template <int NP>
struct PairRing {
  static constexpr int kPieces = SplitPlan<NP>::kPieces;
  static constexpr uint32_t kPieceTile = kPairHalf * kBK * 2;            // 8 KB
  static constexpr uint32_t kStageBytes = 2 * kPieces * kPieceTile;      // this CTA's A and B pieces
  static constexpr int kStages = NP == 3 ? 6 : 4;
};

// Tile order for the pair kernel: groups of `group` M-tiles sweep all N-tiles.
__device__ __forceinline__ void tile_coords_g(int tile, int m_tiles, int group, int& mt, int& nt,
                                              int n_tiles) {
  const int per_group = group * n_tiles;
  const int g = tile / per_group;
  const int gm0 = g * group;
  const int gsz = min(group, m_tiles - gm0);
  const int within = tile - g * per_group;
  mt = gm0 + within % gsz;
  nt = within / gsz;
}

template <typename Plan>
__device__ __forceinline__ void mma_plan_pair(int q, uint32_t acc, uint64_t ad, uint64_t bd,
                                              uint32_t idesc, uint32_t accumulate) {
  switch (Plan::collect(q)) {
    case tc::kCollectFill: tc::mma_f16_pair<tc::kCollectFill>(acc, ad, bd, idesc, accumulate); break;
    case tc::kCollectUse: tc::mma_f16_pair<tc::kCollectUse>(acc, ad, bd, idesc, accumulate); break;
    case tc::kCollectLastUse: tc::mma_f16_pair<tc::kCollectLastUse>(acc, ad, bd, idesc, accumulate); break;
    default: tc::mma_f16_pair<tc::kCollectNone>(acc, ad, bd, idesc, accumulate); break;
  }
}

template <int NP>
__global__ void __launch_bounds__(kSplitThreads, 1)
k_gemm_split_pair(const __grid_constant__ SplitMaps maps, int kdim, int m_tiles, int n_tiles, int group,
                  int chunk_kb, int splits, float* ws, int ws_cols, EpiParams ep, unsigned* status,
                  uint64_t limit_ns) {
  using Plan = SplitPlan<NP>;
  using Ring = PairRing<NP>;
  constexpr int kPieces = Ring::kPieces;
  constexpr int kS = Ring::kStages;
  constexpr uint32_t kPieceTile = Ring::kPieceTile;
  constexpr uint32_t kStageBytes = Ring::kStageBytes;
  constexpr uint32_t kIdesc = tc::idesc_bf16_f32(kPairTile, kPairTile);
  constexpr int kCols = kPairTile / 2;  // accumulator columns per epilogue thread
  constexpr uint16_t kPairMask = 3;

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = tc::align1024_shared(smem_raw);
  __shared__ __align__(8) uint64_t full_bar[kS], empty_bar[kS];
  __shared__ __align__(8) uint64_t chunk_full[2], chunk_empty[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = tc::cluster_ctarank();
  const int cluster = (int)(blockIdx.x >> 1), nclusters = (int)(gridDim.x >> 1);
  const int nk = (kdim + kBK - 1) / kBK;
  const int total_items = m_tiles * n_tiles * splits;
  const int sk = (nk + splits - 1) / splits;
  auto slab_range = [&](int item, int& lo, int& hi) {
    const int part = item % splits;
    lo = min(nk, part * sk);
    hi = min(nk, lo + sk);
  };

  if (threadIdx.x == 0) {
    for (int s = 0; s < kS; ++s) {
      tc::mbar_init(&full_bar[s], 1);
      tc::mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&chunk_full[b], 1);
      tc::mbar_init(&chunk_empty[b], 2 * kEpiWarps);
    }
    abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 1) {
    tc::tmem_alloc_pair(&tmem_slot, 2 * kPairTile);
    tc::tmem_relinquish_pair();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::cluster_sync();  // both CTAs' barriers exist before any remote use
  tc::tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer (both CTAs) ----
      for (int p = 0; p < kPieces; ++p) {
        tc::prefetch_tmap(&maps.a[p]);
        tc::prefetch_tmap(&maps.b[p]);
      }
      int it = 0;
      for (int item = cluster; item < total_items && !abort_flag; item += nclusters) {
        int mt, nt, kb_lo, kb_hi;
        tile_coords_g(item / splits, m_tiles, group, mt, nt, n_tiles);
        slab_range(item, kb_lo, kb_hi);
        const bool down = ((item / nclusters) & 1) != 0;
        const int row_a = mt * kPairTile + (int)rank * kPairHalf;
        const int row_b = nt * kPairTile + (int)rank * kPairHalf;
        for (int j = 0; j < kb_hi - kb_lo; ++j, ++it) {
          const int kb = down ? kb_hi - 1 - j : kb_lo + j;
          const int s = it % kS;
          if (it >= kS && !tc::mbar_wait(&empty_bar[s], ((it / kS) - 1) & 1, limit_ns)) {
            atomicOr(status, kStatusTimeout);
            atomicExch(&abort_flag, 1);
            break;
          }
          if (*(volatile int*)&abort_flag) break;
          uint8_t* st = smem + (size_t)s * kStageBytes;
          if (rank == 0) tc::mbar_expect_tx(&full_bar[s], 2 * kStageBytes);
          const uint32_t fb = tc::mapa_shared(tc::smem_u32(&full_bar[s]), 0);
          for (int p = 0; p < kPieces; ++p) {
            tc::tma_load_2d_pair(st + p * kPieceTile, &maps.a[p], fb, kb * kBK, row_a);
            tc::tma_load_2d_pair(st + (kPieces + p) * kPieceTile, &maps.b[p], fb, kb * kBK, row_b);
          }
        }
      }
      // Drain: a slab's loads have landed once the MMA that read it released
      // the slot, so wait for the last slots' releases before exiting.
      for (int j = (it > kS ? it - kS : 0); j < it; ++j)
        tc::mbar_wait(&empty_bar[j % kS], (j / kS) & 1, limit_ns);
    }
  } else if (warp == 1) {
    if (lane == 0 && rank == 0) {
      // ---- MMA issuer (even CTA) ----
      int it = 0, gc = 0;
      bool stop = false;
      for (int item = cluster; item < total_items && !stop; item += nclusters) {
        int kb_lo, kb_hi;
        slab_range(item, kb_lo, kb_hi);
        const int chunks = (kb_hi - kb_lo + chunk_kb - 1) / chunk_kb;
        for (int c = 0; c < chunks && !stop; ++c, ++gc) {
          const int b = gc & 1;
          if (gc >= 2 && !tc::mbar_wait(&chunk_empty[b], ((gc >> 1) - 1) & 1, limit_ns)) {
            atomicOr(status, kStatusTimeout);
            atomicExch(&abort_flag, 1);
            stop = true;
            break;
          }
          tc::tc_fence_after();
          const uint32_t acc = tmem + b * kPairTile;
          const int kb0 = kb_lo + c * chunk_kb, kb1 = min(kb_hi, kb0 + chunk_kb);
          for (int kb = kb0; kb < kb1; ++kb, ++it) {
            const int s = it % kS;
            if (!tc::mbar_wait(&full_bar[s], (it / kS) & 1, limit_ns)) {
              atomicOr(status, kStatusTimeout);
              atomicExch(&abort_flag, 1);
              stop = true;
              break;
            }
            tc::tc_fence_after();
            const uint32_t sa = tc::smem_u32(smem + (size_t)s * kStageBytes);
            const uint32_t sb = sa + kPieces * kPieceTile;
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk) {
#pragma unroll
              for (int q = 0; q < Plan::kProducts; ++q) {
                const uint64_t ad = slab_desc(sa + Plan::a(q) * kPieceTile + kk * 32);
                const uint64_t bd = slab_desc(sb + Plan::b(q) * kPieceTile + kk * 32);
                mma_plan_pair<Plan>(q, acc, ad, bd, kIdesc, ((kb - kb0) | kk | q) != 0);
              }
            }
            tc::mma_commit_pair(&empty_bar[s], kPairMask);
          }
          tc::mma_commit_pair(&chunk_full[b], kPairMask);
        }
      }
    }
  } else {
    // ---- epilogue warps (both CTAs): rows [128 r, 128 r + 128) of the tile ----
    const int ew = warp - 2;
    const int quad = warp & 3;
    const int half = ew >> 2;
    const uint32_t lane_base = (uint32_t)(quad * 32) << 16;
    const bool beta0 = ep.beta_re == 0.f && ep.beta_im == 0.f;
    const bool beta1 = ep.beta_re == 1.f && ep.beta_im == 0.f;
    int gc = 0;
    bool stop = false;
    for (int item = cluster; item < total_items && !stop; item += nclusters) {
      int mt, nt, kb_lo, kb_hi;
      tile_coords_g(item / splits, m_tiles, group, mt, nt, n_tiles);
      slab_range(item, kb_lo, kb_hi);
      const int chunks = (kb_hi - kb_lo + chunk_kb - 1) / chunk_kb;
      float sum[kCols];
#pragma unroll
      for (int j = 0; j < kCols; ++j) sum[j] = 0.f;
      for (int c = 0; c < chunks; ++c, ++gc) {
        const int b = gc & 1;
        if (!tc::mbar_wait(&chunk_full[b], (gc >> 1) & 1, limit_ns)) {
          atomicOr(status, kStatusTimeout);
          stop = true;
          break;
        }
        tc::tc_fence_after();
        const uint32_t acc = tmem + b * kPairTile + half * kCols + lane_base;
#pragma unroll
        for (int c0 = 0; c0 < kCols; c0 += 32) {
          uint32_t r[32];
          tc::tmem_ld32(acc + c0, r);
          tc::tmem_wait_ld();
#pragma unroll
          for (int j = 0; j < 32; ++j) sum[c0 + j] += __uint_as_float(r[j]);
        }
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive_cluster(tc::mapa_shared(tc::smem_u32(&chunk_empty[b]), 0));
      }
      if (stop || *(volatile int*)&abort_flag) break;
      const int row = mt * kPairTile + (int)rank * kPairHalf + quad * 32 + lane;
      if (row >= ep.m) continue;
      const int col0 = nt * kPairTile + half * kCols;
      if (splits > 1) {
        float* wp = ws + ((size_t)(item % splits) * ws_cols) * ep.m + row;
#pragma unroll
        for (int j = 0; j < kCols; ++j)
          if (col0 + j < ws_cols) wp[(size_t)(col0 + j) * ep.m] = sum[j];
      } else if (!ep.complex_out) {
        float* crow = ep.C + row;
#pragma unroll
        for (int g = 0; g < kCols; g += kCGroup) {
          float cv[kCGroup];
#pragma unroll
          for (int j = 0; j < kCGroup; ++j)
            cv[j] = (!beta0 && col0 + g + j < ep.n) ? crow[(size_t)(col0 + g + j) * ep.ldc] : 0.f;
#pragma unroll
          for (int j = 0; j < kCGroup; ++j) {
            const int col = col0 + g + j;
            if (col < ep.n) {
              const float v = ep.alpha_re * sum[g + j];
              crow[(size_t)col * ep.ldc] = beta0 ? v : beta1 ? cv[j] + v : ep.beta_re * cv[j] + v;
            }
          }
        }
      } else {
        float2* crow = reinterpret_cast<float2*>(ep.C) + row;
#pragma unroll
        for (int g = 0; g < kCols / 2; g += kCGroup / 2) {
          float2 cvs[kCGroup / 2];
#pragma unroll
          for (int j = 0; j < kCGroup / 2; ++j)
            cvs[j] = (!beta0 && col0 / 2 + g + j < ep.n) ? crow[(size_t)(col0 / 2 + g + j) * ep.ldc]
                                                          : make_float2(0.f, 0.f);
#pragma unroll
          for (int j = 0; j < kCGroup / 2; ++j) {
            const int col = col0 / 2 + g + j;
            if (col < ep.n) {
              const float ar = sum[2 * (g + j)], ai = sum[2 * (g + j) + 1];
              float2 v = make_float2(ep.alpha_re * ar - ep.alpha_im * ai, ep.alpha_re * ai + ep.alpha_im * ar);
              if (!beta0) {
                const float2 cv = cvs[j];
                if (beta1) { v.x += cv.x; v.y += cv.y; }
                else {
                  v.x += ep.beta_re * cv.x - ep.beta_im * cv.y;
                  v.y += ep.beta_re * cv.y + ep.beta_im * cv.x;
                }
              }
              crow[(size_t)col * ep.ldc] = v;
            }
          }
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::cluster_sync();  // no CTA leaves while its partner may still signal or read it
  tc::tc_fence_after();
  if (warp == 1) tc::tmem_dealloc_pair(tmem, 2 * kPairTile);
}

// Split-K combine: C = alpha * sum_p ws[p] + beta * C in a fixed part order.
__global__ void k_split_reduce(const float* __restrict__ ws, int splits, int ws_cols, EpiParams ep) {
  const size_t total = (size_t)ep.m * ep.n;
  const bool beta0 = ep.beta_re == 0.f && ep.beta_im == 0.f;
  const bool beta1 = ep.beta_re == 1.f && ep.beta_im == 0.f;
  const size_t part = (size_t)ws_cols * ep.m;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(t % ep.m), col = (int)(t / ep.m);
    if (!ep.complex_out) {
      float s = 0.f;
      for (int p = 0; p < splits; ++p) s += ws[p * part + (size_t)col * ep.m + row];
      float* cp = ep.C + row + (size_t)col * ep.ldc;
      const float v = ep.alpha_re * s;
      if (beta0) *cp = v;
      else if (beta1) *cp = *cp + v;
      else *cp = ep.beta_re * *cp + v;
    } else {
      float ar = 0.f, ai = 0.f;
      for (int p = 0; p < splits; ++p) {
        ar += ws[p * part + (size_t)(2 * col) * ep.m + row];
        ai += ws[p * part + (size_t)(2 * col + 1) * ep.m + row];
      }
      float2* cp = reinterpret_cast<float2*>(ep.C) + row + (size_t)col * ep.ldc;
      float2 v = make_float2(ep.alpha_re * ar - ep.alpha_im * ai, ep.alpha_re * ai + ep.alpha_im * ar);
      if (!beta0) {
        const float2 cv = *cp;
        if (beta1) { v.x += cv.x; v.y += cv.y; }
        else {
          v.x += ep.beta_re * cv.x - ep.beta_im * cv.y;
          v.y += ep.beta_re * cv.y + ep.beta_im * cv.x;
        }
      }
      *cp = v;
    }
  }
}

template <int NP, int BN>
size_t gemm_smem_bytes() {
  return (size_t)kStages * SplitPlan<NP>::kPieces * (kBM * kBK * 2 + BN * kBK * 2) + 1024;
}

// Runs the GEMM kernel over prepared pieces: A pieces [mr][kp], B pieces [nr][kp];
// with splits > 1, `ws` holds splits x nr x mr floats of partial sums.
template <int NP, int BN>
coral_status_t run_split_gemm(Handle* h, const __nv_bfloat16* ap, size_t a_piece, int mr,
                              const __nv_bfloat16* bp, size_t b_piece, int nr, int kd, size_t kp,
                              int splits, float* ws, const EpiParams& ep) {
  SplitMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  for (int p = 0; p < SplitPlan<NP>::kPieces; ++p) {
    if (!encode_kmajor_map(&maps.a[p], ap + p * a_piece, 2, (uint64_t)kd, (uint64_t)mr, kp * 2, kBK, kBM,
                           kSwizzle) ||
        !encode_kmajor_map(&maps.b[p], bp + p * b_piece, 2, (uint64_t)kd, (uint64_t)nr, kp * 2, kBK, BN,
                           kSwizzle))
      return CORAL_ERR_NOT_SUPPORTED;
  }
  const size_t smem = gemm_smem_bytes<NP, BN>();
  static uint64_t attr_devices = 0;  // bit d: attribute set on device d
  const uint64_t bit = h->device < 64 ? (1ull << h->device) : 0;
  if (!(attr_devices & bit) || !bit) {
    CORAL_CUDA(h, cudaFuncSetAttribute(k_gemm_split<NP, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    attr_devices |= bit;
  }
  const int m_tiles = (mr + kBM - 1) / kBM, n_tiles = (nr + BN - 1) / BN;
  const int items = m_tiles * n_tiles * splits;
  const int grid = items < h->sm_count ? items : h->sm_count;
  const uint64_t limit_ns = h->wait_limit * 32ull;  // default 2^26 * 32 ns ~ 2.1 s
  timed_begin(h);
  k_gemm_split<NP, BN><<<grid, kSplitThreads, smem, h->stream>>>(
      maps, kd, m_tiles, n_tiles, h->split_chunk_kb * kSlabsPer64, splits, ws, nr, ep, &h->words->status,
      limit_ns);
  coral_status_t s = launch_status(h);
  timed_end(h);
  if (s != CORAL_OK || splits == 1) return s;
  unsigned g = stream_grid((size_t)ep.m * ep.n, 256 * 4, h->sm_count, 8);
  k_split_reduce<<<g, 256, 0, h->stream>>>(ws, splits, nr, ep);
  return launch_status(h);
}

template <int NP>
size_t pair_smem_bytes() {
  return (size_t)PairRing<NP>::kStages * PairRing<NP>::kStageBytes + 1024;
}

// Clusters of two that can be resident at once (per device, queried once).
template <int NP>
int pair_cluster_capacity(Handle* h, size_t smem) {
  static int cap[64] = {0};
  const int d = h->device < 64 ? h->device : 0;
  if (cap[d] > 0) return cap[d];
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)h->sm_count, 1, 1);
  cfg.blockDim = dim3(kSplitThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_gemm_split_pair<NP>, &cfg) != cudaSuccess || n < 1) {
    cudaGetLastError();
    n = h->sm_count / 2;
  }
  cap[d] = n;
  return n;
}

// The pair kernel over prepared pieces (same operands and workspace as
// run_split_gemm); `group` M-tiles per raster group.
template <int NP>
coral_status_t run_split_gemm_pair(Handle* h, const __nv_bfloat16* ap, size_t a_piece, int mr,
                                   const __nv_bfloat16* bp, size_t b_piece, int nr, int kd, size_t kp,
                                   int splits, float* ws, const EpiParams& ep) {
  SplitMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  for (int p = 0; p < SplitPlan<NP>::kPieces; ++p) {
    if (!encode_kmajor_map(&maps.a[p], ap + p * a_piece, 2, (uint64_t)kd, (uint64_t)mr, kp * 2, kBK,
                           kPairHalf, kSwizzle) ||
        !encode_kmajor_map(&maps.b[p], bp + p * b_piece, 2, (uint64_t)kd, (uint64_t)nr, kp * 2, kBK,
                           kPairHalf, kSwizzle))
      return CORAL_ERR_NOT_SUPPORTED;
  }
  const size_t smem = pair_smem_bytes<NP>();
  static uint64_t attr_devices = 0;
  const uint64_t bit = h->device < 64 ? (1ull << h->device) : 0;
  if (!(attr_devices & bit) || !bit) {
    CORAL_CUDA(h, cudaFuncSetAttribute(k_gemm_split_pair<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    attr_devices |= bit;
  }
  const int m_tiles = (mr + kPairTile - 1) / kPairTile, n_tiles = (nr + kPairTile - 1) / kPairTile;
  const int items = m_tiles * n_tiles * splits;
  const int cap = pair_cluster_capacity<NP>(h, smem);
  const int clusters = items < cap ? items : cap;
  const int group = h->pair_group > 0 ? h->pair_group : 8;
  const uint64_t limit_ns = h->wait_limit * 32ull;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(2 * clusters), 1, 1);
  cfg.blockDim = dim3(kSplitThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  timed_begin(h);
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_gemm_split_pair<NP>, maps, kd, m_tiles, n_tiles, group,
                                     h->split_chunk_kb * kSlabsPer64, splits, ws, nr, ep,
                                     &h->words->status, limit_ns);
  count_launch();
  coral_status_t s = cuda_status(h, e != cudaSuccess ? e : cudaGetLastError());
  timed_end(h);
  if (s != CORAL_OK || splits == 1) return s;
  unsigned g = stream_grid((size_t)ep.m * ep.n, 256 * 4, h->sm_count, 8);
  k_split_reduce<<<g, 256, 0, h->stream>>>(ws, splits, nr, ep);
  return launch_status(h);
}

}  // namespace

// Tile width and split-K factor for a split-BF16 GEMM of op(A) (mr x kd)
// times B-rows (nr x kd): the handle's explicit choice, else its selector,
// else the default rule (full-width tiles; split K when the output tiles
// cannot fill the GPU and K is deep).
SplitConfig choose_split_config(Handle* h, const SplitShape& sh) {
  const int products = sh.products, mr = sh.mr, nr = sh.nr, kd = sh.kd;
  SplitConfig c{products == 3 ? 256 : 128, 1};
  const int nk = (kd + 63) / 64;   // 64-deep K units (independent of the kernel's slab depth)
  if (h->cfg_bn > 0 || h->cfg_splits > 0 || h->cfg_bm > 0) {
    if (h->cfg_bn > 0) c.bn = h->cfg_bn;
    if (h->cfg_splits > 0) c.splits = h->cfg_splits;
    if (h->cfg_bm == 256) {
      c.pair = 1;
      c.bn = 256;
    }
  } else if (h->selector && select_split_config(h, sh, &c)) {
    // selector decided
  } else {
    const int tiles = ((mr + kBM - 1) / kBM) * ((nr + c.bn - 1) / c.bn);
    const int pair_tiles = ((mr + kPairTile - 1) / kPairTile) * ((nr + kPairTile - 1) / kPairTile);
    if (pair_tiles >= h->sm_count) {
      // At least two waves of 256 x 256 tiles over the resident CTA pairs:
      // the pair tiles read half as much of B per flop from shared memory.
      c.pair = 1;
      c.bn = 256;
    } else if (tiles * 2 <= h->sm_count && nk >= 16) {
      int sp = h->sm_count / tiles;
      sp = sp > 16 ? 16 : sp;
      sp = sp > nk ? nk : sp;
      int p2 = 1;  // largest power of two <= sp (the tuned candidate set)
      while (p2 * 2 <= sp) p2 *= 2;
      c.splits = p2;
    }
  }
  if (products == 6 && !c.pair) c.bn = 128;
  if (c.bn != 128 && c.bn != 256) c.bn = 256;
  if (c.splits > nk) c.splits = nk > 0 ? nk : 1;
  if (c.splits < 1) c.splits = 1;
  return c;
}

namespace {

template <int NP>
coral_status_t dispatch_split_gemm(Handle* h, const __nv_bfloat16* ap, size_t a_piece, int mr,
                                   const __nv_bfloat16* bp, size_t b_piece, int nr, int kd,
                                   size_t kp, const SplitConfig& c, float* ws, const EpiParams& ep) {
  if (c.pair)
    return run_split_gemm_pair<NP>(h, ap, a_piece, mr, bp, b_piece, nr, kd, kp, c.splits, ws, ep);
  if (NP == 3 && c.bn == 256)
    return run_split_gemm<NP, 256>(h, ap, a_piece, mr, bp, b_piece, nr, kd, kp, c.splits, ws, ep);
  return run_split_gemm<NP, 128>(h, ap, a_piece, mr, bp, b_piece, nr, kd, kp, c.splits, ws, ep);
}

template <int NP>
coral_status_t sgemm_split_impl(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                float alpha, const float* A, size_t lda, const float* B, size_t ldb,
                                float beta, float* C, size_t ldc) {
  constexpr int NPC = SplitPlan<NP>::kPieces;
  const size_t kp = (k + 7) & ~size_t(7);
  const size_t a_piece = m * kp, b_piece = n * kp;
  const size_t a_bytes = (NPC * a_piece * 2 + 255) & ~size_t(255);
  const size_t b_bytes = (NPC * b_piece * 2 + 255) & ~size_t(255);
  const SplitConfig cfg = choose_split_config(h, SplitShape{(int)m, (int)n, (int)k, NP, op_a, op_b, 0, 1});
  const size_t ws_bytes = cfg.splits > 1 ? (size_t)cfg.splits * m * n * sizeof(float) : 0;
  char* sc = static_cast<char*>(scratch(h, a_bytes + b_bytes + ws_bytes));
  if (!sc) return CORAL_ERR_ALLOC;
  __nv_bfloat16* ap = reinterpret_cast<__nv_bfloat16*>(sc);
  __nv_bfloat16* bp = reinterpret_cast<__nv_bfloat16*>(sc + a_bytes);
  // op(A) rows are i: storage K-major iff op_a is (conjugate) transpose.
  launch_split_real<NPC>(h->stream, A, lda, (int)m, (int)k, op_a != CORAL_NO_TRANSPOSE, ap, kp, a_piece);
  coral_status_t s = launch_status(h);
  if (s != CORAL_OK) return s;
  // op(B)^T rows are j: storage K-major iff op_b is NoTranspose.
  launch_split_real<NPC>(h->stream, B, ldb, (int)n, (int)k, op_b == CORAL_NO_TRANSPOSE, bp, kp, b_piece);
  s = launch_status(h);
  if (s != CORAL_OK) return s;
  EpiParams ep{C, ldc, (int)m, (int)n, alpha, 0.f, beta, 0.f, 0};
  float* ws = reinterpret_cast<float*>(sc + a_bytes + b_bytes);
  return dispatch_split_gemm<NP>(h, ap, a_piece, (int)m, bp, b_piece, (int)n, (int)k, kp, cfg, ws, ep);
}

// 3M mapping: three real split GEMMs of m x n x k (Re A Re B, Im A Im B and
// (Re A + Im A)(Re B + Im B)) into fp32 workspace, then k_combine_3m.  Three
// quarters of the 4M mapping's tensor work; the imaginary part is formed as
// T3 - T1 - T2, so its error is bounded by (|Re A| + |Im A|)(|Re B| + |Im B|)
// rather than |A| |B| per term.
template <int NP>
coral_status_t cgemm_split_3m(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                              float2 alpha, const float2* A, size_t lda, const float2* B, size_t ldb,
                              float2 beta, float2* C, size_t ldc) {
  constexpr int NPC = SplitPlan<NP>::kPieces;
  const size_t kp = (k + 7) & ~size_t(7);
  const size_t a_piece = m * kp, b_piece = n * kp;
  const size_t a_part = NPC * a_piece, b_part = NPC * b_piece;
  const size_t a_bytes = (3 * a_part * 2 + 255) & ~size_t(255);
  const size_t b_bytes = (3 * b_part * 2 + 255) & ~size_t(255);
  const size_t t_bytes = (m * n * sizeof(float) + 255) & ~size_t(255);
  const SplitConfig cfg = choose_split_config(h, SplitShape{(int)m, (int)n, (int)k, NP, op_a, op_b, 1, 1});
  const size_t ws_bytes = cfg.splits > 1 ? (size_t)cfg.splits * m * n * sizeof(float) : 0;
  char* sc = static_cast<char*>(scratch(h, a_bytes + b_bytes + 3 * t_bytes + ws_bytes));
  if (!sc) return CORAL_ERR_ALLOC;
  __nv_bfloat16* ap = reinterpret_cast<__nv_bfloat16*>(sc);
  __nv_bfloat16* bp = reinterpret_cast<__nv_bfloat16*>(sc + a_bytes);
  float* t[3];
  for (int i = 0; i < 3; ++i) t[i] = reinterpret_cast<float*>(sc + a_bytes + b_bytes + i * t_bytes);
  float* ws = reinterpret_cast<float*>(sc + a_bytes + b_bytes + 3 * t_bytes);
  const bool ca = op_a == CORAL_CONJ_TRANSPOSE, cbj = op_b == CORAL_CONJ_TRANSPOSE;
  dim3 ga((unsigned)((kp + 31) / 32), (unsigned)((m + 31) / 32));
  if (op_a == CORAL_NO_TRANSPOSE)
    k_split_cplx3<NPC, false><<<ga, 256, 0, h->stream>>>(A, lda, (int)m, (int)k, ca, ap, kp, a_piece, a_part);
  else
    k_split_cplx3<NPC, true><<<ga, 256, 0, h->stream>>>(A, lda, (int)m, (int)k, ca, ap, kp, a_piece, a_part);
  coral_status_t s = launch_status(h);
  if (s != CORAL_OK) return s;
  // op(B)^T rows are j: storage K-major iff op_b is NoTranspose
  dim3 gb((unsigned)((kp + 31) / 32), (unsigned)((n + 31) / 32));
  if (op_b == CORAL_NO_TRANSPOSE)
    k_split_cplx3<NPC, true><<<gb, 256, 0, h->stream>>>(B, ldb, (int)n, (int)k, cbj, bp, kp, b_piece, b_part);
  else
    k_split_cplx3<NPC, false><<<gb, 256, 0, h->stream>>>(B, ldb, (int)n, (int)k, cbj, bp, kp, b_piece, b_part);
  if ((s = launch_status(h)) != CORAL_OK) return s;
  for (int part = 0; part < 3; ++part) {
    EpiParams ep{t[part], m, (int)m, (int)n, 1.f, 0.f, 0.f, 0.f, 0};
    s = dispatch_split_gemm<NP>(h, ap + part * a_part, a_piece, (int)m, bp + part * b_part, b_piece, (int)n,
                                (int)k, kp, cfg, ws, ep);
    if (s != CORAL_OK) return s;
  }
  unsigned g = stream_grid(m * n, 256 * 4, h->sm_count, 8);
  k_combine_3m<<<g, 256, 0, h->stream>>>(t[0], t[1], t[2], (int)m, (int)n, alpha, beta, C, ldc);
  return launch_status(h);
}

template <int NP>
coral_status_t cgemm_split_impl(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                float2 alpha, const float2* A, size_t lda, const float2* B,
                                size_t ldb, float2 beta, float2* C, size_t ldc) {
  if (h->complex_mapping == CORAL_COMPLEX_3M)
    return cgemm_split_3m<NP>(h, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  constexpr int NPC = SplitPlan<NP>::kPieces;
  const size_t k2 = 2 * k;
  const size_t kp = (k2 + 7) & ~size_t(7);
  const size_t a_piece = m * kp, b_piece = 2 * n * kp;
  const size_t a_bytes = (NPC * a_piece * 2 + 255) & ~size_t(255);
  const size_t b_bytes = (NPC * b_piece * 2 + 255) & ~size_t(255);
  const SplitConfig cfg =
      choose_split_config(h, SplitShape{(int)m, (int)(2 * n), (int)k2, NP, op_a, op_b, 1, 1});
  const size_t ws_bytes = cfg.splits > 1 ? (size_t)cfg.splits * m * 2 * n * sizeof(float) : 0;
  char* sc = static_cast<char*>(scratch(h, a_bytes + b_bytes + ws_bytes));
  if (!sc) return CORAL_ERR_ALLOC;
  __nv_bfloat16* ap = reinterpret_cast<__nv_bfloat16*>(sc);
  __nv_bfloat16* bp = reinterpret_cast<__nv_bfloat16*>(sc + a_bytes);
  if (kp != k2) {  // zero the row tails so every byte TMA may read is defined
    CORAL_CUDA(h, cudaMemsetAsync(sc, 0, a_bytes + b_bytes, h->stream));
  }
  dim3 ga((unsigned)((k + 31) / 32), (unsigned)((m + 31) / 32));
  const bool ca = op_a == CORAL_CONJ_TRANSPOSE, cbj = op_b == CORAL_CONJ_TRANSPOSE;
  if (op_a == CORAL_NO_TRANSPOSE)
    k_split_cplx<NPC, false, false><<<ga, 256, 0, h->stream>>>(A, lda, (int)m, (int)k, ca, ap, kp, a_piece);
  else
    k_split_cplx<NPC, true, false><<<ga, 256, 0, h->stream>>>(A, lda, (int)m, (int)k, ca, ap, kp, a_piece);
  coral_status_t s = launch_status(h);
  if (s != CORAL_OK) return s;
  dim3 gb((unsigned)((k + 31) / 32), (unsigned)((n + 31) / 32));
  if (op_b == CORAL_NO_TRANSPOSE)
    k_split_cplx<NPC, true, true><<<gb, 256, 0, h->stream>>>(B, ldb, (int)n, (int)k, cbj, bp, kp, b_piece);
  else
    k_split_cplx<NPC, false, true><<<gb, 256, 0, h->stream>>>(B, ldb, (int)n, (int)k, cbj, bp, kp, b_piece);
  s = launch_status(h);
  if (s != CORAL_OK) return s;
  EpiParams ep{reinterpret_cast<float*>(C), ldc, (int)m, (int)n, alpha.x, alpha.y, beta.x, beta.y, 1};
  float* ws = reinterpret_cast<float*>(sc + a_bytes + b_bytes);
  return dispatch_split_gemm<NP>(h, ap, a_piece, (int)m, bp, b_piece, (int)(2 * n), (int)k2, kp, cfg,
                                 ws, ep);
}

}  // namespace

coral_status_t enqueue_sgemm_split(Handle* h, int terms, int op_a, int op_b, size_t m, size_t n,
                                   size_t k, float alpha, const float* A, size_t lda,
                                   const float* B, size_t ldb, float beta, float* C, size_t ldc) {
  if (m > (size_t)INT32_MAX / 2 || n > (size_t)INT32_MAX / 2 || k > (size_t)INT32_MAX / 2)
    return CORAL_ERR_NOT_SUPPORTED;
  return terms == 6 ? sgemm_split_impl<6>(h, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
                    : sgemm_split_impl<3>(h, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

coral_status_t enqueue_cgemm_split(Handle* h, int terms, int op_a, int op_b, size_t m, size_t n,
                                   size_t k, float2 alpha, const float2* A, size_t lda,
                                   const float2* B, size_t ldb, float2 beta, float2* C, size_t ldc) {
  if (m > (size_t)INT32_MAX / 4 || n > (size_t)INT32_MAX / 4 || k > (size_t)INT32_MAX / 4)
    return CORAL_ERR_NOT_SUPPORTED;
  return terms == 6 ? cgemm_split_impl<6>(h, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc)
                    : cgemm_split_impl<3>(h, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

}  // namespace coral

// ---- allocation-free split-BF16x3 SGEMM ----------------------------------------
// Some callers cannot let a library call cudaMalloc: a serving process that
// reserves nearly all of HBM at start-up and sub-allocates it itself, a
// latency-critical loop that cannot afford the implicit synchronisation of
// cudaMalloc/cudaFree, or a deployment that forbids device allocation after
// initialisation.  coral_sgemm_bf16x3_noalloc serves them: the bf16 pieces of
// op(A) and op(B) go into this fixed array instead of handle scratch.
//
// The array is a file-scope __device__ variable, so every GPU that loads this
// library holds it until the process exits.  Host code must not use its name
// as a device address (on the host it is only a stand-in); the address comes
// from cudaGetSymbolAddress, once per device, in noalloc_setup().
namespace coral {
namespace {
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB per device
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;
  unsigned* status = nullptr;
  int sm_count = 0;
};
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

__global__ void k_noalloc_scale(int m, int n, float beta, float* __restrict__ C, size_t ldc) {
  size_t total = (size_t)m * n;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    float* cp = C + t % m + (t / m) * ldc;
    *cp = beta == 0.f ? 0.f : beta * *cp;
  }
}
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static __device__ __align__(256) unsigned g_noalloc_status;

// One-time set-up for the current device: device addresses of the fixed
// scratch and status word, the SM count, and the kernel's shared-memory limit.
static coral_status_t noalloc_setup(NoAllocDevice** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
    return CORAL_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc_dev[dev];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(nullptr, e);
    d.scratch = static_cast<unsigned char*>(p);
    e = cudaGetSymbolAddress(&p, g_noalloc_status);
    if (e != cudaSuccess) return cuda_status(nullptr, e);
    d.status = static_cast<unsigned*>(p);
    e = cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_status(nullptr, e);
    e = cudaFuncSetAttribute(k_gemm_split<3, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)gemm_smem_bytes<3, 256>());
    if (e != cudaSuccess) return cuda_status(nullptr, e);
    d.ready = true;
  }
  *out = &d;
  return CORAL_OK;
}

}  // namespace coral

extern "C" coral_status_t coral_sgemm_bf16x3_noalloc(void* stream, int op_a, int op_b, size_t m,
                                                     size_t n, size_t k, float alpha,
                                                     const float* a, size_t lda, const float* b,
                                                     size_t ldb, float beta, float* c, size_t ldc) {
  using namespace coral;
  if (gemm_bad_arg(op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc, false) > 0)
    return CORAL_ERR_INVALID_ARG;
  if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX || k > (size_t)INT32_MAX)
    return CORAL_ERR_NOT_SUPPORTED;
  if (m == 0 || n == 0) return CORAL_OK;
  NoAllocDevice* d = nullptr;
  coral_status_t s = noalloc_setup(&d);
  if (s != CORAL_OK) return s;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (alpha == 0.0f || k == 0) {  // scale-only, no scratch used (sgemm_nn.rs:29-45)
    if (beta == 1.0f) return CORAL_OK;
    unsigned g = stream_grid(m * n, 256 * 4, d->sm_count, 8);
    k_noalloc_scale<<<g, 256, 0, st>>>((int)m, (int)n, beta, c, ldc);
    return launch_status(nullptr);
  }
  // The two pieces of each operand need 4 * (m + n) * kp bytes plus the
  // 256-byte rounding of A's part.  Compared by division: with m, n, k up to
  // 2^31 the product itself could wrap around 64 bits.
  const size_t kp = (k + 7) & ~size_t(7);
  if (m + n > ((kNoAllocScratchBytes - 256) / 4) / kp)
    return CORAL_ERR_NOT_SUPPORTED;  // the pieces do not fit the fixed scratch
  const size_t a_piece = m * kp, b_piece = n * kp;
  const size_t a_bytes = (2 * a_piece * 2 + 255) & ~size_t(255);
  // The status word is not cleared here: it collects the give-ups of every
  // call until coral_sgemm_bf16x3_noalloc_status reads and clears it.
  __nv_bfloat16* ap = reinterpret_cast<__nv_bfloat16*>(d->scratch);
  __nv_bfloat16* bp = reinterpret_cast<__nv_bfloat16*>(d->scratch + a_bytes);
  // Every piece element the GEMM reads is rewritten here, so stale contents
  // of the shared array from an earlier call never leak into this one.
  launch_split_real<2>(st, a, lda, (int)m, (int)k, op_a != CORAL_NO_TRANSPOSE, ap, kp, a_piece);
  if ((s = launch_status(nullptr)) != CORAL_OK) return s;
  launch_split_real<2>(st, b, ldb, (int)n, (int)k, op_b == CORAL_NO_TRANSPOSE, bp, kp, b_piece);
  if ((s = launch_status(nullptr)) != CORAL_OK) return s;
  SplitMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  for (int p = 0; p < 2; ++p) {
    if (!encode_kmajor_map(&maps.a[p], ap + p * a_piece, 2, k, m, kp * 2, kBK, kBM, kSwizzle) ||
        !encode_kmajor_map(&maps.b[p], bp + p * b_piece, 2, k, n, kp * 2, kBK, 256, kSwizzle))
      return CORAL_ERR_NOT_SUPPORTED;
  }
  const int m_tiles = (int)((m + kBM - 1) / kBM), n_tiles = (int)((n + 255) / 256);
  const int tiles = m_tiles * n_tiles;
  const int grid = tiles < d->sm_count ? tiles : d->sm_count;
  EpiParams ep{c, ldc, (int)m, (int)n, alpha, 0.f, beta, 0.f, 0};
  k_gemm_split<3, 256><<<grid, kSplitThreads, gemm_smem_bytes<3, 256>(), st>>>(
      maps, (int)k, m_tiles, n_tiles, 16 * kSlabsPer64, 1, nullptr, (int)n, ep, d->status,
      kDefaultWaitLimit * 32ull);
  return launch_status(nullptr);
}

// The GEMM's bounded waits report a give-up in the fixed status word of the
// device, not in a return value (the call returns before the kernel runs).
// This waits for `stream`, then reads and clears that word for the current
// device: CORAL_ERR_TIMEOUT means a C written since the last query may be
// incomplete.  No allocation: the word is copied into a host variable.
extern "C" coral_status_t coral_sgemm_bf16x3_noalloc_status(void* stream) {
  using namespace coral;
  NoAllocDevice* d = nullptr;
  coral_status_t s = noalloc_setup(&d);
  if (s != CORAL_OK) return s;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  unsigned word = 0;
  cudaError_t e = cudaMemcpyAsync(&word, d->status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(nullptr, e);
  if (word) {
    e = cudaMemsetAsync(d->status, 0, sizeof(unsigned), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(nullptr, e);
    if (word & kStatusTimeout) return CORAL_ERR_TIMEOUT;
  }
  return CORAL_OK;
}
