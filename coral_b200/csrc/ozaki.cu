// Ozaki-scheme DGEMM / ZGEMM on the INT8 tensor pipe (tcgen05 kind::i8).
//
// No reference counterpart: an FP64 GEMM (dgemm.rs:107 semantics, zgemm.rs:123
// through the 4M mapping) emulated with exact integer products.
//
//   1. Scaling: each row i of op(A) gets e_i with max_l |a_il| * 2^-e_i < 1, each
//      column j of op(B) gets f_j likewise (frexp exponents, reduced with
//      atomicMax -- exact and order independent).
//   2. Slicing: v = a * 2^-e_i (exact) is cut into S signed 7-bit slices,
//      v = sum_p A_p 2^-7p + r with A_p = trunc(2^7 r_{p-1}) in [-127, 127]
//      and |r| < 2^-7S: every step is exact in FP64.  Slices are stored
//      K-major, int8, [S][rows][kp] (kp = k rounded up to 16 bytes).
//   3. GEMM: for a 128 x 64 tile of C, the products A_p B_q^T with p + q <= S+1
//      (S(S+1)/2 of them; the rest are below 2^-7(S+1)) are accumulated in
//      INT32 in TMEM, one accumulator per anti-diagonal d = p + q, exactly as
//      long as (#products on d) * 127^2 * kchunk < 2^31 -- K is cut into
//      chunks that satisfy it.  After each chunk the epilogue warps convert
//      each diagonal accumulator to FP64 and add 2^-7d times it to registers
//      (exact scaling, one FP64 rounding per add).
//   4. Epilogue: C = alpha * 2^(e_i + f_j) * acc + beta * C in FP64 (beta == 0
//      does not read C, as f64_edge / f32_edge.rs:37-58 do).
// Complex operands (ZGEMM) use the same 4M folding as the split-BF16 CGEMM:
// A'' = [Re A | Im A], B'' rows (2j, 2j+1) = ([Re B_j | -Im B_j], [Im B_j | Re B_j]);
// or, with the handle's complex mapping set to 3M, three real Ozaki GEMMs
// combined as Re = T1 - T2, Im = T3 - T1 - T2 (zgemm_ozaki_3m).
//
// Pipeline: warp 0 lane 0 = TMA producer (2 stages of S slices of A and B,
// 64-byte K slabs, 64-byte swizzle); warp 1 lane 0 = MMA issuer (kind::i8,
// M=128, N=64, K=32 per instruction); warps 2-9 = epilogue.  All waits are
// bounded and report through the handle's status word.
#include "common.cuh"
#include "tc_common.cuh"

#include <climits>

namespace coral {
namespace {

constexpr int kOzBM = 128, kOzBN = 64, kOzBK = 64;  // BK in int8 elements (64 bytes)
constexpr int kOzStages = 2;
constexpr int kOzEpiWarps = 8;
constexpr int kOzThreads = 64 + 32 * kOzEpiWarps;

// ---- 1. exponents ---------------------------------------------------------------
// e[r] = max over l of the exponent of |op(X)(r, l)| (frexp: |v| 2^-e < 1),
// combined across column chunks with atomicMax, which is exact in any order.
// Complex: magnitude max(|re|, |im|) covers every real entry the 4M folding
// makes. Column-major rows (element (r, l) at X[r + l ld]): a thread owns a
// row and streams kExpChunkN columns with 8 loads in flight, so a warp reads
// 32 consecutive elements per column. K-major rows (element (r, l) at
// X[l + r ld]): a warp owns a row and streams kExpChunkK contiguous columns.
constexpr int kExpChunkN = 64, kExpChunkK = 256;

template <typename T>
__device__ __forceinline__ double mag(const T& a) {
  if constexpr (sizeof(T) == 16)
    return fmax(fabs(reinterpret_cast<const double2&>(a).x), fabs(reinterpret_cast<const double2&>(a).y));
  else
    return fabs(reinterpret_cast<const double&>(a));
}

template <typename T, bool kKMajorSrc>
__global__ void __launch_bounds__(256)
k_row_exponent(const T* __restrict__ X, size_t ld, int R, int Kd, int* __restrict__ e) {
  double m = 0.0;
  int r;
  if constexpr (!kKMajorSrc) {
    r = blockIdx.y * 256 + threadIdx.x;
    if (r >= R) return;
    const int l0 = blockIdx.x * kExpChunkN, l1 = min(Kd, l0 + kExpChunkN);
    const T* p = X + r;
    int l = l0;
    for (; l + 8 <= l1; l += 8) {
      T a[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) a[u] = __ldg(p + (size_t)(l + u) * ld);
#pragma unroll
      for (int u = 0; u < 8; ++u) m = fmax(m, mag(a[u]));
    }
    for (; l < l1; ++l) m = fmax(m, mag(__ldg(p + (size_t)l * ld)));
  } else {
    const int lane = threadIdx.x & 31;
    r = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (r >= R) return;
    const int l0 = blockIdx.x * kExpChunkK;
    const T* p = X + (size_t)r * ld;
    T a[kExpChunkK / 32];
#pragma unroll
    for (int u = 0; u < kExpChunkK / 32; ++u) {
      const int l = l0 + lane + 32 * u;
      a[u] = l < Kd ? __ldg(p + l) : T{};
    }
#pragma unroll
    for (int u = 0; u < kExpChunkK / 32; ++u) m = fmax(m, mag(a[u]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane != 0) return;
  }
  if (m > 0.0) {
    int ex;
    frexp(m, &ex);  // m = f 2^ex, f in [0.5, 1) -> m 2^-ex < 1
    atomicMax(e + r, ex);
  }
}

// Launches k_row_exponent over R rows of Kd columns (e must hold INT_MIN-like
// starting values).
template <typename T>
coral_status_t launch_row_exponent(Handle* h, const T* X, size_t ld, int R, int Kd, bool kmajor, int* e) {
  if (kmajor) {
    const dim3 g((unsigned)((Kd + kExpChunkK - 1) / kExpChunkK), (unsigned)((R + 7) / 8));
    if (g.y > 65535) return CORAL_ERR_NOT_SUPPORTED;
    k_row_exponent<T, true><<<g, 256, 0, h->stream>>>(X, ld, R, Kd, e);
  } else {
    const dim3 g((unsigned)((Kd + kExpChunkN - 1) / kExpChunkN), (unsigned)((R + 255) / 256));
    if (g.y > 65535) return CORAL_ERR_NOT_SUPPORTED;
    k_row_exponent<T, false><<<g, 256, 0, h->stream>>>(X, ld, R, Kd, e);
  }
  return launch_status(h);
}

// ---- 2. slicing ----------------------------------------------------------------
template <int S>
__device__ __forceinline__ void slice_value(double a, int ex, int8_t (&s)[S]) {
  double r = ldexp(a, -ex);  // |r| < 1
#pragma unroll
  for (int p = 0; p < S; ++p) {
    r *= 128.0;
    const double t = trunc(r);
    s[p] = (int8_t)(int)t;
    r -= t;
  }
}

// Real: dst[p][row][l] for op(X) rows (K contiguous).
template <int S, bool kKMajorSrc>
__global__ void __launch_bounds__(256)
k_slice_real(const double* __restrict__ X, size_t ld, int R, int Kd, const int* __restrict__ e,
             int8_t* __restrict__ dst, size_t kp, size_t piece) {
  __shared__ double tile[32][33];
  const int r0 = blockIdx.y * 32, l0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (kKMajorSrc) {
      int r = r0 + ty + 8 * q, l = l0 + tx;
      tile[ty + 8 * q][tx] = (r < R && l < Kd) ? __ldg(X + l + (size_t)r * ld) : 0.0;
    } else {
      int l = l0 + ty + 8 * q, r = r0 + tx;
      tile[tx][ty + 8 * q] = (r < R && l < Kd) ? __ldg(X + r + (size_t)l * ld) : 0.0;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int r = r0 + ty + 8 * q, l = l0 + tx;
    if (r < R && l < (int)kp) {
      int8_t s[S];
      slice_value<S>(tile[ty + 8 * q][tx], e[r], s);
      const size_t o = (size_t)r * kp + l;
#pragma unroll
      for (int p = 0; p < S; ++p) dst[p * piece + o] = s[p];
    }
  }
}

// Complex, 4M layout (see k_split_cplx in gemm_split.cu): A rows [Re | Im];
// B rows 2r = [Re | -Im], 2r+1 = [Im | Re].  Exponent per source row r.
template <int S, bool kKMajorSrc, bool kIsB>
__global__ void __launch_bounds__(256)
k_slice_cplx(const double2* __restrict__ X, size_t ld, int R, int Kd, bool conj,
             const int* __restrict__ e, int8_t* __restrict__ dst, size_t kp, size_t piece) {
  __shared__ double2 tile[32][33];
  const int r0 = blockIdx.y * 32, l0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (kKMajorSrc) {
      int r = r0 + ty + 8 * q, l = l0 + tx;
      tile[ty + 8 * q][tx] = (r < R && l < Kd) ? __ldg(X + l + (size_t)r * ld) : make_double2(0.0, 0.0);
    } else {
      int l = l0 + ty + 8 * q, r = r0 + tx;
      tile[tx][ty + 8 * q] = (r < R && l < Kd) ? __ldg(X + r + (size_t)l * ld) : make_double2(0.0, 0.0);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int r = r0 + ty + 8 * q, l = l0 + tx;
    if (r >= R || l >= Kd) continue;
    double2 v = tile[ty + 8 * q][tx];
    if (conj) v.y = -v.y;
    int8_t sr[S], si[S], sn[S];
    slice_value<S>(v.x, e[r], sr);
    slice_value<S>(v.y, e[r], si);
#pragma unroll
    for (int p = 0; p < S; ++p) sn[p] = (int8_t)(-si[p]);
    if (!kIsB) {
      const size_t o = (size_t)r * kp;
#pragma unroll
      for (int p = 0; p < S; ++p) {
        dst[p * piece + o + l] = sr[p];
        dst[p * piece + o + Kd + l] = si[p];
      }
    } else {
      const size_t o0 = (size_t)(2 * r) * kp, o1 = o0 + kp;
#pragma unroll
      for (int p = 0; p < S; ++p) {
        dst[p * piece + o0 + l] = sr[p];
        dst[p * piece + o0 + Kd + l] = sn[p];
        dst[p * piece + o1 + l] = si[p];
        dst[p * piece + o1 + Kd + l] = sr[p];
      }
    }
  }
}

// ---- 3./4. integer GEMM and FP64 recombination -----------------------------------
struct OzMaps {
  CUtensorMap a[8];
  CUtensorMap b[8];
};

struct OzEpi {
  double* C;
  size_t ldc;
  int m, n;               // logical C (complex: n complex columns)
  const int* ea;          // row exponents of op(A) (length m)
  const int* eb;          // row exponents of B-rows (length n, or 2n complex)
  double alpha_re, alpha_im, beta_re, beta_im;
  int complex_out;
};

__device__ __forceinline__ void oz_tile_coords(int tile, int m_tiles, int n_tiles, int& mt, int& nt) {
  const int group = 16;
  const int per_group = group * n_tiles;
  const int g = tile / per_group;
  const int gm0 = g * group;
  const int gsz = min(group, m_tiles - gm0);
  const int within = tile - g * per_group;
  mt = gm0 + within % gsz;
  nt = within / gsz;
}

template <int S>
__global__ void __launch_bounds__(kOzThreads, 1)
k_gemm_ozaki(const __grid_constant__ OzMaps maps, int kdim, int m_tiles, int n_tiles,
             int chunk_kb, OzEpi ep, unsigned* status, uint64_t limit_ns) {
  constexpr uint32_t kATile = kOzBM * kOzBK;  // bytes
  constexpr uint32_t kBTile = kOzBN * kOzBK;
  constexpr uint32_t kStageBytes = S * (kATile + kBTile);
  constexpr uint32_t kIdesc = tc::idesc_s8_s32(kOzBM, kOzBN);
  constexpr int kCols = kOzBN / 2;  // columns per epilogue thread

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = tc::align1024_shared(smem_raw);
  __shared__ __align__(8) uint64_t full_bar[kOzStages], empty_bar[kOzStages];
  __shared__ __align__(8) uint64_t acc_full, acc_empty;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nk = (kdim + kOzBK - 1) / kOzBK;
  const int chunks = (nk + chunk_kb - 1) / chunk_kb;
  const int total_tiles = m_tiles * n_tiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kOzStages; ++s) {
      tc::mbar_init(&full_bar[s], 1);
      tc::mbar_init(&empty_bar[s], 1);
    }
    tc::mbar_init(&acc_full, 1);
    tc::mbar_init(&acc_empty, kOzEpiWarps);
    abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(&tmem_slot, 512);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int it = 0;
      for (int tile = blockIdx.x; tile < total_tiles && !abort_flag; tile += gridDim.x) {
        int mt, nt;
        oz_tile_coords(tile, m_tiles, n_tiles, mt, nt);
        for (int kb = 0; kb < nk; ++kb, ++it) {
          const int s = it % kOzStages;
          if (it >= kOzStages && !tc::mbar_wait(&empty_bar[s], ((it / kOzStages) - 1) & 1, limit_ns)) {
            atomicOr(status, kStatusTimeout);
            atomicExch(&abort_flag, 1);
            break;
          }
          if (*(volatile int*)&abort_flag) break;
          uint8_t* st = smem + (size_t)s * kStageBytes;
          tc::mbar_expect_tx(&full_bar[s], kStageBytes);
          for (int p = 0; p < S; ++p) {
            tc::tma_load_2d(st + p * kATile, &maps.a[p], &full_bar[s], kb * kOzBK, mt * kOzBM);
            tc::tma_load_2d(st + S * kATile + p * kBTile, &maps.b[p], &full_bar[s], kb * kOzBK, nt * kOzBN);
          }
        }
      }
      for (int j = (it > kOzStages ? it - kOzStages : 0); j < it; ++j)
        tc::mbar_wait(&full_bar[j % kOzStages], (j / kOzStages) & 1, limit_ns);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int it = 0, gc = 0;
      bool stop = false;
      for (int tile = blockIdx.x; tile < total_tiles && !stop; tile += gridDim.x) {
        for (int c = 0; c < chunks && !stop; ++c, ++gc) {
          // the epilogue must have drained the previous chunk
          if (gc >= 1 && !tc::mbar_wait(&acc_empty, (gc - 1) & 1, limit_ns)) {
            atomicOr(status, kStatusTimeout);
            atomicExch(&abort_flag, 1);
            stop = true;
            break;
          }
          tc::tc_fence_after();
          const int kb0 = c * chunk_kb, kb1 = min(nk, kb0 + chunk_kb);
          for (int kb = kb0; kb < kb1; ++kb, ++it) {
            const int s = it % kOzStages;
            if (!tc::mbar_wait(&full_bar[s], (it / kOzStages) & 1, limit_ns)) {
              atomicOr(status, kStatusTimeout);
              atomicExch(&abort_flag, 1);
              stop = true;
              break;
            }
            tc::tc_fence_after();
            const uint32_t sa = tc::smem_u32(smem + (size_t)s * kStageBytes);
            const uint32_t sb = sa + S * kATile;
#pragma unroll
            for (int kk = 0; kk < kOzBK / 32; ++kk) {
#pragma unroll
              for (int d = 2; d <= S + 1; ++d) {
                const uint32_t acc = tmem + (d - 2) * kOzBN;
#pragma unroll
                for (int p = 1; p <= S; ++p) {
                  const int q = d - p;
                  if (q < 1 || q > S) continue;
                  const uint64_t ad = tc::desc_k_sw64(sa + (p - 1) * kATile + kk * 32);
                  const uint64_t bd = tc::desc_k_sw64(sb + (q - 1) * kBTile + kk * 32);
                  const bool first = (kb == kb0) && kk == 0 && p == max(1, d - S);
                  tc::mma_i8(acc, ad, bd, kIdesc, first ? 0u : 1u);
                }
              }
            }
            tc::mma_commit(&empty_bar[s]);
          }
          tc::mma_commit(&acc_full);
        }
      }
    }
  } else {
    const int ew = warp - 2;
    const int quad = warp & 3;
    const int half = ew >> 2;
    const uint32_t lane_base = (uint32_t)(quad * 32) << 16;
    const bool beta0 = ep.beta_re == 0.0 && ep.beta_im == 0.0;
    const bool beta1 = ep.beta_re == 1.0 && ep.beta_im == 0.0;
    int gc = 0;
    bool stop = false;
    for (int tile = blockIdx.x; tile < total_tiles && !stop; tile += gridDim.x) {
      int mt, nt;
      oz_tile_coords(tile, m_tiles, n_tiles, mt, nt);
      double sum[kCols];
#pragma unroll
      for (int j = 0; j < kCols; ++j) sum[j] = 0.0;
      for (int c = 0; c < chunks; ++c, ++gc) {
        if (!tc::mbar_wait(&acc_full, gc & 1, limit_ns)) {
          atomicOr(status, kStatusTimeout);
          stop = true;
          break;
        }
        tc::tc_fence_after();
#pragma unroll 1
        for (int d = 2; d <= S + 1; ++d) {
          uint32_t r[32];
          tc::tmem_ld32(tmem + (d - 2) * kOzBN + half * kCols + lane_base, r);
          tc::tmem_wait_ld();
          const double sc = ldexp(1.0, -7 * d);
#pragma unroll
          for (int j = 0; j < kCols; ++j) sum[j] = fma((double)(int)r[j], sc, sum[j]);
        }
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&acc_empty);
      }
      if (stop || *(volatile int*)&abort_flag) break;
      const int row = mt * kOzBM + quad * 32 + lane;
      if (row >= ep.m) continue;
      const int ei = max(ep.ea[row], -4000);  // all-zero rows keep the INT_MIN-like fill
      const int col0 = nt * kOzBN + half * kCols;
      // All C loads (and column exponents) of the tile row before any store:
      // a store followed by a load the compiler cannot prove disjoint would
      // cost a memory round trip per column.
      constexpr int G = 8;  // columns per group of loads
      if (!ep.complex_out) {
        double* crow = ep.C + row;
#pragma unroll
        for (int g = 0; g < kCols; g += G) {
          double cv[G];
          int ej[G];
#pragma unroll
          for (int j = 0; j < G; ++j) {
            const int col = col0 + g + j;
            cv[j] = (!beta0 && col < ep.n) ? crow[(size_t)col * ep.ldc] : 0.0;
            ej[j] = col < ep.n ? max(ep.eb[col], -4000) : 0;
          }
#pragma unroll
          for (int j = 0; j < G; ++j) {
            const int col = col0 + g + j;
            if (col >= ep.n) continue;
            const double v = ep.alpha_re * ldexp(sum[g + j], ei + ej[j]);
            crow[(size_t)col * ep.ldc] = beta0 ? v : beta1 ? cv[j] + v : ep.beta_re * cv[j] + v;
          }
        }
      } else {
        double2* crow = reinterpret_cast<double2*>(ep.C) + row;
#pragma unroll
        for (int g = 0; g < kCols / 2; g += G / 2) {
        double2 cvs[G / 2];
#pragma unroll
        for (int j0 = 0; j0 < G / 2; ++j0) {
          const int col = col0 / 2 + g + j0;
          cvs[j0] = (!beta0 && col < ep.n) ? crow[(size_t)col * ep.ldc] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int j0 = 0; j0 < G / 2; ++j0) {
          const int j = g + j0;
          const int col = col0 / 2 + j;
          if (col >= ep.n) continue;
          const double ar = ldexp(sum[2 * j], ei + max(ep.eb[2 * col], -4000));
          const double ai = ldexp(sum[2 * j + 1], ei + max(ep.eb[2 * col + 1], -4000));
          double2 v = make_double2(ep.alpha_re * ar - ep.alpha_im * ai, ep.alpha_re * ai + ep.alpha_im * ar);
          if (!beta0) {
            const double2 cv = cvs[j0];
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
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) tc::tmem_dealloc(tmem, 512);
}

template <int S>
size_t oz_smem_bytes() {
  return (size_t)kOzStages * S * (kOzBM * kOzBK + kOzBN * kOzBK) + 1024;
}

// K slabs per exact INT32 chunk: (products on the fullest diagonal) * 127^2 * k < 2^31.
template <int S>
int oz_chunk_slabs() {
  const long long kmax = (long long)INT32_MAX / (127LL * 127LL * S);
  return (int)(kmax / kOzBK);
}

template <int S>
coral_status_t run_ozaki_gemm(Handle* h, const int8_t* ap, size_t a_piece, int mr, const int8_t* bp,
                              size_t b_piece, int nr, int kd, size_t kp, const OzEpi& ep) {
  OzMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  for (int p = 0; p < S; ++p) {
    if (!encode_kmajor_map(&maps.a[p], ap + p * a_piece, 1, (uint64_t)kd, (uint64_t)mr, kp, kOzBK, kOzBM, 64) ||
        !encode_kmajor_map(&maps.b[p], bp + p * b_piece, 1, (uint64_t)kd, (uint64_t)nr, kp, kOzBK, kOzBN, 64))
      return CORAL_ERR_NOT_SUPPORTED;
  }
  const size_t smem = oz_smem_bytes<S>();
  static uint64_t attr_devices = 0;  // bit d: attribute set on device d
  const uint64_t bit = h->device < 64 ? (1ull << h->device) : 0;
  if (!(attr_devices & bit) || !bit) {
    CORAL_CUDA(h, cudaFuncSetAttribute(k_gemm_ozaki<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_devices |= bit;
  }
  const int m_tiles = (mr + kOzBM - 1) / kOzBM, n_tiles = (nr + kOzBN - 1) / kOzBN;
  const int tiles = m_tiles * n_tiles;
  const int grid = tiles < h->sm_count ? tiles : h->sm_count;
  timed_begin(h);
  k_gemm_ozaki<S><<<grid, kOzThreads, smem, h->stream>>>(maps, kd, m_tiles, n_tiles, oz_chunk_slabs<S>(),
                                                         ep, &h->words->status, h->wait_limit * 32ull);
  coral_status_t s = launch_status(h);
  timed_end(h);
  return s;
}

constexpr int kOzSlices = 7;

// Device bytes the real Ozaki GEMM needs for its slices and exponents.
size_t dgemm_ozaki_bytes(size_t m, size_t n, size_t k) {
  constexpr int S = kOzSlices;
  const size_t kp = (k + 15) & ~size_t(15);
  const size_t a_bytes = (S * m * kp + 1023) & ~size_t(1023);
  const size_t b_bytes = (S * n * kp + 1023) & ~size_t(1023);
  const size_t e_bytes = ((m + n) * sizeof(int) + 255) & ~size_t(255);
  return a_bytes + b_bytes + e_bytes;
}

// The real Ozaki GEMM with its slices and exponents in `sc`
// (dgemm_ozaki_bytes(m, n, k) bytes, 1024-byte aligned).
coral_status_t dgemm_ozaki_core(Handle* h, char* sc, int op_a, int op_b, size_t m, size_t n, size_t k,
                                double alpha, const double* A, size_t lda, const double* B,
                                size_t ldb, double beta, double* C, size_t ldc) {
  constexpr int S = kOzSlices;
  const size_t kp = (k + 15) & ~size_t(15);
  const size_t a_piece = m * kp, b_piece = n * kp;
  const size_t a_bytes = (S * a_piece + 1023) & ~size_t(1023);
  const size_t b_bytes = (S * b_piece + 1023) & ~size_t(1023);
  int8_t* ap = reinterpret_cast<int8_t*>(sc);
  int8_t* bp = reinterpret_cast<int8_t*>(sc + a_bytes);
  int* ea = reinterpret_cast<int*>(sc + a_bytes + b_bytes);
  int* eb = ea + m;
  CORAL_CUDA(h, cudaMemsetAsync(ea, 0x80, (m + n) * sizeof(int), h->stream));  // INT_MIN-ish
  const bool a_km = op_a != CORAL_NO_TRANSPOSE, b_km = op_b == CORAL_NO_TRANSPOSE;
  coral_status_t s = launch_row_exponent(h, A, lda, (int)m, (int)k, a_km, ea);
  if (s != CORAL_OK) return s;
  if ((s = launch_row_exponent(h, B, ldb, (int)n, (int)k, b_km, eb)) != CORAL_OK) return s;
  dim3 gsa((unsigned)((kp + 31) / 32), (unsigned)((m + 31) / 32));
  dim3 gsb((unsigned)((kp + 31) / 32), (unsigned)((n + 31) / 32));
  if (a_km) k_slice_real<S, true><<<gsa, 256, 0, h->stream>>>(A, lda, (int)m, (int)k, ea, ap, kp, a_piece);
  else k_slice_real<S, false><<<gsa, 256, 0, h->stream>>>(A, lda, (int)m, (int)k, ea, ap, kp, a_piece);
  if ((s = launch_status(h)) != CORAL_OK) return s;
  if (b_km) k_slice_real<S, true><<<gsb, 256, 0, h->stream>>>(B, ldb, (int)n, (int)k, eb, bp, kp, b_piece);
  else k_slice_real<S, false><<<gsb, 256, 0, h->stream>>>(B, ldb, (int)n, (int)k, eb, bp, kp, b_piece);
  if ((s = launch_status(h)) != CORAL_OK) return s;
  OzEpi ep{C, ldc, (int)m, (int)n, ea, eb, alpha, 0.0, beta, 0.0, 0};
  return run_ozaki_gemm<S>(h, ap, a_piece, (int)m, bp, b_piece, (int)n, (int)k, kp, ep);
}

coral_status_t dgemm_ozaki_impl(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                double alpha, const double* A, size_t lda, const double* B,
                                size_t ldb, double beta, double* C, size_t ldc) {
  char* sc = static_cast<char*>(scratch(h, dgemm_ozaki_bytes(m, n, k)));
  if (!sc) return CORAL_ERR_ALLOC;
  return dgemm_ozaki_core(h, sc, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

// 3M operands: the real matrices Re, Im and Re + Im of op(X) (conjugated when
// `conj`), R x L, column-major with leading dimension R.  Element (r, l) of
// op(X) is X[r + l * ld] (trans == false) or X[l + r * ld]; 32 x 32 tiles
// through shared memory so both the loads and the stores are coalesced.
__global__ void __launch_bounds__(256)
k_cplx_parts(const double2* __restrict__ X, size_t ld, bool trans, bool conj, int R, int L,
             double* __restrict__ re, double* __restrict__ im, double* __restrict__ sum) {
  __shared__ double2 tile[32][33];
  const int r0 = blockIdx.y * 32, l0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (trans) {  // contiguous along l
      const int r = r0 + ty + 8 * q, l = l0 + tx;
      if (r < R && l < L) tile[ty + 8 * q][tx] = X[l + (size_t)r * ld];
    } else {      // contiguous along r
      const int l = l0 + ty + 8 * q, r = r0 + tx;
      if (r < R && l < L) tile[tx][ty + 8 * q] = X[r + (size_t)l * ld];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int l = l0 + ty + 8 * q, r = r0 + tx;
    if (r < R && l < L) {
      double2 v = tile[tx][ty + 8 * q];
      if (conj) v.y = -v.y;
      const size_t o = r + (size_t)l * R;
      re[o] = v.x;
      im[o] = v.y;
      sum[o] = v.x + v.y;
    }
  }
}

// C = alpha (T1 - T2 + i (T3 - T1 - T2)) + beta C, T* m x n with ld m.
__global__ void k_combine_3m_z(const double* __restrict__ t1, const double* __restrict__ t2,
                               const double* __restrict__ t3, int m, int n, double2 alpha, double2 beta,
                               double2* __restrict__ C, size_t ldc) {
  const size_t total = (size_t)m * n;
  const bool beta0 = beta.x == 0.0 && beta.y == 0.0;
  const bool beta1 = beta.x == 1.0 && beta.y == 0.0;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const double a = t1[t], b = t2[t], c3 = t3[t];
    const double re = a - b, im = c3 - a - b;
    double2 v = make_double2(alpha.x * re - alpha.y * im, alpha.x * im + alpha.y * re);
    double2* cp = C + t % m + (t / m) * ldc;
    if (!beta0) {
      const double2 cv = *cp;
      if (beta1) { v.x += cv.x; v.y += cv.y; }
      else {
        v.x += beta.x * cv.x - beta.y * cv.y;
        v.y += beta.x * cv.y + beta.y * cv.x;
      }
    }
    *cp = v;
  }
}

// ZGEMM by the 3M mapping: three real Ozaki GEMMs of m x n x k (Re A Re B,
// Im A Im B, (Re A + Im A)(Re B + Im B)) into fp64 workspace, then the
// combine.  Three quarters of the 4M work; Im C = T3 - T1 - T2, whose error is
// bounded by (|Re A| + |Im A|)(|Re B| + |Im B|) instead of |A| |B| per term.
coral_status_t zgemm_ozaki_3m(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                              double2 alpha, const double2* A, size_t lda, const double2* B,
                              size_t ldb, double2 beta, double2* C, size_t ldc) {
  auto up = [](size_t b) { return (b + 1023) & ~size_t(1023); };
  const size_t pa = up(m * k * sizeof(double)), pb = up(k * n * sizeof(double));
  const size_t pt = up(m * n * sizeof(double));
  const size_t oz = dgemm_ozaki_bytes(m, n, k);
  char* sc = static_cast<char*>(scratch(h, 3 * pa + 3 * pb + 3 * pt + oz));
  if (!sc) return CORAL_ERR_ALLOC;
  double* ar[3];
  double* br[3];
  double* t[3];
  for (int i = 0; i < 3; ++i) {
    ar[i] = reinterpret_cast<double*>(sc + i * pa);
    br[i] = reinterpret_cast<double*>(sc + 3 * pa + i * pb);
    t[i] = reinterpret_cast<double*>(sc + 3 * pa + 3 * pb + i * pt);
  }
  char* ozs = sc + 3 * pa + 3 * pb + 3 * pt;
  // op(A): m x k; op(B): k x n
  const dim3 ga((unsigned)((k + 31) / 32), (unsigned)((m + 31) / 32));
  k_cplx_parts<<<ga, 256, 0, h->stream>>>(A, lda, op_a != CORAL_NO_TRANSPOSE, op_a == CORAL_CONJ_TRANSPOSE,
                                          (int)m, (int)k, ar[0], ar[1], ar[2]);
  coral_status_t s = launch_status(h);
  if (s != CORAL_OK) return s;
  const dim3 gb((unsigned)((n + 31) / 32), (unsigned)((k + 31) / 32));
  k_cplx_parts<<<gb, 256, 0, h->stream>>>(B, ldb, op_b != CORAL_NO_TRANSPOSE, op_b == CORAL_CONJ_TRANSPOSE,
                                          (int)k, (int)n, br[0], br[1], br[2]);
  if ((s = launch_status(h)) != CORAL_OK) return s;
  for (int i = 0; i < 3; ++i) {
    s = dgemm_ozaki_core(h, ozs, CORAL_NO_TRANSPOSE, CORAL_NO_TRANSPOSE, m, n, k, 1.0, ar[i], m, br[i], k,
                         0.0, t[i], m);
    if (s != CORAL_OK) return s;
  }
  const unsigned g = stream_grid(m * n, 256 * 4, h->sm_count, 8);
  k_combine_3m_z<<<g, 256, 0, h->stream>>>(t[0], t[1], t[2], (int)m, (int)n, alpha, beta, C, ldc);
  return launch_status(h);
}

coral_status_t zgemm_ozaki_impl(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                double2 alpha, const double2* A, size_t lda, const double2* B,
                                size_t ldb, double2 beta, double2* C, size_t ldc) {
  constexpr int S = kOzSlices;
  const size_t k2 = 2 * k;
  const size_t kp = (k2 + 15) & ~size_t(15);
  const size_t a_piece = m * kp, b_piece = 2 * n * kp;
  const size_t a_bytes = (S * a_piece + 1023) & ~size_t(1023);
  const size_t b_bytes = (S * b_piece + 1023) & ~size_t(1023);
  const size_t e_bytes = ((m + 2 * n + n) * sizeof(int) + 255) & ~size_t(255);
  char* sc = static_cast<char*>(scratch(h, a_bytes + b_bytes + e_bytes));
  if (!sc) return CORAL_ERR_ALLOC;
  int8_t* ap = reinterpret_cast<int8_t*>(sc);
  int8_t* bp = reinterpret_cast<int8_t*>(sc + a_bytes);
  int* ea = reinterpret_cast<int*>(sc + a_bytes + b_bytes);
  int* ebs = ea + m;          // per source column j of op(B) (length n)
  int* eb2 = ebs + n;         // per B'' row (length 2n)
  CORAL_CUDA(h, cudaMemsetAsync(ea, 0x80, (m + n) * sizeof(int), h->stream));
  const bool a_km = op_a != CORAL_NO_TRANSPOSE, b_km = op_b == CORAL_NO_TRANSPOSE;
  coral_status_t s = launch_row_exponent(h, A, lda, (int)m, (int)k, a_km, ea);
  if (s != CORAL_OK) return s;
  if ((s = launch_row_exponent(h, B, ldb, (int)n, (int)k, b_km, ebs)) != CORAL_OK) return s;
  // B'' rows 2j and 2j+1 share column j's exponent.
  CORAL_CUDA(h, cudaMemcpy2DAsync(eb2, 2 * sizeof(int), ebs, sizeof(int), sizeof(int), n,
                                  cudaMemcpyDeviceToDevice, h->stream));
  CORAL_CUDA(h, cudaMemcpy2DAsync(eb2 + 1, 2 * sizeof(int), ebs, sizeof(int), sizeof(int), n,
                                  cudaMemcpyDeviceToDevice, h->stream));
  if (kp != k2) CORAL_CUDA(h, cudaMemsetAsync(sc, 0, a_bytes + b_bytes, h->stream));
  const bool ca = op_a == CORAL_CONJ_TRANSPOSE, cbj = op_b == CORAL_CONJ_TRANSPOSE;
  const dim3 ga((unsigned)((k + 31) / 32), (unsigned)((m + 31) / 32));  // 32 x 32 slicing tiles
  const dim3 gb((unsigned)((k + 31) / 32), (unsigned)((n + 31) / 32));
  if (a_km) k_slice_cplx<S, true, false><<<ga, 256, 0, h->stream>>>(A, lda, (int)m, (int)k, ca, ea, ap, kp, a_piece);
  else k_slice_cplx<S, false, false><<<ga, 256, 0, h->stream>>>(A, lda, (int)m, (int)k, ca, ea, ap, kp, a_piece);
  if ((s = launch_status(h)) != CORAL_OK) return s;
  if (b_km) k_slice_cplx<S, true, true><<<gb, 256, 0, h->stream>>>(B, ldb, (int)n, (int)k, cbj, ebs, bp, kp, b_piece);
  else k_slice_cplx<S, false, true><<<gb, 256, 0, h->stream>>>(B, ldb, (int)n, (int)k, cbj, ebs, bp, kp, b_piece);
  if ((s = launch_status(h)) != CORAL_OK) return s;
  OzEpi ep{reinterpret_cast<double*>(C), ldc, (int)m, (int)n, ea, eb2,
           alpha.x, alpha.y, beta.x, beta.y, 1};
  return run_ozaki_gemm<S>(h, ap, a_piece, (int)m, bp, b_piece, (int)(2 * n), (int)k2, kp, ep);
}

}  // namespace

coral_status_t enqueue_dgemm_ozaki(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                   double alpha, const double* A, size_t lda, const double* B,
                                   size_t ldb, double beta, double* C, size_t ldc) {
  if (m > (size_t)INT32_MAX / 2 || n > (size_t)INT32_MAX / 2 || k > (size_t)INT32_MAX / 2)
    return CORAL_ERR_NOT_SUPPORTED;
  return dgemm_ozaki_impl(h, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

coral_status_t enqueue_zgemm_ozaki(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                   double2 alpha, const double2* A, size_t lda, const double2* B,
                                   size_t ldb, double2 beta, double2* C, size_t ldc) {
  if (m > (size_t)INT32_MAX / 4 || n > (size_t)INT32_MAX / 4 || k > (size_t)INT32_MAX / 4)
    return CORAL_ERR_NOT_SUPPORTED;
  if (h->complex_mapping == CORAL_COMPLEX_3M)
    return zgemm_ozaki_3m(h, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  return zgemm_ozaki_impl(h, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

}  // namespace coral
