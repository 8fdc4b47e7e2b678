// Native-precision SGEMM / DGEMM on the FMA pipes with TMA-staged operand
// tiles: C <- alpha * op(A) op(B) + beta * C, column-major.
//
// Replaces CORAL's packing and register-tile microkernels
// (coral-aarch64/src/level3/f32_packers.rs:113-170, microkernel/f32_mrxnr.rs:46-158,
// f64_packers.rs, microkernel/f64_mrxnr.rs): instead of packing panels on the
// host core, one producer warp streams the operand tiles of each K slab into a
// 4-stage shared-memory ring with cp.async.bulk.tensor (TMA), and eight
// consumer warps (16 x 16 threads, TM x TN outputs each) run the register
// outer products straight from shared memory.
//
// Tile layout follows the operand's storage, so the TMA box is a plain copy:
//   - stored contiguous along M (A with op N) or N (B with op T): [BK][E]
//     rows of E elements, no swizzle; a thread owns groups of V = 16 / sizeof(T)
//     consecutive rows and reads them with 16-byte shared loads;
//   - stored contiguous along K (A with op T, B with op N): [E][BK] rows of
//     128 bytes in the 128-byte swizzle (16-byte chunk q of row r at q ^ (r & 7));
//     a thread owns rows t, t + 16, ... and reads V consecutive K values of a
//     row with one 16-byte load, conflict-free across the 8 chunk positions.
// A slab is BK = 128 / sizeof(T) deep (32 floats, 16 doubles).  Rows and K past
// the matrix are zero-filled by TMA.  The epilogue follows f32_edge.rs:37-58
// (beta == 0 writes alpha * acc without reading C; beta == 1 accumulates).
// Every wait is bounded: a give-up sets the handle's status word.
#include "common.cuh"
#include "tc_common.cuh"

namespace coral {

template <typename T> struct TmaFmaCfg;
template <> struct TmaFmaCfg<float> { static constexpr int TM = 8, TN = 8; };
template <> struct TmaFmaCfg<double> { static constexpr int TM = 8, TN = 4; };

namespace {

constexpr int kTfConsumers = 8;                       // consumer warps: 16 x 16 threads
constexpr int kTfThreads = 32 * (1 + kTfConsumers);   // + one producer warp
constexpr int kTfStages = 4;

template <typename T>
struct TfShape {
  static constexpr int TM = TmaFmaCfg<T>::TM, TN = TmaFmaCfg<T>::TN;
  static constexpr int BM = 16 * TM, BN = 16 * TN;
  static constexpr int V = 16 / (int)sizeof(T);     // elements per 16-byte load
  static constexpr int BK = 128 / (int)sizeof(T);   // slab depth: one 128-byte row
  static constexpr uint32_t kABytes = BM * BK * sizeof(T);
  static constexpr uint32_t kBBytes = BN * BK * sizeof(T);
  static constexpr uint32_t kStage = kABytes + kBBytes;
  static constexpr size_t kSmem = (size_t)kTfStages * kStage + 1024;
};

// Row (of the operand tile) held in slot i by thread coordinate t.
template <int R, int V, bool KMaj>
__device__ __forceinline__ int tile_row(int t, int i) {
  return KMaj ? t + 16 * i : (i / V) * (16 * V) + t * V + (i % V);
}

// Loads the values thread t needs for K values kq*V .. kq*V + V - 1 of a tile:
// x[i][v] = tile(row(i), kq * V + v).
template <typename T, int R, int E, bool KMaj>
__device__ __forceinline__ void load_block(const uint8_t* tile, int t, int kq, T (&x)[R][16 / sizeof(T)]) {
  constexpr int V = 16 / (int)sizeof(T);
  if constexpr (KMaj) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int r = t + 16 * i;
      const uint4 u = *reinterpret_cast<const uint4*>(tile + r * 128 + ((kq ^ (r & 7)) << 4));
      const T* p = reinterpret_cast<const T*>(&u);
#pragma unroll
      for (int v = 0; v < V; ++v) x[i][v] = p[v];
    }
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const T* row = reinterpret_cast<const T*>(tile) + (size_t)(kq * V + v) * E;
#pragma unroll
      for (int g = 0; g < R / V; ++g) {
        const uint4 u = *reinterpret_cast<const uint4*>(row + g * 16 * V + t * V);
        const T* p = reinterpret_cast<const T*>(&u);
#pragma unroll
        for (int w = 0; w < V; ++w) x[g * V + w][v] = p[w];
      }
    }
  }
}

__device__ __forceinline__ float tf_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double tf_fma(double a, double b, double c) { return fma(a, b, c); }

struct TfMaps {
  CUtensorMap a, b;
};

template <typename T, bool AK, bool BK_>
__global__ void __launch_bounds__(kTfThreads, 1)
k_gemm_tma_fma(const __grid_constant__ TfMaps maps, int m, int n, int k, T alpha, T beta,
               T* __restrict__ C, size_t ldc, unsigned* status, uint64_t limit_ns) {
  using S = TfShape<T>;
  constexpr int TM = S::TM, TN = S::TN, V = S::V, BKd = S::BK;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = tc::align1024_shared(smem_raw);
  __shared__ __align__(8) uint64_t full_bar[kTfStages], empty_bar[kTfStages];
  __shared__ int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * S::BM, n0 = blockIdx.y * S::BN;
  const int nk = (k + BKd - 1) / BKd;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kTfStages; ++s) {
      tc::mbar_init(&full_bar[s], 1);
      tc::mbar_init(&empty_bar[s], kTfConsumers);
    }
    abort_flag = 0;
    tc::fence_mbar_init();
  }
  __syncthreads();

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer ----
      tc::prefetch_tmap(&maps.a);
      tc::prefetch_tmap(&maps.b);
      int kb = 0;
      for (; kb < nk; ++kb) {
        const int s = kb % kTfStages;
        if (kb >= kTfStages && !tc::mbar_wait(&empty_bar[s], ((kb / kTfStages) - 1) & 1, limit_ns)) {
          atomicOr(status, kStatusTimeout);
          atomicExch(&abort_flag, 1);
          break;
        }
        if (*(volatile int*)&abort_flag) break;
        uint8_t* st = smem + (size_t)s * S::kStage;
        const int k0 = kb * BKd;
        tc::mbar_expect_tx(&full_bar[s], S::kStage);
        if (AK) tc::tma_load_2d(st, &maps.a, &full_bar[s], k0, m0);
        else tc::tma_load_2d(st, &maps.a, &full_bar[s], m0, k0);
        if (BK_) tc::tma_load_2d(st + S::kABytes, &maps.b, &full_bar[s], k0, n0);
        else tc::tma_load_2d(st + S::kABytes, &maps.b, &full_bar[s], n0, k0);
      }
      // every issued load lands before the CTA may exit
      for (int j = (kb > kTfStages ? kb - kTfStages : 0); j < kb; ++j)
        tc::mbar_wait(&full_bar[j % kTfStages], (j / kTfStages) & 1, 1000000000ull);
    }
  } else {
    // ---- FMA consumers ----
    const int c = threadIdx.x - 32;
    const int tx = c & 15, ty = c >> 4;
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % kTfStages;
      if (!tc::mbar_wait(&full_bar[s], (kb / kTfStages) & 1, limit_ns)) {
        atomicOr(status, kStatusTimeout);
        atomicExch(&abort_flag, 1);
        break;
      }
      const uint8_t* ta = smem + (size_t)s * S::kStage;
      const uint8_t* tb = ta + S::kABytes;
      // fully unrolled for both types: with the tiles addressed in the
      // shared window the fp32 kernel fits it (NN 8192^3: 47.9 TFLOP/s
      // rolled, 50.9 unrolled)
#pragma unroll
      for (int kq = 0; kq < BKd / V; ++kq) {
        T a[TM][V], b[TN][V];
        load_block<T, TM, S::BM, AK>(ta, ty, kq, a);
        load_block<T, TN, S::BN, BK_>(tb, tx, kq, b);
#pragma unroll
        for (int v = 0; v < V; ++v)
#pragma unroll
          for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] = tf_fma(a[i][v], b[j][v], acc[i][j]);
      }
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&empty_bar[s]);
    }
    if (!*(volatile int*)&abort_flag) {
      const bool beta0 = beta == T(0), beta1 = beta == T(1);
      // every C load of a column before its stores: a load behind a store
      // the compiler cannot prove disjoint would cost a round trip each
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const int gc = n0 + tile_row<TN, V, BK_>(tx, j);
        if (gc >= n) continue;
        T cv[TM];
#pragma unroll
        for (int i = 0; i < TM; ++i) {
          const int gr = m0 + tile_row<TM, V, AK>(ty, i);
          cv[i] = (!beta0 && gr < m) ? C[gr + (size_t)gc * ldc] : T(0);
        }
#pragma unroll
        for (int i = 0; i < TM; ++i) {
          const int gr = m0 + tile_row<TM, V, AK>(ty, i);
          if (gr >= m) continue;
          const T v = alpha * acc[i][j];
          C[gr + (size_t)gc * ldc] = beta0 ? v : beta1 ? cv[i] + v : beta * cv[i] + v;
        }
      }
    }
  }
}

template <typename T, bool AK, bool BK_>
coral_status_t launch_tma_fma(Handle* h, const TfMaps& maps, int m, int n, int k, T alpha, T beta, T* C,
                              size_t ldc) {
  using S = TfShape<T>;
  static uint64_t attr_devices = 0;  // bit d: attribute set on device d
  const uint64_t bit = h->device < 64 ? (1ull << h->device) : 0;
  if (!(attr_devices & bit) || !bit) {
    CORAL_CUDA(h, cudaFuncSetAttribute(k_gemm_tma_fma<T, AK, BK_>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)S::kSmem));
    attr_devices |= bit;
  }
  const dim3 grid((unsigned)((m + S::BM - 1) / S::BM), (unsigned)((n + S::BN - 1) / S::BN));
  timed_begin(h);
  k_gemm_tma_fma<T, AK, BK_><<<grid, kTfThreads, S::kSmem, h->stream>>>(
      maps, m, n, k, alpha, beta, C, ldc, &h->words->status, h->wait_limit * 32ull);
  coral_status_t s = launch_status(h);
  timed_end(h);
  return s;
}

}  // namespace

// Enqueues the TMA-fed kernel when tensor maps can describe both operands
// (16-byte aligned bases, leading dimensions multiples of 16 bytes, sizes
// within int range); returns CORAL_ERR_NOT_SUPPORTED otherwise so the caller
// takes the register-staged kernel.  m, n, k > 0 and alpha != 0 here.
template <typename T>
coral_status_t enqueue_gemm_tma_fma(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k, T alpha,
                                    const T* A, size_t lda, const T* B, size_t ldb, T beta, T* C,
                                    size_t ldc) {
  using S = TfShape<T>;
  if (!aligned16(A) || !aligned16(B) || (lda * sizeof(T)) % 16 || (ldb * sizeof(T)) % 16)
    return CORAL_ERR_NOT_SUPPORTED;
  if ((m + S::BM - 1) / S::BM > 0x7fffffffu || (n + S::BN - 1) / S::BN > 65535) return CORAL_ERR_NOT_SUPPORTED;
  const bool ak = op_a != CORAL_NO_TRANSPOSE, bk = op_b == CORAL_NO_TRANSPOSE;
  TfMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  const int es = (int)sizeof(T);
  // K-contiguous operands: box {BK, rows}, 128-byte swizzle; others: box {rows, BK}.
  const bool ok_a = ak ? encode_kmajor_map(&maps.a, A, es, k, m, lda * es, S::BK, S::BM, 128)
                       : encode_kmajor_map(&maps.a, A, es, m, k, lda * es, S::BM, S::BK, 0);
  const bool ok_b = bk ? encode_kmajor_map(&maps.b, B, es, k, n, ldb * es, S::BK, S::BN, 128)
                       : encode_kmajor_map(&maps.b, B, es, n, k, ldb * es, S::BN, S::BK, 0);
  if (!ok_a || !ok_b) return CORAL_ERR_NOT_SUPPORTED;
  const int mi = (int)m, ni = (int)n, ki = (int)k;
  if (ak && bk) return launch_tma_fma<T, true, true>(h, maps, mi, ni, ki, alpha, beta, C, ldc);
  if (ak) return launch_tma_fma<T, true, false>(h, maps, mi, ni, ki, alpha, beta, C, ldc);
  if (bk) return launch_tma_fma<T, false, true>(h, maps, mi, ni, ki, alpha, beta, C, ldc);
  return launch_tma_fma<T, false, false>(h, maps, mi, ni, ki, alpha, beta, C, ldc);
}

template coral_status_t enqueue_gemm_tma_fma<float>(Handle*, int, int, size_t, size_t, size_t, float,
                                                    const float*, size_t, const float*, size_t, float,
                                                    float*, size_t);
template coral_status_t enqueue_gemm_tma_fma<double>(Handle*, int, int, size_t, size_t, size_t, double,
                                                     const double*, size_t, const double*, size_t, double,
                                                     double*, size_t);

}  // namespace coral
