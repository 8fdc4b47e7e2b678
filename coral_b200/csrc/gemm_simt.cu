// Native-precision GEMM on the FMA pipes: C <- alpha * op(A) op(B) + beta * C,
// column-major, for float, double, complex64 and complex128.
//
// Replaces CORAL's packing + macro/micro-kernel subsystem
// (coral-aarch64/src/level3/*_packers.rs, *_macro_kernel.rs, microkernel/).
// One CTA computes a BM x BN tile of C with 256 threads, each holding a TM x TN
// register tile split in two halves along each dimension (rows
// {ty*TM/2 + i} and {BM/2 + ty*TM/2 + i}) so the shared-memory reads of a warp
// are broadcast or consecutive.  Operand tiles are staged global -> registers
// -> shared memory, double buffered, one barrier per k-step.  op(A)/op(B)
// (N, T and, for complex, C = conjugate transpose) are resolved while staging:
// the tile in shared memory is always op(A)[k][m] / op(B)[k][n], with the
// conjugation applied on load as CORAL applies it in its packers
// (c32_packers.rs:83-108).
//
// Epilogue follows f32_edge.rs:37-58: beta == 0 writes alpha*acc without
// reading C, beta == 1 accumulates, else beta*C + alpha*acc.  alpha == 0 or
// k == 0 only scales C (sgemm_nn.rs:29-45, cgemm_nn.rs scale-only path).
#include "common.cuh"

#include <cuComplex.h>
#include <type_traits>

namespace coral {

// ---- arithmetic traits ------------------------------------------------------
template <typename T> struct Arith;

template <> struct Arith<float> {
  static __device__ __forceinline__ float zero() { return 0.f; }
  static __device__ __forceinline__ void mac(float& c, float a, float b) { c = fmaf(a, b, c); }
  static __device__ __forceinline__ float conj(float a) { return a; }
  static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
  static __device__ __forceinline__ float add(float a, float b) { return a + b; }
  static __host__ __device__ __forceinline__ bool is_zero(float a) { return a == 0.f; }
  static __host__ __device__ __forceinline__ bool is_one(float a) { return a == 1.f; }
};
template <> struct Arith<double> {
  static __device__ __forceinline__ double zero() { return 0.0; }
  static __device__ __forceinline__ void mac(double& c, double a, double b) { c = fma(a, b, c); }
  static __device__ __forceinline__ double conj(double a) { return a; }
  static __device__ __forceinline__ double mul(double a, double b) { return a * b; }
  static __device__ __forceinline__ double add(double a, double b) { return a + b; }
  static __host__ __device__ __forceinline__ bool is_zero(double a) { return a == 0.0; }
  static __host__ __device__ __forceinline__ bool is_one(double a) { return a == 1.0; }
};
template <> struct Arith<float2> {
  static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
  static __device__ __forceinline__ void mac(float2& c, float2 a, float2 b) {
    c.x = fmaf(a.x, b.x, c.x);
    c.x = fmaf(-a.y, b.y, c.x);
    c.y = fmaf(a.x, b.y, c.y);
    c.y = fmaf(a.y, b.x, c.y);
  }
  static __device__ __forceinline__ float2 conj(float2 a) { return make_float2(a.x, -a.y); }
  static __device__ __forceinline__ float2 mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
  static __device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
  static __host__ __device__ __forceinline__ bool is_zero(float2 a) { return a.x == 0.f && a.y == 0.f; }
  static __host__ __device__ __forceinline__ bool is_one(float2 a) { return a.x == 1.f && a.y == 0.f; }
};
template <> struct Arith<double2> {
  static __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
  static __device__ __forceinline__ void mac(double2& c, double2 a, double2 b) {
    c.x = fma(a.x, b.x, c.x);
    c.x = fma(-a.y, b.y, c.x);
    c.y = fma(a.x, b.y, c.y);
    c.y = fma(a.y, b.x, c.y);
  }
  static __device__ __forceinline__ double2 conj(double2 a) { return make_double2(a.x, -a.y); }
  static __device__ __forceinline__ double2 mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
  static __device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
  static __host__ __device__ __forceinline__ bool is_zero(double2 a) { return a.x == 0.0 && a.y == 0.0; }
  static __host__ __device__ __forceinline__ bool is_one(double2 a) { return a.x == 1.0 && a.y == 0.0; }
};

// Tile configuration per element type.
template <typename T> struct SimtCfg;
template <> struct SimtCfg<float>   { static constexpr int TM = 8, TN = 8, BK = 8; };
template <> struct SimtCfg<double>  { static constexpr int TM = 8, TN = 4, BK = 8; };
template <> struct SimtCfg<float2>  { static constexpr int TM = 4, TN = 4, BK = 8; };
template <> struct SimtCfg<double2> { static constexpr int TM = 4, TN = 2, BK = 8; };

namespace {

constexpr int kSimtThreads = 256;  // 16 x 16 thread grid

template <typename T>
__device__ __forceinline__ T load_op(const T* p, bool conj) {
  T v = __ldg(p);
  return conj ? Arith<T>::conj(v) : v;
}

// Stage one BK-slab of op(X) (X is A with extent `mn` = m, or B with extent n)
// into registers: element (kk, r) of the slab is op(X)(r0 + r, k0 + kk) for A
// and op(X)(k0 + kk, r0 + r) for B; `kmajor` says whether the stored matrix is
// contiguous along k (A transposed, B not transposed).
template <typename T, int BMN, int BK>
struct SlabLoader {
  static constexpr int kElems = BMN * BK / kSimtThreads;  // per thread
  T reg[kElems];

  __device__ __forceinline__ void load(const T* X, size_t ld, bool kmajor, bool conj, int r0,
                                       int k0, int mn, int k) {
#pragma unroll
    for (int e = 0; e < kElems; ++e) {
      int idx = threadIdx.x + e * kSimtThreads;
      int r, kk;
      if (kmajor) { kk = idx % BK; r = idx / BK; }
      else        { r = idx % BMN; kk = idx / BMN; }
      int gr = r0 + r, gk = k0 + kk;
      T v = Arith<T>::zero();
      if (gr < mn && gk < k) v = load_op(kmajor ? X + gk + (size_t)gr * ld : X + gr + (size_t)gk * ld, conj);
      reg[e] = v;
    }
  }
  __device__ __forceinline__ void store(T (*S)[BMN + 16 / sizeof(T)], bool kmajor) {
#pragma unroll
    for (int e = 0; e < kElems; ++e) {
      int idx = threadIdx.x + e * kSimtThreads;
      int r, kk;
      if (kmajor) { kk = idx % BK; r = idx / BK; }
      else        { r = idx % BMN; kk = idx / BMN; }
      S[kk][r] = reg[e];
    }
  }
};

template <typename T>
__global__ void __launch_bounds__(kSimtThreads)
k_gemm_simt(int m, int n, int k, T alpha, const T* __restrict__ A, size_t lda, int op_a,
            const T* __restrict__ B, size_t ldb, int op_b, T beta, T* __restrict__ C, size_t ldc) {
  constexpr int TM = SimtCfg<T>::TM, TN = SimtCfg<T>::TN, BK = SimtCfg<T>::BK;
  constexpr int BM = 16 * TM, BN = 16 * TN;
  constexpr int PAD = 16 / sizeof(T);
  constexpr int HM = TM / 2, HN = TN / 2;
  __shared__ __align__(16) T As[2][BK][BM + PAD];
  __shared__ __align__(16) T Bs[2][BK][BN + PAD];

  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const bool a_kmajor = op_a != CORAL_NO_TRANSPOSE, a_conj = op_a == CORAL_CONJ_TRANSPOSE;
  const bool b_kmajor = op_b == CORAL_NO_TRANSPOSE, b_conj = op_b == CORAL_CONJ_TRANSPOSE;

  SlabLoader<T, BM, BK> la;
  SlabLoader<T, BN, BK> lb;
  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = Arith<T>::zero();

  la.load(A, lda, a_kmajor, a_conj, m0, 0, m, k);
  lb.load(B, ldb, b_kmajor, b_conj, n0, 0, n, k);
  la.store(As[0], a_kmajor);
  lb.store(Bs[0], b_kmajor);
  __syncthreads();

  const int ktiles = (k + BK - 1) / BK;
  for (int kt = 0; kt < ktiles; ++kt) {
    const int cur = kt & 1;
    const bool more = kt + 1 < ktiles;
    if (more) {
      la.load(A, lda, a_kmajor, a_conj, m0, (kt + 1) * BK, m, k);
      lb.load(B, ldb, b_kmajor, b_conj, n0, (kt + 1) * BK, n, k);
    }
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[TM], b[TN];
#pragma unroll
      for (int i = 0; i < HM; ++i) {
        a[i] = As[cur][kk][ty * HM + i];
        a[HM + i] = As[cur][kk][BM / 2 + ty * HM + i];
      }
#pragma unroll
      for (int j = 0; j < HN; ++j) {
        b[j] = Bs[cur][kk][tx * HN + j];
        b[HN + j] = Bs[cur][kk][BN / 2 + tx * HN + j];
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) Arith<T>::mac(acc[i][j], a[i], b[j]);
    }
    if (more) {
      la.store(As[cur ^ 1], a_kmajor);
      lb.store(Bs[cur ^ 1], b_kmajor);
    }
    __syncthreads();
  }

  const bool beta0 = Arith<T>::is_zero(beta), beta1 = Arith<T>::is_one(beta);
  // every C load of a column before its stores: a load behind a store the
  // compiler cannot prove disjoint would cost a memory round trip each
#pragma unroll
  for (int j = 0; j < TN; ++j) {
    const int gc = n0 + (j < HN ? tx * HN + j : BN / 2 + tx * HN + (j - HN));
    if (gc >= n) continue;
    T cv[TM];
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int gr = m0 + (i < HM ? ty * HM + i : BM / 2 + ty * HM + (i - HM));
      cv[i] = (!beta0 && gr < m) ? C[gr + (size_t)gc * ldc] : Arith<T>::zero();
    }
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int gr = m0 + (i < HM ? ty * HM + i : BM / 2 + ty * HM + (i - HM));
      if (gr >= m) continue;
      const T v = Arith<T>::mul(alpha, acc[i][j]);
      C[gr + (size_t)gc * ldc] =
          beta0 ? v : beta1 ? Arith<T>::add(cv[i], v) : Arith<T>::add(Arith<T>::mul(beta, cv[i]), v);
    }
  }
}

// C <- beta * C (beta == 0 writes zeros without reading C).
template <typename T>
__global__ void k_scale_c(int m, int n, T beta, T* __restrict__ C, size_t ldc) {
  const bool beta0 = Arith<T>::is_zero(beta);
  size_t total = (size_t)m * n;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    size_t i = t % m, j = t / m;
    T* cp = C + i + j * ldc;
    *cp = beta0 ? Arith<T>::zero() : Arith<T>::mul(beta, *cp);
  }
}

}  // namespace

// Validates the GEMM arguments the way the reference's debug_asserts do
// (sgemm_nn.rs:24-27) and reports the 1-based position of the first bad one.
int gemm_bad_arg(int op_a, int op_b, size_t m, size_t n, size_t k, const void* a, size_t lda,
                 const void* b, size_t ldb, const void* c, size_t ldc, bool complex_ops) {
  const int maxop = complex_ops ? CORAL_CONJ_TRANSPOSE : CORAL_CONJ_TRANSPOSE;
  if (op_a < 0 || op_a > maxop) return 1;
  if (op_b < 0 || op_b > maxop) return 2;
  const size_t a_rows = op_a == CORAL_NO_TRANSPOSE ? m : k;
  const size_t b_rows = op_b == CORAL_NO_TRANSPOSE ? k : n;
  if (m && n && !c) return 12;
  if (ldc < (m ? m : 1)) return 13;
  if (m && n && k) {
    if (!a) return 7;
    if (lda < (a_rows ? a_rows : 1)) return 8;
    if (!b) return 9;
    if (ldb < (b_rows ? b_rows : 1)) return 10;
  }
  if (m > INT32_MAX || n > INT32_MAX || k > INT32_MAX) return -1;
  return 0;
}

template <typename T>
coral_status_t enqueue_gemm_tma_fma(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k, T alpha,
                                    const T* A, size_t lda, const T* B, size_t ldb, T beta, T* C,
                                    size_t ldc);

// Real types take the TMA-fed kernel (gemm_tma_fma.cu) whenever tensor maps
// can describe the operands, the register-staged kernel below otherwise;
// complex types always take the register-staged kernel.
template <typename T>
coral_status_t enqueue_gemm_simt(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                 T alpha, const T* A, size_t lda, const T* B, size_t ldb, T beta,
                                 T* C, size_t ldc) {
  if (m == 0 || n == 0) return CORAL_OK;
  if (Arith<T>::is_zero(alpha) || k == 0) {
    if (Arith<T>::is_one(beta)) return CORAL_OK;
    unsigned g = stream_grid(m * n, 256 * 4, h->sm_count, 8);
    k_scale_c<T><<<g, 256, 0, h->stream>>>((int)m, (int)n, beta, C, ldc);
    return launch_status(h);
  }
  if constexpr (std::is_same<T, float>::value || std::is_same<T, double>::value) {
    const coral_status_t s = enqueue_gemm_tma_fma<T>(h, op_a, op_b, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    if (s != CORAL_ERR_NOT_SUPPORTED) return s;
  }
  constexpr int BM = 16 * SimtCfg<T>::TM, BN = 16 * SimtCfg<T>::TN;
  dim3 grid((unsigned)((m + BM - 1) / BM), (unsigned)((n + BN - 1) / BN));
  if (grid.y > 65535) return CORAL_ERR_NOT_SUPPORTED;
  // ConjugateTranspose on a real type means Transpose (sgemm.rs:97-103).
  timed_begin(h);
  k_gemm_simt<T><<<grid, kSimtThreads, 0, h->stream>>>((int)m, (int)n, (int)k, alpha, A, lda, op_a,
                                                        B, ldb, op_b, beta, C, ldc);
  coral_status_t s = launch_status(h);
  timed_end(h);
  return s;
}

template coral_status_t enqueue_gemm_simt<float>(Handle*, int, int, size_t, size_t, size_t, float,
                                                 const float*, size_t, const float*, size_t, float,
                                                 float*, size_t);
template coral_status_t enqueue_gemm_simt<double>(Handle*, int, int, size_t, size_t, size_t, double,
                                                  const double*, size_t, const double*, size_t,
                                                  double, double*, size_t);
template coral_status_t enqueue_gemm_simt<float2>(Handle*, int, int, size_t, size_t, size_t, float2,
                                                  const float2*, size_t, const float2*, size_t,
                                                  float2, float2*, size_t);
template coral_status_t enqueue_gemm_simt<double2>(Handle*, int, int, size_t, size_t, size_t,
                                                   double2, const double2*, size_t, const double2*,
                                                   size_t, double2, double2*, size_t);

}  // namespace coral
