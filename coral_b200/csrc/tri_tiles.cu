// Level-2 routines that read one triangle of a square matrix: SSYMV, CHEMV
// and STRMV (N and T), sharing one tile kernel.
//
// The stored triangle is cut into 64 x 64 tiles; every stored tile is read
// from HBM exactly once (128-bit loads when aligned), staged in shared memory
// and used for up to two products:
//   row part    tile * v_J        -> contribution to output rows of tile-row I
//   column part tile^T * v_I      -> contribution to output rows of tile-row J
// SYMV/HEMV use both (the unstored triangle is the (conjugate) transpose of
// the stored one -- reading the triangle once, where CORAL's lda == n fast
// path walks it column by column, ssymv.rs:144-211, chemv.rs:142-231);
// TRMV N uses the row part, TRMV T the column part.  Diagonal tiles are
// completed in shared memory (mirrored for SYMV/HEMV with Re(a_jj) for HEMV,
// chemv.rs:179-182; masked to the triangle, unit diagonal = 1, for TRMV).
//
// A CTA handles a run of up to kSeg tiles of one tile-column J; row parts are
// written per tile, column parts summed over the run.  A second kernel adds,
// for each tile-row, its partials in a fixed order and applies beta (SYMV:
// beta == 0 fills zeros, else multiplies, ssymv.rs:137-141) or writes x
// (TRMV).  Results are deterministic.
#include "common.cuh"

namespace coral {
namespace {

constexpr int kT = 64;        // tile edge
constexpr int kSeg = 8;       // tiles per CTA run
constexpr int kTriThreads = 256;

enum TriMode { kSymv = 0, kHemv = 1, kTrmvN = 2, kTrmvT = 3 };

template <typename T> struct Cx;
template <> struct Cx<float> {
  static __device__ __forceinline__ float zero() { return 0.f; }
  static __device__ __forceinline__ float conj(float a) { return a; }
  static __device__ __forceinline__ float re(float a) { return a; }
  static __device__ __forceinline__ void mac(float& c, float a, float b) { c = fmaf(a, b, c); }
  static __device__ __forceinline__ float add(float a, float b) { return a + b; }
  static __device__ __forceinline__ float one() { return 1.f; }
};
template <> struct Cx<float2> {
  static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
  static __device__ __forceinline__ float2 conj(float2 a) { return make_float2(a.x, -a.y); }
  static __device__ __forceinline__ float2 re(float2 a) { return make_float2(a.x, 0.f); }
  static __device__ __forceinline__ void mac(float2& c, float2 a, float2 b) {
    c.x = fmaf(a.x, b.x, c.x);
    c.x = fmaf(-a.y, b.y, c.x);
    c.y = fmaf(a.x, b.y, c.y);
    c.y = fmaf(a.y, b.x, c.y);
  }
  static __device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
  static __device__ __forceinline__ float2 one() { return make_float2(1.f, 0.f); }
};

__device__ __forceinline__ float scale_x(float alpha, float x) { return alpha * x; }
__device__ __forceinline__ float2 scale_x(float2 alpha, float2 x) {
  return make_float2(alpha.x * x.x - alpha.y * x.y, alpha.x * x.y + alpha.y * x.x);
}

// Index of stored tile (I, J) in packed triangular order.
__host__ __device__ __forceinline__ size_t tri_index(int I, int J, bool lower) {
  return lower ? (size_t)I * (I + 1) / 2 + J : (size_t)J * (J + 1) / 2 + I;
}

template <typename T, int kMode>
__global__ void __launch_bounds__(kTriThreads)
k_tri_tiles(int n, const T* __restrict__ A, size_t lda, const T* __restrict__ x, size_t incx,
            T alpha, bool lower, bool unit, T* __restrict__ rowpart, T* __restrict__ colpart,
            int max_seg, int diag_only) {
  constexpr bool kSym = kMode == kSymv || kMode == kHemv;
  constexpr bool kRow = kMode != kTrmvT;
  constexpr bool kCol = kMode == kSymv || kMode == kHemv || kMode == kTrmvT;
  __shared__ T tile[kT][kT + 1];   // tile[c][r] = element (row r, col c)
  __shared__ T vJ[kT], vI[kT];
  __shared__ T red[4][kT];

  const int NT = (n + kT - 1) / kT;
  const int J = blockIdx.x, seg = blockIdx.y;
  // Stored tiles of tile-column J: upper I = 0..J, lower I = J..NT-1.
  const int first = diag_only ? J : (lower ? J : 0);
  const int count = diag_only ? 1 : (lower ? NT - J : J + 1);
  const int t0 = seg * kSeg;
  if (t0 >= count) return;
  const int t1 = min(count, t0 + kSeg);
  const int tid = threadIdx.x;
  const int r = tid % kT, q = tid / kT;  // 4 quarters of 16 columns / rows
  const int c0 = J * kT;

  if (tid < kT) {
    const int gc = c0 + tid;
    T v = gc < n ? x[(size_t)gc * incx] : Cx<T>::zero();
    vJ[tid] = kSym ? scale_x(alpha, v) : v;
  }
  T colacc = Cx<T>::zero();  // column part for column r, quarter q of the rows
  // Tile elements of this thread (element e = tid + p * 256: row e % 64,
  // column e / 64), loaded for tile ti+1 while tile ti is computed.
  constexpr int kPer = kT * kT / kTriThreads;
  T reg[kPer];
  auto load_tile = [&](int I) {
    const int r0 = I * kT;
#pragma unroll
    for (int p = 0; p < kPer; ++p) {
      const int e = tid + p * kTriThreads;
      const int gr = r0 + e % kT, gc = c0 + e / kT;
      reg[p] = (gr < n && gc < n) ? __ldcs(A + gr + (size_t)gc * lda) : Cx<T>::zero();
    }
  };
  load_tile(first + t0);
  for (int ti = t0; ti < t1; ++ti) {
    const int I = first + ti;
    const int r0 = I * kT;
    __syncthreads();
#pragma unroll
    for (int p = 0; p < kPer; ++p) {
      const int e = tid + p * kTriThreads;
      tile[e / kT][e % kT] = reg[p];
    }
    if (tid < kT) {
      const int gr = r0 + tid;
      T v = gr < n ? x[(size_t)gr * incx] : Cx<T>::zero();
      vI[tid] = kSym ? scale_x(alpha, v) : v;
    }
    if (ti + 1 < t1) load_tile(I + 1);
    __syncthreads();
    const bool diag = I == J;
    if (diag) {
      // Complete the diagonal tile in place: element (rr, cc) with rr, cc in tile.
      for (int e = tid; e < kT * kT; e += kTriThreads) {
        const int rr = e % kT, cc = e / kT;
        const bool stored = lower ? rr >= cc : rr <= cc;
        if (rr == cc) {
          if (kMode == kHemv) tile[cc][rr] = Cx<T>::re(tile[cc][rr]);
          if ((kMode == kTrmvN || kMode == kTrmvT) && unit) tile[cc][rr] = Cx<T>::one();
        } else if (!stored) {
          if (kSym) {
            // unstored (rr, cc) = stored (cc, rr), conjugated for HEMV; read
            // from the stored half, which this pass never overwrites.
            T s = tile[rr][cc];
            tile[cc][rr] = kMode == kHemv ? Cx<T>::conj(s) : s;
          } else {
            tile[cc][rr] = Cx<T>::zero();
          }
        }
      }
      __syncthreads();
    }
    // Row part: out[r] = sum_c tile(r, c) * vJ[c], quarter q of the columns.
    if (kRow) {
      T acc = Cx<T>::zero();
#pragma unroll
      for (int c = q * 16; c < q * 16 + 16; ++c) Cx<T>::mac(acc, tile[c][r], vJ[c]);
      red[q][r] = acc;
    }
    // Column part (off-diagonal tiles for SYMV/HEMV; every tile for TRMV T):
    // out[c = r] += sum_rr conj?(tile(rr, c)) * vI[rr], quarter q of the rows.
    if (kCol && (!diag || kMode == kTrmvT)) {
#pragma unroll
      for (int rr = q * 16; rr < q * 16 + 16; ++rr) {
        T a = tile[r][rr];
        Cx<T>::mac(colacc, kMode == kHemv ? Cx<T>::conj(a) : a, vI[rr]);
      }
    }
    __syncthreads();
    if (kRow && tid < kT) {
      T s = Cx<T>::add(Cx<T>::add(red[0][tid], red[1][tid]), Cx<T>::add(red[2][tid], red[3][tid]));
      rowpart[(diag_only ? (size_t)J : tri_index(I, J, lower)) * kT + tid] = s;
    }
  }
  if (kCol) {
    __syncthreads();
    red[q][r] = colacc;
    __syncthreads();
    if (tid < kT) {
      T s = Cx<T>::add(Cx<T>::add(red[0][tid], red[1][tid]), Cx<T>::add(red[2][tid], red[3][tid]));
      colpart[(diag_only ? (size_t)J : ((size_t)J * max_seg + seg)) * kT + tid] = s;
    }
  }
}

__device__ __forceinline__ float beta_apply(float beta, float y) {
  return beta == 0.f ? 0.f : (beta != 1.f ? y * beta : y);
}
__device__ __forceinline__ float2 beta_apply(float2 beta, float2 y) {
  if (beta.x == 0.f && beta.y == 0.f) return make_float2(0.f, 0.f);
  if (beta.x == 1.f && beta.y == 0.f) return y;
  return make_float2(y.x * beta.x - y.y * beta.y, y.x * beta.y + y.y * beta.x);
}

// Sums the partials of tile-row t in a fixed order.
template <typename T, int kMode>
__global__ void k_tri_combine(int n, T beta, T* __restrict__ y, size_t incy, bool lower,
                              const T* __restrict__ rowpart, const T* __restrict__ colpart,
                              int max_seg) {
  constexpr bool kRow = kMode != kTrmvT;
  constexpr bool kCol = kMode == kSymv || kMode == kHemv || kMode == kTrmvT;
  const int NT = (n + kT - 1) / kT;
  const int t = blockIdx.x, i = threadIdx.x;
  const int gr = t * kT + i;
  if (gr >= n) return;
  T s = Cx<T>::zero();
  if (kRow) {
    const int j0 = lower ? 0 : t, j1 = lower ? t : NT - 1;
    for (int J = j0; J <= j1; ++J) s = Cx<T>::add(s, rowpart[tri_index(t, J, lower) * kT + i]);
  }
  if (kCol) {
    const int count = lower ? NT - t : t + 1;
    const int nseg = (count + kSeg - 1) / kSeg;
    for (int g = 0; g < nseg; ++g) s = Cx<T>::add(s, colpart[((size_t)t * max_seg + g) * kT + i]);
  }
  T* yp = y + (size_t)gr * incy;
  if (kMode == kTrmvN || kMode == kTrmvT) *yp = s;
  else *yp = Cx<T>::add(beta_apply(beta, *yp), s);
}

template <typename T, int kMode>
coral_status_t run_tri(Handle* h, int n, const T* A, size_t lda, const T* x, size_t incx, T alpha,
                       T beta, T* y, size_t incy, bool lower, bool unit) {
  const int NT = (n + kT - 1) / kT;
  const int max_seg = (NT + kSeg - 1) / kSeg;
  const size_t rp = (size_t)NT * (NT + 1) / 2 * kT;
  const size_t cp = (size_t)NT * max_seg * kT;
  T* sc = static_cast<T*>(scratch(h, (rp + cp) * sizeof(T)));
  if (!sc) return CORAL_ERR_ALLOC;
  dim3 grid(NT, max_seg);
  timed_begin(h);
  k_tri_tiles<T, kMode><<<grid, kTriThreads, 0, h->stream>>>(n, A, lda, x, incx, alpha, lower, unit,
                                                             sc, sc + rp, max_seg, 0);
  coral_status_t s = launch_status(h);
  timed_end(h);
  if (s != CORAL_OK) return s;
  k_tri_combine<T, kMode><<<NT, kT, 0, h->stream>>>(n, beta, y, incy, lower, sc, sc + rp, max_seg);
  return launch_status(h);
}


// ---- register-resident off-diagonal pass ----------------------------------------
// Off-diagonal stored tiles, processed as 32-row strips of a kC-column tile
// column J by one warp each (lane = row).  A strip's kC column values stay in
// registers: the row part (A_strip * v_J) is complete per lane; the column
// part (A_strip^T v_I) is accumulated per lane across every strip the warp
// handles and reduced across lanes once at the end.  No shared-memory
// staging, no barrier per tile, kC independent loads in flight per lane.
// kC columns per tile column (the diagonal tile width); kH columns loaded per
// pass (complex values take two passes so a strip fits in registers).
template <typename T> struct StripCfg { static constexpr int kC = 64, kH = 64; };
template <> struct StripCfg<float2> { static constexpr int kC = 64, kH = 32; };
constexpr int kStripWarps = 4;

template <typename T>
__device__ __forceinline__ T shfl_xor_t(T v, int o);
template <> __device__ __forceinline__ float shfl_xor_t<float>(float v, int o) {
  return __shfl_xor_sync(0xffffffffu, v, o);
}
template <> __device__ __forceinline__ float2 shfl_xor_t<float2>(float2 v, int o) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}

template <int W, typename T, int N>
__device__ __forceinline__ void butterfly(T (&acc)[N], int lane, int o) {
  const bool up = (lane & o) != 0;
#pragma unroll
  for (int c = 0; c < W; ++c) {
    const T mine = up ? acc[c + W] : acc[c];
    const T theirs = shfl_xor_t(up ? acc[c] : acc[c + W], o);
    acc[c] = Cx<T>::add(mine, theirs);
  }
}

// Off-diagonal rows of column block J: upper [0, J*kC), lower [(J+1)*kC, n).
template <typename T, int kMode>
__global__ void __launch_bounds__(32 * kStripWarps)
k_tri_strips(int n, const T* __restrict__ A, size_t lda, const T* __restrict__ x, size_t incx,
             T alpha, bool lower, T* __restrict__ rowpart, T* __restrict__ colpart, int nstrip_rows) {
  constexpr int kC = StripCfg<T>::kC, kH = StripCfg<T>::kH;
  constexpr bool kSym = kMode == kSymv || kMode == kHemv;
  constexpr bool kRow = kMode != kTrmvT;
  constexpr bool kCol = kMode == kSymv || kMode == kHemv || kMode == kTrmvT;
  __shared__ T vJ[kC];
  __shared__ T red[kStripWarps][kC];
  const int J = blockIdx.x;
  const int c0 = J * kC;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row_lo = lower ? c0 + kC : 0;
  const int row_hi = lower ? n : c0;
  const int nstrip = row_hi > row_lo ? (row_hi - row_lo + 31) / 32 : 0;
  if (threadIdx.x < kC) {
    const int gc = c0 + threadIdx.x;
    T v = gc < n ? x[(size_t)gc * incx] : Cx<T>::zero();
    vJ[threadIdx.x] = kSym ? scale_x(alpha, v) : v;
  }
  __syncthreads();
  T colacc[kC];
#pragma unroll
  for (int c = 0; c < kC; ++c) colacc[c] = Cx<T>::zero();
  const int step = gridDim.y * kStripWarps;
  for (int st = blockIdx.y * kStripWarps + warp; st < nstrip; st += step) {
    const int r = row_lo + st * 32 + lane;
    const bool rv = r < row_hi;
    const T* ap = A + r + (size_t)c0 * lda;
    T xi = Cx<T>::zero();
    if (kCol) {
      xi = rv ? x[(size_t)r * incx] : Cx<T>::zero();
      if (kSym) xi = scale_x(alpha, xi);
    }
    T racc = Cx<T>::zero();
#pragma unroll
    for (int h0 = 0; h0 < kC; h0 += kH) {
      T a[kH];
#pragma unroll
      for (int c = 0; c < kH; ++c)
        a[c] = (rv && c0 + h0 + c < n) ? __ldcs(ap + (size_t)(h0 + c) * lda) : Cx<T>::zero();
      if (kRow) {
#pragma unroll
        for (int c = 0; c < kH; ++c) Cx<T>::mac(racc, a[c], vJ[h0 + c]);
      }
      if (kCol) {
#pragma unroll
        for (int c = 0; c < kH; ++c)
          Cx<T>::mac(colacc[h0 + c], kMode == kHemv ? Cx<T>::conj(a[c]) : a[c], xi);
      }
    }
    if (kRow) {
      // row strip index within the whole matrix (32-row strips)
      const int gstrip = (row_lo / 32) + st;
      rowpart[((size_t)gstrip * gridDim.x + J) * 32 + lane] = rv ? racc : Cx<T>::zero();
    }
  }
  if (!kCol) return;
  // Cross-lane sum of colacc[c] for every c: a butterfly that halves the
  // values per lane each step (lanes with bit o set keep the upper half).
  // After the 5 steps, entry j of lane l holds the sum for column
  // j + (kC / 32) * l.
  butterfly<kC / 2>(colacc, lane, 16);
  butterfly<kC / 4>(colacc, lane, 8);
  butterfly<kC / 8>(colacc, lane, 4);
  butterfly<kC / 16>(colacc, lane, 2);
  butterfly<kC / 32>(colacc, lane, 1);
  int col_of[kC / 32];
#pragma unroll
  for (int j = 0; j < kC / 32; ++j) col_of[j] = j + (kC / 32) * lane;
#pragma unroll
  for (int j = 0; j < kC / 32; ++j) red[warp][col_of[j]] = colacc[j];
  __syncthreads();
  if (threadIdx.x < kC) {
    T s = red[0][threadIdx.x];
#pragma unroll
    for (int w2 = 1; w2 < kStripWarps; ++w2) s = Cx<T>::add(s, red[w2][threadIdx.x]);
    colpart[((size_t)J * gridDim.y + blockIdx.y) * kC + threadIdx.x] = s;
  }
}

// Per 32-row strip: y = beta*y (or 0 for TRMV) + row parts of every
// off-diagonal column block + the diagonal block's parts + column parts.
template <typename T, int kMode>
__global__ void k_strip_combine(int n, T beta, T* __restrict__ y, size_t incy, bool lower,
                                const T* __restrict__ rowpart, const T* __restrict__ colpart,
                                int ncolblk, int nsplit, const T* __restrict__ drow,
                                const T* __restrict__ dcol) {
  constexpr int kC = StripCfg<T>::kC;
  constexpr bool kRow = kMode != kTrmvT;
  constexpr bool kCol = kMode == kSymv || kMode == kHemv || kMode == kTrmvT;
  const int gr = blockIdx.x * 32 + threadIdx.x;
  if (gr >= n) return;
  const int gstrip = blockIdx.x;
  const int Jr = gr / kC;  // column block containing this row
  T s = Cx<T>::zero();
  if (kRow) {
    // off-diagonal column blocks J whose stored strips cover row gr
    const int j0 = lower ? 0 : Jr + 1, j1 = lower ? Jr : ncolblk;
    for (int J = j0; J < j1; ++J) s = Cx<T>::add(s, rowpart[((size_t)gstrip * ncolblk + J) * 32 + threadIdx.x]);
    s = Cx<T>::add(s, drow[gr]);
  }
  if (kCol) {
    for (int q = 0; q < nsplit; ++q) s = Cx<T>::add(s, colpart[((size_t)Jr * nsplit + q) * kC + gr % kC]);
    if (kMode == kTrmvT) s = Cx<T>::add(s, dcol[gr]);
  }
  T* yp = y + (size_t)gr * incy;
  if (kMode == kTrmvN || kMode == kTrmvT) *yp = s;
  else *yp = Cx<T>::add(beta_apply(beta, *yp), s);
}

template <typename T, int kMode>
coral_status_t run_tri_strips(Handle* h, int n, const T* A, size_t lda, const T* x, size_t incx,
                              T alpha, T beta, T* y, size_t incy, bool lower, bool unit) {
  constexpr int kC = StripCfg<T>::kC;
  static_assert(kC == kT || kC == kT / 2, "diagonal tiles are kT wide");
  const int ncol = (n + kC - 1) / kC;
  const int nstrips = (n + 31) / 32;
  // CTAs per column block: enough warps to cover the longest column with ~4 strips each
  int nsplit = (nstrips / kStripWarps + 3) / 4;
  nsplit = nsplit < 1 ? 1 : (nsplit > 64 ? 64 : nsplit);
  const size_t rp = (size_t)nstrips * ncol * 32;
  const size_t cp = (size_t)ncol * nsplit * kC;
  // diagonal pass on kT-wide tiles: row parts and (TRMV T) column parts per row
  const int NT = (n + kT - 1) / kT;
  const size_t dlen = (size_t)NT * kT;
  T* sc = static_cast<T*>(scratch(h, (rp + cp + 2 * dlen) * sizeof(T)));
  if (!sc) return CORAL_ERR_ALLOC;
  T* drow = sc + rp + cp;
  T* dcol = drow + dlen;
  if (kC != kT) return CORAL_ERR_NOT_SUPPORTED;
  timed_begin(h);
  k_tri_strips<T, kMode><<<dim3(ncol, nsplit), 32 * kStripWarps, 0, h->stream>>>(
      n, A, lda, x, incx, alpha, lower, sc, sc + rp, nstrips);
  coral_status_t s = launch_status(h);
  timed_end(h);
  if (s != CORAL_OK) return s;
  k_tri_tiles<T, kMode><<<dim3(NT, 1), kTriThreads, 0, h->stream>>>(n, A, lda, x, incx, alpha, lower,
                                                                    unit, drow, dcol, 1, 1);
  if ((s = launch_status(h)) != CORAL_OK) return s;
  k_strip_combine<T, kMode><<<nstrips, 32, 0, h->stream>>>(n, beta, y, incy, lower, sc, sc + rp, ncol,
                                                           nsplit, drow, dcol);
  return launch_status(h);
}

}  // namespace
}  // namespace coral

using namespace coral;

extern "C" {

coral_status_t coral_ssymv(coral_handle_t hh, int uplo, size_t n, float alpha, const float* matrix,
                           size_t lda, const float* x, size_t incx, float beta, float* y,
                           size_t incy) {
  CORAL_HANDLE(hh);
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (n == 0) return CORAL_OK;                          // ssymv.rs:112
  if (alpha == 0.0f && beta == 1.0f) return CORAL_OK;   // ssymv.rs:113
  if (!matrix) return bad_arg(H, 4);
  if (lda < n) return bad_arg(H, 5);
  if (!x) return bad_arg(H, 6);
  if (incx == 0) return bad_arg(H, 7);
  if (!y) return bad_arg(H, 9);
  if (incy == 0) return bad_arg(H, 10);
  if (n > (size_t)(1 << 20)) return CORAL_ERR_NOT_SUPPORTED;
  return run_tri_strips<float, kSymv>(H, (int)n, matrix, lda, x, incx, alpha, beta, y, incy,
                                      uplo == CORAL_LOWER, false);
}

coral_status_t coral_chemv(coral_handle_t hh, int uplo, size_t n, const float alpha[2],
                           const float* matrix, size_t lda, const float* x, size_t incx,
                           const float beta[2], float* y, size_t incy) {
  CORAL_HANDLE(hh);
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (!alpha) return bad_arg(H, 3);
  if (!beta) return bad_arg(H, 8);
  if (n == 0) return CORAL_OK;  // chemv.rs:109
  if (alpha[0] == 0.f && alpha[1] == 0.f && beta[0] == 1.f && beta[1] == 0.f) return CORAL_OK;
  if (!matrix) return bad_arg(H, 4);
  if (lda < n) return bad_arg(H, 5);
  if (!x) return bad_arg(H, 6);
  if (incx == 0) return bad_arg(H, 7);
  if (!y) return bad_arg(H, 9);
  if (incy == 0) return bad_arg(H, 10);
  if (((uintptr_t)matrix | (uintptr_t)x | (uintptr_t)y) & 7) return bad_arg(H, 4);
  if (n > (size_t)(1 << 20)) return CORAL_ERR_NOT_SUPPORTED;
  return run_tri_strips<float2, kHemv>(H, (int)n, reinterpret_cast<const float2*>(matrix), lda,
                                reinterpret_cast<const float2*>(x), incx,
                                make_float2(alpha[0], alpha[1]), make_float2(beta[0], beta[1]),
                                reinterpret_cast<float2*>(y), incy, uplo == CORAL_LOWER, false);
}

coral_status_t coral_strmv(coral_handle_t hh, int uplo, int trans, int diag, size_t n,
                           const float* matrix, size_t lda, float* x, size_t incx) {
  CORAL_HANDLE(hh);
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (trans < CORAL_NO_TRANSPOSE || trans > CORAL_CONJ_TRANSPOSE) return bad_arg(H, 2);
  if (diag != CORAL_UNIT && diag != CORAL_NON_UNIT) return bad_arg(H, 3);
  if (n == 0) return CORAL_OK;
  if (!matrix) return bad_arg(H, 5);
  if (lda < n) return bad_arg(H, 6);
  if (!x) return bad_arg(H, 7);
  if (incx == 0) return bad_arg(H, 8);
  if (n > (size_t)(1 << 20)) return CORAL_ERR_NOT_SUPPORTED;
  const bool lower = uplo == CORAL_LOWER, unit = diag == CORAL_UNIT;
  if (trans == CORAL_NO_TRANSPOSE)
    return run_tri<float, kTrmvN>(H, (int)n, matrix, lda, x, incx, 1.f, 0.f, x, incx, lower, unit);
  return run_tri<float, kTrmvT>(H, (int)n, matrix, lda, x, incx, 1.f, 0.f, x, incx, lower, unit);
}

}  // extern "C"
