// Level-2 routines that read one triangle of a square matrix: SSYMV, CHEMV
// and STRMV (N and T).  The stored triangle is read from HBM exactly once:
//
//   * off-diagonal part -- k_tri_strips: one warp per 32-row strip of a
//     64-column tile column J, the strip held in registers (lane = row);
//     it yields a row part (strip * v_J -> output rows of the strip) and a
//     column part (strip^T v_I, accumulated per lane over the warp's strips,
//     reduced across lanes once) -> output rows of block J.  SYMV/HEMV use
//     both, the unstored triangle being the (conjugate) transpose of the
//     stored one -- where CORAL's lda == n fast path walks the triangle column
//     by column (ssymv.rs:144-211, chemv.rs:142-231); TRMV N uses the row
//     part, TRMV T the column part;
//   * diagonal 64 x 64 blocks -- k_tri_tiles: staged in shared memory and
//     completed there (mirrored for SYMV/HEMV with Re(a_jj) for HEMV,
//     chemv.rs:179-182; masked to the triangle, unit diagonal = 1, for TRMV);
//   * k_strip_combine adds, per 32-row strip, its partials in a fixed order
//     and applies beta (SYMV/HEMV: beta == 0 fills zeros, else multiplies,
//     ssymv.rs:137-141) or writes x (TRMV).  Results are deterministic.
//
// With coral_set_strip_form(CORAL_STRIPS_TMA) an aligned matrix instead takes
// k_tri_strips_tma, one TMA-fed persistent pass over the whole stored triangle
// (diagonal blocks included), then the combine: two launches instead of three.
// On the measured sizes (SSYMV n = 8192, CHEMV n = 4096) it is not faster than
// the register form, which stays the default.
#include "common.cuh"
#include "tc_common.cuh"

#include <cstring>
#include <type_traits>

namespace coral {
namespace {

constexpr int kT = 64;        // tile edge
constexpr int kSeg = 8;       // tiles per CTA run
constexpr int kTriThreads = 256;

enum TriMode { kSymv = 0, kHemv = 1, kTrmvN = 2, kTrmvT = 3, kTrmvC = 4 };
// Mode traits: which parts a mode uses, and whether the column part (the
// transposed use of a stored element) conjugates it.
template <int kMode> struct ModeT {
  static constexpr bool kSym = kMode == kSymv || kMode == kHemv;
  static constexpr bool kTr = kMode == kTrmvN || kMode == kTrmvT || kMode == kTrmvC;
  static constexpr bool kColOnly = kMode == kTrmvT || kMode == kTrmvC;
  static constexpr bool kRow = !kColOnly;
  static constexpr bool kCol = kSym || kColOnly;
  static constexpr bool kConjCol = kMode == kHemv || kMode == kTrmvC;
};

template <typename T> struct Cx;
template <> struct Cx<float> {
  static __host__ __device__ __forceinline__ float zero() { return 0.f; }
  static __device__ __forceinline__ float conj(float a) { return a; }
  static __device__ __forceinline__ float re(float a) { return a; }
  static __device__ __forceinline__ void mac(float& c, float a, float b) { c = fmaf(a, b, c); }
  static __device__ __forceinline__ float add(float a, float b) { return a + b; }
  static __host__ __device__ __forceinline__ float one() { return 1.f; }
};
template <> struct Cx<double> {
  static __host__ __device__ __forceinline__ double zero() { return 0.0; }
  static __device__ __forceinline__ double conj(double a) { return a; }
  static __device__ __forceinline__ double re(double a) { return a; }
  static __device__ __forceinline__ void mac(double& c, double a, double b) { c = fma(a, b, c); }
  static __device__ __forceinline__ double add(double a, double b) { return a + b; }
  static __host__ __device__ __forceinline__ double one() { return 1.0; }
};
template <> struct Cx<double2> {
  static __host__ __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
  static __device__ __forceinline__ double2 conj(double2 a) { return make_double2(a.x, -a.y); }
  static __device__ __forceinline__ double2 re(double2 a) { return make_double2(a.x, 0.0); }
  static __device__ __forceinline__ void mac(double2& c, double2 a, double2 b) {
    c.x = fma(a.x, b.x, c.x);
    c.x = fma(-a.y, b.y, c.x);
    c.y = fma(a.x, b.y, c.y);
    c.y = fma(a.y, b.x, c.y);
  }
  static __device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
  static __host__ __device__ __forceinline__ double2 one() { return make_double2(1.0, 0.0); }
};
template <> struct Cx<float2> {
  static __host__ __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
  static __device__ __forceinline__ float2 conj(float2 a) { return make_float2(a.x, -a.y); }
  static __device__ __forceinline__ float2 re(float2 a) { return make_float2(a.x, 0.f); }
  static __device__ __forceinline__ void mac(float2& c, float2 a, float2 b) {
    c.x = fmaf(a.x, b.x, c.x);
    c.x = fmaf(-a.y, b.y, c.x);
    c.y = fmaf(a.x, b.y, c.y);
    c.y = fmaf(a.y, b.x, c.y);
  }
  static __device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
  static __host__ __device__ __forceinline__ float2 one() { return make_float2(1.f, 0.f); }
};

__device__ __forceinline__ float scale_x(float alpha, float x) { return alpha * x; }
__device__ __forceinline__ double scale_x(double alpha, double x) { return alpha * x; }
__device__ __forceinline__ double2 scale_x(double2 alpha, double2 x) {
  return make_double2(alpha.x * x.x - alpha.y * x.y, alpha.x * x.y + alpha.y * x.x);
}
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
  constexpr bool kSym = ModeT<kMode>::kSym;
  constexpr bool kRow = ModeT<kMode>::kRow;
  constexpr bool kCol = ModeT<kMode>::kCol;
  // tile[c][r] = element (row r, col c); dynamic, as complex128 tiles pass 48 KB
  extern __shared__ __align__(16) unsigned char tile_raw[];
  T(*tile)[kT + 1] = reinterpret_cast<T(*)[kT + 1]>(tile_raw);
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
          if (ModeT<kMode>::kTr && unit) tile[cc][rr] = Cx<T>::one();
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
    if (kCol && (!diag || ModeT<kMode>::kColOnly)) {
#pragma unroll
      for (int rr = q * 16; rr < q * 16 + 16; ++rr) {
        T a = tile[r][rr];
        Cx<T>::mac(colacc, ModeT<kMode>::kConjCol ? Cx<T>::conj(a) : a, vI[rr]);
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
__device__ __forceinline__ double beta_apply(double beta, double y) {
  return beta == 0.0 ? 0.0 : (beta != 1.0 ? y * beta : y);
}
__device__ __forceinline__ double2 beta_apply(double2 beta, double2 y) {
  if (beta.x == 0.0 && beta.y == 0.0) return make_double2(0.0, 0.0);
  if (beta.x == 1.0 && beta.y == 0.0) return y;
  return make_double2(y.x * beta.x - y.y * beta.y, y.x * beta.y + y.y * beta.x);
}
__device__ __forceinline__ float2 beta_apply(float2 beta, float2 y) {
  if (beta.x == 0.f && beta.y == 0.f) return make_float2(0.f, 0.f);
  if (beta.x == 1.f && beta.y == 0.f) return y;
  return make_float2(y.x * beta.x - y.y * beta.y, y.x * beta.y + y.y * beta.x);
}

// ---- register-resident off-diagonal pass ----------------------------------------
// kC = 64 columns per tile column (the diagonal tile width).  A warp owns a
// strip of 32*V rows: each lane V consecutive rows, loaded as one 16-byte
// vector per column (V = 4 floats or 2 complex; V = 1 when lda or the base
// are not 16-byte aligned), so a warp load covers a 512-byte contiguous
// segment of a column.  Columns are taken kP per pass to bound registers.
// Strips sit on a global grid of 32*V-row strips; rows outside this column
// block's stored off-diagonal range [row_lo, row_hi) are masked out.
constexpr int kC = 64;
constexpr int kStripWarps = 4;

template <typename T>
__device__ __forceinline__ T shfl_xor_t(T v, int o);
template <> __device__ __forceinline__ float shfl_xor_t<float>(float v, int o) {
  return __shfl_xor_sync(0xffffffffu, v, o);
}
template <> __device__ __forceinline__ double shfl_xor_t<double>(double v, int o) {
  return __shfl_xor_sync(0xffffffffu, v, o);
}
template <> __device__ __forceinline__ double2 shfl_xor_t<double2>(double2 v, int o) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}
template <> __device__ __forceinline__ float2 shfl_xor_t<float2>(float2 v, int o) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}

// The value of lane `src`, for each type.
__device__ __forceinline__ float shfl_idx_t(float v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ double shfl_idx_t(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ float2 shfl_idx_t(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ double2 shfl_idx_t(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
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

template <typename T, int V> struct Vec;
template <> struct Vec<float, 4> {
  using type = float4;
  static __device__ __forceinline__ void split(const float4& v, float (&o)[4]) { o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w; }
};
template <> struct Vec<double, 2> {
  using type = double2;
  static __device__ __forceinline__ void split(const double2& v, double (&o)[2]) { o[0] = v.x; o[1] = v.y; }
};
template <> struct Vec<float2, 2> {
  using type = float4;
  static __device__ __forceinline__ void split(const float4& v, float2 (&o)[2]) { o[0] = make_float2(v.x, v.y); o[1] = make_float2(v.z, v.w); }
};

template <typename T, int kMode, int V>
__global__ void __launch_bounds__(32 * kStripWarps, sizeof(T) >= 16 ? 3 : 4)
k_tri_strips(int n, const T* __restrict__ A, size_t lda, const T* __restrict__ x, size_t incx,
             T alpha, bool lower, T* __restrict__ rowpart, T* __restrict__ colpart, int nsplit) {
  constexpr int kS = 32 * V;                 // strip height
  constexpr int kP = 16;                     // columns per pass
  constexpr bool kSym = ModeT<kMode>::kSym;
  constexpr bool kRow = ModeT<kMode>::kRow;
  constexpr bool kCol = ModeT<kMode>::kCol;
  __shared__ T vJ[kC];
  __shared__ T red[kStripWarps][kC];
  const int J = blockIdx.x;
  const int c0 = J * kC;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row_lo = lower ? c0 + kC : 0;
  const int row_hi = lower ? n : c0;
  const int s_lo = row_lo / kS;
  const int s_hi = row_hi > row_lo ? (row_hi + kS - 1) / kS : s_lo;
  // A CTA past its column's last strip leaves at once: it writes no partial
  // (the combine reads only the splits that hold strips).
  if (s_lo + (int)blockIdx.y * kStripWarps >= s_hi) return;
  if (threadIdx.x < kC) {
    const int gc = c0 + threadIdx.x;
    T v = gc < n ? x[(size_t)gc * incx] : Cx<T>::zero();
    vJ[threadIdx.x] = kSym ? scale_x(alpha, v) : v;
  }
  for (int i = threadIdx.x; i < kStripWarps * kC; i += blockDim.x) (&red[0][0])[i] = Cx<T>::zero();
  __syncthreads();
  // One strip per warp (the grid has enough warps for the longest column).
  const int gs = s_lo + blockIdx.y * kStripWarps + warp;
  if (gs < s_hi) {
    const int r0 = gs * kS + lane * V;      // first row of this lane
    bool rv[V];
    T xi[V];
#pragma unroll
    for (int e = 0; e < V; ++e) {
      const int r = r0 + e;
      rv[e] = r >= row_lo && r < row_hi;
      xi[e] = Cx<T>::zero();
      if (kCol && rv[e]) {
        xi[e] = x[(size_t)r * incx];
        if (kSym) xi[e] = scale_x(alpha, xi[e]);
      }
    }
    const bool all_in = V > 1 && rv[0] && rv[V - 1];
    T racc[V];
#pragma unroll
    for (int e = 0; e < V; ++e) racc[e] = Cx<T>::zero();
#pragma unroll 1
    for (int h0 = 0; h0 < kC; h0 += kP) {
      T a[kP][V];
      const T* base = A + r0 + (size_t)(c0 + h0) * lda;
      if constexpr (V > 1) {
        using VT = typename Vec<T, V>::type;
        if (all_in) {
          VT raw[kP];
#pragma unroll
          for (int c = 0; c < kP; ++c)
            raw[c] = (c0 + h0 + c < n) ? __ldcs(reinterpret_cast<const VT*>(base + (size_t)c * lda)) : VT{};
#pragma unroll
          for (int c = 0; c < kP; ++c) Vec<T, V>::split(raw[c], a[c]);
        } else {
#pragma unroll
          for (int c = 0; c < kP; ++c)
#pragma unroll
            for (int e = 0; e < V; ++e)
              a[c][e] = (rv[e] && c0 + h0 + c < n) ? __ldcs(base + (size_t)c * lda + e) : Cx<T>::zero();
        }
      } else {
#pragma unroll
        for (int c = 0; c < kP; ++c)
          a[c][0] = (rv[0] && c0 + h0 + c < n) ? __ldcs(base + (size_t)c * lda) : Cx<T>::zero();
      }
      if (kRow) {
#pragma unroll
        for (int c = 0; c < kP; ++c)
#pragma unroll
          for (int e = 0; e < V; ++e) Cx<T>::mac(racc[e], a[c][e], vJ[h0 + c]);
      }
      if (kCol) {
        // per-lane column partials of this pass, reduced across the warp now:
        // butterfly 16 -> 1 values per lane, then a final pairwise add; lane l
        // (even) ends with the sum for column h0 + (l >> 1).
        T v[kP];
#pragma unroll
        for (int c = 0; c < kP; ++c) {
          v[c] = Cx<T>::zero();
#pragma unroll
          for (int e = 0; e < V; ++e)
            Cx<T>::mac(v[c], ModeT<kMode>::kConjCol ? Cx<T>::conj(a[c][e]) : a[c][e], xi[e]);
        }
        butterfly<8>(v, lane, 16);
        butterfly<4>(v, lane, 8);
        butterfly<2>(v, lane, 4);
        butterfly<1>(v, lane, 2);
        const T tot = Cx<T>::add(v[0], shfl_xor_t(v[0], 1));
        if ((lane & 1) == 0) red[warp][h0 + (lane >> 1)] = tot;
      }
    }
    if (kRow) {
      T* rp = rowpart + ((size_t)gs * gridDim.x + J) * kS + lane * V;
#pragma unroll
      for (int e = 0; e < V; ++e) rp[e] = rv[e] ? racc[e] : Cx<T>::zero();
    }
  }
  if (kCol) {
    __syncthreads();
    if (threadIdx.x < kC) {
      T s = red[0][threadIdx.x];
#pragma unroll
      for (int w2 = 1; w2 < kStripWarps; ++w2) s = Cx<T>::add(s, red[w2][threadIdx.x]);
      colpart[((size_t)J * nsplit + blockIdx.y) * kC + threadIdx.x] = s;
    }
  }
  // This CTA's share is written: the combine grid may start launching (its
  // griddepcontrol.wait still waits for the whole of this grid).
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---- TMA-fed persistent pass ------------------------------------------------------
// One launch for the whole stored triangle (off-diagonal strips and diagonal
// blocks), for matrices a tensor map can describe.  A unit is the kS x 64 block of rows
// [s*kS, s*kS + kS) and columns [J*64, J*64 + 64), kS = 32 * (16 / sizeof(T)):
// 32 KB for every type.  One CTA per SM takes an equal share of the units,
// numbered in column-block order (equal-sized units, so the static share is
// balanced to one unit); its producer thread loads each unit with
// TMA into a kTsStages-deep ring.  Two groups of four consumer warps take
// alternate units, so one group's reductions overlap the other's; in a group,
// warp w reduces columns [16w, 16w + 16): lane l holds rows l*V .. l*V + V - 1
// of each column (one conflict-free 16-byte shared load per column), forms the
// row part over its 16 columns and the column part of its 16 columns
// (butterfly across the lanes, as in k_tri_strips); the four warps' row parts
// are added in shared memory in warp order.  The x values of a group's next
// unit are loaded while it reduces the current one.  Column block J's units
// are the strips meeting its stored rows including its diagonal block (upper:
// rows [0, J*64 + 64); lower: rows [J*64, n)).  Each stored element (r, c)
// with r != c adds A(r, c) x(c) to the row part of r and, for SYMV / HEMV,
// conj?(A(r, c)) x(r) to the column part of c; the diagonal element adds once
// (a_jj, Re(a_jj) for HEMV, 1 for a unit TRMV), to the row part or, for TRMV
// T / C, to the column part.  Unstored elements are masked with a select (the
// unstored triangle may hold NaN); rows and columns past n are zero-filled by
// TMA.  Column parts are kept per (J, s) unit.  Every wait is bounded: a
// give-up sets the status word and the CTA drains.
constexpr int kTsStages = 4;
constexpr int kTsConsumers = 4;   // warps per consumer group
constexpr int kTsGroups = 2;
constexpr int kTsThreads = 32 * (1 + kTsGroups * kTsConsumers);
constexpr int kTsCtasPerSm = 1;
constexpr int kTsBoxCols = 64;   // columns per TMA copy (a unit takes kC / kTsBoxCols copies)
// 1: each CTA takes a contiguous run of units (it streams its column blocks
// top to bottom); 0: units are dealt round-robin across the CTAs.
constexpr int kTsContiguous = 1;

// The units of CTA b of g: count, and the i-th one.
struct UnitShare {
  int first, count, stride;
  __device__ __forceinline__ UnitShare(int total, int b, int g) {
    if (kTsContiguous) {
      const int per = total / g, rem = total % g;
      first = b * per + min(b, rem);
      count = per + (b < rem ? 1 : 0);
      stride = 1;
    } else {
      first = b;
      count = b < total ? (total - b + g - 1) / g : 0;
      stride = g;
    }
  }
  __device__ __forceinline__ int unit(int i) const { return first + i * stride; }
};

// Strips [s_lo, s_hi) holding column block J's stored rows, its diagonal
// block included: the units of block J in the TMA-fed pass.
__host__ __device__ __forceinline__ void strip_range_fold(int J, int n, int kS, bool lower, int& s_lo,
                                                          int& s_hi) {
  const int c0 = J * kC;
  const int row_lo = lower ? c0 : 0;
  const int row_hi = lower ? n : min(c0 + kC, n);
  s_lo = row_lo / kS;
  s_hi = row_hi > row_lo ? (row_hi + kS - 1) / kS : s_lo;
}

// Walks the units of one CTA (or consumer group) in increasing order: unit u
// lies in column block J, whose units are base .. base + cnt - 1 and start at
// strip s_lo.  Each walker passes over the column blocks once in all.
struct UnitWalk {
  int J = 0, base = 0, cnt = 0, s_lo = 0;
  __device__ __forceinline__ void start(int n, int kS, bool lower) {
    int hi;
    strip_range_fold(0, n, kS, lower, s_lo, hi);
    cnt = hi - s_lo;
  }
  // -> strip of unit u; J names its column block
  __device__ __forceinline__ int seek(int u, int n, int kS, bool lower) {
    while (u >= base + cnt) {
      base += cnt;
      ++J;
      int hi;
      strip_range_fold(J, n, kS, lower, s_lo, hi);
      cnt = hi - s_lo;
    }
    return s_lo + (u - base);
  }
};

template <typename T> struct TsVec { using type = T; };
template <> struct TsVec<float> { using type = float4; };
template <> struct TsVec<double> { using type = double2; };
template <> struct TsVec<float2> { using type = float4; };

template <typename T, int V>
__device__ __forceinline__ void ts_split(const typename TsVec<T>::type& raw, T (&o)[V]) {
  if constexpr (V == 1) {
    o[0] = raw;
  } else {
    Vec<T, V>::split(raw, o);
  }
}

// One consumer lane's view of a unit: where it is and the x values it needs.
template <typename T, int V>
struct UnitX {
  int J, gs;
  int row_lo, row_hi;   // the block's stored rows, its diagonal block included
  bool diag;            // the strip meets the diagonal block: classify each element
  bool rv[V];           // lane's row is a stored off-diagonal row (the rule when !diag)
  T xi[V];              // x of the lane's rows (column part)
  T vj;                 // x of column cw * 16 + lane (row part), lanes 0..15
};

template <typename T, int kMode, int V>
__device__ __forceinline__ void unit_x(UnitWalk& w, int u, int n, bool lower, const T* __restrict__ x,
                                       size_t incx, int cw, int lane, UnitX<T, V>& o) {
  constexpr int kS = 32 * V;
  constexpr int kP = kC / kTsConsumers;
  o.gs = w.seek(u, n, kS, lower);
  o.J = w.J;
  const int c0 = o.J * kC;
  o.row_lo = lower ? c0 : 0;
  o.row_hi = lower ? n : min(c0 + kC, n);
  o.diag = o.gs * kS < c0 + kC && o.gs * kS + kS > c0;
  const int off_lo = lower ? c0 + kC : 0, off_hi = lower ? n : c0;
  const int r0 = o.gs * kS + lane * V;
#pragma unroll
  for (int e = 0; e < V; ++e) {
    const int r = r0 + e;
    o.rv[e] = r >= off_lo && r < off_hi;
    o.xi[e] = Cx<T>::zero();
    if (ModeT<kMode>::kCol && r >= o.row_lo && r < o.row_hi) o.xi[e] = x[(size_t)r * incx];
  }
  o.vj = Cx<T>::zero();
  if (ModeT<kMode>::kRow && lane < kP) {
    const int gc = c0 + cw * kP + lane;
    if (gc < n) o.vj = x[(size_t)gc * incx];
  }
}

// Element weights of a unit: what element (row rb + e, column cb + c) with
// value a adds to the row part (row) and to the column part (col).
// Off-diagonal strips: the stored off-diagonal rows, others masked.
template <typename T, int V>
struct PlainWeight {
  const bool (&rv)[V];
  __device__ __forceinline__ T row(int, int e, T a) const { return rv[e] ? a : Cx<T>::zero(); }
  __device__ __forceinline__ T col(int, int e, T a) const { return rv[e] ? a : Cx<T>::zero(); }
};
// Strips meeting the diagonal block: the strict triangle (r < c upper, r > c
// lower) adds to both parts; the diagonal adds a_jj (Re(a_jj) for HEMV, 1 for
// a unit TRMV) once, to the column part for TRMV T / C, else to the row part.
template <typename T, int kMode>
struct DiagWeight {
  int rb, cb, n;
  bool lower, unit;
  __device__ __forceinline__ bool strict(int r, int c) const { return lower ? (r > c && r < n) : r < c; }
  __device__ __forceinline__ T dval(T a) const {
    if (kMode == kHemv) return Cx<T>::re(a);
    if (ModeT<kMode>::kTr && unit) return Cx<T>::one();
    return a;
  }
  __device__ __forceinline__ T row(int c, int e, T a) const {
    const int r = rb + e, cc = cb + c;
    return strict(r, cc) ? a : (r == cc && !ModeT<kMode>::kColOnly) ? dval(a) : Cx<T>::zero();
  }
  __device__ __forceinline__ T col(int c, int e, T a) const {
    const int r = rb + e, cc = cb + c;
    return strict(r, cc) ? a : (r == cc && ModeT<kMode>::kColOnly) ? dval(a) : Cx<T>::zero();
  }
};

// A warp's share of a unit: row part into racc (this lane's V rows over the
// warp's kP columns), column part of the kP columns into colpart.
template <typename T, int kMode, int V, int kP, typename W>
__device__ __forceinline__ void reduce_unit(const T (&a)[kP][V], const W& w, const UnitX<T, V>& cur,
                                            T alpha, int lane, T (&racc)[V], T* __restrict__ colpart, int nstrips,
                                            int cw) {
  constexpr bool kSym = ModeT<kMode>::kSym;
  if (ModeT<kMode>::kRow) {
    const T vjs = kSym ? scale_x(alpha, cur.vj) : cur.vj;
#pragma unroll
    for (int c = 0; c < kP; ++c) {
      const T vc = shfl_idx_t(vjs, c);
#pragma unroll
      for (int e = 0; e < V; ++e) Cx<T>::mac(racc[e], w.row(c, e, a[c][e]), vc);
    }
  }
  if (ModeT<kMode>::kCol) {
    T xs[V];
#pragma unroll
    for (int e = 0; e < V; ++e) xs[e] = kSym ? scale_x(alpha, cur.xi[e]) : cur.xi[e];
    T v[kP];
#pragma unroll
    for (int c = 0; c < kP; ++c) {
      v[c] = Cx<T>::zero();
#pragma unroll
      for (int e = 0; e < V; ++e) {
        const T wa = w.col(c, e, a[c][e]);
        Cx<T>::mac(v[c], ModeT<kMode>::kConjCol ? Cx<T>::conj(wa) : wa, xs[e]);
      }
    }
    butterfly<8>(v, lane, 16);
    butterfly<4>(v, lane, 8);
    butterfly<2>(v, lane, 4);
    butterfly<1>(v, lane, 2);
    const T tot = Cx<T>::add(v[0], shfl_xor_t(v[0], 1));
    if ((lane & 1) == 0) colpart[((size_t)cur.J * nstrips + cur.gs) * kC + cw * kP + (lane >> 1)] = tot;
  }
}

template <typename T, int kMode>
__global__ void __launch_bounds__(kTsThreads, kTsCtasPerSm)
k_tri_strips_tma(const __grid_constant__ CUtensorMap map, int n, const T* __restrict__ x, size_t incx,
                 T alpha, bool lower, bool unit, int total, T* __restrict__ rowpart, T* __restrict__ colpart,
                 unsigned* status, uint64_t limit_ns) {
  constexpr int V = 16 / (int)sizeof(T);
  constexpr int kS = 32 * V;
  constexpr int kP = kC / kTsConsumers;              // columns per consumer warp
  constexpr uint32_t kUnitBytes = kS * kC * sizeof(T);
  constexpr int kMapPerElem = sizeof(T) > 8 ? 2 : 1;   // map elements per T
  constexpr bool kRow = ModeT<kMode>::kRow;
  using VT = typename TsVec<T>::type;
  extern __shared__ __align__(128) uint8_t ts_raw[];
  uint8_t* ring = ts_raw + ((128u - (tc::smem_u32(ts_raw) & 127u)) & 127u);  // stays in the shared window
  __shared__ __align__(8) uint64_t full_bar[kTsStages], empty_bar[kTsStages];
  __shared__ __align__(16) T red[kTsGroups][2][kTsConsumers][kS];
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ncol = (n + kC - 1) / kC;
  const int nstrips = (n + kS - 1) / kS;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kTsStages; ++s) {
      tc::mbar_init(&full_bar[s], 1);
      tc::mbar_init(&empty_bar[s], kTsConsumers);
    }
    abort_flag = 0;
    tc::fence_mbar_init();
  }
  __syncthreads();
  UnitWalk walk;
  walk.start(n, kS, lower);

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer ----
      tc::prefetch_tmap(&map);
      const UnitShare share(total, blockIdx.x, gridDim.x);
      int i = 0;
      for (; i < share.count; ++i) {
        const int u = share.unit(i);
        const int st = i % kTsStages;
        if (i >= kTsStages && !tc::mbar_wait(&empty_bar[st], ((i / kTsStages) - 1) & 1, limit_ns)) {
          atomicOr(status, kStatusTimeout);
          atomicExch(&abort_flag, 1);
          break;
        }
        if (*(volatile int*)&abort_flag) break;
        const int gs = walk.seek(u, n, kS, lower);
        tc::mbar_expect_tx(&full_bar[st], kUnitBytes);
#pragma unroll
        for (int b = 0; b < kC / kTsBoxCols; ++b)
          tc::tma_load_2d(ring + (size_t)st * kUnitBytes + (size_t)b * kS * kTsBoxCols * sizeof(T), &map,
                          &full_bar[st], gs * kS * kMapPerElem, walk.J * kC + b * kTsBoxCols);
      }
      // every issued copy lands before the CTA may exit
      for (int j = (i > kTsStages ? i - kTsStages : 0); j < i; ++j)
        tc::mbar_wait(&full_bar[j % kTsStages], (j / kTsStages) & 1, 1000000000ull);
    }
  } else {
    // ---- consumers: group cg takes the CTA's units cg, cg + 2, ...; warp cw
    // of the group takes columns [cw * kP, cw * kP + kP) of each ----
    const int cg = (warp - 1) / kTsConsumers;
    const int cw = (warp - 1) % kTsConsumers;
    const int ct = (warp - 1 - cg * kTsConsumers) * 32 + lane;  // 0 .. 127 within the group
    const UnitShare share(total, blockIdx.x, gridDim.x);
    UnitX<T, V> nx;
    if (cg < share.count) unit_x<T, kMode, V>(walk, share.unit(cg), n, lower, x, incx, cw, lane, nx);
    for (int i = cg, k = 0; i < share.count; i += kTsGroups, ++k) {
      const UnitX<T, V> cur = nx;
      if (i + kTsGroups < share.count)
        unit_x<T, kMode, V>(walk, share.unit(i + kTsGroups), n, lower, x, incx, cw, lane, nx);
      const int st = i % kTsStages;
      bool ok = !*(volatile int*)&abort_flag;
      if (ok && !tc::mbar_wait(&full_bar[st], (i / kTsStages) & 1, limit_ns)) {
        atomicOr(status, kStatusTimeout);
        atomicExch(&abort_flag, 1);
        ok = false;
      }
      T racc[V];
#pragma unroll
      for (int e = 0; e < V; ++e) racc[e] = Cx<T>::zero();
      if (ok) {
        const T* tile = reinterpret_cast<const T*>(ring + (size_t)st * kUnitBytes);
        T a[kP][V];
#pragma unroll
        for (int c = 0; c < kP; ++c) {
          const VT raw = *reinterpret_cast<const VT*>(tile + (size_t)(cw * kP + c) * kS + lane * V);
          ts_split<T, V>(raw, a[c]);
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty_bar[st]);
        if (cur.diag) {
          const DiagWeight<T, kMode> w{cur.gs * kS + lane * V, cur.J * kC + cw * kP, n, lower, unit};
          reduce_unit<T, kMode, V, kP>(a, w, cur, alpha, lane, racc, colpart, nstrips, cw);
        } else {
          const PlainWeight<T, V> w{cur.rv};
          reduce_unit<T, kMode, V, kP>(a, w, cur, alpha, lane, racc, colpart, nstrips, cw);
        }
      }
      if (kRow) {
        // row part: the group's four partials added in warp order (the buffer
        // alternates with the unit, so one barrier per unit suffices)
#pragma unroll
        for (int e = 0; e < V; ++e) red[cg][k & 1][cw][lane * V + e] = racc[e];
        asm volatile("bar.sync %0, %1;" ::"r"(1 + cg), "n"(32 * kTsConsumers) : "memory");
        if (ok && ct < kS) {
          T t = Cx<T>::add(Cx<T>::add(red[cg][k & 1][0][ct], red[cg][k & 1][1][ct]),
                           Cx<T>::add(red[cg][k & 1][2][ct], red[cg][k & 1][3][ct]));
          const int r = cur.gs * kS + ct;
          if (r < cur.row_lo || r >= cur.row_hi) t = Cx<T>::zero();
          rowpart[((size_t)cur.gs * ncol + cur.J) * kS + ct] = t;
        }
      }
    }
  }
  // this CTA's share is written: the combine grid may start launching
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Per 32 output rows: y = beta*y (or 0 for TRMV) + row parts of every
// off-diagonal column block + the diagonal block's parts + column parts.
// 8 groups of 32 threads (lane = row) split the column blocks; a group loads
// up to 16 of its partials at once (one L2 round trip covers 128 column
// blocks, n = 8192) and adds them in a fixed tree order, then a fixed-order
// shared-memory sum across the groups.
constexpr int kCombineGroups = 8;
constexpr int kCombineBatch = 16;

template <typename T, int N>
__device__ __forceinline__ T tree_sum(T (&a)[N]) {
#pragma unroll
  for (int w = N / 2; w >= 1; w /= 2)
#pragma unroll
    for (int u = 0; u < w; ++u) a[u] = Cx<T>::add(a[u], a[u + w]);
  return a[0];
}
template <typename T, int kMode, int V>
__global__ void __launch_bounds__(32 * kCombineGroups)
k_strip_combine(int n, T beta, T* __restrict__ y, size_t incy, bool lower,
                const T* __restrict__ rowpart, const T* __restrict__ colpart, int ncolblk,
                int nsplit, int folded, const T* __restrict__ drow, const T* __restrict__ dcol) {
  constexpr int kS = 32 * V;
  constexpr bool kRow = ModeT<kMode>::kRow;
  constexpr bool kCol = ModeT<kMode>::kCol;
  __shared__ T part[kCombineGroups][32];
  // Launched as a programmatic dependent of k_tri_strips: wait until that
  // grid has completed and its writes are visible (a no-op when launched
  // without the dependency).
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int g = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gr = blockIdx.x * 32 + lane;
  const int gs = gr / kS, li = gr % kS;   // strip and row within it
  const int Jr = min(gr, n - 1) / kC;
  T s = Cx<T>::zero();
  if (kRow) {
    // column blocks whose stored range covers row gr: the off-diagonal ones,
    // and with the layout of k_tri_strips_tma (folded) block Jr itself
    const int j0 = lower ? 0 : (folded ? Jr : Jr + 1), j1 = lower ? (folded ? Jr + 1 : Jr) : ncolblk;
    const T* rp = rowpart + (size_t)gs * ncolblk * kS + li;
    for (int Jb = j0 + g; Jb < j1; Jb += kCombineBatch * kCombineGroups) {
      T a[kCombineBatch];
#pragma unroll
      for (int u = 0; u < kCombineBatch; ++u) {
        const int J = Jb + u * kCombineGroups;
        a[u] = J < j1 ? __ldcs(rp + (size_t)J * kS) : Cx<T>::zero();
      }
      s = Cx<T>::add(s, tree_sum(a));
    }
  }
  if (kCol) {
    // column parts of block Jr: one per CTA split (k_tri_strips), or one per
    // stored strip [q_lo, q_hi) of the block, its diagonal block included
    // (k_tri_strips_tma, nsplit = strips)
    int q_lo = 0, q_hi = nsplit;
    if (folded) {
      strip_range_fold(Jr, n, kS, lower, q_lo, q_hi);
    } else {
      // the splits of column block Jr that hold strips (k_tri_strips)
      const int c0 = Jr * kC;
      const int row_lo = lower ? c0 + kC : 0, row_hi = lower ? n : c0;
      const int s_lo = row_lo / kS;
      const int s_hi = row_hi > row_lo ? (row_hi + kS - 1) / kS : s_lo;
      q_hi = min(nsplit, (s_hi - s_lo + kStripWarps - 1) / kStripWarps);
    }
    const T* cp = colpart + (size_t)Jr * nsplit * kC + gr % kC;
    for (int qb = q_lo + g; qb < q_hi; qb += kCombineBatch * kCombineGroups) {
      T a[kCombineBatch];
#pragma unroll
      for (int u = 0; u < kCombineBatch; ++u) {
        const int q = qb + u * kCombineGroups;
        a[u] = q < q_hi ? cp[(size_t)q * kC] : Cx<T>::zero();
      }
      s = Cx<T>::add(s, tree_sum(a));
    }
  }
  part[g][lane] = s;
  __syncthreads();
  if (g != 0 || gr >= n) return;
  T t = part[0][lane];
#pragma unroll
  for (int q = 1; q < kCombineGroups; ++q) t = Cx<T>::add(t, part[q][lane]);
  if (!folded) {
    if (kRow) t = Cx<T>::add(t, drow[gr]);
    if (ModeT<kMode>::kColOnly) t = Cx<T>::add(t, dcol[gr]);
  }
  T* yp = y + (size_t)gr * incy;
  if (ModeT<kMode>::kTr) *yp = t;
  else *yp = Cx<T>::add(beta_apply(beta, *yp), t);
}

template <typename T, int kMode, int V>
coral_status_t launch_strips(Handle* h, int n, const T* A, size_t lda, const T* x, size_t incx,
                             T alpha, T beta, T* y, size_t incy, bool lower, bool unit) {
  constexpr int kS = 32 * V;
  const int ncol = (n + kC - 1) / kC;
  const int nstrips = (n + kS - 1) / kS;
  // CTAs per column block: one strip per warp in the longest column, so no
  // warp streams more than one strip (CTAs past a short column's end exit)
  int nsplit = (nstrips + kStripWarps - 1) / kStripWarps;
  nsplit = nsplit < 1 ? 1 : (nsplit > 256 ? 256 : nsplit);
  const size_t rp = (size_t)nstrips * ncol * kS;
  const size_t cp = (size_t)ncol * nsplit * kC;
  const int NT = (n + kT - 1) / kT;  // diagonal tiles (kT == kC)
  const size_t dlen = (size_t)NT * kT;
  T* sc = static_cast<T*>(scratch(h, (rp + cp + 2 * dlen) * sizeof(T)));
  if (!sc) return CORAL_ERR_ALLOC;
  T* drow = sc + rp + cp;
  T* dcol = drow + dlen;
  // The diagonal tiles are independent of the strips: run them on the
  // handle's side stream, forked from and joined back into the main stream.
  CORAL_CUDA(h, cudaEventRecord(h->fork_event, h->stream));
  CORAL_CUDA(h, cudaStreamWaitEvent(h->side_stream, h->fork_event, 0));
  constexpr size_t kTileSmem = (size_t)kT * (kT + 1) * sizeof(T);
  if (kTileSmem > 48 * 1024) {
    static uint64_t attr_devices = 0;  // bit d: attribute set on device d
    const uint64_t bit = h->device < 64 ? (1ull << h->device) : 0;
    if (!(attr_devices & bit) || !bit) {
      CORAL_CUDA(h, cudaFuncSetAttribute(k_tri_tiles<T, kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTileSmem));
      attr_devices |= bit;
    }
  }
  k_tri_tiles<T, kMode><<<dim3(NT, 1), kTriThreads, kTileSmem, h->side_stream>>>(n, A, lda, x, incx, alpha,
                                                                         lower, unit, drow, dcol, 1, 1);
  coral_status_t s = launch_status(h);
  if (s != CORAL_OK) return s;
  CORAL_CUDA(h, cudaEventRecord(h->join_event, h->side_stream));
  timed_begin(h);
  k_tri_strips<T, kMode, V><<<dim3(ncol, nsplit), 32 * kStripWarps, 0, h->stream>>>(
      n, A, lda, x, incx, alpha, lower, sc, sc + rp, nsplit);
  s = launch_status(h);
  timed_end(h);
  if (s != CORAL_OK) return s;
  CORAL_CUDA(h, cudaStreamWaitEvent(h->stream, h->join_event, 0));
  // Programmatic dependent launch: the combine's CTAs are scheduled as the
  // strips grid drains instead of after it has fully retired.
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((n + 31) / 32);
  cfg.blockDim = dim3(32 * kCombineGroups);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CORAL_CUDA(h, cudaLaunchKernelEx(&cfg, k_strip_combine<T, kMode, V>, n, beta, y, incy, lower,
                                   static_cast<const T*>(sc), static_cast<const T*>(sc + rp), ncol, nsplit, 0,
                                   static_cast<const T*>(drow), static_cast<const T*>(dcol)));
  return launch_status(h);
}

// TMA-fed form, one launch over the whole stored triangle plus the combine:
// returns CORAL_ERR_NOT_SUPPORTED, having enqueued nothing, when the matrix
// cannot be described by a tensor map (the caller then takes the
// register-streaming form).
template <typename T, int kMode>
coral_status_t launch_strips_tma(Handle* h, int n, const T* A, size_t lda, const T* x, size_t incx,
                                 T alpha, T beta, T* y, size_t incy, bool lower, bool unit) {
  constexpr int V = 16 / (int)sizeof(T);
  constexpr int kS = 32 * V;
  constexpr int kMapElem = sizeof(T) > 8 ? 8 : (int)sizeof(T);
  constexpr int kMapPerElem = (int)sizeof(T) / kMapElem;
  constexpr size_t kSmem = (size_t)kTsStages * kS * kC * sizeof(T) + 128;
  if (!aligned16(A) || (lda * sizeof(T)) % 16) return CORAL_ERR_NOT_SUPPORTED;
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  if (!encode_kmajor_map(&map, A, kMapElem, (uint64_t)n * kMapPerElem, (uint64_t)n, lda * sizeof(T),
                         (uint32_t)(kS * kMapPerElem), (uint32_t)kTsBoxCols, 0))
    return CORAL_ERR_NOT_SUPPORTED;
  const int ncol = (n + kC - 1) / kC;
  const int nstrips = (n + kS - 1) / kS;
  int total = 0;
  for (int J = 0; J < ncol; ++J) {
    int lo, hi;
    strip_range_fold(J, n, kS, lower, lo, hi);
    total += hi - lo;
  }
  const size_t rp = (size_t)nstrips * ncol * kS;
  const size_t cp = (size_t)ncol * nstrips * kC;
  T* sc = static_cast<T*>(scratch(h, (rp + cp) * sizeof(T)));
  if (!sc) return CORAL_ERR_ALLOC;
  static uint64_t attr_devices = 0;  // bit d: attribute set on device d
  const uint64_t bit = h->device < 64 ? (1ull << h->device) : 0;
  if (!(attr_devices & bit) || !bit) {
    CORAL_CUDA(h, cudaFuncSetAttribute(k_tri_strips_tma<T, kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmem));
    attr_devices |= bit;
  }
  const int slots = h->sm_count * kTsCtasPerSm;
  const int grid = total < slots ? total : slots;   // n >= 1: every block has its diagonal unit
  timed_begin(h);
  k_tri_strips_tma<T, kMode><<<grid, kTsThreads, kSmem, h->stream>>>(
      map, n, x, incx, alpha, lower, unit, total, sc, sc + rp, &h->words->status, h->wait_limit * 32ull);
  coral_status_t s = launch_status(h);
  timed_end(h);
  if (s != CORAL_OK) return s;
  // Programmatic dependent launch: the combine's CTAs are scheduled as the
  // pass drains instead of after it has fully retired.
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((n + 31) / 32);
  cfg.blockDim = dim3(32 * kCombineGroups);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CORAL_CUDA(h, cudaLaunchKernelEx(&cfg, k_strip_combine<T, kMode, V>, n, beta, y, incy, lower,
                                   static_cast<const T*>(sc), static_cast<const T*>(sc + rp), ncol, nstrips, 1,
                                   static_cast<const T*>(nullptr), static_cast<const T*>(nullptr)));
  return launch_status(h);
}

template <typename T, int kMode>
coral_status_t run_tri_strips(Handle* h, int n, const T* A, size_t lda, const T* x, size_t incx,
                              T alpha, T beta, T* y, size_t incy, bool lower, bool unit) {
  static_assert(kC == kT, "diagonal tiles are as wide as the tile columns");
  constexpr int V = (int)(16 / sizeof(T));  // one 16-byte vector per lane and column
  const bool vec = aligned16(A) && (lda * sizeof(T)) % 16 == 0;
  if (vec && h->tri_tma) {
    const coral_status_t s = launch_strips_tma<T, kMode>(h, n, A, lda, x, incx, alpha, beta, y, incy, lower, unit);
    if (s != CORAL_ERR_NOT_SUPPORTED) return s;
  }
  if (vec) return launch_strips<T, kMode, V>(h, n, A, lda, x, incx, alpha, beta, y, incy, lower, unit);
  return launch_strips<T, kMode, 1>(h, n, A, lda, x, incx, alpha, beta, y, incy, lower, unit);
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
    return run_tri_strips<float, kTrmvN>(H, (int)n, matrix, lda, x, incx, 1.f, 0.f, x, incx, lower, unit);
  return run_tri_strips<float, kTrmvT>(H, (int)n, matrix, lda, x, incx, 1.f, 0.f, x, incx, lower, unit);
}

// dsymv.rs:99-210: the ssymv order in double.
coral_status_t coral_dsymv(coral_handle_t hh, int uplo, size_t n, double alpha, const double* matrix,
                           size_t lda, const double* x, size_t incx, double beta, double* y,
                           size_t incy) {
  CORAL_HANDLE(hh);
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (n == 0) return CORAL_OK;                          // dsymv.rs:112
  if (alpha == 0.0 && beta == 1.0) return CORAL_OK;     // dsymv.rs:113
  if (!matrix) return bad_arg(H, 4);
  if (lda < n) return bad_arg(H, 5);
  if (!x) return bad_arg(H, 6);
  if (incx == 0) return bad_arg(H, 7);
  if (!y) return bad_arg(H, 9);
  if (incy == 0) return bad_arg(H, 10);
  if (((uintptr_t)matrix | (uintptr_t)x | (uintptr_t)y) & 7) return bad_arg(H, 4);
  if (n > (size_t)(1 << 20)) return CORAL_ERR_NOT_SUPPORTED;
  return run_tri_strips<double, kSymv>(H, (int)n, matrix, lda, x, incx, alpha, beta, y, incy,
                                       uplo == CORAL_LOWER, false);
}

// zhemv.rs:96-230: the chemv order in double (Re of the diagonal only; beta
// == 0 fills zeros, beta != 1 multiplies by zscal, zhemv.rs:135-138).
coral_status_t coral_zhemv(coral_handle_t hh, int uplo, size_t n, const double alpha[2],
                           const double* matrix, size_t lda, const double* x, size_t incx,
                           const double beta[2], double* y, size_t incy) {
  CORAL_HANDLE(hh);
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (!alpha) return bad_arg(H, 3);
  if (!beta) return bad_arg(H, 8);
  if (n == 0) return CORAL_OK;  // zhemv.rs:110
  if (alpha[0] == 0.0 && alpha[1] == 0.0 && beta[0] == 1.0 && beta[1] == 0.0) return CORAL_OK;
  if (!matrix) return bad_arg(H, 4);
  if (lda < n) return bad_arg(H, 5);
  if (!x) return bad_arg(H, 6);
  if (incx == 0) return bad_arg(H, 7);
  if (!y) return bad_arg(H, 9);
  if (incy == 0) return bad_arg(H, 10);
  if (((uintptr_t)matrix | (uintptr_t)x | (uintptr_t)y) & 15) return bad_arg(H, 4);
  if (n > (size_t)(1 << 20)) return CORAL_ERR_NOT_SUPPORTED;
  return run_tri_strips<double2, kHemv>(H, (int)n, reinterpret_cast<const double2*>(matrix), lda,
                                        reinterpret_cast<const double2*>(x), incx,
                                        make_double2(alpha[0], alpha[1]), make_double2(beta[0], beta[1]),
                                        reinterpret_cast<double2*>(y), incy, uplo == CORAL_LOWER, false);
}

}  // extern "C"

namespace coral {
namespace {
// x <- op(A) x for d/c/z TRMV (dtrmv.rs, ctrmv.rs:58-72, ztrmv.rs); for real
// data ConjugateTranspose == Transpose.
template <typename T>
coral_status_t trmv_any(Handle* H, int uplo, int trans, int diag, size_t n, const void* matrix,
                        size_t lda, void* x, size_t incx, size_t align) {
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (trans < CORAL_NO_TRANSPOSE || trans > CORAL_CONJ_TRANSPOSE) return bad_arg(H, 2);
  if (diag != CORAL_UNIT && diag != CORAL_NON_UNIT) return bad_arg(H, 3);
  if (n == 0) return CORAL_OK;
  if (!matrix) return bad_arg(H, 5);
  if (lda < n) return bad_arg(H, 6);
  if (!x) return bad_arg(H, 7);
  if (incx == 0) return bad_arg(H, 8);
  if (((uintptr_t)matrix | (uintptr_t)x) & (align - 1)) return bad_arg(H, 5);
  if (n > (size_t)(1 << 20)) return CORAL_ERR_NOT_SUPPORTED;
  const bool lower = uplo == CORAL_LOWER, unit = diag == CORAL_UNIT;
  const T* A = static_cast<const T*>(matrix);
  T* X = static_cast<T*>(x);
  const T one = Cx<T>::one(), zero = Cx<T>::zero();
  if (trans == CORAL_NO_TRANSPOSE)
    return run_tri_strips<T, kTrmvN>(H, (int)n, A, lda, X, incx, one, zero, X, incx, lower, unit);
  if (trans == CORAL_CONJ_TRANSPOSE && !std::is_same<T, double>::value)
    return run_tri_strips<T, kTrmvC>(H, (int)n, A, lda, X, incx, one, zero, X, incx, lower, unit);
  return run_tri_strips<T, kTrmvT>(H, (int)n, A, lda, X, incx, one, zero, X, incx, lower, unit);
}
}  // namespace
}  // namespace coral

extern "C" {
coral_status_t coral_dtrmv(coral_handle_t hh, int uplo, int trans, int diag, size_t n,
                           const double* matrix, size_t lda, double* x, size_t incx) {
  CORAL_HANDLE(hh);
  return trmv_any<double>(H, uplo, trans, diag, n, matrix, lda, x, incx, 8);
}
coral_status_t coral_ctrmv(coral_handle_t hh, int uplo, int trans, int diag, size_t n,
                           const float* matrix, size_t lda, float* x, size_t incx) {
  CORAL_HANDLE(hh);
  return trmv_any<float2>(H, uplo, trans, diag, n, matrix, lda, x, incx, 8);
}
coral_status_t coral_ztrmv(coral_handle_t hh, int uplo, int trans, int diag, size_t n,
                           const double* matrix, size_t lda, double* x, size_t incx) {
  CORAL_HANDLE(hh);
  return trmv_any<double2>(H, uplo, trans, diag, n, matrix, lda, x, incx, 16);
}
}  // extern "C"
