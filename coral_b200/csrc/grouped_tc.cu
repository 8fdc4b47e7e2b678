// Grouped (uneven) SGEMM on the 5th-generation tensor cores (tcgen05 + TMEM).
//
// No reference counterpart: each instance has the semantics of coral_sgemm
// (sgemm.rs:106-130; quick returns sgemm_nn.rs:29-45; epilogue
// f32_edge.rs:37-58).  Two arithmetic forms share one kernel:
//   - bf16 inputs, fp32 accumulation: one tcgen05 product per K step;
//   - fp32 inputs as split-BF16x3: each value split into two bf16 pieces
//     (a = a0 + a1 + r, |r| <= 2^-18 |a|) and A0 B0 + A0 B1 + A1 B0 summed in
//     the fp32 TMEM accumulator, as the single split GEMM does.
//
// The instances' operands have arbitrary leading dimensions and alignments,
// which tensor maps cannot describe without per-instance host work, so the
// operands are staged by producer warps instead of TMA: each thread takes
// items of 8 consecutive K values of one row -- one contiguous segment (16-byte
// loads where it is aligned) for an operand stored along K, or 8 row-coalesced
// loads for one stored along the rows -- converts them to bf16 pieces in
// registers, and writes each piece with one 16-byte shared store into the
// K-major 64-byte-swizzled layout that a TMA
// CU_TENSOR_MAP_SWIZZLE_64B load would write (rows of 32 bf16, 8-row / 512-byte
// atoms, 16-byte chunk c of row r at chunk c ^ ((r >> 1) & 3)), so the MMA
// descriptors are the same as the TMA-fed kernels'.
//
// Plan (k_grouped_plan, one CTA): every instance gets a tile width BN from the
// handle's per-class policy (classes by n: <= 64, <= 128, <= 256, > 256;
// BN in {64, 128, 256}; a descriptor's `reserved` field of 64/128/256
// overrides it), instances are ordered by decreasing K bucket (longest tiles
// first), and the exclusive prefix sum of 128 x BN output tiles is formed.
//
// GEMM (k_gemm_grouped_tc, persistent, one CTA per SM, 22 warps):
//   warp 0      scheduler: takes tile indices from a global atomic counter
//               (dynamic load balance), decodes (instance, m0, n0, BN) and
//               publishes them through a 16-deep shared queue;
//   warps 1-16  producers: stage the K slabs of each tile into a ring of
//               shared-memory stages (4 for fp32 pieces, 8 for bf16), each
//               thread issuing all its loads of a slab before converting any;
//   warp 17     MMA issuer (lane 0): tcgen05.mma M=128, N=BN, K=16 into one of
//               two TMEM accumulators of 256 columns, in chunks of at most
//               32 slabs (1024 K) per accumulation;
//   warps 18-21 epilogue: tcgen05.ld the accumulator (thread = row), apply
//               alpha / beta to C with coalesced column accesses (the C loads
//               of 16 columns issued together before their stores, so a tile
//               costs a few memory round trips, not one per column); chunks
//               after the first add alpha * partial into C.
// Every wait is bounded: a wait that gives up sets the handle's status word
// (reported by coral_sync) and the CTA winds down.
#include "common.cuh"
#include "tc_common.cuh"

#include <cuda_bf16.h>

#include <type_traits>

namespace coral {
namespace {

constexpr int kTM = 128;          // tile rows (TMEM lanes)
constexpr int kTK = 32;           // K slab: one 64-byte swizzled row of bf16
constexpr int kMaxBN = 256;
constexpr int kProdWarps = 16;
constexpr int kEpiWarps = 4;
constexpr int kMmaWarp = 1 + kProdWarps;
constexpr int kEpiWarp0 = kMmaWarp + 1;
constexpr int kTcThreads = 32 * (kEpiWarp0 + kEpiWarps);  // 704
constexpr int kQueue = 16;
constexpr int kChunkSlabs = 32;
constexpr uint32_t kAPieceBytes = kTM * kTK * 2;       // 8 KiB
constexpr uint32_t kBPieceBytes = kMaxBN * kTK * 2;    // 16 KiB

template <int NPC> struct TcCfg;
template <> struct TcCfg<2> {
  static constexpr int kStages = 4, kProducts = 3;
  // (A piece, B piece) per product, smallest terms first: A1 B0, A0 B1, A0 B0;
  // A0 stays in the tensor core's A collector between its two products
  __device__ static constexpr int a(int q) { return q == 0 ? 1 : 0; }
  __device__ static constexpr int b(int q) { return q == 1 ? 1 : 0; }
  __device__ static constexpr int collect(int q) {
    return q == 1 ? tc::kCollectFill : q == 2 ? tc::kCollectLastUse : tc::kCollectNone;
  }
};
template <> struct TcCfg<1> {
  static constexpr int kStages = 8, kProducts = 1;
  __device__ static constexpr int a(int) { return 0; }
  __device__ static constexpr int b(int) { return 0; }
  __device__ static constexpr int collect(int) { return tc::kCollectNone; }
};

template <int NPC>
constexpr uint32_t tc_stage_bytes() { return NPC * (kAPieceBytes + kBPieceBytes); }
template <int NPC>
constexpr size_t tc_smem_bytes() { return (size_t)TcCfg<NPC>::kStages * tc_stage_bytes<NPC>() + 1024; }

struct TileInfo {
  int inst;    // instance, -1: no more tiles
  int m0, n0, bn;
  int nslabs;  // K slabs; 0: scale-only tile (alpha == 0 or k == 0)
};

__device__ __forceinline__ int policy_bn(const GroupedPolicy& pol, const coral_sgemm_problem_t& p) {
  if (p.reserved == 64 || p.reserved == 128 || p.reserved == 256) return p.reserved;
  const int cls = p.n <= 64 ? 0 : p.n <= 128 ? 1 : p.n <= 256 ? 2 : 3;
  return pol.bn[cls];
}

// One CTA.  order[pos] = instance, bn_pos[pos] = its tile width, prefix[pos] =
// tiles before position pos (prefix[count] = total).  Positions follow
// decreasing K bucket, so the longest tiles are handed out first.
__global__ void __launch_bounds__(1024)
k_grouped_plan(const coral_sgemm_problem_t* __restrict__ probs, int count, GroupedPolicy pol,
               int* __restrict__ order, int* __restrict__ bn_pos, long long* __restrict__ prefix) {
  __shared__ int hist[32], start[32], cursor[32];
  __shared__ long long warp_tot[32];
  __shared__ long long carry;
  if (threadIdx.x < 32) { hist[threadIdx.x] = 0; cursor[threadIdx.x] = 0; }
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  auto key_of = [&](const coral_sgemm_problem_t& p) {
    if (p.m <= 0 || p.n <= 0 || p.k <= 0 || p.alpha == 0.f) return 0;
    return 31 - __clz(p.k);
  };
  for (int i = threadIdx.x; i < count; i += blockDim.x) atomicAdd(&hist[key_of(probs[i])], 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int b = 31; b >= 0; --b) { start[b] = s; s += hist[b]; }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    const int b = key_of(probs[i]);
    order[start[b] + atomicAdd(&cursor[b], 1)] = i;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < count; base += blockDim.x) {
    const int pos = base + threadIdx.x;
    long long t = 0;
    if (pos < count) {
      const coral_sgemm_problem_t p = probs[order[pos]];
      const int bn = policy_bn(pol, p);
      bn_pos[pos] = bn;
      if (p.m > 0 && p.n > 0) t = (long long)((p.m + kTM - 1) / kTM) * ((p.n + bn - 1) / bn);
    }
    long long v = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    if (lane == 31) warp_tot[w] = v;
    __syncthreads();
    if (w == 0) {
      long long s = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += u;
      }
      warp_tot[lane] = s;
    }
    __syncthreads();
    const long long excl = carry + (w ? warp_tot[w - 1] : 0) + v - t;
    if (pos < count) prefix[pos] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + t;
    __syncthreads();
  }
  if (threadIdx.x == 0) prefix[count] = carry;
}

template <typename TIn> __device__ __forceinline__ float ld_val(const TIn* p);
template <> __device__ __forceinline__ float ld_val<float>(const float* p) { return __ldg(p); }

// Operand views of one tile's K slab for the producers.
template <typename TIn>
struct SlabSrc {
  const TIn* a;
  const TIn* b;
  long long lda, ldb;
  bool a_kc, b_kc;  // stored contiguous along K
  int m, n, k;      // valid rows of A, of B, and K
  int m0, n0, bn;
};

// Byte offset of element (row r, K position kk) of a slab tile in the
// 64-byte-swizzled K-major layout (rows of 32 bf16, 8-row / 512-byte atoms,
// 16-byte chunk c of row r at chunk c ^ ((r >> 1) & 3)).
__device__ __forceinline__ uint32_t sw64_offset(int r, int kk) {
  return (uint32_t)(r >> 3) * 512u + (uint32_t)(r & 7) * 64u + (uint32_t)((((kk >> 3) ^ ((r >> 1) & 3)) << 4) +
                                                                           (kk & 7) * 2);
}

// Eight consecutive floats p[0..8), with two 16-byte loads when p is 16-byte
// aligned (bf16 operands are staged raw by load_share_bf16 instead).
__device__ __forceinline__ void ld8(const float* p, float* v) {
  if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    const float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  } else {
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = __ldg(p + j);
  }
}
// Item e of an operand tile: 8 consecutive K values of one row.  Along K the
// items run row-major (4 per row: lanes on the chunks of 8 consecutive rows,
// each item one contiguous 16- or 32-byte segment); along the rows they run
// chunk-major (lanes on consecutive rows, each of the 8 loads one coalesced
// row segment).
__device__ __forceinline__ void item_rc(bool kc, int e, int rows, int& r, int& c) {
  if (kc) {
    r = e >> 2;
    c = e & 3;
  } else {
    r = e % rows;
    c = e / rows;
  }
}

// Loads one operand's share of a 32-deep slab for this producer thread into
// v[0 .. kVals): rows [row0, row0 + rows) of an operand stored contiguous
// along K (element (r, k) at X[k + r ld]) or along the rows (X[r + k ld]),
// one item of 8 K values per 8 entries of v.  Everything outside R x Kd (and
// rows past `rows`) reads as zero.
template <typename TIn, int kVals>
__device__ __forceinline__ void load_share(const TIn* __restrict__ X, long long ld, bool kc, int R, int Kd,
                                           int row0, int rows, int k0, int ptid, float (&v)[kVals]) {
  constexpr int kPT = 32 * kProdWarps;
#pragma unroll
  for (int i = 0; i < kVals; ++i) v[i] = 0.f;
#pragma unroll
  for (int it = 0; it < kVals / 8; ++it) {
    const int e = ptid + it * kPT;
    if (e >= rows * 4) continue;
    int r, c;
    item_rc(kc, e, rows, r, c);
    const int gr = row0 + r, gk = k0 + 8 * c;
    if (gr >= R) continue;
    if (kc) {
      const TIn* p = X + (size_t)gr * ld + gk;
      if (gk + 8 <= Kd) {
        ld8(p, &v[it * 8]);
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (gk + j < Kd) v[it * 8 + j] = ld_val<TIn>(p + j);
      }
    } else {
      const TIn* p = X + gr + (size_t)gk * ld;
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (gk + j < Kd) v[it * 8 + j] = ld_val<TIn>(p + (size_t)j * ld);
    }
  }
}

// Converts and stores what load_share loaded: NPC bf16 pieces of each value,
// one 16-byte store per item and piece at dst + pc * piece_bytes.
template <int NPC, int kVals>
__device__ __forceinline__ void store_share(uint8_t* dst, uint32_t piece_bytes, bool kc, int rows, int ptid,
                                            const float (&v)[kVals]) {
  constexpr int kPT = 32 * kProdWarps;
#pragma unroll
  for (int it = 0; it < kVals / 8; ++it) {
    const int e = ptid + it * kPT;
    if (e >= rows * 4) continue;
    int r, c;
    item_rc(kc, e, rows, r, c);
    __align__(16) __nv_bfloat16 q[NPC][8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const __nv_bfloat16 h0 = __float2bfloat16_rn(v[it * 8 + j]);
      q[0][j] = h0;
      if constexpr (NPC == 2) q[1][j] = __float2bfloat16_rn(v[it * 8 + j] - __bfloat162float(h0));
    }
    const uint32_t off = sw64_offset(r, 8 * c);
#pragma unroll
    for (int pc = 0; pc < NPC; ++pc)
      *reinterpret_cast<uint4*>(dst + pc * piece_bytes + off) = *reinterpret_cast<const uint4*>(q[pc]);
  }
}

// bf16 inputs need no conversion: their bits go to shared memory as loaded.
// Loads one operand's share of a slab as packed bf16 pairs (w[it * 4 + h] =
// K values 2h and 2h + 1 of item it), with the items of load_share; zero
// bits (+0.0) outside R x Kd.
template <int kItems>
__device__ __forceinline__ void load_share_bf16(const __nv_bfloat16* __restrict__ X, long long ld, bool kc, int R,
                                                int Kd, int row0, int rows, int k0, int ptid,
                                                uint32_t (&w)[4 * kItems]) {
  constexpr int kPT = 32 * kProdWarps;
  const unsigned short* Xs = reinterpret_cast<const unsigned short*>(X);
#pragma unroll
  for (int i = 0; i < 4 * kItems; ++i) w[i] = 0u;
#pragma unroll
  for (int it = 0; it < kItems; ++it) {
    const int e = ptid + it * kPT;
    if (e >= rows * 4) continue;
    int r, c;
    item_rc(kc, e, rows, r, c);
    const int gr = row0 + r, gk = k0 + 8 * c;
    if (gr >= R) continue;
    unsigned short h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (kc) {
      const unsigned short* p = Xs + (size_t)gr * ld + gk;
      if (gk + 8 <= Kd && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
        const uint4 u = __ldg(reinterpret_cast<const uint4*>(p));
        w[it * 4 + 0] = u.x;
        w[it * 4 + 1] = u.y;
        w[it * 4 + 2] = u.z;
        w[it * 4 + 3] = u.w;
        continue;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (gk + j < Kd) h[j] = __ldg(p + j);
    } else {
      const unsigned short* p = Xs + gr + (size_t)gk * ld;
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (gk + j < Kd) h[j] = __ldg(p + (size_t)j * ld);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) w[it * 4 + j] = (uint32_t)h[2 * j] | ((uint32_t)h[2 * j + 1] << 16);
  }
}

template <int kItems>
__device__ __forceinline__ void store_share_bf16(uint8_t* dst, bool kc, int rows, int ptid,
                                                 const uint32_t (&w)[4 * kItems]) {
  constexpr int kPT = 32 * kProdWarps;
#pragma unroll
  for (int it = 0; it < kItems; ++it) {
    const int e = ptid + it * kPT;
    if (e >= rows * 4) continue;
    int r, c;
    item_rc(kc, e, rows, r, c);
    *reinterpret_cast<uint4*>(dst + sw64_offset(r, 8 * c)) =
        make_uint4(w[it * 4], w[it * 4 + 1], w[it * 4 + 2], w[it * 4 + 3]);
  }
}

// Stages one 32-deep K slab of a tile: A rows [m0, m0 + 128) and B rows
// [n0, n0 + bn) as NPC bf16 piece tiles, A pieces at st + i * kAPieceBytes
// and B pieces after them, 64-byte swizzled.  Every load of the thread's share
// of both operands is issued before any value is converted, so a slab costs
// one memory round trip.
template <typename TIn, int NPC>
__device__ __forceinline__ void stage_slab(const SlabSrc<TIn>& src, int k0, uint8_t* st, int ptid) {
  constexpr int kAVals = kTM / kProdWarps;       // 8: one item of 8 K values per producer thread
  constexpr int kBVals = kMaxBN / kProdWarps;    // 16: two items
  if constexpr (std::is_same<TIn, __nv_bfloat16>::value) {
    uint32_t wa[kAVals / 2], wb[kBVals / 2];
    load_share_bf16<kAVals / 8>(src.a, src.lda, src.a_kc, src.m, src.k, src.m0, kTM, k0, ptid, wa);
    load_share_bf16<kBVals / 8>(src.b, src.ldb, src.b_kc, src.n, src.k, src.n0, src.bn, k0, ptid, wb);
    store_share_bf16<kAVals / 8>(st, src.a_kc, kTM, ptid, wa);
    store_share_bf16<kBVals / 8>(st + kAPieceBytes, src.b_kc, src.bn, ptid, wb);
  } else {
    float va[kAVals], vb[kBVals];
    load_share<TIn, kAVals>(src.a, src.lda, src.a_kc, src.m, src.k, src.m0, kTM, k0, ptid, va);
    load_share<TIn, kBVals>(src.b, src.ldb, src.b_kc, src.n, src.k, src.n0, src.bn, k0, ptid, vb);
    store_share<NPC, kAVals>(st, kAPieceBytes, src.a_kc, kTM, ptid, va);
    store_share<NPC, kBVals>(st + NPC * kAPieceBytes, kBPieceBytes, src.b_kc, src.bn, ptid, vb);
  }
}

template <typename TIn, int NPC>
__global__ void __launch_bounds__(kTcThreads, 1)
k_gemm_grouped_tc(const coral_sgemm_problem_t* __restrict__ probs, int count,
                  const int* __restrict__ order, const int* __restrict__ bn_pos,
                  const long long* __restrict__ prefix, unsigned long long* tile_counter,
                  unsigned* status, uint64_t limit_ns) {
  using Cfg = TcCfg<NPC>;
  constexpr int S = Cfg::kStages;
  constexpr uint32_t kStage = tc_stage_bytes<NPC>();

  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = tc::align1024_shared(smem_raw);
  __shared__ __align__(8) uint64_t full_bar[S], empty_bar[S];
  __shared__ __align__(8) uint64_t acc_full[2], acc_empty[2];
  __shared__ __align__(8) uint64_t tq_full[kQueue], tq_empty[kQueue];
  __shared__ __align__(8) uint64_t drain_bar;
  __shared__ TileInfo tq[kQueue];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      tc::mbar_init(&full_bar[s], kProdWarps);
      tc::mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&acc_full[b], 1);
      tc::mbar_init(&acc_empty[b], kEpiWarps);
    }
    for (int q = 0; q < kQueue; ++q) {
      tc::mbar_init(&tq_full[q], 1);
      tc::mbar_init(&tq_empty[q], kProdWarps + 1 + kEpiWarps);
    }
    tc::mbar_init(&drain_bar, 1);
    abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == kMmaWarp) {
    tc::tmem_alloc(&tmem_slot, 2 * kMaxBN);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_slot;

  auto give_up = [&]() {
    atomicOr(status, kStatusTimeout);
    atomicExch(&abort_flag, 1);
  };
  // Consumer side of the tile queue: the info of the j-th tile of this CTA.
  // A whole warp calls it (one arrival per warp), or a single thread with
  // single == true.
  auto next_tile = [&](int j, TileInfo& ti, bool single) -> bool {
    const int q = j % kQueue;
    if (!tc::mbar_wait(&tq_full[q], (j / kQueue) & 1, limit_ns)) {
      give_up();
      return false;
    }
    ti = tq[q];
    if (!single) __syncwarp();
    if (single || lane == 0) tc::mbar_arrive(&tq_empty[q]);
    return ti.inst >= 0 && !*(volatile int*)&abort_flag;
  };

  if (warp == 0) {
    if (lane == 0) {
      // ---- scheduler ----
      const long long total = prefix[count];
      for (int j = 0;; ++j) {
        const int q = j % kQueue;
        if (j >= kQueue && !tc::mbar_wait(&tq_empty[q], ((j / kQueue) - 1) & 1, limit_ns)) {
          give_up();
          break;
        }
        TileInfo ti{-1, 0, 0, 0, 0};
        const long long t = *(volatile int*)&abort_flag ? total : (long long)atomicAdd(tile_counter, 1ull);
        if (t < total) {
          int lo = 0, hi = count - 1;  // last position with prefix <= t
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= t) lo = mid; else hi = mid - 1;
          }
          const int inst = order[lo];
          const coral_sgemm_problem_t p = probs[inst];
          const int bn = bn_pos[lo];
          const long long local = t - prefix[lo];
          const int mt = (p.m + kTM - 1) / kTM;
          ti.inst = inst;
          ti.bn = bn;
          ti.m0 = (int)(local % mt) * kTM;
          ti.n0 = (int)(local / mt) * bn;
          ti.nslabs = (p.alpha == 0.f || p.k <= 0) ? 0 : (p.k + kTK - 1) / kTK;
        }
        tq[q] = ti;
        tc::mbar_arrive(&tq_full[q]);
        if (ti.inst < 0) break;
      }
    }
  } else if (warp < kMmaWarp) {
    // ---- producers ----
    const int ptid = threadIdx.x - 32;
    int it = 0;
    TileInfo ti;
    for (int j = 0; next_tile(j, ti, false); ++j) {
      if (ti.nslabs == 0) continue;
      const coral_sgemm_problem_t p = probs[ti.inst];
      const SlabSrc<TIn> src{static_cast<const TIn*>(p.a), static_cast<const TIn*>(p.b), p.lda, p.ldb,
                             p.op_a != CORAL_NO_TRANSPOSE, p.op_b == CORAL_NO_TRANSPOSE, p.m, p.n, p.k,
                             ti.m0, ti.n0, ti.bn};
      bool stop = false;
      for (int kb = 0; kb < ti.nslabs; ++kb, ++it) {
        const int s = it % S;
        if (it >= S && !tc::mbar_wait(&empty_bar[s], ((it / S) - 1) & 1, limit_ns)) {
          give_up();
          stop = true;
          break;
        }
        uint8_t* st = smem + (size_t)s * kStage;
        stage_slab<TIn, NPC>(src, kb * kTK, st, ptid);
        tc::fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&full_bar[s]);
      }
      if (stop) break;
    }
  } else if (warp == kMmaWarp) {
    if (lane == 0) {
      // ---- MMA issuer ----
      int it = 0, gc = 0;
      bool stop = false;
      TileInfo ti;
      for (int j = 0; !stop && next_tile(j, ti, true); ++j) {
        if (ti.nslabs == 0) continue;
        const uint32_t idesc = tc::idesc_bf16_f32(kTM, ti.bn);
        const int chunks = (ti.nslabs + kChunkSlabs - 1) / kChunkSlabs;
        for (int c = 0; c < chunks && !stop; ++c, ++gc) {
          const int b = gc & 1;
          if (gc >= 2 && !tc::mbar_wait(&acc_empty[b], ((gc >> 1) - 1) & 1, limit_ns)) {
            give_up();
            stop = true;
            break;
          }
          tc::tc_fence_after();
          const uint32_t acc = tmem + b * kMaxBN;
          const int kb0 = c * kChunkSlabs, kb1 = min(ti.nslabs, kb0 + kChunkSlabs);
          for (int kb = kb0; kb < kb1; ++kb, ++it) {
            const int s = it % S;
            if (!tc::mbar_wait(&full_bar[s], (it / S) & 1, limit_ns)) {
              give_up();
              stop = true;
              break;
            }
            tc::tc_fence_after();
            const uint32_t sa = tc::smem_u32(smem + (size_t)s * kStage);
            const uint32_t sb = sa + NPC * kAPieceBytes;
#pragma unroll
            for (int kk = 0; kk < kTK / 16; ++kk) {
#pragma unroll
              for (int q = 0; q < Cfg::kProducts; ++q) {
                const uint64_t ad = tc::desc_k_sw64(sa + Cfg::a(q) * kAPieceBytes + kk * 32);
                const uint64_t bd = tc::desc_k_sw64(sb + Cfg::b(q) * kBPieceBytes + kk * 32);
                const uint32_t accum = ((kb - kb0) | kk | q) != 0;
                switch (Cfg::collect(q)) {
                  case tc::kCollectFill: tc::mma_f16_ca<tc::kCollectFill>(acc, ad, bd, idesc, accum); break;
                  case tc::kCollectLastUse:
                    tc::mma_f16_ca<tc::kCollectLastUse>(acc, ad, bd, idesc, accum);
                    break;
                  default: tc::mma_f16(acc, ad, bd, idesc, accum); break;
                }
              }
            }
            tc::mma_commit(&empty_bar[s]);
          }
          if (!stop) tc::mma_commit(&acc_full[b]);
        }
      }
      // every MMA issued by this thread completes before TMEM is released
      // (own 1 s bound: the configured limit may be tiny)
      tc::mma_commit(&drain_bar);
      tc::mbar_wait(&drain_bar, 0, 1000000000ull);
    }
  } else {
    // ---- epilogue ----
    const int quad = warp & 3;
    const uint32_t lane_base = (uint32_t)(quad * 32) << 16;
    int gc = 0;
    TileInfo ti;
    for (int j = 0; next_tile(j, ti, false); ++j) {
      const coral_sgemm_problem_t p = probs[ti.inst];
      const int row = ti.m0 + quad * 32 + lane;
      const bool beta0 = p.beta == 0.f, beta1 = p.beta == 1.f;
      const int ncols = min(ti.bn, p.n - ti.n0);
      float* crow = p.c + row;
      if (ti.nslabs == 0) {  // scale-only (sgemm_nn.rs:29-45), 16 C loads before their stores
        if (!beta1 && row < p.m)
          for (int g = 0; g < ncols; g += 16) {
            float cv[16];
#pragma unroll
            for (int jj = 0; jj < 16; ++jj)
              cv[jj] = (!beta0 && g + jj < ncols) ? crow[(size_t)(ti.n0 + g + jj) * p.ldc] : 0.f;
#pragma unroll
            for (int jj = 0; jj < 16; ++jj)
              if (g + jj < ncols) crow[(size_t)(ti.n0 + g + jj) * p.ldc] = beta0 ? 0.f : p.beta * cv[jj];
          }
        continue;
      }
      const int chunks = (ti.nslabs + kChunkSlabs - 1) / kChunkSlabs;
      bool stop = false;
      for (int c = 0; c < chunks; ++c, ++gc) {
        const int b = gc & 1;
        if (!tc::mbar_wait(&acc_full[b], (gc >> 1) & 1, limit_ns)) {
          give_up();
          stop = true;
          break;
        }
        tc::tc_fence_after();
        const bool read_c = c > 0 || !beta0;
        for (int col0 = 0; col0 < ncols; col0 += 16) {
          // 16 accumulator columns, then every C load of them before any store
          uint32_t r[16];
          tc::tmem_ld16(tmem + b * kMaxBN + col0 + lane_base, r);
          tc::tmem_wait_ld();
          if (row < p.m) {
            const int lim = min(16, ncols - col0);
            float cv[16];
#pragma unroll
            for (int jj = 0; jj < 16; ++jj)
              cv[jj] = (read_c && jj < lim) ? crow[(size_t)(ti.n0 + col0 + jj) * p.ldc] : 0.f;
#pragma unroll
            for (int jj = 0; jj < 16; ++jj) {
              if (jj >= lim) break;
              const float v = p.alpha * __uint_as_float(r[jj]);
              crow[(size_t)(ti.n0 + col0 + jj) * p.ldc] =
                  (c > 0 || beta1) ? cv[jj] + v : beta0 ? v : p.beta * cv[jj] + v;
            }
          }
        }
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&acc_empty[b]);
      }
      if (stop) break;
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) tc::tmem_dealloc(tmem, 2 * kMaxBN);
}

template <typename TIn, int NPC>
coral_status_t launch_grouped_tc(Handle* h, int count, const coral_sgemm_problem_t* probs, const int* order,
                                 const int* bn_pos, const long long* prefix, unsigned long long* counter) {
  const size_t smem = tc_smem_bytes<NPC>();
  static uint64_t attr_devices = 0;  // bit d: attribute set on device d
  const uint64_t bit = h->device < 64 ? (1ull << h->device) : 0;
  if (!(attr_devices & bit) || !bit) {
    CORAL_CUDA(h, cudaFuncSetAttribute(k_gemm_grouped_tc<TIn, NPC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_devices |= bit;
  }
  const uint64_t limit_ns = h->wait_limit * 32ull;
  timed_begin(h);
  k_gemm_grouped_tc<TIn, NPC><<<h->sm_count, kTcThreads, smem, h->stream>>>(
      probs, count, order, bn_pos, prefix, counter, &h->words->status, limit_ns);
  coral_status_t s = launch_status(h);
  timed_end(h);
  return s;
}

}  // namespace

// Enqueues the plan and the tensor-core grouped GEMM: bf16 inputs (npc 1) or
// fp32 inputs as split-BF16x3 (npc 2).
coral_status_t enqueue_grouped_tc(Handle* h, bool bf16_inputs, size_t count,
                                  const coral_sgemm_problem_t* probs) {
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t o_order = 0, o_bn = up(count * 4), o_prefix = o_bn + up(count * 4);
  const size_t o_ctr = o_prefix + up((count + 1) * 8);
  char* sc = static_cast<char*>(scratch(h, o_ctr + 256));
  if (!sc) return CORAL_ERR_ALLOC;
  int* order = reinterpret_cast<int*>(sc + o_order);
  int* bn_pos = reinterpret_cast<int*>(sc + o_bn);
  long long* prefix = reinterpret_cast<long long*>(sc + o_prefix);
  unsigned long long* counter = reinterpret_cast<unsigned long long*>(sc + o_ctr);
  CORAL_CUDA(h, cudaMemsetAsync(counter, 0, sizeof(unsigned long long), h->stream));
  k_grouped_plan<<<1, 1024, 0, h->stream>>>(probs, (int)count, h->grouped_policy, order, bn_pos, prefix);
  coral_status_t s = launch_status(h);
  if (s != CORAL_OK) return s;
  return bf16_inputs
             ? launch_grouped_tc<__nv_bfloat16, 1>(h, (int)count, probs, order, bn_pos, prefix, counter)
             : launch_grouped_tc<float, 2>(h, (int)count, probs, order, bn_pos, prefix, counter);
}

}  // namespace coral
