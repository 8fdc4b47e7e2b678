// STRSV: solve op(A) x = b in place, A triangular (strsv.rs:60-74 ->
// strlsv.rs / strusv.rs).  ConjugateTranspose == Transpose.
//
// Two kernels.  k_trsv_cluster (below) is the path for any A that a tensor
// map can describe; k_trsv, one CTA per block reading A with plain loads, is
// the path for the rest (lda % 4 != 0 or A not 16-byte aligned).
//
// k_trsv: op(A) is cut into 64-row blocks; each CTA takes a ticket from a
// per-call counter, so block b is handled by the b-th CTA to start (in solve
// order: forward when op(A) is lower, backward when upper) and only ever
// waits for blocks whose CTAs started earlier -- no dependency on scheduling
// order, no deadlock.  A CTA
//   1. stages its diagonal block of op(A) (triangle masked, unit diagonal
//      applied) in shared memory and inverts it (independent of every other
//      block, so it overlaps the solve of earlier blocks);
//   2. streams its row panel of op(A), 256 KB of tiles in flight, and
//      for each tile waits for the solution x_k of that block, then
//      accumulates tile * x_k -- tiles of early blocks are ready long before
//      the last one, so the panel streams while the solve front advances;
//   3. forms x_b = inv(D_b) (b_b - acc), writes it over b, and publishes it
//      as NB epoch-tagged 64-bit slots ((epoch << 32) | float bits, store
//      release).  A consumer polls the slots themselves: one round trip
//      through L2 both signals readiness and delivers the values.
// CORAL solves its diagonal blocks by substitution (strlsv.rs:66-140) with the
// panel update through saxpyf/sdotf; here the blocked diagonal solve uses the
// inverted NB x NB block as a small GEMV, which takes the serial substitution
// off the critical path.  Waits are bounded by the handle's wait limit and
// abort early once any CTA has set the status word.
#include "common.cuh"
#include "tc_common.cuh"

namespace coral {
namespace {

// Block size NB rows; 4 threads per row.
template <int NB> struct TrsvCfg {
  static constexpr int kThreads = 4 * NB;
  static constexpr int kPer = NB * NB / kThreads;  // tile elements per thread
  static constexpr int kG = 4;                    // panel tiles loaded per group
  static constexpr int kQ = 4;                    // thread groups per row
};

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <int kNB>
__global__ void __launch_bounds__(4 * kNB, 1)
k_trsv(int n, const float* __restrict__ A, size_t lda, float* x, size_t incx, bool lower_eff,
       bool trans, bool unit, unsigned long long* slots, unsigned* ticket, unsigned* done,
       unsigned* epoch_word, unsigned* status, uint64_t limit_ns) {
  constexpr int kTrsvThreads = TrsvCfg<kNB>::kThreads, kPer = TrsvCfg<kNB>::kPer;
  constexpr int kG = TrsvCfg<kNB>::kG, kQ = TrsvCfg<kNB>::kQ;
  extern __shared__ float smem_f[];
  float (*D)[kNB + 1] = reinterpret_cast<float (*)[kNB + 1]>(smem_f);               // op(A) block, then inverse
  float (*T)[kNB + 1] = reinterpret_cast<float (*)[kNB + 1]>(smem_f + kNB * (kNB + 1));  // panel tile / scratch
  __shared__ float xk[kNB];
  __shared__ float red[kQ][kNB];
  __shared__ float rhs[kNB];
  __shared__ int sblk;
  __shared__ int abort_flag;

  const int nblk = (n + kNB - 1) / kNB;
  const int tid = threadIdx.x;
  __shared__ unsigned sepoch;
  if (tid == 0) {
    // Tickets start at 0 in every call (the last CTA resets the counter);
    // the call's epoch is one past the last completed call's, read before
    // any CTA of this call can finish and advance it.
    const unsigned t = atomicAdd(ticket, 1u);
    sepoch = *(volatile unsigned*)epoch_word + 1u;
    if (sepoch == 0u) sepoch = 1u;  // slots start at 0: never a live epoch
    abort_flag = 0;
    sblk = lower_eff ? (int)t : nblk - 1 - (int)t;
  }
  __syncthreads();
  const unsigned epoch = sepoch;
  const int blk = sblk;
  const int b0 = blk * kNB;

  // ---- 1. diagonal block of op(A), masked, and its inverse ----
  for (int e = tid; e < kNB * kNB; e += kTrsvThreads) {
    const int rr = e % kNB, cc = e / kNB;       // stored element (b0+rr, b0+cc)
    const int gr = b0 + rr, gc = b0 + cc;
    float v = (gr < n && gc < n) ? __ldg(A + gr + (size_t)gc * lda) : 0.f;
    const int r = trans ? cc : rr, c = trans ? rr : cc;   // op(A)(r, c)
    const bool in_tri = lower_eff ? r >= c : r <= c;
    if (r == c) v = (unit || b0 + r >= n) ? 1.f : v;
    else if (!in_tri) v = 0.f;
    D[r][c] = v;
  }
  __syncthreads();
  {
    // Column c of inv(D) by substitution on e_c, 4 lanes per column (the 4
    // share a warp and split each dot product); result kept in T[c][*].  A
    // warp holds columns [8w, 8w + 8): every lane runs the warp's full
    // iteration range so the full-mask shuffles always have all 32 lanes.
    const int c = tid >> 2, part = tid & 3;
    const int cw0 = (tid >> 5) * 8, cw1 = cw0 + 7;
    if (lower_eff) {
      for (int i = part; i < c; i += 4) T[c][i] = 0.f;
      if (part == 0) T[c][c] = 1.f / D[c][c];
      __syncwarp();
      for (int i = cw0 + 1; i < kNB; ++i) {
        float s = 0.f;
        if (i > c)
          for (int j = c + part; j < i; j += 4) s = fmaf(D[i][j], T[c][j], s);
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        if (i > c && part == 0) T[c][i] = -s / D[i][i];
        __syncwarp();
      }
    } else {
      for (int i = c + 1 + part; i < kNB; i += 4) T[c][i] = 0.f;
      if (part == 0) T[c][c] = 1.f / D[c][c];
      __syncwarp();
      for (int i = cw1 - 1; i >= 0; --i) {
        float s = 0.f;
        if (i < c)
          for (int j = i + 1 + part; j <= c; j += 4) s = fmaf(D[i][j], T[c][j], s);
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        if (i < c && part == 0) T[c][i] = -s / D[i][i];
        __syncwarp();
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < kNB * kNB; e += kTrsvThreads) {  // D <- inv(D)
    const int r = e % kNB, c = e / kNB;
    D[r][c] = T[c][r];
  }
  if (tid < kNB) rhs[tid] = (b0 + tid < n) ? x[(size_t)(b0 + tid) * incx] : 0.f;
  __syncthreads();

  // ---- 2. panel: acc = sum over solved blocks k of op(A)(blk, k) x_k, in
  // solve order, so the blocks solved first are applied first ----
  const int r = tid % kNB, q = tid / kNB;
  float acc = 0.f;
  const int npanel = lower_eff ? blk : nblk - 1 - blk;
  for (int g0 = 0; g0 < npanel; g0 += kG) {
    float reg[kG][kPer];
#pragma unroll
    for (int g = 0; g < kG; ++g) {
      const int idx = g0 + g;
      const int k = lower_eff ? idx : nblk - 1 - idx;  // solve order: earliest first
      // stored block: rows (trans ? k : blk), cols (trans ? blk : k)
      const int R0 = (trans ? k : blk) * kNB, C0 = (trans ? blk : k) * kNB;
#pragma unroll
      for (int p = 0; p < kPer; ++p) {
        const int e = tid + p * kTrsvThreads;
        const int rr = e % kNB, cc = e / kNB;
        const int gr = R0 + rr, gc = C0 + cc;
        reg[g][p] = (idx < npanel && gr < n && gc < n) ? __ldcs(A + gr + (size_t)gc * lda) : 0.f;
      }
    }
#pragma unroll
    for (int g = 0; g < kG; ++g) {
      const int idx = g0 + g;
      if (idx >= npanel) break;
      const int k = lower_eff ? idx : nblk - 1 - idx;  // solve order: earliest first
#pragma unroll
      for (int p = 0; p < kPer; ++p) {
        const int e = tid + p * kTrsvThreads;
        T[e / kNB][e % kNB] = reg[g][p];
      }
      if (tid < kNB) {
        const unsigned long long* sp = slots + (size_t)k * kNB + tid;
        unsigned long long v = ld_acquire64(sp);
        if ((unsigned)(v >> 32) != epoch) {
          const uint64_t t0 = gtimer();
          unsigned spins = 0;
          while ((unsigned)((v = ld_acquire64(sp)) >> 32) != epoch) {
            // the status word (another block gave up) is read only once the
            // wait is long; a healthy wait never pays its round trip
            const uint64_t el = gtimer() - t0;
            if (el > limit_ns ||
                ((++spins & 15u) == 0 && el > 20000ull && *(volatile unsigned*)status != 0)) {
              atomicOr(status, kStatusTimeout);
              abort_flag = 1;
              break;
            }
          }
        }
        xk[tid] = __uint_as_float((unsigned)v);
      }
      __syncthreads();
      if (abort_flag) break;
      // op(A)(r, c) = stored(r, c) = T[c][r], or stored(c, r) = T[r][c] when transposed
      const int cq = q * (kNB / kQ);
      if (!trans) {
#pragma unroll 8
        for (int c = cq; c < cq + kNB / kQ; ++c) acc = fmaf(T[c][r], xk[c], acc);
      } else {
#pragma unroll 8
        for (int c = cq; c < cq + kNB / kQ; ++c) acc = fmaf(T[r][c], xk[c], acc);
      }
      __syncthreads();
    }
    if (abort_flag) break;
  }
  if (!abort_flag) {
  red[q][r] = acc;
  __syncthreads();
  if (tid < kNB) rhs[tid] -= (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]);
  __syncthreads();

  // ---- 3. x_b = inv(D) rhs, publish ----
  float s = 0.f;
  const int cq = q * (kNB / kQ);
#pragma unroll 8
  for (int c = cq; c < cq + kNB / kQ; ++c) s = fmaf(D[r][c], rhs[c], s);
  red[q][r] = s;
  __syncthreads();
  if (tid < kNB) {
    const float v = (b0 + tid < n) ? (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]) : 0.f;
    if (b0 + tid < n) x[(size_t)(b0 + tid) * incx] = v;
    st_release64(slots + (size_t)blk * kNB + tid,
                 ((unsigned long long)epoch << 32) | __float_as_uint(v));
  }
  }  // !abort_flag
  // The last CTA to finish (aborted or not) resets the ticket counter and
  // publishes this call's epoch for the next call.
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(done, 1u) == (unsigned)nblk - 1) {
      *ticket = 0u;
      *done = 0u;
      __threadfence();
      atomicExch(epoch_word, epoch);
    }
  }
}


// ---- cluster path ---------------------------------------------------------
// Same block decomposition (64-row blocks in solve order), restructured so
// that the chain from one block to the next is as short as the hardware
// allows:
//   * CTAs run in clusters of 16 (8 where the hardware cannot place 16) that
//     take consecutive blocks.  A CTA pushes its solution straight into the
//     shared memory of the later CTAs of its cluster (st.shared::cluster,
//     epoch-tagged like the global slots), so 15 of every 16 hand-offs skip
//     the L2 round trip; the global slots serve later clusters.
//   * At setup each CTA inverts its diagonal block D and forms
//     M1 = inv(D) op(A)(b, b-1) and M2 = inv(D) op(A)(b, b-2) in registers.
//     With y = inv(D) (rhs - sum_{k <= b-3} op(A)(b, k) x_k), the solution is
//     x_b = y - M2 x_{b-2} - M1 x_{b-1}: once x_{b-1} lands, each row costs 16
//     FMAs and a 4-lane shuffle reduction -- no block-wide barrier.
//   * The panel tiles op(A)(b, k), k <= b-3, stream through a 4-stage TMA ring
//     (64 x 64 fp32 boxes, zero fill past n) fed by a producer warp, which
//     also polls the solution slots of 8 tiles at once and stages ready ones
//     in a shared-memory ring, so neither the tile nor the solution latency
//     sits on the consumers' path.
// Requires lda % 4 == 0 and a 16-byte aligned A (tensor-map rules).
constexpr int kCB = 64;          // rows per block
constexpr int kClMax = 16;       // CTAs per cluster: 16, or 8 where 16 cannot be placed
constexpr int kCStages = 4;      // panel tile ring
constexpr int kXRing = 32;       // staged solutions of panel tiles
constexpr int kLook = 8;         // panel solutions polled at once
constexpr int kCons = 256;       // consumer threads (8 warps)
constexpr int kCThreads = kCons + 32;
constexpr uint32_t kTileBytes = kCB * kCB * 4;
constexpr int kLd = kCB + 4;     // row stride of the square work arrays (16-byte rows)

struct ClusterSmem {
  float ring[kCStages][kCB][kCB];     // panel tiles as loaded: [stored col][stored row]
  float raw[3][kCB][kCB];             // diagonal block, tiles (b-1), (b-2) as loaded
  float Dm[kCB][kLd];                 // op(D) masked, in lower form
  float W[kCB][kLd];                  // op(tile b-2), rows in the order of Dm
  float Top[kCB][kLd];                // op(tile b-1), rows in the order of Dm
  float rdiag[kCB];                   // reciprocals of Dm's diagonal
  float xs[kXRing][kCB];              // staged solutions of panel tiles
  unsigned long long xin[kClMax][kCB];  // solutions pushed by earlier CTAs of the cluster
  float part[8][kCB];
  float v[kCB + 4];                   // v[vi(c)]: one pad word per 16 values
  float rhs[kCB];
  uint64_t full[kCStages];
  uint64_t empty[kCStages];
  uint64_t xfull[kXRing];
  uint64_t xempty[kXRing];
  uint64_t setup_bar;
  unsigned ticket, epoch, my_ticket, my_epoch;
  int abort_flag;
  int issued;                         // panel tile loads the producer issued
};

// v keeps one pad word after every 16 values, so the four 16-value groups
// read by a warp's lane quads start in different banks.
__device__ __forceinline__ int vi(int c) { return c + (c >> 4); }

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t map_rank(const void* p, unsigned rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(tc::smem_u32(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ unsigned ld_cluster_u32(uint32_t addr) {
  unsigned v;
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ void st_cluster_u64(uint32_t addr, unsigned long long v) {
  asm volatile("st.relaxed.cluster.shared::cluster.u64 [%0], %1;" ::"r"(addr), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_local_tag(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.cluster.shared::cta.u64 %0, [%1];" : "=l"(v) : "r"(tc::smem_u32(p)) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void bar_consumers() {
  asm volatile("bar.sync 1, %0;" ::"n"(kCons) : "memory");
}
__device__ __forceinline__ float quad_sum(float v) {
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  return v;
}

// Reads one block's 64 epoch-tagged solution values (global slots, or this
// CTA's copies pushed by earlier CTAs of the cluster): lane l polls values 2l
// and 2l + 1 (16 contiguous bytes) until the whole warp sees `epoch`, then
// shuffles give each lane xv[j] = x[16 (lane & 3) + j], j < 16.  The poll
// touches only the values, the timer and the CTA's abort flag; the global
// status word (an L2 round trip) is read only after 20 us without the values.
// False (warp-uniform) on timeout or abort.
__device__ __forceinline__ bool fetch_x(const unsigned long long* src, bool local, unsigned epoch,
                                        int lane, float (&xv)[16], const unsigned* status,
                                        const int* abort_flag, uint64_t limit_ns) {
  unsigned long long v0, v1;
  uint64_t t0 = 0;
  for (unsigned spins = 0;; ++spins) {
    if (local) {
      v0 = ld_local_tag(src + 2 * lane);
      v1 = ld_local_tag(src + 2 * lane + 1);
    } else {
      v0 = ld_relaxed64(src + 2 * lane);
      v1 = ld_relaxed64(src + 2 * lane + 1);
    }
    const bool ok = (unsigned)(v0 >> 32) == epoch && (unsigned)(v1 >> 32) == epoch;
    if (__all_sync(0xffffffffu, ok)) break;
    // the timer is read on every 4th poll only, so a healthy poll stays short
    if ((spins & 3u) != 0) continue;
    const uint64_t now = tc::globaltimer();
    if (spins == 0) {
      t0 = now;
      continue;
    }
    const uint64_t el = now - t0;
    bool quit = el > limit_ns;
    if ((spins & 15u) == 0)
      quit = quit || *(volatile const int*)abort_flag ||
             (el > 20000ull && *(volatile const unsigned*)status != 0);
    if (__any_sync(0xffffffffu, quit)) return false;
  }
  const float f0 = __uint_as_float((unsigned)v0), f1 = __uint_as_float((unsigned)v1);
  const int base = 8 * (lane & 3);
#pragma unroll
  for (int j = 0; j < 16; ++j) xv[j] = __shfl_sync(0xffffffffu, (j & 1) ? f1 : f0, base + (j >> 1));
  return true;
}

// Sum of m[j] * x[j], j < 16, over four independent chains.
__device__ __forceinline__ float dot16(const float (&m)[16], const float (&x)[16]) {
  float a[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int j = 0; j < 16; ++j) a[j & 3] = fmaf(m[j], x[j], a[j & 3]);
  return (a[0] + a[1]) + (a[2] + a[3]);
}

// Column `col` of X = inv(L) B for the 64 x 64 lower-triangular L in Dm
// (reciprocal diagonal in rdiag), B = [I | Top | W] (192 columns), by forward
// substitution with the column in registers: x_i = (b_i - sum_{j<i} L_ij x_j)
// / L_ii, the sum over j split four ways.  Each thread solves its column with
// no barrier; L's rows are read as broadcast 16-byte shared loads.  Column c
// of X goes to out[c / 64] at row i, position (c % 64) ^ (4 (i % 8)): the
// swizzle keeps both this column-wise store and the row-wise 16-byte reads of
// the later register loads free of bank conflicts.
__device__ __forceinline__ void solve_column(const ClusterSmem& S, int col, float (*out)[kCB][kCB]) {
  const int part = col >> 6, c = col & 63;
  float xc[kCB];
#pragma unroll
  for (int i = 0; i < kCB; ++i) {
    float a0 = part == 0 ? (i == c ? 1.f : 0.f) : part == 1 ? S.Top[i][c] : S.W[i][c];
    float a1 = 0.f, a2 = 0.f, a3 = 0.f;
#pragma unroll
    for (int j = 0; j + 4 <= i; j += 4) {
      const float4 l = *reinterpret_cast<const float4*>(&S.Dm[i][j]);
      a0 = fmaf(-l.x, xc[j], a0);
      a1 = fmaf(-l.y, xc[j + 1], a1);
      a2 = fmaf(-l.z, xc[j + 2], a2);
      a3 = fmaf(-l.w, xc[j + 3], a3);
    }
#pragma unroll
    for (int j = i & ~3; j < i; ++j) a0 = fmaf(-S.Dm[i][j], xc[j], a0);
    xc[i] = ((a0 + a1) + (a2 + a3)) * S.rdiag[i];
  }
#pragma unroll
  for (int i = 0; i < kCB; ++i) out[part][i][c ^ ((i & 7) << 2)] = xc[i];
}

__global__ void __launch_bounds__(kCThreads, 1)
k_trsv_cluster(const __grid_constant__ CUtensorMap amap, int n, float* x, size_t incx,
               bool lower_eff, bool trans, bool unit, unsigned long long* slots, unsigned* ticket,
               unsigned* done, unsigned* epoch_word, unsigned* status, uint64_t limit_ns) {
  // Offsetting the __shared__ array itself (not an integer address) keeps the
  // accesses below in the shared window (LDS/STS rather than generic loads).
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  ClusterSmem& S = *reinterpret_cast<ClusterSmem*>(
      smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned rank = cluster_rank();

  unsigned ncl;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(ncl));
  const int kCl = (int)ncl;
  for (int i = tid; i < kCl * kCB; i += kCThreads) (&S.xin[0][0])[i] = 0ull;
  if (tid == 0) {
    for (int i = 0; i < kCStages; ++i) {
      tc::mbar_init(&S.full[i], 1);
      tc::mbar_init(&S.empty[i], 8);
    }
    for (int i = 0; i < kXRing; ++i) {
      tc::mbar_init(&S.xfull[i], 32);
      tc::mbar_init(&S.xempty[i], 8);
    }
    tc::mbar_init(&S.setup_bar, 1);
    tc::fence_mbar_init();
    S.abort_flag = 0;
    S.issued = 0;
    if (rank == 0) {
      // Tickets start at 0 in every call (the last CTA resets the counter);
      // the epoch is one past the last completed call's, read before any CTA
      // of this call can finish and advance it.
      S.ticket = atomicAdd(ticket, 1u);
      unsigned e = *(volatile unsigned*)epoch_word + 1u;
      S.epoch = e ? e : 1u;  // slots start at 0: never a live epoch
    }
  }
  cluster_sync_all();
  if (tid == 0) {
    S.my_ticket = ld_cluster_u32(map_rank(&S.ticket, 0));
    S.my_epoch = ld_cluster_u32(map_rank(&S.epoch, 0));
  }
  __syncthreads();
  const unsigned epoch = S.my_epoch;
  const int nblk = (n + kCB - 1) / kCB;
  const int s_first = (int)S.my_ticket * kCl;        // first solve index of this cluster
  const int s = s_first + (int)rank;                   // this CTA's solve index
  const bool active = s < nblk;
  auto blk_of = [&](int sp) { return lower_eff ? sp : nblk - 1 - sp; };
  const int blk = active ? blk_of(s) : 0;
  const int b0 = blk * kCB;
  const int npanel = s >= 3 ? s - 2 : 0;              // panel tiles: solve indices 0 .. s-3
  // TMA coordinates of tile op(A)(blk, kb): stored rows x, stored columns y
  auto tile_x = [&](int kb) { return trans ? kb * kCB : b0; };
  auto tile_y = [&](int kb) { return trans ? b0 : kb * kCB; };

  if (active && warp == 8) {
    // ---------------- producer warp ----------------
    if (lane == 0) {
      tc::prefetch_tmap(&amap);
      uint32_t bytes = kTileBytes * (1 + (s >= 1) + (s >= 2));
      tc::mbar_expect_tx(&S.setup_bar, bytes);
      tc::tma_load_2d(S.raw[0], &amap, &S.setup_bar, b0, b0);
      if (s >= 1) tc::tma_load_2d(S.raw[1], &amap, &S.setup_bar, tile_x(blk_of(s - 1)), tile_y(blk_of(s - 1)));
      if (s >= 2) tc::tma_load_2d(S.raw[2], &amap, &S.setup_bar, tile_x(blk_of(s - 2)), tile_y(blk_of(s - 2)));
    }
    int tma_next = 0, x_next = 0;
    uint64_t t_last = 0;  // start of the current stretch without progress (0: none)
    unsigned iter = 0;
    const int nstaged = npanel < s_first ? npanel : s_first;  // panel tiles of earlier clusters
    while (x_next < nstaged || tma_next < npanel) {
      if (lane == 0) {
        while (tma_next < npanel) {
          const int st = tma_next % kCStages;
          if (tma_next >= kCStages && !tc::mbar_try_wait(&S.empty[st], ((tma_next / kCStages) - 1) & 1))
            break;
          const int kb = blk_of(tma_next);
          tc::mbar_expect_tx(&S.full[st], kTileBytes);
          tc::tma_load_2d(S.ring[st], &amap, &S.full[st], tile_x(kb), tile_y(kb));
          ++tma_next;
        }
      }
      tma_next = __shfl_sync(0xffffffffu, tma_next, 0);
      // solutions of panel tiles x_next .. x_next + kLook - 1: load all, then
      // publish the ready prefix in order
      unsigned long long va[kLook], vb[kLook];
#pragma unroll
      for (int w = 0; w < kLook; ++w) {
        const int i = x_next + w;
        va[w] = vb[w] = 0ull;
        if (i < nstaged) {
          va[w] = ld_relaxed64(slots + (size_t)i * kCB + lane);
          vb[w] = ld_relaxed64(slots + (size_t)i * kCB + lane + 32);
        }
      }
      bool go = true;
      const int x_start = x_next;
#pragma unroll
      for (int w = 0; w < kLook; ++w) {
        const int i = x_start + w;
        if (go && i < nstaged) {
          const int j = i % kXRing;
          bool ok = (unsigned)(va[w] >> 32) == epoch && (unsigned)(vb[w] >> 32) == epoch;
          ok = __all_sync(0xffffffffu, ok);
          if (ok && i >= kXRing) ok = tc::mbar_try_wait(&S.xempty[j], ((i / kXRing) - 1) & 1);
          ok = __all_sync(0xffffffffu, ok);
          if (ok) {
            S.xs[j][lane] = __uint_as_float((unsigned)va[w]);
            S.xs[j][lane + 32] = __uint_as_float((unsigned)vb[w]);
            tc::mbar_arrive(&S.xfull[j]);
            x_next = i + 1;
          } else {
            go = false;
          }
        }
      }
      // progress check every 16 idle rounds: timer and abort flag, and the
      // global status word only after 20 us without progress
      bool quit = false;
      if (x_next != x_start) {
        iter = 0;
        t_last = 0;
      } else if ((++iter & 15u) == 0) {
        const uint64_t now = tc::globaltimer();
        if (t_last == 0) t_last = now;
        const uint64_t el = now - t_last;
        quit = el > limit_ns || *(volatile int*)&S.abort_flag ||
               (el > 20000ull && *(volatile unsigned*)status != 0);
      }
      quit = __any_sync(0xffffffffu, quit);
      if (quit) {
        if (lane == 0) {
          atomicOr(status, kStatusTimeout);
          S.abort_flag = 1;
        }
        break;
      }
    }
    if (lane == 0) S.issued = tma_next;
  } else if (active) {
    // ---------------- consumer warps ----------------
    // the right-hand side is read first so its latency hides behind the wait
    const float rhs_v = (tid < kCB && b0 + tid < n) ? x[(size_t)(b0 + tid) * incx] : 0.f;
    bool ok = tc::mbar_wait(&S.setup_bar, 0, limit_ns);
    // op(D) masked: stored element (b0 + rr, b0 + cc) sits at raw[0][cc][rr].
    // An upper op(D) is stored index-reversed (L = P op(D) P, P the reversal),
    // which is lower triangular, and so are the rows of the right-hand sides.
    // Every load of a loop before its stores: a store the compiler cannot
    // prove disjoint from the next load would cost a shared-memory round trip
    // per element.
    constexpr int kPerT = kCB * kCB / kCons;
    {
      float vals[kPerT];
#pragma unroll
      for (int k = 0; k < kPerT; ++k) {
        const int e = tid + k * kCons;
        vals[k] = S.raw[0][e / kCB][e % kCB];
      }
#pragma unroll
      for (int k = 0; k < kPerT; ++k) {
        const int e = tid + k * kCons;
        const int rr = e % kCB, cc = e / kCB;
        float v = vals[k];
        const int r = trans ? cc : rr, c = trans ? rr : cc;
        const bool in_tri = lower_eff ? r >= c : r <= c;
        if (r == c) v = (unit || b0 + r >= n) ? 1.f : v;
        else if (!in_tri) v = 0.f;
        S.Dm[lower_eff ? r : kCB - 1 - r][lower_eff ? c : kCB - 1 - c] = v;
      }
    }
    // op(tile) row-major for blocks b-1 (Top) and b-2 (W), rows in L's order;
    // zero where absent
    {
      float t1[kPerT], t2[kPerT];
#pragma unroll
      for (int k = 0; k < kPerT; ++k) {
        const int e = tid + k * kCons;
        const int i = trans ? e / kCB : e % kCB, c = trans ? e % kCB : e / kCB;
        t1[k] = s >= 1 ? (trans ? S.raw[1][i][c] : S.raw[1][c][i]) : 0.f;
        t2[k] = s >= 2 ? (trans ? S.raw[2][i][c] : S.raw[2][c][i]) : 0.f;
      }
#pragma unroll
      for (int k = 0; k < kPerT; ++k) {
        const int e = tid + k * kCons;
        const int i = trans ? e / kCB : e % kCB, c = trans ? e % kCB : e / kCB;
        const int li = lower_eff ? i : kCB - 1 - i;
        S.Top[li][c] = t1[k];
        S.W[li][c] = t2[k];
      }
    }
    if (tid < kCB) S.rhs[tid] = rhs_v;
    bar_consumers();
    if (tid < kCB) S.rdiag[tid] = 1.f / S.Dm[tid][tid];
    bar_consumers();
    // [inv(L) | inv(L) Top | inv(L) W] by column substitutions into raw[0..2]
    // (the raw tiles are consumed); the products the block does not need
    // (no block b-1 or b-2) are skipped.
    {
      const int ncols = kCB * (1 + (s >= 1) + (s >= 2));
      if (tid < ncols) solve_column(S, tid, S.raw);
    }
    bar_consumers();
    // Registers of thread (r, q): inv(op(D))[r][16q + j], and rows r of
    // M1 = inv(op(D)) op(tile b-1), M2 = inv(op(D)) op(tile b-2), columns
    // 16q + j.  With op(D) upper, inv(op(D)) = P inv(L) P and M = P X.
    const int r = tid >> 2, q = tid & 3, c0 = q * 16;
    float inv[16], M1[16], M2[16];
    const int xr = lower_eff ? r : kCB - 1 - r;
    const int sw = (xr & 7) << 2;  // the swizzle moves whole aligned groups of 4
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      // inv: columns c0 + 4g .. c0 + 4g + 3, or (upper) 63 - c0 - 4g down to 60 - c0 - 4g
      const int ci = lower_eff ? c0 + 4 * g : kCB - 4 - c0 - 4 * g;
      const float4 vi4 = *reinterpret_cast<const float4*>(&S.raw[0][xr][ci ^ sw]);
      const float4 m14 = *reinterpret_cast<const float4*>(&S.raw[1][xr][(c0 + 4 * g) ^ sw]);
      const float4 m24 = *reinterpret_cast<const float4*>(&S.raw[2][xr][(c0 + 4 * g) ^ sw]);
      inv[4 * g + 0] = lower_eff ? vi4.x : vi4.w;
      inv[4 * g + 1] = lower_eff ? vi4.y : vi4.z;
      inv[4 * g + 2] = lower_eff ? vi4.z : vi4.y;
      inv[4 * g + 3] = lower_eff ? vi4.w : vi4.x;
      M1[4 * g + 0] = s >= 1 ? m14.x : 0.f;
      M1[4 * g + 1] = s >= 1 ? m14.y : 0.f;
      M1[4 * g + 2] = s >= 1 ? m14.z : 0.f;
      M1[4 * g + 3] = s >= 1 ? m14.w : 0.f;
      M2[4 * g + 0] = s >= 2 ? m24.x : 0.f;
      M2[4 * g + 1] = s >= 2 ? m24.y : 0.f;
      M2[4 * g + 2] = s >= 2 ? m24.z : 0.f;
      M2[4 * g + 3] = s >= 2 ? m24.w : 0.f;
    }

    // panel: acc = sum over solve indices k <= s-3 of op(A)(b, k) x_k
    float acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = 0.f;
    for (int i = 0; i < npanel && ok; ++i) {
      const int st = i % kCStages, j = i % kXRing;
      const bool staged = i < s_first;  // earlier cluster: staged by the producer
      ok = tc::mbar_wait(&S.full[st], (i / kCStages) & 1, limit_ns) &&
           (!staged || tc::mbar_wait(&S.xfull[j], (i / kXRing) & 1, limit_ns));
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      // solution values lane and lane + 32 of block i
      float x0, x1;
      if (staged) {
        x0 = S.xs[j][lane];
        x1 = S.xs[j][lane + 32];
      } else {
        // this cluster: read the pushed copy directly
        const unsigned long long* src = S.xin[i - s_first];
        unsigned long long v0, v1;
        uint64_t t0 = 0;
        for (unsigned spins = 0;; ++spins) {
          v0 = ld_local_tag(src + lane);
          v1 = ld_local_tag(src + lane + 32);
          const bool got = (unsigned)(v0 >> 32) == epoch && (unsigned)(v1 >> 32) == epoch;
          if (__all_sync(0xffffffffu, got)) break;
          const uint64_t now = tc::globaltimer();
          if (spins == 0) t0 = now;
          bool quit = now - t0 > limit_ns;
          if ((spins & 15u) == 0) quit = quit || *(volatile int*)&S.abort_flag;
          if (__any_sync(0xffffffffu, quit)) {
            ok = false;
            break;
          }
        }
        if (!ok) break;
        x0 = __uint_as_float((unsigned)v0);
        x1 = __uint_as_float((unsigned)v1);
      }
      const float (*T)[kCB] = S.ring[st];
      if (!trans) {
        // T[c][r]: rows lane, lane + 32; this warp's columns 8w .. 8w + 7,
        // whose solution values sit in lanes (8w + u) mod 32 of x0 or x1
        const float xsrc = warp < 4 ? x0 : x1;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const float xu = __shfl_sync(0xffffffffu, xsrc, (warp * 8 + u) & 31);
          acc[0] = fmaf(T[warp * 8 + u][lane], xu, acc[0]);
          acc[1] = fmaf(T[warp * 8 + u][lane + 32], xu, acc[1]);
        }
      } else {
        // T[r][c]: this warp's rows 8w .. 8w + 7; columns lane, lane + 32
#pragma unroll
        for (int u = 0; u < 8; ++u)
          acc[u] = fmaf(T[warp * 8 + u][lane], x0, fmaf(T[warp * 8 + u][lane + 32], x1, acc[u]));
      }
      __syncwarp();
      if (lane == 0) {
        tc::mbar_arrive(&S.empty[st]);
        if (staged) tc::mbar_arrive(&S.xempty[j]);
      }
    }
    if (!ok && lane == 0) {
      atomicOr(status, kStatusTimeout);
      S.abort_flag = 1;
    }
    // v = rhs - acc
    if (!trans) {
      S.part[warp][lane] = acc[0];
      S.part[warp][lane + 32] = acc[1];
      bar_consumers();
      if (tid < kCB) {
        float a = 0.f;
#pragma unroll
        for (int w = 0; w < 8; ++w) a += S.part[w][tid];
        S.v[vi(tid)] = S.rhs[tid] - a;
      }
    } else {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        float a = acc[u];
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == u) S.v[vi(warp * 8 + u)] = S.rhs[warp * 8 + u] - a;
      }
    }
    bar_consumers();
    // y = inv(D) v, then the two most recent blocks through M2 and M1
    float y = 0.f;
    {
#pragma unroll
      for (int j = 0; j < 16; ++j) y = fmaf(inv[j], S.v[vi(c0 + j)], y);
      y = quad_sum(y);
    }
    float xv[16];
    if (s >= 2) {
      const bool local = (int)rank >= 2;
      const unsigned long long* src = local ? &S.xin[rank - 2][0] : slots + (size_t)(s - 2) * kCB;
      bool got = ok && fetch_x(src, local, epoch, lane, xv, status, &S.abort_flag, limit_ns);
      y -= quad_sum(dot16(M2, xv));
      ok = __all_sync(0xffffffffu, got);
    }
    if (s >= 1) {
      const bool local = (int)rank >= 1;
      const unsigned long long* src = local ? &S.xin[rank - 1][0] : slots + (size_t)(s - 1) * kCB;
      bool got = ok && fetch_x(src, local, epoch, lane, xv, status, &S.abort_flag, limit_ns);
      y -= quad_sum(dot16(M1, xv));
      ok = __all_sync(0xffffffffu, got);
    }
    if (ok) {
      // rows past n solve to 0 (identity diagonal, zero-filled tiles)
      const unsigned long long val = ((unsigned long long)epoch << 32) | __float_as_uint(y);
      if (q == 3) st_relaxed64(slots + (size_t)s * kCB + r, val);
      for (int d = (int)rank + 1 + q; d < kCl; d += 4) st_cluster_u64(map_rank(&S.xin[rank][r], d), val);
      if (q == 1 && b0 + r < n) x[(size_t)(b0 + r) * incx] = y;
    } else if (lane == 0) {
      atomicOr(status, kStatusTimeout);
      S.abort_flag = 1;
    }
  }
  __syncthreads();
  if (active && tid == kCons) {
    // Every issued tile load lands before the CTA leaves (after an abort some
    // may never have been consumed).  Loads of tiles before issued - stages
    // were consumed, so only the last ring's worth can be in flight.  This
    // wait is bounded by its own second, not the caller's wait limit, which
    // may be far shorter than a copy.
    const int issued = S.issued;
    const int first = issued > kCStages ? issued - kCStages : 0;
    const uint64_t drain_ns = limit_ns > 1000000000ull ? limit_ns : 1000000000ull;
    for (int i = first; i < issued; ++i)
      tc::mbar_wait(&S.full[i % kCStages], (i / kCStages) & 1, drain_ns);
    tc::mbar_wait(&S.setup_bar, 0, drain_ns);
  }
  __syncthreads();
  cluster_sync_all();
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(done, 1u) == gridDim.x - 1) {
      *ticket = 0u;
      *done = 0u;
      __threadfence();
      atomicExch(epoch_word, epoch);
    }
  }
}

}  // namespace
}  // namespace coral

using namespace coral;

extern "C" coral_status_t coral_strsv(coral_handle_t hh, int uplo, int trans, int diag, size_t n,
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
  constexpr int nb = 64;
  const size_t nblk = (n + nb - 1) / nb;
  if (n > (size_t)INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  if (H->trsv_slots_len < nblk * nb) {
    if (H->trsv_slots) {
      CORAL_CUDA(H, cudaStreamSynchronize(H->stream));
      cudaFree(H->trsv_slots);
      H->trsv_slots = nullptr;
      H->trsv_slots_len = 0;
    }
    const size_t len = ((nblk * nb + 65535) / 65536) * 65536;
    CORAL_CUDA(H, cudaMalloc(&H->trsv_slots, len * sizeof(unsigned long long)));
    CORAL_CUDA(H, cudaMemsetAsync(H->trsv_slots, 0, len * sizeof(unsigned long long), H->stream));
    H->trsv_slots_len = len;
  }
  const bool t = trans != CORAL_NO_TRANSPOSE;
  const bool lower_eff = (uplo == CORAL_LOWER) != t;
  const uint64_t limit_ns = H->wait_limit * 32ull;
  static uint64_t attr_devices[2] = {0, 0};  // bit d: attribute set on device d, per kernel
  const uint64_t bit = H->device < 64 ? (1ull << H->device) : 0;
  CUtensorMap map;
  const bool tma_ok = (lda % 4) == 0 && aligned16(matrix) &&
                      encode_kmajor_map(&map, matrix, 4, n, n, lda * 4, kCB, kCB, 0);
  if (tma_ok) {
    const size_t smem = sizeof(ClusterSmem) + 1024;
    static int cluster_size[64] = {0};  // per device: 16 where the hardware places it, else 8
    int& cl = cluster_size[H->device < 64 ? H->device : 63];
    if (!(attr_devices[0] & bit) || !bit || cl == 0) {
      CORAL_CUDA(H, cudaFuncSetAttribute(k_trsv_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      cl = 8;
      if (cudaFuncSetAttribute(k_trsv_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
        cudaLaunchConfig_t q = {};
        cudaLaunchAttribute qa[1];
        qa[0].id = cudaLaunchAttributeClusterDimension;
        qa[0].val.clusterDim.x = 16;
        qa[0].val.clusterDim.y = qa[0].val.clusterDim.z = 1;
        q.gridDim = dim3(16);
        q.blockDim = dim3(kCThreads);
        q.dynamicSmemBytes = smem;
        q.attrs = qa;
        q.numAttrs = 1;
        int active = 0;
        if (cudaOccupancyMaxActiveClusters(&active, k_trsv_cluster, &q) == cudaSuccess && active >= 1) cl = 16;
      }
      cudaGetLastError();  // a refused query leaves cl at 8, not an error
      attr_devices[0] |= bit;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(((nblk + cl - 1) / cl) * cl));
    cfg.blockDim = dim3(kCThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = H->stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    timed_begin(H);
    const cudaError_t le = cudaLaunchKernelEx(
        &cfg, k_trsv_cluster, map, (int)n, x, incx, lower_eff, t, diag == CORAL_UNIT, H->trsv_slots,
        &H->words->trsv_ticket, &H->words->trsv_done, &H->words->trsv_epoch, &H->words->status,
        limit_ns);
    if (le != cudaSuccess) {
      timed_end(H);
      count_launch();
      cudaGetLastError();
      return cuda_status(H, le);
    }
  } else {
    const size_t smem = 2 * (size_t)nb * (nb + 1) * sizeof(float);
    if (!(attr_devices[1] & bit) || !bit) {
      CORAL_CUDA(H, cudaFuncSetAttribute(k_trsv<nb>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr_devices[1] |= bit;
    }
    timed_begin(H);
    k_trsv<nb><<<(unsigned)nblk, 4 * nb, smem, H->stream>>>(
        (int)n, matrix, lda, x, incx, lower_eff, t, diag == CORAL_UNIT, H->trsv_slots,
        &H->words->trsv_ticket, &H->words->trsv_done, &H->words->trsv_epoch, &H->words->status,
        limit_ns);
  }
  coral_status_t s = launch_status(H);
  timed_end(H);
  return s;
}
