// DTRSV, CTRSV, ZTRSV: solve op(A) x = b in place, A triangular, op in
// {N, T, C} (dtrsv.rs, ctrsv.rs, ztrsv.rs -> the *trlsv / *trusv files).
// Complex data is interleaved (re, im) with lda / incx in complex units.
//
// One launch, one 64-row block of the solve per CTA, in clusters of 16 CTAs
// (8 where 16 cannot be placed).  Rank 0 of each cluster takes a ticket, so
// the cluster with ticket t solves blocks 16 t .. 16 t + 15 in solve order and
// only waits for clusters that started earlier -- no deadlock whatever the
// scheduling.  A CTA
//   1. stages its diagonal block of op(A) in shared memory (unstored triangle
//      masked, unit diagonal applied, conjugated for op C), forms the
//      reciprocals of its diagonal and scales each row by its reciprocal
//      (negated, ready for the updates), and reads its right-hand side;
//   2. for every earlier block k in solve order: loads its panel tile of
//      op(A) into registers, then reads x_k from block k's published slots
//      and accumulates op(A)(b, k) x_k -- four threads per row, 16 columns
//      each;
//   3. solves the row-scaled system by forward (backward) substitution in
//      one warp, fully unrolled (the diagonal block is never inverted: FP64
//      substitution as the reference does, dtrlsv.rs);
//   4. writes x_b over b, pushes it into the shared memory of the later CTAs
//      of its cluster (the next block's first) and publishes it in its slots
//      for later clusters: within a cluster a block's solution reaches the
//      next one through distributed shared memory instead of an L2 round trip.
// Slots: every 32-bit word of a block's solution is published as one 64-bit
// slot (epoch << 32) | word, so a single load delivers both the readiness of
// that word and its value (aligned 64-bit accesses are single-copy atomic):
// a consumer's poll is its data load.  The last CTA resets the ticket counter
// and publishes the call's epoch, so no reset pass is needed.  Waits give up
// after the handle's wait limit and set the status word.
#include "common.cuh"
#include "field.cuh"
#include "tc_common.cuh"

#include <type_traits>

namespace coral {
namespace {

// Block edge: 64 rows for every element type, four threads per block row.
// 128-row blocks halve the serial hand-offs but double each block's
// substitution chain; at n = 4096 they measured slower (dtrsv 253 against
// 200 us, ctrsv 250 against 187 us), and a complex128 block of 128 rows
// would not fit in shared memory.
template <typename T> constexpr int kTBOf = 64;
// Substitution form per element type (see substitute_strided() and
// substitute()), as measured at n = 4096: two consecutive rows per lane for
// double (dtrsv 173 us, against 200 strided); rows 32 apart for complex,
// whose wider elements make the consecutive form slower (ctrsv 236 against
// 187 us, ztrsv 356 against 277 us).
template <typename T> constexpr int kRowsPerLaneOf = std::is_same<T, double>::value ? 2 : 0;   // 0: strided

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Cluster shared-memory accesses: a 32-bit load from another CTA's shared
// memory, a 64-bit store into it, and a 64-bit load of this CTA's shared
// memory that observes those stores.
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
constexpr int kDczClMax = 16;  // CTAs per cluster: 16, or 8 where 16 cannot be placed

// 32-bit words per element (slots per element).
template <typename T> constexpr int kWords = (int)(sizeof(T) / 4);

// Substitution on the row-scaled diagonal block in one warp, fully unrolled.
// D holds -op(A)(i, j) / op(A)(i, i) off the diagonal and v the scaled
// right-hand side, so every x_i is its row's final v_i.
//
// Strided form: lane owns rows lane + 32 m (m < TB / 32).  At step j the
// owner's value is x_j; it is broadcast and every later row i takes
// v_i += D[i][j] x_j -- one shuffle round per row on the critical path.
template <typename T, int TB, bool kLower>
__device__ __forceinline__ void substitute_strided(const T (*D)[TB + 1], T (&v)[TB / 32], int lane) {
  using F = Fld<T>;
#pragma unroll
  for (int s = 0; s < TB; ++s) {
    const int j = kLower ? s : TB - 1 - s;
    const T xj = F::shfl(v[j / 32], j & 31);
#pragma unroll
    for (int m = 0; m < TB / 32; ++m) {
      const int i = lane + 32 * m;
      if (kLower ? i > j : i < j) F::mac(v[m], D[i][j], xj);
    }
  }
}

// Consecutive form: lane l < TB / R owns
// the R consecutive rows R l .. R l + R - 1 (v[0..R-1]).  In solve order, the
// owner of the next R rows finishes them among themselves (R - 1 dependent
// multiply-adds, no communication), broadcasts the R values, and every lane
// whose rows come later applies them.  The critical path per R rows is R
// multiply-adds and one shuffle round, against one shuffle per row when each
// lane owns rows 32 apart.
template <typename T, int TB, int R, bool kLower>
__device__ __forceinline__ void substitute(const T (*D)[TB + 1], T (&v)[R], int lane) {
  using F = Fld<T>;
  constexpr int P = TB / R;   // owner lanes
#pragma unroll
  for (int s = 0; s < P; ++s) {
    const int p = kLower ? s : P - 1 - s;
    const int j0 = p * R;
    if (lane == p) {
      if (kLower) {
#pragma unroll
        for (int a = 0; a < R; ++a)
#pragma unroll
          for (int b = a + 1; b < R; ++b) F::mac(v[b], D[j0 + b][j0 + a], v[a]);
      } else {
#pragma unroll
        for (int a = R - 1; a >= 0; --a)
#pragma unroll
          for (int b = a - 1; b >= 0; --b) F::mac(v[b], D[j0 + b][j0 + a], v[a]);
      }
    }
    T xr[R];
#pragma unroll
    for (int a = 0; a < R; ++a) xr[a] = F::shfl(v[a], p);
    if (lane < P && (kLower ? lane > p : lane < p)) {
      const int i0 = lane * R;
      // the next owner's first row to finish gets its updates first
#pragma unroll
      for (int bb = 0; bb < R; ++bb) {
        const int b = kLower ? bb : R - 1 - bb;
#pragma unroll
        for (int a = 0; a < R; ++a) F::mac(v[b], D[i0 + b][j0 + a], xr[a]);
      }
    }
  }
}
__device__ __forceinline__ uint64_t gtime() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T, bool kConj, int kTB = kTBOf<T>, int kTThr = 4 * kTBOf<T>>
__global__ void __launch_bounds__(kTThr, 1)
k_trsv_g(int n, const T* __restrict__ A, size_t lda, T* x, size_t incx, bool lower_eff, bool trans,
         bool unit, unsigned long long* slots, unsigned* ticket, unsigned* done, unsigned* epoch_word,
         unsigned* status, uint64_t limit_ns) {
  using F = Fld<T>;
  constexpr int W = kWords<T>;
  constexpr int kSlotWords = kTB * W;   // slots per block (<= kTThr)
  extern __shared__ __align__(16) unsigned char smem[];
  T(*D)[kTB + 1] = reinterpret_cast<T(*)[kTB + 1]>(smem);   // op(A) diagonal block
  // solutions pushed by the earlier CTAs of the cluster: xin[rank][word]
  unsigned long long(*xin)[kSlotWords] =
      reinterpret_cast<unsigned long long(*)[kSlotWords]>(smem + sizeof(T) * kTB * (kTB + 1));
  __shared__ T xk[kTB];        // solution of the block being applied
  __shared__ T rv[kTB];        // right-hand side, then this block's solution
  __shared__ T rdiag[kTB];     // reciprocals of the diagonal
  __shared__ int abort_flag;
  __shared__ unsigned sticket, sepoch, my_ticket, my_epoch;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nblk = (n + kTB - 1) / kTB;
  const unsigned rank = tc::cluster_ctarank();
  unsigned ncl_u;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(ncl_u));
  const int ncl = (int)ncl_u;
  for (int i = tid; i < ncl * kSlotWords; i += kTThr) (&xin[0][0])[i] = 0ull;
  if (tid == 0) {
    abort_flag = 0;
    if (rank == 0) {
      // one ticket per cluster: the cluster takes the next ncl blocks in solve
      // order, so it only ever waits for clusters that started earlier
      sticket = atomicAdd(ticket, 1u);
      const unsigned e = *(volatile unsigned*)epoch_word + 1u;
      sepoch = e ? e : 1u;   // slots start at 0: never a live epoch
    }
  }
  tc::cluster_sync();
  if (tid == 0) {
    my_ticket = ld_cluster_u32(tc::mapa_shared(tc::smem_u32(&sticket), 0));
    my_epoch = ld_cluster_u32(tc::mapa_shared(tc::smem_u32(&sepoch), 0));
  }
  __syncthreads();
  const unsigned epoch = my_epoch;
  const int s_first = (int)my_ticket * ncl;   // solve index of this cluster's rank 0
  const int s = s_first + (int)rank;          // this CTA's solve index
  const bool active = s < nblk;
  auto blk_of = [&](int sp) { return lower_eff ? sp : nblk - 1 - sp; };
  const int blk = active ? blk_of(s) : 0;
  const int b0 = blk * kTB;
  auto opv = [](T v) { return kConj ? F::conj(v) : v; };

  if (active) {
  // ---- 1. diagonal block, its reciprocals, the row scaling; right-hand side ----
  for (int e = tid; e < kTB * kTB; e += kTThr) {
    const int rr = e % kTB, cc = e / kTB;          // stored element (b0 + rr, b0 + cc)
    const int gr = b0 + rr, gc = b0 + cc;
    T v = (gr < n && gc < n) ? A[gr + (size_t)gc * lda] : F::zero();
    const int r = trans ? cc : rr, c = trans ? rr : cc;   // op(A)(r, c)
    const bool in_tri = lower_eff ? r >= c : r <= c;
    if (r == c) v = (unit || b0 + r >= n) ? F::one() : opv(v);
    else v = in_tri ? opv(v) : F::zero();
    D[r][c] = v;
  }
  if (tid < kTB) rv[tid] = (b0 + tid < n) ? x[(size_t)(b0 + tid) * incx] : F::zero();
  __syncthreads();
  if (tid < kTB) rdiag[tid] = F::div(F::one(), D[tid][tid]);
  __syncthreads();
  for (int e = tid; e < kTB * kTB; e += kTThr) {
    const int r = e / kTB, c = e % kTB;
    if (r != c) D[r][c] = F::neg(F::mul(D[r][c], rdiag[r]));
  }

  // ---- 2. panel: acc(r) = sum over earlier blocks k of op(A)(b, k) x_k,
  // in solve order; a block of this cluster is read from the copy its CTA
  // pushed into this CTA's shared memory, an earlier cluster's from its slots
  constexpr int kQ = kTB / 4;           // columns per thread of a panel tile
  static_assert(kSlotWords <= kTThr, "one slot per thread");
  uint32_t* xkw = reinterpret_cast<uint32_t*>(xk);
  const int r = tid >> 2, q = tid & 3;
  T acc = F::zero();
  for (int idx = 0; idx < s; ++idx) {
    const int k = blk_of(idx);
    const int k0 = k * kTB;
    // thread (r, q) takes columns q * kQ + j of the tile when A is read as
    // stored (lanes of a warp on 8 consecutive rows of 4 column runs), and
    // q + 4 j when it is read transposed, where the 4 threads of a row then
    // read 4 consecutive elements of one stored column (measured: DTRSV T
    // 221 -> 134-140 us, CTRSV T 221 -> 146-153, ZTRSV T 274 -> 204-216 at
    // n = 4096).  The tile is held as stored; the conjugation of op C is
    // applied where an element is used.
    const bool tcols = trans;
    T a[kQ];
#pragma unroll
    for (int j = 0; j < kQ; ++j) {
      const int gr = b0 + r, gc = k0 + (tcols ? q + 4 * j : q * kQ + j);   // op(A)(gr, gc)
      const bool in = gr < n && gc < n;
      a[j] = in ? (trans ? A[gc + (size_t)gr * lda] : A[gr + (size_t)gc * lda]) : F::zero();
    }
    if (tid < kSlotWords) {
      const bool local = idx >= s_first;
      const unsigned long long* sp = local ? &xin[idx - s_first][tid] : slots + (size_t)k * kSlotWords + tid;
      unsigned long long w = local ? ld_local_tag(sp) : ld_relaxed_u64(sp);
      if ((unsigned)(w >> 32) != epoch) {
        const uint64_t t0 = gtime();
        for (unsigned spins = 1;; ++spins) {
          w = local ? ld_local_tag(sp) : ld_relaxed_u64(sp);
          if ((unsigned)(w >> 32) == epoch) break;
          const uint64_t el = gtime() - t0;
          if (el > limit_ns || ((spins & 15u) == 0 && el > 20000ull && *(volatile unsigned*)status != 0)) {
            atomicOr(status, kStatusTimeout);
            abort_flag = 1;
            break;
          }
        }
      }
      xkw[tid] = (uint32_t)w;
    }
    __syncthreads();
    if (abort_flag) break;
#pragma unroll
    for (int j = 0; j < kQ; ++j) F::mac(acc, opv(a[j]), xk[tcols ? q + 4 * j : q * kQ + j]);
    __syncthreads();
  }
  acc = F::add(acc, F::shfl_xor(acc, 1));
  acc = F::add(acc, F::shfl_xor(acc, 2));
  if (q == 0) rv[r] = F::mul(F::sub(rv[r], acc), rdiag[r]);
  __syncthreads();

  // ---- 3. substitution on the row-scaled diagonal block (one warp) ----
  if (warp == 0 && !abort_flag) {
    constexpr int R = kRowsPerLaneOf<T>;
    if constexpr (R == 0) {
      T v[kTB / 32];
#pragma unroll
      for (int m = 0; m < kTB / 32; ++m) v[m] = rv[lane + 32 * m];
      if (lower_eff) substitute_strided<T, kTB, true>(D, v, lane);
      else substitute_strided<T, kTB, false>(D, v, lane);
#pragma unroll
      for (int m = 0; m < kTB / 32; ++m) rv[lane + 32 * m] = v[m];
    } else {
      T v[R];
      const bool owner = lane < kTB / R;
#pragma unroll
      for (int a = 0; a < R; ++a) v[a] = owner ? rv[lane * R + a] : F::zero();
      if (lower_eff) substitute<T, kTB, R, true>(D, v, lane);
      else substitute<T, kTB, R, false>(D, v, lane);
      if (owner) {
#pragma unroll
        for (int a = 0; a < R; ++a) rv[lane * R + a] = v[a];
      }
    }
  }
  __syncthreads();

  // ---- 4. publish: x_b over b, every word of it into the shared memory of
  // the later CTAs of the cluster (the next one first) and into the block's
  // slots for later clusters ----
  if (!abort_flag) {
    if (tid < kTB && b0 + tid < n) x[(size_t)(b0 + tid) * incx] = rv[tid];
    if (tid < kSlotWords) {
      const unsigned long long val =
          ((unsigned long long)epoch << 32) | reinterpret_cast<const uint32_t*>(rv)[tid];
      const uint32_t mine = tc::smem_u32(&xin[rank][tid]);
      for (int d = (int)rank + 1; d < ncl && s_first + d < nblk; ++d)
        st_cluster_u64(tc::mapa_shared(mine, (uint32_t)d), val);
      st_relaxed_u64(slots + (size_t)blk * kSlotWords + tid, val);
    }
  }
  }  // active
  // No CTA leaves while a CTA of its cluster may still push into it.
  __syncthreads();
  tc::cluster_sync();
  // The last CTA to finish (aborted or not) resets the ticket counter and
  // publishes this call's epoch for the next call.
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

template <typename T>
coral_status_t trsv_g(Handle* H, int uplo, int trans, int diag, size_t n, const void* matrix, size_t lda,
                      void* x, size_t incx, size_t align) {
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (trans < CORAL_NO_TRANSPOSE || trans > CORAL_CONJ_TRANSPOSE) return bad_arg(H, 2);
  if (diag != CORAL_UNIT && diag != CORAL_NON_UNIT) return bad_arg(H, 3);
  if (n == 0) return CORAL_OK;
  if (!matrix) return bad_arg(H, 5);
  if (lda < n) return bad_arg(H, 6);
  if (!x) return bad_arg(H, 7);
  if (incx == 0) return bad_arg(H, 8);
  if (((uintptr_t)matrix | (uintptr_t)x) & (align - 1)) return bad_arg(H, 5);
  if (n > (size_t)INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  constexpr int kTB = kTBOf<T>, kTThr = 4 * kTBOf<T>;
  const size_t nblk = (n + kTB - 1) / kTB;
  const size_t nslots = nblk * kTB * kWords<T>;   // one slot per 32-bit word of x
  if (H->trsv_slots_len < nslots) {
    if (H->trsv_slots) {
      CORAL_CUDA(H, cudaStreamSynchronize(H->stream));
      cudaFree(H->trsv_slots);
      H->trsv_slots = nullptr;
      H->trsv_slots_len = 0;
    }
    const size_t len = ((nslots + 65535) / 65536) * 65536;
    CORAL_CUDA(H, cudaMalloc(&H->trsv_slots, len * sizeof(unsigned long long)));
    CORAL_CUDA(H, cudaMemsetAsync(H->trsv_slots, 0, len * sizeof(unsigned long long), H->stream));
    H->trsv_slots_len = len;
  }
  const bool t = trans != CORAL_NO_TRANSPOSE;
  const bool cj = trans == CORAL_CONJ_TRANSPOSE && !std::is_same<T, double>::value;
  const bool lower_eff = (uplo == CORAL_LOWER) != t;
  const size_t smem = (size_t)kTB * (kTB + 1) * sizeof(T) + (size_t)kDczClMax * kTB * kWords<T> * 8;
  // per device and kernel form: the attributes are set, and the cluster size
  // (16 where the hardware places it, else 8) is chosen, on the first call
  static int cluster_size[2][64] = {{0}};
  int& cl = cluster_size[cj][H->device < 64 ? H->device : 63];
  auto kern = cj ? k_trsv_g<T, true> : k_trsv_g<T, false>;
  if (cl == 0) {
    CORAL_CUDA(H, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int c = 8;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
      cudaLaunchConfig_t q = {};
      cudaLaunchAttribute qa[1];
      qa[0].id = cudaLaunchAttributeClusterDimension;
      qa[0].val.clusterDim.x = 16;
      qa[0].val.clusterDim.y = qa[0].val.clusterDim.z = 1;
      q.gridDim = dim3(16);
      q.blockDim = dim3(kTThr);
      q.dynamicSmemBytes = smem;
      q.attrs = qa;
      q.numAttrs = 1;
      int activec = 0;
      if (cudaOccupancyMaxActiveClusters(&activec, kern, &q) == cudaSuccess && activec >= 1) c = 16;
    }
    cudaGetLastError();  // a refused query leaves the size at 8, not an error
    cl = c;
  }
  T* X = static_cast<T*>(x);
  const T* Am = static_cast<const T*>(matrix);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cl;
  at[0].val.clusterDim.y = at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3((unsigned)(((nblk + cl - 1) / cl) * cl));
  cfg.blockDim = dim3(kTThr);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = H->stream;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  timed_begin(H);
  const cudaError_t le = cudaLaunchKernelEx(&cfg, kern, (int)n, Am, lda, X, incx, lower_eff, t, diag == CORAL_UNIT,
                                            H->trsv_slots, &H->words->trsv_ticket, &H->words->trsv_done,
                                            &H->words->trsv_epoch, &H->words->status, H->wait_limit * 32ull);
  if (le != cudaSuccess) {
    timed_end(H);
    count_launch();
    cudaGetLastError();
    return cuda_status(H, le);
  }
  coral_status_t s = launch_status(H);
  timed_end(H);
  return s;
}

}  // namespace
}  // namespace coral

using namespace coral;

extern "C" {

coral_status_t coral_dtrsv(coral_handle_t hh, int uplo, int trans, int diag, size_t n, const double* matrix,
                           size_t lda, double* x, size_t incx) {
  CORAL_HANDLE(hh);
  return trsv_g<double>(H, uplo, trans, diag, n, matrix, lda, x, incx, 8);
}

coral_status_t coral_ctrsv(coral_handle_t hh, int uplo, int trans, int diag, size_t n, const float* matrix,
                           size_t lda, float* x, size_t incx) {
  CORAL_HANDLE(hh);
  return trsv_g<float2>(H, uplo, trans, diag, n, matrix, lda, x, incx, 8);
}

coral_status_t coral_ztrsv(coral_handle_t hh, int uplo, int trans, int diag, size_t n, const double* matrix,
                           size_t lda, double* x, size_t incx) {
  CORAL_HANDLE(hh);
  return trsv_g<double2>(H, uplo, trans, diag, n, matrix, lda, x, incx, 16);
}

}  // extern "C"
