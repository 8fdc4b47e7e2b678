// STRSV: solve op(A) x = b in place, A triangular (strsv.rs:60-74 ->
// strlsv.rs / strusv.rs).  ConjugateTranspose == Transpose.
//
// One launch.  op(A) is cut into NB-row blocks (NB = 64, or 128 for large n or
// when the handle asks for it); each CTA takes a ticket from a
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

namespace coral {
namespace {

// Block size NB (64 or 128 rows); 4 threads per row.
template <int NB> struct TrsvCfg {
  static constexpr int kThreads = 4 * NB;
  static constexpr int kPer = NB * NB / kThreads;  // tile elements per thread
  static constexpr int kG = NB == 64 ? 4 : 2;     // panel tiles loaded per group
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

  // ---- 2. panel: acc = sum over solved blocks k of op(A)(blk, k) x_k ----
  const int r = tid % kNB, q = tid / kNB;
  float acc = 0.f;
  const int npanel = lower_eff ? blk : nblk - 1 - blk;
  for (int g0 = 0; g0 < npanel; g0 += kG) {
    float reg[kG][kPer];
#pragma unroll
    for (int g = 0; g < kG; ++g) {
      const int idx = g0 + g;
      const int k = lower_eff ? idx : blk + 1 + idx;
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
      const int k = lower_eff ? idx : blk + 1 + idx;
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
            if (gtimer() - t0 > limit_ns ||
                ((++spins & 15u) == 0 && *(volatile unsigned*)status != 0)) {
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
  const int nb = H->trsv_block == 128 || (H->trsv_block == 0 && n >= 8192) ? 128 : 64;
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
  const size_t smem = 2 * (size_t)nb * (nb + 1) * sizeof(float);
  static uint64_t attr_devices[2] = {0, 0};  // bit d: attribute set on device d, per block size
  const uint64_t bit = H->device < 64 ? (1ull << H->device) : 0;
  uint64_t& mask = attr_devices[nb == 128];
  if (!(mask & bit) || !bit) {
    if (nb == 128)
      CORAL_CUDA(H, cudaFuncSetAttribute(k_trsv<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else
      CORAL_CUDA(H, cudaFuncSetAttribute(k_trsv<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mask |= bit;
  }
  timed_begin(H);
  if (nb == 128)
    k_trsv<128><<<(unsigned)nblk, 512, smem, H->stream>>>(
        (int)n, matrix, lda, x, incx, lower_eff, t, diag == CORAL_UNIT, H->trsv_slots,
        &H->words->trsv_ticket, &H->words->trsv_done, &H->words->trsv_epoch, &H->words->status,
        H->wait_limit * 32ull);
  else
    k_trsv<64><<<(unsigned)nblk, 256, smem, H->stream>>>(
        (int)n, matrix, lda, x, incx, lower_eff, t, diag == CORAL_UNIT, H->trsv_slots,
        &H->words->trsv_ticket, &H->words->trsv_done, &H->words->trsv_epoch, &H->words->status,
        H->wait_limit * 32ull);
  coral_status_t s = launch_status(H);
  timed_end(H);
  return s;
}
