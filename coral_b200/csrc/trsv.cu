// STRSV: solve op(A) x = b in place, A triangular (strsv.rs:60-74 ->
// strlsv.rs / strusv.rs).  ConjugateTranspose == Transpose.
//
// One launch.  op(A) is cut into 64-row blocks; each CTA takes a ticket from a
// running counter, so block b is handled by the b-th CTA to start (in solve
// order: forward when op(A) is lower, backward when upper) and only ever
// waits for blocks whose CTAs started earlier -- no dependency on scheduling
// order, no deadlock.  A CTA
//   1. stages its diagonal block of op(A) (triangle masked, unit diagonal
//      applied) in shared memory and inverts it (independent of every other
//      block, so it overlaps the solve of earlier blocks);
//   2. streams its row panel of op(A), 4 tiles of 64 x 64 in flight, and
//      for each tile waits for the solution x_k of that block, then
//      accumulates tile * x_k -- tiles of early blocks are ready long before
//      the last one, so the panel streams while the solve front advances;
//   3. forms x_b = inv(D_b) (b_b - acc), writes it over b, and publishes it
//      as 64 epoch-tagged 64-bit slots ((epoch << 32) | float bits, store
//      release).  A consumer polls the slots themselves: one round trip
//      through L2 both signals readiness and delivers the values.
// CORAL solves its diagonal blocks by substitution (strlsv.rs:66-140) with the
// panel update through saxpyf/sdotf; here the blocked diagonal solve uses the
// inverted 64 x 64 block as a small GEMV, which takes the serial substitution
// off the critical path.  Waits are bounded by the handle's wait limit and
// abort early once any CTA has set the status word.
#include "common.cuh"

namespace coral {
namespace {

constexpr int kNB = 64;
constexpr int kG = 4;          // panel tiles loaded per group
constexpr int kTrsvThreads = 256;
constexpr int kPer = kNB * kNB / kTrsvThreads;  // tile elements per thread (16)

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

__global__ void __launch_bounds__(kTrsvThreads)
k_trsv(int n, const float* __restrict__ A, size_t lda, float* x, size_t incx, bool lower_eff,
       bool trans, bool unit, unsigned long long* slots, unsigned long long* ticket,
       unsigned long long ticket_base, unsigned epoch, unsigned* status, uint64_t limit_ns) {
  __shared__ float D[kNB][kNB + 1];    // D[r][c] = op(A)(r, c) of the diagonal block, then inv
  __shared__ float T[kNB][kNB + 1];    // T[c][r] = stored block element (row r, col c)
  __shared__ float xk[kNB];
  __shared__ float red[4][kNB];
  __shared__ float rhs[kNB];
  __shared__ int sblk;
  __shared__ int abort_flag;

  const int nblk = (n + kNB - 1) / kNB;
  const int tid = threadIdx.x;
  if (tid == 0) {
    unsigned long long t = atomicAdd(ticket, 1ull) - ticket_base;
    abort_flag = 0;
    if (t >= (unsigned long long)nblk) {  // ticket count out of step with the host
      atomicOr(status, kStatusTimeout);
      abort_flag = 1;
      t = 0;
    }
    sblk = lower_eff ? (int)t : nblk - 1 - (int)t;
  }
  __syncthreads();
  if (abort_flag) return;
  const int blk = sblk;
  const int b0 = blk * kNB;

  // ---- 1. diagonal block of op(A), masked, and its inverse ----
  for (int e = tid; e < kNB * kNB; e += kTrsvThreads) {
    const int rr = e % kNB, cc = e / kNB;       // stored element (b0+rr, b0+cc)
    const int gr = b0 + rr, gc = b0 + cc;
    float v = (gr < n && gc < n) ? __ldg(A + gr + (size_t)gc * lda) : 0.f;
    // op(A)(r, c): stored (rr, cc) is op element (rr, cc) or (cc, rr).
    const int r = trans ? cc : rr, c = trans ? rr : cc;
    const bool in_tri = lower_eff ? r >= c : r <= c;
    if (r == c) v = (unit || b0 + r >= n) ? 1.f : v;
    else if (!in_tri) v = 0.f;
    D[r][c] = v;
  }
  __syncthreads();
  if (tid < kNB) {
    // Column `c` of inv(D) by substitution on the unit vector e_c, kept in
    // T[c][*] (T is free until the panel phase).
    const int c = tid;
    if (lower_eff) {
      for (int i = 0; i < c; ++i) T[c][i] = 0.f;
      T[c][c] = 1.f / D[c][c];
      for (int i = c + 1; i < kNB; ++i) {
        float s = 0.f;
        for (int j = c; j < i; ++j) s = fmaf(D[i][j], T[c][j], s);
        T[c][i] = -s / D[i][i];
      }
    } else {
      for (int i = c + 1; i < kNB; ++i) T[c][i] = 0.f;
      T[c][c] = 1.f / D[c][c];
      for (int i = c - 1; i >= 0; --i) {
        float s = 0.f;
        for (int j = i + 1; j <= c; ++j) s = fmaf(D[i][j], T[c][j], s);
        T[c][i] = -s / D[i][i];
      }
    }
  }
  __syncthreads();
  // D <- inv(D) (D[r][c] = inv(r, c) = T[c][r])
  for (int e = tid; e < kNB * kNB; e += kTrsvThreads) {
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
      if (abort_flag) return;
      // op(A)(r, c) = stored(r, c) = T[c][r], or stored(c, r) = T[r][c] when transposed
      if (!trans) {
#pragma unroll
        for (int c = q * 16; c < q * 16 + 16; ++c) acc = fmaf(T[c][r], xk[c], acc);
      } else {
#pragma unroll
        for (int c = q * 16; c < q * 16 + 16; ++c) acc = fmaf(T[r][c], xk[c], acc);
      }
      __syncthreads();
    }
  }
  red[q][r] = acc;
  __syncthreads();
  if (tid < kNB) rhs[tid] -= (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]);
  __syncthreads();

  // ---- 3. x_b = inv(D) rhs, publish ----
  float s = 0.f;
#pragma unroll
  for (int c = q * 16; c < q * 16 + 16; ++c) s = fmaf(D[r][c], rhs[c], s);
  red[q][r] = s;
  __syncthreads();
  if (tid < kNB) {
    const float v = (b0 + tid < n) ? (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]) : 0.f;
    if (b0 + tid < n) x[(size_t)(b0 + tid) * incx] = v;
    st_release64(slots + (size_t)blk * kNB + tid,
                 ((unsigned long long)epoch << 32) | __float_as_uint(v));
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
  const size_t nblk = (n + kNB - 1) / kNB;
  if (n > (size_t)INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  if (H->trsv_slots_len < nblk * kNB) {
    if (H->trsv_slots) {
      CORAL_CUDA(H, cudaStreamSynchronize(H->stream));
      cudaFree(H->trsv_slots);
      H->trsv_slots = nullptr;
      H->trsv_slots_len = 0;
    }
    const size_t len = ((nblk * kNB + 65535) / 65536) * 65536;
    CORAL_CUDA(H, cudaMalloc(&H->trsv_slots, len * sizeof(unsigned long long)));
    CORAL_CUDA(H, cudaMemsetAsync(H->trsv_slots, 0, len * sizeof(unsigned long long), H->stream));
    H->trsv_slots_len = len;
  }
  const bool t = trans != CORAL_NO_TRANSPOSE;
  const bool lower_eff = (uplo == CORAL_LOWER) != t;
  H->trsv_epoch += 1;
  if (H->trsv_epoch == 0) H->trsv_epoch = 1;  // flags start at 0: never a valid epoch
  const unsigned long long base = H->trsv_tickets;
  H->trsv_tickets += nblk;
  timed_begin(H);
  k_trsv<<<(unsigned)nblk, kTrsvThreads, 0, H->stream>>>(
      (int)n, matrix, lda, x, incx, lower_eff, t, diag == CORAL_UNIT, H->trsv_slots,
      &H->words->trsv_ticket, base, H->trsv_epoch, &H->words->status, H->wait_limit * 32ull);
  coral_status_t s = launch_status(H);
  timed_end(H);
  return s;
}
