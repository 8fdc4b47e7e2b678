// Internal declarations shared by every translation unit of libcoral_b200.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/coral_b200.h"

namespace coral {

constexpr int kNumSMs = 148;                 // B200: 2 dies x 74 SMs
constexpr uint64_t kDefaultWaitLimit = 1ull << 26;  // ~1 s of 20-ns spins

// Device status word bits (written by bounded waits, read by coral_sync).
constexpr unsigned kStatusTimeout = 1u;

// Tile width policy of the tensor-core grouped GEMM: N tile width (64, 128
// or 256) per instance class by n (<= 64, <= 128, <= 256, > 256).
struct GroupedPolicy {
  int bn[4];
};

struct Handle {
  int device = 0;
  int sm_count = kNumSMs;
  cudaStream_t stream = nullptr;
  // Side stream and events for work that forks from and joins back into
  // `stream` within one call (created with the handle).
  cudaStream_t side_stream = nullptr;
  cudaEvent_t fork_event = nullptr, join_event = nullptr;
  int pointer_mode = CORAL_POINTER_HOST;
  int gemm_mode = CORAL_GEMM_NATIVE;
  uint64_t wait_limit = kDefaultWaitLimit;
  // K slabs (64 deep) per tensor-core accumulation chunk of the split GEMMs.
  int split_chunk_kb = 16;
  // Explicit split-GEMM configuration (0 = not set): N tile width, split-K,
  // and tile height (128: one CTA per tile; 256: a CTA pair per 256 x 256 tile).
  int cfg_bn = 0, cfg_splits = 0, cfg_bm = 0;
  // M-tiles per raster group of the CTA-pair split GEMM (0: the default, 8).
  int pair_group = 0;
  // Complex GEMM mapping onto real tensor-core products (CORAL_COMPLEX_4M or 3M).
  int complex_mapping = CORAL_COMPLEX_4M;
  // SYMV / HEMV / TRMV: the TMA-fed single pass (when the matrix allows)
  // instead of the register-streaming strips.
  bool tri_tma = false;
  // Tile widths of the tensor-core grouped GEMM per instance class.
  GroupedPolicy grouped_policy{{64, 128, 128, 256}};
  // Learned configuration selector (see selector.cu), or null.
  struct Selector* selector = nullptr;
  int bad_arg = 0;
  std::string cuda_error;

  // Growable device scratch (partials of multi-block reductions, split
  // operands of emulated GEMMs).  Never shrinks until coral_destroy.
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // Small zero-initialised device area: reduction arrival counters, the
  // status word and scalar results.  Laid out as `DeviceWords`.
  struct DeviceWords* words = nullptr;
  void* host_pinned = nullptr;  // 64 B pinned staging for scalar results
  // Zeroed pool of per-tile arrival counters for single-launch multi-block
  // combines; every kernel returns the counters it used to zero.
  unsigned* counters = nullptr;
  // TRSV epoch-tagged solution slots ((epoch << 32) | float bits), zeroed when
  // (re)allocated so stale memory never carries a live epoch.
  unsigned long long* trsv_slots = nullptr;
  size_t trsv_slots_len = 0;
  // Optional event timing of the dominant kernel of each call.
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timing_events;
  size_t timing_used = 0;
};

// Brackets one dominant-kernel launch with events when the handle's timing is
// on: call timed_begin() before the launch and timed_end() after it.
void timed_begin(Handle* h);
void timed_end(Handle* h);

constexpr size_t kCounterPool = 1u << 16;
// Counters [0, kTrsvFlagBase) are zero-reset arrival counters; the rest are
// TRSV ready flags.
constexpr size_t kTrsvFlagBase = 1u << 15;

// Fixed device-side bookkeeping; counters are returned to zero by the last
// block of the reduction that used them, so the area stays reusable.
struct DeviceWords {
  unsigned status;                 // kStatus* bits
  unsigned pad0;
  unsigned counters[30];           // arrival counters of single-launch reductions
  double dresult[4];               // scalar results (device pointer mode staging)
  unsigned long long uresult[4];
  unsigned trsv_ticket;   // TRSV: tickets handed out in the current call
  unsigned trsv_done;     // TRSV: CTAs finished in the current call
  unsigned trsv_epoch;    // TRSV: epoch of the last completed call
  unsigned pad1;
  double stage[8];        // scalar arguments of the rotation constructors
  unsigned char reserved[1024 - 4 * 32 - 64 - 16 - 64];
};
static_assert(sizeof(DeviceWords) == 1024, "DeviceWords layout");

enum CounterSlot { kCtrDot = 0, kCtrNrm2 = 1, kCtrIamax = 2, kCtrGemv = 3, kCtrTrsv = 4,
                   kCtrSymv = 5, kCtrMisc = 6 };

// Ensure the handle owns at least `bytes` of scratch; returns nullptr on failure.
void* scratch(Handle* h, size_t bytes);

// Records the CUDA error text in the handle and maps it to a status.
coral_status_t cuda_status(Handle* h, cudaError_t err);
// GEMM argument check (gemm_simt.cu): 1-based position of the first bad
// argument, -1 for sizes past INT32_MAX, 0 when all are valid.
int gemm_bad_arg(int op_a, int op_b, size_t m, size_t n, size_t k, const void* a, size_t lda,
                 const void* b, size_t ldb, const void* c, size_t ldc, bool complex_ops);
// Every kernel launch site reports through launch_status(), which also
// counts the launch (coral_kernel_launches()).
void count_launch();
inline coral_status_t launch_status(Handle* h) {
  count_launch();
  return cuda_status(h, cudaGetLastError());
}

inline coral_status_t bad_arg(Handle* h, int pos) {
  if (h) h->bad_arg = pos;
  return CORAL_ERR_INVALID_ARG;
}

// Grid size for a streaming kernel of `work` independent items with `per_block`
// items per block, capped at `waves` resident waves of the SM count.
inline unsigned stream_grid(size_t work, size_t per_block, int sm_count, int blocks_per_sm) {
  size_t g = (work + per_block - 1) / per_block;
  size_t cap = (size_t)sm_count * blocks_per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Copies a scalar result produced at device address `src` to `dst` per the
// pointer mode (host: waits on the stream).
coral_status_t deliver_result(Handle* h, void* dst, const void* src, size_t bytes);

// Split-BF16 GEMM configuration (tile width BN, split-K factor, and whether a
// CTA pair computes a 256 x 256 tile).
struct SplitConfig {
  int bn;
  int splits;
  int pair = 0;
};
// Shape of a split-BF16 GEMM call as the configuration policy sees it:
// op(A) rows mr, B-rows nr (2n for complex), depth kd (2k for complex).
struct SplitShape {
  int mr, nr, kd;
  int products;  // 3 or 6
  int op_a, op_b;
  int complex_;
  int batch;
};
SplitConfig choose_split_config(Handle* h, const SplitShape& sh);
// Asks the handle's selector for a configuration; false if it has none.
bool select_split_config(Handle* h, const SplitShape& sh, SplitConfig* out);
// Features of (shape, configuration) for the selector network.
constexpr int kSelectorFeatures = 13;
void selector_features(const SplitShape& sh, int bm, int bn, int splits, float* f);
// Split-GEMM configurations the selector and the exhaustive tile autotuner
// consider, in their documented order: tiles (256 x 256 CTA pair, 128 x 256,
// 128 x 128) x split-K (1, 2, 4, 8, 16); the 3-piece mode has no 128 x 256
// tile.  Writes up to 15 configurations; returns the count.
int split_candidates(int products, SplitConfig* out);

// Tensor-core grouped GEMM (grouped_tc.cu): bf16 inputs, or fp32 inputs as
// split-BF16x3; descriptors in device memory.
coral_status_t enqueue_grouped_tc(Handle* h, bool bf16_inputs, size_t count,
                                  const coral_sgemm_problem_t* probs);

// Per-thread default handle for the coral_host_* entry points.
Handle* thread_handle();

}  // namespace coral

#define CORAL_CUDA(h, call)                                   \
  do {                                                        \
    cudaError_t e__ = (call);                                 \
    if (e__ != cudaSuccess) return ::coral::cuda_status((h), e__); \
  } while (0)

#define CORAL_HANDLE(hh) \
  ::coral::Handle* H = reinterpret_cast<::coral::Handle*>(hh); \
  if (!H) return CORAL_ERR_INVALID_ARG; \
  H->bad_arg = 0
