// Exhaustive autotuning of the split-BF16 SGEMM configuration for one shape
// (no reference counterpart).  Every candidate (tile shape x split-K) runs
// once untimed and `reps` times between CUDA events on the handle's stream;
// all candidates are enqueued before the single synchronisation, so the
// measurement does not include host round trips.
#include "common.cuh"

#include <vector>

using namespace coral;

extern "C" coral_status_t coral_autotune_sgemm(coral_handle_t hh, int products, int op_a, int op_b,
                                               size_t m, size_t n, size_t k, const float* a,
                                               size_t lda, const float* b, size_t ldb, float* c,
                                               size_t ldc, int reps, float* ms_out, int* best) {
  CORAL_HANDLE(hh);
  if (products != 3 && products != 6) return bad_arg(H, 1);
  if (reps < 1) return bad_arg(H, 14);
  if (!ms_out) return bad_arg(H, 15);
  if (!best) return bad_arg(H, 16);
  static const int kBn[2] = {256, 128};
  static const int kSp[5] = {1, 2, 4, 8, 16};
  struct Cand {
    int bn, sp;
  };
  std::vector<Cand> cands;
  for (int bi = 0; bi < 2; ++bi) {
    if (products == 6 && kBn[bi] == 256) continue;
    for (int si = 0; si < 5; ++si) cands.push_back({kBn[bi], kSp[si]});
  }
  const int saved_mode = H->gemm_mode, saved_bn = H->cfg_bn, saved_sp = H->cfg_splits;
  H->gemm_mode = products == 6 ? CORAL_GEMM_SPLIT_BF16X6 : CORAL_GEMM_SPLIT_BF16X3;
  std::vector<cudaEvent_t> ev(2 * cands.size(), nullptr);
  coral_status_t st = CORAL_OK;
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) st = CORAL_ERR_CUDA;
  const int saved_bm = H->cfg_bm;
  H->cfg_bm = 128;
  for (size_t i = 0; i < cands.size() && st == CORAL_OK; ++i) {
    H->cfg_bn = cands[i].bn;
    H->cfg_splits = cands[i].sp;
    st = coral_sgemm(hh, op_a, op_b, m, n, k, 1.0f, a, lda, b, ldb, 0.0f, c, ldc);
    if (st != CORAL_OK) break;
    cudaEventRecord(ev[2 * i], H->stream);
    for (int r = 0; r < reps && st == CORAL_OK; ++r)
      st = coral_sgemm(hh, op_a, op_b, m, n, k, 1.0f, a, lda, b, ldb, 0.0f, c, ldc);
    cudaEventRecord(ev[2 * i + 1], H->stream);
  }
  if (st == CORAL_OK && cudaStreamSynchronize(H->stream) != cudaSuccess) st = CORAL_ERR_CUDA;
  if (st == CORAL_OK) {
    int bi = 0;
    for (size_t i = 0; i < cands.size(); ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
      ms_out[i] = ms / (float)reps;
      if (ms_out[i] < ms_out[bi]) bi = (int)i;
    }
    *best = bi;
  }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  H->gemm_mode = saved_mode;
  H->cfg_bn = saved_bn;
  H->cfg_splits = saved_sp;
  H->cfg_bm = saved_bm;
  return st;
}

// Exhaustive tuning over the tile shapes as well: the configurations of
// split_candidates() (CTA-pair 256 x 256, 128 x 256 and 128 x 128 tiles, each
// with split-K 1..16), timed like coral_autotune_sgemm.
extern "C" coral_status_t coral_autotune_sgemm_tiles(coral_handle_t hh, int products, int op_a, int op_b,
                                                     size_t m, size_t n, size_t k, const float* a,
                                                     size_t lda, const float* b, size_t ldb, float* c,
                                                     size_t ldc, int reps, float* ms_out, int capacity,
                                                     int* count, int* best) {
  CORAL_HANDLE(hh);
  if (products != 3 && products != 6) return bad_arg(H, 1);
  if (reps < 1) return bad_arg(H, 14);
  if (!ms_out) return bad_arg(H, 15);
  if (!count) return bad_arg(H, 17);
  if (!best) return bad_arg(H, 18);
  SplitConfig cands[15];
  const int nc = split_candidates(products, cands);
  if (capacity < nc) return bad_arg(H, 16);
  const int saved_mode = H->gemm_mode, saved_bn = H->cfg_bn, saved_sp = H->cfg_splits, saved_bm = H->cfg_bm;
  H->gemm_mode = products == 6 ? CORAL_GEMM_SPLIT_BF16X6 : CORAL_GEMM_SPLIT_BF16X3;
  std::vector<cudaEvent_t> ev(2 * nc, nullptr);
  coral_status_t st = CORAL_OK;
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) st = CORAL_ERR_CUDA;
  for (int i = 0; i < nc && st == CORAL_OK; ++i) {
    H->cfg_bm = cands[i].pair ? 256 : 128;
    H->cfg_bn = cands[i].bn;
    H->cfg_splits = cands[i].splits;
    st = coral_sgemm(hh, op_a, op_b, m, n, k, 1.0f, a, lda, b, ldb, 0.0f, c, ldc);
    if (st != CORAL_OK) break;
    cudaEventRecord(ev[2 * i], H->stream);
    for (int r = 0; r < reps && st == CORAL_OK; ++r)
      st = coral_sgemm(hh, op_a, op_b, m, n, k, 1.0f, a, lda, b, ldb, 0.0f, c, ldc);
    cudaEventRecord(ev[2 * i + 1], H->stream);
  }
  if (st == CORAL_OK && cudaStreamSynchronize(H->stream) != cudaSuccess) st = CORAL_ERR_CUDA;
  if (st == CORAL_OK) {
    int bi = 0;
    for (int i = 0; i < nc; ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
      ms_out[i] = ms / (float)reps;
      if (ms_out[i] < ms_out[bi]) bi = i;
    }
    *best = bi;
    *count = nc;
  }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  H->gemm_mode = saved_mode;
  H->cfg_bn = saved_bn;
  H->cfg_splits = saved_sp;
  H->cfg_bm = saved_bm;
  return st;
}

// Exhaustive tuning of the tensor-core grouped GEMM's tile-width policy on one
// batch: every assignment of N tile widths to the four instance classes
// (n <= 64: {64, 128}; n <= 128: {64, 128}; n <= 256 and n > 256:
// {64, 128, 256}) -- 36 candidates, class 0 varying slowest -- runs once
// untimed and `reps` times between CUDA events.  Installs the fastest policy
// on the handle and returns it in `tile_n`.  The instances' C is overwritten.
extern "C" coral_status_t coral_autotune_sgemm_grouped(coral_handle_t hh, int input_type, size_t count,
                                                       const coral_sgemm_problem_t* problems, int reps,
                                                       float* ms_out, int* best, int tile_n[4]) {
  CORAL_HANDLE(hh);
  if (input_type != CORAL_INPUT_F32 && input_type != CORAL_INPUT_BF16) return bad_arg(H, 1);
  if (!problems) return bad_arg(H, 3);
  if (reps < 1) return bad_arg(H, 4);
  if (!ms_out) return bad_arg(H, 5);
  if (!best) return bad_arg(H, 6);
  if (!tile_n) return bad_arg(H, 7);
  static const int kC01[2] = {64, 128};
  static const int kC23[3] = {64, 128, 256};
  std::vector<GroupedPolicy> cands;
  for (int a : kC01)
    for (int b : kC01)
      for (int c : kC23)
        for (int d : kC23) cands.push_back(GroupedPolicy{{a, b, c, d}});
  const GroupedPolicy saved = H->grouped_policy;
  const int saved_mode = H->gemm_mode;
  if (input_type == CORAL_INPUT_F32) H->gemm_mode = CORAL_GEMM_SPLIT_BF16X3;
  std::vector<cudaEvent_t> ev(2 * cands.size(), nullptr);
  coral_status_t st = CORAL_OK;
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) st = CORAL_ERR_CUDA;
  for (size_t i = 0; i < cands.size() && st == CORAL_OK; ++i) {
    H->grouped_policy = cands[i];
    st = coral_sgemm_grouped(hh, input_type, count, problems);
    if (st != CORAL_OK) break;
    cudaEventRecord(ev[2 * i], H->stream);
    for (int r = 0; r < reps && st == CORAL_OK; ++r) st = coral_sgemm_grouped(hh, input_type, count, problems);
    cudaEventRecord(ev[2 * i + 1], H->stream);
  }
  if (st == CORAL_OK && cudaStreamSynchronize(H->stream) != cudaSuccess) st = CORAL_ERR_CUDA;
  H->gemm_mode = saved_mode;
  H->grouped_policy = saved;
  if (st == CORAL_OK) {
    int bi = 0;
    for (size_t i = 0; i < cands.size(); ++i) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
      ms_out[i] = ms / (float)reps;
      if (ms_out[i] < ms_out[bi]) bi = (int)i;
    }
    *best = bi;
    H->grouped_policy = cands[bi];
    for (int c = 0; c < 4; ++c) tile_n[c] = cands[bi].bn[c];
  }
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  return st;
}
