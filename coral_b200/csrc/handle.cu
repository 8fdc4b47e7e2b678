// Handle lifecycle, status reporting, scratch management and the host-slice
// drop-in wrappers of the C ABI.
#include "common.cuh"

#include <atomic>
#include <cstdio>
#include <mutex>

namespace coral {

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

coral_status_t cuda_status(Handle* h, cudaError_t err) {
  if (err == cudaSuccess) return CORAL_OK;
  if (h) h->cuda_error = cudaGetErrorString(err);
  if (err == cudaErrorMemoryAllocation) return CORAL_ERR_ALLOC;
  if (err == cudaErrorNoDevice || err == cudaErrorInsufficientDriver) return CORAL_ERR_NO_DEVICE;
  return CORAL_ERR_CUDA;
}

void* scratch(Handle* h, size_t bytes) {
  if (bytes <= h->scratch_bytes) return h->scratch;
  // Round up to 64 MiB granules past the first 16 MiB to avoid re-allocation churn.
  size_t want = bytes < (16u << 20) ? (16u << 20) : ((bytes + (64u << 20) - 1) & ~size_t((64u << 20) - 1));
  if (h->scratch) {
    // The old buffer may still be read by queued kernels of this stream.
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return nullptr;
    cudaFree(h->scratch);
    h->scratch = nullptr;
    h->scratch_bytes = 0;
  }
  void* p = nullptr;
  if (cudaMalloc(&p, want) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  h->scratch = p;
  h->scratch_bytes = want;
  return p;
}

coral_status_t deliver_result(Handle* h, void* dst, const void* src, size_t bytes) {
  if (h->pointer_mode == CORAL_POINTER_DEVICE) {
    CORAL_CUDA(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, h->stream));
    return CORAL_OK;
  }
  CORAL_CUDA(h, cudaMemcpyAsync(h->host_pinned, src, bytes, cudaMemcpyDeviceToHost, h->stream));
  CORAL_CUDA(h, cudaStreamSynchronize(h->stream));
  std::memcpy(dst, h->host_pinned, bytes);
  return CORAL_OK;
}

static coral_status_t create_handle(Handle** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { cudaGetLastError(); return CORAL_ERR_NO_DEVICE; }
  int major = 0, sms = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (major != 10) return CORAL_ERR_NO_DEVICE;  // kernels are built for sm_100a only
  Handle* h = new Handle();
  h->device = dev;
  h->sm_count = sms > 0 ? sms : kNumSMs;
  if (cudaMalloc(&h->words, sizeof(DeviceWords)) != cudaSuccess ||
      cudaMemset(h->words, 0, sizeof(DeviceWords)) != cudaSuccess ||
      cudaMalloc(&h->counters, kCounterPool * sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(h->counters, 0, kCounterPool * sizeof(unsigned)) != cudaSuccess ||
      cudaMallocHost(&h->host_pinned, 64) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->fork_event, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->join_event, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (h->words) cudaFree(h->words);
    if (h->counters) cudaFree(h->counters);
    delete h;
    return CORAL_ERR_ALLOC;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) { delete h; return CORAL_ERR_CUDA; }
  *out = h;
  return CORAL_OK;
}

void timed_begin(Handle* h) {
  if (!h->timing) return;
  if (h->timing_used == h->timing_events.size()) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    h->timing_events.emplace_back(a, b);
  }
  cudaEventRecord(h->timing_events[h->timing_used].first, h->stream);
}

void timed_end(Handle* h) {
  if (!h->timing || h->timing_used == h->timing_events.size()) return;
  cudaEventRecord(h->timing_events[h->timing_used].second, h->stream);
  ++h->timing_used;
}

extern "C" coral_status_t coral_set_selector(coral_handle_t, coral_mlp_t);

static void destroy_handle(Handle* h) {
  if (!h) return;
  cudaStreamSynchronize(h->stream);
  if (h->selector) coral_set_selector(reinterpret_cast<coral_handle_t>(h), nullptr);
  for (auto& e : h->timing_events) {
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  if (h->scratch) cudaFree(h->scratch);
  if (h->words) cudaFree(h->words);
  if (h->counters) cudaFree(h->counters);
  if (h->trsv_slots) cudaFree(h->trsv_slots);
  if (h->host_pinned) cudaFreeHost(h->host_pinned);
  if (h->side_stream) {
    cudaStreamSynchronize(h->side_stream);
    cudaStreamDestroy(h->side_stream);
  }
  if (h->fork_event) cudaEventDestroy(h->fork_event);
  if (h->join_event) cudaEventDestroy(h->join_event);
  delete h;
}

// Per-thread handle plus growable device staging for the host-slice wrappers,
// and the copy streams / events of the pipelined host SGEMM.
constexpr int kHostPanels = 16;
struct ThreadState {
  Handle* h = nullptr;
  void* dev = nullptr;
  size_t dev_bytes = 0;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t ev_a = nullptr, ev_in[kHostPanels] = {}, ev_c[kHostPanels] = {}, ev_out = nullptr;
  ~ThreadState() {
    if (dev) cudaFree(dev);
    if (s_in) cudaStreamDestroy(s_in);
    if (s_out) cudaStreamDestroy(s_out);
    if (ev_a) cudaEventDestroy(ev_a);
    if (ev_out) cudaEventDestroy(ev_out);
    for (int i = 0; i < kHostPanels; ++i) {
      if (ev_in[i]) cudaEventDestroy(ev_in[i]);
      if (ev_c[i]) cudaEventDestroy(ev_c[i]);
    }
    destroy_handle(h);
  }
};
static thread_local ThreadState tls;

Handle* thread_handle() {
  if (!tls.h) {
    Handle* h = nullptr;
    if (create_handle(&h) != CORAL_OK) return nullptr;
    tls.h = h;
  }
  return tls.h;
}

static void* thread_staging(size_t bytes) {
  if (bytes <= tls.dev_bytes) return tls.dev;
  if (tls.dev) { cudaStreamSynchronize(tls.h->stream); cudaFree(tls.dev); tls.dev = nullptr; tls.dev_bytes = 0; }
  size_t want = (bytes + (1u << 20) - 1) & ~size_t((1u << 20) - 1);
  if (cudaMalloc(&tls.dev, want) != cudaSuccess) { cudaGetLastError(); return nullptr; }
  tls.dev_bytes = want;
  return tls.dev;
}

}  // namespace coral

using namespace coral;

extern "C" {

int coral_abi_version(void) { return CORAL_B200_ABI_VERSION; }

uint64_t coral_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

coral_status_t coral_create(coral_handle_t* handle) {
  if (!handle) return CORAL_ERR_INVALID_ARG;
  Handle* h = nullptr;
  coral_status_t s = create_handle(&h);
  *handle = reinterpret_cast<coral_handle_t>(h);
  return s;
}

coral_status_t coral_destroy(coral_handle_t handle) {
  destroy_handle(reinterpret_cast<Handle*>(handle));
  return CORAL_OK;
}

coral_status_t coral_set_stream(coral_handle_t handle, void* stream) {
  CORAL_HANDLE(handle);
  H->stream = reinterpret_cast<cudaStream_t>(stream);
  return CORAL_OK;
}

coral_status_t coral_get_stream(coral_handle_t handle, void** stream) {
  CORAL_HANDLE(handle);
  if (!stream) return bad_arg(H, 1);
  *stream = H->stream;
  return CORAL_OK;
}

coral_status_t coral_set_pointer_mode(coral_handle_t handle, int mode) {
  CORAL_HANDLE(handle);
  if (mode != CORAL_POINTER_HOST && mode != CORAL_POINTER_DEVICE) return bad_arg(H, 1);
  H->pointer_mode = mode;
  return CORAL_OK;
}

coral_status_t coral_set_gemm_mode(coral_handle_t handle, int mode) {
  CORAL_HANDLE(handle);
  if (mode < CORAL_GEMM_NATIVE || mode > CORAL_GEMM_SPLIT_BF16X6) return bad_arg(H, 1);
  H->gemm_mode = mode;
  return CORAL_OK;
}

coral_status_t coral_get_gemm_mode(coral_handle_t handle, int* mode) {
  CORAL_HANDLE(handle);
  if (!mode) return bad_arg(H, 1);
  *mode = H->gemm_mode;
  return CORAL_OK;
}

coral_status_t coral_set_complex_mapping(coral_handle_t handle, int mapping) {
  CORAL_HANDLE(handle);
  if (mapping != CORAL_COMPLEX_4M && mapping != CORAL_COMPLEX_3M) return bad_arg(H, 1);
  H->complex_mapping = mapping;
  return CORAL_OK;
}

coral_status_t coral_set_strip_form(coral_handle_t handle, int form) {
  CORAL_HANDLE(handle);
  if (form != CORAL_STRIPS_REGISTER && form != CORAL_STRIPS_TMA) return bad_arg(H, 1);
  H->tri_tma = form == CORAL_STRIPS_TMA;
  return CORAL_OK;
}

coral_status_t coral_set_split_chunk(coral_handle_t handle, int slabs) {
  CORAL_HANDLE(handle);
  if (slabs < 1 || slabs > 1 << 20) return bad_arg(H, 1);
  H->split_chunk_kb = slabs;
  return CORAL_OK;
}

coral_status_t coral_set_wait_limit(coral_handle_t handle, uint64_t spins) {
  CORAL_HANDLE(handle);
  H->wait_limit = spins ? spins : kDefaultWaitLimit;
  return CORAL_OK;
}

coral_status_t coral_set_kernel_timing(coral_handle_t handle, int enable) {
  CORAL_HANDLE(handle);
  H->timing = enable != 0;
  H->timing_used = 0;
  return CORAL_OK;
}

coral_status_t coral_get_kernel_timing(coral_handle_t handle, double* total_ms, uint64_t* launches) {
  CORAL_HANDLE(handle);
  if (!total_ms) return bad_arg(H, 1);
  if (!launches) return bad_arg(H, 2);
  CORAL_CUDA(H, cudaStreamSynchronize(H->stream));
  double sum = 0.0;
  for (size_t i = 0; i < H->timing_used; ++i) {
    float ms = 0.f;
    CORAL_CUDA(H, cudaEventElapsedTime(&ms, H->timing_events[i].first, H->timing_events[i].second));
    sum += ms;
  }
  *total_ms = sum;
  *launches = H->timing_used;
  H->timing_used = 0;
  return CORAL_OK;
}

coral_status_t coral_sync(coral_handle_t handle) {
  CORAL_HANDLE(handle);
  CORAL_CUDA(H, cudaStreamSynchronize(H->stream));
  unsigned status = 0;
  CORAL_CUDA(H, cudaMemcpy(&status, &H->words->status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (status) {
    unsigned zero = 0;
    CORAL_CUDA(H, cudaMemcpy(&H->words->status, &zero, sizeof(unsigned), cudaMemcpyHostToDevice));
    if (status & kStatusTimeout) return CORAL_ERR_TIMEOUT;
  }
  return CORAL_OK;
}

int coral_last_bad_arg(coral_handle_t handle) {
  Handle* h = reinterpret_cast<Handle*>(handle);
  return h ? h->bad_arg : 0;
}

const char* coral_last_cuda_error(coral_handle_t handle) {
  Handle* h = reinterpret_cast<Handle*>(handle);
  return h ? h->cuda_error.c_str() : "";
}

const char* coral_status_string(coral_status_t s) {
  switch (s) {
    case CORAL_OK: return "CORAL_OK";
    case CORAL_ERR_INVALID_ARG: return "CORAL_ERR_INVALID_ARG";
    case CORAL_ERR_CUDA: return "CORAL_ERR_CUDA";
    case CORAL_ERR_TIMEOUT: return "CORAL_ERR_TIMEOUT";
    case CORAL_ERR_ALLOC: return "CORAL_ERR_ALLOC";
    case CORAL_ERR_NOT_SUPPORTED: return "CORAL_ERR_NOT_SUPPORTED";
    case CORAL_ERR_NO_DEVICE: return "CORAL_ERR_NO_DEVICE";
  }
  return "CORAL_ERR_UNKNOWN";
}

// ---- host-slice drop-ins --------------------------------------------------

static size_t vec_len(size_t n, size_t inc) { return n ? (n - 1) * inc + 1 : 0; }
static size_t mat_len(size_t rows, size_t cols, size_t ld) {
  return (rows && cols) ? (cols - 1) * ld + rows : 0;
}
static size_t up256(size_t bytes) { return (bytes + 255) & ~size_t(255); }

#define HOST_PROLOGUE()                              \
  Handle* H = thread_handle();                       \
  if (!H) return CORAL_ERR_NO_DEVICE;                \
  coral_handle_t hh = reinterpret_cast<coral_handle_t>(H)

coral_status_t coral_host_set_gemm_mode(int mode) {
  HOST_PROLOGUE();
  return coral_set_gemm_mode(hh, mode);
}

// Host-resident operands: for a large problem the PCIe transfers, not the
// GEMM, bound the call.  A is copied first; then column panels of op(B) and C
// (16 panels, widths a multiple of 256) stream in on one copy stream, the GEMM
// of panel j runs on the handle's stream as soon as its inputs land, and C
// panel j streams back on a second copy stream -- so host-to-device,
// device-to-host and the compute overlap.  C is not copied in when beta == 0
// (the GEMM does not read it then).  Small problems take one copy each way.
coral_status_t coral_host_sgemm(int op_a, int op_b, size_t m, size_t n, size_t k, float alpha,
                                const float* a, size_t lda, const float* b, size_t ldb,
                                float beta, float* c, size_t ldc) {
  HOST_PROLOGUE();
  bool ta = op_a != CORAL_NO_TRANSPOSE, tb = op_b != CORAL_NO_TRANSPOSE;
  // arguments are checked before any copy touches the caller's buffers
  const int bad = gemm_bad_arg(op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc, false);
  if (bad > 0) return bad_arg(H, bad);
  if (bad < 0) return CORAL_ERR_NOT_SUPPORTED;
  if (m == 0 || n == 0) return CORAL_OK;
  size_t la = mat_len(ta ? k : m, ta ? m : k, lda);
  size_t lb = mat_len(tb ? n : k, tb ? k : n, ldb);
  size_t lc = mat_len(m, n, ldc);
  size_t oa = 0, ob = up256(la * 4), oc = ob + up256(lb * 4);
  char* d = static_cast<char*>(thread_staging(oc + up256(lc * 4) + 256));
  if (!d) return CORAL_ERR_ALLOC;
  float* da = reinterpret_cast<float*>(d + oa);
  float* db = reinterpret_cast<float*>(d + ob);
  float* dc = reinterpret_cast<float*>(d + oc);
  const bool read_c = beta != 0.f;
  const size_t bytes = (la + lb + lc) * 4;
  if (n < 2 * 256 || m == 0 || k == 0 || bytes < (64u << 20)) {
    if (la) CORAL_CUDA(H, cudaMemcpyAsync(da, a, la * 4, cudaMemcpyHostToDevice, H->stream));
    if (lb) CORAL_CUDA(H, cudaMemcpyAsync(db, b, lb * 4, cudaMemcpyHostToDevice, H->stream));
    if (lc) CORAL_CUDA(H, cudaMemcpyAsync(dc, c, lc * 4, cudaMemcpyHostToDevice, H->stream));
    coral_status_t s = coral_sgemm(hh, op_a, op_b, m, n, k, alpha, da, lda, db, ldb, beta, dc, ldc);
    if (s != CORAL_OK) return s;
    if (lc) CORAL_CUDA(H, cudaMemcpyAsync(c, dc, lc * 4, cudaMemcpyDeviceToHost, H->stream));
    return coral_sync(hh);
  }
  if (!tls.s_in) {
    CORAL_CUDA(H, cudaStreamCreateWithFlags(&tls.s_in, cudaStreamNonBlocking));
    CORAL_CUDA(H, cudaStreamCreateWithFlags(&tls.s_out, cudaStreamNonBlocking));
    CORAL_CUDA(H, cudaEventCreateWithFlags(&tls.ev_a, cudaEventDisableTiming));
    CORAL_CUDA(H, cudaEventCreateWithFlags(&tls.ev_out, cudaEventDisableTiming));
    for (int i = 0; i < kHostPanels; ++i) {
      CORAL_CUDA(H, cudaEventCreateWithFlags(&tls.ev_in[i], cudaEventDisableTiming));
      CORAL_CUDA(H, cudaEventCreateWithFlags(&tls.ev_c[i], cudaEventDisableTiming));
    }
  }
  // After the first asynchronous copy every early return first waits for the
  // copy streams, so no transfer still touches the caller's buffers.
  auto drain = [&](coral_status_t st) {
    cudaStreamSynchronize(tls.s_in);
    cudaStreamSynchronize(tls.s_out);
    return st;
  };
#define PIPE_CUDA(call)                                        \
  do {                                                         \
    cudaError_t e__ = (call);                                  \
    if (e__ != cudaSuccess) return drain(cuda_status(H, e__)); \
  } while (0)
  // the staging buffers may still be read by the previous call's stream
  PIPE_CUDA(cudaEventRecord(tls.ev_out, H->stream));
  PIPE_CUDA(cudaStreamWaitEvent(tls.s_in, tls.ev_out, 0));
  PIPE_CUDA(cudaMemcpyAsync(da, a, la * 4, cudaMemcpyHostToDevice, tls.s_in));
  PIPE_CUDA(cudaEventRecord(tls.ev_a, tls.s_in));
  size_t nb = (n + kHostPanels - 1) / kHostPanels;
  nb = (nb + 255) / 256 * 256;
  int panels = 0;
  for (size_t j0 = 0; j0 < n; j0 += nb, ++panels) {
    const size_t nj = n - j0 < nb ? n - j0 : nb;
    // op(B) columns j0 .. j0 + nj: stored columns (N) or stored rows (T)
    if (!tb)
      PIPE_CUDA(cudaMemcpy2DAsync(db + j0 * ldb, ldb * 4, b + j0 * ldb, ldb * 4, k * 4, nj,
                                      cudaMemcpyHostToDevice, tls.s_in));
    else
      PIPE_CUDA(cudaMemcpy2DAsync(db + j0, ldb * 4, b + j0, ldb * 4, nj * 4, k,
                                      cudaMemcpyHostToDevice, tls.s_in));
    if (read_c)
      PIPE_CUDA(cudaMemcpy2DAsync(dc + j0 * ldc, ldc * 4, c + j0 * ldc, ldc * 4, m * 4, nj,
                                      cudaMemcpyHostToDevice, tls.s_in));
    PIPE_CUDA(cudaEventRecord(tls.ev_in[panels], tls.s_in));
  }
  PIPE_CUDA(cudaStreamWaitEvent(H->stream, tls.ev_a, 0));
  int p = 0;
  for (size_t j0 = 0; j0 < n; j0 += nb, ++p) {
    const size_t nj = n - j0 < nb ? n - j0 : nb;
    PIPE_CUDA(cudaStreamWaitEvent(H->stream, tls.ev_in[p], 0));
    coral_status_t s = coral_sgemm(hh, op_a, op_b, m, nj, k, alpha, da, lda,
                                   tb ? db + j0 : db + j0 * ldb, ldb, beta, dc + j0 * ldc, ldc);
    if (s != CORAL_OK) return drain(s);
    PIPE_CUDA(cudaEventRecord(tls.ev_c[p], H->stream));
    PIPE_CUDA(cudaStreamWaitEvent(tls.s_out, tls.ev_c[p], 0));
    PIPE_CUDA(cudaMemcpy2DAsync(c + j0 * ldc, ldc * 4, dc + j0 * ldc, ldc * 4, m * 4, nj,
                                    cudaMemcpyDeviceToHost, tls.s_out));
  }
  PIPE_CUDA(cudaEventRecord(tls.ev_out, tls.s_out));
  PIPE_CUDA(cudaStreamWaitEvent(H->stream, tls.ev_out, 0));
#undef PIPE_CUDA
  return coral_sync(hh);
}

coral_status_t coral_host_sgemv(int trans, size_t n_rows, size_t n_cols, float alpha,
                                const float* matrix, size_t lda, const float* x, size_t incx,
                                float beta, float* y, size_t incy) {
  HOST_PROLOGUE();
  bool t = trans != CORAL_NO_TRANSPOSE;
  size_t lm = mat_len(n_rows, n_cols, lda);
  size_t lx = vec_len(t ? n_rows : n_cols, incx);
  size_t ly = vec_len(t ? n_cols : n_rows, incy);
  size_t ox = up256(lm * 4), oy = ox + up256(lx * 4);
  char* d = static_cast<char*>(thread_staging(oy + up256(ly * 4) + 256));
  if (!d) return CORAL_ERR_ALLOC;
  float* dm = reinterpret_cast<float*>(d);
  float* dx = reinterpret_cast<float*>(d + ox);
  float* dy = reinterpret_cast<float*>(d + oy);
  if (lm) CORAL_CUDA(H, cudaMemcpyAsync(dm, matrix, lm * 4, cudaMemcpyHostToDevice, H->stream));
  if (lx) CORAL_CUDA(H, cudaMemcpyAsync(dx, x, lx * 4, cudaMemcpyHostToDevice, H->stream));
  if (ly) CORAL_CUDA(H, cudaMemcpyAsync(dy, y, ly * 4, cudaMemcpyHostToDevice, H->stream));
  coral_status_t s = coral_sgemv(hh, trans, n_rows, n_cols, alpha, dm, lda, dx, incx, beta, dy, incy);
  if (s != CORAL_OK) return s;
  if (ly) CORAL_CUDA(H, cudaMemcpyAsync(y, dy, ly * 4, cudaMemcpyDeviceToHost, H->stream));
  return coral_sync(hh);
}

coral_status_t coral_host_sdot(size_t n, const float* x, size_t incx, const float* y,
                               size_t incy, float* result) {
  HOST_PROLOGUE();
  if (!result) return CORAL_ERR_INVALID_ARG;
  size_t lx = vec_len(n, incx), ly = vec_len(n, incy);
  size_t oy = up256(lx * 4);
  char* d = static_cast<char*>(thread_staging(oy + up256(ly * 4) + 256));
  if (!d) return CORAL_ERR_ALLOC;
  float* dx = reinterpret_cast<float*>(d);
  float* dy = reinterpret_cast<float*>(d + oy);
  if (lx) CORAL_CUDA(H, cudaMemcpyAsync(dx, x, lx * 4, cudaMemcpyHostToDevice, H->stream));
  if (ly) CORAL_CUDA(H, cudaMemcpyAsync(dy, y, ly * 4, cudaMemcpyHostToDevice, H->stream));
  int mode = H->pointer_mode;
  H->pointer_mode = CORAL_POINTER_HOST;
  coral_status_t s = coral_sdot(hh, n, dx, incx, dy, incy, result);
  H->pointer_mode = mode;
  if (s != CORAL_OK) return s;
  return coral_sync(hh);
}

coral_status_t coral_host_saxpy(size_t n, float alpha, const float* x, size_t incx, float* y,
                                size_t incy) {
  HOST_PROLOGUE();
  size_t lx = vec_len(n, incx), ly = vec_len(n, incy);
  size_t oy = up256(lx * 4);
  char* d = static_cast<char*>(thread_staging(oy + up256(ly * 4) + 256));
  if (!d) return CORAL_ERR_ALLOC;
  float* dx = reinterpret_cast<float*>(d);
  float* dy = reinterpret_cast<float*>(d + oy);
  if (lx) CORAL_CUDA(H, cudaMemcpyAsync(dx, x, lx * 4, cudaMemcpyHostToDevice, H->stream));
  if (ly) CORAL_CUDA(H, cudaMemcpyAsync(dy, y, ly * 4, cudaMemcpyHostToDevice, H->stream));
  coral_status_t s = coral_saxpy(hh, n, alpha, dx, incx, dy, incy);
  if (s != CORAL_OK) return s;
  if (ly) CORAL_CUDA(H, cudaMemcpyAsync(y, dy, ly * 4, cudaMemcpyDeviceToHost, H->stream));
  return coral_sync(hh);
}

coral_status_t coral_host_isamax(size_t n, const float* x, size_t incx, size_t* index) {
  HOST_PROLOGUE();
  if (!index) return CORAL_ERR_INVALID_ARG;
  size_t lx = vec_len(n, incx);
  float* dx = static_cast<float*>(thread_staging(up256(lx * 4) + 256));
  if (!dx) return CORAL_ERR_ALLOC;
  if (lx) CORAL_CUDA(H, cudaMemcpyAsync(dx, x, lx * 4, cudaMemcpyHostToDevice, H->stream));
  int mode = H->pointer_mode;
  H->pointer_mode = CORAL_POINTER_HOST;
  coral_status_t s = coral_isamax(hh, n, dx, incx, index);
  H->pointer_mode = mode;
  if (s != CORAL_OK) return s;
  return coral_sync(hh);
}

coral_status_t coral_host_strsv(int uplo, int trans, int diag, size_t n, const float* matrix,
                                size_t lda, float* x, size_t incx) {
  HOST_PROLOGUE();
  size_t lm = mat_len(n, n, lda), lx = vec_len(n, incx);
  size_t ox = up256(lm * 4);
  char* d = static_cast<char*>(thread_staging(ox + up256(lx * 4) + 256));
  if (!d) return CORAL_ERR_ALLOC;
  float* dm = reinterpret_cast<float*>(d);
  float* dx = reinterpret_cast<float*>(d + ox);
  if (lm) CORAL_CUDA(H, cudaMemcpyAsync(dm, matrix, lm * 4, cudaMemcpyHostToDevice, H->stream));
  if (lx) CORAL_CUDA(H, cudaMemcpyAsync(dx, x, lx * 4, cudaMemcpyHostToDevice, H->stream));
  coral_status_t s = coral_strsv(hh, uplo, trans, diag, n, dm, lda, dx, incx);
  if (s != CORAL_OK) return s;
  if (lx) CORAL_CUDA(H, cudaMemcpyAsync(x, dx, lx * 4, cudaMemcpyDeviceToHost, H->stream));
  return coral_sync(hh);
}


}  // extern "C"

// ---- host-slice drop-ins built on one staging helper ---------------------
// Each operand is a host span: copied to the thread's device staging before
// the call when `in`, back after it when `out`.  Arguments are checked first
// (the same positions the device entry points report), so no copy ever reads
// past what the reference's own length checks would allow.
namespace {
struct Span {
  const void* host;
  size_t bytes;
  bool in, out;
  void* dev;
};

template <typename F>
coral_status_t host_stage_call(Span* spans, int count, F&& call) {
  HOST_PROLOGUE();
  size_t total = 0;
  for (int i = 0; i < count; ++i) total += up256(spans[i].bytes);
  char* d = static_cast<char*>(thread_staging(total + 256));
  if (!d) return CORAL_ERR_ALLOC;
  for (int i = 0; i < count; ++i) {
    spans[i].dev = d;
    d += up256(spans[i].bytes);
    if (spans[i].in && spans[i].bytes)
      CORAL_CUDA(H, cudaMemcpyAsync(spans[i].dev, spans[i].host, spans[i].bytes,
                                    cudaMemcpyHostToDevice, H->stream));
  }
  const int mode = H->pointer_mode;
  H->pointer_mode = CORAL_POINTER_HOST;  // scalar results land in host memory
  coral_status_t s = call(hh);
  H->pointer_mode = mode;
  if (s != CORAL_OK) {
    cudaStreamSynchronize(H->stream);  // no copy in flight may outlive the call
    return s;
  }
  for (int i = 0; i < count; ++i)
    if (spans[i].out && spans[i].bytes)
      CORAL_CUDA(H, cudaMemcpyAsync(const_cast<void*>(spans[i].host), spans[i].dev, spans[i].bytes,
                                    cudaMemcpyDeviceToHost, H->stream));
  return coral_sync(hh);
}

bool bad_uplo(int u) { return u != CORAL_UPPER && u != CORAL_LOWER; }
bool bad_trans(int t) { return t < CORAL_NO_TRANSPOSE || t > CORAL_CONJ_TRANSPOSE; }
bool bad_diag(int d) { return d != CORAL_UNIT && d != CORAL_NON_UNIT; }

// GEMM operands of any element size (es bytes); arguments already checked.
template <typename T, typename F>
coral_status_t host_gemm(int op_a, int op_b, size_t m, size_t n, size_t k, const T* a, size_t lda,
                         const T* b, size_t ldb, bool read_c, T* c, size_t ldc, bool complex_ops,
                         F&& call) {
  const int bad = gemm_bad_arg(op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc, complex_ops);
  if (bad > 0) { Handle* H = thread_handle(); if (H) H->bad_arg = bad; return CORAL_ERR_INVALID_ARG; }
  if (bad < 0) return CORAL_ERR_NOT_SUPPORTED;
  if (m == 0 || n == 0) return CORAL_OK;
  const bool ta = op_a != CORAL_NO_TRANSPOSE, tb = op_b != CORAL_NO_TRANSPOSE;
  const bool use_ab = k != 0;
  Span sp[3] = {{a, use_ab ? mat_len(ta ? k : m, ta ? m : k, lda) * sizeof(T) : 0, true, false, nullptr},
                {b, use_ab ? mat_len(tb ? n : k, tb ? k : n, ldb) * sizeof(T) : 0, true, false, nullptr},
                // C is uploaded when read, and when ldc > m: the rows between its
                // columns must come back to the caller unchanged
                {c, mat_len(m, n, ldc) * sizeof(T), read_c || ldc > m, true, nullptr}};
  return host_stage_call(sp, 3, [&](coral_handle_t hh) {
    return call(hh, static_cast<const T*>(sp[0].dev), static_cast<const T*>(sp[1].dev),
                static_cast<T*>(sp[2].dev));
  });
}
}  // namespace

extern "C" {

#define HOST_ARG(cond, pos)                                                  \
  do {                                                                      \
    if (cond) {                                                             \
      Handle* H__ = thread_handle();                                        \
      if (H__) H__->bad_arg = (pos);                                        \
      return CORAL_ERR_INVALID_ARG;                                         \
    }                                                                       \
  } while (0)

coral_status_t coral_host_ssymv(int uplo, size_t n, float alpha, const float* matrix, size_t lda,
                                const float* x, size_t incx, float beta, float* y, size_t incy) {
  HOST_ARG(bad_uplo(uplo), 1);
  if (n == 0) return CORAL_OK;
  HOST_ARG(!matrix, 4); HOST_ARG(lda < n, 5); HOST_ARG(!x, 6); HOST_ARG(incx == 0, 7);
  HOST_ARG(!y, 9); HOST_ARG(incy == 0, 10);
  Span sp[3] = {{matrix, mat_len(n, n, lda) * 4, true, false, nullptr},
                {x, vec_len(n, incx) * 4, true, false, nullptr},
                {y, vec_len(n, incy) * 4, true, true, nullptr}};
  return host_stage_call(sp, 3, [&](coral_handle_t hh) {
    return coral_ssymv(hh, uplo, n, alpha, static_cast<const float*>(sp[0].dev), lda,
                       static_cast<const float*>(sp[1].dev), incx, beta, static_cast<float*>(sp[2].dev),
                       incy);
  });
}

coral_status_t coral_host_chemv(int uplo, size_t n, const float alpha[2], const float* matrix,
                                size_t lda, const float* x, size_t incx, const float beta[2],
                                float* y, size_t incy) {
  HOST_ARG(bad_uplo(uplo), 1);
  HOST_ARG(!alpha, 3); HOST_ARG(!beta, 8);
  if (n == 0) return CORAL_OK;
  HOST_ARG(!matrix, 4); HOST_ARG(lda < n, 5); HOST_ARG(!x, 6); HOST_ARG(incx == 0, 7);
  HOST_ARG(!y, 9); HOST_ARG(incy == 0, 10);
  Span sp[3] = {{matrix, mat_len(n, n, lda) * 8, true, false, nullptr},
                {x, vec_len(n, incx) * 8, true, false, nullptr},
                {y, vec_len(n, incy) * 8, true, true, nullptr}};
  return host_stage_call(sp, 3, [&](coral_handle_t hh) {
    return coral_chemv(hh, uplo, n, alpha, static_cast<const float*>(sp[0].dev), lda,
                       static_cast<const float*>(sp[1].dev), incx, beta, static_cast<float*>(sp[2].dev),
                       incy);
  });
}

coral_status_t coral_host_strmv(int uplo, int trans, int diag, size_t n, const float* matrix,
                                size_t lda, float* x, size_t incx) {
  HOST_ARG(bad_uplo(uplo), 1); HOST_ARG(bad_trans(trans), 2); HOST_ARG(bad_diag(diag), 3);
  if (n == 0) return CORAL_OK;
  HOST_ARG(!matrix, 5); HOST_ARG(lda < n, 6); HOST_ARG(!x, 7); HOST_ARG(incx == 0, 8);
  Span sp[2] = {{matrix, mat_len(n, n, lda) * 4, true, false, nullptr},
                {x, vec_len(n, incx) * 4, true, true, nullptr}};
  return host_stage_call(sp, 2, [&](coral_handle_t hh) {
    return coral_strmv(hh, uplo, trans, diag, n, static_cast<const float*>(sp[0].dev), lda,
                       static_cast<float*>(sp[1].dev), incx);
  });
}

coral_status_t coral_host_sger(size_t n_rows, size_t n_cols, float alpha, const float* x,
                               size_t incx, const float* y, size_t incy, float* matrix, size_t lda) {
  if (n_rows == 0 || n_cols == 0) return CORAL_OK;
  HOST_ARG(!x, 4); HOST_ARG(incx == 0, 5); HOST_ARG(!y, 6); HOST_ARG(incy == 0, 7);
  HOST_ARG(!matrix, 8); HOST_ARG(lda < n_rows, 9);
  Span sp[3] = {{x, vec_len(n_rows, incx) * 4, true, false, nullptr},
                {y, vec_len(n_cols, incy) * 4, true, false, nullptr},
                {matrix, mat_len(n_rows, n_cols, lda) * 4, true, true, nullptr}};
  return host_stage_call(sp, 3, [&](coral_handle_t hh) {
    return coral_sger(hh, n_rows, n_cols, alpha, static_cast<const float*>(sp[0].dev), incx,
                      static_cast<const float*>(sp[1].dev), incy, static_cast<float*>(sp[2].dev), lda);
  });
}

coral_status_t coral_host_ssyr(int uplo, size_t n, float alpha, const float* x, size_t incx,
                               float* matrix, size_t lda) {
  HOST_ARG(bad_uplo(uplo), 1);
  if (n == 0) return CORAL_OK;
  HOST_ARG(!x, 4); HOST_ARG(incx == 0, 5); HOST_ARG(!matrix, 6); HOST_ARG(lda < n, 7);
  Span sp[2] = {{x, vec_len(n, incx) * 4, true, false, nullptr},
                {matrix, mat_len(n, n, lda) * 4, true, true, nullptr}};
  return host_stage_call(sp, 2, [&](coral_handle_t hh) {
    return coral_ssyr(hh, uplo, n, alpha, static_cast<const float*>(sp[0].dev), incx,
                      static_cast<float*>(sp[1].dev), lda);
  });
}

coral_status_t coral_host_ssyr2(int uplo, size_t n, float alpha, const float* x, size_t incx,
                                const float* y, size_t incy, float* matrix, size_t lda) {
  HOST_ARG(bad_uplo(uplo), 1);
  if (n == 0) return CORAL_OK;
  HOST_ARG(!x, 4); HOST_ARG(incx == 0, 5); HOST_ARG(!y, 6); HOST_ARG(incy == 0, 7);
  HOST_ARG(!matrix, 8); HOST_ARG(lda < n, 9);
  Span sp[3] = {{x, vec_len(n, incx) * 4, true, false, nullptr},
                {y, vec_len(n, incy) * 4, true, false, nullptr},
                {matrix, mat_len(n, n, lda) * 4, true, true, nullptr}};
  return host_stage_call(sp, 3, [&](coral_handle_t hh) {
    return coral_ssyr2(hh, uplo, n, alpha, static_cast<const float*>(sp[0].dev), incx,
                       static_cast<const float*>(sp[1].dev), incy, static_cast<float*>(sp[2].dev), lda);
  });
}

coral_status_t coral_host_snrm2(size_t n, const float* x, size_t incx, float* result) {
  HOST_ARG(!result, 4);
  if (n == 0 || incx == 0) { *result = 0.0f; return CORAL_OK; }
  HOST_ARG(!x, 2);
  Span sp[1] = {{x, vec_len(n, incx) * 4, true, false, nullptr}};
  return host_stage_call(sp, 1, [&](coral_handle_t hh) {
    return coral_snrm2(hh, n, static_cast<const float*>(sp[0].dev), incx, result);
  });
}

coral_status_t coral_host_scopy(size_t n, const float* x, size_t incx, float* y, size_t incy) {
  if (n == 0) return CORAL_OK;
  HOST_ARG(!x, 2); HOST_ARG(incx == 0, 3); HOST_ARG(!y, 4); HOST_ARG(incy == 0, 5);
  // y is read too: the stride holes between its elements keep the caller's values
  Span sp[2] = {{x, vec_len(n, incx) * 4, true, false, nullptr},
                {y, vec_len(n, incy) * 4, incy > 1, true, nullptr}};
  return host_stage_call(sp, 2, [&](coral_handle_t hh) {
    return coral_scopy(hh, n, static_cast<const float*>(sp[0].dev), incx, static_cast<float*>(sp[1].dev),
                       incy);
  });
}

coral_status_t coral_host_sswap(size_t n, float* x, size_t incx, float* y, size_t incy) {
  if (n == 0) return CORAL_OK;
  HOST_ARG(!x, 2); HOST_ARG(incx == 0, 3); HOST_ARG(!y, 4); HOST_ARG(incy == 0, 5);
  Span sp[2] = {{x, vec_len(n, incx) * 4, true, true, nullptr},
                {y, vec_len(n, incy) * 4, true, true, nullptr}};
  return host_stage_call(sp, 2, [&](coral_handle_t hh) {
    return coral_sswap(hh, n, static_cast<float*>(sp[0].dev), incx, static_cast<float*>(sp[1].dev), incy);
  });
}

coral_status_t coral_host_sscal(size_t n, float alpha, float* x, size_t incx) {
  if (n == 0 || incx == 0) return CORAL_OK;
  HOST_ARG(!x, 3);
  Span sp[1] = {{x, vec_len(n, incx) * 4, true, true, nullptr}};
  return host_stage_call(sp, 1, [&](coral_handle_t hh) {
    return coral_sscal(hh, n, alpha, static_cast<float*>(sp[0].dev), incx);
  });
}

coral_status_t coral_host_dgemm(int op_a, int op_b, size_t m, size_t n, size_t k, double alpha,
                                const double* a, size_t lda, const double* b, size_t ldb,
                                double beta, double* c, size_t ldc) {
  return host_gemm<double>(op_a, op_b, m, n, k, a, lda, b, ldb, beta != 0.0, c, ldc, false,
                           [&](coral_handle_t hh, const double* da, const double* db, double* dc) {
                             return coral_dgemm(hh, op_a, op_b, m, n, k, alpha, da, lda, db, ldb,
                                                beta, dc, ldc);
                           });
}

coral_status_t coral_host_cgemm(int op_a, int op_b, size_t m, size_t n, size_t k,
                                const float alpha[2], const float* a, size_t lda, const float* b,
                                size_t ldb, const float beta[2], float* c, size_t ldc) {
  HOST_ARG(!alpha, 6); HOST_ARG(!beta, 11);
  struct C64 { float re, im; };
  return host_gemm<C64>(op_a, op_b, m, n, k, reinterpret_cast<const C64*>(a), lda,
                        reinterpret_cast<const C64*>(b), ldb, beta[0] != 0.f || beta[1] != 0.f,
                        reinterpret_cast<C64*>(c), ldc, true,
                        [&](coral_handle_t hh, const C64* da, const C64* db, C64* dc) {
                          return coral_cgemm(hh, op_a, op_b, m, n, k, alpha,
                                             reinterpret_cast<const float*>(da), lda,
                                             reinterpret_cast<const float*>(db), ldb, beta,
                                             reinterpret_cast<float*>(dc), ldc);
                        });
}

coral_status_t coral_host_zgemm(int op_a, int op_b, size_t m, size_t n, size_t k,
                                const double alpha[2], const double* a, size_t lda, const double* b,
                                size_t ldb, const double beta[2], double* c, size_t ldc) {
  HOST_ARG(!alpha, 6); HOST_ARG(!beta, 11);
  struct C128 { double re, im; };
  return host_gemm<C128>(op_a, op_b, m, n, k, reinterpret_cast<const C128*>(a), lda,
                         reinterpret_cast<const C128*>(b), ldb, beta[0] != 0.0 || beta[1] != 0.0,
                         reinterpret_cast<C128*>(c), ldc, true,
                         [&](coral_handle_t hh, const C128* da, const C128* db, C128* dc) {
                           return coral_zgemm(hh, op_a, op_b, m, n, k, alpha,
                                              reinterpret_cast<const double*>(da), lda,
                                              reinterpret_cast<const double*>(db), ldb, beta,
                                              reinterpret_cast<double*>(dc), ldc);
                         });
}

#undef HOST_ARG

}  // extern "C"
