// Learned configuration selector: a small MLP (in -> H -> H -> out, ReLU)
// whose forward pass, backward pass, MSE loss and Adam update are the CUDA
// kernels below, plus the glue that lets a handle consult it when it picks a
// split-BF16 GEMM configuration.  No reference counterpart.
//
// Parameters are one packed fp32 array: W1[H][in], b1[H], W2[H][H], b2[H],
// W3[out][H], b3[out].  Row-major activations: X[batch][in].
// Training minimises mean((y - t)^2) over the batch (y, t: [batch][out]).
//
// The selector's network predicts log(milliseconds) of one call from the
// features of (shape, configuration); for a new shape it scores every
// candidate configuration in one batched forward pass and takes the argmin
// (cached per shape, so only the first call for a shape waits for it).
#include "common.cuh"

#include <algorithm>
#include <climits>

#include <cmath>
#include <mutex>
#include <random>
#include <unordered_map>

namespace coral {

struct Mlp {
  Handle* h = nullptr;
  int in = 0, hid = 0, out = 0;
  size_t nparams = 0;
  float* params = nullptr;  // device
  float* grads = nullptr;   // device
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  long long step = 0;
  // activation buffers for the largest batch seen
  float* act = nullptr;
  size_t act_batch = 0;
  float* loss_dev = nullptr;
};

struct Selector {
  Mlp* mlp = nullptr;
  std::mutex mu;
  std::unordered_map<unsigned long long, SplitConfig> cache;
  float* feat_dev = nullptr;
  float* pred_dev = nullptr;
};

namespace {

constexpr int kMT = 32;  // tile of the small GEMM kernel

// C[M][N] = alpha * op(A) op(B) + beta * C, row-major:
//   op(A) = A[M][K] (ta = 0) or A^T with A[K][M] (ta = 1);
//   op(B) = B[K][N] (tb = 0) or B^T with B[N][K] (tb = 1).
// Optional bias[N] added and ReLU applied (forward layers).
__global__ void k_mlp_gemm(int M, int N, int K, const float* __restrict__ A, int ta,
                           const float* __restrict__ B, int tb, float* __restrict__ Cm, float beta,
                           const float* __restrict__ bias, int relu) {
  __shared__ float As[kMT][kMT + 1], Bs[kMT][kMT + 1];
  const int tx = threadIdx.x % kMT, ty = threadIdx.x / kMT;  // 32 x 8 threads
  const int row0 = blockIdx.y * kMT, col0 = blockIdx.x * kMT;
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += kMT) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ty + 8 * q;
      // As[r][tx] = op(A)(row0 + r, k0 + tx)
      const int ar = row0 + r, ak = k0 + tx;
      float av = 0.f;
      if (ar < M && ak < K) av = ta ? A[(size_t)ak * M + ar] : A[(size_t)ar * K + ak];
      As[r][tx] = av;
      // Bs[r][tx] = op(B)(k0 + r, col0 + tx)
      const int bk = k0 + r, bc = col0 + tx;
      float bv = 0.f;
      if (bk < K && bc < N) bv = tb ? B[(size_t)bc * K + bk] : B[(size_t)bk * N + bc];
      Bs[r][tx] = bv;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < kMT; ++kk) {
      const float b = Bs[kk][tx];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fmaf(As[ty + 8 * q][kk], b, acc[q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int r = row0 + ty + 8 * q, c = col0 + tx;
    if (r >= M || c >= N) continue;
    float v = acc[q];
    if (bias) v += bias[c];
    if (relu) v = fmaxf(v, 0.f);
    float* cp = Cm + (size_t)r * N + c;
    *cp = beta == 0.f ? v : fmaf(beta, *cp, v);
  }
}

// out[c] = sum_r X[r][c] (column sums). A block takes 32 columns (lane =
// column, so a warp reads 128 contiguous bytes of a row); warp w sums rows
// w, w + 32, ... with 8 loads in flight, and the 32 warp sums are added in
// warp order. The order is fixed, so the result is deterministic.
constexpr int kColSumWarps = 32;
__global__ void __launch_bounds__(32 * kColSumWarps)
k_col_sum(int R, int Cn, const float* __restrict__ X, float* __restrict__ out) {
  __shared__ float part[kColSumWarps][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = blockIdx.x * 32 + lane;
  float s = 0.f;
  if (c < Cn) {
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    int r = w;
    for (; r + 7 * kColSumWarps < R; r += 8 * kColSumWarps) {
#pragma unroll
      for (int u = 0; u < 8; ++u) acc[u] += X[(size_t)(r + u * kColSumWarps) * Cn + c];
    }
    for (; r < R; r += kColSumWarps) acc[0] += X[(size_t)r * Cn + c];
    s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  }
  part[w][lane] = s;
  __syncthreads();
  if (w != 0 || c >= Cn) return;
  float t = 0.f;
#pragma unroll 8
  for (int k = 0; k < kColSumWarps; ++k) t += part[k][lane];
  out[c] = t;
}

// dY = 2 (y - t) / (batch * out); loss partial sums via a single-block reduction.
__global__ void k_mse_grad(int n, float scale, const float* __restrict__ y, const float* __restrict__ t,
                           float* __restrict__ dy, float* __restrict__ loss) {
  __shared__ float sh[32];
  float s = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float d = y[i] - t[i];
    dy[i] = 2.f * d * scale;
    s += d * d;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *loss = s * scale;
  }
}

// dA *= (A > 0) (ReLU backward, A = post-activation).
__global__ void k_relu_back(size_t n, const float* __restrict__ a, float* __restrict__ d) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (a[i] <= 0.f) d[i] = 0.f;
}

__global__ void k_adam(size_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

coral_status_t gemm(Mlp* n, int M, int N, int K, const float* A, int ta, const float* B, int tb,
                    float* C, float beta, const float* bias, int relu) {
  dim3 grid((N + kMT - 1) / kMT, (M + kMT - 1) / kMT);
  if (grid.y > 65535) return CORAL_ERR_NOT_SUPPORTED;
  k_mlp_gemm<<<grid, 256, 0, n->h->stream>>>(M, N, K, A, ta, B, tb, C, beta, bias, relu);
  return launch_status(n->h);
}

struct Views {
  const float *W1, *b1, *W2, *b2, *W3, *b3;
};
Views views(const Mlp* n, const float* base) {
  Views v;
  v.W1 = base;
  v.b1 = v.W1 + (size_t)n->hid * n->in;
  v.W2 = v.b1 + n->hid;
  v.b2 = v.W2 + (size_t)n->hid * n->hid;
  v.W3 = v.b2 + n->hid;
  v.b3 = v.W3 + (size_t)n->out * n->hid;
  return v;
}

coral_status_t ensure_act(Mlp* n, size_t batch) {
  if (batch <= n->act_batch) return CORAL_OK;
  if (n->act) cudaFree(n->act);
  n->act = nullptr;
  // A1, A2 (post-ReLU), Y, dY, dA2, dA1
  const size_t elems = batch * (4 * (size_t)n->hid + 2 * (size_t)n->out);
  CORAL_CUDA(n->h, cudaMalloc(&n->act, elems * sizeof(float)));
  n->act_batch = batch;
  return CORAL_OK;
}

coral_status_t forward(Mlp* n, const float* x, int batch, float* y_out) {
  coral_status_t s = ensure_act(n, batch);
  if (s != CORAL_OK) return s;
  Views w = views(n, n->params);
  float* A1 = n->act;
  float* A2 = A1 + (size_t)batch * n->hid;
  if ((s = gemm(n, batch, n->hid, n->in, x, 0, w.W1, 1, A1, 0.f, w.b1, 1)) != CORAL_OK) return s;
  if ((s = gemm(n, batch, n->hid, n->hid, A1, 0, w.W2, 1, A2, 0.f, w.b2, 1)) != CORAL_OK) return s;
  return gemm(n, batch, n->out, n->hid, A2, 0, w.W3, 1, y_out, 0.f, w.b3, 0);
}

// Forward + backward; leaves dLoss/dparams in n->grads and the loss in n->loss_dev.
coral_status_t backward(Mlp* n, const float* x, const float* t, int batch) {
  coral_status_t s = ensure_act(n, batch);
  if (s != CORAL_OK) return s;
  float* A1 = n->act;
  float* A2 = A1 + (size_t)batch * n->hid;
  float* Y = A2 + (size_t)batch * n->hid;
  float* dY = Y + (size_t)batch * n->out;
  float* dA2 = dY + (size_t)batch * n->out;
  float* dA1 = dA2 + (size_t)batch * n->hid;
  if ((s = forward(n, x, batch, Y)) != CORAL_OK) return s;
  const int cnt = batch * n->out;
  k_mse_grad<<<1, 1024, 0, n->h->stream>>>(cnt, 1.f / (float)cnt, Y, t, dY, n->loss_dev);
  if ((s = launch_status(n->h)) != CORAL_OK) return s;
  Views w = views(n, n->params);
  Views g = views(n, n->grads);
  float* gW1 = const_cast<float*>(g.W1);
  float* gb1 = const_cast<float*>(g.b1);
  float* gW2 = const_cast<float*>(g.W2);
  float* gb2 = const_cast<float*>(g.b2);
  float* gW3 = const_cast<float*>(g.W3);
  float* gb3 = const_cast<float*>(g.b3);
  // layer 3: dW3 = dY^T A2, db3 = colsum(dY), dA2 = dY W3
  if ((s = gemm(n, n->out, n->hid, batch, dY, 1, A2, 0, gW3, 0.f, nullptr, 0)) != CORAL_OK) return s;
  k_col_sum<<<(n->out + 31) / 32, 32 * kColSumWarps, 0, n->h->stream>>>(batch, n->out, dY, gb3);
  if ((s = launch_status(n->h)) != CORAL_OK) return s;
  if ((s = gemm(n, batch, n->hid, n->out, dY, 0, w.W3, 0, dA2, 0.f, nullptr, 0)) != CORAL_OK) return s;
  const size_t bh = (size_t)batch * n->hid;
  unsigned gr = stream_grid(bh, 256 * 4, n->h->sm_count, 8);
  k_relu_back<<<gr, 256, 0, n->h->stream>>>(bh, A2, dA2);
  if ((s = launch_status(n->h)) != CORAL_OK) return s;
  // layer 2
  if ((s = gemm(n, n->hid, n->hid, batch, dA2, 1, A1, 0, gW2, 0.f, nullptr, 0)) != CORAL_OK) return s;
  k_col_sum<<<(n->hid + 31) / 32, 32 * kColSumWarps, 0, n->h->stream>>>(batch, n->hid, dA2, gb2);
  if ((s = launch_status(n->h)) != CORAL_OK) return s;
  if ((s = gemm(n, batch, n->hid, n->hid, dA2, 0, w.W2, 0, dA1, 0.f, nullptr, 0)) != CORAL_OK) return s;
  k_relu_back<<<gr, 256, 0, n->h->stream>>>(bh, A1, dA1);
  if ((s = launch_status(n->h)) != CORAL_OK) return s;
  // layer 1
  if ((s = gemm(n, n->hid, n->in, batch, dA1, 1, x, 0, gW1, 0.f, nullptr, 0)) != CORAL_OK) return s;
  k_col_sum<<<(n->hid + 31) / 32, 32 * kColSumWarps, 0, n->h->stream>>>(batch, n->hid, dA1, gb1);
  return launch_status(n->h);
}

}  // namespace

// Selector hook used by choose_split_config(): features of (shape, config),
// one forward pass over all candidates, argmin of the predicted log time.
bool select_split_config(Handle* h, const SplitShape& sh, SplitConfig* out) {
  Selector* sel = h->selector;
  if (!sel || !sel->mlp || sel->mlp->in != kSelectorFeatures || sel->mlp->out != 1) return false;
  const int products = sh.products;
  unsigned long long key = 1469598103934665603ull;  // FNV-1a over the shape fields
  for (int v : {sh.mr, sh.nr, sh.kd, sh.products, sh.op_a, sh.op_b, sh.complex_, sh.batch}) {
    key ^= (unsigned long long)(unsigned)v;
    key *= 1099511628211ull;
  }
  std::lock_guard<std::mutex> lock(sel->mu);
  auto it = sel->cache.find(key);
  if (it != sel->cache.end()) {
    *out = it->second;
    return true;
  }
  float feats[15 * kSelectorFeatures];
  SplitConfig cand[15];
  const int nc = split_candidates(products, cand);
  for (int i = 0; i < nc; ++i)
    selector_features(sh, cand[i].pair ? 256 : 128, cand[i].bn, cand[i].splits, feats + i * kSelectorFeatures);
  if (cudaMemcpyAsync(sel->feat_dev, feats, sizeof(float) * nc * kSelectorFeatures,
                      cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
    return false;
  Handle* saved = sel->mlp->h;
  cudaStream_t saved_stream = saved->stream;
  saved->stream = h->stream;
  coral_status_t s = forward(sel->mlp, sel->feat_dev, nc, sel->pred_dev);
  saved->stream = saved_stream;
  float pred[15];
  if (s != CORAL_OK ||
      cudaMemcpyAsync(pred, sel->pred_dev, sizeof(float) * nc, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return false;
  int best = 0;
  for (int i = 1; i < nc; ++i)
    if (pred[i] < pred[best]) best = i;
  sel->cache[key] = cand[best];
  *out = cand[best];
  return true;
}

int split_candidates(int products, SplitConfig* out) {
  static const int kSp[5] = {1, 2, 4, 8, 16};
  int nc = 0;
  for (int t = 0; t < 3; ++t) {
    if (products == 6 && t == 1) continue;  // 3 pieces: no 128 x 256 single-CTA tile
    for (int s = 0; s < 5; ++s) {
      SplitConfig c{t == 2 ? 128 : 256, kSp[s]};
      c.pair = t == 0 ? 1 : 0;
      out[nc++] = c;
    }
  }
  return nc;
}

// Feature vector of (shape, configuration) for the selector network:
// log2 m, n, k; transpose flags; data type (products, complex); log2 batch;
// tile area (bm x bn over 128 x 256: 0.5, 1, or 2 for the CTA-pair tile) and
// log2 split-K; and the occupancy the configuration implies (log2 of output
// tiles, resident waves of work items -- 148 single CTAs or 74 pairs --, log2
// K slabs per split).
void selector_features(const SplitShape& sh, int bm, int bn, int splits, float* f) {
  const float m = (float)(sh.mr > 0 ? sh.mr : 1), n = (float)(sh.nr > 0 ? sh.nr : 1);
  const float k = (float)(sh.kd > 0 ? sh.kd : 1);
  f[0] = std::log2(m) / 16.f;
  f[1] = std::log2(n) / 16.f;
  f[2] = std::log2(k) / 16.f;
  f[3] = sh.op_a != 0 ? 1.f : 0.f;
  f[4] = sh.op_b != 0 ? 1.f : 0.f;
  f[5] = (float)sh.products / 6.f;
  f[6] = sh.complex_ ? 1.f : 0.f;
  f[7] = std::log2((float)(sh.batch > 0 ? sh.batch : 1)) / 12.f;
  f[8] = (float)(bm * bn) / (128.f * 256.f);
  f[9] = std::log2((float)splits) / 4.f;
  const float tiles = std::ceil(m / (float)bm) * std::ceil(n / (float)bn);
  const float items = tiles * (float)splits;
  const float resident = bm == 256 ? 74.f : 148.f;
  f[10] = std::log2(tiles) / 16.f;
  f[11] = std::min(items / resident, 8.f) / 8.f;
  f[12] = std::log2(std::max(1.f, std::ceil(k / 64.f) / (float)splits)) / 12.f;
}

// Features of a batch of `batch` instances of one shape under grouped tile
// width bn, in the layout of selector_features: log2 m, n, k; transpose flags;
// data type (3 products for fp32 inputs, 1 for bf16); log2 batch; tile width;
// log2 tiles per instance, resident waves of the batch's tiles, log2 K slabs.
void grouped_features(int input_type, int op_a, int op_b, int mi, int ni, int ki, int batch, int bn, float* f) {
  const float m = (float)(mi > 0 ? mi : 1), n = (float)(ni > 0 ? ni : 1), k = (float)(ki > 0 ? ki : 1);
  const float b = (float)(batch > 0 ? batch : 1);
  f[0] = std::log2(m) / 16.f;
  f[1] = std::log2(n) / 16.f;
  f[2] = std::log2(k) / 16.f;
  f[3] = op_a != 0 ? 1.f : 0.f;
  f[4] = op_b != 0 ? 1.f : 0.f;
  f[5] = (input_type == CORAL_INPUT_BF16 ? 1.f : 3.f) / 6.f;
  f[6] = 0.f;
  f[7] = std::log2(b) / 12.f;
  f[8] = (float)bn / 256.f;
  f[9] = 0.f;
  const float tiles = std::ceil(m / 128.f) * std::ceil(n / (float)bn);
  f[10] = std::log2(tiles) / 16.f;
  f[11] = std::min(tiles * b / 148.f, 8.f) / 8.f;
  f[12] = std::log2(std::max(1.f, std::ceil(k / 32.f))) / 12.f;
}

}  // namespace coral

using namespace coral;

extern "C" {

coral_status_t coral_grouped_features(int input_type, int op_a, int op_b, size_t m, size_t n, size_t k,
                                      size_t batch, int tile_n, float* out) {
  if (!out) return CORAL_ERR_INVALID_ARG;
  grouped_features(input_type, op_a, op_b, (int)m, (int)n, (int)k,
                   (int)(batch < (size_t)INT32_MAX ? batch : INT32_MAX), tile_n, out);
  return CORAL_OK;
}

// Learned choice of the grouped tile-width policy: for each instance class
// (n <= 64, <= 128, <= 256, > 256) present in the host copy of the
// descriptors, the class's median m, n, k, majority operations and instance
// count describe a uniform batch; the network predicts its log time under each
// allowed width (64 or 128 for the two small classes, 64, 128 or 256 for the
// others) and the class takes the argmin.  Classes without instances keep the
// handle's width.  Synchronises with the handle's stream.
coral_status_t coral_select_grouped_config(coral_handle_t hh, coral_mlp_t mlp, int input_type, size_t count,
                                           const coral_sgemm_problem_t* problems_host, int tile_n[4]) {
  CORAL_HANDLE(hh);
  Mlp* net = reinterpret_cast<Mlp*>(mlp);
  if (!net || net->in != kSelectorFeatures || net->out != 1) return bad_arg(H, 1);
  if (input_type != CORAL_INPUT_F32 && input_type != CORAL_INPUT_BF16) return bad_arg(H, 2);
  if (count && !problems_host) return bad_arg(H, 4);
  if (!tile_n) return bad_arg(H, 5);
  std::vector<int> ms[4], ns[4], ks[4];
  int ta[4] = {0, 0, 0, 0}, tb[4] = {0, 0, 0, 0};
  for (size_t i = 0; i < count; ++i) {
    const coral_sgemm_problem_t& p = problems_host[i];
    if (p.m <= 0 || p.n <= 0) continue;
    const int c = p.n <= 64 ? 0 : p.n <= 128 ? 1 : p.n <= 256 ? 2 : 3;
    ms[c].push_back(p.m);
    ns[c].push_back(p.n);
    ks[c].push_back(p.k);
    ta[c] += p.op_a != 0;
    tb[c] += p.op_b != 0;
  }
  auto median = [](std::vector<int>& v) {
    std::nth_element(v.begin(), v.begin() + v.size() / 2, v.end());
    return v[v.size() / 2];
  };
  float feats[12 * kSelectorFeatures];
  int cls[12], width[12], rows = 0;
  for (int c = 0; c < 4; ++c) {
    if (ms[c].empty()) continue;
    const int b = (int)ms[c].size();
    const int m = median(ms[c]), n = median(ns[c]), k = median(ks[c]);
    for (int bn : {64, 128, 256}) {
      if (c < 2 && bn == 256) continue;
      grouped_features(input_type, 2 * ta[c] > b, 2 * tb[c] > b, m, n, k, b, bn, feats + rows * kSelectorFeatures);
      cls[rows] = c;
      width[rows] = bn;
      ++rows;
    }
  }
  GroupedPolicy pol = H->grouped_policy;
  if (rows > 0) {
    char* d = static_cast<char*>(scratch(H, 16 * kSelectorFeatures * sizeof(float) + 256));
    if (!d) return CORAL_ERR_ALLOC;
    float* fx = reinterpret_cast<float*>(d);
    float* py = reinterpret_cast<float*>(d + 12 * kSelectorFeatures * sizeof(float));
    CORAL_CUDA(H, cudaMemcpyAsync(fx, feats, sizeof(float) * rows * kSelectorFeatures, cudaMemcpyHostToDevice,
                                  H->stream));
    Handle* owner = net->h;
    cudaStream_t saved = owner->stream;
    owner->stream = H->stream;
    coral_status_t s = forward(net, fx, rows, py);
    owner->stream = saved;
    if (s != CORAL_OK) return s;
    float pred[12];
    CORAL_CUDA(H, cudaMemcpyAsync(pred, py, sizeof(float) * rows, cudaMemcpyDeviceToHost, H->stream));
    CORAL_CUDA(H, cudaStreamSynchronize(H->stream));
    float best[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    for (int r = 0; r < rows; ++r)
      if (pred[r] < best[cls[r]]) {
        best[cls[r]] = pred[r];
        pol.bn[cls[r]] = width[r];
      }
  }
  H->grouped_policy = pol;
  for (int c = 0; c < 4; ++c) tile_n[c] = pol.bn[c];
  return CORAL_OK;
}

coral_status_t coral_mlp_create(coral_handle_t hh, int in_dim, int hidden, int out_dim,
                                uint64_t seed, coral_mlp_t* out) {
  CORAL_HANDLE(hh);
  if (in_dim < 1) return bad_arg(H, 1);
  if (hidden < 1) return bad_arg(H, 2);
  if (out_dim < 1) return bad_arg(H, 3);
  if (!out) return bad_arg(H, 5);
  Mlp* n = new Mlp();
  n->h = H;
  n->in = in_dim;
  n->hid = hidden;
  n->out = out_dim;
  n->nparams = (size_t)hidden * in_dim + hidden + (size_t)hidden * hidden + hidden +
               (size_t)out_dim * hidden + out_dim;
  if (cudaMalloc(&n->params, n->nparams * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&n->grads, n->nparams * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&n->adam_m, n->nparams * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&n->adam_v, n->nparams * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&n->loss_dev, sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    coral_mlp_destroy(reinterpret_cast<coral_mlp_t>(n));
    return CORAL_ERR_ALLOC;
  }
  // He-uniform initialisation (host, seeded), zero biases.
  std::vector<float> p(n->nparams, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](size_t off, int fan_in, size_t count) {
    const float lim = std::sqrt(6.f / (float)fan_in);
    std::uniform_real_distribution<float> u(-lim, lim);
    for (size_t i = 0; i < count; ++i) p[off + i] = u(rng);
  };
  size_t off = 0;
  fill(off, in_dim, (size_t)hidden * in_dim);
  off += (size_t)hidden * in_dim + hidden;
  fill(off, hidden, (size_t)hidden * hidden);
  off += (size_t)hidden * hidden + hidden;
  fill(off, hidden, (size_t)out_dim * hidden);
  CORAL_CUDA(H, cudaMemcpy(n->params, p.data(), n->nparams * sizeof(float), cudaMemcpyHostToDevice));
  CORAL_CUDA(H, cudaMemset(n->adam_m, 0, n->nparams * sizeof(float)));
  CORAL_CUDA(H, cudaMemset(n->adam_v, 0, n->nparams * sizeof(float)));
  *out = reinterpret_cast<coral_mlp_t>(n);
  return CORAL_OK;
}

coral_status_t coral_mlp_destroy(coral_mlp_t mlp) {
  Mlp* n = reinterpret_cast<Mlp*>(mlp);
  if (!n) return CORAL_OK;
  if (n->h) cudaStreamSynchronize(n->h->stream);
  cudaFree(n->params);
  cudaFree(n->grads);
  cudaFree(n->adam_m);
  cudaFree(n->adam_v);
  cudaFree(n->act);
  cudaFree(n->loss_dev);
  delete n;
  return CORAL_OK;
}

size_t coral_mlp_param_count(coral_mlp_t mlp) {
  Mlp* n = reinterpret_cast<Mlp*>(mlp);
  return n ? n->nparams : 0;
}

coral_status_t coral_mlp_get_params(coral_mlp_t mlp, float* host, size_t count) {
  Mlp* n = reinterpret_cast<Mlp*>(mlp);
  if (!n || !host || count != n->nparams) return CORAL_ERR_INVALID_ARG;
  CORAL_CUDA(n->h, cudaMemcpyAsync(host, n->params, count * sizeof(float), cudaMemcpyDeviceToHost, n->h->stream));
  CORAL_CUDA(n->h, cudaStreamSynchronize(n->h->stream));
  return CORAL_OK;
}

coral_status_t coral_mlp_set_params(coral_mlp_t mlp, const float* host, size_t count) {
  Mlp* n = reinterpret_cast<Mlp*>(mlp);
  if (!n || !host || count != n->nparams) return CORAL_ERR_INVALID_ARG;
  CORAL_CUDA(n->h, cudaMemcpyAsync(n->params, host, count * sizeof(float), cudaMemcpyHostToDevice, n->h->stream));
  CORAL_CUDA(n->h, cudaMemsetAsync(n->adam_m, 0, count * sizeof(float), n->h->stream));
  CORAL_CUDA(n->h, cudaMemsetAsync(n->adam_v, 0, count * sizeof(float), n->h->stream));
  CORAL_CUDA(n->h, cudaStreamSynchronize(n->h->stream));
  n->step = 0;
  return CORAL_OK;
}

coral_status_t coral_mlp_forward(coral_mlp_t mlp, const float* x, int batch, float* y) {
  Mlp* n = reinterpret_cast<Mlp*>(mlp);
  if (!n) return CORAL_ERR_INVALID_ARG;
  if (batch < 0 || (batch > 0 && (!x || !y))) return bad_arg(n->h, 2);
  if (batch == 0) return CORAL_OK;
  return forward(n, x, batch, y);
}

coral_status_t coral_mlp_gradients(coral_mlp_t mlp, const float* x, const float* target, int batch,
                                   float* grads, float* loss) {
  Mlp* n = reinterpret_cast<Mlp*>(mlp);
  if (!n) return CORAL_ERR_INVALID_ARG;
  if (batch < 1 || !x || !target) return bad_arg(n->h, 2);
  coral_status_t s = backward(n, x, target, batch);
  if (s != CORAL_OK) return s;
  if (grads)
    CORAL_CUDA(n->h, cudaMemcpyAsync(grads, n->grads, n->nparams * sizeof(float), cudaMemcpyDeviceToDevice, n->h->stream));
  if (loss) {
    CORAL_CUDA(n->h, cudaMemcpyAsync(loss, n->loss_dev, sizeof(float), cudaMemcpyDeviceToHost, n->h->stream));
    CORAL_CUDA(n->h, cudaStreamSynchronize(n->h->stream));
  }
  return CORAL_OK;
}

coral_status_t coral_mlp_train_step(coral_mlp_t mlp, const float* x, const float* target, int batch,
                                    float lr, float* loss) {
  Mlp* n = reinterpret_cast<Mlp*>(mlp);
  if (!n) return CORAL_ERR_INVALID_ARG;
  if (batch < 1 || !x || !target) return bad_arg(n->h, 2);
  coral_status_t s = backward(n, x, target, batch);
  if (s != CORAL_OK) return s;
  n->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)n->step), c2 = 1.f - std::pow(b2, (float)n->step);
  unsigned g = stream_grid(n->nparams, 256 * 4, n->h->sm_count, 4);
  k_adam<<<g, 256, 0, n->h->stream>>>(n->nparams, n->params, n->grads, n->adam_m, n->adam_v, lr, b1, b2,
                                      1e-8f, c1, c2);
  if ((s = launch_status(n->h)) != CORAL_OK) return s;
  if (loss) {
    CORAL_CUDA(n->h, cudaMemcpyAsync(loss, n->loss_dev, sizeof(float), cudaMemcpyDeviceToHost, n->h->stream));
    CORAL_CUDA(n->h, cudaStreamSynchronize(n->h->stream));
  }
  return CORAL_OK;
}

coral_status_t coral_set_selector(coral_handle_t hh, coral_mlp_t mlp) {
  CORAL_HANDLE(hh);
  Mlp* n = reinterpret_cast<Mlp*>(mlp);
  if (H->selector) {
    cudaStreamSynchronize(H->stream);
    cudaFree(H->selector->feat_dev);
    cudaFree(H->selector->pred_dev);
    delete H->selector;
    H->selector = nullptr;
  }
  if (!n) return CORAL_OK;
  if (n->in != kSelectorFeatures || n->out != 1) return bad_arg(H, 1);
  Selector* sel = new Selector();
  sel->mlp = n;
  if (cudaMalloc(&sel->feat_dev, 16 * kSelectorFeatures * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&sel->pred_dev, 16 * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    delete sel;
    return CORAL_ERR_ALLOC;
  }
  H->selector = sel;
  return CORAL_OK;
}

coral_status_t coral_set_gemm_config(coral_handle_t hh, int tile_n, int split_k) {
  CORAL_HANDLE(hh);
  if (tile_n != 0 && tile_n != 128 && tile_n != 256) return bad_arg(H, 1);
  if (split_k < 0 || split_k > 64) return bad_arg(H, 2);
  H->cfg_bn = tile_n;
  H->cfg_splits = split_k;
  H->cfg_bm = 0;
  return CORAL_OK;
}

coral_status_t coral_set_gemm_tile(coral_handle_t hh, int tile_m, int tile_n, int split_k) {
  CORAL_HANDLE(hh);
  if (tile_m != 0 && tile_m != 128 && tile_m != 256) return bad_arg(H, 1);
  if (tile_n != 0 && tile_n != 128 && tile_n != 256) return bad_arg(H, 2);
  if (tile_m == 256 && tile_n != 256) return bad_arg(H, 2);
  if (split_k < 0 || split_k > 64) return bad_arg(H, 3);
  H->cfg_bm = tile_m;
  H->cfg_bn = tile_n;
  H->cfg_splits = split_k;
  return CORAL_OK;
}

// Shapes whose sides do not fit an int have no configuration (the GEMM entry
// points report those sizes as not supported).
static bool shape_fits(size_t m, size_t n, size_t k) {
  return m <= (size_t)INT_MAX && n <= (size_t)INT_MAX && k <= (size_t)INT_MAX;
}

coral_status_t coral_get_gemm_tile(coral_handle_t hh, int products, int op_a, int op_b, size_t m,
                                   size_t n, size_t k, int* tile_m, int* tile_n, int* split_k) {
  CORAL_HANDLE(hh);
  if (products != 3 && products != 6) return bad_arg(H, 1);
  if (!shape_fits(m, n, k)) return CORAL_ERR_NOT_SUPPORTED;
  if (!tile_m) return bad_arg(H, 7);
  if (!tile_n) return bad_arg(H, 8);
  if (!split_k) return bad_arg(H, 9);
  SplitConfig c = choose_split_config(H, SplitShape{(int)m, (int)n, (int)k, products, op_a, op_b, 0, 1});
  *tile_m = c.pair ? 256 : 128;
  *tile_n = c.bn;
  *split_k = c.splits;
  return CORAL_OK;
}

coral_status_t coral_set_pair_raster(coral_handle_t hh, int group) {
  CORAL_HANDLE(hh);
  if (group < 0 || group > 64) return bad_arg(H, 1);
  H->pair_group = group;
  return CORAL_OK;
}

coral_status_t coral_get_gemm_config(coral_handle_t hh, int products, int op_a, int op_b, size_t m,
                                     size_t n, size_t k, int* tile_n, int* split_k) {
  CORAL_HANDLE(hh);
  if (products != 3 && products != 6) return bad_arg(H, 1);
  if (!shape_fits(m, n, k)) return CORAL_ERR_NOT_SUPPORTED;
  if (!tile_n) return bad_arg(H, 7);
  if (!split_k) return bad_arg(H, 8);
  SplitConfig c = choose_split_config(H, SplitShape{(int)m, (int)n, (int)k, products, op_a, op_b, 0, 1});
  *tile_n = c.bn;
  *split_k = c.splits;
  return CORAL_OK;
}

coral_status_t coral_selector_features(int products, int op_a, int op_b, size_t m, size_t n, size_t k,
                                       int tile_n, int split_k, float* out) {
  if (!out || tile_n <= 0 || split_k <= 0) return CORAL_ERR_INVALID_ARG;
  if (!shape_fits(m, n, k)) return CORAL_ERR_NOT_SUPPORTED;
  selector_features(SplitShape{(int)m, (int)n, (int)k, products, op_a, op_b, 0, 1}, 128, tile_n, split_k, out);
  return CORAL_OK;
}

coral_status_t coral_selector_features_tile(int products, int op_a, int op_b, size_t m, size_t n, size_t k,
                                            int tile_m, int tile_n, int split_k, float* out) {
  if (!out || tile_n <= 0 || split_k <= 0) return CORAL_ERR_INVALID_ARG;
  if (tile_m != 128 && tile_m != 256) return CORAL_ERR_INVALID_ARG;
  if (!shape_fits(m, n, k)) return CORAL_ERR_NOT_SUPPORTED;
  selector_features(SplitShape{(int)m, (int)n, (int)k, products, op_a, op_b, 0, 1}, tile_m, tile_n, split_k,
                    out);
  return CORAL_OK;
}

}  // extern "C"
