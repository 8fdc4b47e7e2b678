// coral_safe.hpp routines on a B200 against host loops in double: every view
// has an offset, most a stride, so the pointer arithmetic of the views is
// exercised.  Bounds: |got - want| <= 1e-5 (|terms| summed) for fp32 data;
// indices and copies exact.  Exit status 0 on success.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <random>
#include <stdexcept>
#include <vector>

#include "coral_safe.hpp"

using namespace coral::safe;

static int failures = 0;
#define EXPECT(cond)                                              \
  do {                                                            \
    if (!(cond)) {                                                \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #cond); \
      ++failures;                                                 \
    }                                                             \
  } while (0)

struct Dev {
  float* p = nullptr;
  size_t n = 0;
  explicit Dev(const std::vector<float>& h) : n(h.size()) {
    if (cudaMalloc(&p, n * sizeof(float)) != cudaSuccess) throw std::runtime_error("cudaMalloc");
    cudaMemcpy(p, h.data(), n * sizeof(float), cudaMemcpyHostToDevice);
  }
  ~Dev() { cudaFree(p); }
  std::vector<float> get() const {
    std::vector<float> h(n);
    cudaDeviceSynchronize();
    cudaMemcpy(h.data(), p, n * sizeof(float), cudaMemcpyDeviceToHost);
    return h;
  }
  DeviceSlice<float> mut() const { return {p, n}; }
  DeviceSlice<const float> ref() const { return {p, n}; }
};

static std::vector<float> rnd(size_t n, unsigned seed) {
  std::mt19937 g(seed);
  std::uniform_real_distribution<float> u(-1.f, 1.f);
  std::vector<float> v(n);
  for (auto& e : v) e = u(g);
  return v;
}

static bool near(double got, double want, double scale) { return std::fabs(got - want) <= 1e-5 * scale + 1e-30; }

int main() {
  Handle h;
  const size_t n = 1000, ox = 3, sx = 2, oy = 5, sy = 1;
  auto hx = rnd(ox + (n - 1) * sx + 1, 1), hy = rnd(oy + (n - 1) * sy + 1, 2);
  Dev dx(hx), dy(hy);
  auto X = [&] { return VectorRef<float>::make(dx.ref(), n, sx, ox).unwrap(); };
  auto Y = [&] { return VectorRef<float>::make(dy.ref(), n, sy, oy).unwrap(); };
  auto XM = [&] { return VectorMut<float>::make(dx.mut(), n, sx, ox).unwrap(); };
  auto YM = [&] { return VectorMut<float>::make(dy.mut(), n, sy, oy).unwrap(); };
  auto xi = [&](const std::vector<float>& v, size_t i) { return (double)v[ox + i * sx]; };
  auto yi = [&](const std::vector<float>& v, size_t i) { return (double)v[oy + i * sy]; };

  // sdot, sasum, snrm2, isamax
  double dot = 0, adot = 0, asum = 0, ss = 0;
  size_t imax = 0;
  double best = -1;
  for (size_t i = 0; i < n; ++i) {
    dot += xi(hx, i) * yi(hy, i);
    adot += std::fabs(xi(hx, i) * yi(hy, i));
    asum += std::fabs(xi(hx, i));
    ss += xi(hx, i) * xi(hx, i);
    if (std::fabs(xi(hx, i)) > best) { best = std::fabs(xi(hx, i)); imax = i; }
  }
  EXPECT(near(sdot(h, X(), Y()), dot, adot));
  EXPECT(near(sasum(h, X()), asum, asum));
  EXPECT(near(snrm2(h, X()), std::sqrt(ss), std::sqrt(ss)));
  EXPECT(isamax(h, X()) == imax);
  // length mismatch -> std::invalid_argument (debug_assert_n_eq!)
  bool threw = false;
  try {
    sdot(h, X(), VectorRef<float>::make(dy.ref(), n - 1, 1, 0).unwrap());
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  EXPECT(threw);

  // saxpy, sscal, scopy, sswap, srot, srotm
  saxpy(h, 0.5f, X(), YM());
  auto gy = dy.get();
  bool ok = true;
  for (size_t i = 0; i < n; ++i) ok &= near(yi(gy, i), yi(hy, i) + 0.5 * xi(hx, i), 2.0);
  EXPECT(ok);
  hy = gy;
  sscal(h, -2.0f, XM());
  auto gx = dx.get();
  ok = true;
  for (size_t i = 0; i < n; ++i) ok &= gx[ox + i * sx] == -2.0f * hx[ox + i * sx];
  for (size_t i = 0; i < ox; ++i) ok &= gx[i] == hx[i];  // before the offset: untouched
  EXPECT(ok);
  hx = gx;
  scopy(h, X(), YM());
  gy = dy.get();
  ok = true;
  for (size_t i = 0; i < n; ++i) ok &= gy[oy + i * sy] == hx[ox + i * sx];
  EXPECT(ok);
  hy = rnd(hy.size(), 3);
  cudaMemcpy(dy.p, hy.data(), hy.size() * sizeof(float), cudaMemcpyHostToDevice);
  sswap(h, XM(), YM());
  gx = dx.get();
  gy = dy.get();
  ok = true;
  for (size_t i = 0; i < n; ++i) ok &= gx[ox + i * sx] == hy[oy + i * sy] && gy[oy + i * sy] == hx[ox + i * sx];
  EXPECT(ok);
  hx = gx;
  hy = gy;
  srot(h, XM(), YM(), 0.6f, 0.8f);
  gx = dx.get();
  gy = dy.get();
  ok = true;
  for (size_t i = 0; i < n; ++i) {
    ok &= near(xi(gx, i), 0.6 * xi(hx, i) + 0.8 * yi(hy, i), 2.0);
    ok &= near(yi(gy, i), 0.6 * yi(hy, i) - 0.8 * xi(hx, i), 2.0);
  }
  EXPECT(ok);
  hx = gx;
  hy = gy;
  const float param[5] = {-1.f, 1.1f, -0.4f, 0.7f, 0.9f};
  srotm(h, XM(), YM(), param);
  gx = dx.get();
  gy = dy.get();
  ok = true;
  for (size_t i = 0; i < n; ++i) {
    ok &= near(xi(gx, i), 1.1 * xi(hx, i) + 0.7 * yi(hy, i), 3.0);
    ok &= near(yi(gy, i), -0.4 * xi(hx, i) + 0.9 * yi(hy, i), 3.0);
  }
  EXPECT(ok);

  // srotg / srotmg on host scalars
  float a = 3.f, b = 4.f, c = 0, s = 0;
  srotg(h, a, b, c, s);
  EXPECT(std::fabs(a - 5.f) < 1e-6f && std::fabs(c - 0.6f) < 1e-6f && std::fabs(s - 0.8f) < 1e-6f);
  float d1 = 1.f, d2 = 2.f, x1 = 3.f, p[5] = {};
  srotmg(h, d1, d2, x1, 4.f, p);
  EXPECT(p[0] == 1.f && std::fabs(p[1] - 0.375f) < 1e-7f && std::fabs(p[4] - 0.75f) < 1e-7f);

  // sgemv N and T, sger, saxpyf, sdotf on a 300 x 200 matrix at offset 7, lda 305
  const size_t m = 300, k = 200, lda = 305, oa = 7;
  auto ha = rnd(oa + (k - 1) * lda + m, 4);
  Dev da(ha);
  auto A = [&] { return MatrixRef<float>::make(da.ref(), m, k, lda, oa).unwrap(); };
  auto AM = [&] { return MatrixMut<float>::make(da.mut(), m, k, lda, oa).unwrap(); };
  auto aij = [&](const std::vector<float>& v, size_t i, size_t j) { return (double)v[oa + j * lda + i]; };
  auto hv = rnd(1 + (k - 1) * 3 + 1, 5), hw = rnd(2 + (m - 1) * 2 + 1, 6);
  Dev dv(hv), dw(hw);
  auto V = VectorRef<float>::make(dv.ref(), k, 3, 1).unwrap();   // length n_cols
  auto W = VectorMut<float>::make(dw.mut(), m, 2, 2).unwrap();   // length n_rows
  sgemv(h, CoralTranspose::NoTrans, 1.5f, 0.5f, A(), V, W);
  auto gw = dw.get();
  ok = true;
  for (size_t i = 0; i < m; ++i) {
    double acc = 0, sc = 0;
    for (size_t j = 0; j < k; ++j) {
      acc += aij(ha, i, j) * hv[1 + j * 3];
      sc += std::fabs(aij(ha, i, j) * hv[1 + j * 3]);
    }
    ok &= near(gw[2 + i * 2], 1.5 * acc + 0.5 * hw[2 + i * 2], 1.5 * sc + 1.0);
  }
  EXPECT(ok);
  hw = gw;
  // y += A^T w through sdotf with a strided output (length n_cols)
  auto hz = rnd(4 + (k - 1) * 2 + 1, 7);
  Dev dz(hz);
  auto Wr = VectorRef<float>::make(dw.ref(), m, 2, 2).unwrap();
  sdotf(h, A(), Wr, VectorMut<float>::make(dz.mut(), k, 2, 4).unwrap());
  auto gz = dz.get();
  ok = true;
  for (size_t j = 0; j < k; ++j) {
    double acc = 0, sc = 0;
    for (size_t i = 0; i < m; ++i) {
      acc += aij(ha, i, j) * hw[2 + i * 2];
      sc += std::fabs(aij(ha, i, j) * hw[2 + i * 2]);
    }
    ok &= near(gz[4 + j * 2], hz[4 + j * 2] + acc, sc + 1.0);
  }
  EXPECT(ok);
  // saxpyf: w += A v
  saxpyf(h, A(), V, W);
  gw = dw.get();
  ok = true;
  for (size_t i = 0; i < m; ++i) {
    double acc = 0, sc = 0;
    for (size_t j = 0; j < k; ++j) {
      acc += aij(ha, i, j) * hv[1 + j * 3];
      sc += std::fabs(aij(ha, i, j) * hv[1 + j * 3]);
    }
    ok &= near(gw[2 + i * 2], hw[2 + i * 2] + acc, sc + 1.0);
  }
  EXPECT(ok);
  hw = gw;
  // sger: A += 0.25 w v^T
  sger(h, 0.25f, AM(), VectorRef<float>::make(dw.ref(), m, 2, 2).unwrap(), V);
  auto ga = da.get();
  ok = true;
  for (size_t j = 0; j < k; ++j)
    for (size_t i = 0; i < m; ++i)
      ok &= near(aij(ga, i, j), aij(ha, i, j) + 0.25 * hw[2 + i * 2] * hv[1 + j * 3], 2.0);
  for (size_t i = 0; i < oa; ++i) ok &= ga[i] == ha[i];
  EXPECT(ok);

  // strsv lower, non-unit, diagonally dominant 256 x 256 at offset 9
  const size_t nt = 256, ot = 9;
  auto hl = rnd(ot + nt * nt, 8);
  for (size_t i = 0; i < nt; ++i) hl[ot + i * nt + i] = (float)nt;
  Dev dl(hl);
  auto hb = rnd(nt, 9);
  Dev db(hb);
  strsv(h, CoralTriangular::Lower, CoralTranspose::NoTrans, CoralDiagonal::NonUnit,
        MatrixRef<float>::make(dl.ref(), nt, nt, nt, ot).unwrap(), VectorMut<float>::make(db.mut(), nt, 1, 0).unwrap());
  auto gb = db.get();
  ok = true;
  for (size_t i = 0; i < nt; ++i) {  // residual of L x = b
    double r = 0;
    for (size_t j = 0; j <= i; ++j) r += (double)hl[ot + j * nt + i] * gb[j];
    ok &= std::fabs(r - hb[i]) <= 1e-4 * (1.0 + std::fabs(hb[i]));
  }
  EXPECT(ok);
  // a non-square matrix is refused before any call
  threw = false;
  try {
    strsv(h, CoralTriangular::Lower, CoralTranspose::NoTrans, CoralDiagonal::NonUnit, A(),
          VectorMut<float>::make(db.mut(), nt, 1, 0).unwrap());
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  EXPECT(threw);

  const cudaError_t e = cudaDeviceSynchronize();
  EXPECT(e == cudaSuccess);
  std::printf("%s (%d failures)\n", failures ? "FAILED" : "ok", failures);
  return failures ? 1 : 0;
}
