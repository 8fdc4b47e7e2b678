// Builds every wrapper of coral_b200/host/coral.hpp against libcoral_b200 and
// calls each once on small host operands.
//
// Without an sm_100 device every call must throw coral::Error carrying
// CORAL_ERR_NO_DEVICE (the library never falls back to the CPU); the program
// prints "no-device" and exits 0.  With a device, each result is checked
// against the reference's own small known answers (the sgemm doctest of
// sgemm.rs:36-81 and hand-checked level-1/2 values), and the program prints
// "device" and exits 0.  Any other outcome exits 1.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "coral.hpp"

namespace {

using coral::CoralDiagonal;
using coral::CoralTranspose;
using coral::CoralTriangular;

int g_failures = 0;

bool near(double got, double want) { return std::fabs(got - want) <= 1e-5 * (1.0 + std::fabs(want)); }

void expect(bool ok, const char* what) {
  if (!ok) {
    std::printf("FAIL %s\n", what);
    ++g_failures;
  }
}

// Runs one call; returns true when it ran on a device, false when it
// reported CORAL_ERR_NO_DEVICE.  Any other error is a failure.
template <typename F>
bool run(const char* name, bool device, F&& f) {
  try {
    f();
    if (!device) {
      std::printf("FAIL %s: returned without a device\n", name);
      ++g_failures;
    }
    return true;
  } catch (const coral::Error& e) {
    if (e.status == CORAL_ERR_NO_DEVICE && !device) return false;
    std::printf("FAIL %s: %s\n", name, e.what());
    ++g_failures;
    return false;
  }
}

}  // namespace

int main() {
  // Probe with the sgemm doctest: C = 2 * A B + C, A = [1 3; 2 4],
  // B = [5 7; 6 8], C = I (column-major), C becomes [47 62; 68 93].
  float a[4] = {1, 2, 3, 4}, b[4] = {5, 6, 7, 8}, c[4] = {1, 0, 0, 1};
  bool device = true;
  try {
    coral::level3::sgemm(CoralTranspose::NoTranspose, CoralTranspose::NoTranspose, 2, 2, 2, 2.0f, a, 2,
                         b, 2, 1.0f, c, 2);
  } catch (const coral::Error& e) {
    if (e.status != CORAL_ERR_NO_DEVICE) {
      std::printf("FAIL sgemm probe: %s\n", e.what());
      return 1;
    }
    device = false;
  }
  if (device) {
    const float want[4] = {47, 68, 62, 93};
    for (int i = 0; i < 4; ++i) expect(near(c[i], want[i]), "sgemm doctest");
  }

  double ad[4] = {1, 2, 3, 4}, bd[4] = {5, 6, 7, 8}, cd[4] = {1, 0, 0, 1};
  if (run("dgemm", device, [&] {
        coral::level3::dgemm(CoralTranspose::NoTranspose, CoralTranspose::NoTranspose, 2, 2, 2, 2.0, ad, 2,
                             bd, 2, 1.0, cd, 2);
      })) {
    const double want[4] = {47, 68, 62, 93};
    for (int i = 0; i < 4; ++i) expect(near(cd[i], want[i]), "dgemm");
  }

  // 1 x 1 complex products: (1 + 2i)(3 - i) = 5 + 5i; alpha = 1, beta = 0.
  float ac[2] = {1, 2}, bc[2] = {3, -1}, cc[2] = {9, 9}, one_c[2] = {1, 0}, zero_c[2] = {0, 0};
  if (run("cgemm", device, [&] {
        coral::level3::cgemm(CoralTranspose::NoTranspose, CoralTranspose::NoTranspose, 1, 1, 1, one_c, ac, 1,
                             bc, 1, zero_c, cc, 1);
      })) {
    expect(near(cc[0], 5) && near(cc[1], 5), "cgemm");
  }
  double az[2] = {1, 2}, bz[2] = {3, -1}, cz[2] = {9, 9}, one_z[2] = {1, 0}, zero_z[2] = {0, 0};
  if (run("zgemm", device, [&] {
        coral::level3::zgemm(CoralTranspose::NoTranspose, CoralTranspose::NoTranspose, 1, 1, 1, one_z, az, 1,
                             bz, 1, zero_z, cz, 1);
      })) {
    expect(near(cz[0], 5) && near(cz[1], 5), "zgemm");
  }

  // Level 2 on the 2 x 2 matrix M = [1 3; 2 4] and x = (1, 1).
  float m2[4] = {1, 2, 3, 4}, x2[2] = {1, 1}, y2[2] = {0, 0};
  if (run("sgemv", device, [&] {
        coral::level2::sgemv(CoralTranspose::NoTranspose, 2, 2, 1.0f, m2, 2, x2, 1, 0.0f, y2, 1);
      })) {
    expect(near(y2[0], 4) && near(y2[1], 6), "sgemv");
  }
  // upper triangle of M: [1 3; . 4]; solve [1 3; 0 4] x = (4, 4) -> (1, 1)
  float xs[2] = {4, 4};
  if (run("strsv", device, [&] {
        coral::level2::strsv(CoralTriangular::UpperTriangular, CoralTranspose::NoTranspose,
                             CoralDiagonal::NonUnitDiagonal, 2, m2, 2, xs, 1);
      })) {
    expect(near(xs[0], 1) && near(xs[1], 1), "strsv");
  }
  float xm[2] = {1, 1};
  if (run("strmv", device, [&] {
        coral::level2::strmv(CoralTriangular::UpperTriangular, CoralTranspose::NoTranspose,
                             CoralDiagonal::NonUnitDiagonal, 2, m2, 2, xm, 1);
      })) {
    expect(near(xm[0], 4) && near(xm[1], 4), "strmv");
  }
  // ssymv from the upper triangle: S = [1 3; 3 4], S (1, 1) = (4, 7)
  float ys[2] = {0, 0};
  if (run("ssymv", device, [&] {
        coral::level2::ssymv(CoralTriangular::UpperTriangular, 2, 1.0f, m2, 2, x2, 1, 0.0f, ys, 1);
      })) {
    expect(near(ys[0], 4) && near(ys[1], 7), "ssymv");
  }
  // chemv, 1 x 1: H = [2], x = 1 + i, y = H x = 2 + 2i
  float h1[2] = {2, 0}, xh[2] = {1, 1}, yh[2] = {0, 0};
  if (run("chemv", device, [&] {
        coral::level2::chemv(CoralTriangular::UpperTriangular, 1, one_c, h1, 1, xh, 1, zero_c, yh, 1);
      })) {
    expect(near(yh[0], 2) && near(yh[1], 2), "chemv");
  }
  float g[4] = {0, 0, 0, 0}, u[2] = {1, 2}, v[2] = {3, 4};
  if (run("sger", device, [&] { coral::level2::sger(2, 2, 1.0f, u, 1, v, 1, g, 2); })) {
    const float want[4] = {3, 6, 4, 8};
    for (int i = 0; i < 4; ++i) expect(near(g[i], want[i]), "sger");
  }
  float s1[4] = {0, 0, 0, 0};
  if (run("ssyr", device, [&] { coral::level2::ssyr(CoralTriangular::UpperTriangular, 2, 1.0f, u, 1, s1, 2); })) {
    expect(near(s1[0], 1) && near(s1[2], 2) && near(s1[3], 4) && s1[1] == 0.0f, "ssyr");
  }
  float s2[4] = {0, 0, 0, 0};
  if (run("ssyr2", device,
          [&] { coral::level2::ssyr2(CoralTriangular::LowerTriangular, 2, 1.0f, u, 1, v, 1, s2, 2); })) {
    // x y^T + y x^T = [6 10; 10 16], lower triangle only
    expect(near(s2[0], 6) && near(s2[1], 10) && near(s2[3], 16) && s2[2] == 0.0f, "ssyr2");
  }

  // Level 1 on x = (3, -4, 1).
  float x3[3] = {3, -4, 1}, y3[3] = {1, 1, 1};
  float dot = 0.0f, nrm = 0.0f;
  size_t imax = 99;
  if (run("sdot", device, [&] { dot = coral::level1::sdot(3, x3, 1, y3, 1); })) expect(near(dot, 0), "sdot");
  if (run("snrm2", device, [&] { nrm = coral::level1::snrm2(3, x3, 1); }))
    expect(near(nrm, std::sqrt(26.0)), "snrm2");
  if (run("isamax", device, [&] { imax = coral::level1::isamax(3, x3, 1); })) expect(imax == 1, "isamax");
  float y4[3] = {1, 1, 1};
  if (run("saxpy", device, [&] { coral::level1::saxpy(3, 2.0f, x3, 1, y4, 1); }))
    expect(near(y4[0], 7) && near(y4[1], -7) && near(y4[2], 3), "saxpy");
  float y5[3] = {0, 0, 0};
  if (run("scopy", device, [&] { coral::level1::scopy(3, x3, 1, y5, 1); }))
    expect(std::memcmp(x3, y5, sizeof x3) == 0, "scopy");
  float p[2] = {1, 2}, q[2] = {3, 4};
  if (run("sswap", device, [&] { coral::level1::sswap(2, p, 1, q, 1); }))
    expect(p[0] == 3 && p[1] == 4 && q[0] == 1 && q[1] == 2, "sswap");
  float r[2] = {1, -2};
  if (run("sscal", device, [&] { coral::level1::sscal(2, -0.5f, r, 1); }))
    expect(near(r[0], -0.5) && near(r[1], 1), "sscal");
  run("set_gemm_mode", device, [&] { coral::set_gemm_mode(0); });

  if (g_failures) return 1;
  std::printf(device ? "device\n" : "no-device\n");
  return 0;
}
