/*
 * oracle.c -- CPU restatement of CORAL's BLAS semantics.  TEST INFRASTRUCTURE
 * ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * arm as the checker; nothing in the coral_b200 product links or calls it.
 *
 * Three kinds of functions:
 *   or_*_exact  fp32 restatements that reproduce the reference's rounding
 *               element for element (the GPU must match these bit for bit);
 *   or_*_f64    FP64 (or double-double, `dd`) references of the mathematical
 *               result, following the reference's quick returns and scaling
 *               order, for tolerance-based parity and error measurement;
 *   port_*      restatements of CORAL's own CPU algorithms (blocking, loop
 *               order, fp32 accumulation) that bench.py times as the
 *               reference CPU path, because the Rust crate cannot be built
 *               here (no cargo, and coral-aarch64 is aarch64-only).
 *
 * Reference paths are relative to the devdeliw/CORAL checkout
 * (coral-aarch64/src/...).  Compile with -ffp-contract=off: the reference's
 * `a += b * c` in Rust is two roundings, and only explicit fmaf()/fma() may
 * fuse.
 */
#include <immintrin.h>
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define UPPER 0
#define LOWER 1
#define UNIT 0
#define NON_UNIT 1
#define NOTRANS 0
#define TRANS 1
#define CONJTRANS 2

/* ---------------- double-double helpers (Dekker/Knuth, with fma) --------- */
typedef struct { double hi, lo; } dd;

static inline dd dd_two_sum(double a, double b) {
  double s = a + b, bb = s - a, e = (a - (s - bb)) + (b - bb);
  dd r = {s, e};
  return r;
}
static inline dd dd_add_prod(dd acc, double a, double b) {
  double p = a * b, pe = fma(a, b, -p);
  dd s = dd_two_sum(acc.hi, p);
  s.lo += acc.lo + pe;
  return dd_two_sum(s.hi, s.lo);
}
static inline double dd_val(dd a) { return a.hi + a.lo; }

/* ============================ level 1 ==================================== */

/* level1/saxpy.rs:42-131: fused body for the first n - n%8 elements of the
 * unit-stride path (16- and 8-wide vfmaq_f32), `*y += alpha * x` otherwise. */
void or_saxpy_exact(size_t n, float alpha, const float* x, size_t incx, float* y, size_t incy) {
  if (n == 0 || alpha == 0.0f) return;
  if (incx == 1 && incy == 1) {
    size_t nf = n - (n % 8);
    for (size_t i = 0; i < nf; ++i) y[i] = fmaf(alpha, x[i], y[i]);
    for (size_t i = nf; i < n; ++i) y[i] += alpha * x[i];
  } else {
    for (size_t i = 0; i < n; ++i) y[i * incy] += alpha * x[i * incx];
  }
}

/* level1/sscal.rs:30-66: multiplies even when alpha == 0. */
void or_sscal_exact(size_t n, float alpha, float* x, size_t incx) {
  if (n == 0 || incx == 0) return;
  for (size_t i = 0; i < n; ++i) x[i * incx] = x[i * incx] * alpha;
}

/* level1/scopy.rs:28-58 */
void or_scopy_exact(size_t n, const float* x, size_t incx, float* y, size_t incy) {
  for (size_t i = 0; i < n; ++i) y[i * incy] = x[i * incx];
}

/* level1/sswap.rs:35-118 */
void or_sswap_exact(size_t n, float* x, size_t incx, float* y, size_t incy) {
  for (size_t i = 0; i < n; ++i) {
    float t = x[i * incx];
    x[i * incx] = y[i * incy];
    y[i * incy] = t;
  }
}

/* level1/isamax.rs:43-151: first index of the largest |x_i|; NaN never wins
 * (mapped to -inf in the SIMD body, rejected by `v > best` in the scalar
 * paths); n == 0 or incx == 0 -> 0. */
size_t or_isamax_exact(size_t n, const float* x, size_t incx) {
  if (n == 0 || incx == 0) return 0;
  float best = -INFINITY;
  size_t idx = 0;
  for (size_t i = 0; i < n; ++i) {
    float v = fabsf(x[i * incx]);
    if (v > best) { best = v; idx = i; }
  }
  return idx;
}

/* level1/sdot.rs:42-161 (exact value of the fp32 inputs' dot product). */
double or_sdot_f64(size_t n, const float* x, size_t incx, const float* y, size_t incy) {
  dd acc = {0.0, 0.0};
  for (size_t i = 0; i < n; ++i) acc = dd_add_prod(acc, x[i * incx], y[i * incy]);
  return dd_val(acc);
}

/* level1/snrm2.rs:45-149 -- ||x||_2; n == 0 or incx == 0 -> 0. */
double or_snrm2_f64(size_t n, const float* x, size_t incx) {
  if (n == 0 || incx == 0) return 0.0;
  dd acc = {0.0, 0.0};
  for (size_t i = 0; i < n; ++i) acc = dd_add_prod(acc, x[i * incx], x[i * incx]);
  return sqrt(dd_val(acc));
}

/* ---------------- double and complex level 1 ------------------------------
 * kind: 0 = s (float), 1 = d (double), 2 = c (complex64), 3 = z (complex128);
 * complex data interleaved, increments in complex elements.  The reference's
 * unit-stride loops run a NEON body over the first n - n % W elements and a
 * scalar tail; the body fuses where the tail rounds every product, so the
 * exact restatements take `nf` = n - n % W (unit strides) or 0. */
#define L1_LOAD(kind, p, i, re, im)                                           \
  do {                                                                        \
    if ((kind) == 0) { re = ((const float*)(p))[i]; im = 0; }                 \
    else if ((kind) == 1) { re = ((const double*)(p))[i]; im = 0; }           \
    else if ((kind) == 2) { re = ((const float*)(p))[2 * (i)]; im = ((const float*)(p))[2 * (i) + 1]; } \
    else { re = ((const double*)(p))[2 * (i)]; im = ((const double*)(p))[2 * (i) + 1]; } \
  } while (0)

static size_t nf_of(size_t n, size_t incx, size_t incy, size_t w) {
  return (incx == 1 && incy == 1) ? n - n % w : 0;
}

/* daxpy.rs:42-133 (W 4), caxpy.rs:45-172 (W 4), zaxpy.rs:44-172 (W 2):
 * body y += a x fused (complex: yr = fma(ar, xr, yr), yr = fma(-ai, xi, yr),
 * yi = fma(ar, xi, yi), yi = fma(ai, xr, yi)); tail y += a x /
 * yr += ar xr - ai xi, yi += ar xi + ai xr.  n == 0 or alpha == 0 returns. */
#define OR_AXPY_C(T, FMA)                                                       \
  {                                                                           \
    const T ar = (T)alpha[0], ai = (T)alpha[1];                               \
    if (ar == 0 && ai == 0) return;                                           \
    T* xx = (T*)x; T* yy = (T*)y;                                             \
    for (size_t i = 0; i < n; ++i) {                                          \
      T xr = xx[2 * i * incx], xi = xx[2 * i * incx + 1];                     \
      T* yp = yy + 2 * i * incy;                                              \
      if (i < nf) {                                                           \
        yp[0] = FMA(ar, xr, yp[0]); yp[0] = FMA(-ai, xi, yp[0]);              \
        yp[1] = FMA(ar, xi, yp[1]); yp[1] = FMA(ai, xr, yp[1]);               \
      } else {                                                                \
        yp[0] += ar * xr - ai * xi;                                           \
        yp[1] += ar * xi + ai * xr;                                           \
      }                                                                       \
    }                                                                         \
  }
void or_axpy_exact(int kind, size_t n, const double alpha[2], const void* x, size_t incx, void* y,
                   size_t incy) {
  if (n == 0) return;
  const size_t nf = nf_of(n, incx, incy, kind == 3 ? 2 : 4);
  if (kind == 1) {
    const double a = alpha[0];
    if (a == 0.0) return;
    const double* xx = (const double*)x;
    double* yy = (double*)y;
    for (size_t i = 0; i < n; ++i)
      yy[i * incy] = i < nf ? fma(a, xx[i * incx], yy[i * incy]) : yy[i * incy] + a * xx[i * incx];
  } else if (kind == 2) OR_AXPY_C(float, fmaf)
  else OR_AXPY_C(double, fma)
}

/* dscal.rs:30-66 (kind 1), cscal.rs:43-111 (kind 2, W 4), zscal.rs:41-109
 * (kind 3, W 2), csscal.rs:39-88 (kind 4: real alpha, complex64) and
 * zdscal.rs:38-88 (kind 5: real alpha, complex128).  Complex body:
 * re = fma(-xi, ai, xr ar), im = fma(xr, ai, xi ar); tail re = ar xr - ai xi,
 * im = ar xi + ai xr.  Real alpha multiplies each part.  n == 0 or incx == 0
 * returns; alpha == 0 still multiplies. */
#define OR_SCAL_C(T, FMA, W)                                                    \
  {                                                                           \
    const T ar = (T)alpha[0], ai = (T)alpha[1];                               \
    T* xx = (T*)x;                                                            \
    const size_t nf = nf_of(n, incx, 1, W);                                   \
    for (size_t i = 0; i < n; ++i) {                                          \
      T* p = xx + 2 * i * incx;                                               \
      T re, im;                                                               \
      if (i < nf) { re = FMA(-p[1], ai, p[0] * ar); im = FMA(p[0], ai, p[1] * ar); } \
      else { re = ar * p[0] - ai * p[1]; im = ar * p[1] + ai * p[0]; }        \
      p[0] = re; p[1] = im;                                                   \
    }                                                                         \
  }
void or_scal_exact(int kind, size_t n, const double alpha[2], void* x, size_t incx) {
  if (n == 0 || incx == 0) return;
  if (kind == 1) {
    double* xx = (double*)x;
    for (size_t i = 0; i < n; ++i) xx[i * incx] = xx[i * incx] * alpha[0];
  } else if (kind == 2) OR_SCAL_C(float, fmaf, 4)
  else if (kind == 3) OR_SCAL_C(double, fma, 2)
  else if (kind == 4) {
    float* xx = (float*)x;
    const float a = (float)alpha[0];
    for (size_t i = 0; i < n; ++i) { xx[2 * i * incx] *= a; xx[2 * i * incx + 1] *= a; }
  } else {
    double* xx = (double*)x;
    for (size_t i = 0; i < n; ++i) { xx[2 * i * incx] *= alpha[0]; xx[2 * i * incx + 1] *= alpha[0]; }
  }
}

/* srot.rs:51-180 (kind 0, W 4), drot.rs:48-178 (kind 1, W 2), csrot.rs:50-166
 * (kind 2, W 2 complex) and zdrot.rs:51-166 (kind 3, every unit-stride
 * element in the body): x' = c x + s y, y' = c y - s x per real part.  Body:
 * x' = fma(y, s, c x); real kinds y' = fma(-s, x, c y), complex kinds round
 * both products of y'.  n == 0 returns. */
#define OR_ROT_PART(T, FMA, FUSEY, xp, yp, fused)                               \
  do {                                                                        \
    T xv = *(xp), yv = *(yp), xn, yn;                                         \
    if (fused) {                                                              \
      xn = FMA(yv, s, c * xv);                                                \
      yn = (FUSEY) ? FMA(-s, xv, c * yv) : c * yv - s * xv;                   \
    } else { xn = c * xv + s * yv; yn = c * yv - s * xv; }                    \
    *(xp) = xn; *(yp) = yn;                                                   \
  } while (0)
void or_rot_exact(int kind, size_t n, void* x, size_t incx, void* y, size_t incy, double cc, double ss) {
  if (n == 0) return;
  static const size_t W[4] = {4, 2, 2, 1};
  const size_t nf = nf_of(n, incx, incy, W[kind]);
  if (kind == 0 || kind == 2) {
    const float c = (float)cc, s = (float)ss;
    float* xx = (float*)x; float* yy = (float*)y;
    for (size_t i = 0; i < n; ++i) {
      if (kind == 0) OR_ROT_PART(float, fmaf, 1, xx + i * incx, yy + i * incy, i < nf);
      else for (int h = 0; h < 2; ++h) OR_ROT_PART(float, fmaf, 0, xx + 2 * i * incx + h, yy + 2 * i * incy + h, i < nf);
    }
  } else {
    const double c = cc, s = ss;
    double* xx = (double*)x; double* yy = (double*)y;
    for (size_t i = 0; i < n; ++i) {
      if (kind == 1) OR_ROT_PART(double, fma, 1, xx + i * incx, yy + i * incy, i < nf);
      else for (int h = 0; h < 2; ++h) OR_ROT_PART(double, fma, 0, xx + 2 * i * incx + h, yy + 2 * i * incy + h, i < nf);
    }
  }
}

/* srotm.rs:47-412 (kind 0, W 4) and drotm.rs:47-410 (kind 1, W 2):
 * param = [flag, h11, h21, h12, h22]; flag == -2 or n == 0 returns; flag < 0
 * full H (body x' = fma(y, h12, h11 x), y' = fma(x, h21, h22 y); tail
 * h11 x + h12 y, h21 x + h22 y); flag == 0 (body fma(y, h12, x),
 * fma(x, h21, y); tail x + h12 y, h21 x + y); otherwise (body fma(x, h11, y),
 * h22 y - x; tail h11 x + y, -x + h22 y). */
#define OR_ROTM(T, FMA)                                                         \
  {                                                                           \
    const T flag = (T)param[0], h11 = (T)param[1], h21 = (T)param[2],         \
            h12 = (T)param[3], h22 = (T)param[4];                             \
    if (flag == (T)-2) return;                                                \
    T* xx = (T*)x; T* yy = (T*)y;                                             \
    for (size_t i = 0; i < n; ++i) {                                          \
      const T a = xx[i * incx], b = yy[i * incy];                             \
      const int f = i < nf;                                                   \
      T xn, yn;                                                               \
      if (flag < 0) {                                                         \
        xn = f ? FMA(b, h12, h11 * a) : h11 * a + h12 * b;                    \
        yn = f ? FMA(a, h21, h22 * b) : h21 * a + h22 * b;                    \
      } else if (flag == 0) {                                                 \
        xn = f ? FMA(b, h12, a) : a + h12 * b;                                \
        yn = f ? FMA(a, h21, b) : h21 * a + b;                                \
      } else {                                                                \
        xn = f ? FMA(a, h11, b) : h11 * a + b;                                \
        yn = f ? h22 * b - a : -a + h22 * b;                                  \
      }                                                                       \
      xx[i * incx] = xn; yy[i * incy] = yn;                                   \
    }                                                                         \
  }
void or_rotm_exact(int kind, size_t n, void* x, size_t incx, void* y, size_t incy, const double param[5]) {
  if (n == 0) return;
  const size_t nf = nf_of(n, incx, incy, kind == 0 ? 4 : 2);
  if (kind == 0) OR_ROTM(float, fmaf)
  else OR_ROTM(double, fma)
}

/* srotg.rs:40-75 / drotg.rs:40-71: r = scale sqrt((a/scale)^2 + (b/scale)^2)
 * with the sign of the larger of a, b; c = a / r, s = b / r; z = s when
 * |a| > |b|, 1 / c when |b| >= |a| and c != 0, else 1; a <- r, b <- z.
 * scale == 0 gives c = 1, s = 0, a = b = 0.  v = {a, b, c, s}. */
#define OR_ROTG(T, FABS, SQRT)                                                  \
  {                                                                           \
    T a = (T)v[0], b = (T)v[1];                                               \
    T roe = FABS(a) > FABS(b) ? a : b, scale = FABS(a) + FABS(b);             \
    if (scale == 0) { v[0] = 0; v[1] = 0; v[2] = 1; v[3] = 0; return; }       \
    T qa = a / scale, qb = b / scale;                                         \
    T r = scale * SQRT(qa * qa + qb * qb);                                    \
    if (roe < 0) r = -r;                                                      \
    T c = a / r, s = b / r, z = 1;                                            \
    if (FABS(a) > FABS(b)) z = s;                                             \
    if (FABS(b) >= FABS(a) && c != 0) z = (T)1 / c;                           \
    v[0] = r; v[1] = z; v[2] = c; v[3] = s;                                   \
  }
void or_rotg_exact(int dbl, double v[4]) {
  if (dbl) OR_ROTG(double, fabs, sqrt)
  else OR_ROTG(float, fabsf, sqrtf)
}

/* srotmg.rs:42-199 / drotmg.rs:41-195: modified Givens construction with
 * rescaling by gam = 4096 (the loops stop after 256 steps, which finite
 * inputs never reach).  v = {d1, d2, x1, y1}; param[5] written (param[0] = -2
 * only when d2 y1 == 0, leaving v untouched). */
#define OR_ROTMG(T, FABS)                                                       \
  {                                                                           \
    const T gam = 4096, gamsq = gam * gam, rgamsq = (T)1 / gamsq;             \
    T d1 = (T)v[0], d2 = (T)v[1], x1 = (T)v[2], y1 = (T)v[3];                 \
    T flag, h11 = 0, h12 = 0, h21 = 0, h22 = 0;                               \
    if (d1 < 0) { flag = -1; d1 = 0; d2 = 0; x1 = 0; }                        \
    else {                                                                    \
      T p2 = d2 * y1;                                                         \
      if (p2 == 0) { param[0] = -2; return; }                                 \
      T p1 = d1 * x1, q2 = p2 * y1, q1 = p1 * x1;                             \
      if (FABS(q1) > FABS(q2)) {                                              \
        h21 = -y1 / x1; h12 = p2 / p1;                                        \
        T u = 1 - h12 * h21;                                                  \
        if (u <= 0) { flag = -1; d1 = d2 = x1 = 0; h11 = h12 = h21 = h22 = 0; } \
        else { flag = 0; d1 /= u; d2 /= u; x1 *= u; }                         \
      } else if (q2 < 0) { flag = -1; d1 = d2 = x1 = 0; h11 = h12 = h21 = h22 = 0; } \
      else {                                                                  \
        flag = 1; h11 = p1 / p2; h22 = x1 / y1;                               \
        T u = 1 + h11 * h22, t = d2 / u;                                      \
        d2 = d1 / u; d1 = t; x1 = y1 * u;                                     \
      }                                                                       \
      if (d1 != 0)                                                            \
        for (int it = 0; it < 256 && (d1 <= rgamsq || d1 >= gamsq); ++it) {   \
          if (flag == 0) { h11 = 1; h22 = 1; } else { h21 = -1; h12 = 1; }    \
          flag = -1;                                                          \
          if (d1 <= rgamsq) { d1 *= gamsq; x1 /= gam; h11 /= gam; h12 /= gam; } \
          else { d1 /= gamsq; x1 *= gam; h11 *= gam; h12 *= gam; }            \
        }                                                                     \
      if (d2 != 0)                                                            \
        for (int it = 0; it < 256 && (FABS(d2) <= rgamsq || FABS(d2) >= gamsq); ++it) { \
          if (flag == 0) { h11 = 1; h22 = 1; } else { h21 = -1; h12 = 1; }    \
          flag = -1;                                                          \
          if (FABS(d2) <= rgamsq) { d2 *= gamsq; h21 /= gam; h22 /= gam; }    \
          else { d2 /= gamsq; h21 *= gam; h22 *= gam; }                       \
        }                                                                     \
    }                                                                         \
    param[1] = param[2] = param[3] = param[4] = 0;                            \
    if (flag < 0) { param[1] = h11; param[2] = h21; param[3] = h12; param[4] = h22; } \
    else if (flag == 0) { param[2] = h21; param[3] = h12; }                   \
    else { param[1] = h11; param[4] = h22; }                                  \
    param[0] = flag;                                                          \
    v[0] = d1; v[1] = d2; v[2] = x1;                                          \
  }
void or_rotmg_exact(int dbl, double v[4], double param[5]) {
  if (dbl) OR_ROTMG(double, fabs)
  else OR_ROTMG(float, fabsf)
}

/* idamax.rs:43-159, icamax.rs:48-166, izamax.rs:33-163: first index of the
 * largest |x| (|re| + |im| summed in the element precision); NaN never wins;
 * n == 0 or incx == 0 -> 0. */
size_t or_iamax_exact(int kind, size_t n, const void* x, size_t incx) {
  if (n == 0 || incx == 0) return 0;
  double best = -INFINITY;
  size_t idx = 0;
  for (size_t i = 0; i < n; ++i) {
    double v;
    if (kind == 1) v = fabs(((const double*)x)[i * incx]);
    else if (kind == 2) v = (double)(fabsf(((const float*)x)[2 * i * incx]) + fabsf(((const float*)x)[2 * i * incx + 1]));
    else v = fabs(((const double*)x)[2 * i * incx]) + fabs(((const double*)x)[2 * i * incx + 1]);
    if (v > best) { best = v; idx = i; }
  }
  return idx;
}

/* ddot.rs:43-163, cdotu.rs / cdotc.rs / zdotu.rs / zdotc.rs (conj: sum
 * conj(x_i) y_i) in double-double; n == 0 -> 0. */
void or_dot_f64(int kind, int conj, size_t n, const void* x, size_t incx, const void* y, size_t incy,
                double out[2]) {
  dd re = {0, 0}, im = {0, 0};
  for (size_t i = 0; i < n; ++i) {
    double xr, xi, yr, yi;
    L1_LOAD(kind, x, i * incx, xr, xi);
    L1_LOAD(kind, y, i * incy, yr, yi);
    if (conj) xi = -xi;
    re = dd_add_prod(re, xr, yr);
    re = dd_add_prod(re, -xi, yi);
    im = dd_add_prod(im, xr, yi);
    im = dd_add_prod(im, xi, yr);
  }
  out[0] = dd_val(re);
  out[1] = dd_val(im);
}

/* sasum.rs:40-107, dasum.rs:41-110, scasum.rs:40-108, dzasum.rs:40-111:
 * sum of |re| + |im| in long double; n == 0 or incx == 0 -> 0. */
double or_asum_f64(int kind, size_t n, const void* x, size_t incx) {
  if (n == 0 || incx == 0) return 0.0;
  long double s = 0;
  for (size_t i = 0; i < n; ++i) {
    double r, m;
    L1_LOAD(kind, x, i * incx, r, m);
    s += fabsl((long double)r) + fabsl((long double)m);
  }
  return (double)s;
}

/* dnrm2.rs:45-152, scnrm2.rs:44-155, dznrm2.rs:43-156: ||x||_2 with the sum
 * of squares in long double (no overflow or underflow for double data);
 * n == 0 or incx == 0 -> 0. */
double or_nrm2_f64(int kind, size_t n, const void* x, size_t incx) {
  if (n == 0 || incx == 0) return 0.0;
  long double s = 0;
  for (size_t i = 0; i < n; ++i) {
    double r, m;
    L1_LOAD(kind, x, i * incx, r, m);
    s += (long double)r * r + (long double)m * m;
  }
  return (double)sqrtl(s);
}

/* ============================ level 2 ==================================== */

/* level2/sgemv_notranspose.rs:63-177, sgemv_transpose.rs:64-182:
 * empty matrix or (alpha == 0 && beta == 1) -> no-op; beta != 1 -> y *= beta
 * in fp32 (sscal); alpha == 0 -> done; x is scaled by alpha in fp32, then
 * y += op(A) xs.  Output in double: y_out = fl32(beta*y) + sum. */
void or_sgemv_f64(int trans, size_t m, size_t n, float alpha, const float* A, size_t lda,
                  const float* x, size_t incx, float beta, const float* y, size_t incy,
                  double* y_out) {
  const int t = trans != NOTRANS;
  const size_t ylen = t ? n : m, xlen = t ? m : n;
  for (size_t i = 0; i < ylen; ++i) y_out[i] = y[i * incy];
  if (m == 0 || n == 0) return;
  if (alpha == 0.0f && beta == 1.0f) return;
  if (beta != 1.0f)
    for (size_t i = 0; i < ylen; ++i) y_out[i] = (double)(y[i * incy] * beta);
  if (alpha == 0.0f) return;
  float* xs = (float*)malloc(sizeof(float) * (xlen ? xlen : 1));
  for (size_t j = 0; j < xlen; ++j) xs[j] = alpha * x[j * incx];
  for (size_t i = 0; i < ylen; ++i) {
    dd acc = {0.0, 0.0};
    for (size_t j = 0; j < xlen; ++j) {
      float a = t ? A[j + i * lda] : A[i + j * lda];
      acc = dd_add_prod(acc, a, xs[j]);
    }
    y_out[i] += dd_val(acc);
  }
  free(xs);
}

/* level2/dgemv_notranspose.rs, dgemv_transpose.rs: the sgemv order in
 * double -- empty matrix or (alpha == 0 && beta == 1) -> no-op; beta != 1 ->
 * y *= beta (dscal: a multiplication, so 0 * NaN stays NaN); alpha == 0 ->
 * done; xs = alpha * x; y += op(A) xs, summed in double-double. */
void or_dgemv_f64(int trans, size_t m, size_t n, double alpha, const double* A, size_t lda,
                  const double* x, size_t incx, double beta, const double* y, size_t incy,
                  double* y_out) {
  const int t = trans != NOTRANS;
  const size_t ylen = t ? n : m, xlen = t ? m : n;
  for (size_t i = 0; i < ylen; ++i) y_out[i] = y[i * incy];
  if (m == 0 || n == 0) return;
  if (alpha == 0.0 && beta == 1.0) return;
  if (beta != 1.0)
    for (size_t i = 0; i < ylen; ++i) y_out[i] = y[i * incy] * beta;
  if (alpha == 0.0) return;
  double* xs = (double*)malloc(sizeof(double) * (xlen ? xlen : 1));
  for (size_t j = 0; j < xlen; ++j) xs[j] = alpha * x[j * incx];
  for (size_t i = 0; i < ylen; ++i) {
    dd acc = {0.0, 0.0};
    for (size_t j = 0; j < xlen; ++j) acc = dd_add_prod(acc, t ? A[j + i * lda] : A[i + j * lda], xs[j]);
    y_out[i] += dd_val(acc);
  }
  free(xs);
}

/* level2/cgemv_*.rs and zgemv_*.rs (zgemv_notranspose.rs:76-101): empty or
 * (alpha == 0 && beta == 1) -> no-op; beta != 1 -> y *= beta in the element
 * precision, by csscal/zdscal when Im(beta) == 0 (both parts times Re(beta))
 * and cscal/zscal otherwise; alpha == 0 -> done; xs = alpha * x in the
 * element precision; y += op(A) xs with op N, T or C (conjugated A), summed
 * in double-double.  Interleaved (re, im); ld and inc in complex units. */
#define OR_CGEMV_BODY(R)                                                                     \
  const int t = trans != NOTRANS, cj = trans == CONJTRANS;                                   \
  const size_t ylen = t ? n : m, xlen = t ? m : n;                                           \
  for (size_t i = 0; i < ylen; ++i) {                                                        \
    y_out[2 * i] = y[2 * i * incy];                                                          \
    y_out[2 * i + 1] = y[2 * i * incy + 1];                                                  \
  }                                                                                          \
  if (m == 0 || n == 0) return;                                                              \
  if (alpha[0] == 0 && alpha[1] == 0 && beta[0] == 1 && beta[1] == 0) return;                \
  if (!(beta[0] == 1 && beta[1] == 0))                                                       \
    for (size_t i = 0; i < ylen; ++i) {                                                      \
      R yr = y[2 * i * incy], yi = y[2 * i * incy + 1];                                      \
      if (beta[1] == 0) { y_out[2 * i] = (R)(yr * beta[0]); y_out[2 * i + 1] = (R)(yi * beta[0]); } \
      else {                                                                                 \
        y_out[2 * i] = (R)(beta[0] * yr - beta[1] * yi);                                     \
        y_out[2 * i + 1] = (R)(beta[0] * yi + beta[1] * yr);                                 \
      }                                                                                      \
    }                                                                                        \
  if (alpha[0] == 0 && alpha[1] == 0) return;                                                \
  R* xs = (R*)malloc(sizeof(R) * 2 * (xlen ? xlen : 1));                                     \
  for (size_t j = 0; j < xlen; ++j) {                                                        \
    R xr = x[2 * j * incx], xi = x[2 * j * incx + 1];                                        \
    xs[2 * j] = alpha[0] * xr - alpha[1] * xi;                                               \
    xs[2 * j + 1] = alpha[0] * xi + alpha[1] * xr;                                           \
  }                                                                                          \
  for (size_t i = 0; i < ylen; ++i) {                                                        \
    dd re = {0.0, 0.0}, im = {0.0, 0.0};                                                     \
    for (size_t j = 0; j < xlen; ++j) {                                                      \
      size_t e = t ? j + i * lda : i + j * lda;                                              \
      double ar = A[2 * e], ai = cj ? -(double)A[2 * e + 1] : (double)A[2 * e + 1];          \
      re = dd_add_prod(re, ar, xs[2 * j]);                                                   \
      re = dd_add_prod(re, -ai, xs[2 * j + 1]);                                              \
      im = dd_add_prod(im, ar, xs[2 * j + 1]);                                               \
      im = dd_add_prod(im, ai, xs[2 * j]);                                                   \
    }                                                                                        \
    y_out[2 * i] += dd_val(re);                                                              \
    y_out[2 * i + 1] += dd_val(im);                                                          \
  }                                                                                          \
  free(xs);

void or_cgemv_f64(int trans, size_t m, size_t n, const float alpha[2], const float* A, size_t lda,
                  const float* x, size_t incx, const float beta[2], const float* y, size_t incy,
                  double* y_out) {
  OR_CGEMV_BODY(float)
}

void or_zgemv_f64(int trans, size_t m, size_t n, const double alpha[2], const double* A, size_t lda,
                  const double* x, size_t incx, const double beta[2], const double* y, size_t incy,
                  double* y_out) {
  OR_CGEMV_BODY(double)
}

/* level2/ssymv.rs:99-394: n == 0 or (alpha == 0 && beta == 1) -> no-op;
 * x scaled by alpha in fp32; beta == 0 -> y = 0 (fill), beta != 1 -> y *= beta;
 * only the `uplo` triangle of A is referenced. */
void or_ssymv_f64(int uplo, size_t n, float alpha, const float* A, size_t lda, const float* x,
                  size_t incx, float beta, const float* y, size_t incy, double* y_out) {
  for (size_t i = 0; i < n; ++i) y_out[i] = y[i * incy];
  if (n == 0) return;
  if (alpha == 0.0f && beta == 1.0f) return;
  float* xs = (float*)malloc(sizeof(float) * n);
  for (size_t j = 0; j < n; ++j) xs[j] = alpha * x[j * incx];
  for (size_t i = 0; i < n; ++i) {
    float yb = beta == 0.0f ? 0.0f : (beta != 1.0f ? y[i * incy] * beta : y[i * incy]);
    dd acc = {0.0, 0.0};
    for (size_t j = 0; j < n; ++j) {
      int stored = uplo == UPPER ? (i <= j) : (i >= j);
      float a = stored ? A[i + j * lda] : A[j + i * lda];
      acc = dd_add_prod(acc, a, xs[j]);
    }
    y_out[i] = (double)yb + dd_val(acc);
  }
  free(xs);
}

/* level2/chemv.rs:96-447: as ssymv for a Hermitian matrix stored in the
 * `uplo` triangle; the other triangle is conj of the stored one and only
 * Re(a_jj) is used on the diagonal (chemv.rs:179-182).  Complex scalars as
 * (re, im); alpha*x and beta*y rounded in fp32 as the reference does. */
void or_chemv_f64(int uplo, size_t n, const float alpha[2], const float* A, size_t lda,
                  const float* x, size_t incx, const float beta[2], const float* y, size_t incy,
                  double* y_out) {
  for (size_t i = 0; i < n; ++i) {
    y_out[2 * i] = y[2 * i * incy];
    y_out[2 * i + 1] = y[2 * i * incy + 1];
  }
  if (n == 0) return;
  if (alpha[0] == 0.0f && alpha[1] == 0.0f && beta[0] == 1.0f && beta[1] == 0.0f) return;
  float* xs = (float*)malloc(sizeof(float) * 2 * n);
  for (size_t j = 0; j < n; ++j) {
    float xr = x[2 * j * incx], xi = x[2 * j * incx + 1];
    xs[2 * j] = alpha[0] * xr - alpha[1] * xi;
    xs[2 * j + 1] = alpha[0] * xi + alpha[1] * xr;
  }
  for (size_t i = 0; i < n; ++i) {
    float yr = y[2 * i * incy], yi = y[2 * i * incy + 1], br, bi;
    if (beta[0] == 0.0f && beta[1] == 0.0f) { br = 0.0f; bi = 0.0f; }
    else if (beta[0] == 1.0f && beta[1] == 0.0f) { br = yr; bi = yi; }
    else { br = yr * beta[0] - yi * beta[1]; bi = yr * beta[1] + yi * beta[0]; }
    dd re = {0.0, 0.0}, im = {0.0, 0.0};
    for (size_t j = 0; j < n; ++j) {
      double ar, ai;
      if (i == j) { ar = A[2 * (i + j * lda)]; ai = 0.0; }
      else {
        int stored = uplo == UPPER ? (i < j) : (i > j);
        if (stored) { ar = A[2 * (i + j * lda)]; ai = A[2 * (i + j * lda) + 1]; }
        else { ar = A[2 * (j + i * lda)]; ai = -A[2 * (j + i * lda) + 1]; }
      }
      re = dd_add_prod(re, ar, xs[2 * j]);
      re = dd_add_prod(re, -ai, xs[2 * j + 1]);
      im = dd_add_prod(im, ar, xs[2 * j + 1]);
      im = dd_add_prod(im, ai, xs[2 * j]);
    }
    y_out[2 * i] = (double)br + dd_val(re);
    y_out[2 * i + 1] = (double)bi + dd_val(im);
  }
  free(xs);
}

static inline double tri_elem(int uplo, int diag, const float* A, size_t lda, size_t i, size_t j) {
  if (i == j) return diag == UNIT ? 1.0 : (double)A[i + j * lda];
  if (uplo == UPPER ? (i < j) : (i > j)) return A[i + j * lda];
  return 0.0;
}

/* level2/strsv.rs:60-74 -> strlsv.rs / strusv.rs: solve op(A) x = b in place
 * (op = A or A^T; ConjugateTranspose == Transpose), in double. */
void or_strsv_f64(int uplo, int trans, int diag, size_t n, const float* A, size_t lda,
                  const float* b, size_t incx, double* x_out) {
  const int t = trans != NOTRANS;
  /* op(A) is lower when (uplo==LOWER) xor t */
  const int lower = (uplo == LOWER) != t;
  for (size_t i = 0; i < n; ++i) x_out[i] = b[i * incx];
  if (lower) {
    for (size_t i = 0; i < n; ++i) {
      dd acc = {x_out[i], 0.0};
      for (size_t k = 0; k < i; ++k) {
        double a = t ? tri_elem(uplo, diag, A, lda, k, i) : tri_elem(uplo, diag, A, lda, i, k);
        acc = dd_add_prod(acc, -a, x_out[k]);
      }
      double d = tri_elem(uplo, diag, A, lda, i, i);
      x_out[i] = dd_val(acc) / d;
    }
  } else {
    for (size_t ii = n; ii-- > 0;) {
      dd acc = {x_out[ii], 0.0};
      for (size_t k = ii + 1; k < n; ++k) {
        double a = t ? tri_elem(uplo, diag, A, lda, k, ii) : tri_elem(uplo, diag, A, lda, ii, k);
        acc = dd_add_prod(acc, -a, x_out[k]);
      }
      double d = tri_elem(uplo, diag, A, lda, ii, ii);
      x_out[ii] = dd_val(acc) / d;
    }
  }
}

/* level2/strmv.rs:59-73 -> strlmv.rs / strumv.rs: x <- op(A) x, in double. */
void or_strmv_f64(int uplo, int trans, int diag, size_t n, const float* A, size_t lda,
                  const float* x, size_t incx, double* x_out) {
  const int t = trans != NOTRANS;
  for (size_t i = 0; i < n; ++i) {
    dd acc = {0.0, 0.0};
    for (size_t k = 0; k < n; ++k) {
      double a = t ? tri_elem(uplo, diag, A, lda, k, i) : tri_elem(uplo, diag, A, lda, i, k);
      if (a != 0.0) acc = dd_add_prod(acc, a, x[k * incx]);
    }
    x_out[i] = dd_val(acc);
  }
}

/* level2/dsymv.rs:99-210: the ssymv order in double -- n == 0 or
 * (alpha == 0 && beta == 1) -> no-op; xs = alpha * x; beta == 0 -> y = 0
 * (fill), beta != 1 -> y *= beta; only the `uplo` triangle of A is read. */
void or_dsymv_f64(int uplo, size_t n, double alpha, const double* A, size_t lda, const double* x,
                  size_t incx, double beta, const double* y, size_t incy, double* y_out) {
  for (size_t i = 0; i < n; ++i) y_out[i] = y[i * incy];
  if (n == 0) return;
  if (alpha == 0.0 && beta == 1.0) return;
  double* xs = (double*)malloc(sizeof(double) * n);
  for (size_t j = 0; j < n; ++j) xs[j] = alpha * x[j * incx];
  for (size_t i = 0; i < n; ++i) {
    double yb = beta == 0.0 ? 0.0 : (beta != 1.0 ? y[i * incy] * beta : y[i * incy]);
    dd acc = {0.0, 0.0};
    for (size_t j = 0; j < n; ++j) {
      int stored = uplo == UPPER ? (i <= j) : (i >= j);
      acc = dd_add_prod(acc, stored ? A[i + j * lda] : A[j + i * lda], xs[j]);
    }
    y_out[i] = yb + dd_val(acc);
  }
  free(xs);
}

/* level2/zhemv.rs:96-230: the chemv order in double -- Re of the diagonal
 * only; the unstored triangle is the conjugate of the stored one; beta == 0
 * -> y = 0, beta != 1 -> y *= beta (zscal). */
void or_zhemv_f64(int uplo, size_t n, const double alpha[2], const double* A, size_t lda,
                  const double* x, size_t incx, const double beta[2], const double* y, size_t incy,
                  double* y_out) {
  for (size_t i = 0; i < n; ++i) {
    y_out[2 * i] = y[2 * i * incy];
    y_out[2 * i + 1] = y[2 * i * incy + 1];
  }
  if (n == 0) return;
  if (alpha[0] == 0.0 && alpha[1] == 0.0 && beta[0] == 1.0 && beta[1] == 0.0) return;
  double* xs = (double*)malloc(sizeof(double) * 2 * n);
  for (size_t j = 0; j < n; ++j) {
    double xr = x[2 * j * incx], xi = x[2 * j * incx + 1];
    xs[2 * j] = alpha[0] * xr - alpha[1] * xi;
    xs[2 * j + 1] = alpha[0] * xi + alpha[1] * xr;
  }
  for (size_t i = 0; i < n; ++i) {
    double yr = y[2 * i * incy], yi = y[2 * i * incy + 1], br, bi;
    if (beta[0] == 0.0 && beta[1] == 0.0) { br = 0.0; bi = 0.0; }
    else if (beta[0] == 1.0 && beta[1] == 0.0) { br = yr; bi = yi; }
    else { br = yr * beta[0] - yi * beta[1]; bi = yr * beta[1] + yi * beta[0]; }
    dd re = {0.0, 0.0}, im = {0.0, 0.0};
    for (size_t j = 0; j < n; ++j) {
      double ar, ai;
      if (i == j) { ar = A[2 * (i + j * lda)]; ai = 0.0; }
      else if (uplo == UPPER ? (i < j) : (i > j)) { ar = A[2 * (i + j * lda)]; ai = A[2 * (i + j * lda) + 1]; }
      else { ar = A[2 * (j + i * lda)]; ai = -A[2 * (j + i * lda) + 1]; }
      re = dd_add_prod(re, ar, xs[2 * j]);
      re = dd_add_prod(re, -ai, xs[2 * j + 1]);
      im = dd_add_prod(im, ar, xs[2 * j + 1]);
      im = dd_add_prod(im, ai, xs[2 * j]);
    }
    y_out[2 * i] = br + dd_val(re);
    y_out[2 * i + 1] = bi + dd_val(im);
  }
  free(xs);
}

/* level2/dtrmv.rs (dtrlmv.rs / dtrumv.rs): x <- op(A) x, A triangular in the
 * `uplo` half, unit diagonal = 1; ConjugateTranspose == Transpose. */
void or_dtrmv_f64(int uplo, int trans, int diag, size_t n, const double* A, size_t lda,
                  const double* x, size_t incx, double* x_out) {
  const int t = trans != NOTRANS;
  for (size_t i = 0; i < n; ++i) {
    dd acc = {0.0, 0.0};
    for (size_t k = 0; k < n; ++k) {
      size_t r = t ? k : i, c = t ? i : k;  /* element (r, c) of A */
      double a;
      if (r == c) a = diag == UNIT ? 1.0 : A[r + c * lda];
      else if (uplo == UPPER ? (r < c) : (r > c)) a = A[r + c * lda];
      else continue;
      acc = dd_add_prod(acc, a, x[k * incx]);
    }
    x_out[i] = dd_val(acc);
  }
}

/* level2/ctrmv.rs:58-72 / ztrmv.rs (c/z trlmv, trumv): x <- op(A) x with op
 * N, T or C (conjugated elements), interleaved complex, unit diagonal = 1. */
#define OR_CTRMV_BODY                                                                        \
  const int t = trans != NOTRANS, cj = trans == CONJTRANS;                                   \
  for (size_t i = 0; i < n; ++i) {                                                           \
    dd re = {0.0, 0.0}, im = {0.0, 0.0};                                                     \
    for (size_t k = 0; k < n; ++k) {                                                         \
      size_t r = t ? k : i, c = t ? i : k;                                                   \
      double ar, ai;                                                                         \
      if (r == c && diag == UNIT) { ar = 1.0; ai = 0.0; }                                    \
      else if (r == c || (uplo == UPPER ? (r < c) : (r > c))) {                             \
        ar = A[2 * (r + c * lda)];                                                           \
        ai = cj ? -(double)A[2 * (r + c * lda) + 1] : (double)A[2 * (r + c * lda) + 1];     \
      } else continue;                                                                       \
      double xr = x[2 * k * incx], xi = x[2 * k * incx + 1];                                 \
      re = dd_add_prod(re, ar, xr);                                                          \
      re = dd_add_prod(re, -ai, xi);                                                         \
      im = dd_add_prod(im, ar, xi);                                                          \
      im = dd_add_prod(im, ai, xr);                                                          \
    }                                                                                        \
    x_out[2 * i] = dd_val(re);                                                               \
    x_out[2 * i + 1] = dd_val(im);                                                           \
  }

void or_ctrmv_f64(int uplo, int trans, int diag, size_t n, const float* A, size_t lda,
                  const float* x, size_t incx, double* x_out) {
  OR_CTRMV_BODY
}
void or_ztrmv_f64(int uplo, int trans, int diag, size_t n, const double* A, size_t lda,
                  const double* x, size_t incx, double* x_out) {
  OR_CTRMV_BODY
}

/* level2/dger.rs: per column j, coeff = alpha * y_j (a zero coefficient
 * leaves the column untouched); A_ij += x_i * coeff with one rounding (the
 * reference's daxpy / mul_add).  A is updated in place. */
void or_dger_f64(size_t m, size_t n, double alpha, const double* x, size_t incx, const double* y,
                 size_t incy, double* A, size_t lda) {
  if (m == 0 || n == 0 || alpha == 0.0) return;
  for (size_t j = 0; j < n; ++j) {
    double c = alpha * y[j * incy];
    if (c == 0.0) continue;
    for (size_t i = 0; i < m; ++i) A[i + j * lda] = fma(x[i * incx], c, A[i + j * lda]);
  }
}

/* Complex rank updates, interleaved (re, im), A (double, interleaved) updated
 * in place; coefficients are formed in the element precision R as the
 * reference forms them, the update A_ij += x_i * c in double:
 *   cgeru/zgeru (cj = 0): c = alpha * y_j;  cgerc/zgerc (cj = 1): alpha * conj(y_j)
 *   (cgeru.rs / cgerc.rs: a zero coefficient leaves the column untouched). */
#define OR_CGER(NAME, R)                                                                        \
  void NAME(int cj, size_t m, size_t n, const R alpha[2], const R* x, size_t incx, const R* y,   \
            size_t incy, double* A, size_t lda) {                                               \
    if (m == 0 || n == 0 || (alpha[0] == 0 && alpha[1] == 0)) return;                           \
    for (size_t j = 0; j < n; ++j) {                                                            \
      R yr = y[2 * j * incy], yi = cj ? -y[2 * j * incy + 1] : y[2 * j * incy + 1];             \
      R cr = alpha[0] * yr - alpha[1] * yi, ci = alpha[0] * yi + alpha[1] * yr;                 \
      if (cr == 0 && ci == 0) continue;                                                         \
      for (size_t i = 0; i < m; ++i) {                                                          \
        double xr = x[2 * i * incx], xi = x[2 * i * incx + 1];                                  \
        A[2 * (i + j * lda)] += xr * (double)cr - xi * (double)ci;                              \
        A[2 * (i + j * lda) + 1] += xr * (double)ci + xi * (double)cr;                          \
      }                                                                                         \
    }                                                                                           \
  }
OR_CGER(or_cger_f64, float)
OR_CGER(or_zger_f64, double)

/* level2/dsyr.rs / dsyr2.rs: the `uplo` triangle of column j gets
 * x_i * (alpha x_j)  (syr), or  x_i * (alpha y_j) + y_i * (alpha x_j)  (syr2),
 * each term skipped when its coefficient is zero; one rounding per term. */
void or_dsyr_f64(int uplo, size_t n, double alpha, const double* x, size_t incx, const double* y,
                 size_t incy, int two, double* A, size_t lda) {
  if (n == 0 || alpha == 0.0) return;
  for (size_t j = 0; j < n; ++j) {
    size_t lo = uplo == UPPER ? 0 : j, hi = uplo == UPPER ? j + 1 : n;
    double c1 = two ? alpha * y[j * incy] : alpha * x[j * incx];
    double c2 = two ? alpha * x[j * incx] : 0.0;
    for (size_t i = lo; i < hi; ++i) {
      double a = A[i + j * lda];
      if (c1 != 0.0) a = fma(x[i * incx], c1, a);
      if (c2 != 0.0) a = fma(y[i * incy], c2, a);
      A[i + j * lda] = a;
    }
  }
}

/* level2/cher.rs, zher.rs (two = 0; real alpha): c = alpha * conj(x_j); the
 * column's triangle gets x_i * c and, when updated, a real diagonal.
 * cher2.rs, zher2.rs (two = 1): c1 = alpha * conj(y_j) on x,
 * c2 = conj(alpha) * conj(x_j) on y, each skipped when zero; the diagonal is
 * made real for every column. */
#define OR_CHER(NAME, R)                                                                        \
  void NAME(int uplo, size_t n, const R alpha[2], const R* x, size_t incx, const R* y,          \
            size_t incy, int two, double* A, size_t lda) {                                      \
    if (n == 0 || (alpha[0] == 0 && alpha[1] == 0)) return;                                     \
    for (size_t j = 0; j < n; ++j) {                                                            \
      size_t lo = uplo == UPPER ? 0 : j, hi = uplo == UPPER ? j + 1 : n;                        \
      R c1r, c1i, c2r = 0, c2i = 0;                                                             \
      R xjr = x[2 * j * incx], xji = x[2 * j * incx + 1];                                       \
      if (!two) { c1r = alpha[0] * xjr; c1i = -alpha[0] * xji; }                                \
      else {                                                                                    \
        R yjr = y[2 * j * incy], yji = y[2 * j * incy + 1];                                     \
        c1r = alpha[0] * yjr + alpha[1] * yji; c1i = -alpha[0] * yji + alpha[1] * yjr;          \
        c2r = alpha[0] * xjr - alpha[1] * xji; c2i = -alpha[0] * xji - alpha[1] * xjr;          \
      }                                                                                         \
      int u1 = c1r != 0 || c1i != 0, u2 = c2r != 0 || c2i != 0;                                \
      if (!u1 && !u2 && !two) continue;                                                         \
      for (size_t i = lo; i < hi; ++i) {                                                        \
        double* a = A + 2 * (i + j * lda);                                                      \
        if (u1) {                                                                               \
          double xr = x[2 * i * incx], xi = x[2 * i * incx + 1];                                \
          a[0] += xr * (double)c1r - xi * (double)c1i;                                          \
          a[1] += xr * (double)c1i + xi * (double)c1r;                                          \
        }                                                                                       \
        if (u2) {                                                                               \
          double yr = y[2 * i * incy], yi = y[2 * i * incy + 1];                                \
          a[0] += yr * (double)c2r - yi * (double)c2i;                                          \
          a[1] += yr * (double)c2i + yi * (double)c2r;                                          \
        }                                                                                       \
        if (i == j) a[1] = 0.0;                                                                 \
      }                                                                                         \
    }                                                                                           \
  }
OR_CHER(or_cher_f64, float)
OR_CHER(or_zher_f64, double)

/* level2/dtrsv.rs, ctrsv.rs, ztrsv.rs (the *trlsv / *trusv files): solve
 * op(A) x = b by substitution in long double (64-bit significand), op N, T
 * or C, unit diagonal = 1; only the `uplo` triangle is read.  Complex data
 * interleaved.  Output in double. */
#define OR_TRSV_BODY(CPLX)                                                                      \
  const int t = trans != NOTRANS, cj = trans == CONJTRANS;                                      \
  const int lower_eff = (uplo == LOWER) != t;                                                   \
  long double* vr = (long double*)malloc(sizeof(long double) * (n ? n : 1));                    \
  long double* vi = (long double*)malloc(sizeof(long double) * (n ? n : 1));                    \
  for (size_t i = 0; i < n; ++i) {                                                              \
    vr[i] = CPLX ? x[2 * i * incx] : x[i * incx];                                               \
    vi[i] = CPLX ? x[2 * i * incx + 1] : 0;                                                     \
  }                                                                                             \
  for (size_t s = 0; s < n; ++s) {                                                              \
    size_t i = lower_eff ? s : n - 1 - s;                                                       \
    long double sr = vr[i], si = vi[i];                                                         \
    for (size_t s2 = 0; s2 < s; ++s2) {                                                         \
      size_t k = lower_eff ? s2 : n - 1 - s2;                                                   \
      size_t e = t ? k + i * lda : i + k * lda;                                                 \
      long double ar = CPLX ? A[2 * e] : A[e];                                                  \
      long double ai = CPLX ? (cj ? -(long double)A[2 * e + 1] : (long double)A[2 * e + 1]) : 0; \
      sr -= ar * vr[k] - ai * vi[k];                                                            \
      si -= ar * vi[k] + ai * vr[k];                                                            \
    }                                                                                           \
    if (diag != UNIT) {                                                                         \
      size_t e = i + i * lda;                                                                   \
      long double dr = CPLX ? A[2 * e] : A[e];                                                  \
      long double di = CPLX ? (cj ? -(long double)A[2 * e + 1] : (long double)A[2 * e + 1]) : 0; \
      long double den = dr * dr + di * di;                                                      \
      long double qr = (sr * dr + si * di) / den, qi = (si * dr - sr * di) / den;               \
      sr = qr; si = qi;                                                                         \
    }                                                                                           \
    vr[i] = sr; vi[i] = si;                                                                     \
  }                                                                                             \
  for (size_t i = 0; i < n; ++i) {                                                              \
    if (CPLX) { x_out[2 * i] = (double)vr[i]; x_out[2 * i + 1] = (double)vi[i]; }               \
    else x_out[i] = (double)vr[i];                                                              \
  }                                                                                             \
  free(vr); free(vi);

void or_dtrsv_f64(int uplo, int trans, int diag, size_t n, const double* A, size_t lda,
                  const double* x, size_t incx, double* x_out) {
  OR_TRSV_BODY(0)
}
void or_ctrsv_f64(int uplo, int trans, int diag, size_t n, const float* A, size_t lda,
                  const float* x, size_t incx, double* x_out) {
  OR_TRSV_BODY(1)
}
void or_ztrsv_f64(int uplo, int trans, int diag, size_t n, const double* A, size_t lda,
                  const double* x, size_t incx, double* x_out) {
  OR_TRSV_BODY(1)
}

/* level2/sger.rs:68-132 (bit-exact): unit strides go through saxpy per
 * column (fused first m - m%8 rows, `+= a*x` for the rest), strided through
 * mul_add; a column whose coefficient alpha*y_j is 0 is skipped. */
void or_sger_exact(size_t m, size_t n, float alpha, const float* x, size_t incx, const float* y,
                   size_t incy, float* A, size_t lda) {
  if (m == 0 || n == 0 || alpha == 0.0f) return;
  for (size_t j = 0; j < n; ++j) {
    float coeff = alpha * y[j * incy];
    if (coeff == 0.0f) continue;
    float* col = A + j * lda;
    if (incx == 1 && incy == 1) or_saxpy_exact(m, coeff, x, 1, col, 1);
    else
      for (size_t i = 0; i < m; ++i) col[i] = fmaf(x[i * incx], coeff, col[i]);
  }
}

/* level2/ssyr.rs:63-181 (bit-exact). */
void or_ssyr_exact(int uplo, size_t n, float alpha, const float* x, size_t incx, float* A,
                   size_t lda) {
  if (n == 0 || alpha == 0.0f) return;
  for (size_t j = 0; j < n; ++j) {
    float aj = alpha * x[j * incx];
    if (aj == 0.0f) continue;
    size_t lo = uplo == UPPER ? 0 : j, hi = uplo == UPPER ? j + 1 : n;
    if (incx == 1) or_saxpy_exact(hi - lo, aj, x + lo, 1, A + j * lda + lo, 1);
    else
      for (size_t i = lo; i < hi; ++i) A[i + j * lda] = fmaf(x[i * incx], aj, A[i + j * lda]);
  }
}

/* level2/ssyr2.rs:59-197 (bit-exact). */
void or_ssyr2_exact(int uplo, size_t n, float alpha, const float* x, size_t incx, const float* y,
                    size_t incy, float* A, size_t lda) {
  if (n == 0 || alpha == 0.0f) return;
  for (size_t j = 0; j < n; ++j) {
    float ay = alpha * y[j * incy], ax = alpha * x[j * incx];
    size_t lo = uplo == UPPER ? 0 : j, hi = uplo == UPPER ? j + 1 : n;
    float* col = A + j * lda;
    if (incx == 1 && incy == 1) {
      if (ay != 0.0f) or_saxpy_exact(hi - lo, ay, x + lo, 1, col + lo, 1);
      if (ax != 0.0f) or_saxpy_exact(hi - lo, ax, y + lo, 1, col + lo, 1);
    } else {
      if (ay == 0.0f && ax == 0.0f) continue;
      for (size_t i = lo; i < hi; ++i) {
        float a = fmaf(x[i * incx], ay, col[i]);
        col[i] = fmaf(y[i * incy], ax, a);
      }
    }
  }
}

/* ============================ level 3 ==================================== */

/* level3/sgemm.rs:106-130 / dgemm.rs:107 / cgemm.rs:127-157 / zgemm.rs:123
 * evaluated on selected entries (rows[s], cols[s]) of C, in double-double:
 * C_ij <- alpha * sum_l op(A)_il op(B)_lj + beta * C_ij, with
 * beta == 0 -> C not read (f32_edge.rs:37-58) and alpha == 0 or k == 0 ->
 * scale only (sgemm_nn.rs:29-45).  `absval[s]` receives
 * |alpha| * sum_l |op(A)_il||op(B)_lj| + |beta||C_ij| for component-wise
 * error bounds.  `cplx` selects interleaved complex storage (ld in complex
 * units); `dbl` selects double inputs.  Results are written as (re, im)
 * pairs in out[2*s] (im = 0 for real). */
void or_gemm_sample(int dbl, int cplx, int op_a, int op_b, size_t m, size_t n, size_t k,
                    const double alpha[2], const void* A, size_t lda, const void* B, size_t ldb,
                    const double beta[2], const void* C, size_t ldc, size_t count,
                    const int64_t* rows, const int64_t* cols, double* out, double* absval) {
  (void)m; (void)n;
  const int w = cplx ? 2 : 1;
#define LD(P, idx) (dbl ? ((const double*)(P))[idx] : (double)((const float*)(P))[idx])
  for (size_t s = 0; s < count; ++s) {
    size_t i = (size_t)rows[s], j = (size_t)cols[s];
    dd re = {0.0, 0.0}, im = {0.0, 0.0};
    double asum = 0.0;
    int scale_only = (alpha[0] == 0.0 && alpha[1] == 0.0) || k == 0;
    if (!scale_only) {
      for (size_t l = 0; l < k; ++l) {
        size_t ia = op_a == NOTRANS ? i + l * lda : l + i * lda;
        size_t ib = op_b == NOTRANS ? l + j * ldb : j + l * ldb;
        double ar = LD(A, w * ia), ai = cplx ? LD(A, w * ia + 1) : 0.0;
        double br = LD(B, w * ib), bi = cplx ? LD(B, w * ib + 1) : 0.0;
        if (cplx && op_a == CONJTRANS) ai = -ai;
        if (cplx && op_b == CONJTRANS) bi = -bi;
        re = dd_add_prod(re, ar, br);
        asum += fabs(ar) * fabs(br);
        if (cplx) {
          re = dd_add_prod(re, -ai, bi);
          im = dd_add_prod(im, ar, bi);
          im = dd_add_prod(im, ai, br);
          asum += fabs(ai) * fabs(bi) + fabs(ar) * fabs(bi) + fabs(ai) * fabs(br);
        }
      }
    }
    double pr = dd_val(re), pi = dd_val(im);
    double cr = 0.0, ci = 0.0;
    int beta0 = beta[0] == 0.0 && beta[1] == 0.0;
    if (!beta0) {
      cr = LD(C, w * (i + j * ldc));
      ci = cplx ? LD(C, w * (i + j * ldc) + 1) : 0.0;
    }
    double rr = alpha[0] * pr - alpha[1] * pi + beta[0] * cr - beta[1] * ci;
    double ri = alpha[0] * pi + alpha[1] * pr + beta[0] * ci + beta[1] * cr;
    if (scale_only) {
      rr = beta[0] * cr - beta[1] * ci;
      ri = beta[0] * ci + beta[1] * cr;
    }
    out[2 * s] = rr;
    out[2 * s + 1] = cplx ? ri : 0.0;
    if (absval)
      absval[s] = hypot(alpha[0], alpha[1]) * (scale_only ? 0.0 : asum) +
                  hypot(beta[0], beta[1]) * hypot(cr, ci);
  }
#undef LD
}

/* ===================== CORAL CPU algorithm restatements =================== */

/* level3/sgemm_nn.rs:10-99 with f32_packers.rs (MR x NR = 8 x 12 register
 * tile, MC/NC/KC = 384/576/256 from sgemm.rs:92-94) and the microkernel's
 * rank-1 update order (microkernel/f32_mrxnr.rs:46-95): NN only, fp32, with
 * the NEON 4-wide FMAs restated as AVX2 8-wide FMAs (the host is x86-64). */
#define P_MR 8
#define P_NR 12
#define P_MC 384
#define P_NC 576
#define P_KC 256

static void port_pack_a(size_t mc, size_t kc, const float* a, size_t lda, float* buf) {
  for (size_t i0 = 0; i0 < mc; i0 += P_MR) {
    size_t mr = mc - i0 < P_MR ? mc - i0 : P_MR;
    for (size_t l = 0; l < kc; ++l)
      for (size_t r = 0; r < P_MR; ++r) *buf++ = r < mr ? a[(i0 + r) + l * lda] : 0.0f;
  }
}

static void port_pack_b(size_t kc, size_t nc, const float* b, size_t ldb, float* buf) {
  for (size_t j0 = 0; j0 < nc; j0 += P_NR) {
    size_t nr = nc - j0 < P_NR ? nc - j0 : P_NR;
    for (size_t l = 0; l < kc; ++l)
      for (size_t c = 0; c < P_NR; ++c) *buf++ = c < nr ? b[l + (j0 + c) * ldb] : 0.0f;
  }
}

void port_sgemm_nn(size_t m, size_t n, size_t k, float alpha, const float* a, size_t lda,
                   const float* b, size_t ldb, float beta, float* c, size_t ldc) {
  if (alpha == 0.0f || k == 0) {
    for (size_t j = 0; j < n; ++j)
      for (size_t i = 0; i < m; ++i)
        c[i + j * ldc] = beta == 0.0f ? 0.0f : (beta != 1.0f ? c[i + j * ldc] * beta : c[i + j * ldc]);
    return;
  }
  float* abuf = (float*)aligned_alloc(64, sizeof(float) * (P_MC + P_MR) * P_KC);
  float* bbuf = (float*)aligned_alloc(64, sizeof(float) * (P_NC + P_NR) * P_KC);
  for (size_t j0 = 0; j0 < n; j0 += P_NC) {
    size_t nc = n - j0 < P_NC ? n - j0 : P_NC;
    for (size_t l0 = 0; l0 < k; l0 += P_KC) {
      size_t kc = k - l0 < P_KC ? k - l0 : P_KC;
      port_pack_b(kc, nc, b + l0 + j0 * ldb, ldb, bbuf);
      float bp = l0 == 0 ? beta : 1.0f;
      for (size_t i0 = 0; i0 < m; i0 += P_MC) {
        size_t mc = m - i0 < P_MC ? m - i0 : P_MC;
        port_pack_a(mc, kc, a + i0 + l0 * lda, lda, abuf);
        for (size_t jr = 0; jr < nc; jr += P_NR) {
          size_t nr = nc - jr < P_NR ? nc - jr : P_NR;
          const float* bpan = bbuf + (jr / P_NR) * P_NR * kc;
          for (size_t ir = 0; ir < mc; ir += P_MR) {
            size_t mr = mc - ir < P_MR ? mc - ir : P_MR;
            const float* apan = abuf + (ir / P_MR) * P_MR * kc;
            /* 8 x 12 register tile: the 8 rows of one ymm per column, 12
             * accumulators, one broadcast FMA per (k, column) -- the x86
             * counterpart of the NEON vfmaq_laneq rank-1 update
             * (microkernel/f32_mrxnr.rs:46-95). */
            float acc[P_NR][P_MR];
            __m256 c0 = _mm256_setzero_ps(), c1 = c0, c2 = c0, c3 = c0, c4 = c0, c5 = c0;
            __m256 c6 = c0, c7 = c0, c8 = c0, c9 = c0, c10 = c0, c11 = c0;
            for (size_t l = 0; l < kc; ++l) {
              const __m256 av = _mm256_loadu_ps(apan + l * P_MR);
              const float* bv = bpan + l * P_NR;
              c0 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 0), c0);
              c1 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 1), c1);
              c2 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 2), c2);
              c3 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 3), c3);
              c4 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 4), c4);
              c5 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 5), c5);
              c6 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 6), c6);
              c7 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 7), c7);
              c8 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 8), c8);
              c9 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 9), c9);
              c10 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 10), c10);
              c11 = _mm256_fmadd_ps(av, _mm256_broadcast_ss(bv + 11), c11);
            }
            _mm256_storeu_ps(acc[0], c0); _mm256_storeu_ps(acc[1], c1);
            _mm256_storeu_ps(acc[2], c2); _mm256_storeu_ps(acc[3], c3);
            _mm256_storeu_ps(acc[4], c4); _mm256_storeu_ps(acc[5], c5);
            _mm256_storeu_ps(acc[6], c6); _mm256_storeu_ps(acc[7], c7);
            _mm256_storeu_ps(acc[8], c8); _mm256_storeu_ps(acc[9], c9);
            _mm256_storeu_ps(acc[10], c10); _mm256_storeu_ps(acc[11], c11);
            for (size_t cc = 0; cc < nr; ++cc) {
              float* col = c + (i0 + ir) + (j0 + jr + cc) * ldc;
              for (size_t r = 0; r < mr; ++r) {
                if (bp == 0.0f) col[r] = alpha * acc[cc][r];
                else if (bp == 1.0f) col[r] += alpha * acc[cc][r];
                else col[r] = bp * col[r] + alpha * acc[cc][r];
              }
            }
          }
        }
      }
    }
  }
  free(abuf);
  free(bbuf);
}

/* level1_special/saxpyf.rs:59-499 as used by sgemv_notranspose.rs:108-115
 * (lda == m fast path): y *= beta, xs = alpha*x, then y += A xs with 8-column
 * blocks, fp32 FMA. */
void port_sgemv_n(size_t m, size_t n, float alpha, const float* A, size_t lda, const float* x,
                  float beta, float* y) {
  if (m == 0 || n == 0 || (alpha == 0.0f && beta == 1.0f)) return;
  if (beta != 1.0f)
    for (size_t i = 0; i < m; ++i) y[i] = y[i] * beta;
  if (alpha == 0.0f) return;
  float* xs = (float*)malloc(sizeof(float) * n);
  for (size_t j = 0; j < n; ++j) xs[j] = alpha * x[j];
  size_t j = 0;
  for (; j + 8 <= n; j += 8) {
    const float* c0 = A + j * lda;
    for (size_t i = 0; i < m; ++i) {
      float acc = y[i];
      for (int q = 0; q < 8; ++q) acc = fmaf(c0[i + q * lda], xs[j + q], acc);
      y[i] = acc;
    }
  }
  for (; j < n; ++j)
    for (size_t i = 0; i < m; ++i) y[i] = fmaf(A[i + j * lda], xs[j], y[i]);
  free(xs);
}

/* level1_special/sdotf.rs:59-289 as used by sgemv_transpose.rs (lda == m):
 * y_j = beta*y_j + dot(A[:, j], alpha*x), 8 fp32 lane accumulators. */
void port_sgemv_t(size_t m, size_t n, float alpha, const float* A, size_t lda, const float* x,
                  float beta, float* y) {
  if (m == 0 || n == 0 || (alpha == 0.0f && beta == 1.0f)) return;
  if (beta != 1.0f)
    for (size_t j = 0; j < n; ++j) y[j] = y[j] * beta;
  if (alpha == 0.0f) return;
  float* xs = (float*)malloc(sizeof(float) * m);
  for (size_t i = 0; i < m; ++i) xs[i] = alpha * x[i];
  for (size_t j = 0; j < n; ++j) {
    const float* col = A + j * lda;
    float acc[8] = {0};
    size_t i = 0;
    for (; i + 8 <= m; i += 8)
      for (int q = 0; q < 8; ++q) acc[q] = fmaf(col[i + q], xs[i + q], acc[q]);
    float s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    for (; i < m; ++i) s += col[i] * xs[i];
    y[j] += s;
  }
  free(xs);
}

/* level1/sdot.rs:60-145: 8 x 4-lane fp32 accumulators over 32-element steps. */
float port_sdot(size_t n, const float* x, const float* y) {
  float acc[32] = {0};
  size_t i = 0;
  for (; i + 32 <= n; i += 32)
    for (int q = 0; q < 32; ++q) acc[q] = fmaf(x[i + q], y[i + q], acc[q]);
  float s = 0.0f;
  for (int q = 0; q < 32; ++q) s += acc[q];
  for (; i < n; ++i) s += x[i] * y[i];
  return s;
}
