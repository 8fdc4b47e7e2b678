// coral_safe.hpp -- checked views and routines over device buffers, after
// coral-safe (coral-safe/src/types.rs, errors.rs, level1/, level2/, fused/).
//
// A view is validated once, when it is built, and the routines take views
// instead of (pointer, n, inc) triples:
//
//   DeviceSlice<T>{ptr, len}       device memory, len counted in elements
//   VectorRef<T> / VectorMut<T>    (slice, n, stride, offset)
//   MatrixRef<T> / MatrixMut<T>    (slice, n_rows, n_cols, lda, offset)
//
// `make(...)` returns Result<View>: the view, or the reference's BufferError
// (ZeroStride, OutOfBounds{required, len}, BadOffset{offset, len},
// InvalidLda{lda, n_rows}) with its Display text.  Empty views skip the
// checks, as in the reference.  The routines call the coral_* entry points on
// a Handle's stream at ptr + offset.  Logical lengths that disagree throw
// std::invalid_argument, where the reference has debug_assert!s
// (types.rs:324-332, sgemv_n.rs:23-24, sger.rs:227-228).  A failing entry
// point throws coral::Error.
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <variant>

#include "coral.hpp"

namespace coral {
namespace safe {

enum class CoralTranspose : int { NoTrans = 0, Trans = 1 };
enum class CoralTriangular : int { Upper = 0, Lower = 1 };
enum class CoralDiagonal : int { Unit = 0, NonUnit = 1 };

// errors.rs: BufferError and its Display text.
struct BufferError : std::exception {
  enum class Kind { ZeroStride, OutOfBounds, BadOffset, InvalidLda };
  Kind kind = Kind::ZeroStride;
  size_t a = 0, b = 0;  // OutOfBounds: required, len; BadOffset: offset, len; InvalidLda: lda, n_rows
  std::string text;

  static BufferError zero_stride() { return make(Kind::ZeroStride, 0, 0); }
  static BufferError out_of_bounds(size_t required, size_t len) { return make(Kind::OutOfBounds, required, len); }
  static BufferError bad_offset(size_t offset, size_t len) { return make(Kind::BadOffset, offset, len); }
  static BufferError invalid_lda(size_t lda, size_t n_rows) { return make(Kind::InvalidLda, lda, n_rows); }

  const char* what() const noexcept override { return text.c_str(); }
  bool operator==(const BufferError& o) const { return kind == o.kind && a == o.a && b == o.b; }

 private:
  static BufferError make(Kind k, size_t a, size_t b) {
    BufferError e;
    e.kind = k;
    e.a = a;
    e.b = b;
    switch (k) {
      case Kind::ZeroStride: e.text = "stride must be nonzero"; break;
      case Kind::OutOfBounds:
        e.text = "buffer too small: required " + std::to_string(a) + ", have " + std::to_string(b);
        break;
      case Kind::BadOffset:
        e.text = "offset " + std::to_string(a) + " out of range for buffer of len " + std::to_string(b);
        break;
      case Kind::InvalidLda:
        e.text = "leading dimension " + std::to_string(a) + " must exceed num rows " + std::to_string(b);
        break;
    }
    return e;
  }
};

// Result<V>: a view or the BufferError that refused it.
template <class V>
class Result {
 public:
  Result(V v) : r_(std::move(v)) {}            // NOLINT(google-explicit-constructor)
  Result(BufferError e) : r_(std::move(e)) {}  // NOLINT(google-explicit-constructor)
  bool is_ok() const { return r_.index() == 0; }
  bool is_err() const { return r_.index() == 1; }
  // the view; throws the BufferError when there is none
  V unwrap() const {
    if (is_err()) throw std::get<1>(r_);
    return std::get<0>(r_);
  }
  BufferError unwrap_err() const {
    if (is_ok()) throw std::logic_error("unwrap_err on a valid view");
    return std::get<1>(r_);
  }

 private:
  std::variant<V, BufferError> r_;
};

template <class T>
struct DeviceSlice {
  T* ptr = nullptr;
  size_t len = 0;
};

namespace detail {
inline size_t sat_mul(size_t a, size_t b) {
  if (a != 0 && b > std::numeric_limits<size_t>::max() / a) return std::numeric_limits<size_t>::max();
  return a * b;
}
inline size_t sat_add(size_t a, size_t b) {
  return b > std::numeric_limits<size_t>::max() - a ? std::numeric_limits<size_t>::max() : a + b;
}
// types.rs:76-103: n == 0 skips the checks; stride 0 -> ZeroStride;
// (n - 1) stride + offset + 1 elements must fit.
inline const BufferError* check_vector(size_t len, size_t n, size_t stride, size_t offset, BufferError* out) {
  if (n == 0) return nullptr;
  if (stride == 0) return &(*out = BufferError::zero_stride());
  const size_t required = sat_add(sat_add(sat_mul(n - 1, stride), offset), 1);
  if (required > len) return &(*out = BufferError::out_of_bounds(required, len));
  return nullptr;
}
// types.rs:174-201: empty -> no checks; lda 0 -> ZeroStride; lda < n_rows ->
// InvalidLda; (n_cols - 1) lda + n_rows + offset elements must fit.
inline const BufferError* check_matrix(size_t len, size_t m, size_t n, size_t lda, size_t offset,
                                       BufferError* out) {
  if (m == 0 || n == 0) return nullptr;
  if (lda == 0) return &(*out = BufferError::zero_stride());
  if (lda < m) return &(*out = BufferError::invalid_lda(lda, m));
  const size_t required = sat_add(sat_add(sat_mul(n - 1, lda), m), offset);
  if (required > len) return &(*out = BufferError::out_of_bounds(required, len));
  return nullptr;
}
}  // namespace detail

template <class T, class P>
class VectorView {
 public:
  static Result<VectorView> make(DeviceSlice<P> data, size_t n, size_t stride, size_t offset) {
    BufferError e;
    if (detail::check_vector(data.len, n, stride, offset, &e)) return e;
    return VectorView(data, n, stride, offset);
  }
  size_t n() const { return n_; }
  size_t stride() const { return stride_; }
  size_t offset() const { return offset_; }
  DeviceSlice<P> as_slice() const { return data_; }
  bool compare_n(size_t n) const { return n_ == n; }
  // the first logical element (device address)
  P* ptr() const { return data_.ptr + offset_; }

 private:
  VectorView(DeviceSlice<P> d, size_t n, size_t s, size_t o) : data_(d), n_(n), stride_(s), offset_(o) {}
  DeviceSlice<P> data_;
  size_t n_, stride_, offset_;
};

template <class T>
using VectorRef = VectorView<T, const T>;
template <class T>
using VectorMut = VectorView<T, T>;

template <class T, class P>
class MatrixView {
 public:
  static Result<MatrixView> make(DeviceSlice<P> data, size_t n_rows, size_t n_cols, size_t lda, size_t offset) {
    BufferError e;
    if (detail::check_matrix(data.len, n_rows, n_cols, lda, offset, &e)) return e;
    return MatrixView(data, n_rows, n_cols, lda, offset);
  }
  size_t n_rows() const { return m_; }
  size_t n_cols() const { return n_; }
  size_t lda() const { return lda_; }
  size_t offset() const { return offset_; }
  DeviceSlice<P> as_slice() const { return data_; }
  bool compare_m_n() const { return m_ == n_; }
  P* ptr() const { return data_.ptr + offset_; }

 private:
  MatrixView(DeviceSlice<P> d, size_t m, size_t n, size_t lda, size_t o)
      : data_(d), m_(m), n_(n), lda_(lda), offset_(o) {}
  DeviceSlice<P> data_;
  size_t m_, n_, lda_, offset_;
};

template <class T>
using MatrixRef = MatrixView<T, const T>;
template <class T>
using MatrixMut = MatrixView<T, T>;

// A coral handle bound to a CUDA stream (nullptr: the legacy default stream).
class Handle {
 public:
  explicit Handle(void* stream = nullptr) {
    check("coral_create", coral_create(&h_));
    check("coral_set_stream", coral_set_stream(h_, stream));
  }
  ~Handle() {
    if (h_) coral_destroy(h_);
  }
  Handle(const Handle&) = delete;
  Handle& operator=(const Handle&) = delete;
  coral_handle_t get() const { return h_; }

 private:
  coral_handle_t h_ = nullptr;
};

namespace detail {
template <class X, class Y>
void same_n(const X& x, const Y& y) {
  if (!x.compare_n(y.n())) throw std::invalid_argument("number of logical elements must be equal");
}
}  // namespace detail

// ---- level 1 (coral-safe/src/level1) ---------------------------------------------
inline size_t isamax(Handle& h, VectorRef<float> x) {
  size_t r = 0;
  check("isamax", coral_isamax(h.get(), x.n(), x.ptr(), x.stride(), &r));
  return r;
}
inline float sasum(Handle& h, VectorRef<float> x) {
  float r = 0;
  check("sasum", coral_sasum(h.get(), x.n(), x.ptr(), x.stride(), &r));
  return r;
}
inline float snrm2(Handle& h, VectorRef<float> x) {
  float r = 0;
  check("snrm2", coral_snrm2(h.get(), x.n(), x.ptr(), x.stride(), &r));
  return r;
}
inline float sdot(Handle& h, VectorRef<float> x, VectorRef<float> y) {
  detail::same_n(x, y);
  float r = 0;
  check("sdot", coral_sdot(h.get(), x.n(), x.ptr(), x.stride(), y.ptr(), y.stride(), &r));
  return r;
}
inline void saxpy(Handle& h, float alpha, VectorRef<float> x, VectorMut<float> y) {
  detail::same_n(x, y);
  check("saxpy", coral_saxpy(h.get(), x.n(), alpha, x.ptr(), x.stride(), y.ptr(), y.stride()));
}
inline void scopy(Handle& h, VectorRef<float> x, VectorMut<float> y) {
  detail::same_n(x, y);
  check("scopy", coral_scopy(h.get(), x.n(), x.ptr(), x.stride(), y.ptr(), y.stride()));
}
inline void sswap(Handle& h, VectorMut<float> x, VectorMut<float> y) {
  detail::same_n(x, y);
  check("sswap", coral_sswap(h.get(), x.n(), x.ptr(), x.stride(), y.ptr(), y.stride()));
}
inline void sscal(Handle& h, float alpha, VectorMut<float> x) {
  check("sscal", coral_sscal(h.get(), x.n(), alpha, x.ptr(), x.stride()));
}
inline void srot(Handle& h, VectorMut<float> x, VectorMut<float> y, float c, float s) {
  detail::same_n(x, y);
  check("srot", coral_srot(h.get(), x.n(), x.ptr(), x.stride(), y.ptr(), y.stride(), c, s));
}
// param = [flag, h11, h21, h12, h22] (host memory)
inline void srotm(Handle& h, VectorMut<float> x, VectorMut<float> y, const float (&param)[5]) {
  detail::same_n(x, y);
  check("srotm", coral_srotm(h.get(), x.n(), x.ptr(), x.stride(), y.ptr(), y.stride(), param));
}
// host scalars, updated in place as in the reference
inline void srotg(Handle& h, float& a, float& b, float& c, float& s) {
  check("srotg", coral_srotg(h.get(), &a, &b, &c, &s));
}
inline void srotmg(Handle& h, float& sd1, float& sd2, float& sx1, float sy1, float (&param)[5]) {
  check("srotmg", coral_srotmg(h.get(), &sd1, &sd2, &sx1, sy1, param));
}

// ---- level 2 (coral-safe/src/level2) ---------------------------------------------
inline void sgemv(Handle& h, CoralTranspose op, float alpha, float beta, MatrixRef<float> a, VectorRef<float> x,
                  VectorMut<float> y) {
  const bool t = op == CoralTranspose::Trans;
  if (!x.compare_n(t ? a.n_rows() : a.n_cols()))
    throw std::invalid_argument(t ? "logical length of x must equal n_rows" : "logical length of x must equal n_cols");
  if (!y.compare_n(t ? a.n_cols() : a.n_rows()))
    throw std::invalid_argument(t ? "logical length of y must equal n_cols" : "logical length of y must equal n_rows");
  check("sgemv", coral_sgemv(h.get(), static_cast<int>(op), a.n_rows(), a.n_cols(), alpha, a.ptr(), a.lda(), x.ptr(),
                             x.stride(), beta, y.ptr(), y.stride()));
}
inline void sger(Handle& h, float alpha, MatrixMut<float> a, VectorRef<float> x, VectorRef<float> y) {
  if (y.n() != a.n_cols()) throw std::invalid_argument("logical length of y must equal n_cols");
  if (x.n() != a.n_rows()) throw std::invalid_argument("logical length of x must equal n_rows");
  if (a.n_rows() == 0 || a.n_cols() == 0) return;
  check("sger", coral_sger(h.get(), a.n_rows(), a.n_cols(), alpha, x.ptr(), x.stride(), y.ptr(), y.stride(),
                           a.ptr(), a.lda()));
}
inline void strsv(Handle& h, CoralTriangular uplo, CoralTranspose trans, CoralDiagonal diag, MatrixRef<float> a,
                  VectorMut<float> x) {
  if (!a.compare_m_n()) throw std::invalid_argument("matrix must be square");
  if (!x.compare_n(a.n_rows())) throw std::invalid_argument("logical length of x must equal n");
  if (a.n_rows() == 0) return;
  check("strsv", coral_strsv(h.get(), static_cast<int>(uplo), static_cast<int>(trans), static_cast<int>(diag),
                             a.n_rows(), a.ptr(), a.lda(), x.ptr(), x.stride()));
}

// ---- fused (coral-safe/src/fused) ---------------------------------------------------
inline void saxpyf(Handle& h, MatrixRef<float> a, VectorRef<float> x, VectorMut<float> y) {
  if (!x.compare_n(a.n_cols())) throw std::invalid_argument("logical length of x must equal n_cols");
  if (!y.compare_n(a.n_rows())) throw std::invalid_argument("logical length of y must equal n_rows");
  check("saxpyf", coral_saxpyf(h.get(), a.n_rows(), a.n_cols(), x.ptr(), x.stride(), a.ptr(), a.lda(), y.ptr(),
                               y.stride()));
}
// y += A^T x; a strided y goes through SGEMV T with alpha = beta = 1 (the same sum)
inline void sdotf(Handle& h, MatrixRef<float> a, VectorRef<float> x, VectorMut<float> y) {
  if (!x.compare_n(a.n_rows())) throw std::invalid_argument("logical length of x must equal n_rows");
  if (!y.compare_n(a.n_cols())) throw std::invalid_argument("logical length of y must equal n_cols");
  if (y.stride() == 1 || y.n() == 0)
    check("sdotf", coral_sdotf(h.get(), a.n_rows(), a.n_cols(), a.ptr(), a.lda(), x.ptr(), x.stride(), y.ptr()));
  else
    check("sdotf", coral_sgemv(h.get(), 1, a.n_rows(), a.n_cols(), 1.0f, a.ptr(), a.lda(), x.ptr(), x.stride(),
                               1.0f, y.ptr(), y.stride()));
}

}  // namespace safe
}  // namespace coral
