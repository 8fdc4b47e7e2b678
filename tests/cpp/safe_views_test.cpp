// Checks of coral_safe.hpp's view validation on the host (no GPU, no calls):
// the cases of coral-safe/tests/types.rs (ZeroStride, OutOfBounds{6, 5},
// InvalidLda{4, 5}) plus empty views, offsets, saturation and the Display
// text of each BufferError variant.
#include <cstdio>
#include <limits>
#include <string>

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

int main() {
  // views are never dereferenced here: any non-null address will do
  float* fake = reinterpret_cast<float*>(uintptr_t{0x1000});
  // types.rs ensure_nonzero_stride_vec: n 5, stride 0
  EXPECT(VectorRef<float>::make({fake, 5}, 5, 0, 0).unwrap_err() == BufferError::zero_stride());
  EXPECT(VectorMut<float>::make({fake, 5}, 5, 0, 0).unwrap_err() == BufferError::zero_stride());
  // types.rs ensure_within_bounds_vec: n 3, stride 2, offset 1 needs 6
  EXPECT(VectorRef<float>::make({fake, 5}, 3, 2, 1).unwrap_err() == BufferError::out_of_bounds(6, 5));
  EXPECT(VectorRef<float>::make({fake, 6}, 3, 2, 1).is_ok());
  EXPECT(VectorMut<float>::make({fake, 5}, 3, 2, 1).unwrap_err() == BufferError::out_of_bounds(6, 5));
  // types.rs ensure_valid_lda_mat: 5 x 6, lda 4 -> InvalidLda{4, 5}; lda 7 fits
  EXPECT(MatrixRef<float>::make({fake, 24}, 5, 6, 4, 0).unwrap_err() == BufferError::invalid_lda(4, 5));
  EXPECT(MatrixMut<float>::make({fake, 24}, 5, 6, 4, 0).unwrap_err() == BufferError::invalid_lda(4, 5));
  EXPECT(MatrixRef<float>::make({fake, 42}, 5, 6, 7, 0).is_ok());
  // (n_cols - 1) lda + n_rows + offset: 5*7 + 5 + 3 = 43 > 42
  EXPECT(MatrixRef<float>::make({fake, 42}, 5, 6, 7, 3).unwrap_err() == BufferError::out_of_bounds(43, 42));
  EXPECT(MatrixRef<float>::make({fake, 42}, 5, 6, 0, 0).unwrap_err() == BufferError::zero_stride());
  // empty views skip every check
  EXPECT(VectorRef<float>::make({nullptr, 0}, 0, 0, 99).is_ok());
  EXPECT(MatrixRef<float>::make({nullptr, 0}, 0, 6, 0, 0).is_ok());
  EXPECT(MatrixRef<float>::make({nullptr, 0}, 5, 0, 1, 0).is_ok());
  // usize saturation of the required length
  const size_t big = std::numeric_limits<size_t>::max();
  EXPECT(VectorRef<float>::make({fake, 10}, big, 2, 0).unwrap_err() == BufferError::out_of_bounds(big, 10));
  // accessors and the offset pointer
  auto v = VectorRef<float>::make({fake, 100}, 10, 3, 7).unwrap();
  EXPECT(v.n() == 10 && v.stride() == 3 && v.offset() == 7 && v.ptr() == fake + 7 && v.compare_n(10));
  auto m = MatrixMut<float>::make({fake, 100}, 4, 5, 6, 2).unwrap();
  EXPECT(m.n_rows() == 4 && m.n_cols() == 5 && m.lda() == 6 && m.ptr() == fake + 2 && !m.compare_m_n());
  // Display text (errors.rs)
  EXPECT(std::string(BufferError::zero_stride().what()) == "stride must be nonzero");
  EXPECT(std::string(BufferError::out_of_bounds(6, 5).what()) == "buffer too small: required 6, have 5");
  EXPECT(std::string(BufferError::bad_offset(9, 4).what()) == "offset 9 out of range for buffer of len 4");
  EXPECT(std::string(BufferError::invalid_lda(4, 5).what()) == "leading dimension 4 must exceed num rows 5");
  // unwrap of an error throws the BufferError
  bool threw = false;
  try {
    (void)VectorRef<float>::make({fake, 5}, 5, 0, 0).unwrap();
  } catch (const BufferError& e) {
    threw = e == BufferError::zero_stride();
  }
  EXPECT(threw);
  std::printf("%s (%d failures)\n", failures ? "FAILED" : "ok", failures);
  return failures ? 1 : 0;
}
