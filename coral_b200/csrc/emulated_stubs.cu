// Emulated-precision GEMM entry points whose tensor-core kernels are not
// built into this library yet report CORAL_ERR_NOT_SUPPORTED.
#include "common.cuh"

namespace coral {

coral_status_t enqueue_dgemm_ozaki(Handle*, int, int, size_t, size_t, size_t, double,
                                   const double*, size_t, const double*, size_t, double, double*,
                                   size_t) {
  return CORAL_ERR_NOT_SUPPORTED;
}
coral_status_t enqueue_zgemm_ozaki(Handle*, int, int, size_t, size_t, size_t, double2,
                                   const double2*, size_t, const double2*, size_t, double2,
                                   double2*, size_t) {
  return CORAL_ERR_NOT_SUPPORTED;
}

}  // namespace coral
