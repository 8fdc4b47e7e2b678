// Level-2 routines whose kernels are not in this build report
// CORAL_ERR_NOT_SUPPORTED.
#include "common.cuh"

extern "C" {

coral_status_t coral_ssymv(coral_handle_t, int, size_t, float, const float*, size_t, const float*,
                           size_t, float, float*, size_t) {
  return CORAL_ERR_NOT_SUPPORTED;
}
coral_status_t coral_chemv(coral_handle_t, int, size_t, const float*, const float*, size_t,
                           const float*, size_t, const float*, float*, size_t) {
  return CORAL_ERR_NOT_SUPPORTED;
}
coral_status_t coral_strsv(coral_handle_t, int, int, int, size_t, const float*, size_t, float*,
                           size_t) {
  return CORAL_ERR_NOT_SUPPORTED;
}
coral_status_t coral_strmv(coral_handle_t, int, int, int, size_t, const float*, size_t, float*,
                           size_t) {
  return CORAL_ERR_NOT_SUPPORTED;
}

}  // extern "C"
