// Read-only view of an operator handle's device state for entry points that
// live outside engine.cu.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

struct defmm_handle;

namespace dfb {

struct HandleView {
  int device = -1;
  cudaStream_t stream = nullptr;  // the handle's own stream
  int64_t nS = 0;                 // sources
  const double* S_pos = nullptr;  // 3 per source, tree order (device)
  const int32_t* S_perm = nullptr;  // tree position -> user index (device)
  const double2* qin = nullptr;   // charges of the last host gemv, user order (device)
  // record on the stream that last reads qin: the handle's next host gemv
  // waits for it before overwriting qin
  cudaEvent_t qin_read = nullptr;
  double kappa = 0.;
};

// Fills `v` for a handle that has run a host gemv; otherwise records the
// reason in the handle and returns DEFMM_ERR_ARG.
int handle_view(defmm_handle* h, HandleView* v);
// Records `msg` as the handle's last error and returns `code`.
int handle_fail(defmm_handle* h, int code, const char* msg);

}  // namespace dfb
