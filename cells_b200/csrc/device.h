// Device memory, stream and error plumbing shared by the 2D and 3D solvers.
//
// A Device is either a CUDA device (one non-blocking stream per solver handle) or the fake device
// (CELLS_FAKE_DEVICE): host memory, no kernels, used only by the host-logic tests.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace cells {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

// Thrown by Device::alloc; the solver turns it into "Solver3D allocation failed: <what>".
struct AllocError : std::runtime_error {
  explicit AllocError(const std::string& m) : std::runtime_error(m) {}
};

void check_cuda(cudaError_t e, const char* what);

struct Device {
  bool fake = false;
  int ordinal = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evRead = nullptr;
  int failAllocAt = 0;  // fake device only: the n-th allocation (1-based) fails
  int nAllocs = 0;
  std::vector<void*> owned;
  int64_t launches = 0;

  void open(int device_ordinal, int fail_alloc_at);
  void close();
  void* alloc(size_t bytes, const char* what);
  void h2d(void* d, const void* h, size_t bytes);
  void d2h(void* h, const void* d, size_t bytes);
  // Device-to-host copy of a large buffer into pageable memory, waiting for it: through two pinned
  // 2 MiB buffers (allocated on first use, freed by close), the copy of chunk k out of one overlapping
  // the DMA of chunk k + 1 into the other. A pageable destination otherwise runs at a fraction of the
  // pinned rate. Small copies take d2h and a sync.
  void d2h_large(void* h, const void* d, size_t bytes);
  void* stage[2] = {nullptr, nullptr};
  cudaEvent_t stageEv[2] = {nullptr, nullptr};
  void memset0(void* d, size_t bytes);
  void sync();
  void* host_pinned(size_t bytes);
  void free_host_pinned(void* p);
  void release(void* d);  // frees one buffer from alloc() before close()
  size_t free_bytes();
};

// Number of live fake-device buffers in the process (host-logic tests check that a failed create
// frees everything).
extern int64_t g_fake_live_buffers;

// First base of every handle type: cells_last_error reads the message through it.
struct HandleBase {
  std::string lastError;
};

// Message of the last failed create on this thread (cells_last_error(NULL)).
extern thread_local std::string g_create_error;

}  // namespace cells
