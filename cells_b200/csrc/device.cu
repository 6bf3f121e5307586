#include "device.h"

#include <string>

#include "../../include/cells.h"

#include <cstdlib>

namespace cells {

int64_t g_fake_live_buffers = 0;

void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  if (e == cudaErrorMemoryAllocation) throw AllocError(std::string(what) + ": " + cudaGetErrorString(e));
  throw Error(4 /*CELLS_E_CUDA*/, std::string(what) + ": " + cudaGetErrorString(e));
}

void Device::open(int device_ordinal, int fail_alloc_at) {
  ordinal = device_ordinal;
  failAllocAt = fail_alloc_at;
  if (device_ordinal == -2) {
    fake = true;
    return;
  }
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    throw Error(4, std::string("no CUDA device available: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
  if (device_ordinal < 0 || device_ordinal >= n) throw Error(3, "device ordinal out of range");
  check_cuda(cudaSetDevice(device_ordinal), "cudaSetDevice");
  check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
  check_cuda(cudaEventCreate(&ev0), "cudaEventCreate");
  check_cuda(cudaEventCreate(&ev1), "cudaEventCreate");
  check_cuda(cudaEventCreateWithFlags(&evRead, cudaEventDisableTiming), "cudaEventCreate");
}

void Device::close() {
  if (fake) {
    for (void* p : owned) {
      std::free(p);
      g_fake_live_buffers--;
    }
    owned.clear();
    return;
  }
  if (stream) cudaStreamSynchronize(stream);
  for (int b = 0; b < 2; b++) {
    if (stage[b]) cudaFreeHost(stage[b]);
    if (stageEv[b]) cudaEventDestroy(stageEv[b]);
    stage[b] = nullptr;
    stageEv[b] = nullptr;
  }
  for (void* p : owned) cudaFree(p);
  owned.clear();
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (evRead) cudaEventDestroy(evRead);
  if (stream) cudaStreamDestroy(stream);
  ev0 = ev1 = evRead = nullptr;
  stream = nullptr;
}

void* Device::alloc(size_t bytes, const char* what) {
  nAllocs++;
  if (bytes == 0) bytes = 16;
  if (fake) {
    if (failAllocAt > 0 && nAllocs == failAllocAt)
      throw AllocError(std::string("fake out-of-memory allocating ") + what);
    void* p = std::calloc(1, bytes);
    if (!p) throw AllocError(std::string("host out of memory allocating ") + what);
    owned.push_back(p);
    g_fake_live_buffers++;
    return p;
  }
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear the sticky-free allocation error
    throw AllocError(std::string(what) + " (" + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e));
  }
  owned.push_back(p);
  return p;
}

void Device::h2d(void* d, const void* h, size_t bytes) {
  if (fake) {
    std::memcpy(d, h, bytes);
    return;
  }
  check_cuda(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync H2D");
}

constexpr size_t kStageBytes = 2u << 20;

// Whether host memory is page-locked (allocated or registered with CUDA): such memory takes a
// direct DMA copy.
static bool host_is_pinned(const void* h) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, h) != cudaSuccess) {
    cudaGetLastError();  // clear the error of an unknown pointer
    return false;
  }
  return attr.type == cudaMemoryTypeHost;
}

void Device::d2h_large(void* h, const void* d, size_t bytes) {
  if (fake || bytes < 2 * kStageBytes || host_is_pinned(h)) {
    d2h(h, d, bytes);
    sync();
    return;
  }
  if (!stage[0]) {
    for (int b = 0; b < 2; b++) {
      check_cuda(cudaMallocHost(&stage[b], kStageBytes), "cudaMallocHost");
      check_cuda(cudaEventCreateWithFlags(&stageEv[b], cudaEventDisableTiming), "cudaEventCreate");
    }
  }
  const size_t chunks = (bytes + kStageBytes - 1) / kStageBytes;
  auto issue = [&](size_t k) {
    const size_t off = k * kStageBytes, n = bytes - off < kStageBytes ? bytes - off : kStageBytes;
    check_cuda(cudaMemcpyAsync(stage[k & 1], (const char*)d + off, n, cudaMemcpyDeviceToHost, stream),
               "cudaMemcpyAsync D2H");
    check_cuda(cudaEventRecord(stageEv[k & 1], stream), "cudaEventRecord");
  };
  issue(0);
  issue(1);
  for (size_t k = 0; k < chunks; k++) {
    const size_t off = k * kStageBytes, n = bytes - off < kStageBytes ? bytes - off : kStageBytes;
    check_cuda(cudaEventSynchronize(stageEv[k & 1]), "cudaEventSynchronize");
    std::memcpy((char*)h + off, stage[k & 1], n);
    if (k + 2 < chunks) issue(k + 2);  // the buffer is free again: its chunk has been copied out
  }
}

void Device::d2h(void* h, const void* d, size_t bytes) {
  if (fake) {
    std::memcpy(h, d, bytes);
    return;
  }
  check_cuda(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, stream), "cudaMemcpyAsync D2H");
}

void Device::memset0(void* d, size_t bytes) {
  if (fake) {
    std::memset(d, 0, bytes);
    return;
  }
  check_cuda(cudaMemsetAsync(d, 0, bytes, stream), "cudaMemsetAsync");
}

void Device::sync() {
  if (fake) return;
  check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
}

void* Device::host_pinned(size_t bytes) {
  if (fake) return std::calloc(1, bytes);
  void* p = nullptr;
  check_cuda(cudaMallocHost(&p, bytes), "cudaMallocHost");
  return p;
}

void Device::release(void* d) {
  if (!d) return;
  for (size_t k = 0; k < owned.size(); k++) {
    if (owned[k] != d) continue;
    owned.erase(owned.begin() + (long)k);
    if (fake) {
      std::free(d);
      g_fake_live_buffers--;
    } else {
      cudaFree(d);
    }
    return;
  }
}

void Device::free_host_pinned(void* p) {
  if (!p) return;
  if (fake) {
    std::free(p);
    return;
  }
  cudaFreeHost(p);
}

size_t Device::free_bytes() {
  if (fake) return (size_t)1 << 40;
  size_t fr = 0, tot = 0;
  check_cuda(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
  return fr;
}

}  // namespace cells

// ---------------- pinned host buffers for callers (include/cells.h) ----------------
namespace cells {
extern thread_local std::string g_create_error;
}

extern "C" int cells_host_alloc(size_t bytes, void** out) {
  if (!out || bytes == 0) return CELLS_E_INVALID;
  *out = nullptr;
  const cudaError_t e = cudaMallocHost(out, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cells::g_create_error = std::string("cells_host_alloc: ") + cudaGetErrorString(e);
    *out = nullptr;
    return CELLS_E_ALLOC;
  }
  return CELLS_OK;
}

extern "C" void cells_host_free(void* p) {
  if (p) cudaFreeHost(p);
}
