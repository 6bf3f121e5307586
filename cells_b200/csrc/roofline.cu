// The copy roofline of the reference's benchmark (src/bench.ts:61-95): the memory traffic of one
// step with no arithmetic. `q` SoA population arrays of `cells` elements are copied from one buffer
// to another (optionally reading one u32 flag word per cell as the reference's copy does), the
// buffers swapping every launch as a step's do; the time per launch is measured with CUDA events.
// The step kernel's throughput divided by this copy's is the fraction of the achievable stream.
#include <cuda_runtime.h>

#include <string>

#include "../../include/cells.h"
#include "device.h"

namespace cells {
namespace {

// Each thread moves one word of every population array: 4 bytes (one f32 cell or two 16-bit
// cells, the widths the step kernel moves) or 8 bytes (one f64 cell).
template <class T>
__global__ void copy_roofline_kernel(const T* __restrict__ src, T* __restrict__ dst, const uint32_t* __restrict__ flags,
                                     long long words, int q, int cellsPerWord) {
  const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= words) return;
  T add = 0;
  if (flags) add = (T)__ldg(flags + w * cellsPerWord);
  for (int i = 0; i < q; i++) dst[(long long)i * words + w] = __ldg(src + (long long)i * words + w) + add;
}

template <class T>
cudaError_t launch_copy(const void* src, void* dst, const uint32_t* flags, long long words, int q, int cpw,
                        cudaStream_t s) {
  const unsigned blocks = (unsigned)((words + 255) / 256);
  copy_roofline_kernel<T><<<blocks, 256, 0, s>>>((const T*)src, (T*)dst, flags, words, q, cpw);
  return cudaGetLastError();
}

}  // namespace
}  // namespace cells

using namespace cells;

int cells_copy_roofline(int device, int precision, int q, int64_t n_cells, int launches, int with_flags,
                        double* ms_per_launch) {
  g_create_error.clear();
  if (!ms_per_launch || precision < 0 || precision > 3 || q <= 0 || q > 64 || n_cells <= 0 || launches <= 0) {
    g_create_error = "copy roofline: bad arguments";
    return CELLS_E_INVALID;
  }
  const int bytes = precision == 0 ? 4 : (precision == 3 ? 8 : 2);
  if (bytes == 2 && (n_cells % 2) != 0) {
    g_create_error = "copy roofline: 16-bit storage needs an even cell count";
    return CELLS_E_INVALID;
  }
  const int wordBytes = bytes == 8 ? 8 : 4;
  const int cpw = wordBytes / bytes;
  const long long words = n_cells / cpw;
  const size_t arr = (size_t)q * (size_t)words * wordBytes;
  void* buf[2] = {nullptr, nullptr};
  uint32_t* flags = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int status = CELLS_OK;
  auto fail = [&](cudaError_t e, const char* what) {
    g_create_error = std::string("copy roofline: ") + what + ": " + cudaGetErrorString(e);
    status = e == cudaErrorMemoryAllocation ? CELLS_E_ALLOC : CELLS_E_CUDA;
  };
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) fail(e, "cudaSetDevice");
  if (status == CELLS_OK && (e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess)
    fail(e, "cudaStreamCreate");
  if (status == CELLS_OK && ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess))
    fail(e, "cudaEventCreate");
  for (int k = 0; k < 2 && status == CELLS_OK; k++) {
    if ((e = cudaMalloc(&buf[k], arr)) != cudaSuccess) fail(e, "cudaMalloc");
    else if ((e = cudaMemsetAsync(buf[k], 0, arr, s)) != cudaSuccess) fail(e, "cudaMemset");
  }
  if (status == CELLS_OK && with_flags) {
    if ((e = cudaMalloc(&flags, (size_t)n_cells * 4)) != cudaSuccess) fail(e, "cudaMalloc");
    else if ((e = cudaMemsetAsync(flags, 0, (size_t)n_cells * 4, s)) != cudaSuccess) fail(e, "cudaMemset");
  }
  auto run = [&](int n) {
    for (int k = 0; k < n && status == CELLS_OK; k++) {
      const void* src = buf[k & 1];
      void* dst = buf[(k & 1) ^ 1];
      e = wordBytes == 8 ? launch_copy<unsigned long long>(src, dst, flags, words, q, cpw, s)
                         : launch_copy<uint32_t>(src, dst, flags, words, q, cpw, s);
      if (e != cudaSuccess) fail(e, "copy kernel");
    }
  };
  const int warm = launches < 10 ? launches : 10;
  run(warm);
  if (status == CELLS_OK && (e = cudaEventRecord(e0, s)) != cudaSuccess) fail(e, "cudaEventRecord");
  run(launches);
  if (status == CELLS_OK && (e = cudaEventRecord(e1, s)) != cudaSuccess) fail(e, "cudaEventRecord");
  if (status == CELLS_OK && (e = cudaEventSynchronize(e1)) != cudaSuccess) fail(e, "cudaEventSynchronize");
  float ms = 0.0f;
  if (status == CELLS_OK && (e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) fail(e, "cudaEventElapsedTime");
  if (status == CELLS_OK) *ms_per_launch = (double)ms / launches;
  if (s) cudaStreamSynchronize(s);
  for (void* p : buf)
    if (p) cudaFree(p);
  if (flags) cudaFree(flags);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  return status;
}
