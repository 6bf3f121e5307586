// Allocation-free variant of the f64 mass reduction (cells3d_mass_noalloc in include/cells.h).
//
// Some callers cannot allocate device memory at the point where they need a result: a host
// application or plugin framework that owns every device buffer and forbids allocations after
// start-up, or a real-time loop that must not risk an allocation failure or the implicit
// synchronisation that cudaMalloc/cudaFree cause. This entry point serves them: the caller passes
// the populations, the flags and a device location for the result, and the per-block partial sums
// live in a file-scope __device__ array of fixed size instead of a buffer the library allocates.
//
// Limits and behaviour
//   * the scratch holds 8192 doubles (64 KiB) on every GPU that loads the library, for the life of
//     the process;
//   * one partial per 8192 cells, so at most 8192 * 8192 = 67,108,864 cells; larger grids are
//     rejected with CELLS_E_INVALID before anything is enqueued;
//   * every call overwrites every partial it reads, so nothing has to be cleared between calls;
//     the array keeps the last call's partials afterwards;
//   * all calls share the one array per device: calls that can overlap on the GPU (different
//     streams, or different host threads) race on it and must be serialised by the caller;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//     that device current and keeps it for that device's current CUDA context; make that first
//     call before any stream capture that uses it. A call under a different context of the device
//     (after a cudaDeviceReset, or with another context made current) looks the address up again.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/cells.h"
#include "d3q19.cuh"

namespace cells {

constexpr int kNoallocMaxPartials = 8192;
constexpr long long kNoallocCellsPerBlock = 8192;

static __device__ __align__(256) double g_mass_scratch[kNoallocMaxPartials];

// Sum of rho = 1 + sum_i f_i over the fluid cells of one contiguous range of cells.
template <class C>
__global__ void mass3_noalloc_partial_kernel(const typename C::S* __restrict__ f, const uint32_t* __restrict__ flags,
                                             long long n, double* __restrict__ partials) {
  __shared__ double red[8];
  const long long begin = (long long)blockIdx.x * kNoallocCellsPerBlock;
  const long long end = min(begin + kNoallocCellsPerBlock, n);
  double acc = 0.0;
  for (long long idx = begin + threadIdx.x; idx < end; idx += blockDim.x) {
    if (flags[idx] & FLAG3_SOLID) continue;
    double drho = 0.0;
    for (int i = 0; i < Q3; i++) drho += (double)C::load(f + (size_t)i * (size_t)n + idx);
    acc += 1.0 + drho;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    partials[blockIdx.x] = s;
  }
}

__global__ void mass3_noalloc_final_kernel(const double* __restrict__ partials, int n, double* __restrict__ out) {
  __shared__ double red[8];
  double acc = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) acc += partials[k];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    *out = s;
  }
}

namespace {
std::mutex g_scratch_mutex;
constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
void* g_scratch_ctx[kMaxDevices] = {nullptr};  // the context each cached address belongs to

// The driver's current context (cuCtxGetCurrent through the runtime's entry-point query, so the
// library needs no link to libcuda); nullptr when it cannot be found, which disables caching.
void* current_context() {
  using GetCurrent = int (*)(void**);
  static GetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (GetCurrent) nullptr;
    return (GetCurrent)f;
  }();
  void* ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// The device address of the scratch array on the current device, looked up with that device
// current and kept for the device's current context.
cudaError_t scratch_on_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  // no current context yet (before the runtime's first use of the device): nullptr, and the
  // address is looked up again on the next call
  void* ctx = current_context();
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev] || !ctx || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_mass_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = (double*)p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}
}  // namespace

// failures are reported through cells_last_error(NULL), like a failed create
extern thread_local std::string g_create_error;

}  // namespace cells

using namespace cells;

extern "C" int cells3d_mass_noalloc(const void* populations, const uint32_t* flags, int64_t n_cells, int32_t precision,
                                    double* out_device, void* stream) {
  g_create_error.clear();
  if (!populations || !flags || !out_device || n_cells <= 0) {
    g_create_error = "cells3d_mass_noalloc: populations, flags and out_device must be device pointers and n_cells > 0";
    return CELLS_E_INVALID;
  }
  const long long blocks = (n_cells + kNoallocCellsPerBlock - 1) / kNoallocCellsPerBlock;
  if (blocks > kNoallocMaxPartials) {
    g_create_error = "cells3d_mass_noalloc: " + std::to_string((long long)n_cells) + " cells exceed the maximum of " +
                      std::to_string((long long)kNoallocMaxPartials * kNoallocCellsPerBlock) +
                      " (the fixed scratch holds " + std::to_string(kNoallocMaxPartials) + " partial sums)";
    return CELLS_E_INVALID;
  }
  if (precision < CELLS_FP32 || precision > CELLS_FP64) {
    g_create_error = "cells3d_mass_noalloc: unknown precision " + std::to_string(precision);
    return CELLS_E_PRECISION_UNSUPPORTED;
  }
  double* scratch = nullptr;
  cudaError_t e = scratch_on_current_device(&scratch);
  if (e != cudaSuccess) {
    g_create_error = std::string("cells3d_mass_noalloc: scratch address lookup failed: ") + cudaGetErrorString(e);
    return CELLS_E_CUDA;
  }
  cudaStream_t s = (cudaStream_t)stream;
  switch (precision) {
    case CELLS_FP32:
      mass3_noalloc_partial_kernel<CodecF32><<<(unsigned)blocks, 256, 0, s>>>((const float*)populations, flags, n_cells, scratch);
      break;
    case CELLS_FP16:
      mass3_noalloc_partial_kernel<CodecF16><<<(unsigned)blocks, 256, 0, s>>>((const __half*)populations, flags, n_cells, scratch);
      break;
    case CELLS_BF16:
      mass3_noalloc_partial_kernel<CodecBF16><<<(unsigned)blocks, 256, 0, s>>>((const __nv_bfloat16*)populations, flags, n_cells,
                                                                             scratch);
      break;
    default:
      mass3_noalloc_partial_kernel<CodecF64><<<(unsigned)blocks, 256, 0, s>>>((const double*)populations, flags, n_cells, scratch);
      break;
  }
  e = cudaGetLastError();
  if (e == cudaSuccess) {
    mass3_noalloc_final_kernel<<<1, 256, 0, s>>>(scratch, (int)blocks, out_device);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    g_create_error = std::string("cells3d_mass_noalloc: launch failed: ") + cudaGetErrorString(e);
    return CELLS_E_CUDA;
  }
  return CELLS_OK;
}
