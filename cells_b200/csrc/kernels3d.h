// Host-visible declarations of the 3D kernels' launchers (implemented in step3d.cu and aux3d.cu).
#pragma once

#include "d3q19.cuh"

namespace cells {

struct StepLaunch3 {
  const void* src;
  void* dst;
  const uint32_t* flags;
  const float* sdf;
  const uint8_t* rowBody;
  const void* xTab;
  const int* blockSlot;
  double4* partials;
  double4* history;
  DevState3* st;
  int W, H, D, N;
  int bx, by;
  int nForceBlocks;
  int rampKind, rampEvery;
  double rampTarget, rampSteps;
  double lambda, smagC2;
  int par, sample;
};

// precision: cells_precision (0 f32, 1 f16, 2 bf16, 3 f64). fast: FMA contraction allowed;
// exact: no contraction, every operation rounds as written.
namespace fast {
cudaError_t launch_step3(int precision, const StepLaunch3& a, cudaStream_t s);
}
namespace exact {
cudaError_t launch_step3(int precision, const StepLaunch3& a, cudaStream_t s);
}

struct AuxLaunch3 {
  int W, H, D, N;
  double uIn;   // inflow speed for init / refill fallback
};

// flags3dShader (src/shaders/aux3d.ts:20-101): flags, refill of uncovered cells from mac, and the
// body-row marks (rowBody must be zeroed first).
cudaError_t launch_flags3(int precision, const AuxLaunch3& a, const float* sdf, uint32_t* flags, uint8_t* rowBody,
                          void* fA, void* fB, const float4* mac, cudaStream_t s);
// init3dShader (src/shaders/aux3d.ts:105-125); mac (optional, (ux,uy,uz,rho) per cell) sets each
// fluid cell to its own equilibrium instead of feq(1, uIn, 0, 0).
cudaError_t launch_init3(int precision, const AuxLaunch3& a, void* fA, void* fB, const uint32_t* flags,
                         const float4* mac, cudaStream_t s);
// macro3dShader (src/shaders/aux3d.ts:128-152); sets status bit 1 on a non-finite value.
cudaError_t launch_macro3(int precision, const AuxLaunch3& a, const void* f, const uint32_t* flags, float4* mac,
                          DevState3* st, cudaStream_t s);
// sum(rho) over fluid cells in f64: per-block partials, then one block sums them in order.
cudaError_t launch_mass3(int precision, const AuxLaunch3& a, const void* f, const uint32_t* flags, double* partials,
                         int nPartials, double* out, cudaStream_t s);
// Writes parts of the device state in stream order. which: bit 0 both step counters, bit 1 both
// inlet speeds, bit 2 clears the force sample counter, bit 3 clears the status word.
cudaError_t launch_set_state3(DevState3* st, int which, unsigned step, double uIn0, double uIn1, cudaStream_t s);

}  // namespace cells
