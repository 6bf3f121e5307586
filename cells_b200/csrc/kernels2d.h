// Host-visible declarations of the 2D kernels' launchers (step2d.cu and aux2d.cu).
#pragma once

#include "d2q9.cuh"

namespace cells {

// One step (or, persistent, nSteps steps) of every tunnel of a batch. A tile is one block's cells:
// tileX x (rows tileY) cells of one tunnel, each thread taking rows y and, with rows = 2, y + tileY;
// the tiles of all tunnels are numbered consecutively.
struct Step2Launch {
  const Tunnel2* tunnels;            // device array, one per tunnel
  const unsigned short* tileTunnel;  // device array: the tunnel of each tile
  int nTiles;                        // tiles of all tunnels
  int tileX, tileY;                  // block shape
  int rows;                          // cell rows per thread: 1 or 2
  int par;                           // parity of the first step
  int allowSample;                   // 0: no force sampling (autotuner trials)
  int nSteps;                        // persistent launch: steps per launch
  int gridBlocks;                    // persistent launch: resident blocks
  unsigned* barrier;                 // persistent launch: grid barrier counter (zeroed per launch)
  int* error;                        // persistent launch: set to 1 when a barrier wait ran out
  unsigned barrierExtra;             // persistent launch: arrivals added to every barrier's target
                                     // (0; 1 only to test the time-out path)
};

// precision: 0 f32, 3 f64. fast: FMA contraction allowed; exact: every operation rounds as written.
namespace fast {
cudaError_t launch_step2(int precision, const Step2Launch& a, cudaStream_t s);
cudaError_t launch_step2_persistent(int precision, const Step2Launch& a, cudaStream_t s);
int persistent_blocks2(int precision, int threads);  // resident blocks of the persistent kernel
}
namespace exact {
cudaError_t launch_step2(int precision, const Step2Launch& a, cudaStream_t s);
cudaError_t launch_step2_persistent(int precision, const Step2Launch& a, cudaStream_t s);
int persistent_blocks2(int precision, int threads);
}

struct AuxLaunch2 {
  int W, H, N;
  int left, right, bottom, top;
  int forcing;
  double fx, fy;
};

// flagsShader (src/shaders/aux.ts:22-88): flags with force slots from *counter (zeroed first) and
// the refill of uncovered cells from mac.
cudaError_t launch_flags2(int precision, const AuxLaunch2& a, const float* sdf, uint32_t* flags, void* fA, void* fB,
                          const float4* mac, unsigned* counter, cudaStream_t s);
// initShader (src/shaders/aux.ts:92-111): both buffers to feq(rho, ux, uy) of mac.
cudaError_t launch_init2(int precision, const AuxLaunch2& a, const float4* mac, void* fA, void* fB, cudaStream_t s);
// macroShader (src/shaders/aux.ts:115-140); sets status bit 1 on a non-finite value.
cudaError_t launch_macro2(int precision, const AuxLaunch2& a, const void* f, const uint32_t* flags, float4* mac,
                          DevState2* st, cudaStream_t s);
// sum(rho) over fluid cells in f64, per-block partials then one ordered sum.
cudaError_t launch_mass2(int precision, const AuxLaunch2& a, const void* f, const uint32_t* flags, double* partials,
                         int nPartials, double* out, cudaStream_t s);
// brushShader (src/shaders/aux.ts:177-194) over the box [x0, x0 + w) x [y0, y0 + h).
cudaError_t launch_brush2(float* sdf, int W, int H, float cx, float cy, float r, int erase, int x0, int y0, int w,
                          int h, cudaStream_t s);
// Writes parts of a tunnel's device state: bit 0 both step counters, bit 1 both inlet speeds,
// bit 2 clears the force sample counter, bit 3 clears the status word.
cudaError_t launch_set_state2(DevState2* st, int which, unsigned step, double uIn, cudaStream_t s);

}  // namespace cells
