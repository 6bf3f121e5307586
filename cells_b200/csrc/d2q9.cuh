// D2Q9 lattice constants and the device-side tunnel descriptor of the 2D engine.
//
// Lattice: src/lattice.ts:2-33 (velocity set, OPP, MIRROR_Y, TRT pairs (1,3) (2,4) (5,7) (6,8), flag
// bits 9-11 and the force-slot field from bit 12, the X/Y boundary modes).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cells {

constexpr int Q2 = 9;
constexpr uint32_t FLAG2_SOLID = 1u << 9;
constexpr uint32_t FLAG2_INLET = 1u << 10;
constexpr uint32_t FLAG2_OUTLET = 1u << 11;
constexpr int BIDX2_SHIFT = 12;
constexpr int HISTORY2_LEN = 8192;  // src/shaders/aux.ts:4

// XMode / YMode (src/lattice.ts:17-28)
constexpr int X2_PERIODIC = 0, X2_WALL = 1, X2_OPEN = 2;
constexpr int Y2_PERIODIC = 0, Y2_NOSLIP = 1, Y2_SLIP = 2, Y2_MOVING = 3;

__host__ __device__ __forceinline__ constexpr int cx2(int i) {
  constexpr int v[Q2] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
  return v[i];
}
__host__ __device__ __forceinline__ constexpr int cy2(int i) {
  constexpr int v[Q2] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
  return v[i];
}
__host__ __device__ __forceinline__ constexpr int opp2(int i) {
  constexpr int v[Q2] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
  return v[i];
}
__host__ __device__ __forceinline__ constexpr int mirror_y2(int i) {
  constexpr int v[Q2] = {0, 1, 4, 3, 2, 8, 7, 6, 5};
  return v[i];
}
// 4/9, 1/9, 1/36: the WGSL literals of the JS doubles, rounded to R
template <class R>
__host__ __device__ __forceinline__ R w2(int i) {
  return i == 0 ? (R)(4.0 / 9.0) : (i <= 4 ? (R)(1.0 / 9.0) : (R)(1.0 / 36.0));
}

// Per-tunnel device state. step[] and uIn[] are double-buffered by parity: the step of parity p
// reads slot p, and the tunnel's first tile writes slot p^1 for the next step.
struct DevState2 {
  unsigned int step[2];
  unsigned int sample;  // force samples written so far (the reference's histState)
  unsigned int done;    // tiles finished in the current sampled step
  unsigned int status;  // bit 0: non-finite force sample, bit 1: non-finite macro value
  unsigned int pad[3];
  double uIn[2];
};

// Index of each float parameter in Tunnel2::pf / pd (Params, src/shaders/common.ts:14-22).
enum Param2 : int {
  P2_TAU = 0,
  P2_LAMBDA,
  P2_SMAGC2,
  P2_SPONGE_START,
  P2_TAU_SPONGE,
  P2_ULID,
  P2_FX,
  P2_FY,
  P2_ABSORB,
  P2_INLET_LAYER,
  P2_COUNT
};

// One tunnel of a batch, as the step kernel sees it. A batch of one is the reference's Solver.
struct Tunnel2 {
  void* f[2];             // populations A and B (storage type), f[i * N + x + W * y]
  const uint32_t* flags;  // N
  const float* sdf;       // N
  double2* partials;      // one force partial per tile
  double2* history;       // HISTORY2_LEN force samples
  DevState2* st;
  // per x, in the arithmetic type (float4 or double4): omega+ without Smagorinsky (the sponge's
  // 1 / mix(tau, tauSponge, sOut)), omega- for that omega+, the absorbing strength sigma, and
  // 1 / omega+ -- filled on the host with the kernel's own expressions (src/shaders/step.ts:48-63,
  // :215-223), so the step reads them instead of evaluating two smoothsteps and four divisions per cell
  const void* xtab;
  int W, H;
  int tilesX, nTiles;     // tiles of this tunnel (tile = one block's cells)
  int firstTile;          // index of its first tile in the batch
  int left, right, bottom, top;
  int parabolic, forcing;
  int forceEvery;
  int rampKind, rampEvery;
  double rampTarget, rampSteps;
  float pf[P2_COUNT];     // parameters rounded to f32 (f32 arithmetic)
  double pd[P2_COUNT];    // the same in f64 (f64 arithmetic)
};

}  // namespace cells
