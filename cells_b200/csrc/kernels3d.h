// Host-visible declarations of the 3D kernels' launchers (implemented in step3d.cu and aux3d.cu).
#pragma once

#include "d3q19.cuh"

namespace cells {

// How a body cell obtains population i (pullSlow3, src/shaders/step3d.ts:119-168, resolved once
// per SDF): the value and the momentum exchange follow from one or two source elements.
enum LinkKind3 : uint8_t {
  LINK_LOAD = 0,        // v = f[e1]: plain pull, outlet copy, edge bounce-back, mirror from a fluid node
  LINK_SLIP_SOLID = 1,  // v = fj = f[e1]; force += c_j * (2 fj): a body meets a slip face
  LINK_BOUZIDI_N = 2,   // fj = f[e1], v = c1 fj + c2 f[e2] (q < 1/2, fluid node behind): c1 = 2q, c2 = 1 - 2q
  LINK_BOUZIDI_0 = 3,   // v = fj = f[e1] (q < 1/2, no fluid node behind)
  LINK_BOUZIDI_H = 4    // fj = f[e1], v = fj / c1 + c2 f[e2] (q >= 1/2): c1 = 2q, c2 = (2q - 1) / (2q)
};

// One link: the element indices (population * N + cell) of its sources and its coefficients in the
// arithmetic type R. e2 equals e1 for links with a single source. 32 bytes, two 16-byte loads.
template <class R>
struct alignas(16) Link3 {
  long long e1, e2;
  R c1, c2;
};
static_assert(sizeof(Link3<float>) == 32 && sizeof(Link3<double>) == 32, "link records are 32 bytes");

// Link tables of the body cells: records [direction 1..18][body cell], and per body cell the 18
// link kinds packed 3 bits each (direction i at bit 3 (i - 1)) and x with the inlet/outlet marks.
struct BodyLinks3 {
  void* rec;                   // Link3<R>[18 * cap]
  unsigned long long* kinds;  // [cap]
  int* meta;                   // [cap]: x | 1 << 29 (outlet) | 1 << 30 (inlet)
  int cap;                     // capacity in body cells
};

struct StepLaunch3 {
  const void* src;
  void* dst;
  const uint32_t* flags;
  const float* sdf;
  const uint8_t* rowBody;
  const void* xTab;
  BodyLinks3 links;
  const int* bodyCells;  // sorted cell indices handled by the body kernel
  double4* partials;     // one per body block
  double4* history;
  DevState3* st;
  long long N;
  int W, H, D;
  int tileTX, tileTY;  // interior tile of the step kernel: tileTY rows of tileTX cells
  int pairTiles;       // f32 / 16-bit storage with an even width: two cells per thread
  int absorbX0;        // first x of the absorbing layer (W when it is off): interior tiles before
                       // it compile without the absorbing sources
  int nBody;
  int rampKind, rampEvery;
  double rampTarget, rampSteps;
  double lambda, smagC2;
  int par, sample;
};

// One time step: one launch of the step kernel. precision: cells_precision (0 f32, 1 f16, 2 bf16,
// 3 f64). fast: FMA contraction allowed; exact: no contraction, every operation rounds as written.
namespace fast {
cudaError_t launch_step3(int precision, const StepLaunch3& a, cudaStream_t s);
int body_blocks3(int nBody);
}
namespace exact {
cudaError_t launch_step3(int precision, const StepLaunch3& a, cudaStream_t s);
int body_blocks3(int nBody);
}

struct AuxLaunch3 {
  int W, H, D, N;
  double uIn;   // inflow speed for init / refill fallback
};

// flags3dShader (src/shaders/aux3d.ts:20-101): flags, refill of uncovered cells from mac, and the
// body-row marks (rowBody must be zeroed first).
cudaError_t launch_flags3(int precision, const AuxLaunch3& a, const float* sdf, uint32_t* flags, uint8_t* rowBody,
                          void* fA, void* fB, const float4* mac, cudaStream_t s);
// The body cells of the rows marked in rowBody, in increasing index order: counts per row (H * D
// ints), then, from the host's exclusive scan of the counts, the cells themselves.
cudaError_t launch_body_count3(int W, int nRows, const uint8_t* rowBody, const uint32_t* flags, int* counts,
                               cudaStream_t s);
cudaError_t launch_body_write3(int W, int nRows, const uint8_t* rowBody, const uint32_t* flags, const int* offsets,
                               int* cells, cudaStream_t s);
// Resolves the 18 pulls of each listed body cell into link records (run after the flags pass).
cudaError_t launch_links3(int precision, const AuxLaunch3& a, const int* cells, int n, const uint32_t* flags,
                          const float* sdf, const BodyLinks3& L, cudaStream_t s);
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
cudaError_t launch_set_state3(int precision, DevState3* st, int which, unsigned step, double uIn0, double uIn1,
                              cudaStream_t s);

}  // namespace cells
