// Discrete adjoint of the D3Q19 step (no counterpart in the reference): the recorded forward run
// and the buffers of the backward sweep.
//
// The forward map of one step is f^{n+1} = C(P(f^n)): P pulls every population (a plain copy from
// the upstream node, or at boundaries a combination of one or two source elements: outlet copy,
// bounce-back, slip mirror, Bouzidi interpolation with link fraction q from the SDF), C collides
// each cell (TRT with sponge and absorbing layer; the inlet stores feq(1, u_n); the outlet stores
// feq(1, u)). The objective is J = scale * mean_{n in window} F_c(n), F the momentum-exchange force.
// The backward sweep runs lambda^n = P^T (dC/dg)^T lambda^{n+1} + dJ_n/df^n from lambda^T down to
// lambda^0 over states recomputed segment by segment from checkpoints taken every K steps, and
// accumulates dJ/dq per Bouzidi link (then dJ/dsdf) and dJ/du_n per step (then dJ/du_in).
#pragma once

#include <cstdint>
#include <vector>

#include "kernels3d.h"

// A resolved pull of a flagged fluid cell's direction: g = a1 f[e1] + a2 f[e2] (e2 < 0: one source).
// Force links add cF (fj + g) to the objective's force component, fj = f[ej] with ej = e1.
struct AdjLink3Host {
  long long e1, e2;
  double a1, a2;
  double cF;      // c_{j, component} for force links (Bouzidi, slip face meeting a solid), else 0
  int qKind;      // 0: g does not depend on q; 1: q < 1/2 with a fluid node behind; 2: q >= 1/2
  double q;       // link fraction in the arithmetic type, for dg/dq
  double dqdF, dqdS;  // dq/dsdf at the cell and at the solid node (0 where q is clamped)
  int cell, solid;    // node indices of the SDF values q reads
};

struct Adjoint3D {
  // recorded run
  int64_t s0 = 0;         // step count when the recorded forward run started
  int64_t steps = 0;
  int64_t w0 = 0, w1 = 0;  // objective window (inclusive step labels)
  int K = 100;
  int component = 0;
  double scale = 1.0;
  double objective = 0.0;
  int parity0 = 0;
  uint64_t argGen = 0;     // the handle's argument generation at record time
  int64_t endStep = 0;     // the handle's step after the recorded run
  std::vector<double> uStep;    // inlet speed of each recorded step
  std::vector<double> rampStep; // d u_n / d u_in of each recorded step

  // checkpoints: the populations and device state at the start of every segment
  std::vector<void*> ck;       // into the handle's adjStore
  std::vector<void*> ckState;  // into ckStateBlock
  cells::DevState3* ckStateBlock = nullptr;
  void* endState = nullptr;  // device state after the run (restored after the backward sweep)
  std::vector<void*> seg[2];  // two sets of K recomputed states: the segment being swept and the next

  // link tables (device)
  int nLinks = 0;
  std::vector<AdjLink3Host> hostLinks;
  int* linkBase = nullptr;      // N: first link of a flagged fluid cell, -1 otherwise
  long long* le1 = nullptr;
  long long* le2 = nullptr;
  void* la1 = nullptr;          // R
  void* la2 = nullptr;          // R
  void* lcF = nullptr;          // R
  void* lq = nullptr;           // R
  signed char* lqk = nullptr;
  void* lamG = nullptr;         // R, the adjoint of each link's pulled value in the current step
  double* dqAcc = nullptr;      // dJ/dq per link, summed over the steps

  // transposed map: elements with irregular readers or no regular reader
  int nRows = 0;
  long long* rowElem = nullptr;
  unsigned char* rowSet = nullptr;  // 1: the element has no regular reader (its adjoint is set, not added)
  int* rowStart = nullptr;          // nRows + 1
  int* entLink = nullptr;
  void* entAlpha = nullptr;         // R
  void* rowPhi = nullptr;           // R: sum of cF of the force links whose fj is this element

  // adjoint state
  void* lam[2] = {nullptr, nullptr};  // R, 19 N each
  double* blockPart = nullptr;
  unsigned* counter = nullptr;
  double* dudn = nullptr;            // dJ/du_n per recorded step
  int nBlocks = 0;  // blocks of the cell kernel
  int tileX = 128;
  double* uDev = nullptr;    // inlet speed of each recorded step (device)
  double* wDev = nullptr;    // objective weight of each recorded step (device)
  int* n0Dev = nullptr;      // first step of the segment being swept (device)
  int* n0Host = nullptr;     // pinned, one slot per segment (the source of each n0Dev copy)
  size_t n0Cap = 0;          // slots n0Host holds
  // device buffers of this run: carved from the handle's adjTab block while it has room (tabUsed
  // bytes taken), else allocated on their own (own, freed with the run); tabNeed is the total
  size_t tabUsed = 0, tabNeed = 0;
  std::vector<void*> own;
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaStream_t side2 = nullptr;          // the next segment's recompute, beside the sweep
  cudaEvent_t fork2 = nullptr, join2 = nullptr;
  // full segments replay captured graphs: [state set of the swept segment][with the next recompute]
  cudaGraphExec_t segGraph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int64_t segGraphLaunches[2][2] = {{0, 0}, {0, 0}};
  int segGraphCur = -1;                 // the adjoint buffer the graphs start from
  int* slowCells = nullptr;  // flagged fluid cells (device), in index order
  int nSlow = 0;
  int* sE1 = nullptr;        // [19][nSlow] pull records of the flagged cells
  int* sE2 = nullptr;
  int* sTgt = nullptr;
  void* sA1 = nullptr;       // R
  void* sA2 = nullptr;       // R
  int nParts = 0;            // entries of blockPart
};

namespace cells {

struct AdjLaunch3 {
  const void* f;         // f^n (storage type == arithmetic type: f32 or f64)
  const void* lamNext;   // lambda^{n+1}
  void* lamOut;          // lambda^n
  const uint32_t* flags;
  const void* xTab;      // per x: omega+, omega-, sigma, 0
  const int* linkBase;
  const long long* le1;
  const long long* le2;
  const void* la1;
  const void* la2;
  const void* lcF;
  const void* lq;
  const signed char* lqk;
  void* lamG;
  double* dqAcc;
  double* blockPart;
  unsigned* counter;
  const int* n0Dev;      // first recorded step of the current segment (device)
  int t;                 // this step's position in the segment: step n = *n0Dev + t
  const double* uDev;    // inlet speed of each recorded step
  const double* wDev;    // objective weight of each recorded step's force
  double* dudn;          // dJ/du_n of each recorded step
  long long N;
  int W, H, D;
  int tileX;             // cell kernel block: tileX x (kAdjThreads / tileX) cells of x-rows
  int absorbX0;          // first x of the absorbing layer (W when there is none)
  int nCellBlocks;       // blocks of the cell kernel
  const int* slowCells;  // the flagged fluid cells, in index order
  int nSlow;
  const int* sE1;        // [19][nSlow]: the source of a one-source pull (coefficient 1), or the first
                         // of two sources with the sign bit set (then sE2, sA1, sA2 apply)
  const int* sE2;
  const int* sTgt;       // [19][nSlow]: element of a plain pull's adjoint, or -(link + 1)
  const void* sA1;       // R: coefficients (a2 = 0 for one source)
  const void* sA2;
  int nParts;            // blockPart entries: nCellBlocks + blocks of the flagged-cell kernel
  // transposed map
  int nRows;
  const long long* rowElem;
  const unsigned char* rowSet;
  const int* rowStart;
  const int* entLink;
  const void* entAlpha;
  const void* rowPhi;
};

constexpr int kAdjThreads = 128;
// One adjoint step (precision 0 or 3): the interior-cell kernel on `s` and the flagged-cell kernel
// on `side` run concurrently (they write disjoint elements), then the boundary-element kernel on
// `s`. fork and join are events used to order the two streams.
cudaError_t launch_adjoint_step3(int precision, const AdjLaunch3& a, cudaStream_t s, cudaStream_t side,
                                 cudaEvent_t fork, cudaEvent_t join);

}  // namespace cells
