// Host state of a Solver3D handle, shared by the solver (solver3d.cu) and its discrete adjoint
// (adjoint3d.cu).
//
// Mirrors class Solver3D, src/solver3d.ts:42-320: buffers, parameter derivation (writeParams
// :197-208), host bookkeeping (:48-54) and the force ring's read window.
#pragma once

#include <cmath>
#include <deque>
#include <memory>
#include <string>
#include <vector>

#include "../../include/cells.h"
#include "device.h"
#include "kernels3d.h"

struct Adjoint3D;  // adjoint3d.cu

struct Cells3D : cells::HandleBase {
  cells::Device dev;
  Cells3DConfig cfg{};
  int W = 0, H = 0, D = 0;
  long long N = 0;
  int prec = 0;
  size_t bpp = 4;  // bytes per stored population
  int bx = 128, by = 1;  // interior tile of the step kernel: by rows of bx cells
  int pairTiles = 0;     // two cells per thread (f32 or 16-bit storage, even width)
  int absorbX0 = -1;     // first x of the absorbing layer (W when there is none), from the x table

  void* f[2] = {nullptr, nullptr};
  uint32_t* flags = nullptr;
  float* sdf = nullptr;
  uint8_t* rowBody = nullptr;
  void* xTab = nullptr;
  int* bodyCells = nullptr;  // capacity N
  double4* partials = nullptr;  // one per body block
  double4* history = nullptr;
  cells::DevState3* st = nullptr;
  float4* macro = nullptr;
  double* massPartials = nullptr;
  double* massOut = nullptr;
  int nMassPartials = 0;

  // host bookkeeping (src/solver3d.ts:48-54)
  int64_t step = 0;
  int parity = 0;
  uint64_t forceSamplesRead = 0;
  std::deque<uint32_t> forceSteps;
  uint64_t forceGeneration = 0;
  int nBody = 0;
  cells::BodyLinks3 links{};

  // inlet
  double uIn = 0.0;
  int rampKind = 0;
  double rampTarget = 0.0;
  int64_t rampSteps = 1, rampEvery = 1;

  // staging for readForces
  double4* stageHist = nullptr;  // pinned, HISTORY_LEN entries
  unsigned* stageState = nullptr;
  bool readPending = false;
  uint64_t readGeneration = 0;
  uint64_t readFirst = 0, readWritten = 0;

  double fakeForce[3] = {0, 0, 0};

  // the discrete adjoint's recorded forward run (checkpoints, link tables), when one exists
  std::unique_ptr<Adjoint3D> adj;
  // device memory the adjoint keeps between recorded runs: the checkpoints, the two sets of
  // recomputed states and the two adjoint states, carved from one block that a later run reuses
  // while it fits (freed by cells3d_adjoint_release or destroy)
  void* adjStore = nullptr;
  size_t adjStoreBytes = 0;
  // one device block for the recorded run's tables and small buffers, grown to a run's needs when
  // its tables are built and kept for the next run while they fit
  void* adjTab = nullptr;
  size_t adjTabBytes = 0;

  // device scratch of the macro-field products (fields3d.cu), grown on demand
  void* scratch = nullptr;
  size_t scratchBytes = 0;
  void* scratch_buffer(size_t bytes);

  double lambda_value() const {
    if (std::isnan(cfg.lambda)) return std::fmin(3.0 / 16.0, 50.0 * (cfg.tau - 0.5) * (cfg.tau - 0.5));
    return cfg.lambda;
  }
  double sponge_start() const { return cfg.sponge_fraction > 0 ? (W - 1) * (1 - cfg.sponge_fraction) : 1e9; }
  double tau_sponge() const { return std::fmax(cfg.sponge_tau, cfg.tau); }
  double ramp_speed(int64_t s) const {
    const int64_t q = (s / rampEvery) * rampEvery;
    const double t = std::fmin(1.0, (double)q / (double)rampSteps);
    return rampKind == 1 ? rampTarget * t : rampTarget * (t * t * (3.0 - 2.0 * t));
  }
  double current_uin() const { return rampKind ? ramp_speed(step) : uIn; }
  // the inlet speed of the step that starts at step s
  double uin_at(int64_t s) const { return rampKind ? ramp_speed(s) : uIn; }

  // CUDA graphs of kGraphSteps steps, one per phase of the launch-argument period; argGen counts
  // changes of the arguments the graphs bake in (parameters, ramp, body links), so a stale graph is
  // rebuilt on its next use. CELLS_GRAPHS=0 in the environment launches every step directly.
  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    uint64_t gen = 0;
    int launches = 0;
  };
  static constexpr int kGraphSteps = 128;
  static constexpr int kMaxGraphPeriod = 16;
  std::vector<StepGraph> graphs = std::vector<StepGraph>(kMaxGraphPeriod);
  uint64_t argGen = 1;
  bool useGraphs = true;

  Cells3D();
  ~Cells3D();
  void choose_launch();
  void upload_xtab();
  void rebuild_flags();
  void build_body_list();
  int enqueue_step(int par, bool sample, cudaStream_t main);
  // one step from src to dst (any buffers of 19 N populations), parity par of the device state, on
  // `stream` (nullptr: the handle's stream)
  void enqueue_step_between(const void* src, void* dst, int par, bool sample, cudaStream_t stream = nullptr);
  int graph_period() const;
  void build_graph(int phase);
  void launch_steps(int64_t n);
  void prepare_steps(int64_t n);
  void write_state(int which);
  void free_all();
};
