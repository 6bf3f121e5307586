// Solver (D2Q9) host state: batches of independent 2D tunnels and the 2D half of the C ABI
// (include/cells.h).
//
// Mirrors class Solver, src/solver.ts:50-340: buffers, parameter derivation (writeParams
// :180-197), setSdf / rebuildFlags (:200-217), initField (:219-234), resetForces (:236-241),
// brush (:243-268), encodeSteps (:270-286), run (:294-307), readMacro (:309-311) and readForces with
// its ring window and generation check (:314-335). A batch holds many tunnels; one kernel launch
// steps them all (src has no batches: they are this engine's addition). Each tunnel's parameters
// live in a device-side descriptor that the kernel reads every step, so parameter changes need no
// graph rebuild; the inlet speed and step counter live in per-tunnel device state.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <deque>
#include <string>
#include <vector>

#include "../../include/cells.h"
#include "device.h"
#include "kernels2d.h"

using namespace cells;

namespace {

constexpr int kGraphSteps2 = 100;
constexpr int kPersistentChunk = 500;

struct Shape2 {
  int tx, ty;
};
// launch shapes the autotuner tries: 64, 128 and 256 threads, rows of 32 to 256 cells
const Shape2 kShapes[] = {{32, 2}, {64, 1}, {32, 4}, {64, 2}, {128, 1}, {32, 8}, {64, 4}, {128, 2}, {256, 1}};

struct Tunnel2Host {
  Cells2DConfig cfg{};
  int W = 0, H = 0;
  long long N = 0;
  void* f[2] = {nullptr, nullptr};
  uint32_t* flags = nullptr;
  float* sdf = nullptr;
  float4* macro = nullptr;
  double2* partials = nullptr;
  int partialsCap = 0;
  double2* history = nullptr;
  DevState2* st = nullptr;
  void* xtab = nullptr;  // W entries of 4 values in the arithmetic type (Tunnel2::xtab)
  int tilesX = 0, nTiles = 0, firstTile = 0;

  // host bookkeeping (src/solver.ts:57-61)
  int64_t step = 0;
  uint64_t forceSamplesRead = 0;
  std::deque<uint32_t> forceSteps;
  uint64_t forceGeneration = 0;

  int rampKind = 0;
  double rampTarget = 0.0;
  int64_t rampSteps = 1, rampEvery = 1;

  double2* stageHist = nullptr;  // pinned
  unsigned* stageState = nullptr;  // pinned, 64 bytes
  bool readPending = false;
  uint64_t readGeneration = 0, readFirst = 0, readWritten = 0;
  double fakeForce[2] = {0.0, 0.0};

  double ramp_speed(int64_t s) const {
    const int64_t q = (s / rampEvery) * rampEvery;
    const double t = std::fmin(1.0, (double)q / (double)rampSteps);
    return rampKind == 1 ? rampTarget * t : rampTarget * (t * t * (3.0 - 2.0 * t));
  }
  double current_uin() const { return rampKind ? ramp_speed(step) : cfg.u_in; }
  double sponge_start() const { return cfg.sponge_fraction > 0 ? (W - 1) * (1 - cfg.sponge_fraction) : 1e9; }
  double tau_sponge() const { return std::fmax(cfg.sponge_tau, cfg.tau); }
  int forcing() const { return (cfg.body_force[0] != 0.0 || cfg.body_force[1] != 0.0) ? 1 : 0; }
};

void validate_config(const Cells2DConfig& c) {
  if (c.width < 2 || c.height < 1) throw Error(CELLS_E_INVALID, "grid must be at least 2 x 1");
  if ((long long)c.width * c.height > 0x7fffffffLL / 9) throw Error(CELLS_E_INVALID, "grid has too many cells");
  if (c.precision != CELLS_FP32 && c.precision != CELLS_FP64)
    throw Error(CELLS_E_PRECISION_UNSUPPORTED,
                "precision " + std::to_string(c.precision) + " is not available for the 2D solver (FP32 or FP64)");
  if (!(c.tau > 0.5)) throw Error(CELLS_E_INVALID, "tau must be above 1/2");
  if (c.left < 0 || c.left > 2 || c.right < 0 || c.right > 2) throw Error(CELLS_E_INVALID, "unknown x boundary mode");
  if (c.bottom < 0 || c.bottom > 3 || c.top < 0 || c.top > 3) throw Error(CELLS_E_INVALID, "unknown y boundary mode");
  if (c.force_every < 0) throw Error(CELLS_E_INVALID, "force_every must be >= 0");
  if (c.workgroup_size != 0 && c.workgroup_size != 64 && c.workgroup_size != 128 && c.workgroup_size != 256)
    throw Error(CELLS_E_INVALID, "workgroup_size must be 0, 64, 128 or 256");
}

}  // namespace

struct Cells2DBatch : HandleBase {
  Device dev;
  int prec = 0;
  int arithmetic = 0;
  size_t bpp = 4;
  std::vector<Tunnel2Host> t;
  std::vector<Cells2D*> views;
  int parity = 0;

  // launch layout
  int tileX = 32, tileY = 4;
  int rows = 1;  // cell rows per thread of the step kernel
  int persistent = 0;
  int persistentBlocks = 0;
  int nTiles = 0;
  int maxTiles = 0;
  Tunnel2* dTunnels = nullptr;
  unsigned short* dTileTunnel = nullptr;
  unsigned* dBarrier = nullptr;
  int* dError = nullptr;
  unsigned* dCounter = nullptr;
  double* massPartials = nullptr;
  double* massOut = nullptr;
  int nMassPartials = 4 * 148;
  uint64_t layoutGen = 1;
  bool useGraphs = true;
  unsigned barrierErrors = 0;
  unsigned barrierExtra = 0;  // test hook: arrivals a persistent launch waits for that never come

  struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    uint64_t gen = 0;
  };
  StepGraph graphs[2][2];  // [allowSample][starting parity]

  void set_layout(int tx, int ty, int pers);
  void upload_tunnel(int k);
  void write_state(int k, int which);
  void rebuild_flags(int k);
  AuxLaunch2 aux(int k) const;
  void launch_raw(int64_t n, int par, int allowSample);
  void launch_steps(int64_t n);
  void advance(int64_t n);
  void build_graph(int allowSample, int par);
  void check_barrier();
  void free_all();
};

struct Cells2D : HandleBase {
  Cells2DBatch* b = nullptr;
  int k = 0;
  bool owner = false;
  Tunnel2Host& T() { return b->t[(size_t)k]; }
};

AuxLaunch2 Cells2DBatch::aux(int k) const {
  const Tunnel2Host& T = t[(size_t)k];
  AuxLaunch2 a;
  a.W = T.W;
  a.H = T.H;
  a.N = (int)T.N;
  a.left = T.cfg.left;
  a.right = T.cfg.right;
  a.bottom = T.cfg.bottom;
  a.top = T.cfg.top;
  a.forcing = T.forcing();
  a.fx = T.cfg.body_force[0];
  a.fy = T.cfg.body_force[1];
  return a;
}

// Tiles of every tunnel for a tile shape, numbered tunnel by tunnel, and the tile -> tunnel map.
void Cells2DBatch::set_layout(int tx, int ty, int pers) {
  tileX = tx;
  tileY = ty;
  persistent = pers;
  // two cell rows per thread (both rows' loads in flight together) when the batch is large enough
  // to fill the GPU with the halved block count; small grids keep one row and twice the blocks
  long long tiles1 = 0;
  for (const Tunnel2Host& T : t) tiles1 += (long long)((T.W + tx - 1) / tx) * ((T.H + ty - 1) / ty);
  rows = tiles1 >= 4096 ? 2 : 1;
  std::vector<unsigned short> map;
  int first = 0;
  for (size_t k = 0; k < t.size(); k++) {
    Tunnel2Host& T = t[k];
    T.tilesX = (T.W + tx - 1) / tx;
    T.nTiles = T.tilesX * ((T.H + rows * ty - 1) / (rows * ty));
    if (T.nTiles > T.partialsCap) throw Error(CELLS_E_INVALID, "tile shape needs more force partials than allocated");
    T.firstTile = first;
    first += T.nTiles;
    map.insert(map.end(), (size_t)T.nTiles, (unsigned short)k);
  }
  if (first > maxTiles) throw Error(CELLS_E_INVALID, "tile shape needs more tiles than allocated");
  nTiles = first;
  if (!dev.fake) {
    dev.h2d(dTileTunnel, map.data(), map.size() * sizeof(unsigned short));
    dev.sync();
    persistentBlocks = arithmetic == CELLS_ARITH_EXACT ? exact::persistent_blocks2(prec, tx * ty)
                                                       : fast::persistent_blocks2(prec, tx * ty);
    if (persistent && persistentBlocks <= 0) throw Error(CELLS_E_CUDA, "persistent kernel cannot be resident");
  }
  for (size_t k = 0; k < t.size(); k++) upload_tunnel((int)k);
  layoutGen++;
}

// The per-x rates of a tunnel (Tunnel2::xtab) in the arithmetic type R, by the step kernel's
// expressions for the sponge, inlet layer and TRT rates (src/shaders/step.ts:48-63, :215-223) in the
// same operation order, so the values equal what the kernel computed per cell before.
template <class R>
static void fill_xtab2(std::vector<R>& t, int W, const double* p) {
  const R tau = (R)p[P2_TAU], lam = (R)p[P2_LAMBDA], ss = (R)p[P2_SPONGE_START], ts = (R)p[P2_TAU_SPONGE];
  const R ab = (R)p[P2_ABSORB], il = (R)p[P2_INLET_LAYER];
  auto smooth = [](R e0, R e1, R x) {
    R u = (x - e0) / (e1 - e0);
    u = u < R(0) ? R(0) : (R(1) < u ? R(1) : u);
    return u * u * (R(3) - R(2) * u);
  };
  t.assign((size_t)W * 4, R(0));
  for (int x = 0; x < W; x++) {
    R omegaBase = R(1) / tau;
    R sOut = R(0);
    if (ss < R(W - 1)) {
      sOut = smooth(ss, R(W - 1), R(x));
      omegaBase = R(1) / (tau * (R(1) - sOut) + ts * sOut);
    }
    R sIn = R(0);
    if (il > R(0)) sIn = R(1) - smooth(R(0), il, R(x));
    const R sOut2 = sOut * sOut, sIn2 = sIn * sIn;
    t[4 * (size_t)x] = omegaBase;
    t[4 * (size_t)x + 1] = R(1) / (R(0.5) + lam / (R(1) / omegaBase - R(0.5)));
    t[4 * (size_t)x + 2] = ab * (sOut2 < sIn2 ? sIn2 : sOut2);
    t[4 * (size_t)x + 3] = R(1) / omegaBase;
  }
}

// The tunnel's descriptor, with every parameter derived as writeParams does (src/solver.ts:180-197)
// and rounded once into f32 (and kept in f64 for f64 arithmetic).
void Cells2DBatch::upload_tunnel(int k) {
  Tunnel2Host& T = t[(size_t)k];
  Tunnel2 d;
  std::memset(&d, 0, sizeof(d));
  d.f[0] = T.f[0];
  d.f[1] = T.f[1];
  d.flags = T.flags;
  d.sdf = T.sdf;
  d.partials = T.partials;
  d.history = T.history;
  d.st = T.st;
  d.xtab = T.xtab;
  d.W = T.W;
  d.H = T.H;
  d.tilesX = T.tilesX;
  d.nTiles = T.nTiles;
  d.firstTile = T.firstTile;
  d.left = T.cfg.left;
  d.right = T.cfg.right;
  d.bottom = T.cfg.bottom;
  d.top = T.cfg.top;
  d.parabolic = T.cfg.parabolic ? 1 : 0;
  d.forcing = T.forcing();
  d.forceEvery = T.cfg.force_every;
  d.rampKind = T.rampKind;
  d.rampEvery = (int)T.rampEvery;
  d.rampTarget = T.rampTarget;
  d.rampSteps = (double)T.rampSteps;
  double p[P2_COUNT];
  p[P2_TAU] = T.cfg.tau;
  p[P2_LAMBDA] = T.cfg.lambda;
  p[P2_SMAGC2] = T.cfg.smagorinsky * T.cfg.smagorinsky;
  p[P2_SPONGE_START] = T.sponge_start();
  p[P2_TAU_SPONGE] = T.tau_sponge();
  p[P2_ULID] = T.cfg.u_lid;
  p[P2_FX] = T.cfg.body_force[0];
  p[P2_FY] = T.cfg.body_force[1];
  p[P2_ABSORB] = T.cfg.absorb;
  p[P2_INLET_LAYER] = T.cfg.inlet_layer_fraction * (T.W - 1);
  for (int i = 0; i < P2_COUNT; i++) {
    d.pf[i] = (float)p[i];
    d.pd[i] = p[i];
  }
  std::vector<float> tf;
  std::vector<double> td;
  if (prec == CELLS_FP64) {
    fill_xtab2<double>(td, T.W, p);
    dev.h2d(T.xtab, td.data(), td.size() * sizeof(double));
  } else {
    fill_xtab2<float>(tf, T.W, p);
    dev.h2d(T.xtab, tf.data(), tf.size() * sizeof(float));
  }
  if (dev.fake) return;
  dev.h2d(dTunnels + k, &d, sizeof(d));
  dev.sync();  // d and the tables die here
}

void Cells2DBatch::write_state(int k, int which) {
  Tunnel2Host& T = t[(size_t)k];
  if (dev.fake) {
    if (which & 1) T.st->step[0] = T.st->step[1] = (unsigned)T.step;
    if (which & 2) T.st->uIn[0] = T.st->uIn[1] = T.current_uin();
    if (which & 4) T.st->sample = T.st->done = 0;
    if (which & 8) T.st->status = 0;
    return;
  }
  check_cuda(launch_set_state2(T.st, which, (unsigned)T.step, T.current_uin(), dev.stream), "set_state kernel");
  dev.launches++;
}

// rebuildFlags, src/solver.ts:205-217: the macro of the latest populations (the refill reads it),
// then the flags pass with a zeroed slot counter.
void Cells2DBatch::rebuild_flags(int k) {
  if (dev.fake) return;
  Tunnel2Host& T = t[(size_t)k];
  const AuxLaunch2 a = aux(k);
  check_cuda(launch_macro2(prec, a, T.f[parity], T.flags, T.macro, T.st, dev.stream), "macro kernel");
  dev.memset0(dCounter, sizeof(unsigned));
  check_cuda(launch_flags2(prec, a, T.sdf, T.flags, T.f[0], T.f[1], T.macro, dCounter, dev.stream), "flags kernel");
  dev.launches += 2;
}

// n steps from parity par on the device only (no host bookkeeping).
void Cells2DBatch::launch_raw(int64_t n, int par, int allowSample) {
  Step2Launch a;
  a.tunnels = dTunnels;
  a.tileTunnel = dTileTunnel;
  a.nTiles = nTiles;
  a.tileX = tileX;
  a.tileY = tileY;
  a.rows = rows;
  a.allowSample = allowSample;
  a.barrier = dBarrier;
  a.error = dError;
  a.barrierExtra = barrierExtra;
  a.gridBlocks = std::min(nTiles, persistentBlocks);
  const bool ex = arithmetic == CELLS_ARITH_EXACT;
  while (n > 0) {
    if (persistent) {
      const int k = (int)std::min<int64_t>(n, kPersistentChunk);
      a.par = par;
      a.nSteps = k;
      check_cuda(ex ? exact::launch_step2_persistent(prec, a, dev.stream)
                    : fast::launch_step2_persistent(prec, a, dev.stream),
                 "persistent step kernel");
      dev.launches += 1;
      if (k & 1) par ^= 1;
      n -= k;
      continue;
    }
    if (useGraphs && n >= kGraphSteps2) {
      StepGraph& g = graphs[allowSample][par];
      if (!g.exec || g.gen != layoutGen) build_graph(allowSample, par);
      check_cuda(cudaGraphLaunch(g.exec, dev.stream), "cudaGraphLaunch");
      dev.launches += kGraphSteps2;
      n -= kGraphSteps2;  // even: the parity comes back
      continue;
    }
    a.par = par;
    a.nSteps = 1;
    check_cuda(ex ? exact::launch_step2(prec, a, dev.stream) : fast::launch_step2(prec, a, dev.stream), "step kernel");
    dev.launches++;
    par ^= 1;
    n--;
  }
}

void Cells2DBatch::build_graph(int allowSample, int par) {
  static_assert(kGraphSteps2 % 2 == 0, "a graph must end on its starting parity");
  StepGraph& g = graphs[allowSample][par];
  if (g.exec) cudaGraphExecDestroy(g.exec);
  g.exec = nullptr;
  Step2Launch a;
  a.tunnels = dTunnels;
  a.tileTunnel = dTileTunnel;
  a.nTiles = nTiles;
  a.tileX = tileX;
  a.tileY = tileY;
  a.rows = rows;
  a.allowSample = allowSample;
  a.nSteps = 1;
  a.gridBlocks = 0;
  a.barrier = nullptr;
  a.barrierExtra = 0;
  a.error = nullptr;
  const bool ex = arithmetic == CELLS_ARITH_EXACT;
  check_cuda(cudaStreamBeginCapture(dev.stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  int p = par;
  cudaError_t err = cudaSuccess;
  for (int s = 0; s < kGraphSteps2 && err == cudaSuccess; s++) {
    a.par = p;
    err = ex ? exact::launch_step2(prec, a, dev.stream) : fast::launch_step2(prec, a, dev.stream);
    p ^= 1;
  }
  cudaGraph_t graph = nullptr;
  cudaError_t e2 = cudaStreamEndCapture(dev.stream, &graph);
  check_cuda(err, "step kernel (capture)");
  check_cuda(e2, "cudaStreamEndCapture");
  cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  check_cuda(e, "cudaGraphInstantiate");
  g.gen = layoutGen;
}

// Host bookkeeping of n steps of every tunnel (encodeSteps, src/solver.ts:270-286); on the fake
// device it also writes the force samples the kernel would.
void Cells2DBatch::advance(int64_t n) {
  for (int64_t s = 0; s < n; s++) {
    for (Tunnel2Host& T : t) {
      const int every = T.cfg.force_every;
      const bool sample = every > 0 && ((T.step + 1) % every) == 0;
      if (sample && dev.fake) {
        const unsigned c = T.st->sample;
        T.history[c % HISTORY2_LEN] = make_double2(T.fakeForce[0], T.fakeForce[1]);
        T.st->sample = c + 1;
      }
      T.step++;
      if (sample) T.forceSteps.push_back((uint32_t)T.step);
    }
    parity ^= 1;
  }
}

void Cells2DBatch::launch_steps(int64_t n) {
  if (n <= 0) return;
  if (!dev.fake) launch_raw(n, parity, 1);
  advance(n);
}

// A persistent launch whose barrier wait ran out has left its tunnels part-stepped.
void Cells2DBatch::check_barrier() {
  if (dev.fake || !persistent) return;
  int e = 0;
  check_cuda(cudaMemcpy(&e, dError, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy error flag");
  if (e) {
    barrierErrors++;
    // the flag is cleared so that later launches run; the tunnels stay part-stepped until the
    // caller re-initialises them
    dev.memset0(dError, sizeof(int));
    dev.sync();
    throw Error(CELLS_E_TIMEOUT, "a grid barrier of the persistent step kernel timed out");
  }
}

void Cells2DBatch::free_all() {
  for (auto& row : graphs)
    for (auto& g : row) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
  for (Tunnel2Host& T : t) {
    if (T.stageHist) dev.free_host_pinned(T.stageHist);
    if (T.stageState) dev.free_host_pinned(T.stageState);
    T.stageHist = nullptr;
    T.stageState = nullptr;
  }
  dev.close();
}

// ---------------- creation ----------------

static Cells2DBatch* create_batch(const Cells2DConfig* cfgs, int count) {
  if (!cfgs || count <= 0) throw Error(CELLS_E_INVALID, "need at least one config");
  if (count > 65535) throw Error(CELLS_E_INVALID, "at most 65535 tunnels per batch");
  for (int k = 0; k < count; k++) {
    validate_config(cfgs[k]);
    if (cfgs[k].precision != cfgs[0].precision || cfgs[k].device != cfgs[0].device ||
        cfgs[k].arithmetic != cfgs[0].arithmetic)
      throw Error(CELLS_E_INVALID, "tunnels of a batch share precision, device and arithmetic");
  }
  Cells2DBatch* b = new Cells2DBatch();
  b->prec = cfgs[0].precision;
  b->arithmetic = cfgs[0].arithmetic;
  b->bpp = b->prec == CELLS_FP64 ? 8 : 4;
  if (const char* gv = std::getenv("CELLS_GRAPHS")) b->useGraphs = std::atoi(gv) != 0;
  try {
    b->dev.open(cfgs[0].device, cfgs[0].fake_fail_alloc);
    b->t.resize((size_t)count);
    unsigned long long total = 1u << 22;
    for (int k = 0; k < count; k++) {
      Tunnel2Host& T = b->t[(size_t)k];
      T.cfg = cfgs[k];
      T.W = cfgs[k].width;
      T.H = cfgs[k].height;
      T.N = (long long)T.W * T.H;
      const unsigned long long fBytes = 9ull * b->bpp * (unsigned long long)T.N;
      if (cfgs[k].max_buffer_bytes > 0 && fBytes > cfgs[k].max_buffer_bytes)
        throw AllocError("one distribution buffer needs " + std::to_string(fBytes) + " bytes; this device allows " +
                         std::to_string(cfgs[k].max_buffer_bytes) + " per buffer");
      total += 2 * fBytes + (unsigned long long)T.N * (4 + 4 + 16);
    }
    const size_t freeB = b->dev.free_bytes();
    if (total > freeB)
      throw AllocError("the solver needs " + std::to_string(total) + " bytes; this device has " +
                       std::to_string(freeB) + " bytes free");
    int maxTiles = 0;
    for (const Shape2& sh : kShapes) {
      int tiles = 0;
      for (Tunnel2Host& T : b->t) tiles += ((T.W + sh.tx - 1) / sh.tx) * ((T.H + sh.ty - 1) / sh.ty);
      maxTiles = std::max(maxTiles, tiles);
    }
    b->maxTiles = maxTiles;
    for (int k = 0; k < count; k++) {
      Tunnel2Host& T = b->t[(size_t)k];
      const size_t fBytes = 9ull * b->bpp * (size_t)T.N;
      // the step kernel issues every cell's nine fast-path pulls before it knows whether the cell
      // takes them; on the top row direction 8's pull lands up to W - 1 elements past the nine
      // arrays, so each buffer carries W elements of padding (never used as a population)
      const size_t padBytes = (size_t)T.W * b->bpp;
      T.f[0] = b->dev.alloc(fBytes + padBytes, "distribution buffer A");
      T.f[1] = b->dev.alloc(fBytes + padBytes, "distribution buffer B");
      T.flags = (uint32_t*)b->dev.alloc((size_t)T.N * 4, "flags");
      T.sdf = (float*)b->dev.alloc((size_t)T.N * 4, "sdf");
      T.macro = (float4*)b->dev.alloc((size_t)T.N * 16, "macro");
      int cap = 0;
      for (const Shape2& sh : kShapes) cap = std::max(cap, ((T.W + sh.tx - 1) / sh.tx) * ((T.H + sh.ty - 1) / sh.ty));
      T.partialsCap = cap;
      T.partials = (double2*)b->dev.alloc((size_t)cap * sizeof(double2), "force partials");
      T.history = (double2*)b->dev.alloc((size_t)HISTORY2_LEN * sizeof(double2), "force history");
      T.st = (DevState2*)b->dev.alloc(sizeof(DevState2), "state");
      T.xtab = b->dev.alloc((size_t)T.W * 4 * b->bpp, "x table");
      T.stageHist = (double2*)b->dev.host_pinned((size_t)HISTORY2_LEN * sizeof(double2));
      T.stageState = (unsigned*)b->dev.host_pinned(64);
      b->dev.memset0(T.st, sizeof(DevState2));
      b->dev.memset0(T.f[0], fBytes + padBytes);
      b->dev.memset0(T.f[1], fBytes + padBytes);
      b->dev.memset0(T.flags, (size_t)T.N * 4);
      std::vector<float> far((size_t)T.N, 1e6f);  // src/solver.ts:133
      b->dev.h2d(T.sdf, far.data(), far.size() * 4);
      b->dev.sync();
    }
    b->dTunnels = (Tunnel2*)b->dev.alloc((size_t)count * sizeof(Tunnel2), "tunnel descriptors");
    b->dTileTunnel = (unsigned short*)b->dev.alloc((size_t)maxTiles * sizeof(unsigned short), "tile map");
    b->dBarrier = (unsigned*)b->dev.alloc(64, "grid barrier");
    b->dError = (int*)b->dev.alloc(64, "barrier error");
    b->dCounter = (unsigned*)b->dev.alloc(64, "slot counter");
    b->massPartials = (double*)b->dev.alloc((size_t)b->nMassPartials * 8, "mass partials");
    b->massOut = (double*)b->dev.alloc(8, "mass result");
    b->dev.memset0(b->dError, 64);
    // the initial launch shape: 32 x (workgroup_size / 32) threads when a size is given; by default
    // 64 x 2, which the autotuner picked for a single 400 x 100 tunnel (cells2d_batch_autotune
    // retunes a batch for its own sizes)
    const int wg = cfgs[0].workgroup_size;
    if (wg == 0)
      b->set_layout(64, 2, 0);
    else
      b->set_layout(32, wg == 64 ? 2 : (wg == 256 ? 8 : 4), 0);
    for (int k = 0; k < count; k++) {
      b->write_state(k, 1 | 2 | 4 | 8);
      b->rebuild_flags(k);
    }
    b->dev.sync();
  } catch (...) {
    b->free_all();
    delete b;
    throw;
  }
  return b;
}

// ---------------- C ABI ----------------

#define C2_TRY try {
#define C2_CATCH(h, prefix)                                     \
  }                                                             \
  catch (const AllocError& e) {                                 \
    (h)->lastError = std::string(prefix) + e.what();            \
    return CELLS_E_ALLOC;                                       \
  }                                                             \
  catch (const Error& e) {                                      \
    (h)->lastError = e.what();                                  \
    return e.status;                                            \
  }                                                             \
  catch (const std::exception& e) {                             \
    (h)->lastError = e.what();                                  \
    return CELLS_E_INVALID;                                     \
  }                                                             \
  return CELLS_OK;

static const char* kAllocPrefix = "Solver allocation failed: ";

static int create_failed(const std::exception& e, int status) {
  g_create_error = e.what();
  return status;
}

extern "C" {

void cells2d_config_default(Cells2DConfig* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->width = 0;
  c->height = 0;
  c->left = CELLS_X_PERIODIC;
  c->right = CELLS_X_PERIODIC;
  c->bottom = CELLS_Y_PERIODIC;
  c->top = CELLS_Y_PERIODIC;
  c->precision = CELLS_FP32;
  c->parabolic = 0;
  c->tau = 0.6;
  c->lambda = 3.0 / 16.0;
  c->smagorinsky = 0.0;
  c->u_in = 0.0;
  c->u_lid = 0.0;
  c->sponge_fraction = 0.0;
  c->sponge_tau = 1.0;
  c->body_force[0] = c->body_force[1] = 0.0;
  c->absorb = 0.0;
  c->inlet_layer_fraction = 0.0;
  c->workgroup_size = 0;
  c->force_every = 1;
  c->device = 0;
}

int cells2d_batch_create(const Cells2DConfig* cfgs, int32_t count, Cells2DBatch** out) {
  if (!out) return CELLS_E_INVALID;
  *out = nullptr;
  g_create_error.clear();
  try {
    Cells2DBatch* b = create_batch(cfgs, count);
    b->views.resize((size_t)count, nullptr);
    for (int k = 0; k < count; k++) {
      Cells2D* v = new Cells2D();
      v->b = b;
      v->k = k;
      b->views[(size_t)k] = v;
    }
    *out = b;
  } catch (const AllocError& e) {
    g_create_error = std::string(kAllocPrefix) + e.what();
    return CELLS_E_ALLOC;
  } catch (const Error& e) {
    return create_failed(e, e.status);
  } catch (const std::exception& e) {
    return create_failed(e, CELLS_E_INVALID);
  }
  return CELLS_OK;
}

int cells2d_create(const Cells2DConfig* cfg, Cells2D** out) {
  if (!out) return CELLS_E_INVALID;
  *out = nullptr;
  if (!cfg) {
    g_create_error = "config is NULL";
    return CELLS_E_INVALID;
  }
  Cells2DBatch* b = nullptr;
  int rc = cells2d_batch_create(cfg, 1, &b);
  if (rc != CELLS_OK) return rc;
  Cells2D* v = b->views[0];
  v->owner = true;
  *out = v;
  return CELLS_OK;
}

void cells2d_batch_destroy(Cells2DBatch* b) {
  if (!b) return;
  b->free_all();
  for (Cells2D* v : b->views) delete v;
  delete b;
}

void cells2d_destroy(Cells2D* h) {
  if (!h) return;
  if (h->owner) cells2d_batch_destroy(h->b);  // deletes h with the views
}

int cells2d_batch_tunnel(Cells2DBatch* b, int32_t k, Cells2D** out) {
  if (!b || !out) return CELLS_E_INVALID;
  if (k < 0 || k >= (int)b->t.size()) {
    b->lastError = "tunnel index out of range";
    return CELLS_E_INVALID;
  }
  *out = b->views[(size_t)k];
  return CELLS_OK;
}

int cells2d_update(Cells2D* h, const Cells2DConfig* c) {
  if (!h || !c) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  if (c->width != T.cfg.width || c->height != T.cfg.height || c->precision != T.cfg.precision ||
      c->device != T.cfg.device || c->arithmetic != T.cfg.arithmetic)
    throw Error(CELLS_E_INVALID, "update cannot change the grid, precision, device or arithmetic");
  validate_config(*c);
  const bool modes = c->left != T.cfg.left || c->right != T.cfg.right || c->bottom != T.cfg.bottom ||
                     c->top != T.cfg.top;
  const bool uin = c->u_in != T.cfg.u_in;
  T.cfg = *c;
  if (uin) T.rampKind = 0;
  h->b->upload_tunnel(h->k);
  if (uin) h->b->write_state(h->k, 2);
  // the boundary modes enter the flags (src/shaders/aux.ts:33-67); the reference rebuilds them on
  // the next setSdf only, which leaves flags that disagree with the new modes: rebuild now
  if (modes) h->b->rebuild_flags(h->k);
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_get_config(Cells2D* h, Cells2DConfig* c) {
  if (!h || !c) return CELLS_E_INVALID;
  *c = h->T().cfg;
  return CELLS_OK;
}

int cells2d_set_inlet(Cells2D* h, double u) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  T.cfg.u_in = u;
  if (T.rampKind) {
    T.rampKind = 0;
    h->b->upload_tunnel(h->k);
  }
  h->b->write_state(h->k, 2);
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_set_inlet_ramp(Cells2D* h, int kind, double target, int64_t ramp_steps, int64_t update_every) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  if (kind < 0 || kind > 2) throw Error(CELLS_E_INVALID, "unknown ramp kind");
  if (kind != 0 && (ramp_steps <= 0 || update_every <= 0))
    throw Error(CELLS_E_INVALID, "ramp_steps and update_every must be positive");
  Tunnel2Host& T = h->T();
  T.rampKind = kind;
  T.rampTarget = target;
  T.rampSteps = ramp_steps > 0 ? ramp_steps : 1;
  T.rampEvery = update_every > 0 ? update_every : 1;
  if (kind == 0) T.cfg.u_in = target;
  h->b->upload_tunnel(h->k);
  h->b->write_state(h->k, 2);
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_set_sdf(Cells2D* h, const float* sdf, size_t n) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  if (!sdf || n != (size_t)T.N) throw Error(CELLS_E_INVALID, "set_sdf needs W*H floats");
  h->b->dev.h2d(T.sdf, sdf, n * 4);
  h->b->dev.sync();
  h->b->rebuild_flags(h->k);
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_read_sdf(Cells2D* h, float* out, size_t n) {
  if (!h || !out) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  if (n != (size_t)T.N) throw Error(CELLS_E_INVALID, "read_sdf needs W*H floats");
  h->b->dev.d2h(out, T.sdf, n * 4);
  h->b->dev.sync();
  C2_CATCH(h, kAllocPrefix)
}

// the bounding box of brush (src/solver.ts:249-255), then the SDF kernel
static void brush_one(Cells2D* h, double cx, double cy, double r, int erase) {
  Tunnel2Host& T = h->T();
  const int pad = 2;
  const int x0 = std::max(0, (int)std::floor(cx - r - pad));
  const int y0 = std::max(0, (int)std::floor(cy - r - pad));
  const int x1 = std::min(T.W - 1, (int)std::ceil(cx + r + pad));
  const int y1 = std::min(T.H - 1, (int)std::ceil(cy + r + pad));
  if (x1 < x0 || y1 < y0) return;
  if (h->b->dev.fake) {
    for (int y = y0; y <= y1; y++)
      for (int x = x0; x <= x1; x++) {
        const float dx = (float)x - (float)cx, dy = (float)y - (float)cy;
        const float d = std::sqrt(dx * dx + dy * dy) - (float)r;
        float& s = T.sdf[(size_t)y * T.W + x];
        s = erase == 0 ? std::fmin(s, d) : std::fmax(s, -d);
      }
    return;
  }
  check_cuda(launch_brush2(T.sdf, T.W, T.H, (float)cx, (float)cy, (float)r, erase ? 1 : 0, x0, y0, x1 - x0 + 1,
                           y1 - y0 + 1, h->b->dev.stream),
             "brush kernel");
  h->b->dev.launches++;
}

int cells2d_brush(Cells2D* h, double cx, double cy, double r, int erase, int rebuild) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  brush_one(h, cx, cy, r, erase);
  if (rebuild) h->b->rebuild_flags(h->k);
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_brush_stroke(Cells2D* h, const double* xy, size_t n_points, double r, int erase) {
  if (!h || (!xy && n_points)) return CELLS_E_INVALID;
  C2_TRY
  for (size_t p = 0; p < n_points; p++) brush_one(h, xy[2 * p], xy[2 * p + 1], r, erase);
  h->b->rebuild_flags(h->k);
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_init_field(Cells2D* h, const float* macro4n) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  Cells2DBatch* b = h->b;
  Tunnel2Host& T = h->T();
  std::vector<float> rest;
  const float* m = macro4n;
  if (!m) {
    rest.assign((size_t)T.N * 4, 0.0f);
    for (long long i = 0; i < T.N; i++) rest[(size_t)i * 4] = 1.0f;
    m = rest.data();
  }
  b->dev.h2d(T.macro, m, (size_t)T.N * 16);
  if (!b->dev.fake) {
    check_cuda(launch_init2(b->prec, b->aux(h->k), T.macro, T.f[0], T.f[1], b->dev.stream), "init kernel");
    b->dev.launches++;
  }
  b->dev.sync();
  T.step = 0;
  // a new flow clears the divergence status, as recoverFromBlowup's re-init starts over
  b->write_state(h->k, 1 | 2 | 4 | 8);
  T.forceSamplesRead = 0;
  T.forceSteps.clear();
  T.forceGeneration++;
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_reset_forces(Cells2D* h) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  h->b->write_state(h->k, 4);
  T.forceSamplesRead = 0;
  T.forceSteps.clear();
  T.forceGeneration++;
  C2_CATCH(h, kAllocPrefix)
}

static void require_single(Cells2D* h) {
  if (h->b->t.size() != 1) throw Error(CELLS_E_INVALID, "this tunnel belongs to a batch: step the batch");
}

int cells2d_step(Cells2D* h, int64_t n) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  require_single(h);
  if (n < 0) throw Error(CELLS_E_INVALID, "negative step count");
  h->b->launch_steps(n);
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_update_macro(Cells2D* h) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  Cells2DBatch* b = h->b;
  Tunnel2Host& T = h->T();
  if (!b->dev.fake) {
    check_cuda(launch_macro2(b->prec, b->aux(h->k), T.f[b->parity], T.flags, T.macro, T.st, b->dev.stream),
               "macro kernel");
    b->dev.launches++;
  }
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_run(Cells2D* h, int64_t n, int64_t chunk) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  require_single(h);
  if (n < 0) throw Error(CELLS_E_INVALID, "negative step count");
  (void)chunk;  // only the last macro refresh of the reference's chunk loop is observable
  h->b->launch_steps(n);
  int rc = cells2d_update_macro(h);
  if (rc != CELLS_OK) return rc;
  h->b->dev.sync();
  h->b->check_barrier();
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_synchronize(Cells2D* h) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  h->b->dev.sync();
  h->b->check_barrier();
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_read_macro(Cells2D* h, float* out4n) {
  if (!h || !out4n) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  h->b->dev.d2h(out4n, T.macro, (size_t)T.N * 16);
  h->b->dev.sync();
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_read_forces_begin(Cells2D* h) {
  if (!h) return CELLS_E_INVALID;
  C2_TRY
  Cells2DBatch* b = h->b;
  Tunnel2Host& T = h->T();
  T.readPending = false;
  if (T.forceSteps.empty()) return CELLS_OK;
  const uint64_t written = T.forceSamplesRead + T.forceSteps.size();
  const uint64_t first =
      std::max<uint64_t>(T.forceSamplesRead, written > (uint64_t)HISTORY2_LEN ? written - HISTORY2_LEN : 0);
  uint64_t k = first;
  size_t outPos = 0;
  while (k < written) {
    const size_t r = (size_t)(k % HISTORY2_LEN);
    const size_t run = (size_t)std::min<uint64_t>(written - k, (uint64_t)(HISTORY2_LEN - r));
    b->dev.d2h(T.stageHist + outPos, T.history + r, run * sizeof(double2));
    outPos += run;
    k += run;
  }
  b->dev.d2h(T.stageState, &T.st->sample, sizeof(unsigned));
  if (!b->dev.fake) check_cuda(cudaEventRecord(b->dev.evRead, b->dev.stream), "cudaEventRecord");
  T.readPending = true;
  T.readGeneration = T.forceGeneration;
  T.readFirst = first;
  T.readWritten = written;
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_read_forces_end(Cells2D* h, CellsForceSample* out, size_t cap, size_t* n_out) {
  if (!h || !n_out) return CELLS_E_INVALID;
  *n_out = 0;
  C2_TRY
  Cells2DBatch* b = h->b;
  Tunnel2Host& T = h->T();
  if (!T.readPending) return CELLS_OK;
  if (!b->dev.fake) check_cuda(cudaEventSynchronize(b->dev.evRead), "cudaEventSynchronize");
  if (T.readGeneration != T.forceGeneration) {  // a reset while the copy was in flight
    T.readPending = false;
    return CELLS_OK;
  }
  const uint64_t n = T.readWritten - T.readFirst;
  if (n > cap) throw Error(CELLS_E_INVALID, "read_forces needs room for " + std::to_string(n) + " samples");
  if ((uint64_t)*T.stageState != (T.readWritten & 0xffffffffull))
    throw Error(CELLS_E_INVALID, "force ring counter " + std::to_string(*T.stageState) + " does not match the " +
                                     std::to_string(T.readWritten) + " samples enqueued");
  for (uint64_t q = 0; q < n; q++) {
    const double2 v = T.stageHist[q];
    out[q].step = T.forceSteps[(size_t)(T.readFirst + q - T.forceSamplesRead)];
    out[q].reserved = 0;
    out[q].fx = v.x;
    out[q].fy = v.y;
    out[q].fz = 0.0;
  }
  const size_t consumed = (size_t)(T.readWritten - T.forceSamplesRead);
  T.forceSteps.erase(T.forceSteps.begin(), T.forceSteps.begin() + consumed);
  T.forceSamplesRead = T.readWritten;
  T.readPending = false;
  *n_out = (size_t)n;
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_read_forces(Cells2D* h, CellsForceSample* out, size_t cap, size_t* n_out) {
  int rc = cells2d_read_forces_begin(h);
  if (rc != CELLS_OK) return rc;
  return cells2d_read_forces_end(h, out, cap, n_out);
}

int cells2d_read_status(Cells2D* h, uint32_t* status) {
  if (!h || !status) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  h->b->dev.d2h(T.stageState + 1, &T.st->status, sizeof(unsigned));
  h->b->dev.sync();
  uint32_t s = T.stageState[1];
  if (!h->b->dev.fake && h->b->persistent) {
    int e = 0;
    check_cuda(cudaMemcpy(&e, h->b->dError, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy error flag");
    if (e) s |= 4u;
  }
  *status = s;
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_check_diverged(Cells2D* h) {
  if (!h) return CELLS_E_INVALID;
  uint32_t st = 0;
  const int rc = cells2d_read_status(h, &st);
  if (rc != CELLS_OK) return rc;
  if ((st & 3u) == 0) return CELLS_OK;
  C2_TRY
  std::string m = "the flow diverged:";
  if (st & 1u) m += " a non-finite force sample";
  if (st & 2u) m += (st & 1u) ? " and a non-finite macro value" : " a non-finite macro value";
  throw Error(CELLS_E_DIVERGED, m);
  C2_CATCH(h, kAllocPrefix)
}

static void fill_info(Cells2DBatch* b, const Tunnel2Host& T, Cells2DInfo* info) {
  info->W = T.W;
  info->H = T.H;
  info->precision = b->prec;
  info->force_every = T.cfg.force_every;
  info->N = T.N;
  info->step = T.step;
  info->tile_x = b->tileX;
  info->tile_y = b->tileY;
  info->persistent = b->persistent;
  info->tunnels = (int32_t)b->t.size();
}

int cells2d_get_info(Cells2D* h, Cells2DInfo* info) {
  if (!h || !info) return CELLS_E_INVALID;
  fill_info(h->b, h->T(), info);
  return CELLS_OK;
}

int cells2d_read_params(Cells2D* h, void* out96) {
  if (!h || !out96) return CELLS_E_INVALID;
  const Tunnel2Host& T = h->T();
  uint32_t u[24] = {0};
  float* f = (float*)u;
  const int wg = T.cfg.workgroup_size > 0 ? T.cfg.workgroup_size : 128;
  const long long total = (T.N + wg - 1) / wg;  // src/solver.ts:117-119
  u[0] = (uint32_t)T.W;
  u[1] = (uint32_t)T.H;
  u[2] = (uint32_t)T.N;
  u[3] = (uint32_t)std::min<long long>(total, 65535);
  u[4] = (uint32_t)T.cfg.left;
  u[5] = (uint32_t)T.cfg.right;
  u[6] = (uint32_t)T.cfg.bottom;
  u[7] = (uint32_t)T.cfg.top;
  f[8] = (float)T.cfg.tau;
  f[9] = (float)T.cfg.lambda;
  f[10] = (float)(T.cfg.smagorinsky * T.cfg.smagorinsky);
  f[11] = (float)T.current_uin();
  u[12] = T.cfg.parabolic ? 1u : 0u;
  f[13] = (float)T.sponge_start();
  f[14] = (float)T.tau_sponge();
  f[15] = (float)T.cfg.u_lid;
  f[16] = (float)T.cfg.body_force[0];
  f[17] = (float)T.cfg.body_force[1];
  u[18] = (uint32_t)T.forcing();
  f[19] = (float)T.cfg.absorb;
  f[20] = (float)(T.cfg.inlet_layer_fraction * (T.W - 1));
  std::memcpy(out96, u, 96);
  return CELLS_OK;
}

int cells2d_mass(Cells2D* h, double* out) {
  if (!h || !out) return CELLS_E_INVALID;
  C2_TRY
  Cells2DBatch* b = h->b;
  Tunnel2Host& T = h->T();
  if (b->dev.fake) throw Error(CELLS_E_INVALID, "mass needs a CUDA device");
  check_cuda(launch_mass2(b->prec, b->aux(h->k), T.f[b->parity], T.flags, b->massPartials, b->nMassPartials,
                          b->massOut, b->dev.stream),
             "mass kernel");
  b->dev.launches += 2;
  b->dev.d2h(T.stageState + 2, b->massOut, 8);
  b->dev.sync();
  std::memcpy(out, T.stageState + 2, 8);
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_read_populations(Cells2D* h, void* out, size_t bytes) {
  if (!h || !out) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  const size_t need = 9ull * h->b->bpp * (size_t)T.N;
  if (bytes != need) throw Error(CELLS_E_INVALID, "read_populations needs " + std::to_string(need) + " bytes");
  h->b->dev.d2h(out, T.f[h->b->parity], need);
  h->b->dev.sync();
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_write_populations(Cells2D* h, const void* in, size_t bytes) {
  if (!h || !in) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  const size_t need = 9ull * h->b->bpp * (size_t)T.N;
  if (bytes != need) throw Error(CELLS_E_INVALID, "write_populations needs " + std::to_string(need) + " bytes");
  h->b->dev.h2d(T.f[h->b->parity], in, need);
  h->b->dev.sync();
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_read_flags(Cells2D* h, uint32_t* out, size_t n) {
  if (!h || !out) return CELLS_E_INVALID;
  C2_TRY
  Tunnel2Host& T = h->T();
  if (n != (size_t)T.N) throw Error(CELLS_E_INVALID, "read_flags needs N entries");
  h->b->dev.d2h(out, T.flags, n * 4);
  h->b->dev.sync();
  C2_CATCH(h, kAllocPrefix)
}

int cells2d_batch_timer_start(Cells2DBatch* b) {
  if (!b) return CELLS_E_INVALID;
  C2_TRY
  if (!b->dev.fake) check_cuda(cudaEventRecord(b->dev.ev0, b->dev.stream), "cudaEventRecord");
  C2_CATCH(b, kAllocPrefix)
}

int cells2d_batch_timer_stop(Cells2DBatch* b, float* ms) {
  if (!b || !ms) return CELLS_E_INVALID;
  C2_TRY
  *ms = 0.f;
  if (!b->dev.fake) {
    check_cuda(cudaEventRecord(b->dev.ev1, b->dev.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(b->dev.ev1), "cudaEventSynchronize");
    check_cuda(cudaEventElapsedTime(ms, b->dev.ev0, b->dev.ev1), "cudaEventElapsedTime");
  }
  C2_CATCH(b, kAllocPrefix)
}

int cells2d_timer_start(Cells2D* h) {
  if (!h) return CELLS_E_INVALID;
  int rc = cells2d_batch_timer_start(h->b);
  if (rc != CELLS_OK) h->lastError = h->b->lastError;
  return rc;
}

int cells2d_timer_stop(Cells2D* h, float* ms) {
  if (!h) return CELLS_E_INVALID;
  int rc = cells2d_batch_timer_stop(h->b, ms);
  if (rc != CELLS_OK) h->lastError = h->b->lastError;
  return rc;
}

int cells2d_launch_count(Cells2D* h, int64_t* count) {
  if (!h || !count) return CELLS_E_INVALID;
  *count = h->b->dev.launches;
  return CELLS_OK;
}

int cells2d_batch_launch_count(Cells2DBatch* b, int64_t* count) {
  if (!b || !count) return CELLS_E_INVALID;
  *count = b->dev.launches;
  return CELLS_OK;
}

int cells2d_fake_set_force(Cells2D* h, double fx, double fy) {
  if (!h) return CELLS_E_INVALID;
  if (!h->b->dev.fake) {
    h->lastError = "fake_set_force is only for CELLS_FAKE_DEVICE handles";
    return CELLS_E_INVALID;
  }
  h->T().fakeForce[0] = fx;
  h->T().fakeForce[1] = fy;
  return CELLS_OK;
}

int cells2d_batch_step(Cells2DBatch* b, int64_t n) {
  if (!b) return CELLS_E_INVALID;
  C2_TRY
  if (n < 0) throw Error(CELLS_E_INVALID, "negative step count");
  b->launch_steps(n);
  C2_CATCH(b, kAllocPrefix)
}

int cells2d_batch_run(Cells2DBatch* b, int64_t n) {
  if (!b) return CELLS_E_INVALID;
  C2_TRY
  if (n < 0) throw Error(CELLS_E_INVALID, "negative step count");
  b->launch_steps(n);
  if (!b->dev.fake) {
    for (size_t k = 0; k < b->t.size(); k++) {
      Tunnel2Host& T = b->t[k];
      check_cuda(launch_macro2(b->prec, b->aux((int)k), T.f[b->parity], T.flags, T.macro, T.st, b->dev.stream),
                 "macro kernel");
      b->dev.launches++;
    }
  }
  b->dev.sync();
  b->check_barrier();
  C2_CATCH(b, kAllocPrefix)
}

int cells2d_batch_synchronize(Cells2DBatch* b) {
  if (!b) return CELLS_E_INVALID;
  C2_TRY
  b->dev.sync();
  b->check_barrier();
  C2_CATCH(b, kAllocPrefix)
}

int cells2d_batch_get_info(Cells2DBatch* b, Cells2DInfo* info) {
  if (!b || !info) return CELLS_E_INVALID;
  fill_info(b, b->t[0], info);
  long long N = 0;
  for (const Tunnel2Host& T : b->t) N += T.N;
  info->N = N;
  return CELLS_OK;
}

int cells2d_batch_set_launch(Cells2DBatch* b, int32_t tile_x, int32_t tile_y, int32_t persistent) {
  if (!b) return CELLS_E_INVALID;
  C2_TRY
  bool known = false;
  for (const Shape2& sh : kShapes) known = known || (sh.tx == tile_x && sh.ty == tile_y);
  if (!known) throw Error(CELLS_E_INVALID, "unsupported tile shape");
  b->dev.sync();
  b->set_layout(tile_x, tile_y, persistent ? 1 : 0);
  C2_CATCH(b, kAllocPrefix)
}

int cells2d_batch_set_barrier_test(Cells2DBatch* b, int32_t extra_arrivals) {
  if (!b) return CELLS_E_INVALID;
  C2_TRY
  if (extra_arrivals < 0 || extra_arrivals > 1) throw Error(CELLS_E_INVALID, "extra_arrivals must be 0 or 1");
  b->dev.sync();
  b->barrierExtra = (unsigned)extra_arrivals;
  C2_CATCH(b, kAllocPrefix)
}

int cells2d_batch_autotune(Cells2DBatch* b, int32_t trial_steps, Cells2DInfo* info) {
  if (!b) return CELLS_E_INVALID;
  C2_TRY
  if (trial_steps <= 0) throw Error(CELLS_E_INVALID, "trial_steps must be positive");
  if (!b->dev.fake) {
    b->dev.sync();
    const int par0 = b->parity;
    const int tx0 = b->tileX, ty0 = b->tileY, pers0 = b->persistent;
    std::vector<void*> save;  // per tunnel: its populations and device state before the trials
    // copies the snapshots back into the current parity's buffers and releases them
    auto restore = [&]() {
      for (size_t k = 0; k < save.size(); k++) {
        Tunnel2Host& T = b->t[k];
        check_cuda(cudaMemcpyAsync(T.f[par0], save[k], 9ull * b->bpp * (size_t)T.N, cudaMemcpyDeviceToDevice,
                                   b->dev.stream),
                   "restore copy");
        check_cuda(cudaMemcpyAsync(T.st, (char*)save[k] + 9ull * b->bpp * (size_t)T.N, sizeof(DevState2),
                                   cudaMemcpyDeviceToDevice, b->dev.stream),
                   "restore copy");
      }
      b->dev.sync();
      for (void* p : save) b->dev.release(p);
      save.clear();
      b->parity = par0;
    };
    try {
      for (Tunnel2Host& T : b->t) {
        void* p = b->dev.alloc(9ull * b->bpp * (size_t)T.N + sizeof(DevState2), "autotune snapshot");
        save.push_back(p);
        check_cuda(cudaMemcpyAsync(p, T.f[b->parity], 9ull * b->bpp * (size_t)T.N, cudaMemcpyDeviceToDevice,
                                   b->dev.stream),
                   "snapshot copy");
        check_cuda(cudaMemcpyAsync((char*)p + 9ull * b->bpp * (size_t)T.N, T.st, sizeof(DevState2),
                                   cudaMemcpyDeviceToDevice, b->dev.stream),
                   "snapshot copy");
      }
      float best = 1e30f;
      Shape2 bestShape = {b->tileX, b->tileY};
      int bestPers = b->persistent;
      const int warm = std::min(trial_steps, 20);
      for (const Shape2& sh : kShapes) {
        for (int pers = 0; pers <= 1; pers++) {
          b->set_layout(sh.tx, sh.ty, pers);
          if (pers && b->persistentBlocks <= 0) continue;
          b->dev.memset0(b->dError, sizeof(int));
          b->launch_raw(warm, par0, 0);
          // a graph-replayed trial times the replay, not the capture: the layout change invalidated
          // the step graphs, so they are rebuilt here, outside the timed region
          if (!pers && b->useGraphs && trial_steps >= kGraphSteps2) {
            b->build_graph(0, 0);
            b->build_graph(0, 1);
          }
          check_cuda(cudaEventRecord(b->dev.ev0, b->dev.stream), "cudaEventRecord");
          b->launch_raw(trial_steps, par0 ^ (warm & 1), 0);
          check_cuda(cudaEventRecord(b->dev.ev1, b->dev.stream), "cudaEventRecord");
          check_cuda(cudaEventSynchronize(b->dev.ev1), "cudaEventSynchronize");
          float ms = 0.f;
          check_cuda(cudaEventElapsedTime(&ms, b->dev.ev0, b->dev.ev1), "cudaEventElapsedTime");
          int err = 0;
          check_cuda(cudaMemcpy(&err, b->dError, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy error flag");
          if (err) {
            b->dev.memset0(b->dError, sizeof(int));
            continue;
          }
          if (ms < best) {
            best = ms;
            bestShape = sh;
            bestPers = pers;
          }
        }
      }
      b->set_layout(bestShape.tx, bestShape.ty, bestPers);
      restore();
    } catch (...) {
      // a failed trial leaves the previous layout and the state before the call in place
      try {
        b->set_layout(tx0, ty0, pers0);
        restore();
      } catch (...) {
        for (void* p : save) b->dev.release(p);
        b->parity = par0;
      }
      throw;
    }
  }
  if (info) {
    fill_info(b, b->t[0], info);
    long long N = 0;
    for (const Tunnel2Host& T : b->t) N += T.N;
    info->N = N;
  }
  C2_CATCH(b, kAllocPrefix)
}

}  // extern "C"
