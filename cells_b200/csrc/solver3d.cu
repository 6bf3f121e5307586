// Solver3D host state and the 3D half of the C ABI (include/cells.h).
//
// Mirrors class Solver3D, src/solver3d.ts:42-320: buffers, parameter derivation (writeParams
// :197-208), setSdf/rebuildFlags (:211-228), initField (:231-242), resetForces (:244-249),
// encodeSteps (:252-267), run (:276-288), readMacro (:290-292) and readForces with its ring window
// and generation check (:295-315). Everything is enqueued on the handle's own CUDA stream.
#include <cmath>
#include <cstdlib>
#include <deque>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cells.h"
#include "adjoint3d.h"
#include "device.h"
#include "kernels3d.h"
#include "solver3d_state.h"

namespace cells {
thread_local std::string g_create_error;
}

using namespace cells;

Cells3D::Cells3D() = default;
Cells3D::~Cells3D() = default;

// ---------------- helpers ----------------

// Per-x table (omega+ without Smagorinsky, omega-, sigma, 0). The reference computes these per
// cell in f32 (src/shaders/step3d.ts:72-74 and :213-219); the same f32 operations in the same order
// give the same values here (the host build does not contract multiply-adds).
template <class R>
static void fill_xtab(std::vector<R>& t, int W, double tau, double lambda, double spongeStart, double tauSponge,
                      double absorb) {
  const R tauR = (R)tau, lamR = (R)lambda, ssR = (R)spongeStart, tsR = (R)tauSponge, abR = (R)absorb;
  const R e1 = (R)(W - 1);
  t.resize(4 * (size_t)W);
  for (int x = 0; x < W; x++) {
    R omegaBase = R(1) / tauR;
    R sOut = R(0);
    if (ssR < e1) {
      R tt = (R(x) - ssR) / (e1 - ssR);
      tt = std::fmin(std::fmax(tt, R(0)), R(1));
      sOut = tt * tt * (R(3) - R(2) * tt);
      const R mix = tauR * (R(1) - sOut) + tsR * sOut;
      omegaBase = R(1) / mix;
    }
    t[4 * x] = omegaBase;
    t[4 * x + 1] = R(1) / (R(0.5) + lamR / (R(1) / omegaBase - R(0.5)));
    t[4 * x + 2] = abR * sOut * sOut;
    t[4 * x + 3] = R(0);
  }
}

// Interior tile of the step kernel (128 threads per block): 128 cells, or 256 cells as x-pairs for
// f32, f16 or bf16 storage with an even width (f64 and odd widths take one cell per thread). The
// tile width is workgroup_size when given (the autotuner's knob), else the candidate that wastes
// the fewest threads at the end of a row: the widest for one cell per thread, the narrowest (64
// cells, 32 pairs x 4 rows) for pairs, so that more tiles fall wholly outside the absorbing layer
// and the outlet column.
void Cells3D::choose_launch() {
  pairTiles = (bpp <= 4 && (W % 2) == 0) ? 1 : 0;
  const int cells = pairTiles ? 256 : 128;
  const int lo = pairTiles ? 64 : 32;
  int best = -1;
  long long bestWaste = -1;
  for (int c = cells; c >= lo; c >>= 1) {
    const long long waste = (long long)((W + c - 1) / c) * c - W;
    if (best < 0 || waste < bestWaste || (pairTiles && waste == bestWaste)) {
      best = c;
      bestWaste = waste;
    }
  }
  if (cfg.workgroup_size > 0) {
    best = lo;
    while (best * 2 <= cells && best * 2 <= cfg.workgroup_size) best *= 2;
  }
  bx = best;
  by = cells / bx;
}

void Cells3D::upload_xtab() {
  int firstAbsorb = W;  // the first x with a nonzero absorbing strength
  if (prec == 3) {
    std::vector<double> t;
    fill_xtab<double>(t, W, cfg.tau, lambda_value(), sponge_start(), tau_sponge(), cfg.absorb);
    for (int x = W - 1; x >= 0; x--)
      if (t[4 * x + 2] > 0.0) firstAbsorb = x;
    dev.h2d(xTab, t.data(), t.size() * sizeof(double));
  } else {
    std::vector<float> t;
    fill_xtab<float>(t, W, cfg.tau, lambda_value(), sponge_start(), tau_sponge(), cfg.absorb);
    for (int x = W - 1; x >= 0; x--)
      if (t[4 * x + 2] > 0.0f) firstAbsorb = x;
    // the x-pair layout of the same values after the W per-x entries: entry x0 (even) holds
    // (omega+ of x0, of x0 + 1, omega- of x0, of x0 + 1), entry x0 + 1 (sigma of x0, of x0 + 1, 0, 0)
    t.resize(8 * (size_t)W, 0.0f);
    float* pairTab = t.data() + 4 * (size_t)W;
    for (int x0 = 0; x0 + 1 < W; x0 += 2) {
      const float* c0 = t.data() + 4 * (size_t)x0;
      const float* c1 = c0 + 4;
      float* e = pairTab + 4 * (size_t)x0;
      e[0] = c0[0];
      e[1] = c1[0];
      e[2] = c0[1];
      e[3] = c1[1];
      e[4] = c0[2];
      e[5] = c1[2];
    }
    dev.h2d(xTab, t.data(), t.size() * sizeof(float));
  }
  if (firstAbsorb != absorbX0) {
    absorbX0 = firstAbsorb;
    argGen++;  // step graphs bake the absorbing layer's first x
  }
  if (!dev.fake) dev.sync();  // the host vectors die here
}

void Cells3D::write_state(int which) {
  // which: 1 step counters, 2 inlet speeds, 4 clear samples, 8 clear status
  if (dev.fake) {
    if (which & 1) st->step[0] = st->step[1] = (unsigned)step;
    if (which & 2) st->uIn[0] = st->uIn[1] = current_uin();
    if (which & 4) st->sample = st->done = 0;
    if (which & 8) st->status = 0;
    return;
  }
  const double u = current_uin();
  check_cuda(launch_set_state3(prec, st, which, (unsigned)step, u, u, dev.stream), "set_state kernel");
  dev.launches++;
}

// The body kernel's cells: every fluid cell with a non-zero flag in a row that holds a body cell,
// in increasing index order (so the force reduction order is fixed).
void Cells3D::build_body_list() {
  nBody = 0;
  if (!dev.fake) {
    // counts per row on the device, offsets on the host (H * D ints each way), cells on the device
    const int nRows = H * D;
    int* counts = (int*)scratch_buffer((size_t)nRows * 4 * 2);
    int* offsets = counts + nRows;
    check_cuda(launch_body_count3(W, nRows, rowBody, flags, counts, dev.stream), "body count kernel");
    std::vector<int> c((size_t)nRows);
    dev.d2h(c.data(), counts, (size_t)nRows * 4);
    dev.sync();
    long long total = 0;
    for (int r = 0; r < nRows; r++) {
      const int k = c[(size_t)r];
      c[(size_t)r] = (int)total;
      total += k;
    }
    nBody = (int)total;
    if (nBody > 0) {
      dev.h2d(offsets, c.data(), (size_t)nRows * 4);
      check_cuda(launch_body_write3(W, nRows, rowBody, flags, offsets, bodyCells, dev.stream), "body list kernel");
      dev.launches += 2;
      dev.sync();
    }
  }
  if (nBody > links.cap) {
    // grow the link tables (18 links per body cell)
    for (void* p : {links.rec, (void*)links.kinds, (void*)links.meta}) dev.release(p);
    links = BodyLinks3{};
    const int cap = std::max(nBody, 4096);
    links.rec = dev.alloc(18 * (size_t)cap * 32, "body links");  // sizeof(Link3<R>) is 32 for f32 and f64
    links.kinds = (unsigned long long*)dev.alloc((size_t)cap * 8, "body links");
    links.meta = (int*)dev.alloc((size_t)cap * 4, "body links");
    links.cap = cap;
  }
  if (nBody > 0 && !dev.fake) {
    AuxLaunch3 a{W, H, D, (int)N, current_uin()};
    check_cuda(launch_links3(prec, a, bodyCells, nBody, flags, sdf, links, dev.stream), "links kernel");
    dev.launches++;
    dev.sync();
  }
}

// rebuildFlags, src/solver3d.ts:216-228: a macro pass on the latest populations (the refill reads
// it), then the flags pass, then the body-row map and the body cell list.
void Cells3D::rebuild_flags() {
  if (!dev.fake) {
    AuxLaunch3 a{W, H, D, (int)N, uIn};
    a.uIn = current_uin();
    check_cuda(launch_macro3(prec, a, f[parity], flags, macro, st, dev.stream), "macro kernel");
    dev.memset0(rowBody, (size_t)H * D);
    check_cuda(launch_flags3(prec, a, sdf, flags, rowBody, f[0], f[1], macro, dev.stream), "flags kernel");
    dev.launches += 2;
  }
  build_body_list();
  argGen++;  // the body list and links are baked into step graphs
}

// Enqueues the step kernel of one step of parity par on `main`; returns the kernels launched.
int Cells3D::enqueue_step(int par, bool sample, cudaStream_t main) {
  (void)main;
  enqueue_step_between(f[par], f[par ^ 1], par, sample);
  return 1;
}

void Cells3D::enqueue_step_between(const void* src, void* dst, int par, bool sample, cudaStream_t stream) {
  cudaStream_t main = stream ? stream : dev.stream;
  StepLaunch3 a;
  a.src = src;
  a.dst = dst;
  a.flags = flags;
  a.sdf = sdf;
  a.rowBody = rowBody;
  a.xTab = xTab;
  a.bodyCells = bodyCells;
  a.links = links;
  a.partials = partials;
  a.history = history;
  a.st = st;
  a.W = W;
  a.H = H;
  a.D = D;
  a.N = N;
  a.tileTX = bx;
  a.tileTY = by;
  a.pairTiles = pairTiles;
  a.absorbX0 = absorbX0;
  a.nBody = nBody;
  a.rampKind = rampKind;
  a.rampEvery = (int)rampEvery;
  a.rampTarget = rampTarget;
  a.rampSteps = (double)rampSteps;
  a.lambda = lambda_value();
  a.smagC2 = cfg.smagorinsky * cfg.smagorinsky;
  a.par = par;
  a.sample = sample ? 1 : 0;
  check_cuda(cfg.arithmetic == CELLS_ARITH_EXACT ? exact::launch_step3(prec, a, main)
                                                 : fast::launch_step3(prec, a, main),
             "step kernel");
}

// Steps repeat with period lcm(2, force_every) in their launch arguments (parity and sampling);
// graphs are kept per phase of that period. Longer periods run without graphs.
int Cells3D::graph_period() const {
  const int every = cfg.force_every;
  if (every <= 0) return 2;
  return (every % 2 == 0) ? every : 2 * every;
}

void Cells3D::build_graph(int phase) {
  StepGraph& g = graphs[phase];
  if (g.exec) cudaGraphExecDestroy(g.exec);
  g.exec = nullptr;
  const int every = cfg.force_every;
  int launches = 0;
  check_cuda(cudaStreamBeginCapture(dev.stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  int par = phase % 2;
  int64_t s = phase;
  for (int k = 0; k < kGraphSteps; k++) {
    const bool sample = every > 0 && ((s + 1) % every) == 0;
    launches += enqueue_step(par, sample, dev.stream);
    par ^= 1;
    s++;
  }
  cudaGraph_t graph = nullptr;
  check_cuda(cudaStreamEndCapture(dev.stream, &graph), "cudaStreamEndCapture");
  cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  check_cuda(e, "cudaGraphInstantiate");
  g.gen = argGen;
  g.launches = launches;
}

void Cells3D::launch_steps(int64_t n) {
  const int every = cfg.force_every;
  const int period = graph_period();
  while (n > 0) {
    if (!dev.fake && useGraphs && period <= kMaxGraphPeriod && n >= kGraphSteps) {
      // kGraphSteps steps as one graph launch: parity and sampling depend on step % period only
      const int phase = (int)(step % period);
      if (!graphs[phase].exec || graphs[phase].gen != argGen) build_graph(phase);
      check_cuda(cudaGraphLaunch(graphs[phase].exec, dev.stream), "cudaGraphLaunch");
      dev.launches += graphs[phase].launches;
      for (int k = 0; k < kGraphSteps; k++) {
        const bool sample = every > 0 && ((step + 1) % every) == 0;
        parity ^= 1;
        step++;
        if (sample) forceSteps.push_back((uint32_t)step);
      }
      n -= kGraphSteps;
      continue;
    }
    const bool sample = every > 0 && ((step + 1) % every) == 0;
    if (dev.fake) {
      if (sample) {
        const unsigned s = st->sample;
        history[s % HISTORY_LEN] = make_double4(fakeForce[0], fakeForce[1], fakeForce[2], 0.0);
        st->sample = s + 1;
      }
    } else {
      dev.launches += enqueue_step(parity, sample, dev.stream);
    }
    parity ^= 1;
    step++;
    if (sample) forceSteps.push_back((uint32_t)step);
    n--;
  }
}

// Builds (captures and instantiates) every step graph that launch_steps(n) from the current step
// would replay, without running anything, so a timed or latency-critical run that follows replays
// graphs only.
void Cells3D::prepare_steps(int64_t n) {
  const int period = graph_period();
  if (dev.fake || !useGraphs || period > kMaxGraphPeriod) return;
  int64_t s = step;
  while (n >= kGraphSteps) {
    const int phase = (int)(s % period);
    if (!graphs[phase].exec || graphs[phase].gen != argGen) build_graph(phase);
    s += kGraphSteps;
    n -= kGraphSteps;
  }
}

void Cells3D::free_all() {
  adj.reset();  // its buffers are the device's; freed by dev.close below
  for (auto& g : graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  graphs.assign(kMaxGraphPeriod, StepGraph{});
  if (stageHist) dev.free_host_pinned(stageHist);
  if (stageState) dev.free_host_pinned(stageState);
  stageHist = nullptr;
  stageState = nullptr;
  dev.close();
}

// ---------------- C ABI ----------------

#define CELLS_TRY(h)                                   \
  try {
#define CELLS_CATCH(h)                                 \
  }                                                    \
  catch (const AllocError& e) {                        \
    (h)->lastError = std::string("Solver3D allocation failed: ") + e.what(); \
    return CELLS_E_ALLOC;                              \
  }                                                    \
  catch (const Error& e) {                             \
    (h)->lastError = e.what();                         \
    return e.status;                                   \
  }                                                    \
  catch (const std::exception& e) {                    \
    (h)->lastError = e.what();                         \
    return CELLS_E_INVALID;                            \
  }                                                    \
  return CELLS_OK;

extern "C" {

void cells3d_config_default(Cells3DConfig* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->precision = CELLS_FP32;
  c->tau = 0.6;
  c->lambda = NAN;
  c->smagorinsky = 0.0;
  c->u_in = 0.0;
  c->sponge_fraction = 0.0;
  c->sponge_tau = 1.0;
  c->absorb = 0.0;
  c->workgroup_size = 0;
  c->force_every = 1;
  c->device = 0;
}

const char* cells_last_error(const void* h) {
  if (!h) return g_create_error.c_str();
  // every handle type (Cells3D, Cells2D, Cells2DBatch) has HandleBase as its first base
  return ((const HandleBase*)h)->lastError.c_str();
}

int cells3d_create(const Cells3DConfig* cfg, Cells3D** out) {
  if (!out) return CELLS_E_INVALID;
  *out = nullptr;
  g_create_error.clear();
  if (!cfg) {
    g_create_error = "config is NULL";
    return CELLS_E_INVALID;
  }
  if (cfg->width < 3 || cfg->height < 1 || cfg->depth < 1) {
    g_create_error = "grid must be at least 3 x 1 x 1";
    return CELLS_E_INVALID;
  }
  if (cfg->precision < 0 || cfg->precision > 3) {
    g_create_error = "precision " + std::to_string(cfg->precision) + " is not available on this device";
    return CELLS_E_PRECISION_UNSUPPORTED;
  }
  if (!(cfg->tau > 0.5)) {
    g_create_error = "tau must be above 1/2";
    return CELLS_E_INVALID;
  }
  const long long N = (long long)cfg->width * cfg->height * cfg->depth;
  if (N > 0x7fffffffLL) {
    g_create_error = "grid has more than 2^31 cells";
    return CELLS_E_INVALID;
  }
  Cells3D* h = new Cells3D();
  h->cfg = *cfg;
  h->W = cfg->width;
  h->H = cfg->height;
  h->D = cfg->depth;
  h->N = N;
  h->prec = cfg->precision;
  h->bpp = h->prec == 0 ? 4 : (h->prec == 3 ? 8 : 2);
  h->uIn = cfg->u_in;
  if (const char* gv = std::getenv("CELLS_GRAPHS")) h->useGraphs = std::atoi(gv) != 0;
  try {
    h->dev.open(cfg->device, cfg->fake_fail_alloc);
    const unsigned long long fBytes = 19ull * h->bpp * (unsigned long long)N;
    // fitsLimits (src/shaders/common3d.ts:67-70): checked before anything is allocated
    if (cfg->max_buffer_bytes > 0 && fBytes > cfg->max_buffer_bytes) {
      throw AllocError("one distribution buffer needs " + std::to_string(fBytes) + " bytes; this device allows " +
                       std::to_string(cfg->max_buffer_bytes) + " per buffer");
    }
    h->choose_launch();
    const unsigned long long total = 2 * fBytes + (unsigned long long)N * (4 + 4 + 16) + (1u << 22);
    const size_t freeB = h->dev.free_bytes();
    if (total > freeB) {
      throw AllocError("the solver needs " + std::to_string(total) + " bytes; this device has " +
                       std::to_string(freeB) + " bytes free");
    }
    h->f[0] = h->dev.alloc(fBytes, "distribution buffer A");
    h->f[1] = h->dev.alloc(fBytes, "distribution buffer B");
    h->flags = (uint32_t*)h->dev.alloc((size_t)N * 4, "flags");
    h->sdf = (float*)h->dev.alloc((size_t)N * 4, "sdf");
    h->macro = (float4*)h->dev.alloc((size_t)N * 16, "macro");
    h->rowBody = (uint8_t*)h->dev.alloc((size_t)h->H * h->D, "row map");
    // f64 rates: 4 per x; f32 rates: 4 per x and the x-pair layout of the same values
    h->xTab = h->dev.alloc((size_t)h->W * (h->prec == 3 ? 4 * 8 : 8 * 4), "x table");
    h->bodyCells = (int*)h->dev.alloc((size_t)N * 4, "body cell list");
    h->partials = (double4*)h->dev.alloc((size_t)(N / 32 + 2) * sizeof(double4), "force partials");
    h->history = (double4*)h->dev.alloc((size_t)HISTORY_LEN * sizeof(double4), "force history");
    h->st = (DevState3*)h->dev.alloc(sizeof(DevState3), "state");
    h->nMassPartials = 4 * 148;
    h->massPartials = (double*)h->dev.alloc((size_t)h->nMassPartials * 8, "mass partials");
    h->massOut = (double*)h->dev.alloc(8, "mass result");
    h->stageHist = (double4*)h->dev.host_pinned((size_t)HISTORY_LEN * sizeof(double4));
    h->stageState = (unsigned*)h->dev.host_pinned(64);
    // zero state, fill the SDF with FAR = 1e6 (src/solver3d.ts:142)
    h->dev.memset0(h->st, sizeof(DevState3));
    h->dev.memset0(h->f[0], fBytes);
    h->dev.memset0(h->f[1], fBytes);
    h->dev.memset0(h->flags, (size_t)N * 4);
    {
      std::vector<float> far((size_t)N, 1e6f);
      h->dev.h2d(h->sdf, far.data(), far.size() * 4);
      h->dev.sync();
    }
    h->upload_xtab();
    h->write_state(1 | 2 | 4 | 8);
    h->rebuild_flags();
  } catch (const AllocError& e) {
    g_create_error = std::string("Solver3D allocation failed: ") + e.what();
    h->free_all();
    delete h;
    return CELLS_E_ALLOC;
  } catch (const Error& e) {
    g_create_error = e.what();
    h->free_all();
    delete h;
    return e.status;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    h->free_all();
    delete h;
    return CELLS_E_INVALID;
  }
  *out = h;
  return CELLS_OK;
}

void cells3d_destroy(Cells3D* h) {
  if (!h) return;
  h->free_all();
  delete h;
}

int cells3d_set_tau(Cells3D* h, double tau) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (!(tau > 0.5)) throw Error(CELLS_E_INVALID, "tau must be above 1/2");
  h->cfg.tau = tau;
  h->argGen++;
  h->upload_xtab();
  CELLS_CATCH(h)
}

int cells3d_set_smagorinsky(Cells3D* h, double cs) {
  if (!h) return CELLS_E_INVALID;
  h->cfg.smagorinsky = cs;
  h->argGen++;
  return CELLS_OK;
}

int cells3d_set_lambda(Cells3D* h, double lambda) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  h->cfg.lambda = lambda;
  h->argGen++;
  h->upload_xtab();
  CELLS_CATCH(h)
}

int cells3d_set_inlet(Cells3D* h, double u) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  h->uIn = u;
  h->cfg.u_in = u;
  h->rampKind = 0;
  h->write_state(2);
  CELLS_CATCH(h)
}

int cells3d_set_inlet_ramp(Cells3D* h, int kind, double target, int64_t ramp_steps, int64_t update_every) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (kind < 0 || kind > 2) throw Error(CELLS_E_INVALID, "unknown ramp kind");
  if (kind != 0 && (ramp_steps <= 0 || update_every <= 0))
    throw Error(CELLS_E_INVALID, "ramp_steps and update_every must be positive");
  h->rampKind = kind;
  h->argGen++;
  h->rampTarget = target;
  h->rampSteps = ramp_steps > 0 ? ramp_steps : 1;
  h->rampEvery = update_every > 0 ? update_every : 1;
  if (kind == 0) h->uIn = target;
  h->write_state(2);
  CELLS_CATCH(h)
}

int cells3d_set_sdf(Cells3D* h, const float* sdf, size_t n) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (!sdf || n != (size_t)h->N) throw Error(CELLS_E_INVALID, "set_sdf needs W*H*D floats");
  h->dev.h2d(h->sdf, sdf, n * 4);
  h->dev.sync();
  h->rebuild_flags();
  CELLS_CATCH(h)
}

int cells3d_init_field(Cells3D* h, const float* macro4n) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  h->step = 0;
  h->parity = 0;
  if (!h->dev.fake) {
    if (macro4n) {
      h->dev.h2d(h->macro, macro4n, (size_t)h->N * 16);
    }
    AuxLaunch3 a{h->W, h->H, h->D, (int)h->N, h->current_uin()};
    check_cuda(launch_init3(h->prec, a, h->f[0], h->f[1], h->flags, macro4n ? h->macro : nullptr, h->dev.stream),
               "init kernel");
    h->dev.launches++;
    if (macro4n) h->dev.sync();
  }
  // a new flow clears the divergence status, as recoverFromBlowup's re-init starts over
  h->write_state(1 | 2 | 8);
  // resetForces (src/solver3d.ts:244-249)
  h->write_state(4);
  h->forceSamplesRead = 0;
  h->forceSteps.clear();
  h->forceGeneration++;
  CELLS_CATCH(h)
}

int cells3d_reset_forces(Cells3D* h) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  h->write_state(4);
  h->forceSamplesRead = 0;
  h->forceSteps.clear();
  h->forceGeneration++;
  CELLS_CATCH(h)
}

int cells3d_step(Cells3D* h, int64_t n) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (n < 0) throw Error(CELLS_E_INVALID, "negative step count");
  h->launch_steps(n);
  CELLS_CATCH(h)
}

int cells3d_prepare_steps(Cells3D* h, int64_t n) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (n < 0) throw Error(CELLS_E_INVALID, "negative step count");
  h->prepare_steps(n);
  CELLS_CATCH(h)
}

int cells3d_update_macro(Cells3D* h) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (!h->dev.fake) {
    AuxLaunch3 a{h->W, h->H, h->D, (int)h->N, h->current_uin()};
    check_cuda(launch_macro3(h->prec, a, h->f[h->parity], h->flags, h->macro, h->st, h->dev.stream), "macro kernel");
    h->dev.launches++;
  }
  CELLS_CATCH(h)
}

int cells3d_run(Cells3D* h, int64_t n, int64_t chunk) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (n < 0) throw Error(CELLS_E_INVALID, "negative step count");
  if (chunk <= 0) chunk = 500;
  for (int64_t done = 0; done < n;) {
    const int64_t k = std::min(chunk, n - done);
    h->launch_steps(k);
    done += k;
  }
  int rc = cells3d_update_macro(h);
  if (rc != CELLS_OK) return rc;
  h->dev.sync();
  CELLS_CATCH(h)
}

int cells3d_synchronize(Cells3D* h) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  h->dev.sync();
  CELLS_CATCH(h)
}

int cells3d_read_macro(Cells3D* h, float* out4n) {
  if (!h || !out4n) return CELLS_E_INVALID;
  CELLS_TRY(h)
  h->dev.d2h_large(out4n, h->macro, (size_t)h->N * 16);
  CELLS_CATCH(h)
}

int cells3d_read_forces_begin(Cells3D* h) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  h->readPending = false;
  if (h->forceSteps.empty()) return CELLS_OK;
  const uint64_t written = h->forceSamplesRead + h->forceSteps.size();
  const uint64_t first = std::max<uint64_t>(h->forceSamplesRead, written > (uint64_t)HISTORY_LEN ? written - HISTORY_LEN : 0);
  // copy ring entries [first, written) in order into the staging buffer (at most two runs)
  uint64_t k = first;
  size_t outPos = 0;
  while (k < written) {
    const size_t r = (size_t)(k % HISTORY_LEN);
    const size_t run = (size_t)std::min<uint64_t>(written - k, (uint64_t)(HISTORY_LEN - r));
    h->dev.d2h(h->stageHist + outPos, h->history + r, run * sizeof(double4));
    outPos += run;
    k += run;
  }
  h->dev.d2h(h->stageState, &h->st->sample, sizeof(unsigned));
  if (!h->dev.fake) check_cuda(cudaEventRecord(h->dev.evRead, h->dev.stream), "cudaEventRecord");
  h->readPending = true;
  h->readGeneration = h->forceGeneration;
  h->readFirst = first;
  h->readWritten = written;
  CELLS_CATCH(h)
}

int cells3d_read_forces_end(Cells3D* h, CellsForceSample* out, size_t cap, size_t* n_out) {
  if (!h || !n_out) return CELLS_E_INVALID;
  *n_out = 0;
  CELLS_TRY(h)
  if (!h->readPending) return CELLS_OK;
  if (!h->dev.fake) check_cuda(cudaEventSynchronize(h->dev.evRead), "cudaEventSynchronize");
  // a reset while the copy was in flight makes these samples stale
  if (h->readGeneration != h->forceGeneration) {
    h->readPending = false;
    return CELLS_OK;
  }
  const uint64_t n = h->readWritten - h->readFirst;
  if (n > cap) throw Error(CELLS_E_INVALID, "read_forces needs room for " + std::to_string(n) + " samples");
  if ((uint64_t)*h->stageState != (h->readWritten & 0xffffffffull))
    throw Error(CELLS_E_INVALID, "force ring counter " + std::to_string(*h->stageState) + " does not match the " +
                                     std::to_string(h->readWritten) + " samples enqueued");
  for (uint64_t k = 0; k < n; k++) {
    const double4 v = h->stageHist[k];
    out[k].step = h->forceSteps[(size_t)(h->readFirst + k - h->forceSamplesRead)];
    out[k].reserved = 0;
    out[k].fx = v.x;
    out[k].fy = v.y;
    out[k].fz = v.z;
  }
  const size_t consumed = (size_t)(h->readWritten - h->forceSamplesRead);
  h->forceSteps.erase(h->forceSteps.begin(), h->forceSteps.begin() + consumed);
  h->forceSamplesRead = h->readWritten;
  h->readPending = false;
  *n_out = (size_t)n;
  CELLS_CATCH(h)
}

int cells3d_read_forces(Cells3D* h, CellsForceSample* out, size_t cap, size_t* n_out) {
  int rc = cells3d_read_forces_begin(h);
  if (rc != CELLS_OK) return rc;
  return cells3d_read_forces_end(h, out, cap, n_out);
}

int cells3d_read_status(Cells3D* h, uint32_t* status) {
  if (!h || !status) return CELLS_E_INVALID;
  CELLS_TRY(h)
  h->dev.d2h(h->stageState + 1, &h->st->status, sizeof(unsigned));
  h->dev.sync();
  *status = h->stageState[1];
  CELLS_CATCH(h)
}

int cells3d_check_diverged(Cells3D* h) {
  if (!h) return CELLS_E_INVALID;
  uint32_t st = 0;
  const int rc = cells3d_read_status(h, &st);
  if (rc != CELLS_OK) return rc;
  if (st == 0) return CELLS_OK;
  CELLS_TRY(h)
  std::string m = "the flow diverged:";
  if (st & 1u) m += " a non-finite force sample";
  if (st & 2u) m += (st & 1u) ? " and a non-finite macro value" : " a non-finite macro value";
  throw Error(CELLS_E_DIVERGED, m);
  CELLS_CATCH(h)
}

int cells3d_get_info(Cells3D* h, Cells3DInfo* info) {
  if (!h || !info) return CELLS_E_INVALID;
  info->W = h->W;
  info->H = h->H;
  info->D = h->D;
  info->precision = h->prec;
  info->N = h->N;
  info->step = h->step;
  info->block_x = h->bx;
  info->block_y = h->by;
  info->force_every = h->cfg.force_every;
  info->n_body_cells = h->nBody;
  return CELLS_OK;
}

int cells3d_read_params(Cells3D* h, void* out64) {
  if (!h || !out64) return CELLS_E_INVALID;
  uint32_t u[16] = {0};
  float* f = (float*)u;
  u[0] = (uint32_t)h->W;
  u[1] = (uint32_t)h->H;
  u[2] = (uint32_t)h->D;
  u[3] = (uint32_t)h->N;
  // groupsX as the reference derives it for its default workgroup of 128 (src/solver3d.ts:124-127)
  u[4] = (uint32_t)std::min<long long>((h->N + 127) / 128, 65535);
  f[8] = (float)h->cfg.tau;
  f[9] = (float)h->lambda_value();
  f[10] = (float)(h->cfg.smagorinsky * h->cfg.smagorinsky);
  f[11] = (float)h->current_uin();
  f[12] = (float)h->sponge_start();
  f[13] = (float)h->tau_sponge();
  f[14] = (float)h->cfg.absorb;
  std::memcpy(out64, u, 64);
  return CELLS_OK;
}

int cells3d_mass(Cells3D* h, double* out) {
  if (!h || !out) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (h->dev.fake) throw Error(CELLS_E_INVALID, "mass needs a CUDA device");
  AuxLaunch3 a{h->W, h->H, h->D, (int)h->N, h->current_uin()};
  check_cuda(launch_mass3(h->prec, a, h->f[h->parity], h->flags, h->massPartials, h->nMassPartials, h->massOut,
                          h->dev.stream),
             "mass kernel");
  h->dev.launches += 2;
  double v = 0;
  h->dev.d2h(h->stageState + 2, h->massOut, 8);  // 8-byte aligned slot in the pinned block
  h->dev.sync();
  std::memcpy(&v, h->stageState + 2, 8);
  *out = v;
  CELLS_CATCH(h)
}

int cells3d_read_populations(Cells3D* h, void* out, size_t bytes) {
  if (!h || !out) return CELLS_E_INVALID;
  CELLS_TRY(h)
  const size_t need = 19ull * h->bpp * (size_t)h->N;
  if (bytes != need) throw Error(CELLS_E_INVALID, "read_populations needs " + std::to_string(need) + " bytes");
  h->dev.d2h(out, h->f[h->parity], need);
  h->dev.sync();
  CELLS_CATCH(h)
}

int cells3d_write_populations(Cells3D* h, const void* in, size_t bytes) {
  if (!h || !in) return CELLS_E_INVALID;
  CELLS_TRY(h)
  const size_t need = 19ull * h->bpp * (size_t)h->N;
  if (bytes != need) throw Error(CELLS_E_INVALID, "write_populations needs " + std::to_string(need) + " bytes");
  h->dev.h2d(h->f[h->parity], in, need);
  h->dev.sync();
  CELLS_CATCH(h)
}

// Snapshot layout: this header, then 19 N populations of the storage type.
struct StateHeader3 {
  uint64_t magic;  // "CELLS3D1"
  int32_t W, H, D, precision;
  int64_t step;
  int32_t parity, rampKind;
  double uIn, rampTarget;
  int64_t rampSteps, rampEvery;
};
static constexpr uint64_t kStateMagic3 = 0x3144334c4c4543ull;

int cells3d_state_size(Cells3D* h, size_t* bytes) {
  if (!h || !bytes) return CELLS_E_INVALID;
  *bytes = sizeof(StateHeader3) + 19ull * h->bpp * (size_t)h->N;
  return CELLS_OK;
}

int cells3d_save_state(Cells3D* h, void* out, size_t bytes) {
  if (!h || !out) return CELLS_E_INVALID;
  CELLS_TRY(h)
  const size_t pop = 19ull * h->bpp * (size_t)h->N;
  if (bytes != sizeof(StateHeader3) + pop) throw Error(CELLS_E_INVALID, "save_state needs state_size bytes");
  StateHeader3 s{};
  s.magic = kStateMagic3;
  s.W = h->W;
  s.H = h->H;
  s.D = h->D;
  s.precision = h->prec;
  s.step = h->step;
  s.parity = h->parity;
  s.rampKind = h->rampKind;
  s.uIn = h->uIn;
  s.rampTarget = h->rampTarget;
  s.rampSteps = h->rampSteps;
  s.rampEvery = h->rampEvery;
  std::memcpy(out, &s, sizeof(s));
  h->dev.d2h((char*)out + sizeof(s), h->f[h->parity], pop);
  h->dev.sync();
  CELLS_CATCH(h)
}

int cells3d_load_state(Cells3D* h, const void* in, size_t bytes) {
  if (!h || !in) return CELLS_E_INVALID;
  CELLS_TRY(h)
  const size_t pop = 19ull * h->bpp * (size_t)h->N;
  if (bytes != sizeof(StateHeader3) + pop) throw Error(CELLS_E_INVALID, "load_state needs state_size bytes");
  StateHeader3 s;
  std::memcpy(&s, in, sizeof(s));
  if (s.magic != kStateMagic3) throw Error(CELLS_E_INVALID, "not a Solver3D state snapshot");
  if (s.W != h->W || s.H != h->H || s.D != h->D || s.precision != h->prec)
    throw Error(CELLS_E_INVALID, "the snapshot's grid or precision differs from this solver's");
  h->step = s.step;
  h->parity = s.parity & 1;
  h->uIn = s.uIn;
  h->cfg.u_in = s.uIn;
  h->rampKind = s.rampKind;
  h->rampTarget = s.rampTarget;
  h->rampSteps = s.rampSteps > 0 ? s.rampSteps : 1;
  h->rampEvery = s.rampEvery > 0 ? s.rampEvery : 1;
  h->argGen++;
  h->dev.h2d(h->f[h->parity], (const char*)in + sizeof(s), pop);
  h->dev.sync();
  h->write_state(1 | 2 | 4);
  h->forceSamplesRead = 0;
  h->forceSteps.clear();
  h->forceGeneration++;
  CELLS_CATCH(h)
}

int cells3d_read_flags(Cells3D* h, uint32_t* out, size_t n) {
  if (!h || !out) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (n != (size_t)h->N) throw Error(CELLS_E_INVALID, "read_flags needs N entries");
  h->dev.d2h(out, h->flags, n * 4);
  h->dev.sync();
  CELLS_CATCH(h)
}

int cells3d_timer_start(Cells3D* h) {
  if (!h) return CELLS_E_INVALID;
  CELLS_TRY(h)
  if (!h->dev.fake) check_cuda(cudaEventRecord(h->dev.ev0, h->dev.stream), "cudaEventRecord");
  CELLS_CATCH(h)
}

int cells3d_timer_stop(Cells3D* h, float* ms) {
  if (!h || !ms) return CELLS_E_INVALID;
  CELLS_TRY(h)
  *ms = 0.f;
  if (!h->dev.fake) {
    check_cuda(cudaEventRecord(h->dev.ev1, h->dev.stream), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(h->dev.ev1), "cudaEventSynchronize");
    check_cuda(cudaEventElapsedTime(ms, h->dev.ev0, h->dev.ev1), "cudaEventElapsedTime");
  }
  CELLS_CATCH(h)
}

int cells3d_launch_count(Cells3D* h, int64_t* count) {
  if (!h || !count) return CELLS_E_INVALID;
  *count = h->dev.launches;
  return CELLS_OK;
}

int cells3d_fake_set_force(Cells3D* h, double fx, double fy, double fz) {
  if (!h) return CELLS_E_INVALID;
  if (!h->dev.fake) {
    h->lastError = "fake_set_force is only for CELLS_FAKE_DEVICE handles";
    return CELLS_E_INVALID;
  }
  h->fakeForce[0] = fx;
  h->fakeForce[1] = fy;
  h->fakeForce[2] = fz;
  return CELLS_OK;
}

int64_t cells_fake_live_buffers(void) { return g_fake_live_buffers; }

}  // extern "C"
