/*
 * cells.h — C ABI of the B200 lattice Boltzmann wind-tunnel step engine (libcells.so).
 *
 * This is the drop-in boundary for the step API of slowernet/cells:
 *   class Solver3D   src/solver3d.ts:42-320   (D3Q19, FP32 / FP16 storage; BF16 and FP64 added here)
 *   class Solver     src/solver.ts:50-340     (D2Q9)
 * A Node-API addon (or ctypes, or any FFI) binds these functions one to one; each handle owns one
 * CUDA stream, and every call on a handle is ordered on that stream. Calls on one handle are not
 * thread-safe; different handles are independent.
 *
 * Conventions
 *   - Every function returns a cells_status; CELLS_OK is 0. cells_last_error(handle) gives the
 *     message of the last failure on that handle (or of the last failed create when handle is NULL).
 *   - Allocation failures use CELLS_E_ALLOC and a message that begins "Solver3D allocation failed: "
 *     (or "Solver allocation failed: " in 2D), the prefix the reference's callers test for
 *     (src/solver3d.ts:84-95, src/app3d.ts:180-190). A failed create frees everything it allocated.
 *   - Distributions are stored shifted (f_i - w_i), structure-of-arrays f[i*N + cell] with
 *     cell = x + W*(y + H*z), as in the reference (src/shaders/common3d.ts:34).
 */
#ifndef CELLS_H
#define CELLS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CELLS_OK = 0,
  CELLS_E_ALLOC = 1,                 /* "Solver3D allocation failed: ..." */
  CELLS_E_PRECISION_UNSUPPORTED = 2, /* reference: 'shader-f16 is not available on this device' */
  CELLS_E_INVALID = 3,               /* bad argument or call order */
  CELLS_E_CUDA = 4,                  /* a CUDA runtime error; message has the CUDA error string */
  CELLS_E_DIVERGED = 5,              /* a non-finite force or macro value was seen on the device */
  CELLS_E_TIMEOUT = 6                /* a bounded device-side wait ran out */
} cells_status;

/* Storage precision of the distributions. Arithmetic is f32 except for CELLS_FP64 (f64).
 * reference: Precision = 'fp16' | 'fp32' (src/shaders/common3d.ts:4). */
typedef enum {
  CELLS_FP32 = 0,
  CELLS_FP16 = 1, /* f16 scaled by 2^15, clamped to +-1.99 before the store (src/shaders/common3d.ts:52-63) */
  CELLS_BF16 = 2, /* bf16, unscaled, round to nearest even (not in the reference) */
  CELLS_FP64 = 3  /* f64 storage and arithmetic: the GPU oracle run (not in the reference) */
} cells_precision;

/* Device ordinal that selects the fake device: buffers live in host memory and kernels are not
 * run. It exists only to test the host-side logic (parameter packing, force-ring bookkeeping,
 * error conventions) without a GPU, as the reference's fakeDevice() does in src/solver3d.test.ts:13-69. */
#define CELLS_FAKE_DEVICE (-2)

/* Step-kernel arithmetic. FAST lets the compiler fuse multiply-adds (the tuned default). EXACT
 * rounds every operation as written (no contraction), which reproduces a non-FMA CPU evaluation of
 * the reference formulas bit for bit; it is slower only in arithmetic-bound configurations. */
#define CELLS_ARITH_FAST 0
#define CELLS_ARITH_EXACT 1

/* Inlet ramp kinds for cells3d_set_inlet_ramp (the reference ramps on the host: src/cases.ts:52-53). */
typedef enum { CELLS_RAMP_NONE = 0, CELLS_RAMP_LINEAR = 1, CELLS_RAMP_SMOOTHSTEP = 2 } cells_ramp_kind;

/* Solver3DConfig, src/solver3d.ts:11-31. Call cells3d_config_default() first: it fills the
 * reference defaults (src/solver3d.ts:110-119); then set the fields you need. */
typedef struct {
  int32_t width, height, depth;
  int32_t precision;        /* cells_precision */
  double tau;
  double lambda;            /* fixed TRT Lambda; NaN (default) follows trtLambda3(tau) */
  double smagorinsky;       /* C_s; 0 disables the subgrid model */
  double u_in;              /* inflow speed, already ramped by the caller */
  double sponge_fraction;   /* fraction of the length, ending at the outlet, where tau rises */
  double sponge_tau;
  double absorb;            /* peak rate of the outlet absorbing layer; 0 disables it */
  int32_t workgroup_size;   /* threads per block; 0 picks the tuned default */
  int32_t force_every;      /* sample the obstacle force every n steps; 0 disables sampling */
  int32_t device;           /* CUDA device ordinal, or CELLS_FAKE_DEVICE */
  int32_t fake_fail_alloc;  /* fake device only: the n-th allocation fails (0 = none) */
  uint64_t max_buffer_bytes; /* largest single buffer allowed; 0 = the device's free memory */
  int32_t arithmetic;       /* CELLS_ARITH_FAST (default) or CELLS_ARITH_EXACT */
  int32_t reserved1;
} Cells3DConfig;

/* One force sample: ForceSample3 {step, fx, fy, fz} (src/solver3d.ts:33-38), summed in f64. */
typedef struct {
  uint32_t step;
  uint32_t reserved;
  double fx, fy, fz;
} CellsForceSample;

typedef struct {
  int32_t W, H, D, precision;
  int64_t N;
  int64_t step;
  int32_t block_x, block_y; /* launch shape of the step kernel */
  int32_t force_every;
  int32_t n_body_cells;     /* cells the body kernel updates (fluid cells with a flag in rows with a body) */
} Cells3DInfo;

typedef struct Cells3D Cells3D;

/* ---------------- lifecycle ---------------- */

/* Fills the reference defaults: smagorinsky 0, u_in 0, sponge_fraction 0, sponge_tau 1, absorb 0,
 * workgroup_size 0 (tuned), force_every 1, lambda NaN, precision FP32, device 0. */
void cells3d_config_default(Cells3DConfig* cfg);

/* Solver3D.create (src/solver3d.ts:79-104). Checks the size before allocating anything, allocates
 * every buffer, fills the SDF with FAR = 1e6 and builds the flags. On failure *out is NULL and all
 * buffers are freed. */
int cells3d_create(const Cells3DConfig* cfg, Cells3D** out);
/* Solver3D.destroy (src/solver3d.ts:317-319). NULL is a no-op. */
void cells3d_destroy(Cells3D* h);
const char* cells_last_error(const void* handle_or_null);

/* ---------------- setters (src/solver3d.ts:183-194) ---------------- */
int cells3d_set_tau(Cells3D* h, double tau);               /* setTau */
int cells3d_set_smagorinsky(Cells3D* h, double cs);        /* setSmagorinsky: stores C_s^2 */
int cells3d_set_inlet(Cells3D* h, double u);               /* setInlet: already-ramped speed */
int cells3d_set_lambda(Cells3D* h, double lambda);         /* cfg.lambda; NaN restores trtLambda3(tau) */
/* Device-side inlet ramp (not in the reference, whose callers ramp on the host between chunks,
 * src/cases.ts:52-54): before the step that starts at step s the inlet speed is
 *   target * ramp(min(1, s_q / ramp_steps)),  s_q = s rounded down to a multiple of update_every,
 * ramp(t) = t (LINEAR) or t*t*(3-2t) (SMOOTHSTEP). update_every = 400 reproduces runRamped's
 * chunking exactly; 1 ramps every step. kind NONE returns to cells3d_set_inlet. */
int cells3d_set_inlet_ramp(Cells3D* h, int kind, double target, int64_t ramp_steps, int64_t update_every);

/* ---------------- geometry and state ---------------- */
/* setSdf (src/solver3d.ts:211-228): copies n = W*H*D floats (cells, negative inside) and rebuilds
 * flags; cells that stop being solid are refilled from their fluid neighbours. */
int cells3d_set_sdf(Cells3D* h, const float* sdf, size_t n);
/* initField (src/solver3d.ts:231-242): every fluid cell to equilibrium at the current inflow speed,
 * solids to rest; resets step, parity and forces. macro4n (may be NULL) is the 3D macro layout
 * (ux, uy, uz, rho) per cell and, when given, sets each fluid cell to its own equilibrium
 * (the 2D reference's initField(macro), src/solver.ts:220-234, extended to 3D). */
int cells3d_init_field(Cells3D* h, const float* macro4n);
int cells3d_reset_forces(Cells3D* h);                       /* resetForces */

/* ---------------- stepping ---------------- */
/* encodeSteps (src/solver3d.ts:252-267): enqueue n steps; returns without waiting. */
int cells3d_step(Cells3D* h, int64_t n);
/* No counterpart in the reference: builds the CUDA graphs that cells3d_step(h, n) from the current
 * step would replay (128 steps each), without running anything, so that a timed or latency-critical
 * run replays graphs only. A later parameter, SDF or ramp change invalidates them. */
int cells3d_prepare_steps(Cells3D* h, int64_t n);
/* encodeMacro (src/solver3d.ts:269-273): refresh the macro buffer from the latest populations. */
int cells3d_update_macro(Cells3D* h);
/* run (src/solver3d.ts:276-288): n steps, then the macro refresh, then wait for the GPU. The
 * reference refreshes the macro after every chunk; only the last refresh is observable, so the
 * chunk argument only bounds how many steps are enqueued before the host waits. */
int cells3d_run(Cells3D* h, int64_t n, int64_t chunk);
int cells3d_synchronize(Cells3D* h);

/* ---------------- readback ---------------- */
/* readMacro (src/solver3d.ts:290-292): 4N floats (ux, uy, uz, rho), rho = 0 in solids. Waits. */
int cells3d_read_macro(Cells3D* h, float* out4n);
/* readForces (src/solver3d.ts:295-315): the samples produced since the last call, oldest first,
 * at most 8192 (older ones are dropped, as the ring overwrote them). cap must be at least the
 * number available (8192 always suffices). */
int cells3d_read_forces(Cells3D* h, CellsForceSample* out, size_t cap, size_t* n_out);
/* The two halves of readForces, for callers that overlap the copy with other work: begin enqueues
 * the device-to-host copy; end waits for it. A reset_forces or init_field between the two makes the
 * read stale: end then returns 0 samples and keeps the later samples aligned (the reference's
 * generation check, src/solver3d.ts:298-304). */
int cells3d_read_forces_begin(Cells3D* h);
int cells3d_read_forces_end(Cells3D* h, CellsForceSample* out, size_t cap, size_t* n_out);
/* Device-side status bits: 1 = a non-finite force sample, 2 = a non-finite macro value. The word
 * is cleared at create and by init_field. */
int cells3d_read_status(Cells3D* h, uint32_t* status);
/* The divergence checks of the reference's pages (hasDiverged / fieldDiverged,
 * src/tunnel3d.ts:97-105: a non-finite force sample or macro value), answered from the device-side
 * status word instead of a scan of the read-back samples: CELLS_OK, or CELLS_E_DIVERGED with the
 * reason in cells_last_error. Waits for the stream. */
int cells3d_check_diverged(Cells3D* h);
int cells3d_get_info(Cells3D* h, Cells3DInfo* info);
/* The 64-byte Params3 block exactly as the reference packs it (src/shaders/common3d.ts:9-16,
 * src/solver3d.ts:197-208): u32 W,H,D,N,groupsX,0,0,0; f32 tau, lambda, smagC2, uIn,
 * spongeStart, tauSponge, absorb, 0. */
int cells3d_read_params(Cells3D* h, void* out64);
/* Total mass sum(rho) over fluid cells, accumulated in f64 on the device. Waits. */
int cells3d_mass(Cells3D* h, double* out);
/* Raw state access: the latest populations (19*N elements of the storage type), flags (N u32). */
int cells3d_read_populations(Cells3D* h, void* out, size_t bytes);
int cells3d_write_populations(Cells3D* h, const void* in, size_t bytes);
int cells3d_read_flags(Cells3D* h, uint32_t* out, size_t n);

/* ---------------- macro-field products (src/shaders/render3d.ts:33-65, 159-230) ----------------
 * Both read the macro buffer as of the last cells3d_update_macro or cells3d_run, as the
 * reference's slice and tracer passes read solver.macro, and wait for the result. */
#define CELLS_FIELD_SPEED 0     /* |u| / (1.6 u_ref), the slice's speed mode */
#define CELLS_FIELD_VORTICITY 1 /* |curl u| / (0.3 u_ref), curl from trilinear velocity at +-1 cell */
/* The slice quad of sliceShader (render3d.ts:159-177): axis 0/1/2 = x/y/z at pos * (dim - 1),
 * pos in [0, 1]; the two other axes span [-0.5, dim - 0.5] in order (y, z), (x, z) or (x, y) and are
 * sampled at the centres of nu x nv pixels: out[j * nu + i]. Solid nodes (nearest node, ties to
 * even) give NaN. With nu and nv equal to the in-plane dimensions the pixels are the cell centres. */
int cells3d_sample_slice(Cells3D* h, int axis, double pos, int mode, double u_ref, int nu, int nv, float* out);
/* advectShader (render3d.ts:196-230): one frame of `steps` lattice steps for `count` tracers.
 * particles: count x 8 floats (x, y, z, 0, ux, uy, uz, 0), updated in place; seeds: count x 4
 * floats (x, y, z, 0), where a tracer restarts when it leaves the box or enters a solid. */
int cells3d_advect_tracers(Cells3D* h, const float* seeds, float* particles, int count, double steps, double u_ref);

/* Allocation-free mass reduction. It has no counterpart in the reference. It is for callers that
 * cannot allocate device memory when they need the result: host applications or plugin frameworks
 * that own every device buffer and fix their device memory at start-up, and real-time loops that
 * must not risk the failure or the implicit synchronisation of cudaMalloc/cudaFree. The array it
 * uses is held by every GPU that loads the library until the process exits. The caller passes device pointers to
 * the populations (19 * n_cells values of the storage type, layout f[i * n_cells + cell]) and to
 * the flags (n_cells u32), a device pointer for the f64 result, and a CUDA stream (NULL = the
 * default stream); the call enqueues the work and returns without waiting. The partial sums live in
 * a fixed 64 KiB __device__ array, one partial per 8192 cells: grids above 67,108,864 cells are
 * rejected with CELLS_E_INVALID. Calls share that array, so calls that can overlap on the GPU
 * race and must be serialised by the caller; the array keeps the last call's partial sums, and
 * every call overwrites each partial it reads. The first call on a device (and the first under a
 * new context of it, e.g. after cudaDeviceReset) looks up the array's address; that first call
 * should come before any stream capture. Errors: cells_last_error(NULL). */
int cells3d_mass_noalloc(const void* populations, const uint32_t* flags, int64_t n_cells, int32_t precision,
                         double* out_device, void* stream);

/* ---------------- measurement ----------------
 * copyRoofline (src/bench.ts:61-95): the memory traffic of a step with no arithmetic. Copies q SoA
 * population arrays of n_cells elements of the precision's storage type between two device
 * buffers (swapped every launch), 4-byte words per thread (8 for f64), reading one u32 flag word
 * per word when with_flags is set (the reference's copy reads one per cell); runs `launches`
 * launches after up to 10 untimed ones and returns the CUDA-event time per launch. Allocates and
 * frees its own buffers (2 q n_cells bytes-per-element, plus flags). Errors: cells_last_error(NULL). */
int cells_copy_roofline(int device, int precision, int q, int64_t n_cells, int launches, int with_flags,
                        double* ms_per_launch);

/* ---------------- pinned host memory (no counterpart in the reference) ----------------
 * Page-locked host buffers for the arrays a caller passes in and reads back (SDF, macro fields,
 * populations): copies from and into them go straight over DMA, where pageable memory takes a
 * staged copy. Allocation is slow; allocate once and reuse. Errors: cells_last_error(NULL). */
int cells_host_alloc(size_t bytes, void** out);
void cells_host_free(void* p);

/* ---------------- discrete adjoint (no counterpart in the reference) ----------------
 * The forward/backward pair of a differentiable run: adjoint_forward steps the solver `steps`
 * steps from its current state (exactly like cells3d_step, plus a checkpoint of the populations
 * every checkpoint_every steps) and returns J = scale * mean over the window of the force
 * component; adjoint_backward then sweeps the discrete adjoint of those steps back to the start,
 * recomputing each segment of checkpoint_every steps from its checkpoint, and returns
 *   dJ_dsdf[N]  dJ/d(SDF value of every node): the shape gradient through the Bouzidi link
 *               fractions q(sdf) (cells whose solidity would flip are a discrete change and have
 *               no derivative);
 *   dJ_du_in    dJ/d(inflow speed): the ramp target when a device ramp is set, else the inlet speed,
 *               with `scale` held fixed (a caller whose scale is 2/(u^2 A) adds -2 J / u);
 *   adjoint_out the adjoint of the initial populations (19 N values of the storage type), for
 *               adjoint tests; terminal_adjoint (or NULL = 0) seeds the adjoint of the final state.
 * FP32 or FP64 storage, Smagorinsky off. Force samples of the window go to the force ring as usual
 * (other steps of the recorded run are not sampled). Any change to the solver after the forward
 * run (parameters, SDF, steps) invalidates it. */
typedef struct {
  int64_t steps;             /* steps of the recorded run */
  int64_t window_begin;      /* first and last step label (the step count after the step) */
  int64_t window_end;        /*   averaged by the objective; inside the recorded run */
  int32_t checkpoint_every;  /* K: one checkpoint of the populations every K steps */
  int32_t component;         /* force component: 0 x (drag), 1 y, 2 z */
  double scale;              /* J = scale * mean of the force component over the window */
} Cells3DAdjointSpec;

int cells3d_adjoint_forward(Cells3D* h, const Cells3DAdjointSpec* spec, double* objective);
int cells3d_adjoint_backward(Cells3D* h, const void* terminal_adjoint, double* dJ_dsdf, double* dJ_du_in,
                             void* adjoint_out);
/* Star-shaped body of the shape-gradient problem: r(theta, phi) = r0 (1 + sum_k coef[k] Y_k) about
 * (cx, cy, cz), theta the polar angle from +z, phi = atan2(dy, dx), Y_k the orthonormal real
 * spherical harmonics of degree l <= 3 in the order (l, m) = (0,0), (1,-1), (1,0), (1,1), (2,-2) ...
 * (3,3), without the Condon-Shortley phase. Host functions; no device work.
 *   star_sdf            stamps min(sdf, |p - c| - r(theta, phi)) over the body's bounding box
 *                       grown by 3 cells (the margin of every shape, src/geometry3d.ts:15-27);
 *   star_coef_gradient  dJ/dcoef_k = sum_n dJ_dsdf[n] * (-r0 Y_k(theta_n, phi_n)), the chain rule
 *                       from adjoint_backward's dJ/dSDF to the 16 coefficients;
 *   adjoint_backward_star  adjoint_backward followed by that projection: the shape gradient in
 *                       coefficients and dJ/du_in (same meaning as in adjoint_backward).
 * Errors of the first two: cells_last_error(NULL); of the third: cells_last_error(h). */
typedef struct {
  double cx, cy, cz, r0;
  double coef[16];
} CellsStar3D;

int cells3d_star_sdf(float* sdf, int32_t W, int32_t H, int32_t D, const CellsStar3D* star);
int cells3d_star_coef_gradient(const CellsStar3D* star, int32_t W, int32_t H, int32_t D, const double* dJ_dsdf,
                               double* dJ_dcoef16);
int cells3d_adjoint_backward_star(Cells3D* h, const CellsStar3D* star, double* dJ_dcoef16, double* dJ_du_in);
/* Frees the recorded run's checkpoints and tables. Without it two device blocks stay with the
 * handle after a run -- one holding the checkpoints, the recompute buffers and the adjoint states,
 * one sized by the run for its link tables and small buffers -- and the next adjoint_forward
 * reuses them while they fit (an optimisation loop allocates them once). */
int cells3d_adjoint_release(Cells3D* h);

/* ---------------- state save / restore (no counterpart in the reference) ----------------
 * A snapshot of the simulation state for resuming long runs: the latest populations, the step
 * count, the parity, the inlet speed and the device-side ramp. The geometry (SDF) and the
 * parameters are not included: restore into a handle created with the same config and SDF.
 * Loading resets the force ring (like init_field). */
int cells3d_state_size(Cells3D* h, size_t* bytes);
int cells3d_save_state(Cells3D* h, void* out, size_t bytes);
int cells3d_load_state(Cells3D* h, const void* in, size_t bytes);

/* ---------------- timing (CUDA events on the handle's stream) ---------------- */
int cells3d_timer_start(Cells3D* h);
int cells3d_timer_stop(Cells3D* h, float* ms);
/* Kernel launches this handle has issued since it was created (graph replays count each node). */
int cells3d_launch_count(Cells3D* h, int64_t* count);

/* ---------------- fake-device hooks (host-logic tests only) ---------------- */
/* On a CELLS_FAKE_DEVICE handle, every force sample that a step would reduce is written as
 * (fx, fy, fz). Any other handle returns CELLS_E_INVALID. */
int cells3d_fake_set_force(Cells3D* h, double fx, double fy, double fz);
/* Live fake-device buffers in this process (a failed create must leave this unchanged). */
int64_t cells_fake_live_buffers(void);

/* =====================================================================================
 * D2Q9: class Solver, src/solver.ts:50-340, and batches of independent 2D tunnels.
 *
 * A Cells2D handle is one tunnel. cells2d_create makes a batch of one and returns its tunnel;
 * cells2d_batch_create makes many tunnels of different sizes that advance together, one kernel
 * launch per step for all of them (or one persistent launch for many steps), and
 * cells2d_batch_tunnel gives a handle to each for the per-tunnel calls (geometry, parameters,
 * readback). Stepping a tunnel of a batch of more than one is an error: step the batch.
 * Distributions are f[i*N + x + W*y], shifted by w_i (src/shaders/step.ts:7).
 * ===================================================================================== */

/* XMode and YMode, src/lattice.ts:17-28 */
typedef enum { CELLS_X_PERIODIC = 0, CELLS_X_WALL = 1, CELLS_X_OPEN = 2 } cells_x_mode;
typedef enum { CELLS_Y_PERIODIC = 0, CELLS_Y_NOSLIP = 1, CELLS_Y_SLIP = 2, CELLS_Y_MOVING = 3 } cells_y_mode;

/* SolverConfig, src/solver.ts:15-40. cells2d_config_default() fills the reference defaults
 * (src/solver.ts:98-112); then set the fields you need. */
typedef struct {
  int32_t width, height;
  int32_t left, right;        /* cells_x_mode; OPEN makes x = 0 a Zou-He velocity inlet and x = W-1 a
                                 Zou-He pressure outlet (rho = 1) */
  int32_t bottom, top;        /* cells_y_mode */
  int32_t precision;          /* CELLS_FP32 (the reference) or CELLS_FP64 */
  int32_t parabolic;          /* parabolic inlet profile with peak u_in (src/shaders/common.ts:39-45) */
  double tau;
  double lambda;              /* TRT magic parameter; default 3/16 (MAGIC_LAMBDA, src/lattice.ts:35) */
  double smagorinsky;         /* C_s; 0 disables the subgrid model */
  double u_in;                /* inflow speed (peak of the parabola when parabolic) */
  double u_lid;               /* moving-wall speed */
  double sponge_fraction;     /* fraction of the length, ending at the outlet, where tau rises */
  double sponge_tau;
  double body_force[2];       /* Guo body force (fx, fy) */
  double absorb;              /* peak rate of the absorbing layers */
  double inlet_layer_fraction;/* fraction of the length, from the inlet, with an absorbing layer */
  int32_t workgroup_size;     /* threads per block: 64, 128 or 256 (rows of 32); 0 = default (64 x 2) */
  int32_t force_every;        /* sample the obstacle force every n steps; 0 disables */
  int32_t device;             /* CUDA device ordinal, or CELLS_FAKE_DEVICE */
  int32_t fake_fail_alloc;    /* fake device only: the n-th allocation fails (0 = none) */
  uint64_t max_buffer_bytes;  /* largest single buffer allowed; 0 = the device's free memory */
  int32_t arithmetic;         /* CELLS_ARITH_FAST (default) or CELLS_ARITH_EXACT */
  int32_t reserved1;
} Cells2DConfig;

typedef struct {
  int32_t W, H, precision, force_every;
  int64_t N;
  int64_t step;
  int32_t tile_x, tile_y;     /* block shape of the batch's step kernel */
  int32_t persistent;         /* 1 when the batch steps with the persistent kernel */
  int32_t tunnels;            /* tunnels in the batch */
} Cells2DInfo;

typedef struct Cells2D Cells2D;
typedef struct Cells2DBatch Cells2DBatch;

void cells2d_config_default(Cells2DConfig* cfg);
/* Solver.create (src/solver.ts:87-134): allocates, fills the SDF with 1e6 and builds the flags. On
 * failure *out is NULL, everything allocated is freed, and allocation failures carry the message
 * prefix "Solver allocation failed: ". */
int cells2d_create(const Cells2DConfig* cfg, Cells2D** out);
/* destroy (src/solver.ts:337-339). For a tunnel of a batch this releases only the handle. */
void cells2d_destroy(Cells2D* h);
/* update(partial) (src/solver.ts:175-178): takes a whole config, of which every field but width,
 * height, precision, device and arithmetic may differ from the current one. */
int cells2d_update(Cells2D* h, const Cells2DConfig* cfg);
int cells2d_get_config(Cells2D* h, Cells2DConfig* cfg);
int cells2d_set_inlet(Cells2D* h, double u);  /* update({ uIn: u }) */
/* Device-side inlet ramp, as cells3d_set_inlet_ramp; update_every = 400 with SMOOTHSTEP reproduces
 * the reference's runRamped (src/cases.ts:41-59). */
int cells2d_set_inlet_ramp(Cells2D* h, int kind, double target, int64_t ramp_steps, int64_t update_every);
/* setSdf (src/solver.ts:200-203): W*H floats, negative inside; rebuilds flags and refills
 * uncovered cells. */
int cells2d_set_sdf(Cells2D* h, const float* sdf, size_t n);
/* brush / brushStroke (src/solver.ts:244-268): union (erase 0) or subtract (erase 1) a disc of
 * radius r into the SDF; brush_stroke stamps n_points discs at xy[2k], xy[2k+1] and rebuilds once. */
int cells2d_brush(Cells2D* h, double cx, double cy, double r, int erase, int rebuild);
int cells2d_brush_stroke(Cells2D* h, const double* xy, size_t n_points, double r, int erase);
int cells2d_read_sdf(Cells2D* h, float* out, size_t n);
/* initField(macro?) (src/solver.ts:219-234): macro4n is (rho, ux, uy, unused) per cell, NULL = rest.
 * Resets the tunnel's step and forces. */
int cells2d_init_field(Cells2D* h, const float* macro4n);
int cells2d_reset_forces(Cells2D* h);
/* encodeSteps / encodeMacro / run (src/solver.ts:270-307); tunnels of a multi-tunnel batch step
 * with cells2d_batch_step. */
int cells2d_step(Cells2D* h, int64_t n);
int cells2d_update_macro(Cells2D* h);
int cells2d_run(Cells2D* h, int64_t n, int64_t chunk);
int cells2d_synchronize(Cells2D* h);
/* readMacro (src/solver.ts:309-311): 4N floats (rho, ux, uy, solid) as of the last macro refresh. */
int cells2d_read_macro(Cells2D* h, float* out4n);
/* readForces (src/solver.ts:314-335) with the same ring window and generation check as 3D; fz = 0. */
int cells2d_read_forces(Cells2D* h, CellsForceSample* out, size_t cap, size_t* n_out);
int cells2d_read_forces_begin(Cells2D* h);
int cells2d_read_forces_end(Cells2D* h, CellsForceSample* out, size_t cap, size_t* n_out);
/* bits: 1 non-finite force sample, 2 non-finite macro value (both cleared by init_field), 4 a
 * persistent-launch barrier timed out */
int cells2d_read_status(Cells2D* h, uint32_t* status);
/* CELLS_OK, or CELLS_E_DIVERGED when status bit 1 or 2 is set (hasDiverged / fieldDiverged of
 * src/tunnel3d.ts:97-105, as the 2D page applies them, src/app.ts:433-460). */
int cells2d_check_diverged(Cells2D* h);
int cells2d_get_info(Cells2D* h, Cells2DInfo* info);
/* The 96-byte Params block as the reference packs it (src/shaders/common.ts:14-22,
 * src/solver.ts:180-197). */
int cells2d_read_params(Cells2D* h, void* out96);
int cells2d_mass(Cells2D* h, double* out);
int cells2d_read_populations(Cells2D* h, void* out, size_t bytes);
int cells2d_write_populations(Cells2D* h, const void* in, size_t bytes);
int cells2d_read_flags(Cells2D* h, uint32_t* out, size_t n);
int cells2d_timer_start(Cells2D* h);
int cells2d_timer_stop(Cells2D* h, float* ms);
int cells2d_launch_count(Cells2D* h, int64_t* count);
int cells2d_fake_set_force(Cells2D* h, double fx, double fy);

/* ---------------- batches (no counterpart in the reference) ---------------- */
/* count tunnels, each with its own config; precision, device and arithmetic must agree. */
int cells2d_batch_create(const Cells2DConfig* cfgs, int32_t count, Cells2DBatch** out);
void cells2d_batch_destroy(Cells2DBatch* b);
/* A handle to tunnel k for the per-tunnel calls; valid until the batch is destroyed. */
int cells2d_batch_tunnel(Cells2DBatch* b, int32_t k, Cells2D** out);
/* n steps of every tunnel: one launch per step (replayed from CUDA graphs of 100 steps), or
 * persistent launches of many steps when the autotuner chose that. */
int cells2d_batch_step(Cells2DBatch* b, int64_t n);
/* n steps, then every tunnel's macro refresh, then wait. */
int cells2d_batch_run(Cells2DBatch* b, int64_t n);
int cells2d_batch_synchronize(Cells2DBatch* b);
/* Times trial_steps steps of each candidate launch shape (block shapes x per-step graphs or the
 * persistent kernel) on a copy of the current state, keeps the fastest, and restores the state:
 * populations, step counters, inlet speeds and force rings are as before the call. Writes the
 * chosen shape to *info when info is not NULL. */
int cells2d_batch_autotune(Cells2DBatch* b, int32_t trial_steps, Cells2DInfo* info);
/* Fixes the launch shape by hand: tile_x * tile_y threads (64, 128 or 256, tile_x a multiple of 32),
 * persistent 0 or 1. A block covers tile_x x tile_y cells, or tile_x x 2 tile_y (two rows per
 * thread) when the batch has 4,096 tiles or more at one row per thread. */
int cells2d_batch_set_launch(Cells2DBatch* b, int32_t tile_x, int32_t tile_y, int32_t persistent);
int cells2d_batch_get_info(Cells2DBatch* b, Cells2DInfo* info);
/* Test hook of the persistent kernel's time-out path: with extra_arrivals = 1 every grid barrier of
 * the following persistent launches waits for one arrival that never comes, so the bounded wait
 * (one second) runs out, the kernel winds down, and the call that waits for it returns
 * CELLS_E_TIMEOUT and clears the device error flag; the tunnels are then part-stepped until they
 * are re-initialised. 0 (the default) restores normal barriers. */
int cells2d_batch_set_barrier_test(Cells2DBatch* b, int32_t extra_arrivals);
int cells2d_batch_timer_start(Cells2DBatch* b);
int cells2d_batch_timer_stop(Cells2DBatch* b, float* ms);
int cells2d_batch_launch_count(Cells2DBatch* b, int64_t* count);

#ifdef __cplusplus
}
#endif

#endif /* CELLS_H */
