// Fused D3Q19 step: pull streaming, boundaries (inlet, outlet, slip faces, Bouzidi walls), TRT
// collision with optional Smagorinsky, absorbing layer and sponge, momentum-exchange force and its
// reduction into the force history ring.
//
// Semantics follow the reference kernel src/shaders/step3d.ts:170-223 (main) and :119-168
// (pullSlow3); the arithmetic order of the moments, equilibria and collision is the generated WGSL's.
//
// B200 work split: one time step is two kernels that update disjoint sets of cells, both reading
// the source buffer and writing the destination buffer.
//   * bulk3d_kernel: every cell except the body cells. One thread per cell, blocks of (BX x BY)
//     cells of one z plane, x along warps, so each population load and store of a warp is one
//     contiguous run of the SoA array f[i*N + cell]. Interior cells take the fast path (19 plain
//     pulls, no flag read); the inlet plane, the outlet plane and the four slip faces take a
//     geometric boundary path whose pull sources follow from the coordinates alone. A cell reads
//     its flag word only when its row (y, z) holds a body cell (rowBody[]); such a cell with a
//     non-zero flag belongs to the body kernel and is skipped here. No forces arise in this kernel.
//   * body3d_kernel: the body cells, from a compact list built when the SDF changes: every fluid
//     cell with a non-zero flag in a row that holds a body cell. It runs the reference's full
//     pullSlow3 (Bouzidi walls, mirrored sources on solids, momentum exchange) and, on sampled
//     steps, reduces the forces: warp shuffles in f64, one partial per block, and the last block
//     to finish sums the partials in a fixed order into the force ring, so the result is
//     deterministic (the reference sums in atomic slot order, src/shaders/aux3d.ts:80).
//   * the relaxation rates and absorbing strength depend on x alone (without Smagorinsky) and come
//     from a W-entry table that the host fills with the reference's f32 arithmetic.
#include "kernels3d.h"

// Compiled twice: the product build (FMA contraction allowed) into cells::fast, and with
// -fmad=false -DCELLS_EXACT_ARITH into cells::exact, whose f32/f64 results round exactly as the
// written expressions state (bit-reproducible against a non-FMA CPU build of the same formulas).
#ifdef CELLS_EXACT_ARITH
#define CELLS_ARITH exact
constexpr bool kExact = true;
#else
#define CELLS_ARITH fast
constexpr bool kExact = false;
#endif

namespace cells {
namespace CELLS_ARITH {

template <class C>
struct StepArgs3 {
  using S = typename C::S;
  using R = typename C::R;
  // src + i*N - (c_ix + c_iy W + c_iz W H): the interior source of population i of cell idx is
  // pull[i][idx], one multiply-add from a constant-bank base
  const S* pull[Q3];
  S* out[Q3];  // dst + i*N
  const S* src;
  S* dst;
  const uint32_t* flags;
  const float* sdf;
  const uint8_t* rowBody;
  const typename Vec4<R>::T* xTab;  // per x: (omega+ without Smagorinsky, omega-, sigma, 0)
  BodyLinks3 links;
  const int* bodyCells;
  double4* partials;
  double4* history;
  DevState3* st;
  long long N;
  int W, H, D;
  int nBody;
  int rampKind, rampEvery;
  int par, sample;
  double rampTarget, rampSteps;
  R lambda, smagC2;
};

template <class R>
__device__ __forceinline__ R cu_of(int p, R ux, R uy, R uz) {
  // cu_a = 3 (c_a . u) for the lower member a of each pair, as cDotU writes it (step3d.ts:15-17)
  switch (p) {
    case 1: return R(3) * (ux);
    case 3: return R(3) * (uy);
    case 5: return R(3) * (uz);
    case 7: return R(3) * (ux + uy);
    case 9: return R(3) * (ux + uz);
    case 11: return R(3) * (uy + uz);
    case 13: return R(3) * (ux - uy);
    case 15: return R(3) * (ux - uz);
    default: return R(3) * (uy - uz);
  }
}

// w_i * SCALE: the equilibrium weights in storage units (exact, SCALE is a power of two)
template <class C>
__device__ __forceinline__ typename C::R ws3(int i) {
  using R = typename C::R;
  return w3<R>(i) * R(C::SCALE);
}

// feq(i, ...) in storage units (src/shaders/common3d.ts:38-41 times SCALE)
template <class C>
__device__ __forceinline__ typename C::R feq3s(int i, typename C::R rho, typename C::R ux, typename C::R uy,
                                               typename C::R uz) {
  using R = typename C::R;
  R cu = R(3) * (R(cx3(i)) * ux + R(cy3(i)) * uy + R(cz3(i)) * uz);
  return ws3<C>(i) * (rho - R(1) + rho * (cu + R(0.5) * cu * cu - R(1.5) * (ux * ux + uy * uy + uz * uz)));
}

// Moments, the outlet equilibrium or the TRT collision, and the 19 stores of one cell
// (src/shaders/step3d.ts:38-102 and :205-223). f holds the pulled populations in storage units;
// dividing the sums by SCALE and multiplying the weights by SCALE are exact, so every stored value
// equals the reference formula's.
template <class C, bool SMAG>
__device__ __forceinline__ void collide_store(const StepArgs3<C>& a, const typename C::R (&f)[Q3], int x, int idx,
                                              bool outlet) {
  using R = typename C::R;
  constexpr R IS = R(1) / R(C::SCALE);
  // moments, in the generated WGSL's left-to-right order
  R dsum = f[0];
#pragma unroll
  for (int i = 1; i < Q3; i++) dsum = dsum + f[i];
  const R drho = dsum * IS;
  const R rho = R(1) + drho;
  const R invRho = R(1) / rho;
  const R ux = ((f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16]) * IS) * invRho;
  const R uy = ((f[3] - f[4] + f[7] - f[8] + f[11] - f[12] - f[13] + f[14] + f[17] - f[18]) * IS) * invRho;
  const R uz = ((f[5] - f[6] + f[9] - f[10] + f[11] - f[12] - f[15] + f[16] - f[17] + f[18]) * IS) * invRho;
  const R usq = R(1.5) * (ux * ux + uy * uy + uz * uz);
  if (outlet) {
    // pressure outlet: equilibrium at rho = 1 with the node's own velocity
#pragma unroll
    for (int i = 0; i < Q3; i++) a.out[i][idx] = C::enc_raw(feq3s<C>(i, R(1), ux, uy, uz));
    return;
  }
  const auto tab = a.xTab[x];
  R omP = tab.x, omM = tab.y;
  const R sigma = tab.z;
  if (SMAG) {
    const R omegaBase = tab.x;
    R pxx = R(0), pyy = R(0), pzz = R(0), pxy = R(0), pxz = R(0), pyz = R(0);
    // each second moment accumulates in increasing index order, as the generated sums are written
#pragma unroll
    for (int p = 1; p < Q3; p += 2) {
      const R cu = cu_of<R>(p, ux, uy, uz);
      const R eqS = ws3<C>(p) * (drho + rho * (R(0.5) * cu * cu - usq));
      const R eqA = ws3<C>(p) * rho * cu;
      const R na = f[p] - (eqS + eqA);
      const R nb = f[p + 1] - (eqS - eqA);
      if (p == 1) pxx = na + nb;
      else if (cx3(p) != 0) pxx = pxx + na + nb;
      if (p == 3) pyy = na + nb;
      else if (cy3(p) != 0) pyy = pyy + na + nb;
      if (p == 5) pzz = na + nb;
      else if (cz3(p) != 0) pzz = pzz + na + nb;
      if (p == 7) pxy = na + nb;
      else if (cx3(p) * cy3(p) == -1) pxy = pxy - na - nb;
      if (p == 9) pxz = na + nb;
      else if (cx3(p) * cz3(p) == -1) pxz = pxz - na - nb;
      if (p == 11) pyz = na + nb;
      else if (cy3(p) * cz3(p) == -1) pyz = pyz - na - nb;
    }
    // sqrt(SCALE^2 x) = SCALE sqrt(x) exactly (SCALE^2 is a power of four)
    const R pi = sqrt(pxx * pxx + pyy * pyy + pzz * pzz + R(2) * (pxy * pxy + pxz * pxz + pyz * pyz)) * IS;
    const R t0 = R(1) / omegaBase;
    const R tEff = R(0.5) * (t0 + sqrt(t0 * t0 + R(25.45584412271571) * a.smagC2 * pi * invRho));
    omP = R(1) / tEff;
    omM = R(1) / (R(0.5) + a.lambda / (R(1) / omP - R(0.5)));
  }
  // absorbing layer: relax toward the inflow equilibrium
  R ut = R(0), dq = R(0);
  const bool absorb = sigma > R(0);
  if (absorb) {
    ut = (R)a.st->uIn[a.par];
    dq = R(1.5) * rho * (ut * ut - ux * ux - uy * uy - uz * uz);
  }
  {
    R s0 = R(0);
    if (absorb) s0 += sigma * ws3<C>(0) * -dq;
    R v = f[0] - omP * (f[0] - ws3<C>(0) * (drho - rho * usq));
    if (kExact || absorb) v = v + s0;
    a.out[0][idx] = C::enc_raw(v);
  }
#pragma unroll
  for (int p = 1; p < Q3; p += 2) {
    const R cu = cu_of<R>(p, ux, uy, uz);
    const R eqS = ws3<C>(p) * (drho + rho * (R(0.5) * cu * cu - usq));
    const R eqA = ws3<C>(p) * rho * cu;
    const R sym = omP * (R(0.5) * (f[p] + f[p + 1]) - eqS);
    const R asym = omM * (R(0.5) * (f[p] - f[p + 1]) - eqA);
    R va = f[p] - sym - asym;
    R vb = f[p + 1] - sym + asym;
    if (kExact || absorb) {
      R sS = R(0), sA = R(0);
      if (absorb) {
        const R cut = R(3) * R(cx3(p)) * ut;
        sS += sigma * ws3<C>(p) * (R(0.5) * rho * (cut * cut - cu * cu) - dq);
        sA += sigma * ws3<C>(p) * rho * (cut - cu);
      }
      va = va + sS + sA;
      vb = vb + sS - sA;
    }
    a.out[p][idx] = C::enc_raw(va);
    a.out[p + 1][idx] = C::enc_raw(vb);
  }
}

__device__ __forceinline__ double ramp_speed(int kind, double target, double rampSteps, int every, unsigned step) {
  const double sq = (double)((step / (unsigned)every) * (unsigned)every);
  const double t = fmin(1.0, sq / rampSteps);
  return kind == 1 ? target * t : target * (t * t * (3.0 - 2.0 * t));
}

// ---------------- bulk kernel ----------------

template <class C, bool SMAG>
__global__ void __launch_bounds__(256, sizeof(typename C::R) == 8 ? 2 : 4)
    bulk3d_kernel(const __grid_constant__ StepArgs3<C> a) {
  using R = typename C::R;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
    const unsigned s = a.st->step[a.par];
    a.st->step[a.par ^ 1] = s + 1u;
    if (a.rampKind != 0)
      a.st->uIn[a.par ^ 1] = ramp_speed(a.rampKind, a.rampTarget, a.rampSteps, a.rampEvery, s + 1u);
  }
  const int W = a.W, H = a.H, D = a.D;
  if (x >= W || y >= H) return;
  const int row = y + H * z;
  const int idx = x + W * row;
  const bool interior = x > 0 && x < W - 1 && y > 0 && y < H - 1 && z > 0 && z < D - 1;
  if (a.rowBody[row]) {
    // rows holding a body cell: any cell with a flag belongs to the body kernel
    if (__ldg(a.flags + idx) != 0u) return;
  }
  R f[Q3];
  bool outlet = false;
  if (interior) {
#pragma unroll
    for (int i = 0; i < Q3; i++) f[i] = C::raw(a.pull[i] + idx);
  } else {
    if (x == 0) {
      // inlet: equilibrium at the inflow speed, no collision (step3d.ts:190-193)
      const R u = (R)a.st->uIn[a.par];
#pragma unroll
      for (int i = 0; i < Q3; i++) a.out[i][idx] = C::enc_raw(feq3s<C>(i, R(1), u, R(0), R(0)));
      return;
    }
    outlet = x == W - 1;
    // geometric boundary pull: pullSlow3 (step3d.ts:119-168) for a cell without solid neighbours,
    // so every mirrored source is fluid
    const long long N = a.N;
    const long long WH = (long long)W * H;
    f[0] = C::raw(a.src + idx);
#pragma unroll
    for (int i = 1; i < Q3; i++) {
      const int sx = x - cx3(i), sy = y - cy3(i), sz = z - cz3(i);
      const bool outX = sx < 0 || sx >= W;
      const bool outY = sy < 0 || sy >= H;
      const bool outZ = sz < 0 || sz >= D;
      int pop = i;
      long long cell;
      if (!(outX || outY || outZ)) {
        cell = idx - (cx3(i) + cy3(i) * (long long)W + cz3(i) * WH);
      } else if (outX && outlet) {
        cell = (long long)(W - 2) + (long long)W * row;  // outlet: zero-gradient copy
      } else if (outY && outZ) {
        pop = opp3(i);  // edge: the double mirror equals bounce-back
        cell = idx;
      } else if (outY || outZ) {
        pop = outY ? mirror_y3(i) : mirror_z3(i);  // slip: specular reflection
        const int ry = outY ? y : sy;
        const int rz = outY ? sz : z;
        cell = (long long)sx + (long long)W * (ry + (long long)H * rz);
      } else {
        pop = opp3(i);
        cell = idx;
      }
      f[i] = C::raw(a.src + (long long)pop * N + cell);
    }
  }
  collide_store<C, SMAG>(a, f, x, idx, outlet);
}

// ---------------- body kernel ----------------

template <class C>
__device__ __forceinline__ void finish_forces(typename C::R fx, typename C::R fy, typename C::R fz, int nSlots,
                                              double4* __restrict__ partials, double4* __restrict__ history,
                                              DevState3* __restrict__ st) {
  __shared__ double red[3][32];
  __shared__ int amLast;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int lane = tid & 31, warp = tid >> 5, nwarps = (blockDim.x * blockDim.y + 31) >> 5;
  double dx = (double)fx, dy = (double)fy, dz = (double)fz;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dx += __shfl_down_sync(0xffffffffu, dx, o);
    dy += __shfl_down_sync(0xffffffffu, dy, o);
    dz += __shfl_down_sync(0xffffffffu, dz, o);
  }
  if (lane == 0) {
    red[0][warp] = dx;
    red[1][warp] = dy;
    red[2][warp] = dz;
  }
  __syncthreads();
  if (tid == 0) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int w = 0; w < nwarps; w++) {
      sx += red[0][w];
      sy += red[1][w];
      sz += red[2][w];
    }
    partials[blockIdx.x] = make_double4(sx, sy, sz, 0.0);
    __threadfence();
    const unsigned prev = atomicAdd(&st->done, 1u);
    amLast = (prev == (unsigned)(nSlots - 1));
  }
  __syncthreads();
  if (amLast && warp == 0) {
    __threadfence();
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int k = lane; k < nSlots; k += 32) {
      const double2* pk = reinterpret_cast<const double2*>(partials + k);
      const double2 v0 = __ldcg(pk);  // L2, bypassing L1: written by other blocks in this launch
      const double2 v1 = __ldcg(pk + 1);
      ax += v0.x;
      ay += v0.y;
      az += v1.x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ax += __shfl_down_sync(0xffffffffu, ax, o);
      ay += __shfl_down_sync(0xffffffffu, ay, o);
      az += __shfl_down_sync(0xffffffffu, az, o);
    }
    if (lane == 0) {
      const unsigned s = st->sample;
      history[s % HISTORY_LEN] = make_double4(ax, ay, az, 0.0);
      st->sample = s + 1u;
      st->done = 0u;
      if (!isfinite(ax) || !isfinite(ay) || !isfinite(az)) atomicOr(&st->status, 1u);
    }
  }
}

// One block handles 32 body cells with 32 x 19 threads: thread (lane, i) resolves link i of cell
// lane (a record load, then one or two source loads, all independent across threads) into shared
// memory; then one thread per cell sums the momentum exchange in the reference's direction order
// and collides.
template <class C, bool SMAG>
__global__ void __launch_bounds__(32 * Q3) body3d_kernel(const __grid_constant__ StepArgs3<C> a) {
  using R = typename C::R;
  __shared__ R sv[Q3][32];  // pulled populations in storage units
  __shared__ R sm[Q3][32];  // momentum-exchange term of each link (0 when the link exchanges none)
  const int lane = threadIdx.x, dir = threadIdx.y;
  const int t = blockIdx.x * 32 + lane;
  const bool valid = t < a.nBody;
  if (valid) {
    const int idx = a.bodyCells[t];
    if (dir == 0) {
      sv[0][lane] = C::raw(a.src + idx);
    } else {
      const int kind = (int)((__ldg(a.links.kinds + t) >> (3 * (dir - 1))) & 7ull);
      const Link3<R> L = ((const Link3<R>*)a.links.rec)[(long long)(dir - 1) * a.links.cap + t];
      const R fj = C::raw(a.src + L.e1);
      R v = fj, m = R(0);
      if (kind == LINK_SLIP_SOLID) {
        m = R(2) * fj;  // a body meets the slip face: bounce-back
      } else if (kind >= LINK_BOUZIDI_N) {
        // Bouzidi linear interpolated bounce-back (step3d.ts:152-167)
        if (kind == LINK_BOUZIDI_N) v = L.c1 * fj + L.c2 * C::raw(a.src + L.e2);
        else if (kind == LINK_BOUZIDI_H) v = fj / L.c1 + L.c2 * C::raw(a.src + L.e2);
        m = fj + v;
      }
      sv[dir][lane] = v;
      sm[dir][lane] = m;
    }
  }
  __syncthreads();
  R fx = R(0), fy = R(0), fz = R(0);
  if (dir == 0 && valid) do {
      const int idx = a.bodyCells[t];
      const int meta = a.links.meta[t];
      const int x = meta & ((1 << 29) - 1);
      if (meta & (1 << 30)) {
        // inlet cell of a body row: equilibrium at the inflow speed
        const R u = (R)a.st->uIn[a.par];
#pragma unroll
        for (int i = 0; i < Q3; i++) a.out[i][idx] = C::enc_raw(feq3s<C>(i, R(1), u, R(0), R(0)));
        break;
      }
      const unsigned long long kinds = __ldg(a.links.kinds + t);
      R f[Q3];
#pragma unroll
      for (int i = 0; i < Q3; i++) {
        f[i] = sv[i][lane];
        if (i > 0 && ((kinds >> (3 * (i - 1))) & 7ull) != LINK_LOAD) {
          const int j = opp3(i);
          const R m = sm[i][lane];
          fx += R(cx3(j)) * m;
          fy += R(cy3(j)) * m;
          fz += R(cz3(j)) * m;
        }
      }
      collide_store<C, SMAG>(a, f, x, idx, (meta & (1 << 29)) != 0);
    } while (0);
  // the momentum exchange was summed in storage units
  constexpr R IS = R(1) / R(C::SCALE);
  if (a.sample) finish_forces<C>(fx * IS, fy * IS, fz * IS, (int)gridDim.x, a.partials, a.history, a.st);
}

// ---------------- host-side launcher ----------------

int body_blocks3(int nBody);

template <class C>
static cudaError_t launch_step3_t(const StepLaunch3& L, const StepStreams3& ss) {
  using R = typename C::R;
  using S = typename C::S;
  StepArgs3<C> a;
  a.src = (const S*)L.src;
  a.dst = (S*)L.dst;
  const long long W = L.W, WH = (long long)L.W * L.H;
  for (int i = 0; i < Q3; i++) {
    const long long off = (long long)i * L.N - (cx3(i) + cy3(i) * W + cz3(i) * WH);
    a.pull[i] = (const S*)((uintptr_t)a.src + (intptr_t)(off * (long long)sizeof(S)));
    a.out[i] = a.dst + (size_t)i * (size_t)L.N;
  }
  a.flags = L.flags;
  a.sdf = L.sdf;
  a.rowBody = L.rowBody;
  a.xTab = (const typename Vec4<R>::T*)L.xTab;
  a.bodyCells = L.bodyCells;
  a.links = L.links;
  a.partials = L.partials;
  a.history = L.history;
  a.st = L.st;
  a.N = L.N;
  a.W = L.W;
  a.H = L.H;
  a.D = L.D;
  a.nBody = L.nBody;
  a.rampKind = L.rampKind;
  a.rampEvery = L.rampEvery > 0 ? L.rampEvery : 1;
  a.par = L.par;
  a.sample = L.sample;
  a.rampTarget = L.rampTarget;
  a.rampSteps = L.rampSteps;
  a.lambda = (R)L.lambda;
  a.smagC2 = (R)L.smagC2;
  dim3 block(L.bx, L.by, 1);
  dim3 grid((L.W + L.bx - 1) / L.bx, (L.H + L.by - 1) / L.by, L.D);
  const bool smag = L.smagC2 > 0;
  cudaError_t e;
  // the body kernel runs when there are body cells, and on sampled steps even without them (a
  // sample of zero force is still written to the ring, as the reference's reduce pass does). The
  // two kernels touch disjoint cells, so the body kernel runs on a side stream beside the bulk one.
  const bool body = L.nBody > 0 || L.sample;
  const bool side = body && ss.side != nullptr;
  cudaStream_t bs = side ? ss.side : ss.main;
  if (side) {
    if ((e = cudaEventRecord(ss.fork, ss.main)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ss.side, ss.fork, 0)) != cudaSuccess) return e;
  }
  if (body) {
    const int blocks = body_blocks3(L.nBody);
    const dim3 bblock(32, Q3, 1);
    if (smag)
      body3d_kernel<C, true><<<blocks, bblock, 0, bs>>>(a);
    else
      body3d_kernel<C, false><<<blocks, bblock, 0, bs>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (side && (e = cudaEventRecord(ss.join, ss.side)) != cudaSuccess) return e;
  if (smag)
    bulk3d_kernel<C, true><<<grid, block, 0, ss.main>>>(a);
  else
    bulk3d_kernel<C, false><<<grid, block, 0, ss.main>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (side) e = cudaStreamWaitEvent(ss.main, ss.join, 0);
  return e;
}

cudaError_t launch_step3(int precision, const StepLaunch3& a, const StepStreams3& ss) {
  switch (precision) {
    case 0: return launch_step3_t<CodecF32>(a, ss);
    case 1: return launch_step3_t<CodecF16>(a, ss);
    case 2: return launch_step3_t<CodecBF16>(a, ss);
    case 3: return launch_step3_t<CodecF64>(a, ss);
  }
  return cudaErrorInvalidValue;
}

int body_blocks3(int nBody) { return nBody > 0 ? (nBody + 31) / 32 : 1; }

}  // namespace CELLS_ARITH
}  // namespace cells
