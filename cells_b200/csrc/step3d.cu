// Fused D3Q19 step: pull streaming, boundaries (inlet, outlet, slip faces, Bouzidi walls), TRT
// collision with optional Smagorinsky, absorbing layer and sponge, momentum-exchange force and its
// reduction into the force history ring, all in one kernel per time step.
//
// Semantics follow the reference kernel src/shaders/step3d.ts:170-223 (main) and :119-168
// (pullSlow3); the arithmetic order of the moments, equilibria and collision is the generated WGSL's.
//
// B200 layout and work split
//   * one thread per cell, blocks of (BX x BY) cells in one z plane: x runs along warps, so every
//     population load and store of a warp is one contiguous 32-element run (SoA f[i*N + cell]);
//   * interior cells take the fast path with exactly 19 loads and no flag read: a cell needs its
//     flag word only when its row (y, z) holds a body cell (rowBody[]), otherwise the flag is
//     derived from its coordinates (inlet plane, outlet plane, the four slip faces);
//   * the relaxation rate and absorbing strength depend on x alone and come from a W-entry table;
//   * forces: each cell's momentum exchange stays in registers; blocks that contain body rows
//     (force blocks) reduce it with warp shuffles in f64 into one partial each on sampled steps,
//     and the last force block to finish sums the partials in a fixed order into the ring. The
//     result is deterministic, unlike the reference's atomic slot order (src/shaders/aux3d.ts:80).
#include "kernels3d.h"

// Compiled twice: the product build (FMA contraction allowed) into cells::fast, and with
// -fmad=false -DCELLS_EXACT_ARITH into cells::exact, whose f32/f64 results round exactly as the
// written expressions state (bit-reproducible against a non-FMA CPU build of the same formulas).
#ifdef CELLS_EXACT_ARITH
#define CELLS_ARITH exact
#else
#define CELLS_ARITH fast
#endif

namespace cells {
namespace CELLS_ARITH {

template <class R>
__device__ __forceinline__ R feq3(int i, R rho, R ux, R uy, R uz) {
  R cu = R(3) * (R(cx3(i)) * ux + R(cy3(i)) * uy + R(cz3(i)) * uz);
  return w3<R>(i) * (rho - R(1) + rho * (cu + R(0.5) * cu * cu - R(1.5) * (ux * ux + uy * uy + uz * uz)));
}

// Flag word of a cell in a row without body cells: inlet/outlet bits plus the directions whose
// upstream node is off the grid (what flags3dShader computes when no neighbour is solid).
__device__ __forceinline__ uint32_t geom_flag3(int x, int y, int z, int W, int H, int D) {
  if (x > 0 && x < W - 1 && y > 0 && y < H - 1 && z > 0 && z < D - 1) return 0u;
  uint32_t bits = 0u;
  if (x == 0) bits = FLAG3_INLET;
  if (x == W - 1) bits = FLAG3_OUTLET;
#pragma unroll
  for (int i = 1; i < Q3; i++) {
    const int sx = x - cx3(i), sy = y - cy3(i), sz = z - cz3(i);
    if (sx < 0 || sx >= W || sy < 0 || sy >= H || sz < 0 || sz >= D) bits |= 1u << i;
  }
  return bits;
}

template <class C>
struct Cell3 {
  using S = typename C::S;
  using R = typename C::R;
  const S* __restrict__ src;
  const uint32_t* __restrict__ flags;
  const float* __restrict__ sdf;
  int W, H, D;
  size_t N;

  __device__ __forceinline__ int at(int x, int y, int z) const { return x + W * (y + H * z); }
  __device__ __forceinline__ R ld(int i, int cell) const { return C::load(src + (size_t)i * N + cell); }
  __device__ __forceinline__ bool solid(int cell) const { return (__ldg(flags + cell) & FLAG3_SOLID) != 0u; }

  // src/shaders/step3d.ts:119-168
  __device__ __forceinline__ R pull_slow(int i, int x, int y, int z, int idx, uint32_t fl, bool outlet, R& fx, R& fy,
                                         R& fz) const {
    const int j = opp3(i);
    const int sx = x - cx3(i), sy = y - cy3(i), sz = z - cz3(i);
    if ((fl & (1u << i)) == 0u) return ld(i, at(sx, sy, sz));
    const bool outX = sx < 0 || sx >= W;
    const bool outY = sy < 0 || sy >= H;
    const bool outZ = sz < 0 || sz >= D;
    if (outX && outlet) return ld(i, at(W - 2, y, z));  // outlet: zero-gradient copy
    if (outY && outZ) return ld(j, idx);                // edge: double mirror = bounce-back
    if (outY || outZ) {
      // slip: specular reflection across the face, bounce-back where a body meets the face
      const int ry = outY ? y : sy;
      const int rz = outY ? sz : z;
      const int m = outY ? mirror_y3(i) : mirror_z3(i);
      const int rs = at(sx, ry, rz);
      if (solid(rs)) {
        const R fj = ld(j, idx);
        const R t = R(2) * fj;
        fx += R(cx3(j)) * t;
        fy += R(cy3(j)) * t;
        fz += R(cz3(j)) * t;
        return fj;
      }
      return ld(m, rs);
    }
    if (outX) return ld(j, idx);
    const int s = at(sx, sy, sz);
    if (!solid(s)) return ld(i, s);
    // Bouzidi linear interpolated bounce-back; q is the fluid fraction of the link
    const R fj = ld(j, idx);
    const R dF = R(__ldg(sdf + idx));
    const R dS = R(__ldg(sdf + s));
    R q = dF / max(dF - dS, R(1e-6));
    q = min(max(q, R(1e-3)), R(1));
    R fi = fj;
    if (q < R(0.5)) {
      const int nx = x + cx3(i), ny = y + cy3(i), nz = z + cz3(i);
      if (nx >= 0 && nx < W && ny >= 0 && ny < H && nz >= 0 && nz < D) {
        const int n = at(nx, ny, nz);
        if (!solid(n)) fi = R(2) * q * fj + (R(1) - R(2) * q) * ld(j, n);
      }
    } else {
      fi = fj / (R(2) * q) + (R(2) * q - R(1)) / (R(2) * q) * ld(i, idx);
    }
    const R t = fj + fi;
    fx += R(cx3(j)) * t;
    fy += R(cy3(j)) * t;
    fz += R(cz3(j)) * t;
    return fi;
  }
};

template <class C>
__device__ __forceinline__ void store_pop(typename C::S* __restrict__ dst, int i, size_t N, int idx,
                                          typename C::R v) {
  dst[(size_t)i * N + idx] = C::enc(v);
}

template <class C>
__device__ __forceinline__ void finish_forces(typename C::R fx, typename C::R fy, typename C::R fz, int slot,
                                              int nSlots, double4* __restrict__ partials,
                                              double4* __restrict__ history, DevState3* __restrict__ st) {
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
    partials[slot] = make_double4(sx, sy, sz, 0.0);
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

__device__ __forceinline__ double ramp_speed(int kind, double target, double rampSteps, int every, unsigned step) {
  const double sq = (double)((step / (unsigned)every) * (unsigned)every);
  const double t = fmin(1.0, sq / rampSteps);
  return kind == 1 ? target * t : target * (t * t * (3.0 - 2.0 * t));
}

template <class C>
__global__ void __launch_bounds__(256) step3d_kernel(const typename C::S* __restrict__ src,
                                                     typename C::S* __restrict__ dst,
                                                     const uint32_t* __restrict__ flags,
                                                     const float* __restrict__ sdf,
                                                     const uint8_t* __restrict__ rowBody,
                                                     const typename C::R* __restrict__ xTab,
                                                     const int* __restrict__ blockSlot,
                                                     double4* __restrict__ partials, double4* __restrict__ history,
                                                     DevState3* __restrict__ st, const StepParams3<typename C::R> p,
                                                     const int par, const int sample) {
  using R = typename C::R;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  R fx = R(0), fy = R(0), fz = R(0);

  if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
    const unsigned s = st->step[par];
    st->step[par ^ 1] = s + 1u;
    if (p.rampKind != 0) st->uIn[par ^ 1] = ramp_speed(p.rampKind, p.rampTarget, p.rampSteps, p.rampEvery, s + 1u);
  }

  if (x < p.W && y < p.H) do {
      const int W = p.W, H = p.H;
      const size_t N = (size_t)p.N;
      const int row = y + H * z;
      const int idx = x + W * row;
      const uint32_t fl = rowBody[row] ? __ldg(flags + idx) : geom_flag3(x, y, z, W, H, p.D);
      R f[Q3];
      bool outlet = false;
      if (fl == 0u) {
        // fast path: 19 plain pulls
        const typename C::S* s0 = src + idx;
        const int WH = W * H;
#pragma unroll
        for (int i = 0; i < Q3; i++) {
          const long off = (long)i * (long)N - (long)(cx3(i) + cy3(i) * W + cz3(i) * WH);
          f[i] = C::load(s0 + off);
        }
      } else {
        if (fl & FLAG3_SOLID) break;  // solids keep their stale values, as in the reference
        if (fl & FLAG3_INLET) {
          const R u = (R)st->uIn[par];
#pragma unroll
          for (int i = 0; i < Q3; i++) store_pop<C>(dst, i, N, idx, feq3<R>(i, R(1), u, R(0), R(0)));
          break;
        }
        outlet = (fl & FLAG3_OUTLET) != 0u;
        Cell3<C> c{src, flags, sdf, W, H, p.D, N};
        f[0] = c.ld(0, idx);
#pragma unroll
        for (int i = 1; i < Q3; i++) f[i] = c.pull_slow(i, x, y, z, idx, fl, outlet, fx, fy, fz);
      }

      // moments, in the generated WGSL's left-to-right order
      R drho = f[0];
#pragma unroll
      for (int i = 1; i < Q3; i++) drho = drho + f[i];
      const R rho = R(1) + drho;
      const R invRho = R(1) / rho;
      const R ux = (f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16]) * invRho;
      const R uy = (f[3] - f[4] + f[7] - f[8] + f[11] - f[12] - f[13] + f[14] + f[17] - f[18]) * invRho;
      const R uz = (f[5] - f[6] + f[9] - f[10] + f[11] - f[12] - f[15] + f[16] - f[17] + f[18]) * invRho;
      const R usq = R(1.5) * (ux * ux + uy * uy + uz * uz);
      if (outlet) {
        // pressure outlet: equilibrium at rho = 1 with the node's own velocity
#pragma unroll
        for (int i = 0; i < Q3; i++) store_pop<C>(dst, i, N, idx, feq3<R>(i, R(1), ux, uy, uz));
        break;
      }
      R cu[Q3];
      cu[1] = R(3) * (ux);
      cu[3] = R(3) * (uy);
      cu[5] = R(3) * (uz);
      cu[7] = R(3) * (ux + uy);
      cu[9] = R(3) * (ux + uz);
      cu[11] = R(3) * (uy + uz);
      cu[13] = R(3) * (ux - uy);
      cu[15] = R(3) * (ux - uz);
      cu[17] = R(3) * (uy - uz);
      R eqS[Q3], eqA[Q3];
#pragma unroll
      for (int a = 1; a < Q3; a += 2) {
        eqS[a] = w3<R>(a) * (drho + rho * (R(0.5) * cu[a] * cu[a] - usq));
        eqA[a] = w3<R>(a) * rho * cu[a];
      }
      const R omegaBase = xTab[2 * x];
      const R sigma = xTab[2 * x + 1];
      R omP = omegaBase;
      if (p.smagC2 > R(0)) {
        R n[Q3];
#pragma unroll
        for (int a = 1; a < Q3; a += 2) {
          n[a] = f[a] - (eqS[a] + eqA[a]);
          n[a + 1] = f[a + 1] - (eqS[a] - eqA[a]);
        }
        const R pxx = n[1] + n[2] + n[7] + n[8] + n[9] + n[10] + n[13] + n[14] + n[15] + n[16];
        const R pyy = n[3] + n[4] + n[7] + n[8] + n[11] + n[12] + n[13] + n[14] + n[17] + n[18];
        const R pzz = n[5] + n[6] + n[9] + n[10] + n[11] + n[12] + n[15] + n[16] + n[17] + n[18];
        const R pxy = n[7] + n[8] - n[13] - n[14];
        const R pxz = n[9] + n[10] - n[15] - n[16];
        const R pyz = n[11] + n[12] - n[17] - n[18];
        const R pi = sqrt(pxx * pxx + pyy * pyy + pzz * pzz + R(2) * (pxy * pxy + pxz * pxz + pyz * pyz));
        const R t0 = R(1) / omegaBase;
        const R tEff = R(0.5) * (t0 + sqrt(t0 * t0 + R(25.45584412271571) * p.smagC2 * pi * invRho));
        omP = R(1) / tEff;
      }
      const R omM = R(1) / (R(0.5) + p.lambda / (R(1) / omP - R(0.5)));
      R s0 = R(0);
      R sS[Q3], sA[Q3];
#pragma unroll
      for (int a = 1; a < Q3; a += 2) sS[a] = sA[a] = R(0);
      if (sigma > R(0)) {
        // absorbing layer: relax toward the inflow equilibrium
        const R ut = (R)st->uIn[par];
        const R dq = R(1.5) * rho * (ut * ut - ux * ux - uy * uy - uz * uz);
        s0 += sigma * w3<R>(0) * -dq;
#pragma unroll
        for (int a = 1; a < Q3; a += 2) {
          const R cut = R(3) * R(cx3(a)) * ut;
          sS[a] += sigma * w3<R>(a) * (R(0.5) * rho * (cut * cut - cu[a] * cu[a]) - dq);
          sA[a] += sigma * w3<R>(a) * rho * (cut - cu[a]);
        }
      }
      store_pop<C>(dst, 0, N, idx, f[0] - omP * (f[0] - w3<R>(0) * (drho - rho * usq)) + s0);
#pragma unroll
      for (int a = 1; a < Q3; a += 2) {
        const int b = a + 1;
        const R sym = omP * (R(0.5) * (f[a] + f[b]) - eqS[a]);
        const R asym = omM * (R(0.5) * (f[a] - f[b]) - eqA[a]);
        store_pop<C>(dst, a, N, idx, f[a] - sym - asym + sS[a] + sA[a]);
        store_pop<C>(dst, b, N, idx, f[b] - sym + asym + sS[a] - sA[a]);
      }
    } while (0);

  if (sample) {
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const int slot = blockSlot[bid];
    if (slot >= 0) finish_forces<C>(fx, fy, fz, slot, p.nForceBlocks, partials, history, st);
  }
}

// ---------------- host-side launchers ----------------



template <class C>
static cudaError_t launch_step3_t(const StepLaunch3& a, cudaStream_t s) {
  using R = typename C::R;
  StepParams3<R> p;
  p.W = a.W;
  p.H = a.H;
  p.D = a.D;
  p.N = a.N;
  p.nForceBlocks = a.nForceBlocks;
  p.rampKind = a.rampKind;
  p.rampEvery = a.rampEvery > 0 ? a.rampEvery : 1;
  p.pad = 0;
  p.rampTarget = a.rampTarget;
  p.rampSteps = a.rampSteps;
  p.lambda = (R)a.lambda;
  p.smagC2 = (R)a.smagC2;
  dim3 block(a.bx, a.by, 1);
  dim3 grid((a.W + a.bx - 1) / a.bx, (a.H + a.by - 1) / a.by, a.D);
  step3d_kernel<C><<<grid, block, 0, s>>>((const typename C::S*)a.src, (typename C::S*)a.dst, a.flags, a.sdf,
                                          a.rowBody, (const R*)a.xTab, a.blockSlot, a.partials, a.history, a.st,
                                          p, a.par, a.sample);
  return cudaGetLastError();
}

cudaError_t launch_step3(int precision, const StepLaunch3& a, cudaStream_t s) {
  switch (precision) {
    case 0: return launch_step3_t<CodecF32>(a, s);
    case 1: return launch_step3_t<CodecF16>(a, s);
    case 2: return launch_step3_t<CodecBF16>(a, s);
    case 3: return launch_step3_t<CodecF64>(a, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace CELLS_ARITH
}  // namespace cells
