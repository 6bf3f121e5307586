// The D2Q9 step kernel: pull streaming, every boundary rule of the reference's 2D solver, Zou-He
// inlet and outlet, TRT collision with Smagorinsky, absorbing layers and the Guo body force, and
// the momentum-exchange force of the step reduced in f64 — for every tunnel of a batch in one
// launch (src/shaders/step.ts:9-229, src/shaders/common.ts:39-57, src/shaders/aux.ts:143-172).
//
// Each block updates one tile (blockDim.x x blockDim.y cells) of one tunnel; the tiles of all
// tunnels of a batch form one grid, so tunnels of different sizes advance in the same launch. A
// cell whose flag word is 0 pulls its 9 populations straight from the neighbours; any other cell
// resolves each direction with the reference's pullSlow rules. The arithmetic follows the
// reference's expressions operation by operation; the exact build (-fmad=false) reproduces the
// oracle's bits.
//
// Force: every tile of a sampled step writes the f64 sum of its cells' forces to its partial slot;
// the tunnel's last tile to finish (an atomic count) sums the partials in slot order into the
// history ring. The reference sums f32 slots in atomic order instead (src/shaders/aux.ts:143-172).
//
// This file is compiled twice: into cells::fast (contraction allowed) and, with
// -fmad=false -DCELLS_EXACT_ARITH, into cells::exact.
#include "kernels2d.h"

#ifdef CELLS_EXACT_ARITH
#define CELLS_NS exact
constexpr bool kExact2 = true;
#else
#define CELLS_NS fast
constexpr bool kExact2 = false;
#endif

namespace cells {
namespace CELLS_NS {

// Storage type S, arithmetic type R, and how populations are loaded: through the read-only path
// when a launch never writes what it reads (one step per launch), through L2 when it does (the
// persistent kernel rewrites the buffer it read two steps earlier, which a stale read-only line
// would miss).
template <class S_, class R_, bool COHERENT>
struct Store2 {
  using S = S_;
  using R = R_;
  __device__ __forceinline__ static S ld(const S* p) { return COHERENT ? __ldcg(p) : __ldg(p); }
};
using Store2F32 = Store2<float, float, false>;
using Store2F64 = Store2<double, double, false>;
using Store2F32P = Store2<float, float, true>;
using Store2F64P = Store2<double, double, true>;

template <class R>
__device__ __forceinline__ R prm(const Tunnel2& T, int k);
template <>
__device__ __forceinline__ float prm<float>(const Tunnel2& T, int k) {
  return __ldg(&T.pf[k]);
}
template <>
__device__ __forceinline__ double prm<double>(const Tunnel2& T, int k) {
  return __ldg(&T.pd[k]);
}

template <class R>
__device__ __forceinline__ R clampR(R v, R lo, R hi) {
  return v < lo ? lo : (hi < v ? hi : v);
}
// 1 / v: IEEE in the exact build and for f64; the hardware reciprocal (within 2 ulp, no branch)
// for f32 in the fast build
template <class R>
__device__ __forceinline__ R recip2(R v) {
  if constexpr (!kExact2 && sizeof(R) == 4)
    return __fdividef(R(1), v);
  else
    return R(1) / v;
}
template <class R>
struct XTab2;
template <>
struct XTab2<float> {
  using T = float4;
};
template <>
struct XTab2<double> {
  using T = double4;
};

struct Geo2 {
  int W, H;
  int left, right, bottom, top;
};

// wrapPeriodic, src/shaders/common.ts:48-57
__device__ __forceinline__ void wrap2(const Geo2& g, int& x, int& y) {
  if (x < 0 && g.left == X2_PERIODIC) x += g.W;
  if (x >= g.W && g.right == X2_PERIODIC) x -= g.W;
  if (y < 0 && g.bottom == Y2_PERIODIC) y += g.H;
  if (y >= g.H && g.top == Y2_PERIODIC) y -= g.H;
}

// inletVelocity, src/shaders/common.ts:39-45
template <class R>
__device__ __forceinline__ R inlet_velocity2(int parabolic, R uIn, int H, int y) {
  if (parabolic == 0) return uIn;
  const R h = R(H);
  const R s = R(y) + R(0.5);
  return R(4) * uIn * s * (h - s) / (h * h);
}

// pullSlow, src/shaders/step.ts:119-175
template <class C>
__device__ __forceinline__ typename C::R pull_slow2(int i, const Geo2& g, const typename C::S* __restrict__ src,
                                                    const uint32_t* __restrict__ flags, const float* __restrict__ sdf,
                                                    long long N, int x, int y, long long idx, uint32_t fl,
                                                    typename C::R uLid, typename C::R force[2]) {
  using R = typename C::R;
  const int j = opp2(i);
  int sx = x - cx2(i);
  int sy = y - cy2(i);
  if ((fl & (1u << i)) == 0u) return (R)C::ld(&src[i * N + (long long)sy * g.W + sx]);
  wrap2(g, sx, sy);
  const bool inX = sx >= 0 && sx < g.W;
  const bool inY = sy >= 0 && sy < g.H;
  if (inX && inY) {
    const long long s = (long long)sy * g.W + sx;
    if ((__ldg(&flags[s]) & FLAG2_SOLID) == 0u) return (R)C::ld(&src[i * N + s]);
    // Bouzidi linear interpolated bounce-back with q from the SDF
    const R fj = (R)C::ld(&src[j * N + idx]);
    const R dF = (R)__ldg(&sdf[idx]);
    const R dS = (R)__ldg(&sdf[s]);
    const R den = (dF - dS) < (R)1e-6 ? (R)1e-6 : (dF - dS);
    const R q = clampR<R>(dF / den, (R)1e-3, R(1));
    R fi = fj;
    if (q < R(0.5)) {
      int nx = x + cx2(i), ny = y + cy2(i);
      wrap2(g, nx, ny);
      if (nx >= 0 && nx < g.W && ny >= 0 && ny < g.H) {
        const long long n = (long long)ny * g.W + nx;
        if ((__ldg(&flags[n]) & FLAG2_SOLID) == 0u)
          fi = R(2) * q * fj + (R(1) - R(2) * q) * (R)C::ld(&src[j * N + n]);
      }
    } else {
      fi = fj / (R(2) * q) + (R(2) * q - R(1)) / (R(2) * q) * (R)C::ld(&src[i * N + idx]);
    }
    const R t = fj + fi;
    force[0] += R(cx2(j)) * t;
    force[1] += R(cy2(j)) * t;
    return fi;
  }
  if (!inY) {
    const int mode = sy < 0 ? g.bottom : g.top;
    if (mode == Y2_SLIP) {
      const int rx = sx < 0 ? 0 : (sx > g.W - 1 ? g.W - 1 : sx);
      return (R)C::ld(&src[mirror_y2(i) * N + (long long)y * g.W + rx]);
    }
    if (mode == Y2_MOVING) return (R)C::ld(&src[j * N + idx]) + R(6) * w2<R>(i) * R(cx2(i)) * uLid;
    return (R)C::ld(&src[j * N + idx]);
  }
  // walls, and placeholders that the open-boundary fix-up overwrites
  return (R)C::ld(&src[j * N + idx]);
}

// The fields of a tunnel that every cell of a tile reads, loaded once per thread.
template <class C>
struct Hot2 {
  const typename C::S* __restrict__ src;
  typename C::S* __restrict__ dst;
  const uint32_t* __restrict__ flags;
  const typename XTab2<typename C::R>::T* __restrict__ xtab;
  int W, H, N;
  int forcing;
  typename C::R smagC2;
};

// The loads of the cell (x, y): its flag word and the fast path's nine pulls, issued together (one
// memory round trip per cell, not two); a flagged cell replaces the pulls in cell2. Every address is
// inside the allocation: the largest, direction 8 on the top row, is at most W - 1 elements past the
// nine arrays, which the host pads.
template <class C>
__device__ __forceinline__ uint32_t load2(const Hot2<C>& h, int x, int y, typename C::R (&f)[Q2]) {
  using R = typename C::R;
  const int idx = y * h.W + x;
#pragma unroll
  for (int i = 0; i < Q2; i++) f[i] = (R)C::ld(h.src + (i * h.N + idx - cy2(i) * h.W - cx2(i)));
  return __ldg(&h.flags[idx]);
}

// main, src/shaders/step.ts:177-227, for the cell (x, y) of tunnel T, whose loads load2 made.
// Returns whether the cell has a force slot (its force is then in force[0..1]). The x-dependent
// rates come from the tunnel's x table; the exact build evaluates every other expression in the
// reference's order.
template <class C>
__device__ __forceinline__ bool cell2(const Tunnel2& T, const Hot2<C>& h, typename C::R uIn, int x, int y,
                                      uint32_t fl, typename C::R (&f)[Q2], typename C::R force[2]) {
  using R = typename C::R;
  using S = typename C::S;
  const int W = h.W;
  const int N = h.N;  // 9 N < 2^31: checked when the tunnel is created
  const S* __restrict__ src = h.src;
  S* __restrict__ dst = h.dst;
  const int idx = y * W + x;
  bool slot = false;
  if (fl != 0u) {
    if (fl & FLAG2_SOLID) return false;
    // pullSlow's first rule: a direction without its flag bit is the plain pull, which load2
    // already made (same element), so the general rules run for the flagged directions only. An
    // inlet (outlet) cell whose only flagged directions are the three entering from outside the
    // grid skips them altogether: Zou-He replaces those three pulls.
    constexpr uint32_t kInletPlain = FLAG2_INLET | (1u << 1) | (1u << 5) | (1u << 8);
    constexpr uint32_t kOutletPlain = FLAG2_OUTLET | (1u << 3) | (1u << 6) | (1u << 7);
    if (fl != kInletPlain && fl != kOutletPlain) {
      Geo2 g;
      g.W = W;
      g.H = h.H;
      g.left = T.left;
      g.right = T.right;
      g.bottom = T.bottom;
      g.top = T.top;
      const R uLid = prm<R>(T, P2_ULID);
#pragma unroll
      for (int i = 1; i < Q2; i++)
        if (fl & (1u << i))
          f[i] = pull_slow2<C>(i, g, src, h.flags, T.sdf, (long long)N, x, y, (long long)idx, fl, uLid, force);
      slot = (fl >> BIDX2_SHIFT) != 0u;
    }
    // Zou-He (populations stored shifted by w_i)
    if (fl & FLAG2_INLET) {
      const R u = inlet_velocity2<R>(T.parabolic, uIn, h.H, y);
      const R r = (R(1) + f[0] + f[2] + f[4] + R(2) * (f[3] + f[6] + f[7])) / (R(1) - u);
      f[1] = f[3] + (R)(2.0 / 3.0) * r * u;
      f[5] = f[7] - R(0.5) * (f[2] - f[4]) + (R)(1.0 / 6.0) * r * u;
      f[8] = f[6] + R(0.5) * (f[2] - f[4]) + (R)(1.0 / 6.0) * r * u;
    } else if (fl & FLAG2_OUTLET) {
      const R u = f[0] + f[2] + f[4] + R(2) * (f[1] + f[5] + f[8]);
      f[3] = f[1] - (R)(2.0 / 3.0) * u;
      f[7] = f[5] + R(0.5) * (f[2] - f[4]) - (R)(1.0 / 6.0) * u;
      f[6] = f[8] - R(0.5) * (f[2] - f[4]) - (R)(1.0 / 6.0) * u;
    }
  }
  // moments (src/shaders/step.ts:22-32)
  const R drho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
  const R rho = R(1) + drho;
  const R invRho = recip2<R>(rho);
  R ux = (f[1] - f[3] + f[5] - f[6] - f[7] + f[8]) * invRho;
  R uy = (f[2] - f[4] + f[5] + f[6] - f[7] - f[8]) * invRho;
  const int forcing = h.forcing;
  R bfx = R(0), bfy = R(0);
  if (forcing != 0) {
    bfx = prm<R>(T, P2_FX);
    bfy = prm<R>(T, P2_FY);
    ux += R(0.5) * bfx * invRho;
    uy += R(0.5) * bfy * invRho;
  }
  const R usq = R(1.5) * (ux * ux + uy * uy);
  R cu[Q2];
  cu[1] = R(3) * (ux);
  cu[2] = R(3) * (uy);
  cu[5] = R(3) * (ux + uy);
  cu[6] = R(3) * (-ux + uy);
  R eqS[Q2], eqA[Q2];
#pragma unroll
  for (int a : {1, 2, 5, 6}) {
    eqS[a] = w2<R>(a) * (drho + rho * (R(0.5) * cu[a] * cu[a] - usq));
    eqA[a] = w2<R>(a) * rho * cu[a];
  }
  // sponge and absorbing layers (src/shaders/step.ts:215-223), from the x table
  const auto xt = h.xtab[x];  // read-only for the whole launch
  const R omegaBase = xt.x;
  const R sigma = xt.z;
  // Smagorinsky (src/shaders/step.ts:48-63)
  R omP = omegaBase, omM = xt.y;
  if (h.smagC2 > R(0)) {
    R n[Q2];
#pragma unroll
    for (int a : {1, 2, 5, 6}) {
      const int b = opp2(a);
      n[a] = f[a] - (eqS[a] + eqA[a]);
      n[b] = f[b] - (eqS[a] - eqA[a]);
    }
    const R pxx = n[1] + n[3] + n[5] + n[6] + n[7] + n[8];
    const R pyy = n[2] + n[4] + n[5] + n[6] + n[7] + n[8];
    const R pxy = n[5] - n[6] + n[7] - n[8];
    const R pi = sqrt(pxx * pxx + pyy * pyy + R(2) * pxy * pxy);
    const R t0 = xt.w;  // 1 / omegaBase
    const R tEff = R(0.5) * (t0 + sqrt(t0 * t0 + (R)25.45584412271571 * h.smagC2 * pi * invRho));
    omP = recip2<R>(tEff);
    // the exact build divides 1 by omega+ again, as the reference does; the fast build uses tEff
    const R tP = kExact2 ? R(1) / omP : tEff;
    omM = recip2<R>(R(0.5) + prm<R>(T, P2_LAMBDA) / (tP - R(0.5)));
  }
  // absorbing-layer and Guo body-force sources (src/shaders/step.ts:65-91)
  R s0 = R(0);
  R sS[Q2], sA[Q2];
#pragma unroll
  for (int a : {1, 2, 5, 6}) {
    sS[a] = R(0);
    sA[a] = R(0);
  }
  if (sigma > R(0)) {
    const R ut = inlet_velocity2<R>(T.parabolic, uIn, h.H, y);
    const R dq = R(1.5) * rho * (ut * ut - ux * ux - uy * uy);
    s0 += sigma * w2<R>(0) * -dq;
#pragma unroll
    for (int a : {1, 2, 5, 6}) {
      const R cut = R(3) * R(cx2(a)) * ut;
      sS[a] += sigma * w2<R>(a) * (R(0.5) * rho * (cut * cut - cu[a] * cu[a]) - dq);
      sA[a] += sigma * w2<R>(a) * rho * (cut - cu[a]);
    }
  }
  if (forcing != 0) {
    const R uF = ux * bfx + uy * bfy;
    s0 += (R(1) - R(0.5) * omP) * w2<R>(0) * (R(-3) * uF);
#pragma unroll
    for (int a : {1, 2, 5, 6}) {
      const R cF = (R(cx2(a)) * bfx + R(cy2(a)) * bfy);
      sS[a] += (R(1) - R(0.5) * omP) * w2<R>(a) * (R(-3) * uF + R(9) * (cu[a] / R(3)) * cF);
      sA[a] += (R(1) - R(0.5) * omM) * w2<R>(a) * R(3) * cF;
    }
  }
  // TRT collide + store (src/shaders/step.ts:93-103)
  dst[idx] = (S)(f[0] - omP * (f[0] - w2<R>(0) * (drho - rho * usq)) + s0);
#pragma unroll
  for (int a : {1, 2, 5, 6}) {
    const int b = opp2(a);
    const R sym = omP * (R(0.5) * (f[a] + f[b]) - eqS[a]);
    const R asym = omM * (R(0.5) * (f[a] - f[b]) - eqA[a]);
    dst[a * N + idx] = (S)(f[a] - sym - asym + sS[a] + sA[a]);
    dst[b * N + idx] = (S)(f[b] - sym + asym + sS[a] - sA[a]);
  }
  return slot;
}

__device__ __forceinline__ double ramp_speed2(int kind, double target, double rampSteps, int every, unsigned step) {
  const double sq = (double)((step / (unsigned)every) * (unsigned)every);
  const double t = fmin(1.0, sq / rampSteps);
  return kind == 1 ? target * t : target * (t * t * (3.0 - 2.0 * t));
}

// One tile (lb-th of its tunnel t) of the step of parity par.
template <class C, int ROWS>
__device__ __forceinline__ void tile2(const Tunnel2* __restrict__ tunnels, int t, int lb, int par, int allowSample) {
  using R = typename C::R;
  const Tunnel2& T = tunnels[t];
  __shared__ double2 warpSum[32];
  __shared__ int lastTile;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int nthreads = blockDim.x * blockDim.y;
  const int tilesX = T.tilesX;
  const int tyi = lb / tilesX;
  const int txi = lb - tyi * tilesX;
  const int x = txi * blockDim.x + threadIdx.x;
  const int y = tyi * (ROWS * blockDim.y) + threadIdx.y;  // this thread's rows: y (+ blockDim.y)
  DevState2* st = T.st;
  const unsigned step = __ldcg(&st->step[par]);
  const double uInD = __ldcg(&st->uIn[par]);
  const int every = T.forceEvery;
  const bool sample = allowSample && every > 0 && ((step + 1u) % (unsigned)every) == 0u;
  if (lb == 0 && tid == 0) {
    // the next step's counter and inlet speed (slot par^1; this step reads slot par only)
    st->step[par ^ 1] = step + 1u;
    st->uIn[par ^ 1] = T.rampKind != 0 ? ramp_speed2(T.rampKind, T.rampTarget, T.rampSteps, T.rampEvery, step + 1u)
                                       : uInD;
  }
  // each cell's force stays in its own accumulator and is widened to f64 before the two are added,
  // as every cell's force enters the f64 tile sum on its own
  R force[2] = {R(0), R(0)}, force1[2] = {R(0), R(0)};
  bool slot = false, slot1 = false;
  if (x < T.W && y < T.H) {
    Hot2<C> h;
    h.W = T.W;
    h.H = T.H;
    h.N = h.W * h.H;
    h.src = (const typename C::S*)T.f[par];
    h.dst = (typename C::S*)T.f[par ^ 1];
    h.flags = T.flags;
    h.xtab = (const typename XTab2<R>::T*)T.xtab;
    h.forcing = T.forcing;
    h.smagC2 = prm<R>(T, P2_SMAGC2);
    R f0[Q2];
    const uint32_t fl0 = load2<C>(h, x, y, f0);
    if constexpr (ROWS == 2) {
      // both rows' loads go out before either cell computes
      const int y1 = y + blockDim.y;
      const bool second = y1 < h.H;
      R f1[Q2];
      uint32_t fl1 = 0u;
      if (second) fl1 = load2<C>(h, x, y1, f1);
      slot = cell2<C>(T, h, (R)uInD, x, y, fl0, f0, force);
      if (second) slot1 = cell2<C>(T, h, (R)uInD, x, y1, fl1, f1, force1);
    } else {
      slot = cell2<C>(T, h, (R)uInD, x, y, fl0, f0, force);
    }
  }
  if (!sample) return;
  // f64 sum of the tile's forces: warp shuffles, then warps in order
  if (__syncthreads_or((slot || slot1) ? 1 : 0)) {
    double sx = slot ? (double)force[0] : 0.0, sy = slot ? (double)force[1] : 0.0;
    if (slot1) {
      sx += (double)force1[0];
      sy += (double)force1[1];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sx += __shfl_down_sync(0xffffffffu, sx, o);
      sy += __shfl_down_sync(0xffffffffu, sy, o);
    }
    if ((tid & 31) == 0) warpSum[tid >> 5] = make_double2(sx, sy);
    __syncthreads();
    if (tid == 0) {
      double ax = 0.0, ay = 0.0;
      for (int w = 0; w < (nthreads + 31) / 32; w++) {
        ax += warpSum[w].x;
        ay += warpSum[w].y;
      }
      T.partials[lb] = make_double2(ax, ay);
    }
  } else if (tid == 0) {
    T.partials[lb] = make_double2(0.0, 0.0);
  }
  if (tid == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&st->done, 1u);
    lastTile = prev == (unsigned)(T.nTiles - 1);
  }
  __syncthreads();
  if (!lastTile) return;
  // the tunnel's last tile: partials in slot order, strided per thread, then threads in order
  __threadfence();
  double ax = 0.0, ay = 0.0;
  for (int k = tid; k < T.nTiles; k += nthreads) {
    const double2 v = __ldcg(&T.partials[k]);
    ax += v.x;
    ay += v.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_down_sync(0xffffffffu, ax, o);
    ay += __shfl_down_sync(0xffffffffu, ay, o);
  }
  __syncthreads();
  if ((tid & 31) == 0) warpSum[tid >> 5] = make_double2(ax, ay);
  __syncthreads();
  if (tid == 0) {
    double bx = 0.0, by = 0.0;
    for (int w = 0; w < (nthreads + 31) / 32; w++) {
      bx += warpSum[w].x;
      by += warpSum[w].y;
    }
    const unsigned s = __ldcg(&st->sample);
    T.history[s % HISTORY2_LEN] = make_double2(bx, by);
    st->sample = s + 1u;
    st->done = 0u;
    if (!isfinite(bx) || !isfinite(by)) atomicOr(&st->status, 1u);
  }
}

// Register cap of the f32 kernel (blocks of 256 threads per SM it must fit): 3 (up to 85
// registers); measured against 4 (64 registers, a few spilled words) the batch is as fast and one
// tunnel at a time 3% faster, while 5 and 6 (51 and 42 registers) spill and lose 12-28%. The f64
// kernel keeps its registers.
template <class C>
constexpr int min_blocks2() {
  return sizeof(typename C::R) == 4 ? 3 : 1;
}

template <class C, int ROWS>
__global__ void __launch_bounds__(256, min_blocks2<C>()) step2d_kernel(const Tunnel2* __restrict__ tunnels,
                                                     const unsigned short* __restrict__ tileTunnel, int par,
                                                     int allowSample) {
  // programmatic dependent launch, as in the 3D step: the next step's grid is scheduled during
  // this one's tail and waits here for the previous grid to complete
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int b = blockIdx.x;
  const int t = __ldg(&tileTunnel[b]);
  tile2<C, ROWS>(tunnels, t, b - __ldg(&tunnels[t].firstTile), par, allowSample);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier of the persistent kernel: arrivals count up a counter that the host zeroes
// before each launch; barrier k of the launch waits for k * gridDim.x arrivals. The wait is
// bounded by one second of the global timer and, as a backstop, by 2^23 polls; on time-out the
// block sets *error and the kernel winds down (every other block's wait then ends at its next
// poll).
__device__ __forceinline__ bool grid_barrier2(unsigned* counter, unsigned target, int* error) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    ok = 1;
    __threadfence();
    atomicAdd(counter, 1u);
    long long spins = 0;
    const unsigned long long t0 = global_ns();
    while (true) {
      unsigned seen;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(counter) : "memory");
      if (seen >= target) break;
      if (*(volatile int*)error != 0 || ++spins > (1ll << 23) || global_ns() - t0 > 1000000000ull) {
        atomicExch(error, 1);
        ok = 0;
        break;
      }
      __nanosleep(100);
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// nSteps steps of every tunnel in one launch: each resident block walks the tiles with a grid
// stride, then all blocks meet at the barrier before the next step.
template <class C, int ROWS>
__global__ void __launch_bounds__(256, min_blocks2<C>()) step2d_persistent_kernel(const Tunnel2* __restrict__ tunnels,
                                                                const unsigned short* __restrict__ tileTunnel,
                                                                int nTiles, int par, int nSteps, int allowSample,
                                                                unsigned* barrier, int* error, unsigned extra) {
  for (int s = 0; s < nSteps; s++) {
    for (int b = blockIdx.x; b < nTiles; b += gridDim.x) {
      const int t = __ldg(&tileTunnel[b]);
      tile2<C, ROWS>(tunnels, t, b - __ldg(&tunnels[t].firstTile), par, allowSample);
      __syncthreads();
    }
    par ^= 1;
    if (s + 1 < nSteps && !grid_barrier2(barrier, (unsigned)(s + 1) * gridDim.x + extra, error)) return;
  }
}

template <class C>
static cudaError_t launch_step2_t(const Step2Launch& a, cudaStream_t s) {
  if (a.nTiles <= 0) return cudaSuccess;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(a.nTiles);
  cfg.blockDim = dim3(a.tileX, a.tileY);
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, a.rows == 2 ? step2d_kernel<C, 2> : step2d_kernel<C, 1>, a.tunnels, a.tileTunnel,
                            a.par, a.allowSample);
}

template <class C>
static cudaError_t launch_step2_persistent_t(const Step2Launch& a, cudaStream_t s) {
  if (a.nTiles <= 0 || a.nSteps <= 0) return cudaSuccess;
  dim3 block(a.tileX, a.tileY);
  const Tunnel2* tunnels = a.tunnels;
  const unsigned short* tileTunnel = a.tileTunnel;
  int nTiles = a.nTiles, par = a.par, nSteps = a.nSteps, allowSample = a.allowSample;
  unsigned* barrier = a.barrier;
  int* error = a.error;
  unsigned extra = a.barrierExtra;
  void* args[] = {&tunnels, &tileTunnel, &nTiles, &par, &nSteps, &allowSample, &barrier, &error, &extra};
  cudaError_t e = cudaMemsetAsync(barrier, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  const void* fn = a.rows == 2 ? (const void*)step2d_persistent_kernel<C, 2> : (const void*)step2d_persistent_kernel<C, 1>;
  return cudaLaunchCooperativeKernel(fn, dim3(a.gridBlocks), block, args, 0, s);
}

template <class C>
static int persistent_blocks2_t(int threads) {
  int dev = 0, sms = 0, perSm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  // resident blocks of either rows variant (the smaller, so that both launch cooperatively)
  int perSm2 = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, step2d_persistent_kernel<C, 1>, threads, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm2, step2d_persistent_kernel<C, 2>, threads, 0) != cudaSuccess)
    return 0;
  if (perSm2 < perSm) perSm = perSm2;
  return perSm * sms;
}

cudaError_t launch_step2(int precision, const Step2Launch& a, cudaStream_t s) {
  if (precision == 0) return launch_step2_t<Store2F32>(a, s);
  if (precision == 3) return launch_step2_t<Store2F64>(a, s);
  return cudaErrorInvalidValue;
}

cudaError_t launch_step2_persistent(int precision, const Step2Launch& a, cudaStream_t s) {
  if (precision == 0) return launch_step2_persistent_t<Store2F32P>(a, s);
  if (precision == 3) return launch_step2_persistent_t<Store2F64P>(a, s);
  return cudaErrorInvalidValue;
}

int persistent_blocks2(int precision, int threads) {
  if (precision == 0) return persistent_blocks2_t<Store2F32P>(threads);
  if (precision == 3) return persistent_blocks2_t<Store2F64P>(threads);
  return 0;
}

}  // namespace CELLS_NS
}  // namespace cells
