// Discrete adjoint of the D3Q19 step: the adjoint step kernels, the recorded forward run with
// checkpoints, the backward sweep with recomputation, and their C ABI (include/cells.h). No
// counterpart in the reference.
//
// Adjoint step n (from lambda^{n+1} to lambda^n over the recomputed state f^n), per cell x:
//   g = P(f^n)(x): the 19 pulled values (plain pulls, or the cell's link records at boundaries);
//   lambda_g = (dC/dg)^T lambda^{n+1}(x): the transposed Jacobian of the TRT collision (or of the
//     outlet's feq(1, u), or zero at the inlet, whose output does not depend on g);
//   the streaming transpose: a plain pull of direction i from x - c_i is the only regular reader of
//     that element, so lambda^n_i(x - c_i) = lambda_g,i is a plain store; a link's adjoint goes to
//     lamG and a second kernel adds it, with the objective's direct force terms, to the link's
//     source elements (a fixed-order sum per element: deterministic).
// Shape: dJ/dq per Bouzidi link accumulates (lambda_g + w cF) dg/dq; dq/dsdf then gives dJ/dsdf.
// Inflow: dJ/du_n from the inlet's feq(1, u_n) and the absorbing layer's target u_n, summed per
// step in f64 with a fixed order.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "adjoint3d.h"
#include "solver3d_state.h"

using namespace cells;

namespace {

__host__ __device__ __forceinline__ long long off3(int i, int W, int H) {
  return (long long)cx3(i) + (long long)W * ((long long)cy3(i) + (long long)H * cz3(i));
}

template <class R>
struct XRow {
  R omP, omM, sigma;
};

// (dC/dg)^T lp for the TRT collision with sponge rate omP/omM and absorbing strength sigma toward
// the inflow speed ut (src/shaders/step3d.ts:38-102, Smagorinsky off). Also returns dJ/dut.
// ABS = false: a cell known to lie outside the absorbing layer, compiled without its terms (as a
// run-time branch the compiler evaluates them for every cell). f32 takes the hardware reciprocal.
template <class R, bool ABS = true>
__device__ __forceinline__ void collide_adjoint3(const R g[Q3], const R lp[Q3], R omP, R omM, R sigma, R ut,
                                                 R lg[Q3], R& dut) {
  R drho = R(0);
#pragma unroll
  for (int i = 0; i < Q3; i++) drho += g[i];
  const R rho = R(1) + drho;
  R inv;
  if constexpr (sizeof(R) == 4)
    inv = __fdividef(R(1), rho);
  else
    inv = R(1) / rho;
  R jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
  for (int i = 1; i < Q3; i++) {
    jx += R(cx3(i)) * g[i];
    jy += R(cy3(i)) * g[i];
    jz += R(cz3(i)) * g[i];
  }
  const R ux = jx * inv, uy = jy * inv, uz = jz * inv;
  const R uu = ux * ux + uy * uy + uz * uz;
  const R usq = R(1.5) * uu;
  const R w0 = w3<R>(0);
  R rhoB = R(0), usqB = R(0), uxB = R(0), uyB = R(0), uzB = R(0), dqB = R(0), utB = R(0);
  lg[0] = lp[0] * (R(1) - omP);
  {
    const R e0 = omP * lp[0];
    rhoB += e0 * w0 * (R(1) - usq);
    usqB -= e0 * w0 * rho;
  }
  const bool absorb = ABS && sigma > R(0);
  if (absorb) dqB -= lp[0] * sigma * w0;
#pragma unroll
  for (int a = 1; a < Q3; a += 2) {
    const int b = a + 1;
    const R wa = w3<R>(a);
    const R cu = R(3) * (R(cx3(a)) * ux + R(cy3(a)) * uy + R(cz3(a)) * uz);
    const R S = lp[a] + lp[b];
    const R Dd = lp[a] - lp[b];
    lg[a] = lp[a] - R(0.5) * omP * S - R(0.5) * omM * Dd;
    lg[b] = lp[b] - R(0.5) * omP * S + R(0.5) * omM * Dd;
    const R eS = omP * S, eA = omM * Dd;
    rhoB += eS * wa * (R(1) + R(0.5) * cu * cu - usq) + eA * wa * cu;
    R cuB = eS * wa * rho * cu + eA * wa * rho;
    usqB -= eS * wa * rho;
    if (absorb) {
      const R cut = R(3) * R(cx3(a)) * ut;
      const R sw = sigma * wa;
      rhoB += S * sw * R(0.5) * (cut * cut - cu * cu) + Dd * sw * (cut - cu);
      cuB -= S * sw * rho * cu + Dd * sw * rho;
      dqB -= S * sw;
      utB += R(3) * R(cx3(a)) * (S * sw * rho * cut + Dd * sw * rho);
    }
    uxB += R(3) * R(cx3(a)) * cuB;
    uyB += R(3) * R(cy3(a)) * cuB;
    uzB += R(3) * R(cz3(a)) * cuB;
  }
  if (absorb) {  // dq = 1.5 rho (ut^2 - |u|^2)
    rhoB += dqB * R(1.5) * (ut * ut - uu);
    uxB -= dqB * R(3) * rho * ux;
    uyB -= dqB * R(3) * rho * uy;
    uzB -= dqB * R(3) * rho * uz;
    utB += dqB * R(3) * rho * ut;
  }
  uxB += R(3) * ux * usqB;
  uyB += R(3) * uy * usqB;
  uzB += R(3) * uz * usqB;
  const R jxB = uxB * inv, jyB = uyB * inv, jzB = uzB * inv;
  rhoB -= (ux * uxB + uy * uyB + uz * uzB) * inv;
#pragma unroll
  for (int i = 0; i < Q3; i++) lg[i] += rhoB + R(cx3(i)) * jxB + R(cy3(i)) * jyB + R(cz3(i)) * jzB;
  dut = utB;
}

// (d feq(1, u(g)) / dg)^T lp: the outlet stores feq(1, u) with u the velocity of the pulled values.
template <class R>
__device__ __forceinline__ void outlet_adjoint3(const R g[Q3], const R lp[Q3], R lg[Q3]) {
  R drho = R(0);
#pragma unroll
  for (int i = 0; i < Q3; i++) drho += g[i];
  const R rho = R(1) + drho;
  const R inv = R(1) / rho;
  R jx = R(0), jy = R(0), jz = R(0);
#pragma unroll
  for (int i = 1; i < Q3; i++) {
    jx += R(cx3(i)) * g[i];
    jy += R(cy3(i)) * g[i];
    jz += R(cz3(i)) * g[i];
  }
  const R ux = jx * inv, uy = jy * inv, uz = jz * inv;
  R uxB = R(0), uyB = R(0), uzB = R(0);
#pragma unroll
  for (int i = 0; i < Q3; i++) {
    const R cu = R(3) * (R(cx3(i)) * ux + R(cy3(i)) * uy + R(cz3(i)) * uz);
    const R k = lp[i] * w3<R>(i);
    uxB += k * (R(3) * R(cx3(i)) * (R(1) + cu) - R(3) * ux);
    uyB += k * (R(3) * R(cy3(i)) * (R(1) + cu) - R(3) * uy);
    uzB += k * (R(3) * R(cz3(i)) * (R(1) + cu) - R(3) * uz);
  }
  const R jxB = uxB * inv, jyB = uyB * inv, jzB = uzB * inv;
  const R rhoB = -(ux * uxB + uy * uyB + uz * uzB) * inv;
#pragma unroll
  for (int i = 0; i < Q3; i++) lg[i] = rhoB + R(cx3(i)) * jxB + R(cy3(i)) * jyB + R(cz3(i)) * jzB;
}

// The recorded step this adjoint step undoes: the segment's first step (device memory, written
// before the segment's kernels run, so one captured graph serves every segment) plus the kernel's
// position t within the segment.
__device__ __forceinline__ int adj_step(const AdjLaunch3& a) { return __ldg(a.n0Dev) + a.t; }

// The block's f64 sum of dJ/du_n into part[slot] (the rows kernel sums the slots in order).
__device__ __forceinline__ void block_du_partial(double du, double* part, int slot, double* red, int tid) {
  for (int o = 16; o > 0; o >>= 1) du += __shfl_down_sync(0xffffffffu, du, o);
  if ((tid & 31) == 0) red[tid >> 5] = du;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int k = 0; k < kAdjThreads / 32; k++) s += red[k];
    part[slot] = s;
  }
}

template <class R>
__global__ void __launch_bounds__(kAdjThreads) adj_cells3_kernel(AdjLaunch3 a) {
  __shared__ double red[kAdjThreads / 32];
  // a tile of x-rows per block (no division per cell); 32-bit element indices (19 N < 2^31)
  const int W = a.W, H = a.H;
  const int N = (int)a.N;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const R* __restrict__ f = (const R*)a.f;
  const R* __restrict__ lamNext = (const R*)a.lamNext;
  R* __restrict__ lamOut = (R*)a.lamOut;
  double du = 0.0;
  const int idx = x + W * (y + H * (int)blockIdx.z);
  const bool in = x < W && y < H;
  // the plain pulls and lambda^{n+1} go out with the flag load rather than after it: for every cell
  // of the grid each address lies inside the 19 N arrays (no D3Q19 direction reaches further than
  // one plane, and the arrays of directions 1 and 18 are not the first and last), and flagged cells
  // discard the values
  R g[Q3], lp[Q3];
  if (in) {
#pragma unroll
    for (int i = 0; i < Q3; i++) {
      const int o = i * N + idx;
      lp[i] = __ldg(&lamNext[o]);
      g[i] = __ldg(&f[o - (int)off3(i, W, H)]);
    }
  }
  const uint32_t fl = in ? __ldg(&a.flags[idx]) : FLAG3_SOLID;
  if (fl == 0u) {
    // interior cell: plain pulls, the collision's transposed Jacobian, plain pushes
    R lg[Q3];
    const R* xt = (const R*)a.xTab + 4 * x;
    R dut = R(0);
    // block-uniform: tiles that end before the absorbing layer take the code without it
    if ((int)((blockIdx.x + 1) * blockDim.x) > a.absorbX0)
      collide_adjoint3<R, true>(g, lp, xt[0], xt[1], xt[2], (R)__ldg(&a.uDev[adj_step(a)]), lg, dut);
    else
      collide_adjoint3<R, false>(g, lp, xt[0], xt[1], xt[2], (R)__ldg(&a.uDev[adj_step(a)]), lg, dut);
    du = (double)dut;
#pragma unroll
    for (int i = 0; i < Q3; i++) lamOut[i * N + idx - (int)off3(i, W, H)] = lg[i];
  }
  // flagged fluid cells (faces, inlet, outlet, body) are done by adj_slow3_kernel
  block_du_partial(du, a.blockPart, blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z), red, tid);
}

// The flagged fluid cells (faces, inlet, outlet, body), kSlowCells per block in three phases so
// that their many independent loads are in flight together: (cell, direction) items pull through
// the cells' records into shared memory; one thread per cell applies the transposed Jacobian of its
// collision (or of the outlet equilibrium; the inlet only feeds dJ/du_n); (cell, direction) items
// push the plain pulls' adjoints and store the links' adjoints (with dJ/dq of Bouzidi links).
constexpr int kSlowCells = 32;

template <class R>
__global__ void __launch_bounds__(kAdjThreads) adj_slow3_kernel(AdjLaunch3 a) {
  __shared__ double red[kAdjThreads / 32];
  __shared__ R sg[Q3][kSlowCells + 1];
  __shared__ R slp[Q3][kSlowCells + 1];
  __shared__ R slg[Q3][kSlowCells + 1];
  __shared__ uint32_t sfl[kSlowCells];
  const int N = (int)a.N;
  const int n = a.nSlow;
  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * kSlowCells;
  const R* __restrict__ f = (const R*)a.f;
  const R* __restrict__ lamNext = (const R*)a.lamNext;
  R* __restrict__ lamOut = (R*)a.lamOut;
  const R* sA1 = (const R*)a.sA1;
  const R* sA2 = (const R*)a.sA2;
  for (int it = tid; it < Q3 * kSlowCells; it += kAdjThreads) {
    const int c = it % kSlowCells, i = it / kSlowCells, s = c0 + c;
    if (s >= n) continue;
    const int idx = a.slowCells[s];
    const int r = i * n + s;
    slp[i][c] = lamNext[i * N + idx];
    const int e = a.sE1[r];
    if (e >= 0) {  // one source with coefficient 1: plain pulls, copies, mirrors, bounce-back
      sg[i][c] = f[e];
    } else {       // Bouzidi interpolation: two sources
      sg[i][c] = sA1[r] * f[e & 0x7fffffff] + sA2[r] * f[a.sE2[r]];
    }
  }
  __syncthreads();
  double du = 0.0;
  if (tid < kSlowCells && c0 + tid < n) {
    const int idx = a.slowCells[c0 + tid];
    const uint32_t fl = a.flags[idx];
    sfl[tid] = fl;
    R g[Q3], lp[Q3], lg[Q3];
#pragma unroll
    for (int i = 0; i < Q3; i++) {
      g[i] = sg[i][tid];
      lp[i] = slp[i][tid];
    }
    const R u = (R)__ldg(&a.uDev[adj_step(a)]);
    if (fl & FLAG3_INLET) {
      // f' = feq(1, u, 0, 0): d/du = w_i (3 c_ix + 9 c_ix^2 u - 3 u); the inlet reads nothing
      R sum = R(0);
#pragma unroll
      for (int i = 0; i < Q3; i++) {
        const R c = R(cx3(i));
        sum += lp[i] * w3<R>(i) * (R(3) * c + R(9) * c * c * u - R(3) * u);
        lg[i] = R(0);
      }
      du = (double)sum;
    } else if (fl & FLAG3_OUTLET) {
      outlet_adjoint3<R>(g, lp, lg);
    } else {
      const R* xt = (const R*)a.xTab + 4 * (idx % a.W);
      R dut = R(0);
      collide_adjoint3<R>(g, lp, xt[0], xt[1], xt[2], u, lg, dut);
      du = (double)dut;
    }
#pragma unroll
    for (int i = 0; i < Q3; i++) slg[i][tid] = lg[i];
  }
  __syncthreads();
  const R* lcF = (const R*)a.lcF;
  const R* lq = (const R*)a.lq;
  R* lamG = (R*)a.lamG;
  const R w = (R)__ldg(&a.wDev[adj_step(a)]);
  for (int it = tid; it < Q3 * kSlowCells; it += kAdjThreads) {
    const int c = it % kSlowCells, i = it / kSlowCells, s = c0 + c;
    if (s >= n || (sfl[c] & FLAG3_INLET)) continue;
    const R v = slg[i][c];
    const int t = a.sTgt[i * n + s];
    if (t >= 0) {  // a plain pull: the element's only regular reader
      lamOut[t] = v;
    } else {       // a link: its adjoint, and dJ/dq of a Bouzidi link
      const int k = -t - 1;
      lamG[k] = v;
      const int qk = a.lqk[k];
      if (qk) {
        const R fj = f[a.le1[k]], f2 = f[a.le2[k]], q = lq[k];
        const R dgdq = qk == 1 ? R(2) * (fj - f2) : (f2 - fj) / (R(2) * q * q);
        a.dqAcc[k] += (double)((v + w * lcF[k]) * dgdq);
      }
    }
  }
  block_du_partial(du, a.blockPart, a.nCellBlocks + (int)blockIdx.x, red, tid);
}

// Elements with an irregular reader or no regular reader: lambda^n[e] (= 0 when no regular reader
// wrote it) plus each link's adjoint times its coefficient, plus the direct force terms.
template <class R>
__global__ void __launch_bounds__(256) adj_rows3_kernel(AdjLaunch3 a) {
  if (blockIdx.x == gridDim.x - 1) {
    // the extra last block: dJ/du_n = the cell kernel's block sums, strided per thread, then in order
    __shared__ double red[8];
    double s = 0.0;
    for (int k = threadIdx.x; k < a.nParts; k += 256) s += a.blockPart[k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < 8; k++) t += red[k];
      a.dudn[adj_step(a)] = t;
    }
    return;
  }
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.nRows) return;
  R* lamOut = (R*)a.lamOut;
  const R* lamG = (const R*)a.lamG;
  const R* lcF = (const R*)a.lcF;
  const R* alpha = (const R*)a.entAlpha;
  const R w = (R)__ldg(&a.wDev[adj_step(a)]);
  const long long e = a.rowElem[r];
  R v = a.rowSet[r] ? R(0) : lamOut[e];
  for (int k = a.rowStart[r]; k < a.rowStart[r + 1]; k++) {
    const int L = a.entLink[k];
    v += alpha[k] * (lamG[L] + w * lcF[L]);
  }
  v += w * ((const R*)a.rowPhi)[r];
  lamOut[e] = v;
}

template <class R>
cudaError_t launch_adjoint_step3_t(const AdjLaunch3& a, cudaStream_t s, cudaStream_t side, cudaEvent_t fork,
                                   cudaEvent_t join) {
  const dim3 block(a.tileX, kAdjThreads / a.tileX);
  const dim3 grid((unsigned)((a.W + block.x - 1) / block.x), (unsigned)((a.H + block.y - 1) / block.y),
                  (unsigned)a.D);
  if ((long long)grid.x * grid.y * grid.z != a.nCellBlocks) return cudaErrorInvalidValue;
  const int slowBlocks = (a.nSlow + kSlowCells - 1) / kSlowCells;
  if (a.nCellBlocks + slowBlocks != a.nParts) return cudaErrorInvalidValue;
  cudaError_t e;
  if (slowBlocks > 0) {  // the flagged cells on the side stream, beside the interior cells
    if ((e = cudaEventRecord(fork, s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(side, fork, 0)) != cudaSuccess) return e;
    adj_slow3_kernel<R><<<slowBlocks, kAdjThreads, 0, side>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaEventRecord(join, side)) != cudaSuccess) return e;
  }
  adj_cells3_kernel<R><<<grid, block, 0, s>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (slowBlocks > 0 && (e = cudaStreamWaitEvent(s, join, 0)) != cudaSuccess) return e;
  adj_rows3_kernel<R><<<(unsigned)((a.nRows + 255) / 256) + 1, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace

namespace cells {
cudaError_t launch_adjoint_step3(int precision, const AdjLaunch3& a, cudaStream_t s, cudaStream_t side,
                                 cudaEvent_t fork, cudaEvent_t join) {
  if (precision == 0) return launch_adjoint_step3_t<float>(a, s, side, fork, join);
  if (precision == 3) return launch_adjoint_step3_t<double>(a, s, side, fork, join);
  return cudaErrorInvalidValue;
}
}  // namespace cells

// ---------------- host: link resolution (the rules of pullSlow3, src/shaders/step3d.ts:119-168) ----

namespace {

// Host threads for the table builds: the machine's, at most 16.
int table_threads() {
  const unsigned n = std::thread::hardware_concurrency();
  return (int)std::max(1u, std::min(16u, n));
}

// Runs fn(t) for t = 0 .. n-1 on n host threads (t = 0 on the caller's).
template <class F>
void run_threads(int n, F fn) {
  std::vector<std::thread> pool;
  for (int t = 1; t < n; t++) pool.emplace_back(fn, t);
  fn(0);
  for (std::thread& th : pool) th.join();
}

// The links of the flagged fluid cells of planes z0 .. z1-1, in cell order; base[idx] is set to the
// first link of each such cell, counted within this slab's links.
template <class R>
void resolve_links_slab(const Cells3D* h, const std::vector<uint32_t>& fl, const std::vector<float>& sdf, int comp,
                        int z0, int z1, std::vector<int>& base, std::vector<AdjLink3Host>& links) {
  const int W = h->W, H = h->H, D = h->D;
  const long long N = h->N;
  auto at = [&](int x, int y, int z) { return (long long)x + (long long)W * ((long long)y + (long long)H * z); };
  auto solid = [&](long long c) { return (fl[(size_t)c] & FLAG3_SOLID) != 0u; };
  auto cc = [&](int j) { return comp == 0 ? cx3(j) : (comp == 1 ? cy3(j) : cz3(j)); };
  links.clear();
  for (int z = z0; z < z1; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        const long long idx = at(x, y, z);
        const uint32_t f = fl[(size_t)idx];
        if (f == 0u || (f & (FLAG3_SOLID | FLAG3_INLET))) continue;
        const bool outlet = (f & FLAG3_OUTLET) != 0u;
        bool any = false;
        for (int i = 1; i < Q3; i++) {
          if (!(f & (1u << i))) continue;
          if (!any) {
            base[(size_t)idx] = (int)links.size();
            any = true;
          }
          AdjLink3Host L{};
          L.e2 = -1;
          L.a1 = 1.0;
          L.a2 = 0.0;
          L.cell = (int)idx;
          L.solid = -1;
          const int j = opp3(i);
          const int sx = x - cx3(i), sy = y - cy3(i), sz = z - cz3(i);
          const bool outX = sx < 0 || sx >= W, outY = sy < 0 || sy >= H, outZ = sz < 0 || sz >= D;
          if (outX && outlet) {
            L.e1 = i * N + at(W - 2, y, z);
          } else if (outY && outZ) {
            L.e1 = j * N + idx;
          } else if (outY || outZ) {
            int rx = sx, ry = sy, rz = sz, m = mirror_y3(i);
            if (outY) {
              ry = y;
            } else {
              rz = z;
              m = mirror_z3(i);
            }
            const long long rs = at(rx, ry, rz);
            if (solid(rs)) {  // a body meets a slip face: bounce-back with force 2 c_j f_j
              L.e1 = j * N + idx;
              L.cF = cc(j);
            } else {
              L.e1 = m * N + rs;
            }
          } else if (outX) {
            L.e1 = j * N + idx;
          } else {
            const long long s = at(sx, sy, sz);
            if (!solid(s)) {
              L.e1 = i * N + s;
            } else {
              // Bouzidi: q in the arithmetic type, as the step kernel computes it
              const R dF = (R)sdf[(size_t)idx], dS = (R)sdf[(size_t)s];
              const R den = std::max(dF - dS, (R)1e-6);
              const R raw = dF / den;
              const R q = std::min(std::max(raw, (R)1e-3), R(1));
              L.e1 = j * N + idx;
              L.cF = cc(j);
              L.q = (double)q;
              L.cell = (int)idx;
              L.solid = (int)s;
              const bool free = raw > (R)1e-3 && raw < R(1) && (dF - dS) > (R)1e-6;
              if (free) {
                L.dqdF = -(double)dS / ((double)den * (double)den);
                L.dqdS = (double)dF / ((double)den * (double)den);
              }
              if (q < R(0.5)) {
                const int nx = x + cx3(i), ny = y + cy3(i), nz = z + cz3(i);
                if (nx >= 0 && nx < W && ny >= 0 && ny < H && nz >= 0 && nz < D && !solid(at(nx, ny, nz))) {
                  L.a1 = (double)(R(2) * q);
                  L.e2 = j * N + at(nx, ny, nz);
                  L.a2 = (double)(R(1) - R(2) * q);
                  L.qKind = 1;
                }
              } else {
                L.a1 = (double)(R(1) / (R(2) * q));
                L.e2 = i * N + idx;
                L.a2 = (double)((R(2) * q - R(1)) / (R(2) * q));
                L.qKind = 2;
              }
            }
          }
          links.push_back(L);
        }
      }
}

// The link records of every flagged fluid cell in cell order (the order a sequential pass gives),
// built by slabs of planes on host threads and joined.
template <class R>
void resolve_links(const Cells3D* h, const std::vector<uint32_t>& fl, const std::vector<float>& sdf, int comp,
                   std::vector<int>& base, std::vector<AdjLink3Host>& links) {
  const int D = h->D;
  const long long plane = (long long)h->W * h->H;
  base.assign((size_t)h->N, -1);
  const int T = std::min(table_threads(), D);
  std::vector<std::vector<AdjLink3Host>> part((size_t)T);
  auto z_begin = [&](int t) { return (int)((long long)D * t / T); };
  run_threads(T, [&](int t) { resolve_links_slab<R>(h, fl, sdf, comp, z_begin(t), z_begin(t + 1), base, part[(size_t)t]); });
  std::vector<int> offset((size_t)T + 1, 0);
  for (int t = 0; t < T; t++) offset[(size_t)t + 1] = offset[(size_t)t] + (int)part[(size_t)t].size();
  run_threads(T, [&](int t) {
    const int o = offset[(size_t)t];
    if (o == 0) return;
    for (long long c = z_begin(t) * plane; c < z_begin(t + 1) * plane; c++)
      if (base[(size_t)c] >= 0) base[(size_t)c] += o;
  });
  links.clear();
  links.reserve((size_t)offset[(size_t)T]);
  for (auto& p : part) links.insert(links.end(), p.begin(), p.end());
}

template <class R>
void upload_typed(cells::Device& dev, void* d, const std::vector<double>& v) {
  std::vector<R> t(v.begin(), v.end());
  if (!t.empty()) dev.h2d(d, t.data(), t.size() * sizeof(R));
  dev.sync();
}

// A device buffer of the recorded run: from the handle's table block while it has room (256-byte
// aligned), else a buffer of its own that the run frees.
void* adj_alloc(Cells3D* h, Adjoint3D* A, size_t bytes, const char* what) {
  bytes = (std::max<size_t>(bytes, 1) + 255) / 256 * 256;
  A->tabNeed += bytes;
  if (h->adjTab && A->tabUsed + bytes <= h->adjTabBytes) {
    void* p = (char*)h->adjTab + A->tabUsed;
    A->tabUsed += bytes;
    return p;
  }
  void* p = h->dev.alloc(bytes, what);
  A->own.push_back(p);
  return p;
}

// Makes the handle's table block hold `bytes` (with room for a somewhat larger body next time),
// before the run has taken anything from it; without the memory for it the run's buffers are
// allocated one by one.
void reserve_adj_tables(Cells3D* h, Adjoint3D* A, size_t bytes) {
  if (h->adjTabBytes >= bytes || A->tabUsed != 0) return;
  if (h->adjTab) h->dev.release(h->adjTab);
  h->adjTab = nullptr;
  h->adjTabBytes = 0;
  const size_t want = bytes + bytes / 8 + ((size_t)1 << 20);
  if (want + (size_t)h->N * 16 < h->dev.free_bytes()) {
    h->adjTab = h->dev.alloc(want, "adjoint tables");
    h->adjTabBytes = want;
  }
}

void release_adjoint(Cells3D* h) {
  if (!h->adj) return;
  Adjoint3D* A = h->adj.get();
  // the checkpoints, recompute buffers and adjoint states live in h->adjStore and the tables in
  // h->adjTab, which both stay; only the run's own buffers go
  if (!h->dev.fake) h->dev.sync();
  if (A->side) cudaStreamSynchronize(A->side);
  if (A->side2) cudaStreamSynchronize(A->side2);
  for (auto& row : A->segGraph)
    for (auto& g : row)
      if (g) cudaGraphExecDestroy(g);
  if (A->fork2) cudaEventDestroy(A->fork2);
  if (A->join2) cudaEventDestroy(A->join2);
  if (A->side2) cudaStreamDestroy(A->side2);
  if (A->fork) cudaEventDestroy(A->fork);
  if (A->join) cudaEventDestroy(A->join);
  if (A->side) cudaStreamDestroy(A->side);
  if (A->n0Host) h->dev.free_host_pinned(A->n0Host);
  for (void* p : A->own) h->dev.release(p);
  h->adj.reset();
}

// Link tables and the transposed element map for the current flags and SDF.
void build_tables(Cells3D* h, Adjoint3D* A) {
  cells::Device& dev = h->dev;
  const long long N = h->N;
  const int W = h->W, H = h->H, D = h->D;
  std::vector<uint32_t> fl((size_t)N);
  std::vector<float> sdf((size_t)N);
  dev.d2h(fl.data(), h->flags, (size_t)N * 4);
  dev.d2h(sdf.data(), h->sdf, (size_t)N * 4);
  dev.sync();
  std::vector<int> base;
  if (h->prec == 3)
    resolve_links<double>(h, fl, sdf, A->component, base, A->hostLinks);
  else
    resolve_links<float>(h, fl, sdf, A->component, base, A->hostLinks);
  const std::vector<AdjLink3Host>& L = A->hostLinks;
  A->nLinks = (int)L.size();
  // transposed map: (element, link, alpha) entries, direct force terms, and elements without a
  // regular reader
  struct Ent {
    long long e;
    int link;  // -1: no regular reader; -2: a force term
    double alpha;
  };
  // the links' entries, sorted by element (ties keep their order of insertion: link order, then
  // e1, e2, force within a link)
  std::vector<Ent> lent;
  lent.reserve(L.size() * 3);
  for (int k = 0; k < A->nLinks; k++) {
    lent.push_back({L[k].e1, k, L[k].a1});
    if (L[k].e2 >= 0) lent.push_back({L[k].e2, k, L[k].a2});
    if (L[k].cF != 0.0) lent.push_back({L[k].e1, -2, L[k].cF});
  }
  // entry indices in element order, ties in insertion order: a stable LSD radix sort on the
  // element index (below 19 N < 2^31), 8 bits a pass, as many passes as the largest element needs
  std::vector<int> key(lent.size()), tmp(lent.size());
  for (size_t p = 0; p < lent.size(); p++) key[p] = (int)p;
  {
    long long maxE = 0;
    for (const Ent& en : lent) maxE = std::max(maxE, en.e);
    for (int shift = 0; shift < 32 && (maxE >> shift) != 0; shift += 8) {
      size_t count[257] = {0};
      for (int p : key) count[(((uint32_t)lent[(size_t)p].e >> shift) & 255u) + 1]++;
      for (int d = 0; d < 256; d++) count[d + 1] += count[d];
      for (int p : key) tmp[count[((uint32_t)lent[(size_t)p].e >> shift) & 255u]++] = p;
      key.swap(tmp);
    }
  }
  // elements without a regular reader, generated in increasing element order (direction outer)
  auto at = [&](int x, int y, int z) { return (long long)x + (long long)W * ((long long)y + (long long)H * z); };
  std::vector<std::vector<long long>> irr(Q3);  // per direction, on host threads
  {
    const int T = std::min(table_threads(), Q3);
    run_threads(T, [&](int t) {
      for (int i = t; i < Q3; i += T) {
        std::vector<long long>& out = irr[(size_t)i];
        for (int z = 0; z < D; z++)
          for (int y = 0; y < H; y++) {
            const int ry = y + cy3(i), rz = z + cz3(i);
            const bool rowIn = ry >= 0 && ry < H && rz >= 0 && rz < D;
            for (int x = 0; x < W; x++) {
              const long long c = at(x, y, z);
              if (fl[(size_t)c] & FLAG3_SOLID) continue;
              const int rx = x + cx3(i);
              bool regular = rowIn && rx >= 0 && rx < W;
              if (regular) {
                const uint32_t g = fl[(size_t)at(rx, ry, rz)];
                regular = !(g & (FLAG3_SOLID | FLAG3_INLET)) && (i == 0 || !(g & (1u << i)));
              }
              if (!regular) out.push_back(i * N + c);
            }
          }
      }
    });
  }
  std::vector<long long> irregular;
  for (auto& v : irr) irregular.insert(irregular.end(), v.begin(), v.end());
  // merge: for one element the link entries come before its no-reader mark
  std::vector<Ent> ents;
  ents.reserve(lent.size() + irregular.size());
  {
    size_t p = 0, q = 0;
    while (p < key.size() || q < irregular.size()) {
      if (q >= irregular.size() || (p < key.size() && lent[(size_t)key[p]].e <= irregular[q]))
        ents.push_back(lent[(size_t)key[p++]]);
      else
        ents.push_back({irregular[q++], -1, 0.0});
    }
  }
  std::vector<long long> rowElem;
  std::vector<unsigned char> rowSet;
  std::vector<int> rowStart, entLink;
  std::vector<double> entAlpha, rowPhi;
  rowElem.reserve(ents.size());
  rowSet.reserve(ents.size());
  rowStart.reserve(ents.size() + 1);
  rowPhi.reserve(ents.size());
  entLink.reserve(lent.size());
  entAlpha.reserve(lent.size());
  for (size_t p = 0; p < ents.size();) {
    const long long e = ents[p].e;
    unsigned char set = 0;
    double phi = 0.0;
    rowElem.push_back(e);
    rowStart.push_back((int)entLink.size());
    for (; p < ents.size() && ents[p].e == e; p++) {
      if (ents[p].link == -1) {
        set = 1;
      } else if (ents[p].link == -2) {
        phi += ents[p].alpha;
      } else {
        entLink.push_back(ents[p].link);
        entAlpha.push_back(ents[p].alpha);
      }
    }
    rowSet.push_back(set);
    rowPhi.push_back(phi);
  }
  rowStart.push_back((int)entLink.size());
  A->nRows = (int)rowElem.size();
  const size_t rb = h->prec == 3 ? 8 : 4;
  auto up_r = [&](void* d, const std::vector<double>& v) {
    if (h->prec == 3)
      upload_typed<double>(dev, d, v);
    else
      upload_typed<float>(dev, d, v);
  };
  const size_t nl = std::max<size_t>(1, L.size());
  std::vector<int> slow;
  for (long long c = 0; c < N; c++) {
    const uint32_t v = fl[(size_t)c];
    if (v != 0u && !(v & FLAG3_SOLID)) slow.push_back((int)c);
  }
  {
    // every device buffer of the run, as adj_alloc rounds them (these tables, then the forward
    // run's): the handle's table block grows to hold them all before the first is taken
    auto al = [](size_t b) { return (std::max<size_t>(b, 1) + 255) / 256 * 256; };
    const size_t ns = slow.size(), nsr = std::max<size_t>(1, 19 * ns);
    const size_t nr = std::max<size_t>(1, rowElem.size()), ne = std::max<size_t>(1, entLink.size());
    const size_t nSeg = (size_t)((A->steps + A->K - 1) / A->K);
    const int tileY = kAdjThreads / 32;
    const size_t nBlocks = (size_t)((W + 31) / 32) * (size_t)((H + tileY - 1) / tileY) * (size_t)D;
    const size_t nParts = nBlocks + (ns + kSlowCells - 1) / kSlowCells;
    const size_t need = al((size_t)N * 4) + al(ns * 4) + 3 * al(nsr * 4) + 2 * al(nsr * rb) + 2 * al(nl * 8) +
                        5 * al(nl * rb) + al(nl) + al(nl * 8) + al(nr * 8) + al(nr) + al((nr + 1) * 4) +
                        al(nr * rb) + al(ne * 4) + al(ne * rb) + al(nSeg * sizeof(DevState3)) +
                        al(sizeof(DevState3)) + al(nParts * 8) + 2 * al(64) + 3 * al((size_t)A->steps * 8);
    reserve_adj_tables(h, A, need);
  }
  A->linkBase = (int*)adj_alloc(h, A, (size_t)N * 4, "adjoint link base");
  dev.h2d(A->linkBase, base.data(), (size_t)N * 4);
  dev.sync();
  A->nSlow = (int)slow.size();
  A->slowCells = (int*)adj_alloc(h, A, std::max<size_t>(1, slow.size()) * 4, "adjoint flagged cells");
  if (!slow.empty()) {
    dev.h2d(A->slowCells, slow.data(), slow.size() * 4);
    dev.sync();
  }
  // per flagged cell and direction, [i][cell]: the pull's sources and coefficients, and where its
  // adjoint goes (an element index, or -(link + 1))
  const size_t ns = slow.size();
  std::vector<int> sE1(19 * ns), sE2(19 * ns), sTgt(19 * ns);
  std::vector<double> sA1(19 * ns), sA2(19 * ns);
  std::atomic<bool> mismatch(false);
  // each cell's 19 records are independent: chunks of cells on host threads
  const int TS = (int)std::min<size_t>((size_t)table_threads(), std::max<size_t>(1, ns / 4096));
  run_threads(TS, [&](int t) {
    for (size_t c = ns * t / TS; c < ns * (t + 1) / TS; c++) {
      const int idx = slow[c];
      const uint32_t v = fl[(size_t)idx];
      if (v & FLAG3_INLET) {  // the inlet reads nothing (and has no link records)
        for (int i = 0; i < Q3; i++) {
          const size_t r = (size_t)i * ns + c;
          sE1[r] = sE2[r] = sTgt[r] = 0;
          sA1[r] = sA2[r] = 0.0;
        }
        continue;
      }
      const int bse = base[(size_t)idx];
      int rank = 0;
      for (int i = 0; i < Q3; i++) {
        const size_t r = (size_t)i * ns + c;
        sA2[r] = 0.0;
        if (i == 0 || !(v & (1u << i))) {
          const int e = (int)(i * N + idx - off3(i, W, H));
          sE1[r] = sE2[r] = sTgt[r] = e;
          sA1[r] = 1.0;
        } else {
          const int k = bse + rank++;
          if (bse < 0 || k >= A->nLinks) {
            mismatch = true;
            sE1[r] = sE2[r] = sTgt[r] = 0;
            sA1[r] = 0.0;
            continue;
          }
          const AdjLink3Host& Lk = A->hostLinks[(size_t)k];
          const bool single = Lk.e2 < 0 && Lk.a1 == 1.0;
          // a single source with coefficient 1 is the plain index; otherwise the sign bit marks the
          // record's two sources and coefficients
          sE1[r] = single ? (int)Lk.e1 : (int)((uint32_t)Lk.e1 | 0x80000000u);
          sE2[r] = Lk.e2 >= 0 ? (int)Lk.e2 : (int)Lk.e1;
          sA1[r] = Lk.a1;
          sA2[r] = Lk.e2 >= 0 ? Lk.a2 : 0.0;
          sTgt[r] = -(k + 1);
        }
      }
    }
  });
  if (mismatch) throw Error(CELLS_E_INVALID, "adjoint link table does not match the flags");
  const size_t nsr = std::max<size_t>(1, 19 * ns);
  A->sE1 = (int*)adj_alloc(h, A, nsr * 4, "adjoint flagged-cell records");
  A->sE2 = (int*)adj_alloc(h, A, nsr * 4, "adjoint flagged-cell records");
  A->sTgt = (int*)adj_alloc(h, A, nsr * 4, "adjoint flagged-cell records");
  A->sA1 = adj_alloc(h, A, nsr * (h->prec == 3 ? 8 : 4), "adjoint flagged-cell records");
  A->sA2 = adj_alloc(h, A, nsr * (h->prec == 3 ? 8 : 4), "adjoint flagged-cell records");
  if (ns) {
    dev.h2d(A->sE1, sE1.data(), sE1.size() * 4);
    dev.h2d(A->sE2, sE2.data(), sE2.size() * 4);
    dev.h2d(A->sTgt, sTgt.data(), sTgt.size() * 4);
    dev.sync();
    if (h->prec == 3) {
      upload_typed<double>(dev, A->sA1, sA1);
      upload_typed<double>(dev, A->sA2, sA2);
    } else {
      upload_typed<float>(dev, A->sA1, sA1);
      upload_typed<float>(dev, A->sA2, sA2);
    }
  }
  std::vector<long long> e1(L.size()), e2(L.size());
  std::vector<double> a1(L.size()), a2(L.size()), cF(L.size()), q(L.size());
  std::vector<signed char> qk(L.size());
  for (size_t k = 0; k < L.size(); k++) {
    e1[k] = L[k].e1;
    e2[k] = L[k].e2;
    a1[k] = L[k].a1;
    a2[k] = L[k].a2;
    cF[k] = L[k].cF;
    q[k] = L[k].q;
    qk[k] = (signed char)L[k].qKind;
  }
  A->le1 = (long long*)adj_alloc(h, A, nl * 8, "adjoint links");
  A->le2 = (long long*)adj_alloc(h, A, nl * 8, "adjoint links");
  A->la1 = adj_alloc(h, A, nl * rb, "adjoint links");
  A->la2 = adj_alloc(h, A, nl * rb, "adjoint links");
  A->lcF = adj_alloc(h, A, nl * rb, "adjoint links");
  A->lq = adj_alloc(h, A, nl * rb, "adjoint links");
  A->lqk = (signed char*)adj_alloc(h, A, nl, "adjoint links");
  A->lamG = adj_alloc(h, A, nl * rb, "adjoint link values");
  A->dqAcc = (double*)adj_alloc(h, A, nl * 8, "adjoint dJ/dq");
  if (!L.empty()) {
    dev.h2d(A->le1, e1.data(), L.size() * 8);
    dev.h2d(A->le2, e2.data(), L.size() * 8);
    dev.h2d(A->lqk, qk.data(), L.size());
    dev.sync();
    up_r(A->la1, a1);
    up_r(A->la2, a2);
    up_r(A->lcF, cF);
    up_r(A->lq, q);
  }
  const size_t nr = std::max<size_t>(1, rowElem.size());
  const size_t ne = std::max<size_t>(1, entLink.size());
  A->rowElem = (long long*)adj_alloc(h, A, nr * 8, "adjoint rows");
  A->rowSet = (unsigned char*)adj_alloc(h, A, nr, "adjoint rows");
  A->rowStart = (int*)adj_alloc(h, A, (nr + 1) * 4, "adjoint rows");
  A->rowPhi = adj_alloc(h, A, nr * rb, "adjoint rows");
  A->entLink = (int*)adj_alloc(h, A, ne * 4, "adjoint rows");
  A->entAlpha = adj_alloc(h, A, ne * rb, "adjoint rows");
  if (!rowElem.empty()) {
    dev.h2d(A->rowElem, rowElem.data(), rowElem.size() * 8);
    dev.h2d(A->rowSet, rowSet.data(), rowSet.size());
    dev.h2d(A->rowStart, rowStart.data(), rowStart.size() * 4);
    if (!entLink.empty()) dev.h2d(A->entLink, entLink.data(), entLink.size() * 4);
    dev.sync();
    up_r(A->rowPhi, rowPhi);
    if (!entAlpha.empty()) up_r(A->entAlpha, entAlpha);
  }
}

}  // namespace

namespace {

// The launch arguments of the adjoint step kernels for the recorded run (all but f, the adjoint
// buffers and the step position t, which enqueue_segment sets per step).
AdjLaunch3 adj_args(Cells3D* h, Adjoint3D* A) {
  AdjLaunch3 a;
  std::memset(&a, 0, sizeof(a));
  a.flags = h->flags;
  a.xTab = h->xTab;
  a.linkBase = A->linkBase;
  a.le1 = A->le1;
  a.le2 = A->le2;
  a.la1 = A->la1;
  a.la2 = A->la2;
  a.lcF = A->lcF;
  a.lq = A->lq;
  a.lqk = A->lqk;
  a.lamG = A->lamG;
  a.dqAcc = A->dqAcc;
  a.blockPart = A->blockPart;
  a.counter = A->counter;
  a.N = h->N;
  a.W = h->W;
  a.H = h->H;
  a.D = h->D;
  a.tileX = A->tileX;
  a.absorbX0 = h->absorbX0;
  a.nCellBlocks = A->nBlocks;
  a.slowCells = A->slowCells;
  a.nSlow = A->nSlow;
  a.sE1 = A->sE1;
  a.sE2 = A->sE2;
  a.sTgt = A->sTgt;
  a.sA1 = A->sA1;
  a.sA2 = A->sA2;
  a.nParts = A->nParts;
  a.nRows = A->nRows;
  a.rowElem = A->rowElem;
  a.rowSet = A->rowSet;
  a.rowStart = A->rowStart;
  a.entLink = A->entLink;
  a.entAlpha = A->entAlpha;
  a.rowPhi = A->rowPhi;
  a.n0Dev = A->n0Dev;
  a.uDev = A->uDev;
  a.wDev = A->wDev;
  a.dudn = A->dudn;
  return a;
}

// Recompute a segment's len states into state set `set` from its checkpoint copy in set[0].
void enqueue_recompute(Cells3D* h, Adjoint3D* A, int set, int len, int par0, cudaStream_t stream) {
  for (int t = 0; t + 1 < len; t++) {
    h->enqueue_step_between(A->seg[set][(size_t)t], A->seg[set][(size_t)t + 1], par0 ^ (t & 1), false, stream);
    h->dev.launches++;
  }
}

// The adjoint steps of a segment whose states are in set `set`, from the last to the first,
// starting from adjoint buffer c; with `next`, the next (earlier) segment's recompute into the
// other set runs beside them on side2.
void enqueue_sweep(Cells3D* h, Adjoint3D* A, AdjLaunch3& a, int set, int len, int c, bool next, int nextLen,
                   int nextPar0) {
  cudaStream_t s = h->dev.stream;
  if (next) {
    check_cuda(cudaEventRecord(A->fork2, s), "cudaEventRecord");
    check_cuda(cudaStreamWaitEvent(A->side2, A->fork2, 0), "cudaStreamWaitEvent");
    enqueue_recompute(h, A, set ^ 1, nextLen, nextPar0, A->side2);
    check_cuda(cudaEventRecord(A->join2, A->side2), "cudaEventRecord");
  }
  for (int t = len - 1; t >= 0; t--) {
    a.f = A->seg[set][(size_t)t];
    a.lamNext = A->lam[c];
    a.lamOut = A->lam[c ^ 1];
    a.t = t;
    check_cuda(launch_adjoint_step3(h->prec, a, s, A->side, A->fork, A->join), "adjoint step kernel");
    h->dev.launches += 3;
    c ^= 1;
  }
  if (next) check_cuda(cudaStreamWaitEvent(s, A->join2, 0), "cudaStreamWaitEvent");
}

// Full segments replay graphs when K is even (the parity pattern and buffers repeat).
bool segment_graphs(const Cells3D* h, const Adjoint3D* A) { return h->useGraphs && A->K % 2 == 0; }

void build_segment_graph(Cells3D* h, Adjoint3D* A, int set, int next, int cur) {
  cudaGraphExec_t& g = A->segGraph[set][next];
  if (g) cudaGraphExecDestroy(g);
  g = nullptr;
  AdjLaunch3 a = adj_args(h, A);
  const int par0 = A->parity0 & 1;  // the parity at every full segment's start (K even)
  const int64_t before = h->dev.launches;
  check_cuda(cudaStreamBeginCapture(h->dev.stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  enqueue_sweep(h, A, a, set, A->K, cur, next != 0, A->K, par0);
  cudaGraph_t graph = nullptr;
  check_cuda(cudaStreamEndCapture(h->dev.stream, &graph), "cudaStreamEndCapture");
  cudaError_t e = cudaGraphInstantiate(&g, graph, 0);
  cudaGraphDestroy(graph);
  check_cuda(e, "cudaGraphInstantiate");
  A->segGraphLaunches[set][next] = h->dev.launches - before;
  h->dev.launches = before;
}

// The state set of segment s: the sweep alternates sets, starting with set 0 at the last segment.
int seg_set(const Adjoint3D* A, int64_t s) {
  const int64_t nSeg = (A->steps + A->K - 1) / A->K;
  return (int)((nSeg - 1 - s) & 1);
}

// The sweep reaches its full segments with adjoint buffer 0, or 1 after an odd-length last segment.
int full_segment_cur(const Adjoint3D* A) {
  const int64_t nSeg = (A->steps + A->K - 1) / A->K;
  const int64_t lenLast = A->steps - (nSeg - 1) * A->K;
  return (lenLast < A->K && (lenLast & 1)) ? 1 : 0;
}

void build_segment_graphs(Cells3D* h, Adjoint3D* A) {
  const int64_t nSeg = (A->steps + A->K - 1) / A->K;
  const int cur = full_segment_cur(A);
  for (int64_t s = nSeg - 1; s >= 0; s--) {
    const int64_t len = std::min<int64_t>(A->K, A->steps - s * A->K);
    if (len != A->K) continue;
    const int set = seg_set(A, s), next = s > 0 ? 1 : 0;
    if (!A->segGraph[set][next]) build_segment_graph(h, A, set, next, cur);
  }
  A->segGraphCur = cur;
}

}  // namespace

// ---------------- C ABI ----------------

#define ADJ_TRY(h) try {
#define ADJ_CATCH(h)                                                         \
  }                                                                          \
  catch (const AllocError& e) {                                              \
    release_adjoint(h);                                                      \
    (h)->lastError = std::string("Solver3D allocation failed: ") + e.what(); \
    return CELLS_E_ALLOC;                                                    \
  }                                                                          \
  catch (const Error& e) {                                                   \
    (h)->lastError = e.what();                                               \
    return e.status;                                                         \
  }                                                                          \
  catch (const std::exception& e) {                                          \
    (h)->lastError = e.what();                                               \
    return CELLS_E_INVALID;                                                  \
  }                                                                          \
  return CELLS_OK;

extern "C" {

int cells3d_adjoint_forward(Cells3D* h, const Cells3DAdjointSpec* spec, double* objective) {
  if (!h || !spec) return CELLS_E_INVALID;
  ADJ_TRY(h)
  if (h->dev.fake) throw Error(CELLS_E_INVALID, "the adjoint needs a CUDA device");
  if (h->prec != CELLS_FP32 && h->prec != CELLS_FP64)
    throw Error(CELLS_E_PRECISION_UNSUPPORTED, "the adjoint runs with FP32 or FP64 storage");
  if (h->cfg.smagorinsky != 0.0) throw Error(CELLS_E_INVALID, "the adjoint supports smagorinsky = 0 only");
  if (spec->steps <= 0 || spec->checkpoint_every <= 0) throw Error(CELLS_E_INVALID, "steps and checkpoint_every must be positive");
  if (spec->component < 0 || spec->component > 2) throw Error(CELLS_E_INVALID, "component must be 0, 1 or 2");
  const int64_t s0 = h->step;
  if (spec->window_begin > spec->window_end || spec->window_begin <= s0 || spec->window_end > s0 + spec->steps)
    throw Error(CELLS_E_INVALID, "the objective window must lie within the recorded steps");
  const int64_t nWin = spec->window_end - spec->window_begin + 1;
  if (nWin > HISTORY_LEN) throw Error(CELLS_E_INVALID, "the objective window exceeds the 8192-sample force ring");
  if (19ll * h->N >= (1ll << 31)) throw Error(CELLS_E_INVALID, "the adjoint supports grids of fewer than 2^31 / 19 cells");
  // the previous run's streams, events and pinned segment slots carry over (detached here, after
  // their work has finished, so release_adjoint keeps them)
  Adjoint3D carry;
  if (Adjoint3D* old = h->adj.get()) {
    if (old->side) cudaStreamSynchronize(old->side);
    if (old->side2) cudaStreamSynchronize(old->side2);
    std::swap(carry.side, old->side);
    std::swap(carry.side2, old->side2);
    std::swap(carry.fork, old->fork);
    std::swap(carry.join, old->join);
    std::swap(carry.fork2, old->fork2);
    std::swap(carry.join2, old->join2);
    std::swap(carry.n0Host, old->n0Host);
    std::swap(carry.n0Cap, old->n0Cap);
  }
  release_adjoint(h);
  h->adj.reset(new Adjoint3D());
  Adjoint3D* A = h->adj.get();
  std::swap(A->side, carry.side);
  std::swap(A->side2, carry.side2);
  std::swap(A->fork, carry.fork);
  std::swap(A->join, carry.join);
  std::swap(A->fork2, carry.fork2);
  std::swap(A->join2, carry.join2);
  std::swap(A->n0Host, carry.n0Host);
  std::swap(A->n0Cap, carry.n0Cap);
  A->s0 = s0;
  A->steps = spec->steps;
  A->w0 = spec->window_begin;
  A->w1 = spec->window_end;
  A->K = spec->checkpoint_every;
  A->component = spec->component;
  A->scale = spec->scale;
  A->parity0 = h->parity;
  cells::Device& dev = h->dev;
  const size_t fBytes = 19ull * h->bpp * (size_t)h->N;
  const int64_t nSeg = (A->steps + A->K - 1) / A->K;
  const int segBufs = (int)std::min<int64_t>(A->K, A->steps);
  // one block for the checkpoints, both sets of recompute buffers and both adjoint states, each
  // at a 256-byte aligned stride; kept for the next recorded run while it fits
  const size_t stride = (fBytes + 255) / 256 * 256;
  const size_t need = (size_t)(nSeg + 2 * segBufs + 2) * stride;
  if (!h->adjStore || h->adjStoreBytes < need) {
    if (h->adjStore) {
      dev.release(h->adjStore);
      h->adjStore = nullptr;
      h->adjStoreBytes = 0;
    }
    if (need + (size_t)h->N * 16 > dev.free_bytes())
      throw AllocError("the adjoint's checkpoints need " + std::to_string(need) + " bytes; the device has " +
                       std::to_string(dev.free_bytes()) + " free");
    h->adjStore = dev.alloc(need, "adjoint checkpoints");
    h->adjStoreBytes = need;
  }
  build_tables(h, A);
  char* store = (char*)h->adjStore;
  A->ckStateBlock = (DevState3*)adj_alloc(h, A, (size_t)nSeg * sizeof(DevState3), "adjoint checkpoint");
  for (int64_t k = 0; k < nSeg; k++) {
    A->ck.push_back(store + (size_t)k * stride);
    A->ckState.push_back(A->ckStateBlock + k);
  }
  for (int set = 0; set < 2; set++)
    for (int k = 0; k < segBufs; k++) A->seg[set].push_back(store + (size_t)(nSeg + set * segBufs + k) * stride);
  A->endState = adj_alloc(h, A, sizeof(DevState3), "adjoint end state");
  A->lam[0] = store + (size_t)(nSeg + 2 * segBufs) * stride;
  A->lam[1] = store + (size_t)(nSeg + 2 * segBufs + 1) * stride;
  // 32-cell x tiles: each warp still reads 128-byte rows, and the tiles before the absorbing layer
  // take the collision code without it
  A->tileX = 32;
  const int tileY = kAdjThreads / A->tileX;
  A->nBlocks = ((h->W + A->tileX - 1) / A->tileX) * ((h->H + tileY - 1) / tileY) * h->D;
  A->nParts = A->nBlocks + (A->nSlow + kSlowCells - 1) / kSlowCells;
  A->blockPart = (double*)adj_alloc(h, A, (size_t)A->nParts * 8, "adjoint partials");
  A->counter = (unsigned*)adj_alloc(h, A, 64, "adjoint counter");
  A->dudn = (double*)adj_alloc(h, A, (size_t)A->steps * 8, "adjoint du");
  A->uDev = (double*)adj_alloc(h, A, (size_t)A->steps * 8, "adjoint step speeds");
  A->wDev = (double*)adj_alloc(h, A, (size_t)A->steps * 8, "adjoint step weights");
  A->n0Dev = (int*)adj_alloc(h, A, 64, "adjoint segment index");
  if (A->n0Cap < (size_t)nSeg) {
    if (A->n0Host) dev.free_host_pinned(A->n0Host);
    A->n0Host = nullptr;
    A->n0Cap = 0;
    A->n0Host = (int*)dev.host_pinned((size_t)nSeg * sizeof(int));
    A->n0Cap = (size_t)nSeg;
  }
  if (!A->side) check_cuda(cudaStreamCreateWithFlags(&A->side, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!A->side2) check_cuda(cudaStreamCreateWithFlags(&A->side2, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!A->fork2) check_cuda(cudaEventCreateWithFlags(&A->fork2, cudaEventDisableTiming), "cudaEventCreate");
  if (!A->join2) check_cuda(cudaEventCreateWithFlags(&A->join2, cudaEventDisableTiming), "cudaEventCreate");
  if (!A->fork) check_cuda(cudaEventCreateWithFlags(&A->fork, cudaEventDisableTiming), "cudaEventCreate");
  if (!A->join) check_cuda(cudaEventCreateWithFlags(&A->join, cudaEventDisableTiming), "cudaEventCreate");
  // the recorded run: a checkpoint at the start of every segment, force samples in the window
  const uint64_t written0 = h->forceSamplesRead + h->forceSteps.size();
  A->uStep.resize((size_t)A->steps);
  A->rampStep.resize((size_t)A->steps);
  for (int64_t n = 0; n < A->steps; n++) {
    const int64_t s = s0 + n;
    A->uStep[(size_t)n] = h->uin_at(s);
    A->rampStep[(size_t)n] = h->rampKind ? (h->rampTarget != 0.0 ? h->ramp_speed(s) / h->rampTarget : 0.0) : 1.0;
  }
  // Segments of K steps (K even) that are all sampled or all unsampled replay a graph of K steps
  // captured once per recorded run: with K even every segment starts at the parity of the first.
  cudaGraphExec_t recGraph[2] = {nullptr, nullptr};  // [sampled]
  int64_t recGraphLaunches[2] = {0, 0};
  const bool recGraphs = h->useGraphs && A->K % 2 == 0;
  auto record_graph = [&](int sampled) {
    const int64_t before = dev.launches;
    const int p0 = h->parity;
    check_cuda(cudaStreamBeginCapture(dev.stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    for (int t = 0; t < A->K; t++) {
      const int p = p0 ^ (t & 1);
      h->enqueue_step_between(h->f[p], h->f[p ^ 1], p, sampled != 0);
      dev.launches++;
    }
    cudaGraph_t graph = nullptr;
    check_cuda(cudaStreamEndCapture(dev.stream, &graph), "cudaStreamEndCapture");
    const cudaError_t e = cudaGraphInstantiate(&recGraph[sampled], graph, 0);
    cudaGraphDestroy(graph);
    check_cuda(e, "cudaGraphInstantiate");
    recGraphLaunches[sampled] = dev.launches - before;
    dev.launches = before;
  };
  try {
    for (int64_t n = 0; n < A->steps;) {
      if (n % A->K == 0) {
        const int64_t k = n / A->K;
        check_cuda(cudaMemcpyAsync(A->ck[(size_t)k], h->f[h->parity], fBytes, cudaMemcpyDeviceToDevice, dev.stream),
                   "checkpoint copy");
        check_cuda(cudaMemcpyAsync(A->ckState[(size_t)k], h->st, sizeof(DevState3), cudaMemcpyDeviceToDevice,
                                   dev.stream),
                   "checkpoint copy");
        const int64_t first = s0 + n + 1, last = s0 + n + A->K;  // the segment's step labels
        const bool all = first >= A->w0 && last <= A->w1, none = last < A->w0 || first > A->w1;
        if (recGraphs && n + A->K <= A->steps && (all || none)) {
          const int sampled = all ? 1 : 0;
          if (!recGraph[sampled]) record_graph(sampled);
          check_cuda(cudaGraphLaunch(recGraph[sampled], dev.stream), "cudaGraphLaunch");
          dev.launches += recGraphLaunches[sampled];
          for (int t = 0; t < A->K; t++) {
            h->step++;
            if (all) h->forceSteps.push_back((uint32_t)h->step);
          }
          n += A->K;
          continue;
        }
      }
      const int64_t label = s0 + n + 1;
      const bool sample = label >= A->w0 && label <= A->w1;
      h->enqueue_step_between(h->f[h->parity], h->f[h->parity ^ 1], h->parity, sample);
      dev.launches++;
      h->parity ^= 1;
      h->step++;
      if (sample) h->forceSteps.push_back((uint32_t)h->step);
      n++;
    }
  } catch (...) {
    for (cudaGraphExec_t g : recGraph)
      if (g) cudaGraphExecDestroy(g);
    throw;
  }
  for (cudaGraphExec_t g : recGraph)
    if (g) cudaGraphExecDestroy(g);
  check_cuda(cudaMemcpyAsync(A->endState, h->st, sizeof(DevState3), cudaMemcpyDeviceToDevice, dev.stream),
             "end state copy");
  // the objective from the window's samples (ring slots written0 .. written0 + nWin - 1)
  std::vector<double4> hist((size_t)nWin);
  size_t got = 0;
  for (uint64_t k = written0; k < written0 + (uint64_t)nWin;) {
    const size_t r = (size_t)(k % HISTORY_LEN);
    const size_t run = (size_t)std::min<uint64_t>(written0 + nWin - k, (uint64_t)(HISTORY_LEN - r));
    dev.d2h(hist.data() + got, h->history + r, run * sizeof(double4));
    got += run;
    k += run;
  }
  dev.sync();
  double sum = 0.0;
  for (const double4& v : hist) sum += A->component == 0 ? v.x : (A->component == 1 ? v.y : v.z);
  A->objective = A->scale * sum / (double)nWin;
  std::vector<double> wStep((size_t)A->steps, 0.0);
  for (int64_t n = 0; n < A->steps; n++) {
    const int64_t label = s0 + n + 1;
    if (label >= A->w0 && label <= A->w1) wStep[(size_t)n] = A->scale / (double)nWin;
  }
  dev.h2d(A->uDev, A->uStep.data(), (size_t)A->steps * 8);
  dev.h2d(A->wDev, wStep.data(), (size_t)A->steps * 8);
  dev.sync();
  A->endStep = h->step;
  A->argGen = h->argGen;
  // the backward sweep's segment graphs, built now (record time) rather than inside the sweep
  if (segment_graphs(h, A)) build_segment_graphs(h, A);
  if (objective) *objective = A->objective;
  ADJ_CATCH(h)
}

int cells3d_adjoint_backward(Cells3D* h, const void* terminal_adjoint, double* dJ_dsdf, double* dJ_du_in,
                             void* adjoint_out) {
  if (!h) return CELLS_E_INVALID;
  ADJ_TRY(h)
  Adjoint3D* A = h->adj.get();
  if (!A) throw Error(CELLS_E_INVALID, "adjoint_backward needs a recorded adjoint_forward");
  if (h->step != A->endStep || h->argGen != A->argGen)
    throw Error(CELLS_E_INVALID, "the solver changed after adjoint_forward: record the run again");
  cells::Device& dev = h->dev;
  const long long N = h->N;
  const size_t fBytes = 19ull * h->bpp * (size_t)N;
  dev.memset0(A->lam[0], fBytes);
  dev.memset0(A->lam[1], fBytes);
  dev.memset0(A->dqAcc, (size_t)std::max(1, A->nLinks) * 8);
  dev.memset0(A->dudn, (size_t)A->steps * 8);
  dev.memset0(A->counter, 4);
  int cur = 0;
  if (terminal_adjoint) {
    dev.h2d(A->lam[0], terminal_adjoint, fBytes);
    dev.sync();
  }
  const int64_t nSeg = (A->steps + A->K - 1) / A->K;
  AdjLaunch3 a = adj_args(h, A);
  const bool graphs = segment_graphs(h, A);
  if (graphs && A->segGraphCur != full_segment_cur(A)) build_segment_graphs(h, A);
  // restore a segment's device state and first state (its checkpoint) into its state set
  auto restore = [&](int64_t s) {
    check_cuda(cudaMemcpyAsync(h->st, A->ckState[(size_t)s], sizeof(DevState3), cudaMemcpyDeviceToDevice,
                               dev.stream),
               "checkpoint restore");
    check_cuda(cudaMemcpyAsync(A->seg[seg_set(A, s)][0], A->ck[(size_t)s], fBytes, cudaMemcpyDeviceToDevice,
                               dev.stream),
               "checkpoint restore");
  };
  auto seg_len = [&](int64_t s) { return (int)std::min<int64_t>(A->K, A->steps - s * A->K); };
  auto seg_par0 = [&](int64_t s) { return (int)((A->parity0 + s * A->K) & 1); };
  // the last segment's states first; every other segment's recompute runs beside the sweep of the
  // segment after it
  restore(nSeg - 1);
  enqueue_recompute(h, A, seg_set(A, nSeg - 1), seg_len(nSeg - 1), seg_par0(nSeg - 1), dev.stream);
  for (int64_t sgi = nSeg - 1; sgi >= 0; sgi--) {
    const int len = seg_len(sgi);
    const int set = seg_set(A, sgi);
    const bool next = sgi > 0;
    A->n0Host[sgi] = (int)(sgi * A->K);
    check_cuda(cudaMemcpyAsync(A->n0Dev, A->n0Host + sgi, sizeof(int), cudaMemcpyHostToDevice, dev.stream),
               "segment index copy");
    if (next) restore(sgi - 1);
    if (graphs && len == A->K && cur == A->segGraphCur) {
      check_cuda(cudaGraphLaunch(A->segGraph[set][next ? 1 : 0], dev.stream), "cudaGraphLaunch");
      dev.launches += A->segGraphLaunches[set][next ? 1 : 0];
    } else {
      enqueue_sweep(h, A, a, set, len, cur, next, next ? seg_len(sgi - 1) : 0, next ? seg_par0(sgi - 1) : 0);
    }
    if (len & 1) cur ^= 1;
  }
  check_cuda(cudaMemcpyAsync(h->st, A->endState, sizeof(DevState3), cudaMemcpyDeviceToDevice, dev.stream),
             "end state restore");
  if (adjoint_out) dev.d2h(adjoint_out, A->lam[cur], fBytes);
  std::vector<double> dq((size_t)std::max(1, A->nLinks)), dudn((size_t)A->steps);
  dev.d2h(dq.data(), A->dqAcc, dq.size() * 8);
  dev.d2h(dudn.data(), A->dudn, dudn.size() * 8);
  dev.sync();
  if (dJ_dsdf) {
    std::fill(dJ_dsdf, dJ_dsdf + N, 0.0);
    for (int k = 0; k < A->nLinks; k++) {
      const AdjLink3Host& L = A->hostLinks[(size_t)k];
      if (L.qKind == 0 || L.solid < 0) continue;
      dJ_dsdf[L.cell] += dq[(size_t)k] * L.dqdF;
      dJ_dsdf[L.solid] += dq[(size_t)k] * L.dqdS;
    }
  }
  if (dJ_du_in) {
    double s = 0.0;
    for (int64_t n = 0; n < A->steps; n++) s += dudn[(size_t)n] * A->rampStep[(size_t)n];
    *dJ_du_in = s;
  }
  ADJ_CATCH(h)
}

int cells3d_adjoint_release(Cells3D* h) {
  if (!h) return CELLS_E_INVALID;
  ADJ_TRY(h)
  release_adjoint(h);
  if (h->adjStore) {
    h->dev.release(h->adjStore);
    h->adjStore = nullptr;
    h->adjStoreBytes = 0;
  }
  if (h->adjTab) {
    h->dev.release(h->adjTab);
    h->adjTab = nullptr;
    h->adjTabBytes = 0;
  }
  ADJ_CATCH(h)
}

}  // extern "C"
