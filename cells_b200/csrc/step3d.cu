// Fused D3Q19 step: pull streaming, boundaries (inlet, outlet, slip faces, Bouzidi walls), TRT
// collision with optional Smagorinsky, absorbing layer and sponge, momentum-exchange force and its
// reduction into the force history ring.
//
// Semantics follow the reference kernel src/shaders/step3d.ts:170-223 (main) and :119-168
// (pullSlow3); the arithmetic order of the moments, equilibria and collision is the generated WGSL's.
//
// B200 work split: one launch per time step, its blocks in three roles that update disjoint sets
// of cells, all reading the source buffer and writing the destination buffer (see step3d_kernel):
//   * interior rows (y = 1 .. H-2, z = 1 .. D-2): x runs along warps, so each population load and
//     store of a warp is one contiguous run of the SoA array f[i*N + cell]; the 19 pulls come from
//     constant-bank bases already shifted by each direction's offset, with no flag read except in
//     rows that hold a body cell (rowBody[]); the inlet and outlet cells of each row ride along in
//     the same coalesced loads; with an even width f32, f16 and bf16 storage move two cells per
//     thread (an x-pair: one word per population for both) and collide them with packed f32x2
//     instructions; every step grid is launched as a programmatic dependent of the previous one;
//   * the y and z faces: the geometric boundary pull (slip mirrors, edges, outlet copy); with
//     x-pairs, the face rows with one outside side run the interior pair code with per-side pull
//     bases (the specular reflection is a pull of the mirrored population from the same plane or
//     row), and only the four edge rows take the one-cell face code;
//   * the body cells (every fluid cell with a flag in a row that holds a body cell): their pulls
//     (Bouzidi walls, mirrored sources on solids) are resolved into link records when the SDF is
//     set, so a step reads them with independent loads; on sampled steps the body blocks reduce
//     the momentum exchange in f64 (warp shuffles, one partial per block, the last block sums the
//     partials in a fixed order into the force ring), which is deterministic, unlike the
//     reference's atomic slot order (src/shaders/aux3d.ts:80);
//   * the relaxation rates and absorbing strength depend on x alone (without Smagorinsky) and come
//     from a W-entry table that the host fills with the reference's f32 arithmetic;
//   * every block first asks L2 for the pull sources of the interior tile a few z planes ahead of
//     its own (prefetch.global.L2, one 128-byte line per thread, no registers held), so the loads
//     of the blocks that start later find their lines in L2 instead of waiting for DRAM.
#include <algorithm>

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
  // per x-pair (x0 = 2j, x0 + 1), for f32 rates: entry 2j (omega+ of both, omega- of both),
  // entry 2j + 1 (sigma of both, 0, 0); the same values as xTab, laid out so a pair's rates load
  // as register pairs of the packed f32x2 collision
  const float4* xPair;
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
  int shellBlocks, bodyBlocks;   // block ranges of the face and body roles
  int tileTX, tileTY;            // interior tile: tileTY rows of tileTX cells
  int roleZ;                     // grid z-slices holding the face and body roles
  int absorbX0;                  // first x of the absorbing layer (W when there is none)
  int pfPlanes;                  // L2 prefetch distance in z planes of interior tiles (0: none)
  int pfShift, pfRowShift;       // log2 of the 128-byte stretches per tile row and of the rows
  // x-pair face tiles (facePairs = 1): the rows with one outside side -- rows y = 1 .. H-2 of the
  // z = 0 / z = D-1 planes (sides 0 / 1) and the y = 0 / y = H-1 rows of the planes between
  // (sides 2 / 3), tileTY rows per tile -- take the interior pair code with per-side pull bases:
  // fpull[side][i] + idx is the source of population i of cell idx (the slip face's specular
  // reflection for the directions that enter from outside), and fout[side][i] the offset from it
  // of the outlet copy's source for the directions with c_x = -1. The shell role keeps the edge
  // rows (two outside sides).
  const S* fpull[4][Q3];
  int fout[4][Q3];
  int facePairs, faceBlocks;
  int faceZTiles;                // tiles of the two z planes: 2 tilesX tilesY
  int faceYGroups;               // groups of tileTY rows along z per y side
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

// Moments, then the outlet equilibrium or the TRT collision of one cell (src/shaders/step3d.ts:38-102
// and :205-223), into o. f and o are in storage units; dividing the sums by SCALE and multiplying
// the weights by SCALE are exact, so every value equals the reference formula's.
//   * exact arithmetic evaluates the generated WGSL's expressions in its order;
//   * fast arithmetic evaluates the same TRT update in an equivalent form with about half the
//     operations per pair: A = omega+ w e - omega+/2 (fa + fb), B = omega- w rho cu - omega-/2 (fa - fb),
//     fa' = fa + A + B, fb' = fb + A - B, with e = drho + rho (cu^2/2 - 3u^2/2);
//   * the absorbing layer depends on x alone, so its branch is taken by whole warps (lanes outside
//     the layer add sources of zero);
//   * ABS = false compiles the collision of a cell outside the absorbing layer with no code for it:
//     left as a run-time branch, the compiler evaluates the absorbing sources for every cell.
template <class C, bool SMAG, bool ABS = true>
__device__ __forceinline__ void collide3(const StepArgs3<C>& a, const typename C::R (&f)[Q3], int x, bool outlet,
                                         typename C::R (&o)[Q3]) {
  using R = typename C::R;
  constexpr R IS = R(1) / R(C::SCALE);
  // 16-bit storage is issue-bound rather than bandwidth-bound, so its fast arithmetic uses the
  // leanest form: the pair sums s_p = f_p + f_p+1 and differences d_p = f_p - f_p+1 (p odd) feed both
  // the moments and the TRT update. Wider storage keeps the form with fewer live registers.
  constexpr bool kLean = !kExact && sizeof(typename C::S) == 2;
  R sp[Q3], dp[Q3];
  R drho, rho, ux, uy, uz, invRho;
  if constexpr (!kLean) {
    // moments, in the generated WGSL's left-to-right order
    R dsum = f[0];
#pragma unroll
    for (int i = 1; i < Q3; i++) dsum = dsum + f[i];
    drho = dsum * IS;
    rho = R(1) + drho;
    // fast arithmetic: the hardware reciprocal (branch-free, within 2 ulp) instead of IEEE division
    if constexpr (!kExact && sizeof(R) == 4)
      invRho = __fdividef(R(1), rho);
    else
      invRho = R(1) / rho;
    ux = ((f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16]) * IS) * invRho;
    uy = ((f[3] - f[4] + f[7] - f[8] + f[11] - f[12] - f[13] + f[14] + f[17] - f[18]) * IS) * invRho;
    uz = ((f[5] - f[6] + f[9] - f[10] + f[11] - f[12] - f[15] + f[16] - f[17] + f[18]) * IS) * invRho;
  } else {
#pragma unroll
    for (int p = 1; p < Q3; p += 2) {
      sp[p] = f[p] + f[p + 1];
      dp[p] = f[p] - f[p + 1];
    }
    drho = (f[0] + ((sp[1] + sp[3]) + (sp[5] + sp[7])) + ((sp[9] + sp[11]) + (sp[13] + (sp[15] + sp[17])))) * IS;
    rho = R(1) + drho;
    // the hardware reciprocal (branch-free, within 2 ulp) instead of IEEE division, with 1/SCALE folded in
    R invRhoS;
    if constexpr (sizeof(R) == 4)
      invRhoS = __fdividef(IS, rho);
    else
      invRhoS = IS / rho;
    invRho = invRhoS * R(C::SCALE);  // exact: SCALE is a power of two
    ux = (((dp[1] + dp[7]) + (dp[9] + dp[13])) + dp[15]) * invRhoS;
    uy = (((dp[3] + dp[7]) + (dp[11] - dp[13])) + dp[17]) * invRhoS;
    uz = (((dp[5] + dp[9]) + (dp[11] - dp[15])) - dp[17]) * invRhoS;
  }
  const R usq = R(1.5) * (ux * ux + uy * uy + uz * uz);
  if (outlet) {
    // pressure outlet: equilibrium at rho = 1 with the node's own velocity; fast arithmetic uses
    // feq_a,b = w (t +- cu) with t = cu^2/2 - 3u^2/2, sharing t between the pair
    if (kExact) {
#pragma unroll
      for (int i = 0; i < Q3; i++) o[i] = feq3s<C>(i, R(1), ux, uy, uz);
    } else {
      o[0] = -ws3<C>(0) * usq;
#pragma unroll
      for (int p = 1; p < Q3; p += 2) {
        const R cu = cu_of<R>(p, ux, uy, uz);
        const R t = cu * (R(0.5) * cu) - usq;
        o[p] = ws3<C>(p) * (t + cu);
        o[p + 1] = ws3<C>(p) * (t - cu);
      }
    }
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
  const bool absorb = !ABS ? false : (kExact ? sigma > R(0) : __any_sync(__activemask(), sigma > R(0)));
  R ut = R(0), dq = R(0);
  if (absorb) {
    ut = (R)a.st->uIn[a.par];
    dq = R(1.5) * rho * (ut * ut - ux * ux - uy * uy - uz * uz);
  }
  if (kExact) {
    {
      R s0 = R(0);
      if (absorb) s0 += sigma * ws3<C>(0) * -dq;
      o[0] = f[0] - omP * (f[0] - ws3<C>(0) * (drho - rho * usq)) + s0;
    }
#pragma unroll
    for (int p = 1; p < Q3; p += 2) {
      const R cu = cu_of<R>(p, ux, uy, uz);
      const R eqS = ws3<C>(p) * (drho + rho * (R(0.5) * cu * cu - usq));
      const R eqA = ws3<C>(p) * rho * cu;
      const R sym = omP * (R(0.5) * (f[p] + f[p + 1]) - eqS);
      const R asym = omM * (R(0.5) * (f[p] - f[p + 1]) - eqA);
      R sS = R(0), sA = R(0);
      if (absorb) {
        const R cut = R(3) * R(cx3(p)) * ut;
        sS += sigma * ws3<C>(p) * (R(0.5) * rho * (cut * cut - cu * cu) - dq);
        sA += sigma * ws3<C>(p) * rho * (cut - cu);
      }
      o[p] = f[p] - sym - asym + sS + sA;
      o[p + 1] = f[p + 1] - sym + asym + sS - sA;
    }
  } else {
   if constexpr (kLean) {
    // e_p = rho cu^2 / 2 + K0 with K0 = drho - rho usq, so with cP = omega+ w and cM = omega- w rho:
    //   A = cP e - omega+/2 s_p = (cP rho / 2) cu cu + (cP K0 - omega+/2 s_p)
    //   B = cM cu - omega-/2 d_p
    const R K0 = drho - rho * usq;
    const R nhP = R(-0.5) * omP, nhM = R(-0.5) * omM;
    const R u3[3] = {R(3) * ux, R(3) * uy, R(3) * uz};
    const R cP0 = omP * ws3<C>(1), cP1 = omP * ws3<C>(7);
    const R cPr[2] = {cP0 * (R(0.5) * rho), cP1 * (R(0.5) * rho)};
    const R cK[2] = {cP0 * K0, cP1 * K0};
    const R cM[2] = {omM * ws3<C>(1) * rho, omM * ws3<C>(7) * rho};
    R v0 = f[0] - omP * (f[0] - ws3<C>(0) * K0);
    if (absorb) v0 += sigma * ws3<C>(0) * -dq;
    o[0] = v0;
#pragma unroll
    for (int p = 1; p < Q3; p += 2) {
      const int k = p <= 5 ? 0 : 1;
      R cu;
      switch (p) {  // 3 (c_p . u) from the precomputed 3u
        case 1: cu = u3[0]; break;
        case 3: cu = u3[1]; break;
        case 5: cu = u3[2]; break;
        case 7: cu = u3[0] + u3[1]; break;
        case 9: cu = u3[0] + u3[2]; break;
        case 11: cu = u3[1] + u3[2]; break;
        case 13: cu = u3[0] - u3[1]; break;
        case 15: cu = u3[0] - u3[2]; break;
        default: cu = u3[1] - u3[2]; break;
      }
      R A = (cPr[k] * cu) * cu + (cK[k] + nhP * sp[p]);
      R B = cM[k] * cu + nhM * dp[p];
      if (absorb) {
        const R cut = R(3) * R(cx3(p)) * ut;
        const R sw = sigma * ws3<C>(p);
        A += sw * (R(0.5) * rho * (cut * cut - cu * cu) - dq);
        B += sw * rho * (cut - cu);
      }
      o[p] = f[p] + A + B;
      o[p + 1] = f[p + 1] + A - B;
    }
   } else {
    const R hP = R(0.5) * omP, hM = R(0.5) * omM;
    const R u3[3] = {R(3) * ux, R(3) * uy, R(3) * uz};
    const R cP[2] = {omP * ws3<C>(1), omP * ws3<C>(7)};
    const R cM[2] = {omM * ws3<C>(1) * rho, omM * ws3<C>(7) * rho};
    R v0 = f[0] - omP * (f[0] - ws3<C>(0) * (drho - rho * usq));
    if (absorb) v0 += sigma * ws3<C>(0) * -dq;
    o[0] = v0;
#pragma unroll
    for (int p = 1; p < Q3; p += 2) {
      const int k = p <= 5 ? 0 : 1;
      R cu;
      switch (p) {  // 3 (c_p . u) from the precomputed 3u
        case 1: cu = u3[0]; break;
        case 3: cu = u3[1]; break;
        case 5: cu = u3[2]; break;
        case 7: cu = u3[0] + u3[1]; break;
        case 9: cu = u3[0] + u3[2]; break;
        case 11: cu = u3[1] + u3[2]; break;
        case 13: cu = u3[0] - u3[1]; break;
        case 15: cu = u3[0] - u3[2]; break;
        default: cu = u3[1] - u3[2]; break;
      }
      const R e = rho * (cu * (R(0.5) * cu) - usq) + drho;
      R A = cP[k] * e - hP * (f[p] + f[p + 1]);
      R B = cM[k] * cu - hM * (f[p] - f[p + 1]);
      if (absorb) {
        const R cut = R(3) * R(cx3(p)) * ut;
        const R sw = sigma * ws3<C>(p);
        A += sw * (R(0.5) * rho * (cut * cut - cu * cu) - dq);
        B += sw * rho * (cut - cu);
      }
      o[p] = f[p] + A + B;
      o[p + 1] = f[p + 1] + A - B;
    }
   }
  }
}


// ---------------- packed f32x2 arithmetic (sm_100) ----------------
// One FADD2 / FMUL2 / FFMA2 instruction applies the same f32 operation to two values, each
// component rounding exactly as the scalar instruction would. The x-pair kernel keeps cell x0 in .x
// and cell x0 + 1 in .y, so one instruction stream updates both cells.
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(d)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)), "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&d);
}
__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }

// 3 (c_p . u) for the lower member p of each pair, from u3 = 3u
__device__ __forceinline__ float2 cu3x2(int p, const float2 (&u3)[3]) {
  switch (p) {
    case 1: return u3[0];
    case 3: return u3[1];
    case 5: return u3[2];
    case 7: return add2(u3[0], u3[1]);
    case 9: return add2(u3[0], u3[2]);
    case 11: return add2(u3[1], u3[2]);
    case 13: return sub2(u3[0], u3[1]);
    case 15: return sub2(u3[0], u3[2]);
    default: return sub2(u3[1], u3[2]);
  }
}

// The fast TRT collision of the two cells of an x-pair (cell x0 in .x, x0 + 1 in .y) with packed
// f32x2 instructions, stored as one 32-bit word per population. It evaluates the lean pair form of
// collide3 per component in f32: with s_p = f_p + f_p+1 and d_p = f_p - f_p+1 (exact for values
// of 16-bit storage, whose sums and differences fit the f32 significand; rounded once for f32),
//   o_p = S + T, o_p+1 = S - T,  S = (1 - omega+)/2 s_p + omega+ w (rho cu^2/2 + K0),
//                                T = (1 - omega-)/2 d_p + omega- w rho cu,   K0 = drho - rho usq,
// which is f_p + A + B and f_p+1 + A - B of collide3 rearranged, so only s_p and d_p stay live.
// Only the reciprocal of rho, and with Smagorinsky the relaxation time, run per cell.
// The inlet cell (x0 = 0, when IN) and the outlet cell (x0 + 1 = W - 1, when OUT) go through the
// same instructions: with omega+ = omega- = 1, rho = 1, drho = 0 and no absorbing source the update
// is exactly the equilibrium feq(1, u), at u = (uIn, 0, 0) for the inlet (step3d.ts:190-193) and at
// the node's own velocity for the outlet.
template <class C, bool SMAG, bool ABS, bool IN, bool OUT>
__device__ __forceinline__ void collide3x2_store(const StepArgs3<C>& a, const typename C::Pair (&r)[Q3], int x0,
                                                 int idx) {
  constexpr float IS = 1.0f / C::SCALE;
  float2 sp[Q3], dp[Q3];  // entries p = 1, 3, .., 17
  const float2 f0 = make_float2(C::lo(r[0]), C::hi(r[0]));
#pragma unroll
  for (int p = 1; p < Q3; p += 2) {
    const float2 fa = make_float2(C::lo(r[p]), C::hi(r[p]));
    const float2 fb = make_float2(C::lo(r[p + 1]), C::hi(r[p + 1]));
    sp[p] = add2(fa, fb);
    dp[p] = sub2(fa, fb);
  }
  const float2 dsum = add2(add2(f0, add2(add2(sp[1], sp[3]), add2(sp[5], sp[7]))),
                           add2(add2(sp[9], sp[11]), add2(sp[13], add2(sp[15], sp[17]))));
  float2 drho = mul2(dsum, bc2(IS));
  float2 rho = add2(drho, bc2(1.0f));
  // the hardware reciprocal (branch-free, within 2 ulp) with 1/SCALE folded in, per cell
  const float2 invRhoS = make_float2(__fdividef(IS, rho.x), __fdividef(IS, rho.y));
  float2 ux = mul2(add2(add2(add2(dp[1], dp[7]), add2(dp[9], dp[13])), dp[15]), invRhoS);
  float2 uy = mul2(add2(add2(add2(dp[3], dp[7]), sub2(dp[11], dp[13])), dp[17]), invRhoS);
  float2 uz = mul2(sub2(add2(add2(dp[5], dp[9]), sub2(dp[11], dp[15])), dp[17]), invRhoS);
  const bool inlet = IN && x0 == 0, outlet = OUT && x0 + 1 == a.W - 1;
  if (inlet) {
    ux.x = (float)a.st->uIn[a.par];
    uy.x = 0.0f;
    uz.x = 0.0f;
  }
  const float2 u2 = fma2(uz, uz, fma2(uy, uy, mul2(ux, ux)));
  const float2 nusq = mul2(bc2(-1.5f), u2);  // -3u^2/2
  const float2 u3[3] = {mul2(bc2(3.0f), ux), mul2(bc2(3.0f), uy), mul2(bc2(3.0f), uz)};
  const float4 t0 = a.xPair[x0];
  float2 omP = make_float2(t0.x, t0.y), omM = make_float2(t0.z, t0.w);
  if (SMAG) {
    // second moments of the non-equilibrium part, per pair: n_p + n_p+1 = s_p - 2 w (rho cu^2/2 + K0)
    const float2 K0s = fma2(rho, nusq, drho);
    const float2 hr = mul2(bc2(0.5f), rho);
    float2 pxx, pyy, pzz, pxy, pxz, pyz;
#pragma unroll
    for (int p = 1; p < Q3; p += 2) {
      const float2 cu = cu3x2(p, u3);
      const float2 n = fma2(bc2(-2.0f * ws3<C>(p)), fma2(mul2(hr, cu), cu, K0s), sp[p]);
      if (p == 1) pxx = n;
      else if (cx3(p) != 0) pxx = add2(pxx, n);
      if (p == 3) pyy = n;
      else if (cy3(p) != 0) pyy = add2(pyy, n);
      if (p == 5) pzz = n;
      else if (cz3(p) != 0) pzz = add2(pzz, n);
      if (p == 7) pxy = n;
      else if (cx3(p) * cy3(p) == -1) pxy = sub2(pxy, n);
      if (p == 9) pxz = n;
      else if (cx3(p) * cz3(p) == -1) pxz = sub2(pxz, n);
      if (p == 11) pyz = n;
      else if (cy3(p) * cz3(p) == -1) pyz = sub2(pyz, n);
    }
    const float2 off = fma2(pyz, pyz, fma2(pxz, pxz, mul2(pxy, pxy)));
    const float2 q = fma2(bc2(2.0f), off, fma2(pzz, pzz, fma2(pyy, pyy, mul2(pxx, pxx))));
    float om[2], omm[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const float qc = c ? q.y : q.x, omegaBase = c ? omP.y : omP.x;
      const float ir = (c ? invRhoS.y : invRhoS.x) * C::SCALE;  // 1/rho, exact: SCALE is a power of two
      const float pi = sqrtf(qc) * IS;                          // sqrt(SCALE^2 x) = SCALE sqrt(x) exactly
      const float tt = 1.0f / omegaBase;
      const float tEff = 0.5f * (tt + sqrtf(tt * tt + 25.45584412271571f * a.smagC2 * pi * ir));
      om[c] = 1.0f / tEff;
      omm[c] = 1.0f / (0.5f + a.lambda / (1.0f / om[c] - 0.5f));
    }
    omP = make_float2(om[0], om[1]);
    omM = make_float2(omm[0], omm[1]);
  }
  float2 sigma = bc2(0.0f);
  if (ABS) {
    const float4 t1 = a.xPair[x0 + 1];
    sigma = make_float2(t1.x, t1.y);
  }
  // the boundary cells relax fully to feq(1, u)
  if (inlet) {
    omP.x = omM.x = 1.0f;
    rho.x = 1.0f;
    drho.x = 0.0f;
    sigma.x = 0.0f;
  }
  if (outlet) {
    omP.y = omM.y = 1.0f;
    rho.y = 1.0f;
    drho.y = 0.0f;
    sigma.y = 0.0f;
  }
  const bool absorb = ABS && __any_sync(__activemask(), sigma.x > 0.0f || sigma.y > 0.0f);
  const float2 K0 = fma2(rho, nusq, drho);  // drho - rho usq
  const float2 aP = fma2(bc2(-0.5f), omP, bc2(0.5f)), aM = fma2(bc2(-0.5f), omM, bc2(0.5f));
  const float2 hrho = mul2(bc2(0.5f), rho);
  const float2 cP0 = mul2(omP, bc2(ws3<C>(1))), cP1 = mul2(omP, bc2(ws3<C>(7)));
  const float2 cPr[2] = {mul2(cP0, hrho), mul2(cP1, hrho)};
  const float2 cK[2] = {mul2(cP0, K0), mul2(cP1, K0)};
  const float2 omMr = mul2(omM, rho);
  const float2 cM[2] = {mul2(omMr, bc2(ws3<C>(1))), mul2(omMr, bc2(ws3<C>(7)))};
  float2 ut = bc2(0.0f), ndq = bc2(0.0f), sr = bc2(0.0f);
  if (absorb) {
    ut = bc2((float)a.st->uIn[a.par]);
    ndq = mul2(mul2(bc2(-1.5f), rho), fma2(ut, ut, mul2(bc2(-1.0f), u2)));  // -3/2 rho (ut^2 - u^2)
    sr = mul2(sigma, rho);
  }
  {
    // rest population: (1 - omega+) f0 + omega+ w0 K0
    float2 v0 = fma2(add2(aP, aP), f0, mul2(omP, mul2(bc2(ws3<C>(0)), K0)));
    if (absorb) v0 = fma2(mul2(sigma, bc2(ws3<C>(0))), ndq, v0);
    C::st_pair_fast(a.out[0] + idx, v0.x, v0.y);
  }
#pragma unroll
  for (int p = 1; p < Q3; p += 2) {
    const int k = p <= 5 ? 0 : 1;
    const float2 cu = cu3x2(p, u3);
    float2 S = fma2(aP, sp[p], fma2(mul2(cPr[k], cu), cu, cK[k]));
    float2 T = fma2(aM, dp[p], mul2(cM[k], cu));
    if (absorb) {
      const float2 cut = mul2(bc2(3.0f * (float)cx3(p)), ut);
      // S += sigma w (rho/2 (cut^2 - cu^2) - dq); T += sigma w rho (cut - cu)
      const float2 d2 = sub2(mul2(cut, cut), mul2(cu, cu));
      S = fma2(mul2(sigma, bc2(ws3<C>(p))), fma2(hrho, d2, ndq), S);
      T = fma2(mul2(sr, bc2(ws3<C>(p))), sub2(cut, cu), T);
    }
    const float2 oa = add2(S, T), ob = sub2(S, T);
    C::st_pair_fast(a.out[p] + idx, oa.x, oa.y);
    C::st_pair_fast(a.out[p + 1] + idx, ob.x, ob.y);
  }
}

template <class C, bool SMAG, bool ABS = true>
__device__ __forceinline__ void collide_store(const StepArgs3<C>& a, const typename C::R (&f)[Q3], int x, int idx,
                                              bool outlet) {
  typename C::R o[Q3];
  collide3<C, SMAG, ABS>(a, f, x, outlet, o);
#pragma unroll
  for (int i = 0; i < Q3; i++) a.out[i][idx] = C::enc_raw(o[i]);
}

__device__ __forceinline__ double ramp_speed(int kind, double target, double rampSteps, int every, unsigned step) {
  const double sq = (double)((step / (unsigned)every) * (unsigned)every);
  const double t = fmin(1.0, sq / rampSteps);
  return kind == 1 ? target * t : target * (t * t * (3.0 - 2.0 * t));
}

// ---------------- the step kernel: one launch per time step ----------------
//
// Blocks of 128 threads take one of three roles by block index (computed on the host):
//   [0, shellBlocks)                      the face cells: z = 0 and z = D-1 planes, y = 0 and y = H-1
//                                         rows of the planes between, one cell per thread, x fastest;
//   [shellBlocks, + bodyBlocks)           32 body cells per block, their 19 links resolved in parallel;
//   [shellBlocks + bodyBlocks, + tiles)   the rows y = 1 .. H-2 of planes z = 1 .. D-2 in tiles of
//                                         tileTY rows of tileTX cells (two cells per thread for
//                                         f32 / 16-bit storage with an even width, one otherwise).
// The face and body blocks have the lowest indices, so they are dispatched first and run beside
// the first interior tiles. Cells a role does not own it leaves alone: in a row that holds a body
// cell, every cell with a flag belongs to the body role. Block 0 also advances the device step
// counter and the device-side inlet ramp for the next step.

constexpr int kStepThreads = 128;

// Number of cells on the faces: the z = 0 and z = D-1 planes and the y = 0 and y = H-1 rows of the
// planes between.
__host__ __device__ __forceinline__ long long shell_cells3(int W, int H, int D) {
  const long long nz = D >= 2 ? 2 : 1, ny = H >= 2 ? 2 : 1;
  const long long inD = D > 2 ? D - 2 : 0;
  return nz * W * H + ny * W * inD;
}

// Whether direction i enters a face row's cells from outside the grid: SIDE 0 / 1 are the rows
// y = 1 .. H-2 of the z = 0 / z = D-1 planes, 2 / 3 the y = 0 / y = H-1 rows of the planes between.
template <int SIDE>
__host__ __device__ __forceinline__ constexpr bool face_out3(int i) {
  return SIDE == 0 ? cz3(i) == 1 : (SIDE == 1 ? cz3(i) == -1 : (SIDE == 2 ? cy3(i) == 1 : cy3(i) == -1));
}

// A cell of a face row with one outside side (pullSlow3, step3d.ts:119-168, for a cell without solid
// neighbours): every direction's rule is fixed at compile time -- a plain pull, the slip face's
// specular reflection from the same row or plane, or at the outlet column the zero-gradient copy
// from x = W-2 -- and the pulls go out before the body-row test. x >= 1 (the caller handles the
// inlet), so every source is inside the grid.
template <class C, bool SMAG, int SIDE>
__device__ __forceinline__ void face_row_cell3(const StepArgs3<C>& a, int x, int row, int idx) {
  using R = typename C::R;
  const int W = a.W, WH = a.W * a.H;
  const bool outlet = x == W - 1;
  R f[Q3];
  f[0] = C::raw(a.src + idx);
#pragma unroll
  for (int i = 1; i < Q3; i++) {
    int pop = i, cell;
    if (cx3(i) == -1 && outlet) {
      cell = (W - 2) + W * row;  // outlet: zero-gradient copy (the x rule comes first)
    } else if (face_out3<SIDE>(i)) {
      pop = SIDE < 2 ? mirror_z3(i) : mirror_y3(i);  // slip: specular reflection, own plane / row
      cell = SIDE < 2 ? idx - (cx3(i) + cy3(i) * W) : idx - (cx3(i) + cz3(i) * WH);
    } else {
      cell = idx - (cx3(i) + cy3(i) * W + cz3(i) * WH);
    }
    f[i] = C::raw(a.src + (long long)pop * a.N + cell);
  }
  if (a.rowBody[row] && __ldg(a.flags + idx) != 0u) return;
  collide_store<C, SMAG>(a, f, x, idx, outlet);
}

// A face cell: pullSlow3 (step3d.ts:119-168) for a cell without solid neighbours, every mirrored
// source being fluid; the inlet cell stores the inflow equilibrium. With 16-bit storage, cells of
// rows with one outside side take face_row_cell3 (its per-side code measured faster in the
// issue-bound 16-bit kernels and slower in the memory-bound f32 / f64 ones, where the general
// rules below stay).
template <class C, bool SMAG>
__device__ __forceinline__ void shell_role(const StepArgs3<C>& a, int b, int tid) {
  using R = typename C::R;
  const int W = a.W, H = a.H, D = a.D;
  long long t = (long long)b * kStepThreads + tid;
  int x, y, z;
  bool onZ = false;  // a cell of the z = 0 or z = D-1 plane
  const long long nzp = D >= 2 ? 2 : 1, nyr = H >= 2 ? 2 : 1;
  const long long inD = D > 2 ? D - 2 : 0;
  const long long cz = nzp * W * H, cy = nyr * W * inD;
  if (a.facePairs) {
    // the face rows went to the x-pair face tiles: the four edge rows (y = 0 or H-1, z = 0 or D-1)
    if (t >= 4LL * W) return;
    const int e = (int)(t / W);
    x = (int)(t - (long long)e * W);
    y = (e & 1) ? H - 1 : 0;
    z = (e & 2) ? D - 1 : 0;
    onZ = true;
  } else if (t < cz) {
    const long long plane = t / ((long long)W * H);
    const long long r = t - plane * W * H;
    z = plane == 0 ? 0 : D - 1;
    y = (int)(r / W);
    x = (int)(r - (long long)y * W);
    onZ = true;
  } else if ((t -= cz) < cy) {
    const long long side = t / (W * inD);
    const long long r = t - side * W * inD;
    y = side == 0 ? 0 : H - 1;
    z = 1 + (int)(r / W);
    x = (int)(r - (long long)(z - 1) * W);
  } else {
    return;
  }
  const int row = y + H * z;
  const int idx = x + W * row;
  if constexpr (sizeof(typename C::S) == 2) {
    // side as in face_out3 for rows with one outside side (edge rows and thin grids take the rules below)
    const int side = onZ ? ((D >= 2 && y >= 1 && y <= H - 2) ? (z == 0 ? 0 : 1) : 4) : (H >= 2 ? (y == 0 ? 2 : 3) : 4);
    if (x != 0 && side < 4) {
      switch (side) {
        case 0: face_row_cell3<C, SMAG, 0>(a, x, row, idx); return;
        case 1: face_row_cell3<C, SMAG, 1>(a, x, row, idx); return;
        case 2: face_row_cell3<C, SMAG, 2>(a, x, row, idx); return;
        default: face_row_cell3<C, SMAG, 3>(a, x, row, idx); return;
      }
    }
  }
  if (a.rowBody[row] && __ldg(a.flags + idx) != 0u) return;
  if (x == 0) {
    // inlet: equilibrium at the inflow speed, no collision (step3d.ts:190-193)
    const double* eq = a.st->inletEq[a.par];
#pragma unroll
    for (int i = 0; i < Q3; i++) a.out[i][idx] = C::enc_raw((R)eq[i]);
    return;
  }
  const bool outlet = x == W - 1;
  const long long N = a.N;
  const long long WH = (long long)W * H;
  R f[Q3];
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
  collide_store<C, SMAG>(a, f, x, idx, outlet);
}

// Sum of the block's forces in f64 (warp shuffles, then the warps in order) into partials[slot];
// the last of the nSlots body blocks to finish sums the partials in slot order into the force
// ring. Deterministic for a fixed body list.
template <class C>
__device__ __forceinline__ void finish_forces(typename C::R fx, typename C::R fy, typename C::R fz, int slot,
                                              int nSlots, double4* __restrict__ partials,
                                              double4* __restrict__ history, DevState3* __restrict__ st, int tid) {
  __shared__ double red[3][kStepThreads / 32];
  __shared__ int amLast;
  const int lane = tid & 31, warp = tid >> 5;
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
    for (int w = 0; w < kStepThreads / 32; w++) {
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

// 32 body cells: item (lane, i) resolves link i of cell lane (a record load, then one or two
// source loads, independent across items) into shared memory; then one thread per cell sums the
// momentum exchange in the reference's direction order and collides.
template <class C, bool SMAG>
__device__ __forceinline__ void body_role(const StepArgs3<C>& a, int bb, int tid) {
  using R = typename C::R;
  __shared__ R sv[Q3][32];  // pulled populations in storage units
  __shared__ R sm[Q3][32];  // momentum-exchange term of each link (0 when the link exchanges none)
  for (int item = tid; item < 32 * Q3; item += kStepThreads) {
    const int lane = item & 31, dir = item >> 5;
    const int t = bb * 32 + lane;
    if (t >= a.nBody) continue;
    const int idx = a.bodyCells[t];
    if (dir == 0) {
      sv[0][lane] = C::raw(a.src + idx);
      continue;
    }
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
  __syncthreads();
  R fx = R(0), fy = R(0), fz = R(0);
  const int lane = tid;
  const int t = bb * 32 + lane;
  if (lane < 32 && t < a.nBody) do {
      const int idx = a.bodyCells[t];
      const int meta = a.links.meta[t];
      const int x = meta & ((1 << 29) - 1);
      if (meta & (1 << 30)) {
        // inlet cell of a body row: equilibrium at the inflow speed
        const double* eq = a.st->inletEq[a.par];
#pragma unroll
        for (int i = 0; i < Q3; i++) a.out[i][idx] = C::enc_raw((R)eq[i]);
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
  if (a.sample) finish_forces<C>(fx * IS, fy * IS, fz * IS, bb, a.bodyBlocks, a.partials, a.history, a.st, tid);
}

// Interior rows, one cell per thread. Interior cells pull their 19 populations from the
// constant-bank shifted bases. The outlet cell (x = W-1) pulls the same way except for the five
// directions with c_x = -1, whose source is the copy from (W-2, y, z): a fixed index offset per
// direction, so all lanes of a warp still issue the same coalesced loads. The inlet cell (x = 0)
// loads nothing and stores the inflow equilibrium; inlet and outlet stores are short tails, paid
// once per row. ABS / OUT: the tile overlaps the absorbing layer / holds the outlet column.
template <class C, bool SMAG, bool ABS, bool OUT>
__device__ __forceinline__ void bulk_role(const StepArgs3<C>& a, int tz) {
  using R = typename C::R;
  const int x = blockIdx.x * a.tileTX + threadIdx.x;
  const int y = 1 + blockIdx.y * a.tileTY + threadIdx.y;
  const int z = 1 + tz;
  const int W = a.W, H = a.H;
  if (x >= W || y >= H - 1) return;
  const int row = y + H * z;
  const int idx = x + W * row;
  const bool outlet = OUT && x == W - 1;
  const long long WH = (long long)W * H;
  // the pulls go out before the body-row and inlet tests, so they do not wait for them (every
  // interior pull address is inside the grid; body and inlet cells discard them)
  R f[Q3];
#pragma unroll
  for (int i = 0; i < Q3; i++) {
    int e = idx;
    // outlet: zero-gradient copy from (W-2, y, z) for the directions entering through x = W-1
    if (cx3(i) == -1 && outlet) e += (int)(-2 + cy3(i) * (long long)W + cz3(i) * WH);
    f[i] = C::raw(a.pull[i] + e);
  }
  if (a.rowBody[row] && __ldg(a.flags + idx) != 0u) return;
  if (x == 0) {
    // inlet: equilibrium at the inflow speed, no collision (step3d.ts:190-193)
    const double* eq = a.st->inletEq[a.par];
#pragma unroll
    for (int i = 0; i < Q3; i++) a.out[i][idx] = C::enc_raw((R)eq[i]);
    return;
  }
  collide_store<C, SMAG, ABS>(a, f, x, idx, outlet);
}

// Interior rows for f32, f16 and bf16 storage and an even width: each thread updates the x-pair
// (x0, x0 + 1), x0 even. One address per population serves both cells; the populations with c_x = 0
// arrive as one word holding both cells' values (8 bytes for f32, 4 for 16-bit storage), the
// others as two single-cell loads; the 19 results are stored as one word per population. Cells of
// the pair that belong to the body role are left alone. ABS / OUT: the tile overlaps the absorbing
// layer / holds the outlet column. FACE: the pair lies in a face row of side `side` (see
// StepArgs3::fpull), whose pull bases come from the per-side tables.
template <class C, bool SMAG, bool ABS, bool OUT, bool FACE>
__device__ __forceinline__ void pair_cells(const StepArgs3<C>& a, int x0, int y, int z, int side) {
  using R = typename C::R;
  using S = typename C::S;
  const int W = a.W, H = a.H;
  const int row = y + H * z;
  const int idx = x0 + W * row;
  const bool inlet0 = x0 == 0;
  const bool outlet1 = OUT && x0 + 1 == W - 1;
  const long long WH = (long long)W * H;
  // the pulls go out before the body-row test, so they do not wait for it (every pull address is
  // inside the source buffer; a pair of body cells discards them)
  typename C::Pair r[Q3];  // populations of the pair: x0 in the low half (.x), x0 + 1 in the high half
#pragma unroll
  for (int i = 0; i < Q3; i++) {
    const S* p = (FACE ? a.fpull[side][i] : a.pull[i]) + idx;
    if (cx3(i) == 0) {
      r[i] = C::ld_pair(p);
    } else {
      int e1 = 1;
      // outlet: zero-gradient copy from (W-2, y, z) for the directions entering through x = W-1
      if (cx3(i) == -1 && outlet1) e1 = FACE ? a.fout[side][i] : (int)(-1 + cy3(i) * (long long)W + cz3(i) * WH);
      r[i] = C::ld_pair2(p, p + e1);
    }
  }
  bool act0 = true, act1 = true;
  if (a.rowBody[row]) {
    act0 = __ldg(a.flags + idx) == 0u;
    act1 = __ldg(a.flags + idx + 1) == 0u;
    if (!act0 && !act1) return;
  }
  if constexpr (!kExact) {
    // fast arithmetic: both cells through the packed f32x2 collision; a pair with one body cell
    // takes the per-cell code below
    if (act0 && act1) {
      // the inlet and outlet tests run per thread (one variant per ABS instead of four)
      collide3x2_store<C, SMAG, ABS, true, true>(a, r, x0, idx);
      return;
    }
  }
  R o0[Q3];
  if (act0) {
    if (inlet0) {
      // inlet: equilibrium at the inflow speed, no collision (step3d.ts:190-193)
      const double* eq = a.st->inletEq[a.par];
#pragma unroll
      for (int i = 0; i < Q3; i++) o0[i] = (R)eq[i];
    } else {
      R f[Q3];
#pragma unroll
      for (int i = 0; i < Q3; i++) f[i] = C::lo(r[i]);
      collide3<C, SMAG, ABS>(a, f, x0, false, o0);
    }
  }
  R o1[Q3];
  if (act1) {
    R f[Q3];
#pragma unroll
    for (int i = 0; i < Q3; i++) f[i] = C::hi(r[i]);
    collide3<C, SMAG, ABS>(a, f, x0 + 1, outlet1, o1);
  }
  if (act0 && act1) {
#pragma unroll
    for (int i = 0; i < Q3; i++)
      kExact ? C::st_pair(a.out[i] + idx, o0[i], o1[i]) : C::st_pair_fast(a.out[i] + idx, o0[i], o1[i]);
  } else if (act0) {
#pragma unroll
    for (int i = 0; i < Q3; i++) a.out[i][idx] = C::enc_raw(o0[i]);
  } else {
#pragma unroll
    for (int i = 0; i < Q3; i++) a.out[i][idx + 1] = C::enc_raw(o1[i]);
  }
}

// The interior pairs of tile (blockIdx.x, blockIdx.y) in plane z = 1 + tz.
template <class C, bool SMAG, bool ABS, bool OUT>
__device__ __forceinline__ void bulk_pair_role(const StepArgs3<C>& a, int tz) {
  const int x0 = blockIdx.x * a.tileTX + 2 * threadIdx.x;
  const int y = 1 + blockIdx.y * a.tileTY + threadIdx.y;
  if (x0 >= a.W || y >= a.H - 1) return;
  pair_cells<C, SMAG, ABS, OUT, false>(a, x0, y, 1 + tz, 0);
}

// Face tile f: the first faceZTiles are the tiles of the z = 0 and z = D-1 planes (rows 1 .. H-2,
// laid out as an interior plane), the others tileTY consecutive planes of the y = 0 / y = H-1 row.
// The absorbing layer and the outlet column are decided per thread.
template <class C, bool SMAG>
__device__ __forceinline__ void face_pair_role(const StepArgs3<C>& a, int f) {
  const int tilesX = (a.W + a.tileTX - 1) / a.tileTX;
  int side, tx, y, z;
  if (f < a.faceZTiles) {
    const int perPlane = a.faceZTiles / 2;
    side = f >= perPlane ? 1 : 0;
    const int rem = f - side * perPlane;
    const int ty = rem / tilesX;
    tx = rem - ty * tilesX;
    y = 1 + ty * a.tileTY + threadIdx.y;
    z = side ? a.D - 1 : 0;
    if (y >= a.H - 1) return;
  } else {
    f -= a.faceZTiles;
    const int perSide = a.faceYGroups * tilesX;
    side = f >= perSide ? 3 : 2;
    const int rem = f - (side - 2) * perSide;
    const int g = rem / tilesX;
    tx = rem - g * tilesX;
    y = side == 3 ? a.H - 1 : 0;
    z = 1 + g * a.tileTY + threadIdx.y;
    if (z >= a.D - 1) return;
  }
  const int x0 = tx * a.tileTX + 2 * threadIdx.x;
  if (x0 >= a.W) return;
  pair_cells<C, SMAG, true, true, true>(a, x0, y, z, side);
}

// Resident blocks per SM the register allocation must allow: 16-bit x-pairs 6 (80 registers;
// measured faster at 6 than at 7, 5 or 4), f32 x-pairs 5 (up to 102 registers, no spills; with
// the L2 prefetch 3.5% faster at 192x96x96 than at 6, where 68 bytes spilled), 8 for one f32 cell
// per thread (odd widths), 4 for f64.
template <class C>
constexpr int step_min_blocks(bool pair) {
  return pair ? (sizeof(typename C::S) == 4 ? 5 : 6) : (sizeof(typename C::R) == 8 ? 4 : 8);
}

// L2 prefetch of the pull sources of the interior tile at the same (x, y) tile position pfPlanes
// z planes later: one thread per 128-byte stretch of each of the tile's rows (2^pfShift stretches
// per row, 2^pfRowShift rows) in each of the 19 source arrays, each addressed at the stretch's
// middle so the pull's one-element x offset still names the stretch's own line. Every address is
// the pull source of an interior cell, inside the source buffer. A hint only: it changes no
// result. (One bulk prefetch per row instead measured 8-10% slower.)
template <class C>
__device__ __forceinline__ void prefetch_tile_ahead(const StepArgs3<C>& a) {
  using S = typename C::S;
  constexpr int kLine = 128;
  const int bz = blockIdx.z + a.pfPlanes;
  if (bz < a.roleZ || bz >= (int)gridDim.z) return;
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int perDir = a.pfRowShift + a.pfShift;  // log2 of the stretches per population
  const long long plane = (long long)a.H * (1 + bz - a.roleZ);
  for (int t = tid; t < (Q3 << perDir); t += kStepThreads) {
    const int i = t >> perDir;
    const int r = (t >> a.pfShift) & ((1 << a.pfRowShift) - 1);
    const int l = t & ((1 << a.pfShift) - 1);
    const int y = 1 + blockIdx.y * a.tileTY + r;
    if (y >= a.H - 1) continue;
    const int x = min((int)blockIdx.x * a.tileTX + l * (kLine / (int)sizeof(S)) + kLine / 2 / (int)sizeof(S), a.W - 2);
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a.pull[i] + (x + (long long)a.W * (y + plane))));
  }
}

template <class C, bool SMAG, bool PAIR>
__global__ void __launch_bounds__(kStepThreads, step_min_blocks<C>(PAIR))
    step3d_kernel(const __grid_constant__ StepArgs3<C> a) {
  // Programmatic dependent launch: the next step's grid may be scheduled once every block of this
  // one has started, so its blocks fill the SMs this grid's tail leaves idle; each of them waits
  // here until the previous grid (launched before it on the stream) has completed and its writes
  // are visible. Launched without the attribute (or after a non-kernel operation) the wait
  // returns at once.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (a.pfPlanes > 0) prefetch_tile_ahead<C>(a);
  // grid (tilesX, tilesY, roleZ + D - 2): the first roleZ slices of blocks hold the face and body
  // roles (dispatched first), the others the interior tiles, one z plane per slice
  if ((int)blockIdx.z < a.roleZ) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int r = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (r == 0 && tid < Q3) {
      // the next step's counter, inlet speed and inlet equilibrium (slot par ^ 1; this step reads par)
      const unsigned s = a.st->step[a.par];
      if (tid == 0) a.st->step[a.par ^ 1] = s + 1u;
      if (a.rampKind != 0) {
        using R = typename C::R;
        const double u = ramp_speed(a.rampKind, a.rampTarget, a.rampSteps, a.rampEvery, s + 1u);
        if (tid == 0) a.st->uIn[a.par ^ 1] = u;
        a.st->inletEq[a.par ^ 1][tid] = (double)feq3s<C>(tid, R(1), (R)u, R(0), R(0));
      }
    }
    if (r < a.shellBlocks)
      shell_role<C, SMAG>(a, r, tid);
    else if (r < a.shellBlocks + a.bodyBlocks)
      body_role<C, SMAG>(a, r - a.shellBlocks, tid);
    else if constexpr (PAIR) {
      if (r < a.shellBlocks + a.bodyBlocks + a.faceBlocks) face_pair_role<C, SMAG>(a, r - a.shellBlocks - a.bodyBlocks);
    }
    return;
  }
  // block-uniform choice of the code for tiles that overlap the absorbing layer or hold the outlet
  const int tx1 = (blockIdx.x + 1) * a.tileTX;  // end of the tile's x range
  const bool abs = tx1 > a.absorbX0, out = tx1 >= a.W;
  const int tz = blockIdx.z - a.roleZ;
  if constexpr (PAIR) {
    if (out)
      abs ? bulk_pair_role<C, SMAG, true, true>(a, tz) : bulk_pair_role<C, SMAG, false, true>(a, tz);
    else
      abs ? bulk_pair_role<C, SMAG, true, false>(a, tz) : bulk_pair_role<C, SMAG, false, false>(a, tz);
  } else {
    if (out)
      abs ? bulk_role<C, SMAG, true, true>(a, tz) : bulk_role<C, SMAG, false, true>(a, tz);
    else
      abs ? bulk_role<C, SMAG, true, false>(a, tz) : bulk_role<C, SMAG, false, false>(a, tz);
  }
}

// ---------------- host-side launcher ----------------

template <class C>
static cudaError_t launch_step3_t(const StepLaunch3& L, cudaStream_t s) {
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
  // the pair layout follows the W per-x entries in the same buffer (f32 rates only)
  a.xPair = sizeof(R) == 4 ? (const float4*)((const float*)L.xTab + 4 * (size_t)L.W) : nullptr;
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
  a.absorbX0 = L.absorbX0;
  // work split
  const bool pair = sizeof(S) <= 4 && (L.W % 2) == 0 && L.tileTX >= 64 && L.pairTiles;
  if (!pair && L.tileTX > kStepThreads) return cudaErrorInvalidValue;
  a.tileTX = L.tileTX;
  a.tileTY = L.tileTY;
  const int tilesX = (L.W + L.tileTX - 1) / L.tileTX;
  const int tilesY = L.H > 2 ? (L.H - 2 + L.tileTY - 1) / L.tileTY : 1;
  const int zInterior = (L.H > 2 && L.D > 2) ? L.D - 2 : 0;
  const int perSlice = tilesX * tilesY;
  // the face rows with one outside side as x-pair tiles (the 16-bit face code spent about 10% of
  // the step on 4% of the cells); the outlet offsets must fit an int
  a.facePairs = (pair && L.H >= 3 && L.D >= 3 && 19LL * L.N < (1LL << 31)) ? 1 : 0;
  a.faceZTiles = a.facePairs ? 2 * tilesX * tilesY : 0;
  a.faceYGroups = a.facePairs ? (L.D - 2 + L.tileTY - 1) / L.tileTY : 0;
  a.faceBlocks = a.facePairs ? a.faceZTiles + 2 * a.faceYGroups * tilesX : 0;
  for (int side = 0; side < 4; side++) {
    for (int i = 0; i < Q3; i++) {
      // the slip face's specular reflection for the directions that enter from outside: the
      // mirrored population from the same z plane (sides 0, 1) or the same y row (sides 2, 3)
      const bool out = side == 0 ? cz3(i) == 1 : (side == 1 ? cz3(i) == -1 : (side == 2 ? cy3(i) == 1 : cy3(i) == -1));
      const int pop = !out ? i : (side < 2 ? mirror_z3(i) : mirror_y3(i));
      const long long off = !out ? cx3(i) + cy3(i) * W + cz3(i) * WH
                                 : (side < 2 ? cx3(i) + cy3(i) * W : cx3(i) + cz3(i) * WH);
      const long long base = (long long)pop * L.N - off;
      a.fpull[side][i] = (const S*)((uintptr_t)a.src + (intptr_t)(base * (long long)sizeof(S)));
      // the outlet copy's source of the pair's second cell, population i at (W-2, y, z), relative
      // to its pull address
      a.fout[side][i] = (int)((long long)i * L.N - base);
    }
  }
  const long long nShell = a.facePairs ? 4LL * L.W : shell_cells3(L.W, L.H, L.D);
  a.shellBlocks = (int)((nShell + kStepThreads - 1) / kStepThreads);
  // the body role runs when there are body cells, and on sampled steps even without them (a
  // sample of zero force is still written to the ring, as the reference's reduce pass does)
  a.bodyBlocks = (L.nBody > 0 || L.sample) ? body_blocks3(L.nBody) : 0;
  a.roleZ = (a.shellBlocks + a.bodyBlocks + a.faceBlocks + perSlice - 1) / perSlice;
  const dim3 grid(tilesX, tilesY, a.roleZ + zInterior);
  // prefetch distance, measured on B200 at 192x96x96 and 256x128x128 (sphere tunnel, 1000 steps):
  // 16-bit storage 4 planes (+1.5-3% and +6.5-8%), f32 1 plane (+0.5-1.5%), f64 the plane count
  // nearest 270 tiles (+5% and +2%); farther prefetches lost to the demand loads
  a.pfShift = 0;
  while ((128 << a.pfShift) < a.tileTX * (int)sizeof(S)) a.pfShift++;  // 2^shift lines hold a tile row
  a.pfRowShift = 0;
  while ((1 << a.pfRowShift) < a.tileTY) a.pfRowShift++;  // tileTY = 128 / block width, a power of two
  if (sizeof(S) == 2)
    a.pfPlanes = 4;
  else if (sizeof(S) == 4)
    a.pfPlanes = 1;
  else
    a.pfPlanes = std::max(1, (270 + perSlice / 2) / perSlice);
  const dim3 block(pair ? L.tileTX / 2 : L.tileTX, kStepThreads / (pair ? L.tileTX / 2 : L.tileTX), 1);
  const bool smag = L.smagC2 > 0;
  void (*fn)(StepArgs3<C>) = nullptr;
  if (pair) {
    if constexpr (sizeof(S) <= 4) fn = smag ? step3d_kernel<C, true, true> : step3d_kernel<C, false, true>;
  } else {
    fn = smag ? step3d_kernel<C, true, false> : step3d_kernel<C, false, false>;
  }
  if (!fn) return cudaErrorInvalidValue;
  // launched with programmatic stream serialisation: consecutive steps on a stream (and in the
  // captured step graphs) overlap one grid's launch with the previous grid's tail
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, fn, a);
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

int body_blocks3(int nBody) { return nBody > 0 ? (nBody + 31) / 32 : 1; }

}  // namespace CELLS_ARITH
}  // namespace cells
