// CPU restatement of the reference D2Q9 step path — TEST INFRASTRUCTURE ONLY.
//
// The oracle that the CUDA 2D kernels in cells_b200/csrc are checked against. Only the tests, the
// smoke check and the CPU-baseline leg of the benchmark load it; the product library never links
// or calls it.
//
// It restates, in the same order of floating-point operations, the WGSL that slowernet/cells
// generates at run time for its 2D solver:
//   src/lattice.ts:2-33            D2Q9 velocity set, OPP, MIRROR_Y, PAIRS, modes, flag bits
//   src/shaders/common.ts:10-57    Params, inletVelocity (parabolic profile), wrapPeriodic
//   src/shaders/step.ts:9-229      fused pull-stream + boundaries + Zou-He + TRT collide (+ pullSlow)
//   src/shaders/aux.ts:14-194      feq, flags + refill, init, macro, force reduce, brush
// Storage: f32 (the reference) and f64 (f64 arithmetic; the GPU FP64 run's second reference).
//
// Parity status: the reference has no golden vectors for step results. The 2D restatement is
// pinned end to end by the reference's own physics acceptance tests (src/cases.ts: Poiseuille L2
// error below 2e-4, Taylor-Green viscosity within 1%), run on this oracle by the CPU test suite.
//
// Build: oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

constexpr int Q = 9;
// src/lattice.ts:2-7
constexpr int CX[Q] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
constexpr int CY[Q] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
constexpr int OPP[Q] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
constexpr int MIRROR_Y[Q] = {0, 1, 4, 3, 2, 8, 7, 6, 5};
constexpr int PAIRS[4][2] = {{1, 3}, {2, 4}, {5, 7}, {6, 8}};  // src/lattice.ts:10-15
// src/lattice.ts:29-32
constexpr uint32_t FLAG_SOLID = 1u << 9;
constexpr uint32_t FLAG_INLET = 1u << 10;
constexpr uint32_t FLAG_OUTLET = 1u << 11;
constexpr int BIDX_SHIFT = 12;
// XMode / YMode, src/lattice.ts:17-27
constexpr int X_PERIODIC = 0, X_OPEN = 2;  // X_WALL = 1 needs no test: it falls through to bounce-back
constexpr int Y_PERIODIC = 0, Y_SLIP = 2, Y_MOVING = 3;  // Y_NOSLIP = 1 likewise

struct CodecF32 {
  using S = float;
  using R = float;
  static R load(S v) { return v; }
  static S store(R v) { return v; }
};
struct CodecF64 {
  using S = double;
  using R = double;
  static R load(S v) { return v; }
  static S store(R v) { return v; }
};

// The weights as WGSL literals of the JS doubles 4/9, 1/9, 1/36 (src/lattice.ts:4), rounded to R.
template <class R>
R wt(int i) {
  return i == 0 ? (R)(4.0 / 9.0) : (i <= 4 ? (R)(1.0 / 9.0) : (R)(1.0 / 36.0));
}

}  // namespace

// Params (src/shaders/common.ts:14-22) as the host derives it (src/solver.ts:180-197), with the
// float fields in double; the oracle rounds each once into the arithmetic type.
struct HostParams2 {
  int32_t W, H;
  int32_t left, right, bottom, top;
  int32_t parabolic, forcing;
  double tau, lambda, smagC2, uIn, spongeStart, tauSponge, uLid, fx, fy, absorb, inletLayer;
};

namespace {

template <class R>
struct P2 {
  int W, H, N;
  int left, right, bottom, top, parabolic, forcing;
  R tau, lambda, smagC2, uIn, spongeStart, tauSponge, uLid, fx, fy, absorb, inletLayer;
};

template <class R>
P2<R> toP2(const HostParams2* h) {
  P2<R> p;
  p.W = h->W;
  p.H = h->H;
  p.N = h->W * h->H;
  p.left = h->left;
  p.right = h->right;
  p.bottom = h->bottom;
  p.top = h->top;
  p.parabolic = h->parabolic;
  p.forcing = h->forcing;
  p.tau = (R)h->tau;
  p.lambda = (R)h->lambda;
  p.smagC2 = (R)h->smagC2;
  p.uIn = (R)h->uIn;
  p.spongeStart = (R)h->spongeStart;
  p.tauSponge = (R)h->tauSponge;
  p.uLid = (R)h->uLid;
  p.fx = (R)h->fx;
  p.fy = (R)h->fy;
  p.absorb = (R)h->absorb;
  p.inletLayer = (R)h->inletLayer;
  return p;
}

template <class R>
R clampR(R v, R lo, R hi) { return std::min(std::max(v, lo), hi); }
template <class R>
R smoothstepR(R e0, R e1, R x) {
  R t = clampR<R>((x - e0) / (e1 - e0), R(0), R(1));
  return t * t * (R(3) - R(2) * t);
}
template <class R>
R mixR(R a, R b, R t) { return a * (R(1) - t) + b * t; }

// feq, shifted by w_i (src/shaders/aux.ts:14-19)
template <class R>
R feq2(int i, R rho, R ux, R uy) {
  R cu = R(3) * (R(CX[i]) * ux + R(CY[i]) * uy);
  return wt<R>(i) * (rho - R(1) + rho * (cu + R(0.5) * cu * cu - R(1.5) * (ux * ux + uy * uy)));
}

// inletVelocity, src/shaders/common.ts:39-45
template <class R>
R inletVelocity(const P2<R>& P, int y) {
  if (P.parabolic == 0) return P.uIn;
  const R h = R(P.H);
  const R s = R(y) + R(0.5);
  return R(4) * P.uIn * s * (h - s) / (h * h);
}

// wrapPeriodic, src/shaders/common.ts:48-57
template <class R>
void wrapPeriodic(const P2<R>& P, int& x, int& y) {
  if (x < 0 && P.left == X_PERIODIC) x += P.W;
  if (x >= P.W && P.right == X_PERIODIC) x -= P.W;
  if (y < 0 && P.bottom == Y_PERIODIC) y += P.H;
  if (y >= P.H && P.top == Y_PERIODIC) y -= P.H;
}

template <class C>
struct Step2 {
  using S = typename C::S;
  using R = typename C::R;
  const P2<R>& P;
  const S* src;
  S* dst;
  const uint32_t* flags;
  const float* sdf;

  R ld(size_t k) const { return C::load(src[k]); }
  void st(size_t k, R v) const { dst[k] = C::store(v); }
  bool isSolid(size_t s) const { return (flags[s] & FLAG_SOLID) != 0u; }

  // pullSlow, src/shaders/step.ts:119-175
  R pullSlow(int i, int x, int y, size_t idx, uint32_t fl, R force[2]) const {
    const size_t N = (size_t)P.N;
    const int W = P.W, H = P.H;
    const int j = OPP[i];
    int sx = x - CX[i];
    int sy = y - CY[i];
    if ((fl & (1u << i)) == 0u) return ld(i * N + (size_t)(sy * W + sx));
    wrapPeriodic(P, sx, sy);
    const bool inX = sx >= 0 && sx < W;
    const bool inY = sy >= 0 && sy < H;
    if (inX && inY) {
      const size_t s = (size_t)(sy * W + sx);
      if (!isSolid(s)) return ld(i * N + s);
      const R fj = ld(j * N + idx);
      const R dF = (R)sdf[idx];
      const R dS = (R)sdf[s];
      const R q = clampR<R>(dF / std::max(dF - dS, (R)1e-6), (R)1e-3, R(1));
      R fi = fj;
      if (q < R(0.5)) {
        int nx = x + CX[i], ny = y + CY[i];
        wrapPeriodic(P, nx, ny);
        if (nx >= 0 && nx < W && ny >= 0 && ny < H) {
          const size_t n = (size_t)(ny * W + nx);
          if (!isSolid(n)) fi = R(2) * q * fj + (R(1) - R(2) * q) * ld(j * N + n);
        }
      } else {
        fi = fj / (R(2) * q) + (R(2) * q - R(1)) / (R(2) * q) * ld(i * N + idx);
      }
      const R t = fj + fi;
      force[0] += R(CX[j]) * t;
      force[1] += R(CY[j]) * t;
      return fi;
    }
    if (!inY) {
      const int mode = sy < 0 ? P.bottom : P.top;
      if (mode == Y_SLIP) {
        const int rx = std::min(std::max(sx, 0), W - 1);
        return ld(MIRROR_Y[i] * N + (size_t)y * W + rx);
      }
      if (mode == Y_MOVING) return ld(j * N + idx) + R(6) * wt<R>(i) * R(CX[i]) * P.uLid;
      return ld(j * N + idx);
    }
    // walls, and placeholders that the open-boundary fix-up overwrites
    return ld(j * N + idx);
  }

  // main, src/shaders/step.ts:177-227. Returns true when the cell has a force slot; its
  // momentum-exchange force is then in force[0..1].
  bool cell(int x, int y, R force[2]) const {
    const size_t N = (size_t)P.N;
    const size_t idx = (size_t)y * P.W + x;
    const uint32_t fl = flags[idx];
    R f[Q];
    bool slot = false;
    if (fl == 0u) {
      for (int i = 0; i < Q; i++) f[i] = ld(i * N + (size_t)((y - CY[i]) * P.W + (x - CX[i])));
    } else {
      if (fl & FLAG_SOLID) return false;
      f[0] = ld(idx);
      for (int i = 1; i < Q; i++) f[i] = pullSlow(i, x, y, idx, fl, force);
      slot = (fl >> BIDX_SHIFT) != 0u;
      // Zou-He (populations stored shifted by w_i)
      if (fl & FLAG_INLET) {
        const R u = inletVelocity(P, y);
        const R r = (R(1) + f[0] + f[2] + f[4] + R(2) * (f[3] + f[6] + f[7])) / (R(1) - u);
        f[1] = f[3] + (R)(2.0 / 3.0) * r * u;
        f[5] = f[7] - R(0.5) * (f[2] - f[4]) + (R)(1.0 / 6.0) * r * u;
        f[8] = f[6] + R(0.5) * (f[2] - f[4]) + (R)(1.0 / 6.0) * r * u;
      } else if (fl & FLAG_OUTLET) {
        const R u = f[0] + f[2] + f[4] + R(2) * (f[1] + f[5] + f[8]);
        f[3] = f[1] - (R)(2.0 / 3.0) * u;
        f[7] = f[5] + R(0.5) * (f[2] - f[4]) - (R)(1.0 / 6.0) * u;
        f[6] = f[8] - R(0.5) * (f[2] - f[4]) - (R)(1.0 / 6.0) * u;
      }
    }
    // moments (src/shaders/step.ts:22-32)
    const R drho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    const R rho = R(1) + drho;
    const R invRho = R(1) / rho;
    R ux = (f[1] - f[3] + f[5] - f[6] - f[7] + f[8]) * invRho;
    R uy = (f[2] - f[4] + f[5] + f[6] - f[7] - f[8]) * invRho;
    if (P.forcing != 0) {
      ux += R(0.5) * P.fx * invRho;
      uy += R(0.5) * P.fy * invRho;
    }
    const R usq = R(1.5) * (ux * ux + uy * uy);
    // cu_a for the lower member of each pair (src/shaders/step.ts:34-40)
    R cu[Q] = {};
    cu[1] = R(3) * (ux);
    cu[2] = R(3) * (uy);
    cu[5] = R(3) * (ux + uy);
    cu[6] = R(3) * (-ux + uy);
    R eqS[Q] = {}, eqA[Q] = {};
    for (const auto& pr : PAIRS) {
      const int a = pr[0];
      eqS[a] = wt<R>(a) * (drho + rho * (R(0.5) * cu[a] * cu[a] - usq));
      eqA[a] = wt<R>(a) * rho * cu[a];
    }
    // sponge and absorbing layers (src/shaders/step.ts:215-223)
    R omegaBase = R(1) / P.tau;
    R sOut = R(0);
    if (P.spongeStart < R(P.W - 1)) {
      sOut = smoothstepR<R>(P.spongeStart, R(P.W - 1), R(x));
      omegaBase = R(1) / mixR<R>(P.tau, P.tauSponge, sOut);
    }
    R sIn = R(0);
    if (P.inletLayer > R(0)) sIn = R(1) - smoothstepR<R>(R(0), P.inletLayer, R(x));
    const R sigma = P.absorb * std::max(sOut * sOut, sIn * sIn);
    // Smagorinsky (src/shaders/step.ts:48-63)
    R omP = omegaBase;
    if (P.smagC2 > R(0)) {
      R n[Q];
      for (const auto& pr : PAIRS) {
        const int a = pr[0], b = pr[1];
        n[a] = f[a] - (eqS[a] + eqA[a]);
        n[b] = f[b] - (eqS[a] - eqA[a]);
      }
      const R pxx = n[1] + n[3] + n[5] + n[6] + n[7] + n[8];
      const R pyy = n[2] + n[4] + n[5] + n[6] + n[7] + n[8];
      const R pxy = n[5] - n[6] + n[7] - n[8];
      const R pi = std::sqrt(pxx * pxx + pyy * pyy + R(2) * pxy * pxy);
      const R t0 = R(1) / omegaBase;
      const R tEff = R(0.5) * (t0 + std::sqrt(t0 * t0 + (R)25.45584412271571 * P.smagC2 * pi * invRho));
      omP = R(1) / tEff;
    }
    const R omM = R(1) / (R(0.5) + P.lambda / (R(1) / omP - R(0.5)));
    // absorbing-layer and Guo body-force sources (src/shaders/step.ts:65-91)
    R s0 = R(0);
    R sS[Q] = {}, sA[Q] = {};
    if (sigma > R(0)) {
      const R ut = inletVelocity(P, y);
      const R dq = R(1.5) * rho * (ut * ut - ux * ux - uy * uy);
      s0 += sigma * wt<R>(0) * -dq;
      for (const auto& pr : PAIRS) {
        const int a = pr[0];
        const R cut = R(3) * R(CX[a]) * ut;
        sS[a] += sigma * wt<R>(a) * (R(0.5) * rho * (cut * cut - cu[a] * cu[a]) - dq);
        sA[a] += sigma * wt<R>(a) * rho * (cut - cu[a]);
      }
    }
    if (P.forcing != 0) {
      const R uF = ux * P.fx + uy * P.fy;
      s0 += (R(1) - R(0.5) * omP) * wt<R>(0) * (R(-3) * uF);
      for (const auto& pr : PAIRS) {
        const int a = pr[0];
        const R cF = (R(CX[a]) * P.fx + R(CY[a]) * P.fy);
        sS[a] += (R(1) - R(0.5) * omP) * wt<R>(a) * (R(-3) * uF + R(9) * (cu[a] / R(3)) * cF);
        sA[a] += (R(1) - R(0.5) * omM) * wt<R>(a) * R(3) * cF;
      }
    }
    // TRT collide + store (src/shaders/step.ts:93-103)
    st(idx, f[0] - omP * (f[0] - wt<R>(0) * (drho - rho * usq)) + s0);
    for (const auto& pr : PAIRS) {
      const int a = pr[0], b = pr[1];
      const R sym = omP * (R(0.5) * (f[a] + f[b]) - eqS[a]);
      const R asym = omM * (R(0.5) * (f[a] - f[b]) - eqA[a]);
      st(a * N + idx, f[a] - sym - asym + sS[a] + sA[a]);
      st(b * N + idx, f[b] - sym + asym + sS[a] - sA[a]);
    }
    return slot;
  }
};

template <class C>
void step2(const HostParams2* hp, const void* src, void* dst, const uint32_t* flags, const float* sdf,
           double* cellForce) {
  using R = typename C::R;
  const P2<R> P = toP2<R>(hp);
  Step2<C> k{P, (const typename C::S*)src, (typename C::S*)dst, flags, sdf};
#pragma omp parallel for schedule(static)
  for (int y = 0; y < P.H; y++)
    for (int x = 0; x < P.W; x++) {
      R force[2] = {R(0), R(0)};
      const bool slot = k.cell(x, y, force);
      if (cellForce) {
        const size_t idx = (size_t)y * P.W + x;
        cellForce[2 * idx + 0] = slot ? (double)force[0] : 0.0;
        cellForce[2 * idx + 1] = slot ? (double)force[1] : 0.0;
      }
    }
}

// flagsShader, src/shaders/aux.ts:22-88. Force slots are numbered in cell order (the reference
// numbers them in atomic order; only their existence matters to the step).
template <class C>
void flags2(const HostParams2* hp, const float* sdf, uint32_t* flags, void* fA, void* fB, const float* mac) {
  using R = typename C::R;
  using S = typename C::S;
  const P2<R> P = toP2<R>(hp);
  const int W = P.W, H = P.H;
  const size_t N = (size_t)P.N;
  auto solidAt = [&](int x, int y) {
    const bool open = (P.left == X_OPEN && x == 0) || (P.right == X_OPEN && x == W - 1);
    return !open && sdf[(size_t)y * W + x] < 0.0f;
  };
  uint32_t counter = 0;
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      const size_t idx = (size_t)y * W + x;
      const uint32_t old = flags[idx];
      if (solidAt(x, y)) {
        flags[idx] = FLAG_SOLID;
        continue;
      }
      uint32_t bits = 0;
      if (P.left == X_OPEN && x == 0) bits = FLAG_INLET;
      if (P.right == X_OPEN && x == W - 1) bits = FLAG_OUTLET;
      bool touchesBody = false;
      for (int i = 1; i < Q; i++) {
        int sx = x - CX[i], sy = y - CY[i];
        wrapPeriodic(P, sx, sy);
        const bool inside = sx >= 0 && sy >= 0 && sx < W && sy < H;
        if (inside && solidAt(sx, sy)) {
          bits |= 1u << i;
          touchesBody = true;
        } else if (!inside || sx != x - CX[i] || sy != y - CY[i]) {
          bits |= 1u << i;
        }
      }
      if (touchesBody) {
        const uint32_t slot = ++counter;
        if (slot < (1u << (32 - BIDX_SHIFT))) bits |= slot << BIDX_SHIFT;
      }
      flags[idx] = bits;
      if ((old & FLAG_SOLID) != 0u) {
        // refill from the fluid neighbours' macro values (rho, ux, uy, solid)
        R rho = R(0), u[2] = {R(0), R(0)}, n = R(0);
        for (int i = 1; i < Q; i++) {
          const int sx = x + CX[i], sy = y + CY[i];
          if (sx < 0 || sy < 0 || sx >= W || sy >= H) continue;
          const float* m = mac + 4 * ((size_t)sy * W + sx);
          if (m[3] == 0.0f) {
            rho += (R)m[0];
            u[0] += (R)m[1];
            u[1] += (R)m[2];
            n += R(1);
          }
        }
        if (n > R(0)) {
          rho /= n;
          u[0] /= n;
          u[1] /= n;
        } else {
          rho = R(1);
        }
        for (int i = 0; i < Q; i++) {
          const S v = C::store(feq2<R>(i, rho, u[0], u[1]));
          ((S*)fA)[i * N + idx] = v;
          ((S*)fB)[i * N + idx] = v;
        }
      }
    }
}

// initShader, src/shaders/aux.ts:92-111: both buffers to feq(rho, ux, uy) of mac (rho, ux, uy, _).
template <class C>
void init2(const HostParams2* hp, const float* mac, void* fA, void* fB) {
  using R = typename C::R;
  using S = typename C::S;
  const size_t N = (size_t)hp->W * hp->H;
#pragma omp parallel for schedule(static)
  for (long long idx = 0; idx < (long long)N; idx++) {
    const float* m = mac + 4 * idx;
    for (int i = 0; i < Q; i++) {
      const S v = C::store(feq2<R>(i, (R)m[0], (R)m[1], (R)m[2]));
      ((S*)fA)[i * N + idx] = v;
      ((S*)fB)[i * N + idx] = v;
    }
  }
}

// macroShader, src/shaders/aux.ts:115-140: (rho, ux, uy, 0), solids (1, 0, 0, 1); with a body force
// the momentum loses half the force (the stored populations carry the full impulse).
template <class C>
void macro2(const HostParams2* hp, const void* f, const uint32_t* flags, float* mac) {
  using R = typename C::R;
  using S = typename C::S;
  const P2<R> P = toP2<R>(hp);
  const size_t N = (size_t)P.N;
#pragma omp parallel for schedule(static)
  for (long long idx = 0; idx < (long long)N; idx++) {
    float* m = mac + 4 * idx;
    if (flags[idx] & FLAG_SOLID) {
      m[0] = 1.0f;
      m[1] = m[2] = 0.0f;
      m[3] = 1.0f;
      continue;
    }
    R v[Q];
    for (int i = 0; i < Q; i++) v[i] = C::load(((const S*)f)[i * N + idx]);
    const R rho = R(1) + v[0] + v[1] + v[2] + v[3] + v[4] + v[5] + v[6] + v[7] + v[8];
    R jx = v[1] - v[3] + v[5] - v[6] - v[7] + v[8];
    R jy = v[2] - v[4] + v[5] + v[6] - v[7] - v[8];
    if (P.forcing != 0) {
      jx -= R(0.5) * P.fx;
      jy -= R(0.5) * P.fy;
    }
    m[0] = (float)rho;
    m[1] = (float)(jx / rho);
    m[2] = (float)(jy / rho);
    m[3] = 0.0f;
  }
}

template <class C>
double mass2(const HostParams2* hp, const void* f, const uint32_t* flags) {
  using S = typename C::S;
  const size_t N = (size_t)hp->W * hp->H;
  double total = 0.0;
  for (size_t idx = 0; idx < N; idx++) {
    if (flags[idx] & FLAG_SOLID) continue;
    double drho = 0.0;
    for (int i = 0; i < Q; i++) drho += (double)C::load(((const S*)f)[i * N + idx]);
    total += 1.0 + drho;
  }
  return total;
}

}  // namespace

extern "C" {

#define ORACLE2_DISPATCH(prec, call)              \
  switch (prec) {                                \
    case 0: { using C = CodecF32; call; break; } \
    case 3: { using C = CodecF64; call; break; } \
    default: return -1;                          \
  }

int oracle2d_step(int precision, const HostParams2* p, const void* src, void* dst, const uint32_t* flags,
                  const float* sdf, double* cellForce) {
  ORACLE2_DISPATCH(precision, (step2<C>(p, src, dst, flags, sdf, cellForce)));
  return 0;
}

// n steps without force sampling, alternating A and B from parity par; returns the final parity.
int oracle2d_run(int precision, const HostParams2* p, void* fA, void* fB, int par, long long n,
                 const uint32_t* flags, const float* sdf) {
  for (long long k = 0; k < n; k++) {
    void* src = par ? fB : fA;
    void* dst = par ? fA : fB;
    ORACLE2_DISPATCH(precision, (step2<C>(p, src, dst, flags, sdf, nullptr)));
    par ^= 1;
  }
  return par;
}

int oracle2d_flags(int precision, const HostParams2* p, const float* sdf, uint32_t* flags, void* fA, void* fB,
                   const float* mac) {
  ORACLE2_DISPATCH(precision, (flags2<C>(p, sdf, flags, fA, fB, mac)));
  return 0;
}

int oracle2d_init(int precision, const HostParams2* p, const float* mac, void* fA, void* fB) {
  ORACLE2_DISPATCH(precision, (init2<C>(p, mac, fA, fB)));
  return 0;
}

int oracle2d_macro(int precision, const HostParams2* p, const void* f, const uint32_t* flags, float* mac) {
  ORACLE2_DISPATCH(precision, (macro2<C>(p, f, flags, mac)));
  return 0;
}

int oracle2d_mass(int precision, const HostParams2* p, const void* f, const uint32_t* flags, double* out) {
  ORACLE2_DISPATCH(precision, (*out = mass2<C>(p, f, flags)));
  return 0;
}

// brushShader, src/shaders/aux.ts:177-194, over the box Solver.brush derives (src/solver.ts:249-258):
// the SDF unions (erase = 0) or subtracts (erase = 1) a disc of radius r at (cx, cy).
int oracle2d_brush(int W, int H, float* sdf, double cx, double cy, double r, int erase) {
  const int pad = 2;
  const int x0 = std::max(0, (int)std::floor(cx - r - pad));
  const int y0 = std::max(0, (int)std::floor(cy - r - pad));
  const int x1 = std::min(W - 1, (int)std::ceil(cx + r + pad));
  const int y1 = std::min(H - 1, (int)std::ceil(cy + r + pad));
  if (x1 < x0 || y1 < y0) return 0;
  const float fcx = (float)cx, fcy = (float)cy, fr = (float)r;
  for (int y = y0; y <= y1; y++)
    for (int x = x0; x <= x1; x++) {
      const float dx = (float)x - fcx, dy = (float)y - fcy;
      const float d = std::sqrt(dx * dx + dy * dy) - fr;
      float& s = sdf[(size_t)y * W + x];
      s = erase == 0 ? std::min(s, d) : std::max(s, -d);
    }
  return 0;
}

}  // extern "C"
