// CPU restatement of the reference D3Q19 step path — TEST INFRASTRUCTURE ONLY.
//
// This file is the oracle that the CUDA kernels in cells_b200/csrc are checked against. Only the
// tests, the smoke check and the CPU-baseline leg of the benchmark load it; the product library
// never links or calls it.
//
// It restates, in the same order of floating-point operations, the WGSL that slowernet/cells
// generates at run time:
//   src/shaders/common3d.ts:9-63   Params3, feq (shifted equilibrium), storage codec
//   src/shaders/step3d.ts:24-225   fused pull-stream + boundaries + TRT collide (+ pullSlow3)
//   src/shaders/aux3d.ts:20-182    flags + refill, init, macro, force reduce
//   src/lattice3d.ts:4-31          D3Q19 velocity set, OPP, MIRROR_Y/Z, PAIRS, flag bits
// Storage variants: f32 (reference), f16 scaled by 2^15 with the +-1.99 clamp (reference), and two
// variants the reference lacks: bf16 (unscaled, round-to-nearest-even) and f64 (f64 arithmetic).
//
// Parity status: the reference has no golden vectors for step results (it only runs in a browser
// WebGPU device), so bit-level step parity is unpinned by the reference itself. The pieces the
// reference's own unit tests do pin (lattice tables, trtLambda3, equilibrium moments, geometry,
// params semantics) are checked in tests/test_oracle_known_answers.py, and the 2D restatement is
// checked against the reference's own physics acceptance ranges (Poiseuille, Taylor-Green).
//
// Build: oracle/Makefile (g++ -O2 -fopenmp -ffp-contract=off). No FMA contraction, so every f32
// operation rounds exactly as the WGSL source states it.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

constexpr int Q = 19;
// src/lattice3d.ts:4-6 — odd i and i+1 are opposite and form TRT pairs.
constexpr int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0};
constexpr int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1};
constexpr int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1};
// src/lattice3d.ts:19-26
constexpr uint32_t FLAG_SOLID = 1u << 19;
constexpr uint32_t FLAG_INLET = 1u << 20;
constexpr uint32_t FLAG_OUTLET = 1u << 21;

int opp(int i) { return i == 0 ? 0 : (i % 2 ? i + 1 : i - 1); }  // src/lattice3d.ts:9
int find_dir(int cx, int cy, int cz) {
  for (int i = 0; i < Q; i++)
    if (CX[i] == cx && CY[i] == cy && CZ[i] == cz) return i;
  return -1;
}
int mirror_y(int i) { return find_dir(CX[i], -CY[i], CZ[i]); }  // src/lattice3d.ts:17
int mirror_z(int i) { return find_dir(CX[i], CY[i], -CZ[i]); }  // src/lattice3d.ts:19

// ---- storage codecs (src/shaders/common3d.ts:52-63) ----
struct CodecF32 {
  using S = float;
  using R = float;
  static R load(S v) { return v; }
  static S store(R v) { return v; }
};
struct CodecF16 {
  using S = _Float16;
  using R = float;
  static R load(S v) { return (float)v * (1.0f / 32768.0f); }
  // clamp(v, -1.99, 1.99) = min(max(v, lo), hi); f16() rounds to nearest even.
  static S store(R v) {
    float c = std::min(std::max(v, -1.99f), 1.99f);
    return (_Float16)(c * 32768.0f);
  }
};
// bf16 (not in the reference): the top 16 bits of the f32 pattern, rounded to nearest even.
struct CodecBF16 {
  using S = uint16_t;
  using R = float;
  static R load(S v) {
    uint32_t u = (uint32_t)v << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  }
  static S store(R v) {
    uint32_t u;
    std::memcpy(&u, &v, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);  // quiet NaN
    uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
  }
};
struct CodecF64 {
  using S = double;
  using R = double;
  static R load(S v) { return v; }
  static S store(R v) { return v; }
};

// Params3 (src/shaders/common3d.ts:9-16) with its float fields in the arithmetic type R. The host
// computes every derived field in double (as the reference's writeParams does in JS numbers,
// src/solver3d.ts:197-208) and the value is rounded once into R.
template <class R>
struct P3 {
  int W, H, D, N;
  R tau, lambda, smagC2, uIn, spongeStart, tauSponge, absorb;
};

template <class R>
R wt(int i) {
  // 1/3, 1/18, 1/36 rounded to R (src/lattice3d.ts:8)
  return i == 0 ? R(1) / R(3) : (i <= 6 ? R(1) / R(18) : R(1) / R(36));
}

// feq, shifted by w_i (src/shaders/common3d.ts:38-41)
template <class R>
R feq(int i, R rho, R ux, R uy, R uz) {
  R cu = R(3) * (R(CX[i]) * ux + R(CY[i]) * uy + R(CZ[i]) * uz);
  return wt<R>(i) * (rho - R(1) + rho * (cu + R(0.5) * cu * cu - R(1.5) * (ux * ux + uy * uy + uz * uz)));
}

template <class R>
R clampR(R v, R lo, R hi) { return std::min(std::max(v, lo), hi); }

// WGSL smoothstep(low, high, x): t = clamp((x - low) / (high - low), 0, 1); t * t * (3 - 2 t)
template <class R>
R smoothstepR(R e0, R e1, R x) {
  R t = clampR<R>((x - e0) / (e1 - e0), R(0), R(1));
  return t * t * (R(3) - R(2) * t);
}
// WGSL mix(a, b, t) = a * (1 - t) + b * t
template <class R>
R mixR(R a, R b, R t) { return a * (R(1) - t) + b * t; }

template <class C>
struct Step3 {
  using S = typename C::S;
  using R = typename C::R;
  const P3<R>& P;
  const S* src;
  S* dst;
  const uint32_t* flags;
  const float* sdf;

  size_t at(int x, int y, int z) const { return (size_t)(x + P.W * (y + P.H * z)); }
  R ld(size_t k) const { return C::load(src[k]); }
  void st(size_t k, R v) const { dst[k] = C::store(v); }
  bool isSolid(size_t s) const { return (flags[s] & FLAG_SOLID) != 0u; }

  // pullSlow3, src/shaders/step3d.ts:119-168
  R pullSlow3(int i, int x, int y, int z, size_t idx, uint32_t fl, bool outlet, R force[3]) const {
    const size_t N = (size_t)P.N;
    const int j = opp(i);
    const int sx = x - CX[i], sy = y - CY[i], sz = z - CZ[i];
    if ((fl & (1u << i)) == 0u) return ld(i * N + at(sx, sy, sz));
    const bool outX = sx < 0 || sx >= P.W;
    const bool outY = sy < 0 || sy >= P.H;
    const bool outZ = sz < 0 || sz >= P.D;
    if (outX && outlet) return ld(i * N + at(P.W - 2, y, z));
    if (outY && outZ) return ld(j * N + idx);
    if (outY || outZ) {
      int rx = sx, ry = sy, rz = sz;
      int m = mirror_y(i);
      if (outY) {
        ry = y;
      } else {
        rz = z;
        m = mirror_z(i);
      }
      const size_t rs = at(rx, ry, rz);
      if (isSolid(rs)) {
        R fj = ld(j * N + idx);
        R t = R(2) * fj;
        force[0] += R(CX[j]) * t;
        force[1] += R(CY[j]) * t;
        force[2] += R(CZ[j]) * t;
        return fj;
      }
      return ld(m * N + rs);
    }
    if (outX) return ld(j * N + idx);
    const size_t s = at(sx, sy, sz);
    if (!isSolid(s)) return ld(i * N + s);
    // Bouzidi linear interpolated bounce-back
    R fj = ld(j * N + idx);
    R dF = R(sdf[idx]);
    R dS = R(sdf[s]);
    R q = clampR<R>(dF / std::max(dF - dS, R(1e-6)), R(1e-3), R(1));
    R fi = fj;
    if (q < R(0.5)) {
      int nx = x + CX[i], ny = y + CY[i], nz = z + CZ[i];
      if (nx >= 0 && nx < P.W && ny >= 0 && ny < P.H && nz >= 0 && nz < P.D) {
        size_t n = at(nx, ny, nz);
        if (!isSolid(n)) fi = R(2) * q * fj + (R(1) - R(2) * q) * ld(j * N + n);
      }
    } else {
      fi = fj / (R(2) * q) + (R(2) * q - R(1)) / (R(2) * q) * ld(i * N + idx);
    }
    R t = fj + fi;
    force[0] += R(CX[j]) * t;
    force[1] += R(CY[j]) * t;
    force[2] += R(CZ[j]) * t;
    return fi;
  }

  // main, src/shaders/step3d.ts:170-223. Returns true when the cell ran the slow path; its
  // momentum-exchange force is left in force[0..2].
  bool cell(int x, int y, int z, R force[3]) const {
    const size_t N = (size_t)P.N;
    const size_t idx = at(x, y, z);
    const uint32_t fl = flags[idx];
    R f[Q];
    bool outlet = false;
    bool slow = false;
    if (fl == 0u) {
      for (int i = 0; i < Q; i++) f[i] = ld(i * N + at(x - CX[i], y - CY[i], z - CZ[i]));
    } else {
      if (fl & FLAG_SOLID) return false;
      if (fl & FLAG_INLET) {
        for (int i = 0; i < Q; i++) st(i * N + idx, feq<R>(i, R(1), P.uIn, R(0), R(0)));
        return false;
      }
      outlet = (fl & FLAG_OUTLET) != 0u;
      slow = true;
      f[0] = ld(idx);
      for (int i = 1; i < Q; i++) f[i] = pullSlow3(i, x, y, z, idx, fl, outlet, force);
    }
    // moments (generated by sum() in src/shaders/step3d.ts:8-12,38-45): left-to-right order
    R drho = f[0];
    for (int i = 1; i < Q; i++) drho = drho + f[i];
    const R rho = R(1) + drho;
    const R invRho = R(1) / rho;
    const R jx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[13] - f[14] + f[15] - f[16];
    const R jy = f[3] - f[4] + f[7] - f[8] + f[11] - f[12] - f[13] + f[14] + f[17] - f[18];
    const R jz = f[5] - f[6] + f[9] - f[10] + f[11] - f[12] - f[15] + f[16] - f[17] + f[18];
    const R ux = jx * invRho, uy = jy * invRho, uz = jz * invRho;
    const R usq = R(1.5) * (ux * ux + uy * uy + uz * uz);
    if (outlet) {
      for (int i = 0; i < Q; i++) st(i * N + idx, feq<R>(i, R(1), ux, uy, uz));
      return slow;
    }
    // cu_a = 3 (c_a . u) for the lower member a of each pair (cDotU, src/shaders/step3d.ts:15-17)
    R cu[Q] = {};
    cu[1] = R(3) * (ux);
    cu[3] = R(3) * (uy);
    cu[5] = R(3) * (uz);
    cu[7] = R(3) * (ux + uy);
    cu[9] = R(3) * (ux + uz);
    cu[11] = R(3) * (uy + uz);
    cu[13] = R(3) * (ux - uy);
    cu[15] = R(3) * (ux - uz);
    cu[17] = R(3) * (uy - uz);
    R eqS[Q] = {}, eqA[Q] = {};
    for (int a = 1; a < Q; a += 2) {
      eqS[a] = wt<R>(a) * (drho + rho * (R(0.5) * cu[a] * cu[a] - usq));
      eqA[a] = wt<R>(a) * rho * cu[a];
    }
    R omegaBase = R(1) / P.tau;
    R sOut = R(0);
    if (P.spongeStart < R(P.W - 1)) {
      sOut = smoothstepR<R>(P.spongeStart, R(P.W - 1), R(x));
      omegaBase = R(1) / mixR<R>(P.tau, P.tauSponge, sOut);
    }
    const R sigma = P.absorb * sOut * sOut;
    // Smagorinsky, src/shaders/step3d.ts:54-74
    R omP = omegaBase;
    if (P.smagC2 > R(0)) {
      R n[Q];
      for (int a = 1; a < Q; a += 2) {
        n[a] = f[a] - (eqS[a] + eqA[a]);
        n[a + 1] = f[a + 1] - (eqS[a] - eqA[a]);
      }
      const R pxx = n[1] + n[2] + n[7] + n[8] + n[9] + n[10] + n[13] + n[14] + n[15] + n[16];
      const R pyy = n[3] + n[4] + n[7] + n[8] + n[11] + n[12] + n[13] + n[14] + n[17] + n[18];
      const R pzz = n[5] + n[6] + n[9] + n[10] + n[11] + n[12] + n[15] + n[16] + n[17] + n[18];
      const R pxy = n[7] + n[8] - n[13] - n[14];
      const R pxz = n[9] + n[10] - n[15] - n[16];
      const R pyz = n[11] + n[12] - n[17] - n[18];
      const R pi = std::sqrt(pxx * pxx + pyy * pyy + pzz * pzz + R(2) * (pxy * pxy + pxz * pxz + pyz * pyz));
      const R t0 = R(1) / omegaBase;
      const R tEff = R(0.5) * (t0 + std::sqrt(t0 * t0 + R(25.45584412271571) * P.smagC2 * pi * invRho));
      omP = R(1) / tEff;
    }
    const R omM = R(1) / (R(0.5) + P.lambda / (R(1) / omP - R(0.5)));
    // absorbing layer, src/shaders/step3d.ts:76-90
    R s0 = R(0);
    R sS[Q] = {}, sA[Q] = {};
    if (sigma > R(0)) {
      const R ut = P.uIn;
      const R dq = R(1.5) * rho * (ut * ut - ux * ux - uy * uy - uz * uz);
      s0 += sigma * wt<R>(0) * -dq;
      for (int a = 1; a < Q; a += 2) {
        const R cut = R(3) * R(CX[a]) * ut;
        sS[a] += sigma * wt<R>(a) * (R(0.5) * rho * (cut * cut - cu[a] * cu[a]) - dq);
        sA[a] += sigma * wt<R>(a) * rho * (cut - cu[a]);
      }
    }
    // TRT collide + store, src/shaders/step3d.ts:92-102
    st(idx, f[0] - omP * (f[0] - wt<R>(0) * (drho - rho * usq)) + s0);
    for (int a = 1; a < Q; a += 2) {
      const int b = a + 1;
      const R sym = omP * (R(0.5) * (f[a] + f[b]) - eqS[a]);
      const R asym = omM * (R(0.5) * (f[a] - f[b]) - eqA[a]);
      st(a * N + idx, f[a] - sym - asym + sS[a] + sA[a]);
      st(b * N + idx, f[b] - sym + asym + sS[a] - sA[a]);
    }
    return slow;
  }
};

struct HostParams3 {
  int32_t W, H, D;
  int32_t pad;
  double tau, lambda, smagC2, uIn, spongeStart, tauSponge, absorb;
};

template <class R>
P3<R> toP3(const HostParams3* h) {
  P3<R> p;
  p.W = h->W;
  p.H = h->H;
  p.D = h->D;
  p.N = h->W * h->H * h->D;
  p.tau = (R)h->tau;
  p.lambda = (R)h->lambda;
  p.smagC2 = (R)h->smagC2;
  p.uIn = (R)h->uIn;
  p.spongeStart = (R)h->spongeStart;
  p.tauSponge = (R)h->tauSponge;
  p.absorb = (R)h->absorb;
  return p;
}

template <class C>
void step3(const HostParams3* hp, const void* src, void* dst, const uint32_t* flags, const float* sdf,
           double* cellForce) {
  using R = typename C::R;
  const P3<R> P = toP3<R>(hp);
  Step3<C> k{P, (const typename C::S*)src, (typename C::S*)dst, flags, sdf};
#pragma omp parallel for schedule(static)
  for (int z = 0; z < P.D; z++)
    for (int y = 0; y < P.H; y++)
      for (int x = 0; x < P.W; x++) {
        R force[3] = {R(0), R(0), R(0)};
        k.cell(x, y, z, force);
        if (cellForce) {
          size_t idx = k.at(x, y, z);
          cellForce[3 * idx + 0] = (double)force[0];
          cellForce[3 * idx + 1] = (double)force[1];
          cellForce[3 * idx + 2] = (double)force[2];
        }
      }
}

// flags3dShader, src/shaders/aux3d.ts:20-101. touches[idx] = 1 marks a cell that the reference gives
// a force slot (a body link or a slip-face mirror onto a solid node).
template <class C>
void flags3(const HostParams3* hp, const float* sdf, uint32_t* flags, uint8_t* touches, void* fA, void* fB,
            const float* mac) {
  using R = typename C::R;
  using S = typename C::S;
  const P3<R> P = toP3<R>(hp);
  const int W = P.W, H = P.H, D = P.D;
  const size_t N = (size_t)P.N;
  auto inRange = [&](int x, int y, int z) { return x >= 0 && y >= 0 && z >= 0 && x < W && y < H && z < D; };
  auto solidAt = [&](int x, int y, int z) {
    if (x == 0 || x == W - 1) return false;
    return sdf[(size_t)(x + W * (y + H * z))] < 0.0f;
  };
#pragma omp parallel for schedule(static)
  for (int z = 0; z < D; z++)
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        const size_t idx = (size_t)(x + W * (y + H * z));
        const uint32_t old = flags[idx];
        if (solidAt(x, y, z)) {
          flags[idx] = FLAG_SOLID;
          touches[idx] = 0;
          continue;
        }
        uint32_t bits = 0;
        if (x == 0) bits = FLAG_INLET;
        if (x == W - 1) bits = FLAG_OUTLET;
        bool touchesBody = false;
        for (int i = 1; i < Q; i++) {
          const int sx = x - CX[i], sy = y - CY[i], sz = z - CZ[i];
          if (inRange(sx, sy, sz)) {
            if (solidAt(sx, sy, sz)) {
              bits |= 1u << i;
              touchesBody = true;
            }
            continue;
          }
          bits |= 1u << i;
          const bool outX = sx < 0 || sx >= W;
          const bool outY = sy < 0 || sy >= H;
          const bool outZ = sz < 0 || sz >= D;
          if (!outX && outY != outZ) {
            int rx = sx, ry = sy, rz = sz;
            if (outY) ry = y; else rz = z;
            if (solidAt(rx, ry, rz)) touchesBody = true;
          }
        }
        flags[idx] = bits;
        touches[idx] = touchesBody ? 1 : 0;
        if ((old & FLAG_SOLID) != 0u) {
          // refill a cell the obstacle uncovered (src/shaders/aux3d.ts:83-99)
          R rho = R(0), u[3] = {R(0), R(0), R(0)}, n = R(0);
          for (int i = 1; i < Q; i++) {
            const int qx = x + CX[i], qy = y + CY[i], qz = z + CZ[i];
            if (!inRange(qx, qy, qz)) continue;
            const float* m = mac + 4 * (size_t)(qx + W * (qy + H * qz));
            if (m[3] != 0.0f) {
              rho += (R)m[3];
              u[0] += (R)m[0];
              u[1] += (R)m[1];
              u[2] += (R)m[2];
              n += R(1);
            }
          }
          if (n > R(0)) {
            rho /= n;
            u[0] /= n;
            u[1] /= n;
            u[2] /= n;
          } else {
            rho = R(1);
            u[0] = P.uIn;
            u[1] = R(0);
            u[2] = R(0);
          }
          for (int i = 0; i < Q; i++) {
            const S v = C::store(feq<R>(i, rho, u[0], u[1], u[2]));
            ((S*)fA)[i * N + idx] = v;
            ((S*)fB)[i * N + idx] = v;
          }
        }
      }
}

// init3dShader (src/shaders/aux3d.ts:105-125), plus the macro-field variant the 3D reference lacks:
// when mac is given, fluid cells get feq(rho, u) from mac = (ux, uy, uz, rho) per cell.
template <class C>
void init3(const HostParams3* hp, void* fA, void* fB, const uint32_t* flags, const float* mac) {
  using R = typename C::R;
  using S = typename C::S;
  const P3<R> P = toP3<R>(hp);
  const size_t N = (size_t)P.N;
#pragma omp parallel for schedule(static)
  for (long long idx = 0; idx < (long long)N; idx++) {
    const bool solid = (flags[idx] & FLAG_SOLID) != 0u;
    for (int i = 0; i < Q; i++) {
      R v;
      if (solid) {
        v = R(0);
      } else if (mac) {
        const float* m = mac + 4 * idx;
        v = feq<R>(i, (R)m[3], (R)m[0], (R)m[1], (R)m[2]);
      } else {
        v = feq<R>(i, R(1), P.uIn, R(0), R(0));
      }
      const S s = C::store(v);
      ((S*)fA)[i * N + idx] = s;
      ((S*)fB)[i * N + idx] = s;
    }
  }
}

// macro3dShader, src/shaders/aux3d.ts:128-152: (ux, uy, uz, rho), rho = 0 in solids.
template <class C>
void macro3(const HostParams3* hp, const void* f, const uint32_t* flags, float* mac) {
  using R = typename C::R;
  using S = typename C::S;
  const P3<R> P = toP3<R>(hp);
  const size_t N = (size_t)P.N;
#pragma omp parallel for schedule(static)
  for (long long idx = 0; idx < (long long)N; idx++) {
    float* m = mac + 4 * idx;
    if (flags[idx] & FLAG_SOLID) {
      m[0] = m[1] = m[2] = m[3] = 0.0f;
      continue;
    }
    R drho = R(0), j[3] = {R(0), R(0), R(0)};
    for (int i = 0; i < Q; i++) {
      const R v = C::load(((const S*)f)[i * N + idx]);
      drho += v;
      j[0] += R(CX[i]) * v;
      j[1] += R(CY[i]) * v;
      j[2] += R(CZ[i]) * v;
    }
    const R rho = R(1) + drho;
    m[0] = (float)(j[0] / rho);
    m[1] = (float)(j[1] / rho);
    m[2] = (float)(j[2] / rho);
    m[3] = (float)rho;
  }
}

template <class C>
double mass3(const HostParams3* hp, const void* f, const uint32_t* flags) {
  using S = typename C::S;
  const size_t N = (size_t)hp->W * hp->H * hp->D;
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

// precision: 0 = f32, 1 = f16 x 2^15, 2 = bf16, 3 = f64 (same numbering as the product library)
#define ORACLE_DISPATCH(prec, call) \
  switch (prec) {                   \
    case 0: { using C = CodecF32; call; break; } \
    case 1: { using C = CodecF16; call; break; } \
    case 2: { using C = CodecBF16; call; break; } \
    case 3: { using C = CodecF64; call; break; } \
    default: return -1;             \
  }

int oracle3d_step(int precision, const HostParams3* p, const void* src, void* dst, const uint32_t* flags,
                  const float* sdf, double* cellForce) {
  ORACLE_DISPATCH(precision, (step3<C>(p, src, dst, flags, sdf, cellForce)));
  return 0;
}

int oracle3d_flags(int precision, const HostParams3* p, const float* sdf, uint32_t* flags, uint8_t* touches,
                   void* fA, void* fB, const float* mac) {
  ORACLE_DISPATCH(precision, (flags3<C>(p, sdf, flags, touches, fA, fB, mac)));
  return 0;
}

int oracle3d_init(int precision, const HostParams3* p, void* fA, void* fB, const uint32_t* flags,
                  const float* mac) {
  ORACLE_DISPATCH(precision, (init3<C>(p, fA, fB, flags, mac)));
  return 0;
}

int oracle3d_macro(int precision, const HostParams3* p, const void* f, const uint32_t* flags, float* mac) {
  ORACLE_DISPATCH(precision, (macro3<C>(p, f, flags, mac)));
  return 0;
}

int oracle3d_mass(int precision, const HostParams3* p, const void* f, const uint32_t* flags, double* out) {
  ORACLE_DISPATCH(precision, (*out = mass3<C>(p, f, flags)));
  return 0;
}

// trtLambda3, src/lattice3d.ts:29-31
double oracle_trt_lambda3(double tau) { return std::min(3.0 / 16.0, 50.0 * (tau - 0.5) * (tau - 0.5)); }

// codec round trips, for the known-answer tests of the storage formats
float oracle_codec_roundtrip(int precision, float v) {
  switch (precision) {
    case 0: return CodecF32::load(CodecF32::store(v));
    case 1: return CodecF16::load(CodecF16::store(v));
    case 2: return CodecBF16::load(CodecBF16::store(v));
    case 3: return (float)CodecF64::load(CodecF64::store(v));
  }
  return NAN;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  extern int omp_get_max_threads(void);
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
