// CPU restatement of the reference's macro-field sampling (TEST INFRASTRUCTURE ONLY: the CUDA
// kernels of cells_b200/csrc/fields3d.cu are checked against it bit for bit).
//
// src/shaders/render3d.ts:33-65 (MACRO_SAMPLE_WGSL: macAt with clamped indices, trilinear
// velocity, nearest-node solid test, |curl u| from central differences of the trilinear velocity at
// +-1 cell, fieldValue), :159-177 (the slice quad spanning [-0.5, dim - 0.5] on the two in-plane
// axes at slicePos * (dim - 1) on the slice axis), :196-230 (tracer advection: midpoint rule over the
// frame's lattice steps, split into ceil(uRef * steps) sub-steps when that travel exceeds
// SUBSTEP_TRAVEL = 2 cells, src/view3d.ts:85-92; a tracer that leaves the box or enters a solid
// restarts at its seed). The headless slice samples the quad at pixel centres. Every float
// operation is written out in the order the CUDA kernels use; WGSL's mix(a, b, t) is
// a * (1 - t) + b * t, round() rounds half to even, length(v) is sqrt((x*x + y*y) + z*z).
#include <cmath>
#include <cstdint>

namespace {

struct Field3 {
  const float* mac;  // (ux, uy, uz, rho) per cell, rho = 0 in solids
  int W, H, D;
};

struct V3 {
  float x, y, z;
};

inline V3 v3(float x, float y, float z) { return {x, y, z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 scale(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline V3 mix3(V3 a, V3 b, float t) { return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)}; }
inline float len3(V3 a) { return std::sqrt((a.x * a.x + a.y * a.y) + a.z * a.z); }

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

inline const float* mac_at(const Field3& F, int x, int y, int z) {
  x = clampi(x, 0, F.W - 1);
  y = clampi(y, 0, F.H - 1);
  z = clampi(z, 0, F.D - 1);
  return F.mac + 4 * ((long long)x + (long long)F.W * (y + (long long)F.H * z));
}

inline V3 vel_at(const Field3& F, int x, int y, int z) {
  const float* m = mac_at(F, x, y, z);
  return {m[0], m[1], m[2]};
}

V3 velocity(const Field3& F, V3 p) {
  const float fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
  const int bx = (int)fx, by = (int)fy, bz = (int)fz;
  const float tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
  const V3 x00 = mix3(vel_at(F, bx, by, bz), vel_at(F, bx + 1, by, bz), tx);
  const V3 x10 = mix3(vel_at(F, bx, by + 1, bz), vel_at(F, bx + 1, by + 1, bz), tx);
  const V3 x01 = mix3(vel_at(F, bx, by, bz + 1), vel_at(F, bx + 1, by, bz + 1), tx);
  const V3 x11 = mix3(vel_at(F, bx, by + 1, bz + 1), vel_at(F, bx + 1, by + 1, bz + 1), tx);
  return mix3(mix3(x00, x10, ty), mix3(x01, x11, ty), tz);
}

bool solid_at(const Field3& F, V3 p) {
  return mac_at(F, (int)std::nearbyint(p.x), (int)std::nearbyint(p.y), (int)std::nearbyint(p.z))[3] == 0.0f;
}

float vorticity(const Field3& F, V3 p) {
  const V3 dx = sub(velocity(F, add(p, v3(1, 0, 0))), velocity(F, sub(p, v3(1, 0, 0))));
  const V3 dy = sub(velocity(F, add(p, v3(0, 1, 0))), velocity(F, sub(p, v3(0, 1, 0))));
  const V3 dz = sub(velocity(F, add(p, v3(0, 0, 1))), velocity(F, sub(p, v3(0, 0, 1))));
  return len3(scale(0.5f, v3(dy.z - dz.y, dz.x - dx.z, dx.y - dy.x)));
}

float field_value(const Field3& F, V3 p, V3 u, int mode, float uRef) {
  if (mode == 0) return len3(u) / (1.6f * uRef);
  return vorticity(F, p) / (0.3f * uRef);
}

// the slice point of pixel (i, j) of an nu x nv sampling of the quad
V3 slice_point(int W, int H, int D, int axis, float pos, int i, int j, int nu, int nv) {
  const float cu = ((float)i + 0.5f) / (float)nu;
  const float cv = ((float)j + 0.5f) / (float)nv;
  const float dimX = (float)W, dimY = (float)H, dimZ = (float)D;
  if (axis == 0) return {pos * (dimX - 1.0f), mixf(-0.5f, dimY - 0.5f, cu), mixf(-0.5f, dimZ - 0.5f, cv)};
  if (axis == 1) return {mixf(-0.5f, dimX - 0.5f, cu), pos * (dimY - 1.0f), mixf(-0.5f, dimZ - 0.5f, cv)};
  return {mixf(-0.5f, dimX - 0.5f, cu), mixf(-0.5f, dimY - 0.5f, cv), pos * (dimZ - 1.0f)};
}

bool inside(const Field3& F, V3 p) {
  return p.x >= -0.5f && p.y >= -0.5f && p.z >= -0.5f && p.x <= (float)F.W - 0.5f && p.y <= (float)F.H - 0.5f &&
         p.z <= (float)F.D - 0.5f;
}

}  // namespace

extern "C" {

// out[j * nu + i]: NaN on a solid node, else the field value (speed / (1.6 uRef) for mode 0,
// |curl u| / (0.3 uRef) for mode 1) at the quad's pixel centre (i, j).
int oracle3d_sample_slice(const float* mac, int W, int H, int D, int axis, float pos, int mode, float uRef, int nu,
                          int nv, float* out) {
  if (axis < 0 || axis > 2 || nu <= 0 || nv <= 0) return -1;
  const Field3 F{mac, W, H, D};
  for (int j = 0; j < nv; j++)
    for (int i = 0; i < nu; i++) {
      const V3 p = slice_point(W, H, D, axis, pos, i, j, nu, nv);
      out[(long long)j * nu + i] = solid_at(F, p) ? NAN : field_value(F, p, velocity(F, p), mode, uRef);
    }
  return 0;
}

// particles: count x (position xyz_, velocity xyz_); seeds: count x (xyz_).
int oracle3d_advect(const float* mac, int W, int H, int D, const float* seeds, float* particles, int count,
                    float steps, float uRef) {
  const Field3 F{mac, W, H, D};
  const float travel = uRef * steps;
  const int n = travel > 2.0f ? (int)std::ceil(travel) : 1;
  const float h = steps / (float)n;
  for (int i = 0; i < count; i++) {
    float* q = particles + 8 * (long long)i;
    V3 p{q[0], q[1], q[2]};
    for (int k = 0; k < n; k++) {
      const V3 v1 = velocity(F, p);
      p = add(p, scale(h, velocity(F, add(p, scale(0.5f * h, v1)))));
      if (!inside(F, p) || solid_at(F, p)) {
        p = {seeds[4 * (long long)i], seeds[4 * (long long)i + 1], seeds[4 * (long long)i + 2]};
        break;
      }
    }
    const V3 u = velocity(F, p);
    q[0] = p.x;
    q[1] = p.y;
    q[2] = p.z;
    q[3] = 0.0f;
    q[4] = u.x;
    q[5] = u.y;
    q[6] = u.z;
    q[7] = 0.0f;
  }
  return 0;
}

}  // extern "C"
