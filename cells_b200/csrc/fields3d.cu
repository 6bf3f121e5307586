// Macro-field products of the 3D solver on the device: speed or vorticity magnitude on an
// axis-aligned slice, and tracer advection through the velocity field, both read from the macro
// buffer (ux, uy, uz, rho; rho = 0 in solids) as of the last cells3d_update_macro / cells3d_run.
//
// The math is the reference's visualisation sampler, src/shaders/render3d.ts:33-65 (clamped node
// reads, trilinear velocity, nearest-node solid test, |curl u| from central differences of the
// trilinear velocity at +-1 cell, the field value scaled by 1.6 uRef or 0.3 uRef), the slice quad
// :159-177 (the two in-plane axes span [-0.5, dim - 0.5], the slice axis sits at slicePos * (dim - 1)),
// and the tracer advection :196-230 (midpoint rule over a frame of lattice steps, ceil(uRef * steps)
// sub-steps when that travel exceeds 2 cells, src/view3d.ts:85-92; a tracer that leaves the box or
// enters a solid restarts at its seed). There is no graphics pipeline: the slice is sampled at pixel
// centres of an nu x nv grid into a buffer the caller reads back. Built without FMA contraction, so
// every value rounds as the written expressions state (mix(a, b, t) = a (1 - t) + b t).
#include <cmath>
#include <cstring>

#include "solver3d_state.h"

namespace cells {
namespace {

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 f3add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 f3sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 f3scale(float s, F3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ F3 f3mix(F3 a, F3 b, float t) {
  return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)};
}
__device__ __forceinline__ float f3len(F3 a) { return sqrtf((a.x * a.x + a.y * a.y) + a.z * a.z); }

struct MacField {
  const float4* mac;
  int W, H, D;
  __device__ __forceinline__ float4 at(int x, int y, int z) const {
    x = min(max(x, 0), W - 1);
    y = min(max(y, 0), H - 1);
    z = min(max(z, 0), D - 1);
    return __ldg(mac + ((long long)x + (long long)W * (y + (long long)H * z)));
  }
  __device__ __forceinline__ F3 vel(int x, int y, int z) const {
    const float4 m = at(x, y, z);
    return {m.x, m.y, m.z};
  }
  __device__ F3 velocity(F3 p) const {
    const float fx = floorf(p.x), fy = floorf(p.y), fz = floorf(p.z);
    const int bx = (int)fx, by = (int)fy, bz = (int)fz;
    const float tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
    const F3 x00 = f3mix(vel(bx, by, bz), vel(bx + 1, by, bz), tx);
    const F3 x10 = f3mix(vel(bx, by + 1, bz), vel(bx + 1, by + 1, bz), tx);
    const F3 x01 = f3mix(vel(bx, by, bz + 1), vel(bx + 1, by, bz + 1), tx);
    const F3 x11 = f3mix(vel(bx, by + 1, bz + 1), vel(bx + 1, by + 1, bz + 1), tx);
    return f3mix(f3mix(x00, x10, ty), f3mix(x01, x11, ty), tz);
  }
  // round() rounds half to even, as rintf does
  __device__ __forceinline__ bool solid(F3 p) const {
    return at((int)rintf(p.x), (int)rintf(p.y), (int)rintf(p.z)).w == 0.0f;
  }
  __device__ float vorticity(F3 p) const {
    const F3 dx = f3sub(velocity(f3add(p, {1, 0, 0})), velocity(f3sub(p, {1, 0, 0})));
    const F3 dy = f3sub(velocity(f3add(p, {0, 1, 0})), velocity(f3sub(p, {0, 1, 0})));
    const F3 dz = f3sub(velocity(f3add(p, {0, 0, 1})), velocity(f3sub(p, {0, 0, 1})));
    return f3len(f3scale(0.5f, {dy.z - dz.y, dz.x - dx.z, dx.y - dy.x}));
  }
  __device__ __forceinline__ bool inside(F3 p) const {
    return p.x >= -0.5f && p.y >= -0.5f && p.z >= -0.5f && p.x <= (float)W - 0.5f && p.y <= (float)H - 0.5f &&
           p.z <= (float)D - 0.5f;
  }
};

__global__ void slice3_kernel(MacField F, int axis, float pos, int mode, float uRef, int nu, int nv, float* out) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)nu * nv) return;
  const int i = (int)(k % nu), j = (int)(k / nu);
  const float cu = ((float)i + 0.5f) / (float)nu;
  const float cv = ((float)j + 0.5f) / (float)nv;
  const float dimX = (float)F.W, dimY = (float)F.H, dimZ = (float)F.D;
  F3 p;
  if (axis == 0)
    p = {pos * (dimX - 1.0f), mixf(-0.5f, dimY - 0.5f, cu), mixf(-0.5f, dimZ - 0.5f, cv)};
  else if (axis == 1)
    p = {mixf(-0.5f, dimX - 0.5f, cu), pos * (dimY - 1.0f), mixf(-0.5f, dimZ - 0.5f, cv)};
  else
    p = {mixf(-0.5f, dimX - 0.5f, cu), mixf(-0.5f, dimY - 0.5f, cv), pos * (dimZ - 1.0f)};
  float v;
  if (F.solid(p))
    v = __int_as_float(0x7fc00000);  // NaN marks a solid node
  else if (mode == 0)
    v = f3len(F.velocity(p)) / (1.6f * uRef);
  else
    v = F.vorticity(p) / (0.3f * uRef);
  out[k] = v;
}

// particles: count x (position xyz_, velocity xyz_); seeds: count x (xyz_)
__global__ void advect3_kernel(MacField F, const float4* seeds, float4* particles, int count, int n, float h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float4 q = particles[2 * i];
  F3 p{q.x, q.y, q.z};
  for (int k = 0; k < n; k++) {
    const F3 v1 = F.velocity(p);
    p = f3add(p, f3scale(h, F.velocity(f3add(p, f3scale(0.5f * h, v1)))));
    if (!F.inside(p) || F.solid(p)) {
      const float4 s = seeds[i];
      p = {s.x, s.y, s.z};
      break;
    }
  }
  const F3 u = F.velocity(p);
  particles[2 * i] = make_float4(p.x, p.y, p.z, 0.0f);
  particles[2 * i + 1] = make_float4(u.x, u.y, u.z, 0.0f);
}

}  // namespace
}  // namespace cells

using namespace cells;

void* Cells3D::scratch_buffer(size_t bytes) {
  if (bytes > scratchBytes) {
    if (scratch) dev.release(scratch);
    scratch = nullptr;
    scratchBytes = 0;
    scratch = dev.alloc(bytes, "field scratch");
    scratchBytes = bytes;
  }
  return scratch;
}

int cells3d_sample_slice(Cells3D* h, int axis, double pos, int mode, double u_ref, int nu, int nv, float* out) {
  if (!h || !out) return CELLS_E_INVALID;
  try {
    if (axis < 0 || axis > 2) throw Error(CELLS_E_INVALID, "axis must be 0 (x), 1 (y) or 2 (z)");
    if (mode != CELLS_FIELD_SPEED && mode != CELLS_FIELD_VORTICITY) throw Error(CELLS_E_INVALID, "unknown field mode");
    if (!(pos >= 0.0 && pos <= 1.0)) throw Error(CELLS_E_INVALID, "slice position must be within [0, 1]");
    if (!(u_ref > 0.0) || !std::isfinite(u_ref)) throw Error(CELLS_E_INVALID, "u_ref must be positive");
    if (nu <= 0 || nv <= 0 || (long long)nu * nv > (1LL << 28)) throw Error(CELLS_E_INVALID, "bad slice size");
    const size_t bytes = (size_t)nu * nv * sizeof(float);
    if (h->dev.fake) {
      std::memset(out, 0, bytes);
      return CELLS_OK;
    }
    float* d = (float*)h->scratch_buffer(bytes);
    const MacField F{h->macro, h->W, h->H, h->D};
    const long long total = (long long)nu * nv;
    slice3_kernel<<<(unsigned)((total + 255) / 256), 256, 0, h->dev.stream>>>(F, axis, (float)pos, mode, (float)u_ref,
                                                                              nu, nv, d);
    check_cuda(cudaGetLastError(), "slice kernel");
    h->dev.launches++;
    h->dev.d2h(out, d, bytes);
    h->dev.sync();
  } catch (const AllocError& e) {
    h->lastError = std::string("Solver3D allocation failed: ") + e.what();
    return CELLS_E_ALLOC;
  } catch (const Error& e) {
    h->lastError = e.what();
    return e.status;
  }
  return CELLS_OK;
}

int cells3d_advect_tracers(Cells3D* h, const float* seeds, float* particles, int count, double steps, double u_ref) {
  if (!h || count < 0 || (count > 0 && (!seeds || !particles))) return CELLS_E_INVALID;
  try {
    if (!(u_ref > 0.0) || !std::isfinite(u_ref)) throw Error(CELLS_E_INVALID, "u_ref must be positive");
    if (!(steps >= 0.0) || !std::isfinite(steps)) throw Error(CELLS_E_INVALID, "steps must be finite and >= 0");
    if (count == 0 || h->dev.fake) return CELLS_OK;
    // sub-steps of the frame (src/view3d.ts:89-92), in f32 as the shader computes them
    const float travel = (float)u_ref * (float)steps;
    const float nf = travel > 2.0f ? std::ceil(travel) : 1.0f;
    if (nf > 1e7f) throw Error(CELLS_E_INVALID, "u_ref * steps is too large for one frame");
    const int n = (int)nf;
    const float hstep = (float)steps / (float)n;
    const size_t seedBytes = (size_t)count * 16, partBytes = (size_t)count * 32;
    char* d = (char*)h->scratch_buffer(seedBytes + partBytes);
    h->dev.h2d(d, seeds, seedBytes);
    h->dev.h2d(d + seedBytes, particles, partBytes);
    const MacField F{h->macro, h->W, h->H, h->D};
    advect3_kernel<<<(count + 127) / 128, 128, 0, h->dev.stream>>>(F, (const float4*)d, (float4*)(d + seedBytes),
                                                                   count, n, hstep);
    check_cuda(cudaGetLastError(), "advect kernel");
    h->dev.launches++;
    h->dev.d2h(particles, d + seedBytes, partBytes);
    h->dev.sync();
  } catch (const AllocError& e) {
    h->lastError = std::string("Solver3D allocation failed: ") + e.what();
    return CELLS_E_ALLOC;
  } catch (const Error& e) {
    h->lastError = e.what();
    return e.status;
  }
  return CELLS_OK;
}
