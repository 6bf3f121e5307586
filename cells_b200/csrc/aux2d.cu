// Auxiliary D2Q9 kernels: flags + refill, init, macro, mass, the SDF brush and the device-state
// writer. Reference: src/shaders/aux.ts:14-194. They run once per set_sdf / init_field / readback,
// not per step, so they use a flat one-thread-per-cell launch. Compiled with -fmad=false: the
// equilibria they write round exactly as the reference's expressions state.
#include "kernels2d.h"

namespace cells {

namespace {

struct A2F32 {
  using S = float;
  using R = float;
};
struct A2F64 {
  using S = double;
  using R = double;
};

inline unsigned blocks_for2(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// feq, shifted by w_i (src/shaders/aux.ts:14-19)
template <class R>
__device__ __forceinline__ R feq2a(int i, R rho, R ux, R uy) {
  R cu = R(3) * (R(cx2(i)) * ux + R(cy2(i)) * uy);
  return w2<R>(i) * (rho - R(1) + rho * (cu + R(0.5) * cu * cu - R(1.5) * (ux * ux + uy * uy)));
}

__device__ __forceinline__ void wrap2a(const AuxLaunch2& a, int& x, int& y) {
  if (x < 0 && a.left == X2_PERIODIC) x += a.W;
  if (x >= a.W && a.right == X2_PERIODIC) x -= a.W;
  if (y < 0 && a.bottom == Y2_PERIODIC) y += a.H;
  if (y >= a.H && a.top == Y2_PERIODIC) y -= a.H;
}

// flagsShader, src/shaders/aux.ts:22-88
template <class C>
__global__ void flags2_kernel(AuxLaunch2 a, const float* __restrict__ sdf, uint32_t* __restrict__ flags,
                              typename C::S* __restrict__ fA, typename C::S* __restrict__ fB,
                              const float4* __restrict__ mac, unsigned* __restrict__ counter) {
  using R = typename C::R;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.N) return;
  const int W = a.W, H = a.H;
  const int y = (int)(idx / W);
  const int x = (int)(idx - (long long)y * W);
  // open boundary columns stay fluid even when an obstacle is drawn over them
  auto solidAt = [&](int qx, int qy) {
    const bool open = (a.left == X2_OPEN && qx == 0) || (a.right == X2_OPEN && qx == W - 1);
    return !open && sdf[(long long)qy * W + qx] < 0.0f;
  };
  const uint32_t old = flags[idx];
  if (solidAt(x, y)) {
    flags[idx] = FLAG2_SOLID;
    return;
  }
  uint32_t bits = 0;
  if (a.left == X2_OPEN && x == 0) bits = FLAG2_INLET;
  if (a.right == X2_OPEN && x == W - 1) bits = FLAG2_OUTLET;
  bool touchesBody = false;
  for (int i = 1; i < Q2; i++) {
    int sx = x - cx2(i), sy = y - cy2(i);
    wrap2a(a, sx, sy);
    const bool inside = sx >= 0 && sy >= 0 && sx < W && sy < H;
    if (inside && solidAt(sx, sy)) {
      bits |= 1u << i;
      touchesBody = true;
    } else if (!inside || sx != x - cx2(i) || sy != y - cy2(i)) {
      // off the grid or across a periodic seam: the slow path resolves it
      bits |= 1u << i;
    }
  }
  if (touchesBody) {
    const unsigned slot = atomicAdd(counter, 1u) + 1u;
    if (slot < (1u << (32 - BIDX2_SHIFT))) bits |= slot << BIDX2_SHIFT;
  }
  flags[idx] = bits;
  if ((old & FLAG2_SOLID) != 0u) {
    R rho = R(0), ux = R(0), uy = R(0), n = R(0);
    for (int i = 1; i < Q2; i++) {
      const int sx = x + cx2(i), sy = y + cy2(i);
      if (sx < 0 || sy < 0 || sx >= W || sy >= H) continue;
      const float4 m = mac[(long long)sy * W + sx];
      if (m.w == 0.0f) {
        rho += (R)m.x;
        ux += (R)m.y;
        uy += (R)m.z;
        n += R(1);
      }
    }
    if (n > R(0)) {
      rho /= n;
      ux /= n;
      uy /= n;
    } else {
      rho = R(1);
    }
    for (int i = 0; i < Q2; i++) {
      const typename C::S v = (typename C::S)feq2a<R>(i, rho, ux, uy);
      fA[i * (long long)a.N + idx] = v;
      fB[i * (long long)a.N + idx] = v;
    }
  }
}

// initShader, src/shaders/aux.ts:92-111
template <class C>
__global__ void init2_kernel(AuxLaunch2 a, const float4* __restrict__ mac, typename C::S* __restrict__ fA,
                             typename C::S* __restrict__ fB) {
  using R = typename C::R;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.N) return;
  const float4 m = mac[idx];
  for (int i = 0; i < Q2; i++) {
    const typename C::S v = (typename C::S)feq2a<R>(i, (R)m.x, (R)m.y, (R)m.z);
    fA[i * (long long)a.N + idx] = v;
    fB[i * (long long)a.N + idx] = v;
  }
}

// macroShader, src/shaders/aux.ts:115-140: (rho, ux, uy, 0); solids (1, 0, 0, 1)
template <class C>
__global__ void macro2_kernel(AuxLaunch2 a, const typename C::S* __restrict__ f, const uint32_t* __restrict__ flags,
                              float4* __restrict__ mac, DevState2* st) {
  using R = typename C::R;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.N) return;
  if (flags[idx] & FLAG2_SOLID) {
    mac[idx] = make_float4(1.0f, 0.0f, 0.0f, 1.0f);
    return;
  }
  const long long N = a.N;
  R v[Q2];
  for (int i = 0; i < Q2; i++) v[i] = (R)f[i * N + idx];
  const R rho = R(1) + v[0] + v[1] + v[2] + v[3] + v[4] + v[5] + v[6] + v[7] + v[8];
  R jx = v[1] - v[3] + v[5] - v[6] - v[7] + v[8];
  R jy = v[2] - v[4] + v[5] + v[6] - v[7] - v[8];
  if (a.forcing != 0) {
    jx -= R(0.5) * (R)a.fx;
    jy -= R(0.5) * (R)a.fy;
  }
  const float4 m = make_float4((float)rho, (float)(jx / rho), (float)(jy / rho), 0.0f);
  if (!isfinite(m.x) || !isfinite(m.y) || !isfinite(m.z)) atomicOr(&st->status, 2u);
  mac[idx] = m;
}

template <class C>
__global__ void mass2_partial_kernel(AuxLaunch2 a, const typename C::S* __restrict__ f,
                                     const uint32_t* __restrict__ flags, double* __restrict__ partials) {
  __shared__ double red[32];
  const long long N = a.N;
  double acc = 0.0;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < N;
       idx += (long long)gridDim.x * blockDim.x) {
    if (flags[idx] & FLAG2_SOLID) continue;
    double drho = 0.0;
    for (int i = 0; i < Q2; i++) drho += (double)f[i * N + idx];
    acc += 1.0 + drho;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    partials[blockIdx.x] = s;
  }
}

__global__ void sum_partials2_kernel(const double* __restrict__ partials, int n, double* __restrict__ out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) acc += partials[k];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    *out = s;
  }
}

// brushShader, src/shaders/aux.ts:177-194
__global__ void brush2_kernel(float* __restrict__ sdf, int W, int H, float cx, float cy, float r, int erase, int x0,
                              int y0, int w, int h) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x;
  const int gy = blockIdx.y * blockDim.y + threadIdx.y;
  if (gx >= w || gy >= h) return;
  const int x = x0 + gx, y = y0 + gy;
  if (x >= W || y >= H) return;
  const long long idx = (long long)y * W + x;
  const float dx = (float)x - cx, dy = (float)y - cy;
  const float d = sqrtf(dx * dx + dy * dy) - r;
  const float s = sdf[idx];
  sdf[idx] = erase == 0 ? fminf(s, d) : fmaxf(s, -d);
}

__global__ void set_state2_kernel(DevState2* st, int which, unsigned step, double u) {
  if (which & 1) st->step[0] = st->step[1] = step;
  if (which & 2) st->uIn[0] = st->uIn[1] = u;
  if (which & 4) {
    st->sample = 0;
    st->done = 0;
  }
  if (which & 8) st->status = 0;
}

}  // namespace

#define CELLS2_DISPATCH(prec, expr)                      \
  do {                                                   \
    if ((prec) == 0) {                                   \
      using C = A2F32;                                   \
      expr;                                              \
    } else if ((prec) == 3) {                            \
      using C = A2F64;                                   \
      expr;                                              \
    } else {                                             \
      return cudaErrorInvalidValue;                      \
    }                                                    \
  } while (0)

cudaError_t launch_flags2(int precision, const AuxLaunch2& a, const float* sdf, uint32_t* flags, void* fA, void* fB,
                          const float4* mac, unsigned* counter, cudaStream_t s) {
  CELLS2_DISPATCH(precision, (flags2_kernel<C><<<blocks_for2(a.N, 256), 256, 0, s>>>(
                                 a, sdf, flags, (typename C::S*)fA, (typename C::S*)fB, mac, counter)));
  return cudaGetLastError();
}

cudaError_t launch_init2(int precision, const AuxLaunch2& a, const float4* mac, void* fA, void* fB, cudaStream_t s) {
  CELLS2_DISPATCH(precision, (init2_kernel<C><<<blocks_for2(a.N, 256), 256, 0, s>>>(
                                 a, mac, (typename C::S*)fA, (typename C::S*)fB)));
  return cudaGetLastError();
}

cudaError_t launch_macro2(int precision, const AuxLaunch2& a, const void* f, const uint32_t* flags, float4* mac,
                          DevState2* st, cudaStream_t s) {
  CELLS2_DISPATCH(precision, (macro2_kernel<C><<<blocks_for2(a.N, 256), 256, 0, s>>>(
                                 a, (const typename C::S*)f, flags, mac, st)));
  return cudaGetLastError();
}

cudaError_t launch_mass2(int precision, const AuxLaunch2& a, const void* f, const uint32_t* flags, double* partials,
                         int nPartials, double* out, cudaStream_t s) {
  CELLS2_DISPATCH(precision, (mass2_partial_kernel<C><<<nPartials, 256, 0, s>>>(
                                 a, (const typename C::S*)f, flags, partials)));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  sum_partials2_kernel<<<1, 256, 0, s>>>(partials, nPartials, out);
  return cudaGetLastError();
}

cudaError_t launch_brush2(float* sdf, int W, int H, float cx, float cy, float r, int erase, int x0, int y0, int w,
                          int h, cudaStream_t s) {
  if (w <= 0 || h <= 0) return cudaSuccess;
  dim3 block(8, 8);
  dim3 grid((unsigned)((w + 7) / 8), (unsigned)((h + 7) / 8));
  brush2_kernel<<<grid, block, 0, s>>>(sdf, W, H, cx, cy, r, erase, x0, y0, w, h);
  return cudaGetLastError();
}

cudaError_t launch_set_state2(DevState2* st, int which, unsigned step, double uIn, cudaStream_t s) {
  set_state2_kernel<<<1, 1, 0, s>>>(st, which, step, uIn);
  return cudaGetLastError();
}

}  // namespace cells
