// Auxiliary D3Q19 kernels: flags + refill, init, macro, mass and the device-state writer.
// Reference: src/shaders/aux3d.ts:20-152. These run once per set_sdf / init_field / readback, not
// per step, so they use a flat one-thread-per-cell launch.
#include "kernels3d.h"

namespace cells {

template <class R>
__device__ __forceinline__ R feq3a(int i, R rho, R ux, R uy, R uz) {
  R cu = R(3) * (R(cx3(i)) * ux + R(cy3(i)) * uy + R(cz3(i)) * uz);
  return w3<R>(i) * (rho - R(1) + rho * (cu + R(0.5) * cu * cu - R(1.5) * (ux * ux + uy * uy + uz * uz)));
}

static inline unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

template <class C>
__global__ void flags3_kernel(AuxLaunch3 a, const float* __restrict__ sdf, uint32_t* __restrict__ flags,
                              uint8_t* __restrict__ rowBody, typename C::S* __restrict__ fA,
                              typename C::S* __restrict__ fB, const float4* __restrict__ mac) {
  using R = typename C::R;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.N) return;
  const int W = a.W, H = a.H, D = a.D;
  const int WH = W * H;
  const int z = (int)(idx / WH);
  const int rem = (int)(idx - (long long)z * WH);
  const int y = rem / W;
  const int x = rem - y * W;
  const int row = y + H * z;
  auto inRange = [&](int qx, int qy, int qz) { return qx >= 0 && qy >= 0 && qz >= 0 && qx < W && qy < H && qz < D; };
  // the inlet and outlet planes stay fluid even when an obstacle reaches them
  auto solidAt = [&](int qx, int qy, int qz) {
    if (qx == 0 || qx == W - 1) return false;
    return sdf[qx + W * (qy + H * qz)] < 0.0f;
  };
  const uint32_t old = flags[idx];
  if (solidAt(x, y, z)) {
    flags[idx] = FLAG3_SOLID;
    rowBody[row] = 1;
    return;
  }
  uint32_t bits = 0u;
  if (x == 0) bits = FLAG3_INLET;
  if (x == W - 1) bits = FLAG3_OUTLET;
  bool touchesBody = false;
  for (int i = 1; i < Q3; i++) {
    const int sx = x - cx3(i), sy = y - cy3(i), sz = z - cz3(i);
    if (inRange(sx, sy, sz)) {
      if (solidAt(sx, sy, sz)) {
        bits |= 1u << i;
        touchesBody = true;
      }
      continue;
    }
    bits |= 1u << i;
    // a slip face mirrors from the reflected node, which is a body link when that node is solid
    const bool outX = sx < 0 || sx >= W;
    const bool outY = sy < 0 || sy >= H;
    const bool outZ = sz < 0 || sz >= D;
    if (!outX && outY != outZ) {
      const int ry = outY ? y : sy;
      const int rz = outY ? sz : z;
      if (solidAt(sx, ry, rz)) touchesBody = true;
    }
  }
  flags[idx] = bits;
  if (touchesBody) rowBody[row] = 1;
  if ((old & FLAG3_SOLID) != 0u) {
    // refill a cell the obstacle uncovered from its fluid neighbours (rho != 0 marks fluid)
    R rho = R(0), ux = R(0), uy = R(0), uz = R(0), n = R(0);
    for (int i = 1; i < Q3; i++) {
      const int qx = x + cx3(i), qy = y + cy3(i), qz = z + cz3(i);
      if (!inRange(qx, qy, qz)) continue;
      const float4 m = mac[qx + W * (qy + H * qz)];
      if (m.w != 0.0f) {
        rho += (R)m.w;
        ux += (R)m.x;
        uy += (R)m.y;
        uz += (R)m.z;
        n += R(1);
      }
    }
    if (n > R(0)) {
      rho /= n;
      ux /= n;
      uy /= n;
      uz /= n;
    } else {
      rho = R(1);
      ux = (R)a.uIn;
      uy = R(0);
      uz = R(0);
    }
    const size_t N = (size_t)a.N;
    for (int i = 0; i < Q3; i++) {
      const typename C::S v = C::enc(feq3a<R>(i, rho, ux, uy, uz));
      fA[i * N + idx] = v;
      fB[i * N + idx] = v;
    }
  }
}

// pullSlow3 (src/shaders/step3d.ts:119-168) resolved per (body cell, direction): which source
// elements a step reads and with which Bouzidi coefficients. q and the coefficients are computed
// with the reference's operations in the arithmetic type, so the step reproduces its rounding.
template <class C>
__global__ void links3_kernel(AuxLaunch3 a, const int* __restrict__ cells, int n, const uint32_t* __restrict__ flags,
                              const float* __restrict__ sdf, BodyLinks3 L) {
  using R = typename C::R;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const int W = a.W, H = a.H, D = a.D;
  const long long N = a.N;
  const int idx = cells[b];
  const int WH = W * H;
  const int z = idx / WH;
  const int rem = idx - z * WH;
  const int y = rem / W;
  const int x = rem - y * W;
  const uint32_t fl = flags[idx];
  const bool outlet = (fl & FLAG3_OUTLET) != 0u;
  L.meta[b] = x | (outlet ? (1 << 29) : 0) | ((fl & FLAG3_INLET) ? (1 << 30) : 0);
  auto at = [&](int qx, int qy, int qz) { return (long long)qx + (long long)W * (qy + (long long)H * qz); };
  auto solid = [&](long long cell) { return (flags[cell] & FLAG3_SOLID) != 0u; };
  Link3<R>* recs = (Link3<R>*)L.rec;
  unsigned long long kinds = 0ull;
  for (int i = 1; i < Q3; i++) {
    const int j = opp3(i);
    const int sx = x - cx3(i), sy = y - cy3(i), sz = z - cz3(i);
    uint8_t kind = LINK_LOAD;
    long long e1 = 0, e2 = -1;
    R k1 = R(0), k2 = R(0);
    if ((fl & (1u << i)) == 0u) {
      e1 = (long long)i * N + at(sx, sy, sz);
    } else {
      const bool outX = sx < 0 || sx >= W;
      const bool outY = sy < 0 || sy >= H;
      const bool outZ = sz < 0 || sz >= D;
      if (outX && outlet) {
        e1 = (long long)i * N + at(W - 2, y, z);
      } else if (outY && outZ) {
        e1 = (long long)j * N + idx;
      } else if (outY || outZ) {
        const int ry = outY ? y : sy;
        const int rz = outY ? sz : z;
        const long long rs = at(sx, ry, rz);
        if (solid(rs)) {
          kind = LINK_SLIP_SOLID;
          e1 = (long long)j * N + idx;
        } else {
          e1 = (long long)(outY ? mirror_y3(i) : mirror_z3(i)) * N + rs;
        }
      } else if (outX) {
        e1 = (long long)j * N + idx;
      } else {
        const long long s = at(sx, sy, sz);
        if (!solid(s)) {
          e1 = (long long)i * N + s;
        } else {
          e1 = (long long)j * N + idx;
          const R dF = R(sdf[idx]);
          const R dS = R(sdf[s]);
          R q = dF / max(dF - dS, R(1e-6));
          q = min(max(q, R(1e-3)), R(1));
          if (q < R(0.5)) {
            kind = LINK_BOUZIDI_0;
            const int nx = x + cx3(i), ny = y + cy3(i), nz = z + cz3(i);
            if (nx >= 0 && nx < W && ny >= 0 && ny < H && nz >= 0 && nz < D) {
              const long long nn = at(nx, ny, nz);
              if (!solid(nn)) {
                kind = LINK_BOUZIDI_N;
                e2 = (long long)j * N + nn;
                k1 = R(2) * q;
                k2 = R(1) - R(2) * q;
              }
            }
          } else {
            kind = LINK_BOUZIDI_H;
            e2 = (long long)i * N + idx;
            k1 = R(2) * q;
            k2 = (R(2) * q - R(1)) / (R(2) * q);
          }
        }
      }
    }
    Link3<R> rec;
    rec.e1 = e1;
    rec.e2 = e2 >= 0 ? e2 : e1;
    rec.c1 = k1;
    rec.c2 = k2;
    recs[(long long)(i - 1) * L.cap + b] = rec;
    kinds |= (unsigned long long)kind << (3 * (i - 1));
  }
  L.kinds[b] = kinds;
}

template <class C>
__global__ void init3_kernel(AuxLaunch3 a, typename C::S* __restrict__ fA, typename C::S* __restrict__ fB,
                             const uint32_t* __restrict__ flags, const float4* __restrict__ mac) {
  using R = typename C::R;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.N) return;
  const size_t N = (size_t)a.N;
  const bool solid = (flags[idx] & FLAG3_SOLID) != 0u;
  R rho = R(1), ux = (R)a.uIn, uy = R(0), uz = R(0);
  if (mac) {
    const float4 m = mac[idx];
    rho = (R)m.w;
    ux = (R)m.x;
    uy = (R)m.y;
    uz = (R)m.z;
  }
  for (int i = 0; i < Q3; i++) {
    const R v = solid ? R(0) : feq3a<R>(i, rho, ux, uy, uz);
    const typename C::S s = C::enc(v);
    fA[i * N + idx] = s;
    fB[i * N + idx] = s;
  }
}

template <class C>
__global__ void macro3_kernel(AuxLaunch3 a, const typename C::S* __restrict__ f, const uint32_t* __restrict__ flags,
                              float4* __restrict__ mac, DevState3* __restrict__ st) {
  using R = typename C::R;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.N) return;
  if (flags[idx] & FLAG3_SOLID) {
    mac[idx] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  const size_t N = (size_t)a.N;
  R drho = R(0), jx = R(0), jy = R(0), jz = R(0);
  for (int i = 0; i < Q3; i++) {
    const R v = C::load(f + i * N + idx);
    drho += v;
    jx += R(cx3(i)) * v;
    jy += R(cy3(i)) * v;
    jz += R(cz3(i)) * v;
  }
  const R rho = R(1) + drho;
  const float4 m = make_float4((float)(jx / rho), (float)(jy / rho), (float)(jz / rho), (float)rho);
  mac[idx] = m;
  if (!isfinite(m.x) || !isfinite(m.y) || !isfinite(m.z) || !isfinite(m.w)) atomicOr(&st->status, 2u);
}

template <class C>
__global__ void mass3_partial_kernel(AuxLaunch3 a, const typename C::S* __restrict__ f,
                                     const uint32_t* __restrict__ flags, double* __restrict__ partials) {
  __shared__ double red[32];
  const size_t N = (size_t)a.N;
  double acc = 0.0;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < a.N;
       idx += (long long)gridDim.x * blockDim.x) {
    if (flags[idx] & FLAG3_SOLID) continue;
    double drho = 0.0;
    for (int i = 0; i < Q3; i++) drho += (double)C::load(f + i * N + idx);
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

__global__ void sum_partials_kernel(const double* __restrict__ partials, int n, double* __restrict__ out) {
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

// which: bit 0 writes the step counters, bit 1 the inlet speeds, bit 2 clears the sample counter,
// bit 3 clears the status word.
template <class C>
__global__ void set_state3_kernel(DevState3* st, int which, unsigned step, double u0, double u1) {
  using R = typename C::R;
  if (which & 1) {
    st->step[0] = step;
    st->step[1] = step;
  }
  if (which & 2) {
    st->uIn[0] = u0;
    st->uIn[1] = u1;
    // inlet equilibrium in storage units, as the step kernels compute it (src/shaders/common3d.ts:38-41)
    for (int k = 0; k < 2; k++) {
      const R u = (R)(k == 0 ? u0 : u1);
      for (int i = 0; i < Q3; i++)
        st->inletEq[k][i] = (double)(feq3a<R>(i, R(1), u, R(0), R(0)) * R(C::SCALE));
    }
  }
  if (which & 4) {
    st->sample = 0u;
    st->done = 0u;
  }
  if (which & 8) st->status = 0u;
}

// The body role's cells (fluid cells with a non-zero flag word in a row that holds a body cell), in
// increasing index order, built on the device: one warp per row counts them, the host turns the
// counts into offsets, and one warp per row writes its cells in x order with ballots.
__global__ void body_count3_kernel(int W, int nRows, const uint8_t* __restrict__ rowBody,
                                   const uint32_t* __restrict__ flags, int* __restrict__ counts) {
  const int row = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= nRows) return;
  int c = 0;
  if (rowBody[row]) {
    for (int x = lane; x < W; x += 32) {
      const uint32_t f = flags[(long long)row * W + x];
      c += (f != 0u && !(f & FLAG3_SOLID)) ? 1 : 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  }
  if (lane == 0) counts[row] = c;
}

__global__ void body_write3_kernel(int W, int nRows, const uint8_t* __restrict__ rowBody,
                                   const uint32_t* __restrict__ flags, const int* __restrict__ offsets,
                                   int* __restrict__ cells) {
  const int row = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= nRows || !rowBody[row]) return;
  int base = offsets[row];
  for (int x0 = 0; x0 < W; x0 += 32) {
    const int x = x0 + lane;
    bool take = false;
    if (x < W) {
      const uint32_t f = flags[(long long)row * W + x];
      take = f != 0u && !(f & FLAG3_SOLID);
    }
    const unsigned m = __ballot_sync(0xffffffffu, take);
    if (take) cells[base + __popc(m & ((1u << lane) - 1u))] = row * W + x;
    base += __popc(m);
  }
}

cudaError_t launch_body_count3(int W, int nRows, const uint8_t* rowBody, const uint32_t* flags, int* counts,
                               cudaStream_t s) {
  body_count3_kernel<<<(unsigned)((nRows * 32LL + 255) / 256), 256, 0, s>>>(W, nRows, rowBody, flags, counts);
  return cudaGetLastError();
}

cudaError_t launch_body_write3(int W, int nRows, const uint8_t* rowBody, const uint32_t* flags, const int* offsets,
                               int* cells, cudaStream_t s) {
  body_write3_kernel<<<(unsigned)((nRows * 32LL + 255) / 256), 256, 0, s>>>(W, nRows, rowBody, flags, offsets, cells);
  return cudaGetLastError();
}

#define CELLS_DISPATCH(prec, expr)        \
  switch (prec) {                         \
    case 0: { using C = CodecF32; expr; } break; \
    case 1: { using C = CodecF16; expr; } break; \
    case 2: { using C = CodecBF16; expr; } break; \
    case 3: { using C = CodecF64; expr; } break; \
    default: return cudaErrorInvalidValue; \
  }

cudaError_t launch_flags3(int precision, const AuxLaunch3& a, const float* sdf, uint32_t* flags, uint8_t* rowBody,
                          void* fA, void* fB, const float4* mac, cudaStream_t s) {
  CELLS_DISPATCH(precision, (flags3_kernel<C><<<blocks_for(a.N, 256), 256, 0, s>>>(
                                a, sdf, flags, rowBody, (typename C::S*)fA, (typename C::S*)fB, mac)));
  return cudaGetLastError();
}

cudaError_t launch_links3(int precision, const AuxLaunch3& a, const int* cells, int n, const uint32_t* flags,
                          const float* sdf, const BodyLinks3& L, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  CELLS_DISPATCH(precision, (links3_kernel<C><<<blocks_for(n, 128), 128, 0, s>>>(a, cells, n, flags, sdf, L)));
  return cudaGetLastError();
}

cudaError_t launch_init3(int precision, const AuxLaunch3& a, void* fA, void* fB, const uint32_t* flags,
                         const float4* mac, cudaStream_t s) {
  CELLS_DISPATCH(precision, (init3_kernel<C><<<blocks_for(a.N, 256), 256, 0, s>>>(
                                a, (typename C::S*)fA, (typename C::S*)fB, flags, mac)));
  return cudaGetLastError();
}

cudaError_t launch_macro3(int precision, const AuxLaunch3& a, const void* f, const uint32_t* flags, float4* mac,
                          DevState3* st, cudaStream_t s) {
  CELLS_DISPATCH(precision, (macro3_kernel<C><<<blocks_for(a.N, 256), 256, 0, s>>>(
                                a, (const typename C::S*)f, flags, mac, st)));
  return cudaGetLastError();
}

cudaError_t launch_mass3(int precision, const AuxLaunch3& a, const void* f, const uint32_t* flags, double* partials,
                         int nPartials, double* out, cudaStream_t s) {
  CELLS_DISPATCH(precision, (mass3_partial_kernel<C><<<nPartials, 256, 0, s>>>(
                                a, (const typename C::S*)f, flags, partials)));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  sum_partials_kernel<<<1, 256, 0, s>>>(partials, nPartials, out);
  return cudaGetLastError();
}

cudaError_t launch_set_state3(int precision, DevState3* st, int which, unsigned step, double uIn0, double uIn1,
                              cudaStream_t s) {
  CELLS_DISPATCH(precision, (set_state3_kernel<C><<<1, 1, 0, s>>>(st, which, step, uIn0, uIn1)));
  return cudaGetLastError();
}

}  // namespace cells
