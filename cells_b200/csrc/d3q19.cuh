// D3Q19 lattice constants, storage codecs and the shared device/host structures of the 3D engine.
//
// Lattice: src/lattice3d.ts:4-26 (velocity set with odd i and i+1 opposite, weights 1/3, 1/18, 1/36,
// MIRROR_Y/Z, flag bits 19-21). Codec: src/shaders/common3d.ts:52-63 (f16 scaled by 2^15 and
// clamped to +-1.99 before the store); bf16 and f64 are additions of this engine.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cells {

constexpr int Q3 = 19;
constexpr uint32_t FLAG3_SOLID = 1u << 19;
constexpr uint32_t FLAG3_INLET = 1u << 20;
constexpr uint32_t FLAG3_OUTLET = 1u << 21;
constexpr int HISTORY_LEN = 8192;  // src/shaders/aux3d.ts:5

__host__ __device__ __forceinline__ constexpr int cx3(int i) {
  constexpr int v[Q3] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0};
  return v[i];
}
__host__ __device__ __forceinline__ constexpr int cy3(int i) {
  constexpr int v[Q3] = {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1};
  return v[i];
}
__host__ __device__ __forceinline__ constexpr int cz3(int i) {
  constexpr int v[Q3] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1};
  return v[i];
}
__host__ __device__ __forceinline__ constexpr int opp3(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
// Direction with its y (z) component negated, for slip on the y (z) faces.
__host__ __device__ __forceinline__ constexpr int mirror_y3(int i) {
  constexpr int v[Q3] = {0, 1, 2, 4, 3, 5, 6, 13, 14, 9, 10, 18, 17, 7, 8, 15, 16, 12, 11};
  return v[i];
}
__host__ __device__ __forceinline__ constexpr int mirror_z3(int i) {
  constexpr int v[Q3] = {0, 1, 2, 3, 4, 6, 5, 7, 8, 15, 16, 17, 18, 13, 14, 9, 10, 11, 12};
  return v[i];
}

template <class R>
__host__ __device__ __forceinline__ R w3(int i) {
  return i == 0 ? R(1) / R(3) : (i <= 6 ? R(1) / R(18) : R(1) / R(36));
}

template <class R>
struct Vec4;
template <>
struct Vec4<float> {
  using T = float4;
};
template <>
struct Vec4<double> {
  using T = double4;
};

// ---------------- storage codecs ----------------
// load/enc convert between stored values and populations (f_i - w_i). raw/enc_raw work in storage
// units, populations times SCALE: the step kernel computes in those units, which is exact because
// SCALE is a power of two, so it gives the same bits as scaling every load and store.
struct CodecF32 {
  using S = float;
  using R = float;
  static constexpr int prec = 0;
  static constexpr float SCALE = 1.0f;
  __device__ __forceinline__ static R load(const S* p) { return __ldg(p); }
  __device__ __forceinline__ static S enc(R v) { return v; }
  __device__ __forceinline__ static R raw(const S* p) { return __ldg(p); }
  __device__ __forceinline__ static S enc_raw(R v) { return v; }
  // x-pairs (cells x0, x0 + 1, x0 even): one 8-byte word, or two 4-byte loads for a shifted pair
  using Pair = float2;
  __device__ __forceinline__ static Pair ld_pair(const S* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
  __device__ __forceinline__ static Pair ld_pair2(const S* p0, const S* p1) {
    return make_float2(__ldg(p0), __ldg(p1));
  }
  __device__ __forceinline__ static R lo(Pair w) { return w.x; }
  __device__ __forceinline__ static R hi(Pair w) { return w.y; }
  __device__ __forceinline__ static void st_pair(S* p, R a, R b) { *reinterpret_cast<float2*>(p) = make_float2(a, b); }
  __device__ __forceinline__ static void st_pair_fast(S* p, R a, R b) { st_pair(p, a, b); }
};
struct CodecF16 {
  using S = __half;
  using R = float;
  static constexpr int prec = 1;
  static constexpr float SCALE = 32768.0f;
  __device__ __forceinline__ static R load(const S* p) { return __half2float(__ldg(p)) * (1.0f / 32768.0f); }
  __device__ __forceinline__ static S enc(R v) {
    return __float2half_rn(fminf(fmaxf(v, -1.99f), 1.99f) * 32768.0f);
  }
  __device__ __forceinline__ static R raw(const S* p) { return __half2float(__ldg(p)); }
  // clamp(v, -1.99, 1.99) * 2^15 == clamp(v * 2^15, -1.99 * 2^15, 1.99 * 2^15): both products are exact
  __device__ __forceinline__ static S enc_raw(R v) {
    return __float2half_rn(fminf(fmaxf(v, -1.99f * 32768.0f), 1.99f * 32768.0f));
  }
  // Two values in the halves of one 32-bit word (lo = first cell). Rounding first and clamping the
  // halves to +-65216 gives the same bits as enc_raw: 65216 is the f16 nearest to 1.99 * 2^15, and
  // rounding is monotonic, so every value beyond the clamp bound rounds to 65216 or further out.
  __device__ __forceinline__ static R lo(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)w)); }
  __device__ __forceinline__ static R hi(uint32_t w) { return __half2float(__ushort_as_half((unsigned short)(w >> 16))); }
  __device__ __forceinline__ static uint32_t pack2(R a, R b) {
    __half2 h = __floats2half2_rn(a, b);
    const __half2 bound = __float2half2_rn(65216.0f);
    h = __hmin2(__hmax2(h, __hneg2(bound)), bound);
    return *reinterpret_cast<uint32_t*>(&h);
  }
  // The fast-arithmetic store: one saturating conversion, which bounds the stored values at
  // +-65504 (|f - w| <= 1.999) instead of the reference's +-1.99 clamp. Both keep the store finite;
  // they differ only for |f - w| > 1.99, far outside any stable flow.
  __device__ __forceinline__ static uint32_t pack2_fast(R a, R b) {
    uint32_t d;
    asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
    return d;
  }
  using Pair = uint32_t;
  __device__ __forceinline__ static Pair ld_pair(const S* p) { return __ldg(reinterpret_cast<const unsigned int*>(p)); }
  __device__ __forceinline__ static Pair ld_pair2(const S* p0, const S* p1) {
    return (uint32_t)__ldg(reinterpret_cast<const unsigned short*>(p0)) |
           ((uint32_t)__ldg(reinterpret_cast<const unsigned short*>(p1)) << 16);
  }
  __device__ __forceinline__ static void st_pair(S* p, R a, R b) { *reinterpret_cast<uint32_t*>(p) = pack2(a, b); }
  __device__ __forceinline__ static void st_pair_fast(S* p, R a, R b) { *reinterpret_cast<uint32_t*>(p) = pack2_fast(a, b); }
};
struct CodecBF16 {
  using S = __nv_bfloat16;
  using R = float;
  static constexpr int prec = 2;
  static constexpr float SCALE = 1.0f;
  __device__ __forceinline__ static R load(const S* p) { return __bfloat162float(__ldg(p)); }
  __device__ __forceinline__ static S enc(R v) { return __float2bfloat16_rn(v); }
  __device__ __forceinline__ static R raw(const S* p) { return __bfloat162float(__ldg(p)); }
  __device__ __forceinline__ static S enc_raw(R v) { return __float2bfloat16_rn(v); }
  __device__ __forceinline__ static R lo(uint32_t w) { return __uint_as_float(w << 16); }
  __device__ __forceinline__ static R hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }
  __device__ __forceinline__ static uint32_t pack2(R a, R b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
  }
  __device__ __forceinline__ static uint32_t pack2_fast(R a, R b) { return pack2(a, b); }
  using Pair = uint32_t;
  __device__ __forceinline__ static Pair ld_pair(const S* p) { return __ldg(reinterpret_cast<const unsigned int*>(p)); }
  __device__ __forceinline__ static Pair ld_pair2(const S* p0, const S* p1) {
    return (uint32_t)__ldg(reinterpret_cast<const unsigned short*>(p0)) |
           ((uint32_t)__ldg(reinterpret_cast<const unsigned short*>(p1)) << 16);
  }
  __device__ __forceinline__ static void st_pair(S* p, R a, R b) { *reinterpret_cast<uint32_t*>(p) = pack2(a, b); }
  __device__ __forceinline__ static void st_pair_fast(S* p, R a, R b) { *reinterpret_cast<uint32_t*>(p) = pack2_fast(a, b); }
};
struct CodecF64 {
  using S = double;
  using R = double;
  static constexpr int prec = 3;
  static constexpr double SCALE = 1.0;
  __device__ __forceinline__ static R load(const S* p) { return __ldg(p); }
  __device__ __forceinline__ static S enc(R v) { return v; }
  __device__ __forceinline__ static R raw(const S* p) { return __ldg(p); }
  __device__ __forceinline__ static S enc_raw(R v) { return v; }
};

// Per-handle device state. step[] and uIn[] are double-buffered by parity: the step kernel of
// parity p reads slot p and block 0 writes slot p^1 for the next step, so no kernel ever reads a
// slot that the same kernel writes.
struct DevState3 {
  unsigned int step[2];
  unsigned int sample;  // force samples written so far (the reference's histState)
  unsigned int done;    // force blocks finished in the current sampled step
  unsigned int status;  // bit 0: non-finite force sample, bit 1: non-finite macro value
  unsigned int pad[3];
  double uIn[2];
  // the inlet's 19 equilibrium values feq(i, 1, uIn, 0, 0) in storage units, per parity slot (they
  // depend on uIn alone, so a step reads them instead of every inlet cell computing them)
  double inletEq[2][Q3];
};

// Launch-invariant parameters of a step (kernel arguments). The x-dependent relaxation rate and
// absorbing strength come from a per-x table that the host fills with the reference's arithmetic.
template <class R>
struct StepParams3 {
  int W, H, D, N;
  int nForceBlocks;
  int rampKind;       // 0 none, 1 linear, 2 smoothstep
  int rampEvery;
  int pad;
  double rampTarget;
  double rampSteps;
  R lambda;
  R smagC2;
};

}  // namespace cells
