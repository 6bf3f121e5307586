// Star-shaped body of the shape-gradient problem (no counterpart in the reference): its SDF, and the
// chain rule from the adjoint's dJ/dSDF to the body's 16 spherical-harmonic coefficients.
//
// The body is r(theta, phi) = r0 (1 + sum_k coef[k] Y_k(theta, phi)) about (cx, cy, cz), theta the
// polar angle from +z and phi = atan2(dy, dx); Y_k are the orthonormal real spherical harmonics of
// degree l <= 3 in the order (l, m) = (0,0), (1,-1), (1,0), (1,1), (2,-2) ... (3,3), without the
// Condon-Shortley phase (m > 0: sqrt(2) N P_l^m cos(m phi); m < 0: sqrt(2) N P_l^|m| sin(|m| phi)).
// Its SDF value is the signed radial distance |p - c| - r(theta, phi), stamped as min(sdf, value)
// over the body's bounding box grown by the same 3-cell margin as every other shape
// (src/geometry3d.ts:15-27). Host code only: these run once per shape, not per step.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/cells.h"
#include "device.h"
#include "solver3d_state.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kStampMargin = 3;

// The 16 harmonics at one direction, from the unit-sphere coordinates x = cos(theta),
// s = sin(theta) and the azimuth phi.
void star_harmonics(double x, double s, double phi, double Y[16]) {
  // associated Legendre P_l^m(x), m >= 0, without the Condon-Shortley phase
  const double P[4][4] = {
      {1.0, 0, 0, 0},
      {x, s, 0, 0},
      {0.5 * (3 * x * x - 1), 3 * x * s, 3 * s * s, 0},
      {0.5 * (5 * x * x * x - 3 * x), 1.5 * (5 * x * x - 1) * s, 15 * x * s * s, 15 * s * s * s},
  };
  static const double fact[7] = {1, 1, 2, 6, 24, 120, 720};
  int k = 0;
  for (int l = 0; l <= 3; l++) {
    for (int m = -l; m <= l; m++, k++) {
      const int am = m < 0 ? -m : m;
      const double norm = std::sqrt((2 * l + 1) / (4 * kPi) * fact[l - am] / fact[l + am]);
      if (m == 0)
        Y[k] = norm * P[l][0];
      else if (m > 0)
        Y[k] = std::sqrt(2.0) * norm * P[l][am] * std::cos(m * phi);
      else
        Y[k] = std::sqrt(2.0) * norm * P[l][am] * std::sin(am * phi);
    }
  }
}

// Direction of node (x, y, z) from the centre: fills Y and returns the distance.
double star_direction(const CellsStar3D& b, double x, double y, double z, double Y[16]) {
  const double dx = x - b.cx, dy = y - b.cy, dz = z - b.cz;
  const double rr = std::sqrt(dx * dx + dy * dy + dz * dz);
  const double c = rr > 0 ? std::min(1.0, std::max(-1.0, dz / rr)) : 1.0;
  const double theta = std::acos(c);
  star_harmonics(std::cos(theta), std::sin(theta), std::atan2(dy, dx), Y);
  return rr;
}

bool star_valid(const CellsStar3D* b, int32_t W, int32_t H, int32_t D) {
  if (!b || W <= 0 || H <= 0 || D <= 0) return false;
  if (!std::isfinite(b->cx) || !std::isfinite(b->cy) || !std::isfinite(b->cz) || !std::isfinite(b->r0)) return false;
  for (double c : b->coef)
    if (!std::isfinite(c)) return false;
  return b->r0 > 0;
}

}  // namespace

extern "C" int cells3d_star_sdf(float* sdf, int32_t W, int32_t H, int32_t D, const CellsStar3D* star) {
  if (!sdf || !star_valid(star, W, H, D)) {
    cells::g_create_error = "cells3d_star_sdf: null buffer, non-positive size or radius, or a non-finite parameter";
    return CELLS_E_INVALID;
  }
  const CellsStar3D& b = *star;
  double sumAbs = 0;
  for (double c : b.coef) sumAbs += std::fabs(c);
  // |Y_lm| <= sqrt(7 / (4 pi)) for l <= 3 (the l = 3, m = 0 harmonic at the poles)
  const double rmax = b.r0 * (1 + sumAbs * 0.5 * std::sqrt(7 / kPi)) + 1;
  const long long x0 = std::max(0LL, (long long)std::floor(b.cx - rmax - kStampMargin));
  const long long y0 = std::max(0LL, (long long)std::floor(b.cy - rmax - kStampMargin));
  const long long z0 = std::max(0LL, (long long)std::floor(b.cz - rmax - kStampMargin));
  const long long x1 = std::min((long long)W - 1, (long long)std::ceil(b.cx + rmax + kStampMargin));
  const long long y1 = std::min((long long)H - 1, (long long)std::ceil(b.cy + rmax + kStampMargin));
  const long long z1 = std::min((long long)D - 1, (long long)std::ceil(b.cz + rmax + kStampMargin));
  double Y[16];
  for (long long z = z0; z <= z1; z++)
    for (long long y = y0; y <= y1; y++)
      for (long long x = x0; x <= x1; x++) {
        const double rr = star_direction(b, (double)x, (double)y, (double)z, Y);
        double s = 0;
        for (int k = 0; k < 16; k++) s += b.coef[k] * Y[k];
        const double v = rr - b.r0 * (1 + s);
        float& cell = sdf[((size_t)z * H + (size_t)y) * W + (size_t)x];
        cell = (float)std::min((double)cell, v);
      }
  return CELLS_OK;
}

extern "C" int cells3d_star_coef_gradient(const CellsStar3D* star, int32_t W, int32_t H, int32_t D,
                                          const double* dJ_dsdf, double* dJ_dcoef16) {
  if (!dJ_dsdf || !dJ_dcoef16 || !star_valid(star, W, H, D)) {
    cells::g_create_error =
        "cells3d_star_coef_gradient: null buffer, non-positive size or radius, or a non-finite parameter";
    return CELLS_E_INVALID;
  }
  const long long N = (long long)W * H * D;
  double acc[16] = {0};
  double Y[16];
  for (long long n = 0; n < N; n++) {
    const double g = dJ_dsdf[n];
    if (g == 0) continue;
    const long long x = n % W, y = (n / W) % H, z = n / ((long long)W * H);
    star_direction(*star, (double)x, (double)y, (double)z, Y);
    // d(sdf)/d(coef_k) = -r0 Y_k at the node
    for (int k = 0; k < 16; k++) acc[k] += g * (-star->r0 * Y[k]);
  }
  std::copy(acc, acc + 16, dJ_dcoef16);
  return CELLS_OK;
}

extern "C" int cells3d_adjoint_backward_star(Cells3D* h, const CellsStar3D* star, double* dJ_dcoef16,
                                             double* dJ_du_in) {
  if (!h) return CELLS_E_INVALID;
  Cells3DInfo info;
  int rc = cells3d_get_info(h, &info);
  if (rc != CELLS_OK) return rc;
  if (!dJ_dcoef16 || !star_valid(star, info.W, info.H, info.D)) {
    h->lastError = "adjoint_backward_star: null gradient buffer, non-positive radius or a non-finite parameter";
    return CELLS_E_INVALID;
  }
  std::vector<double> dsdf((size_t)info.N);
  rc = cells3d_adjoint_backward(h, nullptr, dsdf.data(), dJ_du_in, nullptr);
  if (rc != CELLS_OK) return rc;
  return cells3d_star_coef_gradient(star, info.W, info.H, info.D, dsdf.data(), dJ_dcoef16);
}
