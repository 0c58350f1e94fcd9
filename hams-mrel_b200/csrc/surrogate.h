// surrogate.h -- shape, input scaling and parameter layout of the MLP
// surrogate of the finite-depth evanescent Green function (surrogate.cu).
//
// The network maps four nondimensional inputs of a panel pair -- R/h,
// (zq + h)/h, (zp + h)/h (source and field depths above the bottom) and
// K = k0 h tanh(k0 h) (the dispersion parameter of the frequency) -- to the
// sum of the evanescent modes of FINGREEN3D's wave term, in depth units
// h = 1 and scaled to order one:
//   t0 = X (fg0 - prop0 - rk0),  t1 = X^2 (fg1 - prop1 - rk1),  t2 = X^2 (fg2 - prop2 - rk2)
// (real parts), X = R/h, fg = G and its R / zq derivatives before the 1/r,
// 1/r1 terms are added back (FinGreen3D.f90:124-150), prop = the
// propagating-mode part (FinGreen3D.f90:311-322) and rk = the point-source
// terms the series subtract (FinGreen3D.f90:349-359); prop and rk stay exact.
#pragma once

namespace sg {

constexpr int kIn = 4, kOut = 3, kWidth = 128, kHidden = 4, kLayers = kHidden + 1;
// training domain (pairs outside it keep the series)
constexpr double kXmin = 0.05, kXmax = 3.0, kZmin = 0.5, kZmax = 1.0, kKmin = 0.04, kKmax = 40.0;

__host__ __device__ constexpr int layer_in(int l) { return l == 0 ? kIn : kWidth; }
__host__ __device__ constexpr int layer_out(int l) { return l == kLayers - 1 ? kOut : kWidth; }
// parameters: for each layer W (out x in, column-major) then b (out); then the
// output mean and scale the network's outputs are normalised by
__host__ __device__ constexpr int w_off(int l) {
  int o = 0;
  for (int k = 0; k < l; ++k) o += layer_in(k) * layer_out(k) + layer_out(k);
  return o;
}
__host__ __device__ constexpr int b_off(int l) { return w_off(l) + layer_in(l) * layer_out(l); }
constexpr int kNormOff = w_off(kLayers);
constexpr int kParams = kNormOff + 2 * kOut;

__host__ __device__ inline bool in_domain(double X, double Zq, double Zp, double K) {
  return X >= kXmin && X <= kXmax && Zq >= kZmin && Zq <= kZmax && Zp >= kZmin && Zp <= kZmax && K >= kKmin &&
         K <= kKmax;
}

// inputs mapped to [-1, 1]: log X, Zq, Zp, log K
__host__ __device__ inline void features(double X, double Zq, double Zp, double K, float f[kIn]) {
  f[0] = (float)(2.0 * log(X / kXmin) / log(kXmax / kXmin) - 1.0);
  f[1] = (float)(2.0 * (Zq - kZmin) / (kZmax - kZmin) - 1.0);
  f[2] = (float)(2.0 * (Zp - kZmin) / (kZmax - kZmin) - 1.0);
  f[3] = (float)(2.0 * log(K / kKmin) / log(kKmax / kKmin) - 1.0);
}

// The point-source terms removed by the series (FinGreen3D.f90:349-359):
// -(1/r + 1/r1) and the R and zq derivatives of that, at horizontal distance
// R, source depth zq, field depth zp (any length unit).
__host__ __device__ inline void rankine_parts(double R, double zq, double zp, double rk[3]) {
  double sr = sqrt(R * R + (zq - zp) * (zq - zp)), sr1 = sqrt(R * R + (zq + zp) * (zq + zp));
  rk[0] = -(1.0 / sr + 1.0 / sr1);
  rk[1] = R / sr / (sr * sr) + R / sr1 / (sr1 * sr1);
  rk[2] = (zq - zp) / sr / (sr * sr) + (zq + zp) / sr1 / (sr1 * sr1);
}

}  // namespace sg
