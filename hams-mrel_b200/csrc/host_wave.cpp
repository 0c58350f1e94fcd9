// host_wave.cpp -- per-frequency wave properties on the host.
//
// hams_wave_properties replaces CalWaveProperts (src/ImplementSubs.f90:40-151)
// and DISPERSION (src/WavDynSubs.f90:40-127, J.N. Newman 1990): Newton-Halley
// iterations for k tanh(kh) = w^2/g and the 199 evanescent roots
// mu tan(mu h) = -w^2/g.  DISPERSION carries its own g = 9.807 (:58) while
// the rest of the program uses the caller's g; both are kept, so a deck
// gives the same roots as the reference.  This runs once per frequency and
// is a few microseconds of scalar work, so it stays on the host.
#include <cmath>
#include <cstring>

#include "../../include/hams_gpu.h"

#include "host_wave.h"

namespace {
constexpr double kPi = 3.141592653589793;
}  // namespace

void hams_dispersion(double* wvn, int nrt, double w, double h) {
  const double g = 9.807;
  double x = w * w * h / g, y, t;
  if (x > 0.0 && x <= 2.0) {
    y = std::sqrt(x) * (0.9994 + 0.1701 * x + (double)0.0305f * x * x);  // 0.0305 is single precision (:71)
  } else {
    t = x * std::exp(-2.0 * x);
    y = x + 2.0 * t - 6.0 * t * t;
  }
  if (std::fabs(y - x) < (double)1.E-10f) {
    wvn[0] = x / h;
  } else {
    double exx = 1.0;
    for (int it = 0; exx > 1.0e-10 && it < 200; ++it) {
      double trial = y, dnm = trial * trial - x * x;
      double fun = std::log((trial + x) / (trial - x)) / 2.0 - trial;
      double dfun = -x / dnm - 1.0;
      double d2fun = 2.0 * x * trial / (dnm * dnm);
      y = trial - fun / dfun * (1.0 + (fun / dfun) * (d2fun / dfun) / 2.0);
      exx = std::fabs(y - trial);
    }
    wvn[0] = y / h;
  }
  double u = 3.0 * x / (7.0 + 3.0 * x);
  t = 0.0159 + 0.1032 * u + 4.3152 * u * u - 2.8768 * u * u * u;
  for (int i = 2; i <= nrt; ++i) {
    double exx = 1.0;
    for (int it = 0; exx > 1.0e-10 && it < 200; ++it) {
      double trial = t, yy = (i - 1) * kPi - trial, dnm = yy * yy + x * x;
      double fun = std::atan2(x, yy) - trial;
      double dfun = x / dnm - 1.0;
      double d2fun = 2.0 * x * trial / (dnm * dnm);
      t = trial - fun / dfun * (1.0 + (fun / dfun) * (d2fun / dfun) / 2.0);
      exx = std::fabs(t - trial);
    }
    wvn[i - 1] = ((i - 1) * kPi - t) / h;
    t = t - kPi * x / (x * x + kPi * i * (kPi * (i - 1) - t));
  }
}

extern "C" int hams_wave_properties(int32_t inft, double value, double depth, double g, int32_t sybo_kk,
                                    hams_wave* o) {
  if (!o) return HAMS_ERR_ARG;
  std::memset(o, 0, sizeof(*o));
  if (sybo_kk == 1) {  // zero-frequency limit
    o->tp = -1.0;
    o->wl = -1.0;
    return HAMS_OK;
  }
  if (sybo_kk == 2) {  // infinite-frequency limit
    o->v = o->wk = o->w1 = -1.0;
    return HAMS_OK;
  }
  if (!(g > 0.0) || !(value > 0.0)) return HAMS_ERR_ARG;
  const bool deep = depth <= 0.0;
  switch (inft) {
    case 1:
      o->v = value;
      o->w1 = std::sqrt(g * o->v);
      if (deep) o->wk = o->v;
      else { hams_dispersion(o->wvn, HAMS_NK, o->w1, depth); o->wk = o->wvn[0]; }
      o->wl = 2.0 * kPi / o->wk;
      o->tp = 2.0 * kPi / o->w1;
      break;
    case 2:
      o->wk = value;
      o->v = deep ? o->wk : o->wk * std::tanh(o->wk * depth);
      o->w1 = std::sqrt(g * o->v);
      if (!deep) hams_dispersion(o->wvn, HAMS_NK, o->w1, depth);
      o->wl = 2.0 * kPi / o->wk;
      o->tp = 2.0 * kPi / o->w1;
      break;
    case 3:
      o->w1 = value;
      o->v = o->w1 * o->w1 / g;
      if (deep) o->wk = o->v;
      else { hams_dispersion(o->wvn, HAMS_NK, o->w1, depth); o->wk = o->wvn[0]; }
      o->wl = 2.0 * kPi / o->wk;
      o->tp = 2.0 * kPi / o->w1;
      break;
    case 4:
      o->tp = value;
      o->w1 = 2.0 * kPi / o->tp;
      o->v = o->w1 * o->w1 / g;
      if (deep) o->wk = o->v;
      else { hams_dispersion(o->wvn, HAMS_NK, o->w1, depth); o->wk = o->wvn[0]; }
      o->wl = 2.0 * kPi / o->wk;
      break;
    case 5:
      o->wl = value;
      o->wk = 2.0 * kPi / o->wl;
      o->v = deep ? o->wk : o->wk * std::tanh(o->wk * depth);
      o->w1 = std::sqrt(g * o->v);
      if (!deep) hams_dispersion(o->wvn, HAMS_NK, o->w1, depth);
      break;
    default:
      return HAMS_ERR_ARG;
  }
  return HAMS_OK;
}
