// rankine.cuh -- analytic 1/r source integral and its gradient over a flat
// triangle or quadrilateral at a field point (J.N. Newman 1986).
//
// Follows SGLINTBD_TRI / SGLINTBD_QUAD of HAMS-MREL src/SingularIntgr.f90
// (:44-245, :252-445): the panel is projected on its mean plane through the
// centre (quad) or the foot of the altitude (triangle), and each edge adds
// an atan2 (solid angle) and a log term.  The two panel types keep the
// reference's opposite orientation conventions.
#pragma once
#include <math.h>

namespace hams {

struct rk4 {
  double s, dx, dy, dz;  // SIJ and DIJ(1:3)
};

__device__ inline rk4 sglint_tri(const double xf[3], const double q[3][3]) {
  double p12[3], p13[3], po[3], po3[3], ui[3], uj[3], uk[3];
  for (int j = 0; j < 3; ++j) {
    p12[j] = q[1][j] - q[0][j];
    p13[j] = q[2][j] - q[0][j];
  }
  double n12s = p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2];
  double alfa = (p12[0] * p13[0] + p12[1] * p13[1] + p12[2] * p13[2]) / n12s;
  for (int j = 0; j < 3; ++j) {
    po[j] = q[0][j] + alfa * p12[j];
    po3[j] = q[2][j] - po[j];
  }
  double n12 = sqrt(n12s), n3 = sqrt(po3[0] * po3[0] + po3[1] * po3[1] + po3[2] * po3[2]);
  for (int j = 0; j < 3; ++j) {
    ui[j] = p12[j] / n12;
    uj[j] = po3[j] / n3;
  }
  uk[0] = ui[1] * uj[2] - ui[2] * uj[1];
  uk[1] = ui[2] * uj[0] - ui[0] * uj[2];
  uk[2] = ui[0] * uj[1] - ui[1] * uj[0];
  double pf[3] = {xf[0] - po[0], xf[1] - po[1], xf[2] - po[2]};
  double x = ui[0] * pf[0] + ui[1] * pf[1] + ui[2] * pf[2];
  double y = uj[0] * pf[0] + uj[1] * pf[1] + uj[2] * pf[2];
  double z = uk[0] * pf[0] + uk[1] * pf[1] + uk[2] * pf[2];
  double d1[3] = {q[0][0] - po[0], q[0][1] - po[1], q[0][2] - po[2]};
  double d2[3] = {q[1][0] - po[0], q[1][1] - po[1], q[1][2] - po[2]};
  double ksi[4], eta[4];
  ksi[0] = -copysign(1.0, alfa) * sqrt(d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
  eta[0] = 0.0;
  ksi[1] = 0.0;
  eta[1] = n3;
  ksi[2] = sqrt(d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2]);
  eta[2] = 0.0;
  ksi[3] = ksi[0];
  eta[3] = eta[0];
  double st = 0.0, sxt = 0.0, syt = 0.0, szt = 0.0;
  for (int i = 0; i < 3; ++i) {
    double dk = ksi[i + 1] - ksi[i], de = eta[i + 1] - eta[i];
    double ax = ksi[i] - x, ay = eta[i] - y, bx = ksi[i + 1] - x, by = eta[i + 1] - y;
    double r1 = sqrt(ax * ax + ay * ay + z * z), r2 = sqrt(bx * bx + by * by + z * z);
    double l = sqrt(dk * dk + de * de);
    double b1 = de * (ax * ax + z * z) - dk * ax * ay, a1 = r1 * z * dk;
    double b2 = de * (bx * bx + z * z) - dk * bx * by, a2 = r2 * z * dk;
    if (!(fabs(z) < 1.0e-6)) szt += atan2(b1 * a2 - b2 * a1, a1 * a2 + b1 * b2);
    if (fabs(r1 + r2 - l) < 1.0e-6) continue;
    double lg = log((r1 + r2 + l) / (r1 + r2 - l));
    sxt = sxt - de / l * lg;
    syt = syt + dk / l * lg;
    st = st + (de * (x - ksi[i]) - dk * (y - eta[i])) / l * lg;
  }
  st = st - z * szt;
  rk4 o;
  o.s = st;
  o.dx = ui[0] * sxt + uj[0] * syt + uk[0] * szt;
  o.dy = ui[1] * sxt + uj[1] * syt + uk[1] * szt;
  o.dz = ui[2] * sxt + uj[2] * syt + uk[2] * szt;
  return o;
}

__device__ inline rk4 sglint_quad(const double xf[3], const double q[4][3]) {
  double po[3], pov[4][3], un[3], ui[3], uj[3], uk[3];
  for (int j = 0; j < 3; ++j) po[j] = (q[0][j] + q[1][j] + q[2][j] + q[3][j]) / 4.0;
  for (int v = 0; v < 4; ++v)
    for (int j = 0; j < 3; ++j) pov[v][j] = q[v][j] - po[j];
  un[0] = pov[0][1] * pov[1][2] - pov[0][2] * pov[1][1];
  un[1] = pov[0][2] * pov[1][0] - pov[0][0] * pov[1][2];
  un[2] = pov[0][0] * pov[1][1] - pov[0][1] * pov[1][0];
  double n1 = sqrt(pov[0][0] * pov[0][0] + pov[0][1] * pov[0][1] + pov[0][2] * pov[0][2]);
  double nu = sqrt(un[0] * un[0] + un[1] * un[1] + un[2] * un[2]);
  for (int j = 0; j < 3; ++j) {
    ui[j] = pov[0][j] / n1;
    uk[j] = un[j] / nu;
  }
  uj[0] = uk[1] * ui[2] - uk[2] * ui[1];
  uj[1] = uk[2] * ui[0] - uk[0] * ui[2];
  uj[2] = uk[0] * ui[1] - uk[1] * ui[0];
  double pf[3] = {xf[0] - po[0], xf[1] - po[1], xf[2] - po[2]};
  double x = ui[0] * pf[0] + ui[1] * pf[1] + ui[2] * pf[2];
  double y = uj[0] * pf[0] + uj[1] * pf[1] + uj[2] * pf[2];
  double z = uk[0] * pf[0] + uk[1] * pf[1] + uk[2] * pf[2];
  double ksi[5], eta[5];
  for (int v = 0; v < 4; ++v) {
    double d = uk[0] * pov[v][0] + uk[1] * pov[v][1] + uk[2] * pov[v][2];
    double p0 = pov[v][0] - d * uk[0], p1 = pov[v][1] - d * uk[1], p2 = pov[v][2] - d * uk[2];
    ksi[v] = ui[0] * p0 + ui[1] * p1 + ui[2] * p2;
    eta[v] = uj[0] * p0 + uj[1] * p1 + uj[2] * p2;
  }
  ksi[4] = ksi[0];
  eta[4] = eta[0];
  double st = 0.0, sxt = 0.0, syt = 0.0, szt = 0.0;
  for (int i = 0; i < 4; ++i) {
    double dk = ksi[i + 1] - ksi[i], de = eta[i + 1] - eta[i];
    double ax = ksi[i] - x, ay = eta[i] - y, bx = ksi[i + 1] - x, by = eta[i + 1] - y;
    double r1 = sqrt(ax * ax + ay * ay + z * z), r2 = sqrt(bx * bx + by * by + z * z);
    double l = sqrt(dk * dk + de * de);
    if (fabs(l) < 1.0e-8) continue;  // coincident vertices (degenerate quad)
    double b1 = de * (ax * ax + z * z) - dk * ax * ay, a1 = r1 * z * dk;
    double b2 = de * (bx * bx + z * z) - dk * bx * by, a2 = r2 * z * dk;
    if (!(fabs(z) < 1.0e-6)) szt += atan2(b1 * a2 - b2 * a1, a1 * a2 + b1 * b2);
    if (fabs(r1 + r2 - l) < 1.0e-6) continue;
    double lg = log((r1 + r2 + l) / (r1 + r2 - l));
    sxt = sxt - de / l * lg;
    syt = syt + dk / l * lg;
    st = st - (de * (x - ksi[i]) - dk * (y - eta[i])) / l * lg;
  }
  st = st + z * szt;
  rk4 o;
  o.s = st;
  o.dx = -(ui[0] * sxt + uj[0] * syt + uk[0] * szt);
  o.dy = -(ui[1] * sxt + uj[1] * syt + uk[1] * szt);
  o.dz = -(ui[2] * sxt + uj[2] * syt + uk[2] * szt);
  return o;
}

}  // namespace hams
