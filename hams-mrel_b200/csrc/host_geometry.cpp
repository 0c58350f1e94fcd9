// host_geometry.cpp -- frequency-independent panel geometry on the host.
//
// hams_prepare_geometry replaces CalNormals / CalNormalsMulti
// (src/ReadPanelMesh.f90:110-150, src/ReadPanelMeshMulti.f90:122-168) and
// the routines of src/NormalProcess.f90 they call: panel centre as the
// vertex average (CalPanelCentre :134, degenerate quads included), area as
// the sum of two triangles by the cancellation-free Heron form
// (CalPanelArea :171, CalDeltaArea_Improved :373), longest edge
// (CalPanelChartLength :401), unit normal from the cross product of the
// diagonals (CalTransNormals :74) and the rotational normals r x n about
// each body's reference point (CalRotNormals :46).  It runs once per mesh.
#include <cmath>

#include "../../include/hams_gpu.h"

namespace {

double tri_area(const double* p1, const double* p2, const double* p3) {
  double v21[3], v13[3], v23[3];
  for (int k = 0; k < 3; ++k) {
    v21[k] = p1[k] - p2[k];
    v23[k] = p3[k] - p2[k];
    v13[k] = p3[k] - p1[k];
  }
  double a = std::sqrt(v21[0] * v21[0] + v21[1] * v21[1] + v21[2] * v21[2]);
  double b = std::sqrt(v13[0] * v13[0] + v13[1] * v13[1] + v13[2] * v13[2]);
  double c = std::sqrt(v23[0] * v23[0] + v23[1] * v23[1] + v23[2] * v23[2]);
  double l1 = a + (b + c), l2 = c - (a - b), l3 = c + (a - b), l4 = a + (b - c);
  return std::sqrt(l1 * l2 * l3 * l4) / 4.0;
}

}  // namespace

extern "C" int hams_prepare_geometry(int32_t ntnd, const double* xyz, int32_t nelem, const int32_t* ncn,
                                     const int32_t* ncon, int32_t nbody, const int32_t* body_nelem, const double* xr,
                                     double* xyz_p, double* ds, double* pnsz, double* dxyz) {
  if (ntnd <= 0 || nelem <= 0 || nbody <= 0 || !xyz || !ncn || !ncon || !body_nelem || !xr || !xyz_p || !ds ||
      !pnsz || !dxyz)
    return HAMS_ERR_ARG;
  int total = 0;
  for (int b = 0; b < nbody; ++b) total += body_nelem[b];
  if (total != nelem) return HAMS_ERR_ARG;
  const long n = nelem;
  for (long iel = 0; iel < n; ++iel) {
    int nc = ncn[iel];
    if (nc != 3 && nc != 4) return HAMS_ERR_ARG;
    double p[4][3];
    for (int j = 0; j < nc; ++j) {
      int id = ncon[iel + n * j];
      if (id < 1 || id > ntnd) return HAMS_ERR_ARG;
      for (int k = 0; k < 3; ++k) p[j][k] = xyz[(id - 1) + (long)ntnd * k];
    }
    double s[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < nc; ++j)
      for (int k = 0; k < 3; ++k) s[k] = s[k] + p[j][k];
    for (int k = 0; k < 3; ++k) xyz_p[iel + n * k] = s[k] / nc;
    ds[iel] = tri_area(p[0], p[1], p[2]);
    if (nc == 4) ds[iel] = ds[iel] + tri_area(p[0], p[3], p[2]);
    double m = 0.0;
    for (int j = 0; j < nc; ++j) {
      int jn = (j + 1) % nc;
      double e = std::sqrt((p[jn][0] - p[j][0]) * (p[jn][0] - p[j][0]) + (p[jn][1] - p[j][1]) * (p[jn][1] - p[j][1]) +
                           (p[jn][2] - p[j][2]) * (p[jn][2] - p[j][2]));
      if (j == 0 || e > m) m = e;
    }
    pnsz[iel] = m;
    double un[3];
    if (nc == 3) {
      double v21[3], v23[3];
      for (int k = 0; k < 3; ++k) {
        v21[k] = p[0][k] - p[1][k];
        v23[k] = p[2][k] - p[1][k];
      }
      un[0] = v21[1] * v23[2] - v21[2] * v23[1];
      un[1] = v21[2] * v23[0] - v21[0] * v23[2];
      un[2] = v21[0] * v23[1] - v21[1] * v23[0];
    } else {
      double v13[3], v24[3];
      for (int k = 0; k < 3; ++k) {
        v13[k] = p[2][k] - p[0][k];
        v24[k] = p[3][k] - p[1][k];
      }
      un[0] = v24[1] * v13[2] - v24[2] * v13[1];
      un[1] = v24[2] * v13[0] - v24[0] * v13[2];
      un[2] = v24[0] * v13[1] - v24[1] * v13[0];
    }
    double aun = std::sqrt(un[0] * un[0] + un[1] * un[1] + un[2] * un[2]);
    for (int k = 0; k < 3; ++k) dxyz[iel + n * k] = un[k] / aun;
  }
  long i0 = 0;
  for (int b = 0; b < nbody; ++b) {
    const double rg[3] = {xr[b], xr[b + nbody], xr[b + 2 * nbody]};
    for (long iel = i0; iel < i0 + body_nelem[b]; ++iel) {
      double x = xyz_p[iel], y = xyz_p[iel + n], z = xyz_p[iel + 2 * n];
      double n1 = dxyz[iel], n2 = dxyz[iel + n], n3 = dxyz[iel + 2 * n];
      dxyz[iel + 3 * n] = (y - rg[1]) * n3 - (z - rg[2]) * n2;
      dxyz[iel + 4 * n] = (z - rg[2]) * n1 - (x - rg[0]) * n3;
      dxyz[iel + 5 * n] = (x - rg[0]) * n2 - (y - rg[1]) * n1;
    }
    i0 += body_nelem[b];
  }
  return HAMS_OK;
}
