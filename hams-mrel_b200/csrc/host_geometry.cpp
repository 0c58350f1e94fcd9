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
#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>
#include <vector>

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

// ---------------------------------------------------------------------------
// Identical bodies (hams_body_blocks).  The finite- and infinite-depth Green
// functions depend on the horizontal distance and the two depths of a pair
// only, and the Rankine panel integrals on the panels' relative position, so
// the (field body, source body) block of the collocation matrices is the same
// for every pair of bodies with the same shapes and the same horizontal
// offset.  Body b is a translate of an earlier body t when both have the same
// panels in the same order, each with the same vertex count, and every
// vertex, centre, area, longest edge and unit normal of b equals t's moved by
// one horizontal offset (coordinates within tol times the mesh size; the
// rotational normals are left out, they enter the right-hand sides only).
// ---------------------------------------------------------------------------
namespace {

struct BodyShape {
  int tmpl;        // the first body of which this one is a translate
  double dx, dy;   // its horizontal offset from that body
};

std::vector<BodyShape> body_shapes(const hams_geom* g, double tol) {
  const int nb = g->nbody, n = g->nelem;
  std::vector<int> st(nb + 1, 0);
  for (int b = 0; b < nb; ++b) st[b + 1] = st[b] + g->body_nelem[b];
  double lo = 0.0, hi = 0.0;
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < n; ++i) {
      lo = std::min(lo, g->xyz_p[i + (size_t)k * n]);
      hi = std::max(hi, g->xyz_p[i + (size_t)k * n]);
    }
  const double eps = tol * std::max(1.0, hi - lo), eps_n = tol;
  auto node = [&](int panel, int v, int k) {
    return g->xyz[(g->ncon[panel + (size_t)v * n] - 1) + (size_t)k * g->ntnd];
  };
  std::vector<BodyShape> s(nb);
  for (int b = 0; b < nb; ++b) {
    s[b] = {b, 0.0, 0.0};
    for (int t = 0; t < b; ++t) {
      if (s[t].tmpl != t || st[t + 1] - st[t] != st[b + 1] - st[b]) continue;
      const int m = st[b + 1] - st[b];
      if (m == 0) continue;
      const double dx = g->xyz_p[st[b]] - g->xyz_p[st[t]], dy = g->xyz_p[st[b] + n] - g->xyz_p[st[t] + n];
      bool same = true;
      for (int q = 0; q < m && same; ++q) {
        const int i = st[b] + q, j = st[t] + q;
        same = g->ncn[i] == g->ncn[j] && std::fabs(g->xyz_p[i] - g->xyz_p[j] - dx) <= eps &&
               std::fabs(g->xyz_p[i + n] - g->xyz_p[j + n] - dy) <= eps &&
               std::fabs(g->xyz_p[i + 2 * (size_t)n] - g->xyz_p[j + 2 * (size_t)n]) <= eps &&
               std::fabs(g->ds[i] - g->ds[j]) <= eps * std::max(1.0, std::fabs(g->pnsz[j])) &&
               std::fabs(g->pnsz[i] - g->pnsz[j]) <= eps;
        for (int k = 0; k < 3 && same; ++k)
          same = std::fabs(g->dxyz[i + (size_t)k * n] - g->dxyz[j + (size_t)k * n]) <= eps_n;
        for (int v = 0; v < g->ncn[i] && same; ++v)
          same = std::fabs(node(i, v, 0) - node(j, v, 0) - dx) <= eps &&
                 std::fabs(node(i, v, 1) - node(j, v, 1) - dy) <= eps &&
                 std::fabs(node(i, v, 2) - node(j, v, 2)) <= eps;
      }
      if (same) {
        s[b] = {t, dx, dy};
        break;
      }
    }
  }
  return s;
}

std::vector<int> body_block_reps(const hams_geom* g, double tol) {
  const int nb = g->nbody;
  std::vector<int> rep((size_t)nb * nb);
  for (size_t k = 0; k < rep.size(); ++k) rep[k] = (int)k;
  if (nb <= 1 || g->inelem > 0) return rep;
  std::vector<BodyShape> s = body_shapes(g, tol);
  double lo = 0.0, hi = 0.0;
  for (int i = 0; i < 2 * g->nelem; ++i) {
    lo = std::min(lo, g->xyz_p[i]);
    hi = std::max(hi, g->xyz_p[i]);
  }
  const double eps = tol * std::max(1.0, hi - lo);
  // block (b1 field, b2 source) = block (c1, c2) when the templates agree and
  // the offset of b2 from b1 equals that of c2 from c1 (within eps); the
  // representatives are filed by templates and offset cell (size eps), so a
  // block looks at its own and the neighbouring cells only, and takes the
  // first representative within eps, in block order
  std::map<std::tuple<int, int, long long, long long>, std::vector<int>> cells;
  for (int b2 = 0; b2 < nb; ++b2)
    for (int b1 = 0; b1 < nb; ++b1) {
      const int k = b1 + nb * b2;
      const double ox = s[b2].dx - s[b1].dx, oy = s[b2].dy - s[b1].dy;
      // floor keeps two offsets within eps of each other at most one cell apart
      // (rounding to nearest would put +-eps/2 two cells apart)
      const long long qx = (long long)std::floor(ox / eps), qy = (long long)std::floor(oy / eps);
      int best = k;
      for (long long ex = -1; ex <= 1; ++ex)
        for (long long ey = -1; ey <= 1; ++ey) {
          auto it = cells.find(std::make_tuple(s[b1].tmpl, s[b2].tmpl, qx + ex, qy + ey));
          if (it == cells.end()) continue;
          for (int c : it->second) {
            const int c1 = c % nb, c2 = c / nb;
            if (c < best && std::fabs(s[c2].dx - s[c1].dx - ox) <= eps && std::fabs(s[c2].dy - s[c1].dy - oy) <= eps)
              best = c;
          }
        }
      rep[k] = best;
      if (best == k) cells[std::make_tuple(s[b1].tmpl, s[b2].tmpl, qx, qy)].push_back(k);
    }
  return rep;
}

}  // namespace

extern "C" int hams_body_blocks(const hams_geom* g, double tol, int32_t* rep) {
  if (!g || !rep || g->nbody < 1 || !g->body_nelem || !g->xyz_p || !g->ncn || !g->ncon || !g->xyz || !g->ds ||
      !g->pnsz || !g->dxyz)
    return -1;
  if (!(tol > 0.0)) tol = 1e-9;
  std::vector<int> r = body_block_reps(g, tol);
  int distinct = 0;
  for (size_t k = 0; k < r.size(); ++k) {
    rep[k] = r[k];
    distinct += r[k] == (int)k;
  }
  return distinct;
}
