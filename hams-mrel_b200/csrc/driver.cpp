// driver.cpp -- hams_b200_run: a HAMS-MREL deck through the B200 library.
//
//   hams_b200_run <inputdir> <outputdir> [--mixed] [--surrogate FILE] [--far F]
//                 [--body-blocks] [--lanes N] [--device D]
//
// Reads the reference's input deck -- ControlFile.in (ReadControlFile,
// src/InputFiles.f90:46-224), HullMesh[_k].pnl and, with IRSP = 1,
// WaterPlaneMesh[_k].pnl (src/ReadPanelMesh.f90:46-99,
// src/ReadPanelMeshMulti.f90:46-111, local coordinate systems applied on
// read), gen_mod_{body}_{dof}.txt generalized normals -- solves every
// frequency and heading through the C ABI of include/hams_gpu.h, and writes
// the HAMS-format added mass, damping and excitation files
// <outputdir>/Hams_format/OAMASS{1..6}.txt, ODAMPING{1..6}.txt,
// OEXFOR{1..6}.txt in the order and formats of RFORCE_MULTI / EFORCE_MULTI
// (src/PotentWavForceMulti.f90).  Constants are the reference's
// (rho 1000, g 9.80665, unit amplitude, wave reference point at the origin).
#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hams_gpu.h"

namespace {

constexpr double kPi = 3.141592653589793;

struct Lines {
  std::vector<std::string> v;
  size_t cur = 0;
  explicit Lines(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::string l;
    while (std::getline(f, l)) {
      while (!l.empty() && (l.back() == '\r' || l.back() == '\n')) l.pop_back();
      v.push_back(l);
    }
  }
  const std::string& next() {
    static const std::string empty;
    return cur < v.size() ? v[cur++] : empty;
  }
  const std::string* peek() const { return cur < v.size() ? &v[cur] : nullptr; }
};

// Columns [skip, skip + w) of a record with blanks removed (Fortran BN editing).
std::string field(const std::string& l, int skip, int w) {
  std::string o;
  for (int i = skip; i < skip + w && i < (int)l.size(); ++i)
    if (l[i] != ' ' && l[i] != '\t') o += l[i];
  return o;
}

// Fortran F/E/D input of a field with d implied decimals when it has no point.
double fortran_real(std::string s, int d) {
  if (s.empty()) return 0.0;
  bool point = false;
  for (char& c : s) {
    if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'E';
    if (c == '.') point = true;
  }
  for (size_t i = 1; i < s.size(); ++i)  // exponent written as a bare sign: 1.0+3
    if ((s[i] == '+' || s[i] == '-') && std::isdigit((unsigned char)s[i - 1]) && s[i - 1] != 'E') {
      s.insert(i, "E");
      break;
    }
  double v = std::strtod(s.c_str(), nullptr);
  if (!point)
    for (int e = 0; e < d; ++e) v /= 10.0;
  return v;
}

double read_f(Lines& r, int skip, int w, int d) { return fortran_real(field(r.next(), skip, w), d); }
int read_i(Lines& r, int skip, int w) { return (int)std::strtol(field(r.next(), skip, w).c_str(), nullptr, 10); }

// List-directed read of n values, across records.
std::vector<double> read_list(Lines& r, int n) {
  std::vector<double> v;
  while ((int)v.size() < n) {
    if (r.cur >= r.v.size()) throw std::runtime_error("unexpected end of file in a list");
    std::string l = r.next();
    for (char& c : l)
      if (c == ',' || c == '\t') c = ' ';
      else if (c == 'd' || c == 'D') c = 'E';
    std::istringstream is(l);
    std::string tok;
    while ((int)v.size() < n && is >> tok) v.push_back(std::strtod(tok.c_str(), nullptr));
  }
  return v;
}

struct Mesh {
  int nelem = 0, ntnd = 0, isx = 0, isy = 0;
  std::vector<double> xyz;  // ntnd x 3, row-major
  std::vector<int> ncn, ncon;  // ncon nelem x 4, row-major
};

Mesh read_pnl(const std::string& path, bool lid) {
  Lines r(path);
  Mesh m;
  r.next();
  r.next();
  r.next();
  auto h = read_list(r, 4);
  m.nelem = (int)h[0];
  m.ntnd = (int)h[1];
  m.isx = (int)h[2];
  m.isy = (int)h[3];
  r.next();
  r.next();
  m.xyz.resize(3 * (size_t)m.ntnd);
  m.ncn.resize(m.nelem);
  m.ncon.assign(4 * (size_t)m.nelem, 0);
  for (int i = 0; i < m.ntnd; ++i) {
    auto v = read_list(r, 4);
    for (int k = 0; k < 3; ++k) m.xyz[3 * i + k] = v[1 + k];
    if (lid && std::fabs(v[3]) > (double)1.E-10f) throw std::runtime_error(path + ": water-plane node off z = 0");
  }
  r.next();
  r.next();
  r.next();
  for (int i = 0; i < m.nelem; ++i) {
    std::istringstream is(r.next());
    int id = 0, nc = 0;
    is >> id >> nc;
    if (nc != 3 && nc != 4) throw std::runtime_error(path + ": panel with " + std::to_string(nc) + " vertices");
    m.ncn[i] = nc;
    for (int k = 0; k < nc; ++k) is >> m.ncon[4 * i + k];
  }
  return m;
}

bool exists(const std::string& p) {
  struct stat st;
  return stat(p.c_str(), &st) == 0;
}

struct Deck {
  double h = 0.0;
  int sybo = 0, inft = 3, ouft = 3, nbody = 1, isol = 1, irsp = 0, isolv = 1;
  std::vector<double> wvnb, wvhd, xr /* (nb,3) */, lcs /* (nb,4) */;
  // combined hull (column-major, 1-based connectivity) and lid centres
  int nelem = 0, ntnd = 0, isx = 0, isy = 0;
  std::vector<double> xyz, xyz_p, ds, pnsz, dxyz, ixyz_p;
  std::vector<int> ncn, ncon, body_nelem;
  int inelem = 0;
  double refl = 1.0;             // reference body length (REFL)
  std::vector<double> xfp;       // field points (nfp,3) column-major
  int nfp = 0;
  bool separate = false;         // separate_wamit_diffraction_radiation_files
  bool genmod = false;           // some gen_mod_* file overrode the normals
};

Deck load(const std::string& dir) {
  Deck d;
  Lines r(dir + "/ControlFile.in");
  r.next();
  r.next();
  d.h = read_f(r, 14, 30, 15);
  r.next();
  r.next();
  d.sybo = read_i(r, 27, 16);
  d.inft = read_i(r, 25, 16);
  d.ouft = read_i(r, 25, 17);
  int npet = read_i(r, 26, 16);
  const int ifs = d.sybo == 1 ? 2 : 0;
  if (npet > 0) {
    auto v = read_list(r, npet);
    d.wvnb.assign(ifs, 0.0);
    d.wvnb.insert(d.wvnb.end(), v.begin(), v.end());
  } else {
    npet = -npet;
    double w1 = read_f(r, 27, 30, 15), dw = read_f(r, 19, 30, 15);
    d.wvnb.assign(ifs, 0.0);
    for (int i = 0; i < npet; ++i) d.wvnb.push_back(w1 + i * dw);
  }
  r.next();
  r.next();
  const std::string bodycheck = r.next();
  d.nbody = bodycheck.find("multi") != std::string::npos ? read_i(r, 24, 16) : 1;
  const int nb = d.nbody;
  if (nb < 1) throw std::runtime_error("number of bodies < 1");
  d.lcs.assign(4 * (size_t)nb, 0.0);
  if (nb > 1) {
    for (int b = 0; b < nb; ++b) {
      const std::string l = r.next();
      for (int k = 0; k < 4; ++k) d.lcs[b + nb * k] = fortran_real(field(l, 26 + 12 * k, 12), 3);
    }
    r.next();
    r.next();
    r.next();
  }
  int nbeta = read_i(r, 23, 16);
  if (nbeta > 0) {
    d.wvhd = read_list(r, nbeta);
  } else {
    nbeta = -nbeta;
    double b1 = read_f(r, 20, 30, 15), db = read_f(r, 17, 30, 15);
    for (int i = 0; i < nbeta; ++i) d.wvhd.push_back(b1 + i * db);
  }
  r.next();
  r.next();
  d.xr.assign(3 * (size_t)nb, 0.0);
  for (int b = 0; b < nb; ++b) {
    const std::string l = r.next();
    for (int k = 0; k < 3; ++k) d.xr[b + nb * k] = fortran_real(field(l, 28 + 12 * k, 12), 3);
  }
  d.refl = read_f(r, 26, 30, 15);
  d.isol = read_i(r, 26, 16);
  d.irsp = read_i(r, 23, 16);
  read_i(r, 23, 16);  // NTHREAD
  if (const std::string* l = r.peek())
    if (l->find("Solver_type") != std::string::npos) {
      d.isolv = (int)std::strtol(field(*l, 26, 16).c_str(), nullptr, 10);
      r.next();
    }
  // field points and the WAMIT output option (InputFiles.f90:190-220)
  r.next();
  r.next();
  if (const std::string* l = r.peek())
    if (l->find("field_points") != std::string::npos) {
      d.nfp = read_i(r, 27, 16);
      if (d.nfp < 0) throw std::runtime_error("negative number of field points");
      d.xfp.assign(3 * (size_t)d.nfp, 0.0);
      for (int i = 0; i < d.nfp; ++i) {
        auto v = read_list(r, 3);
        for (int k = 0; k < 3; ++k) d.xfp[i + (size_t)d.nfp * k] = v[k];
      }
      r.next();
      r.next();
      if (const std::string* o = r.peek())
        if (o->find("separate") != std::string::npos || o->find("Separate") != std::string::npos)
          d.separate = std::strtol(field(*o, 50, 16).c_str(), nullptr, 10) != 0;
    }
  if (d.nbody == 1) d.separate = false;

  // meshes, bodies stacked in order, local coordinates rotated and shifted
  std::vector<Mesh> hull(nb), lid(nb);
  for (int b = 0; b < nb; ++b) {
    const std::string sfx = nb == 1 ? "" : "_" + std::to_string(b + 1);
    hull[b] = read_pnl(dir + "/HullMesh" + sfx + ".pnl", false);
    d.isx = hull[b].isx;
    d.isy = hull[b].isy;
    d.nelem += hull[b].nelem;
    d.ntnd += hull[b].ntnd;
    d.body_nelem.push_back(hull[b].nelem);
    if (d.irsp == 1) {
      const std::string lp = dir + "/WaterPlaneMesh" + sfx + ".pnl";
      if (exists(lp)) lid[b] = read_pnl(lp, true);
      else if (nb == 1) throw std::runtime_error(lp + " is missing (IRSP = 1)");
      d.inelem += lid[b].nelem;
    }
  }
  const int n = d.nelem, nt = d.ntnd;
  d.xyz.assign(3 * (size_t)nt, 0.0);
  d.ncn.assign(n, 0);
  d.ncon.assign(4 * (size_t)n, 0);
  auto place = [&](const Mesh& m, int b, std::vector<double>& xyz, int ntot, int off_n) {
    const double c = std::cos(d.lcs[b + 3 * nb]), s = std::sin(d.lcs[b + 3 * nb]);
    for (int i = 0; i < m.ntnd; ++i) {
      const double x = m.xyz[3 * i], y = m.xyz[3 * i + 1];
      if (nb > 1) {
        xyz[off_n + i] = 0.0 + d.lcs[b] + c * x - s * y;
        xyz[off_n + i + ntot] = 0.0 + d.lcs[b + nb] + s * x + c * y;
      } else {
        xyz[off_n + i] = x;
        xyz[off_n + i + ntot] = y;
      }
      xyz[off_n + i + 2 * (size_t)ntot] = m.xyz[3 * i + 2];
    }
  };
  int off_e = 0, off_n = 0;
  for (int b = 0; b < nb; ++b) {
    place(hull[b], b, d.xyz, nt, off_n);
    for (int i = 0; i < hull[b].nelem; ++i) {
      d.ncn[off_e + i] = hull[b].ncn[i];
      for (int k = 0; k < 4; ++k) {
        int id = hull[b].ncon[4 * i + k];
        d.ncon[off_e + i + (size_t)n * k] = id ? id + off_n : 0;
      }
    }
    off_e += hull[b].nelem;
    off_n += hull[b].ntnd;
  }
  d.xyz_p.assign(3 * (size_t)n, 0.0);
  d.ds.assign(n, 0.0);
  d.pnsz.assign(n, 0.0);
  d.dxyz.assign(6 * (size_t)n, 0.0);
  int rc = hams_prepare_geometry(nt, d.xyz.data(), n, d.ncn.data(), d.ncon.data(), nb, d.body_nelem.data(),
                                 d.xr.data(), d.xyz_p.data(), d.ds.data(), d.pnsz.data(), d.dxyz.data());
  if (rc) throw std::runtime_error(std::string("geometry: ") + hams_last_error());
  // generalized modes override the normals of a body (ReadPanelMeshMulti.f90:170-200)
  int i0 = 0;
  for (int b = 0; b < nb; ++b) {
    for (int dof = 1; dof <= 6; ++dof) {
      const std::string gp = dir + "/gen_mod_" + std::to_string(nb == 1 ? 1 : b + 1) + "_" + std::to_string(dof) + ".txt";
      std::ifstream f(gp);
      if (!f) continue;
      d.genmod = true;
      std::string l;
      for (int i = 0; i < d.body_nelem[b] && std::getline(f, l); ++i) {
        for (char& c : l)
          if (c == 'd' || c == 'D') c = 'E';
        std::istringstream is(l);
        int pid = 0;
        double val = 0.0;
        if (!(is >> pid >> val)) break;
        d.dxyz[i0 + pid - 1 + (size_t)n * (dof - 1)] = val;
      }
    }
    i0 += d.body_nelem[b];
  }
  // lid centres (the lids' own normals are not used by the solve)
  if (d.inelem > 0) {
    int lnt = 0;
    for (int b = 0; b < nb; ++b) lnt += lid[b].ntnd;
    std::vector<double> lxyz(3 * (size_t)lnt, 0.0);
    std::vector<int> lncn(d.inelem), lncon(4 * (size_t)d.inelem, 0), one{d.inelem};
    int le = 0, ln = 0;
    for (int b = 0; b < nb; ++b) {
      place(lid[b], b, lxyz, lnt, ln);
      for (int i = 0; i < lid[b].nelem; ++i) {
        lncn[le + i] = lid[b].ncn[i];
        for (int k = 0; k < 4; ++k) {
          int id = lid[b].ncon[4 * i + k];
          lncon[le + i + (size_t)d.inelem * k] = id ? id + ln : 0;
        }
      }
      le += lid[b].nelem;
      ln += lid[b].ntnd;
    }
    std::vector<double> zero3(3, 0.0), lds(d.inelem), lsz(d.inelem), ldx(6 * (size_t)d.inelem);
    d.ixyz_p.assign(3 * (size_t)d.inelem, 0.0);
    rc = hams_prepare_geometry(lnt, lxyz.data(), d.inelem, lncn.data(), lncon.data(), 1, one.data(), zero3.data(),
                               d.ixyz_p.data(), lds.data(), lsz.data(), ldx.data());
    if (rc) throw std::runtime_error(std::string("lid geometry: ") + hams_last_error());
  }
  return d;
}

// Fortran Ew.d output editing: 0.dddd...E+xx, right-aligned in w columns.
std::string fmt_e(int w, int dg, double v) {
  char out[64], full[64];
  if (v == 0.0) {
    std::string z = "0." + std::string(dg, '0') + "E+00";
    std::snprintf(out, sizeof(out), "%*s", w, z.c_str());
    return out;
  }
  if (std::isnan(v) || std::isinf(v)) {  // the Fortran runtime's spelling, right-aligned
    std::snprintf(out, sizeof(out), "%*s", w, std::isnan(v) ? "NaN" : (v < 0.0 ? "-Infinity" : "Infinity"));
    return out;
  }
  char m[64];
  std::snprintf(m, sizeof(m), "%.*e", dg - 1, std::fabs(v));
  int e = std::atoi(std::strchr(m, 'e') + 1) + 1;
  std::string mant = "0.";
  mant += m[0];
  for (const char* p = m + 2; *p && *p != 'e'; ++p) mant += *p;
  if (e >= -99 && e <= 99)
    std::snprintf(full, sizeof(full), "%s%sE%c%02d", v < 0 ? "-" : "", mant.c_str(), e < 0 ? '-' : '+', std::abs(e));
  else
    std::snprintf(full, sizeof(full), "%s%s%c%03d", v < 0 ? "-" : "", mant.c_str(), e < 0 ? '-' : '+', std::abs(e));
  std::snprintf(out, sizeof(out), "%*s", w, full);
  return out;
}

// Fortran ESw.d (one digit before the point, two-digit exponent).
std::string fmt_es(int w, int dg, double v) {
  char out[64];
  if (std::isnan(v) || std::isinf(v)) {
    std::snprintf(out, sizeof(out), "%*s", w, std::isnan(v) ? "NaN" : (v < 0.0 ? "-Infinity" : "Infinity"));
    return out;
  }
  std::snprintf(out, sizeof(out), "%*.*E", w, dg, v);
  return out;
}

typedef std::complex<double> zc;

// WamitNondimensMulti (PressureElevationMulti.f90:353-399): pressure or
// elevation of a radiation mode md (1..6) or of a diffraction/incident field
// (md = 0) in WAMIT's nondimensional form and sign convention.
zc wamit_nondim(zc vcp, bool pressure, bool radiation, int md, bool limit, double rho, double g, double amp,
                double refl, double w1) {
  const double nfac = pressure ? (limit ? rho * amp : rho * g * amp) : amp;
  zc nv;
  if (!radiation) {
    nv = vcp / nfac;
  } else {
    const int mexp = md <= 3 ? 0 : 1;
    nv = limit ? vcp / nfac * amp / std::pow(refl, mexp + 1) : vcp / nfac * zc(0.0, -w1) * amp / std::pow(refl, mexp);
  }
  if (std::abs(nv) < 1.E-15) nv = 0.0;
  return radiation ? zc(nv.real(), -nv.imag()) : zc(-nv.imag(), -nv.real());
}

// Pressure (i w rho phi) or elevation (i w / g phi) of a potential
// (CalPressureMulti / CalElevationMulti, :305-348), rho phi and phi at the
// zero and infinite frequency limits.
zc pressure_or_elevation(zc pot, bool pressure, bool limit, double rho, double g, double w1) {
  if (pressure) return limit ? rho * pot : zc(0.0, w1 * rho) * pot;
  return limit ? pot : zc(0.0, w1 / g) * pot;
}

std::vector<float> read_params(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  std::vector<float> p(hams_surrogate_param_count());
  f.read(reinterpret_cast<char*>(p.data()), p.size() * sizeof(float));
  if (f.gcount() != (std::streamsize)(p.size() * sizeof(float))) throw std::runtime_error(path + ": short parameter file");
  return p;
}

// Output frequency of a wave (CalWaveProperts OUFR, ImplementSubs.f90:139-149).
double out_freq(const hams_wave& w, int ouft) {
  switch (ouft) {
    case 1: return w.v;
    case 2: return w.wk;
    case 4: return w.tp;
    case 5: return w.wl;
    default: return w.w1;
  }
}

// WAMIT-format field-point files (OutputPressureElevation_*Multi,
// PressureElevationMulti.f90:404-590, and the single-body writers of
// PressureElevation.f90:391-461): per frequency the radiation lines, then per
// heading the diffraction lines and (several bodies) the incident-wave lines.
// Points below the free surface give pressures, points on it elevations.
void write_field_points(const std::string& out, const Deck& d, const std::vector<hams_wave>& waves,
                        const std::vector<std::vector<zc>>& fpot, const hams_opts& o) {
  const std::string wd = out + "/Wamit_format";
  mkdir(out.c_str(), 0755);
  mkdir(wd.c_str(), 0755);
  const int nb = d.nbody, ndof = 6 * nb, nbeta = (int)d.wvhd.size(), nfp = d.nfp;
  const bool multi = nb > 1;
  std::ofstream main_f, dif_f, inc_f;
  std::vector<std::ofstream> rad_f;
  if (d.separate) {
    dif_f.open(wd + "/PressureElevationDiffraction.6p");
    rad_f.resize(nb);
    for (int b = 0; b < nb; ++b) rad_f[b].open(wd + "/PressureElevationRadiation_" + std::to_string(b + 1) + ".6p");
  } else {
    main_f.open(wd + "/PressureElevation.6p");
  }
  if (multi) inc_f.open(wd + "/PressureElevationIncidence.6p");
  std::ofstream& dif = d.separate ? dif_f : main_f;
  const double kPi = 3.141592653589793;
  for (size_t k = 0; k < fpot.size(); ++k) {
    const hams_wave& w = waves[k];
    const bool limit = std::fabs(w.tp + 1.0) < 1.E-6 || std::fabs(w.tp) < 1.E-6;
    const double oufr = out_freq(w, d.ouft);
    auto at = [&](int f, int col) { return fpot[k][f + (size_t)nfp * col]; };
    auto field = [&](int f, int col, bool radiation, int md) {
      const bool pressure = std::fabs(d.xfp[f + 2 * (size_t)nfp]) > 1.E-6;
      const zc v = pressure_or_elevation(at(f, col), pressure, limit, o.rho, o.g, w.w1);
      return wamit_nondim(v, pressure, radiation, md, limit, o.rho, o.g, o.amp, d.refl, w.w1);
    };
    // radiation
    for (int f = 0; f < nfp; ++f) {
      if (!multi) {
        if (!(std::fabs(d.xfp[f + 2 * (size_t)nfp]) > 1.E-6)) continue;  // single body: submerged points only
        main_f << fmt_es(14, 6, oufr) << std::setw(10) << f + 1;
        for (int md = 1; md <= 6; ++md) {
          const zc v = field(f, md - 1, true, md);
          main_f << fmt_es(14, 6, v.real()) << fmt_es(14, 6, v.imag());
        }
        main_f << '\n';
        continue;
      }
      if (!d.separate) main_f << fmt_es(14, 6, oufr) << std::setw(10) << f + 1;
      for (int b = 0; b < nb; ++b) {
        std::ostringstream line;
        for (int md = 1; md <= 6; ++md) {
          const zc v = field(f, 6 * b + md - 1, true, md);
          line << fmt_es(14, 6, v.real()) << fmt_es(14, 6, v.imag());
        }
        if (d.separate)
          rad_f[b] << fmt_es(14, 6, oufr) << std::setw(10) << f + 1 << line.str() << '\n';
        else
          main_f << (b == 0 ? "" : std::string(24, ' ')) << line.str() << '\n';
      }
    }
    // diffraction and incident wave, per heading
    for (int ib = 0; ib < nbeta; ++ib) {
      const double bdeg = (d.wvhd[ib] * kPi / 180.0) * 180.0 / kPi;
      for (int f = 0; f < nfp; ++f) {
        const zc v = field(f, ndof + ib, false, 0);
        dif << fmt_es(14, 6, oufr) << fmt_es(14, 6, bdeg) << std::setw(10) << f + 1;
        if (multi)
          dif << fmt_es(14, 6, v.real()) << fmt_es(14, 6, v.imag()) << '\n';
        else
          dif << fmt_es(14, 6, std::abs(v)) << fmt_es(14, 6, std::atan2(v.imag(), v.real()) * 180.0 / kPi)
              << fmt_es(14, 6, v.real()) << fmt_es(14, 6, v.imag()) << '\n';
      }
      if (multi)
        for (int f = 0; f < nfp; ++f) {
          const zc v = field(f, ndof + nbeta + ib, false, 0);
          inc_f << fmt_es(14, 6, oufr) << fmt_es(14, 6, bdeg) << std::setw(10) << f + 1 << fmt_es(14, 6, std::abs(v))
                << fmt_es(14, 6, std::atan2(v.imag(), v.real()) * 180.0 / kPi) << fmt_es(14, 6, v.real())
                << fmt_es(14, 6, v.imag()) << '\n';
        }
    }
  }
}

// Hydrostatic_k.in / Hydrostatic.in (ReadHydroStatic[Multi],
// HydroStaticMulti.f90:68-118): centre of gravity, then the 6 x 6 mass,
// external linear damping, external quadratic damping, hydrostatic restoring
// and external restoring matrices of one body.
struct Hydro {
  double m[6][6], blin[6][6], bqdr[6][6], crs[6][6], kstf[6][6];
};

Hydro read_hydro(const std::string& path) {
  Lines r(path);
  Hydro h{};
  r.next();
  read_list(r, 3);
  double(*mats[5])[6] = {h.m, h.blin, h.bqdr, h.crs, h.kstf};
  for (auto* a : mats) {
    r.next();
    for (int i = 0; i < 6; ++i) {
      auto v = read_list(r, 6);
      for (int j = 0; j < 6; ++j) a[i][j] = v[j];
    }
  }
  return h;
}

// A x = b for a small complex system by Gaussian elimination with partial
// pivoting on |re| + |im| (ZGESV's choice); b is overwritten with x.
void small_solve(int n, std::vector<zc> a, std::vector<zc>& b) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = -1.0;
    for (int i = k; i < n; ++i) {
      const zc v = a[i + (size_t)n * k];
      const double m = std::fabs(v.real()) + std::fabs(v.imag());
      if (m > best) {
        best = m;
        p = i;
      }
    }
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(a[k + (size_t)n * j], a[p + (size_t)n * j]);
      std::swap(b[k], b[p]);
    }
    const zc d = a[k + (size_t)n * k];
    if (d == zc(0.0, 0.0)) continue;  // singular: the reference's ZGESV leaves INFO > 0 unchecked
    for (int i = k + 1; i < n; ++i) {
      const zc l = a[i + (size_t)n * k] / d;
      if (l == zc(0.0, 0.0)) continue;
      for (int j = k + 1; j < n; ++j) a[i + (size_t)n * j] -= l * a[k + (size_t)n * j];
      b[i] -= l * b[k];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    zc s = b[k];
    for (int j = k + 1; j < n; ++j) s -= a[k + (size_t)n * j] * b[j];
    b[k] = s / a[k + (size_t)n * k];
  }
}

// Motion amplitudes of all bodies for one frequency and heading
// (SolveMotion[Multi], SolveMotionMulti.f90:46-150): block-diagonal body
// matrices, (-w^2 (M + A) + i w (B + Blin [+ Bq w |x|]) + C + K) x = -Im X - i Re X,
// the quadratic damping iterated until the summed relative change is below 1e-6.
std::vector<zc> solve_motion(int nb, const std::vector<Hydro>& hy, double w1, const double* amas, const double* bdmp,
                             size_t stride, const std::vector<zc>& exfc) {
  const int n = 6 * nb;
  auto blk = [&](double(Hydro::*mat)[6][6], int i, int j) {
    return i / 6 == j / 6 ? (hy[i / 6].*mat)[i % 6][j % 6] : 0.0;
  };
  double norm = 0.0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) norm = std::max(norm, std::fabs(blk(&Hydro::bqdr, i, j)));
  auto system = [&](const std::vector<zc>* x) {
    std::vector<zc> a((size_t)n * n);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        const size_t e = (size_t)i + (size_t)n * j;
        double damp = bdmp[e * stride] + blk(&Hydro::blin, i, j);
        if (x) damp += blk(&Hydro::bqdr, i, j) * w1 * std::abs((*x)[j]);
        a[e] = -w1 * w1 * (blk(&Hydro::m, i, j) + amas[e * stride]) + zc(0.0, w1) * damp + blk(&Hydro::crs, i, j) +
               blk(&Hydro::kstf, i, j);
      }
    return a;
  };
  std::vector<zc> rhs(n);
  for (int i = 0; i < n; ++i) rhs[i] = zc(-exfc[i].imag(), -exfc[i].real());
  std::vector<zc> x = rhs;
  small_solve(n, system(nullptr), x);
  if (norm >= 1.0E-6) {
    double rerr = 100.0;
    while (rerr > 1.0E-6) {
      std::vector<zc> x1 = rhs;
      small_solve(n, system(&x), x1);
      rerr = 0.0;
      for (int j = 0; j < n; ++j)
        if (std::abs(x1[j]) > 0.0) rerr += std::abs(x1[j] - x[j]) / std::abs(x1[j]);
      x = x1;
    }
  }
  return x;
}

// WAMIT-format force and motion files (RFORCE[_MULTI] / EFORCE[_MULTI],
// PotentWavForceMulti.f90:122,206-215, ReorderAmssDamp :235-346,
// SolveMotion[Multi], the hydrostatic listing HydroStaticMulti.f90:98-111):
// AmssDamp.1 row-major per frequency, ExcForce.3 and Motion.4 per heading.
// The excitation phase is printed as the reference does, converted to
// degrees twice (ATAN2D(...)*180/PI).
void write_wamit_forces(const std::string& out, const std::string& in, const Deck& d,
                        const std::vector<hams_wave>& waves, const std::vector<double>& amas,
                        const std::vector<double>& bdmp, const std::vector<double>& exfc, const hams_opts& o) {
  const std::string wd = out + "/Wamit_format";
  mkdir(out.c_str(), 0755);
  mkdir(wd.c_str(), 0755);
  const int nb = d.nbody, ndof = 6 * nb, nf = (int)waves.size(), nbeta = (int)d.wvhd.size();
  const double kPi = 3.141592653589793;
  std::vector<Hydro> hy;
  for (int b = 0; b < nb; ++b) {
    const std::string f = in + (nb == 1 ? "/Hydrostatic.in" : "/Hydrostatic_" + std::to_string(b + 1) + ".in");
    if (!exists(f)) {
      hy.clear();
      break;
    }
    hy.push_back(read_hydro(f));
  }
  if (!hy.empty()) {
    std::ofstream hs(wd + "/Hydrostat.hst");
    for (int i = 0; i < ndof; ++i)
      for (int j = 0; j < ndof; ++j) {
        const double v = i / 6 == j / 6 ? hy[i / 6].crs[i % 6][j % 6] / (o.rho * o.g) : 0.0;
        hs << std::setw(6) << i + 1 << std::setw(6) << j + 1 << "  " << fmt_es(14, 6, v) << '\n';
      }
  }
  std::ofstream ad(wd + "/AmssDamp.1"), ef(wd + "/ExcForce.3");
  std::ofstream mo;
  if (!hy.empty()) mo.open(wd + "/Motion.4");
  const size_t sf = (size_t)nf;
  for (int k = 0; k < nf; ++k) {
    const hams_wave& w = waves[k];
    const bool limit = std::fabs(w.tp + 1.0) < 1.E-6 || std::fabs(w.tp) < 1.E-6;
    const double oufr = out_freq(w, d.ouft);
    for (int i = 0; i < ndof; ++i)
      for (int j = 0; j < ndof; ++j) {
        const size_t e = k + sf * ((size_t)i + (size_t)ndof * j);
        ad << fmt_es(14, 6, oufr) << std::setw(6) << i + 1 << std::setw(6) << j + 1 << fmt_es(14, 6, amas[e] / o.rho);
        if (!limit) ad << fmt_es(14, 6, bdmp[e] / (o.rho * w.w1));
        ad << '\n';
      }
    for (int ib = 0; ib < nbeta; ++ib) {
      const double bdeg = (d.wvhd[ib] * kPi / 180.0) * 180.0 / kPi;
      std::vector<zc> x(ndof);
      for (int m = 0; m < ndof; ++m) {
        const size_t e = k + sf * (ib + (size_t)nbeta * m);
        x[m] = zc(exfc[2 * e], exfc[2 * e + 1]);
      }
      if (!limit)
        for (int m = 0; m < ndof; ++m) {
          const double s = o.rho * o.g * o.amp, re = x[m].real() / s, im = x[m].imag() / s;
          const double nrel = -im, nimg = -re;
          ef << fmt_es(14, 6, oufr) << fmt_es(14, 6, bdeg) << std::setw(6) << m + 1 << fmt_es(14, 6, std::abs(x[m]) / s)
             << fmt_es(14, 6, std::atan2(nimg, nrel) * 180.0 / kPi * 180.0 / kPi) << fmt_es(14, 6, nrel)
             << fmt_es(14, 6, nimg) << '\n';
        }
      if (hy.empty() || limit) continue;
      const std::vector<zc> u = solve_motion(nb, hy, w.w1, &amas[k], &bdmp[k], sf, x);
      for (int m = 0; m < ndof; ++m) {
        const double nfac = o.amp / std::pow(d.refl, m % 6 < 3 ? 2 : 3);
        const double nrel = u[m].real() / nfac, nimg = u[m].imag() / nfac;
        mo << fmt_es(14, 6, oufr) << fmt_es(14, 6, bdeg) << std::setw(6) << m + 1
           << fmt_es(14, 6, std::sqrt(nrel * nrel + nimg * nimg)) << fmt_es(14, 6, std::atan2(nimg, nrel) * 180.0 / kPi)
           << fmt_es(14, 6, nrel) << fmt_es(14, 6, nimg) << '\n';
      }
    }
  }
}

int usage() {
  std::fprintf(stderr,
               "usage: hams_b200_run <inputdir> <outputdir> [--mixed] [--surrogate FILE] [--far F] [--body-blocks] "
               "[--lanes N] [--device D]\n");
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) return usage();
  const std::string in = argv[1], out = argv[2];
  int precision = HAMS_PREC_FP64, lanes = 0, device = 0, body_blocks = 0;
  std::string sgfile;
  double far = 3.0;
  for (int a = 3; a < argc; ++a) {
    std::string s = argv[a];
    if (s == "--mixed") precision = HAMS_PREC_MIXED;
    else if (s == "--surrogate" && a + 1 < argc) sgfile = argv[++a];
    else if (s == "--far" && a + 1 < argc) far = std::atof(argv[++a]);
    else if (s == "--body-blocks") body_blocks = 1;
    else if (s == "--lanes" && a + 1 < argc) lanes = std::atoi(argv[++a]);
    else if (s == "--device" && a + 1 < argc) device = std::atoi(argv[++a]);
    else return usage();
  }
  try {
    Deck d = load(in);
    // a half mesh (ISX or ISY = 1) is unfolded by the library; generalized
    // modes would need each mode's parity under the mirror, which the deck
    // does not give
    if ((d.isx || d.isy) && d.genmod)
      throw std::runtime_error("generalized modes (gen_mod_*) with geometric symmetry (ISX/ISY = 1) are not supported");
    const int nb = d.nbody, ndof = 6 * nb, nf = (int)d.wvnb.size(), nbeta = (int)d.wvhd.size();
    const double g = 9.80665;
    hams_geom geo{};
    geo.nelem = d.nelem;
    geo.ntnd = d.ntnd;
    geo.nbody = nb;
    geo.isx = d.isx;
    geo.isy = d.isy;
    geo.xyz = d.xyz.data();
    geo.ncn = d.ncn.data();
    geo.ncon = d.ncon.data();
    geo.xyz_p = d.xyz_p.data();
    geo.ds = d.ds.data();
    geo.pnsz = d.pnsz.data();
    geo.dxyz = d.dxyz.data();
    geo.body_nelem = d.body_nelem.data();
    geo.inelem = d.inelem;
    geo.ixyz_p = d.inelem ? d.ixyz_p.data() : nullptr;
    hams_opts o{};
    o.depth = d.h;
    o.rho = 1000.0;
    o.g = g;
    o.amp = 1.0;
    o.isol = d.isol;
    o.irsp = d.irsp;
    o.precision = precision;
    o.device = device;
    o.batch_lanes = lanes;
    o.body_blocks = body_blocks;
    o.solver = d.isolv == 2 ? HAMS_SOLVER_GMRES : HAMS_SOLVER_LU;
    hams_ctx* ctx = nullptr;
    if (hams_ctx_create(&geo, &o, &ctx)) throw std::runtime_error(std::string("context: ") + hams_last_error());
    if (!sgfile.empty()) {
      auto p = read_params(sgfile);
      if (hams_ctx_set_surrogate(ctx, p.data(), (int32_t)p.size(), far))
        throw std::runtime_error(std::string("surrogate: ") + hams_last_error());
    }
    if (d.nfp > 0 && hams_ctx_set_field_points(ctx, d.nfp, d.xfp.data()))
      throw std::runtime_error(std::string("field points: ") + hams_last_error());
    std::vector<hams_wave> waves(nf);
    for (int k = 0; k < nf; ++k)
      if (hams_wave_properties(d.inft, d.wvnb[k], d.h, g, d.sybo == 1 && k < 2 ? k + 1 : 0, &waves[k]))
        throw std::runtime_error(std::string("wave properties: ") + hams_last_error());
    std::vector<double> beta(nbeta);
    for (int i = 0; i < nbeta; ++i) beta[i] = d.wvhd[i] * kPi / 180.0;
    std::vector<double> amas((size_t)nf * ndof * ndof), bdmp(amas.size()), exfc(2 * (size_t)nf * std::max(nbeta, 1) * ndof);
    int rc = hams_solve_batch(ctx, nf, waves.data(), nbeta, beta.data(), amas.data(), bdmp.data(), exfc.data());
    if (rc >= 0 && *hams_last_note(ctx)) std::fprintf(stderr, "hams_b200_run: %s\n", hams_last_note(ctx));
    // field-point potentials of every frequency: (nfp, 6nb + 2 nbeta) each
    const size_t fpn = (size_t)d.nfp * (ndof + 2 * nbeta);
    std::vector<std::vector<zc>> fpot(d.nfp > 0 && rc >= 0 ? nf : 0, std::vector<zc>(fpn));
    for (int k = 0; k < (int)fpot.size(); ++k)
      if (hams_field_potentials(ctx, k, reinterpret_cast<double*>(fpot[k].data())))
        throw std::runtime_error(std::string("field potentials: ") + hams_last_error());
    hams_ctx_destroy(ctx);
    if (rc < 0) throw std::runtime_error(std::string("solve: ") + hams_last_error());
    if (rc > 0) std::fprintf(stderr, "hams_b200_run: singular pivot %d\n", rc);
    const std::string hd = out + "/Hams_format";
    mkdir(out.c_str(), 0755);
    mkdir(hd.c_str(), 0755);
    for (int md = 0; md < 6; ++md) {
      const std::string s = std::to_string(md + 1) + ".txt";
      std::ofstream fa(hd + "/OAMASS" + s), fd(hd + "/ODAMPING" + s), fx(hd + "/OEXFOR" + s);
      if (!fa || !fd || !fx) throw std::runtime_error("cannot write to " + hd);
      char head[64];
      for (int k = 0; k < nf; ++k) {
        std::snprintf(head, sizeof(head), "%7.3f %7.3f ", waves[k].wk, waves[k].w1);
        // RFORCE_MULTI: body pairs (M, N), row 6M + md, six columns of body N
        for (int b1 = 0; b1 < nb; ++b1)
          for (int b2 = 0; b2 < nb; ++b2) {
            fa << head;
            fd << head;
            for (int c = 0; c < 6; ++c) {
              const size_t e = k + (size_t)nf * ((6 * b1 + md) + (size_t)ndof * (6 * b2 + c));
              fa << fmt_e(14, 5, amas[e]);
              fd << fmt_e(14, 5, bdmp[e]);
            }
            fa << '\n';
            fd << '\n';
          }
        // EFORCE_MULTI: headings outer, bodies inner
        for (int ib = 0; ib < nbeta; ++ib)
          for (int b1 = 0; b1 < nb; ++b1) {
            const size_t e = k + (size_t)nf * (ib + (size_t)nbeta * (6 * b1 + md));
            fx << head << fmt_e(14, 6, exfc[2 * e]) << fmt_e(14, 6, exfc[2 * e + 1]) << '\n';
          }
      }
    }
    write_wamit_forces(out, in, d, waves, amas, bdmp, exfc, o);
    if (d.nfp > 0) write_field_points(out, d, waves, fpot, o);
    std::printf("hams_b200_run: %d frequencies, %d headings, %d panels, %d bodies -> %s\n", nf, nbeta, d.nelem, nb,
                hd.c_str());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "hams_b200_run: %s\n", e.what());
    return 1;
  }
  return 0;
}
