// fullband_tables.cpp -- see fullband_tables.h.
//
// Every numerical expression that feeds a table keeps the reference's
// operand order (IEEE double, no contraction: this file is compiled with
// -ffp-contract=off) so the tables are bit-identical to Band::IELEC's.
// Reference locations are cited per stage.
#include "fullband_tables.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace mcb200 {

namespace {

// Physical constants, include/Constant_GlobalVariable_MathFunction.h:21-79.
constexpr double kPi = 3.141592653589793238462643e0;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kEc = 1.602176e-19;
constexpr double kEm = 9.109383e-31;
constexpr double kPlanck = 6.582119e-16;
constexpr double kClight = 299792458;
constexpr double kBoltz = 8.617343e-5;
constexpr double kEps0 = 8.854187817e-12;
const double kFsc = kEc / (kPlanck * kClight * 4.0 * kPi * kEps0);

double dmax(double a, double b) { return a > b ? a : b; }
double dmin(double a, double b) { return a < b ? a : b; }
int isign(double x) { return int(std::fabs(x) / x); }  // utils.cpp sign()

// Whitespace-separated numeric reader over a whole file (strtod / strtol,
// the same correctly rounded conversion iostream extraction uses).
class Tokens {
 public:
  explicit Tokens(const std::string &path) : path_(path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open table file " + path);
    std::ostringstream ss;
    ss << in.rdbuf();
    buf_ = ss.str();
    p_ = buf_.c_str();
  }
  double real() {
    char *end = nullptr;
    double v = std::strtod(p_, &end);
    if (end == p_) throw std::runtime_error("malformed number in " + path_);
    p_ = end;
    return v;
  }
  long integer() {
    char *end = nullptr;
    long v = std::strtol(p_, &end, 10);
    if (end == p_) throw std::runtime_error("malformed integer in " + path_);
    p_ = end;
    return v;
  }

 private:
  std::string path_, buf_;
  const char *p_;
};

// The 48 point-group operations in the reference's order (SETMATSYM,
// src/Band.cpp:986-1299): for each isym the coordinate permutation
// (matsym[0..2], 1-based source axis of each output axis) and the signs
// (matsym[3..5]).  The order is part of the state encoding (isym / 8 is the
// valley index used by TALIND), so it has to match the reference exactly.
const signed char kSymOps[48][6] = {
    {1, 2, 3, 1, 1, 1},    {1, 2, 3, 1, 1, -1},   {1, 2, 3, 1, -1, 1},   {1, 2, 3, 1, -1, -1},
    {1, 3, 2, 1, 1, 1},    {1, 3, 2, 1, 1, -1},   {1, 3, 2, 1, -1, 1},   {1, 3, 2, 1, -1, -1},
    {1, 2, 3, -1, 1, 1},   {1, 2, 3, -1, 1, -1},  {1, 2, 3, -1, -1, 1},  {1, 2, 3, -1, -1, -1},
    {1, 3, 2, -1, 1, 1},   {1, 3, 2, -1, 1, -1},  {1, 3, 2, -1, -1, 1},  {1, 3, 2, -1, -1, -1},
    {2, 1, 3, 1, 1, 1},    {2, 1, 3, 1, 1, -1},   {2, 1, 3, -1, 1, -1},  {2, 1, 3, -1, 1, 1},
    {3, 1, 2, 1, 1, 1},    {3, 1, 2, 1, 1, -1},   {3, 1, 2, -1, 1, -1},  {3, 1, 2, -1, 1, 1},
    {2, 1, 3, 1, -1, 1},   {2, 1, 3, 1, -1, -1},  {2, 1, 3, -1, -1, -1}, {2, 1, 3, -1, -1, 1},
    {3, 1, 2, 1, -1, 1},   {3, 1, 2, 1, -1, -1},  {3, 1, 2, -1, -1, -1}, {3, 1, 2, -1, -1, 1},
    {2, 3, 1, 1, 1, 1},    {2, 3, 1, 1, -1, 1},   {2, 3, 1, -1, -1, 1},  {2, 3, 1, -1, 1, 1},
    {3, 2, 1, 1, 1, 1},    {3, 2, 1, 1, -1, 1},   {3, 2, 1, -1, -1, 1},  {3, 2, 1, -1, 1, 1},
    {2, 3, 1, 1, 1, -1},   {2, 3, 1, 1, -1, -1},  {2, 3, 1, -1, -1, -1}, {2, 3, 1, -1, 1, -1},
    {3, 2, 1, 1, 1, -1},   {3, 2, 1, 1, -1, -1},  {3, 2, 1, -1, -1, -1}, {3, 2, 1, -1, 1, -1},
};

}  // namespace

// init_phpysical_parameter, src/mcmodel.cpp:4007-4122 (silicon branch).
Units Units::at_temperature(double kelvin) {
  Units u{};
  u.frickel = 1.0;
  double sia0 = 5.43e-10, sirho = 2.33e3, siul = 9.05e3, siut = 9.05e3;
  u.T0 = kelvin;
  u.Tn = u.T0 / 300.0;
  u.eV0 = kBoltz * u.T0;
  u.em0 = kEm;
  u.hq0 = kPlanck;
  u.ec0 = kEc;
  u.rmom0 = std::sqrt((u.em0 / u.ec0) * u.eV0);
  u.spr0 = u.hq0 / u.rmom0;
  u.spk0 = 1.0 / u.spr0;
  u.time0 = u.hq0 / u.eV0;
  u.velo0 = u.spr0 / u.time0;
  u.cvr = kClight / u.velo0;
  u.pot0 = u.eV0;
  u.field0 = u.pot0 / u.spr0;
  u.conc0 = u.spk0 * u.spk0 * u.spk0;
  u.dens0 = u.em0 * u.conc0;
  u.dpc0 = u.field0;
  u.scrt0 = 1.0 / u.time0;
  u.curr0 = u.ec0 / u.time0;
  u.sia0 = sia0 / u.spr0;
  u.sirho = sirho / u.dens0;
  u.siul = siul / u.velo0;
  u.siut = siut / u.velo0;
  const double T0 = u.T0;
  if (T0 < 190.0)
    u.sieg = (1.170 + 1.059e-5 * T0 - 6.05e-7 * T0 * T0) / u.eV0;
  else if (T0 < 250.0)
    u.sieg = (1.17850 - 9.025e-5 * T0 - 3.05e-7 * T0 * T0) / u.eV0;
  else
    u.sieg = (1.2060 - 2.730e-4 * T0) / u.eV0;
  u.a0pi = kTwoPi / u.sia0;
  u.eps_vacuum = 1.00 / (4 * kPi * u.cvr * kFsc);
  u.eps_oxide = 3.90 / (4 * kPi * u.cvr * kFsc);
  u.eps_silicon = 11.70 / (4 * kPi * u.cvr * kFsc);
  return u;
}

double fii(double x1, double y1, double z1, double x2, double y2, double z2, double x3, double y3, double z3) {
  // FII, src/Band.cpp:335-353: half the norm of the edge cross product.
  double sbx = (y2 - y1) * (z3 - z1) - (y3 - y1) * (z2 - z1);
  double sby = (x3 - x1) * (z2 - z1) - (x2 - x1) * (z3 - z1);
  double sbz = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
  return 0.50 * std::sqrt(sbx * sbx + sby * sby + sbz * sbz);
}

// SURF, src/Band.cpp:194-332: area of the iso-energy cut through tet `it`.
double FullBandTables::surf(double eps, int it) const {
  const int n0 = T(0, it), n1 = T(1, it), n2 = T(2, it), n3 = T(3, it);
  const double e0 = eek[n0], e1 = eek[n1], e2 = eek[n2], e3 = eek[n3];
  if (!(eps > e0 && eps < e3)) return 0.0;
  // edge point between nodes p -> q at energy eps, relative (base = 0) or absolute
  auto rel = [&](int p, int q, double &ox, double &oy, double &oz) {
    double r = (eps - eek[p]) / (eek[q] - eek[p]);
    ox = r * (xkk[q] - xkk[p]);
    oy = r * (ykk[q] - ykk[p]);
    oz = r * (zkk[q] - zkk[p]);
  };
  auto abs_ = [&](int p, int q, double &ox, double &oy, double &oz) {
    double r = (eps - eek[p]) / (eek[q] - eek[p]);
    ox = r * (xkk[q] - xkk[p]) + xkk[p];
    oy = r * (ykk[q] - ykk[p]) + ykk[p];
    oz = r * (zkk[q] - zkk[p]) + zkk[p];
  };
  double ax, ay, az, bx, by, bz, cx, cy, cz, dx, dy, dz;
  if (eps <= e1) {
    rel(n0, n1, ax, ay, az);
    rel(n0, n2, bx, by, bz);
    rel(n0, n3, cx, cy, cz);
    return fii(ax, ay, az, bx, by, bz, cx, cy, cz);
  }
  if (eps > e1 && eps < e2) {
    abs_(n0, n2, ax, ay, az);
    abs_(n1, n2, bx, by, bz);
    abs_(n0, n3, cx, cy, cz);
    abs_(n1, n3, dx, dy, dz);
    double a1 = fii(ax, ay, az, bx, by, bz, cx, cy, cz);
    double a2 = fii(dx, dy, dz, bx, by, bz, cx, cy, cz);
    double a3 = fii(ax, ay, az, dx, dy, dz, cx, cy, cz);
    double a4 = fii(ax, ay, az, bx, by, bz, dx, dy, dz);
    return 0.50 * (a1 + a2 + a3 + a4);
  }
  if (eps > e2 && eps < e3) {
    rel(n3, n0, ax, ay, az);
    rel(n3, n1, bx, by, bz);
    rel(n3, n2, cx, cy, cz);
    return fii(ax, ay, az, bx, by, bz, cx, cy, cz);
  }
  return 0.0;
}

// FASTSURF, src/Band.cpp:665-704.
double FullBandTables::fastsurf(double eps, int it) const {
  const double e0 = eek[T(0, it)], e1 = eek[T(1, it)], e2 = eek[T(2, it)], e3 = eek[T(3, it)];
  double r;
  if (eps > e0 && eps < e3) {
    if (eps <= e1)
      r = faclow[it] * (eps - e0) * (eps - e0);
    else if (eps < e2) {
      if (e1 - e0 > 1e-10)
        r = faclow[it] * (eps - e0) * (eps - e0) - facmedium[it] * (eps - e1) * (eps - e1);
      else
        r = surf(eps, it);
    } else
      r = fachigh[it] * (eps - e3) * (eps - e3);
  } else
    r = 0.0;
  if (r < 0.0) throw std::runtime_error("FASTSURF: negative area");
  return r;
}

// CALDOS, src/Band.cpp:2234-2264.
double FullBandTables::caldos(double eed, int ib) const {
  const double *d = &dos[(size_t)ib * (kMaxTab + 1)];
  if (eed <= 0e0) return d[0];
  if (eed >= emax) return d[kMaxTab];
  int itab = (int)(eed / dtable);
  double intp = (eed - energy[itab]) / (energy[itab + 1] - energy[itab]);
  return d[itab] + intp * (d[itab + 1] - d[itab]);
}

// CALDOSSUM, src/Band.cpp:2267-2295.
double FullBandTables::caldossum(double eed, int ip) const {
  if (eed <= 0e0) return sumdos[0 * 3 + ip];
  if (eed >= emax) return sumdos[(size_t)kMaxTab * 3 + ip];
  int itab = (int)(eed / dtable);
  double intp = (eed - energy[itab]) / (energy[itab + 1] - energy[itab]);
  return sumdos[(size_t)itab * 3 + ip] + intp * (sumdos[(size_t)(itab + 1) * 3 + ip] - sumdos[(size_t)itab * 3 + ip]);
}

// CALSCATTSUM, src/Band.cpp:1999-2033.
double FullBandTables::calscattsum(double eed, int ib) const {
  if (eed <= 0.0) return sumscatt[0 * kNumBandsMax + ib];
  if (eed >= emax) return sumscatt[(size_t)kMaxTab * kNumBandsMax + ib];
  int itab = (int)(eed / dtable);
  double intp = (eed - energy[itab]) / (energy[itab + 1] - energy[itab]);
  const double a = sumscatt[(size_t)itab * kNumBandsMax + ib], b = sumscatt[(size_t)(itab + 1) * kNumBandsMax + ib];
  return a + intp * (b - a);
}

FullBandTables FullBandTables::build(const std::string &dir, double kelvin) {
  FullBandTables t;
  t.u = Units::at_temperature(kelvin);
  const Units &u = t.u;

  // ---------------------------------------------------------------- IELEC
  // energy discretisation and phonon / scattering parameters,
  // src/Band.cpp:4293-4392.
  t.dtable = 0.0010 / u.eV0;
  const double emin = 0.0;
  t.emax = (double)(kMaxTab)*t.dtable;
  t.energy.resize(kMaxTab + 1);
  for (int i = 0; i <= kMaxTab; ++i) t.energy[i] = (double)(i)*t.dtable + emin;
  t.temptag = 140.0 / u.T0;
  t.templag = 215.0 / u.T0;
  t.templog = 720.0 / u.T0;
  t.temptaf = 220.0 / u.T0;
  t.templaf = 550.0 / u.T0;
  t.temptof = 685.0 / u.T0;
  const double dftag = 4.65e9 / u.dpc0, dflag = 7.44e9 / u.dpc0, dflog = 1.023e11 / u.dpc0;
  const double dftaf = 2.79e9 / u.dpc0, dflaf = 1.86e10 / u.dpc0, dftof = 1.86e10 / u.dpc0;
  const double dfelast = 8.7 / u.eV0;
  t.temphop = 680.0 / u.T0;
  const double dfhop = 4e10 / u.dpc0, dfhelast = 9.3 / u.eV0;
  const double tempoeop = 735.0 / u.T0, dfoeop = 2.2e10 / u.dpc0, dfoeelast = 25.0 / u.eV0;
  const double iifacelec = 0.16;
  t.difpr[0] = 0.16;
  t.difpr[1] = 0.35;
  t.difpr[2] = 0.16;
  double iifachole = 1.14e12;
  const double hiithresh = 1.49 / u.eV0, hiiexp = 3.4;
  iifachole = iifachole * std::pow(u.eV0, hiiexp) * u.time0;
  const double ephb = 1.6;
  t.mell = 0.9116;
  t.melt = 0.1946;
  t.meld = std::pow((t.mell * t.melt * t.melt), (1.0 / 3.0));

  // --------------------------------------------------------------- READBS
  // src/Band.cpp:754-983
  {
    Tokens in(dir + "/bs.si.asc");
    for (int i = 0; i < 3; ++i) t.nband[i] = (int)in.integer();
    if (t.nband[0] > kElecBandsMax || t.nband[1] > kHoleBandsMax || t.nband[2] > 1)
      throw std::runtime_error("bs.si.asc: too many bands");
    t.nbt = t.nband[0] + t.nband[1] + t.nband[2];
    t.bandof[0] = 0;
    t.bandof[1] = t.nband[0];
    t.bandof[2] = t.nband[0] + t.nband[1];
    t.nk = (int)in.integer();
    t.xkk.resize(t.nk);
    t.ykk.resize(t.nk);
    t.zkk.resize(t.nk);
    t.eek.resize(t.nk);
    for (auto *v : {&t.xkk, &t.ykk, &t.zkk, &t.eek})
      for (int i = 0; i < t.nk; ++i) (*v)[i] = in.real();
    for (int i = 0; i < t.nk; ++i)
      if (t.eek[i] < 0.0) throw std::runtime_error("bs.si.asc: negative energy");
    t.nt = (int)in.integer();
    t.tet.resize((size_t)4 * t.nt);
    t.neib.resize((size_t)4 * t.nt);
    t.ibt.resize(t.nt);
    for (int v = 0; v < 4; ++v)
      for (int it = 0; it < t.nt; ++it) t.tet[(size_t)v * t.nt + it] = (int)in.integer() - 1;
    for (int f = 0; f < 4; ++f)
      for (int it = 0; it < t.nt; ++it) t.neib[(size_t)f * t.nt + it] = (int)in.integer() - 1;
    for (int it = 0; it < t.nt; ++it) t.ibt[it] = (int)in.integer() - 1;
    for (int i = 0; i < t.nk; ++i) {
      t.xkk[i] = t.xkk[i] * u.a0pi;
      t.ykk[i] = t.ykk[i] * u.a0pi;
      t.zkk[i] = t.zkk[i] * u.a0pi;
      t.eek[i] = t.eek[i] / u.eV0;
    }
  }
  const int nt = t.nt;

  // VELOTET, src/Band.cpp:3-68: constant gradient of the linear band in each tet.
  t.vt.resize((size_t)4 * nt);
  t.vgt.resize(nt);
  for (int it = 0; it < nt; ++it) {
    const int n0 = t.T(0, it), n1 = t.T(1, it), n2 = t.T(2, it), n3 = t.T(3, it);
    const double m11 = t.xkk[n1] - t.xkk[n0], m12 = t.ykk[n1] - t.ykk[n0], m13 = t.zkk[n1] - t.zkk[n0];
    const double m21 = t.xkk[n2] - t.xkk[n0], m22 = t.ykk[n2] - t.ykk[n0], m23 = t.zkk[n2] - t.zkk[n0];
    const double m31 = t.xkk[n3] - t.xkk[n0], m32 = t.ykk[n3] - t.ykk[n0], m33 = t.zkk[n3] - t.zkk[n0];
    const double det = m11 * (m22 * m33 - m32 * m23) - m12 * (m21 * m33 - m31 * m23) + m13 * (m21 * m32 - m31 * m22);
    const double i11 = (m22 * m33 - m32 * m23) / det, i21 = -(m21 * m33 - m31 * m23) / det;
    const double i31 = (m21 * m32 - m31 * m22) / det, i12 = -(m12 * m33 - m32 * m13) / det;
    const double i22 = (m11 * m33 - m31 * m13) / det, i32 = -(m11 * m32 - m31 * m12) / det;
    const double i13 = (m12 * m23 - m22 * m13) / det, i23 = -(m11 * m23 - m21 * m13) / det;
    const double i33 = (m11 * m22 - m21 * m12) / det;
    const double a1 = t.eek[n1] - t.eek[n0], a2 = t.eek[n2] - t.eek[n0], a3 = t.eek[n3] - t.eek[n0];
    double *v = &t.vt[(size_t)4 * it];
    v[0] = i11 * a1 + i12 * a2 + i13 * a3;
    v[1] = i21 * a1 + i22 * a2 + i23 * a3;
    v[2] = i31 * a1 + i32 * a2 + i33 * a3;
    v[3] = t.eek[n0];
    t.vgt[it] = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  }

  // HESSTET, src/Band.cpp:356-463: inward normals (n, d) of the four faces,
  // n.k >= d inside.  Face f is opposite node (f+3)%4... as the reference
  // orders them: face 0 through nodes 1,2,3; face 1 through 0,2,3 (wait: the
  // plane of d x f contains nodes 0,2,3); face 2 through 0,1,3; face 3 through 0,1,2.
  t.datantlin.resize((size_t)16 * nt);
  for (int it = 0; it < nt; ++it) {
    const int n[4] = {t.T(0, it), t.T(1, it), t.T(2, it), t.T(3, it)};
    auto X = [&](int v) { return t.xkk[n[v]]; };
    auto Y = [&](int v) { return t.ykk[n[v]]; };
    auto Z = [&](int v) { return t.zkk[n[v]]; };
    const double ax = X(1) - X(0), ay = Y(1) - Y(0), az = Z(1) - Z(0);
    const double bx = X(2) - X(1), by = Y(2) - Y(1), bz = Z(2) - Z(1);
    const double dx = X(3) - X(0), dy = Y(3) - Y(0), dz = Z(3) - Z(0);
    const double ex = X(3) - X(1), ey = Y(3) - Y(1), ez = Z(3) - Z(1);
    const double fx = X(3) - X(2), fy = Y(3) - Y(2), fz = Z(3) - Z(2);
    // (normal, node on the plane, node that must be on the inner side)
    const double nrm[4][3] = {{ey * fz - ez * fy, ez * fx - ex * fz, ex * fy - ey * fx},
                              {dy * fz - dz * fy, dz * fx - dx * fz, dx * fy - dy * fx},
                              {ey * dz - ez * dy, ez * dx - ex * dz, ex * dy - ey * dx},
                              {ay * bz - az * by, az * bx - ax * bz, ax * by - ay * bx}};
    const int on[4] = {1, 2, 3, 0}, inner[4] = {0, 1, 2, 3};
    for (int f = 0; f < 4; ++f) {
      double c0 = nrm[f][0], c1 = nrm[f][1], c2 = nrm[f][2];
      double c3 = c0 * X(on[f]) + c1 * Y(on[f]) + c2 * Z(on[f]);
      if (c0 * X(inner[f]) + c1 * Y(inner[f]) + c2 * Z(inner[f]) < c3) {
        c0 = -c0;
        c1 = -c1;
        c2 = -c2;
        c3 = -c3;
      }
      t.D(0, f, it) = c0;
      t.D(1, f, it) = c1;
      t.D(2, f, it) = c2;
      t.D(3, f, it) = c3;
    }
  }

  // SETMATSYM, src/Band.cpp:986-1299.
  std::memset(t.indmat, 0, sizeof(t.indmat));
  for (int s = 0; s < 48; ++s) {
    for (int c = 0; c < 6; ++c) t.matsym[c][s] = kSymOps[s][c];
    const int idx = ((((((t.matsym[3][s] + 1) * 3 + (t.matsym[4][s] + 1)) * 3 + (t.matsym[5][s] + 1)) * 3 +
                       (t.matsym[0][s] - 1)) * 3 + (t.matsym[1][s] - 1)) * 3 + (t.matsym[2][s] - 1));
    t.indmat[idx] = s;
  }

  // SETNEIBSYM, src/Band.cpp:466-552: lattice shift and new wedge when a
  // particle leaves wedge isym through each of its five outer faces.
  {
    const double a = u.a0pi;
    const double tr[5][3] = {{0.5 * a, 0.3 * a, -0.01 * a},
                             {0.49 * a, 0.51 * a, 0.1 * a},
                             {0.5 * a, 0.24 * a, 0.26 * a},
                             {0.71 * a, 0.51 * a, 0.31 * a},
                             {1.01 * a, 0.1 * a, 0.05 * a}};
    for (int s = 0; s < 48; ++s)
      for (int iv = 0; iv < 5; ++iv) {
        const double vin[3] = {tr[iv][0], tr[iv][1], tr[iv][2]};
        double xk = vin[t.matsym[0][s] - 1] * t.matsym[3][s];
        double yk = vin[t.matsym[1][s] - 1] * t.matsym[4][s];
        double zk = vin[t.matsym[2][s] - 1] * t.matsym[5][s];
        const double xkl = xk, ykl = yk, zkl = zk;
        // CONFBZ, src/Band.cpp:573-616
        for (;;) {
          bool out = std::fabs(xk) > a || std::fabs(yk) > a || std::fabs(zk) > a ||
                     std::fabs(xk) + std::fabs(yk) + std::fabs(zk) > 1.50 * a;
          if (!out) break;
          xk = xk > 0.0 ? xk - a : xk + a;
          yk = yk > 0.0 ? yk - a : yk + a;
          zk = zk > 0.0 ? zk - a : zk + a;
        }
        t.xbz[iv][s] = xk - xkl;
        t.ybz[iv][s] = yk - ykl;
        t.zbz[iv][s] = zk - zkl;
        if (std::fabs(t.xbz[iv][s]) < 1e-10) t.xbz[iv][s] = 0.0;
        if (std::fabs(t.ybz[iv][s]) < 1e-10) t.ybz[iv][s] = 0.0;
        if (std::fabs(t.zbz[iv][s]) < 1e-10) t.zbz[iv][s] = 0.0;
        int pos[3] = {1, 1, 1}, mink, maxk;
        double tmin, tmax;
        if (std::fabs(xk) > std::fabs(yk)) {
          tmin = std::fabs(yk); tmax = std::fabs(xk); mink = 1; maxk = 0;
        } else {
          tmin = std::fabs(xk); tmax = std::fabs(yk); mink = 0; maxk = 1;
        }
        if (std::fabs(zk) < tmin) mink = 2;
        else if (std::fabs(zk) > tmax) maxk = 2;
        pos[mink] = 2;
        pos[maxk] = 0;
        const int idx = (((((isign(xk) + 1) * 3 + (isign(yk) + 1)) * 3 + (isign(zk) + 1)) * 3 + pos[0]) * 3 + pos[1]) * 3 + pos[2];
        t.newisym[iv][s] = t.indmat[idx];
      }
  }

  // CALCFAC, src/Band.cpp:619-662: area(E) is quadratic on each node interval.
  t.faclow.assign(nt, 0.0);
  t.facmedium.assign(nt, 0.0);
  t.fachigh.assign(nt, 0.0);
  for (int it = 0; it < nt; ++it) {
    const double e0 = t.eek[t.T(0, it)], e1 = t.eek[t.T(1, it)], e2 = t.eek[t.T(2, it)], e3 = t.eek[t.T(3, it)];
    if (e1 > e0) {
      double eps = 0.50 * (e0 + e1);
      t.faclow[it] = t.surf(eps, it) / ((eps - e0) * (eps - e0));
    }
    if (e3 > e2) {
      double eps = 0.50 * (e2 + e3);
      t.fachigh[it] = t.surf(eps, it) / ((eps - e3) * (eps - e3));
    }
    if (e2 > e1) {
      double eps = 0.5 * (e2 + e1);
      t.facmedium[it] = (t.faclow[it] * (eps - e0) * (eps - e0) - t.surf(eps, it)) / ((eps - e1) * (eps - e1));
    }
  }

  // ----------------------------------------------------------- BUILDLISTS
  // src/Band.cpp:3843-4268 (energy lists and BZ-surface lists).
  t.dlist = u.eV0 / 0.040;
  t.dlists = u.eV0 / 0.0020;
  t.ntlist.assign((size_t)kCoarseBins * kNumBandsMax, 0);
  t.nslist.assign((size_t)kCoarseBins * kNumBandsMax, 0);
  t.ntlists.assign((size_t)kFineBins * kNumBandsMax, 0);
  auto on_bz_surface = [&](int it) {
    for (int f = 0; f < 4; ++f)
      if (t.N(f, it) == -5 || t.N(f, it) == -6) return true;
    return false;
  };
  auto coarse_span = [&](int it, int &b, int &e) {
    b = int(t.eek[t.T(0, it)] * t.dlist);
    e = int(t.eek[t.T(3, it)] * t.dlist);
  };
  auto fine_span = [&](int it, int &b, int &e) {
    b = int(t.eek[t.T(0, it)] * t.dlists);
    e = int(t.eek[t.T(3, it)] * t.dlists);
    if (e >= kFineBins) e = kFineBins - 1;
  };
  for (int it = 0; it < nt; ++it) {
    int b, e;
    coarse_span(it, b, e);
    if (e >= kCoarseBins) throw std::runtime_error("BUILDLISTS: tetrahedron above the list range");
    const bool s = on_bz_surface(it);
    if (b >= 0)
      for (int i = b; i <= e; ++i) {
        t.ntlist[(size_t)i * kNumBandsMax + t.ibt[it]] += 1;
        if (s) t.nslist[(size_t)i * kNumBandsMax + t.ibt[it]] += 1;
      }
    fine_span(it, b, e);
    if (b >= 0)
      for (int i = b; i <= e; ++i) t.ntlists[(size_t)i * kNumBandsMax + t.ibt[it]] += 1;
  }
  t.ptlist.assign(t.ntlist.size(), 0);
  t.pslist.assign(t.nslist.size(), 0);
  t.ptlists.assign(t.ntlists.size(), 0);
  {
    int ip = 0, ips = 0, ipss = 0;
    for (int ib = 0; ib < t.nbt; ++ib) {
      for (int i = 0; i < kCoarseBins; ++i) {
        ip += t.ntlist[(size_t)i * kNumBandsMax + ib];
        t.ptlist[(size_t)i * kNumBandsMax + ib] = ip;
        ips += t.nslist[(size_t)i * kNumBandsMax + ib];
        t.pslist[(size_t)i * kNumBandsMax + ib] = ips;
      }
      for (int i = 0; i < kFineBins; ++i) {
        ipss += t.ntlists[(size_t)i * kNumBandsMax + ib];
        t.ptlists[(size_t)i * kNumBandsMax + ib] = ipss;
      }
    }
    t.tlist.assign(ip, 0);
    t.slist.assign(ips, 0);
    t.tlists.assign(ipss, 0);
  }
  // fill from the end of each bin, so each bin lists its tets in descending order
  for (int it = 0; it < nt; ++it) {
    int b, e;
    coarse_span(it, b, e);
    const bool s = on_bz_surface(it);
    if (b >= 0)
      for (int i = b; i <= e; ++i) {
        int &p = t.ptlist[(size_t)i * kNumBandsMax + t.ibt[it]];
        t.tlist[--p] = it;
        if (s) {
          int &q = t.pslist[(size_t)i * kNumBandsMax + t.ibt[it]];
          t.slist[--q] = it;
        }
      }
    fine_span(it, b, e);
    if (b >= 0)
      for (int i = b; i <= e; ++i) {
        int &p = t.ptlists[(size_t)i * kNumBandsMax + t.ibt[it]];
        t.tlists[--p] = it;
      }
  }

  // --------------------------------------------------------------- GETDOS
  // src/Band.cpp:3661-3840 (tables read from zd.si.asc, then normalised).
  t.dos.assign((size_t)kNumBandsMax * (kMaxTab + 1), 0.0);
  t.dostetmax.assign((size_t)kNumBandsMax * (kMaxTab + 1), 0.0);
  t.sumdos.assign((size_t)(kMaxTab + 1) * 3, 0.0);
  {
    Tokens in(dir + "/zd.si.asc");
    if (in.integer() != kMaxTab) throw std::runtime_error("zd.si.asc: wrong number of table entries");
    for (int i = 0; i <= kMaxTab; ++i) {
      in.real();
      for (int ib = 0; ib < t.nbt; ++ib) t.dos[(size_t)ib * (kMaxTab + 1) + i] = in.real();
      for (int ip = 0; ip < 3; ++ip) {
        double s = 0.0;
        for (int ib = t.bandof[ip]; ib < t.nband[ip] + t.bandof[ip]; ++ib) s = s + t.dos[(size_t)ib * (kMaxTab + 1) + i];
        t.sumdos[(size_t)i * 3 + ip] = s;
      }
    }
    in.integer();
    for (int i = 0; i <= kMaxTab; ++i) {
      in.real();
      for (int ib = 0; ib < t.nbt; ++ib) t.dostetmax[(size_t)ib * (kMaxTab + 1) + i] = in.real();
    }
  }
  for (int i = 0; i <= kMaxTab; ++i) {
    for (int ib = 0; ib < t.nbt; ++ib) {
      double &d = t.dos[(size_t)ib * (kMaxTab + 1) + i];
      d = d * u.eV0 * std::pow(u.spr0, 3.0);
      double &m = t.dostetmax[(size_t)ib * (kMaxTab + 1) + i];
      m = m * u.velo0 / (u.spk0 * u.spk0);
    }
    for (int ip = 0; ip < 3; ++ip) {
      double &s = t.sumdos[(size_t)i * 3 + ip];
      s = s * u.eV0 * std::pow(u.spr0, 3.0);
      t.dosmax[ip] = dmax(t.dosmax[ip], s);
    }
  }

  // --------------------------------------------------------- BUILDPHSCATT
  // src/Band.cpp:1302-1910, Jacoboni phonon system (jacophfl = true).
  const int NT = kMaxTab + 1;
  t.scatte.assign((size_t)kElecMech * kElecBandsMax * kElecBandsMax, 0.0);
  t.dose.assign((size_t)kElecMech * kElecBandsMax * NT, 0.0);
  t.scattiie.assign((size_t)kElecBandsMax * kElecBandsMax * NT, 0.0);
  t.scatth.assign((size_t)kHoleMech * kHoleBandsMax * kHoleBandsMax, 0.0);
  t.dosh.assign((size_t)kHoleMech * kHoleBandsMax * NT, 0.0);
  t.scattiih.assign((size_t)kHoleBandsMax * kHoleBandsMax * NT, 0.0);
  {
    const double bes[6] = {1.0 / (std::exp(t.temptag) - 1.0), 1.0 / (std::exp(t.templag) - 1.0),
                           1.0 / (std::exp(t.templog) - 1.0), 1.0 / (std::exp(t.temptaf) - 1.0),
                           1.0 / (std::exp(t.templaf) - 1.0), 1.0 / (std::exp(t.temptof) - 1.0)};
    t.scpre = 14;
    const double kint = 2.0 * kPi * dfelast * dfelast / u.sirho / 6e0 / (u.siul * u.siul);
    double kem[6] = {(dftag) * (dftag)*kPi / t.temptag / u.sirho / 6e0, (dflag) * (dflag)*kPi / t.templag / u.sirho / 6e0,
                     (dflog) * (dflog)*kPi / t.templog / u.sirho / 6e0, (dftaf) * (dftaf)*kPi / t.temptaf / u.sirho * 0.666e0,
                     (dflaf) * (dflaf)*kPi / t.templaf / u.sirho * 0.666e0, (dftof) * (dftof)*kPi / t.temptof / u.sirho * 0.666e0};
    double kab[6];
    for (int m = 0; m < 6; ++m) kab[m] = bes[m] * kem[m];
    for (int m = 0; m < 6; ++m) kem[m] = (bes[m] + 1.0) * kem[m];
    const double shift[6] = {t.temptag, t.templag, t.templog, t.temptaf, t.templaf, t.temptof};
    for (int f = 0; f < t.nband[0]; ++f)
      for (int i = 0; i < NT; ++i) {
        const double ee = t.energy[i];
        const int band = f + t.bandof[0];
        t.dose[((size_t)0 * kElecBandsMax + f) * NT + i] = t.caldos(ee, band);
        for (int m = 0; m < 6; ++m) {
          t.dose[((size_t)(1 + 2 * m) * kElecBandsMax + f) * NT + i] = t.caldos(ee + shift[m], band);
          t.dose[((size_t)(2 + 2 * m) * kElecBandsMax + f) * NT + i] = t.caldos(ee - shift[m], band);
        }
      }
    for (int ini = 0; ini < t.nband[0]; ++ini)
      for (int f = 0; f < t.nband[0]; ++f) {
        const double dosfac = (ini == 0 && f == 0) ? 1.0 : ephb;
        auto S = [&](int m) -> double & { return t.scatte[((size_t)m * kElecBandsMax + f) * kElecBandsMax + ini]; };
        S(0) = kint * dosfac;
        for (int m = 0; m < 6; ++m) {
          S(1 + 2 * m) = kab[m] * dosfac;
          S(2 + 2 * m) = kem[m] * dosfac;
        }
      }
    t.scprh = 4;
    const double besh = 1.0 / (std::exp(t.temphop) - 1.0);
    const double kinth = 2e0 * kPi * dfhelast * dfhelast / u.sirho / 2.0 / (u.siul * u.siul);
    double kemh = dfhop * dfhop * kPi / t.temphop / u.sirho;
    const double kabh = besh * kemh;
    kemh = (besh + 1.0) * kemh;
    for (int f = 0; f < t.nband[1]; ++f)
      for (int i = 0; i < NT; ++i) {
        const double ee = t.energy[i];
        const int band = f + t.bandof[1];
        t.dosh[((size_t)0 * kHoleBandsMax + f) * NT + i] = t.caldos(ee, band);
        t.dosh[((size_t)1 * kHoleBandsMax + f) * NT + i] = t.caldos(ee + t.temphop, band);
        t.dosh[((size_t)2 * kHoleBandsMax + f) * NT + i] = t.caldos(ee - t.temphop, band);
      }
    for (int ini = 0; ini < t.nband[1]; ++ini)
      for (int f = 0; f < t.nband[1]; ++f) {
        t.scatth[((size_t)0 * kHoleBandsMax + f) * kHoleBandsMax + ini] = kinth;
        t.scatth[((size_t)1 * kHoleBandsMax + f) * kHoleBandsMax + ini] = kabh;
        t.scatth[((size_t)2 * kHoleBandsMax + f) * kHoleBandsMax + ini] = kemh;
      }
    // impact ionisation, Thoma formula (thomiifl), EIIRATE :1913-1972 and HIIRATE :1975-1996
    auto eiirate = [&](double ee) {
      double eel = ee - u.sieg + 1.1241e0 / u.eV0, sii = 0.0;
      if ((eel * u.eV0 > 1.128e0) && (eel * u.eV0 < 1.75e0))
        sii = 1.25e12 / u.scrt0 * std::pow((eel * u.eV0 - 1.128e0), 3);
      else if (eel * u.eV0 > 1.75e0)
        sii = 9.49e12 / u.scrt0 * (eel * u.eV0 - 1.572e0) * (eel * u.eV0 - 1.572e0);
      return sii * iifacelec;
    };
    auto hiirate = [&](double ee) {
      double eel = ee - u.sieg + 1.1241e0 / u.eV0;
      return eel > hiithresh ? iifachole * std::pow((eel - hiithresh), hiiexp) : 0.0;
    };
    for (int ipt = 0; ipt < 2; ++ipt) {
      const int nb = t.nband[ipt];
      std::vector<double> &dst = ipt == 0 ? t.scattiie : t.scattiih;
      const int stride = ipt == 0 ? kElecBandsMax : kHoleBandsMax;
      for (int ini = 0; ini < nb; ++ini)
        for (int f = 0; f < nb; ++f)
          for (int i = 0; i < NT; ++i) {
            const double ee = t.energy[i];
            const double sii = ipt == 0 ? eiirate(ee) : hiirate(ee);
            const double after = (ee - u.sieg) / 3.0;
            double d1 = 0.0, d2 = 1.0;
            if (after > 0.0) {
              d1 = t.caldos(after, f + t.bandof[ipt]);
              d2 = t.caldossum(after, ipt);
              if (d2 == 0.0) {
                d1 = 0.0;
                d2 = 1.0;
              }
            }
            dst[((size_t)f * stride + ini) * NT + i] = d1 / d2 * sii;
          }
    }
    // oxide electrons, only their total rate is needed (:1772-1817)
    const double besoe = 1.0 / (std::exp(tempoeop) - 1.0);
    const double kintoe = 2.0 * kPi * (dfoeelast * dfoeelast) / u.sirho / 2e0 / (u.siul * u.siul);
    double kemoe = (dfoeop * dfoeop) * 1.5e0 * kPi / tempoeop / u.sirho;
    const double kaboe = besoe * kemoe;
    kemoe = (besoe + 1.0) * kemoe;
    (void)kemoe;

    // total rates per band, :1818-1889
    t.sumscatt.assign((size_t)NT * kNumBandsMax, 0.0);
    for (int i = 0; i < NT; ++i) {
      for (int ini = 0; ini < t.nband[0]; ++ini)
        for (int f = 0; f < t.nband[0]; ++f) {
          double &s = t.sumscatt[(size_t)i * kNumBandsMax + ini + t.bandof[0]];
          for (int m = 0; m < t.scpre - 1; ++m)
            s = s + t.scatte[((size_t)m * kElecBandsMax + f) * kElecBandsMax + ini] * t.dose[((size_t)m * kElecBandsMax + f) * NT + i];
          s = s + t.scattiie[((size_t)f * kElecBandsMax + ini) * NT + i];
        }
    }
    for (int i = 0; i < NT; ++i) {
      for (int ini = 0; ini < t.nband[1]; ++ini)
        for (int f = 0; f < t.nband[1]; ++f) {
          double &s = t.sumscatt[(size_t)i * kNumBandsMax + ini + t.bandof[1]];
          for (int m = 0; m < t.scprh - 1; ++m)
            s = s + t.scatth[((size_t)m * kHoleBandsMax + f) * kHoleBandsMax + ini] * t.dosh[((size_t)m * kHoleBandsMax + f) * NT + i];
          s = s + t.scattiih[((size_t)f * kHoleBandsMax + ini) * NT + i];
        }
    }
    for (int i = 0; i < NT; ++i) {
      const double ee = t.energy[i];
      for (int ini = 0; ini < t.nband[2]; ++ini)
        for (int f = 0; f < t.nband[2]; ++f) {
          const int band = f + t.bandof[2];
          double &s = t.sumscatt[(size_t)i * kNumBandsMax + ini + t.bandof[2]];
          s = s + kintoe * t.caldos(ee, band);
          s = s + kaboe * t.caldos(ee + tempoeop, band);
        }
    }
  }
  // GETINDENS, src/Band.cpp:3609-3656: intrinsic density from the DOS tables.
  {
    double en0 = 0.0, ep0 = 0.0, eelmo = t.energy[0];
    for (int i = 1; i <= kMaxTab; ++i) {
      const double eel = t.energy[i];
      double dosl = t.caldossum(eel, 0), doslmo = t.caldossum(eelmo, 0);
      en0 = en0 + ((doslmo * eel - dosl * eelmo) * (std::exp(-eelmo) - std::exp(-eel)) +
                   (dosl - doslmo) * ((eelmo + 1e0) * std::exp(-eelmo) - (eel + 1e0) * std::exp(-eel))) /
                      (eel - eelmo);
      dosl = t.caldossum(eel, 1);
      doslmo = t.caldossum(eelmo, 1);
      ep0 = ep0 + ((doslmo * eel - dosl * eelmo) * (std::exp(-eelmo) - std::exp(-eel)) +
                   (dosl - doslmo) * ((eelmo + 1e0) * std::exp(-eelmo) - (eel + 1e0) * std::exp(-eel))) /
                      (eel - eelmo);
      eelmo = eel;
    }
    en0 = 2e0 * en0;
    ep0 = 2e0 * ep0;
    t.ni = std::sqrt(en0 * ep0 * std::exp(-u.sieg));
  }
  // gamtet: majorant of the total rate over the tet's energy span, :1890-1906
  t.gamtet.assign(nt, 0.0);
  for (int it = 0; it < nt; ++it) {
    const int itabl = int(dmax(0, (int)(t.eek[t.T(0, it)] / t.dtable)));
    const int itabu = int(dmin(kMaxTab, (int)(t.eek[t.T(3, it)] / t.dtable) + 1));
    double g = 0.0;
    for (int i = itabl; i <= itabu; ++i) g = dmax(g, t.sumscatt[(size_t)i * kNumBandsMax + t.ibt[it]]);
    if (g == 0.0) g = t.sumscatt[(size_t)kMaxTab * kNumBandsMax + t.ibt[it]];
    t.gamtet[it] = g;
  }
  // ------------------------------------------------------------ init_deep
  // src/ParticleUtils.cpp:750-806: for each table, columns (energy bins)
  // outer, rows inner.  All six or none.
  {
    std::vector<double> all;
    bool ok = true;
    for (int d = 0; d < kDispTables && ok; ++d) {
      std::ifstream f(dir + "/" + kDispNames[d] + ".txt");
      if (!f) {
        ok = false;
        break;
      }
      t.disp_off[d] = (int)all.size();
      all.resize(all.size() + (size_t)kDispRows[d] * kDispCols[d]);
      double *tab = all.data() + t.disp_off[d];
      for (int col = 0; col < kDispCols[d] && ok; ++col)
        for (int row = 0; row < kDispRows[d]; ++row)
          if (!(f >> tab[(size_t)row * kDispCols[d] + col])) {
            ok = false;
            break;
          }
    }
    if (ok) t.dispersion.swap(all);
  }
  return t;
}

}  // namespace mcb200
