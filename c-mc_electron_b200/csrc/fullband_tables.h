// fullband_tables.h -- host-side builder for the full-band Monte Carlo tables
// of silicon that the carrier kernels read from HBM / L2.
//
// The tables are the ones the reference builds in Band::IELEC
// (src/Band.cpp:4271-4476) from the reference's own data files
// (input/bs.si.asc: k-grid + tetrahedra, input/zd.si.asc: DOS tables).  This
// builder reads the same files and reproduces every table the carrier path
// consumes, bit for bit (same IEEE double operations in the same order;
// checked against the reference by the CPU parity tests).  Tables only the
// Fischetti phonon model or the injection helpers use (dosfp*, zlist, the
// k-dispersion tables of init_deep) are not built: those models are off on
// this path (fiscphfl = false, src/Band.cpp:4318).
//
// Units are the reference's normalised ones: energy in kB*T, k in 1/spr0,
// time in hbar/(kB*T) (src/mcmodel.cpp:4047-4071).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace mcb200 {

// Sizes fixed by the reference's table layout (include/Constant_GlobalVariable_MathFunction.h).
constexpr int kMaxTab = 7500;          // MTAB: energy table has kMaxTab+1 points
constexpr int kNumBandsMax = 8;        // MNB
constexpr int kElecBandsMax = 4;       // NBE
constexpr int kHoleBandsMax = 3;       // NBH
constexpr int kCoarseBins = 325;       // MWLE: 40 meV tetrahedron lists
constexpr int kFineBins = 60;          // MWLES: 2 meV tetrahedron lists
constexpr int kElecMech = 14;          // MNScaEle
constexpr int kHoleMech = 4;           // MNScaHole

// Normalisation and material constants at one lattice temperature
// (MeshQuantities::init_phpysical_parameter, src/mcmodel.cpp:4007-4122).
struct Units {
  double T0, Tn;
  double eV0, em0, hq0, ec0, rmom0, spr0, spk0, time0, velo0, cvr, pot0, field0, conc0, dens0, dpc0,
      scrt0, curr0;
  double sia0, sirho, siul, siut, sieg, a0pi;
  double eps_vacuum, eps_oxide, eps_silicon;
  double frickel;
  static Units at_temperature(double kelvin);
};

struct FullBandTables {
  Units u;
  // --- k-space grid and tetrahedra (READBS, src/Band.cpp:754-983)
  int nband[3] = {0, 0, 0};  // electron, hole, oxide-electron bands
  int bandof[3] = {0, 0, 0};
  int nbt = 0;
  int nk = 0, nt = 0;
  std::vector<double> xkk, ykk, zkk, eek;  // [nk]
  std::vector<int> tet;                    // [4][nt] node index, energies ascending
  std::vector<int> neib;                   // [4][nt] NeibrTet: >=0 tet, <0 wedge/BZ code
  std::vector<int> ibt;                    // [nt] band of each tet
  std::vector<double> vt;                  // [4*nt] group velocity (3) + base energy
  std::vector<double> vgt;                 // [nt] |v|
  std::vector<double> datantlin;           // [4 comp][4 face][nt] inward face normals + offset
  std::vector<double> faclow, facmedium, fachigh;  // [nt] FASTSURF coefficients
  // --- 48 symmetry operations of the BZ (SETMATSYM / SETNEIBSYM)
  int matsym[6][48];
  int indmat[729];  // [sx+1][sy+1][sz+1][p0][p1][p2] -> isym
  int newisym[5][48];
  double xbz[5][48], ybz[5][48], zbz[5][48];
  // --- energy-binned tetrahedron lists (BUILDLISTS, src/Band.cpp:3843-4268)
  double dlist = 0, dlists = 0;
  std::vector<int> ntlist, ptlist;    // [kCoarseBins][MNB]
  std::vector<int> tlist;
  std::vector<int> nslist, pslist;    // BZ-surface tetrahedra, same binning
  std::vector<int> slist;
  std::vector<int> ntlists, ptlists;  // [kFineBins][MNB]
  std::vector<int> tlists;
  // --- DOS and scattering-rate tables (GETDOS, BUILDPHSCATT)
  double dtable = 0, emax = 0;
  std::vector<double> energy;     // [kMaxTab+1]
  std::vector<double> dos;        // [MNB][kMaxTab+1]
  std::vector<double> sumdos;     // [kMaxTab+1][3]
  std::vector<double> dostetmax;  // [MNB][kMaxTab+1]
  double dosmax[3] = {0, 0, 0};
  int scpre = 14, scprh = 4;
  std::vector<double> scatte;    // [kElecMech][NBE][NBE]   (mech, final, initial)
  std::vector<double> dose;      // [kElecMech][NBE][kMaxTab+1]
  std::vector<double> scattiie;  // [NBE][NBE][kMaxTab+1]   (final, initial, tab)
  std::vector<double> scatth;    // [kHoleMech][NBH][NBH]
  std::vector<double> dosh;      // [kHoleMech][NBH][kMaxTab+1]
  std::vector<double> scattiih;  // [NBH][NBH][kMaxTab+1]
  std::vector<double> sumscatt;  // [kMaxTab+1][MNB]
  std::vector<double> gamtet;    // [nt] majorant of the total rate over the tet's energy span
  // --- phonon energies and scattering parameters (IELEC)
  double temptag, templag, templog, temptaf, templaf, temptof, temphop;
  double difpr[3];
  double mell, melt, meld;
  double ni = 0;         // intrinsic carrier density (GETINDENS), normalised
  // --- phonon dispersion tables (init_deep, src/ParticleUtils.cpp:750-806):
  // the final-energy distributions of the LO / TO / LA phonon events under
  // quantum correction (FEK*, src/ElectronPhononScatter.cpp:633-1022).
  // Table d is [kDispRows[d]][kDispCols[d]] at dispersion[disp_off[d]], in
  // the order of kDispNames; `dispersion` stays empty when a file is absent.
  std::vector<double> dispersion;
  int disp_off[6] = {0, 0, 0, 0, 0, 0};
  bool seciifl = false;  // secondary particles from impact ionisation (off in the reference)

  // Build everything from a directory holding bs.si.asc and zd.si.asc.
  // Throws std::runtime_error with a readable message on a bad file.
  static FullBandTables build(const std::string &table_dir, double kelvin);

  // Reference helpers re-stated for table construction (src/Band.cpp).
  double surf(double eps, int it) const;     // SURF  :194-332
  double fastsurf(double eps, int it) const; // FASTSURF :665-704
  double caldos(double eed, int ib) const;   // CALDOS :2234-2264
  double caldossum(double eed, int ip) const;// CALDOSSUM :2267-2295
  double calscattsum(double eed, int ib) const; // CALSCATTSUM :1999-2033
  int T(int v, int it) const { return tet[(size_t)v * nt + it]; }
  int N(int f, int it) const { return neib[(size_t)f * nt + it]; }
  double &D(int comp, int face, int it) { return datantlin[((size_t)comp * 4 + face) * nt + it]; }
  double D(int comp, int face, int it) const { return datantlin[((size_t)comp * 4 + face) * nt + it]; }
};

double fii(double x1, double y1, double z1, double x2, double y2, double z2, double x3, double y3, double z3);

// The six dispersion tables: LO emission / absorption, TO emission /
// absorption, LA emission / absorption (files <name>.txt in the table
// directory, read column by column as init_deep does).
constexpr int kDispTables = 6;
constexpr const char *kDispNames[kDispTables] = {"kloem", "kloab", "ktoem", "ktoab", "klaem", "klaab"};
constexpr int kDispRows[kDispTables] = {201, 201, 51, 51, 51, 51};
constexpr int kDispCols[kDispTables] = {120, 110, 160, 150, 160, 150};

}  // namespace mcb200
