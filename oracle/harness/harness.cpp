/*
 * harness.cpp -- ORACLE TEST INFRASTRUCTURE (never linked into the engine).
 *
 * Drives the reference's own MeshQuantities routines, compiled unmodified
 * from src/*.cpp against the single-rank shim in oracle/shim, and exposes
 * them through a C ABI for the parity tests (ctypes) and for the CPU
 * baseline leg of bench.py.  MeshQuantities keeps every member private
 * (include/mcmodel.h:28), so this translation unit reads the reference's
 * header with `class` spelled `struct` (same layout, public access); it adds
 * no physics of its own.
 *
 * Random-number hook.  The reference draws every uniform from the free
 * function `double Random()` (declared include/utils.h:171, defined
 * src/utils.cpp:426-470 on top of ran1).  The oracle build compiles
 * src/utils.cpp with -DRandom=ref_ran1_Random, so the definition below is
 * the one every other reference TU calls: it returns draw n of the Philox
 * stream (seed, uid, step, sub) defined in include/mcb200_rng.h, the stream
 * the B200 kernels use.  The harness sets (uid, step, sub) and resets n
 * before each particle's flight, so each particle sees exactly the draws the
 * engine gives the same particle.
 *
 * Mid-step copies.  GENERATE / GENREF (src/CellHit.cpp:435-501) append a copy
 * of the particle to the neighbour cell's list.  The reference's sweep
 * (src/mcmodel.cpp:1460-1505) then flies that copy or not depending on cell
 * iteration order.  The engine defines one behaviour: the copy finishes the
 * rest of its step in the same step, drawing from stream
 * sub' = sub * 16 + 1 + k for the k-th copy made by a particle, and, if it
 * survives that flight, gets a permanent uid afterwards in (parent uid,
 * sub') order.  orc_flight_step applies exactly that rule to the reference
 * routines.
 */
#include <assert.h>
#include <libgen.h>
#include <math.h>
#include <string.h>
#include <time.h>
#include <sys/stat.h>
#include <unistd.h>
#include <algorithm>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <list>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "shim_trilinos.h"
#include "mcb200_rng.h"
#define class struct
#include "mcmodel.h"
#include "PoissonSolver.h"
#undef class

/* ------------------------------------------------------- random hook -- */
static uint64_t g_seed = 1;
static uint32_t g_uid = 0xffffffffu, g_step = 0xfffffffeu, g_sub = 0, g_n = 0;
static uint64_t g_draws = 0;

double Random() {
  ++g_draws;
  double u = mcb200_uniform(g_seed, g_uid, g_step, g_sub, g_n++);
  if (g_n == 0) ++g_sub; /* sequential streams longer than 2^32 draws roll into the next sub */
  return u;
}

static void set_stream(uint32_t uid, uint32_t step, uint32_t sub) {
  g_uid = uid;
  g_step = step;
  g_sub = sub;
  g_n = 0;
}

static MeshQuantities *g_mq = nullptr;

/* Fortran / LAPACK entry points declared by include/utils.h:104-110 and only
 * reached from helpers the carrier path never calls (fermi_integral with
 * aprox=false, the subband eigen-solver). */
extern "C" void fermid_(double *, double *, double *, double *, int *) {
  std::cerr << "oracle: fermid_ is not available" << std::endl;
  std::abort();
}
extern "C" double dspevx_(char *, char *, char *, int *, double *, double *, double *, int *, int *, double *,
                          int *, double *, double *, int *, double *, int *, int *, int *) {
  std::cerr << "oracle: dspevx_ is not available" << std::endl;
  std::abort();
  return 0;
}
static uint32_t g_next_uid = 0;

extern "C" {

/* Run the reference's initialize() sequence (src/mcmodel.cpp:45-146) with the
 * band tables read from `table_dir` instead of <exe>/../input.  Particle
 * initialisation draws from the sequential stream (seed, 0xffffffff,
 * 0xfffffffe, 0).  Every particle gets a uid (stored in par_id) in list
 * order.  The deck is read from its own directory, as the reference
 * expects; the caller's working directory is restored.  Returns 0 on success. */
int orc_init(const char *input_file, const char *table_dir, uint64_t seed, int make_particles) {
  g_seed = seed;
  set_stream(0xffffffffu, 0xfffffffeu, 0);
  std::string path(input_file);
  char saved_cwd[4096];
  if (!getcwd(saved_cwd, sizeof(saved_cwd))) return 1;
  size_t slash = path.rfind('/');
  if (slash != std::string::npos) {
    if (chdir(path.substr(0, slash).c_str()) != 0) return 1;
    path = path.substr(slash + 1);
  }
  std::vector<char> fname(path.begin(), path.end());
  fname.push_back('\0');
  /* The mesh lives in globals that read_grid_file appends to
   * (src/utils.cpp:16-18, src/mcmodel.cpp:4651-4672): start them empty so a
   * second initialisation in the same process sees only its own deck. */
  lx.clear(); ly.clear(); lz.clear();
  dx.clear(); dy.clear(); dz.clear();
  MeshQuantities *mq = new MeshQuantities;
  g_mq = mq;
  mq->init_phpysical_parameter(fname.data());
  mq->getInputData(fname.data());
  mq->bs_path = table_dir;
  mq->read_grid_file();
  mq->init_epetra_map_vector();
  mq->read_device_file();
  mq->init_deep();
  mq->init_by_user_input();
  mq->scaling();
  band.IELEC(mq->bs_path);
  mq->init_cell_data();
  if (mq->Flag_SurfaceScatter) mq->init_surface_roughness();
  mq->init_point_data();
  if (make_particles) {
    mq->init_particle_data();
  } else {
    for (auto &l : mq->par_list) l.clear();
  }
  mq->init_poisson_matrix();
  mq->rcurrent = (double *)calloc(p_numy, sizeof(double));
  mq->lcurrent = (double *)calloc(p_numy, sizeof(double));
  mq->catch_par_num = 0;
  mq->gen_par = 0;
  mq->mr_gen_num = 0;
  mq->flag_heat = false;
  mq->step = 0;
  g_next_uid = 0;
  for (auto &l : mq->par_list)
    for (auto &p : l) p.par_id = (int)g_next_uid++;
  return chdir(saved_cwd) == 0 ? 0 : 1;
}

/* ---- scalar / array accessors --------------------------------------- */
int orc_mesh_dims(int *dims) {
  dims[0] = c_numx; dims[1] = c_numy; dims[2] = c_numz;
  dims[3] = p_numx; dims[4] = p_numy; dims[5] = p_numz;
  return 0;
}
double orc_scalar(const char *name) {
  MeshQuantities *mq = g_mq;
  std::string n(name);
  if (n == "dt") return mq->dt;
  if (n == "time0") return time0;
  if (n == "spr0") return spr0;
  if (n == "eV0") return eV0;
  if (n == "conc0") return conc0;
  if (n == "field0") return field0;
  if (n == "scrt0") return scrt0;
  if (n == "a0pi") return a0pi;
  if (n == "sieg") return sieg;
  if (n == "frickel") return mq->frickel;
  if (n == "eps_si") return eps[SILICON];
  if (n == "eps_ox") return eps[OXIDE];
  if (n == "curr0") return curr0;
  if (n == "pot0") return pot0;
  if (n == "T0") return T0;
  if (n == "Tn") return mq->Tn;
  if (n == "sirho") return sirho;
  if (n == "catch_par_num") return mq->catch_par_num;
  if (n == "gen_par") return mq->gen_par;
  if (n == "phonon_scatter") return mq->sttt.phononScatter;
  if (n == "impurity_scatter") return mq->sttt.impurityScatter;
  if (n == "flag_surface_scatter") return mq->Flag_SurfaceScatter;
  if (n == "flag_surface_roughness") return mq->Flag_SurfaceRoughnessScatter;
  if (n == "flag_surface_phonon") return mq->Flag_SurfacePhononScatter;
  if (n == "flag_surface_impurity") return mq->Flag_SurfaceImpurityScatter;
  if (n == "num_contact") return (double)mq->contact.size();
  if (n == "num_surface") return mq->NumSurface;
  if (n == "total_step") return mq->total_step;
  if (n == "electron_number") return mq->electron_number;
  if (n == "hole_number") return mq->hole_number;
  if (n == "stat_step") return mq->stat_step;
  if (n == "mr_step") return mq->mr_step;
  if (n == "heat_steps") return mq->heat_steps;
  if (n == "default_electron_num") return mq->default_electron_num;
  if (n == "default_hole_num") return mq->default_hole_num;
  if (n == "sum_charge_e") return mq->sum_charge[PELEC];
  if (n == "sum_charge_h") return mq->sum_charge[PHOLE];
  if (n == "par_num") return mq->par_num;
  if (n == "flag_mr") return mq->Flag_MultipleRefresh;
  if (n == "flag_compute_heat") return mq->Flag_compute_heat;
  if (n == "draws") return (double)g_draws;
  if (n == "flag_quantum_correction") return mq->Flag_QuantumCorrection;
  if (n == "quantum_start_step") return mq->quantum_start_step;
  return NAN;
}
int orc_set_scalar(const char *name, double v) {
  std::string n(name);
  if (n == "flag_heat") { g_mq->flag_heat = v != 0; return 0; }
  if (n == "flag_surface_scatter") { g_mq->Flag_SurfaceScatter = v != 0; return 0; }
  if (n == "dt") { g_mq->dt = v; return 0; }
  if (n == "flag_quantum_correction") { g_mq->Flag_QuantumCorrection = v != 0; return 0; }
  if (n == "step") { g_mq->step = (int)v; return 0; }
  if (n == "stat_step") { g_mq->stat_step = (int)v; return 0; }
  /* surface-roughness delta and correlation length (normalised lengths),
   * set by the reference's scaling() from constants (src/mcmodel.cpp:4107-4108) */
  if (n == "SurfSc_delta") { g_mq->SurfSc_delta = v; return 0; }
  if (n == "SurfSc_ail") { g_mq->SurfSc_ail = v; return 0; }
  return 1;
}

static Epetra_Vector *cell_vec(const std::string &n) {
  MeshQuantities *mq = g_mq;
  if (n == "c_field_x") return mq->c_field_x;
  if (n == "c_field_y") return mq->c_field_y;
  if (n == "c_field_z") return mq->c_field_z;
  if (n == "c_h_field_x") return mq->c_h_field_x;
  if (n == "c_h_field_y") return mq->c_h_field_y;
  if (n == "c_h_field_z") return mq->c_h_field_z;
  if (n == "c_par_charge") return mq->c_par_charge;
  if (n == "c_da") return mq->c_da;
  if (n == "c_volume") return mq->c_volume;
  if (n == "c_electron_charge") return mq->c_electron_charge;
  if (n == "c_hole_charge") return mq->c_hole_charge;
  if (n == "c_e_roughnessRate") return mq->c_e_roughnessRate;
  if (n == "c_e_surfPhononRate") return mq->c_e_surfPhononRate;
  if (n == "c_h_roughnessRate") return mq->c_h_roughnessRate;
  if (n == "c_h_surfPhononRate") return mq->c_h_surfPhononRate;
  if (n == "c_donor") return mq->c_donor;
  if (n == "c_init_electron_charge") return mq->c_init_electron_charge;
  if (n == "c_init_hole_charge") return mq->c_init_hole_charge;
  if (n == "c_acceptor") return mq->c_acceptor;
  if (n == "p_electron_heat") return mq->p_electron_heat;
  if (n == "p_hole_heat") return mq->p_hole_heat;
  if (n == "p_poisson_pot") return mq->p_poisson_pot;
  if (n == "p_poisson_pot_saved") return mq->p_poisson_pot_saved;
  if (n == "p_rhs") return mq->p_rhs;
  if (n == "p_par_charge") return mq->p_par_charge;
  if (n == "p_dop") return mq->p_dop;
  if (n == "p_volume") return mq->p_volume;
  if (n == "p_vadd") return mq->p_vadd;
  /* statistic() sums (src/mcmodel.cpp:1167-1408) */
  if (n == "stat_vxE") return mq->stat_vxE;
  if (n == "stat_vyE") return mq->stat_vyE;
  if (n == "stat_vzE") return mq->stat_vzE;
  if (n == "stat_vxH") return mq->stat_vxH;
  if (n == "stat_vyH") return mq->stat_vyH;
  if (n == "stat_vzH") return mq->stat_vzH;
  if (n == "stat_chargeE") return mq->stat_chargeE;
  if (n == "stat_chargeH") return mq->stat_chargeH;
  if (n == "stat_energyE") return mq->stat_energyE;
  if (n == "stat_energyH") return mq->stat_energyH;
  if (n == "stat_pot") return mq->stat_pot;
  if (n == "stat_qc_pot") return mq->stat_qc_pot;
  if (n == "stat_ec") return mq->stat_ec;
  if (n == "stat_enum") return mq->stat_enum;
  if (n == "stat_e_heat") return mq->stat_e_heat;
  if (n == "stat_h_heat") return mq->stat_h_heat;
  return nullptr;
}
static Epetra_IntVector *cell_ivec(const std::string &n) {
  MeshQuantities *mq = g_mq;
  if (n == "c_motion_rule") return mq->c_motion_rule;
  if (n == "c_attached_contact") return mq->c_attached_contact;
  if (n == "c_InSurfRegion") return mq->c_InSurfRegion;
  if (n == "c_nearestSurf") return mq->c_nearestSurf;
  if (n == "c_EeffDirection") return mq->c_EeffDirection;
  if (n == "c_material") return mq->c_material;
  if (n == "c_scatter_type") return mq->c_scatter_type;
  if (n == "c_quantumRegion") return mq->c_quantumRegion;
  if (n == "c_desired_electron_number") return mq->c_desired_electron_number;
  if (n == "c_desired_hole_number") return mq->c_desired_hole_number;
  if (n == "c_electron_num") return mq->c_electron_num;
  if (n == "c_hole_num") return mq->c_hole_num;
  if (n == "p_material") return mq->p_material;
  return nullptr;
}
/* Length of a named mesh vector (reference layout), or -1. */
int orc_array_len(const char *name) {
  std::string n(name);
  if (n == "lx") return (int)lx.size();
  if (n == "ly") return (int)ly.size();
  if (n == "lz") return (int)lz.size();
  if (n == "dx") return (int)dx.size();
  if (n == "dy") return (int)dy.size();
  if (n == "dz") return (int)dz.size();
  if (n == "SurfaceDir" || n == "SurfaceType" || n == "SurfacePosition") return MNSurface;
  if (n == "lcurrent" || n == "rcurrent") return p_numy;
  if (Epetra_Vector *v = cell_vec(n)) return v->MyLength();
  if (Epetra_IntVector *v = cell_ivec(n)) return v->MyLength();
  return -1;
}
int orc_get_array(const char *name, double *out) {
  std::string n(name);
  const std::vector<double> *g = nullptr;
  if (n == "lx") g = &lx;
  if (n == "ly") g = &ly;
  if (n == "lz") g = &lz;
  if (n == "dx") g = &dx;
  if (n == "dy") g = &dy;
  if (n == "dz") g = &dz;
  if (g) { std::copy(g->begin(), g->end(), out); return 0; }
  if (n == "SurfaceDir") { for (int i = 0; i < MNSurface; ++i) out[i] = g_mq->SurfaceDir[i]; return 0; }
  if (n == "SurfaceType") { for (int i = 0; i < MNSurface; ++i) out[i] = g_mq->SurfaceType[i]; return 0; }
  if (n == "SurfacePosition") { for (int i = 0; i < MNSurface; ++i) out[i] = g_mq->SurfacePosition[i]; return 0; }
  if (n == "lcurrent") { std::copy(g_mq->lcurrent, g_mq->lcurrent + p_numy, out); return 0; }
  if (n == "rcurrent") { std::copy(g_mq->rcurrent, g_mq->rcurrent + p_numy, out); return 0; }
  if (Epetra_Vector *v = cell_vec(n)) { for (int i = 0; i < v->MyLength(); ++i) out[i] = (*v)[i]; return 0; }
  if (Epetra_IntVector *v = cell_ivec(n)) { for (int i = 0; i < v->MyLength(); ++i) out[i] = (*v)[i]; return 0; }
  return 1;
}
int orc_set_array(const char *name, const double *in) {
  std::string n(name);
  if (Epetra_Vector *v = cell_vec(n)) { for (int i = 0; i < v->MyLength(); ++i) (*v)[i] = in[i]; return 0; }
  if (Epetra_IntVector *v = cell_ivec(n)) { for (int i = 0; i < v->MyLength(); ++i) (*v)[i] = (int)in[i]; return 0; }
  if (n == "lcurrent") { std::copy(in, in + p_numy, g_mq->lcurrent); return 0; }
  if (n == "rcurrent") { std::copy(in, in + p_numy, g_mq->rcurrent); return 0; }
  return 1;
}

/* Contact tallies: per contact {NumParGen, CharGen, EnergyGen, NumParCatch,
 * CharCatch, EnergyCatch}. */
int orc_contacts(double *out) {
  for (size_t i = 0; i < g_mq->contact.size(); ++i) {
    const Contact &c = g_mq->contact[i];
    out[6 * i + 0] = c.NumParGen;
    out[6 * i + 1] = c.CharGen;
    out[6 * i + 2] = c.EnergyGen;
    out[6 * i + 3] = c.NumParCatch;
    out[6 * i + 4] = c.CharCatch;
    out[6 * i + 5] = c.EnergyCatch;
  }
  return (int)g_mq->contact.size();
}
int orc_reset_tallies() {
  MeshQuantities *mq = g_mq;
  for (auto &c : mq->contact) {
    c.NumParGen = 0; c.CharGen = 0; c.EnergyGen = 0;
    c.NumParCatch = 0; c.CharCatch = 0; c.EnergyCatch = 0;
  }
  for (int i = 0; i < p_numy; ++i) mq->lcurrent[i] = mq->rcurrent[i] = 0;
  mq->sttt.phononScatter = 0;
  mq->sttt.impurityScatter = 0;
  mq->catch_par_num = 0;
  mq->gen_par = 0;
  if (mq->p_electron_heat) mq->p_electron_heat->PutScalar(0);
  if (mq->p_hole_heat) mq->p_hole_heat->PutScalar(0);
  return 0;
}

/* ---- particles --------------------------------------------------------- */
/* Layout per particle: d[9] = x,y,z,kx,ky,kz,charge,energy,left_time;
 * i[9] = i,j,k,itet,isym,par_type,flag,seed,uid. */
int orc_num_particles() {
  size_t n = 0;
  for (auto &l : g_mq->par_list) n += l.size();
  return (int)n;
}
int orc_get_particles(double *d, int *iv) {
  size_t n = 0;
  for (auto &l : g_mq->par_list)
    for (auto &p : l) {
      double *dd = d + 9 * n;
      int *ii = iv + 9 * n;
      dd[0] = p.x; dd[1] = p.y; dd[2] = p.z; dd[3] = p.kx; dd[4] = p.ky; dd[5] = p.kz;
      dd[6] = p.charge; dd[7] = p.energy; dd[8] = p.left_time;
      ii[0] = p.i; ii[1] = p.j; ii[2] = p.k; ii[3] = p.itet; ii[4] = p.isym;
      ii[5] = p.par_type; ii[6] = p.flag; ii[7] = p.seed; ii[8] = p.par_id;
      ++n;
    }
  return (int)n;
}
int orc_set_particles(int n, const double *d, const int *iv) {
  for (auto &l : g_mq->par_list) l.clear();
  uint32_t maxuid = 0;
  for (int q = 0; q < n; ++q) {
    const double *dd = d + 9 * q;
    const int *ii = iv + 9 * q;
    Particle p;
    p.x = dd[0]; p.y = dd[1]; p.z = dd[2]; p.kx = dd[3]; p.ky = dd[4]; p.kz = dd[5];
    p.charge = dd[6]; p.energy = dd[7]; p.left_time = dd[8];
    p.i = ii[0]; p.j = ii[1]; p.k = ii[2]; p.itet = ii[3]; p.isym = ii[4];
    p.par_type = ii[5]; p.flag = ii[6]; p.seed = ii[7]; p.par_id = ii[8];
    if ((uint32_t)ii[8] + 1 > maxuid) maxuid = (uint32_t)ii[8] + 1;
    g_mq->par_list[C_LINDEX_GHOST_ONE(p.i, p.j, p.k)].push_back(p);
  }
  g_next_uid = maxuid;
  return 0;
}

/* The field half of density() (src/mcmodel.cpp:424-471): node charge
 * density from the particles (particle_to_density), the Poisson solve and
 * both carriers' fields (compute_field), then the cell charge
 * (compute_cell_charge). */
int orc_density_and_field() {
  MeshQuantities *mq = g_mq;
  mq->p_par_charge->PutScalar(0);
  mq->particle_to_density(mq->p_par_charge, 2);
  mq->compute_field();
  mq->compute_cell_charge();
  return 0;
}

/* The quantum-correction set-up of the reference's initialisation
 * (src/mcmodel.cpp:136-140): init_effective_potential, init_p_mat,
 * init_ep_range, from the deck's ep_parm and quantumRegion.  Once per
 * orc_init. */
int orc_init_quantum() {
  g_mq->init_effective_potential();
  g_mq->init_p_mat();
  g_mq->init_ep_range();
  return 0;
}

/* The phonon dispersion tables init_deep read (src/ParticleUtils.cpp:
 * 750-806), as [rows][cols]: 0 kloem, 1 kloab, 2 ktoem, 3 ktoab, 4 klaem,
 * 5 klaab. */
int orc_dispersion(int which, double *out) {
  static const int rows[6] = {201, 201, 51, 51, 51, 51}, cols[6] = {120, 110, 160, 150, 160, 150};
  MeshQuantities *mq = g_mq;
  if (which < 0 || which > 5) return 1;
  for (int r = 0; r < rows[which]; ++r)
    for (int c = 0; c < cols[which]; ++c) {
      double v = 0;
      switch (which) {
        case 0: v = mq->kloem[r][c]; break;
        case 1: v = mq->kloab[r][c]; break;
        case 2: v = mq->ktoem[r][c]; break;
        case 3: v = mq->ktoab[r][c]; break;
        case 4: v = mq->klaem[r][c]; break;
        default: v = mq->klaab[r][c]; break;
      }
      out[r * cols[which] + c] = v;
    }
  return 0;
}

/* quantumPotential (src/mcmodel.cpp:2378-2403): p_poisson_pot replaced by
 * the effective potential at every quantum node. */
int orc_quantum_potential() {
  g_mq->quantumPotential();
  return 0;
}

/* Contacts as parsed from the deck (after scaling): per contact
 * {nplanes, Vapp, PhiMS}, planes as {contact, i0, i1, j0, j1, k0, k1}. */
int orc_contact_info(double *per_contact, int *planes, int max_planes) {
  int np = 0;
  for (size_t c = 0; c < g_mq->contact.size(); ++c) {
    const Contact &ct = g_mq->contact[c];
    per_contact[3 * c + 0] = ct.NumContactPlane;
    per_contact[3 * c + 1] = ct.CurrentVapp;
    per_contact[3 * c + 2] = ct.PhiMS;
    for (int p = 0; p < ct.NumContactPlane && np < max_planes; ++p, ++np) {
      int *r = planes + 7 * np;
      r[0] = (int)c;
      r[1] = ct.BeginI[p]; r[2] = ct.EndI[p];
      r[3] = ct.BeginJ[p]; r[4] = ct.EndJ[p];
      r[5] = ct.BeginK[p]; r[6] = ct.EndK[p];
    }
  }
  return np;
}

/* The reference's Poisson matrix (init_matrix, src/mcmodel.cpp:4695-4869) as
 * dense 7-slot rows in the engine's stencil order (-x, +x, -y, +y, -z, +z,
 * diagonal), node index (j*(nx+1)+i)*(nz+1)+k. */
int orc_poisson_stencil(double *out) {
  /* the solver keeps its copy protected; init_matrix builds the same one again */
  std::unique_ptr<Epetra_CrsMatrix> own(g_mq->init_matrix());
  const Epetra_CrsMatrix *A = own.get();
  const Epetra_Map &m = A->RowMap();
  for (int r = 0; r < A->NumMyRows(); ++r) {
    const int g = m.GID(r);
    const int j = g / p_numxz, rem = g % p_numxz, i = rem / p_numz, k = rem % p_numz;
    double *row = out + 7 * (size_t)g;
    for (int s = 0; s < 7; ++s) row[s] = 0;
    for (const auto &e : A->Row(r)) {
      const int q = e.first;
      const int qj = q / p_numxz, qrem = q % p_numxz, qi = qrem / p_numz, qk = qrem % p_numz;
      int slot = 6;
      if (qi == i - 1) slot = 0;
      else if (qi == i + 1) slot = 1;
      else if (qj == j - 1) slot = 2;
      else if (qj == j + 1) slot = 3;
      else if (qk == k - 1) slot = 4;
      else if (qk == k + 1) slot = 5;
      row[slot] = e.second;
    }
  }
  return A->NumMyRows();
}

/* MultipleRefresh (src/MultipleRefresh.cpp:60-143) cell by cell, with the
 * reference's own gen_new_par_mr (:9-58) doing the resampling.  The loop is
 * restated here only to fix the three things the engine defines: a cell's
 * particles are taken in uid order, each (cell, carrier) draws from
 * stream (seed, cell, step, 0x4d520000 + carrier), and resampled particles
 * take new uids in (cell, carrier, draw) order. */
int orc_multiple_refresh(uint32_t step) {
  MeshQuantities *mq = g_mq;
  int *e_num, *h_num;
  mq->c_desired_electron_number->ExtractView(&e_num);
  mq->c_desired_hole_number->ExtractView(&h_num);
  for (size_t c = 0; c < mq->par_list.size(); ++c) {
    std::list<Particle> &lst = mq->par_list[c];
    std::vector<Particle> all(lst.begin(), lst.end());
    std::stable_sort(all.begin(), all.end(),
                     [](const Particle &a, const Particle &b) { return (uint32_t)a.par_id < (uint32_t)b.par_id; });
    std::vector<Particle> vec[2], fresh[2];
    for (const Particle &p : all)
      if (fabs(p.charge) >= mq->pckill) vec[p.par_type == PELEC ? 0 : 1].push_back(p);
    const size_t before = lst.size();
    lst.clear();
    for (int t = 0; t < 2; ++t) {
      set_stream((uint32_t)c, step, 0x4d520000u + (uint32_t)t);
      const bool redone = mq->gen_new_par_mr(vec[t], t == 0 ? e_num[c] : h_num[c], fresh[t]);
      /* A resampled particle is a copy of an old one, par_id included; the
       * reference's single random sequence sets the copies apart at once,
       * but here draws are keyed by par_id, so each copy gets a uid of its
       * own as the engine numbers them (cells in order, electrons then
       * holes, draw order) -- else the copies would fly as one. */
      if (redone)
        for (Particle &p : fresh[t]) p.par_id = (int)g_next_uid++;
      for (const Particle &p : redone ? fresh[t] : vec[t]) lst.push_back(p);
    }
    mq->mr_gen_num += (int)lst.size() - (int)before;
  }
  return mq->mr_gen_num;
}

/* statistic() (src/mcmodel.cpp:1167-1408): one step's sums added to the
 * stat_* vectors; set_stat_zero() (:715-750) clears them with the tallies. */
int orc_statistic() {
  g_mq->statistic();
  return 0;
}
int orc_set_stat_zero() {
  g_mq->set_stat_zero();
  return 0;
}

/* The reference's window outputs for step `step`: output_stat (with
 * current_scatter_info, src/mcmodel.cpp:971-1161, :756-842) and
 * output_for_restart (:895-965), written under <dir>/data/ as the reference
 * writes them under ./data/ (the working directory is restored). */
int orc_write_outputs(const char *dir, int step) {
  char saved_cwd[4096];
  if (!getcwd(saved_cwd, sizeof(saved_cwd))) return 1;
  if (chdir(dir) != 0) return 1;
  mkdir("data", 0755);
  g_mq->step = step;
  g_mq->output_stat();
  g_mq->output_for_restart();
  return chdir(saved_cwd) == 0 ? 0 : 1;
}

/* One particle of the initial ensemble as init_particle_data makes it
 * (src/particle_init.cpp:185-215: three uniform draws place it in cell
 * (i, j, k), then select_kstate, src/mcmodel.cpp:3006-3057, draws its
 * energy, band, wedge and k), drawing from stream (seed, uid, 0xfffffffd, 0)
 * -- the per-particle stream of the engine's GPU seeding.  The position
 * lines are the reference's, restated because init_particle_data loops over
 * every cell of the deck with one sequential stream.  Out: d as
 * orc_get_particles' doubles, iv as its ints. */
int orc_seed_particle(uint64_t seed, uint32_t uid, int i, int j, int k, int type, double charge, double *d, int *iv) {
  MeshQuantities *mq = g_mq;
  const uint64_t saved = g_seed;
  g_seed = seed;
  set_stream(uid, 0xfffffffdu, 0);
  Particle p;
  double lamda = Random();
  p.x = lamda * lx[i] + (1 - lamda) * lx[i + 1];
  lamda = Random();
  p.y = lamda * ly[j] + (1 - lamda) * ly[j + 1];
  lamda = Random();
  p.z = lamda * lz[k] + (1 - lamda) * lz[k + 1];
  p.charge = charge;
  p.i = i;
  p.j = j;
  p.k = k;
  p.par_type = type;
  p.seed = mq->seed;
  p.left_time = mq->dt;
  p.par_id = (int)uid;
  p.flag = 1;
  mq->select_kstate(&p, 0);
  g_seed = saved;
  const double dd[9] = {p.x, p.y, p.z, p.kx, p.ky, p.kz, p.charge, p.energy, p.left_time};
  const int ii[9] = {p.i, p.j, p.k, p.itet, p.isym, p.par_type, p.flag, p.seed, p.par_id};
  for (int q = 0; q < 9; ++q) {
    d[q] = dd[q];
    iv[q] = ii[q];
  }
  return 0;
}

/* Reference charge bookkeeping used by the flight (Rho = screening density):
 * src/mcmodel.cpp:2664-2712. */
int orc_compute_cell_charge() {
  g_mq->compute_cell_charge();
  return 0;
}
int orc_surface_rates() {
  g_mq->GetSurfRoughnessPhononScRate();
  return 0;
}

/* One flight pass over every particle with the reference's particle_fly()
 * (src/mcmodel.cpp:1874-2161), each particle on its own Philox stream,
 * then the mid-step copies (see the file comment), then the reference's
 * removal of caught particles (local_migrate, src/mcmodel.cpp:1615-1638,
 * minus the MPI part).  Particles left unfinished (flag 0: a PASS across
 * the outer y boundary, src/CellHit.cpp:104-107) are counted in *unfinished
 * and kept.  Returns the number of particles after the step. */
int orc_flight_step(uint32_t step, int *unfinished) {
  MeshQuantities *mq = g_mq;
  typedef std::list<Particle>::iterator PIt;
  struct Job { PIt it; std::list<Particle> *lst; uint32_t uid, sub; };
  std::vector<Job> jobs;
  std::vector<size_t> sizes(mq->par_list.size());
  for (size_t c = 0; c < mq->par_list.size(); ++c) {
    sizes[c] = mq->par_list[c].size();
    for (PIt it = mq->par_list[c].begin(); it != mq->par_list[c].end(); ++it)
      jobs.push_back({it, &mq->par_list[c], (uint32_t)it->par_id, 0u});
  }
  std::sort(jobs.begin(), jobs.end(), [](const Job &a, const Job &b) { return a.uid < b.uid; });
  struct Child { uint32_t parent, sub; Particle *p; };
  std::vector<Child> children;
  int n_unfinished = 0;
  std::vector<Job> queue = jobs;
  while (!queue.empty()) {
    std::vector<Job> next;
    for (const Job &jb : queue) {
      mq->current_par_list = jb.lst;
      mq->par_iter = jb.it;
      set_stream(jb.uid, step, jb.sub);
      int gen_before = mq->gen_par;
      mq->particle_fly();
      if (jb.it->i >= 0 && jb.it->flag == 0) ++n_unfinished;
      if (mq->gen_par != gen_before) {
        /* The appended copies sit at the tails of the lists that grew.  A
         * copy keeps the flight time left when it was made, so sorting by
         * left_time (descending) recovers the order they were made in. */
        std::vector<Job> made;
        for (size_t c = 0; c < mq->par_list.size(); ++c) {
          while (mq->par_list[c].size() > sizes[c]) {
            PIt tail = mq->par_list[c].begin();
            std::advance(tail, sizes[c]);
            made.push_back({tail, &mq->par_list[c], jb.uid, 0u});
            ++sizes[c];
          }
        }
        std::stable_sort(made.begin(), made.end(),
                         [](const Job &a, const Job &b) { return a.it->left_time > b.it->left_time; });
        for (size_t k = 0; k < made.size(); ++k) {
          made[k].sub = jb.sub * 16u + 1u + (uint32_t)k;
          made[k].it->flag = 1;
          made[k].it->par_id = -1;
          next.push_back(made[k]);
          children.push_back({jb.uid, made[k].sub, &*made[k].it});
        }
      }
    }
    queue.swap(next);
  }
  std::sort(children.begin(), children.end(), [](const Child &a, const Child &b) {
    return std::tie(a.parent, a.sub) < std::tie(b.parent, b.sub);
  });
  /* uids go to the copies that survive their flight (a copy caught in the
   * rest of its step is removed below without one), as the engine numbers
   * them */
  for (const Child &ch : children)
    if (ch.p->i >= 0) ch.p->par_id = (int)g_next_uid++;
  for (auto &l : mq->par_list)
    for (auto it = l.begin(); it != l.end();) {
      if (it->i < 0) it = l.erase(it);
      else { it->left_time = mq->dt; ++it; }
    }
  /* particles that changed cell move to their new list */
  for (size_t c = 0; c < mq->par_list.size(); ++c) {
    auto &l = mq->par_list[c];
    for (auto it = l.begin(); it != l.end();) {
      size_t want = C_LINDEX_GHOST_ONE(it->i, it->j, it->k);
      if (want != c) {
        mq->par_list[want].push_back(*it);
        it = l.erase(it);
      } else ++it;
    }
  }
  if (unfinished) *unfinished = n_unfinished;
  return orc_num_particles();
}

/* The reference's own sweep for timing: update_particle()
 * (src/mcmodel.cpp:1460-1505) with deposition bookkeeping
 * (compute_cell_charge) as density() does, over nsteps steps, on one
 * sequential Philox stream.  Returns wall seconds spent. */
double orc_time_update_particle(int nsteps, int with_cell_charge) {
  MeshQuantities *mq = g_mq;
  set_stream(0xfffffff0u, 0, 0);
  std::streambuf *old = std::cout.rdbuf(nullptr);
  auto t0 = std::chrono::steady_clock::now();
  for (int s = 0; s < nsteps; ++s) {
    if (with_cell_charge) mq->compute_cell_charge();
    mq->update_particle();
  }
  auto t1 = std::chrono::steady_clock::now();
  std::cout.rdbuf(old);
  return std::chrono::duration<double>(t1 - t0).count();
}

/* Silence the reference's per-step console chatter. */
int orc_quiet(int q) {
  static std::streambuf *saved = nullptr;
  if (q && !saved) saved = std::cout.rdbuf(nullptr);
  if (!q && saved) { std::cout.rdbuf(saved); saved = nullptr; }
  return 0;
}

/* ---- band tables, for the table-builder parity tests ------------------ */
void *orc_band_ptr(const char *name) {
  std::string n(name);
#define B(x) if (n == #x) return (void *)&band.x;
  B(tet) B(NeibrTet) B(ibt) B(xkk) B(ykk) B(zkk) B(eek) B(vt) B(vgt) B(datantlin)
  B(faclow) B(facmedium) B(fachigh) B(maxaovtet) B(gamtet) B(matsym) B(indmat) B(newisym)
  B(xbz) B(ybz) B(zbz) B(ntlist) B(ptlist) B(tlist) B(nslist) B(pslist) B(slist)
  B(ntlists) B(ptlists) B(tlists) B(nclist) B(pclist) B(clist) B(dos) B(sumdos)
  B(dostetmax) B(sumscatt) B(scatte) B(scattiie) B(scatth) B(scattiih) B(dose) B(dosh)
  B(energy) B(DOSMAX) B(gamma) B(nband) B(bandof) B(partyp) B(difpr) B(xkct) B(ykct) B(zkct)
#undef B
  return nullptr;
}
double orc_band_scalar(const char *name) {
  std::string n(name);
  if (n == "nk") return band.nk;
  if (n == "nt") return band.nt;
  if (n == "nbt") return band.nbt;
  if (n == "scpre") return band.scpre;
  if (n == "scprh") return band.scprh;
  if (n == "dtable") return band.dtable;
  if (n == "emax") return band.emax;
  if (n == "dlist") return band.dlist;
  if (n == "dlists") return band.dlists;
  if (n == "temptag") return band.temptag;
  if (n == "templag") return band.templag;
  if (n == "templog") return band.templog;
  if (n == "temptaf") return band.temptaf;
  if (n == "templaf") return band.templaf;
  if (n == "temptof") return band.temptof;
  if (n == "temphop") return band.temphop;
  if (n == "meld") return band.meld;
  if (n == "mell") return band.mell;
  if (n == "melt") return band.melt;
  if (n == "Ni") return band.Ni;
  return NAN;
}

/* Table construction alone (Band::IELEC, src/Band.cpp:4271-4476) for a
 * given temperature, without a deck: sets the normalisation the way
 * init_phpysical_parameter does (src/mcmodel.cpp:4007-4122). */
int orc_build_band_only(const char *table_dir, double temperature) {
  static MeshQuantities *mq = nullptr;
  if (!mq) mq = new MeshQuantities;
  char tmpname[] = "/tmp/orc_temperature_XXXXXX";
  int fd = mkstemp(tmpname);
  if (fd < 0) return 1;
  std::string body = "Temperature=" + std::to_string(temperature) + "\n";
  if (write(fd, body.data(), body.size()) != (ssize_t)body.size()) return 1;
  close(fd);
  mq->init_phpysical_parameter(tmpname);
  unlink(tmpname);
  band.IELEC(table_dir);
  if (!g_mq) g_mq = mq;
  return 0;
}

/* Direct calls of single reference routines on a particle state, for
 * function-level parity.  The state is loaded into the member "registers"
 * (the way InPar does, src/mcmodel.cpp:2169-2190). */
static void load_regs(const double *d, const int *iv) {
  MeshQuantities *mq = g_mq;
  mq->x = d[0]; mq->y = d[1]; mq->z = d[2]; mq->kx = d[3]; mq->ky = d[4]; mq->kz = d[5];
  mq->charge = d[6]; mq->energy = d[7]; mq->left_time = d[8];
  mq->icell = iv[0]; mq->jcell = iv[1]; mq->kcell = iv[2]; mq->itet = iv[3]; mq->isym = iv[4];
  mq->par_type = iv[5];
  mq->iband = band.ibt[mq->itet];
}
static void store_regs(double *d, int *iv) {
  MeshQuantities *mq = g_mq;
  d[0] = mq->x; d[1] = mq->y; d[2] = mq->z; d[3] = mq->kx; d[4] = mq->ky; d[5] = mq->kz;
  d[6] = mq->charge; d[7] = mq->energy; d[8] = mq->left_time;
  iv[0] = mq->icell; iv[1] = mq->jcell; iv[2] = mq->kcell; iv[3] = mq->itet; iv[4] = mq->isym;
  iv[5] = mq->par_type; iv[6] = mq->Flag_SelfScatter; iv[7] = mq->Flag_Catch; iv[8] = mq->iband;
}
/* which: 0 TetTime, 1 HitTet(after TetTime), 2 get_state at current energy
 * and iband, 3 Getisym, 4 GetEnergy, 5 ElectronPhononScatter,
 * 6 HolePhononScatter, 7 TALIND(1), 8 TALIND(2), 9 TALIND(3).
 * out[0] returns the routine's double result (TetTime) or 0. */
int orc_call(int which, double *d, int *iv, double ex, double ey, double ez, uint32_t uid, uint32_t step,
             uint32_t sub, double *out) {
  MeshQuantities *mq = g_mq;
  load_regs(d, iv);
  mq->Ex = ex; mq->Ey = ey; mq->Ez = ez;
  mq->Flag_Catch = false;
  mq->Flag_SelfScatter = false;
  set_stream(uid, step, sub);
  out[0] = 0;
  switch (which) {
    case 0: out[0] = mq->TetTime(); out[1] = mq->itetdir; break;
    case 1: mq->TetTime(); mq->HitTet(); break;
    case 2: mq->get_state(); break;
    case 3: mq->Getisym(); break;
    case 4: mq->GetEnergy(); break;
    case 5: mq->ElectronPhononScatter(); break;
    case 6: mq->HolePhononScatter(); break;
    case 7: mq->TALIND(1); break;
    case 8: mq->TALIND(2); break;
    case 9: mq->TALIND(3); break;
    default: return 1;
  }
  store_regs(d, iv);
  out[2] = (double)g_n;
  return 0;
}

}  // extern "C"
