/*
 * mcb200.h -- C ABI of the B200 ensemble Monte Carlo carrier engine.
 *
 * The engine replaces the per-step carrier update of the reference
 * simulator (chenglinye18-crypto/C-MC_electron), whose seam is the member
 * MeshQuantities::update_particle() (src/mcmodel.cpp:1460) and the routines
 * it reaches: particle_fly (src/mcmodel.cpp:1874-2161), TetHit / CellHit
 * (src/TetHit.cpp, src/CellHit.cpp), the phonon / impurity / surface
 * scattering files, and the bookkeeping local_migrate (:1615-1638).  The
 * reference has no plugin or FFI layer of its own; these entry points are
 * what its host code (or any C / C++ / ctypes caller) binds instead.
 *
 * Conventions.
 *  - Plain pointers and sizes; every host buffer is owned by the caller,
 *    every device buffer by the context.  Nothing here retains a caller
 *    pointer after the call returns.
 *  - Units are the reference's normalised ones (energy kB*T, length spr0,
 *    time hbar/(kB*T)); mcb200_units() returns the scales.
 *  - Mesh cell (i, j, k) has linear index (j * nx + i) * nz + k, the
 *    reference's single-rank layout (C_LINDEX_GHOST_ONE, include/defs.h);
 *    mesh node (i, j, k) has index (j * (nx+1) + i) * (nz+1) + k.
 *  - Every call returns MCB200_OK (0) or an error code; the reference's
 *    exit() paths become error codes or counters, never a process exit.
 *    mcb200_last_error() describes the last failure of a context.
 *  - One context per host thread; each context runs on its own CUDA stream.
 */
#ifndef MCB200_H
#define MCB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCB200_OK 0
#define MCB200_ERR_ARG 1       /* a bad argument or size */
#define MCB200_ERR_CUDA 2      /* a CUDA call failed (no GPU, out of memory, ...) */
#define MCB200_ERR_IO 3        /* a table or deck file could not be read */
#define MCB200_ERR_CAPACITY 4  /* more particles than the context was sized for */
#define MCB200_ERR_STATE 5     /* call made before the data it needs was set */

typedef struct mcb200_ctx mcb200_ctx;

/* Particles as structure-of-arrays host buffers (the reference's Particle,
 * include/utils.h:130-141, minus the per-step bookkeeping fields).
 * i, j, k: cell; itet: tetrahedron; isym: BZ wedge (0..47); type: 0 electron,
 * 1 hole; uid: unique id, the key of the particle's random stream. */
typedef struct {
  double *x, *y, *z;
  double *kx, *ky, *kz;
  double *charge, *energy;
  int32_t *i, *j, *k;
  int32_t *itet, *isym, *type;
  uint32_t *uid;
} mcb200_particles;

/* Counters returned by mcb200_get_tallies (index into counters[]). */
#define MCB200_CNT_PHONON 0        /* real phonon events  (sttt.phononScatter) */
#define MCB200_CNT_IMPURITY 1      /* real impurity events (sttt.impurityScatter) */
#define MCB200_CNT_CAUGHT 2        /* particles removed    (catch_par_num) */
#define MCB200_CNT_GENERATED 3     /* GENERATE copies      (gen_par) */
#define MCB200_CNT_EVENTS 4        /* free-flight loop iterations */
#define MCB200_CNT_UNFINISHED 5    /* PASS across the outer y boundary */
#define MCB200_CNT_TOO_MANY 6      /* particles over the per-step event cap */
#define MCB200_CNT_CHILD_OVERFLOW 7
#define MCB200_CNT_NO_TET 8        /* tetrahedron search failed (particle caught) */
#define MCB200_CNT_ZERO_TIME 9     /* FP32 flight: stuck on zero-length events (particle caught) */
#define MCB200_NUM_COUNTERS 16

/* Build the full-band tables from `table_dir` (the reference's input/
 * directory: bs.si.asc, zd.si.asc; Band::IELEC, src/Band.cpp:4271-4476) at
 * lattice temperature `kelvin`, and upload them to CUDA device `device`.
 * `max_particles` sizes the particle store.  device = -1 builds the tables
 * on the host only (for inspection with mcb200_copy_table; every device
 * call then returns MCB200_ERR_STATE).  On failure *out may still hold a
 * context whose mcb200_last_error() says why; destroy it either way. */
int mcb200_create(const char *table_dir, double kelvin, int device, size_t max_particles, mcb200_ctx **out);
/* A new context on the same device with the same band tables as `like`
 * (shared, not rebuilt or copied; they live until the last context using
 * them is destroyed), its own stream, store of `max_particles`, mesh and
 * tallies.  Contexts made alike can fly together in one batch.  No
 * counterpart in the reference (one simulation per process). */
int mcb200_create_alike(const mcb200_ctx *like, size_t max_particles, mcb200_ctx **out);
void mcb200_destroy(mcb200_ctx *ctx);
const char *mcb200_last_error(const mcb200_ctx *ctx);

/* Flight precision of the context's particle store.
 *  MCB200_FLIGHT_FP64: the reference's arithmetic (IEEE double, reference
 *    operand order; 80 bytes per particle).  The default.
 *  MCB200_FLIGHT_FP32: flight kinematics and rate lookups in float --
 *    positions relative to the cell's low corner, k, velocities, fields,
 *    event times, band and rate tables -- with energy, charge and the
 *    remaining step time in double and the tallies in int64 fixed point
 *    (56 bytes per particle).  Draws come from the float stream of
 *    include/mcb200_rng.h, so results agree with FP64 statistically.
 * No counterpart in the reference (it flies in double only).  Only allowed
 * while the store is empty (before upload / seed); the particle buffers are
 * reallocated.  Host-side particle arrays stay FP64 in both precisions. */
#define MCB200_FLIGHT_FP64 0
#define MCB200_FLIGHT_FP32 1
int mcb200_set_flight_precision(mcb200_ctx *ctx, int precision);
int mcb200_get_flight_precision(const mcb200_ctx *ctx);

/* Sort-bucket width of the step's counting sort (the reference's
 * local_migrate, src/mcmodel.cpp:1615-1638, moves particles between its
 * per-cell lists): the store is
 * grouped by buckets of `cells_per_bucket` consecutive cells of the linear
 * order (z fastest), a power of two from 1 (by cell, the default) to 64.
 * Wider buckets shorten the histogram and its scan and leave a bucket's
 * particles in arrival order.  Results do not depend on it (tallies are
 * fixed point, draws per particle); only the speed of the sort and of the
 * passes over the sorted store does.  ERR_ARG for other widths.  The
 * refresh's own sort stays per cell. */
int mcb200_set_sort_bucket(mcb200_ctx *ctx, int cells_per_bucket);
int mcb200_get_sort_bucket(const mcb200_ctx *ctx);

/* Normalisation scales (MeshQuantities::init_phpysical_parameter,
 * src/mcmodel.cpp:4007-4122): out[0..n) = T0, eV0, spr0, time0, conc0,
 * field0, scrt0, pot0, a0pi, sieg, eps_silicon, eps_oxide, curr0, dens0. */
int mcb200_units(const mcb200_ctx *ctx, double *out, int n);

/* Copy a host-built table (for inspection and parity checks) into `out`
 * (capacity `bytes`); `*needed` receives its size in bytes.  Names follow
 * the reference's Band members: "gamtet", "vt", "vgt", "datantlin",
 * "faclow", "facmedium", "fachigh", "tet", "NeibrTet", "ibt", "xkk", "ykk",
 * "zkk", "eek", "matsym", "indmat", "newisym", "xbz", "ybz", "zbz",
 * "ntlist", "ptlist", "tlist", "nslist", "pslist", "slist", "ntlists",
 * "ptlists", "tlists", "dos", "sumdos", "dostetmax", "sumscatt", "scatte",
 * "dose", "scattiie", "scatth", "dosh", "scattiih", "energy". */
int mcb200_copy_table(const mcb200_ctx *ctx, const char *name, void *out, size_t bytes, size_t *needed);

/* Cells per axis of the mesh set by mcb200_set_mesh (MCB200_ERR_STATE
 * before it). */
int mcb200_get_mesh_dims(const mcb200_ctx *ctx, int *nx, int *ny, int *nz);

/* Mesh node coordinates in normalised length (lx: nx+1 values, ...) and,
 * optionally, the cell widths dx/dy/dz (nx, ny, nz values; NULL: taken as
 * node differences).  The reference scales its widths separately from its
 * node coordinates, so passing its own dx/dy/dz keeps the deposition and
 * Poisson weights bit-identical.  Replaces the lx/ly/lz/dx/dy/dz globals
 * (include/utils.h:81-83).  Resets cells, fields and the device description. */
int mcb200_set_mesh(mcb200_ctx *ctx, int nx, int ny, int nz, const double *lx, const double *ly,
                    const double *lz, const double *dx, const double *dy, const double *dz);

/* Device description for deposition and the Poisson solve: per cell the
 * material (0 void, 1 vacuum, 2 oxide, 3 silicon) and donor / acceptor
 * concentrations (normalised by conc0); contacts: per contact the applied
 * potential Vapp and the work-function difference PhiMS (normalised by
 * pot0), and n_planes planes of 7 ints {contact (0-based), i0, i1, j0, j1,
 * k0, k1} (inclusive node ranges) whose nodes are Dirichlet rows.  Builds
 * node volumes, doping and built-in potential (init_cell_data /
 * init_point_data, src/mcmodel.cpp:3187-3390) and the FV stencil
 * (init_matrix, :4695-4869). */
int mcb200_set_device(mcb200_ctx *ctx, const int32_t *material, const double *donor, const double *acceptor,
                      int n_contacts, const double *vapp, const double *phims, int n_planes, const int32_t *planes);

/* Charge deposition from the particle store: per-cell carrier charge and
 * the screening density Rho the flight uses (compute_cell_charge,
 * src/mcmodel.cpp:2664-2712) and the node charge density of the Poisson
 * right-hand side (particle_to_density, :348-417); int64 fixed point. */
int mcb200_deposit(mcb200_ctx *ctx);

/* Poisson solve from the last deposit (compute_rhs + linear_poisson_solver,
 * src/mcmodel.cpp:2714-2893; the reference factorises with KLU): CG in FP64
 * on the system with the contact rows eliminated, warm-started from the
 * previous potential, to ||b - Ax|| / ||b|| <= rel_tol; then the cell fields
 * of both carriers (pot2field, :2732-2855).  The preconditioner is one
 * geometric-multigrid V-cycle (the default) or Jacobi, selected with
 * mcb200_set_poisson_solver. */
int mcb200_solve_poisson(mcb200_ctx *ctx, double rel_tol, int max_iter, int *iterations, double *rel_residual);
/* With iterations and rel_residual both NULL, mcb200_solve_poisson does not
 * wait for the GPU; every solve adds to statistics kept on the device:
 * solves, CG iterations and the largest relative residual, read (and
 * optionally reset) here. */
int mcb200_poisson_stats(mcb200_ctx *ctx, int64_t *solves, int64_t *iterations, double *max_rel_residual, int reset);

/* No counterpart in the reference (which counts particles crossing the
 * contact planes, current_scatter_info).  The current contact `contact`
 * (0-based, deck order) carries by induction, Ramo-Shockley: the weighting
 * potential of the contact (Laplace's equation on the device's Poisson
 * stencil, 1 on its nodes and 0 on every other contact) is solved once
 * here and its cell field E_w kept ("induced_field" of mcb200_get_array);
 * from then on every transport step (mcb200_step, batched steps) starts by
 * adding the sum over particles of q v . E_w (v the group velocity) to a
 * tally.  mcb200_get_induced_current returns that tally since the last
 * mcb200_reset_tallies and the number of steps it covers: sum / steps *
 * curr0 * 1e-2 (mcb200_units) is in the unit and sign of the reference's
 * `Current = `, and its time average is the contact's terminal current,
 * with far less noise per step than the catch / generate balance.  The
 * particle terms are summed in fixed point, so the tally does not depend
 * on the store's order.  contact < 0 switches it off; MCB200_ERR_STATE
 * before mcb200_set_device. */
int mcb200_set_induced_current(mcb200_ctx *ctx, int contact);
int mcb200_get_induced_current(mcb200_ctx *ctx, double *sum, double *steps);

#define MCB200_POISSON_AUTO 0      /* multigrid when the mesh has a hierarchy, else Jacobi */
#define MCB200_POISSON_JACOBI 1    /* Jacobi-preconditioned CG */
#define MCB200_POISSON_MULTIGRID 2 /* V-cycle-preconditioned CG */
/* Preconditioner and cooperative grid (blocks; 0 = automatic: Jacobi the
 * largest co-resident grid, multigrid one 512-thread block per SM) of the following
 * solves.  No counterpart in the reference. */
int mcb200_set_poisson_solver(mcb200_ctx *ctx, int method, int blocks);
/* Preconditioner (MCB200_POISSON_JACOBI / _MULTIGRID) and grid of the last
 * solve, and the multigrid level count of the device (0: none). */
int mcb200_get_poisson_solver(mcb200_ctx *ctx, int *method_used, int *blocks, int *levels);

/* Surface scattering parameters (the SurfSc_* members set in
 * init_phpysical_parameter, src/mcmodel.cpp:4107-4121): delta and ail are the
 * roughness rms height and correlation length in normalised length; the
 * reference hard-codes 0.1126755 nm and 2 nm. */
typedef struct {
  double delta, ail, xiph, theta, gama, nbmod, npf, pft, pfn, kpha;
  int roughness; /* Flag_SurfaceRoughnessScatter */
  int phonon;    /* Flag_SurfacePhononScatter */
} mcb200_surface_params;

/* Per-cell surface roughness and surface phonon rates of both carriers from
 * the current fields and screening density (GetSurfRoughnessPhononScRate,
 * src/GetSurfRoughnessPhononScRate.cpp:4-70); eeff_direction per cell is the
 * axis (0 x, 1 y, 2 z) of the nearest Si/SiO2 surface (c_EeffDirection,
 * init_surface_roughness, src/mcmodel.cpp:3155-3185). */
int mcb200_surface_rates(mcb200_ctx *ctx, const mcb200_surface_params *params, const int32_t *eeff_direction);

/* MultipleRefresh (src/MultipleRefresh.cpp:9-143): per cell and carrier,
 * particles with |q| < 1e-30 are dropped and, unless the count is within a
 * factor Rpar = 2 of desired and the charge spread within Rsqr = 2, the
 * population is resampled to desired_e / desired_h particles with
 * probability |q| / sum|q|, each carrying sum(q) / desired.  Within a cell
 * particles are taken in uid order; each (cell, carrier) draws from stream
 * (seed, cell, step, 0x4d520000 + carrier); resampled particles get fresh
 * uids.  *generated receives the change in particle count (mr_gen_num);
 * with generated NULL the refresh is only enqueued (its counts stay on the
 * device, nothing waits for the GPU). */
int mcb200_multiple_refresh(mcb200_ctx *ctx, const int32_t *desired_e, const int32_t *desired_h, uint32_t step,
                            uint64_t seed, int64_t *generated);
/* The refresh targets (c_desired_electron_number / c_desired_hole_number,
 * one per cell) uploaded ahead of the first mcb200_multiple_refresh, which
 * otherwise copies them (as it does whenever they change) from the caller's
 * pageable memory: about a millisecond of host time per refresh-sized mesh,
 * taken inside a running simulation.  Waits for the copy; no reference
 * counterpart (the reference keeps the targets in MeshQuantities). */
int mcb200_set_refresh_targets(mcb200_ctx *ctx, const int32_t *desired_e, const int32_t *desired_h);

/* Effective-potential quantum correction (MeshQuantities::
 * effective_potential / quantumPotential, src/mcmodel.cpp:2337-2403, with
 * the set-up of init_effective_potential / init_p_mat / init_ep_range,
 * :2406-2664).  At every node of the quantum region the potential is
 * replaced, for electrons only, by its Gaussian average over a window of
 * ratio * theta per axis (oxide nodes raised by the barrier eb); holes keep
 * the Poisson potential's field (compute_field, :2240-2262).  With params,
 * the set-up is (re)built from the cells' material (as mcb200_set_device)
 * and quantum-region flags; enable switches the correction of every later
 * Poisson solve on or off (the reference applies it from
 * quantum_start_step on).  Lengths normalised like the mesh (nm / (1e9
 * spr0)), eb in pot0.  mcb200_get_array "qc_potential": the corrected
 * potential of the last solve. */
typedef struct {
  double ratio[3]; /* qc_{x,y,z}ratio */
  double theta[3]; /* qc_{x,y,z}theta */
  double eb;       /* Eb */
} mcb200_quantum_params;
int mcb200_set_quantum_correction(mcb200_ctx *ctx, const mcb200_quantum_params *params, const int32_t *material,
                                  const int32_t *quantum_region, int enable);
/* out = the effective potential of a caller's potential (every node; the
 * quantum nodes corrected), as a solve with the correction on applies it.
 * Waits for the result. */
int mcb200_quantum_potential(mcb200_ctx *ctx, const double *potential, double *out);

/* Copy a device array to the host: "rho", "e_rough", "e_phonon", "h_rough",
 * "h_phonon", "efield", "hfield" (3 per cell),
 * "cell_charge_e", "cell_charge_h", "cell_volume" (per cell);
 * "node_density", "node_volume", "node_doping", "vadd", "rhs", "potential"
 * (per node); "stencil" (7 per node); "qc_potential" (per node, with a
 * quantum set-up); "induced_field" (3 per cell, after
 * mcb200_set_induced_current: the weighting field E_w). */
int mcb200_get_array(mcb200_ctx *ctx, const char *name, double *out, size_t n);

#define MCB200_FLAG_SURFACE_SCATTER 1   /* Flag_SurfaceScatter */
#define MCB200_FLAG_SURFACE_IMPURITY 2  /* Flag_SurfaceImpurityScatter */
#define MCB200_FLAG_HEAT 4              /* flag_heat: phonon events tally heat */
#define MCB200_FLAG_QUANTUM 8           /* Flag_QuantumCorrection: LO / TO / LA phonon final energies drawn
                                           from the dispersion tables (FEK*, src/ElectronPhononScatter.cpp:
                                           152-167, 633-1022) */

/* Per-cell data of the device (c_motion_rule: 6 ints per cell in face
 * order UP, DOWN, LEFT, RIGHT, FRONT, BACK; c_attached_contact (1-based);
 * c_InSurfRegion; c_nearestSurf; c_da) and the surface directions
 * (SurfaceDir, up to 30).  NULL optional arrays mean zero. */
int mcb200_set_cells(mcb200_ctx *ctx, const int32_t *motion_rule, const int32_t *attached_contact,
                     const int32_t *in_surf_region, const int32_t *nearest_surf, const int32_t *surface_dir,
                     int n_surface_dir, const double *da, int flags);

/* Cell fields as felt by each carrier type (3 values per cell, the
 * reference's c_field_* / c_h_field_* times ChargeSign), and the screening
 * density Rho (c_par_charge after compute_cell_charge). */
int mcb200_set_fields(mcb200_ctx *ctx, const double *efield_xyz, const double *hfield_xyz, const double *rho);

/* Per-cell surface scattering rates (c_e_roughnessRate, c_e_surfPhononRate,
 * c_h_roughnessRate, c_h_surfPhononRate). */
int mcb200_set_surface_rates(mcb200_ctx *ctx, const double *e_rough, const double *e_phonon,
                             const double *h_rough, const double *h_phonon);

/* Particle store.  The particle count lives on the device (steps change it
 * without the host waiting); mcb200_num_particles and mcb200_download_particles
 * wait for the context's stream to read it. */
int mcb200_upload_particles(mcb200_ctx *ctx, size_t n, const mcb200_particles *p);
int mcb200_download_particles(mcb200_ctx *ctx, mcb200_particles *p, size_t capacity, size_t *n_out);
size_t mcb200_num_particles(const mcb200_ctx *ctx);
/* Particle-steps flown since the context was created (the particle count at
 * the start of every step, summed on the device); waits for the stream. */
int mcb200_particle_steps(mcb200_ctx *ctx, uint64_t *total);
/* Warm start: the particles, uid counter and potential of `src` become those
 * of `dst` (same device, flight precision and mesh dimensions; dst's store
 * must hold them).  Waits for both contexts.  No counterpart in the
 * reference. */
int mcb200_copy_ensemble(mcb200_ctx *dst, mcb200_ctx *src);

/* Append n particles of carrier `type` (0 electron, 1 hole) sampled on the
 * GPU the way the reference initialises them: cell_of[q] is the cell of new
 * particle q and charge[q] its charge; the position is uniform in the cell
 * (init_particle_data, src/particle_init.cpp:112-219) and the k-state follows
 * select_kstate (src/mcmodel.cpp:3006-3057): Boltzmann energy accepted
 * against the DOS, band by DOS share, k uniform on the iso-energy surface.
 * New uids continue after the largest uid in the store; each particle draws
 * from its own stream (seed, uid, 0xfffffffd, 0). */
int mcb200_seed_particles(mcb200_ctx *ctx, size_t n, const int32_t *cell_of, const double *charge, int type,
                          uint64_t seed);

/* One transport step: every particle flies `dt` with the reference's event
 * loop on its own random stream (seed, uid, step), copies made by
 * GENERATE / GENREF finish the step, caught particles are removed, copies
 * join with fresh uids, and the store is counting-sorted by cell.
 * Asynchronous on the context's stream (the host never waits inside it);
 * tallies accumulate.  A store that fills up with copies drops the excess
 * and the next call that reads the count (mcb200_sync, mcb200_get_tallies,
 * mcb200_download_particles, the next mcb200_step) returns
 * MCB200_ERR_CAPACITY. */
int mcb200_step(mcb200_ctx *ctx, uint32_t step, uint64_t seed, double dt);

/* Wait for the context's stream (and report a full store, as above). */
int mcb200_sync(mcb200_ctx *ctx);

/* ---- batches: many simulations stepped together ---------------------------
 * No counterpart in the reference (one simulation per process).  Members
 * are contexts made alike (mcb200_create_alike: one device, one set of band
 * tables, one flight precision), each with its own mesh, fields, store and
 * tallies, of any size.  mcb200_batch_step is mcb200_step for every member
 * at once: the flights of all members run as one persistent launch over a
 * per-member table, likewise each generation of GENERATE copies, and the
 * rest of each member's step (copies joining the store, the cell sort) runs
 * on the member's own stream.  Every particle draws from its own stream
 * (seed, uid, step), so a member's result is the one mcb200_step would give
 * it alone.  A batch step waits on the device for the work already enqueued
 * on the members' streams and the members' later work waits for it; nothing
 * waits on the host.  At most 64 members. */
typedef struct mcb200_batch mcb200_batch;
typedef struct {
  double dt;            /* normalised time step, as mcb200_step */
  uint64_t seed;        /* the member's random-stream key */
  uint32_t first_step;  /* step number of the member's first batch step (+1 per batch step) */
  /* full timesteps (mcb200_batch_run) only: */
  int self_consistent;  /* deposit every step and solve Poisson every poisson_every steps (needs set_device) */
  int poisson_every;    /* 0: 1 (the member solves when its step number is a multiple) */
  double poisson_rel_tol;  /* 0: 1e-10 */
  int surface_rates;    /* recompute the surface rates every step with the member's last mcb200_surface_rates
                           parameters */
} mcb200_batch_member;
int mcb200_batch_create(mcb200_ctx *const *ctxs, const mcb200_batch_member *members, int n, mcb200_batch **out);
void mcb200_batch_destroy(mcb200_batch *batch);
const char *mcb200_batch_last_error(const mcb200_batch *batch);
int mcb200_batch_step(mcb200_batch *batch);
/* `steps` full timesteps of every member, as density() orders them:
 * deposition, Poisson + fields where due (the members' solves run one after
 * another), surface rates, then the transport step of mcb200_batch_step.
 * With graphs on, each step is replayed from a CUDA graph captured the first
 * time its (store parity, solving members) occurs; graphs are dropped when
 * a member's mesh, fields or store change outside the batch. */
int mcb200_batch_run(mcb200_batch *batch, int steps);
int mcb200_batch_use_graphs(mcb200_batch *batch, int enable);
/* Launch shapes picked by measurement: for every candidate (batched-flight
 * blocks per SM in {1, 2} x blocks per SM of the members' per-step kernels
 * -- sort, deposition, copies -- in {2, 4, 8}; then the fastest of those
 * with every combination of overlap, pairing and the member table's place
 * switched; then the fastest of those with the members' sort-bucket width
 * in {1, 2, 4, 8} cells (mcb200_set_sort_bucket); then the fastest of those
 * with no member, every member, or the members above the first, second or
 * third quartile of the particle counts flying solo (mcb200_batch_set_solo))
 * one untimed and `trial_steps` timed full timesteps (mcb200_batch_run:
 * they advance the simulations like any other steps).  The candidates of
 * each of the four stages are timed in order and again in reverse order,
 * so that a steady drift of the simulations (particle counts) cancels; the
 * fastest mean device time is kept and returned. */
typedef struct {
  int flight_blocks_per_sm, grid_per_sm;
  int overlap; /* mcb200_batch_set_overlap */
  double ms_per_step;  /* of the kept setting */
  int candidates;
  int pair_solves; /* mcb200_batch_set_pairing */
  int sort_bucket; /* cells per sort bucket of every member */
  int smem_table;  /* mcb200_batch_set_smem_table */
  uint64_t solo_min_particles; /* mcb200_batch_set_solo (0: none) */
  int solo_members;            /* members flying solo with it */
} mcb200_batch_tuning;
int mcb200_batch_autotune(mcb200_batch *batch, int trial_steps, mcb200_batch_tuning *best);
/* Wait for the batch and every member; reports a member's full store. */
int mcb200_batch_sync(mcb200_batch *batch);
/* Resident blocks per SM of the batched flight launches (0: as many as fit). */
int mcb200_batch_set_grid(mcb200_batch *batch, int blocks_per_sm);
/* Overlap (default on): in a full timestep where some members solve Poisson,
 * the members that do not fly in a launch of their own on a second stream
 * while the solves run (a solve leaves most of the device idle: its passes
 * are bound by grid barriers); the solving members fly after their solves,
 * and a helper launch then takes over what is left of the first launch's
 * particles.  The result is the same either way. */
int mcb200_batch_set_overlap(mcb200_batch *batch, int enable);
/* Solo members (default none): members holding at least min_particles
 * particles now (0: none) fly in launches of their own on their own streams
 * -- the flight and copy flights of mcb200_step, the step number read on the
 * device so that graph replays stay right -- while the others share the
 * batched launches.  Large members fill the GPU alone and gain nothing from
 * sharing a launch; their own launches overlap the batched ones and start
 * their tails without waiting for every member's flight.  The set is fixed
 * until the next call; *members (or null) receives its size.  The result is
 * the same either way. */
int mcb200_batch_set_solo(mcb200_batch *batch, uint64_t min_particles, int *members);
/* Member table (default off): every block of a batched flight copies the
 * table of members (about 0.8 KB each) into shared memory, instead of its
 * lanes reading it from device memory through L1.  The copy costs L1
 * capacity (the shared-memory carve-out grows with it); the reads in place
 * cost L1 traffic.  The result is the same either way. */
int mcb200_batch_set_smem_table(mcb200_batch *batch, int enable);
/* Pairing (default on): two due multigrid Poisson solves whose hierarchies
 * have the same depth, smoothing and solve grid run in one cooperative
 * launch of twice the grid (each on its own half, exactly as alone: the
 * results are bit-identical), sharing the grid barriers that bound a solve.
 * Each pair counts as one batched launch. */
int mcb200_batch_set_pairing(mcb200_batch *batch, int enable);
/* CUDA events after every member's enqueued work (mcb200_mark for a batch). */
int mcb200_batch_mark(mcb200_batch *batch, int slot);
int mcb200_batch_elapsed_ms(mcb200_batch *batch, int from, int to, double *ms);
/* Members, batch steps taken, batched launches made, graphs captured and replayed. */
int mcb200_batch_info(const mcb200_batch *batch, int *members, uint64_t *steps_done, uint64_t *launches,
                      uint64_t *graph_captures, uint64_t *graph_replays);

/* Device timing of mcb200_step with CUDA events on the context's own stream
 * (enable != 0 resets the accumulators and turns timing on): enable = k >= 1
 * brackets one step in k (the first, then every k-th) with events; the
 * others run without them, since an event between two kernels costs the
 * second its overlap with the tail of the first (on the FinFET, events on
 * every step cost 3 % of the step).
 * mcb200_get_timing: out[0..n) = flight-kernel ms and flight-kernel launches
 * of the timed steps, whole-step ms and steps timed, particles flown (all
 * steps), engine kernel launches (all steps). */
int mcb200_set_timing(mcb200_ctx *ctx, int enable);
int mcb200_get_timing(const mcb200_ctx *ctx, double *out, int n);

/* CUDA events on the context's stream: mcb200_mark records event `slot`
 * (0..7); mcb200_elapsed_ms waits for `to` and returns the device time
 * between two recorded marks. */
int mcb200_mark(mcb200_ctx *ctx, int slot);
/* Overwrite a scratch buffer of `bytes` (allocated on first use, held by the
 * context) on the context's stream: evicts the L2 between timed steps. */
int mcb200_flush_l2(mcb200_ctx *ctx, size_t bytes);
int mcb200_elapsed_ms(mcb200_ctx *ctx, int from, int to, double *ms);

/* Tallies since the last reset.  Any output may be NULL.
 * counters[MCB200_NUM_COUNTERS]; contact[16*6] per contact {NumParGen,
 * CharGen, EnergyGen, NumParCatch, CharCatch, EnergyCatch};
 * lcurrent / rcurrent[ny+1]; heat_e / heat_h per mesh node. */
int mcb200_get_tallies(mcb200_ctx *ctx, uint64_t *counters, double *contact, double *lcurrent, double *rcurrent,
                       double *heat_e, double *heat_h);
int mcb200_reset_tallies(mcb200_ctx *ctx);
/* Pipelined readback of the contact tallies (mcb200_get_tallies' contact[16*6]
 * layout).  mcb200_tallies_enqueue copies them, as the work enqueued so far
 * leaves them, into slot `slot` (0..3) of a pinned host ring and returns at
 * once; mcb200_tallies_collect waits for that copy alone (work enqueued after
 * it keeps running) and converts it.  Collecting step s's tallies after step
 * s+1 is enqueued keeps the GPU busy while the host reads (enqueueing a slot
 * that holds an uncollected copy first waits for that copy).  A store that
 * dropped GENERATE copies is reported by the collect (MCB200_ERR_CAPACITY).
 * No counterpart in the reference (its tallies are host memory). */
int mcb200_tallies_enqueue(mcb200_ctx *ctx, int slot);
int mcb200_tallies_collect(mcb200_ctx *ctx, int slot, double *contact);

/* Particle store in device memory in the engine's FP64 layout (what
 * mcb200_step keeps per particle when the flight runs in FP64): absolute
 * positions, k and energy / charge in double; cell packs
 * i | j << 10 | k << 20; meta packs isym | type << 8, and bit 16 set marks a
 * particle to be dropped.  An FP32-flight store (float cell-relative
 * positions and k) has another layout and cannot be passed here. */
typedef struct {
  double *x, *y, *z;
  double *kx, *ky, *kz;
  double *energy, *charge;
  uint32_t *cell;
  int32_t *itet;
  uint32_t *meta;
  uint32_t *uid;
} mcb200_device_particles;

#define MCB200_STATIC_SORT_MAX_CELLS 262144

/* No counterpart in the reference.  Counting sort of a caller-owned device
 * particle store by mesh cell (the sort mcb200_step runs after each flight)
 * that allocates no device memory: for callers that cannot call cudaMalloc,
 * such as a host framework that owns every device buffer and lends out
 * slices of its own pool, or code that must not allocate while other work
 * holds the device.  The caller passes the input and the output arrays
 * (n entries each, in the FP64 layout above; the two stores must not share
 * any bytes, else MCB200_ERR_ARG).  Particles with meta bit 16 are dropped
 * and *n_out receives how many remain.  Every live particle's cell must lie
 * inside the nx x ny x nz mesh: one that does not is left out of the output
 * and the call returns MCB200_ERR_ARG (the kernels never index past the
 * mesh).  The scratch is one static device array of
 * MCB200_STATIC_SORT_MAX_CELLS cells (2 MiB, held by every GPU that loads
 * the library until the process exits), and larger meshes return
 * MCB200_ERR_CAPACITY.  The first call on a device looks the array's device
 * address up and caches it; make that first call before any stream capture,
 * and make no call after cudaDeviceReset (the cached address would be
 * stale).  Every call shares the array, so calls that overlap on the GPU
 * (two streams, two threads) race: serialise them.  The call returns when
 * the sort has finished on `stream` (it reads the kept count and the range
 * check back).  A CUDA error already pending on the calling thread is left
 * in place and the call does nothing but return MCB200_ERR_CUDA.  Order
 * within a cell is not specified.  `stream` is a cudaStream_t (NULL: the
 * legacy default stream). */
int mcb200_sort_particles_static(const mcb200_device_particles *in, size_t n, int nx, int ny, int nz,
                                 const mcb200_device_particles *out, size_t *n_out, void *stream);

/* Node potential (normalised, node layout) set from outside, then the cell
 * fields from it (pot2field): the fixed potential of the reference's heat
 * phase (compute_heat / heat_field, src/heat.cpp:100-128). */
int mcb200_set_potential(mcb200_ctx *ctx, const double *potential);
/* The same with the electrons' field from electron_potential (NULL: from
 * potential): heat_field takes the holes' field from the mean Poisson
 * potential and the electrons' from the mean quantum-corrected one. */
int mcb200_set_potentials(mcb200_ctx *ctx, const double *potential, const double *electron_potential);
/* Phonon events tally heat (flag_heat, src/heat.cpp:108-160) while enabled. */
int mcb200_set_heat_tally(mcb200_ctx *ctx, int enable);

/* ---- window statistics ----------------------------------------------------
 * The sums the reference accumulates every step for its stat_step outputs
 * (MeshQuantities::statistic, src/mcmodel.cpp:1167-1408): per node and
 * carrier type the CIC-weighted |q| v_x, |q| v_y, |q| v_z, |q| and |q| E of
 * every particle, per cell the particle count, per node the potential.
 * mcb200_stat_begin opens a window of `window_steps` steps (zeroes the sums
 * and fixes their int64 fixed-point units from the store's charges);
 * mcb200_stat_accumulate adds the current store and potential (call it once
 * per step); mcb200_stat_get reads a sum as doubles: "electron_qvx",
 * "electron_qvy", "electron_qvz", "electron_q", "electron_qe", "hole_..."
 * (per node, normalised units), "cell_count" (per cell), "pot_sum" (per
 * node), "steps" (1 value). */
int mcb200_stat_begin(mcb200_ctx *ctx, int window_steps);
int mcb200_stat_accumulate(mcb200_ctx *ctx);
int mcb200_stat_get(mcb200_ctx *ctx, const char *name, double *out, size_t n);

/* ---- input decks ---------------------------------------------------------
 * The reference's decks read on the host, with its own semantics:
 * input.txt key = value (MeshQuantities::getInputData,
 * src/mcmodel.cpp:3824-3992; '#' starts a comment), the node coordinates of
 * lgrid.txt in micrometres (read_grid_file, :4595-4693) and the device
 * script ldg.txt (read_device_file, :4190-4479; region, donor, acceptor,
 * motioncube, motionplane, attachcontact, contact, parnumber,
 * default_par_number, ScatterArea, surfaces, surface_scatter_range,
 * quantumRegion, VsVdVg, vgrange, ep_parm, end) applied to the cells as
 * init_by_user_input / SetMRCube / SetMRPlane do (src/mcmodel.cpp:3065-3153,
 * src/set_user_defined_data.cpp).  The grid and device files are looked up
 * relative to the directory of input.txt.  A coordinate off the grid lines
 * (where the reference exits) is MCB200_ERR_IO with the reason in
 * mcb200_deck_error(). */
typedef struct mcb200_deck mcb200_deck;

typedef struct {
  int nx, ny, nz;
  int total_step, electron_number, hole_number, stat_step, stat_heat_step, heat_steps, mr_step;
  double temperature, dt_s;
  int flag_multiple_refresh, flag_compute_potential, flag_compute_heat, flag_surface_scatter,
      flag_surface_roughness, flag_surface_phonon, flag_surface_impurity, flag_restart;
  int n_contacts, n_planes, n_surfaces, default_electrons, default_holes;
  char output_dir[512];
  int prepared;  /* mcb200_deck_prepare has run */
  double dt;     /* dt / time0 once prepared */
  int flag_quantum_correction, quantum_start_step;
  int restart_step; /* with flag_restart: the first step (mcb200_run_deck) */
} mcb200_deck_info;

/* On failure *out may still hold a deck whose mcb200_deck_error() says why. */
int mcb200_deck_load(const char *input_path, mcb200_deck **out);
void mcb200_deck_free(mcb200_deck *deck);
const char *mcb200_deck_error(const mcb200_deck *deck);
int mcb200_deck_get_info(const mcb200_deck *deck, mcb200_deck_info *info);
/* Named arrays; *needed receives the length (out may be NULL to ask).
 * Per cell, index (j * nx + i) * nz + k: int "material", "desired_electrons",
 * "desired_holes", "attached_contact", "scatter_type", "in_surf_region",
 * "quantum_region", "motion_rule" (6 per cell); "contact_planes" (7 per
 * plane: contact, i0, i1, j0, j1, k0, k1 node indices), "surface_type",
 * "surface_dir"; double "lx_m", "ly_m", "lz_m" (metres), "donor_m3",
 * "acceptor_m3", "contact_vapp_v", "contact_phims_v", "surface_pos_nm".
 * After mcb200_deck_prepare, normalised: double "lx", "ly", "lz", "dx",
 * "dy", "dz" (scaling, :4125-4166), "donor", "acceptor", "volume", "da",
 * "init_electron_charge", "init_hole_charge" (init_cell_data, :3187-3270),
 * "contact_vapp", "contact_phims", "surface_pos"; int "nearest_surf",
 * "eeff_direction" (init_surface_roughness, :3155-3185), "electron_num",
 * "hole_num", "refresh_electrons", "refresh_holes" (compute_par_num,
 * src/particle_init.cpp:17-74). */
int mcb200_deck_int_array(const mcb200_deck *deck, const char *name, int32_t *out, size_t n, size_t *needed);
int mcb200_deck_double_array(const mcb200_deck *deck, const char *name, double *out, size_t n, size_t *needed);
/* Normalise the deck with the context's units and intrinsic density; the
 * context's tables must be built at the deck's Temperature. */
int mcb200_deck_prepare(mcb200_deck *deck, const mcb200_ctx *ctx);
/* mcb200_set_mesh + mcb200_set_cells + mcb200_set_device from the deck
 * (prepares it first if needed). */
int mcb200_apply_deck(mcb200_ctx *ctx, mcb200_deck *deck);
/* The initial ensemble of init_particle_data (src/particle_init.cpp:112-219):
 * electron_num / hole_num carriers per silicon cell sharing the cell's
 * neutral charge, electrons first, cells in (i, k, j) order, each sampled by
 * mcb200_seed_particles. */
int mcb200_seed_deck(mcb200_ctx *ctx, mcb200_deck *deck, uint64_t seed);

/* ---- the self-consistent simulation (`main input.txt`) --------------------
 * MeshQuantities::run and compute_heat (src/mcmodel.cpp:499-566,
 * src/heat.cpp:108-160) over this ABI: load and apply the deck, seed the
 * initial ensemble, then total_step transport steps (statistics,
 * deposition, Poisson + fields every poisson_every steps, surface rates,
 * carrier step; MultipleRefresh every mr_step; outputs every stat_step) and,
 * with Flag_compute_heat, heat_steps steps at the last window's mean
 * potential with heat tallies on.  Outputs go to data_dir in the
 * reference's formats: current, section_current<step>, electron_num<step>,
 * pot<step>, qc_pot<step>, Electron<step>, Hole<step>, heat<step>,
 * par_info_restart<step>.  input.txt may also carry keys the reference
 * ignores: poisson_step (solve every N steps), surface_roughness_delta_nm,
 * surface_roughness_lambda_nm. */
typedef struct {
  const char *table_dir;     /* band tables (bs.si.asc, ...) */
  const char *data_dir;      /* NULL: "./data" as the reference */
  int flight_precision;      /* MCB200_FLIGHT_FP64 / MCB200_FLIGHT_FP32 */
  int poisson_every;         /* 0: input.txt's poisson_step, else 1 */
  double poisson_rel_tol;    /* 0: 1e-10 */
  int max_steps;             /* 0: the deck's total_step */
  int max_heat_steps;        /* -1: the deck's heat_steps (when Flag_compute_heat) */
  int write_outputs;
  uint64_t seed;             /* 0: 1 */
  int verbose;
  int warmup_steps;          /* transport steps run before the timed ones (counted in max_steps) */
  int readback_every_step;   /* read the contact tallies back to the host every step (pipelined: a step's
                                copy is read once the next step is enqueued; mcb200_tallies_enqueue) */
  size_t flush_l2_bytes;     /* >0: before every timed step write this many bytes (L2 eviction), timed apart */
  int profile_phases;        /* wait for the GPU after every phase so that report->phase_s holds the
                                device-side time per phase (slows the run; 0: phases are only enqueued
                                and phase_s is host enqueue time) */
} mcb200_run_options;

typedef struct {
  int steps_done, heat_steps_done, windows, refreshes;
  size_t initial_particles, final_particles;
  uint64_t particle_steps;        /* particles flown, summed over steps */
  double wall_s;                  /* host wall time of the step loops */
  double flight_ms, step_ms;      /* device time of the flight kernels / of mcb200_step */
  int poisson_solves;
  long long poisson_iterations;
  double poisson_max_residual;
  double last_current[1];         /* drain current (A/cm) of the last window */
  double heat_total;              /* sum of the heat tallies over the heat windows (kT x charge) */
  double phase_s[8];              /* host wall time per phase: statistics, deposition, Poisson + fields,
                                     surface rates, carrier step, refresh, outputs, (unused); see
                                     profile_phases */
  /* the timed transport steps (after warmup_steps): device time between
     CUDA events on the context's stream, host wall time, particles flown */
  double timed_device_ms, timed_wall_s;
  uint64_t timed_particle_steps;
  int timed_steps;
  double timed_flight_ms;         /* flight-kernel device time within them */
  uint64_t timed_flight_launches, timed_launches;
} mcb200_run_report;

/* The surface-scattering parameters mcb200_run_deck uses for a deck (the
 * reference's constants; roughness delta / Lambda from input.txt's
 * surface_roughness_delta_nm / _lambda_nm keys, else 0.1126755 nm / 2 nm)
 * in ctx's units, and input.txt's poisson_step (1 without it). */
int mcb200_deck_surface_params(const char *input_path, mcb200_ctx *ctx, const mcb200_deck_info *info,
                               mcb200_surface_params *out, int *poisson_every);

/* ---- serving bias-point requests (continuous batching) ---------------------
 * No counterpart in the reference, which runs one bias point per process.
 * A server owns one set of band tables on one device and serves requests,
 * each a device deck (input.txt with its lgrid / ldg files) of a family
 * (requests of a family share the mesh and may warm-start one another) at
 * a bias.  Each mcb200_server_round: admits queued requests in arrival
 * order while a slot (at most 64) is free and the HBM budget holds them
 * (converged ensembles kept for warm starts are evicted least recently used
 * first to make room), runs quantum_steps full timesteps of every active
 * request as one batch (mcb200_batch_run), and retires the requests whose
 * drain-current standard error -- one Ids sample per round, after the
 * discarded transient windows -- is below target_rel_err of |Ids|, or that
 * reached max_steps.  A request's steps, Poisson solves, refreshes and Ids
 * windows count its own steps from admission, so a cold-started request has
 * the same result alone or among others.  Calls are not thread-safe. */
typedef struct mcb200_server mcb200_server;
typedef struct {
  const char *table_dir;
  double kelvin;             /* lattice temperature of the tables (0: 300 K) */
  int device;
  int flight_precision;      /* MCB200_FLIGHT_FP64 / MCB200_FLIGHT_FP32 */
  size_t hbm_budget_bytes;   /* device memory for requests and warm-start entries (0: 160 GB) */
  int max_slots;             /* concurrent requests (0 or > 64: 64) */
  int quantum_steps;         /* timesteps per round = steps per Ids window (0: 50) */
  int use_graphs;            /* replay each round's steps from CUDA graphs (measured slower here: a
                                membership change re-captures every graph, and a batched step is
                                GPU-bound, so replays save little host time; off in the Python API) */
} mcb200_server_options;
typedef struct {
  const char *input_path;    /* the deck's input.txt (copied at submission) */
  const char *family;        /* warm starts stay within a family (same mesh) */
  double bias[2];            /* (Vg, Vd): the distance for nearest-bias warm starts */
  double target_rel_err;     /* complete when stderr(Ids) <= target * |Ids| (0: 0.01) */
  int min_windows;           /* kept Ids windows before completion (at least 2) */
  int max_steps;             /* complete at this many steps regardless (0: no limit) */
  int warm_windows_cold;     /* windows discarded as transient after a cold start */
  int warm_windows_warm;     /* ... after a warm start */
  int warm_start;            /* MCB200_WARM_*: start from the nearest converged bias of the family (and
                                keep this one when it converges); MCB200_WARM_SETTLED: failing a
                                converged one, from the nearest running request of the family that is
                                past its transient windows */
  int poisson_every;         /* 0: the deck's poisson_step */
  int drain_contact;         /* 0-based contact whose current is Ids */
  int ids_estimator;         /* MCB200_IDS_*: how a window's Ids is measured */
  uint64_t seed;
  double arrival_s;          /* arrival time on the server clock (mcb200_server_now), for latency */
} mcb200_request;
/* Ids estimators of a request window: the drain contact's generate / catch
 * balance (the reference's `Current = `), the net flux through the middle
 * third of the y planes (its section currents), or the current the drain
 * carries by induction (Ramo-Shockley, mcb200_set_induced_current): all
 * estimate the same steady-state current, with decreasing noise per window. */
#define MCB200_WARM_OFF 0
#define MCB200_WARM_CONVERGED 1
#define MCB200_WARM_SETTLED 2
#define MCB200_IDS_CONTACT 0
#define MCB200_IDS_SECTIONS 1
#define MCB200_IDS_INDUCED 2
#define MCB200_SERVE_CONVERGED 1
#define MCB200_SERVE_STEP_LIMIT 2
typedef struct {
  uint64_t id;
  int status;                /* MCB200_SERVE_*, or a negative error code of the admission */
  double ids, ids_stderr;    /* mean drain current (A/cm, as the reference's current file) and its stderr */
  int windows, steps;
  uint64_t particle_steps;
  double arrival_s, admit_s, done_s;  /* server clock */
  uint64_t warm_from;        /* request whose ensemble started this one (0: cold start) */
  size_t particles, bytes;   /* final particles; device memory taken */
} mcb200_result;
typedef struct {
  uint64_t rounds, particle_steps;
  double device_ms;          /* device time of the rounds' steps */
  int active, pending, cached;
  size_t bytes_in_use;
} mcb200_server_stats_t;
int mcb200_server_create(const mcb200_server_options *opt, mcb200_server **out);
void mcb200_server_destroy(mcb200_server *server);
const char *mcb200_server_last_error(const mcb200_server *server);
double mcb200_server_now(const mcb200_server *server);
int mcb200_server_submit(mcb200_server *server, const mcb200_request *request, uint64_t *id);
int mcb200_server_round(mcb200_server *server, int *active, int *pending);
/* Moves up to `max` finished results out of the server. */
int mcb200_server_results(mcb200_server *server, mcb200_result *out, int max, int *n);
int mcb200_server_stats(const mcb200_server *server, mcb200_server_stats_t *stats);

/* The window outputs of the reference's run loop for the context's current
 * state, written under data_dir: output_stat with current_scatter_info
 * (src/mcmodel.cpp:971-1161, :756-842) -- `current` (appended), section_current,
 * electron_num, pot, qc_pot, Electron, Hole and, with heat != 0, heat
 * (<name><step>, appended as the reference opens them) -- and
 * output_for_restart (:895-965, par_info_restart<step>).  The sums are those
 * of the statistics window (mcb200_stat_begin / mcb200_stat_accumulate) of
 * `window` steps and the tallies since the last reset; dt is the time step,
 * n_contacts the deck's contacts.  mcb200_run_deck calls the same writer at
 * the end of every window. */
int mcb200_write_outputs(mcb200_ctx *ctx, const char *data_dir, int step, int window, double dt, int n_contacts,
                         int heat);

/* `error` (may be NULL) receives a message on failure. */
int mcb200_run_deck(const char *input_path, int device, const mcb200_run_options *options,
                    mcb200_run_report *report, char *error, size_t error_len);

#ifdef __cplusplus
}
#endif

#endif /* MCB200_H */
