"""Shared parity scenarios: the same device state and the same Philox draws
are given to the CPU oracle (the reference's particle_fly) and to the B200
engine, and the results are compared particle by particle.

TEST INFRASTRUCTURE (used by tests/ and by __graft_entry__.smoke()).
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "c-mc_electron_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import mcb200  # noqa: E402
from mcb200 import decks  # noqa: E402
from oracle_bridge import ORACLE_TABLES, Oracle  # noqa: E402

CONT_FIELDS = ["x", "y", "z", "kx", "ky", "kz", "energy", "charge"]
DISC_FIELDS = ["i", "j", "k", "itet", "isym", "type"]
# Kinematics tolerance: the only differences allowed come from libm
# transcendentals (log / sin / cos / pow with a negative exponent), which
# CUDA and glibc may round 1 ulp apart; a few flight segments later that is
# still a relative 1e-9 at most.
REL_TOL = 1e-9
ABS_TOL = 1e-12


def engine_from_oracle(orc: Oracle, max_particles: int, flags: int = 0) -> mcb200.Engine:
    """Engine context carrying the oracle's mesh, cell data and fields."""
    eng = mcb200.Engine(table_dir=ORACLE_TABLES, kelvin=orc.scalar("T0"), device=0, max_particles=max_particles)
    eng.set_mesh(orc.array("lx"), orc.array("ly"), orc.array("lz"), orc.array("dx"), orc.array("dy"),
                 orc.array("dz"))
    surf_dir = orc.array("SurfaceDir").astype(np.int32)
    eng.set_cells(orc.array("c_motion_rule").astype(np.int32), orc.array("c_da"),
                  attached_contact=orc.array("c_attached_contact").astype(np.int32),
                  in_surf_region=orc.array("c_InSurfRegion").astype(np.int32),
                  nearest_surf=orc.array("c_nearestSurf").astype(np.int32), surface_dir=surf_dir, flags=flags)
    push_fields(orc, eng)
    return eng


def device_engine_from_oracle(orc: Oracle, max_particles: int = 1 << 16, precision: int = mcb200.FLIGHT_FP64,
                              flags: int = 0) -> mcb200.Engine:
    """Engine context carrying the oracle's mesh, cell data and device (doping,
    materials, contacts), so that it deposits and solves Poisson itself."""
    eng = mcb200.Engine(table_dir=ORACLE_TABLES, kelvin=orc.scalar("T0"), device=0, max_particles=max_particles,
                        precision=precision)
    eng.set_mesh(orc.array("lx"), orc.array("ly"), orc.array("lz"), orc.array("dx"), orc.array("dy"),
                 orc.array("dz"))
    eng.set_cells(orc.array("c_motion_rule").astype(np.int32), orc.array("c_da"),
                  attached_contact=orc.array("c_attached_contact").astype(np.int32),
                  in_surf_region=orc.array("c_InSurfRegion").astype(np.int32),
                  nearest_surf=orc.array("c_nearestSurf").astype(np.int32),
                  surface_dir=orc.array("SurfaceDir").astype(np.int32), flags=flags)
    vapp, phims, planes = orc.contact_info()
    eng.set_device(orc.array("c_material").astype(np.int32), orc.array("c_donor"), orc.array("c_acceptor"),
                   vapp, phims, planes)
    return eng


def push_fields(orc: Oracle, eng: mcb200.Engine):
    """Fields as felt by each carrier (ChargeSign = {-1, +1},
    src/Constant_GlobalVariable_MathFunction.cpp:18) and the screening density."""
    e = -np.stack([orc.array("c_field_x"), orc.array("c_field_y"), orc.array("c_field_z")], axis=1)
    h = np.stack([orc.array("c_h_field_x"), orc.array("c_h_field_y"), orc.array("c_h_field_z")], axis=1)
    eng.set_fields(e.ravel(), h.ravel(), orc.array("c_par_charge"))


def set_uniform_field(orc: Oracle, ex_v_per_m: float, ey=0.0, ez=0.0):
    f0 = orc.scalar("field0")
    n = len(orc.array("c_field_x"))
    for name, v in (("x", ex_v_per_m), ("y", ey), ("z", ez)):
        orc.set_array(f"c_field_{name}", np.full(n, v / f0))
        orc.set_array(f"c_h_field_{name}", np.full(n, v / f0))


def compare(a: dict, b: dict) -> dict:
    """Particle-by-particle comparison keyed by uid."""
    ia, ib = np.argsort(a["uid"]), np.argsort(b["uid"])
    ua, ub = a["uid"][ia], b["uid"][ib]
    out = {"n_oracle": len(ua), "n_engine": len(ub)}
    if len(ua) != len(ub) or not np.array_equal(ua, ub):
        out.update(mismatch=-1, uid_mismatch=True)
        return out
    bad = np.zeros(len(ua), dtype=bool)
    worst = 0.0
    for f in DISC_FIELDS:
        bad |= a[f][ia] != b[f][ib]
    for f in CONT_FIELDS:
        x, y = a[f][ia], b[f][ib]
        err = np.abs(x - y)
        lim = ABS_TOL + REL_TOL * np.maximum(np.abs(x), np.abs(y))
        bad |= err > lim
        rel = err / np.maximum(np.maximum(np.abs(x), np.abs(y)), 1e-300)
        worst = max(worst, float(np.max(rel[err > 0], initial=0.0)))
    out.update(mismatch=int(bad.sum()), worst_rel=worst)
    return out


def run_bulk_parity(n_particles: int = 2000, steps: int = 3, seed: int = 11, field_v_per_m: float = 1e6,
                    cells=(8, 6, 6), heat: bool = False, quantum: bool = False) -> dict:
    """Bulk n-Si box, frozen uniform field: `steps` transport steps through
    both implementations from the oracle's own initial ensemble.  quantum:
    Flag_QuantumCorrection on both sides (LO / TO / LA final energies from
    the dispersion tables)."""
    nx, ny, nz = cells
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.bulk_box(tmp, nx=nx, ny=ny, nz=nz, electrons=n_particles, holes=n_particles // 4)
        orc = Oracle()
        orc.init(deck["input"], seed=seed, make_particles=True)
    set_uniform_field(orc, field_v_per_m)
    orc.compute_cell_charge()
    if heat:
        orc.set_scalar("flag_heat", 1)
    if quantum:
        orc.set_scalar("flag_quantum_correction", 1)
    dt = orc.scalar("dt")
    p0 = orc.particles()
    n0 = len(p0["x"])
    flags = (mcb200.FLAG_HEAT if heat else 0) | (mcb200.FLAG_QUANTUM if quantum else 0)
    eng = engine_from_oracle(orc, max_particles=max(4 * n0, 4096), flags=flags)
    eng.upload(p0)
    orc.reset_tallies()
    worst = {"mismatch": 0}
    for s in range(steps):
        orc.flight_step(s)
        eng.step(s, seed, dt)
        res = compare(orc.particles(), eng.download())
        if res["mismatch"] != 0:
            res["step"] = s
            worst = res
            break
        worst = res
    t = eng.tallies()
    worst["energy_sum"] = float(np.sum(eng.download()["energy"]))
    worst.update(n_start=n0, phonon_engine=t["phonon"], phonon_oracle=int(orc.scalar("phonon_scatter")),
                 impurity_engine=t["impurity"], impurity_oracle=int(orc.scalar("impurity_scatter")),
                 events=t["events"], caught_engine=t["caught"], caught_oracle=int(orc.scalar("catch_par_num")))
    if heat:
        worst["heat_engine"] = t["heat_e"]
        worst["heat_oracle"] = orc.array("p_electron_heat")
    eng.close()
    return worst


def action_bar(dirpath: str, nx=6, ny=12, nz=5, cell_nm=2.0, vd=0.5, electrons=6000, holes=1200, dt=1e-15) -> dict:
    """A bar whose cell faces carry every ldg boundary action of HitCell
    (src/CellHit.cpp:96-211) that the other parity decks leave out, in the
    reference's deck language: PERIOD on both x faces (Period, :416-432);
    SCATTOX on both z faces with surface scattering off (Reflect or Diffuse
    by the carrier's diffuse probability, :243-386); contacts on the two
    y end planes (source 0 V, drain vd) with, one cell inside the source, a
    plane that catches carriers going left (CATCH, CatchAtContact :504-543)
    and generates copies of carriers going right (GENERATE, Generate
    :435-501); one cell inside the drain, a plane that catches carriers
    going right without the section-current tally (CATCHGATE, CatchAtGate
    :545-574) and copies carriers going left (GENREF); REFLECT at the y ends.
    The end cells are attached to their contacts (attachcontact)."""
    os.makedirs(dirpath, exist_ok=True)
    X, Y, Z = nx * cell_nm, ny * cell_nm, nz * cell_nm
    decks.write_grid(os.path.join(dirpath, "lgrid.txt"), np.arange(nx + 1) * cell_nm, np.arange(ny + 1) * cell_nm,
                     np.arange(nz + 1) * cell_nm)
    g = lambda v: f"{v:g}"
    box = f"0 {g(X)} 0 {g(Y)} 0 {g(Z)}"
    s_, d_ = cell_nm, Y - cell_nm
    lines = [
        "default_par_number 2 1",
        f"region {box} SILICON",
        f"donor {box} 1e+25",
        f"acceptor {box} 1e+21",
        f"motioncube {box} PASS PASS PASS PASS PASS PASS",
        f"motionplane 0 0 0 {g(Y)} 0 {g(Z)} UP PERIOD",
        f"motionplane {g(X)} {g(X)} 0 {g(Y)} 0 {g(Z)} DOWN PERIOD",
        f"motionplane 0 {g(X)} 0 {g(Y)} 0 0 FRONT SCATTOX",
        f"motionplane 0 {g(X)} 0 {g(Y)} {g(Z)} {g(Z)} BACK SCATTOX",
        f"motionplane 0 {g(X)} 0 0 0 {g(Z)} LEFT REFLECT",
        f"motionplane 0 {g(X)} {g(Y)} {g(Y)} 0 {g(Z)} RIGHT REFLECT",
        f"motionplane 0 {g(X)} {g(s_)} {g(s_)} 0 {g(Z)} LEFT CATCH",
        f"motionplane 0 {g(X)} {g(s_)} {g(s_)} 0 {g(Z)} RIGHT GENERATE",
        f"motionplane 0 {g(X)} {g(d_)} {g(d_)} 0 {g(Z)} RIGHT CATCHGATE",
        f"motionplane 0 {g(X)} {g(d_)} {g(d_)} 0 {g(Z)} LEFT GENREF",
        f"attachcontact 0 {g(X)} 0 {g(s_)} 0 {g(Z)} 1",
        f"attachcontact 0 {g(X)} {g(d_)} {g(Y)} 0 {g(Z)} 2",
        "contact", "1 0", f"0 {g(X)} 0 0 0 {g(Z)}", "0",
        "contact", "1 0", f"0 {g(X)} {g(Y)} {g(Y)} 0 {g(Z)}", f"{vd:g}",
        "end",
    ]
    with open(os.path.join(dirpath, "ldg.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    decks.write_input(os.path.join(dirpath, "input.txt"), dt=dt, ElectronNumber=electrons, HoleNumber=holes)
    return dict(input=os.path.join(dirpath, "input.txt"))


def make_restart(deck: dict, seed: int = 5, restart_step: int = 7) -> np.ndarray:
    """A restart file for the deck (par_info_restart's format: i j k |q|_e
    n_e |q|_h n_h, ended by -1 -1 -1) with seeded counts and charges, a few
    cells left out and one line off the mesh; input.txt switched to restart
    from it.  Returns the (nx, ny, nz) of the mesh."""
    rng = np.random.default_rng(seed)
    dk = mcb200.Deck(deck["input"])
    info = dk.info()
    dk.close()
    nx, ny, nz = info["nx"], info["ny"], info["nz"]
    lines = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                if rng.random() < 0.1:
                    continue  # not in the file: keeps the computed count and a zero charge
                ne, nh = int(rng.integers(0, 6)), int(rng.integers(0, 3))
                lines.append(f"{i} {j} {k} {rng.uniform(0.5, 2.0) * ne:.17g} {ne} {rng.uniform(0.1, 0.5) * nh:.17g} {nh}")
    lines.insert(len(lines) // 2, f"{nx + 3} 0 0 1.0 9 1.0 9")  # off the mesh: skipped
    lines.append("-1 -1 -1")
    folder = os.path.dirname(deck["input"])
    with open(os.path.join(folder, "restart.txt"), "w") as f:
        f.write("\n".join(lines) + "\n")
    with open(deck["input"]) as f:
        kv = [l for l in f.read().splitlines() if not l.startswith(("Flag_restart", "restart_step", "restart_filename"))]
    kv += ["Flag_restart=1", f"restart_step={restart_step}", "restart_filename=restart.txt"]
    with open(deck["input"], "w") as f:
        f.write("\n".join(kv) + "\n")
    return np.array([nx, ny, nz])
