"""The self-consistent loop on the GPU.

* test_self_consistent_steps_match_oracle: deposition -> Poisson -> fields ->
  flight, step after step, against the reference's density() + flight
  (oracle, same Philox streams) on the two-contact bar: the discrete state
  (cells, tetrahedra, wedges, carrier types) stays identical and the
  kinematics agree to 1e-7 relative.  The engine solves Poisson with CG to
  a 1e-12 relative residual and the oracle with BiCGSTAB to 1e-14, so the
  fields differ at the 1e-11 level; the kinematic tolerance covers that,
  the discrete state must not depend on it.
* test_statistics_match_host: the window statistics (statistic(),
  src/mcmodel.cpp:1167-1408) of one step equal a host CIC of the same
  downloaded store to 1e-9 relative (int64 fixed point).
* test_run_deck_*: mcb200_run_deck (the engine's `main input.txt`) on the
  contact bar and on a reduced FinFET, in FP64 and FP32 flight: every output
  file the reference writes exists and parses, the Poisson residual stays
  below 1e-10, the particle count stays within the refresh targets.
"""
import os
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from oracle_bridge import ORACLE_TABLES, Oracle
from parity_cases import DISC_FIELDS, make_restart

pytestmark = pytest.mark.gpu


def _engine_for(orc, max_particles=1 << 16):
    eng = mcb200.Engine(table_dir=ORACLE_TABLES, kelvin=orc.scalar("T0"), device=0, max_particles=max_particles)
    eng.set_mesh(orc.array("lx"), orc.array("ly"), orc.array("lz"), orc.array("dx"), orc.array("dy"),
                 orc.array("dz"))
    eng.set_cells(orc.array("c_motion_rule").astype(np.int32), orc.array("c_da"),
                  attached_contact=orc.array("c_attached_contact").astype(np.int32))
    vapp, phims, planes = orc.contact_info()
    eng.set_device(orc.array("c_material").astype(np.int32), orc.array("c_donor"), orc.array("c_acceptor"),
                   vapp, phims, planes)
    return eng


def test_self_consistent_steps_match_oracle():
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.contact_bar(tmp, vd=0.5, electrons=3000, holes=600)
        orc = Oracle()
        orc.init(deck["input"], seed=33)
    eng = _engine_for(orc)
    eng.upload(orc.particles())
    dt = orc.scalar("dt")
    orc.reset_tallies()
    for s in range(5):
        orc.density_and_field()
        orc.flight_step(s)
        eng.deposit()
        its, res = eng.solve_poisson(rel_tol=1e-12, max_iter=50000)
        assert res <= 1e-12
        eng.step(s, 33, dt)
        a, b = orc.particles(), eng.download()
        ia, ib = np.argsort(a["uid"]), np.argsort(b["uid"])
        assert np.array_equal(a["uid"][ia], b["uid"][ib]), s
        for f in DISC_FIELDS:
            assert np.array_equal(a[f][ia], b[f][ib]), (s, f)
        for f in ("x", "y", "z", "kx", "ky", "kz", "energy", "charge"):
            x, y = a[f][ia], b[f][ib]
            assert np.all(np.abs(x - y) <= 1e-12 + 1e-7 * np.maximum(np.abs(x), np.abs(y))), (s, f)
    t = eng.tallies()
    assert t["generated"] == int(orc.scalar("gen_par"))
    assert t["caught"] == int(orc.scalar("catch_par_num"))
    eng.close()


def test_statistics_match_host():
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.contact_bar(tmp, vd=0.5, electrons=3000, holes=600)
        orc = Oracle()
        orc.init(deck["input"], seed=5)
    eng = _engine_for(orc)
    eng.upload(orc.particles())
    eng.deposit()
    eng.solve_poisson()
    lib = mcb200.lib()
    assert lib.mcb200_stat_begin(eng._ctx, 4) == 0
    assert lib.mcb200_stat_accumulate(eng._ctx) == 0
    nx, ny, nz = eng.mesh.nx, eng.mesh.ny, eng.mesh.nz
    nodes = (nx + 1) * (ny + 1) * (nz + 1)
    got = {}
    for name in ("electron_q", "electron_qe", "electron_qvx", "hole_q", "cell_count", "pot_sum"):
        n = nx * ny * nz if name == "cell_count" else nodes
        out = np.zeros(n)
        assert lib.mcb200_stat_get(eng._ctx, name.encode(), out.ctypes.data_as(mcb200.ctypes.POINTER(mcb200.ctypes.c_double)), n) == 0
        got[name] = out
    p = eng.download()
    lx, ly, lz = orc.array("lx"), orc.array("ly"), orc.array("lz")
    dx, dy, dz = orc.array("dx"), orc.array("dy"), orc.array("dz")
    rx = (p["x"] - lx[p["i"]]) / dx[p["i"]]
    ry = (p["y"] - ly[p["j"]]) / dy[p["j"]]
    rz = (p["z"] - lz[p["k"]]) / dz[p["k"]]
    exp_q = {0: np.zeros(nodes), 1: np.zeros(nodes)}
    exp_qe = np.zeros(nodes)
    for di, wx in ((0, 1 - rx), (1, rx)):
        for dj, wy in ((0, 1 - ry), (1, ry)):
            for dk, wz in ((0, 1 - rz), (1, rz)):
                node = ((p["j"] + dj) * (nx + 1) + p["i"] + di) * (nz + 1) + p["k"] + dk
                w = np.abs(p["charge"] * wx * wy * wz)
                for t in (0, 1):
                    sel = p["type"] == t
                    np.add.at(exp_q[t], node[sel], w[sel])
                np.add.at(exp_qe, node[p["type"] == 0], (w * p["energy"])[p["type"] == 0])
    scale = np.abs(exp_q[0]).max()
    assert np.max(np.abs(got["electron_q"] - exp_q[0])) <= 1e-9 * scale
    assert np.max(np.abs(got["hole_q"] - exp_q[1])) <= 1e-9 * max(np.abs(exp_q[1]).max(), 1e-300)
    assert np.max(np.abs(got["electron_qe"] - exp_qe)) <= 1e-9 * np.abs(exp_qe).max()
    cells = (p["j"] * nx + p["i"]) * nz + p["k"]
    assert np.array_equal(got["cell_count"], np.bincount(cells, minlength=nx * ny * nz).astype(float))
    assert np.array_equal(got["pot_sum"], eng.array("potential"))
    assert np.all(np.isfinite(got["electron_qvx"]))
    eng.close()


def _check_outputs(data, last_step, has_heat=False):
    for prefix in ("section_current", "electron_num", "pot", "qc_pot", "Electron", "Hole", "par_info_restart"):
        path = os.path.join(data, f"{prefix}{last_step}")
        assert os.path.exists(path), path
    pot = np.loadtxt(os.path.join(data, f"pot{last_step}"))
    assert pot.shape[1] == 4 and np.all(np.isfinite(pot[:, 3]))
    el = np.loadtxt(os.path.join(data, f"Electron{last_step}"))
    assert el.shape[1] == 8 and np.all(np.isfinite(el[:, 3:]))
    assert np.all(el[:, 7] >= 0)
    text = open(os.path.join(data, "current")).read()
    assert "Current = " in text and "times of phonon scatter" in text
    rst = open(os.path.join(data, f"par_info_restart{last_step}")).read().split("\n")
    assert rst[-2] == "-1 -1 -1"
    if has_heat:
        assert any(f.startswith("heat") for f in os.listdir(data))


@pytest.mark.parametrize("precision", [mcb200.FLIGHT_FP64, mcb200.FLIGHT_FP32])
def test_run_deck_contact_bar(precision):
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.contact_bar(tmp, vd=0.5, electrons=6000, holes=600)
        text = open(deck["input"]).read()
        text = text.replace("total_step=100", "total_step=40").replace("stat_step=1000000", "stat_step=20")
        text = text.replace("Flag_MultipleRefresh=0", "Flag_MultipleRefresh=1").replace("mr_step=50", "mr_step=10")
        open(deck["input"], "w").write(text)
        data = os.path.join(tmp, "data")
        rep = mcb200.run_deck(deck["input"], data_dir=data, precision=precision, table_dir=ORACLE_TABLES)
        assert rep["steps_done"] == 40 and rep["windows"] == 2 and rep["refreshes"] == 4
        assert rep["poisson_solves"] == 40 and rep["poisson_max_residual"] <= 1e-10
        assert rep["final_particles"] > 0.5 * rep["initial_particles"]
        assert np.isfinite(rep["last_current"])
        _check_outputs(data, 39)


def test_run_deck_readback_every_step_changes_nothing():
    """The per-step (pipelined) readback of the contact tallies only reads:
    the run ends with the same particles, current and outputs."""
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.contact_bar(tmp, vd=0.5, electrons=6000, holes=600)
        text = open(deck["input"]).read().replace("total_step=100", "total_step=30")
        open(deck["input"], "w").write(text)
        reps = [mcb200.run_deck(deck["input"], precision=mcb200.FLIGHT_FP64, table_dir=ORACLE_TABLES,
                                write_outputs=False, readback_every_step=rb) for rb in (False, True)]
    for k in ("steps_done", "final_particles", "last_current", "poisson_solves"):
        assert reps[0][k] == reps[1][k], k


@pytest.mark.parametrize("precision", [mcb200.FLIGHT_FP64, mcb200.FLIGHT_FP32])
def test_run_deck_finfet(precision):
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.finfet(tmp, electrons=40000, holes=5000, total_step=30, heat_steps=10, stat_step=10, mr_step=10)
        data = os.path.join(tmp, "data")
        rep = mcb200.run_deck(deck["input"], data_dir=data, precision=precision, poisson_every=5,
                              table_dir=ORACLE_TABLES)
        assert rep["steps_done"] == 30 and rep["heat_steps_done"] == 10
        assert rep["poisson_solves"] == 6 and rep["poisson_max_residual"] <= 1e-10
        assert rep["final_particles"] > 0.5 * rep["initial_particles"]
        _check_outputs(data, 29, has_heat=True)
        assert np.isfinite(rep["heat_total"])


def test_main_executable_contact_bar():
    """`mcb200_main input.txt` (the drop-in for the reference's `main
    input.txt`) on the contact bar, run from the deck's folder as the
    reference is: exit status 0, ./data/current with one block per
    statistics window, and the same files, byte for byte, as
    mcb200_run_deck writes for the same deck and seed."""
    import shutil
    import subprocess

    exe = os.path.join(os.path.dirname(mcb200.LIB_PATH), "mcb200_main")
    assert os.path.exists(exe), exe
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.contact_bar(tmp, vd=0.5, electrons=4000, holes=400)
        text = open(deck["input"]).read()
        text = text.replace("total_step=100", "total_step=20").replace("stat_step=1000000", "stat_step=10")
        open(deck["input"], "w").write(text)
        env = dict(os.environ, MCB200_TABLES=ORACLE_TABLES)
        run = subprocess.run([exe, "input.txt", "--quiet", "--seed", "5"], cwd=tmp, env=env, capture_output=True,
                             text=True, timeout=300)
        assert run.returncode == 0, run.stderr
        assert "done: 20 steps" in run.stdout, run.stdout
        data = os.path.join(tmp, "data")
        current = open(os.path.join(data, "current")).read()
        assert current.count("step = ") == 2 and "step = 9" in current and "step = 19" in current, current
        assert current.count("Current = ") == 2 * 2  # two contacts per window
        shutil.move(data, os.path.join(tmp, "data_exe"))
        rep = mcb200.run_deck(deck["input"], data_dir=os.path.join(tmp, "data_lib"), table_dir=ORACLE_TABLES, seed=5)
        assert rep["steps_done"] == 20
        names = sorted(os.listdir(os.path.join(tmp, "data_exe")))
        assert names == sorted(os.listdir(os.path.join(tmp, "data_lib")))
        for name in names:
            a = open(os.path.join(tmp, "data_exe", name), "rb").read()
            b = open(os.path.join(tmp, "data_lib", name), "rb").read()
            assert a == b, name


def test_restart_seed_matches_oracle():
    """Flag_restart seeding (init_particle_data with
    read_par_info_for_restart): per cell and carrier type the same number of
    particles as the reference, each with the same charge, bit for bit --
    the file's charge shared away from the contacts, the neutral charge in
    contact cells, nothing in a restarted cell with no carriers."""
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.contact_bar(tmp, vd=0.4, electrons=3000, holes=500)
        make_restart(d)
        orc = Oracle()
        orc.init(d["input"], seed=1)
        ref = orc.particles()
        deck = mcb200.Deck(d["input"])
        eng = mcb200.Engine(table_dir=ORACLE_TABLES, kelvin=deck.info()["temperature"], max_particles=1 << 16)
        deck.apply(eng)
        deck.seed(eng, 1)
        deck.close()
    got = eng.download()
    eng.close()

    def canon(p):
        order = np.lexsort((p["charge"], p["k"], p["j"], p["i"], p["type"]))
        return {k: np.asarray(p[k])[order] for k in ("type", "i", "j", "k", "charge")}

    a, b = canon(got), canon(ref)
    assert len(a["charge"]) == len(b["charge"]) > 0
    for k in ("type", "i", "j", "k"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(a["charge"].view(np.uint64), b["charge"].view(np.uint64))


def test_run_deck_from_restart():
    """mcb200_run_deck on a restart deck: seeded from the file, stepped from
    restart_step (7) on, outputs named by that step count."""
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.contact_bar(tmp, vd=0.4, electrons=3000, holes=500)
        make_restart(d, restart_step=7)
        with open(d["input"]) as f:
            kv = [l for l in f.read().splitlines() if not l.startswith("stat_step")]
        with open(d["input"], "w") as f:
            f.write("\n".join(kv + ["stat_step=3"]) + "\n")
        data = os.path.join(tmp, "data")
        rep = mcb200.run_deck(d["input"], data_dir=data, table_dir=ORACLE_TABLES, max_steps=4, max_heat_steps=0)
        names = set(os.listdir(data))
    assert rep["steps_done"] == 4
    # steps 7..10: the window ends at step 8 (8 % 3 == 2)
    assert "pot8" in names and "pot2" not in names, sorted(names)
