"""FP32 flight on the GPU: state validity, reproducibility, and agreement of
the ensemble observables with the plain FP64 path (which is bit-exact
against the reference's routines, see test_flight_gpu.py).

FP32 flight draws from its own stream and rounds kinematics to float, so it
is compared statistically.  Both precisions start from the same seeded
ensemble (the initial sampling runs in FP64 for both stores) of the bulk
n-Si box (E_x = 10 kV/cm, N_D = 1e17 cm^-3, 300 K, dt = 1 fs) and fly the
same number of steps; each observable must agree within 4 combined standard
errors:
  mean energy, mean x displacement (drift), valley occupation fractions,
  real phonon and impurity events per particle-step.
State validity after the flight (state_checks.consistency):
  k inside its tetrahedron within 4e-5 (FP32; twice the float containment
  tolerance) / 1e-12 (FP64), carried energy equal to the band energy at k
  within 5e-3 kT max and 1e-4 kT rms (FP32) / 1e-9 kT (FP64), positions
  inside their cells.
"""
import numpy as np
import pytest

import mcb200
from mcb200.workloads import bulk_box_engine
from oracle_bridge import ORACLE_TABLES, Oracle
from state_checks import consistency

pytestmark = pytest.mark.gpu

N = 320000
STEPS = 300
SEED = 7


def _run(precision, steps=STEPS, seed=SEED):
    eng, dt, _ = bulk_box_engine(N, seed, 0, precision=precision)
    p0 = eng.download()
    eng.reset_tallies()
    for s in range(steps):
        eng.step(s, seed, dt)
    p = eng.download()
    t = eng.tallies()
    c = consistency(eng, p)
    eng.close()
    o0, o = np.argsort(p0["uid"]), np.argsort(p["uid"])
    return {k: v[o0] for k, v in p0.items()}, {k: v[o] for k, v in p.items()}, t, c


@pytest.fixture(scope="module")
def runs():
    return {"fp64": _run(mcb200.FLIGHT_FP64), "fp32": _run(mcb200.FLIGHT_FP32)}


def test_fp32_store_round_trip():
    import tempfile

    from mcb200 import decks
    from parity_cases import engine_from_oracle

    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.bulk_box(tmp, nx=6, ny=5, nz=4, electrons=2000, holes=400)
        orc = Oracle()
        orc.init(deck["input"], seed=3)
    p = orc.particles()
    eng = engine_from_oracle(orc, max_particles=1 << 14)
    eng.set_flight_precision(mcb200.FLIGHT_FP32)
    assert eng.precision == mcb200.FLIGHT_FP32
    eng.upload(p)
    q = eng.download()
    for f in ("i", "j", "k", "itet", "isym", "type", "uid", "energy", "charge"):
        assert np.array_equal(q[f], p[f]), f
    for f, nodes, idx in (("x", orc.array("lx"), p["i"]), ("y", orc.array("ly"), p["j"]), ("z", orc.array("lz"), p["k"])):
        rel = p[f] - nodes[idx]
        # one float rounding of the offset, plus the double additions
        assert np.all(np.abs(q[f] - p[f]) <= np.abs(rel) * 2.0 ** -23 + 4 * np.spacing(np.abs(p[f]))), f
    for f in ("kx", "ky", "kz"):
        assert np.all(np.abs(q[f] - p[f]) <= np.abs(p[f]) * 2.0 ** -24), f
    with pytest.raises(mcb200.EngineError):
        eng.set_flight_precision(mcb200.FLIGHT_FP64)  # store not empty
    eng.close()


def test_same_initial_ensemble(runs):
    a, b = runs["fp64"][0], runs["fp32"][0]
    for f in ("i", "j", "k", "itet", "isym", "energy", "charge"):
        assert np.array_equal(a[f], b[f]), f


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_state_valid_after_flight(runs, prec):
    _, p, t, c = runs[prec]
    assert c["band_ok"]
    assert len(p["x"]) == N
    assert t["caught"] == 0 and t["no_tet"] == 0 and t["zero_time"] == 0 and t["too_many_events"] == 0
    if prec == "fp64":
        assert c["k_outside_max"] <= 1e-12
        assert c["energy_err_max"] <= 1e-9
        assert c["position_outside_max"] <= 1e-12
    else:
        assert c["k_outside_max"] <= 4e-5
        assert c["energy_err_max"] <= 5e-3
        assert c["energy_err_rms"] <= 1e-4
        assert c["position_outside_max"] <= 1e-5


def _agree(a, b, sa, sb, what):
    sigma = np.sqrt(sa ** 2 + sb ** 2)
    assert abs(a - b) <= 4 * sigma, f"{what}: fp32 {b} vs fp64 {a} (4 sigma = {4 * sigma})"


def test_fp32_observables_match_fp64(runs):
    (p0a, pa, ta, _), (p0b, pb, tb, _) = runs["fp64"], runs["fp32"]
    n = len(pa["x"])
    _agree(pa["energy"].mean(), pb["energy"].mean(), pa["energy"].std() / np.sqrt(n),
           pb["energy"].std() / np.sqrt(n), "mean energy")
    da, db = pa["x"] - p0a["x"], pb["x"] - p0b["x"]
    _agree(da.mean(), db.mean(), da.std() / np.sqrt(n), db.std() / np.sqrt(n), "mean x displacement")
    for v in range(6):
        fa, fb = np.mean(pa["isym"] // 8 == v), np.mean(pb["isym"] // 8 == v)
        _agree(fa, fb, np.sqrt(fa * (1 - fa) / n), np.sqrt(fb * (1 - fb) / n), f"valley {v}")
    for key in ("phonon", "impurity"):
        _agree(ta[key], tb[key], np.sqrt(ta[key]), np.sqrt(tb[key]), key)


def test_fp32_reproducible():
    _, a, ta, _ = _run(mcb200.FLIGHT_FP32, steps=40, seed=11)
    _, b, tb, _ = _run(mcb200.FLIGHT_FP32, steps=40, seed=11)
    for f in a:
        assert np.array_equal(a[f], b[f]), f
    for key in ta:
        assert np.array_equal(np.asarray(ta[key]), np.asarray(tb[key])), key
