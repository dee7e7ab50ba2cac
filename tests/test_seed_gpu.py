"""GPU seeding of the initial ensemble (seed_kernel, mcb200_seed_particles)
against the reference's own select_kstate (src/mcmodel.cpp:3006-3057) and
the placement of init_particle_data (src/particle_init.cpp:185-207), particle
by particle on the same per-particle streams (seed, uid, 0xfffffffd, 0).

* FP64 store: cell, tetrahedron and wedge bit for bit; position, k and
  energy to 1e-9 relative -- the energy draw takes exp and log, which CUDA
  and glibc may round one ulp apart, the flight parity's tolerance.
* FP32 store: the same FP64 draw rounded once -- tetrahedron, wedge and
  cell exact, energy (kept in FP64) to 1e-9; positions (cell-relative
  floats) and k within float rounding.
"""
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from oracle_bridge import Oracle
from parity_cases import REL_TOL, engine_from_oracle

pytestmark = pytest.mark.gpu

SEED = 29


def _case(n_e=2500, n_h=700, seed=SEED):
    with tempfile.TemporaryDirectory() as tmp:
        d = decks.bulk_box(tmp, nx=6, ny=5, nz=4, electrons=10, holes=0)
        orc = Oracle()
        orc.init(d["input"], seed=1, make_particles=False)
    nx, ny, nz = 6, 5, 4
    rng = np.random.default_rng(seed)
    cells_e = rng.integers(0, nx * ny * nz, n_e).astype(np.int32)
    cells_h = rng.integers(0, nx * ny * nz, n_h).astype(np.int32)
    q_e = -rng.uniform(0.5, 2.0, n_e) * 1e-4
    q_h = rng.uniform(0.5, 2.0, n_h) * 1e-4
    ref = []
    uid = 0
    for carrier, cells, q in ((0, cells_e, q_e), (1, cells_h, q_h)):
        for c, qq in zip(cells, q):
            k, i, j = int(c % nz), int((c // nz) % nx), int(c // (nz * nx))
            ref.append(orc.seed_particle(seed, uid, i, j, k, carrier, float(qq)))
            uid += 1
    keys = ref[0].keys()
    ref = {k: np.array([r[k] for r in ref]) for k in keys}
    return orc, (cells_e, q_e, cells_h, q_h), ref


def _seeded(orc, args, precision, seed=SEED):
    eng = engine_from_oracle(orc, max_particles=1 << 14)
    if precision != mcb200.FLIGHT_FP64:
        eng.set_flight_precision(precision)
    cells_e, q_e, cells_h, q_h = args
    eng.seed(cells_e, q_e, 0, seed)
    eng.seed(cells_h, q_h, 1, seed)
    got = eng.download()
    eng.close()
    order = np.argsort(got["uid"])
    return {k: np.asarray(v)[order] for k, v in got.items()}


def test_seed_fp64_matches_select_kstate():
    orc, args, ref = _case()
    got = _seeded(orc, args, mcb200.FLIGHT_FP64)
    n = len(ref["x"])
    assert len(got["x"]) == n and np.array_equal(got["uid"], np.arange(n))
    for f in ("i", "j", "k", "type", "itet", "isym"):
        assert np.array_equal(got[f], ref[f]), f
    assert np.array_equal(got["charge"], ref["charge"])
    for f in ("x", "y", "z", "kx", "ky", "kz", "energy"):
        a, b = got[f], np.asarray(ref[f], dtype=np.float64)
        assert np.all(np.abs(a - b) <= 1e-12 + REL_TOL * np.maximum(np.abs(a), np.abs(b))), f
    # the sampled ensemble is not degenerate: both carrier types, many wedges, an equilibrium energy spread
    assert len(np.unique(ref["isym"])) == 48
    assert 0.5 < np.mean(ref["energy"][ref["type"] == 0]) < 3.0  # mean energy ~1.5 kT


def test_seed_fp32_store_rounds_the_fp64_draw():
    orc, args, ref = _case(n_e=1500, n_h=400, seed=SEED + 3)
    got = _seeded(orc, args, mcb200.FLIGHT_FP32, seed=SEED + 3)
    for f in ("i", "j", "k", "type", "itet", "isym"):
        assert np.array_equal(got[f], ref[f]), f
    assert np.allclose(got["energy"], ref["energy"], rtol=REL_TOL, atol=1e-12)
    for f in ("kx", "ky", "kz"):
        assert np.allclose(got[f], ref[f], rtol=2e-7, atol=1e-7), f
    h = orc.array("dx")[0]
    for f in ("x", "y", "z"):
        assert np.max(np.abs(got[f] - ref[f])) <= 1e-6 * h, f
