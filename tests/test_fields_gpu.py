"""GPU parity of deposition, the Poisson solve and the field update against
the reference's density() pipeline (particle_to_density -> compute_field ->
compute_cell_charge, src/mcmodel.cpp:424-471) on a two-contact n-Si bar.

* node volumes, node doping, built-in potential and the FV matrix are
  bit-identical to the reference's (init_point_data / init_matrix);
* cell charge, screening density and node charge density agree to 1e-12
  (int64 fixed point against FP64 sums);
* the engine's potential satisfies the reference's own matrix and
  right-hand side to a relative residual below 1e-10 (the reference solves
  the same system with KLU; the oracle with BiCGSTAB to 1e-14);
* fields agree with the reference's pot2field to 1e-8 of their scale;
* the multigrid-preconditioned solve (the default) and the Jacobi one reach
  the same potential, the multigrid one in far fewer iterations, and a solve
  repeated from the same start is bit-identical.
"""
import tempfile

import numpy as np
import pytest

import mcb200
from mcb200 import decks
from oracle_bridge import ORACLE_TABLES, Oracle

REF_TABLES = ORACLE_TABLES

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pair():
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.contact_bar(tmp, vd=0.3)
        orc = Oracle()
        orc.init(deck["input"], seed=21)
    orc.density_and_field()
    eng = mcb200.Engine(table_dir=ORACLE_TABLES, kelvin=orc.scalar("T0"), device=0, max_particles=1 << 16)
    eng.set_mesh(orc.array("lx"), orc.array("ly"), orc.array("lz"), orc.array("dx"), orc.array("dy"),
                 orc.array("dz"))
    eng.set_cells(orc.array("c_motion_rule").astype(np.int32), orc.array("c_da"))
    vapp, phims, planes = orc.contact_info()
    eng.set_device(orc.array("c_material").astype(np.int32), orc.array("c_donor"), orc.array("c_acceptor"),
                   vapp, phims, planes)
    eng.upload(orc.particles())
    eng.deposit()
    its, res = eng.solve_poisson(rel_tol=1e-12, max_iter=50000)
    yield orc, eng, its, res
    eng.close()


def bits_equal(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), f"{np.sum(a != b)} entries differ"


def test_device_description_is_bit_exact(pair):
    orc, eng, _, _ = pair
    bits_equal(eng.array("node_volume"), orc.array("p_volume"))
    bits_equal(eng.array("node_doping"), orc.array("p_dop"))
    bits_equal(eng.array("vadd"), orc.array("p_vadd"))
    bits_equal(eng.array("cell_volume"), orc.array("c_volume"))
    bits_equal(eng.array("stencil"), orc.poisson_stencil())


def test_deposition(pair):
    orc, eng, _, _ = pair
    for ours, ref in (("rho", "c_par_charge"), ("cell_charge_e", "c_electron_charge"),
                      ("cell_charge_h", "c_hole_charge"), ("node_density", "p_par_charge")):
        a, b = eng.array(ours), orc.array(ref)
        scale = np.max(np.abs(b))
        assert np.max(np.abs(a - b)) <= 1e-12 * scale, (ours, np.max(np.abs(a - b)) / scale)


def test_poisson_residual_against_reference_matrix(pair):
    orc, eng, its, res = pair
    assert res <= 1e-12, (its, res)
    nx, ny, nz, px, py, pz = orc.dims()
    st = orc.poisson_stencil().reshape(-1, 7)
    x = eng.array("potential").reshape(py, px, pz)
    b = orc.array("p_rhs").reshape(py, px, pz)
    ax = st[:, 6].reshape(py, px, pz) * x
    shifts = [(0, 1, -1), (1, 1, 1), (2, 0, -1), (3, 0, 1), (4, 2, -1), (5, 2, 1)]  # slot, axis, offset
    for slot, axis, off in shifts:
        coeff = st[:, slot].reshape(py, px, pz)
        nb = np.roll(x, -off, axis=axis)
        ax = ax + coeff * nb  # coefficients are zero where the neighbour is off the mesh
    rel = np.linalg.norm(b - ax) / np.linalg.norm(b)
    assert rel <= 1e-10, rel
    ref = orc.array("p_poisson_pot")
    assert np.max(np.abs(eng.array("potential") - ref)) <= 1e-8 * np.max(np.abs(ref))


def test_fields(pair):
    orc, eng, _, _ = pair
    f = np.stack([orc.array("c_field_x"), orc.array("c_field_y"), orc.array("c_field_z")], axis=1)
    e, h = eng.array("efield").reshape(-1, 3), eng.array("hfield").reshape(-1, 3)
    scale = np.max(np.abs(f))
    assert np.max(np.abs(h - f)) <= 1e-8 * scale
    assert np.max(np.abs(e + f)) <= 1e-8 * scale


def _solve_from(eng, start, method, rel_tol=1e-12):
    eng.set_poisson_solver(method)
    eng.set_potential(start)
    its, res = eng.solve_poisson(rel_tol=rel_tol, max_iter=50000)
    return its, res, eng.array("potential")


def test_multigrid_matches_jacobi(pair):
    _, eng, _, _ = pair
    zero = np.zeros(eng.mesh.nnodes)
    its_j, res_j, pot_j = _solve_from(eng, zero, mcb200.POISSON_JACOBI)
    assert eng.poisson_solver()[0] == mcb200.POISSON_JACOBI
    its_m, res_m, pot_m = _solve_from(eng, zero, mcb200.POISSON_MULTIGRID)
    used, blocks, levels = eng.poisson_solver()
    assert used == mcb200.POISSON_MULTIGRID and levels >= 2 and blocks > 0
    assert res_j <= 1e-12 and res_m <= 1e-12, (res_j, res_m)
    assert its_m * 2 < its_j, (its_m, its_j)
    scale = np.max(np.abs(pot_j))
    assert np.max(np.abs(pot_m - pot_j)) <= 1e-9 * scale
    _, _, again = _solve_from(eng, zero, mcb200.POISSON_MULTIGRID)
    assert np.array_equal(again.view(np.uint64), pot_m.view(np.uint64))
    eng.set_poisson_solver(mcb200.POISSON_AUTO)


def test_multigrid_finfet():
    """The FinFET's Poisson system (169,371 nodes, gate and contact planes,
    SiO2 / Si / vacuum): multigrid-preconditioned CG converges in a few
    dozen iterations where Jacobi needs hundreds, to the same potential."""
    with tempfile.TemporaryDirectory() as tmp:
        deck = mcb200.Deck(decks.finfet(tmp)["input"])
        eng = mcb200.Engine(table_dir=REF_TABLES, kelvin=deck.info()["temperature"], device=0, max_particles=1 << 20)
        deck.apply(eng)
    try:
        deck.seed(eng, 7)
        start = np.zeros(eng.mesh.nnodes)
        eng.deposit()
        its_j, res_j, pot_j = _solve_from(eng, start, mcb200.POISSON_JACOBI, rel_tol=1e-10)
        its_m, res_m, pot_m = _solve_from(eng, start, mcb200.POISSON_MULTIGRID, rel_tol=1e-10)
        assert eng.poisson_solver()[2] >= 4
        assert res_j <= 1e-10 and res_m <= 1e-10, (res_j, res_m)
        assert its_m <= 60 and its_m * 5 < its_j, (its_m, its_j)
        scale = np.max(np.abs(pot_j))
        assert np.max(np.abs(pot_m - pot_j)) <= 1e-7 * scale
    finally:
        eng.close()
        deck.close()


def test_induced_current_on_the_contact_bar():
    """Ramo-Shockley on the two-contact bar (uniform silicon, contacts on the
    y = 0 and y = Y node planes): the drain's weighting potential is y / Y,
    so its field is (0, -1/Y, 0) in every cell, and the induced-current
    tally of the transport steps is the sum over steps and particles of
    q v_y / -Y -- the statistic() velocity sums of the same steps (sum |q|
    v_y per carrier type) divided by Y."""
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.contact_bar(tmp, vd=0.5, electrons=3000, holes=600)
        orc = Oracle()
        orc.init(deck["input"], seed=13)
    from parity_cases import device_engine_from_oracle

    eng = device_engine_from_oracle(orc)
    try:
        eng.upload(orc.particles())
        eng.deposit()
        eng.solve_poisson(rel_tol=1e-12, max_iter=50000)
        eng.set_induced_current(1)
        ly = orc.array("ly")
        Y = ly[-1] - ly[0]
        f = eng.array("induced_field").reshape(-1, 3)
        assert np.max(np.abs(f[:, [0, 2]])) <= 1e-12 / Y
        assert np.max(np.abs(f[:, 1] + 1.0 / Y)) <= 1e-9 / Y
        window = 4
        eng.stat_begin(window)
        eng.reset_tallies()
        dt = orc.scalar("dt")
        for s in range(window):
            eng.stat_accumulate()  # the store each transport step starts from
            eng.deposit()
            eng.solve_poisson(rel_tol=1e-10)
            eng.step(s, 13, dt)
        induced, steps = eng.induced_current()
        assert steps == window
        ve, vh = eng.stat("electron_qvy").sum(), eng.stat("hole_qvy").sum()
        expected = (ve - vh) / Y  # electrons carry q = -|q|, holes +|q|; E_w,y = -1/Y
        u = eng.units()
        vbound = 1e6 / (u["spr0"] / u["time0"])  # 1e6 m/s: above any carrier's group velocity
        scale = (eng.stat("electron_q").sum() + eng.stat("hole_q").sum()) * vbound / Y
        assert abs(induced - expected) <= 1e-9 * scale, (induced, expected)
        assert abs(induced) > 1e-4 * scale  # a net drift under the 0.5 V bias
        eng.set_induced_current(-1)
    finally:
        eng.close()
