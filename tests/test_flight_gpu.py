"""GPU parity of the flight step against the reference's particle_fly.

Both sides start from the reference's own initial ensemble (Boltzmann x DOS
k-states, src/mcmodel.cpp:3006-3057) in a bulk n-Si box with a frozen
uniform field, and draw from the same Philox stream per (uid, step).
Discrete state (cell, tetrahedron, wedge, type) must match exactly and the
kinematics to a relative 1e-9 (parity_cases.REL_TOL: libm transcendentals
may round 1 ulp apart between glibc and CUDA).
"""
import numpy as np
import pytest

from parity_cases import run_bulk_parity

pytestmark = pytest.mark.gpu


def test_one_step_bulk():
    r = run_bulk_parity(n_particles=1500, steps=1, seed=11)
    print(r)
    assert r["mismatch"] == 0, r
    assert r["phonon_engine"] == r["phonon_oracle"]
    assert r["impurity_engine"] == r["impurity_oracle"]
    assert r["caught_engine"] == r["caught_oracle"]


@pytest.mark.parametrize("field", [1e5, 1e7])
def test_multi_step_fields(field):
    r = run_bulk_parity(n_particles=1000, steps=4, seed=5, field_v_per_m=field)
    print(r)
    assert r["mismatch"] == 0, r
    assert r["phonon_engine"] == r["phonon_oracle"]
    assert r["impurity_engine"] == r["impurity_oracle"]


def test_heat_tally():
    r = run_bulk_parity(n_particles=800, steps=2, seed=3, field_v_per_m=5e6, heat=True)
    assert r["mismatch"] == 0, r
    he, ho = r["heat_engine"], r["heat_oracle"]
    # int64 fixed point (2^-32 kT units) against the reference's FP64 sums
    assert np.allclose(he, ho, rtol=1e-9, atol=1e-8), np.max(np.abs(he - ho))
