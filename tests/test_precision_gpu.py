"""FP32 flight against FP64 across the bulk velocity-field sweep
(mcb200.precision at its defaults: 100k electrons, 0.3 ps warm-up, 5 x 0.1 ps windows).  For every
field, drift velocity and mean energy agree within 4 combined standard
errors or 1 % (the tolerance the FP32 path is held to), valley fractions
within 4 sigma, phonon / impurity event rates within 1 %; no particle is
lost to FP32-only safeguards."""
import pytest

from mcb200 import precision

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("field", precision.FIELDS_KV_CM)
def test_fp32_matches_fp64_over_the_field_sweep(field):
    row = precision.sweep(electrons=100000, warmup=300, blocks=5, block_steps=100, fields=(field,))[0]
    e = row["error"]
    for key in ("drift_velocity_m_s", "mean_energy_ev"):
        assert abs(e[key]["sigmas"]) <= 4 or abs(e[key]["rel_error"]) <= 0.01, (field, key, e[key])
    assert e["valley_max_sigmas"] <= 4 or e["valley_max_abs_error"] <= 0.005, (field, e)
    for key in ("phonon_per_particle_step", "impurity_per_particle_step"):
        assert abs(e[key]["rel_error"]) <= 0.01 or abs(e[key]["sigmas"]) <= 4, (field, key, e[key])
    assert row["fp32"]["caught"] == 0 and row["fp32"]["zero_time"] == 0
    assert row["fp64"]["caught"] == 0


def test_fp32_finfet_matches_fp64_and_the_reference():
    """The FinFET half of the precision study (mcb200.precision.finfet_report):
    the throughput FinFET run from equilibrium for 300 steps, then 8 windows
    of 100 steps, in FP32 flight and in FP64 flight on the GPU, and the same
    protocol through the reference's own routines (the committed fixture
    tests/golden/finfet_oracle_windows.json, made by
    tests/golden/make_finfet_oracle.py).  Drain, source and section
    currents, the electrons' drift velocity and mean energy, and the heat
    given to the lattice: FP32 against FP64 and FP64 against the reference
    within 3 standard errors of the window-by-window differences."""
    import json
    import os

    fixture = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "finfet_oracle_windows.json")
    oracle = json.load(open(fixture))["windows"]
    rep = precision.finfet_report(seed=1, oracle_windows=oracle)
    for run in ("fp64", "fp32"):
        assert rep[run]["no_tet"] == 0 and rep[run]["zero_time"] == 0, rep[run]
    for pair in ("fp32_vs_fp64", "fp64_vs_oracle", "fp32_vs_oracle"):
        for key, e in rep[pair].items():
            assert abs(e["sigmas"]) <= 3, (pair, key, e)
