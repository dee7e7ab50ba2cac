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
