"""FP32 flight against FP64 (mcb200.precision), with statistics over
independent runs (seeds): a run's observable is its time average, a
precision's standard error is the spread of its runs, and a difference must
stay within the 3-sigma (99.73 %) level of Student's t for its Welch
degrees of freedom.

* the bulk velocity-field sweep (100k electrons, 0.3 ps warm-up, 5 x 0.1 ps
  windows, 8 seeds per precision): drift velocity, mean energy, phonon and
  impurity event rates and every valley's occupation agree, and no particle
  is lost to FP32-only safeguards;
* the FinFET half: the throughput FinFET (511k carriers) run through the
  same protocol in FP32 and FP64 flight (6 seeds each) and by the
  reference's own routines (the committed fixture
  tests/golden/finfet_oracle_windows.json, 6 seeds, made by
  tests/golden/make_finfet_oracle.py): drain current (Ids), drift velocity,
  heat total and mean energy agree FP32 with FP64 and each with the
  reference."""
import json
import os

import pytest

from mcb200 import precision

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("field", precision.FIELDS_KV_CM)
def test_fp32_matches_fp64_over_the_field_sweep(field):
    row = precision.sweep(electrons=100000, warmup=300, blocks=5, block_steps=100, fields=(field,), seeds=8)[0]
    e = row["error"]
    for key in precision.SWEEP_KEYS:
        assert abs(e[key]["sigmas"]) <= e[key]["limit"], (field, key, e[key])
    assert e["valley_max_sigmas"] <= 3.0, (field, e)
    assert all(r["caught"] == 0 and r["zero_time"] == 0 for r in row["fp32"])
    assert all(r["caught"] == 0 for r in row["fp64"])


FINFET_CHECKED = ("drain_current_a", "drift_velocity_y_m_s", "heat_ev_per_step", "mean_energy_ev")


def test_fp32_finfet_matches_fp64_and_the_reference():
    fixture = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "finfet_oracle_windows.json")
    oracle = json.load(open(fixture))["runs"]
    rep = precision.finfet_report(seeds=(1, 2, 3, 4, 5, 6), oracle_runs=oracle)
    for run in rep["fp64"] + rep["fp32"]:
        assert run["no_tet"] == 0 and run["zero_time"] == 0, run
    for pair in ("fp32_vs_fp64", "fp64_vs_oracle", "fp32_vs_oracle"):
        for key in FINFET_CHECKED:
            e = rep[pair][key]
            assert abs(e["sigmas"]) <= e["limit"], (pair, key, e)
