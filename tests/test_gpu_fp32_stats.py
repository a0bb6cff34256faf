"""The FP32-solvent form against the plain FP64 form on the quantities the
physics fixes (rmpcdmd_b200.validate): momentum conservation per MPCD
interval, temperature, the velocity autocorrelation, and the dimer's
propulsion velocity within its statistical error."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_bulk_fp32_against_fp64():
    from rmpcdmd_b200.validate import bulk_check

    r = bulk_check(L=24, n_intervals=20)
    # SRD conserves momentum cell by cell: per interval the FP32 total moves
    # by rounding only (target: 1e-6 of N*sqrt(kT))
    assert r["fp32"]["momentum_step_drift_max"] < 1e-6
    assert r["fp64"]["momentum_step_drift_max"] < 1e-12
    assert r["fp32"]["kinetic_energy_rel_change"] < 1e-6
    assert abs(r["temperature_rel_diff"]) < 2e-3
    # same seeds and start: the first decades of C(t) agree far inside the noise
    c32, c64 = np.array(r["vacf_fp32_first"]), np.array(r["vacf_fp64_first"])
    assert np.abs(c32[:4] - c64[:4]).max() < 1e-3
    assert r["vacf_max_abs_diff"] < 5 * r["vacf_stat_err"] + 1e-3


def test_dimer_propulsion_fp32_against_fp64():
    from rmpcdmd_b200.validate import propulsion_check

    r = propulsion_check(L=16, replicas=16, n_intervals=30, skip=5)
    assert np.isfinite(r["fp32"]["v_prop"]) and np.isfinite(r["fp64"]["v_prop"])
    assert abs(r["diff"]) < 4 * r["diff_err"]
