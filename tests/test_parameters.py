"""Parameter files (the ParseText format of the programs) and the program
runner (``python -m rmpcdmd_b200.run``)."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from rmpcdmd_b200.parameters import ParameterError, Parameters, format_parameters

ROOT = Path(__file__).resolve().parent.parent

DIMER = {"T": 1, "L": [16, 16, 16], "rho": 10, "tau": 1, "probability": 1.0, "bulk_rmpcd": False,
         "bulk_rate": 0.001, "N_MD": 125, "N_loop": 4, "equilibration_loops": 1, "colloid_sampling": 25,
         "sigma_N": 3.0, "sigma_C": 3.0, "d": 6.5, "epsilon_N": [1.0, 0.2], "epsilon_C": [1.0, 1.0],
         "epsilon_N_N": 1.0, "epsilon_N_C": 1.0, "epsilon_C_C": 1.0, "do_hydro": True, "do_thermostat": False}

NCOLL = {"L": [20, 20, 20], "rho": 10, "T": 0.3333, "T_final": 0.4, "tau": 1.0, "N_MD": 20,
         "colloid_sampling": 2, "N_loop": 4, "N_thermo_loop": 2, "N_colloids": 5, "epsilon": 1.0, "sigma": 3.0,
         "do_hydro": True, "do_thermostat": False, "epsilon_colloids": 1.0}


def test_parse_values_and_comments():
    text = "# physical parameters\nT = 1\nL = 32 32 24   # box\nrate = 1.5d-3\nflag = F\nname = dimer run\n\n"
    p = Parameters(text)
    assert p.d("T") == 1.0 and p.i("T") == 1
    assert p.ivec("L", 3) == [32, 32, 24]
    assert p.d("rate") == 1.5e-3
    assert p.l("flag") is False
    assert p.s("name") == "dimer run"
    assert set(p.read) == {"T", "L", "rate", "flag", "name"}


def test_parse_errors():
    p = Parameters("L = 8 8\nflag = maybe\n")
    with pytest.raises(ParameterError, match="needs 3 values"):
        p.ivec("L", 3)
    with pytest.raises(ParameterError, match="not a logical"):
        p.l("flag")
    with pytest.raises(ParameterError, match="not found"):
        p.d("rho")
    with pytest.raises(ParameterError, match="key = value"):
        Parameters("just text\n")


def test_format_round_trip():
    p = Parameters(format_parameters(DIMER))
    assert p.ivec("L", 3) == DIMER["L"]
    assert p.dvec("epsilon_N", 2) == DIMER["epsilon_N"]
    assert p.l("do_hydro") is True and p.l("bulk_rmpcd") is False
    assert p.i("N_MD") == 125


@pytest.mark.gpu
def test_run_single_dimer_pbc(tmp_path):
    prm = tmp_path / "dimer.parameters"
    prm.write_text(format_parameters(DIMER))
    out = tmp_path / "dimer.npz"
    r = subprocess.run([sys.executable, "-m", "rmpcdmd_b200.run", "single_dimer_pbc", str(prm), str(out), "7"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    f = np.load(out)
    n_samples = DIMER["N_loop"] + 1
    E = f["observables/internal_energy/value"]
    V = f["observables/center_of_mass_velocity/value"]
    assert E.shape == (n_samples,) and V.shape == (n_samples, 3)
    # the checks of test/dimer_test.py on this output
    assert (E - E.mean()).std() < 0.1
    assert np.abs(V - V.mean(0)).max() < 1e-15
    assert f["particles/dimer/position/value"].shape == (n_samples * DIMER["N_MD"] // DIMER["colloid_sampling"], 2, 3)
    assert f["observables/n_solvent/value"].shape == (DIMER["N_loop"] + DIMER["equilibration_loops"] + 1, 2)
    assert int(f["parameters/seed"]) == 7 and list(f["parameters/L"]) == DIMER["L"]


@pytest.mark.gpu
def test_run_reports_the_reference_list_overflow(tmp_path):
    # sigma = 2 with the program's own capacity int(300*2**3) overflows, and
    # the run stops with the reference's message; --list-capacity lifts it
    prm = tmp_path / "dimer2.parameters"
    prm.write_text(format_parameters(dict(DIMER, sigma_N=2.0, sigma_C=2.0, d=4.5, N_loop=1, equilibration_loops=0)))
    out = tmp_path / "dimer2.npz"
    cmd = [sys.executable, "-m", "rmpcdmd_b200.run", "single_dimer_pbc", str(prm), str(out), "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode != 0 and "maximum of neighbor list reached" in r.stderr
    r = subprocess.run(cmd + ["--list-capacity", "4000"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.gpu
def test_run_n_colloids_pbc(tmp_path):
    prm = tmp_path / "nc.parameters"
    prm.write_text(format_parameters(NCOLL))
    out = tmp_path / "nc.npz"
    r = subprocess.run([sys.executable, "-m", "rmpcdmd_b200.run", "n_colloids_pbc", str(prm), str(out), "11"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    f = np.load(out)
    T = f["observables/temperature/value"]
    assert T.shape == (NCOLL["N_loop"],) and np.all(np.abs(T - 0.35) < 0.1)
    assert f["particles/colloids/position/value"].shape == (NCOLL["N_loop"] // 2, NCOLL["N_colloids"], 3)
    V = f["observables/center_of_mass_velocity/value"]
    assert np.abs(V - V.mean(0)).max() < 1e-12  # no thermostat in production: momentum conserved
