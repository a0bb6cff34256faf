"""``rmpcdmd run`` for the programs on the solvent path (scripts/rmpcdmd.in:42-81):

    python -m rmpcdmd_b200.run PROGRAM sim.parameters sim.npz SEED [--fp32]

PROGRAM is ``single_dimer_pbc`` or ``n_colloids_pbc``; the parameter file is
the program's own (same keys, read as programs/single_dimer_pbc.f90:127-193
and programs/n_colloids_pbc.f90:87-160 read them); SEED is a signed 64-bit
integer or ``auto``.  The reference writes H5MD; this image has no HDF5
library, so the runner stores the same series under their H5MD paths
(``observables/internal_energy/value``, ``particles/dimer/position/value``,
``parameters/<key>``, ...) in a NumPy ``.npz`` archive.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

from . import api as A
from .parameters import Parameters


def _seed(text: str) -> int:
    if text == "auto":
        return int.from_bytes(os.urandom(8), "little", signed=True)
    return int(text)


def _u64(seed: int) -> int:
    return seed % (1 << 64)


class Series:
    """Append-only series stored as arrays at H5MD-like paths."""

    def __init__(self):
        self.data: dict[str, list] = {}

    def append(self, path: str, value):
        self.data.setdefault(path, []).append(np.asarray(value))

    def arrays(self) -> dict:
        return {k: np.stack(v) for k, v in self.data.items()}


def run_single_dimer_pbc(prm: Parameters, seed: int, precision: int, log=print, list_capacity=None) -> dict:
    """The main loop of programs/single_dimer_pbc.f90:303-445 through the C ABI.
    The neighbor-list capacity defaults to the program's int(300 max(sigma)^3),
    which overflows for sigma = 2 ('maximum of neighbor list reached', as the
    reference stops); list_capacity overrides it."""
    from .programs import SingleDimerPBC

    prob = prm.d("probability")
    bulk_rmpcd = prm.l("bulk_rmpcd")
    bulk_rate = prm.d("bulk_rate")
    L = prm.ivec("L", 3)
    rho = prm.i("rho")
    T = prm.d("T")
    d = prm.d("d")
    tau = prm.d("tau")
    N_MD = prm.i("N_MD")
    colloid_sampling = prm.i("colloid_sampling")
    N_loop = prm.i("N_loop")
    equilibration_loops = prm.i("equilibration_loops")
    sigma_C = prm.d("sigma_C")
    sigma_N = prm.d("sigma_N")
    eps_C = prm.dvec("epsilon_C", 2)
    eps_N = prm.dvec("epsilon_N", 2)
    eps_CC = prm.d("epsilon_C_C")
    eps_NC = prm.d("epsilon_N_C")
    eps_NN = prm.d("epsilon_N_N")
    do_hydro = prm.l("do_hydro")
    do_thermostat = prm.l("do_thermostat")
    g = SingleDimerPBC(L=L, rho=rho, T=T, tau=tau, N_MD=N_MD, sigma_C=sigma_C, sigma_N=sigma_N, d=d,
                       epsilon_C=eps_C, epsilon_N=eps_N, epsilon_CC=eps_CC, epsilon_NC=eps_NC, epsilon_NN=eps_NN,
                       probability=prob, bulk_rmpcd=bulk_rmpcd, bulk_rate=bulk_rate, do_thermostat=do_thermostat,
                       do_hydro=do_hydro, seed=_u64(seed), precision=precision, list_capacity=list_capacity)
    out = Series()
    log(f"Running for {equilibration_loops} + {N_loop} loops; mass {g.mass}")
    for i in range(N_loop + equilibration_loops + 1):
        sampling = i >= equilibration_loops
        for j in range(1, N_MD + 1):
            g.md_step(want_energy=sampling and j == N_MD)
            if sampling and j % colloid_sampling == 0:
                out.append("particles/dimer/position/value", g.colloids.pos)
                out.append("particles/dimer/velocity/value", g.colloids.vel)
                out.append("particles/dimer/image/value", g.colloids.image)
        if sampling:
            th = g.thermo()
            out.append("observables/temperature/value", th["temperature"])
            out.append("observables/potential_energy/value", th["potential"])
            out.append("observables/kinetic_energy/value", th["kinetic"])
            out.append("observables/internal_energy/value", th["internal"])
            out.append("observables/center_of_mass_velocity/value", th["v_com"])
        g.mpcd()
        out.append("observables/n_solvent/value", A.n_solvent(g.solvent, 2))
    res = out.arrays()
    res["observables/n_extra_sorting"] = np.asarray(g.n_extra_sorting)
    return res


def run_n_colloids_pbc(prm: Parameters, seed: int, precision: int, log=print, list_capacity=None) -> dict:
    """programs/n_colloids_pbc.f90: thermalisation (N_thermo_loop) then the
    production loop with the temperature ramp, through rmpcd_ncolloids_run."""
    from .programs import NColloidsPBC

    L = prm.ivec("L", 3)
    rho = prm.i("rho")
    T_init = prm.d("T")
    T_final = prm.d("T_final")
    tau = prm.d("tau")
    N_MD = prm.i("N_MD")
    colloid_sampling = prm.i("colloid_sampling")
    N_loop = prm.i("N_loop")
    N_thermo_loop = prm.i("N_thermo_loop")
    N_colloids = prm.i("N_colloids")
    epsilon = prm.d("epsilon")
    sigma = prm.d("sigma")
    do_hydro = prm.l("do_hydro")
    do_thermostat = prm.l("do_thermostat")
    epsilon_colloids = prm.d("epsilon_colloids")
    g = NColloidsPBC(L=L, rho=rho, T=T_init, T_final=T_final, tau=tau, N_MD=N_MD, N_colloids=N_colloids,
                     sigma=sigma, epsilon=epsilon, epsilon_colloids=epsilon_colloids, do_hydro=do_hydro,
                     do_thermostat=do_thermostat, seed=_u64(seed), precision=precision, list_capacity=list_capacity)
    log(f"{g.N} solvent particles; thermostatting for {N_thermo_loop} loops")
    g.thermalise(N_thermo_loop)
    out = Series()
    Ts = [T_init + (i - 1) * (T_final - T_init) / max(1, N_loop - 1) for i in range(1, N_loop + 1)]
    for i in range(1, N_loop + 1):
        g._native(1, g.do_thermostat, [Ts[i - 1]], 0)
        if i % colloid_sampling == 0:
            out.append("particles/colloids/position/value", g.colloids.pos)
            out.append("particles/colloids/velocity/value", g.colloids.vel)
            out.append("particles/colloids/image/value", g.colloids.image)
        temperature = A.compute_temperature(g.solvent, g.cells)
        vs = A.velocity_sums(g.solvent)
        cv = g.colloids.vel
        kin = vs[0] / 2 + (g.mass * (cv ** 2).sum(1) / 2).sum()
        vcom = (vs[1:] + g.mass * cv.sum(0)) / (g.N + g.mass * len(cv))
        pot = g.e1 + g.e2
        out.append("observables/temperature/value", temperature)
        out.append("observables/potential_energy/value", pot)
        out.append("observables/kinetic_energy/value", kin)
        out.append("observables/internal_energy/value", pot + kin)
        out.append("observables/center_of_mass_velocity/value", vcom)
    res = out.arrays()
    res["observables/n_extra_sorting"] = np.asarray(g.n_extra_sorting)
    return res


PROGRAMS = {"single_dimer_pbc": run_single_dimer_pbc, "n_colloids_pbc": run_n_colloids_pbc}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m rmpcdmd_b200.run",
                                 description="run an RMPCDMD program from its parameter file")
    ap.add_argument("program", choices=sorted(PROGRAMS))
    ap.add_argument("parameters")
    ap.add_argument("output", help=".npz archive (H5MD paths as keys)")
    ap.add_argument("seed", help="signed 64-bit integer, or 'auto'")
    ap.add_argument("--fp32", action="store_true", help="FP32 solvent (colloids stay FP64)")
    ap.add_argument("--list-capacity", type=int, default=None,
                    help="neighbor-list capacity per colloid (default: the program's own formula)")
    args = ap.parse_args(argv)
    seed = _seed(args.seed)
    prm = Parameters.from_file(args.parameters)
    print(f"RMPCDMD running {args.program} {args.parameters} {args.output} {seed}")
    t0 = time.time()
    res = PROGRAMS[args.program](prm, seed, A.FP32 if args.fp32 else A.FP64, list_capacity=args.list_capacity)
    res["parameters/seed"] = np.asarray(seed)
    for k, v in prm.read.items():
        res[f"parameters/{k}"] = np.asarray(v)
    np.savez(args.output, **res)
    print(f"{time.time() - t0:.1f}s elapsed")
    return 0


if __name__ == "__main__":
    sys.exit(main())
