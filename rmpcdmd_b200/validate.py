"""Statistical check of the FP32-solvent form against the plain FP64 form.

The FP32 form cannot match FP64 bit for bit (positions and velocities are
rounded to single precision, cell sums are compensated FP32 sums), so it is
checked on the quantities the physics fixes, each run in both precisions from
the same seeds:

* bulk SRD fluid (the loop of test/setup_bulk_decay.f90): the change of the
  total momentum per MPCD interval relative to N * sqrt(kT) (SRD conserves
  momentum cell by cell), the kinetic temperature, and the solvent velocity
  autocorrelation C(t) = sum_i v_i(0).v_i(t) / sum_i v_i(0)^2;
* single_dimer_pbc (programs/single_dimer_pbc.f90): the dimer's propulsion
  velocity, the centre-of-mass displacement per interval projected on the
  bond direction (catalytic minus noncatalytic bead), averaged over an
  ensemble of replicas run by the batched engine, with its standard error;
* n_colloids_pbc: the colloids' mean-squared displacement per interval,
  paired (an FP32 twin restarted from the FP64 state every interval).

``python -m rmpcdmd_b200.validate [--quick | --bulk L INTERVALS | --paired L
REPLICAS INTERVALS | --colloids L COLLOIDS INTERVALS]`` prints one JSON object.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import api as A
from ._capi import call
from .programs import DimerBatch, NColloidsPBC, SingleDimerPBC

KT = 1.0 / 3.0


def _bulk(L, precision, seed, n_intervals):
    L = [L, L, L]
    cells = A.CellSystem(L, 1.0)
    N = 10 * int(np.prod(L))
    p = A.ParticleSystem(N, 1, None, precision)
    p.random_placement(cells.edges, seed=seed)
    p.maxwell(KT, seed)
    p.species = 1
    rng = A.Rng(seed)
    cells.random_shift(rng)
    p.sort(cells)
    def by_id():
        # velocities in particle-id order (ids are a permutation of a
        # contiguous range): one scatter instead of a sort
        ids, v = p.download("id"), p.download("vel")
        out = np.empty_like(v)
        out[ids - ids.min()] = v
        return out

    v0 = by_id()
    norm = float((v0 * v0).sum())
    mom, temp, vacf, ekin = [], [], [1.0], []
    s = A.velocity_sums(p)
    mom.append(s[1:].copy())
    ekin.append(s[0] / 2)
    for _ in range(n_intervals):
        A.bulk_run(p, cells, rng, 1.0, 1)
        s = A.velocity_sums(p)
        mom.append(s[1:].copy())
        ekin.append(s[0] / 2)
        temp.append(A.compute_temperature(p, cells))
        vacf.append(float((v0 * by_id()).sum()) / norm)
    mom = np.array(mom)
    scale = N * np.sqrt(KT)
    step_drift = np.abs(np.diff(mom, axis=0)).max() / scale
    total_drift = np.abs(mom[-1] - mom[0]).max() / scale
    return dict(N=N, momentum_step_drift_max=float(step_drift), momentum_total_drift=float(total_drift),
                temperature_mean=float(np.mean(temp)), temperature_std=float(np.std(temp)),
                kinetic_energy_rel_change=float(abs(ekin[-1] - ekin[0]) / ekin[0]), vacf=vacf)


def bulk_check(L=32, n_intervals=30, seed=7):
    r32 = _bulk(L, A.FP32, seed, n_intervals)
    r64 = _bulk(L, A.FP64, seed, n_intervals)
    c32, c64 = np.array(r32.pop("vacf")), np.array(r64.pop("vacf"))
    # statistical error of C(t) for N independent particles: ~ sqrt(1 + C^2) / sqrt(3 N)
    err = np.sqrt((1 + c64 ** 2) / (3 * r64["N"]))
    return dict(L=L, intervals=n_intervals, fp32=r32, fp64=r64,
                temperature_rel_diff=(r32["temperature_mean"] - r64["temperature_mean"]) / r64["temperature_mean"],
                vacf_max_abs_diff=float(np.abs(c32 - c64).max()), vacf_stat_err=float(err.max()),
                vacf_fp64_first=[round(float(x), 5) for x in c64[:6]],
                vacf_fp32_first=[round(float(x), 5) for x in c32[:6]])


def _colloids(batch: DimerBatch, r: int):
    d = batch.dimers[r]
    call("rmpcd_dimer_batch_scatter", batch._h, int(r), None, d.colloids.handle, None, None, None)
    pos = d.colloids.download("pos")
    img = d.colloids.download("image")
    return pos + img * d.edges


def _propulsion(L, precision, replicas, n_intervals, skip, seed0):
    dimers = [SingleDimerPBC(L=(L, L, L), rho=10, N_MD=100, seed=seed0 + k, list_capacity=4000,
                             precision=precision) for k in range(replicas)]
    b = DimerBatch(dimers)
    prev = [_colloids(b, r) for r in range(replicas)]
    per_rep = np.zeros((replicas, n_intervals))
    for t in range(n_intervals):
        b.run(1)
        for r in range(replicas):
            x = _colloids(b, r)
            u = prev[r][0] - prev[r][1]
            u = u / np.linalg.norm(u)
            dcom = (x[0] + x[1]) / 2 - (prev[r][0] + prev[r][1]) / 2
            per_rep[r, t] = float(dcom @ u)  # tau = 1
            prev[r] = x
    v = per_rep[:, skip:].mean(axis=1)
    return dict(replicas=replicas, intervals=n_intervals, skipped=skip, v_prop=float(v.mean()),
                v_prop_err=float(v.std(ddof=1) / np.sqrt(replicas)))


def propulsion_check(L=32, replicas=32, n_intervals=60, skip=10, seed0=1000):
    p32 = _propulsion(L, A.FP32, replicas, n_intervals, skip, seed0)
    p64 = _propulsion(L, A.FP64, replicas, n_intervals, skip, seed0)
    diff = p32["v_prop"] - p64["v_prop"]
    err = float(np.hypot(p32["v_prop_err"], p64["v_prop_err"]))
    return dict(L=L, fp32=p32, fp64=p64, diff=diff, diff_err=err,
                rel_diff=diff / p64["v_prop"] if p64["v_prop"] else None,
                rel_err=err / abs(p64["v_prop"]) if p64["v_prop"] else None)


def _unwrapped(d: SingleDimerPBC):
    return d.colloids.download("pos") + d.colloids.download("image") * d.edges


def _sync_twin(twin: SingleDimerPBC, d: SingleDimerPBC) -> None:
    """twin (FP32 solvent) <- the state of d (FP64) at an interval boundary:
    every solvent array rounded to single precision, the colloids as they
    are, the grid origin and the random-number step; then the re-sort the
    program makes at that point (sort, neighbor list, pos_old), so the
    twin's cells and list are those of its own rounded positions."""
    for f in ("pos", "vel", "force", "force_old", "image", "id", "species", "flags"):
        twin.solvent.upload(f, d.solvent.download(f))
    for f in ("pos", "vel", "force", "force_old", "image", "species"):
        twin.colloids.upload(f, d.colloids.download(f))
    twin.cells.origin = d.cells.origin
    twin.rng.step = d.rng.step
    twin._resort()


def paired_propulsion_check(L=16, replicas=8, n_intervals=40, skip=3, seed0=2000):
    """The FP32 form's bias on the propulsion velocity, paired: at every
    interval boundary of plain FP64 runs an FP32 twin takes the FP64 state
    (rounded), both run the same interval with the same random numbers, and
    the difference of their dimer displacements along the bond is recorded.
    The two share their noise for the interval, so the mean difference -- the
    FP32 bias per interval -- is resolved far below the propulsion velocity's
    own statistical error (programs/single_dimer_pbc.f90:364-369)."""
    d64 = [SingleDimerPBC(L=(L, L, L), rho=10, N_MD=100, seed=seed0 + k, list_capacity=4000,
                          precision=A.FP64) for k in range(replicas)]
    tw = [SingleDimerPBC(L=(L, L, L), rho=10, N_MD=100, seed=seed0 + k, list_capacity=4000,
                         precision=A.FP32) for k in range(replicas)]
    for d in d64:
        for _ in range(skip):
            d.interval()
    disp64 = np.zeros((replicas, n_intervals))
    delta = np.zeros((replicas, n_intervals))
    nb64 = np.zeros((replicas, n_intervals))   # change of the B count over the interval (FP64)
    nb_delta = np.zeros((replicas, n_intervals))  # FP32 twin minus FP64

    def n_b(x):
        return int((x.solvent.download("species") == 2).sum())

    for t in range(n_intervals):
        for r in range(replicas):
            d, w = d64[r], tw[r]
            _sync_twin(w, d)
            x0 = _unwrapped(d)
            u = x0[0] - x0[1]
            u = u / np.linalg.norm(u)
            c0 = (x0[0] + x0[1]) / 2
            b0 = n_b(d)
            d.interval()
            w.interval()
            a = float(((_unwrapped(d)[0] + _unwrapped(d)[1]) / 2 - c0) @ u)
            b = float(((_unwrapped(w)[0] + _unwrapped(w)[1]) / 2 - c0) @ u)
            disp64[r, t] = a
            delta[r, t] = b - a
            b64 = n_b(d)
            nb64[r, t] = b64 - b0
            nb_delta[r, t] = n_b(w) - b64
    n = delta.size
    bias = float(delta.mean())
    # replicas are independent; intervals of one replica are nearly so for
    # the paired difference (the twin restarts from the FP64 state each time)
    bias_err = float(delta.std(ddof=1) / np.sqrt(n))
    v = float(disp64.mean())
    v_err = float(disp64.mean(axis=1).std(ddof=1) / np.sqrt(replicas)) if replicas > 1 else float("nan")
    # B species: the net change of the B count per interval (reactions A -> B
    # at the catalytic bead less refuelling B -> A far away), FP64, and the
    # paired FP32-minus-FP64 difference of the count after the interval
    return dict(L=L, replicas=replicas, intervals=n_intervals, skipped=skip, samples=n, bias=bias,
                bias_err=bias_err, delta_std=float(delta.std(ddof=1)), delta_abs_max=float(np.abs(delta).max()),
                v_prop_fp64=v, v_prop_fp64_err=v_err,
                b_change_fp64=float(nb64.mean()), b_change_fp64_err=float(nb64.std(ddof=1) / np.sqrt(n)),
                b_bias=float(nb_delta.mean()), b_bias_err=float(nb_delta.std(ddof=1) / np.sqrt(n)),
                b_delta_abs_max=float(np.abs(nb_delta).max()))


def _sync_nc_twin(twin: NColloidsPBC, d: NColloidsPBC) -> None:
    """twin (FP32 solvent) <- the state of d (FP64) at an interval boundary,
    where every solvent particle is caught up and sorted: the solvent arrays
    rounded to single precision, the colloids as they are, the grid origin,
    the random-number step and the loop counters; then the program's
    catch-up and sort with nothing to catch up, which sorts the twin's
    rounded positions and rebuilds its list and pos_old."""
    for f in ("pos", "vel", "force", "force_old", "image", "id", "species", "flags"):
        twin.solvent.upload(f, d.solvent.download(f))
    for f in ("pos", "vel", "force", "force_old", "image", "species"):
        twin.colloids.upload(f, d.colloids.download(f))
    twin.cells.origin = d.cells.origin
    twin.rng.step = d.rng.step
    twin.t, twin.last_sort = d.t, d.last_sort
    twin._catch_up_and_sort()


def paired_colloids_check(L=128, n_colloids=200, n_intervals=20, skip=2, seed=3000):
    """n_colloids_pbc: the FP32 form's bias on the colloids' mean-squared
    displacement per interval, paired as in paired_propulsion_check: at every
    interval boundary of a plain FP64 run an FP32 twin takes its state, both
    run one production interval with the same random numbers, and the
    difference of the colloids' mean |displacement|^2 over the interval is
    recorded (programs/n_colloids_pbc.f90:304-324)."""
    kw = dict(L=(L, L, L), rho=10, N_MD=100, N_colloids=n_colloids, seed=seed, volume_correction=False)
    d = NColloidsPBC(precision=A.FP64, **kw)
    tw = NColloidsPBC(precision=A.FP32, **kw)
    d.thermalise(skip)
    msd64 = np.zeros(n_intervals)
    delta = np.zeros(n_intervals)
    dmax = 0.0
    for t in range(n_intervals):
        _sync_nc_twin(tw, d)
        x0 = _unwrapped(d)
        d.run(1)
        tw.run(1)
        a, b = _unwrapped(d) - x0, _unwrapped(tw) - x0
        msd64[t] = float((a * a).sum(axis=1).mean())
        delta[t] = float((b * b).sum(axis=1).mean()) - msd64[t]
        dmax = max(dmax, float(np.abs(b - a).max()))
    return dict(L=L, colloids=n_colloids, intervals=n_intervals, msd_per_interval_fp64=float(msd64.mean()),
                msd_per_interval_fp64_err=float(msd64.std(ddof=1) / np.sqrt(n_intervals)),
                msd_bias=float(delta.mean()), msd_bias_err=float(delta.std(ddof=1) / np.sqrt(n_intervals)),
                displacement_diff_abs_max=dmax)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--quick", action="store_true", help="small sizes (a minute)")
    ap.add_argument("--bulk", type=int, nargs=2, metavar=("L", "INTERVALS"),
                    help="only the bulk check, on an L^3 box for INTERVALS intervals")
    ap.add_argument("--paired", type=int, nargs=3, metavar=("L", "REPLICAS", "INTERVALS"),
                    help="only the paired dimer check, on L^3 boxes")
    ap.add_argument("--colloids", type=int, nargs=3, metavar=("L", "COLLOIDS", "INTERVALS"),
                    help="only the paired n_colloids_pbc check")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    if a.bulk:
        out = dict(bulk=bulk_check(L=a.bulk[0], n_intervals=a.bulk[1]))
    elif a.colloids:
        out = dict(colloids=paired_colloids_check(L=a.colloids[0], n_colloids=a.colloids[1],
                                                  n_intervals=a.colloids[2]))
    elif a.paired:
        out = dict(paired=paired_propulsion_check(L=a.paired[0], replicas=a.paired[1], n_intervals=a.paired[2],
                                                  skip=2))
    elif a.quick:
        out = dict(bulk=bulk_check(L=24, n_intervals=20),
                   propulsion=propulsion_check(L=16, replicas=16, n_intervals=30, skip=5),
                   paired=paired_propulsion_check(L=16, replicas=8, n_intervals=20, skip=3))
    else:
        out = dict(bulk=bulk_check(L=48, n_intervals=50),
                   propulsion=propulsion_check(L=32, replicas=64, n_intervals=200, skip=20),
                   paired=paired_propulsion_check(L=32, replicas=16, n_intervals=40, skip=5))
    out["seconds"] = round(time.perf_counter() - t0, 1)
    print(json.dumps(out))
    return out


if __name__ == "__main__":
    main()
