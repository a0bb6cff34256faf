"""Benchmark of the bulk SRD fluid hot path: solvent particle-steps per second.

Workload (one "step" = one MPCD interval of the bulk loop of
test/setup_bulk_decay.f90: simple_mpcd_step -> mpcd_stream_periodic(tau) ->
random_shift -> sort): a 128 x 128 x 128 periodic box at density 10, i.e.
20,971,520 solvent particles, Maxwell velocities at kT = 1/3, alpha = pi/2,
tau = 1.  Inputs are synthetic (seeded placement and velocities); the
particle arrays (~1 GB in FP32, ~1.5 GB in FP64 per copy) exceed the 126 MB
L2, so no L2 flush is needed between steps.

The headline `value` is the FP32 form (the production form); the plain FP64
form, which reproduces the reference arithmetic bit for bit, is reported in
`fp64_plain`.  `--impl reference` times the CPU restatement of the same loop
(the reference is Fortran and cannot be built here) on the host cores.

Multi-GPU: the bulk system does not shard without a halo exchange; N GPUs run
N independent replicas (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L_DEFAULT = 128
RHO = 10
T_INIT = 1.0 / 3.0
TAU = 1.0
SEED = 20241203
# HBM bytes the fused interval kernel must move per particle and per slot:
# read + write of the full particle record (32 B FP32, 56 B FP64), the
# permutation index (4 B) and the next key (4 B); per slot the count and start
# read and the next count written
BYTES_PER_PARTICLE = {32: 72, 64: 120}
BYTES_PER_SLOT = 12
# Minimum bytes of one whole interval (stream + sort + collide) over the
# reference's particle state kept as separate arrays (FP32: pos 12, vel 12,
# image 12, species/flags 4, id 4 = 44 B; FP64: 72 B): key pass reads pos+vel
# and writes a key, the permutation reads the key and moves the state, the
# collision reads vel+species and writes vel; 16 B per slot for counts/starts.
INTERVAL_BYTES_PER_PARTICLE = {32: 148, 64: 252}
INTERVAL_BYTES_PER_SLOT = 16


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(precision):
    """dram bytes per particle of the fused kernel from the committed ncu summary, or None."""
    f = ROOT / "profiles" / "k_bulk_interval.md"
    if not f.exists():
        return None
    key = f"dram_bytes_per_particle_fp{precision}:"
    for line in f.read_text().splitlines():
        if line.strip().startswith(key):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out = ""

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[2:]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


def make_system(rm, L, precision):
    from rmpcdmd_b200 import programs

    cells = rm.CellSystem([L, L, L], 1.0)
    N = RHO * L ** 3
    p = rm.ParticleSystem(N, 1, None, precision)
    p.random_placement(cells.edges, seed=SEED)
    p.maxwell(T_INIT, SEED)
    p.species = 1
    rng = rm.Rng(SEED)
    cells.random_shift(rng)
    p.sort(cells)
    rm.synchronize()
    return p, cells, rng


def timed_run(rm, p, cells, rng, steps, warmup):
    """Device time (ms) of `steps` intervals after `warmup`, plus the average
    duration of the fused interval kernel from its CUDA events."""
    from rmpcdmd_b200._capi import call
    import ctypes as C

    rm.bulk_run(p, cells, rng, TAU, warmup)
    rm.synchronize()
    rm.Timers.enable(True)
    rm.Timers.reset()
    a, b = C.c_int(), C.c_int()
    call("rmpcd_mark", C.byref(a))
    rm.bulk_run(p, cells, rng, TAU, steps)
    call("rmpcd_mark", C.byref(b))
    rm.synchronize()
    ms = C.c_float()
    call("rmpcd_elapsed_ms", a, b, C.byref(ms))
    tm = rm.Timers.read()
    rm.Timers.enable(False)
    return float(ms.value), tm


def call_by_call_ms(rm, p, cells, rng, steps):
    """Device time (ms) of `steps` intervals issued the way the reference's
    bulk loop issues them (test/setup_bulk_decay.f90:112-121), one C-ABI call
    per module procedure: simple_mpcd_step, mpcd_stream_periodic,
    random_shift, sort."""
    from rmpcdmd_b200._capi import call
    import ctypes as C

    def interval():
        rm.simple_mpcd_step(p, cells, rng)
        rm.mpcd_stream_periodic(p, cells, TAU)
        cells.random_shift(rng)
        p.sort(cells)

    interval()
    rm.synchronize()
    a, b = C.c_int(), C.c_int()
    call("rmpcd_mark", C.byref(a))
    for _ in range(steps):
        interval()
    call("rmpcd_mark", C.byref(b))
    rm.synchronize()
    ms = C.c_float()
    call("rmpcd_elapsed_ms", a, b, C.byref(ms))
    return float(ms.value)


def roofline(N, S, precision, phase, peak, peak_kind):
    secs, calls = phase.get("interval_fused", (0.0, 0))
    if not calls:
        return None
    avg = secs / calls
    alg = N * BYTES_PER_PARTICLE[precision] + S * BYTES_PER_SLOT
    achieved = alg / avg / 1e9
    t = profile_traffic(precision)
    return {"kernel": "k_bulk_interval", "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": None if t is None else int(t * N), "algorithmic_bytes": int(alg),
            "avg_launch_ms": round(avg * 1e3, 4), "launches": calls}


# single_dimer_pbc configurations (MD step = tau / N_MD = 0.01)
DIMER_N_MD = 100
DIMER_LIST_CAPACITY = 4000
# HBM bytes per solvent particle and MD step of the two streaming kernels of
# the dimer engine (step begin: flags, pos r/w, vel, pos_old -- species only
# for a batch created with a negative species; step end: flags, plus in the
# FP64 form every velocity, in the FP32 form only those of particles with a
# force; force entries are touched only for flagged particles)
DIMER_BYTES_PER_MD_STEP = {32: 56, 64: 128}


def dimer_boxes_batched(n=512, seed=2024):
    r = np.random.default_rng(seed)
    return [(int(s),) * 3 for s in r.choice([16, 20, 24, 32, 40, 48], size=n)]


def shard(items, rank, world):
    """The replicas rank `rank` of `world` runs: every world-th one from
    `rank` on, so the ranks split a replica ensemble with no overlap and the
    box mix stays alike on every rank."""
    return list(items)[rank::world]


def dimer_time(rm, dimers, n_intervals, use_graph=True, tuned=None):
    """Device time (ms) of n_intervals of a DimerBatch built from `dimers`,
    on the engine shape its autotuner picks (its tuning intervals are real
    intervals of the run), after one warm-up interval (which also captures
    the interval graph).  `tuned`, if a dict, receives the autotuner's
    choice."""
    from rmpcdmd_b200.programs import DimerBatch
    from rmpcdmd_b200._capi import call
    import ctypes as C

    b = DimerBatch(dimers, use_graph=use_graph)
    res = b.autotune(1)
    if tuned is not None:
        prec = int(dimers[0].solvent.precision)
        tuned.update(res, shape=DimerBatch.shapes(prec)[res["best"]])
    b.run(1)
    rm.synchronize()
    a, e = C.c_int(), C.c_int()
    call("rmpcd_mark", C.byref(a))
    b.run(n_intervals)
    call("rmpcd_mark", C.byref(e))
    rm.synchronize()
    ms = C.c_float()
    call("rmpcd_elapsed_ms", a, e, C.byref(ms))
    extra = int(b.n_extra_sorting().sum())
    return float(ms.value), b.n_solvent, extra


def dimer_entry(N, ms, n_intervals, precision, peak, peak_kind, extra=None):
    md_steps = n_intervals * DIMER_N_MD
    secs = ms * 1e-3
    alg = DIMER_BYTES_PER_MD_STEP[precision] * N * md_steps
    achieved = alg / secs / 1e9
    out = {"value": N * md_steps / secs, "us_per_md_step": round(ms * 1e3 / md_steps, 2), "intervals": n_intervals,
           "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind,
                        "unit": "GB/s", "frac": round(achieved / peak, 4),
                        "algorithmic_bytes_per_particle_md_step": DIMER_BYTES_PER_MD_STEP[precision],
                        "note": "streaming bytes of the MD step over the whole interval time (sort, list and "
                                "collision included in the time only)"}}
    if extra is not None:
        out["n_extra_sorting"] = extra
    return out


def run_dimer(rm, peak, peak_kind, local, dist=None, rank=0, world=1):
    """single_dimer_pbc through the batched engine: one dimer at 32^3 (plain
    FP64, FP32 solvent, and the call-by-call driver for comparison), one at
    96^3 (FP32 solvent and FP64), and 512 replicas with uneven boxes (FP32
    solvent).  With N ranks the single dimers run as one independent replica
    per rank and the 512 replicas are split between the ranks (`shard`);
    times are the maximum over ranks and rates count every rank's
    particles."""
    from rmpcdmd_b200.programs import SingleDimerPBC

    def timed(*a, **k):
        barrier(dist)
        ms, N, ex = dimer_time(rm, *a, **k)
        return max_over_ranks(dist, ms), N * world, ex

    def make(boxes, seeds, precision):
        return [SingleDimerPBC(L=L, rho=RHO, N_MD=DIMER_N_MD, seed=s, list_capacity=DIMER_LIST_CAPACITY,
                               precision=precision) for L, s in zip(boxes, seeds)]

    out = {"unit": "particle-steps/s (solvent particles x MD steps / device time, dt = tau/N_MD = 0.01)",
           "data": "synthetic: seeded uniform solvent (rejected inside the colloid cut), Maxwell kT=1/3, "
                   "dimer sigma=2, d=4.5, p(A->B)=1, refuel beyond 0.45 L; list capacity 4000"}
    tu = {}
    ms, N, ex = timed(make([(32, 32, 32)], [SEED], 64), 5, tuned=tu)
    out["single_dimer_32_fp64_plain"] = dict(dimer_entry(N, ms, 5, 64, peak, peak_kind, ex), N=N, replicas=1,
                                             autotune=tu)
    tu = {}
    ms, N, ex = timed(make([(32, 32, 32)], [SEED], 32), 5, tuned=tu)
    out["single_dimer_32_fp32"] = dict(dimer_entry(N, ms, 5, 32, peak, peak_kind, ex), N=N, replicas=1,
                                       autotune=tu)
    d = make([(32, 32, 32)], [SEED], 64)[0]
    d.interval()
    rm.synchronize()
    t0 = time.perf_counter()
    d.interval()
    rm.synchronize()
    cbc = max_over_ranks(dist, time.perf_counter() - t0)
    out["single_dimer_32_fp64_call_by_call"] = {"value": N * DIMER_N_MD / cbc,
                                                "us_per_md_step": round(cbc * 1e6 / DIMER_N_MD, 2),
                                                "path": "one C-ABI call per module procedure (wall clock)"}
    for prec in (32, 64):
        tu = {}
        ms, N, ex = timed(make([(96, 96, 96)], [SEED], prec), 2, tuned=tu)
        out[f"single_dimer_96_fp{prec}"] = dict(dimer_entry(N, ms, 2, prec, peak, peak_kind, ex), N=N, replicas=1,
                                                autotune=tu)
    boxes_all = dimer_boxes_batched()
    mine = shard(zip(boxes_all, range(1, len(boxes_all) + 1)), rank, world)
    boxes = [b for b, _ in mine]
    tu = {}
    with ClockSampler(local) as cs:
        barrier(dist)
        ms, N, ex = dimer_time(rm, make(boxes, [sd for _, sd in mine], 32), 2, tuned=tu)
        ms = max_over_ranks(dist, ms)
        N = int(round(sum_over_ranks(dist, N)))
    e = dimer_entry(N, ms, 2, 32, peak, peak_kind, ex)
    e.update(N=N, replicas=len(boxes_all), replicas_per_rank=len(boxes),
             boxes="cubic sides drawn from {16,20,24,32,40,48}, seed 2024", clocks=cs.summary(), autotune=tu)
    # the same replicas one at a time in plain FP64: every replica of the
    # rank's share, each on its own autotuned engine shape (the tuner
    # remembers one per box size), one timed interval after a warm-up one
    seq_ms, seq_N = 0.0, 0
    for b_k, seed_k in mine:
        m1, n1, _ = dimer_time(rm, make([b_k], [seed_k], 64), 1)
        seq_ms += m1
        seq_N += n1
    seq_ms = max_over_ranks(dist, seq_ms)
    seq_N = int(round(sum_over_ranks(dist, seq_N)))
    e["fp64_plain_one_replica_at_a_time"] = {"value": seq_N * DIMER_N_MD / (seq_ms * 1e-3),
                                             "sample": f"all {len(boxes_all)} replicas (boxes and seeds as in the "
                                                       "batch), one after another, one timed interval each"}
    e["batched_over_sequential_fp64"] = round(e["value"] / e["fp64_plain_one_replica_at_a_time"]["value"], 3)
    out["batched_512_fp32"] = e
    # n_colloids_pbc: 200 passive colloids (sigma 3) in 128^3, the program's
    # loop call by call through the C ABI (lazy cell-wise streaming)
    from rmpcdmd_b200.programs import NColloidsPBC
    for prec in (32, 64):
        g = NColloidsPBC(L=(128, 128, 128), rho=RHO, N_MD=DIMER_N_MD, N_colloids=200, seed=SEED,
                         volume_correction=False, precision=prec)
        g.thermalise(1)
        rm.synchronize()
        # the host reads each MD step's re-sort decision, so the loop's wall
        # clock carries host noise: best of five 2-interval runs
        sec = float("inf")
        for _ in range(5):
            barrier(dist)
            t0 = time.perf_counter()
            g.thermalise(2)
            rm.synchronize()
            sec = min(sec, max_over_ranks(dist, (time.perf_counter() - t0) / 2))
        out[f"n_colloids_128_fp{prec}"] = {
            "value": world * g.N * DIMER_N_MD / sec, "us_per_md_step": round(sec * 1e6 / DIMER_N_MD, 2), "N": g.N,
            "colloids": 200, "n_extra_sorting": g.n_extra_sorting,
            "path": "rmpcd_ncolloids_run (the program's calls issued in C; wall clock, best of 5 runs of 2 "
                    "thermostatted intervals)"}
        if prec == 64:
            t0 = time.perf_counter()
            g.interval(True, g.T_init)
            rm.synchronize()
            sec = max_over_ranks(dist, time.perf_counter() - t0)
            out["n_colloids_128_fp64_call_by_call"] = {
                "value": world * g.N * DIMER_N_MD / sec, "us_per_md_step": round(sec * 1e6 / DIMER_N_MD, 2),
                "path": "one C-ABI call per module procedure from Python (wall clock)"}
        del g
    return out


def e2e_run(rm, p, cells, rng, steps):
    """The same loop through the public API with host arrays: every step
    uploads the particle arrays from page-locked host memory in the reference
    layout, runs one interval and downloads them again."""
    import ctypes as C

    from rmpcdmd_b200._capi import call

    N = p.Nmax
    fields = [("pos", 3, np.float64), ("vel", 3, np.float64), ("image", 3, np.int32), ("id", 1, np.int32),
              ("species", 1, np.int32), ("flags", 1, np.int32)]
    bufs, ptrs = {}, []
    for name, k, dt in fields:
        nbytes = N * k * np.dtype(dt).itemsize
        ptr = C.c_void_p()
        call("rmpcd_host_alloc", C.c_size_t(nbytes), C.byref(ptr))
        ptrs.append(ptr)
        arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_byte)), shape=(nbytes,)).view(dt)
        bufs[name] = arr
        call("rmpcd_particles_download", p.handle, name.encode(), ptr)
    nbytes_step = sum(N * k * np.dtype(dt).itemsize for _, k, dt in fields)
    rm.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        for name, _, _ in fields:
            call("rmpcd_particles_upload", p.handle, name.encode(), bufs[name].ctypes.data_as(C.c_void_p))
        rm.bulk_run(p, cells, rng, TAU, 1)
        for name, _, _ in fields:
            call("rmpcd_particles_download", p.handle, name.encode(), bufs[name].ctypes.data_as(C.c_void_p))
    rm.synchronize()
    dt_s = time.perf_counter() - t0
    for ptr in ptrs:
        call("rmpcd_host_free", ptr)
    return N * steps / dt_s, nbytes_step, nbytes_step


def cpu_model():
    """The host CPU's model name (Linux /proc/cpuinfo), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_sample(L_sample=64, min_seconds=10.0, max_intervals=20, threads=None):
    """The oracle's OpenMP bulk interval on a 64^3 box at the same density."""
    from oracle import oracle as O

    nt = threads or os.cpu_count() or 1
    O.set_threads(nt)
    N = RHO * L_sample ** 3
    c = O.Cells([L_sample] * 3)
    p = O.Particles(N, 1)
    r = np.random.default_rng(SEED)
    p.pos[:] = r.random((N, 3)) * L_sample
    p.vel[:] = r.normal(size=(N, 3)) * np.sqrt(T_INIT)
    p.species[:] = 1
    c.origin = O.random_shift_values(SEED, 0)
    p.sort(c)
    O.bulk_run(p, c, 1, TAU, SEED, 1)  # warm-up interval
    t0 = time.perf_counter()
    n = 0
    while n < max_intervals and (time.perf_counter() - t0) < min_seconds:
        O.bulk_run(p, c, 1, TAU, SEED, 3 + 2 * n)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": N * n / dt, "unit": "particle-steps/s", "cores": nt, "kind": "port", "cpu": cpu_model(),
            "host_threads": os.cpu_count(),
            "sample": f"{n} bulk intervals of the FP64 oracle (C, OpenMP) on {L_sample}^3 cells x rho {RHO} "
                      f"= {N} particles ({n * N} particle-steps, {dt:.1f} s)"}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world == 1:
        return None, rank, local, world
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return dist, rank, local, world


def max_over_ranks(dist, x):
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, x):
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def run_ours(args):
    dist, rank, local, world = dist_init()
    import rmpcdmd_b200 as rm

    rm.set_device(local)
    L = args.L
    N = RHO * L ** 3
    peak, peak_kind = peaks()
    out = {"metric": "solvent particle-steps/s (bulk SRD fluid, 128^3 cells, rho=10; one step = one MPCD "
                     "interval: collide + stream + shift + sort)",
           "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded uniform positions, Maxwell velocities kT=1/3)"}
    results = {}
    tuned = {}
    for precision in (32, 64):
        if args.shapes:
            # a fixed tile shape (for profilers: no autotuning launches)
            rm.set_bulk_shape(precision, args.shapes[0 if precision == 32 else 1])
            tuned[f"fp{precision}"] = {"shape": rm.bulk_shape(precision), "shapes": rm.bulk_shapes(precision),
                                       "fixed": True}
        else:
            # the autotuner times every tile shape of the fused kernel on a
            # synthetic fluid of this box and keeps the fastest (same results)
            best, ms_shapes = rm.bulk_autotune([L, L, L], precision, TAU, 5)
            tuned[f"fp{precision}"] = {"shape": best, "shapes": rm.bulk_shapes(precision),
                                       "ms_per_5_intervals": [round(m, 3) for m in ms_shapes]}
        p, cells, rng = make_system(rm, L, precision)
        barrier(dist)
        with ClockSampler(local) as cs:
            ms, phases = timed_run(rm, p, cells, rng, args.steps, args.warmup)
        ms = max_over_ranks(dist, ms)
        rl = roofline(N, cells.N, precision, phases, peak, peak_kind)
        results[precision] = dict(ms=ms, phases=phases, roofline=rl, clocks=cs.summary(), p=p, cells=cells, rng=rng)
        if precision == 64:
            cbc_steps = max(1, min(3, args.steps))
            results[64]["cbc"] = (max_over_ranks(dist, call_by_call_ms(rm, p, cells, rng, cbc_steps)), cbc_steps)
        del p, cells
    r32, r64 = results[32], results[64]
    value = world * N * args.steps / (r32["ms"] * 1e-3)
    out.update(value=value, ms_per_step=r32["ms"] / args.steps)
    out["config"] = {"workload": f"bulk SRD fluid {L}^3 cells, rho={RHO}, N={N} particles per GPU, "
                                 f"alpha=pi/2, tau=1, FP32 form", "cells": [L, L, L], "particles_per_gpu": N,
                     "parallelism": f"replicas x{world} (independent systems, no collective)",
                     "l2": "inputs larger than L2 (>= 1 GB of particle arrays per copy); no flush"}
    out["roofline"] = r32["roofline"]
    out["interval_roofline"] = {}
    for prec, r in ((32, r32), (64, r64)):
        alg = N * INTERVAL_BYTES_PER_PARTICLE[prec] + r32["cells"].N * INTERVAL_BYTES_PER_SLOT
        ach = alg * args.steps / (r["ms"] * 1e-3) / 1e9
        out["interval_roofline"][f"fp{prec}"] = {
            "bound": "hbm", "achieved": round(ach, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
            "frac": round(ach / peak, 4), "algorithmic_bytes_per_interval": int(alg),
            "note": "minimum bytes of stream+sort+collide over the SoA particle state "
                    f"({INTERVAL_BYTES_PER_PARTICLE[prec]} B/particle + {INTERVAL_BYTES_PER_SLOT} B/slot) "
                    "over the whole device time of an interval"}
    out["autotune"] = tuned
    out["clocks"] = r32["clocks"]
    fp64_value = world * N * args.steps / (r64["ms"] * 1e-3)
    cbc_ms, cbc_steps = r64["cbc"]
    cbc_value = world * N * cbc_steps / (cbc_ms * 1e-3)
    out["fp64_plain"] = {"value": fp64_value, "ms_per_step": r64["ms"] / args.steps, "roofline": r64["roofline"],
                         "clocks": r64["clocks"], "fp32_over_fp64": value / fp64_value,
                         "call_by_call": {"value": cbc_value, "ms_per_step": cbc_ms / cbc_steps, "steps": cbc_steps,
                                          "path": "rmpcd_simple_mpcd_step, rmpcd_mpcd_stream_periodic, "
                                                  "rmpcd_cells_random_shift, rmpcd_particles_sort per interval "
                                                  "(device time)"},
                         "fp32_over_fp64_call_by_call": value / cbc_value}
    out["phases_ms"] = {k: round(v[0] * 1e3 / max(1, args.steps), 4)
                        for k, v in r32["phases"].items()}
    # kernels launched per step: fused interval, 2 scan kernels, placement;
    # plus, once per timed call, the record packing (1) and the FP32 end of
    # the run: entry positions of the records (1), segment sort (2), records
    # back from entry positions (1), gather into the API arrays (1)
    out["gpu_launches"] = 4 * args.steps + 6
    if not args.no_e2e:
        e2e_steps = max(1, min(args.e2e_steps, args.steps))
        path = ("rmpcd_particles_upload x6 (pinned host, reference (3,N) layout) -> rmpcd_bulk_run(1) "
                "-> rmpcd_particles_download x6")
        for prec, key in ((32, "e2e"), (64, "e2e_fp64")):
            r = results[prec]
            v, hb, db = e2e_run(rm, r["p"], r["cells"], r["rng"], e2e_steps)
            v = world * (1.0 / max_over_ranks(dist, 1.0 / v))
            out[key] = {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": hb, "d2h_bytes_per_step": db,
                        "steps": e2e_steps, "dtype": f"f{prec}", "path": path}
            r.pop("p", None)
            r.pop("cells", None)
    if not args.no_dimer:
        for r in (r32, r64):
            r.pop("p", None)
            r.pop("cells", None)
        out["dimer"] = run_dimer(rm, peak, peak_kind, local, dist, rank, world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_sample()
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    from oracle import oracle as O

    nt = os.cpu_count() or 1
    O.set_threads(nt)
    Ls = args.ref_L
    N = RHO * Ls ** 3
    c = O.Cells([Ls] * 3)
    p = O.Particles(N, 1)
    r = np.random.default_rng(SEED)
    p.pos[:] = r.random((N, 3)) * Ls
    p.vel[:] = r.normal(size=(N, 3)) * np.sqrt(T_INIT)
    p.species[:] = 1
    c.origin = O.random_shift_values(SEED, 0)
    p.sort(c)
    step = 1
    for _ in range(args.warmup):
        O.bulk_run(p, c, 1, TAU, SEED, step)
        step += 2
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.bulk_run(p, c, 1, TAU, SEED, step)
        step += 2
    dt = time.perf_counter() - t0
    v = N * args.steps / dt
    sample = (f"each step: one bulk interval of the FP64 CPU restatement (C, OpenMP, {nt} threads) on "
              f"{Ls}^3 cells x rho {RHO} = {N} particles, a bounded 1/{(L_DEFAULT // Ls) ** 3} sample of the "
              f"{L_DEFAULT}^3 workload (particle-steps/s is per-particle intensive)")
    out = {"impl": "reference", "metric": "solvent particle-steps/s (bulk SRD fluid, 128^3 cells, rho=10; one step "
                                          "= one MPCD interval: collide + stream + shift + sort)",
           "value": v, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded uniform positions, Gaussian velocities kT=1/3)",
           "config": {"workload": f"bulk SRD fluid {Ls}^3-cell sample of the {L_DEFAULT}^3 box, rho={RHO}",
                      "cells": [Ls] * 3, "particles": N},
           "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": nt, "kind": "port", "sample": sample,
                            "cpu": cpu_model(), "host_threads": os.cpu_count()},
           "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "note": "the reference (Fortran 2008 + OpenMP) cannot be built here: no Fortran compiler and empty "
                   "dependency submodules; this arm times the C restatement of its loop"}
    print(json.dumps(out))


def cpu_table(args):
    """The CPU restatement (oracle, C + OpenMP) timed on bounded samples of
    the five configurations, with all host threads and with one, for the
    baseline table: particle-steps/s (MD steps for the colloid programs,
    MPCD intervals for the bulk fluid).  Prints one JSON line."""
    from oracle import oracle as O
    from oracle.programs import NColloidsPBC as ONC
    from oracle.programs import SingleDimerPBC as OD

    nt = os.cpu_count() or 1

    def dimer_rate(L, n_md, seed=1):
        o = OD(L=L, rho=RHO, N_MD=DIMER_N_MD, seed=seed, list_capacity=DIMER_LIST_CAPACITY)
        t0 = time.perf_counter()
        for _ in range(n_md):
            o.md_step()
        t_md = (time.perf_counter() - t0) / n_md
        t0 = time.perf_counter()
        o.mpcd()
        t_mpcd = time.perf_counter() - t0
        return o.N, t_md + t_mpcd / DIMER_N_MD

    out = {"impl": "reference", "cpu_table": {}, "threads_all": nt}
    for threads in (nt, 1):
        O.set_threads(threads)
        row = {}
        N, t = dimer_rate((32, 32, 32), 20)
        row["single_dimer_32"] = {"value": N / t, "sample": "20 MD steps + 1 MPCD part, per MD step"}
        Ls = 64
        N = RHO * Ls ** 3
        c = O.Cells([Ls] * 3)
        p = O.Particles(N, 1)
        r = np.random.default_rng(SEED)
        p.pos[:] = r.random((N, 3)) * Ls
        p.vel[:] = r.normal(size=(N, 3)) * np.sqrt(T_INIT)
        p.species[:] = 1
        c.origin = O.random_shift_values(SEED, 0)
        p.sort(c)
        O.bulk_run(p, c, 1, TAU, SEED, 1)
        t0 = time.perf_counter()
        O.bulk_run(p, c, 3, TAU, SEED, 3)
        row["bulk_128"] = {"value": N * 3 / (time.perf_counter() - t0),
                           "sample": "3 intervals on 64^3 cells (per-particle intensive)"}
        del p, c
        N, t = dimer_rate((96, 96, 96), 3 if threads > 1 else 1)
        row["single_dimer_96"] = {"value": N / t, "sample": "1-3 MD steps + 1 MPCD part, per MD step"}
        boxes = dimer_boxes_batched()[:8]
        tot_n = tot_t = 0.0
        for k, L in enumerate(boxes):
            n, t = dimer_rate(L, 5, seed=k + 1)
            tot_n += n
            tot_t += t
        row["batched_512"] = {"value": tot_n / tot_t,
                              "sample": "replicas 0-7 of the 512 (5 MD steps + 1 MPCD part each), run one "
                                        "after the other; the 512 scale with their particle count"}
        o = ONC(L=(128, 128, 128), rho=RHO, N_MD=DIMER_N_MD, N_colloids=200, seed=SEED, volume_correction=False)
        n_md = 3 if threads > 1 else 1
        t0 = time.perf_counter()
        for _ in range(n_md):
            o.md_step()
        t_md = (time.perf_counter() - t0) / n_md
        t0 = time.perf_counter()
        o._catch_up_and_sort()
        t_sort = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.simple_mpcd_step(o.s, o.cells, o.seed, 99, thermostat=True, T=o.T_init, hydro=True)
        t_srd = time.perf_counter() - t0
        row["n_colloids_128"] = {"value": o.N / (t_md + (5 * t_sort + t_srd) / DIMER_N_MD),
                                 "sample": "MD steps + one catch-up/sort and one collision, per MD step with "
                                           "5 sorts per 100-step interval (the rate the GPU runs see)"}
        del o
        out["cpu_table"][f"threads_{threads}"] = row
    print(json.dumps(out))


def profile_dimer(args):
    """A fixed engine workload for profilers: R replicas of the batched
    dimer (cubic sides drawn from {16..48}), FP32 solvent, one interval with
    the kernels launched one by one (profilers cannot see inside a graph that
    holds conditional nodes).  Prints nothing but a line when done."""
    import rmpcdmd_b200 as rm
    from rmpcdmd_b200.programs import DimerBatch, SingleDimerPBC

    boxes = dimer_boxes_batched()[: args.profile_dimer]
    if args.profile_box:
        boxes = [(args.profile_box,) * 3] * args.profile_dimer
    ds = [SingleDimerPBC(L=L, rho=RHO, N_MD=DIMER_N_MD, seed=k + 1, list_capacity=DIMER_LIST_CAPACITY,
                         precision=32) for k, L in enumerate(boxes)]
    b = DimerBatch(ds, use_graph=False)
    b.run(1)
    rm.synchronize()
    print(f"profile_dimer: {len(ds)} replicas, {b.n_solvent} particles, 1 interval")


def profile_ncolloids(args):
    """A fixed n_colloids_pbc workload for profilers: 128^3, rho = 10,
    args.profile_ncolloids colloids, FP32 solvent, one thermostatted interval
    of the native loop (rmpcd_ncolloids_run) after one warm-up interval, with
    its MD steps launched one by one (kernel profilers do not see into the
    conditional nodes of the replayed graphs)."""
    import rmpcdmd_b200 as rm
    from rmpcdmd_b200._capi import call
    from rmpcdmd_b200.programs import NColloidsPBC

    call("rmpcd_ncolloids_set_graphs", 0)

    g = NColloidsPBC(L=(128, 128, 128), rho=RHO, N_MD=DIMER_N_MD, N_colloids=args.profile_ncolloids, seed=SEED,
                     volume_correction=False, precision=32)
    g._native(1, True, [g.T_init], 10)
    g._native(1, True, [g.T_init], 10)
    rm.synchronize()
    print(f"profile_ncolloids: {args.profile_ncolloids} colloids, {g.N} particles, 2 intervals")


def kernel_timeline(run, label):
    """The kernels `run()` puts on the GPU, with their device start and end
    times as CUPTI records them (through torch.profiler), so concurrent and
    graph-launched kernels appear with their real, warm-cache durations:
    prints the span of the run, the time at least one kernel or copy was
    busy, and per kernel its launches, total and share of the busy time."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    torch.zeros(1, device="cuda")
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        run()
    rows = sorted((e.start_ns(), e.duration_ns(), e.name()) for e in prof.profiler.kineto_results.events()
                  if e.device_type().name == "CUDA")
    if not rows:
        print(f"{label}: no device activity recorded")
        return
    t0, busy = rows[0][0], 0
    s0, e0 = rows[0][0], rows[0][0] + rows[0][1]
    for st, d, _ in rows[1:]:
        if st > e0:
            busy += e0 - s0
            s0, e0 = st, st + d
        else:
            e0 = max(e0, st + d)
    busy += e0 - s0
    span = max(st + d for st, d, _ in rows) - t0
    agg = {}
    for _, d, n in rows:
        k = n.split("(")[0]
        c, t = agg.get(k, (0, 0))
        agg[k] = (c + 1, t + d)
    print(f"{label}: span {span / 1e3:.1f} us, busy {busy / 1e3:.1f} us, {len(rows)} kernels and copies")
    print("| kernel | launches | total us | share of busy |")
    print("|---|---|---|---|")
    for k, (c, t) in sorted(agg.items(), key=lambda kv: -kv[1][1]):
        print(f"| {k} | {c} | {t / 1e3:.1f} | {100 * t / busy:.1f} % |")


def timeline(args):
    """One interval of n_colloids_pbc (128^3, 200 colloids, thermostatted,
    after two warm-up intervals) or of one 32^3 single dimer (batched engine,
    graph on, after autotuning and warm-up), FP32 solvent, through
    kernel_timeline."""
    import rmpcdmd_b200 as rm

    if args.timeline == "ncolloids":
        from rmpcdmd_b200.programs import NColloidsPBC

        g = NColloidsPBC(L=(128, 128, 128), rho=RHO, N_MD=DIMER_N_MD, N_colloids=200, seed=SEED,
                         volume_correction=False, precision=32)
        g.thermalise(1)
        g.thermalise(1)
        rm.synchronize()

        def run():
            g.thermalise(1)
            rm.synchronize()

        kernel_timeline(run, "n_colloids 128^3, 200 colloids, FP32, one thermostatted interval (100 MD steps)")
    else:
        from rmpcdmd_b200.programs import DimerBatch, SingleDimerPBC

        d = [SingleDimerPBC(L=(32, 32, 32), rho=RHO, N_MD=DIMER_N_MD, seed=SEED, list_capacity=DIMER_LIST_CAPACITY,
                            precision=32)]
        b = DimerBatch(d, use_graph=True)
        b.autotune(1)
        b.run(2)
        rm.synchronize()

        def run():
            b.run(1)
            rm.synchronize()

        kernel_timeline(run, "single dimer 32^3, FP32 solvent, engine with its interval graph, one interval")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--L", type=int, default=L_DEFAULT)
    ap.add_argument("--ref-L", type=int, default=64)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-dimer", action="store_true", help="skip the single-dimer engine configurations")
    ap.add_argument("--shapes", type=lambda t: [int(x) for x in t.split(",")], default=None, metavar="S32,S64",
                    help="use these fused-interval tile shapes instead of autotuning (for profilers)")
    ap.add_argument("--profile-ncolloids", type=int, default=0, metavar="C",
                    help="only run two intervals of n_colloids_pbc with C colloids at 128^3, for profilers")
    ap.add_argument("--profile-box", type=int, default=0, metavar="L",
                    help="with --profile-dimer: every replica in an L^3 box instead of the drawn sides")
    ap.add_argument("--cpu-table", action="store_true",
                    help="only time the CPU restatement on samples of every configuration (baseline table)")
    ap.add_argument("--timeline", choices=["ncolloids", "dimer32"], default=None,
                    help="only print the kernel timeline of one interval of the named workload")
    ap.add_argument("--profile-dimer", type=int, default=0, metavar="R",
                    help="only run one interval of R batched dimer replicas (graph off), for profilers")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.timeline:
        timeline(args)
    elif args.cpu_table:
        cpu_table(args)
    elif args.profile_dimer:
        profile_dimer(args)
    elif args.profile_ncolloids:
        profile_ncolloids(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
