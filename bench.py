#!/usr/bin/env python
"""Throughput of the MD hot path on B200, one JSON line on rank 0.

Workload (the 1M-molecule LJ configuration): FCC 64x64x64 unit cells
(1,048,576 molecules), density 0.8442, T 0.722 (seeded Maxwell-Boltzmann),
LJ 12-6 truncated and shifted at rc 2.5, skin 0.3, dt 0.005, NVE velocity
Verlet with the reference's vmax rebuild criterion and tplot 100.  A "step"
is one MD timestep of that system.  `value` is the precision form (FP32 pair
forces, FP64 positions / velocities / sums); the plain FP64 drop-in is
reported beside it.  Inputs are larger than L2: the neighbour list alone is
~400 MB, so every step streams it from HBM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 (torchrun) every rank advances its own replica of the system
(replicas only: the hot path has no cross-replica exchange) and the timing is
the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "molecule-steps/s (1M LJ), batched replica agg vs plain on same B200; p50/p99 latency"
UNIT = "molecule-steps/s"
NUNITS = (64, 64, 64)
DENSITY, TEMP, RC, SKIN, DT, TPLOT = 0.8442, 0.722, 2.5, 0.3, 0.005, 100
SEED = 0x466D6F6C + 1


class Ranks:
    """Rank plumbing of replica runs: a barrier, and the MAX over ranks of a
    time, so that a whole-job value is the units all ranks processed divided
    by the slowest rank's time.  `device` None means CPU tensors (gloo)."""

    def __init__(self, dist=None, device=None):
        self.dist = dist
        self.device = device

    @property
    def world(self):
        return self.dist.get_world_size() if self.dist is not None else 1

    def barrier(self):
        import torch
        if self.dist is not None:
            self.dist.barrier()
        if self.device is not None:
            torch.cuda.synchronize(self.device)

    def max(self, x):
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64,
                         device=f"cuda:{self.device}" if self.device is not None else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def whole_job(self, units_per_rank, seconds):
        """Weak-scaling aggregate: world * units / max-over-ranks seconds."""
        return self.world * units_per_rank / self.max(seconds)


def alg_bytes_per_molecule_step(rn=RC + SKIN, rho=DENSITY):
    """192 B of FP64 r, v, a read and written once, plus 4-byte half-list
    indices: n_h = (2/3) pi r_n^3 rho."""
    n_h = (2.0 / 3.0) * np.pi * rn ** 3 * rho
    return 192.0 + 4.0 * n_h


def workload_name():
    return (f"LJ fluid, FCC {NUNITS[0]}x{NUNITS[1]}x{NUNITS[2]} units ({4 * int(np.prod(NUNITS)):,} molecules), "
            f"rho {DENSITY}, T {TEMP}, rc {RC} shifted, skin {SKIN}, dt {DT}, NVE velocity Verlet")


def make_state():
    from flowmol_b200 import lattice
    return lattice.lj_fluid(NUNITS, DENSITY, TEMP, SEED)


def read_peaks():
    try:
        pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """Per-launch DRAM bytes of the force kernel from the committed ncu
    summary (None when no capture has been summarised yet)."""
    p = os.path.join(ROOT, "profiles", "force_kernel_lj1m.json")
    try:
        return json.load(open(p)).get("dram_bytes_per_launch_full_size")
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        # raw samples; the JSON line carries their summary
        out_dir = os.environ.get("FM_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out_dir, f"clocks_bench_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, smax, reasons = [], [], set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); smax.append(float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_form(api, torch, r, v, dom, precision, steps, warmup, dev, timing_pass=True, tpm=0, force_path=0):
    """Device-resident throughput of one precision form."""
    stream = torch.cuda.Stream(device=dev)
    p = api.make_params(len(r), dom, RC, (SKIN,) * 3, DT, TPLOT, density=DENSITY, precision=precision,
                        threads_per_molecule=tpm, force_path=force_path)
    s = api.MDSystem(p, stream=stream)
    s.upload(r, v)
    s.setup()
    s.simulation_md(warmup, blocking=True)
    s.records()
    torch.cuda.synchronize(dev)
    launches0 = s.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    out = {}
    with Clocks(dev) as clk:
        e0.record(stream)
        s.simulation_md(steps, blocking=False)
        e1.record(stream)
        e1.synchronize()
    s.sync()
    out["ms"] = e0.elapsed_time(e1)
    out["clocks"] = clk.summary()
    out["launches"] = s.launch_count() - launches0
    out["rebuilds"] = s.counters()["rebuilds"]
    if timing_pass:
        s.force_kernel_timing(True)
        s.simulation_md(steps, blocking=True)
        ms, nl = s.force_kernel_time()
        s.force_kernel_timing(False)
        out["force_ms_avg"] = ms / max(nl, 1)
        out["force_launches"] = nl
    out["records"] = s.records()
    out["capacity"] = s.counters()["nlist_capacity"]
    out["tpm"] = s.threads_per_molecule
    out["force_path"] = "tiles" if s.force_path()[0] == api.FORCE_PATH_TILES else "gather"
    s.close()
    return out


def run_e2e(api, torch, r, v, dom, precision, steps, dev, tpm=0, force_path=0):
    """Through the public API with host buffers: pinned upload, setup, steps,
    download of the final state and the records, all inside the timed region."""
    n = len(r)
    rh = torch.from_numpy(np.ascontiguousarray(r)).pin_memory()
    vh = torch.from_numpy(np.ascontiguousarray(v)).pin_memory()
    ro = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    vo = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    ao = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    p = api.make_params(n, dom, RC, (SKIN,) * 3, DT, TPLOT, density=DENSITY, precision=precision,
                        threads_per_molecule=tpm, force_path=force_path)
    s = api.MDSystem(p)
    torch.cuda.synchronize(dev)
    import ctypes as C
    dp = lambda t: C.cast(t.data_ptr(), C.POINTER(C.c_double))  # noqa: E731
    t0 = time.perf_counter()
    api.check(api.lib().fm_upload_state(s.h, n, dp(rh), dp(vh), None, None))
    s.setup()
    s.simulation_md(steps, blocking=True)
    api.check(api.lib().fm_download_state(s.h, dp(ro), dp(vo), dp(ao), None))
    recs = s.records()
    t1 = time.perf_counter()
    s.close()
    h2d = 2 * n * 3 * 8
    d2h = 3 * n * 3 * 8 + len(recs) * 80
    return {"value": n * steps / (t1 - t0), "unit": UNIT, "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": d2h / steps, "steps": steps, "seconds": t1 - t0}


def run_drift(api, r, v, dom, precision, nsteps=10000, tplot=1000):
    """NVE energy drift of the 1M fluid over nsteps (records every tplot):
    relative change of the total energy per molecule from the first record."""
    p = api.make_params(len(r), dom, RC, (SKIN,) * 3, DT, tplot, density=DENSITY, precision=precision)
    s = api.MDSystem(p)
    s.upload(r, v)
    s.setup()
    s.simulation_md(nsteps, blocking=True)
    recs = s.records()
    s.close()
    e = np.array([x["totenergy"] for x in recs])
    return {"steps": nsteps, "records": len(e), "totenergy_first": float(e[0]), "totenergy_last": float(e[-1]),
            "rel_drift_end": float((e[-1] - e[0]) / abs(e[0])),
            "rel_drift_max": float(np.abs(e - e[0]).max() / abs(e[0]))}


FENE_CHAINS, FENE_BEADS, FENE_DENSITY, FENE_K, FENE_R0 = 32768, 8, 0.85, 30.0, 1.5


def run_fene(api, torch, dev, steps, warmup):
    """The FENE bead-spring melt: 32768 chains of 8 beads (262,144 beads) at
    density 0.85, WCA + FENE (k 30, R0 1.5, rneighbr = R0), FP32 pair forces
    with FP64 bonds and integration, timed with CUDA events on the handle's
    stream; energy drift from the records of the timed steps."""
    from flowmol_b200 import polymer
    r, v, ch, sub, _fy, bf, dom = polymer.fene_melt(FENE_CHAINS, FENE_BEADS, FENE_DENSITY)
    stream = torch.cuda.Stream(device=dev)
    wca = 2.0 ** (1.0 / 6.0)
    p = api.make_params(len(r), dom, wca, (SKIN,) * 3, DT, TPLOT, density=FENE_DENSITY,
                        precision=api.PRECISION_FP32, potential_flag=1, k_c=FENE_K, R_0=FENE_R0)
    s = api.MDSystem(p, stream=stream)
    s.upload(r, v)
    s.upload_monomers(ch, sub, bf)
    s.setup()
    nbonds = len(s.bonds()[0])
    s.simulation_md(warmup, blocking=True)
    s.records()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.simulation_md(steps, blocking=False)
    e1.record(stream)
    e1.synchronize()
    s.sync()
    ms = e0.elapsed_time(e1)
    recs = s.records()
    rebuilds = s.counters()["rebuilds"]
    s.close()
    e = np.array([x["totenergy"] for x in recs])
    return {"value": len(r) * steps / (ms * 1e-3), "unit": UNIT, "beads": len(r), "steps": steps,
            "ms_per_step": ms / steps, "bond_entries": nbonds, "rebuilds": rebuilds,
            "rel_drift_end": float((e[-1] - e[0]) / abs(e[0])) if len(e) > 1 else None,
            "drift_note": "total energy as the reference reports it: its FENE_energy has the opposite sign "
                          "of the potential its FENE force derives from, so this sum is not conserved",
            "workload": f"FENE melt: {FENE_CHAINS} chains x {FENE_BEADS} beads, rho {FENE_DENSITY}, WCA + FENE "
                        f"k {FENE_K} R0 {FENE_R0} (rneighbr = R0), dt {DT}, VV, FP32 pair forces, FP64 bonds; "
                        "start: self-avoiding walks on FCC sites"}


def batch_replicas(nrep=256, seed=0x466D6F6C + 4):
    """The batched-ensemble configuration: replica sizes log-uniform in
    500-32000 molecules (rounded to 4 n^3 FCC), densities U(0.3, 0.9),
    temperatures U(0.7, 1.5), rc 2.5; boxes below 3 cells run all pairs."""
    from flowmol_b200 import lattice
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for k in range(nrep):
        n_target = float(np.exp(rng.uniform(np.log(500.0), np.log(32000.0))))
        m = max(2, int(round((n_target / 4.0) ** (1.0 / 3.0))))
        rho = float(rng.uniform(0.3, 0.9))
        T = float(rng.uniform(0.7, 1.5))
        r, v, dom = lattice.lj_fluid([m, m, m], rho, T, seed + 1000 + k)
        fl = 0 if min(np.floor(dom / (RC + SKIN))) < 3 else 3
        out.append((r, v, dom, rho, fl))
    return out


def run_batched(api, torch, dev, nsteps, nrep=256):
    """All replicas in one engine (admission and setup inside the timed
    region; the ticks loop on the device in one graph launch, until the
    replicas are done) against the plain single-system form run one
    replica at a time.  The plain form is measured per replica as its setup
    (upload, binning, list, first forces) plus plain_steps steps timed apart
    with CUDA events, and projected to the same nsteps the batch runs:
    t = t_setup + nsteps * t_step.  Both sides therefore pay one setup per
    replica over the same number of steps; the steps-only plain rate is
    reported beside it."""
    reps = batch_replicas(nrep)
    tot = sum(len(x[0]) for x in reps)
    e = api.Engine(max_molecules=tot + 1024, max_cells=2_000_000, max_list_entries=(tot + 1024) * 160,
                   max_slots=nrep, precision=api.PRECISION_FP32, ticks_per_chunk=4096, keep_states=False)
    for r, v, dom, rho, fl in reps:
        e.submit(api.make_job(len(r), dom, RC, nsteps, density=rho, tplot=TPLOT, force_list=fl), r, v)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    e.run()
    t_batch = time.perf_counter() - t0
    res = e.results()
    c = e.counters()
    tune_bb = e.tuning()[1]
    bad = [x for x in res if x["status"] != 0]
    e.close()
    plain_steps = min(nsteps, 200)
    t_setup = t_steps = 0.0  # summed over the replicas; t_steps for plain_steps each
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.Stream(device=dev)
    for r, v, dom, rho, fl in reps:
        p = api.make_params(len(r), dom, RC, (SKIN,) * 3, DT, TPLOT, density=rho, force_list=fl,
                            precision=api.PRECISION_FP32)
        s = api.MDSystem(p, stream=stream)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        s.upload(r, v)
        s.setup()
        s.sync()
        t_setup += time.perf_counter() - t0
        ev0.record(stream)
        s.simulation_md(plain_steps, blocking=False)
        ev1.record(stream)
        ev1.synchronize()
        s.sync()
        t_steps += 1e-3 * ev0.elapsed_time(ev1)
        s.close()
    v_batch = tot * nsteps / t_batch
    v_plain = tot * nsteps / (t_setup + t_steps * nsteps / plain_steps)
    v_plain_steps = tot * plain_steps / t_steps
    return {"value": v_batch, "unit": UNIT, "replicas": nrep, "molecules": tot, "steps_each": nsteps,
            "seconds": t_batch, "plain_one_at_a_time": v_plain, "plain_steps_only": v_plain_steps,
            "plain_setup_seconds": t_setup, "plain_steps_timed_each": plain_steps,
            "ratio_vs_plain": v_batch / v_plain, "ratio_vs_plain_steps_only": v_batch / v_plain_steps,
            "failed": len(bad), "threads_per_molecule": c["threads_per_molecule"],
            "list_build_blocks_below": tune_bb, "gpu_launches": c["launches"],
            "workload": "256 periodic LJ replicas, N log-uniform 500-32000 (4 n^3 FCC), rho U(0.3,0.9), "
                        "T U(0.7,1.5), rc 2.5, skin 0.3, dt 0.005, VV, FP32 forces; boxes < 3 cells: all pairs"}


# Poisson arrivals at this fraction of the service rate probed with 48 jobs resident at once.
ARRIVAL_FRACTION = 0.7


def run_served(api, torch, dev, njobs, seed=0x466D6F6C + 5):
    """Poisson-arriving Couette jobs through the engine's admission loop.
    Job sizes log-uniform in 256-65536 molecules, 200-2000 steps, wall speed
    U(0.5, 2.0); the arrival rate is ARRIVAL_FRACTION x the service rate
    measured with 48 jobs resident at once.  Served jobs overlap less than the
    probe's, so each tick carries fewer molecules and its fixed launch cost
    weighs more: 0.5x left the engine ~77% busy, 0.55x ~79%, 0.6x 80-81%,
    0.65x ~82% and 0.7x ~83% (`gpu_busy_frac`: wall time inside graphs of
    ticks / total), each with a bounded queue (p50 ~0.2 s, p99 0.5-0.7 s).  Latency = finish time -
    scheduled arrival time."""
    from flowmol_b200 import couette
    rng = np.random.Generator(np.random.Philox(seed))

    def make(k, rng):
        n_target = float(np.exp(rng.uniform(np.log(256.0), np.log(65536.0))))
        nu = couette.nunits_for(n_target)
        steps = int(rng.integers(200, 2001))
        speed = float(rng.uniform(0.5, 2.0))
        r, v, tag, rt, sv, dom = couette.couette_job(nu, 0.8, 1.0, speed, seed + 77 + k)
        job = api.make_job(len(r), dom, couette.WCA_RC, steps, tplot=10, integration_algorithm=0, ensemble=6,
                           pressure_outflag=1, nthermo=2, thermostat_temperature=(1.0, 1.0),
                           teth=(0.0, 5000.0, 5.0e6))
        return (job, r, v, tag, rt, sv)

    def new_engine():
        cap = 4_000_000
        return api.Engine(max_molecules=cap, max_cells=4_000_000, max_list_entries=cap * 48, max_slots=512,
                          precision=api.PRECISION_FP32, ticks_per_chunk=20, keep_states=False)

    # service-rate probe: 48 jobs of the same distribution submitted at once
    prng = np.random.Generator(np.random.Philox(seed + 1))
    probe = [make(100000 + k, prng) for k in range(48)]
    e = new_engine()
    for j in probe:
        e.submit(*j)
    t0 = time.perf_counter()
    e.run()
    rate_work = sum(j[0].np * j[0].nsteps for j in probe) / (time.perf_counter() - t0)
    e.close()
    jobs = []
    for k in range(njobs):
        jobs.append(make(k, rng))
    work = sum(j[0].np * j[0].nsteps for j in jobs)
    e = new_engine()
    arrivals = np.cumsum(rng.exponential(1.0, njobs))
    mean_work = work / njobs
    lam = ARRIVAL_FRACTION * rate_work / mean_work
    t_arr = arrivals / lam
    t0 = time.monotonic()
    nxt = 0
    done = []
    busy = 0.0
    while len(done) < njobs:
        now = time.monotonic() - t0
        while nxt < njobs and t_arr[nxt] <= now:
            e.submit(*jobs[nxt])
            nxt += 1
        ticks0 = e.counters()["ticks"]
        ta = time.monotonic()
        res, q = e.step_chunk()
        if e.counters()["ticks"] > ticks0:
            busy += time.monotonic() - ta
        done += e.results()
        if res == 0 and q == 0 and nxt < njobs:
            time.sleep(max(0.0, min(0.01, t_arr[nxt] - (time.monotonic() - t0))))
    t_total = time.monotonic() - t0
    lat = np.array([d["finish_time"] - (t0 + t_arr[d["job_id"] - 1]) for d in done])
    bad = [d for d in done if d["status"] != 0]
    c = e.counters()
    tune_bb = e.tuning()[1]
    e.close()
    # the same kind of jobs run one at a time (an engine with one slot: a job
    # is admitted when the previous one has finished), on a sample of 64
    sample = [make(200000 + k, np.random.Generator(np.random.Philox(seed + 2 + k))) for k in range(64)]
    e1 = api.Engine(max_molecules=200_000, max_cells=400_000, max_list_entries=200_000 * 48, max_slots=1,
                    precision=api.PRECISION_FP32, ticks_per_chunk=20, keep_states=False)
    ts = time.perf_counter()
    for j in sample:
        e1.submit(*j)
        e1.run()
        e1.results()
    t_one = time.perf_counter() - ts
    e1.close()
    v_one = sum(j[0].np * j[0].nsteps for j in sample) / t_one
    return {"value": work / t_total, "unit": UNIT, "jobs": njobs, "molecule_steps": work, "seconds": t_total,
            "one_at_a_time": v_one, "one_at_a_time_jobs": len(sample), "ratio_vs_one_at_a_time": work / t_total / v_one,
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "arrival_rate_per_s": lam, "probe_service_rate": rate_work, "gpu_busy_frac": busy / t_total,
            "failed": len(bad), "threads_per_molecule": c["threads_per_molecule"],
            "list_build_blocks_below": tune_bb,
            "workload": "Couette channels (WCA fluid between tethered, thermostatted FCC walls, top wall "
                        "sliding U(0.5,2.0)), N log-uniform 256-65536, 200-2000 steps, leap-frog + tags, "
                        "time-averaged virial pressure tensor, FP32 forces"}


def _oracle_replica(nsteps, barrier, out):
    """One host core: the FP64 oracle on its own copy of the 1M system; setup
    excluded, `nsteps` velocity-Verlet steps timed after every core is ready."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    r, v, dom = make_state()
    o = O.Oracle(r, v, dom, RC, (SKIN,) * 3, DT, TPLOT, density=DENSITY)
    o.setup()
    barrier.wait()
    t0 = time.perf_counter()
    o.run_vv(nsteps)
    t1 = time.perf_counter()
    out.put((len(r) * nsteps, t0, t1, o.rebuild_count))


def host_cores():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def cpu_baseline(nsteps=16, cores=None):
    """The FP64 oracle (C restatement of the reference's routines; scalar, one
    thread per process) on every host core at once: one replica of the 1M
    system per core, as the reference runs one MPI rank per core.  Value =
    all molecule-steps / (last finish - first start).  Processes are spawned
    (never forked from a process that holds a CUDA context)."""
    import multiprocessing as mp
    cores = cores or host_cores()
    ctx = mp.get_context("spawn")
    barrier, out = ctx.Barrier(cores), ctx.Queue()
    procs = [ctx.Process(target=_oracle_replica, args=(nsteps, barrier, out)) for _ in range(cores)]
    for q in procs:
        q.start()
    res = [out.get() for _ in procs]
    for q in procs:
        q.join()
    work = sum(x[0] for x in res)
    span = max(x[2] for x in res) - min(x[1] for x in res)
    per_core = statistics.median(x[0] / (x[2] - x[1]) for x in res)
    return {"value": work / span, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{cores} concurrent replicas (one per host core) of the {res[0][0] // nsteps:,}-molecule "
                      f"system x {nsteps} velocity-Verlet steps from the FCC start ({res[0][3]} list rebuilds "
                      f"inside each; setup excluded); median single-core rate {per_core:.3g} {UNIT}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--batch-replicas", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=2000)
    ap.add_argument("--serve-jobs", type=int, default=4096)
    ap.add_argument("--no-forms", action="store_true", help="skip the FENE, batched and served forms")
    ap.add_argument("--fene-steps", type=int, default=5000)
    ap.add_argument("--drift-steps", type=int, default=10000,
                    help="NVE drift run of the 1M fluid per precision form (0: skip)")
    ap.add_argument("--tpm", type=int, default=0,
                    help="force-kernel lanes per molecule (0: the autotuner's choice)")
    ap.add_argument("--force-path", type=int, default=0, choices=[0, 1, 2],
                    help="force kernel of the 1M forms: 0 automatic, 1 one gather per list entry, 2 tiles")
    ap.add_argument("--profile-case", choices=["fp32", "fp64", "batched", "fene", "served"], default=None,
                    help="profiling workload, no timing: setup + 10 fused steps of the 1M system "
                         "(fp32, fp64) or of the FENE melt (fene), the batched replicas for "
                         "--batch-steps steps, or --serve-jobs served jobs")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        steps = max(2, min(args.steps, 16))
        cb = cpu_baseline(steps)
        n = NUNITS[0] * NUNITS[1] * NUNITS[2] * 4
        line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "impl": "reference",
                "n_gpus": args.gpus, "steps": steps, "warmup": 0,
                # the CPU sample is bounded (2-16 velocity-Verlet steps of the full
                # 1M system on every core) so that the arm ends within minutes
                "steps_requested": args.steps, "warmup_requested": args.warmup,
                "ms_per_step": 1e3 * n / cb["value"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": workload_name(), "molecules": n, "form": "oracle FP64 CPU restatement"},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    from flowmol_b200 import api, build as fb
    fb.build()
    dev = local
    torch.cuda.set_device(dev)
    if args.profile_case == "batched":
        reps = batch_replicas(args.batch_replicas)
        tot = sum(len(x[0]) for x in reps)
        e = api.Engine(max_molecules=tot + 1024, max_cells=2_000_000, max_list_entries=(tot + 1024) * 160,
                       max_slots=len(reps), precision=api.PRECISION_FP32, ticks_per_chunk=50, keep_states=False,
                       threads_per_molecule=args.tpm)
        for r, v, dom, rho, fl in reps:
            e.submit(api.make_job(len(r), dom, RC, args.batch_steps, density=rho, tplot=TPLOT, force_list=fl), r, v)
        e.run()
        bad = [x for x in e.results() if x["status"] != 0]
        print(json.dumps({"profile_case": "batched", "molecules": tot, "failed": len(bad), **e.counters()}))
        e.close()
        return
    if args.profile_case == "served":
        out = run_served(api, torch, dev, args.serve_jobs)
        print(json.dumps({"profile_case": "served", "jobs": out["jobs"], "failed": out["failed"]}))
        return
    if args.profile_case == "fene":
        from flowmol_b200 import polymer
        r, v, ch, sub, _fy, bf, dom = polymer.fene_melt(FENE_CHAINS, FENE_BEADS, FENE_DENSITY)
        p = api.make_params(len(r), dom, 2.0 ** (1.0 / 6.0), (SKIN,) * 3, DT, TPLOT, density=FENE_DENSITY,
                            precision=api.PRECISION_FP32, potential_flag=1, k_c=FENE_K, R_0=FENE_R0,
                            threads_per_molecule=args.tpm)
        s = api.MDSystem(p)
        s.upload(r, v)
        s.upload_monomers(ch, sub, bf)
        s.setup()
        s.simulation_md(10, blocking=True)
        print(json.dumps({"profile_case": "fene", "beads": len(r), **s.counters()}))
        s.close()
        return
    if args.profile_case:
        r, v, dom = make_state()
        prec = api.PRECISION_FP32 if args.profile_case == "fp32" else api.PRECISION_FP64
        p = api.make_params(len(r), dom, RC, (SKIN,) * 3, DT, TPLOT, density=DENSITY, precision=prec,
                            threads_per_molecule=args.tpm, force_path=args.force_path)
        s = api.MDSystem(p)
        s.upload(r, v)
        s.setup()
        s.simulation_md(10, blocking=True)
        print(json.dumps({"profile_case": args.profile_case, "molecules": len(r), **s.counters()}))
        s.close()
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", dev))
    r, v, dom = make_state()
    n = len(r)
    ranks = Ranks(dist, dev)
    barrier = ranks.barrier
    max_over_ranks = ranks.max

    barrier()
    f32 = run_form(api, torch, r, v, dom, api.PRECISION_FP32, args.steps, args.warmup, dev, tpm=args.tpm,
                   force_path=args.force_path)
    ms32 = max_over_ranks(f32["ms"])
    barrier()
    f64 = run_form(api, torch, r, v, dom, api.PRECISION_FP64, args.steps, args.warmup, dev, tpm=args.tpm,
                   force_path=args.force_path)
    ms64 = max_over_ranks(f64["ms"])
    barrier()
    e2e = None if args.no_e2e else run_e2e(api, torch, r, v, dom, api.PRECISION_FP32, args.steps, dev,
                                           tpm=args.tpm, force_path=args.force_path)
    if e2e is not None:
        e2e["value"] = world * n * args.steps / max_over_ranks(e2e["seconds"])
    barrier()
    drift = None
    if args.drift_steps > 0:
        drift = {"fp32_forces": run_drift(api, r, v, dom, api.PRECISION_FP32, args.drift_steps),
                 "fp64_plain": run_drift(api, r, v, dom, api.PRECISION_FP64, args.drift_steps)}
    barrier()
    batched = served = fene = None
    if not args.no_forms:
        fene = run_fene(api, torch, dev, args.fene_steps, args.warmup)
        fene["value"] = world * fene["value"] * fene["ms_per_step"] / max_over_ranks(fene["ms_per_step"])
        barrier()
        batched = run_batched(api, torch, dev, args.batch_steps, args.batch_replicas)
        batched["value"] = world * batched["value"] * batched["seconds"] / max_over_ranks(batched["seconds"])
        barrier()
        served = run_served(api, torch, dev, args.serve_jobs)
        served["value"] = world * served["value"] * served["seconds"] / max_over_ranks(served["seconds"])
        barrier()

    if rank == 0:
        value = world * n * args.steps / (ms32 * 1e-3)
        peak, peak_kind = read_peaks()
        b_alg = alg_bytes_per_molecule_step()
        achieved = n * b_alg / (f32["force_ms_avg"] * 1e-3) / 1e9
        traffic = profile_traffic()
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_baseline()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": workload_name(), "molecules": n, "replicas": world,
                       "form": "precision: FP32 pair forces, FP64 r/v/a, FP64 compensated sums",
                       "l2": "no flush: per-step working set (neighbour list ~%d MB + state) exceeds the 126 MB L2"
                             % (n * f32["capacity"] * 4 // 2 ** 20),
                       "rebuilds_in_timed_region": f32["rebuilds"], "parallelism": f"replicas x{world}"},
            "forms": {
                "fp32_forces": {"value": value, "ms_per_step": ms32 / args.steps,
                                "force_kernel_ms": f32["force_ms_avg"], "threads_per_molecule": f32["tpm"],
                                "force_path": f32["force_path"]},
                "fp64_plain": {"value": world * n * args.steps / (ms64 * 1e-3), "ms_per_step": ms64 / args.steps,
                               "force_kernel_ms": f64["force_ms_avg"], "threads_per_molecule": f64["tpm"],
                               "force_path": f64["force_path"]},
            },
            "roofline": {"bound": "hbm", "kernel": "k_force (fused forces + move(2) + next move(1))",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": f"{peak_kind} hbm_gbs", "alg_bytes_per_molecule_step": b_alg,
                         "traffic": traffic},
            "clocks": f32["clocks"],
            "gpu_launches": f32["launches"],
            "nve_drift": drift,
            "fene": fene,
            "batched": batched,
            "served": served,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
