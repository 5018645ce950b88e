"""The multi-job slot engine (batched replicas, served jobs) on the GPU.

Tolerances: a job run in the engine follows the single-system path and the
FP64 oracle to 1e-9 in positions after O(100) steps (different kernels sum the
same pairs, so the trajectories agree to rounding that chaos amplifies
slowly); a job's results are bit-identical whether it runs alone or among
other jobs (jobs never share arithmetic)."""
import numpy as np
import pytest

import oracle as O
from flowmol_b200 import api, couette, lattice

pytestmark = pytest.mark.gpu

TPM = 4
TOL32 = 1e-5       # FP32 pair forces: per molecule, relative to max(|F|, F_FLOOR32)
F_FLOOR32 = 10.0


def engine(max_mol=300000, slots=16, ticks=20, tpm=TPM, **kw):
    return api.Engine(max_molecules=max_mol, max_cells=400000, max_list_entries=max_mol * 160,
                      max_slots=slots, threads_per_molecule=tpm, ticks_per_chunk=ticks, **kw)


def lj_replica(nunits, rho, T, seed, jitter=0.03):
    r, v, dom = lattice.lj_fluid(nunits, rho, T, seed)
    return lattice.jitter(r, jitter, seed, dom), v, dom


def test_batch_replicas_follow_single_system(gpu_lib):
    reps = [([6, 6, 6], 0.8, 1.0, 11), ([7, 5, 6], 0.6, 1.3, 12), ([8, 8, 8], 0.85, 0.8, 13),
            ([3, 3, 3], 0.9, 1.0, 14)]  # the last has fewer than 3 cells: all pairs
    nsteps = 150
    e = engine()
    ids = []
    for nu, rho, T, seed in reps:
        r, v, dom = lj_replica(nu, rho, T, seed)
        fl = 0 if min(np.floor(dom / 2.8)) < 3 else 3
        ids.append((e.submit(api.make_job(len(r), dom, 2.5, nsteps, tplot=50, force_list=fl), r, v), r, v, dom, fl))
    e.run()
    res = {x["job_id"]: x for x in e.results()}
    for jid, r, v, dom, fl in ids:
        assert res[jid]["status"] == 0
        assert res[jid]["final_iter"] == nsteps
        rg, vg = e.job_state(jid, len(r))
        p = api.make_params(len(r), dom, 2.5, tplot=50, force_list=fl, threads_per_molecule=TPM)
        s = api.MDSystem(p)
        s.upload(r, v)
        s.setup()
        s.simulation_md(nsteps)
        rs, vs, _, _ = s.download()
        np.testing.assert_allclose(rg, rs, rtol=0, atol=1e-9)
        np.testing.assert_allclose(vg, vs, rtol=0, atol=1e-9)
        last = s.records()[-1]
        assert res[jid]["last"]["iter"] == last["iter"] == nsteps
        assert res[jid]["last"]["totenergy"] == pytest.approx(last["totenergy"], rel=1e-11)
        s.close()


def couette_inputs(n_target, speed, seed):
    nu = couette.nunits_for(n_target)
    r, v, tag, rt, sv, dom = couette.couette_job(nu, 0.8, 1.0, speed, seed)
    job = dict(np_=len(r), domain=dom, rcutoff=couette.WCA_RC, integration_algorithm=0, ensemble=6,
               pressure_outflag=1, nthermo=2, thermostat_temperature=(1.0, 1.0), teth=(0.0, 5000.0, 5.0e6),
               tplot=10)
    return job, r, v, tag, rt, sv, dom


def test_tick_loop_runs_a_batch_in_one_launch(gpu_lib):
    """The chunk's ticks loop on the device (a graph WHILE node): a batch that
    fits the engine runs from admission to its last step in one
    fm_engine_step_chunk -- one graph launch, however large ticks_per_chunk
    -- and the loop stops when the jobs are done, not at the chunk's bound.
    While jobs wait in the queue, a job that finishes ends the launch, so the
    host retires it and admits the next one at once."""
    reps = [([6, 6, 6], 0.8, 1.0, 21), ([7, 5, 6], 0.6, 1.3, 22), ([3, 3, 3], 0.9, 1.0, 23)]
    e = engine(ticks=100000)
    for k, (nu, rho, T, seed) in enumerate(reps):
        r, v, dom = lj_replica(nu, rho, T, seed)
        fl = 0 if min(np.floor(dom / 2.8)) < 3 else 3
        e.submit(api.make_job(len(r), dom, 2.5, 60 * (k + 1), tplot=40, force_list=fl), r, v)
    res, q = e.step_chunk()
    assert res == 0 and q == 0
    out = e.results()
    assert sorted(x["final_iter"] for x in out) == [60, 120, 180] and all(x["status"] == 0 for x in out)
    assert e.counters()["ticks"] <= 181 + 32  # whole iterations of the loop (32 ticks each)
    e.close()
    e = engine(slots=2, ticks=100000)
    for k, (nu, rho, T, seed) in enumerate(reps[:2] + reps[:1]):
        r, v, dom = lj_replica(nu, rho, T, seed)
        e.submit(api.make_job(len(r), dom, 2.5, 120 if k == 1 else 60, tplot=40), r, v)
    res, q = e.step_chunk()  # the third job waits: the first launch ends when the 60-step job is done
    assert (res, q) == (1, 1) and [x["final_iter"] for x in e.results()] == [60]
    res, q = e.step_chunk()
    assert (res, q) == (0, 0) and sorted(x["final_iter"] for x in e.results()) == [60, 120]
    assert e.counters()["ticks"] <= 64 + 96
    e.close()
    # a job whose list overflows ends the launch at once (it is re-queued with
    # more room) instead of waiting for a long job beside it to finish
    e = engine(ticks=100000)
    r, v, dom = lj_replica(*reps[0])
    e.submit(api.make_job(len(r), dom, 2.5, 60, tplot=20, nlist_capacity=8), r, v)
    r2, v2, dom2 = lj_replica(*reps[1])
    e.submit(api.make_job(len(r2), dom2, 2.5, 600, tplot=200), r2, v2)
    e.run()
    out = e.results()
    assert all(x["status"] == 0 for x in out) and max(x["retries"] for x in out) >= 1
    assert e.counters()["ticks"] <= 600 + 64
    e.close()


def test_couette_job_follows_oracle(gpu_lib):
    job, r, v, tag, rt, sv, dom = couette_inputs(500, 1.0, 21)
    nsteps = 200
    e = engine()
    jid = e.submit(api.make_job(nsteps=nsteps, **job), r, v, tag, rt, sv)
    e.run()
    res = e.results()[0]
    assert res["status"] == 0 and res["nsamples"] == nsteps // 10
    rg, vg = e.job_state(jid, len(r))
    o = O.Oracle(r, v, dom, couette.WCA_RC, tplot=10, integration_algorithm=0)
    o.set_tags(6, tag, rt, sv, (0.0, 5000.0, 5.0e6), 2, (1.0, 1.0))
    o.set_pressure(1)
    o.setup()
    o.run_lfv(nsteps)
    P, ns = o.pressure_average()
    assert ns == res["nsamples"]
    np.testing.assert_allclose(res["ptensor"], P, rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(rg, o.r, rtol=0, atol=1e-9)
    np.testing.assert_allclose(vg, o.v, rtol=0, atol=1e-8)


def test_jobs_alone_equal_jobs_in_the_mix(gpu_lib):
    """Served jobs give bit-identical results alone and while other jobs come
    and go (two slots, five jobs: admission and retirement interleave)."""
    inputs = []
    for k, (n, speed) in enumerate([(300, 0.5), (700, 2.0), (420, 1.2), (1100, 0.8)]):
        job, r, v, tag, rt, sv, dom = couette_inputs(n, speed, 30 + k)
        inputs.append((api.make_job(nsteps=60 + 40 * k, **job), r, v, tag, rt, sv))
    rl, vl, doml = lj_replica([6, 6, 6], 0.8, 1.1, 41)
    inputs.append((api.make_job(len(rl), doml, 2.5, 90, tplot=30), rl, vl, None, None, None))
    alone = []
    for job, r, v, tag, rt, sv in inputs:
        e = engine(slots=1)
        jid = e.submit(job, r, v, tag, rt, sv)
        e.run()
        res = e.results()[0]
        alone.append((res, e.job_state(jid, len(r))))
        e.close()
    mix = engine(slots=2)
    ids = [mix.submit(job, r, v, tag, rt, sv) for job, r, v, tag, rt, sv in inputs]
    mix.run()
    res = {x["job_id"]: x for x in mix.results()}
    for jid, (a_res, (ra, va)), (job, r, *_rest) in zip(ids, alone, inputs):
        m = res[jid]
        assert m["status"] == 0 and a_res["status"] == 0
        assert np.array_equal(m["ptensor"], a_res["ptensor"])
        assert m["last"] == a_res["last"]
        rm, vm = mix.job_state(jid, len(r))
        assert np.array_equal(rm, ra) and np.array_equal(vm, va)


def test_list_overflow_is_retried(gpu_lib):
    r, v, dom = lj_replica([6, 6, 6], 0.8, 1.0, 51)
    ref = engine()
    jr = ref.submit(api.make_job(len(r), dom, 2.5, 60, tplot=20), r, v)
    ref.run()
    res_ref = ref.results()[0]
    small = engine()
    js = small.submit(api.make_job(len(r), dom, 2.5, 60, tplot=20, nlist_capacity=8), r, v)
    small.run()
    res = small.results()[0]
    assert res["status"] == 0 and res["retries"] >= 1
    assert np.array_equal(ref.job_state(jr, len(r))[0], small.job_state(js, len(r))[0])
    assert res["last"] == res_ref["last"]


def test_failing_job_does_not_disturb_others(gpu_lib):
    r, v, dom = lj_replica([6, 6, 6], 0.8, 1.0, 61)
    bad = r.copy()
    bad[3] = [5.0 * dom[0], 0.0, 0.0]
    e = engine()
    jb = e.submit(api.make_job(len(r), dom, 2.5, 40, tplot=20), bad, v)
    jg = e.submit(api.make_job(len(r), dom, 2.5, 40, tplot=20), r, v)
    e.run()
    res = {x["job_id"]: x for x in e.results()}
    assert res[jb]["status"] == 4  # FM_ERR_ESCAPE
    assert res[jg]["status"] == 0 and res[jg]["final_iter"] == 40


# ---------------------------------------------------------------------------
# The forms the bench runs: FP32 pair forces at 1 and 2 lanes per molecule.
# ---------------------------------------------------------------------------

# a sample of the uneven batched replicas: LJ rc 2.5 at densities 0.35-0.9 and
# temperatures 0.7-1.4; the last box has fewer than 3 cells per axis and runs
# all pairs with minimum image
FP32_REPLICAS = [([5, 5, 5], 0.35, 1.4, 71), ([6, 6, 6], 0.9, 0.7, 72), ([7, 6, 5], 0.6, 1.0, 73),
                 ([3, 3, 3], 0.8, 1.1, 74)]


def _force_list(dom):
    return 0 if min(np.floor(dom / 2.8)) < 3 else 3


@pytest.mark.parametrize("tpm", [1, 2])
def test_fp32_batch_replicas_follow_single_system(gpu_lib, tpm):
    """FP32 engine replicas against the FP32 single-system path with the same
    lanes per molecule: the same pair magnitudes summed in FP64, so the
    trajectories agree to FP64 rounding (1e-9 after 150 steps)."""
    nsteps = 150
    e = engine(tpm=tpm, precision=1)
    ids = []
    for nu, rho, T, seed in FP32_REPLICAS:
        r, v, dom = lj_replica(nu, rho, T, seed)
        fl = _force_list(dom)
        ids.append((e.submit(api.make_job(len(r), dom, 2.5, nsteps, tplot=50, force_list=fl), r, v), r, v, dom, fl))
    e.run()
    assert e.counters()["threads_per_molecule"] == tpm
    res = {x["job_id"]: x for x in e.results()}
    assert any(fl == 0 for *_x, fl in ids)
    for jid, r, v, dom, fl in ids:
        assert res[jid]["status"] == 0 and res[jid]["final_iter"] == nsteps
        rg, vg = e.job_state(jid, len(r))
        p = api.make_params(len(r), dom, 2.5, tplot=50, force_list=fl, threads_per_molecule=tpm, precision=1)
        s = api.MDSystem(p)
        s.upload(r, v)
        s.setup()
        s.simulation_md(nsteps)
        rs, vs, _, _ = s.download()
        np.testing.assert_allclose(rg, rs, rtol=0, atol=1e-9)
        np.testing.assert_allclose(vg, vs, rtol=0, atol=1e-9)
        last = s.records()[-1]
        assert res[jid]["last"]["totenergy"] == pytest.approx(last["totenergy"], rel=1e-11)
        s.close()


def _min_image(d, dom):
    return d - dom * np.round(d / dom)


@pytest.mark.parametrize("tpm", [1, 2])
def test_fp32_batch_forces_and_records_against_oracle(gpu_lib, tpm):
    """FP32 engine replicas against the FP64 oracle directly.

    Forces of iteration 0: a one-step velocity-Verlet job leaves
    r1 = r0 + dt v0 + (dt^2/2) a0, so a0 = (r1 - r0 - dt v0) / (dt^2/2) to
    ~1e-9 absolute (the rounding of r1, ~2e-15, over dt^2/2 = 1.25e-5) --
    far below the FP32 tolerance 1e-5 * max(|F|, 10).  Records after 100
    steps: kinetic, potential and total energy per molecule within 1e-5
    relative and the pressure within 1e-4 absolute of the oracle's (FP32
    forces move the trajectory by ~1e-6 over 100 steps)."""
    dt = 0.005
    for nu, rho, T, seed in FP32_REPLICAS:
        r, v, dom = lj_replica(nu, rho, T, seed)
        fl = _force_list(dom)
        e = engine(tpm=tpm, precision=1)
        j1 = e.submit(api.make_job(len(r), dom, 2.5, 1, tplot=1000, force_list=fl), r, v)
        j100 = e.submit(api.make_job(len(r), dom, 2.5, 100, tplot=50, force_list=fl), r, v)
        e.run()
        res = {x["job_id"]: x for x in e.results()}
        assert res[j1]["status"] == 0 and res[j100]["status"] == 0
        r1, _ = e.job_state(j1, len(r))
        a0 = _min_image(r1 - r - dt * v, dom) / (0.5 * dt * dt)
        o = O.Oracle(r, v, dom, 2.5, tplot=50, force_list=fl)
        o.setup()
        err = rel_err_rows(a0, o.a, F_FLOOR32)
        assert err.max() <= TOL32, (nu, rho, err.max())
        rec = o.run_vv(100)
        last_o = rec[-1]
        last_g = res[j100]["last"]
        assert last_g["iter"] == int(last_o[0]) == 100
        m = o.macro()
        for k in ("kinenergy", "potenergy", "totenergy"):
            assert last_g[k] == pytest.approx(m[k], rel=TOL32, abs=TOL32), (k, nu, rho)
        assert last_g["pressure"] == pytest.approx(m["pressure"], abs=1e-4)
        e.close()


def rel_err_rows(x, ref, floor):
    d = np.linalg.norm(x - ref, axis=-1)
    return d / np.maximum(np.linalg.norm(ref, axis=-1), floor)


@pytest.mark.parametrize("tpm", [1, 2])
def test_fp32_couette_job_follows_oracle(gpu_lib, tpm):
    """One served Couette job (WCA, tethered sliding walls, thermostatted wall
    regions, leap-frog) in FP32 against the FP64 oracle over 40 steps: the
    time-averaged pressure tensor within 1e-5 relative (1e-5 absolute for the
    small off-diagonal terms) and positions within 2e-6."""
    job, r, v, tag, rt, sv, dom = couette_inputs(500, 1.0, 21)
    nsteps = 40
    e = engine(tpm=tpm, precision=1)
    jid = e.submit(api.make_job(nsteps=nsteps, **job), r, v, tag, rt, sv)
    e.run()
    res = e.results()[0]
    assert res["status"] == 0 and res["nsamples"] == nsteps // 10
    rg, vg = e.job_state(jid, len(r))
    o = O.Oracle(r, v, dom, couette.WCA_RC, tplot=10, integration_algorithm=0)
    o.set_tags(6, tag, rt, sv, (0.0, 5000.0, 5.0e6), 2, (1.0, 1.0))
    o.set_pressure(1)
    o.setup()
    o.run_lfv(nsteps)
    P, ns = o.pressure_average()
    assert ns == res["nsamples"]
    np.testing.assert_allclose(res["ptensor"], P, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(rg, o.r, rtol=0, atol=2e-6)


@pytest.mark.parametrize("tpm", [0, 4])
def test_list_build_tiles_give_identical_jobs(gpu_lib, tpm):
    """The list build's tile (one cell per warp, 2x2x2 cells per warp, or the
    autotuner's choice per job density) changes no result bit: dense and
    sparse jobs run to the same trajectories under all three.  With the lanes
    per molecule autotuned as well (tpm 0), two engines may time their way to
    different lane counts, which sum each row in a different order: such a
    pair is compared to FP64 rounding instead."""
    reps = [([8, 8, 8], 0.85, 1.0, 51), ([7, 7, 7], 0.3, 1.4, 52), ([9, 6, 7], 0.1, 1.2, 53),
            ([6, 6, 6], 0.8, 0.9, 54)]
    out, lanes = {}, {}
    for lb in (api.LIST_BUILD_CELLS, api.LIST_BUILD_BLOCKS, api.LIST_BUILD_AUTO):
        e = engine(tpm=tpm, list_build=lb, ticks=10)
        ids = []
        for nu, rho, T, seed in reps:
            r, v, dom = lj_replica(nu, rho, T, seed)
            ids.append((e.submit(api.make_job(len(r), dom, 2.5, 120, tplot=40), r, v), len(r)))
        e.run()
        res = {x["job_id"]: x for x in e.results()}
        out[lb] = [(res[j]["status"], res[j]["last"], res[j]["rebuilds"]) + e.job_state(j, n) for j, n in ids]
        t, bb = e.tuning()
        lanes[lb] = t
        if lb == api.LIST_BUILD_CELLS:
            assert bb == 0.0
        elif lb == api.LIST_BUILD_BLOCKS:
            assert bb >= 1e30
        else:
            assert bb in (0.0, 4.0, 8.0, 16.0, 1e30)
        assert t in ((1, 2, 4, 8, 16) if tpm == 0 else (tpm,))
        e.close()
    for lb in (api.LIST_BUILD_BLOCKS, api.LIST_BUILD_AUTO):
        same_lanes = lanes[lb] == lanes[api.LIST_BUILD_CELLS]
        for a, b in zip(out[api.LIST_BUILD_CELLS], out[lb]):
            assert a[0] == b[0] == 0 and a[2] == b[2]
            if same_lanes:
                assert a[1] == b[1]
                assert np.array_equal(a[3], b[3]) and np.array_equal(a[4], b[4])
            else:
                assert a[1]["iter"] == b[1]["iter"]
                assert a[1]["totenergy"] == pytest.approx(b[1]["totenergy"], rel=1e-11)
                np.testing.assert_allclose(a[3], b[3], rtol=0, atol=1e-9)
                np.testing.assert_allclose(a[4], b[4], rtol=0, atol=1e-9)
