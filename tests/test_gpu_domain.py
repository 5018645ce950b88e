"""Spatial decomposition on the GPU: all ranks' subdomains of one system as
separate handles on one device, exchanging through device copies
(LocalTransport), against one handle over the whole box.

Tolerances: none for the state.  A subdomain bins, orders and pairs its
molecules exactly as the undivided system does, so after setup and 60
velocity-Verlet steps (rebuilds and migration included) every position and
velocity is bit-identical, in FP64 and in the FP32-forces form.  Records
add the ranks' sums in another order: 1e-12 relative."""
import numpy as np
import pytest

from flowmol_b200 import api, lattice
from flowmol_b200 import domain as D

pytestmark = pytest.mark.gpu

NSTEPS = 60
TPLOT = 10


def _state(seed=lattice.SEED_BASE + 91):
    r, v, dom = lattice.lj_fluid([10, 10, 10], 0.8, 1.0, seed)  # 4000 molecules, 6 cells per axis
    return lattice.jitter(r, 0.05, seed, dom), v, dom


def _params(n, dom, precision):
    return api.make_params(n, dom, 2.5, tplot=TPLOT, density=0.8, threads_per_molecule=4, precision=precision)


@pytest.mark.parametrize("precision", [api.PRECISION_FP64, api.PRECISION_FP32])
@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 1, 1), (3, 1, 1), (2, 2, 2), (3, 2, 1)])
def test_subdomains_equal_the_undivided_system(gpu_lib, dims, precision):
    from helpers import canonical_full

    r, v, dom = _state()
    n = len(r)
    p = _params(n, dom, precision)
    s = api.MDSystem(p)
    s.upload(r, v)
    s.setup()
    pairs_single = canonical_full(*s.pair_list())
    rec0 = s.records()
    s.simulation_md(NSTEPS)
    recs = s.records()
    rs, vs, _, _ = s.download()
    rebuilds = s.counters()["rebuilds"]
    s.close()

    sysd = D.local_system(p, r, v, dims=dims)
    try:
        sysd.setup()
        o, q, c = zip(*[sd.pair_list() for sd in sysd.subs])
        assert np.array_equal(canonical_full(np.concatenate(o) + 1, np.concatenate(q) + 1, np.concatenate(c)),
                              pairs_single)
        owned0 = [np.sort(sd.download()[2]) for sd in sysd.subs]
        sysd.run(NSTEPS)
        rd, vd, gid = sysd.state()
        assert np.array_equal(np.sort(gid), np.arange(n))
        assert np.array_equal(rd, rs[gid]), "positions differ from the undivided system"
        assert np.array_equal(vd, vs[gid]), "velocities differ from the undivided system"
        assert sysd.rebuilds - 1 == rebuilds
        assert len(sysd.records) == len(rec0) + len(recs)
        for a, b in zip(sysd.records, rec0 + recs):
            assert a["iter"] == b["iter"]
            for key in ("totenergy", "potenergy", "kinenergy", "pressure", "virial"):
                assert a[key] == pytest.approx(b[key], rel=1e-12, abs=1e-14)
        if len(sysd.subs) > 1:
            owned1 = [np.sort(sd.download()[2]) for sd in sysd.subs]
            assert any(not np.array_equal(a, b) for a, b in zip(owned0, owned1)), "no molecule changed rank"
    finally:
        sysd.close()


def test_subdomain_rejects_what_it_does_not_run(gpu_lib):
    r, v, dom = _state()
    plan = D.Plan(D.geometry(_params(len(r), dom, 0))["ncells"], (2, 1, 1))
    for kw in (dict(integration_algorithm=0), dict(rebuild_criteria=2), dict(force_list=0),
               dict(potential_flag=1)):
        p = api.make_params(len(r), dom, 2.5, tplot=TPLOT, density=0.8, **kw)
        with pytest.raises(api.FlowmolError):
            D.Subdomain(p, plan, 0, 10000)
