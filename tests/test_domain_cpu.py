"""Spatial decomposition on CPU: the process grid and halo plan, and the
whole host protocol (migration, halo exchange, refresh lists, rebuild
decisions, record sums) over real gloo ranks with a CPU stand-in for each
rank's subdomain, against the single-rank FP64 oracle.

Tolerances: the pair set is compared exactly (canonical multisets, image
codes included); forces per molecule to 1e-12 of max(|F|, 1) (the stand-in
sums the same pairs in another order); after 40 steps positions and
velocities to 1e-9 and total energy to 1e-10 relative (rounding differences
grow slowly in the chaotic trajectory); rebuild steps exactly."""
import os
import pickle
import socket
import tempfile

import numpy as np
import pytest

from flowmol_b200 import domain as D
from flowmol_b200 import lattice

NSTEPS = 40
TPLOT = 10


@pytest.mark.parametrize("n,dims", [(1, (1, 1, 1)), (2, (2, 1, 1)), (3, (3, 1, 1)), (4, (2, 2, 1)),
                                    (6, (2, 3, 1)), (8, (2, 2, 2)), (12, (3, 2, 2)), (7, (7, 1, 1))])
def test_find3factors(n, dims):
    assert D.find3factors(n) == dims


def test_split_cells():
    assert D.split_cells(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert D.split_cells(4, 4) == [(0, 1), (1, 1), (2, 1), (3, 1)]
    with pytest.raises(ValueError):
        D.split_cells(3, 4)


@pytest.mark.parametrize("G,dims", [((5, 4, 6), (1, 1, 1)), ((5, 4, 6), (2, 1, 1)), ((5, 4, 6), (2, 2, 2)),
                                    ((3, 4, 3), (3, 1, 1)), ((4, 4, 4), (2, 2, 1)), ((6, 5, 4), (3, 2, 2))])
def test_plan_covers_the_grid_and_its_images(G, dims):
    """Every global cell is owned once; every halo cell of every rank copies
    the global cell at its position modulo the box, from that cell's owner,
    with the shift that crossing the box edge implies; the needs table is the
    inverse of the halo tables."""
    plan = D.Plan(G, dims)
    owned = np.zeros(G, int)
    for r in range(plan.nranks):
        org, nloc = plan.box(r)
        owned[org[0]:org[0] + nloc[0], org[1]:org[1] + nloc[1], org[2]:org[2] + nloc[2]] += 1
    assert (owned == 1).all()
    total_needs = 0
    for r in range(plan.nranks):
        org, nloc = plan.box(r)
        ne = [n + 2 for n in nloc]
        h = plan.halo_sources(r)
        assert len(h["cell"]) == np.prod(ne) - np.prod(nloc)
        assert (np.diff(h["cell"]) > 0).all()
        for cell, src, src_cell, code in zip(h["cell"], h["src"], h["src_cell"], h["code"]):
            x, y, z = cell % ne[0], (cell // ne[0]) % ne[1], cell // (ne[0] * ne[1])
            g = [org[0] + x - 1, org[1] + y - 1, org[2] + z - 1]
            s = [-1 if g[k] < 0 else (1 if g[k] >= G[k] else 0) for k in range(3)]
            g = [g[k] - s[k] * G[k] for k in range(3)]
            assert code == D.code6(*s)
            o2, n2 = plan.box(int(src))
            assert all(o2[k] <= g[k] < o2[k] + n2[k] for k in range(3))
            ne2 = [c + 2 for c in n2]
            assert src_cell == (g[0] - o2[0] + 1) + ne2[0] * ((g[1] - o2[1] + 1) + ne2[1] * (g[2] - o2[2] + 1))
        nd = plan.needs(r)
        total_needs += len(nd["rank"])
        for c in range(int(np.prod(ne))):
            for k in range(nd["off"][c], nd["off"][c + 1]):
                hr = plan.halo_sources(int(nd["rank"][k]))
                m = np.nonzero(hr["cell"] == nd["cell"][k])[0]
                assert len(m) == 1 and hr["src"][m[0]] == r and hr["src_cell"][m[0]] == c
                assert hr["code"][m[0]] == nd["code"][k]
    assert total_needs == sum(len(plan.halo_sources(r)["cell"]) for r in range(plan.nranks))


def test_one_rank_halo_is_the_periodic_images():
    """With one rank every halo cell copies the interior cell on the far side
    (low halo <- last interior cell shifted by -L, high halo <- first cell
    shifted by +L), as the undivided system forms its images."""
    G = (4, 5, 3)
    plan = D.Plan(G, (1, 1, 1))
    ne = [g + 2 for g in G]
    h = plan.halo_sources(0)
    for cell, src, src_cell, code in zip(h["cell"], h["src"], h["src_cell"], h["code"]):
        c = [cell % ne[0], (cell // ne[0]) % ne[1], cell // (ne[0] * ne[1])]
        s = [-1 if c[k] == 0 else (1 if c[k] == ne[k] - 1 else 0) for k in range(3)]
        srcc = [ne[k] - 2 if c[k] == 0 else (1 if c[k] == ne[k] - 1 else c[k]) for k in range(3)]
        assert src == 0
        assert src_cell == srcc[0] + ne[0] * (srcc[1] + ne[1] * srcc[2])
        assert code == D.code6(*s)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, inp_path, out_dir):
    import datetime

    import torch.distributed as dist

    import dd_cpu
    from flowmol_b200 import api

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=120))
    with open(inp_path, "rb") as f:
        inp = pickle.load(f)
    r, v, dom, rc, dt = inp["r"], inp["v"], inp["dom"], inp["rc"], inp["dt"]
    p = api.make_params(len(r), dom, rc, delta_t=dt, tplot=TPLOT, density=inp["density"])
    geom = D.geometry(p)
    plan = D.Plan(geom["ncells"], D.find3factors(ws))
    parts = D.distribute(p, plan, r, v)
    _, g = api.derive_geometry(p)
    sub = dd_cpu.CpuSubdomain(geom, plan, rank, rc, g["rneighbr2"], dt, TPLOT, 0.5 * 0.3, len(r), inp["density"])
    sub.upload(r[parts[rank]], v[parts[rank]], parts[rank])
    system = D.DecomposedSystem(p, plan, [sub], D.DistTransport())
    system.setup()
    a, pe, gid = sub.owned_forces()
    out = dict(pairs=sub.pair_list(), a=a, gid=gid, n_setup=sub.counts())
    system.run(NSTEPS)
    rr, vv, gg = sub.download()
    out.update(r=rr, v=vv, gid_end=gg, records=system.records, rebuilds=system.rebuilds)
    with open(os.path.join(out_dir, f"rank{rank}.pkl"), "wb") as f:
        pickle.dump(out, f)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 3, 8])
def test_decomposed_ranks_match_the_oracle(ws, tmp_path):
    import torch.multiprocessing as mp

    import oracle as O
    from helpers import canonical_full, canonical_oracle

    seed = lattice.SEED_BASE + 77
    r, v, dom = lattice.lj_fluid([8, 8, 8], 0.8, 1.0, seed)
    r = lattice.jitter(r, 0.05, seed, dom)
    rc, dt = 2.5, 0.005
    inp = dict(r=r, v=v, dom=dom, rc=rc, dt=dt, density=0.8)
    inp_path = str(tmp_path / "inp.pkl")
    with open(inp_path, "wb") as f:
        pickle.dump(inp, f)
    mp.spawn(_rank_main, args=(ws, _free_port(), inp_path, str(tmp_path)), nprocs=ws, join=True)
    outs = []
    for k in range(ws):
        with open(tmp_path / f"rank{k}.pkl", "rb") as f:
            outs.append(pickle.load(f))

    o = O.Oracle(r, v, dom, rc, tplot=TPLOT, delta_t=dt, density=0.8)
    o.setup()
    # pair set: the union of the ranks' rows is the undivided system's
    own = np.concatenate([x["pairs"][0] for x in outs]) + 1
    par = np.concatenate([x["pairs"][1] for x in outs]) + 1
    code = np.concatenate([x["pairs"][2] for x in outs])
    assert np.array_equal(canonical_full(own, par, code), canonical_oracle(*o.pair_list()))
    # every molecule owned once; forces
    gid = np.concatenate([x["gid"] for x in outs])
    assert np.array_equal(np.sort(gid), np.arange(len(r)))
    a = np.concatenate([x["a"] for x in outs])
    ao = o.a[gid]
    scale = np.maximum(np.abs(ao).max(axis=1, keepdims=True), 1.0)
    assert (np.abs(a - ao) / scale).max() < 1e-12
    # 40 velocity-Verlet steps with rebuilds and migration
    recs_o = o.run_vv(NSTEPS)
    assert all(x["rebuilds"] - 1 == o.rebuild_count for x in outs)
    recs = outs[0]["records"][1:]  # [0] is the setup record
    assert [rr["iter"] for rr in recs] == [int(x) for x in recs_o[:, 0]]
    for rr, ro in zip(recs, recs_o):
        assert rr["totenergy"] == pytest.approx(ro[6], rel=1e-10)
    for x in outs[1:]:
        assert x["records"] == outs[0]["records"]
    gid = np.concatenate([x["gid_end"] for x in outs])
    assert np.array_equal(np.sort(gid), np.arange(len(r)))
    rg = np.concatenate([x["r"] for x in outs])
    vg = np.concatenate([x["v"] for x in outs])
    d = rg - o.r[gid]
    d -= dom * np.round(d / dom)
    assert np.abs(d).max() < 1e-9
    assert np.abs(vg - o.v[gid]).max() < 1e-9
    moved = sum(1 for k, x in enumerate(outs) if not np.array_equal(np.sort(x["gid_end"]), np.sort(x["gid"])))
    assert ws == 1 or moved > 0, "no molecule changed rank: the migration path was not exercised"
