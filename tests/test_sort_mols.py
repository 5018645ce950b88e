"""sort_mols (linklist.f90:2744-2869) and its block table Hcurve
(setup_set_parameters.f90:1140-1163, functions_lib.f90:2555-2604).

The reference ships no Hcurve or sort output, so the table is pinned by the
properties of the curve it builds: every block numbered once, consecutive
numbers face-adjacent on a power-of-two cube, a box whose longest axis is not
a power of two numbered in the order of the enclosing power-of-two cube's
curve.  The library's table (an index-by-digits restatement in C++) must equal
the oracle's (the recursive array restatement in C), bit for bit.

The sort itself is integer work and is checked exactly: after each GPU
sort_mols the downloaded r, v and global numbers equal the oracle's sort of
the GPU's own pre-sort state, including the rebuild counter and the skipped
sorts (a block above ave_molperblock) with their growing safety factors; and
the fused device loop, which sorts inside its rebuild branch, ends bit for
bit where the subroutine-by-subroutine mirror ends.
"""
import os

import numpy as np
import pytest

import oracle as O
from flowmol_b200 import api

SHAPES = [(1, 1, 1), (2, 2, 2), (1, 3, 2), (4, 4, 4), (3, 5, 7), (5, 5, 5), (8, 8, 8), (17, 4, 9),
          (12, 12, 12), (16, 16, 16), (20, 3, 3), (33, 2, 2), (7, 31, 2)]


def _cells(t, nb):
    """Block (i, j, k) of each Hcurve number, for a flat x-fastest table."""
    pos = np.zeros((len(t) + 1, 3), np.int64)
    for lin, m in enumerate(t):
        pos[m] = (lin % nb[0], (lin // nb[0]) % nb[1], lin // (nb[0] * nb[1]))
    return pos[1:]


@pytest.mark.parametrize("flag", [1, 2])
@pytest.mark.parametrize("nb", SHAPES)
def test_table_equals_oracle_and_numbers_every_block_once(flag, nb):
    t = api.sort_table(flag, nb)
    assert np.array_equal(t, O.sort_table(flag, nb))
    assert np.array_equal(np.sort(t), np.arange(1, int(np.prod(nb)) + 1))
    if flag == 1:
        assert np.array_equal(t, np.arange(1, t.size + 1))


@pytest.mark.parametrize("side", [2, 4, 8, 16])
def test_hilbert_steps_to_a_face_neighbour(side):
    nb = (side, side, side)
    pos = _cells(api.sort_table(2, nb), nb)
    assert np.all(np.abs(np.diff(pos, axis=0)).sum(axis=1) == 1)


@pytest.mark.parametrize("nb", [(3, 5, 7), (17, 4, 9), (20, 3, 3), (7, 31, 2), (12, 12, 12)])
def test_hilbert_of_a_box_follows_the_enclosing_cube(nb):
    """A longest axis of 17..31 blocks scales the curve to a grid of
    ceiling(8**(5/3)) = 33 cells (the FP64 pow lands above 32); the points
    still fall on cells 1..32, so the box is numbered in the order of the 32^3
    curve, as for any other box inside its power-of-two cube."""
    side = 1 << int(np.ceil(np.log2(max(nb))))
    cube = api.sort_table(2, (side,) * 3)
    order = []
    for m, (i, j, k) in enumerate(_cells(cube, (side,) * 3)):
        if i < nb[0] and j < nb[1] and k < nb[2]:
            order.append((i, j, k))
    pos = _cells(api.sort_table(2, nb), nb)
    assert [tuple(p) for p in pos] == order


def test_table_refusals():
    with pytest.raises(api.FlowmolError):
        api.sort_table(3, (2, 2, 2))
    with pytest.raises(api.FlowmolError):
        api.sort_table(2, (0, 2, 2))


def _blocks(r, dom, cs, bs):
    bsl = bs * np.asarray(cs)
    nb = np.ceil(np.asarray(dom) / bsl).astype(int)
    ib = np.ceil((r + 0.5 * np.asarray(dom)) / bsl).astype(int)
    return nb, ib


def test_oracle_sort_is_a_stable_sort_by_block_number():
    rng = np.random.default_rng(5)
    dom = np.array([10.0, 12.0, 9.0]); cs = dom / np.array([3, 4, 3])
    r = (rng.random((4000, 3)) - 0.5) * dom
    v = rng.standard_normal((4000, 3)); g = np.arange(1, 4001, dtype=np.int32)
    for flag in (1, 2):
        st = O.SortState()
        r2, v2, g2, perm, did = O.sort_mols(r, v, g, dom, cs, flag, 1, 1, st)
        assert did == 1
        nb, ib = _blocks(r, dom, cs, 1)
        hc = O.sort_table(flag, nb)
        key = hc[(ib[:, 0] - 1) + nb[0] * ((ib[:, 1] - 1) + nb[1] * (ib[:, 2] - 1))]
        assert np.array_equal(perm, np.argsort(key, kind="stable"))
        assert np.array_equal(r2, r[perm]) and np.array_equal(v2, v[perm]) and np.array_equal(g2, g[perm])


def test_oracle_counter_and_overflow():
    """nrebuilds runs 1..sort_freq; an overflowing block skips the sort and
    grows sf1 by 0.1 and sf2 by 5 until the blocks fit."""
    rng = np.random.default_rng(6)
    dom = np.array([10.0, 10.0, 10.0]); cs = dom / 4
    r = (rng.random((800, 3)) - 0.5) * dom
    r[:250] = (rng.random((250, 3)) - 0.5) * 2.0 - 3.0  # a clump in block (1,1,1)
    v = np.zeros_like(r); g = np.arange(1, 801, dtype=np.int32)
    st = O.SortState()
    dids = []
    for _ in range(40):
        _, _, _, _, did = O.sort_mols(r, v, g, dom, cs, 2, 2, 2, st)
        dids.append(did)
    assert dids[0::2] == [0] * 20
    skipped = dids[1::2].index(1)
    assert skipped > 0 and dids[1::2][:skipped] == [2] * skipped
    # ave_molperblock = ceiling(100 sf1 + sf2) fits the clump from that sort on
    assert st.sf2 == 5 + 5 * skipped
    assert st.sf1 == pytest.approx(1.5 + 0.1 * skipped, abs=1e-12)


def test_input_deck_sort_flag(tmp_path):
    here = os.path.join(os.path.dirname(__file__), "golden")
    inp = api.read_input(os.path.join(here, "default.in"))
    assert (inp.sort_flag, inp.sort_freq, inp.sortblocksize) == (2, 1, 3)
    deck = open(os.path.join(here, "default.in")).read() + "\nGLOBAL_NUMBERING\n1\n"
    p = tmp_path / "numbered.in"
    p.write_text(deck)
    with pytest.raises(api.FlowmolError, match="Global number does not work with sort flag on"):
        api.read_input(str(p))


# ---------------------------------------------------------------------------
# the CUDA path
# ---------------------------------------------------------------------------

def _system(r, v, dom, **kw):
    p = api.make_params(len(r), dom, 2.5, tplot=kw.pop("tplot", 40), density=0.8442, **kw)
    s = api.MDSystem(p)
    s.upload(r, v)
    return s


@pytest.fixture(scope="module")
def liquid(gpu_lib):
    from helpers import liquid_state
    r, v, dom, _ = liquid_state([8, 8, 8], 0.8442, 0.722, 2.5, steps=100)
    return r, v, dom


@pytest.mark.gpu
@pytest.mark.parametrize("flag,bs", [(2, 1), (1, 1), (2, 2)])
def test_sort_mols_equals_oracle_at_every_rebuild(liquid, flag, bs):
    """md_advance_vv subroutine by subroutine; at each rebuild the state after
    the GPU's sort_mols equals the oracle's sort of the state before it."""
    r, v, dom = liquid
    s = _system(r, v, dom)
    s.set_sort(flag, 1, bs)
    s.setup()
    cs = O.cells(dom, 2.5, (0.3, 0.3, 0.3))[2]
    st = O.SortState()
    sorts = 0
    for _ in range(80):
        s.iter = s.iter + 1
        s.simulation_move_particles_vv(1)
        s.messenger_updateborders(0)
        if s.simulation_checkrebuild():
            s.linklist_deallocateall()
            s.sendmols()
            r0, v0, _, g0 = s.download()
            r1, v1, g1, perm, did = O.sort_mols(r0, v0, g0, dom, cs, flag, 1, bs, st)
            s.sort_mols()
            r2, v2, _, g2 = s.download()
            assert did == 1
            assert np.array_equal(r2, r1) and np.array_equal(v2, v1) and np.array_equal(g2, g1)
            sorts += 1
            s.assign_to_cell()
            s.messenger_updateborders(1)
            s.assign_to_neighbourlist()
        s.simulation_compute_forces()
        s.simulation_move_particles_vv(2)
    assert sorts >= 3 and s.sort_state()["sorts"] == sorts
    # forces of the final (re-numbered) state against the oracle's
    rg, vg, ag, _ = s.download()
    o = O.Oracle(rg, vg, dom, 2.5, tplot=10 ** 6, density=0.8442)
    o.setup()
    np.testing.assert_allclose(ag, o.a, rtol=0, atol=1e-9)
    s.close()


@pytest.mark.gpu
def test_sort_counter_and_overflow_equal_oracle(liquid):
    """Blocks of 3 cells on a 4-cell box: 2 blocks per axis, the first holding
    ~42% of the molecules against ave_molperblock = ceiling(256 sf1 + sf2), so
    sorts are skipped and the safety factors grow until it fits.  Every second
    call sorts (sort_freq 2).  Each call matches the oracle's outcome, state
    and safety factors."""
    r, v, dom = liquid
    s = _system(r, v, dom)
    s.set_sort(2, 2, 3)
    s.setup()
    cs = O.cells(dom, 2.5, (0.3, 0.3, 0.3))[2]
    st = O.SortState()
    outcomes = []
    for _ in range(44):
        r0, v0, _, g0 = s.download()
        r1, v1, g1, perm, did = O.sort_mols(r0, v0, g0, dom, cs, 2, 2, 3, st)
        s.sort_mols()
        r2, v2, _, g2 = s.download()
        assert np.array_equal(r2, r1) and np.array_equal(v2, v1) and np.array_equal(g2, g1)
        q = s.sort_state()
        assert (q["nrebuilds"], q["sf2"], q["sf1"]) == (st.nrebuilds, st.sf2, st.sf1)
        outcomes.append(did)
    assert outcomes.count(2) > 3 and outcomes.count(1) > 0
    q = s.sort_state()
    assert q["skipped"] == outcomes.count(2) and q["sorts"] == outcomes.count(1)
    s.close()


FUSED_CASES = [
    dict(integration_algorithm=1, force_list=3),
    dict(integration_algorithm=0, force_list=3),
    dict(integration_algorithm=1, force_list=0),
    dict(integration_algorithm=1, force_list=3, force_path=api.FORCE_PATH_TILES),
    dict(integration_algorithm=1, force_list=3, precision=api.PRECISION_FP32),
    dict(integration_algorithm=1, force_list=3, rebuild_criteria=2),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", FUSED_CASES, ids=["vv", "lfv", "all_pairs", "tiles", "fp32", "crit2"])
@pytest.mark.parametrize("graphs", ["1", "0"])
def test_fused_loop_sorts_like_the_mirror(liquid, monkeypatch, case, graphs):
    """The fused loop runs sort_mols inside its rebuild branch (in the step
    graphs' conditional body, or as gated launches with FM_STEP_GRAPHS=0):
    120 iterations end bit for bit where the subroutine mirror ends, with the
    same numbering and the same number of sorts (sort_freq 2) -- leap-frog,
    all pairs, the tiled force path, FP32 pair forces and the displacement
    rebuild criterion included."""
    monkeypatch.setenv("FM_STEP_GRAPHS", graphs)
    r, v, dom = liquid
    integration, force_list = case["integration_algorithm"], case["force_list"]
    out = []
    for fused in (False, True):
        s = _system(r, v, dom, **case)
        s.set_sort(2, 2, 1)
        s.setup()
        if fused:
            s.simulation_md(120)
        else:
            for _ in range(120):
                if integration == 1:
                    s.md_advance_vv()
                else:
                    s.md_advance_lfv()
        out.append((s.download(), s.sort_state(), s.counters()["rebuilds"] if force_list else 0))
        s.close()
    (sa, qa, na), (sb, qb, nb) = out
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)
    assert qa == qb and qa["sorts"] >= 2
    assert na == nb
    assert not np.array_equal(sa[3], np.arange(1, len(r) + 1))  # the numbering moved


@pytest.mark.gpu
@pytest.mark.parametrize("flag", [1, 2])
def test_sort_of_molecules_on_the_lower_face_equals_oracle(liquid, flag):
    """A molecule exactly at -L/2 gets block 0, outside Hcurve: the reference
    reads the element before (iblk, jblk, kblk)'s column-major place, which
    both paths reproduce, clamping an offset before the table's start."""
    r, v, dom = liquid
    r = r.copy()
    r[0, 0] = -0.5 * dom[0]
    r[1] = -0.5 * np.asarray(dom)
    r[2, 1] = -0.5 * dom[1]
    s = _system(r, v, dom)
    s.set_sort(flag, 1, 1)
    cs = O.cells(dom, 2.5, (0.3, 0.3, 0.3))[2]
    r0, v0, _, g0 = s.download()
    r1, v1, g1, _, did = O.sort_mols(r0, v0, g0, dom, cs, flag, 1, 1, O.SortState())
    s.sort_mols()
    r2, v2, _, g2 = s.download()
    assert did == 1
    assert np.array_equal(r2, r1) and np.array_equal(v2, v1) and np.array_equal(g2, g1)
    s.close()


@pytest.mark.gpu
def test_step_graphs_carry_the_sort(liquid, monkeypatch):
    """With sorting on, the step graphs still capture the rebuild body (the
    sort kernels and the library radix sort inside the conditional node)
    rather than falling back to per-kernel launches: the same 120 iterations
    launch fewer kernels than FM_STEP_GRAPHS=0, with a bit-identical result."""
    r, v, dom = liquid
    out = []
    for env in ("1", "0"):
        monkeypatch.setenv("FM_STEP_GRAPHS", env)
        s = _system(r, v, dom)
        s.set_sort(2, 1, 1)
        s.setup()
        s.simulation_md(120)
        out.append((s.download(), s.sort_state(), s.launch_count()))
        s.close()
    (sa, qa, la), (sb, qb, lb) = out
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)
    assert qa == qb and qa["sorts"] >= 3
    assert la < lb


@pytest.mark.gpu
def test_sort_refusals(liquid):
    r, v, dom = liquid
    s = _system(r, v, dom)
    with pytest.raises(api.FlowmolError, match="Incorrect value of sort_flag"):
        s.set_sort(3, 1, 1)
    with pytest.raises(api.FlowmolError):
        s.set_sort(2, 1, 0)
    s.set_sort(2, 1, 1)
    from helpers import mie_mixture_tables
    with pytest.raises(api.FlowmolError, match="Mie"):
        s.set_mie(mie_mixture_tables(2.5), (np.arange(len(r)) % 2 + 1).astype(np.int32))
    s.close()
