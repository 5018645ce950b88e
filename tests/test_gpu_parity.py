"""Parity of the CUDA path (through the C ABI) with the FP64 CPU oracle.

Tolerances (the stated contract of the path):
  * pair sets: bit-exact (FP64 distance test, no FMA, same image roundings);
  * FP64 forces: |F_gpu - F_ref| <= 1e-12 * max(|F_ref|, 1), per molecule;
  * FP32 pair forces: |F_gpu - F_ref| <= 1e-5 * max(|F_ref|, F_FLOOR32), per
    molecule, F_FLOOR32 = 10 (the magnitude of one nearest-neighbour pair
    force in the liquid; below it the relative error of a near-cancelling sum
    is not meaningful);
  * per-molecule PE: 1e-12 (FP64) / 1e-5 (FP32) relative with a floor of 1;
  * per-molecule virial: 1e-12 (FP64) relative with a floor of 1; FP32
    1e-5 relative to max(|W_i|, W_FLOOR32), W_FLOOR32 = 100 -- the virial
    is a cancelling sum of pair terms 48(s^6 - s^3/2) that reach ~100 for the
    closest pairs, each carrying FP32 rounding of s = 1/r^2 raised to the 7th
    power (measured max 2.4e-5 against a floor of 1).
"""
import numpy as np
import pytest

import oracle as O
from flowmol_b200 import api, lattice
from helpers import (WCA_RC, canonical_full, canonical_oracle, cfg1_state, digest_oracle, liquid_state,
                     rel_err)

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5
F_FLOOR32 = 10.0
W_FLOOR32 = 100.0


def gpu_system(r, v, dom, rc, precision=0, tplot=10 ** 6, density=None, **kw):
    p = api.make_params(len(r), dom, rc, tplot=tplot, precision=precision,
                        density=density if density is not None else len(r) / float(np.prod(dom)), **kw)
    s = api.MDSystem(p)
    s.upload(r, v)
    return s


@pytest.fixture(scope="module")
def liquid(gpu_lib):
    # LJ rc 2.5 liquid at the large-config density, 2048 molecules, oracle-equilibrated
    r, v, dom, o = liquid_state([8, 8, 8], 0.8442, 0.722, 2.5, steps=150)
    return r, v, dom


def test_cfg1_fcc_kat(gpu_lib):
    r, v, dom = cfg1_state()
    s = gpu_system(r, v, dom, WCA_RC, tplot=100)
    s.setup()
    _, _, a, _ = s.download()
    assert np.all(a == 0.0), "FCC first shell lies beyond the WCA cutoff: forces must be exactly zero"
    pe, vir = s.per_molecule()
    assert np.all(pe == 0.0) and np.all(vir == 0.0)
    own, par, code = s.pair_list()
    assert np.all(np.bincount(own, minlength=len(r) + 1)[1:] == 12)
    o = O.Oracle(r, v, dom, WCA_RC, tplot=100)
    o.setup()
    assert np.array_equal(canonical_full(own, par, code), canonical_oracle(*o.pair_list()))


def test_pairs_forces_energies_fp64(liquid):
    r, v, dom = liquid
    o = O.Oracle(r, v, dom, 2.5, tplot=1, density=0.8442)
    o.setup()
    s = gpu_system(r, v, dom, 2.5, tplot=1, density=0.8442)
    s.setup()
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    pe, vir = s.per_molecule()
    np.testing.assert_allclose(pe, o.potenergymol, rtol=TOL64, atol=TOL64)
    np.testing.assert_allclose(vir, o.virialmol, rtol=TOL64, atol=TOL64)
    m = s.records()[-1]
    mo = o.macro()
    for k in ("kinenergy", "potenergy", "pressure", "temperature", "virial"):
        assert m[k] == pytest.approx(mo[k], rel=1e-12, abs=1e-12), k


def test_fp32_forces_within_tolerance(liquid):
    r, v, dom = liquid
    o = O.Oracle(r, v, dom, 2.5, tplot=1, density=0.8442)
    o.setup()
    s = gpu_system(r, v, dom, 2.5, precision=api.PRECISION_FP32, tplot=1, density=0.8442)
    s.setup()
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    err = rel_err(a, o.a, F_FLOOR32)
    assert err.max() <= TOL32, err.max()
    pe, vir = s.per_molecule()
    assert (np.abs(pe - o.potenergymol) / np.maximum(np.abs(o.potenergymol), 1.0)).max() <= TOL32
    assert (np.abs(vir - o.virialmol) / np.maximum(np.abs(o.virialmol), W_FLOOR32)).max() <= TOL32


def test_trajectory_fp64_follows_oracle(liquid):
    r, v, dom = liquid
    nsteps, tplot = 300, 50
    o = O.Oracle(r, v, dom, 2.5, tplot=tplot, density=0.8442)
    o.setup()
    recs_o = o.run_vv(nsteps)
    s = gpu_system(r, v, dom, 2.5, tplot=tplot, density=0.8442)
    s.setup()
    s.records()
    s.simulation_md(nsteps)
    recs = s.records()
    assert len(recs) == len(recs_o)
    assert s.counters()["rebuilds"] == o.rebuild_count
    for row, ro in zip(recs, recs_o):
        assert row["iter"] == int(ro[0])
        assert row["totenergy"] == pytest.approx(ro[6], rel=1e-10)
        assert row["pressure"] == pytest.approx(ro[7], rel=1e-9)
    rg, vg, _, _ = s.download()
    np.testing.assert_allclose(rg, o.r, rtol=0, atol=1e-8)
    np.testing.assert_allclose(vg, o.v, rtol=0, atol=1e-8)


def test_subroutine_path_equals_fused_loop(liquid):
    """md_advance_vv called subroutine by subroutine through the C ABI gives
    bit-identical state to the fused device loop."""
    r, v, dom = liquid
    a_sys = gpu_system(r, v, dom, 2.5, tplot=40, density=0.8442)
    a_sys.setup()
    for _ in range(60):
        a_sys.md_advance_vv()
    b_sys = gpu_system(r, v, dom, 2.5, tplot=40, density=0.8442)
    b_sys.setup()
    b_sys.simulation_md(60)
    ra, va, aa, _ = a_sys.download()
    rb, vb, ab, _ = b_sys.download()
    assert np.array_equal(ra, rb) and np.array_equal(va, vb) and np.array_equal(aa, ab)
    assert a_sys.counters()["rebuilds"] == b_sys.counters()["rebuilds"]


@pytest.mark.parametrize("integration", [1, 0])
@pytest.mark.parametrize("crit", [0, 2])
def test_step_graphs_equal_per_kernel_launches(liquid, monkeypatch, integration, crit):
    """The step graphs (the decision setting the condition of a rebuild body,
    eight middle iterations per launch) change no result bit against
    launching every kernel of a step on its own (FM_STEP_GRAPHS=0, read when a
    handle is created): 150 iterations with rebuilds and records, velocity
    Verlet and leap-frog, rebuild criteria 0 and 2.  The graphs launch fewer
    kernels: the rebuild kernels run only on rebuild steps."""
    r, v, dom = liquid
    out = []
    for env in ("1", "0"):
        monkeypatch.setenv("FM_STEP_GRAPHS", env)
        s = gpu_system(r, v, dom, 2.5, tplot=40, density=0.8442, integration_algorithm=integration,
                       rebuild_criteria=crit)
        s.setup()
        s.records()
        s.simulation_md(150)
        out.append((s.download(), s.records(), s.counters()["rebuilds"], s.launch_count()))
        s.close()
    (sa, ra, na, la), (sb, rb, nb, lb) = out
    for x, y in zip(sa, sb):
        assert np.array_equal(x, y)
    assert ra == rb and len(ra) == 3
    assert na == nb and na > 2
    assert la < lb


def test_rebuild_lists_equals_the_subroutine_sequence(liquid):
    """fm_rebuild_lists (the rebuild branch in one call) leaves the same
    state as the six subroutine mirrors called one by one: 40 iterations of
    md_advance_vv with either, bit for bit."""
    r, v, dom = liquid
    sys_a = gpu_system(r, v, dom, 2.5, tplot=40, density=0.8442)
    sys_a.setup()
    sys_b = gpu_system(r, v, dom, 2.5, tplot=40, density=0.8442)
    sys_b.setup()
    nreb = 0
    for _ in range(40):
        for s, whole in ((sys_a, False), (sys_b, True)):
            s.iter = s.iter + 1
            s.simulation_move_particles_vv(1)
            s.messenger_updateborders(0)
            if s.simulation_checkrebuild():
                nreb += whole
                if whole:
                    s.rebuild_lists()
                else:
                    s.linklist_deallocateall()
                    s.sendmols()
                    s.sort_mols()
                    s.assign_to_cell()
                    s.messenger_updateborders(1)
                    s.assign_to_neighbourlist()
            s.simulation_compute_forces()
            s.simulation_move_particles_vv(2)
    assert nreb > 0
    ra, va, aa, _ = sys_a.download()
    rb, vb, ab, _ = sys_b.download()
    assert np.array_equal(ra, rb) and np.array_equal(va, vb) and np.array_equal(aa, ab)
    sys_a.close()
    sys_b.close()


def test_all_pairs_matches_oracle(gpu_lib):
    r, v, dom = lattice.lj_fluid([3, 3, 3], 0.8, 1.0, 7)
    r = lattice.jitter(r, 0.08, 7, dom)
    o = O.Oracle(r, v, dom, 2.5, force_list=0, tplot=1)
    o.setup()
    s = gpu_system(r, v, dom, 2.5, force_list=0, tplot=1)
    s.setup()
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    recs_o = o.run_vv(100)
    s.simulation_md(100)
    rg, _, _, _ = s.download()
    np.testing.assert_allclose(rg, o.r, rtol=0, atol=1e-9)


def test_nlist_overflow_is_resized_and_resumed(liquid):
    r, v, dom = liquid
    ref = gpu_system(r, v, dom, 2.5, tplot=25, density=0.8442)
    ref.setup()
    ref.simulation_md(80)
    small = gpu_system(r, v, dom, 2.5, tplot=25, density=0.8442, nlist_capacity=8)
    small.setup()
    small.simulation_md(80)
    assert small.counters()["nlist_capacity"] > 8
    r1, v1, _, _ = ref.download()
    r2, v2, _, _ = small.download()
    assert np.array_equal(r1, r2) and np.array_equal(v1, v2)


def test_nlist_overflow_resumed_with_block_builds(gpu_lib):
    """The same resize-and-resume when the rows are built by 2x2x2-cell
    blocks (a sparse WCA fluid with too small a row capacity)."""
    r, v, dom = lattice.lj_fluid([7, 7, 7], 0.8, 1.0, 81)
    r = lattice.jitter(r, 0.05, 81, dom)
    ref = gpu_system(r, v, dom, WCA_RC, tplot=25, density=0.8, list_build=api.LIST_BUILD_BLOCKS)
    ref.setup()
    ref.simulation_md(80)
    small = gpu_system(r, v, dom, WCA_RC, tplot=25, density=0.8, list_build=api.LIST_BUILD_BLOCKS,
                       nlist_capacity=8)
    small.setup()
    small.simulation_md(80)
    assert small.counters()["nlist_capacity"] > 8
    r1, v1, _, _ = ref.download()
    r2, v2, _, _ = small.download()
    assert np.array_equal(r1, r2) and np.array_equal(v1, v2)


def test_escaped_molecule_is_an_error_code(gpu_lib):
    r, v, dom = cfg1_state()
    r = r.copy()
    r[5] = [3.0 * dom[0], 0.0, 0.0]
    s = gpu_system(r, v, dom, WCA_RC)
    with pytest.raises(api.FlowmolError) as e:
        s.setup()
    assert e.value.code == 4


def test_molecules_on_the_box_faces(gpu_lib):
    """Molecules exactly at -L/2 bin into the low halo cell (reference
    ceiling rule); the pair set still matches the oracle bit for bit."""
    r, v, dom = cfg1_state()
    r = r.copy()
    r[0, 0] = -dom[0] / 2
    r[1, 1] = -dom[1] / 2
    r[2, 2] = -dom[2] / 2
    o = O.Oracle(r, v, dom, WCA_RC, tplot=10 ** 6)
    o.setup()
    s = gpu_system(r, v, dom, WCA_RC)
    s.setup()
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))


def test_cutoff_edge_ulps(gpu_lib):
    """Pairs one ulp either side of rneighbr and rcutoff are classified like
    the FP64 reference (strict `<`)."""
    L = 20.0
    rc = 2.5
    rn = rc + 0.3
    xs = []
    for base in (rc, rn):
        for d in (np.nextafter(base, 0.0), base, np.nextafter(base, 10.0)):
            xs.append(d)
    rows = []
    for k, d in enumerate(xs):
        y = -8.0 + 2.9 * k
        rows += [[-d / 2, y, 0.0], [d / 2, y, 0.0]]
    r = np.array(rows)
    v = np.zeros_like(r)
    o = O.Oracle(r, v, [L, L, L], rc, tplot=1)
    o.setup()
    s = gpu_system(r, v, [L, L, L], rc, tplot=1)
    s.setup()
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    assert np.array_equal(a, o.a)


def test_large_system_pair_digest_and_forces(gpu_lib):
    """1,048,576 molecules (FCC 64^3, rho 0.8442, rc 2.5): the pair-set digest
    equals the oracle's, and FP64 forces agree within 1e-12."""
    r, v, dom = lattice.lj_fluid([64, 64, 64], 0.8442, 0.722, lattice.SEED_BASE + 2)
    r = lattice.jitter(r, 0.04, 11, dom)
    o = O.Oracle(r, v, dom, 2.5, tplot=1, density=0.8442)
    o.setup()
    dig_o = digest_oracle(*o.pair_list())
    s = gpu_system(r, v, dom, 2.5, tplot=1, density=0.8442)
    s.setup()
    assert s.pair_digest() == dig_o
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    s32 = gpu_system(r, v, dom, 2.5, tplot=1, density=0.8442, precision=api.PRECISION_FP32)
    s32.setup()
    _, _, a32, _ = s32.download()
    assert rel_err(a32, o.a, F_FLOOR32).max() <= TOL32


def wrap_diff(a, b, dom):
    d = np.asarray(a) - np.asarray(b)
    dom = np.asarray(dom)
    return d - dom * np.round(d / dom)


def test_leapfrog_trajectory_follows_oracle(liquid):
    """md_advance_lfv (forces, record, move, rebuild check) on the device."""
    r, v, dom = liquid
    nsteps, tplot = 300, 50
    o = O.Oracle(r, v, dom, 2.5, tplot=tplot, density=0.8442, integration_algorithm=0)
    o.setup()
    recs_o = o.run_lfv(nsteps)
    s = gpu_system(r, v, dom, 2.5, tplot=tplot, density=0.8442, integration_algorithm=0)
    s.setup()
    s.records()
    s.simulation_md(nsteps)
    recs = s.records()
    assert len(recs) == len(recs_o)
    for row, ro in zip(recs, recs_o):
        assert row["iter"] == int(ro[0])
        assert row["kinenergy"] == pytest.approx(ro[4], rel=1e-10)
        assert row["totenergy"] == pytest.approx(ro[6], rel=1e-10)
    rg, vg, _, _ = s.download()
    assert np.abs(wrap_diff(rg, o.r, dom)).max() < 1e-8
    np.testing.assert_allclose(vg, o.v, rtol=0, atol=1e-8)


def test_leapfrog_subroutines_equal_fused_loop(liquid):
    r, v, dom = liquid
    a_sys = gpu_system(r, v, dom, 2.5, tplot=40, density=0.8442, integration_algorithm=0)
    a_sys.setup()
    for _ in range(60):
        a_sys.md_advance_lfv()
    b_sys = gpu_system(r, v, dom, 2.5, tplot=40, density=0.8442, integration_algorithm=0)
    b_sys.setup()
    b_sys.simulation_md(60)
    ra, va, _, _ = a_sys.download()
    rb, vb, _, _ = b_sys.download()
    assert np.array_equal(ra, rb) and np.array_equal(va, vb)


def test_reference_restart_liquid_vapour_state(gpu_lib):
    """The reference's runs/Intrinsic_Interface/initial_state (2635 molecules,
    liquid slab + vapour, rc 2.5), read with the library's final_state
    reader: pair set bit-exact and FP64 forces within 1e-12 of the oracle."""
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "intrinsic_interface_initial_state.bin")
    h, a = api.read_final_state(path)
    dom = list(h.globaldomain)
    delta = (h.delta_rneighbr,) * 3
    o = O.Oracle(a["r"], a["v"], dom, h.rcutoff, delta, tplot=1, density=h.density)
    o.setup()
    p = api.make_params(h.globalnp, dom, h.rcutoff, delta, h.delta_t, tplot=1, density=h.density)
    s = api.MDSystem(p)
    s.upload(a["r"], a["v"], glob_no=a["glob_no"])
    s.setup()
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, acc, _ = s.download()
    assert rel_err(acc, o.a, 1.0).max() <= TOL64
    pe, vir = s.per_molecule()
    np.testing.assert_allclose(pe, o.potenergymol, rtol=TOL64, atol=TOL64)


def test_fene_melt_bonds_forces_trajectory(gpu_lib):
    """FENE bead-spring melt (512 chains of 8, WCA + FENE k=30, R0=1.5, the
    rneighbr = R0 override): bonds found at list build equal the reference's
    check_update_adjacentbeadinfo set, pair set bit-exact, forces 1e-12."""
    from flowmol_b200 import polymer
    r, v, ch, sub, fy, bf, dom = polymer.fene_melt(512)
    o = O.Oracle(r, v, dom, WCA_RC, tplot=20, potential_flag=1, k_c=30.0, R_0=1.5, density=0.85)
    o.set_monomers(ch, sub, fy, bf)
    o.setup()
    s = gpu_system(r, v, dom, WCA_RC, tplot=20, density=0.85, potential_flag=1, k_c=30.0, R_0=1.5)
    s.upload_monomers(ch, sub, bf)
    s.setup()
    key = lambda t: np.sort((t[0].astype(np.int64) << 32) | (t[1].astype(np.int64) << 5) | t[2])  # noqa: E731
    assert np.array_equal(key(s.bonds()), key(o.bond_list()))
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    recs_o = o.run_vv(100)
    s.records()
    s.simulation_md(100)
    recs = s.records()
    assert [r_["iter"] for r_ in recs] == [int(x) for x in recs_o[:, 0]]
    for row, ro in zip(recs, recs_o):
        assert row["potenergy"] == pytest.approx(ro[5], rel=1e-9)
    rg, _, _, _ = s.download()
    assert np.abs(wrap_diff(rg, o.r, dom)).max() < 1e-7


def test_cfg1_nve_energy_drift_1e4_steps(gpu_lib):
    """NVE drift over 10^4 steps on the plain configuration (2048 molecules,
    WCA, dt 0.005): the FP64 and FP32 forms and the FP64 oracle all conserve
    the total energy per molecule to well below 1e-3 relative, and the GPU
    forms' records agree with the oracle's (same iterations; total energy to
    1e-3: the trajectories separate by chaos within a few thousand steps and
    the energy then fluctuates around the same value with a different phase)."""
    r, v, dom = cfg1_state()
    nsteps, tplot = 10000, 1000
    o = O.Oracle(r, v, dom, WCA_RC, tplot=tplot)
    o.setup()
    recs_o = o.run_vv(nsteps)
    e_o = recs_o[:, 6]
    drifts = {"oracle": (e_o[-1] - e_o[0]) / abs(e_o[0])}
    assert np.abs(e_o - e_o[0]).max() / abs(e_o[0]) < 1e-3
    for prec, name in ((api.PRECISION_FP64, "fp64"), (api.PRECISION_FP32, "fp32")):
        s = gpu_system(r, v, dom, WCA_RC, precision=prec, tplot=tplot)
        s.setup()
        s.records()  # the setup record (iteration 0)
        s.simulation_md(nsteps)
        recs = s.records()
        s.close()
        assert [x["iter"] for x in recs] == [int(x) for x in recs_o[:, 0]]
        e = np.array([x["totenergy"] for x in recs])
        drifts[name] = (e[-1] - e[0]) / abs(e[0])
        assert np.abs(e - e[0]).max() / abs(e[0]) < 1e-3, (name, e)
        np.testing.assert_allclose(e, e_o, rtol=1e-3)
    print("\ncfg1 NVE relative drift over %d steps: " % nsteps +
          ", ".join("%s %.3e" % (k, x) for k, x in drifts.items()))


def test_mie_mixture_forces_and_trajectory(liquid):
    """Mie_potential 1, two types with different exponents, epsilons and
    masses: pair set bit-exact, a = F/m and per-molecule PE to 1e-12 (FP64;
    the kernels' real powers against the oracle's libm), FP32 within 1e-5,
    and 100 velocity-Verlet steps that follow the oracle."""
    from helpers import mie_mixture_tables
    r, v, dom = liquid
    mt = (np.arange(len(r)) % 2 + 1).astype(np.int32)
    tab = mie_mixture_tables(2.5)
    o = O.Oracle(r, v, dom, 2.5, tplot=20, density=0.8442)
    o.set_mie(tab, mt)
    o.setup()
    s = gpu_system(r, v, dom, 2.5, tplot=20, density=0.8442)
    s.set_mie(tab, mt)
    s.setup()
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    pe, _ = s.per_molecule()
    np.testing.assert_allclose(pe, o.potenergymol, rtol=TOL64, atol=TOL64)
    s32 = gpu_system(r, v, dom, 2.5, tplot=20, density=0.8442, precision=api.PRECISION_FP32)
    s32.set_mie(tab, mt)
    s32.setup()
    _, _, a32, _ = s32.download()
    assert rel_err(a32, o.a, F_FLOOR32).max() <= TOL32
    s32.close()
    recs_o = o.run_vv(100)
    s.records()
    s.simulation_md(100)
    recs = s.records()
    assert [x["iter"] for x in recs] == [int(x) for x in recs_o[:, 0]]
    for row, ro in zip(recs, recs_o):
        assert row["kinenergy"] == pytest.approx(ro[4], rel=1e-9)
        assert row["totenergy"] == pytest.approx(ro[6], rel=1e-9)
    rg, _, _, _ = s.download()
    assert np.abs(wrap_diff(rg, o.r, dom)).max() < 1e-7


def test_mie_polymer_harmonic_bonds(gpu_lib):
    """Mie_potential 1 on a bead-spring melt: bonds become harmonic
    (k 295.3322, r0 1, setup_set_parameters.f90:873, 1215) -- the same bonds
    found, forces to 1e-12, records over 100 steps."""
    from flowmol_b200 import polymer
    from helpers import mie_tables
    r, v, ch, sub, fy, bf, dom = polymer.fene_melt(512)
    tab = mie_tables(WCA_RC, [[1.0]], [[12.0]], [[6.0]], [1.0], k=[[295.3322]], r0=[[1.0]])
    mt = np.ones(len(r), np.int32)
    o = O.Oracle(r, v, dom, WCA_RC, tplot=20, potential_flag=1, k_c=30.0, R_0=1.5, density=0.85)
    o.set_monomers(ch, sub, fy, bf)
    o.set_mie(tab, mt)
    o.setup()
    s = gpu_system(r, v, dom, WCA_RC, tplot=20, density=0.85, potential_flag=1, k_c=30.0, R_0=1.5)
    s.upload_monomers(ch, sub, bf)
    s.set_mie(tab, mt)
    s.setup()
    key = lambda t: np.sort((t[0].astype(np.int64) << 32) | (t[1].astype(np.int64) << 5) | t[2])  # noqa: E731
    assert np.array_equal(key(s.bonds()), key(o.bond_list()))
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    recs_o = o.run_vv(100)
    s.records()
    s.simulation_md(100)
    recs = s.records()
    assert [x["iter"] for x in recs] == [int(x) for x in recs_o[:, 0]]
    for row, ro in zip(recs, recs_o):
        assert row["potenergy"] == pytest.approx(ro[5], rel=1e-9)


@pytest.mark.parametrize("prec", [api.PRECISION_FP64, api.PRECISION_FP32])
def test_soddemann_polymer_solution(gpu_lib, prec):
    """SOLVENT_INFO 1: 8-bead FENE chains in as many solvent molecules
    (chainID 0), WCA + the Soddemann well (eps_pp 1.5, eps_ps 1.0, eps_ss 0.5)
    + FENE bonds.  The Soddemann geometry (cells of rcutoff 1.5 + skin, list
    range rneighbr 1.42246), bonds and pair set bit-exact; forces to 1e-12
    (FP64) or 1e-5 (FP32 pair magnitudes); per-molecule PE; 100 steps."""
    from flowmol_b200 import polymer
    r, v, ch, sub, fy, bf, dom = polymer.fene_solution(192, targetconc=0.5)
    r = lattice.jitter(r, 0.08, 92, dom)  # off the lattice: pairs in the cosine well from the start
    eps = (1.5, 1.0, 0.5)
    o = O.Oracle(r, v, dom, WCA_RC, tplot=20, potential_flag=1, k_c=30.0, R_0=1.5, density=0.85)
    o.set_monomers(ch, sub, fy, bf)
    o.set_solvent(1, *eps)
    o.setup()
    s = gpu_system(r, v, dom, WCA_RC, precision=prec, tplot=20, density=0.85, potential_flag=1, k_c=30.0,
                   R_0=1.5, solvent_flag=1, eps=eps)
    s.upload_monomers(ch, sub, bf)
    s.setup()
    key = lambda t: np.sort((t[0].astype(np.int64) << 32) | (t[1].astype(np.int64) << 5) | t[2])  # noqa: E731
    assert np.array_equal(key(s.bonds()), key(o.bond_list()))
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    pe, _ = s.per_molecule()
    if prec == api.PRECISION_FP32:
        assert rel_err(a, o.a, F_FLOOR32).max() <= TOL32
        s.close()
        return
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    np.testing.assert_allclose(pe, o.potenergymol, rtol=TOL64, atol=TOL64)
    recs_o = o.run_vv(100)
    s.records()
    s.simulation_md(100)
    recs = s.records()
    assert [x["iter"] for x in recs] == [int(x) for x in recs_o[:, 0]]
    for row, ro in zip(recs, recs_o):
        assert row["potenergy"] == pytest.approx(ro[5], rel=1e-9)
    rg, _, _, _ = s.download()
    assert np.abs(wrap_diff(rg, o.r, dom)).max() < 1e-7
    s.close()


@pytest.mark.parametrize("prec", [api.PRECISION_FP64, api.PRECISION_FP32])
def test_mie_soddemann_polymer_solution(gpu_lib, prec):
    """Mie_potential 1 with SOLVENT_INFO 1 (simulation_compute_forces.f90
    :839-872): the WCA branch of the Soddemann force is Mie_accijmag of the
    pair's types (get_accijmag) while its energy stays the LJ-WCA
    expression, the pair accelerations are not divided by a mass but the
    harmonic bonds are (:752-754), and the kinetic sums are mass-weighted.
    A two-type solution (types alternate over the molecules, masses 1 and
    1.5): bonds and pair set bit-exact, forces to 1e-12 (FP64) or 1e-5 (FP32
    pair magnitudes), per-molecule PE, and 100 steps in FP64."""
    from flowmol_b200 import polymer
    from helpers import mie_mixture_tables
    r, v, ch, sub, fy, bf, dom = polymer.fene_solution(192, targetconc=0.5)
    r = lattice.jitter(r, 0.08, 93, dom)
    eps = (1.5, 1.0, 0.5)
    tab = mie_mixture_tables(WCA_RC)
    mt = (np.arange(len(r)) % 2 + 1).astype(np.int32)
    o = O.Oracle(r, v, dom, WCA_RC, tplot=20, potential_flag=1, k_c=30.0, R_0=1.5, density=0.85)
    o.set_monomers(ch, sub, fy, bf)
    o.set_solvent(1, *eps)
    o.set_mie(tab, mt)
    o.setup()
    s = gpu_system(r, v, dom, WCA_RC, precision=prec, tplot=20, density=0.85, potential_flag=1, k_c=30.0,
                   R_0=1.5, solvent_flag=1, eps=eps)
    s.upload_monomers(ch, sub, bf)
    s.set_mie(tab, mt)
    s.setup()
    key = lambda t: np.sort((t[0].astype(np.int64) << 32) | (t[1].astype(np.int64) << 5) | t[2])  # noqa: E731
    assert np.array_equal(key(s.bonds()), key(o.bond_list()))
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    pe, _ = s.per_molecule()
    if prec == api.PRECISION_FP32:
        assert rel_err(a, o.a, F_FLOOR32).max() <= TOL32
        s.close()
        return
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    np.testing.assert_allclose(pe, o.potenergymol, rtol=TOL64, atol=TOL64)
    recs_o = o.run_vv(100)
    s.records()
    s.simulation_md(100)
    recs = s.records()
    assert [x["iter"] for x in recs] == [int(x) for x in recs_o[:, 0]]
    for row, ro in zip(recs, recs_o):
        assert row["kinenergy"] == pytest.approx(ro[4], rel=1e-9)
        assert row["potenergy"] == pytest.approx(ro[5], rel=1e-9)
    rg, _, _, _ = s.download()
    assert np.abs(wrap_diff(rg, o.r, dom)).max() < 1e-7
    s.close()


@pytest.mark.parametrize("crit,fixed", [(0, 1), (1, 7), (2, 1)])
def test_rebuild_criteria_schedule(liquid, crit, fixed):
    """REBUILD_CRITERIA 0 (Rapaport vmax), 1 (every FIXED_REBUILD steps) and 2
    (exact per-molecule displacement, simulation_checkrebuild.f90:83-121):
    the device decides the same rebuilds as the oracle over 300 steps (plus the
    record-forced ones, :34) and the trajectories agree."""
    r, v, dom = liquid
    o = O.Oracle(r, v, dom, 2.5, tplot=50, density=0.8442, rebuild_criteria=crit, fixed_rebuild=fixed)
    o.setup()
    o.run_vv(300)
    s = gpu_system(r, v, dom, 2.5, tplot=50, density=0.8442, rebuild_criteria=crit, fixed_rebuild=fixed)
    s.setup()
    s.simulation_md(300)
    assert s.counters()["rebuilds"] == o.rebuild_count
    if crit == 1:
        assert o.rebuild_count == len([i for i in range(1, 301) if i % fixed == 0 or (i + 1) % 50 == 0])
    rg, _, _, _ = s.download()
    assert np.abs(wrap_diff(rg, o.r, dom)).max() < 1e-7
    s.close()


@pytest.mark.parametrize("case", ["half", "full", "lfv", "fene", "allpairs"])
def test_pressure_tensor_single_system(liquid, case):
    """PRESSURE_OUTFLAG 1 on the single-system path: the time-averaged virial
    pressure tensor sum_i (v v + rf/2)/V over the record steps (cumulative_
    pressure, simulation_record.f90:3151-3220) equals the oracle's for the
    half and full lists, leap-frog, FENE bonds (rf from the bond loop too)
    and all pairs (kinetic part only: LJ_AP records no rf); none at setup."""
    from flowmol_b200 import polymer
    kw, okw, mono = {}, {}, None
    rc, rho = 2.5, 0.8442
    if case == "fene":
        r, v, ch, sub, fy, bf, dom = polymer.fene_melt(256)
        rc, rho = WCA_RC, 0.85
        kw = okw = dict(potential_flag=1, k_c=30.0, R_0=1.5)
        mono = (ch, sub, fy, bf)
    elif case == "allpairs":
        r, v, dom = lattice.lj_fluid([3, 3, 3], 0.8, 1.0, 17)
        kw = okw = dict(force_list=0)
        rho = 0.8
    else:
        r, v, dom = liquid
        if case == "full":
            kw = okw = dict(force_list=2)
        if case == "lfv":
            kw = okw = dict(integration_algorithm=0)
    o = O.Oracle(r, v, dom, rc, tplot=10, density=rho, **okw)
    if mono is not None:
        o.set_monomers(*mono)
    o.set_pressure(1)
    o.setup()
    if case == "lfv":
        o.run_lfv(100)
    else:
        o.run_vv(100)
    po, no = o.pressure_average()
    s = gpu_system(r, v, dom, rc, tplot=10, density=rho, **kw)
    if mono is not None:
        s.upload_monomers(mono[0], mono[1], mono[3])
    s.set_pressure_outflag(1)
    s.setup()
    s.simulation_md(100)
    pg, ng = s.pressure_tensor()
    assert ng == no == 10
    np.testing.assert_allclose(pg, po, rtol=1e-9, atol=1e-9 * np.abs(po).max())
    assert np.allclose(pg, pg.T, rtol=1e-12, atol=1e-12 * np.abs(pg).max())
    pr, nr = s.pressure_tensor(reset=True)
    assert nr == 10 and s.pressure_tensor()[1] == 0
    s.close()


@pytest.mark.parametrize("prec", [api.PRECISION_FP64, api.PRECISION_FP32])
def test_dense_cells_beyond_one_warp(gpu_lib, prec):
    """Cells holding more than 32 molecules (rho 1.05, skin 0.8: cell side
    3.3, ~38 per cell): the build's second owner pass, the per-cell sort's
    one-lane path for large cells and the list's wide rows, against the
    oracle -- pair set bit-exact, forces to 1e-12 (FP64) or 1e-5 (FP32), and
    60 steps with rebuilds."""
    r, v, dom = lattice.lj_fluid([8, 8, 8], 1.05, 1.2, 93)
    r = lattice.jitter(r, 0.04, 93, dom)
    skin = (0.8, 0.8, 0.8)
    o = O.Oracle(r, v, dom, 2.5, skin, tplot=20, density=1.05)
    o.setup()
    g = o.geometry()
    per_cell = len(r) / np.prod(g["ncells"])
    assert per_cell > 32, per_cell
    s = gpu_system(r, v, dom, 2.5, precision=prec, tplot=20, density=1.05, delta_rneighbr=skin)
    s.setup()
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    if prec == api.PRECISION_FP32:
        assert rel_err(a, o.a, F_FLOOR32).max() <= TOL32
        s.close()
        return
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    o.run_vv(60)
    s.simulation_md(60)
    assert s.counters()["rebuilds"] == o.rebuild_count > 0
    rg, _, _, _ = s.download()
    assert np.abs(wrap_diff(rg, o.r, dom)).max() < 1e-7
    s.close()


def test_two_molecules_in_the_cell_path(gpu_lib):
    """The smallest list-path system: two molecules in a box of 3x3x3 cells
    (all other cells empty), one pair inside r_c: the force is the two-body
    LJ force, equal and opposite, and 30 steps follow the oracle."""
    L = 8.5
    r = np.array([[-0.6, 0.1, 0.2], [0.55, 0.1, 0.25]])
    v = np.array([[0.3, -0.1, 0.05], [-0.3, 0.1, -0.05]])
    o = O.Oracle(r, v, [L, L, L], 2.5, tplot=10)
    o.setup()
    s = gpu_system(r, v, [L, L, L], 2.5, tplot=10)
    s.setup()
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    assert np.abs(a[0] + a[1]).max() <= 1e-12 * np.abs(a).max()
    o.run_vv(30)
    s.simulation_md(30)
    rg, vg, _, _ = s.download()
    assert np.abs(wrap_diff(rg, o.r, [L, L, L])).max() < 1e-10
    s.close()


def test_pressure_tensor_mie_mixture(liquid):
    """The pressure tensor of a two-type Mie fluid with unequal masses: the
    pair term uses the Mie accijmag, the kinetic term v v has no mass factor
    (cumulative_pressure, simulation_record.f90:3170-3199), as in the oracle."""
    from helpers import mie_mixture_tables
    r, v, dom = liquid
    mt = (np.arange(len(r)) % 2 + 1).astype(np.int32)
    tab = mie_mixture_tables(2.5)
    o = O.Oracle(r, v, dom, 2.5, tplot=10, density=0.8442)
    o.set_mie(tab, mt)
    o.set_pressure(1)
    o.setup()
    o.run_vv(50)
    po, no = o.pressure_average()
    s = gpu_system(r, v, dom, 2.5, tplot=10, density=0.8442)
    s.set_mie(tab, mt)
    s.set_pressure_outflag(1)
    s.setup()
    s.simulation_md(50)
    pg, ng = s.pressure_tensor()
    assert ng == no == 5
    np.testing.assert_allclose(pg, po, rtol=1e-9, atol=1e-9 * np.abs(po).max())
    s.close()


@pytest.mark.parametrize("crit", [0, 2])
def test_soddemann_leapfrog_trajectory(gpu_lib, crit):
    """Soddemann polymer solution under leap-frog (INTEGRATION_ALGORITHM 0),
    with the Rapaport and the exact-displacement rebuild criteria: the same
    rebuilds as the oracle, records and positions after 80 steps."""
    from flowmol_b200 import polymer
    r, v, ch, sub, fy, bf, dom = polymer.fene_solution(96, targetconc=0.5)
    r = lattice.jitter(r, 0.08, 94, dom)
    eps = (1.5, 1.0, 0.5)
    kw = dict(potential_flag=1, k_c=30.0, R_0=1.5, integration_algorithm=0, rebuild_criteria=crit)
    o = O.Oracle(r, v, dom, WCA_RC, tplot=20, density=0.85, **kw)
    o.set_monomers(ch, sub, fy, bf)
    o.set_solvent(1, *eps)
    o.setup()
    recs_o = o.run_lfv(80)
    s = gpu_system(r, v, dom, WCA_RC, tplot=20, density=0.85, solvent_flag=1, eps=eps, **kw)
    s.upload_monomers(ch, sub, bf)
    s.setup()
    s.records()
    s.simulation_md(80)
    recs = s.records()
    assert s.counters()["rebuilds"] == o.rebuild_count > 0
    assert [x["iter"] for x in recs] == [int(x) for x in recs_o[:, 0]]
    for row, ro in zip(recs, recs_o):
        assert row["potenergy"] == pytest.approx(ro[5], rel=1e-9)
        assert row["kinenergy"] == pytest.approx(ro[4], rel=1e-9)
    rg, _, _, _ = s.download()
    assert np.abs(wrap_diff(rg, o.r, dom)).max() < 1e-7
    s.close()


@pytest.mark.parametrize("case", ["wca", "lj", "fene", "faces"])
def test_list_build_cells_equals_blocks(gpu_lib, case):
    """The per-cell and the 2x2x2-block list builds give identical rows (same
    partners in the same order), equal to the oracle's pair set; odd cell
    counts (partial blocks), box faces and polymers included."""
    from flowmol_b200 import polymer
    kw = {}
    mono = None
    if case == "wca":
        r, v, dom = lattice.lj_fluid([7, 7, 7], 0.8, 1.0, 71)
        r = lattice.jitter(r, 0.05, 71, dom)
        rc, rho = WCA_RC, 0.8
    elif case == "lj":
        r, v, dom = lattice.lj_fluid([7, 6, 8], 0.8442, 0.722, 72)
        r = lattice.jitter(r, 0.05, 72, dom)
        rc, rho = 2.5, 0.8442
    elif case == "faces":
        r, v, dom = lattice.lj_fluid([7, 7, 7], 0.8, 1.0, 73)
        r = r - r.min(axis=0) - 0.5 * np.asarray(dom)  # molecules exactly on the -L/2 faces
        rc, rho = WCA_RC, 0.8
    else:
        r, v, ch, sub, fy, bf, dom = polymer.fene_melt(300)
        rc, rho = WCA_RC, 0.85
        kw = dict(potential_flag=1, k_c=30.0, R_0=1.5)
        mono = (ch, sub, bf, fy)
    rows = {}
    for mode in (api.LIST_BUILD_CELLS, api.LIST_BUILD_BLOCKS):
        s = gpu_system(r, v, dom, rc, density=rho, list_build=mode, **kw)
        if mono is not None:
            s.upload_monomers(*mono[:3])
        s.setup()
        rows[mode] = s.pair_list()
        if mono is not None:
            rows[(mode, "bonds")] = s.bonds()
        _, _, a, _ = s.download()
        rows[(mode, "a")] = a
        s.close()
    c, b = rows[api.LIST_BUILD_CELLS], rows[api.LIST_BUILD_BLOCKS]
    for x, y in zip(c, b):
        assert np.array_equal(x, y)  # same rows, same order
    assert np.array_equal(rows[(api.LIST_BUILD_CELLS, "a")], rows[(api.LIST_BUILD_BLOCKS, "a")])
    if mono is not None:
        for x, y in zip(rows[(api.LIST_BUILD_CELLS, "bonds")], rows[(api.LIST_BUILD_BLOCKS, "bonds")]):
            assert np.array_equal(x, y)
    o = O.Oracle(r, v, dom, rc, density=rho, **kw)
    if mono is not None:
        o.set_monomers(mono[0], mono[1], mono[3], mono[2])
    o.setup()
    assert np.array_equal(canonical_full(*b), canonical_oracle(*o.pair_list()))


# ---------------------------------------------------------------------------
# The two force kernels of the neighbour-list modes: one gather per list entry
# (FORCE_PATH_GATHER, the automatic choice, which the tests above run) and the
# tiled kernel (FORCE_PATH_TILES: the block's neighbourhood staged in shared
# memory, 16-bit offsets in the rows).  These pin both explicitly.
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("prec", [api.PRECISION_FP64, api.PRECISION_FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("path,tpm", [(api.FORCE_PATH_GATHER, 0), (api.FORCE_PATH_TILES, 4),
                                      (api.FORCE_PATH_TILES, 8)], ids=["gather", "tiles4", "tiles8"])
def test_force_paths_pairs_forces_energies(liquid, prec, path, tpm):
    r, v, dom = liquid
    o = O.Oracle(r, v, dom, 2.5, tplot=1, density=0.8442)
    o.setup()
    s = gpu_system(r, v, dom, 2.5, precision=prec, tplot=1, density=0.8442, force_path=path,
                   threads_per_molecule=tpm)
    s.setup()
    assert s.force_path()[0] == path
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    pe, vir = s.per_molecule()
    if prec == api.PRECISION_FP64:
        assert rel_err(a, o.a, 1.0).max() <= TOL64
        np.testing.assert_allclose(pe, o.potenergymol, rtol=TOL64, atol=TOL64)
        np.testing.assert_allclose(vir, o.virialmol, rtol=TOL64, atol=TOL64)
    else:
        assert rel_err(a, o.a, F_FLOOR32).max() <= TOL32
        assert (np.abs(pe - o.potenergymol) / np.maximum(np.abs(o.potenergymol), 1.0)).max() <= TOL32
        assert (np.abs(vir - o.virialmol) / np.maximum(np.abs(o.virialmol), W_FLOOR32)).max() <= TOL32
    m = s.records()[-1]
    mo = o.macro()
    tol = 1e-12 if prec == api.PRECISION_FP64 else TOL32
    for k in ("kinenergy", "potenergy", "pressure", "virial"):
        assert m[k] == pytest.approx(mo[k], rel=tol, abs=tol), k
    s.close()


def test_tiled_and_gather_trajectories_agree(liquid):
    """300 velocity-Verlet steps with rebuilds and records: the tiled kernel
    and the per-entry gather kernel sum the same pairs (in different orders),
    so positions agree to 1e-9 and the records to 1e-10; the rebuild schedule
    is identical."""
    r, v, dom = liquid
    runs = []
    for path in (api.FORCE_PATH_GATHER, api.FORCE_PATH_TILES):
        s = gpu_system(r, v, dom, 2.5, tplot=50, density=0.8442, force_path=path)
        s.setup()
        s.records()
        s.simulation_md(300)
        runs.append((s.download(), s.records(), s.counters()["rebuilds"]))
        s.close()
    (ra, va, _, _), reca, nra = runs[0]
    (rb, vb, _, _), recb, nrb = runs[1]
    assert nra == nrb and nra > 0
    np.testing.assert_allclose(rb, ra, rtol=0, atol=1e-9)
    np.testing.assert_allclose(vb, va, rtol=0, atol=1e-9)
    assert len(reca) == len(recb)
    for x, y in zip(reca, recb):
        assert x["iter"] == y["iter"]
        assert y["totenergy"] == pytest.approx(x["totenergy"], rel=1e-10)
        assert y["pressure"] == pytest.approx(x["pressure"], rel=1e-9)


def test_tiled_staging_grows_then_leaves_tiles(gpu_lib):
    """A dense cube (rho 1.5, 10,976 molecules) in a dilute box with rc 4.5:
    the staging capacity estimated from the mean density is too small (the
    first build raises the staging overflow and the host grows it), and a
    block whose 4x4x4 cells lie inside the cube holds ~10,600 candidates --
    more than shared memory takes -- so the handle leaves the tiled path for
    the gather path.  Pair set and forces still match the oracle."""
    rc = 4.5
    rr, _, _ = lattice.lj_fluid([14, 14, 14], 1.5, 1.0, 81)
    dom = np.array([38.4, 38.4, 38.4])
    rr = rr - rr.mean(axis=0)
    rng = np.random.default_rng(81)
    v = rng.normal(0.0, 1.0, rr.shape)
    o = O.Oracle(rr, v, dom, rc, tplot=1)
    o.setup()
    s = gpu_system(rr, v, dom, rc, tplot=1, force_path=api.FORCE_PATH_TILES)
    assert s.force_path()[0] == api.FORCE_PATH_TILES
    s.setup()
    assert s.force_path()[0] == api.FORCE_PATH_GATHER
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    s.close()


def test_tiled_staging_grows_on_a_liquid_vapour_slab(gpu_lib):
    """Liquid and vapour in one box (a liquid slab at rho 0.8 filling a third
    of the box, vapour elsewhere): the capacity estimated from the mean
    density is below the slab's neighbourhoods, so the first build grows it;
    the handle stays on the tiled path and matches the oracle."""
    rl, _, doml = lattice.lj_fluid([8, 8, 8], 0.8, 1.0, 82)
    dom = np.array([3.0 * doml[0], doml[1], doml[2]])
    rl = lattice.jitter(rl, 0.03, 82, doml)
    rng = np.random.default_rng(82)
    v = rng.normal(0.0, 0.8, rl.shape)
    s = gpu_system(rl, v, dom, 2.5, tplot=1, force_path=api.FORCE_PATH_TILES)
    cap0 = s.force_path()[1]
    s.setup()
    path, cap = s.force_path()
    assert path == api.FORCE_PATH_TILES and cap > cap0
    o = O.Oracle(rl, v, dom, 2.5, tplot=1)
    o.setup()
    assert np.array_equal(canonical_full(*s.pair_list()), canonical_oracle(*o.pair_list()))
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    s.close()


def test_tiled_nlist_overflow_is_resized_and_resumed(liquid):
    """A tiled handle whose rows overflow is grown and resumed from the
    failing iteration, bit for bit as a run with enough capacity."""
    r, v, dom = liquid
    runs = []
    for cap in (0, 8):
        s = gpu_system(r, v, dom, 2.5, tplot=25, density=0.8442, nlist_capacity=cap,
                       force_path=api.FORCE_PATH_TILES, threads_per_molecule=4)
        s.setup()
        s.simulation_md(80)
        assert s.force_path()[0] == api.FORCE_PATH_TILES
        runs.append((s.download(), s.counters()["nlist_capacity"]))
        s.close()
    (r1, v1, _, _), _ = runs[0]
    (r2, v2, _, _), cap2 = runs[1]
    assert cap2 > 8
    assert np.array_equal(r1, r2) and np.array_equal(v1, v2)


def _angular_melt():
    """A bead-spring melt (512 chains of 8, rho 0.85) whose chains with any bead
    within 2.2 cells of a box face are turned to solvent, so no bead of an
    angular triple has a halo image (where the reference's routine reads
    incomplete halo bond rows); types alternate along a chain (1, 2, 1, 2, ...;
    solvent 1), masses 1 and 1.5, harmonic bonds (Mie_potential 1)."""
    from flowmol_b200 import polymer
    from helpers import mie_tables
    r, v, ch, sub, fy, bf, dom = polymer.fene_melt(512)
    _, nc, cs, _ = O.cells(dom, WCA_RC, (0.3, 0.3, 0.3), potential_flag=1, R_0=1.5)
    lim = 0.5 * dom - 2.2 * cs
    near = np.any(np.abs(r) > lim, axis=1)
    drop = np.unique(ch[near])
    ch, sub, fy, bf = polymer.mark_solvent(ch, sub, fy, bf, drop)
    mt = np.where((ch != 0) & (sub % 2 == 0), 2, 1).astype(np.int32)
    tab = mie_tables(WCA_RC, np.ones((2, 2)), np.full((2, 2), 12.0), np.full((2, 2), 6.0), [1.0, 1.5],
                     k=np.full((2, 2), 295.3322), r0=np.ones((2, 2)))
    kk = np.zeros((2, 2, 2)); tt = np.zeros((2, 2, 2))
    kk[0, 1, 0], tt[0, 1, 0] = 4.3196, 2.7751
    kk[1, 0, 1], tt[1, 0, 1] = 3.1, 2.5
    return r, v, ch, sub, fy, bf, dom, mt, tab, kk, tt


def test_angular_potential_forces_and_trajectory(gpu_lib):
    """angular_potential 1 on interior chains: the angular forces with the
    reference's i/k roles (its bond discovery order), forces to 1e-12 and
    positions to 1e-9 after 100 velocity-Verlet steps against the oracle."""
    r, v, ch, sub, fy, bf, dom, mt, tab, kk, tt = _angular_melt()
    assert np.sum(fy == 2) > 300  # enough middle beads left
    o = O.Oracle(r, v, dom, WCA_RC, tplot=20, potential_flag=1, k_c=30.0, R_0=1.5, density=0.85)
    o.set_monomers(ch, sub, fy, bf)
    o.set_mie(tab, mt)
    o.set_angular(kk, tt)
    o.setup()
    s = gpu_system(r, v, dom, WCA_RC, tplot=20, density=0.85, potential_flag=1, k_c=30.0, R_0=1.5)
    s.upload_monomers(ch, sub, bf)
    s.set_mie(tab, mt)
    s.set_angular(kk, tt, fy)
    s.setup()
    _, _, a, _ = s.download()
    assert rel_err(a, o.a, 1.0).max() <= TOL64
    o.run_vv(100)
    s.simulation_md(100)
    rg, vg, _, _ = s.download()
    np.testing.assert_allclose(rg, o.r, rtol=0, atol=1e-9)
    np.testing.assert_allclose(vg, o.v, rtol=0, atol=1e-9)
    s.close()


def test_angular_potential_without_constants_is_an_error(gpu_lib):
    """A triple whose k_ijk < 1e-5 (the reference returns an unset result):
    FM_ERR_BOND."""
    r, v, ch, sub, fy, bf, dom, mt, tab, kk, tt = _angular_melt()
    kk[1, 0, 1] = 0.0
    s = gpu_system(r, v, dom, WCA_RC, tplot=20, density=0.85, potential_flag=1, k_c=30.0, R_0=1.5)
    s.upload_monomers(ch, sub, bf)
    s.set_mie(tab, mt)
    s.set_angular(kk, tt, fy)
    with pytest.raises(api.FlowmolError) as e:
        s.setup()
    assert e.value.code == 8  # FM_ERR_BOND
    s.close()
