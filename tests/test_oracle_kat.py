"""Known-answer and internal-consistency checks of the CPU oracle."""
import numpy as np
import pytest

import oracle as O
from flowmol_b200 import lattice
from helpers import WCA_RC, canonical_oracle, cfg1_state, liquid_state


def test_lj_two_body_analytic():
    # LJ_accijmag(s) = 48 (s^7 - s^4/2), LJ_energy = 4 (s^6 - s^3) - potshift
    for r in (0.95, 1.0, 2 ** (1 / 6), 1.5, 2.4):
        s = 1.0 / (r * r)
        assert O.lib().orc_lj_accijmag(s) == pytest.approx(48.0 * (s ** 7 - 0.5 * s ** 4), rel=1e-15)
        ps = O.lib().orc_potshift(2.5)
        assert O.lib().orc_lj_energy(s, ps) == pytest.approx(4.0 * (r ** -12 - r ** -6) - ps, rel=1e-13, abs=1e-15)
    # WCA shift: potshift(2^(1/6)) = -1 (setup_set_parameters.f90:1222)
    assert O.lib().orc_potshift(WCA_RC) == pytest.approx(-1.0, abs=1e-14)


def two_body(dist, rc=2.5, L=20.0):
    r = np.array([[-dist / 2, 0.1, 0.2], [dist / 2, 0.1, 0.2]])
    v = np.zeros((2, 3))
    o = O.Oracle(r, v, [L, L, L], rc, tplot=1)
    o.setup()
    return o


def test_two_body_force_and_cutoff_edges():
    o = two_body(1.2)
    s = 1.0 / (1.2 * 1.2)
    f = 48.0 * (s ** 7 - 0.5 * s ** 4) * 1.2
    a = o.a
    assert a[0, 0] == pytest.approx(-f, rel=1e-14) and a[1, 0] == pytest.approx(f, rel=1e-14)
    assert np.all(a[:, 1:] == 0.0)
    # strict `<` on rcutoff2: a pair exactly at rc does not interact, one ulp inside does
    rc = 2.5
    assert np.all(two_body(rc).a == 0.0)
    inside = np.nextafter(rc, 0.0)
    o2 = two_body(inside)
    rij2 = (inside / 2 - (-inside / 2)) ** 2
    assert (rij2 < rc * rc) == bool(np.any(o2.a != 0.0))


def test_fcc_first_shell_kat():
    """Perfect FCC at rho 0.8 with WCA: nearest neighbours at 1.2091 > rc, so
    F = PE = virial = 0; every molecule has exactly 12 neighbours in r_n."""
    r, v, dom = cfg1_state()
    o = O.Oracle(r, v, dom, WCA_RC, tplot=1)
    o.setup()
    assert np.all(o.a == 0.0)
    m = o.macro()
    assert m["potenergysum"] == 0.0 and m["virial"] == 0.0
    own, par, code = o.pair_list()
    cnt = np.bincount(own, minlength=len(r) + 1)[1:] + np.bincount(par, minlength=len(r) + 1)[1:]
    # unshifted pairs count once per molecule each side; image pairs are stored
    # on both sides already, so count them on the owner only
    un = code == 13
    cnt = np.bincount(own[un], minlength=len(r) + 1)[1:] + np.bincount(par[un], minlength=len(r) + 1)[1:] \
        + np.bincount(own[~un], minlength=len(r) + 1)[1:]
    assert np.all(cnt == 12)


def brute_force_pairs(r, dom, rn2, ncells):
    """Every (i, j-image) with rij2 < rn2 that the reference's cell stencil can
    see, computed directly: images x + s L with the same FP64 roundings."""
    n = len(r)
    hd = 0.5 * dom
    cs = dom / ncells
    keys = []
    shifts = [(sx, sy, sz) for sz in (-1, 0, 1) for sy in (-1, 0, 1) for sx in (-1, 0, 1)]
    cell = np.ceil((r + hd) / cs).astype(int)  # 0-based extended index
    for (sx, sy, sz) in shifts:
        img = r.copy()
        if sx: img[:, 0] = img[:, 0] + sx * dom[0]
        if sy: img[:, 1] = img[:, 1] + sy * dom[1]
        if sz: img[:, 2] = img[:, 2] + sz * dom[2]
        # images exist only for molecules in the boundary cell facing the shift
        ok = np.ones(n, bool)
        for k, s in enumerate((sx, sy, sz)):
            if s == 1: ok &= cell[:, k] == 1
            if s == -1: ok &= cell[:, k] == ncells[k]
        idx = np.nonzero(ok)[0]
        d = r[:, None, :] - img[None, idx, :]
        d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
        ii, jj = np.nonzero(d2 < rn2)
        jj = idx[jj]
        code = (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1)
        sel = ii != jj if code == 13 else np.ones(len(ii), bool)
        ii, jj = ii[sel], jj[sel]
        if code == 13:
            sel = ii < jj
            ii, jj = ii[sel], jj[sel]
        keys.append(((ii + 1).astype(np.int64) << 32) | ((jj + 1).astype(np.int64) << 5) | code)
    return np.sort(np.concatenate(keys))


def test_halfint_equals_stencil_brute_force():
    """The reference's 13-shift + 27-sweep half list equals the set of all
    (molecule, image) pairs within r_n over adjacent cells: every adjacent
    cell pair with an interior cell visited once, cross-boundary pairs from
    both sides."""
    r, v, dom, o = liquid_state([6, 6, 6], 0.8, 1.0, 2.5, steps=20)
    o.rebuild()
    g = o.geometry()
    got = canonical_oracle(*o.pair_list())
    ref = brute_force_pairs(o.r, dom, g["rneighbr2"], g["ncells"])
    assert np.array_equal(got, ref)


def test_allint_is_symmetric_closure_of_halfint():
    r, v, dom, o = liquid_state([6, 6, 6], 0.8, 1.0, 2.5, steps=10)
    o.rebuild()
    half = canonical_oracle(*o.pair_list())
    o2 = O.Oracle(o.r, o.v, dom, 2.5, force_list=2, tplot=10 ** 6)
    o2.setup()
    from helpers import canonical_full
    full = canonical_full(*o2.pair_list())
    assert np.array_equal(half, full)


def test_halfint_forces_equal_all_pairs():
    r, v, dom, o = liquid_state([6, 6, 6], 0.8, 1.0, 2.5, steps=20)
    o.compute_forces()
    ap = O.Oracle(o.r, o.v, dom, 2.5, force_list=0, tplot=10 ** 6)
    ap.compute_forces()
    np.testing.assert_allclose(o.a, ap.a, rtol=0, atol=1e-11)


def test_molecule_exactly_at_minus_half_domain():
    """A molecule at exactly -L/2 is not wrapped (strict `<`) and bins into the
    low halo cell (ceiling(0)+1 = 1); one at +L/2 wraps to -L/2."""
    r, v, dom = cfg1_state()
    r = r.copy()
    r[0] = [-dom[0] / 2, 0.3, 0.4]
    r[1] = [dom[0] / 2, -1.0, 2.0]
    o = O.Oracle(r, v, dom, WCA_RC, tplot=10 ** 6)
    O.lib().orc_sendmols(o.h)
    assert o.r[0, 0] == -dom[0] / 2
    assert o.r[1, 0] == -dom[0] / 2
    o.setup()  # must not report an escape
    assert o.pair_list()[0].size > 0


def test_nve_energy_conservation_cfg1():
    r, v, dom = cfg1_state()
    o = O.Oracle(r, v, dom, WCA_RC, tplot=100)
    o.setup()
    recs = o.run_vv(1000)
    te = recs[:, 6]
    assert abs(te[-1] - 1.5) < 2e-3
    assert o.rebuild_count > 10


def test_mie_12_6_argon_reproduces_lj():
    """Mie_potential 1 with the argon entry (lambda 12-6, eps 1, C = 4, mass 1)
    is the LJ potential: forces and energies to rounding (real powers against
    integer powers)."""
    from helpers import mie_tables
    r, v, dom, _ = liquid_state([6, 6, 6], 0.8442, 0.722, 2.5, steps=20)
    lj = O.Oracle(r, v, dom, 2.5, tplot=1, density=0.8442)
    lj.setup()
    mie = O.Oracle(r, v, dom, 2.5, tplot=1, density=0.8442)
    mie.set_mie(mie_tables(2.5, [[1.0]], [[12.0]], [[6.0]], [1.0]), np.ones(len(r), np.int32))
    mie.setup()
    np.testing.assert_allclose(mie.a, lj.a, rtol=0, atol=1e-12 * np.abs(lj.a).max())
    np.testing.assert_allclose(mie.potenergymol, lj.potenergymol, rtol=1e-12, atol=1e-12)


def test_mie_mixture_mass_and_records():
    """Two-type Mie fluid: a = F/m per molecule, and the kinetic record sums
    are mass-weighted (simulation_record.f90:1236-1252)."""
    from helpers import mie_mixture_tables
    r, v, dom, _ = liquid_state([6, 6, 6], 0.8, 1.0, 2.5, steps=10)
    mt = (np.arange(len(r)) % 2 + 1).astype(np.int32)
    tab = mie_mixture_tables(2.5)
    o = O.Oracle(r, v, dom, 2.5, tplot=1, density=0.8)
    o.set_mie(tab, mt)
    o.setup()
    m = tab["mass"][mt - 1]
    rec = o.macro()
    assert rec["mv2sum"] == pytest.approx((m[:, None] * v * v).sum(), rel=1e-12)
    # momentum of the forces: sum m a = 0 (Newton's third law over all pairs)
    assert np.abs((m[:, None] * o.a).sum(0)).max() < 1e-9 * np.abs(m[:, None] * o.a).max()
