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


SOD_A = float(np.float32(3.1730728678))       # default-real literals of modules.f90:458-462
SOD_B = float(np.float32(-0.85622864544))
WCA_CUT2_SOD = float(np.float32(1.25992104989487))


def soddemann_pair(dist, beads, eps=(1.7, 1.3, 0.6), L=8.0):
    """Two molecules at `dist` on x; `beads` = how many of them are chain
    beads (chainID 1, a one-bead chain without bonds; the rest solvent)."""
    r = np.array([[-dist / 2, 0.1, 0.2], [dist / 2, 0.1, 0.2]])
    o = O.Oracle(r, np.zeros((2, 3)), [L, L, L], WCA_RC, tplot=1, potential_flag=1, k_c=30.0, R_0=1.5)
    chain = np.array([1 if k < beads else 0 for k in range(2)], np.int32)
    o.set_monomers(chain, np.ones(2, np.int32), np.zeros(2, np.int32), np.zeros((2, 4), np.int32))
    o.set_solvent(1, *eps)
    o.setup()
    return o


def test_soddemann_geometry():
    """SOLVENT_INFO 1 with the WCA cutoff: rneighbr = 1.42246 < sod_cut, so
    rcutoff becomes 1.5 (cells of 1.5 + skin) and rneighbr2 stays -- no R_0
    override (setup_set_parameters.f90:1863-1876); the library's geometry
    says the same."""
    from flowmol_b200 import api
    dom = [8.4453, 9.0, 11.0]
    o = O.Oracle(np.zeros((1, 3)), np.zeros((1, 3)), dom, WCA_RC, potential_flag=1, k_c=30.0, R_0=1.5)
    g0 = o.geometry()
    assert g0["rneighbr2"] == 1.5 * 1.5  # solvent_flag 0: the FENE override
    o.set_solvent(1, 1.0, 1.0, 1.0)
    g = o.geometry()
    rn = WCA_RC + (0.3 + 0.3 + 0.3) / 3.0
    assert g["rcutoff2"] == 2.25 and g["rneighbr2"] == rn * rn
    assert list(g["ncells"]) == [int(np.floor(x / 1.8)) for x in dom]
    p = api.make_params(1, dom, WCA_RC, potential_flag=1, k_c=30.0, R_0=1.5, solvent_flag=1)
    rc, lg = api.derive_geometry(p)
    assert rc == 0
    assert lg["ncells"] == list(g["ncells"]) and lg["rneighbr2"] == g["rneighbr2"]
    assert lg["rcutoff2"] == g["rcutoff2"] and lg["cellside"] == list(g["cellside"])
    assert lg["potshift"] == g["potshift"]


@pytest.mark.parametrize("dist", [1.05, 1.3, 1.41])
@pytest.mark.parametrize("beads", [0, 1, 2])
def test_soddemann_two_body_analytic(dist, beads):
    """simulation_compute_forces_Soddemann_neigbr_halfint (:793-888): WCA
    below wca_cut2 (the REAL(4) rounding of 2^(1/3)), the reference's cosine
    expression eps a s^2 sin(a s + b) (s = 1/r^2) out to 1.5, well depth by
    the number of chain beads; PE per molecule as written there."""
    eps = (1.7, 1.3, 0.6)  # eps_pp, eps_ps, eps_ss
    e = {2: eps[0], 1: eps[1], 0: eps[2]}[beads]
    o = soddemann_pair(dist, beads, eps)
    r2 = (-dist / 2 - dist / 2) ** 2
    s = 1.0 / r2
    if r2 < WCA_CUT2_SOD:
        acc = 48.0 * ((s * s) * (s * s) * (s * s) * s - 0.5 * ((s * s) * (s * s)))
        pe = 4.0 * ((s * s * s) * (s * s * s) - s * s * s + 0.25) - e
    else:
        acc = (e * SOD_A * (s * s)) * np.sin(s * SOD_A + SOD_B)
        pe = 0.5 * e * (np.cos(SOD_A * r2 + SOD_B) - 1.0)
    a = o.a
    assert a[0, 0] == pytest.approx(acc * -dist, rel=1e-14) and a[1, 0] == pytest.approx(acc * dist, rel=1e-14)
    assert np.all(a[:, 1:] == 0.0)
    np.testing.assert_allclose(o.potenergymol, [pe, pe], rtol=1e-13)


@pytest.mark.parametrize("dist", [1.05, 1.3])
def test_mie_soddemann_two_body(dist):
    """Mie_potential 1 with the Soddemann solvent: inside wca_cut2 the force
    is get_accijmag = Mie_accijmag of the two types (setup_set_parameters.f90
    :149-168), the energy the LJ-WCA expression of the Soddemann routine
    (:864-866), and the accelerations are not divided by the masses
    (:852-860); beyond it the cosine well as without Mie."""
    from helpers import mie_mixture_tables
    eps = (1.7, 1.3, 0.6)
    tab = mie_mixture_tables(WCA_RC)
    r = np.array([[-dist / 2, 0.1, 0.2], [dist / 2, 0.1, 0.2]])
    o = O.Oracle(r, np.zeros((2, 3)), [8.0, 8.0, 8.0], WCA_RC, tplot=1, potential_flag=1, k_c=30.0, R_0=1.5)
    o.set_monomers(np.array([1, 0], np.int32), np.ones(2, np.int32), np.zeros(2, np.int32),
                   np.zeros((2, 4), np.int32))
    o.set_solvent(1, *eps)
    o.set_mie(tab, np.array([1, 2], np.int32))
    o.setup()
    r2 = (-dist / 2 - dist / 2) ** 2
    s = 1.0 / r2
    e = eps[1]  # one chain bead in the pair: eps_ps
    if r2 < WCA_CUT2_SOD:
        lr, la = tab["lambdar"][0, 1], tab["lambdaa"][0, 1]
        C, ep, al = tab["C"][0, 1], tab["epsilon"][0, 1], tab["alpha"][0, 1]
        acc = C * ep * (lr * s ** (0.5 * lr + 1) - al * la * s ** (0.5 * la + 1))
        pe = 4.0 * ((s * s * s) * (s * s * s) - s * s * s + 0.25) - e
    else:
        acc = (e * SOD_A * (s * s)) * np.sin(s * SOD_A + SOD_B)
        pe = 0.5 * e * (np.cos(SOD_A * r2 + SOD_B) - 1.0)
    a = o.a
    assert a[0, 0] == pytest.approx(acc * -dist, rel=1e-13) and a[1, 0] == pytest.approx(acc * dist, rel=1e-13)
    np.testing.assert_allclose(o.potenergymol, [pe, pe], rtol=1e-13)


def test_soddemann_pairs_beyond_rneighbr_are_not_seen():
    """A pair inside sod_cut but beyond rneighbr (1.42246) is not in the list
    the forces walk: no force, as in the reference, where rneighbr2 keeps its
    WCA-based value."""
    for dist in (1.45, 1.49):
        assert np.all(soddemann_pair(dist, 2).a == 0.0)


def test_soddemann_solution_wells_act():
    """On a polymer solution the cosine well changes the forces (pairs beyond
    wca_cut2 exist for every bead count) and vanishes with zero well depths,
    leaving WCA + FENE with the Soddemann list geometry."""
    from flowmol_b200 import polymer
    r, v, ch, sub, fy, bf, dom = polymer.fene_solution(48, targetconc=0.5)
    r = lattice.jitter(r, 0.08, 91, dom)  # off the lattice: pairs between the shells
    out = {}
    for eps in ((1.5, 1.0, 0.5), (0.0, 0.0, 0.0)):
        o = O.Oracle(r, v, dom, WCA_RC, tplot=1, potential_flag=1, k_c=30.0, R_0=1.5, density=0.85)
        o.set_monomers(ch, sub, fy, bf)
        o.set_solvent(1, *eps)
        o.setup()
        out[eps] = (o.a, o.potenergymol)
    a1, pe1 = out[(1.5, 1.0, 0.5)]
    a0, pe0 = out[(0.0, 0.0, 0.0)]
    assert np.abs(a1 - a0).max() > 1e-3 and np.all(pe1 <= pe0 + 1e-12)


def test_pressure_tensor_sampling_follows_the_reference_routines():
    """pressure_averaging samples on the record steps of a run, not at setup
    (setup_initial_record.f90:89 calls evaluate_macroscopic_properties only);
    the all-pairs routine adds no rf (kinetic part only), the half list adds
    acc rij rij on both sides."""
    r, v, dom = lattice.lj_fluid([3, 3, 3], 0.8, 1.0, 17)
    o = O.Oracle(r, v, dom, 2.5, tplot=5, force_list=0)
    o.set_pressure(1)
    o.setup()
    assert o.pressure_average()[1] == 0
    o.run_vv(20)
    p, n = o.pressure_average()
    assert n == 4
    # kinetic only: with zero velocities the all-pairs tensor would vanish
    o0 = O.Oracle(r, np.zeros_like(v), dom, 2.5, tplot=1, force_list=0)
    o0.set_pressure(1)
    o0.setup()
    o0.run_vv(1)
    p0, _ = o0.pressure_average()
    vnew = o0.v
    kin = np.einsum("ni,nj->ij", vnew, vnew) / np.prod(dom)
    np.testing.assert_allclose(p0, kin, rtol=1e-12, atol=1e-15)


def _trimer_oracle(angular, k=4.3196, t0=2.7751, kz=0.0):
    """A lone trimer (chain 1: beads 1-2-3, the middle one funcy 2) in the
    middle of a periodic box, Mie 12-6 types 1-2-1 with masses 1 and 1.5,
    harmonic bonds; the angle between the bonds ~150 degrees."""
    from helpers import mie_tables
    from flowmol_b200 import polymer
    r = np.array([[-0.95, 0.05, 0.0], [0.0, 0.0, 0.02], [0.82, 0.47, -0.1]])
    v = np.zeros_like(r)
    dom = np.array([10.0, 10.0, 10.0])
    o = O.Oracle(r, v, dom, WCA_RC, tplot=1, potential_flag=1, k_c=30.0, R_0=1.5)
    bf = np.array([polymer.bflag_words([2]), polymer.bflag_words([1, 3]), polymer.bflag_words([2])], np.int32)
    o.set_monomers([1, 1, 1], [1, 2, 3], [1, 2, 1], bf)
    tab = mie_tables(WCA_RC, np.ones((2, 2)), np.full((2, 2), 12.0), np.full((2, 2), 6.0), [1.0, 1.5],
                     k=np.full((2, 2), 295.3322), r0=np.ones((2, 2)))
    o.set_mie(tab, np.array([1, 2, 1], np.int32))
    if angular:
        kk = np.zeros((2, 2, 2)); tt = np.zeros((2, 2, 2))
        kk[0, 1, 0] = k; tt[0, 1, 0] = t0
        kk[1, 0, 1] = kz
        o.set_angular(kk, tt)
    return o, r


def test_angular_force_follows_the_reference_routine():
    """The oracle's angular term equals a separate restatement of
    simulation_compute_forces_angular / angular_harmonic_force for a lone
    trimer, with i and k the middle bead's first and second bond."""
    import math
    plain, r = _trimer_oracle(False)
    plain.setup()
    o, _ = _trimer_oracle(True)
    o.setup()
    da = o.a - plain.a
    own, par, _code = o.bond_list()
    row = [int(p) for w, p in zip(own, par) if w == 2]
    i, k = row[0] - 1, row[1] - 1
    j = 1
    rij = r[i] - r[j]; rjk = r[j] - r[k]
    mij = math.sqrt(rij @ rij); mjk = math.sqrt(rjk @ rjk)
    th = math.acos((rij @ rjk) / (mij * mjk))
    kk, t0 = 4.3196, 2.7751
    f1 = -(kk * (th - t0) / (mij * math.sin(th))) * (rjk / mjk - rij / mij * math.cos(th))
    f3 = -(kk * (th - t0) / (mjk * math.sin(th))) * (rij / mij - rjk / mjk * math.cos(th))
    f2 = -f1 - f3
    mass = {0: 1.0, 1: 1.5, 2: 1.0}
    want = np.zeros((3, 3))
    want[i] -= f1 / mass[i]; want[j] -= f2 / mass[j]; want[k] -= f3 / mass[k]
    np.testing.assert_allclose(da, want, rtol=1e-12, atol=1e-13)
    assert np.abs(da).max() > 1e-3


def test_angular_force_is_not_the_gradient_on_bead_k():
    """The reference's routine applies -grad U to bead i but +grad U to bead k
    (U = k/2 (theta - theta_0)^2, theta between rij and rjk), so its angular
    force is not conservative; the restatement keeps that, and the total
    force stays zero (the reference's own balance check)."""
    import math
    plain, r = _trimer_oracle(False)
    plain.setup()
    o, _ = _trimer_oracle(True)
    o.setup()
    mass = np.array([1.0, 1.5, 1.0])
    f = (o.a - plain.a) * mass[:, None]
    own, par, _code = o.bond_list()
    row = [int(p) for w, p in zip(own, par) if w == 2]
    i, k = row[0] - 1, row[1] - 1

    def U(x):
        rij = x[i] - x[1]; rjk = x[1] - x[k]
        th = math.acos((rij @ rjk) / math.sqrt((rij @ rij) * (rjk @ rjk)))
        return 0.5 * 4.3196 * (th - 2.7751) ** 2

    g = np.zeros((3, 3))
    for a in range(3):
        for c in range(3):
            xp = r.copy(); xm = r.copy(); xp[a, c] += 1e-6; xm[a, c] -= 1e-6
            g[a, c] = (U(xp) - U(xm)) / 2e-6
    np.testing.assert_allclose(f[i], -g[i], rtol=1e-6, atol=1e-8)
    np.testing.assert_allclose(f[k], g[k], rtol=1e-6, atol=1e-8)
    np.testing.assert_allclose(f.sum(axis=0), 0.0, atol=1e-12)


def test_angular_undefined_cases_are_errors():
    """k_ijk < 1e-5 leaves the reference's result unset: an error, not a
    number."""
    o, _ = _trimer_oracle(True, k=0.0)
    with pytest.raises(O.OracleError):
        o.setup()
