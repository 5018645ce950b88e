"""Shared test helpers: seeded states, pair-set canonicalisation, digests,
error metrics.  Tolerances live in the tests that use them."""
from __future__ import annotations

import numpy as np

from flowmol_b200 import lattice

WCA_RC = 2.0 ** (1.0 / 6.0)
MASK64 = (1 << 64) - 1


def cfg1_state(seed=lattice.SEED_BASE + 0):
    """FCC 8x8x8, rho 0.8, T 1.0, MB velocities (2048 molecules)."""
    r, v, dom = lattice.lj_fluid([8, 8, 8], 0.8, 1.0, seed)
    return r, v, dom


def liquid_state(nunits, density, temperature, rc, steps=200, seed=lattice.SEED_BASE + 1, dt=0.005):
    """A disordered liquid: FCC + jitter, equilibrated by the FP64 oracle for
    `steps` velocity-Verlet steps (so parity starts from a realistic state)."""
    import oracle as O
    r, v, dom = lattice.lj_fluid(nunits, density, temperature, seed)
    r = lattice.jitter(r, 0.05, seed, dom)
    o = O.Oracle(r, v, dom, rc, tplot=10**6, delta_t=dt, density=density)
    o.setup()
    if steps:
        o.run_vv(steps)
    return o.r, o.v, dom, o


def canonical_oracle(owner, partner, code):
    """Canonical multiset of the reference half list: unshifted pairs as
    (min, max, 13), image pairs as directed (owner, partner, code)."""
    owner = owner.astype(np.int64); partner = partner.astype(np.int64); code = code.astype(np.int64)
    un = code == 13
    a = np.where(un, np.minimum(owner, partner), owner)
    b = np.where(un, np.maximum(owner, partner), partner)
    keys = (a << 32) | (b << 5) | code
    return np.sort(keys)


def canonical_full(owner, partner, code):
    """Canonical multiset of a both-directions list; checks the symmetry of
    the unshifted part on the way."""
    owner = owner.astype(np.int64); partner = partner.astype(np.int64); code = code.astype(np.int64)
    un = code == 13
    fwd = np.sort((owner[un] << 32) | partner[un])
    bwd = np.sort((partner[un] << 32) | owner[un])
    assert np.array_equal(fwd, bwd), "unshifted pairs are not stored in both directions"
    keep = ~un | (owner < partner)
    keys = (owner[keep] << 32) | (partner[keep] << 5) | code[keep]
    return np.sort(keys)


def _mix64(x):
    x = x.astype(np.uint64)
    with np.errstate(over="ignore"):
        x ^= x >> np.uint64(30); x *= np.uint64(0xbf58476d1ce4e5b9)
        x ^= x >> np.uint64(27); x *= np.uint64(0x94d049bb133111eb)
        x ^= x >> np.uint64(31)
    return x


def digest_oracle(owner, partner, code):
    """Same order-independent digest as fm_pair_digest, from a half list."""
    owner = owner.astype(np.uint64); partner = partner.astype(np.uint64); code = code.astype(np.uint64)
    un = code == 13
    lo = np.minimum(owner, partner); hi = np.maximum(owner, partner)
    with np.errstate(over="ignore"):
        hu = _mix64((lo[un] << np.uint64(32)) ^ hi[un])
        hs = _mix64(((owner[~un] << np.uint64(32)) ^ partner[~un]) * np.uint64(31) + code[~un]
                    + np.uint64(0x9e3779b97f4a7c15))
    tot = (int(hu.sum(dtype=np.uint64)) + int(hs.sum(dtype=np.uint64))) & MASK64
    return tot, int(un.sum() + (~un).sum())


def rel_err(x, ref, floor):
    """Per-row |x - ref| / max(|ref|, floor)."""
    d = np.linalg.norm(np.asarray(x) - np.asarray(ref), axis=-1)
    s = np.maximum(np.linalg.norm(np.asarray(ref), axis=-1), floor)
    return d / s


def mie_C(lr, la):
    """C_lookup (setup_set_parameters.f90:940-942)."""
    return (lr / (lr - la)) * (lr / la) ** (la / (lr - la))


def mie_tables(rc, eps, lr, la, mass, alpha=None, k=None, r0=None):
    """Symmetric ntypes x ntypes lookup tables as setup_mie_potential leaves
    them: C from (lr, la), potshift_lookup = the unshifted Mie energy at rc
    (:944), alpha 1 by default, harmonic bond constants k and r0."""
    eps = np.asarray(eps, float); lr = np.asarray(lr, float); la = np.asarray(la, float)
    nt = len(mass)
    alpha = np.ones((nt, nt)) if alpha is None else np.asarray(alpha, float)
    C = mie_C(lr, la)
    s = 1.0 / rc ** 2
    shift = C * eps * (s ** (0.5 * lr) - alpha * s ** (0.5 * la))
    return {"mass": np.asarray(mass, float), "epsilon": eps, "lambdar": lr, "lambdaa": la, "C": C,
            "alpha": alpha, "potshift": shift,
            "k_harmonic": np.zeros((nt, nt)) if k is None else np.asarray(k, float),
            "r0": np.zeros((nt, nt)) if r0 is None else np.asarray(r0, float)}


def mie_mixture_tables(rc):
    """Two types: Ar (12-6, eps 1, m 1) and a 15-6 type (eps 0.8, m 1.5);
    cross lambdas by the reference's rule sqrt((l_ii-3)(l_jj-3))+3 and a
    geometric-mean epsilon (setup_set_parameters.f90:918-938)."""
    lr = np.array([[12.0, np.sqrt(9.0 * 12.0) + 3.0], [np.sqrt(9.0 * 12.0) + 3.0, 15.0]])
    la = np.full((2, 2), 6.0)
    eps = np.array([[1.0, np.sqrt(0.8)], [np.sqrt(0.8), 0.8]])
    return mie_tables(rc, eps, lr, la, [1.0, 1.5], k=np.full((2, 2), 295.3322), r0=np.ones((2, 2)))
