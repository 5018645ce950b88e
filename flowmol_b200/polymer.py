"""Seeded FENE bead-spring melts: self-avoiding random walks on FCC sites.

Chains are grown bead by bead, each bead on a random free nearest-neighbour
site of the previous one (restarting a chain that gets stuck), on an FCC
lattice denser than the melt so a fraction of sites stays empty; the box is
sized for the requested bead density.  Lattice sites never overlap, so the
start needs no soft-core relaxation.  Monomer records follow the reference's
polymer_info_MD: chainID, subchainID (1..nmonomers), funcy (1 at the ends,
2 inside) and bin_bflag -- bit (partner subchainID - 1) set for each bonded
partner, 31 bits per word (modules.f90:497, 602-610).
"""
from __future__ import annotations

import numpy as np

from . import lattice


def bflag_words(partners):
    w = [0, 0, 0, 0]
    for sc in partners:
        pos = sc - 1
        w[pos // 31] |= 1 << (pos % 31)
    return w


def fene_melt(nchains, nmonomers=8, density=0.85, temperature=1.0, fill=0.9, seed=lattice.SEED_BASE + 3):
    """(r, v, chain, subchain, funcy, bflag(n,4), domain)."""
    n = nchains * nmonomers
    rng = np.random.Generator(np.random.Philox(int(seed)))
    # FCC as the even sites of a cubic grid of spacing a/2: m^3 cells -> 4 m^3 sites
    sites_needed = n / fill
    m = int(np.ceil((sites_needed / 4.0) ** (1.0 / 3.0)))
    g = 2 * m
    volume = n / density
    L = volume ** (1.0 / 3.0)
    half = L / g  # grid spacing a/2
    occ = bytearray(g * g * g)
    offs = [(1, 1, 0), (1, -1, 0), (-1, 1, 0), (-1, -1, 0), (1, 0, 1), (1, 0, -1), (-1, 0, 1), (-1, 0, -1),
            (0, 1, 1), (0, 1, -1), (0, -1, 1), (0, -1, -1)]

    def idx(i, j, k):
        return (i % g) * g * g + (j % g) * g + (k % g)

    free = [(i, j, k) for i in range(g) for j in range(g) for k in range(g) if (i + j + k) % 2 == 0]
    order = rng.permutation(len(free))
    starts = iter(order.tolist())
    coords = np.empty((n, 3), np.int64)
    pick = rng.integers(0, 1 << 30, size=(n * 4,)).tolist()
    pi = 0
    c = 0
    while c < nchains:
        try:
            s0 = free[next(starts)]
        except StopIteration:
            raise RuntimeError("lattice too full for the requested chains")
        if occ[idx(*s0)]:
            continue
        chain = [s0]
        occ[idx(*s0)] = 1
        ok = True
        while len(chain) < nmonomers:
            x, y, z = chain[-1]
            cand = [((x + a) % g, (y + b) % g, (z + e) % g) for a, b, e in offs]
            cand = [q for q in cand if not occ[idx(*q)]]
            if not cand:
                ok = False
                break
            q = cand[pick[pi % len(pick)] % len(cand)]
            pi += 1
            chain.append(q)
            occ[idx(*q)] = 1
        if not ok:
            for q in chain:
                occ[idx(*q)] = 0
            continue
        coords[c * nmonomers:(c + 1) * nmonomers] = chain
        c += 1
    r = (coords + 0.5) * half - 0.5 * L
    v = lattice.maxwell_boltzmann(n, temperature, seed ^ 0x77)
    chain_id = np.repeat(np.arange(1, nchains + 1, dtype=np.int32), nmonomers)
    sub = np.tile(np.arange(1, nmonomers + 1, dtype=np.int32), nchains)
    funcy = np.where((sub == 1) | (sub == nmonomers), 1, 2).astype(np.int32)
    bf = np.zeros((n, 4), np.int32)
    for s in range(1, nmonomers + 1):
        partners = [p for p in (s - 1, s + 1) if 1 <= p <= nmonomers]
        bf[sub == s] = bflag_words(partners)
    return r, v, chain_id, sub, funcy, bf, np.array([L, L, L])


def mark_solvent(chain, subchain, funcy, bflag, chain_ids):
    """Turns whole chains into solvent molecules as mark_chain_as_solvent does
    (modules.f90:681-707): chainID 0, subchainID 1, funcy 0, no bond flags.
    Returns new arrays."""
    chain, subchain, funcy, bflag = (np.array(x, copy=True) for x in (chain, subchain, funcy, bflag))
    sel = np.isin(chain, np.asarray(chain_ids))
    chain[sel] = 0
    subchain[sel] = 1
    funcy[sel] = 0
    bflag[sel] = 0
    return chain, subchain, funcy, bflag


def fene_solution(nchains, nmonomers=8, density=0.85, targetconc=0.5, temperature=1.0,
                  seed=lattice.SEED_BASE + 3):
    """A bead-spring melt whose chains are turned into solvent (seeded choice)
    until the chain-bead fraction is `targetconc`, the end state of the
    reference's fene_solution start (setup_initialise_microstate.f90:459-486).
    (r, v, chain, subchain, funcy, bflag(n,4), domain)."""
    r, v, ch, sub, fy, bf, dom = fene_melt(nchains, nmonomers, density, temperature, seed=seed)
    rng = np.random.Generator(np.random.Philox(int(seed) ^ 0x5D))
    keep = int(round(targetconc * nchains))
    drop = rng.permutation(np.arange(1, nchains + 1))[:nchains - keep]
    ch, sub, fy, bf = mark_solvent(ch, sub, fy, bf, drop)
    return r, v, ch, sub, fy, bf, dom
