"""Seeded Couette-channel jobs: an FCC WCA fluid between tethered FCC walls.

Tags follow the reference's setup_location_tags for planar regions
(molecular_properties.f90:229-312, get_tag_status :17-154): a molecule is in
a region when, along some axis, it lies within the region's distance of the
bottom (rg <= -L/2 + d_bottom) or the top (rg >= L/2 - d_top) of the domain.
Here the walls are y-slabs: tethered (TETHEREDDISTTOP/BOTTOM), thermostatted
(THERMSTATTOP/BOTTOM, the same slabs) and, for the top wall only, sliding at
WALLSLIDEV along x.  Tether anchors are the lattice sites; tether
coefficients default to the reference's TETHERCOEFFICIENTS 0 5000 5000000.
"""
from __future__ import annotations

import numpy as np

from . import lattice

TAG_FREE, TAG_FIXED, TAG_FIXED_SLIDE, TAG_TETH, TAG_THERMO, TAG_TETH_THERMO, TAG_TETH_SLIDE, \
    TAG_TETH_THERMO_SLIDE = range(8)

WCA_RC = 2.0 ** (1.0 / 6.0)


def tags_for(r, domain, teth_bottom, teth_top, therm_bottom, therm_top, slide_bottom, slide_top):
    """setup_location_tags for y-slab regions (distances per axis, only y set)."""
    half = 0.5 * np.asarray(domain)

    def status(dbot, dtop):
        dbot = np.asarray(dbot, float); dtop = np.asarray(dtop, float)
        hit = np.zeros(len(r), bool)
        for k in range(3):
            if dbot[k] > 0:
                hit |= r[:, k] <= -half[k] + dbot[k]
            if dtop[k] > 0:
                hit |= r[:, k] >= half[k] - dtop[k]
        return hit

    teth = status(teth_bottom, teth_top)
    thermo = status(therm_bottom, therm_top)
    slide = status(slide_bottom, slide_top)
    tag = np.full(len(r), TAG_FREE, np.int32)
    tag[teth & ~thermo & ~slide] = TAG_TETH
    tag[teth & ~thermo & slide] = TAG_TETH_SLIDE
    tag[teth & thermo & ~slide] = TAG_TETH_THERMO
    tag[teth & thermo & slide] = TAG_TETH_THERMO_SLIDE
    tag[thermo & ~teth & ~slide] = TAG_THERMO
    return tag


def couette_job(nunits, density=0.8, temperature=1.0, wall_speed=1.0, seed=lattice.SEED_BASE + 5,
                wall_layers=1.0):
    """(r, v, tag, rtether, slidev, domain) of one channel.  The walls are
    `wall_layers` FCC unit cells thick at the bottom and top in y; the top
    wall slides at +wall_speed along x."""
    r, domain = lattice.fcc_lattice_fast(nunits, density)
    unit = domain[1] / nunits[1]
    d = wall_layers * unit
    tag = tags_for(r, domain, (0, d, 0), (0, d, 0), (0, d, 0), (0, d, 0), (0, 0, 0), (0, d, 0))
    v = lattice.maxwell_boltzmann(len(r), temperature, seed)
    v[tag != TAG_FREE] *= 0.5
    rtether = r.copy()
    slidev = np.zeros_like(r)
    slide = (tag == TAG_TETH_SLIDE) | (tag == TAG_TETH_THERMO_SLIDE)
    slidev[slide, 0] = wall_speed
    return r, v, tag, rtether, slidev, domain


def nunits_for(n_target, aspect_y=2):
    """Unit cells (nx, ny, nz) with ny = aspect_y * nx = aspect_y * nz whose
    4 nx ny nz is closest to n_target."""
    best = None
    for nx in range(2, 64):
        for ny in (aspect_y * nx - 1, aspect_y * nx, aspect_y * nx + 1):
            n = 4 * nx * ny * nx
            if best is None or abs(n - n_target) < abs(best[0] - n_target):
                best = (n, (nx, ny, nx))
    return best[1]
