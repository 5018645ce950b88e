"""Seeded start states for the MD hot path.

``fcc_lattice`` places molecules exactly as the reference's
setup_initialise_lattice does for one rank (setup_initialise_microstate.f90:
197-345): unit cells nz-outer, nx, ny-inner, four sites per cell at
(n - 0.75 + {0, 1/2}) * unitsize, shifted by -domain/2, numbered in that
order.  ``maxwell_boltzmann`` replaces the reference's fixed-speed random
directions (setup_initialise_microstate.f90:4278-4335, which depend on
gfortran's RNG) with seeded Gaussian velocities, zero net momentum and the
kinetic temperature rescaled to exactly T.  Both are FP64 numpy.
"""
from __future__ import annotations

import numpy as np

SEED_BASE = 0x466D6F6C  # "Fmol"


def global_domain(nunits, density):
    """L_i = n_i / (density/4)**(1/3) (setup_set_parameters.f90:1549)."""
    return np.array([float(n) / (density / 4.0) ** (1.0 / 3.0) for n in nunits])


def fcc_lattice(nunits, density):
    nunits = [int(x) for x in nunits]
    domain = global_domain(nunits, density)
    unit = domain / np.array(nunits, dtype=np.float64)
    half = 0.5 * domain
    out = []
    # loops run 0..n like the reference; sites outside [0, domain) are skipped
    for nz in range(0, nunits[2] + 1):
        cz = (nz - 0.75) * unit[2]
        for nx in range(0, nunits[0] + 1):
            cx = (nx - 0.75) * unit[0]
            for ny in range(0, nunits[1] + 1):
                cy = (ny - 0.75) * unit[1]
                for j in range(4):
                    rc = [cx, cy, cz]
                    if j == 1:
                        rc[0] = cx + 0.5 * unit[0]; rc[2] = cz + 0.5 * unit[2]
                    elif j == 2:
                        rc[1] = cy + 0.5 * unit[1]; rc[2] = cz + 0.5 * unit[2]
                    elif j == 3:
                        rc[0] = cx + 0.5 * unit[0]; rc[1] = cy + 0.5 * unit[1]
                    if any(rc[k] < 0.0 or rc[k] >= domain[k] for k in range(3)):
                        continue
                    out.append([rc[0] - half[0], rc[1] - half[1], rc[2] - half[2]])
    return np.array(out, dtype=np.float64), domain


def fcc_lattice_fast(nunits, density):
    """Vectorised fcc_lattice with the same order and values (large N)."""
    nunits = [int(x) for x in nunits]
    domain = global_domain(nunits, density)
    unit = domain / np.array(nunits, dtype=np.float64)
    half = 0.5 * domain
    nz, nx, ny = np.meshgrid(np.arange(nunits[2] + 1), np.arange(nunits[0] + 1), np.arange(nunits[1] + 1),
                             indexing="ij")
    c = np.stack([(nx - 0.75) * unit[0], (ny - 0.75) * unit[1], (nz - 0.75) * unit[2]], axis=-1).reshape(-1, 3)
    sites = np.repeat(c[:, None, :], 4, axis=1)
    sites[:, 1, 0] = c[:, 0] + 0.5 * unit[0]; sites[:, 1, 2] = c[:, 2] + 0.5 * unit[2]
    sites[:, 2, 1] = c[:, 1] + 0.5 * unit[1]; sites[:, 2, 2] = c[:, 2] + 0.5 * unit[2]
    sites[:, 3, 0] = c[:, 0] + 0.5 * unit[0]; sites[:, 3, 1] = c[:, 1] + 0.5 * unit[1]
    sites = sites.reshape(-1, 3)
    keep = np.all((sites >= 0.0) & (sites < domain[None, :]), axis=1)
    return sites[keep] - half[None, :], domain


def maxwell_boltzmann(n, temperature, seed):
    rng = np.random.Generator(np.random.Philox(int(seed)))
    v = rng.standard_normal((n, 3))
    v -= v.mean(axis=0, keepdims=True)
    t_now = float((v * v).sum()) / (3.0 * n)
    v *= np.sqrt(temperature / t_now)
    return v


def lj_fluid(nunits, density, temperature, seed=SEED_BASE):
    """FCC start with Maxwell-Boltzmann velocities: (r, v, domain)."""
    r, domain = fcc_lattice_fast(nunits, density)
    v = maxwell_boltzmann(r.shape[0], temperature, seed)
    return r, v, domain


def jitter(r, amplitude, seed, domain=None):
    """Seeded uniform displacement of every coordinate (a disordered start
    that keeps the lattice's minimum distance well above the LJ core)."""
    rng = np.random.Generator(np.random.Philox(int(seed) ^ 0x5A5A))
    out = r + rng.uniform(-amplitude, amplitude, size=r.shape)
    if domain is not None:
        half = 0.5 * np.asarray(domain)
        out = np.where(out >= half, out - domain, out)
        out = np.where(out < -half, out + domain, out)
    return out
