"""A CPU stand-in for one rank's subdomain (test infrastructure).

It implements the calls ``flowmol_b200.domain.DecomposedSystem`` makes on a
``Subdomain`` -- classification and migration, halo records, the sort by
(cell, global number), neighbour rows, LJ forces and the velocity-Verlet
moves -- in numpy FP64, with the same record layouts and the same global
binning, so that the decomposition's host protocol (plan, counts, all-to-all
exchanges, refresh lists, rebuild decisions) can run over real gloo ranks
on a machine without a GPU and be checked against the FP64 oracle.  The
product path is the CUDA subdomain; nothing outside tests/ imports this.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from flowmol_b200 import domain as D


class CpuSubdomain:
    def __init__(self, geom, plan: D.Plan, rank, rc, rn2, dt, tplot, half_min_delta, np_global, density,
                 rebuild_criteria=0, fixed_rebuild=1):
        self.plan, self.rank = plan, rank
        self.L, self.hd, self.cs = np.asarray(geom["L"]), np.asarray(geom["hd"]), np.asarray(geom["cs"])
        self.G = plan.G
        self.org, self.nloc = plan.box(rank)
        self.ne = [n + 2 for n in self.nloc]
        self.ncell = int(np.prod(self.ne))
        self.rc2 = rc * rc
        self.rn2 = rn2
        self.potshift = 4.0 * (rc ** -12 - rc ** -6)
        self.dt, self.tplot = dt, tplot
        self.half_min_delta = half_min_delta
        self.np_global, self.density = np_global, density
        self.crit, self.fixed = rebuild_criteria, fixed_rebuild
        self.rmax = 0.0
        self.vmax2_bits = 0
        nd = plan.needs(rank)
        self.need_off, self.need_rank, self.need_code, self.need_cell = nd["off"], nd["rank"], nd["code"], nd["cell"]

    # -- state -----------------------------------------------------------------
    def upload(self, r, v, gid):
        n = len(gid)
        self.r = np.array(r, np.float64).reshape(n, 3)
        self.v = np.array(v, np.float64).reshape(n, 3)
        self.a = np.zeros((n, 3))
        self.w = np.zeros(n)
        self.gid = np.array(gid, np.int64)
        self.cell = np.full(n, -1, np.int64)

    def _bin(self, r):
        """(owner rank, local cell or -1, ok) of positions, the undivided grid's binning."""
        g = np.stack([np.ceil((r[:, k] + self.hd[k]) / self.cs[k]).astype(np.int64) for k in range(3)], 1)
        ok = np.all((g >= 1) & (g <= np.asarray(self.G)), axis=1)
        gi = np.clip(g - 1, 0, np.asarray(self.G) - 1)
        own = [self.plan.owner_axis[k][gi[:, k]] for k in range(3)]
        owner = (own[0] * self.plan.dims[1] + own[1]) * self.plan.dims[2] + own[2]
        loc = g - np.asarray(self.org)
        cell = loc[:, 0] + self.ne[0] * (loc[:, 1] + self.ne[1] * loc[:, 2])
        cell = np.where(owner == self.rank, cell, -1)
        return owner, cell, ok

    # -- rebuild ---------------------------------------------------------------
    def classify(self, wrap):
        keep = self.w == 0.0
        for name in ("r", "v", "a", "w", "gid"):
            setattr(self, name, getattr(self, name)[keep])
        if wrap:
            for k in range(3):
                x = self.r[:, k]
                x = np.where(x >= self.hd[k], x - self.L[k], x)
                x = np.where(x < -self.hd[k], x + self.L[k], x)
                self.r[:, k] = x
        owner, cell, ok = self._bin(self.r)
        if not ok.all():
            raise RuntimeError("molecule outside the global interior")
        self.cell = cell
        self.emig = np.nonzero(owner != self.rank)[0]
        self.emig_dest = owner[self.emig]
        return np.bincount(self.emig_dest, minlength=self.plan.nranks).astype(np.int32)

    def pack_emigrants(self, counts):
        order = np.argsort(self.emig_dest, kind="stable")
        idx = self.emig[order]
        rec = np.concatenate([self.r[idx], self.v[idx], self.a[idx], self.gid[idx, None].astype(np.float64)], 1)
        stay = np.ones(len(self.gid), bool)
        stay[self.emig] = False
        for name in ("r", "v", "a", "w", "gid", "cell"):
            setattr(self, name, getattr(self, name)[stay])
        return torch.as_tensor(rec.reshape(-1).copy())

    def immigrate(self, recv, n):
        rec = recv.numpy().reshape(n, D.MREC)
        owner, cell, ok = self._bin(rec[:, 0:3])
        if n and (not ok.all() or (owner != self.rank).any()):
            raise RuntimeError("an immigrant does not bin into this subdomain")
        self.r = np.concatenate([self.r, rec[:, 0:3]])
        self.v = np.concatenate([self.v, rec[:, 3:6]])
        self.a = np.concatenate([self.a, rec[:, 6:9]])
        self.w = np.concatenate([self.w, np.zeros(n)])
        self.gid = np.concatenate([self.gid, rec[:, 9].astype(np.int64)])
        self.cell = np.concatenate([self.cell, cell])

    def halo_counts(self):
        self._hrec = []
        for i in range(len(self.gid)):
            c = self.cell[i]
            for k in range(self.need_off[c], self.need_off[c + 1]):
                self._hrec.append((self.need_rank[k], i, self.need_code[k], self.need_cell[k]))
        dest = np.array([h[0] for h in self._hrec], np.int64)
        return np.bincount(dest, minlength=self.plan.nranks).astype(np.int32)

    def pack_halo(self, counts):
        out = []
        for dest, i, code, hcell in sorted(self._hrec, key=lambda t: t[0]):
            s = [(code & 3) - 1, ((code >> 2) & 3) - 1, ((code >> 4) & 3) - 1]
            x = [self.r[i, k] + s[k] * self.L[k] if s[k] else self.r[i, k] for k in range(3)]
            out.append(x + [float(self.gid[i]), float(hcell)])
        return torch.as_tensor(np.asarray(out, np.float64).reshape(-1))

    def receive_halo(self, recv, n):
        rec = recv.numpy().reshape(n, D.HREC)
        self.r = np.concatenate([self.r, rec[:, 0:3]])
        self.v = np.concatenate([self.v, np.zeros((n, 3))])
        self.a = np.concatenate([self.a, np.zeros((n, 3))])
        self.w = np.concatenate([self.w, np.ones(n)])
        self.gid = np.concatenate([self.gid, rec[:, 3].astype(np.int64)])
        self.cell = np.concatenate([self.cell, rec[:, 4].astype(np.int64)])
        order = np.lexsort((self.gid, self.cell))
        for name in ("r", "v", "a", "w", "gid", "cell"):
            setattr(self, name, getattr(self, name)[order])
        self.starts = np.searchsorted(self.cell, np.arange(self.ncell + 1)).astype(np.int32)
        self._build()

    def _build(self):
        """Rows of the owned molecules: candidates of the 27 cells around the
        owner's cell in the build's visiting order (x offset fastest), in-cell
        order, exact (dx^2 + dy^2) + dz^2 < rneighbr^2."""
        ne = self.ne
        self.rows = [np.zeros(0, np.int64)] * len(self.gid)
        for c in range(self.ncell):
            b, e = self.starts[c], self.starts[c + 1]
            if b == e:
                continue
            cx, cy, cz = c % ne[0], (c // ne[0]) % ne[1], c // (ne[0] * ne[1])
            if cx in (0, ne[0] - 1) or cy in (0, ne[1] - 1) or cz in (0, ne[2] - 1):
                continue  # halo copies get no rows
            cand = []
            for q in range(27):
                x2, y2, z2 = cx + q % 3 - 1, cy + (q // 3) % 3 - 1, cz + q // 9 - 1
                c2 = x2 + ne[0] * (y2 + ne[1] * z2)
                cand.append(np.arange(self.starts[c2], self.starts[c2 + 1]))
            cand = np.concatenate(cand)
            for i in range(b, e):
                d = self.r[i] - self.r[cand]
                r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
                hit = (r2 < self.rn2) & (cand != i)
                self.rows[i] = cand[hit]

    def cell_starts(self):
        return self.starts.copy()

    def to_device(self, a):
        return torch.as_tensor(a)

    def gather_positions(self, idx, code):
        idx = idx.numpy().astype(np.int64)
        code = code.numpy().astype(np.int64)
        out = np.empty((len(idx), 3))
        for k in range(3):
            s = ((code >> (2 * k)) & 3) - 1
            x = self.r[idx, k]
            out[:, k] = np.where(s != 0, x + s * self.L[k], x)
        return torch.as_tensor(out.reshape(-1))

    def scatter_positions(self, idx, t):
        self.r[idx.numpy().astype(np.int64)] = t.numpy().reshape(-1, 3)

    # -- dynamics --------------------------------------------------------------
    def _vmax2_update(self):
        own = self.w == 0.0
        v2 = np.max(np.sum(self.v[own] ** 2, axis=1)) if own.any() else 0.0
        self.vmax2_bits = max(self.vmax2_bits, int(np.float64(v2).view(np.int64)))

    def move1(self):
        own = self.w == 0.0
        self.v[own] = self.v[own] + 0.5 * self.dt * self.a[own]
        self.r[own] = self.r[own] + self.dt * self.v[own]
        self._vmax2_update()

    def vmax2(self):
        return self.vmax2_bits

    def decide(self, vmax2, it, flip):
        rebuild = (it + 1) % self.tplot == 0
        if self.crit == 0:
            vmax = math.sqrt(float(np.int64(vmax2).view(np.float64)))
            self.rmax = self.rmax + vmax * self.dt
            if self.rmax > self.half_min_delta:
                rebuild = True
        elif it % self.fixed == 0:
            rebuild = True
        self.vmax2_bits = 0
        if rebuild:
            self.rmax = 0.0
        return int(rebuild)

    def forces(self, it, record, mode):
        n = len(self.gid)
        self.a = np.zeros((n, 3))
        self.pe = np.zeros(n)
        self.vir = np.zeros(n)
        for i in range(n):
            j = self.rows[i]
            if j.size == 0:
                continue
            d = self.r[i] - self.r[j]
            r2 = np.sum(d * d, axis=1)
            m = r2 < self.rc2
            d, r2 = d[m], r2[m]
            s = 1.0 / r2
            acc = 48.0 * (s ** 7 - 0.5 * s ** 4)
            self.a[i] = np.sum(acc[:, None] * d, axis=0)
            self.pe[i] = np.sum(4.0 * (s ** 6 - s ** 3) - self.potshift)
            self.vir[i] = np.sum(acc * r2)
        own = self.w == 0.0
        if mode >= 1:
            self.v[own] = self.v[own] + 0.5 * self.dt * self.a[own]
        if record:
            self._sums = np.zeros(D.NSUMS)
            self._sums[D.RS_PE] = math.fsum(self.pe[own])
            self._sums[D.RS_VIR] = math.fsum(self.vir[own])
            self._sums[D.RS_MV2] = math.fsum(np.sum(self.v[own] ** 2, axis=1))
            self._sums[D.RS_VSUM] = math.fsum(self.v[own].reshape(-1))
            self._sums[D.RS_PEMAX] = self.pe[own].max() if own.any() else 0.0
        if mode == 2:
            self.move1()

    def sums(self):
        return self._sums.copy()

    def macro(self, sums, it, simtime):
        gnp = float(self.np_global)
        mv2, vir = sums[D.RS_MV2], sums[D.RS_VIR]
        ke = 0.5 * mv2 / gnp
        pe = 0.5 * sums[D.RS_PE] / gnp
        return dict(iter=it, simtime=simtime, vsum=sums[D.RS_VSUM], mv2sum=mv2, temperature=mv2 / (3.0 * gnp),
                    kinenergy=ke, potenergy=pe, totenergy=ke + pe,
                    pressure=(self.density / (gnp * 3.0)) * (mv2 + vir / 2.0), virial=vir)

    def counts(self):
        own = int(np.sum(self.w == 0.0))
        return own, len(self.gid) - own

    def download(self):
        own = self.w == 0.0
        return self.r[own].copy(), self.v[own].copy(), self.gid[own].astype(np.int32)

    def owned_forces(self):
        own = self.w == 0.0
        return self.a[own].copy(), self.pe[own].copy(), self.gid[own].copy()

    def pair_list(self):
        code_of_cell = np.full(self.ncell, 13, np.int64)
        h = self.plan.halo_sources(self.rank)
        code_of_cell[h["cell"]] = D.code27(h["code"])
        o, p, c = [], [], []
        for i, row in enumerate(self.rows):
            if row.size == 0:
                continue
            o.append(np.full(row.size, self.gid[i]))
            p.append(self.gid[row])
            c.append(code_of_cell[self.cell[row]])
        if not o:
            return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.int64)
        return np.concatenate(o), np.concatenate(p), np.concatenate(c)

    def close(self):
        pass
