"""Spatial domain decomposition of one system over ranks (the reference's MPI
build: messenger_init, messenger_updateborders, sendmols in
messenger.MPI.f90), on the subdomain calls of the C ABI (fm_dd_*).

Layout.  The box keeps global coordinates and the undivided system's cell
grid (fm_derive_geometry).  A Cartesian process grid (``find3factors``, or
given dims) splits the interior cells of each axis into contiguous runs;
each rank owns the molecules binned into its cells and holds, in its halo
layer, copies of the neighbouring ranks' boundary cells with the periodic
shift applied by the sender.  Because a rank's cells, the molecules in them
and their in-cell order (by global number) are the undivided system's, its
neighbour rows and forces are bit-identical to one handle over the whole box.

Exchanges are all-to-all of flat FP64 record buffers with per-destination
counts, through a ``Transport``: ``DistTransport`` (torch.distributed, one
subdomain per process: NCCL between GPUs, gloo on CPU) or ``LocalTransport``
(several subdomains in one process, e.g. all on one GPU).  Per step:
  * the rebuild decision takes the largest |v|^2 over ranks (all-reduce max,
    the reference's globalMax), so every rank rebuilds on the same steps;
  * on a rebuild: molecules that left a rank's cells move to their new owner
    (sendmols), then every rank sends the molecules of its boundary cells to
    the ranks whose halo holds them (messenger_updateborders, faces, edges
    and corners at once), sorts and builds its neighbour rows;
  * otherwise the halo copies' positions are refreshed from the same lists.
Records sum the ranks' totals (exactly rounded, in rank order).

Differences from the reference, by design: the reference gives each rank
local coordinates, domain/npx per axis and its own cell count
(setup_set_parameters.f90); here the split follows the global cell grid, so
the result does not depend on the number of ranks.  The reference's
three face-by-face passes of sendmols become one all-to-all (a molecule moves
at most one subdomain between rebuilds).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import api

MREC = 10  # FM_DD_MREC: r, v, a, global number
HREC = 5   # FM_DD_HREC: shifted r, global number, destination halo cell
NSUMS = 11
RS_PE, RS_VIR, RS_MV2, RS_VSUM, RS_PEMAX = 0, 1, 2, 3, 4


def find3factors(n: int):
    """Process grid of n ranks (functions_lib.f90:2735-2800): the cube-root
    guess if it multiplies out, else the prime factors merged smallest-first
    down to three, the largest on x."""
    nx = math.ceil(float(n) ** (1.0 / 3.0))
    ny = math.ceil((float(n) / float(nx)) ** 0.5)
    nz = math.ceil(float(n) / (float(nx) * float(ny)))
    if nx * ny * nz == n:
        return nx, ny, nz
    factors, m, i = [], n, 2
    while m > 1:
        if m % i == 0:
            factors.append(i)
            m //= i
        else:
            i += 1
    if len(factors) == 0:
        factors = [n]
    if len(factors) == 1:
        return factors[0], 1, 1
    if len(factors) == 2:
        return factors[0], factors[1], 1
    f = list(factors)
    while len(f) > 3:
        a = f.pop(f.index(min(f)))
        b = f.pop(f.index(min(f)))
        f.append(a * b)
    f.sort()
    return f[2], f[1], f[0]


def split_cells(ncells: int, parts: int):
    """Contiguous runs of `ncells` interior cells over `parts` ranks, the
    first ncells % parts runs one cell longer: [(origin, count)]."""
    if parts > ncells:
        raise ValueError(f"{parts} ranks along an axis of {ncells} cells")
    base, extra = divmod(ncells, parts)
    out, o = [], 0
    for p in range(parts):
        c = base + (1 if p < extra else 0)
        out.append((o, c))
        o += c
    return out


def code6(sx, sy, sz):
    return (sx + 1) | ((sy + 1) << 2) | ((sz + 1) << 4)


def code27(c6):
    """The 0..26 image code (13 = no shift) of a 6-bit code."""
    c6 = np.asarray(c6)
    return (c6 & 3) + 3 * ((c6 >> 2) & 3) + 9 * ((c6 >> 4) & 3)


class Plan:
    """The static part of a decomposition: the process grid (ranks numbered
    as MPI_Cart_create does, z fastest), each rank's cells, and for every
    halo cell of every rank the rank, cell and periodic shift it copies."""

    def __init__(self, ncells_global, dims):
        self.G = [int(x) for x in ncells_global]
        self.dims = [int(x) for x in dims]
        self.nranks = self.dims[0] * self.dims[1] * self.dims[2]
        self.runs = [split_cells(self.G[k], self.dims[k]) for k in range(3)]
        self.owner_axis = [np.concatenate([np.full(c, p, np.int32) for p, (_, c) in enumerate(self.runs[k])])
                           for k in range(3)]
        self._halo = [self._halo_sources(r) for r in range(self.nranks)]
        self._needs = [None] * self.nranks

    def coords(self, rank):
        return rank // (self.dims[1] * self.dims[2]), (rank // self.dims[2]) % self.dims[1], rank % self.dims[2]

    def rank_of(self, px, py, pz):
        return (px * self.dims[1] + py) * self.dims[2] + pz

    def box(self, rank):
        """(origin, ncells_local) per axis."""
        c = self.coords(rank)
        org = [self.runs[k][c[k]][0] for k in range(3)]
        nloc = [self.runs[k][c[k]][1] for k in range(3)]
        return org, nloc

    def ne(self, rank):
        _, nloc = self.box(rank)
        return [n + 2 for n in nloc]

    def _halo_sources(self, rank):
        """Halo cells of `rank` in ascending local index, as arrays: local
        cell, source rank, source rank's local cell, 6-bit image code."""
        org, nloc = self.box(rank)
        ne = [n + 2 for n in nloc]
        z, y, x = np.meshgrid(np.arange(ne[2]), np.arange(ne[1]), np.arange(ne[0]), indexing="ij")
        x, y, z = x.ravel(), y.ravel(), z.ravel()
        cell = x + ne[0] * (y + ne[1] * z)
        halo = (x == 0) | (y == 0) | (z == 0) | (x == ne[0] - 1) | (y == ne[1] - 1) | (z == ne[2] - 1)
        cell = cell[halo]
        loc = [x[halo], y[halo], z[halo]]
        g, s, own = [], [], []
        for k in range(3):
            gk = org[k] + loc[k] - 1
            sk = np.where(gk < 0, -1, np.where(gk >= self.G[k], 1, 0))
            gk = gk - sk * self.G[k]
            g.append(gk)
            s.append(sk)
            own.append(self.owner_axis[k][gk])
        src = (own[0] * self.dims[1] + own[1]) * self.dims[2] + own[2]
        src_cell = np.zeros_like(cell)
        for r in np.unique(src):
            m = src == r
            o2, n2 = self.box(int(r))
            ne2 = [n + 2 for n in n2]
            lx, ly, lz = (g[k][m] - o2[k] + 1 for k in range(3))
            src_cell[m] = lx + ne2[0] * (ly + ne2[1] * lz)
        code = (s[0] + 1) | ((s[1] + 1) << 2) | ((s[2] + 1) << 4)
        return dict(cell=cell.astype(np.int32), src=src.astype(np.int32), src_cell=src_cell.astype(np.int32),
                    code=code.astype(np.int32))

    def halo_sources(self, rank):
        return self._halo[rank]

    def needs(self, rank):
        """CSR over `rank`'s extended cells of (rank whose halo holds the
        cell, image code, that rank's halo cell)."""
        if self._needs[rank] is None:
            ncell = int(np.prod(self.ne(rank)))
            rk, cl, cd, hc = [], [], [], []
            for r in range(self.nranks):
                h = self._halo[r]
                m = h["src"] == rank
                rk.append(np.full(int(m.sum()), r, np.int32))
                cl.append(h["src_cell"][m])
                cd.append(h["code"][m])
                hc.append(h["cell"][m])
            rk, cl, cd, hc = (np.concatenate(a) for a in (rk, cl, cd, hc))
            order = np.lexsort((hc, rk, cl))
            rk, cl, cd, hc = rk[order], cl[order], cd[order], hc[order]
            off = np.zeros(ncell + 1, np.int32)
            np.add.at(off, cl + 1, 1)
            off = np.cumsum(off).astype(np.int32)
            self._needs[rank] = dict(off=off, rank=rk, code=cd, cell=hc)
        return self._needs[rank]

    def owner_axis_flat(self):
        return np.concatenate(self.owner_axis).astype(np.int32)

    def owner_of_positions(self, r, params_geom):
        """Rank owning each position (global binning of the undivided grid)."""
        hd, cs = params_geom["hd"], params_geom["cs"]
        g = [np.ceil((r[:, k] + hd[k]) / cs[k]).astype(np.int64) - 1 for k in range(3)]
        own = [self.owner_axis[k][np.clip(g[k], 0, self.G[k] - 1)] for k in range(3)]
        return (own[0] * self.dims[1] + own[1]) * self.dims[2] + own[2]


def refresh_lists(plan: Plan, rank: int, starts: np.ndarray, starts_of=None):
    """Per-step halo refresh lists of `rank` from its cell starts after a
    rebuild.  Sending: for each destination rank (ascending), its halo cells
    copied from here in ascending order, each the molecules of the source
    cell with the cell's image code.  Receiving: for each source rank, this
    rank's halo cells copied from it, ascending.  Both sides order a cell's
    molecules by global number, so entry k on one side is entry k on the
    other.  Returns (send_idx, send_code, send_counts, recv_idx, recv_counts)."""
    send_idx, send_code, send_counts = [], [], np.zeros(plan.nranks, np.int64)
    for r in range(plan.nranks):
        h = plan.halo_sources(r)
        m = h["src"] == rank
        cells, codes = h["src_cell"][m], h["code"][m]  # ascending in r's halo cell
        b, e = starts[cells], starts[cells + 1]
        cnt = e - b
        idx = _ranges(b, cnt)
        send_idx.append(idx)
        send_code.append(np.repeat(codes, cnt))
        send_counts[r] = idx.size
    mine = plan.halo_sources(rank)
    recv_idx, recv_counts = [], np.zeros(plan.nranks, np.int64)
    for s in range(plan.nranks):
        m = mine["src"] == s
        cells = mine["cell"][m]
        b, e = starts[cells], starts[cells + 1]
        idx = _ranges(b, e - b)
        recv_idx.append(idx)
        recv_counts[s] = idx.size
    return (np.concatenate(send_idx).astype(np.int32), np.concatenate(send_code).astype(np.int8), send_counts,
            np.concatenate(recv_idx).astype(np.int32), recv_counts)


def _ranges(begin, count):
    begin = np.asarray(begin, np.int64)
    count = np.asarray(count, np.int64)
    tot = int(count.sum())
    if tot == 0:
        return np.zeros(0, np.int64)
    starts = np.repeat(begin - np.concatenate([[0], np.cumsum(count)[:-1]]), count)
    return starts + np.arange(tot)


# ---------------------------------------------------------------------------
# transports
# ---------------------------------------------------------------------------

class LocalTransport:
    """All subdomains in this process; every method takes one item per rank."""

    def alltoall_counts(self, counts):
        c = np.stack([np.asarray(x, np.int64) for x in counts])
        return [c[:, r].copy() for r in range(c.shape[0])]

    def alltoall(self, sends, send_counts, recv_counts, width):
        import torch
        n = len(sends)
        parts = [torch.split(sends[s], [int(c) * width for c in send_counts[s]]) for s in range(n)]
        return [torch.cat([parts[s][r] for s in range(n)]) if n else None for r in range(n)]

    def max_int(self, vals):
        return [max(int(v) for v in vals)] * len(vals)

    def gather_rows(self, rows):
        a = np.stack([np.asarray(x, np.float64) for x in rows])
        return [a] * len(rows)


class DistTransport:
    """One subdomain per process over torch.distributed (NCCL with CUDA
    tensors, gloo with CPU tensors)."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.device = device if device is not None else torch.device("cpu")

    def alltoall_counts(self, counts):
        import torch
        t = torch.as_tensor(np.asarray(counts[0], np.int64), device=self.device)
        out = torch.empty_like(t)
        self.dist.all_to_all_single(out, t, group=self.group)
        return [out.cpu().numpy()]

    def alltoall(self, sends, send_counts, recv_counts, width):
        import torch
        src = sends[0]
        out = torch.empty(int(np.sum(recv_counts[0])) * width, dtype=src.dtype, device=src.device)
        self.dist.all_to_all_single(out, src, [int(c) * width for c in recv_counts[0]],
                                    [int(c) * width for c in send_counts[0]], group=self.group)
        return [out]

    def max_int(self, vals):
        import torch
        t = torch.tensor([int(vals[0])], dtype=torch.int64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
        return [int(t.item())]

    def gather_rows(self, rows):
        import torch
        t = torch.as_tensor(np.asarray(rows[0], np.float64), device=self.device)
        out = [torch.empty_like(t) for _ in range(self.dist.get_world_size(self.group))]
        self.dist.all_gather(out, t, group=self.group)
        return [np.stack([o.cpu().numpy() for o in out])]


# ---------------------------------------------------------------------------
# one rank's subdomain on the GPU (C ABI)
# ---------------------------------------------------------------------------

def _i32(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class Subdomain:
    """One rank's subdomain on a CUDA device (fm_dd_* calls).  Buffers are
    torch tensors on the device, ordered on torch's current stream."""

    def __init__(self, params: api.FmParams, plan: Plan, rank: int, capacity: int, device=None):
        import torch
        self.torch = torch
        self.plan, self.rank = plan, rank
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        org, nloc = plan.box(rank)
        self.h = C.c_void_p()
        G = (C.c_int32 * 3)(*plan.G)
        o = (C.c_int32 * 3)(*org)
        n = (C.c_int32 * 3)(*nloc)
        with torch.cuda.device(self.device):
            api.check(api.lib().fm_dd_create(C.byref(params), G, o, n, int(capacity), C.byref(self.h)))
            api.check(api.lib().fm_set_stream(self.h, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        nd = plan.needs(rank)
        dims = (C.c_int32 * 3)(*plan.dims)
        self._keep = [plan.owner_axis_flat(), nd["off"], nd["rank"], nd["code"], nd["cell"]]
        api.check(api.lib().fm_dd_set_plan(self.h, rank, dims, *[_i32(np.ascontiguousarray(a, np.int32))
                                                                 for a in self._keep]))
        self.ncell = int(np.prod(plan.ne(rank)))

    def close(self):
        if self.h:
            api.lib().fm_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ptr(self, t):
        return C.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else C.c_void_p()

    def upload(self, r, v, gid):
        r = np.ascontiguousarray(r, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        gid = np.ascontiguousarray(gid, np.int32)
        api.check(api.lib().fm_dd_upload(self.h, len(gid), api._dp(r), api._dp(v), _i32(gid)))

    def classify(self, wrap):
        c = np.zeros(self.plan.nranks, np.int32)
        api.check(api.lib().fm_dd_classify(self.h, int(wrap), _i32(c)))
        return c

    def pack_emigrants(self, counts):
        t = self.torch.empty(int(np.sum(counts)) * MREC, dtype=self.torch.float64, device=self.device)
        api.check(api.lib().fm_dd_pack_emigrants(self.h, self._ptr(t)))
        return t

    def immigrate(self, recv, n):
        api.check(api.lib().fm_dd_immigrate(self.h, self._ptr(recv), int(n)))

    def halo_counts(self):
        c = np.zeros(self.plan.nranks, np.int32)
        api.check(api.lib().fm_dd_halo_counts(self.h, _i32(c)))
        return c

    def pack_halo(self, counts):
        t = self.torch.empty(int(np.sum(counts)) * HREC, dtype=self.torch.float64, device=self.device)
        api.check(api.lib().fm_dd_pack_halo(self.h, self._ptr(t)))
        return t

    def receive_halo(self, recv, n):
        api.check(api.lib().fm_dd_receive_halo(self.h, self._ptr(recv), int(n)))

    def cell_starts(self):
        s = np.zeros(self.ncell + 1, np.int32)
        api.check(api.lib().fm_dd_cell_starts(self.h, _i32(s)))
        return s

    def to_device(self, a):
        return self.torch.as_tensor(a).to(self.device)

    def gather_positions(self, idx, code):
        t = self.torch.empty(idx.numel() * 3, dtype=self.torch.float64, device=self.device)
        api.check(api.lib().fm_dd_gather_positions(self.h, self._ptr(idx), self._ptr(code), idx.numel(),
                                                   self._ptr(t)))
        return t

    def scatter_positions(self, idx, t):
        api.check(api.lib().fm_dd_scatter_positions(self.h, self._ptr(idx), self._ptr(t), idx.numel()))

    def move1(self):
        api.check(api.lib().fm_dd_move1(self.h))

    def vmax2(self):
        v = C.c_uint64()
        api.check(api.lib().fm_dd_vmax2(self.h, C.byref(v)))
        return v.value

    def decide(self, vmax2, it, flip):
        rb = C.c_int32()
        api.check(api.lib().fm_dd_decide(self.h, C.c_uint64(int(vmax2)), int(it), int(flip), C.byref(rb)))
        return rb.value

    def forces(self, it, record, mode):
        api.check(api.lib().fm_dd_forces(self.h, int(it), int(record), int(mode)))

    def sums(self):
        s = np.zeros(NSUMS)
        api.check(api.lib().fm_dd_sums(self.h, api._dp(s)))
        return s

    def macro(self, sums, it, simtime):
        m = api.FmMacro()
        s = np.ascontiguousarray(sums, np.float64)
        api.check(api.lib().fm_dd_macro(self.h, api._dp(s), int(it), float(simtime), C.byref(m)))
        return m.as_dict()

    def counts(self):
        a, b = C.c_int32(), C.c_int32()
        api.check(api.lib().fm_dd_counts(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def download(self):
        n_own, _ = self.counts()
        n = C.c_int32()
        r = np.zeros((max(n_own, 1), 3)); v = np.zeros((max(n_own, 1), 3)); g = np.zeros(max(n_own, 1), np.int32)
        api.check(api.lib().fm_dd_download(self.h, n_own, C.byref(n), api._dp(r), api._dp(v), _i32(g)))
        return r[:n.value], v[:n.value], g[:n.value]

    def pair_list(self):
        """(owner gid, partner gid, 0..26 image code) of every row entry."""
        n = C.c_int64()
        api.check(api.lib().fm_dd_pair_list(self.h, None, None, None, 0, C.byref(n)))
        o = np.zeros(max(n.value, 1), np.int32); p = np.zeros_like(o); c = np.zeros_like(o)
        api.check(api.lib().fm_dd_pair_list(self.h, _i32(o), _i32(p), _i32(c), n.value, C.byref(n)))
        o, p, c = o[:n.value], p[:n.value], c[:n.value]
        code_of_cell = np.full(self.ncell, 13, np.int64)
        h = self.plan.halo_sources(self.rank)
        code_of_cell[h["cell"]] = code27(h["code"])
        return o, p, code_of_cell[c]


# ---------------------------------------------------------------------------
# the decomposed system
# ---------------------------------------------------------------------------

@dataclass
class _Lists:
    send_idx: object = None
    send_code: object = None
    send_counts: np.ndarray = None
    recv_idx: object = None
    recv_counts: np.ndarray = None


class DecomposedSystem:
    """Drives the subdomains of this process (all of them with a
    LocalTransport, this rank's with a DistTransport) through setup and
    velocity-Verlet steps (md_advance_vv with the MPI halo exchange and
    sendmols on rebuilds)."""

    def __init__(self, params: api.FmParams, plan: Plan, subs, transport):
        self.p = params
        self.plan = plan
        self.subs = list(subs)
        self.t = transport
        self.iter = int(params.initialstep)
        self.simtime = float(params.simtime)
        self.records = []
        self._lists = [_Lists() for _ in self.subs]
        self.rebuilds = 0

    # -- phases --------------------------------------------------------------
    def rebuild(self, wrap):
        subs, t = self.subs, self.t
        counts = [s.classify(wrap) for s in subs]
        rc = t.alltoall_counts(counts)
        sends = [s.pack_emigrants(c) for s, c in zip(subs, counts)]
        recvs = t.alltoall(sends, counts, rc, MREC)
        for s, buf, c in zip(subs, recvs, rc):
            s.immigrate(buf, int(np.sum(c)))
        hc = [s.halo_counts() for s in subs]
        hrc = t.alltoall_counts(hc)
        hs = [s.pack_halo(c) for s, c in zip(subs, hc)]
        hr = t.alltoall(hs, hc, hrc, HREC)
        for s, buf, c in zip(subs, hr, hrc):
            s.receive_halo(buf, int(np.sum(c)))
        for k, s in enumerate(subs):
            si, sc, sn, ri, rn = refresh_lists(self.plan, s.rank, s.cell_starts())
            self._lists[k] = _Lists(s.to_device(si), s.to_device(sc), sn, s.to_device(ri), rn)
        self.rebuilds += 1

    def refresh(self):
        L = self._lists
        sends = [s.gather_positions(l.send_idx, l.send_code) for s, l in zip(self.subs, L)]
        recvs = self.t.alltoall(sends, [l.send_counts for l in L], [l.recv_counts for l in L], 3)
        for s, l, buf in zip(self.subs, L, recvs):
            s.scatter_positions(l.recv_idx, buf)

    def _record(self, it):
        rows = self.t.gather_rows([s.sums() for s in self.subs])[0]
        tot = np.array([max(rows[:, k]) if k == RS_PEMAX else math.fsum(rows[:, k]) for k in range(NSUMS)])
        self.records.append(self.subs[0].macro(tot, it, self.simtime))

    # -- the md.f90 driver ---------------------------------------------------
    def setup(self):
        """setup_initial_record's first force evaluation: cells (no wrap),
        rows, forces, and the record of the initial step."""
        self.rebuild(wrap=0)
        record = self.iter % self.p.tplot == 0
        for s in self.subs:
            s.forces(self.iter, record, 0)
        if record:
            self._record(self.iter)

    def run(self, nsteps):
        """nsteps velocity-Verlet iterations: move(1) (fused into the previous
        force kernel after the first), the rebuild decision on the ranks'
        largest |v|^2, rebuild or halo refresh, forces with move(2) (and the
        next move(1)), records on tplot steps."""
        first = self.iter + 1
        for k in range(nsteps):
            it = first + k
            if k == 0:
                for s in self.subs:
                    s.move1()
            v = self.t.max_int([s.vmax2() for s in self.subs])
            rb = [s.decide(vv, it, 0 if k == 0 else 1) for s, vv in zip(self.subs, v)]
            if any(rb) != all(rb):
                raise RuntimeError("ranks disagree on the rebuild decision")
            if rb[0]:
                self.rebuild(wrap=1)
            else:
                self.refresh()
            record = it % self.p.tplot == 0
            mode = 1 if k == nsteps - 1 else 2
            for s in self.subs:
                s.forces(it, record, mode)
            self.simtime = self.simtime + self.p.delta_t
            if record:
                self._record(it)
        self.iter = first + nsteps - 1

    def state(self):
        """(r, v, gid) of this process's subdomains, concatenated."""
        parts = [s.download() for s in self.subs]
        return (np.concatenate([p[0] for p in parts]), np.concatenate([p[1] for p in parts]),
                np.concatenate([p[2] for p in parts]))

    def close(self):
        for s in self.subs:
            s.close()


def geometry(params: api.FmParams):
    rc, g = api.derive_geometry(params)
    api.check(rc)
    dom = np.array(list(params.domain))
    return dict(ncells=g["ncells"], cs=np.array(g["cellside"]), hd=0.5 * dom, L=dom)


def distribute(params: api.FmParams, plan: Plan, r, v):
    """Global numbers (0-based upload order) of each rank's molecules, by the
    undivided grid's binning of the (in-box) positions."""
    own = plan.owner_of_positions(np.asarray(r), geometry(params))
    return [np.nonzero(own == k)[0].astype(np.int32) for k in range(plan.nranks)]


def local_system(params: api.FmParams, r, v, dims=None, nranks=None, capacity_factor=2.0):
    """All ranks of a decomposition as subdomains of this process's current
    CUDA device, exchanging through device copies.  Returns the
    DecomposedSystem, uploaded but not set up."""
    g = geometry(params)
    if dims is None:
        dims = find3factors(int(nranks))
    plan = Plan(g["ncells"], dims)
    parts = distribute(params, plan, r, v)
    n = len(r)
    subs = []
    for k in range(plan.nranks):
        org, nloc = plan.box(k)
        ext = np.prod([c + 2 for c in nloc]) / np.prod(nloc)
        cap = int(capacity_factor * ext * max(len(parts[k]), n / plan.nranks)) + 1024
        s = Subdomain(params, plan, k, min(cap, api_max_molecules()))
        s.upload(np.asarray(r)[parts[k]], np.asarray(v)[parts[k]], parts[k])
        subs.append(s)
    return DecomposedSystem(params, plan, subs, LocalTransport())


def api_max_molecules():
    return (1 << 26) - 1
