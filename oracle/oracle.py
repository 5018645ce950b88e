"""ctypes wrapper over the CPU FP64 oracle (fm_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline leg, and never by the product package.  Parity
status: see the header of fm_oracle.c (geometry and restart format pinned by
reference fixtures; forces and pair lists restated from the Fortran but
unpinned by reference outputs).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libfm_oracle.so")
_lib = None

ORC_ERRORS = {1: "allocation", 2: "escaped molecule", 3: "fewer than 3 cells",
              4: "polymer bond error", 5: "bad parameter"}


def build() -> str:
    """Compiles the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
                os.path.join(_HERE, "fm_oracle.c")):
            build()
        L = C.CDLL(_LIB)
        d3 = C.POINTER(C.c_double)
        i3 = C.POINTER(C.c_int)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, d3, C.c_double, d3, C.c_double, C.c_int, C.c_int, C.c_int,
                                 C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, i3]
        L.orc_free.argtypes = [C.c_void_p]
        for name in ("orc_r", "orc_v", "orc_a", "orc_potenergymol", "orc_virialmol"):
            getattr(L, name).restype = d3
            getattr(L, name).argtypes = [C.c_void_p]
        L.orc_glob_no.restype = i3
        L.orc_glob_no.argtypes = [C.c_void_p]
        for name in ("orc_np", "orc_halo_np", "orc_iter", "orc_rebuild_count", "orc_setup",
                     "orc_rebuild", "orc_compute_forces", "orc_assign_to_cell",
                     "orc_assign_to_neighbourlist", "orc_checkrebuild"):
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = [C.c_void_p]
        L.orc_updateborders.restype = C.c_int
        L.orc_updateborders.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_iter.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_integration_algorithm.argtypes = [C.c_void_p, C.c_int]
        L.orc_rmax.restype = C.c_double
        L.orc_rmax.argtypes = [C.c_void_p]
        L.orc_move_vv.argtypes = [C.c_void_p, C.c_int]
        L.orc_move_lfv.argtypes = [C.c_void_p]
        L.orc_sendmols.argtypes = [C.c_void_p]
        L.orc_linklist_deallocateall.argtypes = [C.c_void_p]
        L.orc_evaluate_macroscopic_properties.argtypes = [C.c_void_p]
        L.orc_macro.argtypes = [C.c_void_p, d3]
        L.orc_geometry.argtypes = [C.c_void_p, i3, d3, d3, d3, d3]
        L.orc_pair_list.restype = C.c_long
        L.orc_pair_list.argtypes = [C.c_void_p, i3, i3, i3, C.c_long]
        L.orc_list_length.restype = C.c_long
        L.orc_list_length.argtypes = [C.c_void_p]
        L.orc_run_vv.restype = C.c_int
        L.orc_run_vv.argtypes = [C.c_void_p, C.c_int, d3, C.c_int, i3]
        L.orc_global_domain.argtypes = [i3, C.c_double, d3, d3, d3]
        L.orc_set_parameters_cells.restype = C.c_int
        L.orc_set_parameters_cells.argtypes = [d3, d3, d3, C.c_int, C.c_int, C.c_double, i3, d3, d3]
        L.orc_set_solvent.restype = C.c_int
        L.orc_set_solvent.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_lj_accijmag.restype = C.c_double
        L.orc_lj_accijmag.argtypes = [C.c_double]
        L.orc_lj_energy.restype = C.c_double
        L.orc_lj_energy.argtypes = [C.c_double, C.c_double]
        L.orc_potshift.restype = C.c_double
        L.orc_potshift.argtypes = [C.c_double]
        L.orc_set_monomers.argtypes = [C.c_void_p, i3, i3, i3, i3]
        d8 = C.POINTER(C.c_double)
        L.orc_set_mie.argtypes = [C.c_void_p, C.c_int] + [d8] * 9 + [i3]
        L.orc_set_angular.restype = C.c_int
        L.orc_set_angular.argtypes = [C.c_void_p, C.c_int, d8, d8]
        L.orc_set_tags.argtypes = [C.c_void_p, C.c_int, i3, d3, d3, C.c_double, C.c_double, C.c_double, C.c_int,
                                   C.c_double, C.c_double]
        L.orc_set_pressure.argtypes = [C.c_void_p, C.c_int]
        L.orc_run_lfv.restype = C.c_int
        L.orc_run_lfv.argtypes = [C.c_void_p, C.c_int, d3, C.c_int, i3]
        L.orc_pressure_average.argtypes = [C.c_void_p, d3, i3]
        L.orc_bond_list.restype = C.c_long
        L.orc_bond_list.argtypes = [C.c_void_p, i3, i3, i3, C.c_long]
        L.orc_sort_table.argtypes = [C.c_int, i3, i3]
        L.orc_sort_mols.argtypes = [C.c_int, d3, d3, i3, d3, d3, C.c_int, C.c_int, C.c_int, i3,
                                    C.POINTER(SortState), i3, i3]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class OracleError(RuntimeError):
    pass


def _check(rc):
    if rc:
        raise OracleError(ORC_ERRORS.get(rc, f"error {rc}"))


class SortState(C.Structure):
    """The save variables of sort_mols (linklist.f90:2758-2762)."""
    _fields_ = [("nrebuilds", C.c_int), ("sf2", C.c_int), ("sf1", C.c_double)]

    def __init__(self):
        super().__init__(1, 5, 1.5)


def sort_table(sort_flag, nblocks):
    """Hcurve over nblocks sort blocks per axis, flat and x fastest
    (orc_sort_table)."""
    nb = np.ascontiguousarray(nblocks, dtype=np.int32)
    out = np.zeros(int(np.prod(nb)), np.int32)
    _check(lib().orc_sort_table(int(sort_flag), _ip(nb), _ip(out)))
    return out


def sort_mols(r, v, glob, domain, cellsidelength, sort_flag, sort_freq, sortblocksize, state):
    """One call of sort_mols on (n, 3) r and v and n global numbers.
    Returns (r, v, glob, perm, did): did 0 = order kept by the counter, 1 =
    sorted (perm[p] = old index now at p), 2 = a block overflowed."""
    r = np.array(r, dtype=np.float64, order="C"); v = np.array(v, dtype=np.float64, order="C")
    g = np.array(glob, dtype=np.int32)
    n = r.shape[0]
    nb = np.array([int(np.ceil(domain[k] / (sortblocksize * cellsidelength[k]))) for k in range(3)], np.int32)
    hc = sort_table(sort_flag, nb) if sort_flag else np.zeros(1, np.int32)
    perm = np.zeros(max(n, 1), np.int32); did = np.zeros(1, np.int32)
    dom = np.ascontiguousarray(domain, dtype=np.float64); cs = np.ascontiguousarray(cellsidelength, dtype=np.float64)
    _check(lib().orc_sort_mols(n, _dp(r), _dp(v), _ip(g), _dp(dom), _dp(cs), int(sort_flag), int(sort_freq),
                               int(sortblocksize), _ip(hc), C.byref(state), _ip(perm), _ip(did)))
    return r, v, g, (perm[:n] if did[0] == 1 else None), int(did[0])


def global_domain(nunits, density):
    n = np.ascontiguousarray(nunits, dtype=np.int32)
    dom = np.zeros(3); unit = np.zeros(3); vol = np.zeros(1)
    lib().orc_global_domain(_ip(n), float(density), _dp(dom), _dp(unit), _dp(vol))
    return dom, unit, float(vol[0])


def cells(domain, rcutoff, delta, potential_flag=0, R_0=1.5, solvent_flag=0):
    d = np.ascontiguousarray(domain, dtype=np.float64)
    dl = np.ascontiguousarray(delta, dtype=np.float64)
    nc = np.zeros(3, np.int32); cs = np.zeros(3); rn2 = np.zeros(1)
    rcio = np.array([float(rcutoff)])
    rc = lib().orc_set_parameters_cells(_dp(d), _dp(rcio), _dp(dl), int(potential_flag), int(solvent_flag),
                                        float(R_0), _ip(nc), _dp(cs), _dp(rn2))
    return rc, nc, cs, float(rn2[0])


class Oracle:
    """One FP64 CPU simulation state (single rank, fully periodic)."""

    def __init__(self, r, v, domain, rcutoff, delta_rneighbr=(0.3, 0.3, 0.3), delta_t=0.005,
                 tplot=100, force_list=3, potential_flag=0, k_c=30.0, R_0=1.5,
                 rebuild_criteria=0, fixed_rebuild=1, density=None, sLRC_flag=0, iter0=0,
                 integration_algorithm=1):
        r = np.asarray(r, dtype=np.float64)
        v = np.asarray(v, dtype=np.float64)
        self.np_ = r.shape[0]
        dom = np.ascontiguousarray(domain, dtype=np.float64)
        dl = np.ascontiguousarray(delta_rneighbr, dtype=np.float64)
        if density is None:
            density = self.np_ / float(np.prod(dom))
        err = C.c_int(0)
        L = lib()
        self.h = L.orc_create(self.np_, _dp(dom), float(rcutoff), _dp(dl), float(delta_t), int(tplot),
                              int(force_list), int(potential_flag), float(k_c), float(R_0),
                              int(rebuild_criteria), int(fixed_rebuild), float(density), int(sLRC_flag),
                              C.byref(err))
        if not self.h:
            _check(err.value or 1)
        self.domain = dom
        self._r = np.ctypeslib.as_array(L.orc_r(self.h), shape=(self.np_ * 8 + 1024, 3))
        self._v = np.ctypeslib.as_array(L.orc_v(self.h), shape=(self.np_ * 8 + 1024, 3))
        self._a = np.ctypeslib.as_array(L.orc_a(self.h), shape=(self.np_ * 8 + 1024, 3))
        self._r[:self.np_] = r
        self._v[:self.np_] = v
        L.orc_set_iter(self.h, int(iter0))
        L.orc_set_integration_algorithm(self.h, int(integration_algorithm))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_free(h)
            self.h = None

    # --- state ---
    @property
    def r(self):
        return self._r[:self.np_].copy()

    @property
    def v(self):
        return self._v[:self.np_].copy()

    @property
    def a(self):
        return self._a[:self.np_].copy()

    def set_state(self, r=None, v=None, a=None):
        if r is not None:
            self._r[:self.np_] = r
        if v is not None:
            self._v[:self.np_] = v
        if a is not None:
            self._a[:self.np_] = a

    def set_monomers(self, chain, subchain, funcy, bflag):
        c = np.ascontiguousarray(chain, np.int32)
        s = np.ascontiguousarray(subchain, np.int32)
        f = np.ascontiguousarray(funcy, np.int32)
        b = np.ascontiguousarray(bflag, np.int32).reshape(-1)
        lib().orc_set_monomers(self.h, _ip(c), _ip(s), _ip(f), _ip(b))

    def set_solvent(self, solvent_flag, eps_pp=1.0, eps_ps=1.0, eps_ss=1.0):
        """SOLVENT_INFO: 1 = Soddemann solvent of variable quality (chainID 0
        marks a solvent molecule); re-derives the cells.  Before setup()."""
        _check(lib().orc_set_solvent(self.h, int(solvent_flag), float(eps_pp), float(eps_ps), float(eps_ss)))

    def set_mie(self, tables, moltype):
        """Mie_potential 1: `tables` maps mass, epsilon, lambdar, lambdaa, C,
        alpha, potshift, k_harmonic, r0 to arrays (ntypes, or ntypes x
        ntypes indexed [i-1, j-1]); moltype is 1-based per molecule."""
        nt = len(tables["mass"])
        keep = [np.ascontiguousarray(tables["mass"], np.float64)]
        for k in ("epsilon", "lambdar", "lambdaa", "C", "alpha", "potshift", "k_harmonic", "r0"):
            keep.append(np.ascontiguousarray(np.asarray(tables[k], np.float64).T).reshape(-1))  # (i,j) at i + nt*j
        mt = np.ascontiguousarray(moltype, np.int32)
        _check(lib().orc_set_mie(self.h, nt, *[_dp(a) for a in keep], _ip(mt)))

    def set_angular(self, k, theta0):
        """angular_potential on: k and theta0 as (ntypes, ntypes, ntypes)
        arrays indexed [i-1, j-1, k-1] (angular_k_lookup, angular_r0_lookup).
        After set_mie(), before setup()."""
        kk = np.ascontiguousarray(np.asarray(k, np.float64).transpose(2, 1, 0)).reshape(-1)  # (i,j,k) at i+nt(j+nt k)
        tt = np.ascontiguousarray(np.asarray(theta0, np.float64).transpose(2, 1, 0)).reshape(-1)
        self._ang = (kk, tt)
        _check(lib().orc_set_angular(self.h, int(np.asarray(k).shape[0]), _dp(kk), _dp(tt)))

    @property
    def potenergymol(self):
        return np.ctypeslib.as_array(lib().orc_potenergymol(self.h), shape=(self.np_,)).copy()

    @property
    def virialmol(self):
        return np.ctypeslib.as_array(lib().orc_virialmol(self.h), shape=(self.np_,)).copy()

    @property
    def iter(self):
        return lib().orc_iter(self.h)

    @property
    def halo_np(self):
        return lib().orc_halo_np(self.h)

    @property
    def rebuild_count(self):
        return lib().orc_rebuild_count(self.h)

    def geometry(self):
        nc = np.zeros(3, np.int32); cs = np.zeros(3)
        rn2 = np.zeros(1); rc2 = np.zeros(1); ps = np.zeros(1)
        lib().orc_geometry(self.h, _ip(nc), _dp(cs), _dp(rn2), _dp(rc2), _dp(ps))
        return dict(ncells=nc, cellside=cs, rneighbr2=float(rn2[0]), rcutoff2=float(rc2[0]),
                    potshift=float(ps[0]))

    # --- subroutines ---
    def setup(self):
        _check(lib().orc_setup(self.h))

    def rebuild(self):
        _check(lib().orc_rebuild(self.h))

    def compute_forces(self):
        _check(lib().orc_compute_forces(self.h))

    def move_vv(self, pass_num):
        lib().orc_move_vv(self.h, int(pass_num))

    def checkrebuild(self):
        return lib().orc_checkrebuild(self.h)

    def macro(self):
        o = np.zeros(9)
        lib().orc_macro(self.h, _dp(o))
        keys = ("vsum", "mv2sum", "temperature", "kinenergy", "potenergy", "totenergy", "pressure",
                "virial", "potenergysum")
        return dict(zip(keys, o.tolist()))

    def evaluate_macroscopic_properties(self):
        lib().orc_evaluate_macroscopic_properties(self.h)
        return self.macro()

    def run_vv(self, nsteps, rec_cap=100000):
        out = np.zeros((rec_cap, 10))
        nrec = C.c_int(0)
        _check(lib().orc_run_vv(self.h, int(nsteps), _dp(out), rec_cap, C.byref(nrec)))
        return out[:min(nrec.value, rec_cap)]

    def set_tags(self, ensemble, tag=None, rtether=None, slidev=None, k=(0.0, 0.0, 0.0), nthermo=0,
                 therm_T=(0.0, 0.0)):
        tg = None if tag is None else np.ascontiguousarray(tag, np.int32)
        rt = None if rtether is None else np.ascontiguousarray(rtether, np.float64)
        sv = None if slidev is None else np.ascontiguousarray(slidev, np.float64)
        lib().orc_set_tags(self.h, int(ensemble), None if tg is None else _ip(tg), None if rt is None else _dp(rt),
                           None if sv is None else _dp(sv), float(k[0]), float(k[1]), float(k[2]), int(nthermo),
                           float(therm_T[0]), float(therm_T[1]))

    def set_pressure(self, flag=1):
        lib().orc_set_pressure(self.h, int(flag))

    def run_lfv(self, nsteps, rec_cap=100000):
        out = np.zeros((rec_cap, 10))
        nrec = C.c_int(0)
        _check(lib().orc_run_lfv(self.h, int(nsteps), _dp(out), rec_cap, C.byref(nrec)))
        return out[:min(nrec.value, rec_cap)]

    def pressure_average(self):
        out = np.zeros(9)
        n = C.c_int(0)
        lib().orc_pressure_average(self.h, _dp(out), C.byref(n))
        return out.reshape(3, 3), n.value

    def bond_list(self):
        cap = 4 * self.np_ + 16
        o = np.zeros(cap, np.int32); p = np.zeros(cap, np.int32); c = np.zeros(cap, np.int32)
        n = lib().orc_bond_list(self.h, _ip(o), _ip(p), _ip(c), cap)
        return o[:n], p[:n], c[:n]

    def pair_list(self):
        """(owner, partner, code) arrays, 1-based glob_no; code 13 = no image."""
        n = lib().orc_list_length(self.h)
        o = np.zeros(n, np.int32); p = np.zeros(n, np.int32); c = np.zeros(n, np.int32)
        m = lib().orc_pair_list(self.h, _ip(o), _ip(p), _ip(c), n)
        assert m == n
        return o, p, c
