"""ctypes binding of libflowmol_b200.so (C ABI in include/flowmol_b200.h).

``MDSystem`` exposes the reference's hot-path subroutines under their own
names (simulation_move_particles_vv, messenger_updateborders,
simulation_checkrebuild, linklist_deallocateall, sendmols, assign_to_cell,
assign_to_neighbourlist, simulation_compute_forces,
evaluate_macroscopic_properties) plus ``md_advance_vv`` and the fused
``simulation_md`` loop, so a driver written against Flowmol's md.f90 reads
the same.  Every call goes to the CUDA library; there is no CPU path, and a
missing library raises at import of this module's first use.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libflowmol_b200.so")

FM_OK = 0
ERRORS = {1: "ARG", 2: "CUDA", 3: "FEWCELLS", 4: "ESCAPE", 5: "NLIST", 6: "PE", 7: "STATE", 8: "BOND",
          9: "NODEVICE", 10: "IO"}

FORCE_LIST_ALLPAIRS, FORCE_LIST_FULL, FORCE_LIST_HALF = 0, 2, 3
PRECISION_FP64, PRECISION_FP32 = 0, 1


class FmParams(C.Structure):
    _fields_ = [
        ("np", C.c_int32),
        ("domain", C.c_double * 3),
        ("density", C.c_double),
        ("rcutoff", C.c_double),
        ("delta_rneighbr", C.c_double * 3),
        ("delta_t", C.c_double),
        ("tplot", C.c_int32),
        ("initialstep", C.c_int32),
        ("simtime", C.c_double),
        ("force_list", C.c_int32),
        ("potential_flag", C.c_int32),
        ("rebuild_criteria", C.c_int32),
        ("fixed_rebuild", C.c_int32),
        ("sLRC_flag", C.c_int32),
        ("precision", C.c_int32),
        ("k_c", C.c_double),
        ("R_0", C.c_double),
        ("nlist_capacity", C.c_int32),
        ("threads_per_molecule", C.c_int32),
        ("integration_algorithm", C.c_int32),
        ("list_build", C.c_int32),
        ("solvent_flag", C.c_int32),
        ("force_path", C.c_int32),
        ("eps_pp", C.c_double),
        ("eps_ps", C.c_double),
        ("eps_ss", C.c_double),
    ]


class FmMacro(C.Structure):
    _fields_ = [
        ("iter", C.c_int32), ("pad_", C.c_int32), ("simtime", C.c_double), ("vsum", C.c_double),
        ("mv2sum", C.c_double), ("temperature", C.c_double), ("kinenergy", C.c_double),
        ("potenergy", C.c_double), ("totenergy", C.c_double), ("pressure", C.c_double),
        ("virial", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad_"}


class FmEngineParams(C.Structure):
    _fields_ = [
        ("max_molecules", C.c_int64), ("max_cells", C.c_int64), ("max_list_entries", C.c_int64),
        ("max_slots", C.c_int32), ("precision", C.c_int32), ("threads_per_molecule", C.c_int32),
        ("ticks_per_chunk", C.c_int32), ("keep_states", C.c_int32), ("list_build", C.c_int32),
        ("delta_t", C.c_double),
    ]


class FmMieTables(C.Structure):
    _fields_ = [("ntypes", C.c_int32), ("pad_", C.c_int32)] + [
        (k, C.POINTER(C.c_double)) for k in ("mass", "epsilon", "lambdar", "lambdaa", "C", "alpha", "potshift",
                                             "k_harmonic", "r0")]


LIST_BUILD_AUTO, LIST_BUILD_CELLS, LIST_BUILD_BLOCKS = 0, 1, 2
FORCE_PATH_AUTO, FORCE_PATH_GATHER, FORCE_PATH_TILES = 0, 1, 2
LIST_BUILD_AUTO, LIST_BUILD_CELLS, LIST_BUILD_BLOCKS = 0, 1, 2
MIE_TABLE_KEYS = ("epsilon", "lambdar", "lambdaa", "C", "alpha", "potshift", "k_harmonic", "r0")


class FmJob(C.Structure):
    _fields_ = [
        ("np", C.c_int32), ("tplot", C.c_int32), ("domain", C.c_double * 3), ("density", C.c_double),
        ("rcutoff", C.c_double), ("delta_rneighbr", C.c_double * 3), ("nsteps", C.c_int32),
        ("initialstep", C.c_int32), ("integration_algorithm", C.c_int32), ("ensemble", C.c_int32),
        ("force_list", C.c_int32), ("pressure_outflag", C.c_int32), ("nthermo", C.c_int32),
        ("rebuild_criteria", C.c_int32), ("fixed_rebuild", C.c_int32), ("nlist_capacity", C.c_int32),
        ("thermostat_temperature", C.c_double * 2), ("teth_k2", C.c_double), ("teth_k4", C.c_double),
        ("teth_k6", C.c_double),
    ]


class FmJobResult(C.Structure):
    _fields_ = [
        ("job_id", C.c_int64), ("status", C.c_int32), ("nsamples", C.c_int32), ("final_iter", C.c_int32),
        ("rebuilds", C.c_int32), ("retries", C.c_int32), ("pad_", C.c_int32), ("ptensor", C.c_double * 9),
        ("last", FmMacro), ("submit_time", C.c_double), ("admit_time", C.c_double), ("finish_time", C.c_double),
    ]

    def as_dict(self):
        return dict(job_id=self.job_id, status=self.status, nsamples=self.nsamples, final_iter=self.final_iter,
                    rebuilds=self.rebuilds, retries=self.retries,
                    ptensor=np.array(list(self.ptensor)).reshape(3, 3), last=self.last.as_dict(),
                    submit_time=self.submit_time, admit_time=self.admit_time, finish_time=self.finish_time)


RESTART_MAXPROC = 4096


class FmRestartHeader(C.Structure):
    _fields_ = [
        ("globalnp", C.c_int32), ("initialnunits", C.c_int32 * 3), ("nsteps", C.c_int32), ("tplot", C.c_int32),
        ("seed", C.c_int32 * 2), ("periodic", C.c_int32 * 3), ("potential_flag", C.c_int32),
        ("rtrue_flag", C.c_int32), ("solvent_flag", C.c_int32), ("nmonomers", C.c_int32), ("npx", C.c_int32),
        ("npy", C.c_int32), ("npz", C.c_int32), ("nproc", C.c_int32), ("mie_potential", C.c_int32),
        ("global_numbering", C.c_int32), ("header_pos", C.c_int64), ("globaldomain", C.c_double * 3),
        ("density", C.c_double), ("rcutoff", C.c_double), ("delta_t", C.c_double), ("elapsedtime", C.c_double),
        ("simtime", C.c_double), ("k_c", C.c_double), ("R_0", C.c_double), ("eps_pp", C.c_double),
        ("eps_ps", C.c_double), ("eps_ss", C.c_double), ("delta_rneighbr", C.c_double),
        ("procnp", C.c_int32 * RESTART_MAXPROC), ("proctethernp", C.c_int32 * RESTART_MAXPROC),
    ]


class FmInput(C.Structure):
    _fields_ = [
        ("ensemble", C.c_int32), ("integration_algorithm", C.c_int32), ("force_list", C.c_int32),
        ("potential_flag", C.c_int32), ("nsteps", C.c_int32), ("tplot", C.c_int32),
        ("rebuild_criteria", C.c_int32), ("fixed_rebuild", C.c_int32), ("initialnunits", C.c_int32 * 3),
        ("periodic", C.c_int32 * 3), ("sort_flag", C.c_int32), ("global_numbering", C.c_int32),
        ("pressure_outflag", C.c_int32), ("sLRC_flag", C.c_int32), ("mie_potential", C.c_int32),
        ("nmonomers", C.c_int32), ("nthermo", C.c_int32), ("solvent_flag", C.c_int32),
        ("density", C.c_double), ("rcutoff", C.c_double), ("inputtemperature", C.c_double), ("delta_t", C.c_double),
        ("delta_rneighbr", C.c_double * 3), ("k_c", C.c_double), ("R_0", C.c_double),
        ("tethereddisttop", C.c_double * 3), ("tethereddistbottom", C.c_double * 3),
        ("thermstattop", C.c_double * 3), ("thermstatbottom", C.c_double * 3), ("slidedisttop", C.c_double * 3),
        ("slidedistbottom", C.c_double * 3), ("fixdisttop", C.c_double * 3), ("fixdistbottom", C.c_double * 3),
        ("wallslidev", C.c_double * 3), ("teth_k", C.c_double * 3), ("thermostattemperature", C.c_double * 2),
        ("targetconc", C.c_double), ("eps_pp", C.c_double), ("eps_ps", C.c_double), ("eps_ss", C.c_double),
        ("sort_freq", C.c_int32), ("sortblocksize", C.c_int32),
    ]

    def as_dict(self):
        out = {}
        for k, _ in self._fields_:
            if k == "pad_":
                continue
            x = getattr(self, k)
            out[k] = list(x) if hasattr(x, "__len__") else x
        return out


class FlowmolError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"FM_ERR_{ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m flowmol_b200.build` "
                              "(the MD path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        h = C.c_void_p
        sig = {
            "fm_derive_geometry": [P(FmParams), P(C.c_int32), P(C.c_double), P(C.c_double), P(C.c_double),
                                   P(C.c_double)],
            "fm_global_domain": [P(C.c_int32), C.c_double, P(C.c_double)],
            "fm_create": [P(FmParams), P(h)],
            "fm_destroy": [h],
            "fm_set_stream": [h, C.c_void_p],
            "fm_upload_state": [h, C.c_int32, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_int32)],
            "fm_download_state": [h, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_int32)],
            "fm_upload_state_device": [h, C.c_int32, C.c_void_p, C.c_void_p],
            "fm_download_state_device": [h, C.c_void_p, C.c_void_p, C.c_void_p],
            "fm_setup": [h],
            "fm_move_vv": [h, C.c_int32],
            "fm_move_lfv": [h],
            "fm_upload_monomers": [h, P(C.c_int32), P(C.c_int32), P(C.c_int32)],
            "fm_set_mie": [h, P(FmMieTables), P(C.c_int32)],
            "fm_set_angular": [h, C.c_int32, P(C.c_double), P(C.c_double), P(C.c_int32)],
            "fm_get_bonds": [h, P(C.c_int32), P(C.c_int32), P(C.c_int8), C.c_int64, P(C.c_int64)],
            "fm_update_borders": [h, C.c_int32],
            "fm_check_rebuild": [h, P(C.c_int32)],
            "fm_linklist_deallocateall": [h],
            "fm_sendmols": [h],
            "fm_sort_mols": [h],
            "fm_set_sort": [h, C.c_int32, C.c_int32, C.c_int32],
            "fm_get_sort_state": [h, P(C.c_int64), P(C.c_int64), P(C.c_int32), P(C.c_double), P(C.c_int32)],
            "fm_sort_table": [C.c_int32, P(C.c_int32), P(C.c_int32), C.c_int64],
            "fm_rebuild_lists": [h],
            "fm_assign_to_cell": [h],
            "fm_assign_to_neighbourlist": [h],
            "fm_compute_forces": [h],
            "fm_evaluate_macroscopic_properties": [h, P(FmMacro)],
            "fm_set_iter": [h, C.c_int32],
            "fm_get_iter": [h, P(C.c_int32)],
            "fm_step": [h, C.c_int32, C.c_int32],
            "fm_sync": [h],
            "fm_get_records": [h, P(FmMacro), C.c_int32, P(C.c_int32)],
            "fm_get_per_molecule": [h, P(C.c_double), P(C.c_double)],
            "fm_get_pair_list": [h, P(C.c_int32), P(C.c_int32), P(C.c_int8), C.c_int64, P(C.c_int64)],
            "fm_pair_digest": [h, P(C.c_uint64), P(C.c_int64)],
            "fm_get_counters": [h, P(C.c_int64), P(C.c_int32), P(C.c_int32)],
            "fm_set_pressure_outflag": [h, C.c_int32],
            "fm_get_pressure_tensor": [h, P(C.c_double), P(C.c_int32), C.c_int32],
            "fm_get_threads_per_molecule": [h, P(C.c_int32)],
            "fm_get_force_path": [h, P(C.c_int32), P(C.c_int32)],
            "fm_last_error": [C.c_char_p, C.c_int32],
            "fm_engine_create": [P(FmEngineParams), P(h)],
            "fm_engine_destroy": [h],
            "fm_engine_set_stream": [h, C.c_void_p],
            "fm_engine_submit": [h, P(FmJob), P(C.c_double), P(C.c_double), P(C.c_int32), P(C.c_double),
                                 P(C.c_double), P(C.c_int64)],
            "fm_engine_step_chunk": [h, P(C.c_int32), P(C.c_int32)],
            "fm_engine_run": [h, C.c_int32],
            "fm_engine_take_results": [h, P(FmJobResult), C.c_int32, P(C.c_int32)],
            "fm_engine_job_state": [h, C.c_int64, P(C.c_double), P(C.c_double)],
            "fm_engine_counters": [h, P(C.c_int64), P(C.c_int64), P(C.c_int32), P(C.c_int64)],
            "fm_engine_tuning": [h, P(C.c_int32), P(C.c_double)],
            "fm_read_final_state": [C.c_char_p, P(FmRestartHeader), C.c_int32, P(C.c_double), P(C.c_double),
                                    P(C.c_int32), P(C.c_double), P(C.c_int32), P(C.c_double), P(C.c_int32),
                                    P(C.c_double)],
            "fm_write_final_state": [C.c_char_p, P(FmRestartHeader), P(C.c_double), P(C.c_double), P(C.c_int32),
                                     P(C.c_double), P(C.c_int32), P(C.c_double), P(C.c_int32), P(C.c_double)],
            "fm_read_input": [C.c_char_p, P(FmInput)],
            "fm_force_kernel_timing": [h, C.c_int32],
            "fm_get_force_kernel_time": [h, P(C.c_double), P(C.c_int64)],
            "fm_get_launch_count": [h, P(C.c_int64)],
            "fm_dd_create": [P(FmParams), P(C.c_int32), P(C.c_int32), P(C.c_int32), C.c_int32, P(h)],
            "fm_dd_set_plan": [h, C.c_int32, P(C.c_int32), P(C.c_int32), P(C.c_int32), P(C.c_int32),
                               P(C.c_int32), P(C.c_int32)],
            "fm_dd_upload": [h, C.c_int32, P(C.c_double), P(C.c_double), P(C.c_int32)],
            "fm_dd_classify": [h, C.c_int32, P(C.c_int32)],
            "fm_dd_pack_emigrants": [h, C.c_void_p],
            "fm_dd_immigrate": [h, C.c_void_p, C.c_int32],
            "fm_dd_halo_counts": [h, P(C.c_int32)],
            "fm_dd_pack_halo": [h, C.c_void_p],
            "fm_dd_receive_halo": [h, C.c_void_p, C.c_int32],
            "fm_dd_counts": [h, P(C.c_int32), P(C.c_int32)],
            "fm_dd_cell_starts": [h, P(C.c_int32)],
            "fm_dd_gather_positions": [h, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p],
            "fm_dd_scatter_positions": [h, C.c_void_p, C.c_void_p, C.c_int32],
            "fm_dd_move1": [h],
            "fm_dd_vmax2": [h, P(C.c_uint64)],
            "fm_dd_decide": [h, C.c_uint64, C.c_int32, C.c_int32, P(C.c_int32)],
            "fm_dd_forces": [h, C.c_int32, C.c_int32, C.c_int32],
            "fm_dd_sums": [h, P(C.c_double)],
            "fm_dd_macro": [h, P(C.c_double), C.c_int32, C.c_double, P(FmMacro)],
            "fm_dd_download": [h, C.c_int32, P(C.c_int32), P(C.c_double), P(C.c_double), P(C.c_int32)],
            "fm_dd_pair_list": [h, P(C.c_int32), P(C.c_int32), P(C.c_int32), C.c_int64, P(C.c_int64)],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        _lib = L
    return _lib


def exported_symbols():
    """Names declared in include/flowmol_b200.h that the loaded library exports."""
    L = lib()
    out = []
    hdr = os.path.join(os.path.dirname(_PKG), "include", "flowmol_b200.h")
    import re
    for name in re.findall(r"FM_API int (fm_\w+)\(", open(hdr).read()):
        getattr(L, name)  # raises AttributeError when missing
        out.append(name)
    return out


def last_error() -> str:
    buf = C.create_string_buffer(512)
    lib().fm_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(rc):
    if rc != FM_OK:
        raise FlowmolError(rc, last_error())


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_params(np_, domain, rcutoff, delta_rneighbr=(0.3, 0.3, 0.3), delta_t=0.005, tplot=100,
                density=None, initialstep=0, simtime=0.0, force_list=FORCE_LIST_HALF, potential_flag=0,
                rebuild_criteria=0, fixed_rebuild=1, sLRC_flag=0, precision=PRECISION_FP64, k_c=30.0,
                R_0=1.5, nlist_capacity=0, threads_per_molecule=0, integration_algorithm=1,
                list_build=0, solvent_flag=0, eps=(1.0, 1.0, 1.0), force_path=0) -> FmParams:
    """`eps` = (eps_pp, eps_ps, eps_ss), the SOLVENT_INFO well depths used with
    solvent_flag 1."""
    p = FmParams()
    p.np = int(np_)
    for k in range(3):
        p.domain[k] = float(domain[k])
        p.delta_rneighbr[k] = float(delta_rneighbr[k])
    p.density = float(density) if density is not None else np_ / float(np.prod(domain))
    p.rcutoff = float(rcutoff)
    p.delta_t = float(delta_t)
    p.tplot = int(tplot)
    p.initialstep = int(initialstep)
    p.simtime = float(simtime)
    p.force_list = int(force_list)
    p.potential_flag = int(potential_flag)
    p.rebuild_criteria = int(rebuild_criteria)
    p.fixed_rebuild = int(fixed_rebuild)
    p.sLRC_flag = int(sLRC_flag)
    p.precision = int(precision)
    p.k_c = float(k_c)
    p.R_0 = float(R_0)
    p.nlist_capacity = int(nlist_capacity)
    p.threads_per_molecule = int(threads_per_molecule)
    p.integration_algorithm = int(integration_algorithm)
    p.list_build = int(list_build)
    p.solvent_flag = int(solvent_flag)
    p.force_path = int(force_path)
    p.eps_pp, p.eps_ps, p.eps_ss = (float(x) for x in eps)
    return p


def derive_geometry(params: FmParams):
    nc = (C.c_int32 * 3)()
    cs = (C.c_double * 3)()
    rn2, rc2, ps = C.c_double(), C.c_double(), C.c_double()
    rc = lib().fm_derive_geometry(C.byref(params), nc, cs, C.byref(rn2), C.byref(rc2), C.byref(ps))
    return rc, dict(ncells=list(nc), cellside=list(cs), rneighbr2=rn2.value, rcutoff2=rc2.value,
                    potshift=ps.value)


def global_domain(nunits, density):
    n = (C.c_int32 * 3)(*[int(x) for x in nunits])
    d = (C.c_double * 3)()
    check(lib().fm_global_domain(n, float(density), d))
    return np.array(list(d))


class MDSystem:
    """One simulation on the current CUDA device (a handle of the C ABI)."""

    def __init__(self, params: FmParams, stream=None):
        self.params = params
        self.n = params.np
        hp = C.c_void_p()
        check(lib().fm_create(C.byref(params), C.byref(hp)))
        self.h = hp
        if stream is not None:
            self.set_stream(stream)

    def close(self):
        if getattr(self, "h", None):
            lib().fm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        ptr = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", 0)
        check(lib().fm_set_stream(self.h, C.c_void_p(ptr)))

    # ---- state ----
    def upload(self, r, v, a=None, glob_no=None):
        r = np.ascontiguousarray(r, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        ap = None
        if a is not None:
            a = np.ascontiguousarray(a, dtype=np.float64)
            ap = _dp(a)
        gp = None
        if glob_no is not None:
            glob_no = np.ascontiguousarray(glob_no, dtype=np.int32)
            gp = glob_no.ctypes.data_as(C.POINTER(C.c_int32))
        check(lib().fm_upload_state(self.h, self.n, _dp(r), _dp(v), ap, gp))

    def upload_monomers(self, chain, subchain, bflag):
        c = np.ascontiguousarray(chain, np.int32); sc = np.ascontiguousarray(subchain, np.int32)
        b = np.ascontiguousarray(bflag, np.int32).reshape(-1, 4)
        P = C.POINTER(C.c_int32)
        check(lib().fm_upload_monomers(self.h, c.ctypes.data_as(P), sc.ctypes.data_as(P), b.ctypes.data_as(P)))

    def set_mie(self, tables, moltype):
        """Mie_potential 1 (fm_set_mie): `tables` maps mass (ntypes) and
        epsilon, lambdar, lambdaa, C, alpha, potshift, k_harmonic, r0
        (ntypes x ntypes, indexed [i-1, j-1]) -- the reference's lookup
        arrays; moltype is 1-based in upload order."""
        nt = len(tables["mass"])
        self._mie_keep = [np.ascontiguousarray(tables["mass"], np.float64)]
        t = FmMieTables()
        t.ntypes = nt
        t.mass = self._mie_keep[0].ctypes.data_as(C.POINTER(C.c_double))
        for k in MIE_TABLE_KEYS:
            a = np.ascontiguousarray(np.asarray(tables[k], np.float64).T).reshape(-1)  # (i,j) at i + nt*j
            self._mie_keep.append(a)
            setattr(t, k, a.ctypes.data_as(C.POINTER(C.c_double)))
        mt = np.ascontiguousarray(moltype, np.int32)
        check(lib().fm_set_mie(self.h, C.byref(t), mt.ctypes.data_as(C.POINTER(C.c_int32))))

    def set_angular(self, k, theta0, funcy):
        """angular_potential 1 (fm_set_angular): k and theta0 as (ntypes,
        ntypes, ntypes) arrays indexed [i-1, j-1, k-1] -- the reference's
        angular_k_lookup and angular_r0_lookup -- and funcy per molecule in
        upload order.  After set_mie(), before setup()."""
        kk = np.ascontiguousarray(np.asarray(k, np.float64).transpose(2, 1, 0)).reshape(-1)  # (i,j,k) at i+nt(j+nt k)
        tt = np.ascontiguousarray(np.asarray(theta0, np.float64).transpose(2, 1, 0)).reshape(-1)
        fy = np.ascontiguousarray(funcy, np.int32)
        self._ang_keep = (kk, tt, fy)
        check(lib().fm_set_angular(self.h, int(np.asarray(k).shape[0]), _dp(kk), _dp(tt),
                                   fy.ctypes.data_as(C.POINTER(C.c_int32))))

    def bonds(self):
        n = C.c_int64()
        check(lib().fm_get_bonds(self.h, None, None, None, 0, C.byref(n)))
        o = np.empty(n.value, np.int32); p = np.empty(n.value, np.int32); c = np.empty(n.value, np.int8)
        P = C.POINTER(C.c_int32)
        check(lib().fm_get_bonds(self.h, o.ctypes.data_as(P), p.ctypes.data_as(P),
                                 c.ctypes.data_as(C.POINTER(C.c_int8)), n.value, C.byref(n)))
        return o, p, c.astype(np.int32)

    def download(self):
        r = np.empty((self.n, 3)); v = np.empty((self.n, 3)); a = np.empty((self.n, 3))
        g = np.empty(self.n, np.int32)
        check(lib().fm_download_state(self.h, _dp(r), _dp(v), _dp(a), g.ctypes.data_as(C.POINTER(C.c_int32))))
        return r, v, a, g

    # ---- reference subroutine mirrors (md.f90) ----
    def setup(self):
        check(lib().fm_setup(self.h))

    def simulation_move_particles_vv(self, pass_num):
        check(lib().fm_move_vv(self.h, int(pass_num)))

    def simulation_move_particles_lfv(self):
        check(lib().fm_move_lfv(self.h))

    def md_advance_lfv(self):
        """One leap-frog iteration, subroutine by subroutine (md.f90:109-139)."""
        self.iter = self.iter + 1
        self.simulation_compute_forces()
        self.simulation_move_particles_lfv()
        self.messenger_updateborders(0)
        if self.simulation_checkrebuild():
            self.linklist_deallocateall()
            self.sendmols()
            self.sort_mols()
            self.assign_to_cell()
            self.messenger_updateborders(1)
            self.assign_to_neighbourlist()

    def messenger_updateborders(self, rebuild):
        check(lib().fm_update_borders(self.h, int(rebuild)))

    def simulation_checkrebuild(self) -> int:
        r = C.c_int32()
        check(lib().fm_check_rebuild(self.h, C.byref(r)))
        return r.value

    def linklist_deallocateall(self):
        check(lib().fm_linklist_deallocateall(self.h))

    def sendmols(self):
        check(lib().fm_sendmols(self.h))

    def set_sort(self, sort_flag, sort_freq=1, sortblocksize=1):
        """SORT_FLAG: 0 off, 1 x-fastest blocks, 2 Hilbert-ordered blocks of
        sortblocksize^3 cells, every sort_freq-th rebuild."""
        check(lib().fm_set_sort(self.h, int(sort_flag), int(sort_freq), int(sortblocksize)))

    def sort_mols(self):
        """Every sort_freq-th call re-numbers the molecules by sort block
        (linklist.f90:2744-2869); downloads report the new order."""
        check(lib().fm_sort_mols(self.h))

    def sort_state(self):
        so = C.c_int64(); sk = C.c_int64(); nr = C.c_int32(); f1 = C.c_double(); f2 = C.c_int32()
        check(lib().fm_get_sort_state(self.h, C.byref(so), C.byref(sk), C.byref(nr), C.byref(f1), C.byref(f2)))
        return dict(sorts=so.value, skipped=sk.value, nrebuilds=nr.value, sf1=f1.value, sf2=f2.value)

    def assign_to_cell(self):
        check(lib().fm_assign_to_cell(self.h))

    def rebuild_lists(self):
        """The whole rebuild branch of md_advance_vv in one call."""
        check(lib().fm_rebuild_lists(self.h))

    def assign_to_neighbourlist(self):
        check(lib().fm_assign_to_neighbourlist(self.h))

    def simulation_compute_forces(self):
        check(lib().fm_compute_forces(self.h))

    def evaluate_macroscopic_properties(self):
        m = FmMacro()
        check(lib().fm_evaluate_macroscopic_properties(self.h, C.byref(m)))
        return m.as_dict()

    @property
    def iter(self):
        i = C.c_int32()
        check(lib().fm_get_iter(self.h, C.byref(i)))
        return i.value

    @iter.setter
    def iter(self, value):
        check(lib().fm_set_iter(self.h, int(value)))

    def md_advance_vv(self):
        """One iteration, subroutine by subroutine (md.f90:143-163)."""
        self.iter = self.iter + 1
        self.simulation_move_particles_vv(1)
        self.messenger_updateborders(0)
        if self.simulation_checkrebuild():
            self.linklist_deallocateall()
            self.sendmols()
            self.sort_mols()
            self.assign_to_cell()
            self.messenger_updateborders(1)
            self.assign_to_neighbourlist()
        self.simulation_compute_forces()
        self.simulation_move_particles_vv(2)

    def simulation_md(self, nsteps, blocking=True):
        """The fused device loop over nsteps iterations."""
        check(lib().fm_step(self.h, int(nsteps), 1 if blocking else 0))

    def sync(self):
        check(lib().fm_sync(self.h))

    # ---- results ----
    def records(self, cap=100000):
        arr = (FmMacro * cap)()
        n = C.c_int32()
        check(lib().fm_get_records(self.h, arr, cap, C.byref(n)))
        return [arr[k].as_dict() for k in range(n.value)]

    def per_molecule(self):
        pe = np.empty(self.n); vir = np.empty(self.n)
        check(lib().fm_get_per_molecule(self.h, _dp(pe), _dp(vir)))
        return pe, vir

    def pair_list(self):
        n = C.c_int64()
        check(lib().fm_get_pair_list(self.h, None, None, None, 0, C.byref(n)))
        o = np.empty(n.value, np.int32); p = np.empty(n.value, np.int32); c = np.empty(n.value, np.int8)
        check(lib().fm_get_pair_list(self.h, o.ctypes.data_as(C.POINTER(C.c_int32)),
                                     p.ctypes.data_as(C.POINTER(C.c_int32)),
                                     c.ctypes.data_as(C.POINTER(C.c_int8)), n.value, C.byref(n)))
        return o, p, c.astype(np.int32)

    def pair_digest(self):
        d = C.c_uint64(); n = C.c_int64()
        check(lib().fm_pair_digest(self.h, C.byref(d), C.byref(n)))
        return d.value, n.value

    def force_kernel_timing(self, enable=True):
        check(lib().fm_force_kernel_timing(self.h, 1 if enable else 0))

    def force_kernel_time(self):
        ms = C.c_double(); n = C.c_int64()
        check(lib().fm_get_force_kernel_time(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def launch_count(self):
        n = C.c_int64()
        check(lib().fm_get_launch_count(self.h, C.byref(n)))
        return n.value

    @property
    def threads_per_molecule(self):
        t = C.c_int32()
        check(lib().fm_get_threads_per_molecule(self.h, C.byref(t)))
        return t.value

    def force_path(self):
        """(FORCE_PATH_GATHER or FORCE_PATH_TILES, staged capacity per block)."""
        p = C.c_int32(); cap = C.c_int32()
        check(lib().fm_get_force_path(self.h, C.byref(p), C.byref(cap)))
        return p.value, cap.value

    def counters(self):
        rb = C.c_int64(); cap = C.c_int32(); mx = C.c_int32()
        check(lib().fm_get_counters(self.h, C.byref(rb), C.byref(cap), C.byref(mx)))
        return dict(rebuilds=rb.value, nlist_capacity=cap.value, max_neighbours=mx.value)

    def set_pressure_outflag(self, flag=1):
        check(lib().fm_set_pressure_outflag(self.h, int(flag)))

    def pressure_tensor(self, reset=False):
        """(3x3 mean virial pressure tensor over the record steps sampled, samples)."""
        out = (C.c_double * 9)()
        n = C.c_int32()
        check(lib().fm_get_pressure_tensor(self.h, out, C.byref(n), int(bool(reset))))
        return np.array(list(out)).reshape(3, 3), n.value


def make_job(np_, domain, rcutoff, nsteps, delta_rneighbr=(0.3, 0.3, 0.3), tplot=100, density=None,
             initialstep=0, integration_algorithm=1, ensemble=0, force_list=FORCE_LIST_HALF, pressure_outflag=0,
             nthermo=0, thermostat_temperature=(1.0, 1.0), teth=(0.0, 0.0, 0.0), rebuild_criteria=0,
             fixed_rebuild=1, nlist_capacity=0) -> FmJob:
    j = FmJob()
    j.np = int(np_)
    j.tplot = int(tplot)
    for k in range(3):
        j.domain[k] = float(domain[k])
        j.delta_rneighbr[k] = float(delta_rneighbr[k])
    j.density = float(density) if density is not None else np_ / float(np.prod(domain))
    j.rcutoff = float(rcutoff)
    j.nsteps = int(nsteps)
    j.initialstep = int(initialstep)
    j.integration_algorithm = int(integration_algorithm)
    j.ensemble = int(ensemble)
    j.force_list = int(force_list)
    j.pressure_outflag = int(pressure_outflag)
    j.nthermo = int(nthermo)
    j.thermostat_temperature[0] = float(thermostat_temperature[0])
    j.thermostat_temperature[1] = float(thermostat_temperature[1])
    j.teth_k2, j.teth_k4, j.teth_k6 = (float(x) for x in teth)
    j.rebuild_criteria = int(rebuild_criteria)
    j.fixed_rebuild = int(fixed_rebuild)
    j.nlist_capacity = int(nlist_capacity)
    return j


class Engine:
    """Multi-job slot engine (batched replicas, served jobs)."""

    def __init__(self, max_molecules, max_cells, max_list_entries, max_slots, delta_t=0.005, precision=0,
                 threads_per_molecule=0, ticks_per_chunk=20, keep_states=True, list_build=0):
        p = FmEngineParams()
        p.max_molecules = int(max_molecules)
        p.max_cells = int(max_cells)
        p.max_list_entries = int(max_list_entries)
        p.max_slots = int(max_slots)
        p.precision = int(precision)
        p.threads_per_molecule = int(threads_per_molecule)
        p.ticks_per_chunk = int(ticks_per_chunk)
        p.keep_states = 1 if keep_states else 0
        p.list_build = int(list_build)
        p.delta_t = float(delta_t)
        hp = C.c_void_p()
        check(lib().fm_engine_create(C.byref(p), C.byref(hp)))
        self.h = hp

    def close(self):
        if getattr(self, "h", None):
            lib().fm_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, job: FmJob, r, v, tag=None, rtether=None, slidev=None) -> int:
        r = np.ascontiguousarray(r, np.float64); v = np.ascontiguousarray(v, np.float64)
        args = []
        for x, t in ((tag, np.int32), (rtether, np.float64), (slidev, np.float64)):
            if x is None:
                args.append(None)
            else:
                x = np.ascontiguousarray(x, t)
                args.append(x)
        jid = C.c_int64()
        check(lib().fm_engine_submit(self.h, C.byref(job), _dp(r), _dp(v),
                                     None if args[0] is None else args[0].ctypes.data_as(C.POINTER(C.c_int32)),
                                     None if args[1] is None else _dp(args[1]),
                                     None if args[2] is None else _dp(args[2]), C.byref(jid)))
        return jid.value

    def step_chunk(self):
        res = C.c_int32(); q = C.c_int32()
        check(lib().fm_engine_step_chunk(self.h, C.byref(res), C.byref(q)))
        return res.value, q.value

    def run(self, max_chunks=0):
        check(lib().fm_engine_run(self.h, int(max_chunks)))

    def results(self, cap=100000):
        arr = (FmJobResult * cap)()
        n = C.c_int32()
        check(lib().fm_engine_take_results(self.h, arr, cap, C.byref(n)))
        return [arr[k].as_dict() for k in range(n.value)]

    def job_state(self, job_id, n):
        r = np.empty((n, 3)); v = np.empty((n, 3))
        check(lib().fm_engine_job_state(self.h, int(job_id), _dp(r), _dp(v)))
        return r, v

    def counters(self):
        t = C.c_int64(); m = C.c_int64(); tp = C.c_int32(); la = C.c_int64()
        check(lib().fm_engine_counters(self.h, C.byref(t), C.byref(m), C.byref(tp), C.byref(la)))
        return dict(ticks=t.value, molecule_steps=m.value, threads_per_molecule=tp.value, launches=la.value)

    def tuning(self):
        """(threads per molecule, blocks_below): the autotuner's choices."""
        tp = C.c_int32(); bb = C.c_double()
        check(lib().fm_engine_tuning(self.h, C.byref(tp), C.byref(bb)))
        return tp.value, bb.value


def _ip32(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int32))


def _dpn(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def read_final_state(path):
    """(header, dict of arrays) of a final_state restart file; arrays are
    (n, 3) for r, v, rtether, rtrue and (n, 8) for monomer."""
    h = FmRestartHeader()
    check(lib().fm_read_final_state(os.fsencode(path), C.byref(h), 0, None, None, None, None, None, None, None,
                                    None))
    n = h.globalnp
    r = np.empty((n, 3)); v = np.empty((n, 3)); rt = np.empty((n, 3)); rtrue = np.empty((n, 3))
    tag = np.empty(n, np.int32); glob = np.empty(n, np.int32); mt = np.empty(n, np.int32)
    mono = np.empty((n, 8))
    check(lib().fm_read_final_state(os.fsencode(path), C.byref(h), n, _dpn(r), _dpn(v), _ip32(tag), _dpn(rt),
                                    _ip32(glob), _dpn(rtrue), _ip32(mt), _dpn(mono)))
    return h, dict(r=r, v=v, tag=tag, rtether=rt, glob_no=glob, rtrue=rtrue, moltype=mt, monomer=mono)


def write_final_state(path, h, r, v, tag=None, rtether=None, glob_no=None, rtrue=None, moltype=None, monomer=None):
    arr = lambda x, t: None if x is None else np.ascontiguousarray(x, t)  # noqa: E731
    r = arr(r, np.float64); v = arr(v, np.float64); tag = arr(tag, np.int32); rtether = arr(rtether, np.float64)
    glob_no = arr(glob_no, np.int32); rtrue = arr(rtrue, np.float64); moltype = arr(moltype, np.int32)
    monomer = arr(monomer, np.float64)
    check(lib().fm_write_final_state(os.fsencode(path), C.byref(h), _dpn(r), _dpn(v), _ip32(tag), _dpn(rtether),
                                     _ip32(glob_no), _dpn(rtrue), _ip32(moltype), _dpn(monomer)))


def sort_table(sort_flag, nblocks):
    """Hcurve over nblocks sort blocks per axis, flat and x fastest."""
    nb = (C.c_int32 * 3)(*[int(x) for x in nblocks])
    out = np.zeros(int(np.prod(nblocks)), np.int32)
    check(lib().fm_sort_table(int(sort_flag), nb, out.ctypes.data_as(C.POINTER(C.c_int32)), out.size))
    return out


def read_input(path) -> FmInput:
    x = FmInput()
    check(lib().fm_read_input(os.fsencode(path), C.byref(x)))
    return x


def params_from_input(inp: FmInput, np_, domain, precision=PRECISION_FP64, **overrides) -> FmParams:
    """fm_params for the run an MD.in deck describes (read_input), given the
    molecule count and box -- from a restart header, or global_domain of the
    deck's INITIALNUNITS and DENSITY for a lattice start.  Keyword arguments
    override single fields (e.g. tplot, nlist_capacity)."""
    kw = dict(delta_rneighbr=tuple(inp.delta_rneighbr), delta_t=inp.delta_t, tplot=inp.tplot,
              density=inp.density, force_list=inp.force_list, potential_flag=inp.potential_flag,
              rebuild_criteria=inp.rebuild_criteria, fixed_rebuild=max(1, inp.fixed_rebuild),
              sLRC_flag=inp.sLRC_flag, precision=precision, k_c=inp.k_c, R_0=inp.R_0,
              integration_algorithm=inp.integration_algorithm, solvent_flag=inp.solvent_flag,
              eps=(inp.eps_pp, inp.eps_ps, inp.eps_ss))
    kw.update(overrides)
    return make_params(np_, domain, inp.rcutoff, **kw)
