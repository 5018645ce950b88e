"""fm_compute_forces_noalloc: forces for callers that cannot allocate.

Some callers of this library cannot call cudaMalloc -- a host code whose
device memory is all handed out by its own pool, or a loop that must not take
the synchronisation an allocation can imply.  The no-allocation entry point
keeps its scratch in a fixed __device__ array instead.  This file checks,
through the C ABI, that it returns the same forces, per-molecule PE and
virial as the existing entry point (fm_setup on a handle) within the FP64
tolerance of the parity tests, on two calls in a row with different inputs
(the second call must not see the first call's leftovers), and that inputs
above its fixed limit are refused.  It is collected last so that a failure
here never hides another test's result.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _bind():
    from flowmol_b200 import api, build
    build.build()
    L = api.lib()
    L.fm_compute_forces_noalloc.argtypes = [C.POINTER(api.FmParams), C.c_int32, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p]
    L.fm_compute_forces_noalloc.restype = C.c_int
    L.fm_noalloc_last_error.argtypes = [C.c_char_p, C.c_int32]
    L.fm_noalloc_last_error.restype = C.c_int
    return api, L


def _existing(api, p, r, v):
    s = api.MDSystem(p)
    s.upload(r, v)
    s.setup()
    _, _, a, _ = s.download()
    pe, vir = s.per_molecule()
    s.close()
    return a, pe, vir


def test_noalloc_matches_existing_entry_point_on_two_calls():
    import torch
    api, L = _bind()
    from flowmol_b200 import lattice
    states = []
    for k in range(2):
        r, v, dom = lattice.lj_fluid([8, 8, 8], 0.8442, 0.722, lattice.SEED_BASE + 20 + k)
        r = lattice.jitter(r, 0.04 + 0.02 * k, 40 + k, dom)
        states.append((r, v, dom))
    n = len(states[0][0])
    p = api.make_params(n, states[0][2], 2.5, tplot=1, density=0.8442)
    dr = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    da = torch.empty_like(dr)
    dpe = torch.empty(n, dtype=torch.float64, device="cuda")
    dvir = torch.empty_like(dpe)
    for r, v, dom in states:
        a_ref, pe_ref, vir_ref = _existing(api, p, r, v)
        dr.copy_(torch.from_numpy(np.ascontiguousarray(r)))
        da.fill_(float("nan")); dpe.fill_(float("nan")); dvir.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = L.fm_compute_forces_noalloc(C.byref(p), n, dr.data_ptr(), da.data_ptr(), dpe.data_ptr(),
                                         dvir.data_ptr(), None)
        assert rc == 0, rc
        a = da.cpu().numpy()
        assert rel_err(a, a_ref, 1.0).max() <= TOL64
        np.testing.assert_allclose(dpe.cpu().numpy(), pe_ref, rtol=TOL64, atol=TOL64)
        np.testing.assert_allclose(dvir.cpu().numpy(), vir_ref, rtol=TOL64, atol=TOL64)


def test_noalloc_refuses_inputs_above_its_limit():
    import torch
    api, L = _bind()
    n = 65536 + 1
    p = api.make_params(n, [60.0, 60.0, 60.0], 2.5)
    dr = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    da = torch.empty_like(dr)
    rc = L.fm_compute_forces_noalloc(C.byref(p), n, dr.data_ptr(), da.data_ptr(), None, None, None)
    assert rc == 1  # FM_ERR_ARG
    buf = C.create_string_buffer(256)
    L.fm_noalloc_last_error(buf, 256)
    assert b"65536" in buf.value
