"""fm_compute_forces_noalloc: forces for callers that cannot allocate.

Some callers of this library cannot call cudaMalloc -- a host code whose
device memory is all handed out by its own pool, or a loop that must not take
the synchronisation an allocation can imply.  The no-allocation entry point
keeps its scratch in a fixed __device__ array instead.  This file checks,
through the C ABI:

  * FP64 and FP32 forces, per-molecule PE and virial against the FP64 oracle
    directly, with the parity tolerances of the main force kernel (FP64 1e-12
    relative, floor 1; FP32 1e-5 relative to max(|F|, 10), PE floor 1, virial
    floor 100), on an input with two molecules just outside the box: the
    entry point wraps them by one period on a private copy, so the oracle is
    given the same wrap done on the host;
  * the same results as the existing entry point (fm_setup on a handle) on
    two calls in a row with different inputs (the second call must not see
    the first call's leftovers);
  * refusal of inputs above either fixed limit (molecules, extended cells).

It is collected last so that a failure here never hides another test's
result.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from helpers import rel_err

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5
F_FLOOR32 = 10.0
W_FLOOR32 = 100.0


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


def _state(k):
    from flowmol_b200 import lattice
    r, v, dom = lattice.lj_fluid([8, 8, 8], 0.8442, 0.722, lattice.SEED_BASE + 20 + k)
    return lattice.jitter(r, 0.04 + 0.02 * k, 40 + k, dom), v, dom


def _call(L, p, r):
    import torch
    n = len(r)
    dr = torch.from_numpy(np.ascontiguousarray(r)).cuda()
    da = torch.full_like(dr, float("nan"))
    dpe = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    dvir = torch.full_like(dpe, float("nan"))
    torch.cuda.synchronize()
    rc = L.fm_compute_forces_noalloc(C.byref(p), n, dr.data_ptr(), da.data_ptr(), dpe.data_ptr(),
                                     dvir.data_ptr(), None)
    assert rc == 0, rc
    out = da.cpu().numpy(), dpe.cpu().numpy(), dvir.cpu().numpy()
    assert np.array_equal(dr.cpu().numpy(), r), "the caller's positions must not be written"
    return out


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_noalloc_matches_oracle_with_molecules_outside_the_box(precision):
    api, L = _bind()
    r, v, dom = _state(0)
    hd = 0.5 * dom
    r_in = r.copy()
    lo = int(np.argmin(r[:, 0]))  # nearest the -x face: x + L lies just past +L/2
    hi = int(np.argmax(r[:, 1]))  # nearest the +y face: y - L lies just below -L/2
    assert lo != hi
    r_in[lo, 0] = r[lo, 0] + dom[0]
    r_in[hi, 1] = r[hi, 1] - dom[1]
    assert r_in[lo, 0] >= hd[0] and r_in[hi, 1] < -hd[1]
    # the same one-period wrap on the host (IEEE double, one rounding per op)
    r_w = np.where(r_in >= hd, r_in - dom, r_in)
    r_w = np.where(r_w < -hd, r_w + dom, r_w)
    n = len(r)
    p = api.make_params(n, dom, 2.5, tplot=1, density=0.8442, precision=precision)
    a, pe, vir = _call(L, p, r_in)
    o = O.Oracle(r_w, v, dom, 2.5, tplot=1, density=0.8442)
    o.setup()
    if precision == 0:
        assert rel_err(a, o.a, 1.0).max() <= TOL64
        np.testing.assert_allclose(pe, o.potenergymol, rtol=TOL64, atol=TOL64)
        np.testing.assert_allclose(vir, o.virialmol, rtol=TOL64, atol=TOL64)
    else:
        assert rel_err(a, o.a, F_FLOOR32).max() <= TOL32
        assert (np.abs(pe - o.potenergymol) / np.maximum(np.abs(o.potenergymol), 1.0)).max() <= TOL32
        assert (np.abs(vir - o.virialmol) / np.maximum(np.abs(o.virialmol), W_FLOOR32)).max() <= TOL32
    # the two moved molecules really interact across the faces
    assert np.linalg.norm(o.a[lo]) > 0.0 and np.linalg.norm(o.a[hi]) > 0.0


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_noalloc_matches_existing_entry_point_on_two_calls(precision):
    api, L = _bind()
    states = [_state(k) for k in range(2)]
    n = len(states[0][0])
    p = api.make_params(n, states[0][2], 2.5, tplot=1, density=0.8442, precision=precision)
    tol = TOL64 if precision == 0 else TOL32
    for r, v, dom in states:
        a_ref, pe_ref, vir_ref = _existing(api, p, r, v)
        a, pe, vir = _call(L, p, r)
        # both paths give the oracle's forces within the form's tolerance; the
        # FP64 forms agree to rounding of the summation order
        assert rel_err(a, a_ref, 1.0 if precision == 0 else F_FLOOR32).max() <= tol
        np.testing.assert_allclose(pe, pe_ref, rtol=tol, atol=tol)
        np.testing.assert_allclose(vir, vir_ref, rtol=tol, atol=tol * (1.0 if precision == 0 else W_FLOOR32))


def test_noalloc_refuses_inputs_above_its_limits():
    import torch
    api, L = _bind()
    buf = C.create_string_buffer(256)
    # too many molecules
    n = 65536 + 1
    p = api.make_params(n, [60.0, 60.0, 60.0], 2.5)
    dr = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    da = torch.empty_like(dr)
    rc = L.fm_compute_forces_noalloc(C.byref(p), n, dr.data_ptr(), da.data_ptr(), None, None, None)
    assert rc == 1  # FM_ERR_ARG
    L.fm_noalloc_last_error(buf, 256)
    assert b"65536" in buf.value
    # few molecules but too many cells: 32 interior cells per axis -> 34^3 > 32768
    n = 1000
    p = api.make_params(n, [32 * 2.8, 32 * 2.8, 32 * 2.8], 2.5)
    dr = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    da = torch.empty_like(dr)
    rc = L.fm_compute_forces_noalloc(C.byref(p), n, dr.data_ptr(), da.data_ptr(), None, None, None)
    assert rc == 1
    L.fm_noalloc_last_error(buf, 256)
    assert b"32768" in buf.value
