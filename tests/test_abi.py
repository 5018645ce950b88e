"""The C-ABI library loads and exports every entry point declared in
include/flowmol_b200.h; host-only calls work without a GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

from flowmol_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_header_symbols():
    build.build()
    hdr = open(os.path.join(ROOT, "include", "flowmol_b200.h")).read()
    declared = set(re.findall(r"FM_API int (fm_\w+)\(", hdr))
    assert len(declared) >= 25
    exported = set(api.exported_symbols())
    assert declared == exported


ABI_STRUCTS = {
    "fm_params": api.FmParams, "fm_macro": api.FmMacro, "fm_engine_params": api.FmEngineParams,
    "fm_mie_tables": api.FmMieTables, "fm_job": api.FmJob, "fm_job_result": api.FmJobResult,
    "fm_restart_header": api.FmRestartHeader, "fm_input": api.FmInput,
}


def test_struct_layouts_match_header(tmp_path):
    """Every ctypes mirror has the C struct's size and, field by field, the
    offsets and sizes gcc gives the header's declarations."""
    p = api.make_params(10, [10.0, 10.0, 10.0], 2.5)
    assert p.np == 10 and p.tplot == 100
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "flowmol_b200.h"', "int main(void) {"]
    for cname, ct in ABI_STRUCTS.items():
        lines.append(f'printf("{cname} . %zu 0\\n", sizeof({cname}));')
        for fname, _ in ct._fields_:
            lines.append(f'printf("{cname} {fname} %zu %zu\\n", sizeof((({cname} *)0)->{fname}), '
                         f"offsetof({cname}, {fname}));")
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln.strip():
            cname, fname, size, off = ln.split()
            got[(cname, fname)] = (int(size), int(off))
    for cname, ct in ABI_STRUCTS.items():
        assert got[(cname, ".")][0] == C.sizeof(ct), cname
        for fname, _ in ct._fields_:
            f = getattr(ct, fname)
            assert got[(cname, fname)] == (f.size, f.offset), (cname, fname)


def test_errors_are_codes_not_aborts():
    L = api.lib()
    # null params -> FM_ERR_ARG, message available
    assert L.fm_create(None, None) == 1
    assert "null" in api.last_error()


def test_create_without_device_is_an_error_code():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    p = api.make_params(100, [20.0, 20.0, 20.0], 2.5)
    h = C.c_void_p()
    assert api.lib().fm_create(C.byref(p), C.byref(h)) == 9  # FM_ERR_NODEVICE


def test_combinations_the_reference_refuses_are_argument_errors():
    """Parameter sets the reference stops on with error_abort come back as
    FM_ERR_ARG from fm_create, before any device is touched: polymers with
    all pairs or the full list (simulation_compute_forces.f90:206, 242-246),
    the Soddemann solvent outside the half list, unknown flags."""
    import ctypes as C
    L = api.lib()
    h = C.c_void_p()
    cases = [
        (dict(potential_flag=1, force_list=0), "all pairs"),
        (dict(potential_flag=1, force_list=2), "full interaction"),
        (dict(potential_flag=1, force_list=2, solvent_flag=1), "full interaction"),
        (dict(potential_flag=0, solvent_flag=1), "solvent"),
        (dict(rebuild_criteria=3), "rebuild_criteria"),
        (dict(solvent_flag=2, potential_flag=1), "solvent_flag"),
    ]
    for kw, word in cases:
        p = api.make_params(100, [10.0, 10.0, 10.0], 2.5, **kw)
        assert L.fm_create(C.byref(p), C.byref(h)) == 1, kw
        assert word in api.last_error(), (kw, api.last_error())


def test_plain_c_program_compiles_links_and_gets_codes(tmp_path):
    """A C (not C++) caller: the header compiles under gcc -std=c99, the
    library links, host-only calls answer, and fm_create reports a missing
    device or succeeds -- never aborts."""
    src = tmp_path / "caller.c"
    src.write_text(r"""
#include <stdio.h>
#include "flowmol_b200.h"
int main(void) {
    fm_params p = {0};
    p.np = 2048; p.domain[0] = p.domain[1] = p.domain[2] = 13.68; p.density = 0.8;
    p.rcutoff = 1.12246204830937; p.delta_rneighbr[0] = p.delta_rneighbr[1] = p.delta_rneighbr[2] = 0.3;
    p.delta_t = 0.005; p.tplot = 100; p.force_list = FM_FORCE_LIST_HALF;
    int32_t nc[3]; double cs[3], rn2, rc2, ps;
    int rc = fm_derive_geometry(&p, nc, cs, &rn2, &rc2, &ps);
    fm_handle *h = NULL;
    int rc2_ = fm_create(&p, &h);
    char msg[256]; fm_last_error(msg, sizeof msg);
    printf("%d %d %d %d %.17g %d\n", rc, nc[0], nc[1], nc[2], ps, rc2_);
    if (h) fm_destroy(h);
    return 0;
}
""")
    exe = tmp_path / "caller"
    libdir = os.path.join(ROOT, "flowmol_b200")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                    "-L", libdir, "-lflowmol_b200", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert out[:4] == ["0", "9", "9", "9"]
    assert float(out[4]) == pytest.approx(-1.0, abs=1e-12)  # WCA potshift
    assert out[5] in ("0", "9")  # FM_OK with a GPU, FM_ERR_NODEVICE without
