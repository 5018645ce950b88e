"""The oracle's geometry rules and the library's host-side geometry, pinned
bit for bit against values the reference printed into
runs/Intrinsic_Interface/results/simulation_header (fixture made by
tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def geom():
    return json.load(open(os.path.join(GOLD, "intrinsic_interface_geometry.json")))


def test_global_domain_bitexact(geom):
    dom, unit, vol = O.global_domain(geom["nunits"], geom["density"])
    assert dom.tolist() == geom["globaldomain"]
    assert unit.tolist() == geom["initialunitsize"]
    assert vol == geom["volume"]


def test_cells_bitexact(geom):
    rc, nc, cs, rn2 = O.cells(geom["globaldomain"], geom["rcutoff"], geom["delta_rneighbr"])
    assert rc == 0
    assert nc.tolist() == geom["ncells"]
    assert cs.tolist() == geom["cellsidelength"]
    assert rn2 == (geom["rcutoff"] + sum(geom["delta_rneighbr"]) / 3.0) ** 2


def test_library_geometry_matches_golden(geom):
    """fm_derive_geometry / fm_global_domain run on the host: no GPU needed."""
    from flowmol_b200 import api
    d = api.global_domain(geom["nunits"], geom["density"])
    assert d.tolist() == geom["globaldomain"]
    p = api.make_params(geom["globalnp"], geom["globaldomain"], geom["rcutoff"], geom["delta_rneighbr"])
    rc, g = api.derive_geometry(p)
    assert rc == 0
    assert g["ncells"] == geom["ncells"]
    assert g["cellside"] == geom["cellsidelength"]
    rc_o, nc_o, cs_o, rn2_o = O.cells(geom["globaldomain"], geom["rcutoff"], geom["delta_rneighbr"])
    assert g["rneighbr2"] == rn2_o


def test_fewcells_refused_like_reference():
    """setup_set_parameters.f90:1891-1896 aborts below 3 cells per axis."""
    rc, nc, cs, rn2 = O.cells([8.0, 8.0, 8.0], 2.5, [0.3, 0.3, 0.3])
    assert rc == O.lib().orc_set_parameters_cells.restype(3).value or rc == 3
    from flowmol_b200 import api
    p = api.make_params(100, [8.0, 8.0, 8.0], 2.5)
    assert api.derive_geometry(p)[0] == 3


def test_fene_rneighbr_override():
    """rneighbr < R_0 is raised to R_0 for polymers (setup_set_parameters.f90:1865-1869)."""
    rc, nc, cs, rn2 = O.cells([20.0, 20.0, 20.0], 2 ** (1 / 6), [0.3, 0.3, 0.3], potential_flag=1, R_0=1.5)
    assert rn2 == 1.5 * 1.5
