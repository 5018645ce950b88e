"""final_state reader/writer and keyword-input reader (host only, no GPU).

Pinned against the reference: the header and molecule arrays must equal what
the reference's own reader (src/reorder_restart/read_final_state.py) decoded
from runs/Intrinsic_Interface/initial_state (fixtures in tests/golden, made by
tests/golden/make_golden.py), and writing what was read must reproduce the
file byte for byte."""
import json
import os

import numpy as np
import pytest

from flowmol_b200 import api

GOLD = os.path.join(os.path.dirname(__file__), "golden")
FIXTURE = os.path.join(GOLD, "intrinsic_interface_initial_state.bin")


def test_reader_matches_reference_reader():
    h, a = api.read_final_state(FIXTURE)
    ref = json.load(open(os.path.join(GOLD, "intrinsic_interface_restart.json")))
    st = np.load(os.path.join(GOLD, "intrinsic_interface_state.npz"))
    assert h.globalnp == ref["globalnp"] == 2635
    assert list(h.initialnunits) == [ref["initialunits1"], ref["initialunits2"], ref["initialunits3"]]
    assert h.nsteps == ref["Nsteps"] and h.tplot == ref["tplot"]
    assert list(h.seed) == [ref["seed1"], ref["seed2"]]
    assert list(h.periodic) == [ref["periodic1"], ref["periodic2"], ref["periodic3"]]
    assert (h.npx, h.npy, h.npz) == (ref["npx"], ref["npy"], ref["npz"])
    assert [h.procnp[p] for p in range(h.nproc)] == [ref["procnp0"], ref["procnp1"]]
    assert list(h.globaldomain) == [ref["globaldomain1"], ref["globaldomain2"], ref["globaldomain3"]]
    for k in ("density", "rcutoff", "delta_t", "elapsedtime", "simtime", "k_c", "R_0", "delta_rneighbr"):
        assert getattr(h, k) == ref[k], k
    assert h.header_pos == ref["headerstart"]
    assert np.array_equal(a["r"], st["r"]) and np.array_equal(a["v"], st["v"])
    assert np.array_equal(a["tag"], st["tag"].astype(np.int32))


def test_round_trip_is_byte_identical(tmp_path):
    h, a = api.read_final_state(FIXTURE)
    out = tmp_path / "final_state"
    api.write_final_state(str(out), h, a["r"], a["v"], a["tag"], a["rtether"], a["glob_no"])
    assert out.read_bytes() == open(FIXTURE, "rb").read()


def test_optional_blocks_round_trip(tmp_path):
    """rtrue, tethers, Mie types, global numbering and monomer records."""
    rng = np.random.default_rng(3)
    n = 50
    h = api.FmRestartHeader()
    h.globalnp = n; h.npx = h.npy = h.npz = 1; h.nproc = 1; h.procnp[0] = n
    h.rtrue_flag = 1; h.mie_potential = 1; h.global_numbering = 1; h.potential_flag = 1; h.nmonomers = 8
    h.globaldomain[0] = h.globaldomain[1] = h.globaldomain[2] = 10.0
    tag = rng.integers(0, 8, n).astype(np.int32)
    a = dict(r=rng.normal(size=(n, 3)), v=rng.normal(size=(n, 3)), tag=tag,
             rtether=np.where(np.isin(tag, [3, 5, 6, 7])[:, None], rng.normal(size=(n, 3)), 0.0),
             glob_no=rng.permutation(n).astype(np.int32) + 1, rtrue=rng.normal(size=(n, 3)),
             moltype=rng.integers(1, 3, n).astype(np.int32), monomer=rng.integers(0, 100, (n, 8)).astype(float))
    p = tmp_path / "s"
    api.write_final_state(str(p), h, **a)
    h2, b = api.read_final_state(str(p))
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert h2.nmonomers == 8 and h2.rtrue_flag == 1


def test_truncated_file_is_an_error(tmp_path):
    data = open(FIXTURE, "rb").read()
    p = tmp_path / "bad"
    p.write_bytes(data[:-100])
    with pytest.raises(api.FlowmolError) as e:
        api.read_final_state(str(p))
    assert e.value.code == 10  # FM_ERR_IO


def test_input_reader_default_in():
    x = api.read_input(os.path.join(GOLD, "default.in"))
    assert x.ensemble == 0 and x.density == 0.8 and x.rcutoff == 1.12246204830937
    assert list(x.initialnunits) == [8, 8, 8]
    assert x.nsteps == 1000 and x.tplot == 100 and x.delta_t == 0.005
    assert list(x.delta_rneighbr) == [0.3, 0.3, 0.3]
    assert x.force_list == 3 and x.integration_algorithm == 0


def test_input_reader_two_phase_run():
    x = api.read_input(os.path.join(GOLD, "MD_2_phase.in"))
    assert x.rcutoff == 2.5 and x.delta_t == 0.005 and x.force_list == 1
    assert list(x.initialnunits) == [76, 8, 8]
    assert x.inputtemperature == 0.6057
    assert x.integration_algorithm == 0


def test_input_reader_reports_missing_keywords(tmp_path):
    p = tmp_path / "MD.in"
    p.write_text("DENSITY\n0.8\n")
    with pytest.raises(api.FlowmolError) as e:
        api.read_input(str(p))
    assert "RCUTOFF" in str(e.value)


def test_input_reader_fene_solution_with_soddemann_solvent(tmp_path):
    """INITIAL_CONFIG_FLAG 1 fene_solution: the FENE_SOLUTION block sets
    potential_flag 1, the WCA cutoff and targetconc, and SOLVENT_INFO 1 its
    three well depths (setup_read_input.f90:188-199, 253-296).  With flag 0
    the same blocks are present in default.in but not read."""
    base = open(os.path.join(GOLD, "default.in")).read()
    x0 = api.read_input(os.path.join(GOLD, "default.in"))
    assert x0.potential_flag == 0 and x0.solvent_flag == 0 and x0.targetconc == 0.0
    assert "INITIAL_CONFIG_FLAG\n0\nspecial_case_name" in base and "SOLVENT_INFO\n0\n0.0\n0.0\n0.0" in base
    deck = base.replace("INITIAL_CONFIG_FLAG\n0\nspecial_case_name", "INITIAL_CONFIG_FLAG\n1\nfene_solution")
    deck = deck.replace("SOLVENT_INFO\n0\n0.0\n0.0\n0.0", "SOLVENT_INFO\n1\n1.5\n1.0d0\n0.5")
    p = tmp_path / "MD.in"
    p.write_text(deck)
    x = api.read_input(str(p))
    assert x.potential_flag == 1 and x.rcutoff == 2.0 ** (1.0 / 6.0)
    assert x.nmonomers == 8 and x.k_c == 30.0 and x.R_0 == 1.5 and x.density == 0.5 and x.targetconc == 0.2
    assert x.solvent_flag == 1 and (x.eps_pp, x.eps_ps, x.eps_ss) == (1.5, 1.0, 0.5)
    p.write_text(deck.replace("SOLVENT_INFO\n1\n1.5", "SOLVENT_INFO\n3\n1.5"))
    with pytest.raises(api.FlowmolError) as e:
        api.read_input(str(p))
    assert "solvent flag" in str(e.value)


def test_input_reader_dense_fene_special_case(tmp_path):
    """INITIAL_CONFIG_FLAG 1 dense_fene reads the DENSE_FENE block (nmonomers,
    k_c, r_0, density, initialnunits) and sets potential_flag 1 with the WCA
    cutoff (setup_read_input.f90:229-254); a missing block is an error, not a
    silent LJ run."""
    base = open(os.path.join(GOLD, "default.in")).read()
    deck = base.replace("INITIAL_CONFIG_FLAG\n0\nspecial_case_name", "INITIAL_CONFIG_FLAG\n1\ndense_fene")
    p = tmp_path / "MD.in"
    p.write_text(deck)
    with pytest.raises(api.FlowmolError) as e:
        api.read_input(str(p))
    assert "DENSE_FENE" in str(e.value)
    p.write_text(deck + "\nDENSE_FENE\n8\n30.0\n1.5\n0.85\n16\n16\n16\n")
    x = api.read_input(str(p))
    assert x.potential_flag == 1 and x.nmonomers == 8 and x.k_c == 30.0 and x.R_0 == 1.5
    assert x.density == 0.85 and list(x.initialnunits) == [16, 16, 16] and x.rcutoff == 2.0 ** (1.0 / 6.0)
    assert x.solvent_flag == 0


def test_params_from_input_deck_give_the_reference_geometry():
    """fm_params built from default.in (8x8x8 FCC units at rho 0.8, WCA,
    skin 0.3) give the oracle's cells, rneighbr2 and potshift."""
    import oracle as O
    x = api.read_input(os.path.join(GOLD, "default.in"))
    dom = api.global_domain(list(x.initialnunits), x.density)
    n = 4 * int(np.prod(list(x.initialnunits)))
    p = api.params_from_input(x, n, dom)
    assert p.np == n and p.tplot == x.tplot and p.delta_t == x.delta_t
    rc, g = api.derive_geometry(p)
    assert rc == 0
    rco, nc, cs, rn2 = O.cells(dom, x.rcutoff, list(x.delta_rneighbr))
    assert rco == 0 and g["ncells"] == list(nc) and g["cellside"] == list(cs) and g["rneighbr2"] == rn2
    assert g["potshift"] == O.lib().orc_potshift(x.rcutoff)
