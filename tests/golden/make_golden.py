"""Generates the golden fixtures in this folder from the reference checkout.

Run with the root of a reference checkout as the first argument (or in the
REFERENCE_ROOT environment variable).  It reads, never writes, the reference:
  * runs/Intrinsic_Interface/results/simulation_header -- values the
    reference printed for its domain/cell geometry
    (setup_initial_record.f90:700-930);
  * runs/Intrinsic_Interface/initial_state decoded with the reference's own
    reader src/reorder_restart/read_final_state.py.
Outputs: intrinsic_interface_geometry.json, intrinsic_interface_restart.json
(header as the reference reader decodes it), intrinsic_interface_state.npz
(tag, r, v, glob_no per molecule), and verbatim copies of the restart file
(intrinsic_interface_initial_state.bin) and of two keyword input files
(default.in, MD_2_phase.in) for the reader tests.
"""
from __future__ import annotations

import contextlib
import io
import json
import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT", "")
HERE = os.path.dirname(os.path.abspath(__file__))


def parse_header(path):
    out = {}
    for line in open(path):
        parts = [p.strip() for p in line.split(";")]
        if len(parts) >= 3 and parts[1]:
            out[parts[1]] = parts[2]
    return out


def main():
    if not REF or not os.path.isdir(REF):
        sys.exit("usage: make_golden.py <reference checkout root>  (or set REFERENCE_ROOT)")
    hdr = parse_header(os.path.join(REF, "runs/Intrinsic_Interface/results/simulation_header"))
    sys.path.insert(0, os.path.join(REF, "src/reorder_restart"))
    import read_final_state as rfs  # the reference's own reader

    with contextlib.redirect_stdout(io.StringIO()):
        fs = rfs.final_state(os.path.join(REF, "runs/Intrinsic_Interface/initial_state"))
        tag, r, v = fs.read_moldata()
    h = {k: (float(x) if isinstance(x, float) else int(x)) for k, x in fs.headerDict.items()}
    geom = {
        "nunits": [h["initialunits1"], h["initialunits2"], h["initialunits3"]],
        "density": float(hdr["density"]),
        "rcutoff": float(hdr["rcutoff"]),
        "delta_rneighbr": [float(hdr["delta_rneighbrx"]), float(hdr["delta_rneighbry"]),
                           float(hdr["delta_rneighbrz"])],
        "globaldomain": [float(hdr["globaldomain(1)"]), float(hdr["globaldomain(2)"]),
                         float(hdr["globaldomain(3)"])],
        "initialunitsize": [float(hdr["initialunitsize(1)"]), float(hdr["initialunitsize(2)"]),
                            float(hdr["initialunitsize(3)"])],
        "volume": float(hdr["volume"]),
        "ncells": [int(hdr["globalncells(1)"]), int(hdr["globalncells(2)"]), int(hdr["globalncells(3)"])],
        "cellsidelength": [float(hdr["cellsidelength(1)"]), float(hdr["cellsidelength(2)"]),
                           float(hdr["cellsidelength(3)"])],
        "globalnp": int(hdr["globalnp"]),
    }
    json.dump(geom, open(os.path.join(HERE, "intrinsic_interface_geometry.json"), "w"), indent=1)
    json.dump(h, open(os.path.join(HERE, "intrinsic_interface_restart.json"), "w"), indent=1)
    glob = fs.globnum if h.get("global_numbering") else np.arange(1, len(tag) + 1)
    np.savez_compressed(os.path.join(HERE, "intrinsic_interface_state.npz"), tag=tag, r=r, v=v,
                        glob_no=np.asarray(glob), size=np.array([os.path.getsize(
                            os.path.join(REF, "runs/Intrinsic_Interface/initial_state"))]))
    import shutil
    shutil.copyfile(os.path.join(REF, "runs/Intrinsic_Interface/initial_state"),
                    os.path.join(HERE, "intrinsic_interface_initial_state.bin"))
    shutil.copyfile(os.path.join(REF, "src/default.in"), os.path.join(HERE, "default.in"))
    shutil.copyfile(os.path.join(REF, "runs/Intrinsic_Interface/MD_2_phase.in"), os.path.join(HERE, "MD_2_phase.in"))
    print("wrote fixtures for", geom["globalnp"], "molecules")


if __name__ == "__main__":
    main()
