"""Writes tests/golden/jt_g0.2.npz: the reference's own shipped case (JT.stl
with its config.txt) at a coarser grid, as the reference sets it up and runs
it.

The reference ships one real case: JT.stl (9,712 facets) with config.txt
(grid_size 0.025: a 318 x 407 x 500 grid, which the reference's O(points x
facets) setup takes hours to label). With grid_size 0.2 (spacing 0.4, a
41 x 52 x 64 grid) the reference harness (oracle/_ref/refharness, the
reference's own Geometry, SubDomain and Simulation compiled from its sources)
sets it up in about half a minute; everything else is the shipped config.txt:
tau 0.68, constant inflow 0.1 on the z = -178.5 inlet, and its four outlet
blocks (x planes, and y planes limited by range_x / range_z).

The fixture holds the STL's triangles as the library's reader (the
reference reader's grammar) returns them, the opening blocks as parsed from
the config, the node map the reference built (coordinates, kinds, inlet,
outlet, wall and near-wall lists, near-wall normals), and, after STEPS time
steps of the reference's loop, a seeded sample of the populations and
moments, all WSS values and accumulators and whole-field checksums.

    python tests/golden/make_jt.py <reference source directory>
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "reza-seti_b200"))
sys.path.insert(0, HERE)

import make_golden as M  # noqa: E402

GRID_SIZE = 0.2
STEPS = 50
FIXTURE = os.path.join(HERE, "jt_g0.2.npz")


def main(argv):
    if len(argv) != 2:
        sys.exit(__doc__)
    ref = argv[1]
    from lbm_b200 import geometry as G
    from lbm_b200.config import read_config
    if not os.path.exists(M.HARNESS):
        sys.exit("build the reference harness first: make -C oracle REF=<reference sources>")
    tris = G.read_stl(os.path.join(ref, "JT.stl"))
    with tempfile.TemporaryDirectory() as tmp:
        shutil.copy(os.path.join(ref, "JT.stl"), os.path.join(tmp, "JT.stl"))
        text = open(os.path.join(ref, "config.txt")).read()
        assert "grid_size: 0.025" in text
        text = text.replace("grid_size: 0.025", "grid_size: %r" % GRID_SIZE)
        cfg_path = os.path.join(tmp, "config.txt")
        with open(cfg_path, "w") as fh:
            fh.write(text)
        cfg = read_config(cfg_path)
        dump = os.path.join(tmp, "dump.bin")
        subprocess.run([M.HARNESS, "stl", cfg_path, str(STEPS), dump], check=True, stdout=subprocess.DEVNULL)
        d = M.read_dump(dump)
    assert int(d["meta_i"][6]) == 0, "fluid node with an uninitialised Wall tag"
    out = M.keep_pipe(d)
    out["coords"] = d["coords"].astype(np.int32)
    out["triangles"] = tris
    out["grid_size"] = np.array([GRID_SIZE])
    out["steps"] = np.array([STEPS])
    out["openings"] = np.array(json.dumps(cfg["inlets"] + cfg["outlets"]))
    out["cte_vel"] = np.array([cfg["CteVel"]])
    np.savez_compressed(FIXTURE, **out)
    print("nodes", int(d["meta_i"][0]), "inlet", len(d["inlet"]), "outlets",
          [len(d["outlet_%d" % k]) for k in range(int(d["meta_i"][5]))], "near-wall", len(d["nearwall"]))


if __name__ == "__main__":
    main(sys.argv)
