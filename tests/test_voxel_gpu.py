"""GPU geometry pipeline (lbm_stl_read_ascii + lbm_voxelise) against the
reference's own setup chain.

For every golden case (the STL cylinders of tests/golden/make_golden.py, whose
node maps the reference's Geometry + SubDomain produced), the STL is written
again, read by the library and voxelised on the GPU with the case's inlet and
outlet planes: node coordinates and kinds, the inlet, outlet and wall lists
(same order) and the near-wall set must equal the reference's, and the
near-wall normals (area / distance^2 weighted facet normals) must equal them
bit for bit.
"""
import os
import sys

import numpy as np
import pytest

from lbm_b200 import geometry as G

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as M  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = {c["name"]: c for c in M.small_cases()}
CASES["pipe16"] = M.pipe16_case()
FIXTURE = {name: ("pipe16_2000.npz" if name == "pipe16" else name + ".npz") for name in CASES}


def openings(c):
    def block(kind, b):
        return G.opening(kind, b["plane"], b["coordinate"], b["normal"], b.get("range_x"), b.get("range_y"),
                         b.get("range_z"))
    return [block("inlet", c["inlet"])] + [block("outlet", o) for o in c["outlets"]]


@pytest.mark.parametrize("name", sorted(CASES))
def test_voxeliser_reproduces_reference_node_map(name, tmp_path):
    c = CASES[name]
    tris = M.permute(M.cylinder_triangles(c["R"], c["L"], c["naz"], c["nax"]), c["axis"])
    stl = tmp_path / "geom.stl"
    M.write_stl(str(stl), tris)
    topo, (dims, origin, spacing, ms) = G.voxelise_stl(G.read_stl(stl), 0.5, openings(c), info=True)
    ref = np.load(os.path.join(HERE, "golden", FIXTURE[name]))
    assert spacing == 1.0
    np.testing.assert_array_equal(topo["coords"], ref["coords"].astype(np.int32))
    np.testing.assert_array_equal(topo["kind"], ref["kind"])
    np.testing.assert_array_equal(topo["inlet"], ref["inlet"])
    np.testing.assert_array_equal(topo["wall"], ref["wall"])
    np.testing.assert_array_equal(topo["inlet_normal"], ref["inlet_normal"])
    k = 0
    while "outlet_%d" % k in ref.files:
        np.testing.assert_array_equal(topo["outlet_%d" % k], ref["outlet_%d" % k])
        np.testing.assert_array_equal(topo["outlet_normal_%d" % k], ref["outlet_normal_%d" % k])
        k += 1
    assert "outlet_%d" % k not in topo
    # near-wall list: the reference's order is a hash set's; compare by node
    mine = np.argsort(topo["nearwall"])
    theirs = np.argsort(ref["nearwall"])
    np.testing.assert_array_equal(topo["nearwall"][mine], ref["nearwall"][theirs])
    np.testing.assert_array_equal(topo["nearwall_normal"][mine], ref["nearwall_normal"][theirs])
