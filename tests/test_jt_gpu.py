"""The reference's own shipped case, JT.stl with its config.txt, at grid_size
0.2 (tests/golden/make_jt.py: the reference's setup and 50 steps of its loop).

* The GPU pipeline voxelises the STL with the config's four outlet blocks (x
  planes, y planes limited by range_x / range_z; at this grid only one of
  them meets grid points, as in the reference) into the reference's node
  map: coordinates, kinds, inlet / outlet / wall lists, the near-wall set
  and its normals, bit for bit.
* On that node map the FP64 engine (reference boundaries) reproduces the
  reference's 50 steps bit for bit: sampled populations and moments, every
  WSS value and accumulator, whole-field checksums; FP32 storage stays within
  the FP32 parity bounds of tests/test_parity_gpu.py.
"""
import json
import os

import numpy as np
import pytest

from lbm_b200 import Engine
from lbm_b200 import geometry as G

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "jt_g0.2.npz")


@pytest.fixture(scope="module")
def jt():
    d = np.load(FIXTURE)
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="module")
def topo(jt):
    return G.voxelise_stl(jt["triangles"], float(jt["grid_size"][0]), json.loads(str(jt["openings"])))


def test_voxeliser_reproduces_reference_node_map(jt, topo):
    np.testing.assert_array_equal(topo["coords"], jt["coords"])
    np.testing.assert_array_equal(topo["kind"], jt["kind"])
    np.testing.assert_array_equal(topo["inlet"], jt["inlet"])
    np.testing.assert_array_equal(topo["inlet_normal"], jt["inlet_normal"])
    np.testing.assert_array_equal(topo["wall"], jt["wall"])
    n_out = int(jt["meta_i"][5])
    assert n_out == 4
    for k in range(n_out):
        np.testing.assert_array_equal(topo["outlet_%d" % k], jt["outlet_%d" % k])
        np.testing.assert_array_equal(topo["outlet_normal_%d" % k], jt["outlet_normal_%d" % k])
    assert [len(jt["outlet_%d" % k]) for k in range(n_out)] == [0, 27, 0, 0]
    mine, theirs = np.argsort(topo["nearwall"]), np.argsort(jt["nearwall"])
    np.testing.assert_array_equal(topo["nearwall"][mine], jt["nearwall"][theirs])
    np.testing.assert_array_equal(topo["nearwall_normal"][mine], jt["nearwall_normal"][theirs])


def run(jt, topo, storage):
    meta = jt["meta_d"]
    e = Engine(topo, tau=meta[0], dt=meta[1], spacing=meta[2], storage=storage, numeric_check=False)
    e.set_flow(False, float(jt["cte_vel"][0]))
    e.step(int(jt["steps"][0]))
    f = e.populations()
    rho, u = e.macros()
    w, acc, accm = e.wss()
    e.close()
    return f, rho, u, w, acc, accm


def test_fp64_reproduces_reference_steps(jt, topo):
    f, rho, u, w, acc, accm = run(jt, topo, "f64")
    s = jt["sample"]
    np.testing.assert_array_equal(f[s], jt["final__f_sample"])
    np.testing.assert_array_equal(rho[s], jt["final__rho_sample"])
    np.testing.assert_array_equal(u[s], jt["final__u_sample"])
    # near-wall arrays in the fixture are in the reference's near-wall order,
    # which the voxeliser reproduces as a set: compare by node
    mine, theirs = np.argsort(topo["nearwall"]), np.argsort(jt["nearwall"])
    np.testing.assert_array_equal(w[mine], jt["final__wss"][theirs])
    np.testing.assert_array_equal(acc[mine], jt["final__acc"][theirs])
    np.testing.assert_array_equal(accm[mine], jt["final__accmag"][theirs])
    np.testing.assert_array_equal(np.array([f.sum(), np.abs(f).sum(), (f * f).sum()]), jt["final__f_sum"])


def test_fp32_within_parity_bounds(jt, topo):
    f, rho, u, w, acc, accm = run(jt, topo, "f32")
    s = jt["sample"]
    mine, theirs = np.argsort(topo["nearwall"]), np.argsort(jt["nearwall"])

    def close(a, b, floor):
        return bool(np.all(np.abs(a - b) <= 1e-5 * np.abs(b) + floor * np.max(np.abs(b))))

    assert close(f[s], jt["final__f_sample"], 0.0)
    assert close(rho[s], jt["final__rho_sample"], 0.0)
    assert close(u[s], jt["final__u_sample"], 3e-6)
    assert close(w[mine], jt["final__wss"][theirs], 3e-6)
    assert close(acc[mine], jt["final__acc"][theirs], 3e-6)
    assert close(accm[mine], jt["final__accmag"][theirs], 3e-6)
