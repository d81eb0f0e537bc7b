"""Failure detection on the GPU, without faulting it: a detector that fires
on a real non-finite state, and the geometry inputs the reference only warns
about.

* The reference's own y-branch inlet divides by zero in its first step
  (golden case cyl_y: u_y = 1 gives 1 - u_y = 0, Boundary.cpp:171-221), and
  it runs on with NaN. The engine sets device flag 2 in that step; with the
  numeric check on, lbm_step returns LBM_ERR_NUMERIC once the flag's copy has
  reached the host, runs no further step, and a long call stops early. With
  the check off it runs on like the reference; lbm_set_populations starts a
  new state with the flags cleared.
* lbm_voxelise refuses an inlet plane that matches no grid point, and a
  geometry without an inlet opening, where the reference prints a warning
  (ComplexGeometry.cpp:667-672) and simulates a flow nothing drives; the
  config.txt runner passes that error on.
"""
import os

import numpy as np
import pytest

from lbm_b200 import Engine, capi
from lbm_b200 import geometry as G

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cyl_y(numeric_check=True):
    d = np.load(os.path.join(GOLDEN, "cyl_y.npz"))
    topo = {k: d[k] for k in d.files}
    meta = topo["meta_d"]
    e = Engine(topo, tau=meta[0], dt=meta[1], spacing=meta[2], storage="f64", numeric_check=numeric_check)
    e.set_flow(False, float(meta[4]))
    return e, topo


def test_nonfinite_density_raises_flag_and_numeric_status():
    e, topo = cyl_y()
    e.step(1)
    assert not np.isfinite(e.populations()).all()  # the reference's own NaN (golden p1 state)
    assert e.flags() & capi.FLAG_NONFINITE
    with pytest.raises(capi.LbmError) as ei:
        e.step(3)
    assert ei.value.code == capi.LBM_ERR_NUMERIC
    assert e.time()[0] == 1  # no step ran
    # off: runs on through the NaN, as the reference does
    e.set_numeric_check(False)
    e.step(3)
    assert e.time()[0] == 4
    np.testing.assert_array_equal(e.populations(), topo["final__f"])
    # a finite state uploaded: flags cleared, the check lets the next call run
    e.set_numeric_check(True)
    f = np.tile(np.array([2 / 36] * 6 + [1 / 36] * 12 + [12 / 36]), (len(topo["kind"]), 1))
    e.set_populations(f)
    assert e.flags() == 0
    e.step(1)
    assert e.time()[0] == 5
    e.close()


def test_numeric_check_stops_a_long_call_early():
    e, _ = cyl_y()
    with pytest.raises(capi.LbmError) as ei:
        e.step(200000)
    assert ei.value.code == capi.LBM_ERR_NUMERIC
    steps = e.time()[0]
    assert 256 <= steps < 200000
    e.close()


def test_stable_run_passes_the_check():
    d = np.load(os.path.join(GOLDEN, "cyl_z.npz"))
    topo = {k: d[k] for k in d.files}
    meta = topo["meta_d"]
    e = Engine(topo, tau=meta[0], dt=meta[1], spacing=meta[2], storage="f32")
    e.set_flow(False, float(meta[4]))
    e.step(600)  # three flag copies inside the call
    e.step(10)
    assert e.time()[0] == 610 and e.flags() == 0
    e.close()


def pipe_stl():
    return G.tube_triangles(lambda z: (0.37, 0.21), lambda z: 4.0, 0.0, 16.0, 16, 8)


def test_voxelise_refuses_an_inlet_plane_off_the_geometry():
    tris = pipe_stl()
    ok = [G.opening("inlet", "z", 0.0, (0, 0, -1)), G.opening("outlet", "z", 16.0, (0, 0, 1))]
    topo = G.voxelise_stl(tris, 0.5, ok)
    assert len(topo["inlet"]) > 0
    off = [G.opening("inlet", "z", -7.0, (0, 0, -1)), G.opening("outlet", "z", 16.0, (0, 0, 1))]
    with pytest.raises(capi.LbmError) as ei:
        G.voxelise_stl(tris, 0.5, off)
    assert ei.value.code == capi.LBM_ERR_ARGUMENT and "matches no grid point" in str(ei.value)
    with pytest.raises(capi.LbmError) as ei:
        G.voxelise_stl(tris, 0.5, ok[1:])
    assert "no inlet opening" in str(ei.value)


def test_run_config_passes_the_inlet_error_on(tmp_path):
    from lbm_b200.config import run_config
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    case = [c for c in mg.small_cases() if c["name"] == "cyl_z"][0]
    tris = mg.permute(mg.cylinder_triangles(case["R"], case["L"], case["naz"], case["nax"]), case["axis"])
    mg.write_stl(str(tmp_path / "geom.stl"), tris)
    inlet = dict(case["inlet"])
    inlet["coordinate"] = -50.0
    mg.write_config(str(tmp_path / "config.txt"), inlet=inlet, outlets=case["outlets"], max_iter=2)
    with pytest.raises(capi.LbmError) as ei:
        run_config(tmp_path / "config.txt")
    assert "matches no grid point" in str(ei.value)
