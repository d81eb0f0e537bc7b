"""End to end through the drop-in: the reference's own program (LBM.cpp main,
Geometry, SubDomain) linked with the B200 Simulation replacement
(reza-seti_b200/host/Simulation_b200.cpp) runs the R=4 cylinder from its STL
and config.txt, writing outputs every 20 steps, and its final Node fields must
equal the reference's own run bit for bit."""
import importlib.util
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "reza-seti_b200", "host", "_build", "lbm_dropin")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def make_golden():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_dropin_program_matches_reference(tmp_path):
    assert os.path.exists(BINARY), "drop-in not built: make -C reza-seti_b200/host"
    mg = make_golden()
    case = [c for c in mg.small_cases() if c["name"] == "cyl_z"][0]
    tris = mg.permute(mg.cylinder_triangles(case["R"], case["L"], case["naz"], case["nax"]), case["axis"])
    mg.write_stl(str(tmp_path / "geom.stl"), tris)
    mg.write_config(str(tmp_path / "config.txt"), max_iter=case["steps"], iter_to_write=20,
                    inlet=case["inlet"], outlets=case["outlets"])
    env = dict(os.environ, LBM_B200_DUMP=str(tmp_path / "dump.bin"))
    r = subprocess.run([BINARY], cwd=str(tmp_path), env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Iteration output written: Iteration_40" in r.stdout
    assert "Iteration 59 has been performed successfully" in r.stdout
    d = mg.read_dump(str(tmp_path / "dump.bin"))
    g = np.load(os.path.join(GOLDEN, "cyl_z.npz"))
    np.testing.assert_array_equal(d["final/f"], g["final__f"])
    np.testing.assert_array_equal(d["final/rho"], g["final__rho"])
    np.testing.assert_array_equal(d["final/u"], g["final__u"])
    np.testing.assert_array_equal(d["final/velmag"], g["final__velmag"])
    # near-wall values keyed by node index (both lists come from the same set)
    order = {int(n): k for k, n in enumerate(g["nearwall"])}
    idx = np.array([order[int(n)] for n in d["nearwall"]])
    np.testing.assert_array_equal(d["final/wss"], g["final__wss"][idx])
    np.testing.assert_array_equal(d["final/acc"], g["final__acc"][idx])
    np.testing.assert_array_equal(d["final/accmag"], g["final__accmag"][idx])
