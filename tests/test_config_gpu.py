"""config.txt driving the engine, on the GPU.

* The reference's waveform given as the config's three equations (the
  engine's lbm_set_pulsatile) reproduces the reference's own pulsatile run of
  the golden cylinder bit for bit; a one-constant-piece waveform equals
  constant flow at that speed.
* The drop-in program wires the config's equations into the waveform: with a
  waveform of its own in config.txt, its final state equals the engine's run
  with those pieces.
* run_config does the reference program's whole job from config.txt (STL read,
  GPU voxelisation, steps, WriteOutput at IterToWrite): its state after the
  run equals the reference's golden final state, its surface CSV holds the
  reference's rows for that state (row order aside: the reference's comes
  from a hash set) and its smoothed CSV is the reference's smoothing of it.
"""
import os
import subprocess

import numpy as np
import pytest

from lbm_b200 import Engine
from lbm_b200.config import Pulse, read_config, run_config
from oracle import oracle as orc
from test_config import REFERENCE_PIECES
from test_output_gpu import parse_vtu, reference_csv, reference_smooth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
BINARY = os.path.join(ROOT, "reza-seti_b200", "host", "_build", "lbm_dropin")


def make_golden():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: d[k] for k in d.files}


def engine_for(d):
    meta = d["meta_d"]
    return Engine(d, tau=meta[0], dt=meta[1], spacing=meta[2], storage="f64")


def test_reference_equations_reproduce_reference_run():
    d = load("cyl_z_pulsatile")
    e = engine_for(d)
    e.set_flow(True, 0.0)
    e.set_pulsatile(Pulse(REFERENCE_PIECES))
    e.step(100)
    np.testing.assert_array_equal(e.populations(), d["final__f"])
    wss, acc, accmag = e.wss()
    np.testing.assert_array_equal(wss, d["final__wss"])
    osi, tawss = e.osi_tawss()
    np.testing.assert_array_equal(osi, d["final__osi"])
    np.testing.assert_array_equal(tawss, d["final__tawss"])


def test_constant_piece_equals_constant_flow():
    d = load("cyl_z")
    a, b = engine_for(d), engine_for(d)
    a.set_flow(False, 0.05)
    b.set_flow(True, 0.0)
    b.set_pulsatile(Pulse([[0.05]], bounds=[0.0, 1.0], period=0.9))
    a.step(40)
    b.step(40)
    np.testing.assert_array_equal(a.populations(), b.populations())
    np.testing.assert_array_equal(a.wss()[0], b.wss()[0])
    # back to the built-in waveform
    b.set_pulsatile(None)


def write_case(tmp_path, name, **kw):
    mg = make_golden()
    case = [c for c in mg.small_cases() if c["name"] == name][0]
    tris = mg.permute(mg.cylinder_triangles(case["R"], case["L"], case["naz"], case["nax"]), case["axis"])
    mg.write_stl(str(tmp_path / "geom.stl"), tris)
    args = dict(inlet=case["inlet"], outlets=case["outlets"])
    if "flow" in case:
        args["flow"] = case["flow"]
    if "dt" in case:
        args["dt"] = case["dt"]
    args.update(kw)
    mg.write_config(str(tmp_path / "config.txt"), **args)
    return tris


def test_dropin_takes_waveform_from_equations(tmp_path):
    assert os.path.exists(BINARY), "drop-in not built: make -C reza-seti_b200/host"
    write_case(tmp_path, "cyl_z_pulsatile", max_iter=1)
    text = (tmp_path / "config.txt").read_text()
    pieces = [[2e-3, 0.03], [0.045], [-0.02, 0.04, 0.01]]
    eq = "equations:\n" + "".join("    InletVel%d: [%s]\n" % (k + 1, ", ".join(repr(c) for c in p))
                                  for k, p in enumerate(pieces))
    text = text[:text.index("equations:")] + eq
    (tmp_path / "config.txt").write_text(text)
    env = dict(os.environ, LBM_B200_DUMP=str(tmp_path / "dump.bin"))
    r = subprocess.run([BINARY], cwd=str(tmp_path), env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    dump = make_golden().read_dump(str(tmp_path / "dump.bin"))
    d = load("cyl_z_pulsatile")
    e = engine_for(d)
    e.set_flow(True, 0.0)
    e.set_pulsatile(Pulse(pieces))
    e.step(orc.pulsatile_step_count(float(d["meta_d"][1])))
    np.testing.assert_array_equal(dump["final/f"], e.populations())


def test_run_config_reproduces_reference_outputs(tmp_path):
    write_case(tmp_path, "cyl_z", max_iter=60, iter_to_write=59)
    cfg = read_config(tmp_path / "config.txt")
    assert cfg["MaxIter"] == 60 and cfg["IterToWrite"] == 59
    eng, total, outputs = run_config(tmp_path / "config.txt")
    assert total == 60 and outputs == [(59, "Iteration_59")]
    d = load("cyl_z")
    np.testing.assert_array_equal(eng.populations(), d["final__f"])
    # the reference's file text from its own final state; grid origin =
    # bounding-box minimum of the STL's vertices as read back from the file
    # (Geometry::pointsBox)
    from lbm_b200 import geometry as G
    v = G.read_stl(tmp_path / "geom.stl")[:, :9].reshape(-1, 3)
    origin = tuple(float(x) for x in v.min(axis=0))
    want = reference_csv(d, origin, 2 * cfg["grid_size"], False).splitlines()
    got = (tmp_path / "59_FlowHemodynamics.csv").read_text()
    # rows follow the caller's near-wall list; the reference's is a
    # pointer-keyed hash set, whose order not even the reference repeats
    lines = got.splitlines()
    assert lines[0] == want[0] and sorted(lines[1:]) == sorted(want[1:])
    smooth, _ = reference_smooth(got, 0.25, False)
    assert (tmp_path / "FlowHemodynamics" / "Iteration_59_59_FlowHemodynamics.csv").read_text() == smooth
    npts, ncells, arr = parse_vtu(tmp_path / "Fluid_Variables" / "59.vtu")
    assert npts == len(d["coords"]) and ncells > 0
    assert sorted(arr["Density"].tolist()) == sorted(d["final__rho"].tolist())


def test_physics_mode_pulsatile_setter_order():
    """In physics mode the initial store already applies the inlet correction
    of the waveform at t = 0, so the waveform pieces must reach that store in
    whichever order the setters are called: flow type then pieces gives the
    same populations as pieces then flow type."""
    from lbm_b200 import geometry as G
    topo = G.straight_pipe(radius=5.0, length=24)
    pulse = Pulse([[0.4, 0.02], [0.03], [-0.01, 0.03]], period=0.9)

    def run(order):
        e = Engine(topo, tau=0.7, dt=1e-3, storage="f64", bc="physics")
        e.set_inlet_profile(G.parabolic_inlet(topo, 1.0))
        if order == "flow_first":
            e.set_flow(True, 0.0)
            e.set_pulsatile(pulse)
        else:
            e.set_pulsatile(pulse)
            e.set_flow(True, 0.0)
        e.step(5)
        f = e.populations()
        e.close()
        return f

    a, b = run("flow_first"), run("pieces_first")
    np.testing.assert_array_equal(a, b)
