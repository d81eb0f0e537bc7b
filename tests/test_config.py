"""config.txt parsing (lbm_config_parse) and the piecewise-polynomial
waveform (lbm_pulse_eval), on the CPU.

The parser is pinned to the reference's own parseInputFile (LBM.h:81-188),
compiled into oracle/_ref/refharness ("config" mode prints what it read): on
every file below both must read the same values, bit for bit, including the
grammar's corners (numeric prefixes of std::stod / std::stoi, an int field set
from stod, quotes, comments, whitespace-only lines that do not end a block and
so swallow a following section). The waveform with the reference's pieces
must equal the oracle's restatement of Simulation::getInletVelocity bit for
bit, and a C program built here must see the structures at the offsets the
ctypes binding uses.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from lbm_b200 import capi
from lbm_b200.config import Pulse, output_schedule, read_config, reference_pulse
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "refharness")

FULL = """parameters:

  stl_file: "vessel_a.stl"
  FlowType: "Pulsatile"
  time_resolution: 2e-5
  density: 1060.5
  kinematic_viscosity: 3.3e-6
  relaxation_factor: 0.71
  grid_size: 0.0375
  pressure: 2
  CteVel: 0.125   # inflow
  reynolds_number: 250
  number_of_outlets: 3
  MaxIter: 12001
  IterToWrite: 4000
  Systole: 0.2
  Diastole: 0.85
  period: 0.9
  NumCycle: 3


inlets:

    plane: z
    coordinate: -42.25
    normal: [0, 0, -1]

outlets:

    plane: x
    coordinate: 7.5
    normal: [1, 0, 0]   # first

    plane: y
    coordinate: -61.125
    range_x: [1.5, 4.0]
    range_z: [-30.0, -27.5]
    normal: [0, 1, 0]

    plane: y
    coordinate: -63.5
    range_x: [6.0, 8.5]
    range_z: [-25, -22]
    normal: [0, -1, 0]

equations:
    A: [-2.5e+06, 1.25e+05, -3.1, 0.5]
    B: [4.0, -3.0, 2.0]
    C: [1.5]
"""

# a whitespace-only line does not end a block: the outlet block runs on and
# takes "equations:" and its lines as unknown keys
SWALLOW = """parameters:
  FlowType: "Constant"
  CteVel: 0.05

inlets:
    plane: x
    coordinate: 1
    normal: [-1, 0, 0]

outlets:
    plane: x
    coordinate: 9
    normal: [1, 0, 0]
""" + "    \n" + """equations:
    P1: [1, 2, 3]
"""

# numeric prefixes (stod / stoi), an int field from stod, tabs, quotes,
# comments, a second colon in a value, two inlets, unknown and extension keys
# (the reference skips them)
CORNERS = """# leading comment
parameters:
\tstl_file: "C:/data/v.stl"
  FlowType: Constant
  time_resolution: 1e-5 # comment after a number
  relaxation_factor:   0.6
  MaxIter: 3.9e3
  IterToWrite: 250.75
  NumCycle: 2.7
  Systole: .15
  lattice: D3Q27
  storage: f16
  boundary: physics
  outlet_density: 1.01
  harmonic_period_steps: 4000
  harmonic_amplitudes: [0.5, 0.25]
  harmonic_phases: [0.1, -0.2]
  equation_bounds: [0, 0.5, 1]
  some_key_nobody_reads: 7

inlets:
    plane: y
    coordinate: 3
    range_z: [1, 2]
    normal: [0, -1, 0]

    plane: y
    coordinate: 30
    normal: [0, 1, 0]
    # a comment inside a block

outlets:
    plane: z
    coordinate: 100.25
    range_x: [-1e300, 1e300]
    range_y: [ -5 , 5 ]
    normal: [0, 0, 1]
"""

CASES = {"full": FULL, "swallow": SWALLOW, "corners": CORNERS}


def reference_parse(path):
    r = subprocess.run([HARNESS, "config", str(path)], capture_output=True, text=True, timeout=60)
    out = {"inlets": [], "outlets": [], "equations": []}
    for line in r.stdout.splitlines():
        tok = line.split(" ")
        if tok[0] == "error":
            return {"error": line}
        if tok[0] in ("inlet", "outlet"):
            vals, lists, i = tok[3:], [], 0
            while i < len(vals):
                n = int(vals[i])
                lists.append([float(v) for v in vals[i + 1:i + 1 + n]])
                i += 1 + n
            out[tok[0] + "s"].append({"plane": tok[1], "coordinate": float(tok[2]), "range_x": lists[0],
                                      "range_y": lists[1], "range_z": lists[2], "normal": lists[3]})
        elif tok[0] == "equation":
            n = int(tok[2])
            out["equations"].append((tok[1], [float(v) for v in tok[3:3 + n]]))
        else:
            out[tok[0]] = " ".join(tok[1:])
    assert r.returncode == 0, r.stderr
    return out


def same_float(a, b):
    return (math.isnan(a) and math.isnan(b)) or a == b


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference harness not built (make -C oracle)")
@pytest.mark.parametrize("name", sorted(CASES))
def test_parser_reads_what_the_reference_reads(name, tmp_path):
    path = tmp_path / "config.txt"
    path.write_text(CASES[name])
    ref = reference_parse(path)
    mine = read_config(path)
    assert mine["stl_file"] == ref["stl_file"]
    assert mine["FlowType"] == ref["FlowType"]
    for key in ("dt", "rho", "nu_blood", "tau", "grid_size", "pressure", "CteVel", "reynolds_number", "Systole",
                "Diastole"):
        assert same_float(mine[key], float(ref[key])), key
    for key in ("number_of_outlets", "MaxIter", "IterToWrite", "NumCycle"):
        assert mine[key] == int(ref[key]), key
    for kind in ("inlets", "outlets"):
        assert len(mine[kind]) == len(ref[kind])
        for m, r in zip(mine[kind], ref[kind]):
            assert m["plane"] == r["plane"]
            assert m["coordinate"] == r["coordinate"]
            assert m["normal"] == r["normal"]
            for ax in "xyz":
                want = r["range_" + ax]
                got = m["range_" + ax]
                assert (got is None and want == [-math.inf, math.inf]) or list(got) == want, ax
    assert mine["equations"] == ref["equations"]


def test_parser_corners_and_extensions(tmp_path):
    path = tmp_path / "config.txt"
    path.write_text(CORNERS)
    c = read_config(path)
    assert c["stl_file"] == "C:/data/v.stl" and c["FlowType"] == "Constant"
    assert c["MaxIter"] == 3 and c["IterToWrite"] == 250 and c["NumCycle"] == 2 and c["Systole"] == 0.15
    assert c["lattice"] == "D3Q27" and c["storage"] == "f16" and c["boundary"] == "physics"
    assert c["outlet_density"] == 1.01 and c["harmonic_period_steps"] == 4000
    assert c["harmonic_amplitudes"] == [0.5, 0.25] and c["harmonic_phases"] == [0.1, -0.2]
    assert c["equation_bounds"] == [0, 0.5, 1]
    assert [o["plane"] for o in c["inlets"]] == ["y", "y"] and c["inlets"][0]["range_z"] == (1, 2)
    path.write_text(SWALLOW)
    c = read_config(path)
    assert c["equations"] == [] and len(c["outlets"]) == 1
    assert c["lattice"] == "D3Q19" and c["storage"] == "f64" and c["boundary"] == "reference"
    assert c["period"] == 0.9 and c["outlet_density"] == 1.0


@pytest.mark.parametrize("text,what", [
    ("parameters:\n  time_resolution: fast\n", "bad number"),
    ("inlets:\n    plane: w\n    coordinate: 1\n    normal: [0, 0, 1]\n", "plane"),
    ("inlets:\n    plane: z\n    normal: [0, 0, 1]\n", "coordinate"),
    ("outlets:\n    plane: z\n    coordinate: 1\n    normal: [0, 1]\n", "normal"),
    ("outlets:\n    plane: z\n    coordinate: 1\n    range_x: [2]\n    normal: [0, 0, 1]\n", "range"),
    ("parameters:\n  lattice: D2Q9\n", "lattice"),
    ("parameters:\n  harmonic_amplitudes: [1, 2]\n  harmonic_phases: [0]\n", "harmonic_phases"),
])
def test_parser_rejects_what_the_reference_cannot_read(text, what, tmp_path):
    path = tmp_path / "config.txt"
    path.write_text(text)
    with pytest.raises(capi.LbmError) as ex:
        read_config(path)
    assert what in str(ex.value)
    if what == "bad number" and os.path.exists(HARNESS):
        # the reference's std::stod throws there too
        assert "error" in reference_parse(path)


def test_missing_file_is_an_error(tmp_path):
    with pytest.raises(capi.LbmError) as ex:
        read_config(tmp_path / "nope.txt")
    assert "Unable to open input file" in str(ex.value)


REFERENCE_PIECES = [
    [-8.579e+08, 4.059e+08, -7.817e+07, 7.994e+06, -4.835e+05, 1.782e+04, -321.6, 3.215, 0.1423],
    [-4.32e+06, 7.94e+06, -6.298e+06, 2.82e+06, -7.809e+05, 1.37e+05, -1.484e+04, 901.9, -22.87],
    [-5.123, 14.15, -14.21, 5.865, -0.5696],
]


def test_reference_waveform_bit_for_bit():
    """Built-in and given-as-pieces reference waveforms equal the oracle's
    getInletVelocity at every step time of a pulsatile run and between."""
    ts = np.concatenate([np.cumsum(np.full(3000, 1e-3)), np.linspace(0, 2.7, 20011), [0.09, 0.27, 0.81, 0.9]])
    pieces = Pulse(REFERENCE_PIECES)
    for t in ts:
        want = orc.pulsatile_velocity(float(t))
        assert reference_pulse(t) == want
        assert pieces(t) == want


def test_custom_pieces():
    """Two pieces over half periods of 2 s: each a polynomial summed from the
    highest power down with pow, x * x, x and the constant; 0 outside."""
    p = Pulse([[2.0, -1.0, 0.5, 0.25], [3.0, 0.125]], bounds=[0.0, 0.5, 1.0], period=2.0)
    for t in np.linspace(-0.5, 5.0, 1001):
        x = math.fmod(t, 2.0)
        if 0 <= x < 1.0:
            want = 2.0 * math.pow(x, 3) + -1.0 * (x * x) + 0.5 * x + 0.25
        elif 1.0 <= x < 2.0:
            want = 3.0 * x + 0.125
        else:
            want = 0.0
        assert p(t) == want
    with pytest.raises(ValueError):
        Pulse([[1.0]], bounds=[0.0, 0.5, 1.0])


def test_equations_become_pieces_only_when_whole(tmp_path):
    base = {"equations": [], "equation_bounds": [], "period": 0.9}
    assert Pulse.from_config(base) is None
    assert Pulse.from_config(dict(base, equations=[("InletVel1", [0.0])])) is None
    three = Pulse.from_config(dict(base, equations=[("a", REFERENCE_PIECES[0]), ("b", REFERENCE_PIECES[1]),
                                                    ("c", REFERENCE_PIECES[2])]))
    assert [three(t) for t in (0.05, 0.2, 0.5)] == [reference_pulse(t) for t in (0.05, 0.2, 0.5)]
    two = Pulse.from_config(dict(base, equations=[("a", [1.0]), ("b", [2.0])], equation_bounds=[0, 0.5, 1]))
    assert two(0.1) == 1.0 and two(0.5) == 2.0
    with pytest.raises(ValueError):
        Pulse.from_config(dict(base, equations=[("a", [1.0])], equation_bounds=[0, 0.5, 1]))


def test_pulsatile_schedule_matches_iterate():
    """Step count of the pulsatile stop rule and the Systole/Diastole output
    steps (Simulation.cpp:549-608) for the golden pulsatile case's dt."""
    cfg = {"FlowType": "Pulsatile", "dt": 3e-3, "period": 0.9, "Systole": 0.15, "Diastole": 0.6}
    total, outs = output_schedule(cfg)
    assert total == orc.pulsatile_step_count(3e-3)
    t, want = 0.0, []
    for it in range(total):
        tic = math.fmod(t, 0.9)
        if abs(tic - 0.15) < 1.5e-3:
            want.append(it)
        elif abs(tic - 0.6) < 1.5e-3:
            want.append(it)
        t += 3e-3
    assert [o[0] for o in outs] == want and len(want) == 6
    assert [o[1] for o in outs][:2] == ["Systole_1", "Diastole_1"]
    total, outs = output_schedule({"FlowType": "Constant", "MaxIter": 30001, "IterToWrite": 10000})
    assert total == 30001 and outs == [(10000, "Iteration_10000"), (20000, "Iteration_20000"),
                                       (30000, "Iteration_30000")]


def test_struct_layout_matches_binding(tmp_path):
    """sizeof and field offsets of lbm_config and lbm_pulse_desc as a C
    compiler lays them out, against the ctypes structures."""
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "lbm_b200.h"\n'
        "int main(void) { printf(\"%zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(lbm_config),\n"
        "  offsetof(lbm_config, openings), offsetof(lbm_config, equations), offsetof(lbm_config, flow),\n"
        "  offsetof(lbm_config, equation_bounds), offsetof(lbm_config, harmonic_phases),\n"
        "  sizeof(lbm_pulse_desc)); return 0; }\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    C = capi.LbmConfig
    import ctypes
    assert got == [ctypes.sizeof(C), C.openings.offset, C.equations.offset, C.flow.offset,
                   C.equation_bounds.offset, C.harmonic_phases.offset, ctypes.sizeof(capi.LbmPulseDesc)]
