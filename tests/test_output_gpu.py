"""Result files (lbm_write_surface_csv, lbm_smooth_surface_csv, lbm_write_vtu)
against restatements of the reference's writers on the golden cases' state.

* The surface CSV after the pulsatile cylinder's 100 steps must equal, line for
  line, the reference's WriteSurfaceAttribute text (OutputFile.cpp:234-316:
  header, near-wall order, ostream default number format = printf "%g") of
  the reference's own final WSS, OSI, TAWSS and |u|; constant flow writes the
  five-column form.
* Smoothing must equal OutputFile::processFlowData (:395-483) restated as its
  all-pairs loop, at radii that give every row 0, axis-only and diagonal
  neighbours.
* The VTU must hold the reference's point order (z, then y, x fastest),
  fields, and hexahedra (WriteVTK_Collective, :60-230).
"""
import os
import re
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from lbm_b200 import Engine
from lbm_b200.engine import smooth_surface_csv

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STEPS = {"cyl_z": 60, "cyl_z_pulsatile": 100}


def run(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: d[k] for k in d.files}
    meta = d["meta_d"]
    e = Engine(d, tau=meta[0], dt=meta[1], spacing=meta[2], storage="f64")
    e.set_flow(bool(d["meta_i"][7]), float(meta[4]))
    e.step(STEPS[name])
    return d, e


def g(x):
    """std::ostream << double with default flags: printf %g, 6 digits."""
    return "%g" % x


def reference_csv(d, origin, spacing, pulsatile):
    lines = ["X,Y,Z,WSS" + (",OSI,TAWSS" if pulsatile else "") + ",VelMag"]
    for k, n in enumerate(d["nearwall"]):
        x, y, z = (origin[a] + float(d["coords"][n, a]) * spacing for a in range(3))
        cols = [x, y, z, d["final__wss"][k]]
        if pulsatile:
            cols += [d["final__osi"][k], d["final__tawss"][k]]
        cols.append(d["final__velmag"][n])
        lines.append(",".join(g(v) for v in cols))
    return "\n".join(lines) + "\n"


def reference_smooth(text, radius, pulsatile):
    """processFlowData + smoothData + calculateMeanNeighboringValues: every row
    against every row, sums in file order."""
    lines = text.splitlines()
    rows = np.array([[float(t) for t in ln.split(",")] for ln in lines[1:]])
    xyz = rows[:, :3]
    attrs = [3, 4, 5] if pulsatile else [3]
    out = rows.copy()
    for i in range(len(rows)):
        dd = xyz - xyz[i]
        dist = np.sqrt(dd[:, 0] * dd[:, 0] + dd[:, 1] * dd[:, 1] + dd[:, 2] * dd[:, 2])
        nb = np.nonzero((dist > 0) & (dist <= radius))[0]
        for a in attrs:
            if len(nb):
                s = 0.0
                for j in nb:
                    s += rows[j, a]
                out[i, a] = s / len(nb)
    res = [lines[0]]
    for r in out:
        res.append(",".join(g(v) for v in r))
    return "\n".join(res) + "\n", rows


@pytest.mark.parametrize("name", ["cyl_z_pulsatile", "cyl_z"])
def test_surface_csv_matches_reference_text(name, tmp_path):
    d, e = run(name)
    pulsatile = bool(d["meta_i"][7])
    origin, spacing = (-3.55314112, -3.71314112, 0.125), 0.5
    path = tmp_path / "100_FlowHemodynamics.csv"
    e.write_surface_csv(path, origin, spacing, pulsatile)
    got = path.read_text()
    assert got == reference_csv(d, origin, spacing, pulsatile)
    assert len(got.splitlines()) == len(d["nearwall"]) + 1


@pytest.mark.parametrize("radius", [0.1, 0.25, 0.45, 1.1])
def test_smoothing_matches_all_pairs_loop(radius, tmp_path):
    d, e = run("cyl_z_pulsatile")
    src = tmp_path / "in.csv"
    # spacing 0.2: 0.25 reaches axis neighbours, 0.45 the diagonals, 1.1 many
    e.write_surface_csv(src, (0.1, -2.3, 5.7), 0.2, True)
    dst = tmp_path / "FlowHemodynamics" / "out.csv"
    dst.parent.mkdir()
    smooth_surface_csv(src, dst, radius=radius, pulsatile=True)
    want, rows = reference_smooth(src.read_text(), radius, True)
    assert dst.read_text() == want
    if radius > 0.2:
        assert dst.read_text() != src.read_text()


def test_smoothing_constant_flow_and_bad_rows(tmp_path):
    d, e = run("cyl_z")
    src = tmp_path / "in.csv"
    e.write_surface_csv(src, (0.0, 0.0, 0.0), 0.2, False)
    text = src.read_text()
    lines = text.splitlines()
    # a row that does not parse is dropped, as the reference's try/catch does
    damaged = "\n".join(lines[:3] + ["x,y,z,w,v"] + lines[3:]) + "\n"
    src.write_text(damaged)
    dst = tmp_path / "out.csv"
    smooth_surface_csv(src, dst, radius=0.25, pulsatile=False)
    want, _ = reference_smooth(text, 0.25, False)
    assert dst.read_text() == want


def parse_vtu(path):
    raw = path.read_bytes()
    head, _, tail = raw.partition(b"<AppendedData encoding=\"raw\">")
    start = tail.index(b"_") + 1
    blob = tail[start:]
    root = ET.fromstring(head.decode() + "</VTKFile>")
    piece = root.find("UnstructuredGrid/Piece")
    types = {"Float64": np.float64, "Float32": np.float32, "Int64": np.int64, "UInt8": np.uint8}
    arrays = {}
    for da in root.iter("DataArray"):
        off = int(da.get("offset"))
        nbytes = int(np.frombuffer(blob[off:off + 8], dtype=np.uint64)[0])
        a = np.frombuffer(blob[off + 8:off + 8 + nbytes], dtype=types[da.get("type")])
        nc = int(da.get("NumberOfComponents", "1"))
        arrays[da.get("Name")] = a.reshape(-1, nc) if nc > 1 else a
    return int(piece.get("NumberOfPoints")), int(piece.get("NumberOfCells")), arrays


def test_vtu_matches_reference_layout(tmp_path):
    d, e = run("cyl_z")
    c = d["coords"].astype(np.int64)
    cells = (int(c[:, 0].max()) + 1, int(c[:, 1].max()) + 1, int(c[:, 2].max()))
    path = tmp_path / "0.vtu"
    e.write_vtu(path, cells)
    npts, ncells, arr = parse_vtu(path)
    order = np.lexsort((c[:, 0], c[:, 1], c[:, 2]))
    assert npts == len(c)
    np.testing.assert_array_equal(arr["Points"], c[order].astype(np.float32))
    np.testing.assert_array_equal(arr["Velocity"], d["final__u"][order])
    np.testing.assert_array_equal(arr["Density"], d["final__rho"][order])
    u = d["final__u"][order]
    np.testing.assert_array_equal(arr["VelocityMagnitude"],
                                  np.sqrt(u[:, 0] * u[:, 0] + u[:, 1] * u[:, 1] + u[:, 2] * u[:, 2]))
    # hexahedra of the reference loop (z, y, x; corners in VTK_HEXAHEDRON order)
    pid = {tuple(p): i for i, p in enumerate(c[order])}
    want = []
    for z in range(cells[2] - 1):
        for y in range(cells[1] - 1):
            for x in range(cells[0] - 1):
                ids = [pid.get(k) for k in ((x, y, z), (x + 1, y, z), (x + 1, y + 1, z), (x, y + 1, z),
                                            (x, y, z + 1), (x + 1, y, z + 1), (x + 1, y + 1, z + 1),
                                            (x, y + 1, z + 1))]
                if None not in ids:
                    want.extend(ids)
    assert ncells == len(want) // 8 and ncells > 0
    np.testing.assert_array_equal(arr["connectivity"], np.array(want, dtype=np.int64))
    np.testing.assert_array_equal(arr["offsets"], 8 * np.arange(1, ncells + 1))
    assert np.all(arr["types"] == 12)
    assert re.search(rb"</AppendedData>\n</VTKFile>\n$", path.read_bytes())
