"""Generates the golden fixtures in tests/golden/ by running the reference solver.

Each case writes a synthetic ASCII STL cylinder and a config.txt into a scratch
directory, runs the reference harness (oracle/_ref/refharness, built by
``make -C oracle`` from the reference sources) and keeps a compact .npz of its
dumps: the node map the reference built (coordinates, node kinds, inlet /
outlet / wall / near-wall lists, near-wall normals) and its state after the
phases of step 1 and after the last step.

The fixtures are the pins of the oracle restatement (oracle/lbm_oracle.c):
tests/test_oracle.py replays every case through the oracle and requires
bit-for-bit agreement with these dumps.

Run from the repository root (needs the reference tree, this container only):
    python tests/golden/make_golden.py            # all small cases
    python tests/golden/make_golden.py pipe16     # the R=16, L=128 pipe, 2000 steps

STL conventions (the reference voxeliser's rules, ComplexGeometry.cpp:265-310,
440-514): facet normals point outwards and are written to the file; the axis
sits off the lattice (centre offset 0.37, 0.21) and the ring is rotated by half
a facet, so no +z ray runs along a shared cap edge, which the inclusive
point-in-triangle test would count twice.
"""
from __future__ import annotations

import math
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "refharness")


# ---------------------------------------------------------------- geometry ---
def cylinder_triangles(radius, length, n_az, n_ax, centre=(0.37, 0.21)):
    """Closed cylinder along +z from z=0 to z=length: side quads split in two,
    fan-triangulated caps. Returns a list of (normal, v1, v2, v3)."""
    cx, cy = centre
    ring = []
    for a in range(n_az):
        th = 2.0 * math.pi * (a + 0.5) / n_az
        ring.append((cx + radius * math.cos(th), cy + radius * math.sin(th)))
    tris = []
    for s in range(n_ax):
        z0 = length * s / n_ax
        z1 = length * (s + 1) / n_ax
        for a in range(n_az):
            p0 = ring[a]
            p1 = ring[(a + 1) % n_az]
            mx, my = (p0[0] + p1[0]) / 2 - cx, (p0[1] + p1[1]) / 2 - cy
            nrm = math.hypot(mx, my)
            n = (mx / nrm, my / nrm, 0.0)
            v00 = (p0[0], p0[1], z0)
            v10 = (p1[0], p1[1], z0)
            v01 = (p0[0], p0[1], z1)
            v11 = (p1[0], p1[1], z1)
            tris.append((n, v00, v10, v11))
            tris.append((n, v00, v11, v01))
    for a in range(n_az):
        p0 = ring[a]
        p1 = ring[(a + 1) % n_az]
        tris.append(((0.0, 0.0, -1.0), (cx, cy, 0.0), (p1[0], p1[1], 0.0), (p0[0], p0[1], 0.0)))
        tris.append(((0.0, 0.0, 1.0), (cx, cy, length), (p0[0], p0[1], length),
                     (p1[0], p1[1], length)))
    return tris


def permute(tris, axis):
    """Rotate a z-axis cylinder so its axis is `axis` ('x', 'y' or 'z')."""
    if axis == "z":
        return tris
    # cyclic permutations keep the orientation (outward normals stay outward)
    perm = {"x": lambda p: (p[2], p[0], p[1]), "y": lambda p: (p[1], p[2], p[0])}[axis]
    return [tuple(perm(v) for v in t) for t in tris]


def write_stl(path, tris):
    with open(path, "w") as fh:
        fh.write("solid cylinder\n")
        for n, a, b, c in tris:
            fh.write("facet normal %.17g %.17g %.17g\n" % n)
            fh.write("outer loop\n")
            for v in (a, b, c):
                fh.write("vertex %.17g %.17g %.17g\n" % v)
            fh.write("endloop\nendfacet\n")
        fh.write("endsolid cylinder\n")


def write_config(path, *, flow="Constant", dt=1e-5, tau=0.8, grid_size=0.5, vel=0.05,
                 max_iter=100, iter_to_write=1000000, inlet, outlets):
    lines = ["parameters:", "", '  stl_file: "geom.stl"', '  FlowType: "%s"' % flow,
             "  time_resolution: %r" % dt, "  density: 1060", "  kinematic_viscosity: 3.5e-6",
             "  relaxation_factor: %r" % tau, "  grid_size: %r" % grid_size, "  pressure: 1",
             "  CteVel: %r" % vel, "  reynolds_number: 100",
             "  number_of_outlets: %d" % len(outlets), "  MaxIter: %d" % max_iter,
             "  IterToWrite: %d" % iter_to_write, "  Systole: 0.15", "  Diastole: 0.9", "  period: 0.9",
             "  NumCycle: 1", "", ""]

    def block(b):
        out = ["    plane: %s" % b["plane"], "    coordinate: %r" % b["coordinate"]]
        for k in ("range_x", "range_y", "range_z"):
            if k in b:
                out.append("    %s: [%r, %r]" % (k, b[k][0], b[k][1]))
        out.append("    normal: [%r, %r, %r]" % tuple(b["normal"]))
        return out + [""]

    lines += ["inlets:", ""] + block(inlet) + [""]
    lines += ["outlets:", ""]
    for o in outlets:
        lines += block(o)
    lines += ["", "equations:", "    InletVel1: [0]", ""]
    with open(path, "w") as fh:
        fh.write("\n".join(lines))


# -------------------------------------------------------------- dump reader ---
_DT = {b"d": np.float64, b"i": np.int32, b"q": np.int64, b"b": np.uint8}


def read_dump(path):
    """Reads the harness's record file into a dict of numpy arrays."""
    out = {}
    with open(path, "rb") as fh:
        buf = fh.read()
    pos = 0
    while pos < len(buf):
        (n,) = np.frombuffer(buf, np.uint32, 1, pos)
        pos += 4
        name = buf[pos:pos + n].decode()
        pos += n
        dt = _DT[buf[pos:pos + 1]]
        pos += 1
        (nd,) = np.frombuffer(buf, np.uint32, 1, pos)
        pos += 4
        dims = tuple(int(d) for d in np.frombuffer(buf, np.uint64, nd, pos))
        pos += 8 * nd
        cnt = int(np.prod(dims)) if dims else 1
        arr = np.frombuffer(buf, dt, cnt, pos).reshape(dims).copy()
        pos += cnt * arr.itemsize
        out[name] = arr
    return out


# -------------------------------------------------------------------- cases ---
def _ends(axis, length):
    lo = {"plane": axis, "coordinate": 0.0}
    hi = {"plane": axis, "coordinate": float(length)}
    return lo, hi


def _unit(axis, sign):
    v = [0.0, 0.0, 0.0]
    v["xyz".index(axis)] = float(sign)
    return v


def small_cases():
    """Small cylinders (radius 4, length 16) covering every inlet and outlet
    branch of the reference (Boundary.cpp:115-288, Simulation.cpp:655-739)."""
    # 7 axial segments: segment ends fall between lattice planes, so +z rays of
    # x- and y-axis cylinders never run along a shared side edge.
    R, L, NAZ, NAX = 4.0, 16.0, 16, 7
    cases = []

    def case(name, axis, inlet_at_lo, steps, **kw):
        lo, hi = _ends(axis, L)
        inl, outl = (lo, hi) if inlet_at_lo else (hi, lo)
        inl = dict(inl, normal=_unit(axis, -1 if inlet_at_lo else 1))
        outl = dict(outl, normal=_unit(axis, 1 if inlet_at_lo else -1))
        outlets = kw.pop("outlets", [outl])
        cases.append(dict(name=name, axis=axis, R=R, L=L, naz=NAZ, nax=NAX, steps=steps,
                          inlet=inl, outlets=outlets, **kw))

    case("cyl_z", "z", True, 60)
    case("cyl_z_rev", "z", False, 20)
    case("cyl_x", "x", True, 40)
    case("cyl_x_rev", "x", False, 20)
    case("cyl_y", "y", True, 4)
    case("cyl_y_rev", "y", False, 4)
    # dt 3e-3 over 100 steps spans all three waveform pieces (t < 0.09,
    # 0.09 <= t < 0.27, t >= 0.27; Simulation.cpp:523-531).
    case("cyl_z_pulsatile", "z", True, 100, flow="Pulsatile", dt=3e-3)
    # two outlets on one plane whose normals point along the plane: each outlet
    # node copies from a neighbour in the same plane, so the reference's
    # in-order sweep chains copies (x+ side) or reads values not yet copied
    # (x- side). The x ranges stop one plane short of the box faces: the
    # reference indexes the inward neighbour without a bounds check
    # (Simulation.cpp:663,677), so a node on the face would read outside the
    # lattice.
    cx = 0.37
    case("outlet_chain", "z", True, 12, outlets=[
        {"plane": "z", "coordinate": L, "range_x": [-3.0, cx], "normal": [1.0, 0.0, 0.0]},
        {"plane": "z", "coordinate": L, "range_x": [cx, 3.9], "normal": [-1.0, 0.0, 0.0]},
        {"plane": "z", "coordinate": L, "normal": [0.0, 0.0, 1.0]},
    ])
    return cases


def pipe16_case():
    """The R=16 lu, L=128 lu pipe with 64 x 32 facets on the reference grid
    (grid_size 0.5 -> spacing 1), tau 0.8, plug inlet 0.05, 2000 steps."""
    return dict(name="pipe16", axis="z", R=16.0, L=128.0, naz=64, nax=32, steps=2000,
                inlet={"plane": "z", "coordinate": 0.0, "normal": [0.0, 0.0, -1.0]},
                outlets=[{"plane": "z", "coordinate": 128.0, "normal": [0.0, 0.0, 1.0]}])


TOPO_KEYS = ("meta_i", "meta_d", "coords", "kind", "inlet", "inlet_normal", "wall",
             "nearwall", "nearwall_normal")


def run_case(c, workdir, phases=True):
    tris = permute(cylinder_triangles(c["R"], c["L"], c["naz"], c["nax"]), c["axis"])
    write_stl(os.path.join(workdir, "geom.stl"), tris)
    write_config(os.path.join(workdir, "config.txt"), flow=c.get("flow", "Constant"),
                 dt=c.get("dt", 1e-5), inlet=c["inlet"], outlets=c["outlets"])
    dump = os.path.join(workdir, "dump.bin")
    cmd = [HARNESS, "stl", os.path.join(workdir, "config.txt"), str(c["steps"]), dump]
    if phases:
        cmd.append("--phases")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    return read_dump(dump)


def keep_small(d):
    """Everything: topology, the step-1 phase states and the final state."""
    out = {}
    for k, v in d.items():
        if k.startswith("init/"):
            continue
        out[k.replace("/", "__")] = v
    return out


def keep_pipe(d, n_sample=4096, seed=1234):
    """Topology plus a seeded node sample of the final state, full near-wall
    fields (WSS and its accumulators) and whole-field checksums."""
    out = {k.replace("/", "__"): d[k] for k in d if k in TOPO_KEYS or k.startswith("outlet_")}
    N = int(d["meta_i"][0])
    rng = np.random.default_rng(seed)
    sample = np.sort(rng.choice(N, size=min(n_sample, N), replace=False))
    out["sample"] = sample.astype(np.int64)
    for k in ("f", "rho", "u"):
        out["final__%s_sample" % k] = d["final/" + k][sample]
    for k in ("wss", "acc", "accmag"):
        out["final__" + k] = d["final/" + k]
    for k in ("f", "rho", "u", "feq"):
        a = d["final/" + k]
        out["final__%s_sum" % k] = np.array([a.sum(), np.abs(a).sum(), (a * a).sum()])
    out["coords"] = d["coords"].astype(np.int16)
    return out


def main(argv):
    if not os.path.exists(HARNESS):
        sys.exit("build the reference harness first: make -C oracle")
    which = argv[1:] or ["small"]
    with tempfile.TemporaryDirectory() as tmp:
        if "small" in which:
            for c in small_cases():
                wd = os.path.join(tmp, c["name"])
                os.makedirs(wd)
                d = run_case(c, wd)
                assert int(d["meta_i"][6]) == 0, "fluid node with an uninitialised Wall tag"
                np.savez_compressed(os.path.join(HERE, c["name"] + ".npz"), **keep_small(d))
                print(c["name"], "nodes", int(d["meta_i"][0]), "nearwall", len(d["nearwall"]))
        if "pipe16" in which:
            c = pipe16_case()
            wd = os.path.join(tmp, c["name"])
            os.makedirs(wd)
            d = run_case(c, wd, phases=False)
            assert int(d["meta_i"][6]) == 0, "fluid node with an uninitialised Wall tag"
            np.savez_compressed(os.path.join(HERE, "pipe16_2000.npz"), **keep_pipe(d))
            print(c["name"], "nodes", int(d["meta_i"][0]), "nearwall", len(d["nearwall"]))


if __name__ == "__main__":
    main(sys.argv)
