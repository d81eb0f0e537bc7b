"""Failure detection on the host (no GPU): the inputs where the reference goes
on quietly are refused with a status and a message naming the fault.

* ASCII STL (lbm_stl_read_ascii): the reference's reader skips a facet that
  breaks its grammar, or keeps the previous facet's vertices where a vertex
  line fails (GeometryReader.cpp:88-158), and returns what it has; here a
  truncated file, a malformed line or a file without facets is
  LBM_ERR_ARGUMENT with the file and line.
* config.txt (lbm_config_parse): the reference's parser reads an
  uninitialised coordinate or indexes past a short vector where a block is
  incomplete, and LBM.cpp:94-99 swallows its exceptions; here those blocks are
  errors.
* Both readers, fuzzed with seeded damage (bytes changed, cut, inserted or
  repeated, 1500 files each), either read the file or refuse it with a
  status; neither crashes or fails another way.
"""
import os

import numpy as np
import pytest

from lbm_b200 import capi
from lbm_b200 import config as CF
from lbm_b200 import geometry as G

FACET = ("facet normal 0 0 1\n outer loop\n  vertex 0 0 0\n  vertex 1 0 0\n  vertex 0 1 0\n"
         " endloop\nendfacet\n")


def write(tmp_path, text, name="g.stl"):
    p = tmp_path / name
    p.write_text(text)
    return p


def read_error(path):
    with pytest.raises(capi.LbmError) as ei:
        G.read_stl(path)
    assert ei.value.code == capi.LBM_ERR_ARGUMENT
    return str(ei.value)


def test_well_formed_stl_reads():
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.stl")
        with open(p, "w") as fh:
            fh.write("solid s\n" + FACET + FACET.replace("0 0 1", "0 0 -1") + "endsolid s\n")
        t = G.read_stl(p)
    assert t.shape == (2, 12)
    np.testing.assert_array_equal(t[0], [0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1])
    assert t[1, 11] == -1


def test_truncated_stl_is_refused(tmp_path):
    # ends after the second facet's first vertex
    cut = "solid s\n" + FACET + FACET[: FACET.index("  vertex 1 0 0")]
    msg = read_error(write(tmp_path, cut))
    assert "g.stl:11:" in msg and "ends inside a facet" in msg
    # ends in the middle of a vertex line
    msg = read_error(write(tmp_path, "solid s\n" + FACET[: FACET.index("1 0 0") + 2], "half.stl"))
    assert "half.stl:5:" in msg and "malformed vertex line" in msg


def test_corrupt_vertex_line_is_refused_with_its_line(tmp_path):
    bad = FACET.replace("vertex 1 0 0", "vertex 1 zero 0")
    msg = read_error(write(tmp_path, "solid s\n" + FACET + bad + "endsolid s\n"))
    assert "g.stl:12:" in msg and "malformed vertex line" in msg


def test_missing_endloop_is_refused(tmp_path):
    bad = FACET.replace(" endloop\n", "")
    msg = read_error(write(tmp_path, "solid s\n" + bad))
    assert "expected endloop" in msg


def test_stl_without_facets_is_refused(tmp_path):
    msg = read_error(write(tmp_path, "solid s\nendsolid s\n"))
    assert "no facets" in msg
    read_error(write(tmp_path, "", name="empty.stl"))


def test_missing_stl_is_refused(tmp_path):
    msg = read_error(tmp_path / "nothing.stl")
    assert "cannot open" in msg


def test_config_incomplete_blocks_are_refused(tmp_path):
    from lbm_b200.config import read_config
    base = ("parameters:\n\n  stl_file: \"g.stl\"\n  grid_size: 0.5\n\n\ninlets:\n\n"
            "    plane: z\n    coordinate: 0.0\n    normal: [0, 0, -1]\n\n\noutlets:\n\n"
            "    plane: z\n    coordinate: 8.0\n    normal: [0, 0, 1]\n\n")
    p = write(tmp_path, base, "config.txt")
    cfg = read_config(p)
    assert len(cfg["inlets"]) == 1 and len(cfg["outlets"]) == 1
    for broken in (base.replace("    coordinate: 0.0\n", ""),         # inlet without coordinate
                   base.replace("    normal: [0, 0, 1]\n", ""),        # outlet without normal
                   base.replace("plane: z\n    coordinate: 0.0", "plane: w\n    coordinate: 0.0")):
        write(tmp_path, broken, "config.txt")
        with pytest.raises((capi.LbmError, ValueError)):
            read_config(p)


def mutations(base, rng, n):
    """n damaged copies of base: bytes changed, cut, inserted or repeated."""
    for _ in range(n):
        b = bytearray(base)
        for _ in range(int(rng.integers(1, 4))):
            k = int(rng.integers(5))
            if k == 0 and len(b):
                b[int(rng.integers(len(b)))] = int(rng.integers(256))
            elif k == 1:
                b = b[:int(rng.integers(len(b) + 1))]
            elif k == 2:
                i = int(rng.integers(len(b) + 1))
                b[i:i] = bytes(rng.integers(0, 256, size=int(rng.integers(1, 20)), dtype=np.uint8))
            elif k == 3 and len(b):
                i = int(rng.integers(len(b)))
                b[i:i] = b"\n"
            else:
                i, j = sorted(int(x) for x in rng.integers(len(b) + 1, size=2))
                b[i:j] = b[i:j] * 2
        yield bytes(b)


def test_stl_reader_survives_damaged_files(tmp_path):
    """Seeded fuzzing: every damaged STL reads as facets or is refused with
    LBM_ERR_ARGUMENT; none crashes the reader or fails another way."""
    base = ("solid s\n" + FACET * 3 + "endsolid s\n").encode()
    p = tmp_path / "g.stl"
    refused = 0
    for b in mutations(base, np.random.default_rng(7), 1500):
        p.write_bytes(b)
        try:
            t = G.read_stl(p)
            assert t.ndim == 2 and t.shape[1] == 12 and t.shape[0] >= 1
        except capi.LbmError as e:
            assert e.code == capi.LBM_ERR_ARGUMENT
            refused += 1
    assert refused > 1000


def test_config_parser_survives_damaged_files(tmp_path):
    """Seeded fuzzing of lbm_config_parse through read_config: every damaged
    config.txt parses or is refused with a status; none crashes the parser
    or fails another way (string fields keep bytes that are not UTF-8, as
    the reference's std::string does)."""
    from test_config import FULL
    p = tmp_path / "config.txt"
    refused = parsed = 0
    for b in mutations(FULL.encode(), np.random.default_rng(11), 1500):
        p.write_bytes(b)
        try:
            cfg = CF.read_config(p)
            assert isinstance(cfg, dict)
            parsed += 1
        except capi.LbmError:
            refused += 1
    assert refused > 300 and parsed > 300
