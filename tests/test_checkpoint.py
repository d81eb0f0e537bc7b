"""Checkpoint files on the CPU: the format round-trips, and every kind of
damage is refused with CheckpointError before anything reaches an engine.
The damage covered: a flipped bit (CRC-32), truncation, a foreign file, another
format version, trailing bytes, a missing array. Also checked: a checkpoint is
refused by an engine unlike its writer, and restore() hands the engine the
state blob. A stand-in records the calls; no GPU is used."""
import json
import types
import zlib

import numpy as np
import pytest

from lbm_b200 import checkpoint as C


def sample(seed=0, n=50, q=19, m=7):
    r = np.random.default_rng(seed)
    meta = {"kind": "engine", "n_nodes": n, "lattice": q, "n_nearwall": m, "storage": "f32", "bc": "physics",
            "steps": 1234, "runtime": 0.01234}
    return meta, {"state": r.integers(0, 256, size=5000, dtype=np.uint8)}


def test_round_trip(tmp_path):
    meta, arrays = sample()
    p = str(tmp_path / "a.ckpt")
    C.write(p, meta, arrays)
    got = C.read(p)
    assert got["meta"] == meta
    for k, v in arrays.items():
        np.testing.assert_array_equal(got["arrays"][k], v)


def damaged(tmp_path, edit):
    meta, arrays = sample()
    p = str(tmp_path / "a.ckpt")
    C.write(p, meta, arrays)
    raw = bytearray(open(p, "rb").read())
    raw = edit(raw)
    open(p, "wb").write(bytes(raw))
    return p


def header_len(raw):
    return C.PREFIX.unpack_from(raw, len(C.MAGIC))[0]


HEADER_START = len(C.MAGIC) + C.PREFIX.size


@pytest.mark.parametrize("where", [0.1, 0.5, 0.99])
def test_flipped_bit_is_a_crc_mismatch(tmp_path, where):
    def edit(raw):
        base = HEADER_START + header_len(raw)
        i = base + int(where * (len(raw) - base - 1))
        raw[i] ^= 0x10
        return raw
    with pytest.raises(C.CheckpointError, match="CRC-32 mismatch"):
        C.read(damaged(tmp_path, edit))


def test_truncated_file(tmp_path):
    with pytest.raises(C.CheckpointError, match="truncated"):
        C.read(damaged(tmp_path, lambda raw: raw[:-9]))
    with pytest.raises(C.CheckpointError, match="truncated header"):
        C.read(damaged(tmp_path, lambda raw: raw[:HEADER_START + 5]))
    with pytest.raises(C.CheckpointError, match="bad magic"):
        C.read(damaged(tmp_path, lambda raw: raw[:5]))


def test_foreign_file_and_trailing_bytes(tmp_path):
    with pytest.raises(C.CheckpointError, match="bad magic"):
        C.read(damaged(tmp_path, lambda raw: b"NOTACKPT" + raw[8:]))
    with pytest.raises(C.CheckpointError, match="after the last array"):
        C.read(damaged(tmp_path, lambda raw: raw + b"\0\0\0"))


def rewrite_header(tmp_path, change):
    """A file whose header is changed and re-checksummed: what only the
    content checks can catch."""
    def edit(raw):
        h = header_len(raw)
        header = json.loads(bytes(raw[HEADER_START:HEADER_START + h]).decode())
        change(header)
        new = json.dumps(header).encode()
        return raw[:len(C.MAGIC)] + C.PREFIX.pack(len(new), zlib.crc32(new)) + new + raw[HEADER_START + h:]
    return damaged(tmp_path, edit)


def test_header_is_checksummed(tmp_path):
    def edit(raw):
        i = HEADER_START + header_len(raw) // 2
        raw[i] ^= 0x01
        return raw
    with pytest.raises(C.CheckpointError, match="CRC-32 mismatch in the header"):
        C.read(damaged(tmp_path, edit))


def test_other_version_and_missing_array(tmp_path):
    with pytest.raises(C.CheckpointError, match="format version"):
        C.read(rewrite_header(tmp_path, lambda h: h.update(version=99)))
    with pytest.raises(C.CheckpointError, match="without meta or arrays"):
        C.read(rewrite_header(tmp_path, lambda h: h["arrays"].pop("state")))
    with pytest.raises(C.CheckpointError, match="array state missing"):
        C.read(rewrite_header(tmp_path, lambda h: h["arrays"].update(other=h["arrays"].pop("state"))))
    with pytest.raises(C.CheckpointError, match="inconsistent"):
        C.read(rewrite_header(tmp_path, lambda h: h["arrays"]["state"].update(shape=[5001])))
    with pytest.raises(C.CheckpointError, match="inconsistent"):
        C.read(rewrite_header(tmp_path, lambda h: h["arrays"]["state"].update(dtype="<f8")))


class StandIn:
    """Records what restore() hands the engine."""

    def __init__(self, n=50, q=19, m=7, storage="f32", bc="physics"):
        self.n, self.q, self.n_nearwall, self.storage, self.bc = n, q, m, storage, bc
        self.calls = []

    def set_state(self, blob):
        self.calls.append(("set_state", blob.dtype.str, blob.shape))


def test_restore_hands_over_the_state_and_checks_the_engine(tmp_path):
    meta, arrays = sample()
    p = str(tmp_path / "a.ckpt")
    C.write(p, meta, arrays)
    ck = C.read(p)
    e = StandIn()
    C.restore(e, ck)
    assert e.calls == [("set_state", "|u1", (5000,))]
    for bad in (StandIn(storage="f16"), StandIn(bc="reference"), StandIn(n=51), StandIn(q=27), StandIn(m=8)):
        with pytest.raises(C.CheckpointError):
            C.restore(bad, ck)
        assert bad.calls == []


def test_state_of_reads_meta_and_blob():
    fake = types.SimpleNamespace(
        n=4, q=19, n_nearwall=3, storage="f64", bc="reference",
        time=lambda: (7, 0.5), get_state=lambda: np.arange(10, dtype=np.uint8))
    meta, arrays = C.state_of(fake)
    assert meta == {"kind": "engine", "n_nodes": 4, "lattice": 19, "n_nearwall": 3, "storage": "f64",
                    "bc": "reference", "steps": 7, "runtime": 0.5}
    assert list(arrays) == ["state"]
    np.testing.assert_array_equal(arrays["state"], np.arange(10, dtype=np.uint8))


def test_only_byte_arrays_are_written(tmp_path):
    meta, _ = sample()
    with pytest.raises(C.CheckpointError, match="only"):
        C.write(str(tmp_path / "a.ckpt"), meta, {"state": np.zeros(3)})


def test_unknown_kind_and_overlapping_arrays(tmp_path):
    with pytest.raises(C.CheckpointError, match="unknown kind"):
        C.read(rewrite_header(tmp_path, lambda h: h["meta"].update(kind="something")))

    def two_arrays(h):
        # a second array claiming the first one's bytes
        h["arrays"]["extra"] = dict(h["arrays"]["state"])
    with pytest.raises(C.CheckpointError, match="does not start"):
        C.read(rewrite_header(tmp_path, two_arrays))


class SlabEngine(StandIn):
    def __init__(self, n, blob_len):
        super().__init__(n=n)
        self.blob_len = blob_len

    def time(self):
        return (40, 0.0)

    def get_state(self):
        return np.full(self.blob_len, self.n % 251, dtype=np.uint8)


def test_slab_set_round_trip_and_checks(tmp_path):
    eng = [SlabEngine(30, 100), SlabEngine(25, 90), SlabEngine(28, 96)]
    ss = types.SimpleNamespace(engines=eng, n=80, q=19)
    meta, arrays = C.slab_set_state(ss)
    assert meta["kind"] == "slab_set" and meta["n_slabs"] == 3 and meta["slab_nodes"] == [30, 25, 28]
    p = str(tmp_path / "s.ckpt")
    C.write(p, meta, arrays)
    ck = C.read(p)
    fresh = [SlabEngine(30, 100), SlabEngine(25, 90), SlabEngine(28, 96)]
    C.restore_slab_set(types.SimpleNamespace(engines=fresh, n=80, q=19), ck)
    assert [e.calls for e in fresh] == [[("set_state", "|u1", (100,))], [("set_state", "|u1", (90,))],
                                        [("set_state", "|u1", (96,))]]
    # another cut of the lattice is refused before any engine is touched
    other = [SlabEngine(30, 100), SlabEngine(26, 90), SlabEngine(27, 96)]
    with pytest.raises(C.CheckpointError, match="slab_nodes"):
        C.restore_slab_set(types.SimpleNamespace(engines=other, n=80, q=19), ck)
    assert all(e.calls == [] for e in other)
    # an engine checkpoint is not a slab-set checkpoint, nor the other way round
    with pytest.raises(C.CheckpointError, match="kind"):
        C.restore(StandIn(), ck)
    with pytest.raises(C.CheckpointError, match="array state_2 missing"):
        C.read(rewrite_slab_header(tmp_path, ss))


def rewrite_slab_header(tmp_path, ss):
    meta, arrays = C.slab_set_state(ss)
    arrays.pop("state_2")
    p = str(tmp_path / "short.ckpt")
    C.write(p, meta, arrays)
    return p



def test_any_corruption_is_refused_or_harmless(tmp_path):
    """Seeded fuzzing of the reader: whatever bytes change, go missing or get
    inserted, read() raises CheckpointError or returns exactly the content
    written (a change that JSON ignores, such as one kind of whitespace for
    another). It never fails another way."""
    meta, arrays = sample(n=20, m=3)
    p = str(tmp_path / "a.ckpt")
    C.write(p, meta, arrays)
    good = open(p, "rb").read()
    rng = np.random.default_rng(2024)
    outcomes = {"refused": 0, "same": 0}
    for trial in range(400):
        raw = bytearray(good)
        kind = trial % 4
        if kind == 0:      # flip one byte anywhere
            i = int(rng.integers(len(raw)))
            raw[i] ^= int(rng.integers(1, 256))
        elif kind == 1:    # flip one byte of the header
            i = int(rng.integers(len(C.MAGIC), HEADER_START + header_len(good)))
            raw[i] ^= int(rng.integers(1, 256))
        elif kind == 2:    # cut the file short
            raw = raw[:int(rng.integers(len(raw)))]
        else:              # insert bytes
            i = int(rng.integers(len(raw) + 1))
            raw[i:i] = bytes(rng.integers(0, 256, size=int(rng.integers(1, 9)), dtype=np.uint8))
        q = str(tmp_path / "b.ckpt")
        open(q, "wb").write(bytes(raw))
        try:
            got = C.read(q)
        except C.CheckpointError:
            outcomes["refused"] += 1
            continue
        assert got["meta"] == meta
        np.testing.assert_array_equal(got["arrays"]["state"], arrays["state"])
        outcomes["same"] += 1
    assert outcomes["refused"] > 300


def test_hostile_shapes_are_refused(tmp_path):
    for shape in ([-5000, -1], [2 ** 40, 2 ** 40], [5000, 0]):
        with pytest.raises(C.CheckpointError, match="inconsistent"):
            C.read(rewrite_header(tmp_path, lambda h: h["arrays"]["state"].update(shape=shape)))
