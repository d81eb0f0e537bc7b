"""Checkpoint files: stop a run and resume it bit for bit.

The reference writes no restart files; its only outputs are the result files
of Simulation::WriteOutput (Simulation.cpp:835-856). A checkpoint here holds
the engine's state blob (lbm_get_state): the stored populations in the storage
type, the near-wall moments the next wall shear stress uses, the WSS with its
FP64 accumulators, the step count, the flow clock and the AA phase. FP64
populations would not do for the 16-bit and FP32 storage types: f = w + d
rounds away low bits of small deviations d, and a run restarted from them
drifts in the last bit. The flow settings (waveform, inlet profile, outlet
density) are the caller's, as at the start of a run. To resume, build an
engine from the same topology with the same settings, then call restore():
the steps taken from there equal those of the run that was never stopped.

File layout, all little-endian:
* the 8-byte magic b"LBMCKPT1";
* the header length as a uint64;
* a JSON header: format version, engine settings, step count and clock, and
  per array its dtype, shape, byte offset, length and CRC-32;
* the arrays' raw bytes.
read() checks the magic, the header, and every array's length and CRC-32. It
raises CheckpointError naming the first thing that is wrong, before anything
reaches an engine.
"""
from __future__ import annotations

import json
import os
import struct
import zlib

import numpy as np

MAGIC = b"LBMCKPT1"
VERSION = 1
ARRAYS = ("state",)
DTYPES = {"|u1": 1}


class CheckpointError(ValueError):
    """A checkpoint file that cannot be used: damaged, truncated, of another
    format version, or written by an engine unlike the one restoring it."""


def state_of(engine):
    """(meta, arrays) of an engine's current state."""
    steps, runtime = engine.time()
    meta = {"n_nodes": int(engine.n), "lattice": int(engine.q), "n_nearwall": int(engine.n_nearwall),
            "storage": engine.storage, "bc": engine.bc, "steps": int(steps), "runtime": float(runtime)}
    return meta, {"state": engine.get_state()}


def write(path, meta, arrays):
    """Writes meta and the arrays to path (through a temporary file that
    replaces path once complete)."""
    entries, blobs, offset = {}, [], 0
    for name in ARRAYS:
        a = np.ascontiguousarray(arrays[name])
        dt = a.dtype.str
        if dt not in DTYPES:
            raise CheckpointError("array %s of type %s: only %s are written" % (name, dt, sorted(DTYPES)))
        b = a.tobytes()
        entries[name] = {"dtype": dt, "shape": list(a.shape), "offset": offset, "nbytes": len(b),
                         "crc32": zlib.crc32(b)}
        blobs.append(b)
        offset += len(b)
    header = json.dumps({"version": VERSION, "meta": meta, "arrays": entries}, sort_keys=True).encode()
    tmp = path + ".tmp"
    with open(tmp, "wb") as fh:
        fh.write(MAGIC)
        fh.write(struct.pack("<Q", len(header)))
        fh.write(header)
        for b in blobs:
            fh.write(b)
        fh.flush()
        os.fsync(fh.fileno())
    os.replace(tmp, path)


def save(engine, path):
    meta, arrays = state_of(engine)
    write(path, meta, arrays)


def read(path):
    """{"meta": ..., "arrays": ...} of a checkpoint file, every array checked."""
    with open(path, "rb") as fh:
        data = fh.read()
    start = len(MAGIC) + 8
    if len(data) < start or data[: len(MAGIC)] != MAGIC:
        raise CheckpointError("%s: not a checkpoint file (bad magic)" % path)
    (hlen,) = struct.unpack_from("<Q", data, len(MAGIC))
    if start + hlen > len(data):
        raise CheckpointError("%s: truncated header" % path)
    try:
        header = json.loads(data[start:start + hlen].decode())
    except (UnicodeDecodeError, ValueError) as exc:
        raise CheckpointError("%s: unreadable header (%s)" % (path, exc)) from None
    if not isinstance(header, dict) or header.get("version") != VERSION:
        raise CheckpointError("%s: format version %r, this reader takes %d"
                              % (path, header.get("version") if isinstance(header, dict) else None, VERSION))
    meta, entries = header.get("meta"), header.get("arrays")
    if not isinstance(meta, dict) or not isinstance(entries, dict):
        raise CheckpointError("%s: header without meta or arrays" % path)
    base, end, arrays = start + hlen, start + hlen, {}
    for name in ARRAYS:
        e = entries.get(name)
        if not isinstance(e, dict):
            raise CheckpointError("%s: array %s missing" % (path, name))
        try:
            lo, n, shape, crc = base + int(e["offset"]), int(e["nbytes"]), [int(x) for x in e["shape"]], int(e["crc32"])
        except (KeyError, TypeError, ValueError):
            raise CheckpointError("%s: bad entry for array %s" % (path, name)) from None
        dt = e.get("dtype")
        if dt not in DTYPES or n != DTYPES[dt] * int(np.prod(shape)) or lo < base:
            raise CheckpointError("%s: array %s: shape, type or offset inconsistent" % (path, name))
        if lo + n > len(data):
            raise CheckpointError("%s: truncated in array %s" % (path, name))
        b = data[lo:lo + n]
        if zlib.crc32(b) != crc:
            raise CheckpointError("%s: CRC-32 mismatch in array %s" % (path, name))
        arrays[name] = np.frombuffer(b, dtype=dt).reshape(shape).copy()
        end = max(end, lo + n)
    if end != len(data):
        raise CheckpointError("%s: %d bytes after the last array" % (path, len(data) - end))
    return {"meta": meta, "arrays": arrays}


def check_compatible(engine, meta):
    """Raises CheckpointError unless engine matches the one that wrote meta."""
    mine = {"n_nodes": engine.n, "lattice": engine.q, "n_nearwall": engine.n_nearwall,
            "storage": engine.storage, "bc": engine.bc}
    for k, v in mine.items():
        if meta.get(k) != v:
            raise CheckpointError("checkpoint %s is %r, the engine's %r" % (k, meta.get(k), v))


def restore(engine, ckpt):
    """Puts a checkpoint's state into engine, which must be like the writer's
    (same topology, lattice, storage type and boundary mode) and carry the
    run's flow settings."""
    meta, arrays = ckpt["meta"], ckpt["arrays"]
    check_compatible(engine, meta)
    engine.set_state(arrays["state"])
