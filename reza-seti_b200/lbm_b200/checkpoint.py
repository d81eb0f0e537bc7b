"""Checkpoint files: stop a run and resume it bit for bit.

The reference writes no restart files; its only outputs are the result files
of Simulation::WriteOutput (Simulation.cpp:835-856). An engine checkpoint
holds the engine's state blob (lbm_get_state), and a slab-set checkpoint holds
one blob per slab engine. A blob carries the stored populations in the storage
type, the near-wall moments the next wall shear stress uses, the WSS with its
FP64 accumulators, the step count, the flow clock and the AA phase. FP64
populations would not do for the 16-bit and FP32 storage types: f = w + d
rounds away low bits of small deviations d, and a run restarted from them
drifts in the last bit. The flow settings (waveform, inlet profile, outlet
density) are the caller's, as at the start of a run. To resume, build an
engine from the same topology with the same settings, then call restore():
the steps taken from there equal those of the run that was never stopped.

File layout, all little-endian:
* the 8-byte magic b"LBMCKPT2";
* the header length as a uint64 and the header's CRC-32 as a uint32;
* a JSON header: format version, engine settings, step count and clock, and
  per array its dtype, shape, byte offset, length and CRC-32;
* the arrays' raw bytes, one after another.
read() checks the magic, the header's CRC-32 and contents, and every array's
length and CRC-32. It raises CheckpointError naming the first thing that is
wrong, before anything reaches an engine.
"""
from __future__ import annotations

import json
import math
import os
import struct
import zlib

import numpy as np

MAGIC = b"LBMCKPT2"
VERSION = 2
PREFIX = struct.Struct("<QI")  # header length, header CRC-32
DTYPES = {"|u1": 1}
# the arrays each kind of checkpoint must hold
REQUIRED = {"engine": lambda meta: ["state"],
            "slab_set": lambda meta: ["state_%d" % r for r in range(int(meta.get("n_slabs", 0)))]}


class CheckpointError(ValueError):
    """A checkpoint file that cannot be used: damaged, truncated, of another
    format version, or written by an engine unlike the one restoring it."""


def state_of(engine):
    """(meta, arrays) of an engine's current state."""
    steps, runtime = engine.time()
    meta = {"kind": "engine", "n_nodes": int(engine.n), "lattice": int(engine.q),
            "n_nearwall": int(engine.n_nearwall), "storage": engine.storage, "bc": engine.bc,
            "steps": int(steps), "runtime": float(runtime)}
    return meta, {"state": engine.get_state()}


def write(path, meta, arrays):
    """Writes meta and the arrays to path (through a temporary file that
    replaces path once complete)."""
    if not arrays:
        raise CheckpointError("nothing to write")
    entries, blobs, offset = {}, [], 0
    for name in arrays:
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
        fh.write(PREFIX.pack(len(header), zlib.crc32(header)))
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
    start = len(MAGIC) + PREFIX.size
    if len(data) < start or data[: len(MAGIC)] != MAGIC:
        raise CheckpointError("%s: not a checkpoint file (bad magic)" % path)
    hlen, hcrc = PREFIX.unpack_from(data, len(MAGIC))
    if start + hlen > len(data):
        raise CheckpointError("%s: truncated header" % path)
    if zlib.crc32(data[start:start + hlen]) != hcrc:
        raise CheckpointError("%s: CRC-32 mismatch in the header" % path)
    try:
        header = json.loads(data[start:start + hlen].decode())
    except (UnicodeDecodeError, ValueError) as exc:
        raise CheckpointError("%s: unreadable header (%s)" % (path, exc)) from None
    if not isinstance(header, dict) or header.get("version") != VERSION:
        raise CheckpointError("%s: format version %r, this reader takes %d"
                              % (path, header.get("version") if isinstance(header, dict) else None, VERSION))
    meta, entries = header.get("meta"), header.get("arrays")
    if not isinstance(meta, dict) or not isinstance(entries, dict) or not entries:
        raise CheckpointError("%s: header without meta or arrays" % path)
    kind = meta.get("kind")
    if kind not in REQUIRED:
        raise CheckpointError("%s: unknown kind of checkpoint %r" % (path, kind))
    for name in REQUIRED[kind](meta):
        if name not in entries:
            raise CheckpointError("%s: array %s missing" % (path, name))
    base, end, arrays, spans = start + hlen, start + hlen, {}, []
    for name, e in entries.items():
        if not isinstance(e, dict):
            raise CheckpointError("%s: bad entry for array %s" % (path, name))
        try:
            lo, n, shape, crc = base + int(e["offset"]), int(e["nbytes"]), [int(x) for x in e["shape"]], int(e["crc32"])
        except (KeyError, TypeError, ValueError):
            raise CheckpointError("%s: bad entry for array %s" % (path, name)) from None
        dt = e.get("dtype")
        if (dt not in DTYPES or any(d < 0 for d in shape) or n != DTYPES[dt] * math.prod(shape)
                or lo < base):
            raise CheckpointError("%s: array %s: shape, type or offset inconsistent" % (path, name))
        if lo + n > len(data):
            raise CheckpointError("%s: truncated in array %s" % (path, name))
        b = data[lo:lo + n]
        if zlib.crc32(b) != crc:
            raise CheckpointError("%s: CRC-32 mismatch in array %s" % (path, name))
        arrays[name] = np.frombuffer(b, dtype=dt).reshape(shape).copy()
        spans.append((lo, n, name))
        end = max(end, lo + n)
    # the arrays tile the payload: no overlap, no gap
    at = base
    for lo, n, name in sorted(spans):
        if lo != at:
            raise CheckpointError("%s: array %s does not start where the previous one ends" % (path, name))
        at = lo + n
    if end != len(data):
        raise CheckpointError("%s: %d bytes after the last array" % (path, len(data) - end))
    return {"meta": meta, "arrays": arrays}


def check_compatible(engine, meta):
    """Raises CheckpointError unless engine matches the one that wrote meta."""
    mine = {"kind": "engine", "n_nodes": engine.n, "lattice": engine.q, "n_nearwall": engine.n_nearwall,
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


def slab_set_state(slab_set):
    """(meta, arrays) of a SlabSet (lbm_b200.slabs): every slab engine's state."""
    engines = slab_set.engines
    steps, runtime = engines[0].time()
    meta = {"kind": "slab_set", "n_slabs": len(engines), "n_nodes": int(slab_set.n), "lattice": int(slab_set.q),
            "storage": engines[0].storage, "steps": int(steps), "runtime": float(runtime),
            "slab_nodes": [int(e.n) for e in engines]}
    return meta, {"state_%d" % r: e.get_state() for r, e in enumerate(engines)}


def restore_slab_set(slab_set, ckpt):
    """Puts a slab-set checkpoint into slab_set, which must cut the same
    lattice into the same slabs with the same storage type."""
    meta, arrays = ckpt["meta"], ckpt["arrays"]
    engines = slab_set.engines
    mine = {"kind": "slab_set", "n_slabs": len(engines), "n_nodes": slab_set.n, "lattice": slab_set.q,
            "storage": engines[0].storage, "slab_nodes": [e.n for e in engines]}
    for k, v in mine.items():
        if meta.get(k) != v:
            raise CheckpointError("checkpoint %s is %r, the slab set's %r" % (k, meta.get(k), v))
    for r, e in enumerate(engines):
        e.set_state(arrays["state_%d" % r])

