"""Checkpoint and resume on the GPU: a run saved after some steps and
resumed in a new engine continues bit for bit, in every storage type and
both boundary modes. The comparison covers populations, moments, WSS with its
accumulators, OSI/TAWSS and the clock. Also covered: a pulsatile run (the
flow clock), a harmonic waveform (the step count), and the pair kernels of
physics mode with FP32 and FP16 storage."""
import os

import numpy as np
import pytest

from lbm_b200 import Engine
from lbm_b200 import geometry as G
from lbm_b200.capi import LbmError
from lbm_b200.checkpoint import CheckpointError

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: d[k] for k in d.files}


def reference_engine(storage):
    d = golden("cyl_z_pulsatile")
    meta = d["meta_d"]

    def make():
        e = Engine(d, tau=meta[0], dt=meta[1], spacing=meta[2], storage=storage, numeric_check=False)
        e.set_flow(bool(d["meta_i"][7]), float(meta[4]))
        return e
    return make


def physics_engine(storage, q=19, harmonic=True, bc="physics"):
    topo = G.straight_pipe(radius=6.0, length=40)

    def make():
        e = Engine(topo, tau=0.6, lattice=q, storage=storage, bc=bc)
        e.set_inlet_profile(G.parabolic_inlet(topo, 0.03))
        if harmonic:
            e.set_waveform(50.0, [0.4, 0.1], [0.3, 1.2])
        e.set_flow(False, 0.0, harmonic=harmonic)
        return e
    return make


def observables(e):
    w, acc, accm = e.wss()
    o, t = e.osi_tawss()
    rho, u = e.macros()
    return {"f": e.populations(), "rho": rho, "u": u, "wss": w, "acc": acc, "accmag": accm,
            "osi": o, "tawss": t, "time": np.array(e.time())}


def resume_equals_uninterrupted(make, tmp_path, before=30, after=25, pre_steps=0):
    path = str(tmp_path / "run.ckpt")
    a = make()
    a.step(before)
    a.save_checkpoint(path)
    a.step(after)
    want = observables(a)
    a.close()
    b = make()
    if pre_steps:
        b.step(pre_steps)  # an engine that has run already restores all the same
    b.load_checkpoint(path)
    b.step(after)
    got = observables(b)
    b.close()
    for k in want:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_resume_reference_mode_pulsatile(storage, tmp_path):
    resume_equals_uninterrupted(reference_engine(storage), tmp_path, before=40, after=30)


@pytest.mark.parametrize("storage,q", [("f64", 19), ("f32", 19), ("f16", 19), ("bf16", 19), ("f32", 27)])
def test_resume_physics_mode(storage, q, tmp_path):
    resume_equals_uninterrupted(physics_engine(storage, q), tmp_path, pre_steps=3)


def test_restore_refuses_another_storage_type(tmp_path):
    path = str(tmp_path / "run.ckpt")
    a = physics_engine("f32")()
    a.step(4)
    a.save_checkpoint(path)
    a.close()
    b = physics_engine("f16")()
    with pytest.raises(CheckpointError, match="storage"):
        b.load_checkpoint(path)
    b.close()


def test_set_state_refuses_a_foreign_blob():
    a = physics_engine("f32")()
    a.step(4)
    blob = a.get_state()
    b = physics_engine("f32", harmonic=False, bc="reference")()
    with pytest.raises(LbmError, match="another node set"):
        b.set_state(blob)  # same size, other boundary mode
    bad = blob.copy()
    bad[0] ^= 0xFF
    with pytest.raises(LbmError, match="not a state blob"):
        a.set_state(bad)
    # the C ABI checks the length it is given, both ways
    with pytest.raises(LbmError, match="bytes"):
        a.set_state(blob[:-1])
    from lbm_b200 import capi
    short = np.empty(blob.size - 1, dtype=np.uint8)
    with pytest.raises(LbmError, match="buffer of"):
        capi.check(capi.lib().lbm_get_state(a._h, short.ctypes.data, short.size), a._h)
    a.close()
    b.close()


def test_getters_right_after_a_restore(tmp_path):
    path = str(tmp_path / "run.ckpt")
    a = physics_engine("f16")()
    a.step(9)
    w = a.wss()
    a.save_checkpoint(path)
    b = physics_engine("f16")()
    b.load_checkpoint(path)
    assert b.time() == a.time()
    for x, y in zip(b.wss(), w):
        np.testing.assert_array_equal(x, y)
    # populations and moments come back with the next step
    with pytest.raises(LbmError, match="not observed"):
        b.populations()
    a.step(1)
    b.step(1)
    np.testing.assert_array_equal(b.populations(), a.populations())
    a.close()
    b.close()


def test_damaged_checkpoint_is_refused_before_the_engine(tmp_path):
    path = str(tmp_path / "run.ckpt")
    a = physics_engine("f32")()
    a.step(4)
    a.save_checkpoint(path)
    want = a.populations()
    raw = bytearray(open(path, "rb").read())
    raw[-100] ^= 0x01  # one bit of the state blob
    open(path, "wb").write(bytes(raw))
    with pytest.raises(CheckpointError, match="CRC-32"):
        a.load_checkpoint(path)
    np.testing.assert_array_equal(a.populations(), want)
    a.close()


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_slab_set_resume(storage, tmp_path):
    """A lattice cut into 3 slabs (one engine each, halo exchange after every
    step): a resumed slab set equals the uninterrupted one bit for bit."""
    from lbm_b200.slabs import SlabSet
    topo = G.straight_pipe(radius=6.0, length=40)

    def make():
        s = SlabSet(topo, 3, storage=storage, tau=0.6)
        s.set_inlet_profile(G.parabolic_inlet(topo, 0.03))
        s.set_waveform(50.0, [0.4, 0.1], [0.3, 1.2])
        s.set_flow(False, 0.0, harmonic=True)
        return s

    path = str(tmp_path / "slabs.ckpt")
    a = make()
    a.step(20)
    a.save_checkpoint(path)
    a.step(15)
    want = (a.populations(), *a.wss(), *a.osi_tawss())
    a.close()
    b = make()
    b.step(2)  # a set that has run already restores all the same
    b.load_checkpoint(path)
    b.step(15)
    got = (b.populations(), *b.wss(), *b.osi_tawss())
    b.close()
    for x, y in zip(got, want):
        np.testing.assert_array_equal(x, y)
