"""Slab decomposition on the GPU: the lattice cut into 2-4 slabs, one engine
per slab on one device (SlabSet: the halo exchange of lbm_halo_pack /
lbm_halo_unpack after every step, as the one-GPU-per-rank run does over
NCCL), reproduces the undivided engine's physics-mode run bit for bit:
populations, moments, wall shear stress and its accumulators, OSI / TAWSS;
the fluxes are the slabs' partial sums added (FP64, another summation
order). Pulsatile inflow, D3Q19 and D3Q27, FP64 / FP32 / FP16 storage, and a
vessel large enough that the persistent phase-1 kernel walks several tiles
per CTA in every slab."""
import numpy as np
import pytest

from lbm_b200 import Engine
from lbm_b200 import geometry as G
from lbm_b200.slabs import SlabSet

pytestmark = pytest.mark.gpu


def setup(obj, topo, storage):
    obj.set_inlet_profile(G.parabolic_inlet(topo, 0.03))
    obj.set_waveform(40.0, [0.3, 0.1], [0.0, 1.0])
    obj.set_flow(False, 0.0, harmonic=True)


def compare(topo, q, storage, n_slabs, axis, steps, tau=0.7):
    e = Engine(topo, tau=tau, lattice=q, storage=storage, bc="physics")
    setup(e, topo, storage)
    s = SlabSet(topo, n_slabs, lattice=q, axis=axis, storage=storage, tau=tau)
    setup(s, topo, storage)
    for chunk in steps:
        e.step(chunk)
        s.step(chunk)
        np.testing.assert_array_equal(s.populations(), e.populations())
        r1, u1 = s.macros()
        r0, u0 = e.macros()
        np.testing.assert_array_equal(r1, r0)
        np.testing.assert_array_equal(u1, u0)
        for a, b in zip(s.wss(), e.wss()):
            np.testing.assert_array_equal(a, np.asarray(b).reshape(np.shape(a)))
        for a, b in zip(s.osi_tawss(), e.osi_tawss()):
            np.testing.assert_array_equal(a, b)
        i1, o1 = s.flux()
        i0, o0 = e.flux()
        assert i1 == pytest.approx(i0, rel=1e-12, abs=1e-15)
        np.testing.assert_allclose(o1, o0, rtol=1e-12, atol=1e-15)
    assert s.flags() == 0 and e.flags() == 0
    s.close()
    e.close()


@pytest.mark.parametrize("storage", ["f64", "f32", "f16"])
@pytest.mark.parametrize("n_slabs,axis", [(2, None), (3, 0)])
def test_d3q19_slabs_equal_single_engine(storage, n_slabs, axis):
    topo = G.straight_pipe(radius=6.0, length=40, stenosis=0.4, stenosis_sigma=4.0)
    compare(topo, 19, storage, n_slabs, axis, steps=(1, 4, 25))


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_d3q27_slabs_equal_single_engine(storage):
    topo = G.straight_pipe(radius=6.0, length=40, stenosis=0.4, stenosis_sigma=4.0)
    compare(topo, 27, storage, 3, None, steps=(3, 20))


def test_multi_tile_vessel_four_slabs():
    """R = 24 stenosed pipe (643k nodes, 2513 tiles): every slab's persistent
    phase-1 CTAs walk several tiles, twin and per-node paths both run."""
    topo = G.straight_pipe(radius=24.0, length=384, box=(64, 64, 384), stenosis=0.6, stenosis_sigma=12.0)
    compare(topo, 19, "f32", 4, None, steps=(30,), tau=0.6)
