"""The branching and aneurysm workloads through the engine (physics mode).

Y-bifurcation, D3Q27 (parent R = 24 lu, daughters R = 18 / 16 lu at +-35
degrees, tau 0.55): FP32 storage tracking FP64, the wider daughter carrying
more flow, inflow balancing outflow on time average. Saccular aneurysm on a
90-degree bend, D3Q19: finite state in FP32 and FP16 storage, balanced flux
on time average, slow flow (low wall shear) in the sac relative to the tube.

The instantaneous flux balance is not tested: at these low viscosities
pressure waves travel between the open boundaries for thousands of steps,
so inflow and outflow differ by tens of percent at any one step while
their averages over a window agree.
"""
import numpy as np
import pytest

from lbm_b200 import Engine
from lbm_b200 import geometry as G

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bifurcation():
    return G.y_bifurcation()


@pytest.fixture(scope="module")
def aneurysm():
    return G.saccular_aneurysm()


def engine(topo, q, storage, tau, mean=0.03):
    e = Engine(topo, tau=tau, lattice=q, storage=storage, bc="physics")
    e.set_inlet_profile(G.inlet_disc_profile(topo, mean))
    e.set_flow(False, 0.0)
    return e


def window_flux(e, start, stop, every):
    """Mean inlet and outlet fluxes over samples every `every` steps in [start, stop)."""
    e.step(start)
    ins, outs = [], []
    for _ in range((stop - start) // every):
        e.step(every)
        i, o = e.flux()
        ins.append(i)
        outs.append(o)
    return float(np.mean(ins)), np.mean(outs, axis=0)


def test_bifurcation_fp32_tracks_fp64(bifurcation):
    a = engine(bifurcation, 27, "f64", 0.55)
    b = engine(bifurcation, 27, "f32", 0.55)
    a.step(500)
    b.step(500)
    ua, ub = a.macros()[1], b.macros()[1]
    assert np.linalg.norm(ub - ua) < 1e-4 * np.linalg.norm(ua)
    wa, wb = a.wss()[0], b.wss()[0]
    assert np.linalg.norm(wb - wa) < 1e-4 * np.linalg.norm(wa)


def test_bifurcation_d3q27_split_and_mean_balance(bifurcation):
    e = engine(bifurcation, 27, "f64", 0.55)
    inl, outs = window_flux(e, 3000, 9000, 20)
    print("bifurcation mean fluxes", inl, outs, (inl + outs.sum()) / abs(inl))
    assert e.flags() == 0
    assert len(outs) == 2 and inl < 0 and np.all(outs > 0)
    assert outs[0] > outs[1]  # the R = 18 daughter
    assert abs(inl + outs.sum()) < 0.05 * abs(inl)


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_aneurysm_sac_flow(aneurysm, storage):
    """tau 0.8 (viscous time R^2 / nu = 4000 steps); the 1100-lu tube is
    averaged once its flow has settled, from step 20000 to 26000."""
    e = engine(aneurysm, 19, storage, 0.8, mean=0.02)
    inl, outs = window_flux(e, 20000, 26000, 20)
    print("aneurysm", storage, "mean fluxes", inl, outs, (inl + outs.sum()) / abs(inl))
    assert e.flags() == 0
    assert inl < 0 and abs(inl + outs.sum()) < 0.02 * abs(inl)
    w = e.wss()[0]
    sac = G.sac_wall_targets(aneurysm)
    assert np.all(np.isfinite(w))
    assert w[sac].mean() < 0.5 * w.mean()
