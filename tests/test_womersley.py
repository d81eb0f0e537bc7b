"""The Womersley reference profile used by the physics-mode pulsatile test
(tests/physics_ref.py womersley_shape), checked on its own: it carries the
unit flow rate, reduces to Poiseuille at small alpha, flattens with a phase
lag at large alpha, and satisfies the oscillatory pipe-flow equation."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from physics_ref import womersley_shape  # noqa: E402


def test_unit_flow_rate():
    R = 8.0
    r = np.linspace(0.0, R, 40001)
    for alpha in (0.5, 2.0, 4.0, 10.0):
        s = womersley_shape(r, R, alpha)
        q = np.trapezoid(2 * np.pi * r * s, r)
        assert abs(q - 1.0) < 1e-6


def test_poiseuille_limit_and_flattening():
    R = 8.0
    r = np.linspace(0.0, R, 101)
    pois = 2 * (1 - r ** 2 / R ** 2) / (np.pi * R * R)
    # the deviation is O(alpha^2): 5e-5 of the peak at alpha = 0.05
    s = womersley_shape(r, R, 0.05)
    assert np.max(np.abs(s - pois)) < 1e-4 * np.max(pois)
    big = womersley_shape(r, R, 10.0)
    # centre amplitude below Poiseuille's, and lagging the flow rate
    assert abs(big[0]) < 0.8 * pois[0] and np.angle(big[0]) < -0.1


def test_oscillatory_pipe_equation():
    """i w u = G + nu (u'' + u'/r) with a uniform G: the residual
    i w u - nu lap(u) is constant across the radius."""
    R, nu, alpha = 8.0, 0.1, 4.0
    w = alpha ** 2 * nu / R ** 2
    r = np.linspace(0.5, R - 0.5, 2001)
    h = r[1] - r[0]
    s = womersley_shape(r, R, alpha)
    d1 = np.gradient(s, h)
    d2 = np.gradient(d1, h)
    res = 1j * w * s - nu * (d2 + d1 / r)
    core = res[50:-50]
    assert np.max(np.abs(core - core.mean())) < 1e-3 * np.abs(core.mean())
    # no slip at the wall
    assert abs(womersley_shape(R, R, alpha)) < 1e-12
