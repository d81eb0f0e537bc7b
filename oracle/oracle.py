"""Python driver for the oracle (oracle/lbm_oracle.c) — TEST INFRASTRUCTURE.

The oracle restates the reference solver's FP64 time step on the CPU; it is the
checker the CUDA engine is compared with. Only tests/, the smoke check and the
CPU-baseline leg of bench.py import this module; the engine never does.

A topology is a plain dict of numpy arrays in the reference's node order
(Involved_Lat_, Subdomain.cpp:598-611), the same keys the golden fixtures in
tests/golden/ carry:
    coords [N,3] int, kind [N] uint8 (0 fluid, 1 inlet, 2 outlet, 3 wall),
    inlet [n] int64, inlet_normal [3], outlet_<k> [n_k] int64,
    outlet_normal_<k> [3], wall [n] int64, nearwall [n] int64,
    nearwall_normal [n,3], and meta_d = [tau, dt, spacing, ...].
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbm_oracle.so")

Q = 19
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class _Geom(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int64), ("q", ctypes.c_int32), ("nbr", _i64p), ("kind", _u8p),
        ("n_inlet", ctypes.c_int64), ("inlet", _i64p), ("inlet_normal", ctypes.c_double * 3),
        ("n_outlets", ctypes.c_int32), ("outlet_off", _i64p), ("outlet_nodes", _i64p),
        ("outlet_normal", _f64p), ("n_wall", ctypes.c_int64), ("wall", _i64p),
        ("n_nearwall", ctypes.c_int64), ("nearwall", _i64p), ("nearwall_normal", _f64p),
        ("tau", ctypes.c_double), ("dt", ctypes.c_double), ("spacing", ctypes.c_double),
    ]


class _State(ctypes.Structure):
    _fields_ = [(k, _f64p) for k in ("f", "fnew", "feq", "rho", "u", "velmag", "wss", "acc",
                                     "accmag", "osi", "tawss")]


_lib = None


def build():
    """Compiles liblbm_oracle.so (gcc, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        gp, sp = ctypes.POINTER(_Geom), ctypes.POINTER(_State)
        for name in ("orc_init", "orc_collide", "orc_stream", "orc_outlet", "orc_wall",
                     "orc_wss", "orc_osi_tawss"):
            getattr(L, name).argtypes = [gp, sp]
            getattr(L, name).restype = None
        L.orc_inlet.argtypes = [gp, sp, ctypes.c_double]
        L.orc_inlet.restype = None
        L.orc_run.argtypes = [gp, sp, ctypes.c_int64, ctypes.c_int, ctypes.c_double, _f64p]
        L.orc_run.restype = ctypes.c_int64
        L.orc_pulsatile_velocity.argtypes = [ctypes.c_double, ctypes.c_double]
        L.orc_pulsatile_velocity.restype = ctypes.c_double
        L.orc_pulsatile_step_count.argtypes = [ctypes.c_double]
        L.orc_pulsatile_step_count.restype = ctypes.c_int64
        L.orc_wss_constant.argtypes = [gp]
        L.orc_wss_constant.restype = ctypes.c_double
        L.orc_directions.restype = ctypes.POINTER(ctypes.c_int)
        L.orc_weights.restype = _f64p
        L.orc_opposite.restype = ctypes.POINTER(ctypes.c_int)
        _lib = L
    return _lib


def directions():
    p = lib().orc_directions()
    return np.array([p[i] for i in range(3 * Q)], dtype=np.int64).reshape(Q, 3)


def weights():
    p = lib().orc_weights()
    return np.array([p[i] for i in range(Q)])


def opposite():
    p = lib().orc_opposite()
    return np.array([p[i] for i in range(Q)], dtype=np.int64)


def neighbour_table(coords):
    """[N,Q] index of the node at x + c_q, or -1 (SubDomain::Connectivity,
    Subdomain.cpp:447-471)."""
    coords = np.asarray(coords, dtype=np.int64)
    n = len(coords)
    lo = coords.min(axis=0) - 1
    shape = tuple(coords.max(axis=0) - lo + 2)
    grid = -np.ones(shape, dtype=np.int64)
    c = coords - lo
    grid[c[:, 0], c[:, 1], c[:, 2]] = np.arange(n)
    nb = np.empty((n, Q), dtype=np.int64)
    for q, d in enumerate(directions()):
        t = c + d
        nb[:, q] = grid[t[:, 0], t[:, 1], t[:, 2]]
    return nb


def pulsatile_velocity(t, period=0.9):
    return lib().orc_pulsatile_velocity(t, period)


def pulsatile_step_count(dt):
    return lib().orc_pulsatile_step_count(dt)


def _p(a, t):
    return a.ctypes.data_as(t)


class Oracle:
    """FP64 reference-semantics solver on one topology."""

    def __init__(self, topo, tau=None, dt=None, spacing=None):
        meta = np.asarray(topo["meta_d"], dtype=np.float64)
        self.tau = float(meta[0] if tau is None else tau)
        self.dt = float(meta[1] if dt is None else dt)
        self.spacing = float(meta[2] if spacing is None else spacing)
        coords = np.asarray(topo["coords"])
        self.n = len(coords)
        self.nbr = np.ascontiguousarray(topo["nbr"] if "nbr" in topo else neighbour_table(coords),
                                        dtype=np.int64)
        self.kind = np.ascontiguousarray(topo["kind"], dtype=np.uint8)
        self.inlet = np.ascontiguousarray(topo["inlet"], dtype=np.int64)
        k = 0
        outs, normals = [], []
        while "outlet_%d" % k in topo:
            outs.append(np.asarray(topo["outlet_%d" % k], dtype=np.int64))
            normals.append(np.asarray(topo["outlet_normal_%d" % k], dtype=np.float64))
            k += 1
        self.outlet_off = np.concatenate([[0], np.cumsum([len(o) for o in outs])]).astype(np.int64)
        self.outlet_nodes = np.ascontiguousarray(np.concatenate(outs) if outs else np.zeros(0),
                                                 dtype=np.int64)
        self.outlet_normal = np.ascontiguousarray(np.array(normals).reshape(-1, 3))
        self.wall = np.ascontiguousarray(topo["wall"], dtype=np.int64)
        self.nearwall = np.ascontiguousarray(topo["nearwall"], dtype=np.int64)
        self.nearwall_normal = np.ascontiguousarray(
            np.asarray(topo["nearwall_normal"], dtype=np.float64).reshape(-1, 3))
        g = _Geom()
        g.n_nodes = self.n
        g.q = Q
        g.nbr = _p(self.nbr, _i64p)
        g.kind = _p(self.kind, _u8p)
        g.n_inlet = len(self.inlet)
        g.inlet = _p(self.inlet, _i64p)
        inl = np.asarray(topo["inlet_normal"], dtype=np.float64)
        for i in range(3):
            g.inlet_normal[i] = inl[i] if len(inl) == 3 else 0.0
        g.n_outlets = len(outs)
        g.outlet_off = _p(self.outlet_off, _i64p)
        g.outlet_nodes = _p(self.outlet_nodes, _i64p)
        g.outlet_normal = _p(self.outlet_normal, _f64p)
        g.n_wall = len(self.wall)
        g.wall = _p(self.wall, _i64p)
        g.n_nearwall = len(self.nearwall)
        g.nearwall = _p(self.nearwall, _i64p)
        g.nearwall_normal = _p(self.nearwall_normal, _f64p)
        g.tau, g.dt, g.spacing = self.tau, self.dt, self.spacing
        self._g = g
        nw = len(self.nearwall)
        self.f = np.zeros((self.n, Q))
        self.fnew = np.zeros((self.n, Q))
        self.feq = np.zeros((self.n, Q))
        self.rho = np.zeros(self.n)
        self.u = np.zeros((self.n, 3))
        self.velmag = np.zeros(self.n)
        self.wss = np.zeros(nw)
        self.acc = np.zeros((nw, 3))
        self.accmag = np.zeros(nw)
        self.osi = np.zeros(nw)
        self.tawss = np.zeros(nw)
        s = _State()
        for name in ("f", "fnew", "feq", "rho", "u", "velmag", "wss", "acc", "accmag", "osi",
                     "tawss"):
            setattr(s, name, _p(getattr(self, name), _f64p))
        self._s = s
        self.runtime = ctypes.c_double(0.0)
        lib().orc_init(ctypes.byref(self._g), ctypes.byref(self._s))

    # one phase of the reference step each
    def collide(self):
        lib().orc_collide(ctypes.byref(self._g), ctypes.byref(self._s))

    def stream(self):
        lib().orc_stream(ctypes.byref(self._g), ctypes.byref(self._s))

    def inlet_bc(self, vel):
        lib().orc_inlet(ctypes.byref(self._g), ctypes.byref(self._s), vel)

    def outlet_bc(self):
        lib().orc_outlet(ctypes.byref(self._g), ctypes.byref(self._s))

    def wall_bc(self):
        lib().orc_wall(ctypes.byref(self._g), ctypes.byref(self._s))

    def wall_shear_stress(self):
        lib().orc_wss(ctypes.byref(self._g), ctypes.byref(self._s))

    def osi_tawss(self):
        lib().orc_osi_tawss(ctypes.byref(self._g), ctypes.byref(self._s))

    @property
    def wss_constant(self):
        return lib().orc_wss_constant(ctypes.byref(self._g))

    def run(self, steps, pulsatile=False, cte_vel=0.0):
        return lib().orc_run(ctypes.byref(self._g), ctypes.byref(self._s), steps,
                             1 if pulsatile else 0, cte_vel, ctypes.byref(self.runtime))
