"""Python host mirror of the reference's time-step interface over the C ABI.

``Engine`` wraps one lbm_engine handle. ``Simulation`` mirrors the reference's
Simulation class (Simulation.h:54-90): it is built from a flattened SubDomain
and a parameter set, and ``Iterate()`` runs the reference's loop with its stop
rules (Simulation.cpp:549-550): MaxIter steps for constant flow, or while the
flow clock is <= 2.7 for pulsatile flow.

A topology is a dict of numpy arrays in the caller's node order, with the keys
    coords [N,3], kind [N] (0 fluid, 1 inlet, 2 outlet, 3 wall),
    inlet, inlet_normal [3], outlet_<k>, outlet_normal_<k> [3], wall,
    nearwall, nearwall_normal [n,3]
— the same keys the reference harness dumps.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi


def _p(a, t):
    return a.ctypes.data_as(t)


def outlets_of(topo):
    outs, normals = [], []
    k = 0
    while "outlet_%d" % k in topo:
        outs.append(np.asarray(topo["outlet_%d" % k], dtype=np.int64))
        normals.append(np.asarray(topo["outlet_normal_%d" % k], dtype=np.float64).reshape(3))
        k += 1
    return outs, normals


class Engine:
    """One engine on one GPU."""

    def __init__(self, topo, *, tau, dt=1e-5, spacing=1.0, lattice=19, storage="f64",
                 bc="reference", device=0, numeric_check=True):
        L = capi.lib()
        self.q = lattice
        self.storage = storage
        self.bc = bc
        keep = {}
        keep["coords"] = np.ascontiguousarray(topo["coords"], dtype=np.int32).reshape(-1, 3)
        keep["kind"] = np.ascontiguousarray(topo["kind"], dtype=np.uint8)
        keep["inlet"] = np.ascontiguousarray(topo["inlet"], dtype=np.int64)
        outs, normals = outlets_of(topo)
        keep["outlet_offsets"] = np.concatenate([[0], np.cumsum([len(o) for o in outs])]).astype(np.int64)
        keep["outlet_nodes"] = np.ascontiguousarray(
            np.concatenate(outs) if outs else np.zeros(0), dtype=np.int64)
        keep["outlet_normals"] = np.ascontiguousarray(np.array(normals, dtype=np.float64).reshape(-1))
        keep["wall"] = np.ascontiguousarray(topo.get("wall", np.zeros(0)), dtype=np.int64)
        keep["nearwall"] = np.ascontiguousarray(topo.get("nearwall", np.zeros(0)), dtype=np.int64)
        keep["nearwall_normal"] = np.ascontiguousarray(
            np.asarray(topo.get("nearwall_normal", np.zeros((0, 3))), dtype=np.float64).reshape(-1))
        self.n = len(keep["kind"])
        self.n_nearwall = len(keep["nearwall"])
        self.n_inlet = len(keep["inlet"])
        self.n_outlets = len(outs)
        d = capi.LbmDesc()
        d.lattice = lattice
        d.storage = capi.STORAGE[storage]
        d.bc_mode = capi.BC_REFERENCE if bc == "reference" else capi.BC_PHYSICS
        d.device = device
        d.n_nodes = self.n
        d.coords = _p(keep["coords"], capi._i32p)
        d.kind = _p(keep["kind"], capi._u8p)
        d.n_inlet = self.n_inlet
        d.inlet = _p(keep["inlet"], capi._i64p)
        inl = np.asarray(topo.get("inlet_normal", np.zeros(3)), dtype=np.float64).reshape(-1)
        for i in range(3):
            d.inlet_normal[i] = float(inl[i]) if len(inl) == 3 else 0.0
        d.n_outlets = len(outs)
        d.outlet_offsets = _p(keep["outlet_offsets"], capi._i64p)
        d.outlet_nodes = _p(keep["outlet_nodes"], capi._i64p)
        d.outlet_normals = _p(keep["outlet_normals"], capi._f64p)
        d.n_wall = len(keep["wall"])
        d.wall = _p(keep["wall"], capi._i64p)
        d.n_nearwall = self.n_nearwall
        d.nearwall = _p(keep["nearwall"], capi._i64p)
        d.nearwall_normals = _p(keep["nearwall_normal"], capi._f64p)
        d.tau, d.dt, d.spacing = float(tau), float(dt), float(spacing)
        h = ctypes.c_void_p()
        capi.check(L.lbm_create(ctypes.byref(d), ctypes.byref(h)), None)
        self._h = h
        self._keep = keep
        self.tau, self.dt, self.spacing = float(tau), float(dt), float(spacing)
        if not numeric_check:
            self.set_numeric_check(False)

    # ---- lifecycle
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            capi.lib().lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, code):
        return capi.check(code, self._h)

    # ---- driving
    def set_stream(self, stream_ptr):
        self._check(capi.lib().lbm_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def set_flow(self, pulsatile=False, cte_vel=0.0, harmonic=False):
        kind = capi.FLOW_HARMONIC if harmonic else (capi.FLOW_PULSATILE if pulsatile else capi.FLOW_CONSTANT)
        self._check(capi.lib().lbm_set_flow(self._h, kind, float(cte_vel)))

    def set_waveform(self, period_steps, amplitude, phase):
        a = np.ascontiguousarray(amplitude, dtype=np.float64)
        p = np.ascontiguousarray(phase, dtype=np.float64)
        self._check(capi.lib().lbm_set_waveform(self._h, float(period_steps), len(a), _p(a, capi._f64p),
                                                _p(p, capi._f64p)))

    def set_pulsatile(self, pulse):
        """Pulsatile waveform pieces (lbm_set_pulsatile): a config.Pulse, or
        None for the reference's built-in waveform."""
        self._pulse = pulse  # the descriptor's arrays must outlive the call only; kept for inspection
        self._check(capi.lib().lbm_set_pulsatile(self._h, ctypes.byref(pulse.desc) if pulse is not None else None))

    def set_inlet_profile(self, vel):
        v = np.ascontiguousarray(vel, dtype=np.float64).reshape(self.n_inlet, 3)
        self._check(capi.lib().lbm_set_inlet_profile(self._h, _p(v, capi._f64p)))

    def set_outlet_density(self, rho):
        self._check(capi.lib().lbm_set_outlet_density(self._h, float(rho)))

    def set_numeric_check(self, enabled):
        """With the check on (default), step() raises LbmError with code
        LBM_ERR_NUMERIC once the device has reported non-finite densities;
        off, it runs on through them as the reference does."""
        self._check(capi.lib().lbm_set_numeric_check(self._h, 1 if enabled else 0))

    def set_observation(self, enabled):
        self._check(capi.lib().lbm_set_observation(self._h, 1 if enabled else 0))

    def step(self, n=1):
        self._check(capi.lib().lbm_step(self._h, int(n)))

    def step_timed(self, n):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(capi.lib().lbm_step_timed(self._h, int(n), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    # ---- slab halo lists (lbm_halo_*)
    def halo_define(self, list_id, nodes, dirs):
        n = np.ascontiguousarray(nodes, dtype=np.int64)
        d = np.ascontiguousarray(dirs, dtype=np.int32)
        if len(n) != len(d):
            raise ValueError("nodes and dirs differ in length")
        self._keep["halo_%d" % list_id] = (n, d)
        self._check(capi.lib().lbm_halo_define(self._h, int(list_id), len(n), _p(n, capi._i64p),
                                                _p(d, capi._i32p)))

    def halo_pack(self, list_id, dst_ptr):
        """Copies list list_id's slots to device memory at dst_ptr (storage type)."""
        self._check(capi.lib().lbm_halo_pack(self._h, int(list_id), ctypes.c_void_p(dst_ptr)))

    def halo_unpack(self, list_id, src_ptr):
        self._check(capi.lib().lbm_halo_unpack(self._h, int(list_id), ctypes.c_void_p(src_ptr)))

    def next_phase(self):
        v = ctypes.c_int32()
        self._check(capi.lib().lbm_get_phase(self._h, ctypes.byref(v)))
        return v.value

    # ---- results
    def time(self):
        s, r = ctypes.c_int64(), ctypes.c_double()
        self._check(capi.lib().lbm_get_time(self._h, ctypes.byref(s), ctypes.byref(r)))
        return s.value, r.value

    def get_state(self):
        """The state the next step reads, as bytes (lbm_get_state)."""
        size = ctypes.c_int64()
        self._check(capi.lib().lbm_state_size(self._h, ctypes.byref(size)))
        buf = np.empty(size.value, dtype=np.uint8)
        self._check(capi.lib().lbm_get_state(self._h, buf.ctypes.data, buf.size))
        return buf

    def set_state(self, blob):
        """Restores a state from get_state of an engine like this one
        (lbm_set_state); the steps then continue bit for bit."""
        buf = np.ascontiguousarray(blob, dtype=np.uint8).reshape(-1)
        self._check(capi.lib().lbm_set_state(self._h, buf.ctypes.data, buf.size))

    def populations(self, out=None):
        f = np.empty((self.n, self.q)) if out is None else out
        self._check(capi.lib().lbm_get_populations(self._h, f.ctypes.data))
        return f

    def set_populations(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(self.n, self.q)
        self._check(capi.lib().lbm_set_populations(self._h, f.ctypes.data))

    def macros(self):
        rho, u = np.empty(self.n), np.empty((self.n, 3))
        self._check(capi.lib().lbm_get_macros(self._h, rho.ctypes.data, u.ctypes.data))
        return rho, u

    def wss(self):
        m = self.n_nearwall
        w, a, am = np.empty(m), np.empty((m, 3)), np.empty(m)
        self._check(capi.lib().lbm_get_wss(self._h, w.ctypes.data, a.ctypes.data, am.ctypes.data))
        return w, a, am

    def save_checkpoint(self, path):
        """Writes the state a resumed run needs to path (lbm_b200.checkpoint)."""
        from . import checkpoint
        checkpoint.save(self, path)

    def load_checkpoint(self, path):
        """Restores a checkpoint written by save_checkpoint from an engine of
        the same topology, lattice, storage type and boundary mode, after the
        flow settings; the run then continues as if it had not stopped."""
        from . import checkpoint
        checkpoint.restore(self, checkpoint.read(path))

    def osi_tawss(self):
        m = self.n_nearwall
        o, t = np.empty(m), np.empty(m)
        self._check(capi.lib().lbm_get_osi_tawss(self._h, o.ctypes.data, t.ctypes.data))
        return o, t

    def flux(self):
        """(inlet flux, [outlet fluxes]) of the last observed state, FP64."""
        inl = np.empty(1)
        outs = np.empty(max(1, self.n_outlets))
        self._check(capi.lib().lbm_get_flux(self._h, inl.ctypes.data, outs.ctypes.data))
        return float(inl[0]), outs[: self.n_outlets].copy()

    def flags(self):
        v = ctypes.c_uint32()
        self._check(capi.lib().lbm_get_flags(self._h, ctypes.byref(v)))
        return v.value

    def adjoint(self, n_steps, targets, basis, coeffs, *, gradient=True, checkpoint_every=100,
                precision="f32", final_populations=False, objective="wss2"):
        """Objective over the near-wall entries `targets` — "wss2", the
        time-averaged sum of |WSS|^2, or "osi", their mean oscillatory shear
        index — and, with `gradient`, its adjoint gradient (lbm_adjoint_run). The
        inlet speed along -inlet_normal is coeffs @ basis ([n_coeffs, n_inlet]).
        Returns a dict: J, dJ_dtau, grad_coeffs, grad_inlet, forward_ms,
        reverse_ms, steps_recomputed, device_bytes (and populations)."""
        targets = np.ascontiguousarray(targets, dtype=np.int64).reshape(-1)
        basis = np.ascontiguousarray(basis, dtype=np.float64).reshape(-1, self.n_inlet)
        coeffs = np.ascontiguousarray(coeffs, dtype=np.float64).reshape(-1)
        if len(coeffs) != basis.shape[0]:
            raise ValueError("one coefficient per basis row")
        d = capi.LbmAdjointDesc()
        d.n_steps, d.checkpoint_every = int(n_steps), int(checkpoint_every)
        d.precision = capi.STORAGE[precision]
        d.n_target, d.target = len(targets), _p(targets, capi._i64p)
        d.n_coeffs, d.basis, d.coeffs = len(coeffs), _p(basis, capi._f64p), _p(coeffs, capi._f64p)
        d.objective = capi.ADJOINT_OBJECTIVE[objective]
        gc = np.zeros(max(1, len(coeffs)))
        gi = np.zeros(max(1, self.n_inlet))
        r = capi.LbmAdjointResult()
        r.grad_coeffs, r.grad_inlet = _p(gc, capi._f64p), _p(gi, capi._f64p)
        fp = None
        if final_populations:
            fp = np.empty((self.n, self.q))
            r.final_populations = _p(fp, capi._f64p)
        self._check(capi.lib().lbm_adjoint_run(self._h, ctypes.byref(d), int(bool(gradient)), ctypes.byref(r)))
        out = {"J": r.objective, "dJ_dtau": r.dJ_dtau, "grad_coeffs": gc[: len(coeffs)].copy(),
               "grad_inlet": gi[: self.n_inlet].copy(), "forward_ms": r.forward_ms,
               "reverse_ms": r.reverse_ms, "steps_recomputed": r.steps_recomputed,
               "device_bytes": r.device_bytes}
        if fp is not None:
            out["populations"] = fp
        return out

    def write_surface_csv(self, path, origin=(0.0, 0.0, 0.0), spacing=1.0, pulsatile=False):
        """The reference's <iter>_FlowHemodynamics.csv (lbm_write_surface_csv)."""
        o = np.ascontiguousarray(origin, dtype=np.float64)
        self._check(capi.lib().lbm_write_surface_csv(self._h, str(path).encode(), _p(o, capi._f64p),
                                                     float(spacing), int(bool(pulsatile))))

    def write_vtu(self, path, cells):
        """The reference's Fluid_Variables/<k>.vtu content (lbm_write_vtu);
        cells = the reference grid's interval counts (nx, ny, nz)."""
        c = np.ascontiguousarray(cells, dtype=np.int32)
        self._check(capi.lib().lbm_write_vtu(self._h, str(path).encode(), _p(c, capi._i32p)))

    def info(self):
        vals = [ctypes.c_int64() for _ in range(6)]
        self._check(capi.lib().lbm_get_info(self._h, *[ctypes.byref(v) for v in vals]))
        keys = ("n_nodes", "ld", "n_segments", "n_nearwall", "n_outlet_nodes", "device_bytes")
        return {k: v.value for k, v in zip(keys, vals)}


class Simulation:
    """The reference's Simulation (Simulation.h:54-90) on the engine.

    params: dict with FlowType ("Constant" or "Pulsatile"), CteVel, MaxIter,
    tau, dt and spacing — the SimulationParameters fields the loop uses.
    ``on_output(iter, sim)`` is called where the reference calls WriteOutput
    for constant flow (every IterToWrite steps, Simulation.cpp:596-603)."""

    PERIOD = 0.9
    PULSATILE_END = 2.7

    def __init__(self, topo, params, storage="f64", on_output=None, device=0):
        self.params = dict(params)
        # the reference runs on through non-finite values
        self.engine = Engine(topo, tau=params["tau"], dt=params.get("dt", 1e-5),
                             spacing=params.get("spacing", 1.0), storage=storage,
                             bc="reference", device=device, numeric_check=False)
        self.pulsatile = params.get("FlowType", "Constant") == "Pulsatile"
        self.engine.set_flow(self.pulsatile, params.get("CteVel", 0.0))
        self.on_output = on_output

    def Iterate(self):
        p = self.params
        if not self.pulsatile:
            total = int(p["MaxIter"])
            every = int(p.get("IterToWrite", 0) or 0)
            done = 0
            while done < total:
                # next output point: iter > 0 and iter % IterToWrite == 0, after
                # the step with that index (iter counts from 0)
                chunk = total - done
                if every and self.on_output:
                    nxt = ((done // every) + 1) * every
                    if nxt < total:
                        chunk = nxt + 1 - done
                self.engine.step(chunk)
                done += chunk
                it = done - 1
                if every and self.on_output and it > 0 and it % every == 0:
                    self.on_output(it, self)
        else:
            t, n = 0.0, 0
            while t <= self.PULSATILE_END:
                t += float(p["dt"])
                n += 1
            self.engine.step(n)


def smooth_surface_csv(in_path, out_path, radius=0.25, pulsatile=False, device=0):
    """The reference's FlowHemodynamics/<phase>_<iter>_FlowHemodynamics.csv
    (lbm_smooth_surface_csv; search radius 0.25 in Simulation::WriteOutput)."""
    capi.check(capi.lib().lbm_smooth_surface_csv(str(in_path).encode(), str(out_path).encode(), float(radius),
                                                 int(bool(pulsatile)), int(device)))
