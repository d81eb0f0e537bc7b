"""config.txt and a whole run from it on one GPU.

`read_config` parses a config.txt with the reference's grammar
(parseInputFile, LBM.h:81-188) through lbm_config_parse, including the
extension keys the reference's parser skips (lattice, storage, boundary,
period, equation_bounds, outlet_density, harmonic_*, device).

`run_config` is the reference program (LBM.cpp main: parse, Geometry,
SubDomain, Simulation::Iterate with WriteOutput) on the engine: the STL is
read and voxelised on the GPU, the lattice, storage and boundary mode come
from the file, the pulsatile waveform uses the file's equations: pieces, and
the result files are written where and when the reference writes them
(Simulation.cpp:538-618, 835-856).
"""
import ctypes
import math
import os

import numpy as np

from . import capi

# Pieces of the reference's waveform when a file lists three equations and no
# equation_bounds (Simulation.cpp:523-531): fractions of the period
REFERENCE_BOUNDS = (0.0, 0.1, 0.3, 0.9)
# Iterate's pulsatile stop rule and output radius (Simulation.cpp:549-550, 855)
PULSATILE_END = 2.7
SMOOTHING_RADIUS = 0.25


def _str(b):
    # the reference keeps these fields as raw std::string bytes: decode as
    # file names are, so bytes that are not UTF-8 survive (and still open)
    return os.fsdecode(bytes(b).split(b"\0", 1)[0])


def read_config(path):
    """Parsed config.txt as a dict (lbm_config_parse)."""
    c = capi.LbmConfig()
    capi.check(capi.lib().lbm_config_parse(str(path).encode(), ctypes.byref(c)))
    lattice = {19: "D3Q19", 27: "D3Q27"}[c.lattice]
    storage = {0: "f64", 1: "f32", 2: "f16", 3: "bf16"}[c.storage]

    def opening(o):
        rng = {}
        for a, ax in enumerate("xyz"):
            lo, hi = o.range[a][0], o.range[a][1]
            rng["range_" + ax] = None if (lo == -math.inf and hi == math.inf) else (lo, hi)
        return {"kind": "outlet" if o.outlet else "inlet", "plane": "xyz"[o.axis], "coordinate": o.coordinate,
                "normal": list(o.normal), **rng}

    ops = [opening(c.openings[k]) for k in range(c.n_inlets + c.n_outlets)]
    return {
        "stl_file": _str(c.stl_file), "FlowType": _str(c.flow_type), "dt": c.dt, "rho": c.rho,
        "nu_blood": c.nu_blood, "tau": c.tau, "grid_size": c.grid_size, "pressure": c.pressure,
        "CteVel": c.cte_vel, "reynolds_number": c.reynolds_number, "Systole": c.systole, "Diastole": c.diastole,
        "number_of_outlets": c.number_of_outlets, "MaxIter": c.max_iter, "IterToWrite": c.iter_to_write,
        "NumCycle": c.num_cycle, "inlets": ops[:c.n_inlets], "outlets": ops[c.n_inlets:],
        "equations": [(_str(q.name), list(q.coeffs[:q.n_coeffs])) for q in c.equations[:c.n_equations]],
        "flow": c.flow, "lattice": lattice, "storage": storage,
        "boundary": "physics" if c.bc_mode == 1 else "reference", "device": c.device, "period": c.period,
        "equation_bounds": list(c.equation_bounds[:c.n_bounds]), "outlet_density": c.outlet_density,
        "harmonic_period_steps": c.harmonic_period_steps,
        "harmonic_amplitudes": list(c.harmonic_amplitudes[:c.n_harmonics]),
        "harmonic_phases": list(c.harmonic_phases[:c.n_harmonics]),
    }


class Pulse:
    """A piecewise-polynomial waveform (lbm_pulse_desc). `pieces`: coefficient
    lists, highest power first; `bounds`: fractions of the period, one more
    than pieces."""

    def __init__(self, pieces, bounds=REFERENCE_BOUNDS, period=0.9):
        if len(bounds) != len(pieces) + 1:
            raise ValueError("need one more bound than pieces")
        self.pieces = [list(map(float, p)) for p in pieces]
        self._bounds = np.ascontiguousarray(bounds, dtype=np.float64)
        self._n = np.array([len(p) for p in pieces], dtype=np.int32)
        self._c = np.ascontiguousarray(np.concatenate([np.asarray(p, float) for p in pieces]), dtype=np.float64)
        self.desc = capi.LbmPulseDesc(float(period), len(pieces), self._bounds.ctypes.data_as(capi._f64p),
                                      self._n.ctypes.data_as(capi._i32p), self._c.ctypes.data_as(capi._f64p))

    @classmethod
    def from_config(cls, cfg):
        """The file's equations: as waveform pieces, where they describe a
        whole waveform: any number of equations with equation_bounds (one more
        bound than equations), or three equations without it (the reference's
        bounds, the layout of its config.txt). Otherwise (no equations, or a
        placeholder line) None: the built-in waveform, which is all the
        reference ever uses."""
        pieces = [c for _, c in cfg["equations"] if c]
        if not pieces or len(pieces) != len(cfg["equations"]):
            return None
        if cfg["equation_bounds"]:
            if len(cfg["equation_bounds"]) != len(pieces) + 1:
                raise ValueError("equation_bounds needs one more value than equations")
            return cls(pieces, cfg["equation_bounds"], cfg["period"])
        if len(pieces) == 3:
            return cls(pieces, REFERENCE_BOUNDS, cfg["period"])
        return None

    def __call__(self, t):
        v = ctypes.c_double()
        capi.check(capi.lib().lbm_pulse_eval(ctypes.byref(self.desc), float(t), ctypes.byref(v)))
        return v.value


def reference_pulse(t):
    """The reference's built-in waveform at time t (lbm_pulse_eval, NULL)."""
    v = ctypes.c_double()
    capi.check(capi.lib().lbm_pulse_eval(None, float(t), ctypes.byref(v)))
    return v.value


def output_schedule(cfg):
    """(steps to run, [(step index, phase name)]) of Iterate: Constant and
    Harmonic flow run MaxIter steps with output after every IterToWrite-th
    step index; Pulsatile runs while the clock is <= 2.7 with output where the
    time in the cycle is within dt/2 of Systole or Diastole
    (Simulation.cpp:549-608)."""
    out = []
    if cfg["FlowType"] == "Pulsatile":
        dt, period, tol = cfg["dt"], cfg["period"], cfg["dt"] / 2
        t, it, ns, nd = 0.0, 0, 0, 0
        while t <= PULSATILE_END:
            tic = math.fmod(t, period)
            if abs(tic - cfg["Systole"]) < tol:
                ns += 1
                out.append((it, "Systole_%d" % ns))
            elif abs(tic - cfg["Diastole"]) < tol:
                nd += 1
                out.append((it, "Diastole_%d" % nd))
            t += dt
            it += 1
        return it, out
    total, every = cfg["MaxIter"], cfg["IterToWrite"]
    if every > 0:
        out = [(i, "Iteration_%d" % i) for i in range(every, total, every)]
    return total, out


def run_config(path, out_dir=None, max_steps=None, on_output=None):
    """Runs config.txt at `path` on one GPU and writes the reference's result
    files (<iter>_FlowHemodynamics.csv, FlowHemodynamics/<phase>_<iter>_...csv,
    Fluid_Variables/<iter>.vtu) into out_dir (default: the config's
    directory). Paths in the file are relative to the config's directory, as
    the reference reads them from its working directory. `max_steps` cuts the
    run short (for tests); `on_output(iter, name, engine)` is called after
    each output. Returns (engine, steps run, outputs)."""
    from . import geometry as G
    from .engine import Engine, smooth_surface_csv

    cfg = read_config(path)
    base = os.path.dirname(os.path.abspath(path))
    out_dir = out_dir or base
    if cfg["flow"] < 0:
        raise ValueError("FlowType must be Constant, Pulsatile or Harmonic")
    stl = cfg["stl_file"] if os.path.isabs(cfg["stl_file"]) else os.path.join(base, cfg["stl_file"])
    tris = G.read_stl(stl)
    topo, (dims, origin, spacing, _) = G.voxelise_stl(tris, cfg["grid_size"], cfg["inlets"] + cfg["outlets"],
                                                      device=cfg["device"], info=True)
    q = 27 if cfg["lattice"] == "D3Q27" else 19
    eng = Engine(topo, tau=cfg["tau"], dt=cfg["dt"], spacing=spacing, lattice=q, storage=cfg["storage"],
                 bc=cfg["boundary"], device=cfg["device"])
    pulsatile = cfg["FlowType"] == "Pulsatile"
    if cfg["FlowType"] == "Harmonic":
        eng.set_waveform(cfg["harmonic_period_steps"], cfg["harmonic_amplitudes"], cfg["harmonic_phases"])
        eng.set_flow(harmonic=True, cte_vel=cfg["CteVel"])
    else:
        eng.set_flow(pulsatile, cfg["CteVel"])
    pulse = Pulse.from_config(cfg) if pulsatile else None
    if pulse is not None:
        eng.set_pulsatile(pulse)
    if cfg["boundary"] == "physics":
        # plug inflow against the inlet normal; the waveform factor scales it
        # (1 for constant flow, so the profile carries CteVel there)
        speed = 1.0 if pulsatile else cfg["CteVel"]
        if cfg["FlowType"] == "Harmonic":
            speed = cfg["CteVel"]
        n = np.asarray(topo["inlet_normal"], float)
        eng.set_inlet_profile(np.tile(-speed * n, (len(topo["inlet"]), 1)))
        eng.set_outlet_density(cfg["outlet_density"])
    total, outputs = output_schedule(cfg)
    if max_steps is not None:
        total = min(total, int(max_steps))
        outputs = [o for o in outputs if o[0] < total]
    cells = tuple(int(d) - 1 for d in dims)
    done = 0
    # observation on: the last steps of each call store the state read below
    eng.set_observation(True)
    for it, name in outputs:
        eng.step(it + 1 - done)
        done = it + 1
        csv = os.path.join(out_dir, "%d_FlowHemodynamics.csv" % it)
        eng.write_surface_csv(csv, origin, spacing, pulsatile)
        os.makedirs(os.path.join(out_dir, "FlowHemodynamics"), exist_ok=True)
        smooth_surface_csv(csv, os.path.join(out_dir, "FlowHemodynamics", "%s_%d_FlowHemodynamics.csv" % (name, it)),
                           SMOOTHING_RADIUS, pulsatile, cfg["device"])
        os.makedirs(os.path.join(out_dir, "Fluid_Variables"), exist_ok=True)
        eng.write_vtu(os.path.join(out_dir, "Fluid_Variables", "%d.vtu" % it), cells)
        if on_output:
            on_output(it, name, eng)
    if total > done:
        eng.step(total - done)
    return eng, total, outputs
