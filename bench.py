"""Benchmark of the B200 LBM engine's time step (MLUPS and HBM roofline).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload tortuous8|tortuousR<radius>|pipe] [--storage f32|f16|bf16|f64]

Workload (default): the tortuous stenosed vessel in a 512 x 512 x 1024 box —
sinusoidal centerline (amplitude 30 lu, wavelength 200 lu), Gaussian 50 %-area
stenosis at mid-length, D3Q19, tau 0.52, plug inlet at Re = 300 — at the stated
~8 % fluid fraction of the box (radius from fluid_fraction_radius). The
vessel's own radius 20 lu gives ~0.6 % of the box; that variant is timed too
and reported under "variants". Inputs are synthetic and seeded (none needed:
the geometry is analytic and the initial state is f = w). The population
state (>= 1.6 GB) is larger than L2 (126 MB), so no flush is needed between
steps.

A step is one time step over every fluid node: the AA stream+collide kernel
and the post pass after it (that step's WSS on the near-wall nodes and the
open-boundary corrections; in reference mode a pre-pass with the previous
step's WSS and the outlet sources). `value`
is fluid-node updates per second over all GPUs (MLUPS), timed with CUDA
events on the engine's stream; `e2e` times the same through the C ABI from
host buffers (state upload, steps, state and WSS download). With --gpus N
(torchrun) every rank runs an independent replica: the path has no
inter-GPU exchange on one domain ("replicas only").

--impl reference times the reference solver's own step loop (built from its
sources into oracle/_ref/refharness) on slabs of the same vessel, one process
per host core, and prints the same line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "reza-seti_b200"))

METRIC = "MLUPS"
BYTES_PER_POP = {"f64": 8, "f32": 4, "f16": 2, "bf16": 2}
TAU = 0.52
REYNOLDS = 300.0


def inlet_velocity(radius):
    """Mean inlet velocity (lattice units) giving Re = u D / nu = 300 for the
    vessel diameter, with nu = (tau - 1/2) / 3 — the precision config's Re."""
    return REYNOLDS * (TAU - 0.5) / 3.0 / (2.0 * radius)


def inlet_profile(topo, radius, mean):
    """Parabolic inflow along +z with the given mean velocity over the inlet
    disc (peak 2 x mean), centred on the inlet nodes."""
    xy = topo["coords"][topo["inlet"]][:, :2].astype(np.float64)
    c = xy.mean(axis=0)
    r2 = ((xy - c) ** 2).sum(axis=1)
    v = np.zeros((len(xy), 3))
    v[:, 2] = np.maximum(0.0, 2.0 * mean * (1.0 - r2 / (radius * radius)))
    return v


BOX = (512, 512, 1024)


def build_workload(name):
    from lbm_b200 import geometry as G
    if name == "tortuous8":
        r = G.fluid_fraction_radius(0.08, BOX)
        topo = G.tortuous_vessel(radius=r, box=BOX)
        desc = "tortuous stenosed vessel, 512x512x1024 box, ~8%% fluid (radius %.1f lu)" % r
    elif name.startswith("tortuousR"):
        r = float(name[len("tortuousR"):])
        topo = G.tortuous_vessel(radius=r, box=BOX)
        desc = "tortuous stenosed vessel, 512x512x1024 box, radius %g lu" % r
    elif name == "pipe":
        r = 16.0
        topo = G.straight_pipe(radius=r, length=136, box=(40, 40, 136))
        desc = "straight pipe R=16 lu in a 40x40x136 box"
    elif name == "aneurysm":
        r = 20.0
        topo = G.saccular_aneurysm()
        desc = "saccular aneurysm: R=20 tube, 90 deg bend of radius 120, R=40 sac, box 1024x512x512"
    elif name == "bifurcation":
        r = 24.0
        topo = G.y_bifurcation()
        desc = "Y-bifurcation, parent R=24 L=200, daughters R=18/16 at +-35 deg, box 256x256x348 (D3Q27)"
    elif name == "stenosed":
        r = 24.0
        topo = G.straight_pipe(radius=24.0, length=384, box=(64, 64, 384), stenosis=0.6, stenosis_sigma=12.0)
        desc = "stenosed pipe R=24 lu, 64x64x384 box, 60% radius stenosis"
    else:
        raise SystemExit("unknown workload " + name)
    return topo, desc, r


def workload_lattice(name):
    return 27 if name == "bifurcation" else 19


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes (read + write) per fluid node and step-kernel launch, averaged
# over the two phase kernels of one step, from an ncu capture of
# dram__bytes_read.sum + dram__bytes_write.sum on the step kernels (command
# and case in profiles/step_kernel_traffic_d3q19.md); None where not captured.
STEP_KERNEL_TRAFFIC = {"f32": 156.2, "f16": 80.92}
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one phase-0 and one phase-1 launch "
                  "on the default workload (21,381,419 nodes, 1.6 GB FP32 state, 13x L2), averaged: FP32 "
                  "3.33 and 3.35 GB, FP16 1.712 and 1.748 GB per launch; the excess over the algorithmic "
                  "2 Q S per node is the node words (4 B), segment rows and the near-wall hand-off")


def host_cpu():
    """CPU model and logical core count of this host (for the CPU baselines)."""
    model = None
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def dist_setup(n_gpus, backend="nccl"):
    """World size, rank, local rank and torch.distributed (or None for one
    process) from the torchrun environment. Ranks are independent replicas:
    the process group carries only the barriers and the max-over-ranks time."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(value, dist, device):
    """The largest of every rank's value: the job takes as long as its
    slowest replica."""
    if not dist:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_mlups(n_nodes, steps, max_ms, world):
    """Whole-job MLUPS of `world` replicas of n_nodes each over `steps` steps
    that took at most max_ms."""
    return n_nodes * steps / (max_ms / 1e3) / 1e6 * world


def time_engine(topo, storage, steps, warmup, device, torch, vel, bc="physics", radius=None, before=None, q=19):
    from lbm_b200 import Engine
    # reference boundaries diverge at tau 0.52 (as the reference itself does);
    # their timing runs on through the non-finite values, as the reference would
    eng = Engine(topo, tau=TAU, dt=1e-5, spacing=1.0, lattice=q, storage=storage, device=device, bc=bc,
                 numeric_check=(bc == "physics"))
    eng.set_flow(False, vel)
    if bc == "physics":
        eng.set_inlet_profile(inlet_profile(topo, radius, vel))
    # timed steps store no observable state (the C ABI's observation switch);
    # the end-to-end measurement below turns it back on
    eng.set_observation(False)
    stream = torch.cuda.Stream(device=device)
    eng.set_stream(stream.cuda_stream)
    eng.step(warmup)
    torch.cuda.synchronize(device)
    if before is not None:
        before()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    ms_step, ms_bnd = eng.step_timed(steps)
    stop.record(stream)
    stop.synchronize()
    total_ms = start.elapsed_time(stop)
    return eng, total_ms, ms_step, ms_bnd


def run_gpu(args):
    import torch
    world, rank, local, dist = dist_setup(args.gpus)
    device = local
    torch.cuda.set_device(device)
    topo, desc, radius = build_workload(args.workload)
    vel = inlet_velocity(radius)
    n = len(topo["kind"])
    storage = args.storage
    S = BYTES_PER_POP[storage]
    Q = workload_lattice(args.workload)

    # headline: K steps on the engine stream, CUDA events, barrier + sync on
    # both sides of the timed region
    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize(device)

    with ClockSampler(device) as clk:
        eng, total_ms, ms_step, ms_bnd = time_engine(topo, storage, args.steps, args.warmup, device, torch, vel,
                                                     args.bc, radius, before=barrier, q=Q)
    barrier()
    total_ms = max_over_ranks(total_ms, dist, "cuda")
    clocks = clk.summary()
    info = eng.info()
    flags = eng.flags()
    mlups = replica_mlups(n, args.steps, total_ms, world)
    ms_per_step = total_ms / args.steps

    # roofline of the dominant kernel (stream+collide): algorithmic bytes 2 Q S per node
    peak, peak_kind = measured_peaks()
    alg_bytes = 2 * Q * S * n
    step_avg_ms = ms_step / args.steps
    achieved = alg_bytes / (step_avg_ms / 1e3) / 1e9
    tpn = STEP_KERNEL_TRAFFIC.get(storage) if (args.workload == "tortuous8" and args.bc == "physics") else None
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": round(tpn * n) if tpn else None,
                "traffic_source": TRAFFIC_SOURCE if tpn else "not captured for this storage type",
                "algorithmic_bytes_per_launch": alg_bytes,
                "step_kernel_ms": round(step_avg_ms, 5),
                "boundary_kernel_ms": round(ms_bnd / args.steps, 5)}

    # end to end through the C ABI with host buffers
    e2e = None
    if rank == 0 and not args.no_e2e:
        e2e = end_to_end(eng, n, Q, args.steps, torch)
    eng.close()

    variants = {}
    if rank == 0 and not args.no_variants:
        variants = run_variants(args, topo, n, torch, device, vel, radius)

    precision = None
    if rank == 0 and not args.no_precision:
        precision = run_precision(torch, device)
    adjoint = None
    if rank == 0 and not args.no_adjoint:
        adjoint = run_adjoint(torch, device)
    configs = None
    if rank == 0 and not args.no_configs:
        configs = run_configs(torch, device)
    voxel = None
    if rank == 0 and not args.no_voxel:
        voxel = run_voxel(torch, device)
    jt = None
    if rank == 0 and not args.no_jt:
        jt = run_jt(torch, device)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference(args, sample_only=True)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"f32": "f32 (storage f - w), f32 compute", "f16": "f16 storage, f32 compute",
                      "bf16": "bf16 storage, f32 compute", "f64": "f64"}[storage],
            "data": "synthetic (analytic vessel geometry, f = w initial state)",
            "config": {"workload": desc, "lattice": "D3Q%d" % Q, "fluid_nodes": n,
                       "box_cells": BOX[0] * BOX[1] * BOX[2] if args.workload.startswith("tortuous") else None,
                       "tau": TAU, "inlet_velocity": round(vel, 6), "reynolds": REYNOLDS, "storage": storage,
                       "bc_mode": args.bc, "segments": info["n_segments"],
                       "near_wall_nodes": info["n_nearwall"],
                       "l2": "state larger than L2 (no flush)",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": 2 * args.steps, "clocks": clocks, "device_flags": flags,
            "variants": variants, "precision": precision, "adjoint": adjoint, "configs": configs, "geometry_setup": voxel,
            "shipped_case": jt,
        }
        # the key figures once more, last on the line (a reader of its tail
        # sees them)
        line["summary"] = summary(storage, mlups, roofline, variants, precision, adjoint, configs, cpu, jt)
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def summary(storage, mlups, roofline, variants, precision, adjoint, configs, cpu, jt=None):
    """Headline figures of every section, in one small block."""
    def get(d, *keys):
        for k in keys:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    out = {storage + "_MLUPS": round(mlups, 1), "step_kernel_frac": roofline["frac"]}
    for st in ("f32", "f16", "bf16"):
        v = get(variants, st, "MLUPS")
        if v is not None:
            out[st + "_MLUPS"] = v
    if storage == "f32":
        for st in ("f16", "bf16"):
            if get(variants, st, "MLUPS"):
                out[st + "_vs_f32"] = round(variants[st]["MLUPS"] / mlups, 3)
    ref = get(variants, "reference_bc_f64")
    if ref:
        out["reference_bc_f64"] = {"MLUPS": ref["MLUPS"], "step_kernel_frac": ref["step_kernel_frac"],
                                   "e2e_MLUPS": get(ref, "e2e", "value")}
    for tau in PRECISION_TAUS:
        b = get(precision, "tau_%g" % tau)
        if b:
            out["precision_tau_%g" % tau] = {
                "tawss_rel_l2": {"f32_vs_f64": get(b, "f32", "vs_f64", "tawss_rel_l2"),
                                 "f16_vs_f64": get(b, "f16", "vs_f64", "tawss_rel_l2"),
                                 "f16_vs_f32": get(b, "f16", "vs_f32", "tawss_rel_l2"),
                                 "bf16_vs_f64": get(b, "bf16", "vs_f64", "tawss_rel_l2")},
                "osi_abs_max": {"f32_vs_f64": get(b, "f32", "vs_f64", "osi_abs_max"),
                                "f16_vs_f64": get(b, "f16", "vs_f64", "osi_abs_max"),
                                "f16_vs_f32": get(b, "f16", "vs_f32", "osi_abs_max")}}
    if adjoint:
        out["adjoint_stenosed_pipe"] = {"cost_vs_forward_step": adjoint.get("cost_per_step_vs_forward_step"),
                                        "f32_vs_fd_rel": adjoint.get("f32_vs_fd_rel"),
                                        "f64_vs_fd_rel": adjoint.get("f64_vs_fd_rel")}
    if configs:
        out["aneurysm"] = {"f32_MLUPS": get(configs, "aneurysm", "f32", "MLUPS"),
                           "f16_MLUPS": get(configs, "aneurysm", "f16", "MLUPS"),
                           "adjoint_cost_vs_forward_step": get(configs, "aneurysm_adjoint",
                                                               "cost_per_step_vs_forward_step")}
        out["bifurcation_f32_MLUPS"] = get(configs, "bifurcation", "f32", "MLUPS")
    if jt:
        out["shipped_case_jt"] = {"nodes": jt["nodes"], "gpu_setup_seconds": jt["gpu_setup_seconds"],
                                  "reference_f64_MLUPS": get(jt, "reference_f64", "MLUPS"),
                                  "physics_f32_MLUPS": get(jt, "physics_f32", "MLUPS")}
    if cpu:
        out["cpu_reference_MLUPS"] = {"value": cpu.get("value"), "cores": cpu.get("cores"),
                                      "cpu_model": cpu.get("cpu_model")}
    return out


def timed_steps(e, n, torch, device):
    """n steps of engine e on a torch stream: (device time of the whole call by
    CUDA events around it, the step-kernel and boundary-kernel split of
    lbm_step_timed). A step's kernels overlap (programmatic dependent
    launch), so throughput comes from the first figure, not the split's sum."""
    s = torch.cuda.Stream(device=device)
    e._timing_stream = s  # the engine keeps using it
    e.set_stream(s.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    ms_step, ms_bnd = e.step_timed(n)
    b.record(s)
    b.synchronize()
    return a.elapsed_time(b), ms_step, ms_bnd


def end_to_end(eng, n, Q, steps, torch):
    """State upload, `steps` steps and result download through the C ABI from
    pinned host buffers, timed on the host clock around the synchronous calls."""
    eng.set_observation(True)
    eng.step(1)
    f = torch.empty((n, Q), dtype=torch.float64).pin_memory().numpy()
    f[:] = eng.populations()
    wss = torch.empty(eng.n_nearwall, dtype=torch.float64).pin_memory().numpy()
    t0 = time.perf_counter()
    eng.set_populations(f)
    eng.step(steps)
    eng.populations(out=f)
    from lbm_b200 import capi
    capi.check(capi.lib().lbm_get_wss(eng._h, wss.ctypes.data, None, None), eng._h)
    dt = time.perf_counter() - t0
    h2d = n * Q * 8
    d2h = n * Q * 8 + eng.n_nearwall * 8
    return {"value": round(n * steps / dt / 1e6, 1), "unit": "MLUPS",
            "h2d_bytes_per_step": h2d // steps, "d2h_bytes_per_step": d2h // steps,
            "seconds": round(dt, 4)}


def run_variants(args, topo, n, torch, device, vel, radius):
    out = {}
    steps = max(10, args.steps // 2)
    for storage in ("f16", "bf16", "f64"):
        if storage == args.storage:
            continue
        eng, total_ms, ms_step, _ = time_engine(topo, storage, steps, args.warmup, device, torch, vel,
                                                args.bc, radius)
        S = BYTES_PER_POP[storage]
        out[storage] = {"MLUPS": round(n * steps / (total_ms / 1e3) / 1e6, 1),
                        "step_kernel_GBs": round(2 * 19 * S * n / (ms_step / steps / 1e3) / 1e9, 1)}
        eng.close()
    if args.workload == "tortuous8":
        from lbm_b200 import geometry as G
        t20 = G.tortuous_vessel(radius=20.0, box=BOX)
        n20 = len(t20["kind"])
        eng, total_ms, ms_step, _ = time_engine(t20, "f32", steps, args.warmup, device, torch,
                                                inlet_velocity(20.0), args.bc, 20.0)
        out["radius20_f32"] = {"fluid_nodes": n20,
                               "MLUPS": round(n20 * steps / (total_ms / 1e3) / 1e6, 1)}
        eng.close()
    other = "reference" if args.bc == "physics" else "physics"
    eng, total_ms, ms_step, _ = time_engine(topo, "f32", steps, args.warmup, device, torch, vel, other, radius)
    out[other + "_bc_f32"] = {"MLUPS": round(n * steps / (total_ms / 1e3) / 1e6, 1),
                              "step_kernel_GBs": round(2 * 19 * 4 * n / (ms_step / steps / 1e3) / 1e9, 1),
                              "device_flags": eng.flags()}
    eng.close()
    # like for like with the reference arm: FP64 storage and arithmetic, the
    # reference's boundary rules, same workload; kernel time and end to end
    # through the C ABI from host buffers
    peak, _ = measured_peaks()
    eng, total_ms, ms_step, _ = time_engine(topo, "f64", steps, args.warmup, device, torch, vel, "reference",
                                            radius)
    gbs = 2 * 19 * 8 * n / (ms_step / steps / 1e3) / 1e9
    out["reference_bc_f64"] = {"MLUPS": round(n * steps / (total_ms / 1e3) / 1e6, 1),
                               "step_kernel_GBs": round(gbs, 1), "step_kernel_frac": round(gbs / peak, 4),
                               "algorithmic_bytes_per_node": 2 * 19 * 8,
                               "device_flags": eng.flags(),
                               "e2e": None if args.no_e2e else end_to_end(eng, n, 19, steps, torch)}
    eng.close()
    return out


# --------------------------------------------------------------- precision ---
PRECISION_PERIOD = 4000
PRECISION_PERIODS = 2


def harmonic_waveform(seed=3, n=4):
    """Seeded Womersley-type waveform: harmonic k (1-based) with amplitude
    uniform in [0, 0.5] / k of the mean and a uniform phase."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.0, 0.5, n) / np.arange(1, n + 1)
    phase = rng.uniform(0.0, 2 * np.pi, n)
    return amp, phase


PRECISION_TAUS = (0.52, 0.55)


def run_precision(torch, device, topo=None):
    """TAWSS / OSI (FP64 accumulators) and final-state errors of FP32, FP16 and
    BF16 storage on the radius-20 tortuous vessel over two periods of a
    4-harmonic waveform, at tau 0.52 (Re 300 at the mean flow, the precision
    config) and at tau 0.55 (the same inflow, Re 120), where the flow no longer
    amplifies every perturbation. Each storage type is compared with FP64
    storage, and FP16 / BF16 also with FP32 storage, so that storage rounding
    and the flow's sensitivity can be told apart. Errors are relative L2 norms
    over all near-wall nodes (TAWSS, WSS), over all nodes (velocity,
    populations f - w), the largest relative TAWSS difference (to the largest
    TAWSS) and the largest absolute OSI difference."""
    from lbm_b200 import Engine
    from lbm_b200 import geometry as G
    r = 20.0
    if topo is None:
        topo = G.tortuous_vessel(radius=r, box=BOX)
    n = len(topo["kind"])
    vel = inlet_velocity(r)
    amp, phase = harmonic_waveform()
    steps = PRECISION_PERIOD * PRECISION_PERIODS
    w = np.array([2 / 36] * 6 + [1 / 36] * 12 + [12 / 36])

    def l2(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    def errors(a, b):
        osi, tawss, wss, d, u = a
        return {"tawss_rel_l2": l2(tawss, b[1]),
                "tawss_rel_max": float(np.max(np.abs(tawss - b[1])) / np.max(np.abs(b[1]))),
                "osi_abs_max": float(np.max(np.abs(osi - b[0]))),
                "wss_rel_l2": l2(wss, b[2]), "velocity_rel_l2": l2(u, b[4]), "populations_rel_l2": l2(d, b[3])}

    out = {"workload": "tortuous stenosed vessel radius 20 lu, 512x512x1024 box (%d fluid nodes)" % n,
           "steps": steps, "waveform": {"period_steps": PRECISION_PERIOD, "amplitude": np.round(amp, 4).tolist(),
                                        "phase": np.round(phase, 4).tolist(), "seed": 3},
           "mean_inlet_velocity": round(vel, 6)}
    for tau in PRECISION_TAUS:
        res = {}
        block = {"reynolds": round(vel * 2 * r / ((tau - 0.5) / 3.0), 1)}
        for storage in ("f64", "f32", "f16", "bf16"):
            eng = Engine(topo, tau=tau, dt=1e-5, spacing=1.0, storage=storage, device=device, bc="physics")
            eng.set_inlet_profile(inlet_profile(topo, r, vel))
            eng.set_waveform(float(PRECISION_PERIOD), amp, phase)
            eng.set_flow(False, vel, harmonic=True)
            t0 = time.perf_counter()
            eng.step(steps)
            osi, tawss = eng.osi_tawss()
            wss = eng.wss()[0]
            d = eng.populations() - w
            u = eng.macros()[1]
            flags = eng.flags()
            secs = time.perf_counter() - t0
            eng.close()
            res[storage] = (osi, tawss, wss, d, u)
            row = {"seconds": round(secs, 2), "device_flags": flags}
            if storage == "f64":
                row["tawss_mean"] = float(np.mean(tawss))
                row["osi_max"] = float(np.max(osi))
            else:
                row["vs_f64"] = errors(res[storage], res["f64"])
                if storage != "f32":
                    row["vs_f32"] = errors(res[storage], res["f32"])
            block[storage] = row
        out["tau_%g" % tau] = block
    return out


# ----------------------------------------------- branching and aneurysm ---
CFG_PERIOD, CFG_PERIODS, CFG_MEAN = 4000, 2, 0.03


def run_configs(torch, device):
    """The Y-bifurcation (D3Q27, tau 0.55) and the saccular aneurysm (D3Q19,
    tau 0.55) over two periods of a seeded 4-harmonic waveform (period 4000
    steps, mean inflow 0.03 lu): kernel MLUPS per storage type (fluid nodes
    and, for the aneurysm, box cells), TAWSS / OSI (FP64 accumulators), and
    the errors of FP32 / FP16 storage against FP64 storage."""
    from lbm_b200 import Engine
    from lbm_b200 import geometry as G
    amp, phase = harmonic_waveform(seed=5)
    steps = CFG_PERIOD * CFG_PERIODS

    def l2(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    def one(topo, q, storage, tau):
        e = Engine(topo, tau=tau, dt=1e-5, spacing=1.0, lattice=q, storage=storage, device=device, bc="physics")
        e.set_inlet_profile(G.inlet_disc_profile(topo, CFG_MEAN))
        e.set_waveform(float(CFG_PERIOD), amp, phase)
        e.set_flow(False, 0.0, harmonic=True)
        e.set_observation(False)
        wall_ms, ms_step, ms_bnd = timed_steps(e, steps - 1, torch, device)
        e.set_observation(True)
        e.step(1)
        osi, tawss = e.osi_tawss()
        u = e.macros()[1]
        inl, outs = e.flux()
        res = {"ms_per_step": round(wall_ms / (steps - 1), 5),
               "step_kernel_ms": round(ms_step / (steps - 1), 5), "boundary_kernel_ms": round(ms_bnd / (steps - 1), 5),
               "device_flags": e.flags(), "inlet_flux": inl, "outlet_fluxes": outs.tolist()}
        e.close()
        return res, osi, tawss, u, wall_ms / (steps - 1)

    out = {"waveform": {"period_steps": CFG_PERIOD, "amplitude": np.round(amp, 4).tolist(),
                        "phase": np.round(phase, 4).tolist(), "seed": 5, "mean_inlet_velocity": CFG_MEAN},
           "steps": steps}
    topo = G.y_bifurcation()
    n = len(topo["kind"])
    bif = {"workload": "Y-bifurcation, parent R=24 L=200, daughters R=18/16 L=180 at +-35 deg, box 256x256x348",
           "lattice": "D3Q27", "tau": 0.55, "fluid_nodes": n}
    ref = None
    for storage in ("f64", "f32"):
        res, osi, tawss, u, ms = one(topo, 27, storage, 0.55)
        res["MLUPS"] = round(n / ms / 1e3, 1)
        if ref is None:
            ref = (osi, tawss, u)
        else:
            res.update({"tawss_rel_l2": l2(tawss, ref[1]), "osi_abs_max": float(np.max(np.abs(osi - ref[0]))),
                        "velocity_rel_l2": l2(u, ref[2])})
        bif[storage] = res
    out["bifurcation"] = bif

    topo = G.saccular_aneurysm()
    n = len(topo["kind"])
    cells = 1024 * 512 * 512
    sac = G.sac_wall_targets(topo)
    an = {"workload": "saccular aneurysm: R=20 tube, 90 deg bend of radius 120, R=40 sac on the outer wall, "
                      "box 1024x512x512", "lattice": "D3Q19", "tau": 0.55, "fluid_nodes": n, "box_cells": cells,
          "sac_wall_nodes": int(len(sac))}
    ref = None
    for storage in ("f64", "f32", "f16"):
        res, osi, tawss, u, ms = one(topo, 19, storage, 0.55)
        res["MLUPS"] = round(n / ms / 1e3, 1)
        res["box_cell_MLUPS"] = round(cells / ms / 1e3, 1)
        res["sac_tawss_mean"] = float(np.mean(tawss[sac]))
        res["sac_osi_mean"] = float(np.mean(osi[sac]))
        if ref is None:
            ref = (osi, tawss, u)
        else:
            res.update({"sac_tawss_rel_l2": l2(tawss[sac], ref[1][sac]),
                        "sac_osi_abs_max": float(np.max(np.abs(osi[sac] - ref[0][sac]))),
                        "tawss_rel_l2": l2(tawss, ref[1]), "velocity_rel_l2": l2(u, ref[2])})
        an[storage] = res
    out["aneurysm"] = an

    # adjoint of the sac-averaged OSI w.r.t. 8 inlet modes, over the same run
    basis = G.zernike_inlet_basis(topo, 8)
    rng = np.random.default_rng(13)
    a = 0.006 * rng.standard_normal(8)
    a[0] = 2 * CFG_MEAN  # mode 0: parabola with the mean inflow
    e = Engine(topo, tau=0.55, dt=1e-5, spacing=1.0, storage="f64", device=device, bc="physics")
    e.set_waveform(float(CFG_PERIOD), amp, phase)
    e.set_flow(False, 0.0, harmonic=True)
    r32 = e.adjoint(steps, sac, basis, a, checkpoint_every=100, precision="f32", objective="osi")
    r64 = e.adjoint(steps, sac, basis, a, checkpoint_every=100, precision="f64", objective="osi")
    g32, g64 = np.append(r32["grad_coeffs"], r32["dJ_dtau"]), np.append(r64["grad_coeffs"], r64["dJ_dtau"])
    h = 1e-4
    fd = {}
    for j in (0, 1, 3):
        ap, am = a.copy(), a.copy()
        ap[j] += h
        am[j] -= h
        fd[j] = (e.adjoint(steps, sac, basis, ap, gradient=False, precision="f64", objective="osi")["J"] -
                 e.adjoint(steps, sac, basis, am, gradient=False, precision="f64", objective="osi")["J"]) / (2 * h)
    e.close()
    fwd_ms = an["f32"]["ms_per_step"]
    out["aneurysm_adjoint"] = {
        "objective": "mean OSI over the sac wall nodes", "parameters": "8 inlet modes + tau", "steps": steps,
        "checkpoint_every": 100, "J_f32": r32["J"], "J_f64": r64["J"], "grad_f64": g64.tolist(),
        "grad_f32_vs_f64_rel": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
        "fd_h": h, "fd_checked": {str(j): {"fd": v, "adjoint_f64": float(g64[j]),
                                           "rel": float(abs(g64[j] - v) / abs(v))} for j, v in fd.items()},
        "adjoint_ms_f32": round(r32["forward_ms"] + r32["reverse_ms"], 2),
        "cost_per_step_vs_forward_step": round((r32["forward_ms"] + r32["reverse_ms"]) / steps / fwd_ms, 3),
        "device_bytes_f32": r32["device_bytes"]}
    return out


# -------------------------------------------------------- geometry setup ---
def write_stl_ascii(path, tris):
    with open(path, "w") as fh:
        fh.write("solid vessel\n")
        for t in tris:
            fh.write("facet normal %.17g %.17g %.17g\nouter loop\n" % tuple(t[9:12]))
            for v in range(3):
                fh.write("vertex %.17g %.17g %.17g\n" % tuple(t[3 * v:3 * v + 3]))
            fh.write("endloop\nendfacet\n")
        fh.write("endsolid vessel\n")


def write_reference_config(path, grid_size, length):
    """config.txt of the reference (LBM.h parser) for a tube along z with the
    inlet plane z = 0 and the outlet plane z = length."""
    lines = ["parameters:", "", '  stl_file: "geom.stl"', '  FlowType: "Constant"', "  time_resolution: 1e-05",
             "  density: 1060", "  kinematic_viscosity: 3.5e-6", "  relaxation_factor: 0.8",
             "  grid_size: %r" % grid_size, "  pressure: 1", "  CteVel: 0.05", "  reynolds_number: 100",
             "  number_of_outlets: 1", "  MaxIter: 1", "  IterToWrite: 1000000", "  Systole: 0.15",
             "  Diastole: 0.9", "  period: 0.9", "  NumCycle: 1", "", "",
             "inlets:", "", "    plane: z", "    coordinate: 0.0", "    normal: [0.0, 0.0, -1.0]", "", "",
             "outlets:", "", "    plane: z", "    coordinate: %r" % float(length), "    normal: [0.0, 0.0, 1.0]", "",
             "", "equations:", "    InletVel1: [0]", ""]
    with open(path, "w") as fh:
        fh.write("\n".join(lines))


def run_voxel(torch, device):
    """Geometry setup from an STL: the GPU pipeline (lbm_voxelise) against the
    reference's own Geometry + SubDomain construction (oracle/_ref/refharness,
    stl mode, setup only) on the R = 16 pipe STL, and the GPU pipeline alone on
    a triangulated radius-20 tortuous vessel (the reference needs hours)."""
    from lbm_b200 import geometry as G
    out = {}
    # R = 16, L = 128 pipe, 64 x 32 facets, grid_size 0.5 (spacing 1)
    tris = G.tube_triangles(lambda z: (0.37, 0.21), lambda z: 16.0, 0.0, 128.0, 64, 32)
    ops = [G.opening("inlet", "z", 0.0, (0, 0, -1)), G.opening("outlet", "z", 128.0, (0, 0, 1))]
    G.voxelise_stl(tris, 0.5, ops, device=device)  # warm-up (context, module load)
    wall = None
    for _ in range(3):  # best of three: the call is short, host jitter is not
        t0 = time.perf_counter()
        topo, (dims, origin, sp, ms) = G.voxelise_stl(tris, 0.5, ops, device=device, info=True)
        dt = time.perf_counter() - t0
        wall = dt if wall is None else min(wall, dt)
    pipe = {"triangles": len(tris), "grid_points": int(np.prod(dims)), "nodes": len(topo["kind"]),
            "near_wall_nodes": len(topo["nearwall"]), "gpu_seconds": round(wall, 4)}
    harness = os.path.join(ROOT, "oracle", "_ref", "refharness")
    if os.path.exists(harness):
        with tempfile.TemporaryDirectory() as tmp:
            write_stl_ascii(os.path.join(tmp, "geom.stl"), tris)
            write_reference_config(os.path.join(tmp, "config.txt"), 0.5, 128.0)
            r = subprocess.run([harness, "stl", os.path.join(tmp, "config.txt"), "0", os.path.join(tmp, "d.bin"),
                                "--time"], capture_output=True, text=True, timeout=1800)
            try:
                rep = json.loads(r.stdout.strip().splitlines()[-1])
                pipe["reference_setup_seconds"] = rep["setup_seconds"]
                pipe["reference_nodes"] = int(rep["nodes"])
                pipe["speedup"] = round(rep["setup_seconds"] / wall, 1)
            except (ValueError, IndexError, KeyError):
                pipe["reference_setup_seconds"] = None
    out["pipe16"] = pipe
    # radius-20 tortuous stenosed vessel as an STL: 128 x 1024 facets
    A, lam, R, Z = 30.0, 200.0, 20.0, 1024.0
    tris = G.tube_triangles(lambda z: (256.37 + A * math.sin(2 * math.pi * z / lam), 256.21),
                            lambda z: R * math.sqrt(1 - 0.5 * math.exp(-((z - Z / 2) ** 2) / (2 * (2 * R) ** 2))),
                            0.0, Z, 128, 1024)
    ops = [G.opening("inlet", "z", 0.0, (0, 0, -1)), G.opening("outlet", "z", Z, (0, 0, 1))]
    t0 = time.perf_counter()
    topo, (dims, origin, sp, ms) = G.voxelise_stl(tris, 0.5, ops, device=device, info=True)
    wall = time.perf_counter() - t0
    out["tortuous_R20"] = {"triangles": len(tris), "grid": list(dims), "grid_points": int(np.prod(dims)),
                           "nodes": len(topo["kind"]), "near_wall_nodes": len(topo["nearwall"]),
                           "gpu_seconds": round(wall, 3)}
    return out


# ------------------------------------------------------- the shipped case ---
JT_FIXTURE = os.path.join(ROOT, "tests", "golden", "jt_g0.2.npz")
JT_GRID = 0.025


def run_jt(torch, device, steps=200):
    """The reference's own case: JT.stl (its triangles, as the reference's
    reader reads them, and its config.txt opening blocks are kept in the
    JT test fixture) at the config's grid_size 0.025 (318 x 407 x 500 grid
    points, 64.7M). GPU voxelisation (wall clock, Python array handling
    included), then the config's tau 0.68 and constant inflow 0.1 through
    the engine: FP64 and FP32 storage with the reference's boundaries, FP32
    and FP16 with physics boundaries. The reference's setup labels every grid
    point against every facet: 27.7 s for the 136k points of grid_size 0.2
    on one core, so hours at 0.025; it is not timed here."""
    from lbm_b200 import Engine
    from lbm_b200 import geometry as G
    d = np.load(JT_FIXTURE)
    tris = d["triangles"]
    ops = json.loads(str(d["openings"]))
    tau, vel = 0.68, float(d["cte_vel"][0])
    G.voxelise_stl(tris, 0.2, ops, device=device)  # warm-up (context, module load)
    t0 = time.perf_counter()
    topo, (dims, origin, sp, ms) = G.voxelise_stl(tris, JT_GRID, ops, device=device, info=True)
    wall = time.perf_counter() - t0
    n = len(topo["kind"])
    outs = [len(topo["outlet_%d" % k]) for k in range(4) if "outlet_%d" % k in topo]
    out = {"workload": "JT.stl with its config.txt, grid_size %g" % JT_GRID, "grid": list(dims),
           "grid_points": int(np.prod(dims)), "nodes": n, "inlet_nodes": len(topo["inlet"]),
           "outlet_nodes": outs, "near_wall_nodes": len(topo["nearwall"]), "gpu_setup_seconds": round(wall, 3),
           "tau": tau, "inlet_velocity": vel, "steps": steps}
    for storage, bc in (("f64", "reference"), ("f32", "reference"), ("f32", "physics"), ("f16", "physics")):
        e = Engine(topo, tau=tau, dt=1e-5, spacing=sp, storage=storage, device=device, bc=bc, numeric_check=False)
        e.set_flow(False, vel)
        if bc == "physics":
            nrm = np.asarray(topo["inlet_normal"], float)
            e.set_inlet_profile(np.tile(-vel * nrm, (len(topo["inlet"]), 1)))
        e.set_observation(False)
        e.step(20)
        wall_ms, _, _ = timed_steps(e, steps, torch, device)
        out["%s_%s" % (bc, storage)] = {"MLUPS": round(n * steps / (wall_ms / 1e3) / 1e6, 1),
                                        "device_flags": e.flags()}
        e.close()
    return out


# ----------------------------------------------------------------- adjoint ---
ADJ_STEPS, ADJ_K, ADJ_TAU = 3000, 100, 0.6


def adjoint_workload():
    """Stenosed pipe: radius 24 lu in a 64 x 64 x 384 box, Gaussian stenosis
    narrowing the radius by 60 % at mid-length (sigma 12 lu); objective over
    the near-wall nodes within 12 lu of the throat; 8 Zernike-like inlet modes
    with seeded coefficients (mode 0 peak 0.012 lu)."""
    from lbm_b200 import geometry as G
    topo = G.straight_pipe(radius=24.0, length=384, box=(64, 64, 384), stenosis=0.6, stenosis_sigma=12.0)
    basis = G.zernike_inlet_basis(topo, 8)
    rng = np.random.default_rng(11)
    a = 0.0012 * rng.standard_normal(8)
    a[0] = 0.012
    targets = G.stenotic_throat_targets(topo, 12.0)
    return topo, basis, a, targets


def run_adjoint(torch, device, fd=True, steps=None, k=None):
    """Adjoint gradient of the throat's time-averaged WSS^2 w.r.t. 8 inlet
    coefficients and tau (3000 steps, checkpoint every 100): FP32 cost per
    step against the engine's FP32 forward step on the same pipe, and
    accuracy against an FP64 adjoint and central differences (h = 1e-4) of
    the FP64 objective."""
    from lbm_b200 import Engine
    T = steps or ADJ_STEPS
    K = k or ADJ_K
    topo, basis, a, targets = adjoint_workload()
    n = len(topo["kind"])

    def engine(tau, storage="f64"):
        e = Engine(topo, tau=tau, dt=1e-5, spacing=1.0, storage=storage, device=device, bc="physics")
        return e

    # the engine's own FP32 forward step on this geometry (inlet = the same modes)
    fw = engine(ADJ_TAU, "f32")
    fw.set_inlet_profile((a @ basis)[:, None] * -np.asarray(topo["inlet_normal"], dtype=np.float64)[None, :])
    fw.set_observation(False)
    fw.step(20)
    wall_ms, _, _ = timed_steps(fw, T, torch, device)
    fw.close()
    fwd_ms = wall_ms / T

    e = engine(ADJ_TAU)
    e.adjoint(50, targets, basis, a, checkpoint_every=10, precision="f32")   # warm-up
    r32 = e.adjoint(T, targets, basis, a, checkpoint_every=K, precision="f32")
    r64 = e.adjoint(T, targets, basis, a, checkpoint_every=K, precision="f64")
    g32 = np.append(r32["grad_coeffs"], r32["dJ_dtau"])
    g64 = np.append(r64["grad_coeffs"], r64["dJ_dtau"])
    total32 = r32["forward_ms"] + r32["reverse_ms"]
    out = {"workload": "stenosed pipe R=24 lu, 64x64x384 box, 60%% radius stenosis; %d fluid nodes, "
                       "%d throat near-wall nodes" % (n, len(targets)),
           "steps": T, "checkpoint_every": K, "tau": ADJ_TAU, "parameters": "8 inlet modes + tau",
           "J_f32": r32["J"], "J_f64": r64["J"],
           "engine_forward_step_ms_f32": round(fwd_ms, 5),
           "adjoint_ms_f32": {"forward_sweep": round(r32["forward_ms"], 2),
                              "recompute_and_reverse": round(r32["reverse_ms"], 2)},
           "steps_recomputed": r32["steps_recomputed"],
           "cost_per_step_vs_forward_step": round(total32 / T / fwd_ms, 3),
           "device_bytes_f32": r32["device_bytes"],
           "grad_f32_vs_f64_rel": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
           "grad_f64": g64.tolist()}
    if fd:
        h = 1e-4
        g_fd = np.zeros(9)
        for j in range(8):
            ap, am = a.copy(), a.copy()
            ap[j] += h
            am[j] -= h
            g_fd[j] = (e.adjoint(T, targets, basis, ap, gradient=False, precision="f64")["J"] -
                       e.adjoint(T, targets, basis, am, gradient=False, precision="f64")["J"]) / (2 * h)
        jt = []
        for t in (ADJ_TAU + h, ADJ_TAU - h):
            et = engine(t)
            jt.append(et.adjoint(T, targets, basis, a, gradient=False, precision="f64")["J"])
            et.close()
        g_fd[8] = (jt[0] - jt[1]) / (2 * h)
        out["fd_h"] = h
        out["grad_fd"] = g_fd.tolist()
        out["f64_vs_fd_rel"] = float(np.linalg.norm(g64 - g_fd) / np.linalg.norm(g_fd))
        out["f32_vs_fd_rel"] = float(np.linalg.norm(g32 - g_fd) / np.linalg.norm(g_fd))
        out["f64_vs_fd_rel_per_parameter"] = (np.abs(g64 - g_fd) / np.abs(g_fd)).round(8).tolist()
    e.close()
    return out


# ------------------------------------------------------------ reference arm ---
def write_nodemap(path, topo, zlo, zhi):
    """Node-map file of the slab zlo <= z < zhi for the reference harness
    (format documented in oracle/refharness/harness.cpp). The slab's last
    layer becomes its outlet."""
    c = topo["coords"]
    sel = (c[:, 2] >= zlo) & (c[:, 2] < zhi)
    cs = c[sel]
    kind = topo["kind"][sel].astype(np.int64)
    lo = cs.min(axis=0)
    hi = cs.max(axis=0)
    shape = hi - lo + 1
    cls = np.zeros(tuple(shape), np.uint8)
    code = np.array([1, 2, 4, 3])[kind]
    top = cs[:, 2] == hi[2]
    code[top & (kind != 1)] = 4
    loc = cs - lo
    cls[loc[:, 0], loc[:, 1], loc[:, 2]] = code
    nw = topo["nearwall"]
    nwc = c[nw]
    msel = (nwc[:, 2] >= zlo) & (nwc[:, 2] < zhi)
    with open(path, "wb") as fh:
        fh.write(b"NMAP")
        np.array([shape[0], shape[1], shape[2], 1], np.int32).tofile(fh)
        np.array([1.0, 0, 0, 0, 0, 0, -1.0, 0, 0, 1.0], np.float64).tofile(fh)
        cls.tofile(fh)
        np.array([int(msel.sum())], np.int64).tofile(fh)
        rec = np.zeros(int(msel.sum()), dtype=[("c", np.int32, 4), ("n", np.float64, 3)])
        rec["c"][:, :3] = nwc[msel] - lo
        rec["n"] = topo["nearwall_normal"][msel]
        rec.tofile(fh)
    return int(sel.sum())


def cpu_reference(args, sample_only=False, steps=None, procs=None):
    """Times the reference's own step loop on slabs of the workload, one
    harness process per core; returns MLUPS over all processes."""
    harness = os.path.join(ROOT, "oracle", "_ref", "refharness")
    if not os.path.exists(harness):
        return {"value": None, "unit": "MLUPS", "unavailable": "oracle/_ref/refharness not built"}
    topo, desc, radius = build_workload(args.workload)
    vel = inlet_velocity(radius)
    ncores = os.cpu_count() or 1
    procs = procs or (1 if sample_only else min(ncores, 32))
    steps = steps or (8 if sample_only else max(3, args.steps // 10))
    layers = 12
    work = tempfile.mkdtemp()
    cfg = os.path.join(work, "config.txt")
    with open(cfg, "w") as fh:
        fh.write("parameters:\n\n  FlowType: \"Constant\"\n  time_resolution: 1e-05\n"
                 "  relaxation_factor: %r\n  grid_size: 0.5\n  CteVel: %r\n  MaxIter: %d\n"
                 "  IterToWrite: 100000000\n\n" % (TAU, vel, steps))
    runs = []
    nodes_total = 0
    for p in range(procs):
        zlo = p * layers
        mp = os.path.join(work, "slab%d.bin" % p)
        nodes_total += write_nodemap(mp, topo, zlo, zlo + layers)
        runs.append(subprocess.Popen([harness, "nodemap", cfg, mp, str(steps), "-", "--time"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True))
    results = []
    for r in runs:
        out, _ = r.communicate()
        for line in out.splitlines():
            if line.startswith("{"):
                results.append(json.loads(line))
    if len(results) != procs:
        return {"value": None, "unit": "MLUPS", "unavailable": "reference harness failed"}
    # all processes run concurrently: aggregate = nodes / slowest wall time
    slowest = max(r["seconds"] for r in results)
    value = sum(r["nodes"] for r in results) * steps / slowest / 1e6
    return {"value": round(value, 4), "unit": "MLUPS", "cores": procs, "kind": "reference", **host_cpu(),
            "workload": desc, "inlet_velocity": round(vel, 6),
            "sample": "%d slab(s) of %d z-layers of the workload (%d nodes), %d steps each, "
                      "reference Simulation step methods, serial MPI build"
                      % (procs, layers, nodes_total, steps)}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    t0 = time.perf_counter()
    cpu = cpu_reference(args, sample_only=False)
    if cpu.get("value") is None:
        print(json.dumps({"impl": "reference", "unavailable": cpu.get("unavailable", "failed")}))
        return
    line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": "MLUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (analytic vessel geometry, f = w initial state)",
            "config": {"workload": cpu.get("workload"), "lattice": "D3Q19", "tau": TAU,
                       "inlet_velocity": cpu.get("inlet_velocity"), "reynolds": REYNOLDS},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_seconds": round(time.perf_counter() - t0, 1)}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    # warm-up of at least 200 steps before timing: the flow develops past the
    # start-up transient and the clocks settle
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="engine")
    ap.add_argument("--workload", default="tortuous8")
    ap.add_argument("--storage", default="f32")
    ap.add_argument("--bc", default="physics", choices=["physics", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    ap.add_argument("--no-voxel", action="store_true")
    ap.add_argument("--no-jt", action="store_true")
    ap.add_argument("--adjoint-steps", type=int, default=None,
                    help="--section adjoint: steps of the adjoint runs (default 3000)")
    ap.add_argument("--no-fd", action="store_true", help="--section adjoint: skip the central differences")
    ap.add_argument("--adjoint-k", type=int, default=None,
                    help="--section adjoint: checkpoint interval (default 100)")
    ap.add_argument("--section", default="all", choices=["all", "precision", "adjoint", "configs", "voxel", "jt"],
                    help="run only the precision study, the adjoint measurement or the branching/aneurysm runs")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.section != "all":
        import torch
        torch.cuda.set_device(0)
        run = {"precision": run_precision, "adjoint": run_adjoint, "configs": run_configs,
               "voxel": run_voxel, "jt": run_jt}[args.section]
        if args.section == "adjoint":
            res = run_adjoint(torch, 0, fd=not args.no_fd, steps=args.adjoint_steps, k=args.adjoint_k)
        else:
            res = run(torch, 0)
        print(json.dumps({"section": args.section, **res}))
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
