"""Pins the oracle restatement to the reference solver's own output.

Every golden fixture was produced by the reference sources themselves
(tests/golden/make_golden.py runs oracle/_ref/refharness). The oracle replays
each case phase by phase and must agree bit for bit: same populations after
collision, streaming, inlet, outlet and wall phases of step 1, same WSS, and
the same state after the last step.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as orc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SMALL = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if not os.path.basename(p).startswith(("pipe16", "jt_")))


def load(path):
    d = np.load(path)
    return {k: d[k] for k in d.files}


def same(a, b, what):
    np.testing.assert_array_equal(np.asarray(a), np.asarray(b), err_msg=what)


def check_state(o, d, tag, nearwall=True):
    same(o.f, d[tag + "__f"], tag + " f")
    same(o.fnew, d[tag + "__fnew"], tag + " fnew")
    same(o.feq, d[tag + "__feq"], tag + " feq")
    same(o.rho, d[tag + "__rho"], tag + " rho")
    same(o.u, d[tag + "__u"], tag + " u")
    same(o.velmag, d[tag + "__velmag"], tag + " velmag")
    if nearwall:
        same(o.wss, d[tag + "__wss"], tag + " wss")
        same(o.acc, d[tag + "__acc"], tag + " acc")
        same(o.accmag, d[tag + "__accmag"], tag + " accmag")


def test_lattice_tables():
    c, w, opp = orc.directions(), orc.weights(), orc.opposite()
    assert c.shape == (19, 3)
    assert abs(w.sum() - 1.0) < 1e-15
    assert (c[opp] == -c).all()
    assert (c[18] == 0).all()


@pytest.mark.parametrize("path", SMALL, ids=[os.path.basename(p)[:-4] for p in SMALL])
def test_oracle_matches_reference_bitwise(path):
    d = load(path)
    pulsatile = bool(d["meta_i"][7])
    steps_total = None
    o = orc.Oracle(d)
    cte = float(d["meta_d"][4])
    assert abs(o.wss_constant - d["meta_d"][3]) == 0.0

    # step 1, phase by phase
    o.collide()
    check_state(o, d, "p1_collide", nearwall=False)
    o.stream()
    check_state(o, d, "p1_stream", nearwall=False)
    vel = orc.pulsatile_velocity(o.runtime.value) if pulsatile else cte
    same(vel, d["p1_inlet__inletvel"][0], "inlet velocity")
    o.inlet_bc(vel)
    check_state(o, d, "p1_inlet", nearwall=False)
    o.outlet_bc()
    check_state(o, d, "p1_outlet", nearwall=False)
    o.wall_bc()
    check_state(o, d, "p1_wall", nearwall=False)
    o.wall_shear_stress()
    if pulsatile:
        o.osi_tawss()
        o.runtime.value += o.dt
    check_state(o, d, "p1_wss")

    # remaining steps of the case
    steps_total = {"cyl_z": 60, "cyl_z_rev": 20, "cyl_x": 40, "cyl_x_rev": 20, "cyl_y": 4,
                   "cyl_y_rev": 4, "cyl_z_pulsatile": 100, "outlet_chain": 12}[
        os.path.basename(path)[:-4]]
    o.run(steps_total - 1, pulsatile=pulsatile, cte_vel=cte)
    check_state(o, d, "final")
    if pulsatile:
        same(o.osi, d["final__osi"], "osi")
        same(o.tawss, d["final__tawss"], "tawss")


def test_pulsatile_step_count_matches_loop_rule():
    # Iterate runs while total_runtime <= 2.7 (Simulation.cpp:549-550)
    for dt in (1e-3, 3e-3, 1e-5 * 7):
        t, n = 0.0, 0
        while t <= 2.7:
            t += dt
            n += 1
        assert orc.pulsatile_step_count(dt) == n


def test_oracle_matches_reference_pipe_2000_steps():
    """The R=16, L=128 pipe on the reference grid (102,555 nodes), 2000 steps:
    sampled populations and moments, every near-wall WSS value and the
    whole-field checksums equal the reference's."""
    d = load(os.path.join(GOLDEN, "pipe16_2000.npz"))
    o = orc.Oracle(d)
    o.run(2000, cte_vel=float(d["meta_d"][4]))
    s = d["sample"]
    same(o.f[s], d["final__f_sample"], "f sample")
    same(o.rho[s], d["final__rho_sample"], "rho sample")
    same(o.u[s], d["final__u_sample"], "u sample")
    same(o.wss, d["final__wss"], "wss")
    same(o.acc, d["final__acc"], "acc")
    same(o.accmag, d["final__accmag"], "accmag")
    for k, a in (("f", o.f), ("rho", o.rho), ("u", o.u), ("feq", o.feq)):
        same(np.array([a.sum(), np.abs(a).sum(), (a * a).sum()]), d["final__%s_sum" % k], k + " sums")


def test_oracle_matches_reference_jt_50_steps():
    """The reference's shipped case (JT.stl, its config.txt at grid_size 0.2:
    12,929 nodes, one inlet, four outlet blocks of which one meets the grid),
    50 steps: sampled populations and moments, every WSS value and the
    whole-field checksums equal the reference's."""
    d = load(os.path.join(GOLDEN, "jt_g0.2.npz"))
    o = orc.Oracle(d)
    o.run(int(d["steps"][0]), cte_vel=float(d["cte_vel"][0]))
    s = d["sample"]
    same(o.f[s], d["final__f_sample"], "f sample")
    same(o.rho[s], d["final__rho_sample"], "rho sample")
    same(o.u[s], d["final__u_sample"], "u sample")
    same(o.wss, d["final__wss"], "wss")
    same(o.acc, d["final__acc"], "acc")
    same(o.accmag, d["final__accmag"], "accmag")
    for k, a in (("f", o.f), ("rho", o.rho), ("u", o.u), ("feq", o.feq)):
        same(np.array([a.sum(), np.abs(a).sum(), (a * a).sum()]), d["final__%s_sum" % k], k + " sums")
