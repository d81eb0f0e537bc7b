"""lbm_flux_noalloc, the allocation-free flux entry point, against lbm_get_flux.

Callers that cannot allocate device memory (a framework owning all device
memory through its own pool, a process that may not allocate after start-up,
post-processing of populations in another program's buffers) get the FP64
inlet/outlet mass flux from populations and a node list they already hold on
the device; the block partial sums go to a fixed array inside the library.
These tests allocate their own device buffers with torch (a test may; the
entry point may not), call the entry point twice in a row on every boundary
list of a D3Q19 golden case and of a D3Q27 pipe, and require the engine's
lbm_get_flux result each time, to the 1e-12 relative tolerance the flux tests
use. They also check the limit, that list entries outside the node range add
nothing, and that repeated calls leave the device's free memory unchanged."""
import ctypes
import os

import numpy as np
import pytest

from lbm_b200 import Engine, capi
from lbm_b200 import geometry as G

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-12


def flux_noalloc(torch, f, q, nodes, normal_h):
    """One call through the C ABI; returns the flux (synchronised)."""
    normal = (ctypes.c_double * 3)(*[float(x) for x in normal_h])
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    L = capi.lib()
    rc = L.lbm_flux_noalloc(f.data_ptr(), f.shape[0], q, nodes.data_ptr() if nodes.numel() else None,
                            nodes.numel(), normal, out.data_ptr(), ctypes.c_void_p(stream))
    assert rc == capi.LBM_OK, L.lbm_last_error(None)
    torch.cuda.synchronize()
    return float(out.item())


def boundary_lists(topo, want_in, want_out):
    lists = [(topo["inlet"], topo["inlet_normal"], want_in)]
    lists += [(topo["outlet_%d" % k], topo["outlet_normal_%d" % k], want_out[k]) for k in range(len(want_out))]
    return lists


def check_twice(torch, e, topo, q):
    want_in, want_out = e.flux()
    f = torch.tensor(e.populations(), dtype=torch.float64, device="cuda")
    for nodes_h, normal_h, want in boundary_lists(topo, want_in, want_out):
        nodes = torch.tensor(np.asarray(nodes_h, dtype=np.int64), device="cuda")
        for _ in range(2):
            got = flux_noalloc(torch, f, q, nodes, normal_h)
            assert abs(got - want) <= RTOL * max(1.0, abs(want)), (got, want)


def test_flux_noalloc_matches_engine_flux_twice():
    torch = pytest.importorskip("torch")
    d = np.load(os.path.join(GOLDEN, "outlet_chain.npz"))
    topo = {k: d[k] for k in d.files}
    meta = topo["meta_d"]
    e = Engine(topo, tau=meta[0], dt=meta[1], spacing=meta[2], storage="f64")
    e.set_flow(False, float(meta[4]))
    e.step(12)
    check_twice(torch, e, topo, 19)
    e.close()


def test_flux_noalloc_d3q27_matches_engine_flux_twice():
    torch = pytest.importorskip("torch")
    topo = G.straight_pipe(radius=5.0, length=24)
    e = Engine(topo, tau=0.7, lattice=27, storage="f64", bc="physics")
    e.set_inlet_profile(G.parabolic_inlet(topo, 0.03))
    e.set_flow(False, 0.0)
    e.step(40)
    check_twice(torch, e, topo, 27)
    e.close()


def test_flux_noalloc_ignores_entries_outside_the_node_range():
    torch = pytest.importorskip("torch")
    d = np.load(os.path.join(GOLDEN, "outlet_chain.npz"))
    topo = {k: d[k] for k in d.files}
    meta = topo["meta_d"]
    e = Engine(topo, tau=meta[0], dt=meta[1], spacing=meta[2], storage="f64")
    e.set_flow(False, float(meta[4]))
    e.step(12)
    f = torch.tensor(e.populations(), dtype=torch.float64, device="cuda")
    n = f.shape[0]
    inlet = np.asarray(topo["inlet"], dtype=np.int64)
    want = flux_noalloc(torch, f, 19, torch.tensor(inlet, device="cuda"), topo["inlet_normal"])
    mixed = np.concatenate([[-1], inlet[: len(inlet) // 2], [n, n + 7, -5], inlet[len(inlet) // 2:], [n]])
    got = flux_noalloc(torch, f, 19, torch.tensor(mixed, device="cuda"), topo["inlet_normal"])
    assert abs(got - want) <= RTOL * max(1.0, abs(want)), (got, want)
    # an empty list (the start-up call) writes 0
    assert flux_noalloc(torch, f, 19, torch.zeros(0, dtype=torch.int64, device="cuda"), (0, 0, 1)) == 0.0
    e.close()


def test_flux_noalloc_calls_leave_free_memory_unchanged():
    torch = pytest.importorskip("torch")
    n, q = 200_000, 19
    f = torch.rand((n, q), dtype=torch.float64, device="cuda")
    nodes = torch.arange(0, n, 3, dtype=torch.int64, device="cuda")
    flux_noalloc(torch, f, q, nodes, (0.0, 0.6, 0.8))  # start-up call: loads the device code
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    vals = [flux_noalloc(torch, f, q, nodes, (0.0, 0.6, 0.8)) for _ in range(20)]
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert len(set(vals)) == 1


def test_flux_noalloc_rejects_lists_beyond_the_maximum():
    torch = pytest.importorskip("torch")
    f = torch.zeros((4, 19), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    normal = (ctypes.c_double * 3)(0.0, 0.0, 1.0)
    L = capi.lib()
    rc = L.lbm_flux_noalloc(f.data_ptr(), 4, 19, f.data_ptr(), capi.FLUX_NOALLOC_MAX_NODES + 1, normal,
                            out.data_ptr(), None)
    assert rc == capi.LBM_ERR_ARGUMENT
    assert b"exceeds the maximum" in L.lbm_last_error(None)
