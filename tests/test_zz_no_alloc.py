"""lbm_flux_noalloc, the allocation-free flux entry point, against lbm_get_flux.

Callers that cannot allocate device memory (a framework owning all device
memory through its own pool, a process that may not allocate after start-up,
post-processing of populations in another program's buffers) get the FP64
inlet/outlet mass flux from populations and a node list they already hold on
the device; the block partial sums go to a fixed array inside the library.
This test allocates its own device buffers with torch (the test may; the entry
point may not), calls the entry point twice in a row on every boundary list
of a golden case and requires the engine's lbm_get_flux result each time, to
the 1e-12 relative tolerance the flux tests use. It also checks the limit."""
import ctypes
import os

import numpy as np
import pytest

from lbm_b200 import Engine, capi

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-12


def test_flux_noalloc_matches_engine_flux_twice():
    torch = pytest.importorskip("torch")
    d = np.load(os.path.join(GOLDEN, "outlet_chain.npz"))
    topo = {k: d[k] for k in d.files}
    meta = topo["meta_d"]
    e = Engine(topo, tau=meta[0], dt=meta[1], spacing=meta[2], storage="f64")
    e.set_flow(False, float(meta[4]))
    e.step(12)
    want_in, want_out = e.flux()
    f = torch.tensor(e.populations(), dtype=torch.float64, device="cuda")
    lists = [(topo["inlet"], topo["inlet_normal"], want_in)]
    lists += [(topo["outlet_%d" % k], topo["outlet_normal_%d" % k], want_out[k]) for k in range(len(want_out))]
    stream = torch.cuda.current_stream().cuda_stream
    L = capi.lib()
    for nodes_h, normal_h, want in lists:
        nodes = torch.tensor(np.asarray(nodes_h, dtype=np.int64), device="cuda")
        normal = (ctypes.c_double * 3)(*[float(x) for x in normal_h])
        for _ in range(2):
            out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
            rc = L.lbm_flux_noalloc(f.data_ptr(), f.shape[0], 19, nodes.data_ptr(), nodes.numel(), normal,
                                    out.data_ptr(), ctypes.c_void_p(stream))
            assert rc == capi.LBM_OK, L.lbm_last_error(None)
            torch.cuda.synchronize()
            got = float(out.item())
            assert abs(got - want) <= RTOL * max(1.0, abs(want)), (got, want)
    e.close()


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
