"""Slab decomposition (lbm_b200/slabs.py), host side, on the CPU.

The partition and its halo lists are checked structurally, then on an
emulation of the engine's AA-pattern store rules in numpy: every node, ghosts
included, runs the same per-node update (phase 0: its own slots, written to
the opposite slots; phase 1: pulled from the neighbours' slots or its own
bounce-back slot, pushed to the neighbours' slots or bounced back), with a
nonlinear update that depends on the node's coordinates. A slab run with the
halo exchange after every step must give every owned node exactly the slots
of the undivided run: in one process, and over two gloo ranks through
SlabRank (the code path the multi-GPU run takes, NCCL there)."""
import ctypes
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from lbm_b200 import geometry as G
from lbm_b200 import slabs as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def small_pipe():
    return G.straight_pipe(radius=5.0, length=24, stenosis=0.3, stenosis_sigma=3.0)


class AAEmulator:
    """The engine's store rules on a node set (float64 slots [Q][n])."""

    def __init__(self, coords, q, seed=3):
        self.c = S.lattice_vectors(q)
        self.opp = S.opposite(self.c)
        self.q = q
        self.coords = np.asarray(coords, dtype=np.int64)
        idx = S.NodeIndex(self.coords)
        self.nb = np.stack([idx.find(self.coords + v) for v in self.c], axis=1)  # [n][q], -1: none
        rng = np.random.default_rng(seed)
        key = (self.coords * np.array([7, 13, 17])).sum(axis=1) % 97
        self.f = 0.01 * (np.sin(key[None, :] * (1 + np.arange(q))[:, None]) + 0.1 * rng.standard_normal((1, 1)))
        self.key = key / 97.0
        self.phase = 1  # the initial store has been made
        self.halo = {}

    def update(self, s):
        # nonlinear, per node: the same function for the node wherever it sits
        tot = s.sum(axis=0)
        return 0.7 * s + 0.3 * np.tanh(tot)[None, :] * (0.5 + self.key)[None, :] * (1 + np.arange(self.q))[:, None] / self.q

    def step(self, n=1):
        for _ in range(n):
            q, f, nb, opp = self.q, self.f, self.nb, self.opp
            nodes = np.arange(f.shape[1])
            if self.phase == 0:
                s = f.copy()
                c = self.update(s)
                for p in range(q):
                    f[opp[p]] = c[p]
            else:
                s = np.empty_like(f)
                for p in range(q):
                    o = opp[p]
                    have = nb[:, o] >= 0
                    s[p] = np.where(have, f[o, np.where(have, nb[:, o], 0)], f[p])
                c = self.update(s)
                for p in range(q):
                    have = nb[:, p] >= 0
                    f[p, nb[have, p]] = c[p, have]
                    f[opp[p], nodes[~have]] = c[p, ~have]
            self.phase ^= 1

    # the engine's checkpoint interface (its whole state: slots and phase)
    def save_checkpoint(self, path):
        with open(path, "wb") as fh:
            np.savez(fh, f=self.f, phase=self.phase)

    def load_checkpoint(self, path):
        with np.load(path) as d:
            self.f = d["f"].copy()
            self.phase = int(d["phase"])

    # the engine's halo interface
    def next_phase(self):
        return self.phase

    def halo_define(self, lid, nodes, dirs):
        self.halo[lid] = (np.asarray(nodes), np.asarray(dirs))

    def halo_pack(self, lid, ptr):
        nodes, dirs = self.halo[lid]
        out = np.ctypeslib.as_array((ctypes.c_double * max(len(nodes), 1)).from_address(ptr))
        out[:len(nodes)] = self.f[dirs, nodes]

    def halo_unpack(self, lid, ptr):
        nodes, dirs = self.halo[lid]
        src = np.ctypeslib.as_array((ctypes.c_double * max(len(nodes), 1)).from_address(ptr))
        self.f[dirs, nodes] = src[:len(nodes)]


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("n_slabs,axis", [(2, None), (3, 2), (3, 0)])
def test_partition_structure(q, n_slabs, axis):
    topo = small_pipe()
    n = len(topo["kind"])
    sl = S.partition(topo, n_slabs, lattice=q, axis=axis)
    owned = np.concatenate([s.owned for s in sl])
    assert np.array_equal(np.sort(owned), np.arange(n))
    c = S.lattice_vectors(q)
    idx = S.NodeIndex(topo["coords"])
    for s in sl:
        # ghosts: exactly the other slabs' neighbours of the slab's nodes
        nbs = np.unique(np.concatenate([idx.find(topo["coords"][s.owned] + v) for v in c]))
        nbs = nbs[nbs >= 0]
        assert np.array_equal(np.setdiff1d(nbs, s.owned), s.ghosts)
        assert len(s.topo["kind"]) == s.n_owned + len(s.ghosts)
        assert set(np.unique(s.topo["kind"][s.n_owned:])) <= {0, 3}
        # list j of this slab pairs with the neighbour's list for this slab
        for j, B in enumerate(s.neighbours):
            t = sl[B]
            jb = t.neighbours.index(s.rank)
            own, ghost = s.lists[2 * j], t.lists[2 * jb + 1]
            assert np.array_equal(own[2], ghost[2]) and np.array_equal(own[1], ghost[1])
            assert len(s.lists[2 * j][0]) == len(s.lists[2 * j + 1][0])
    # every inlet, outlet and near-wall entry lands in exactly one slab
    assert sorted(np.concatenate([s.inlet_pos for s in sl]).tolist()) == list(range(len(topo["inlet"])))
    assert sorted(np.concatenate([s.nearwall_pos for s in sl]).tolist()) == list(range(len(topo["nearwall"])))


def run_in_process(topo, q, n_slabs, axis, steps):
    full = AAEmulator(topo["coords"], q)
    sl = S.partition(topo, n_slabs, lattice=q, axis=axis)
    parts = [AAEmulator(s.topo["coords"], q) for s in sl]
    bufs = {}

    def exchange():
        phase = parts[0].next_phase()
        for s, e in zip(sl, parts):
            for j, (pk, _) in enumerate(S._exchange_plan(s, phase)):
                b = np.zeros(max(len(s.lists[pk][0]), 1))
                bufs[(s.rank, s.neighbours[j])] = b
                e.halo_pack(pk, b.ctypes.data)
        for s, e in zip(sl, parts):
            for j, (_, up) in enumerate(S._exchange_plan(s, phase)):
                e.halo_unpack(up, bufs[(s.neighbours[j], s.rank)].ctypes.data)

    for s, e in zip(sl, parts):
        for lid, (nodes, dirs, _) in s.lists.items():
            e.halo_define(lid, nodes, dirs)
    exchange()
    for _ in range(steps):
        full.step()
        for e in parts:
            e.step()
        exchange()
    return full, sl, parts


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("n_slabs,axis", [(2, None), (3, 2), (4, 0)])
def test_slab_run_equals_whole_lattice(q, n_slabs, axis):
    topo = small_pipe()
    full, sl, parts = run_in_process(topo, q, n_slabs, axis, steps=7)
    for s, e in zip(sl, parts):
        np.testing.assert_array_equal(e.f[:, :s.n_owned], full.f[:, s.owned])


def test_without_exchange_the_slabs_diverge():
    """The check above has teeth: skipping the exchanges changes owned slots."""
    topo = small_pipe()
    full = AAEmulator(topo["coords"], 19)
    sl = S.partition(topo, 2, lattice=19)
    parts = [AAEmulator(s.topo["coords"], 19) for s in sl]
    for _ in range(3):
        full.step()
        for e in parts:
            e.step()
    assert any(not np.array_equal(e.f[:, :s.n_owned], full.f[:, s.owned]) for s, e in zip(sl, parts))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "reza-seti_b200"))
    import datetime
    import torch
    import torch.distributed as dist
    from lbm_b200 import slabs as SS
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        topo = small_pipe()
        slab = SS.partition(topo, world, lattice=19)[rank]
        emu = AAEmulator(slab.topo["coords"], 19)
        r = SS.SlabRank(slab, emu, device="cpu", dtype=torch.float64)
        r.step(5)
        out.put((rank, slab.owned, emu.f[:, :slab.n_owned].copy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def rank_resume_main(rank, world, port, out, ckdir):
    """5 steps, a checkpoint, then a new rank object with a fresh engine
    restores it and takes 4 more steps."""
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "reza-seti_b200"))
    import datetime
    import torch
    import torch.distributed as dist
    from lbm_b200 import slabs as SS
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        topo = small_pipe()
        slab = SS.partition(topo, world, lattice=19)[rank]
        r = SS.SlabRank(slab, AAEmulator(slab.topo["coords"], 19), device="cpu", dtype=torch.float64)
        r.step(5)
        path = os.path.join(ckdir, "run")
        r.save_checkpoint(path)
        emu = AAEmulator(slab.topo["coords"], 19, seed=11)  # another initial state
        r2 = SS.SlabRank(slab, emu, device="cpu", dtype=torch.float64)
        r2.load_checkpoint(path)
        r2.step(4)
        out.put((rank, slab.owned, emu.f[:, :slab.n_owned].copy(), os.path.exists(r.checkpoint_path(path))))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_resume_from_checkpoint(tmp_path):
    """Each rank restores its own checkpoint file into a fresh engine; the
    exchange that SlabRank runs again before the next step makes the resumed
    run equal the undivided lattice's 9 steps."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_resume_main, args=(r, 2, port, q, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    topo = small_pipe()
    full = AAEmulator(topo["coords"], 19)
    full.step(9)
    for rank, owned, f, wrote in got:
        assert wrote
        np.testing.assert_array_equal(f, full.f[:, owned])
    assert sorted(os.listdir(tmp_path)) == ["run.slab0", "run.slab1"]


def test_two_gloo_ranks_equal_whole_lattice():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    topo = small_pipe()
    full = AAEmulator(topo["coords"], 19)
    full.step(5)
    for rank, owned, f in got:
        np.testing.assert_array_equal(f, full.f[:, owned])
