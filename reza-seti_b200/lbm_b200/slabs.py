"""Slab decomposition of one lattice over several engines (physics mode).

The reference splits its box over MPI ranks with a Cartesian split and
one-cell halo layers (SubDomain, Subdomain.cpp:96-245) and, every step,
swaps whole halo faces with six MPI_Sendrecv calls (Simulation::Communicate,
Simulation.cpp:270-516). Here the node set is cut into slabs along one axis
(by default the longest), one engine per slab (one GPU per rank, or several
engines on one GPU), and only the populations that cross a cut move.

Each slab's engine holds its own nodes followed by ghost copies of the other
slabs' nodes that neighbour them (plain fluid nodes in no list: no inlet,
outlet or wall-shear work is done for them). For a pair of slabs A, B the
link set L_AB holds every (b, p) with b a node of A and b - c_p a node of B:
in the AA layout the store before a phase-1 step leaves in slot p of b the
population B's node pulls across the cut, and a phase-1 step leaves in B's
ghost copy of b, slot p, the population that crosses back. So after every
step (and once before the first one):

* next phase 1 (after the initialisation or a phase-0 step): A sends slot p
  of its own b for every (b, p) in L_AB, B writes them into its ghosts;
* next phase 0 (after a phase-1 step): B sends those slots of its ghosts
  back, A writes them into its own nodes.

Every other slot of a ghost is never read by an owned node, and whatever a
ghost's own step writes into an owned node's slot is overwritten by the
second exchange before it is read. Each node then sees exactly the values of
the undivided lattice, and the kernels do the same arithmetic per node, so a
slab run reproduces the single-engine run bit for bit.

A list's entries are sorted by (global node, direction) on both sides; list
2 j is the slab's own side of its j-th neighbour's link set, list 2 j + 1
its ghost side of the neighbour's link set towards it.
"""
from __future__ import annotations

import numpy as np

from .geometry import D3Q19, D3Q27


def lattice_vectors(q):
    if q == 19:
        return D3Q19
    if q == 27:
        return D3Q27
    raise ValueError("lattice must be 19 or 27")


def opposite(c):
    return np.array([int(np.nonzero((c == -v).all(axis=1))[0][0]) for v in c])


class NodeIndex:
    """Lookup of node indices by integer coordinates."""

    def __init__(self, coords):
        c = np.asarray(coords, dtype=np.int64).reshape(-1, 3)
        self.lo = c.min(axis=0) - 1
        self.ext = c.max(axis=0) - self.lo + 2
        keys = self._key(c)
        self.order = np.argsort(keys, kind="stable")
        self.sorted = keys[self.order]
        if len(self.sorted) > 1 and np.any(self.sorted[1:] == self.sorted[:-1]):
            raise ValueError("duplicate node coordinates")

    def _key(self, c):
        r = c - self.lo
        return (r[:, 0] * self.ext[1] + r[:, 1]) * self.ext[2] + r[:, 2]

    def find(self, c):
        """Node index at each coordinate row of c, -1 where there is none."""
        c = np.asarray(c, dtype=np.int64).reshape(-1, 3)
        inside = np.all((c > self.lo) & (c < self.lo + self.ext - 1), axis=1)
        out = np.full(len(c), -1, dtype=np.int64)
        if not inside.any():
            return out
        k = self._key(c[inside])
        pos = np.searchsorted(self.sorted, k)
        pos = np.minimum(pos, len(self.sorted) - 1)
        hit = self.sorted[pos] == k
        res = np.full(len(k), -1, dtype=np.int64)
        res[hit] = self.order[pos[hit]]
        out[inside] = res
        return out


def cut_planes(coords, n_slabs, axis):
    """Slab bounds along `axis`: n_slabs + 1 coordinates, slab r owning
    [b_r, b_{r+1}), placed at the node-count quantiles."""
    x = np.sort(np.asarray(coords, dtype=np.int64)[:, axis])
    lo, hi = int(x[0]), int(x[-1]) + 1
    if hi - lo < n_slabs:
        raise ValueError("fewer planes along the cut axis than slabs")
    bounds = [lo]
    for r in range(1, n_slabs):
        b = int(x[min(len(x) - 1, (r * len(x)) // n_slabs)])
        b = max(b, bounds[-1] + 1)
        b = min(b, hi - (n_slabs - r))
        bounds.append(b)
    bounds.append(hi)
    return np.array(bounds, dtype=np.int64)


class Slab:
    """One slab of a partition: its sub-topology (own nodes first, then the
    ghosts) and where its lists sit in the whole lattice's."""

    def __init__(self, rank, owned, ghosts, topo, neighbours, lists):
        self.rank = rank
        self.owned = owned              # global node indices, ascending
        self.ghosts = ghosts            # global node indices, ascending
        self.topo = topo                # the engine's topology
        self.neighbours = neighbours    # slab ranks, ascending
        self.lists = lists              # {list id: (local nodes, dirs, global nodes)}
        self.inlet_pos = topo.pop("_inlet_pos")        # entries of the whole inlet list
        self.nearwall_pos = topo.pop("_nearwall_pos")  # entries of the whole near-wall list
        self.outlet_pos = topo.pop("_outlet_pos")      # per outlet, entries of its list

    @property
    def n_owned(self):
        return len(self.owned)


def link_sets(topo, slab_of, q):
    """{(A, B): (b, p)} with b a node of slab A and b - c_p a node of slab B
    (b's neighbour across the cut in direction -c_p), sorted by (b, p)."""
    c = lattice_vectors(q)
    opp = opposite(c)
    coords = np.asarray(topo["coords"], dtype=np.int64)
    idx = NodeIndex(coords)
    sets = {}
    for p in range(len(c)):
        if not c[p].any():
            continue
        a = idx.find(coords + c[opp[p]])
        b = np.nonzero(a >= 0)[0]
        a = a[b]
        cross = slab_of[b] != slab_of[a]
        for bb, aa in zip(b[cross], a[cross]):
            sets.setdefault((int(slab_of[bb]), int(slab_of[aa])), []).append((int(bb), p))
    return {k: np.array(sorted(v), dtype=np.int64).reshape(-1, 2) for k, v in sets.items()}


def partition(topo, n_slabs, lattice=19, axis=None):
    """Cuts topo into n_slabs slabs along `axis` (default: the longest extent
    of the node set). Returns the list of Slab objects."""
    from .engine import outlets_of
    coords = np.asarray(topo["coords"], dtype=np.int64).reshape(-1, 3)
    kind = np.asarray(topo["kind"], dtype=np.uint8)
    n = len(kind)
    if axis is None:
        axis = int(np.argmax(coords.max(axis=0) - coords.min(axis=0)))
    bounds = cut_planes(coords, n_slabs, axis)
    slab_of = np.searchsorted(bounds, coords[:, axis], side="right") - 1
    sets = link_sets(topo, slab_of, lattice)
    inlet = np.asarray(topo["inlet"], dtype=np.int64)
    nearwall = np.asarray(topo.get("nearwall", np.zeros(0)), dtype=np.int64)
    nw_normal = np.asarray(topo.get("nearwall_normal", np.zeros((0, 3))), dtype=np.float64).reshape(-1, 3)
    wall = np.asarray(topo.get("wall", np.zeros(0)), dtype=np.int64)
    outs, out_normals = outlets_of(topo)
    slabs = []
    for r in range(n_slabs):
        owned = np.nonzero(slab_of == r)[0]
        if len(owned) == 0:
            raise ValueError("slab %d holds no node" % r)
        # ghosts: the other slabs' nodes of every link set towards r
        g = [v[:, 0] for (A, B), v in sets.items() if B == r]
        ghosts = np.unique(np.concatenate(g)) if g else np.zeros(0, dtype=np.int64)
        local = np.full(n, -1, dtype=np.int64)
        local[owned] = np.arange(len(owned))
        local[ghosts] = len(owned) + np.arange(len(ghosts))
        nodes = np.concatenate([owned, ghosts])
        gk = kind[ghosts].copy()
        gk[(gk == 1) | (gk == 2)] = 0   # a ghost does no inlet or outlet work
        sub = {"coords": coords[nodes].astype(np.int32), "kind": np.concatenate([kind[owned], gk])}
        sel = np.nonzero(slab_of[inlet] == r)[0]
        sub["inlet"], sub["_inlet_pos"] = local[inlet[sel]], sel
        sub["inlet_normal"] = np.asarray(topo.get("inlet_normal", np.zeros(3)), dtype=np.float64)
        sub["_outlet_pos"] = []
        for k, (o, nrm) in enumerate(zip(outs, out_normals)):
            sel = np.nonzero(slab_of[o] == r)[0]
            sub["outlet_%d" % k], sub["outlet_normal_%d" % k] = local[o[sel]], nrm
            sub["_outlet_pos"].append(sel)
        sub["wall"] = local[wall[slab_of[wall] == r]]
        sel = np.nonzero(slab_of[nearwall] == r)[0]
        sub["nearwall"], sub["nearwall_normal"], sub["_nearwall_pos"] = local[nearwall[sel]], nw_normal[sel], sel
        neighbours = sorted({B for (A, B) in sets if A == r} | {A for (A, B) in sets if B == r})
        lists = {}
        for j, B in enumerate(neighbours):
            own = sets.get((r, B), np.zeros((0, 2), dtype=np.int64))
            ghost = sets.get((B, r), np.zeros((0, 2), dtype=np.int64))
            lists[2 * j] = (local[own[:, 0]], own[:, 1].astype(np.int32), own[:, 0])
            lists[2 * j + 1] = (local[ghost[:, 0]], ghost[:, 1].astype(np.int32), ghost[:, 0])
        slabs.append(Slab(r, owned, ghosts, sub, neighbours, lists))
    return slabs


TORCH_DTYPE = {"f64": "float64", "f32": "float32", "f16": "float16", "bf16": "bfloat16"}


def _exchange_plan(slab, next_phase):
    """(pack list, unpack list) per neighbour j for the exchange that
    precedes a step of phase next_phase."""
    if next_phase == 1:
        return [(2 * j, 2 * j + 1) for j in range(len(slab.neighbours))]
    return [(2 * j + 1, 2 * j) for j in range(len(slab.neighbours))]


class SlabSet:
    """All slabs of a partition as engines in one process (one GPU), stepped
    in lockstep on one stream, the halo values copied between their device
    buffers. Reproduces the undivided lattice's run."""

    def __init__(self, topo, n_slabs, *, lattice=19, axis=None, storage="f32", device=0, **engine_kw):
        import torch
        from .engine import Engine
        self.torch = torch
        self.n = len(topo["kind"])
        self.q = lattice
        self.n_nearwall = len(topo.get("nearwall", []))
        self.n_inlet = len(topo["inlet"])
        self.slabs = partition(topo, n_slabs, lattice=lattice, axis=axis)
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.current_stream(self.dev)
        self.engines = []
        for s in self.slabs:
            e = Engine(s.topo, lattice=lattice, storage=storage, bc="physics", device=device, **engine_kw)
            e.set_stream(self.stream.cuda_stream)
            for lid, (nodes, dirs, _) in s.lists.items():
                e.halo_define(lid, nodes, dirs)
            self.engines.append(e)
        dt = getattr(torch, TORCH_DTYPE[storage])
        # one buffer per link set (A, B), A < B, shared by both directions
        self.buf = {}
        for s in self.slabs:
            for j, B in enumerate(s.neighbours):
                key = (min(s.rank, B), max(s.rank, B))
                if key not in self.buf:
                    # |L_AB| = |L_BA|: (b, p) <-> (b - c_p, opp p)
                    n_ab = len(s.lists[2 * j][0])
                    self.buf[key] = {s.rank: torch.empty(max(n_ab, 1), dtype=dt, device=self.dev),
                                     B: torch.empty(max(n_ab, 1), dtype=dt, device=self.dev)}
        self._synced = False

    def close(self):
        for e in self.engines:
            e.close()
        self.engines = []

    def _apply(self, name, *args, **kw):
        for e in self.engines:
            getattr(e, name)(*args, **kw)
        self._synced = False

    # setters that re-initialise a fresh engine's store: the halo is
    # exchanged again before the next step
    def set_flow(self, *a, **k):
        self._apply("set_flow", *a, **k)

    def set_waveform(self, *a, **k):
        self._apply("set_waveform", *a, **k)

    def set_outlet_density(self, *a, **k):
        self._apply("set_outlet_density", *a, **k)

    def set_observation(self, *a, **k):
        for e in self.engines:
            e.set_observation(*a, **k)

    def set_inlet_profile(self, vel):
        v = np.asarray(vel, dtype=np.float64).reshape(self.n_inlet, 3)
        for s, e in zip(self.slabs, self.engines):
            if e.n_inlet:
                e.set_inlet_profile(v[s.inlet_pos])
        self._synced = False

    def exchange(self):
        """The halo exchange due before the next step (by the engines' phase)."""
        phase = self.engines[0].next_phase()
        # every link set's values are read before any is written
        for s, e in zip(self.slabs, self.engines):
            for j, (pk, _) in enumerate(_exchange_plan(s, phase)):
                B = s.neighbours[j]
                e.halo_pack(pk, self.buf[(min(s.rank, B), max(s.rank, B))][s.rank].data_ptr())
        for s, e in zip(self.slabs, self.engines):
            for j, (_, up) in enumerate(_exchange_plan(s, phase)):
                B = s.neighbours[j]
                e.halo_unpack(up, self.buf[(min(s.rank, B), max(s.rank, B))][B].data_ptr())
        self._synced = True

    def step(self, n=1):
        for _ in range(int(n)):
            if not self._synced:
                self.exchange()
            for e in self.engines:
                e.step(1)
            self.exchange()

    # ---- checkpoint and resume
    def save_checkpoint(self, path):
        """Writes every slab engine's state to one checkpoint file."""
        from . import checkpoint
        checkpoint.write(path, *checkpoint.slab_set_state(self))

    def load_checkpoint(self, path):
        """Restores a checkpoint of a slab set cut the same way, after the flow
        settings. The halo exchange runs again before the next step. It copies
        the values the checkpointed set had already exchanged, so the steps
        continue bit for bit."""
        from . import checkpoint
        checkpoint.restore_slab_set(self, checkpoint.read(path))
        self._synced = False

    # ---- results in the whole lattice's order
    def populations(self):
        f = np.empty((self.n, self.q))
        for s, e in zip(self.slabs, self.engines):
            f[s.owned] = e.populations()[:s.n_owned]
        return f

    def macros(self):
        rho, u = np.empty(self.n), np.empty((self.n, 3))
        for s, e in zip(self.slabs, self.engines):
            r, v = e.macros()
            rho[s.owned], u[s.owned] = r[:s.n_owned], v[:s.n_owned]
        return rho, u

    def wss(self):
        w, acc, accm = np.empty(self.n_nearwall), np.empty((self.n_nearwall, 3)), np.empty(self.n_nearwall)
        for s, e in zip(self.slabs, self.engines):
            a, b, c = e.wss()
            w[s.nearwall_pos], acc[s.nearwall_pos], accm[s.nearwall_pos] = a, b.reshape(-1, 3), c
        return w, acc, accm

    def osi_tawss(self):
        osi, tawss = np.empty(self.n_nearwall), np.empty(self.n_nearwall)
        for s, e in zip(self.slabs, self.engines):
            o, t = e.osi_tawss()
            osi[s.nearwall_pos], tawss[s.nearwall_pos] = o, t
        return osi, tawss

    def flux(self):
        """Inlet and outlet mass fluxes: the slabs' partial sums added."""
        inl, outs = 0.0, None
        for e in self.engines:
            a, b = e.flux()
            inl += a
            outs = np.asarray(b, dtype=np.float64) if outs is None else outs + np.asarray(b)
        return inl, outs

    def flags(self):
        f = 0
        for e in self.engines:
            f |= e.flags()
        return f


class SlabRank:
    """One slab per process (one GPU per rank), its halo moved with
    torch.distributed point-to-point calls (NCCL on GPUs: the engine runs on
    torch's current stream, so the packs are ordered before the sends and the
    unpacks after the receives). `engine` is the slab's engine, or any object
    with the same halo_* / next_phase / step methods."""

    def __init__(self, slab, engine, *, device, dtype, group=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.slab, self.engine, self.group = slab, engine, group
        for lid, (nodes, dirs, _) in slab.lists.items():
            engine.halo_define(lid, nodes, dirs)
        self.send, self.recv = [], []
        for j in range(len(slab.neighbours)):
            n_ab = max(len(slab.lists[2 * j][0]), 1)
            self.send.append(torch.empty(n_ab, dtype=dtype, device=device))
            self.recv.append(torch.empty(n_ab, dtype=dtype, device=device))
        self._synced = False

    def _peer(self, B):
        # slab ranks are group ranks; point-to-point calls take global ranks
        if self.group is None:
            return B
        return self.dist.get_global_rank(self.group, B)

    def exchange(self):
        phase = self.engine.next_phase()
        plan = _exchange_plan(self.slab, phase)
        ops = []
        for j, (pk, _) in enumerate(plan):
            self.engine.halo_pack(pk, self.send[j].data_ptr())
            B = self._peer(self.slab.neighbours[j])
            ops.append(self.dist.P2POp(self.dist.isend, self.send[j], B, self.group))
            ops.append(self.dist.P2POp(self.dist.irecv, self.recv[j], B, self.group))
        if ops:
            if self.dist.get_backend(self.group) == "nccl":
                works = self.dist.batch_isend_irecv(ops)
            else:
                works = [op.op(op.tensor, op.peer, op.group) for op in ops]
            for w in works:
                w.wait()
        for j, (_, up) in enumerate(plan):
            self.engine.halo_unpack(up, self.recv[j].data_ptr())
        self._synced = True

    def mark_stale(self):
        """After a setter that re-initialised the engine's store."""
        self._synced = False

    def checkpoint_path(self, path):
        """This rank's file of a checkpoint written by every rank."""
        return "%s.slab%d" % (path, self.slab.rank)

    def save_checkpoint(self, path):
        """Every rank writes its engine's state to checkpoint_path(path)."""
        self.engine.save_checkpoint(self.checkpoint_path(path))

    def load_checkpoint(self, path):
        """Every rank restores its engine from checkpoint_path(path); the halo
        exchange runs again before the next step (it copies what the
        checkpointed ranks had already exchanged)."""
        self.engine.load_checkpoint(self.checkpoint_path(path))
        self._synced = False

    def step(self, n=1):
        for _ in range(int(n)):
            if not self._synced:
                self.exchange()
            self.engine.step(1)
            self.exchange()


def slab_rank(topo, n_slabs, rank, *, lattice=19, axis=None, storage="f32", device=0, group=None, **engine_kw):
    """This process's slab of topo (rank `rank` of n_slabs) with its engine on
    cuda:device, ready to step with SlabRank.step."""
    import torch
    from .engine import Engine
    slab = partition(topo, n_slabs, lattice=lattice, axis=axis)[rank]
    e = Engine(slab.topo, lattice=lattice, storage=storage, bc="physics", device=device, **engine_kw)
    e.set_stream(torch.cuda.current_stream(torch.device("cuda", device)).cuda_stream)
    return SlabRank(slab, e, device=torch.device("cuda", device), dtype=getattr(torch, TORCH_DTYPE[storage]),
                    group=group)
