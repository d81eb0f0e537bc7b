"""NumPy restatement of the engine's physics boundary mode — TEST INFRASTRUCTURE.

The reference solver has no such mode (its rules are restated in the oracle);
physics mode is defined by the engine: BGK collision, streaming with halfway
bounce-back for every link whose far node is missing, a velocity correction on
inlet links that point out through the inlet plane, and anti-bounce-back at
the outlet density on outlet links that point out through an outlet plane:

  f_new[n][q] = C[m][q]                                        m = n - c_q exists
  f_new[n][q] = C[n][p] + 6 w_p (c_p . u_w) ... with p = opp q:
      C[n][p]                                   (wall)
      C[n][p] - 6 w_p (c_p . u_in(n))           (inlet node, c_p . n_in > 0)
      -C[n][p] + 2 w_p rho_out (1 + 4.5 (c_p . u_n)^2 - 1.5 |u_n|^2)
                                                 (outlet node, c_p . n_out > 0)

with C the post-collision populations and u_n the node's collision velocity.
Populations are f (not shifted), FP64, dense over the node list.
"""
from __future__ import annotations

import numpy as np

# D3Q19 in the reference's order (LatticeModel.cpp:92-192)
C19 = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0],
                [1, -1, 0], [1, 0, 1], [1, 0, -1], [-1, 1, 0], [-1, -1, 0], [-1, 0, 1],
                [-1, 0, -1], [0, 1, 1], [0, 1, -1], [0, -1, 1], [0, -1, -1], [0, 0, 0]])
W19 = np.array([2.0 / 36.0] * 6 + [1.0 / 36.0] * 12 + [12.0 / 36.0])
# D3Q27 in the reference's order (LatticeModel.cpp:249-375)
C27 = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                [1, 1, 0], [1, -1, 0], [-1, 1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
                [-1, 0, -1], [0, 1, 1], [0, 1, -1], [0, -1, 1], [0, -1, -1], [1, 1, 1],
                [-1, -1, -1], [1, 1, -1], [-1, -1, 1], [1, -1, 1], [-1, 1, -1], [1, -1, -1],
                [-1, 1, 1]])
W27 = np.array([8.0 / 27.0] + [2.0 / 27.0] * 6 + [1.0 / 54.0] * 12 + [1.0 / 216.0] * 8)


def lattice(q):
    c, w = (C19, W19) if q == 19 else (C27, W27)
    opp = np.array([int(np.nonzero((c == -v).all(axis=1))[0][0]) for v in c])
    return c, w, opp


def neighbour_table(coords, c):
    coords = np.asarray(coords, dtype=np.int64)
    lo = coords.min(axis=0) - 1
    shape = tuple(coords.max(axis=0) - lo + 2)
    grid = -np.ones(shape, dtype=np.int64)
    x = coords - lo
    grid[x[:, 0], x[:, 1], x[:, 2]] = np.arange(len(coords))
    nb = np.empty((len(coords), len(c)), dtype=np.int64)
    for q, d in enumerate(c):
        t = x + d
        nb[:, q] = grid[t[:, 0], t[:, 1], t[:, 2]]
    return nb


class PhysicsRef:
    def __init__(self, topo, tau, q=19, out_rho=1.0):
        self.c, self.w, self.opp = lattice(q)
        self.q = q
        self.omega = 1.0 / tau
        self.out_rho = out_rho
        self.nbr = neighbour_table(topo["coords"], self.c)
        self.kind = np.asarray(topo["kind"])
        n = len(self.kind)
        self.n = n
        self.f = np.tile(self.w, (n, 1))
        self.inlet = np.asarray(topo["inlet"], dtype=np.int64)
        self.in_normal = np.asarray(topo["inlet_normal"], dtype=np.float64)
        self.profile = np.zeros((len(self.inlet), 3))
        self.out_normal_of = np.zeros((n, 3))
        k = 0
        while "outlet_%d" % k in topo:
            self.out_normal_of[np.asarray(topo["outlet_%d" % k], dtype=np.int64)] = topo["outlet_normal_%d" % k]
            k += 1
        self.moments = None

    def step(self, scale=1.0):
        c, w, opp = self.c, self.w, self.opp
        f = self.f
        rho = f.sum(axis=1)
        u = (f @ c) / rho[:, None]
        cu = u @ c.T
        usq = (u * u).sum(axis=1)
        feq = w[None, :] * rho[:, None] * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq[:, None])
        C = f + self.omega * (feq - f)
        self.moments = (rho, u)
        fn = np.empty_like(f)
        uw = np.zeros((self.n, 3))
        uw[self.inlet] = self.profile * scale
        for q in range(self.q):
            p = opp[q]
            up = self.nbr[:, p]
            have = up >= 0
            fn[have, q] = C[up[have], q]
            miss = np.nonzero(~have)[0]
            v = C[miss, p].copy()
            kind = self.kind[miss]
            cp = c[p].astype(np.float64)
            inl = (kind == 1) & (self.in_normal @ cp > 0)
            v[inl] -= 6.0 * w[p] * (uw[miss[inl]] @ cp)
            onrm = self.out_normal_of[miss]
            outl = (kind == 2) & (onrm @ cp > 0)
            un = u[miss[outl]]
            cun = un @ cp
            v[outl] = -C[miss[outl], p] + 2.0 * w[p] * self.out_rho * (
                1.0 + 4.5 * cun * cun - 1.5 * (un * un).sum(axis=1))
            fn[miss, q] = v
        self.f = fn

    def run(self, steps, scale=1.0):
        for _ in range(steps):
            self.step(scale)


def womersley_shape(r, R, alpha):
    """Complex axial-velocity shape of oscillatory pipe flow per unit flow-rate
    amplitude (Womersley): u(r, t) = Re{Q e^{iwt} shape(r)}, with
    shape = [1 - J0(b r/R) / J0(b)] / (pi R^2 [1 - 2 J1(b) / (b J0(b))]),
    b = i^{3/2} alpha, alpha = R sqrt(w / nu). It integrates to 1 over the
    cross-section and tends to the Poiseuille shape 2 (1 - r^2/R^2) / (pi R^2)
    as alpha -> 0."""
    from scipy.special import jv
    b = alpha * np.exp(0.75j * np.pi)
    j0 = jv(0, b)
    return (1.0 - jv(0, b * np.asarray(r) / R) / j0) / (np.pi * R * R * (1.0 - 2.0 * jv(1, b) / (b * j0)))
