"""Synthetic vessel geometries voxelised into the engine's node sets.

Each builder evaluates a signed-distance-like field of an analytic vessel on
the lattice and classifies nodes with the reference's rules:
  * fluid: inside the vessel (ComplexGeometry::labelPoints marks points inside
    the STL surface as Fluid, ComplexGeometry.cpp:440-514);
  * boundary: fluid with a non-fluid 26-neighbour or on the box face
    (ComplexGeometry::findBoundaryPoints, :517-564);
  * inlet / outlet: boundary nodes on the configured planes (getInOutBP,
    :567-641); wall: the remaining boundary nodes (excludeInletOutlet, :645-662);
  * near-wall: plain fluid nodes that are a D3Q19 neighbour of a wall node
    (SubDomain::IdentifyNextToWallLattices, Subdomain.cpp:475-493), with the
    outward surface normal of the analytic vessel at the node (the reference
    area-weights STL facet normals, Subdomain.cpp:499-572).
Nodes are listed x-major, z-fastest, the order of the reference's Involved_Lat_.
The result is a topology dict (keys as in lbm_b200.engine).

Work is done on the bounding sub-box of the vessel, one z-slab at a time, so
the 512 x 512 x 1024 boxes stay within a few GB of host memory.
"""
from __future__ import annotations

import math

import numpy as np

D3Q19 = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0],
                  [1, -1, 0], [1, 0, 1], [1, 0, -1], [-1, 1, 0], [-1, -1, 0], [-1, 0, 1],
                  [-1, 0, -1], [0, 1, 1], [0, 1, -1], [0, -1, 1], [0, -1, -1], [0, 0, 0]])
# D3Q27 in the engine's (and the reference's, LatticeModel.cpp:249-375) order
D3Q27 = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
                  [1, 1, 0], [1, -1, 0], [-1, 1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
                  [-1, 0, -1], [0, 1, 1], [0, 1, -1], [0, -1, 1], [0, -1, -1], [1, 1, 1],
                  [-1, -1, -1], [1, 1, -1], [-1, -1, 1], [1, -1, 1], [-1, 1, -1], [1, -1, -1],
                  [-1, 1, 1]])


def _shift(a, d, fill):
    """a shifted so out[i] = a[i + d] (fill outside)."""
    out = np.full_like(a, fill)
    src = tuple(slice(max(0, k), a.shape[i] + min(0, k)) for i, k in enumerate(d))
    dst = tuple(slice(max(0, -k), a.shape[i] + min(0, -k)) for i, k in enumerate(d))
    out[dst] = a[src]
    return out


def classify(fluid, box_shape, offset, inlet_z=None, outlet_z=None, normal_fn=None, openings=None):
    """Node set of a fluid mask given on a sub-box at `offset` of a box of
    `box_shape` (lattice cells). inlet_z / outlet_z: z index of the inlet and
    outlet planes (box faces); normal_fn(points[k,3]) -> outward normals.
    `openings` generalises the planes: a list of (kind, axis, index, normal,
    select) with kind "inlet" (at most one) or "outlet", the boundary nodes
    whose coordinate along `axis` equals `index`, optionally restricted by
    select(coords[k,3]) -> bool[k]; outlets are numbered in list order."""
    if openings is None:
        openings = []
        if inlet_z is not None:
            openings.append(("inlet", 2, inlet_z, (0.0, 0.0, -1.0), None))
        if outlet_z is not None:
            openings.append(("outlet", 2, outlet_z, (0.0, 0.0, 1.0), None))
    F = fluid.astype(bool)
    nf = ~F
    # 26-neighbourhood test against non-fluid; cells outside the sub-box are
    # non-fluid, except beyond the global box faces (reference tests only
    # in-box neighbours and adds the box-face rule separately)
    has_nf = np.zeros_like(F)
    pad_nf = np.pad(nf, 1, constant_values=True)
    ox, oy, oz = offset
    X, Y, Z = box_shape
    sx, sy, sz = F.shape
    # mark out-of-box padding as fluid so it does not count (reference skips
    # out-of-range neighbours)
    if ox == 0:
        pad_nf[0, :, :] = False
    if oy == 0:
        pad_nf[:, 0, :] = False
    if oz == 0:
        pad_nf[:, :, 0] = False
    if ox + sx == X:
        pad_nf[-1, :, :] = False
    if oy + sy == Y:
        pad_nf[:, -1, :] = False
    if oz + sz == Z:
        pad_nf[:, :, -1] = False
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                if dx == dy == dz == 0:
                    continue
                has_nf |= pad_nf[1 + dx:1 + dx + sx, 1 + dy:1 + dy + sy, 1 + dz:1 + dz + sz]
    face = np.zeros_like(F)
    if ox == 0:
        face[0] = True
    if ox + sx == X:
        face[-1] = True
    if oy == 0:
        face[:, 0] = True
    if oy + sy == Y:
        face[:, -1] = True
    if oz == 0:
        face[:, :, 0] = True
    if oz + sz == Z:
        face[:, :, -1] = True
    B = F & (has_nf | face)
    kind = np.zeros(F.shape, np.uint8)
    inl = np.zeros_like(F)
    outl = np.zeros_like(F)
    inlet_normal = np.zeros(3)
    out_masks, out_normals = [], []
    for what, axis, index, normal, select in openings:
        loc = index - offset[axis]
        m = np.zeros_like(F)
        if 0 <= loc < F.shape[axis]:
            sl = [slice(None)] * 3
            sl[axis] = loc
            m[tuple(sl)] = B[tuple(sl)]
        m &= ~inl & ~outl
        if select is not None and m.any():
            pts = np.stack(np.nonzero(m), axis=1) + np.array(offset)
            keep = np.asarray(select(pts.astype(np.float64)), bool)
            sub = np.zeros_like(F)
            sub[tuple((pts - np.array(offset))[keep].T)] = True
            m = sub
        if what == "inlet":
            inl |= m
            inlet_normal = np.asarray(normal, np.float64)
        else:
            outl |= m
            out_masks.append(m)
            out_normals.append(np.asarray(normal, np.float64))
    wall = B & ~inl & ~outl
    kind[inl] = 1
    kind[outl] = 2
    kind[wall] = 3
    # node numbering, x-major z-fastest
    idx = -np.ones(F.shape, np.int64)
    ii = np.nonzero(F)
    n = len(ii[0])
    idx[ii] = np.arange(n)
    coords = np.stack(ii, axis=1).astype(np.int32) + np.array(offset, np.int32)
    kinds = kind[ii]
    plain = F & (kind == 0)
    near = np.zeros_like(F)
    for d in D3Q19[:18]:
        near |= _shift(wall, tuple(d), False)
    near &= plain
    nearwall = idx[np.nonzero(near)]
    topo = {
        "coords": coords,
        "kind": kinds,
        "inlet": idx[np.nonzero(inl)],
        "inlet_normal": inlet_normal,
        "wall": idx[np.nonzero(wall)],
        "nearwall": nearwall,
    }
    for k, (m, nrm) in enumerate(zip(out_masks, out_normals)):
        topo["outlet_%d" % k] = idx[np.nonzero(m)]
        topo["outlet_normal_%d" % k] = nrm
    if normal_fn is not None:
        topo["nearwall_normal"] = normal_fn(coords[nearwall].astype(np.float64))
    else:
        topo["nearwall_normal"] = np.zeros((len(nearwall), 3))
    return topo


def _normals_from_field(field_fn, pts, h=0.5):
    g = np.zeros_like(pts)
    for a in range(3):
        e = np.zeros(3)
        e[a] = h
        g[:, a] = (field_fn(pts + e) - field_fn(pts - e)) / (2 * h)
    nrm = np.linalg.norm(g, axis=1, keepdims=True)
    nrm[nrm == 0] = 1.0
    return g / nrm


def tortuous_vessel(radius=20.0, box=(512, 512, 1024), amplitude=30.0, wavelength=200.0,
                    stenosis_area=0.5, stenosis_sigma=None):
    """Vessel with a sinusoidal centerline x_c(z) = X/2 + A sin(2 pi z / lambda),
    y_c = Y/2, running the full box length along z, with a Gaussian stenosis of
    the given area reduction at mid-length. Inlet plane z = 0, outlet z = Z-1."""
    X, Y, Z = box
    sig = stenosis_sigma if stenosis_sigma is not None else 2.0 * radius
    k = 2 * math.pi / wavelength

    def field(p):
        x, y, z = p[:, 0], p[:, 1], p[:, 2]
        xc = X / 2 + amplitude * np.sin(k * z)
        slope = amplitude * k * np.cos(k * z)
        cos_t = 1.0 / np.sqrt(1.0 + slope * slope)
        r_loc = radius * np.sqrt(1.0 - stenosis_area * np.exp(-((z - Z / 2) ** 2) / (2 * sig * sig)))
        return np.sqrt(((x - xc) * cos_t) ** 2 + (y - Y / 2) ** 2) - r_loc

    x0 = int(max(0, math.floor(X / 2 - amplitude - radius - 3)))
    x1 = int(min(X, math.ceil(X / 2 + amplitude + radius + 3)))
    y0 = int(max(0, math.floor(Y / 2 - radius - 3)))
    y1 = int(min(Y, math.ceil(Y / 2 + radius + 3)))
    xs = np.arange(x0, x1, dtype=np.float64)
    ys = np.arange(y0, y1, dtype=np.float64)
    fluid = np.zeros((x1 - x0, y1 - y0, Z), bool)
    gx, gy = np.meshgrid(xs, ys, indexing="ij")
    for z in range(Z):
        p = np.stack([gx.ravel(), gy.ravel(), np.full(gx.size, float(z))], axis=1)
        fluid[:, :, z] = (field(p) < 0).reshape(gx.shape)
    return classify(fluid, box, (x0, y0, 0), inlet_z=0, outlet_z=Z - 1,
                    normal_fn=lambda pts: _normals_from_field(field, pts))


def _tortuous_volume(radius, box, amplitude, wavelength, every=8):
    """Fluid cell count of tortuous_vessel, counted on every `every`-th slice."""
    X, Y, Z = box
    k = 2 * math.pi / wavelength
    sig = 2.0 * radius
    gx, gy = np.meshgrid(np.arange(X, dtype=float), np.arange(Y, dtype=float), indexing="ij")
    total = 0
    for z in range(0, Z, every):
        xc = X / 2 + amplitude * math.sin(k * z)
        cos_t = 1.0 / math.sqrt(1.0 + (amplitude * k * math.cos(k * z)) ** 2)
        r = radius * math.sqrt(1.0 - 0.5 * math.exp(-((z - Z / 2) ** 2) / (2 * sig * sig)))
        total += int(np.count_nonzero(((gx - xc) * cos_t) ** 2 + (gy - Y / 2) ** 2 < r * r))
    return total * every


def fluid_fraction_radius(fraction, box=(512, 512, 1024), amplitude=30.0, wavelength=200.0):
    """Vessel radius at which the tortuous vessel fills the requested fraction
    of the box (two fixed-point corrections of the cylinder estimate)."""
    X, Y, Z = box
    z = np.arange(Z)
    slope = amplitude * 2 * math.pi / wavelength * np.cos(2 * math.pi * z / wavelength)
    arc = float(np.sum(np.sqrt(1 + slope ** 2)))
    r = math.sqrt(fraction * X * Y * Z / (math.pi * arc))
    for _ in range(2):
        got = _tortuous_volume(r, box, amplitude, wavelength) / float(X * Y * Z)
        r *= math.sqrt(fraction / got)
    return r


def straight_pipe(radius=16.0, length=128, box=None, centre=None, stenosis=0.0, stenosis_sigma=8.0):
    """Straight pipe along z (optional Gaussian stenosis of the given radius
    reduction fraction at mid-length). Inlet z = 0, outlet z = length-1."""
    if box is None:
        w = int(2 * radius + 8)
        box = (w, w, length)
    X, Y, Z = box
    cx, cy = centre if centre is not None else (X / 2 - 0.5 + 0.37, Y / 2 - 0.5 + 0.21)

    def field(p):
        r = radius * (1 - stenosis * np.exp(-((p[:, 2] - Z / 2) ** 2) / (2 * stenosis_sigma ** 2)))
        return np.hypot(p[:, 0] - cx, p[:, 1] - cy) - r

    gx, gy, gz = np.meshgrid(np.arange(X, dtype=float), np.arange(Y, dtype=float),
                             np.arange(Z, dtype=float), indexing="ij")
    p = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)
    fluid = (field(p) < 0).reshape(box)
    topo = classify(fluid, box, (0, 0, 0), inlet_z=0, outlet_z=Z - 1,
                    normal_fn=lambda pts: _normals_from_field(field, pts))
    topo["axis_centre"] = np.array([cx, cy])
    topo["radius"] = np.array([radius])
    return topo


def zernike_inlet_basis(topo, n=8, radius=None, centre=None):
    """Zernike-like inlet speed modes on the pipe's inlet disc, [n, n_inlet]:
    the low-order Zernike polynomials (1, rho cos t, rho sin t, 2 rho^2 - 1,
    rho^2 cos 2t, rho^2 sin 2t, (3 rho^3 - 2 rho) cos t, (3 rho^3 - 2 rho) sin t,
    ...) times (1 - rho^2), so every mode vanishes on the wall; zero outside
    the radius. Mode 0 is the Poiseuille profile with unit peak."""
    R = float(topo["radius"][0]) if radius is None else radius
    cx, cy = topo["axis_centre"] if centre is None else centre
    xy = topo["coords"][topo["inlet"]][:, :2].astype(np.float64)
    dx, dy = xy[:, 0] - cx, xy[:, 1] - cy
    rho = np.hypot(dx, dy) / R
    th = np.arctan2(dy, dx)
    modes = [np.ones_like(rho), rho * np.cos(th), rho * np.sin(th), 2 * rho ** 2 - 1,
             rho ** 2 * np.cos(2 * th), rho ** 2 * np.sin(2 * th),
             (3 * rho ** 3 - 2 * rho) * np.cos(th), (3 * rho ** 3 - 2 * rho) * np.sin(th),
             6 * rho ** 4 - 6 * rho ** 2 + 1, rho ** 3 * np.cos(3 * th), rho ** 3 * np.sin(3 * th)]
    if n > len(modes):
        raise ValueError("at most %d modes" % len(modes))
    env = np.maximum(0.0, 1.0 - rho ** 2)
    return np.stack([m * env for m in modes[:n]])


def stenotic_throat_targets(topo, half_length, z_centre=None):
    """Near-wall list entries within half_length of the throat plane (z =
    length / 2 by default, where straight_pipe centres its stenosis), [k]
    int64."""
    nw = np.asarray(topo["nearwall"], dtype=np.int64)
    z = topo["coords"][nw][:, 2].astype(np.float64)
    zc = (float(topo["coords"][:, 2].max()) + 1.0) / 2 if z_centre is None else z_centre
    return np.nonzero(np.abs(z - zc) <= half_length)[0].astype(np.int64)


def parabolic_inlet(topo, u_max, radius=None, centre=None):
    """Poiseuille inlet profile along +z for the inlet nodes of a pipe:
    u_z = u_max (1 - r^2 / R^2), zero outside R ([n_inlet, 3])."""
    R = float(topo["radius"][0]) if radius is None else radius
    cx, cy = topo["axis_centre"] if centre is None else centre
    xy = topo["coords"][topo["inlet"]][:, :2].astype(np.float64)
    r2 = (xy[:, 0] - cx) ** 2 + (xy[:, 1] - cy) ** 2
    v = np.zeros((len(xy), 3))
    v[:, 2] = np.maximum(0.0, u_max * (1.0 - r2 / (R * R)))
    return v


# ------------------------------------------------------ branching vessels ---
def _voxelise(field, box, lo, hi):
    """Fluid mask (field < 0) on the sub-box [lo, hi) of `box`, z-slab by z-slab."""
    lo = [max(0, int(v)) for v in lo]
    hi = [min(b, int(v)) for b, v in zip(box, hi)]
    gx, gy = np.meshgrid(np.arange(lo[0], hi[0], dtype=np.float64), np.arange(lo[1], hi[1], dtype=np.float64),
                         indexing="ij")
    fluid = np.zeros((hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]), bool)
    for z in range(lo[2], hi[2]):
        p = np.stack([gx.ravel(), gy.ravel(), np.full(gx.size, float(z))], axis=1)
        fluid[:, :, z - lo[2]] = (field(p) < 0).reshape(gx.shape)
    return fluid, tuple(lo)


def _perpendiculars(d):
    d = d / np.linalg.norm(d)
    a = np.array([0.0, 1.0, 0.0]) if abs(d[1]) < 0.9 else np.array([1.0, 0.0, 0.0])
    n1 = np.cross(d, a)
    n1 /= np.linalg.norm(n1)
    return n1, np.cross(d, n1)


def _tube(p0, d, length, radius, wiggle=(0.0, 0.0)):
    """Signed distance of a straight capsule from p0 along d (length, radius)
    whose axis is displaced by wiggle[0] sin(pi s / L) n1 + wiggle[1]
    sin(2 pi s / L) n2 (zero at both ends)."""
    p0 = np.asarray(p0, np.float64)
    d = np.asarray(d, np.float64) / np.linalg.norm(d)
    n1, n2 = _perpendiculars(d)

    def f(p):
        s = np.clip((p - p0) @ d, 0.0, length)
        c = p0 + s[:, None] * d
        c = c + (wiggle[0] * np.sin(np.pi * s / length))[:, None] * n1
        c = c + (wiggle[1] * np.sin(2 * np.pi * s / length))[:, None] * n2
        return np.linalg.norm(p - c, axis=1) - radius
    return f


def y_bifurcation(seed=2, box=(256, 256, 348), parent=(24.0, 200.0), daughters=((18.0, 180.0), (16.0, 180.0)),
                  angle_deg=35.0):
    """Y-bifurcation: a parent tube along +z from the inlet plane z = 0 to the
    branch point at z = parent length, and two daughters at +-angle in the
    x-z plane, their centerlines displaced by seeded smooth wiggles (at most
    2 lu, zero at the ends). The daughters leave through the top face z = Z-1
    (an oblique cut), split into outlet 0 (x < X/2) and outlet 1."""
    X, Y, Z = box
    rng = np.random.default_rng(seed)
    cx, cy = X / 2 - 0.5 + 0.31, Y / 2 - 0.5 + 0.17
    rp, lp = parent
    tubes = [_tube((cx, cy, -30.0), (0, 0, 1), lp + 30.0, rp, rng.uniform(-2, 2, 2))]
    a = math.radians(angle_deg)
    for sign, (rd, ld) in zip((-1.0, 1.0), daughters):
        d = np.array([sign * math.sin(a), 0.0, math.cos(a)])
        # continue past the top face so that the face cuts the tube open
        over = (Z + 30 - lp) / math.cos(a)
        tubes.append(_tube((cx, cy, lp), d, max(ld, over), rd, rng.uniform(-2, 2, 2)))

    def field(p):
        return np.minimum.reduce([t(p) for t in tubes])

    fluid, off = _voxelise(field, box, (0, cy - 40, 0), (X, cy + 40, Z))
    openings = [("inlet", 2, 0, (0.0, 0.0, -1.0), None),
                ("outlet", 2, Z - 1, (0.0, 0.0, 1.0), lambda c: c[:, 0] < X / 2),
                ("outlet", 2, Z - 1, (0.0, 0.0, 1.0), None)]
    topo = classify(fluid, box, off, normal_fn=lambda pts: _normals_from_field(field, pts), openings=openings)
    topo["axis_centre"] = np.array([cx, cy])
    topo["radius"] = np.array([rp])
    return topo


def saccular_aneurysm(box=(1024, 512, 512), radius=20.0, bend_radius=120.0, sac_radius=40.0, neck=15.0,
                      x0=100.0, z0=100.0):
    """90-degree curved tube with a spherical sac on the outer wall of the bend.
    The tube rises along +z from the inlet plane z = 0 to z0 at x = x0, bends
    through a quarter circle of bend_radius in the x-z plane, and runs along
    +x to the outlet plane x = X-1. The sac's centre lies on the bend's
    45-degree ray, sac_radius - neck beyond the outer wall, so the sphere
    overlaps the tube wall by `neck` lu. Also returns the sac centre under
    "sac_centre"."""
    X, Y, Z = box
    yc = Y / 2 - 0.5 + 0.23
    cb = np.array([x0 + bend_radius, yc, z0])  # bend centre
    t_in = _tube((x0, yc, -30.0), (0, 0, 1), z0 + 30.0, radius)
    t_out = _tube((x0 + bend_radius, yc, z0 + bend_radius), (1, 0, 0), X + 30.0 - x0 - bend_radius, radius)
    ray = np.array([-math.cos(math.pi / 4), 0.0, math.sin(math.pi / 4)])
    sac = cb + (bend_radius + radius + sac_radius - neck) * ray

    def bend(p):
        v = p - cb
        phi = np.arctan2(v[:, 2], -v[:, 0])  # 0 at the tube's start, pi/2 at its end
        rho = np.hypot(v[:, 0], v[:, 2])
        d = np.hypot(rho - bend_radius, v[:, 1]) - radius
        return np.where((phi >= 0) & (phi <= math.pi / 2), d, np.inf)

    def field(p):
        return np.minimum.reduce([t_in(p), t_out(p), bend(p), np.linalg.norm(p - sac, axis=1) - sac_radius])

    lo = (x0 - radius - 3, yc - max(radius, sac_radius) - 3, 0)
    hi = (X, yc + max(radius, sac_radius) + 4, max(z0 + bend_radius + radius, sac[2] + sac_radius) + 4)
    fluid, off = _voxelise(field, box, lo, hi)
    openings = [("inlet", 2, 0, (0.0, 0.0, -1.0), None), ("outlet", 0, X - 1, (1.0, 0.0, 0.0), None)]
    topo = classify(fluid, box, off, normal_fn=lambda pts: _normals_from_field(field, pts), openings=openings)
    topo["sac_centre"] = sac
    topo["sac_radius"] = np.array([sac_radius])
    topo["axis_centre"] = np.array([x0, yc])
    topo["radius"] = np.array([radius])
    return topo


def sac_wall_targets(topo, margin=3.0):
    """Near-wall list entries on the sac: within sac_radius + margin of the sac
    centre and farther than sac_radius - 2 margin from it (its wall layer)."""
    nw = np.asarray(topo["nearwall"], np.int64)
    c = topo["coords"][nw].astype(np.float64)
    r = np.linalg.norm(c - topo["sac_centre"], axis=1)
    R = float(topo["sac_radius"][0])
    return np.nonzero((r <= R + margin) & (r >= R - 2 * margin))[0].astype(np.int64)


def inlet_disc_profile(topo, mean, radius=None):
    """Parabolic inflow with the given mean velocity on the inlet disc, along
    -inlet_normal, centred on the inlet nodes ([n_inlet, 3])."""
    xyz = topo["coords"][topo["inlet"]].astype(np.float64)
    nrm = np.asarray(topo["inlet_normal"], np.float64)
    c = xyz.mean(axis=0)
    rel = xyz - c
    rel -= np.outer(rel @ nrm, nrm)
    r2 = (rel ** 2).sum(axis=1)
    R = float(topo["radius"][0]) if radius is None else radius
    v = np.maximum(0.0, 2.0 * mean * (1.0 - r2 / (R * R)))
    return v[:, None] * (-nrm)[None, :]


# ----------------------------------------------------------- STL pipeline ---
def read_stl(path):
    """Triangles of an ASCII STL as [n, 12] (vertex 1, 2, 3, facet normal),
    read by the library with the reference reader's line grammar."""
    import ctypes

    from . import capi
    n = ctypes.c_int64()
    buf = ctypes.POINTER(ctypes.c_double)()
    capi.check(capi.lib().lbm_stl_read_ascii(str(path).encode(), ctypes.byref(n), ctypes.byref(buf)))
    try:
        return np.ctypeslib.as_array(buf, shape=(max(n.value, 1) * 12,))[: n.value * 12].reshape(-1, 12).copy()
    finally:
        capi.lib().lbm_free(buf)


def opening(kind, plane, coordinate, normal, range_x=None, range_y=None, range_z=None):
    """One inlet or outlet block of the reference's config.txt."""
    return {"kind": kind, "plane": plane, "coordinate": float(coordinate), "normal": list(map(float, normal)),
            "range_x": range_x, "range_y": range_y, "range_z": range_z}


def voxelise_stl(triangles, grid_size, openings, device=0, info=False):
    """Node set of an STL surface on the GPU (lbm_voxelise), as a topology dict
    with the reference's classification; coordinates are grid indices.
    `openings`: list of opening(...) dicts, inlets and outlets in config
    order. With info, also returns (dims, origin, spacing, build_ms)."""
    import ctypes

    from . import capi
    tris = np.ascontiguousarray(triangles, dtype=np.float64).reshape(-1, 12)
    ops = (capi.LbmOpening * max(1, len(openings)))()
    for o, b in zip(ops, openings):
        o.outlet = 1 if b["kind"] == "outlet" else 0
        o.axis = "xyz".index(b["plane"])
        o.coordinate = b["coordinate"]
        for a in range(3):
            o.normal[a] = b["normal"][a]
            r = b.get("range_" + "xyz"[a])
            o.range[a][0], o.range[a][1] = (r[0], r[1]) if r is not None else (-np.inf, np.inf)
    d = capi.LbmVoxelDesc()
    d.n_triangles = len(tris)
    d.triangles = tris.ctypes.data_as(capi._f64p)
    d.grid_size = float(grid_size)
    d.n_openings = len(openings)
    d.openings = ops
    d.device = device
    v = ctypes.c_void_p()
    L = capi.lib()
    capi.check(L.lbm_voxelise(ctypes.byref(d), ctypes.byref(v)))
    try:
        desc = capi.LbmDesc()
        capi.check(L.lbm_voxel_describe(v, ctypes.byref(desc)))
        n = desc.n_nodes

        def arr(ptr, count, dtype, shape=None):
            a = np.ctypeslib.as_array(ptr, shape=(max(count, 1),))[:count].astype(dtype)
            return a.reshape(shape) if shape else a

        topo = {"coords": arr(desc.coords, 3 * n, np.int32, (n, 3)), "kind": arr(desc.kind, n, np.uint8),
                "inlet": arr(desc.inlet, desc.n_inlet, np.int64),
                "inlet_normal": np.array(list(desc.inlet_normal)),
                "wall": arr(desc.wall, desc.n_wall, np.int64),
                "nearwall": arr(desc.nearwall, desc.n_nearwall, np.int64),
                "nearwall_normal": arr(desc.nearwall_normals, 3 * desc.n_nearwall, np.float64,
                                       (desc.n_nearwall, 3))}
        off = arr(desc.outlet_offsets, desc.n_outlets + 1, np.int64)
        nodes = arr(desc.outlet_nodes, int(off[-1]) if len(off) else 0, np.int64)
        normals = arr(desc.outlet_normals, 3 * desc.n_outlets, np.float64, (max(desc.n_outlets, 0), 3))
        for k in range(desc.n_outlets):
            topo["outlet_%d" % k] = nodes[off[k]:off[k + 1]]
            topo["outlet_normal_%d" % k] = normals[k]
        if info:
            dims = (ctypes.c_int32 * 3)()
            origin = (ctypes.c_double * 3)()
            sp, ms = ctypes.c_double(), ctypes.c_double()
            capi.check(L.lbm_voxel_info(v, dims, origin, ctypes.byref(sp), None, None, ctypes.byref(ms)))
            return topo, (tuple(dims), tuple(origin), sp.value, ms.value)
        return topo
    finally:
        L.lbm_voxel_destroy(v)


def tube_triangles(center_fn, radius_fn, z0, z1, n_az, n_ax, phase=0.5):
    """Closed triangulated tube around a centerline (x_c(z), y_c(z)) from z0 to
    z1: rings of n_az vertices in the planes of n_ax + 1 stations (azimuthal
    phase in facets, so that no vertex or edge sits on a lattice line), side
    quads split in two, fan caps. Returns [n, 12] (vertices, outward facet
    normal), the layout of lbm_voxel_desc.triangles."""
    zs = np.linspace(z0, z1, n_ax + 1)
    th = 2 * np.pi * (np.arange(n_az) + phase) / n_az
    cen = np.array([center_fn(z) for z in zs])                     # [S, 2]
    rad = np.array([radius_fn(z) for z in zs])                      # [S]
    ring = np.empty((n_ax + 1, n_az, 3))
    ring[..., 0] = cen[:, None, 0] + rad[:, None] * np.cos(th)[None, :]
    ring[..., 1] = cen[:, None, 1] + rad[:, None] * np.sin(th)[None, :]
    ring[..., 2] = zs[:, None]
    a = np.arange(n_az)
    b = (a + 1) % n_az
    lo, hi = ring[:-1], ring[1:]
    # two triangles per quad: (lo a, lo b, hi b), (lo a, hi b, hi a)
    t1 = np.stack([lo[:, a], lo[:, b], hi[:, b]], axis=2).reshape(-1, 3, 3)
    t2 = np.stack([lo[:, a], hi[:, b], hi[:, a]], axis=2).reshape(-1, 3, 3)
    side = np.concatenate([t1, t2])
    mid_c = np.concatenate([np.repeat(0.5 * (cen[:-1] + cen[1:]), n_az, axis=0)] * 2)
    out_side = side.mean(axis=1)
    out_side[:, :2] -= mid_c
    out_side[:, 2] = 0.0
    caps = []
    outs = []
    for k, sign in ((0, -1.0), (n_ax, 1.0)):
        ctr = np.array([cen[k, 0], cen[k, 1], zs[k]])
        caps.append(np.stack([np.broadcast_to(ctr, (n_az, 3)), ring[k, a], ring[k, b]], axis=1))
        outs.append(np.broadcast_to(np.array([0.0, 0.0, sign]), (n_az, 3)))
    tri = np.concatenate([side] + caps)
    out = np.concatenate([out_side] + outs)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    flip = (n * out).sum(axis=1) < 0
    tri[flip] = tri[flip][:, [0, 2, 1]]
    n[flip] = -n[flip]
    return np.concatenate([tri.reshape(-1, 9), n], axis=1)
