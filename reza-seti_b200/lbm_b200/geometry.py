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


def _shift(a, d, fill):
    """a shifted so out[i] = a[i + d] (fill outside)."""
    out = np.full_like(a, fill)
    src = tuple(slice(max(0, k), a.shape[i] + min(0, k)) for i, k in enumerate(d))
    dst = tuple(slice(max(0, -k), a.shape[i] + min(0, -k)) for i, k in enumerate(d))
    out[dst] = a[src]
    return out


def classify(fluid, box_shape, offset, inlet_z=None, outlet_z=None, normal_fn=None):
    """Node set of a fluid mask given on a sub-box at `offset` of a box of
    `box_shape` (lattice cells). inlet_z / outlet_z: z index of the inlet and
    outlet planes (box faces); normal_fn(points[k,3]) -> outward normals."""
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
    if inlet_z is not None:
        inl[:, :, inlet_z - oz] = B[:, :, inlet_z - oz]
    if outlet_z is not None:
        outl[:, :, outlet_z - oz] = B[:, :, outlet_z - oz] & ~inl[:, :, outlet_z - oz]
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
        "inlet_normal": np.array([0.0, 0.0, -1.0]),
        "outlet_0": idx[np.nonzero(outl)],
        "outlet_normal_0": np.array([0.0, 0.0, 1.0]),
        "wall": idx[np.nonzero(wall)],
        "nearwall": nearwall,
    }
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
