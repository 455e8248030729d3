"""Seeded synthetic grain packings for the MELODY 2D step, written in the reference's formats.

The reference preprocessor is MATLAB (Preprocessor/*.m) and cannot run here, so this module
restates the parts of it the solver's inputs depend on:

* Gauss points: 3-point triangle rule of Preprocessor/GaussCoefficientsTriangle.m:4-7 mapped by
  Preprocessor/TriangleGaussPoints.m:17-27 (weights 1/3, jacobian = triangle area).
* MLS shape functions with a linear basis and the cubic-spline weight W1:
  Preprocessor/MLS2DWithDerivatives.m:65-165 and Preprocessor/WeightW1WithDerivatives.m:17-47.
  The basis is expressed relative to the body centre, which leaves the MLS functions unchanged
  and keeps the 3x3 moment matrix well conditioned.
* Support domains: nodes whose influence radius covers the point
  (Preprocessor/SupportDomain.m:16-18).
* Lumped masses = row sums of the consistent mass matrix (Preprocessor/AnalyseSimpleBody.m:316-331).
* Closed borders list their nodes counter-clockwise and repeat the first node at the end
  (Preprocessor/SetUnstructuredNodesForClosedContour.m:154-159), border nodes first.
* Rigid bodies: centre of mass, mass and inertia of Preprocessor/AnalyseRigidBody.m.

File layout follows Preprocessor/ExportStatic.m and Preprocessor/ExportDynamic.m as read by
Load_static (Code/IO.h:598-1861) and Load_dynamic (Code/IO.h:1871-2345).

Deviations from the preprocessor: the support radius is 2.0x the body's mean Delaunay edge
length (the workload's definition) instead of the k-nearest-neighbour rule of
AnalyseSimpleBody.m:64-68; interior nodes come from seeded rejection sampling instead of
Distmesh; the large packings use a box enlarged to hold 2000 discs at random-sequential-addition
density.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, List, Optional, Tuple

import numpy as np
from scipy.spatial import Delaunay, cKDTree

# 3-point rule exactly as typed in Preprocessor/GaussCoefficientsTriangle.m:4-7
_GAUSS3 = np.array([[0.16666666666667, 0.16666666666667, 0.33333333333333],
                    [0.16666666666667, 0.66666666666667, 0.33333333333333],
                    [0.66666666666667, 0.16666666666667, 0.33333333333333]])

BC_NONE, BC_SOFT, BC_DRIVEN, BC_ORIENTED, BC_FOLLOWING = 0, 1, 2, 3, 4
LAW_NAMES = ["Frictionless", "Cohesion", "MohrCoulomb", "DampedMohrCoulomb", "TwoSlopesMohrCoulomb",
             "BondedMohrCoulomb", "CZMlinear", "CZMfatigue"]
LAW_NPARAM_FILE = [1, 4, 5, 6, 6, 11, 6, 9]
MAT_NAMES = ["ElasticLinear", "NeoHookean"]
SOLVER_NAMES = ["Euler", "Adaptive_Euler", "Mass_Scaling", "Adaptive_Mass_Scaling", "Euler_2"]
T_HIST_END = 1.0e3   # last instant of every boundary-condition history (s)


# --------------------------------------------------------------------------------------------
# MLS shape functions (Preprocessor/MLS2DWithDerivatives.m, WeightW1WithDerivatives.m)
# --------------------------------------------------------------------------------------------

def _w1(relx: np.ndarray, rely: np.ndarray, d: np.ndarray):
    """Cubic-spline weight and its gradient with respect to the point of interest
    (Preprocessor/WeightW1WithDerivatives.m:25-44); relx = x_point - x_node."""
    rho = np.sqrt(relx * relx + rely * rely)
    r = rho / d
    w = np.zeros_like(r)
    dwdx = np.zeros_like(r)
    dwdy = np.zeros_like(r)
    inner = r <= 0.5
    outer = (r > 0.5) & (r <= 1.0)
    w[inner] = (2.0 / 3.0) - 4.0 * r[inner] ** 2 + 4.0 * r[inner] ** 3
    d3 = d ** 3
    dwdx[inner] = (-8.0 * d[inner] * relx[inner] + 12.0 * relx[inner] * rho[inner]) / d3[inner]
    dwdy[inner] = (-8.0 * d[inner] * rely[inner] + 12.0 * rely[inner] * rho[inner]) / d3[inner]
    ro = r[outer]
    w[outer] = (4.0 / 3.0) - 4.0 * ro + 4.0 * ro ** 2 - (4.0 / 3.0) * ro ** 3
    # dw/dr * dr/dx with dw/dr = -4 + 8r - 4r^2 and dr/dx = x / (r d^2)
    fac = 4.0 * (-1.0 + 2.0 * ro - ro * ro) / (ro * d[outer] ** 2)
    dwdx[outer] = fac * relx[outer]
    dwdy[outer] = fac * rely[outer]
    return w, dwdx, dwdy


def _supports(points: np.ndarray, nodes: np.ndarray, radii: np.ndarray, kmax: int = 40):
    """Support lists of Preprocessor/SupportDomain.m:16-18 (nodes whose radius covers the point),
    ascending node order, as a padded (P, K) index array and mask."""
    tree = cKDTree(nodes)
    n = nodes.shape[0]
    k = min(kmax, n)
    while True:
        dist, idx = tree.query(points, k=k, distance_upper_bound=float(radii.max()) * (1 + 1e-12))
        if k == 1:
            dist = dist[:, None]; idx = idx[:, None]
        valid = idx < n
        idx_c = np.where(valid, idx, 0)
        dx = points[:, 0:1] - nodes[idx_c, 0]
        dy = points[:, 1:2] - nodes[idx_c, 1]
        keep = valid & (dx * dx + dy * dy - radii[idx_c] ** 2 < 0.0)
        if k >= n or not np.any(keep.sum(axis=1) == k):
            break
        k = min(2 * k, n)
    key = np.where(keep, idx_c, n + 1)
    order = np.argsort(key, axis=1, kind="stable")
    idx_s = np.take_along_axis(idx_c, order, axis=1)
    keep_s = np.take_along_axis(keep, order, axis=1)
    K = int(keep_s.sum(axis=1).max())
    return idx_s[:, :K], keep_s[:, :K]


def mls_shape(points: np.ndarray, nodes: np.ndarray, radii: np.ndarray, origin: np.ndarray):
    """Linear-basis MLS shape functions N, dN/dx, dN/dy at `points` from `nodes` with influence
    radii `radii` (Preprocessor/MLS2DWithDerivatives.m:65-165).

    Returns (ptr, idx, N, dNdx, dNdy) in CSR form with support lists in ascending node order
    (the order Preprocessor/SupportDomain.m:17-18 produces)."""
    idx, mask = _supports(points, nodes, radii)
    P = points.shape[0]
    counts = mask.sum(axis=1).astype(np.int64)
    relx = points[:, 0:1] - nodes[idx, 0]
    rely = points[:, 1:2] - nodes[idx, 1]
    d = radii[idx]
    w, wx, wy = _w1(relx, rely, d)
    w = np.where(mask, w, 0.0)
    wx = np.where(mask, wx, 0.0)
    wy = np.where(mask, wy, 0.0)
    p = np.stack([np.ones_like(relx), nodes[idx, 0] - origin[0], nodes[idx, 1] - origin[1]], axis=-1)
    pp = p[..., :, None] * p[..., None, :]                      # P,K,3,3
    A = np.einsum("pk,pkij->pij", w, pp)
    Ax = np.einsum("pk,pkij->pij", wx, pp)
    Ay = np.einsum("pk,pkij->pij", wy, pp)
    c = np.stack([np.ones(P), points[:, 0] - origin[0], points[:, 1] - origin[1]], axis=-1)
    g1 = np.linalg.solve(A, c[..., None])[..., 0]
    ex = np.zeros((P, 3)); ex[:, 1] = 1.0
    ey = np.zeros((P, 3)); ey[:, 2] = 1.0
    g2 = np.linalg.solve(A, (ex - np.einsum("pij,pj->pi", Ax, g1))[..., None])[..., 0]
    g3 = np.linalg.solve(A, (ey - np.einsum("pij,pj->pi", Ay, g1))[..., None])[..., 0]
    gp1 = np.einsum("pj,pkj->pk", g1, p)
    N = gp1 * w
    dNdx = np.einsum("pj,pkj->pk", g2, p) * w + gp1 * wx
    dNdy = np.einsum("pj,pkj->pk", g3, p) * w + gp1 * wy
    ptr = np.zeros(P + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(counts)
    return ptr, idx[mask], N[mask], dNdx[mask], dNdy[mask]


# --------------------------------------------------------------------------------------------
# Bodies
# --------------------------------------------------------------------------------------------

@dataclasses.dataclass
class Body:
    kind: str                       # "deformable" | "rigid"
    material: int
    nodes: np.ndarray               # (n,2)
    borders: List[dict]             # each: nodes (list, closed repeats first), periodicity, interpolant,
                                    #       before, after, bc: [(type, params(2), hist(t,v))] x2
    cells: np.ndarray               # (m,3) CCW
    nodal_distance: float
    detection: float
    contact: float
    periodic: int = 0
    status: int = 0
    # deformable only
    domain: Optional[np.ndarray] = None
    mass: Optional[np.ndarray] = None            # (n,2)
    sup: Optional[Tuple] = None                  # DOF_TO_DISP csr (ptr, idx, N, dNdx, dNdy)
    gp_xy: Optional[np.ndarray] = None
    gp_w: Optional[np.ndarray] = None
    gp_J: Optional[np.ndarray] = None
    gp: Optional[Tuple] = None                   # csr (ptr, idx, N, dNdx, dNdy)
    n_regions: int = 1
    # rigid only
    centre: Optional[np.ndarray] = None
    rigid_mass: float = 0.0
    rigid_inertia: float = 0.0
    velocity: Tuple[float, float] = (0.0, 0.0)
    angular_velocity: float = 0.0               # rigid only (rad/s)
    dt_terms: Optional[Tuple[float, float]] = None   # critical-step terms (elastic eigenvalue, h/m per kn)
    # MATRICES of STATIC_DATA (Code/IO.h:1827-1851): upper-triangle (dof0, dof1) pairs, dof = 2 node +
    # direction, with their stiffness and damping coefficients; None writes an empty section
    matrices: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]] = None
    # ALID absorbing layer of STATIC_CONTROL (Code/IO.h:1395-1480): keys x_hist and y_hist (lists
    # of (time, value) of the layer's reference velocity) and xmin, xmax, ymin, ymax, range,
    # alphain, alphaout, betain, betaout, exponent; None: no layer
    alid: Optional[dict] = None


def _ccw(nodes: np.ndarray, tri: np.ndarray) -> np.ndarray:
    p0, p1, p2 = nodes[tri[:, 0]], nodes[tri[:, 1]], nodes[tri[:, 2]]
    cross = (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p1[:, 1] - p0[:, 1]) * (p2[:, 0] - p0[:, 0])
    tri = tri.copy()
    flip = cross < 0
    tri[flip] = tri[flip][:, [0, 2, 1]]
    area = 0.5 * np.abs(cross)
    return tri[area > 1e-14 * np.max(area)]


def _rejection_interior(rng, centre, radius, n_target, min_sep, existing, margin, max_tries=200000):
    pts = []
    tree_pts = [tuple(p) for p in existing]
    grid: Dict[Tuple[int, int], List[Tuple[float, float]]] = {}
    cs = min_sep
    def key(x, y):
        return (int(math.floor(x / cs)), int(math.floor(y / cs)))
    for p in tree_pts:
        grid.setdefault(key(*p), []).append(p)
    tries = 0
    rin = radius - margin
    while len(pts) < n_target and tries < max_tries:
        tries += 1
        rr = rin * math.sqrt(rng.random())
        th = 2.0 * math.pi * rng.random()
        x = centre[0] + rr * math.cos(th)
        y = centre[1] + rr * math.sin(th)
        kx, ky = key(x, y)
        ok = True
        for ix in (kx - 1, kx, kx + 1):
            for iy in (ky - 1, ky, ky + 1):
                for q in grid.get((ix, iy), ()):
                    if (q[0] - x) ** 2 + (q[1] - y) ** 2 < min_sep * min_sep:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            pts.append((x, y))
            grid.setdefault((kx, ky), []).append((x, y))
    return np.array(pts).reshape(-1, 2)


# A lumped mass is the integral of the node's MLS shape function; a node placed where its support
# is cut short (next to another node, close to the border) can get a mass far below the others, or
# even a negative one, and with it a critical time step far below its disc's (or no stable step at
# all).  Such a disc is drawn again: MIN_MASS_RATIO is the smallest accepted ratio of a node's mass to
# the disc's median.
MIN_MASS_RATIO = 0.2


# The same holds for the disc's critical time step, 2 / sqrt(largest eigenvalue of its lumped-mass
# elastic operator): over many draws it sits near h_b sqrt(rho / E) (h_b the border-node spacing) with
# a long lower tail, down to a third of that, and one such disc sets the step of a whole sample.
# With dt_check, a disc whose step falls below MIN_DT_RATIO of that nominal value is drawn again.
MIN_DT_RATIO = 0.75


def make_disc(rng, centre, radius, n_border, n_interior, min_sep, material, rho, support_factor=2.0,
              mass_factor=1.0, regions=1, max_draws=20, dt_check=None):
    """Deformable disc: n_border equispaced border nodes (CCW), seeded interior nodes, Delaunay
    cells, 3 Gauss points per cell, MLS shape functions, lumped masses.  The interior nodes are drawn
    again (from the same random stream) while some node's lumped mass is below MIN_MASS_RATIO of the
    median, and, with dt_check = (mu, lambda, E), while the disc's critical step is below MIN_DT_RATIO
    of h_b sqrt(rho mass_factor / E); the disc then carries dt_terms (the two terms of critical_dt)."""
    best = None
    for _ in range(max_draws):
        b = _make_disc_once(rng, centre, radius, n_border, n_interior, min_sep, material, rho, support_factor,
                            mass_factor, regions)
        m = b.mass[:, 0]
        q = float(m.min() / np.median(m)) / MIN_MASS_RATIO
        if dt_check is not None and q >= 1.0:   # (a non-positive mass leaves no stable step to compute)
            mu, lam, E = dt_check
            lam_el = (2.0 / critical_dt(b, mu, lam, 0.0)) ** 2
            b.dt_terms = (lam_el, float(np.max(b.nodal_distance / m[: len(b.borders[0]["nodes"]) - 1])))
            nominal = b.nodal_distance * math.sqrt(rho * mass_factor / E)
            q = min(q, 2.0 / math.sqrt(lam_el) / nominal / MIN_DT_RATIO)
        if q >= 1.0:
            return b
        if best is None or q > best[0]:
            best = (q, b)
    if dt_check is not None and best[1].dt_terms is None:
        raise RuntimeError("no draw of this disc has positive lumped masses")
    return best[1]


def _make_disc_once(rng, centre, radius, n_border, n_interior, min_sep, material, rho, support_factor,
                    mass_factor, regions):
    th = 2.0 * np.pi * np.arange(n_border) / n_border
    border = np.stack([centre[0] + radius * np.cos(th), centre[1] + radius * np.sin(th)], axis=1)
    h_b = 2.0 * math.pi * radius / n_border
    interior = _rejection_interior(rng, centre, radius, n_interior, min_sep, border, margin=0.5 * h_b)
    nodes = np.concatenate([border, interior], axis=0)
    tri = _ccw(nodes, Delaunay(nodes).simplices.astype(np.int64))
    edges = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    edges = np.unique(np.sort(edges, axis=1), axis=0)
    h_mean = float(np.mean(np.linalg.norm(nodes[edges[:, 0]] - nodes[edges[:, 1]], axis=1)))
    domain = np.full(nodes.shape[0], support_factor * h_mean)
    # Gauss points (Preprocessor/TriangleGaussPoints.m)
    X1, X2, X3 = nodes[tri[:, 0]], nodes[tri[:, 1]], nodes[tri[:, 2]]
    J = np.abs(X1[:, 0] * (X2[:, 1] - X3[:, 1]) + X2[:, 0] * (X3[:, 1] - X1[:, 1]) + X3[:, 0] * (X1[:, 1] - X2[:, 1])) / 2.0
    gxy = []
    for a1, a2, _ in _GAUSS3:
        a3 = 1.0 - a1 - a2
        gxy.append(a3 * X1 + a1 * X2 + a2 * X3)
    gp_xy = np.stack(gxy, axis=1).reshape(-1, 2)          # cell-major, 3 per cell
    gp_w = np.tile(_GAUSS3[:, 2], tri.shape[0])
    gp_J = np.repeat(J, 3)
    origin = np.asarray(centre, dtype=np.float64)
    gp = mls_shape(gp_xy, nodes, domain, origin)
    sup = mls_shape(nodes, nodes, domain, origin)
    # lumped mass: m_i = rho * sum_g wJ N_gi sum_j N_gj   (AnalyseSimpleBody.m:316-331)
    ptr, idx, N = gp[0], gp[1], gp[2]
    rowsum = np.add.reduceat(N, ptr[:-1])
    c0 = gp_w * gp_J
    contrib = rho * np.repeat(c0 * rowsum, np.diff(ptr)) * N
    m = np.zeros(nodes.shape[0])
    np.add.at(m, idx, contrib)
    m *= mass_factor
    mass = np.stack([m, m], axis=1)
    bl = list(range(n_border)) + [0]
    border_rec = dict(nodes=bl, periodicity=0, interpolant=0, before=0, after=0,
                      bc=[(BC_NONE, (0.0, 0.0), None), (BC_NONE, (0.0, 0.0), None)])
    return Body(kind="deformable", material=material, nodes=nodes, borders=[border_rec], cells=tri,
                nodal_distance=h_b, detection=0.5 * h_b, contact=0.5 * h_b, domain=domain, mass=mass,
                sup=sup, gp_xy=gp_xy, gp_w=gp_w, gp_J=gp_J, gp=gp, n_regions=regions)


def _rigid_mass_props(nodes: np.ndarray, cells: np.ndarray, rho: float):
    """Centre of mass, mass and inertia about the centre of a rigid body from its cells
    (Preprocessor/AnalyseRigidBody.m)."""
    m = 0.0; cx = 0.0; cy = 0.0
    for tri in cells:
        p = nodes[tri]
        area = 0.5 * abs((p[1, 0] - p[0, 0]) * (p[2, 1] - p[0, 1]) - (p[2, 0] - p[0, 0]) * (p[1, 1] - p[0, 1]))
        xc, yc = p[:, 0].mean(), p[:, 1].mean()
        m += area * rho; cx += area * rho * xc; cy += area * rho * yc
    cx /= m; cy /= m
    inertia = 0.0
    for tri in cells:
        p = nodes[tri]
        area = 0.5 * abs((p[1, 0] - p[0, 0]) * (p[2, 1] - p[0, 1]) - (p[2, 0] - p[0, 0]) * (p[1, 1] - p[0, 1]))
        xc, yc = p[:, 0].mean(), p[:, 1].mean()
        inertia += area * rho * ((xc - cx) ** 2 + (yc - cy) ** 2)
        for (a, b) in ((0, 1), (1, 2), (2, 0)):
            A = 0.5 * abs((p[a, 0] - xc) * (p[b, 1] - yc) - (p[b, 0] - xc) * (p[a, 1] - yc))
            PP = (p[a, 0] - xc) ** 2 + (p[a, 1] - yc) ** 2
            PQ = (p[a, 0] - xc) * (p[b, 0] - xc) + (p[a, 1] - yc) * (p[b, 1] - yc)
            QQ = (p[b, 0] - xc) ** 2 + (p[b, 1] - yc) ** 2
            inertia += rho * A / 6.0 * (PP + PQ + QQ)
    return np.array([cx, cy]), m, abs(inertia)


def make_rect_rigid(x0, y0, x1, y1, spacing, material, rho, bcx, bcy, det, con):
    """Rigid rectangle with CCW border nodes of roughly `spacing` and two cells."""
    pts = []
    def edge(a, b):
        L = math.hypot(b[0] - a[0], b[1] - a[1])
        n = max(1, int(math.ceil(L / spacing)))
        for k in range(n):
            t = k / n
            pts.append((a[0] + t * (b[0] - a[0]), a[1] + t * (b[1] - a[1])))
    c = [(x0, y0), (x1, y0), (x1, y1), (x0, y1)]
    corner_idx = []
    for k in range(4):
        corner_idx.append(len(pts))
        edge(c[k], c[(k + 1) % 4])
    nodes = np.array(pts)
    n = nodes.shape[0]
    cells = np.array([[corner_idx[0], corner_idx[1], corner_idx[2]],
                      [corner_idx[0], corner_idx[2], corner_idx[3]]], dtype=np.int64)
    centre, m, inertia = _rigid_mass_props(nodes, cells, rho)
    bl = list(range(n)) + [0]
    border_rec = dict(nodes=bl, periodicity=0, interpolant=0, before=0, after=0, bc=[bcx, bcy])
    return Body(kind="rigid", material=material, nodes=nodes, borders=[border_rec], cells=cells,
                nodal_distance=spacing, detection=det, contact=con, centre=centre,
                rigid_mass=m, rigid_inertia=inertia)


def make_rigid_disc(centre, radius, n, material, rho, det, con, velocity=(0.0, 0.0), angular_velocity=0.0):
    """Free rigid disc: a regular polygon of n CCW border nodes, cells fanned from node 0, no border
    condition (its centre moves and turns under the contact forces alone)."""
    th = 2.0 * np.pi * np.arange(n) / n
    nodes = np.stack([centre[0] + radius * np.cos(th), centre[1] + radius * np.sin(th)], axis=1)
    cells = np.array([[0, k, k + 1] for k in range(1, n - 1)], dtype=np.int64)
    c, m, inertia = _rigid_mass_props(nodes, cells, rho)
    free = (BC_NONE, (0.0, 0.0), None)
    border_rec = dict(nodes=list(range(n)) + [0], periodicity=0, interpolant=0, before=0, after=0, bc=[free, free])
    return Body(kind="rigid", material=material, nodes=nodes, borders=[border_rec], cells=cells,
                nodal_distance=2.0 * math.pi * radius / n, detection=det, contact=con, centre=c,
                rigid_mass=m, rigid_inertia=inertia, velocity=tuple(velocity), angular_velocity=angular_velocity)


def make_periodic_strip_rigid(W, y0, y1, spacing, material, rho, bcx, bcy, det, con):
    """Rigid strip spanning one period [0, W] of the x-periodic domain, y in [y0, y1]: a body of type
    "Periodic" with two "Periodic" borders (Code/Body.h:403-606): border 0 is the lower edge, nodes at
    x = 0, h, ..., W - h walked in +x (its last entry is the first node one period on), border 1 the
    upper edge, nodes at x = W, W - h, ..., h walked in -x (its last entry is its first node one period
    back).  Each border is its own neighbour before and after.  The two cells only give the strip a
    mass; a periodic body never turns."""
    m = max(2, int(math.ceil(W / spacing)))
    h = W / m
    bottom = [(k * h, y0) for k in range(m)]
    top = [(W - k * h, y1) for k in range(m)]
    nodes = np.array(bottom + top)
    cells = np.array([[0, m - 1, m], [0, m, 2 * m - 1]], dtype=np.int64)
    centre, mass, inertia = _rigid_mass_props(nodes, cells, rho)
    b0 = dict(nodes=list(range(m)) + [0], periodicity=2, interpolant=0, before=0, after=0, bc=[bcx, bcy])
    b1 = dict(nodes=list(range(m, 2 * m)) + [m], periodicity=2, interpolant=0, before=1, after=1, bc=[bcx, bcy])
    return Body(kind="rigid", material=material, nodes=nodes, borders=[b0, b1], cells=cells,
                nodal_distance=h, detection=det, contact=con, centre=centre, rigid_mass=mass,
                rigid_inertia=inertia, periodic=1)


# --------------------------------------------------------------------------------------------
# Scene
# --------------------------------------------------------------------------------------------

@dataclasses.dataclass
class Scene:
    name: str
    bodies: List[Body]
    materials: List[Tuple[str, int, List[float]]]     # name, type, file params (rho, alpha, beta, E, nu, heat)
    laws: List[Tuple[str, str, int, int, List[float]]] # mat1, mat2, type, length(0 fixed), file params
    dt: float
    nsteps: int
    contact_update_period: float
    period: Tuple[float, float] = (-1.0, 1.0)
    gravity: Tuple[float, float] = (0.0, 0.0)
    solver: int = 0
    solver_params: Tuple[float, ...] = (1e-3, 0.2, 1.0, 100.0, 1.0, 1.0, 0.99, 1e3)
    self_contact: bool = True
    initialize_czm: bool = False    # INITIALIZE_CZM: internal variables of the set-up contacts (Code/Proximity.h:481)
    update_matrices: Tuple[bool, bool, bool] = (False, False, False)   # UPDATE_MASS/STIFFNESS/DAMPING_MATRIX (Code/IO.h:1920-1925)
    # output control: MONITORING entries as STATIC_CONTROL lines (the Read_spy_line grammar,
    # Code/IO.h:11-590), MONITOR_ENERGY / MONITOR_BOUNDARIES, Save_period and Print_period (None:
    # one save and one print at the end)
    monitored: List[str] = dataclasses.field(default_factory=list)
    monitor_energy: bool = False
    monitor_boundaries: bool = False
    save_period: Optional[float] = None
    print_period: Optional[float] = None
    # DEACTIVATION entries as STATIC_CONTROL lines: a Read_spy_line quantity, then below / equal /
    # above and the threshold (Code/IO.h:947-968)
    deactivation: List[str] = dataclasses.field(default_factory=list)
    meta: dict = dataclasses.field(default_factory=dict)

    @property
    def n_deformable_nodes(self) -> int:
        return int(sum(b.nodes.shape[0] for b in self.bodies if b.kind == "deformable"))


def material_params_stored(mtype: int, p: List[float]) -> List[float]:
    """Parameters as Load_static stores them (Code/IO.h:672-685): rho, alpha, beta, mu, lambda|kappa, heat."""
    E, nu = p[3], p[4]
    mu = E / (2.0 * (1.0 + nu))
    if mtype == 0:
        lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    else:
        lam = E / (3.0 * (1.0 - 2.0 * nu))
    return [p[0], p[1], p[2], mu, lam, p[5]]


_SPY_CODES = {
    "Position": (0, ["X", "Y", "R"]), "Displacement": (1, ["X", "Y", "Mag", "R"]),
    "Velocity": (2, ["X", "Y", "Mag", "R"]), "Acceleration": (3, ["X", "Y", "Mag", "R"]),
}
_FORCE_KINDS = ["Total", "Internal", "Contact", "Body", "Dirichlet", "Neumann", "Damping", "Alid"]


_libm = None


def _cpow(x: float, y: float) -> float:
    """The C library's pow, the one Load_static calls (CPython's ** refuses a negative base)."""
    global _libm
    if _libm is None:
        import ctypes
        import ctypes.util
        _libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
        _libm.pow.restype = ctypes.c_double
        _libm.pow.argtypes = [ctypes.c_double, ctypes.c_double]
    return _libm.pow(x, y)


def alid_coefficients(body: "Body") -> np.ndarray:
    """alid_alpha and alid_beta of every node of a deformable body, as Load_static computes them
    from the initial position while reading NODES (Code/IO.h:1548-1600): layers of width `range`
    inside [ymin, ymax] (bottom/top) and [xmin, xmax] (left/right), graded from *in to *out with
    the given exponent; a node in a side layer keeps the larger of the two values."""
    n = body.nodes.shape[0]
    out = np.zeros((n, 2))
    A = body.alid
    if A is None or (not A["x_hist"] and not A["y_hist"]):
        return out
    ain, aout, bin_, bout, rng_, ex = A["alphain"], A["alphaout"], A["betain"], A["betaout"], A["range"], A["exponent"]
    for i in range(n):
        x, y = float(body.nodes[i, 0]), float(body.nodes[i, 1])
        al = be = 0.0
        if y < A["ymin"] + rng_:
            ka = (aout - ain) / _cpow(-rng_, ex)
            kb = (bout - bin_) / _cpow(-rng_, ex)
            al = ain + ka * _cpow(y - (A["ymin"] + rng_), ex)
            be = bin_ + kb * _cpow(y - (A["ymin"] + rng_), ex)
        elif y > A["ymax"] - rng_:
            ka = (aout - ain) / _cpow(rng_, ex)
            kb = (bout - bin_) / _cpow(rng_, ex)
            al = ain + ka * _cpow(y - (A["ymax"] - rng_), ex)
            be = bin_ + kb * _cpow(y - (A["ymax"] - rng_), ex)
        if x < A["xmin"] + rng_:
            ka = (aout - ain) / _cpow(-rng_, ex)
            kb = (bout - bin_) / _cpow(-rng_, ex)
            t = ain + ka * _cpow(x - (A["xmin"] + rng_), ex)
            if t > al:
                al = t
            t = bin_ + kb * _cpow(x - (A["xmin"] + rng_), ex)
            if t > be:
                be = t
        elif x > A["xmax"] - rng_:
            ka = (aout - ain) / _cpow(rng_, ex)
            kb = (bout - bin_) / _cpow(rng_, ex)
            t = ain + ka * _cpow(x - (A["xmax"] - rng_), ex)
            if t > al:
                al = t
            t = bin_ + kb * _cpow(x - (A["xmax"] - rng_), ex)
            if t > be:
                be = t
        out[i] = (al, be)
    return out


def deactivation_vector(line: str) -> List[float]:
    """The vector Load_static stores for one DEACTIVATION line (Code/IO.h:955-967): the quantity as
    Read_spy_line encodes it (position, displacement, velocity, acceleration or force entries), then
    0 / 1 / 2 for below / equal / above and the threshold, zero-padded to 8 values."""
    t = line.split()
    if t[0] == "Damage":                      # Read_spy_line: {8, body} (Code/IO.h:454-458)
        v = [8.0, float(t[1])]
        rest = t[2:]
        v += [float(["below", "equal", "above"].index(rest[0])), float(rest[1])]
        return v + [0.0] * (8 - len(v))
    if t[0] == "Force":
        v = [4.0, float(["X", "Y", "Mag", "R"].index(t[1])), float(_FORCE_KINDS.index(t[2])), float(t[3]), float(t[4])]
        rest = t[5:]
    else:
        code, comps = _SPY_CODES[t[0]]
        v = [float(code), float(comps.index(t[1])), float(t[2]), float(t[3])]
        rest = t[4:]
    v += [float(["below", "equal", "above"].index(rest[0])), float(rest[1])]
    return v + [0.0] * (8 - len(v))


def stiffness_matrix(body: Body, mu: float, lam: float):
    """The body's linear elastic stiffness K = sum over Gauss points of w J B^T D B (plane strain,
    the linear part of Update_internal_forces, Body.h:974-997), sparse over dofs 2 node + direction."""
    import scipy.sparse as sp
    n = body.nodes.shape[0]
    ptr, idx, _, dx, dy = body.gp
    c0 = body.gp_w * body.gp_J
    G = ptr.shape[0] - 1
    cnt = np.diff(ptr)
    g_of = np.repeat(np.arange(G), cnt)
    # strain rows: e11 = dx*ux, e22 = dy*uy, g12 = dy*ux + dx*uy
    rows_e11 = 3 * g_of; rows_e22 = 3 * g_of + 1; rows_g = 3 * g_of + 2
    r = np.concatenate([rows_e11, rows_e22, rows_g, rows_g])
    c = np.concatenate([2 * idx, 2 * idx + 1, 2 * idx, 2 * idx + 1])
    v = np.concatenate([dx, dy, dy, dx])
    B = sp.csr_matrix((v, (r, c)), shape=(3 * G, 2 * n))
    D = np.array([[lam + 2 * mu, lam, 0.0], [lam, lam + 2 * mu, 0.0], [0.0, 0.0, mu]])
    Dg = sp.kron(sp.diags(c0), sp.csr_matrix(D))
    return (B.T @ Dg @ B).tocsr()


def add_damping(scene: "Scene", alpha: float, beta: float, mu: float, lam: float) -> None:
    """Gives every deformable body a MATRICES list: the upper triangle of its stiffness matrix in
    row-major order, with Rayleigh damping coefficients alpha K_ij (+ beta m_i on the diagonal), the
    matrix Body::Update_damping_forces (Code/Body.h:1057-1154) applies to the velocity parameters."""
    for b in scene.bodies:
        if b.kind != "deformable":
            continue
        K = stiffness_matrix(b, mu, lam).tocoo()
        keep = K.row <= K.col
        r, c, v = K.row[keep], K.col[keep], K.data[keep]
        order = np.lexsort((c, r))
        r, c, v = r[order], c[order], v[order]
        m = b.mass.reshape(-1)
        d = alpha * v + np.where(r == c, beta * m[r], 0.0)
        b.matrices = (np.stack([r, c], axis=1).astype(np.int64), v.astype(np.float64), d.astype(np.float64))


def critical_dt(body: Body, mu: float, lam: float, kn: float) -> float:
    """2/omega_max of the body's lumped-mass elastic operator (the linear part of
    Update_internal_forces, Body.h:974-997), plus the contact penalty kn*length/m of border nodes."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import eigsh
    K = stiffness_matrix(body, mu, lam)
    minv_sqrt = 1.0 / np.sqrt(body.mass.reshape(-1))
    S = sp.diags(minv_sqrt) @ K @ sp.diags(minv_sqrt)
    v0 = np.ones(S.shape[0])
    lam_max = float(eigsh(S, k=1, which="LA", return_eigenvectors=False, tol=1e-6, v0=v0)[0])
    h_b = body.nodal_distance
    m_border = body.mass[: len(body.borders[0]["nodes"]) - 1, 0]
    lam_c = float(np.max(kn * h_b / m_border))
    return 2.0 / math.sqrt(max(lam_max, lam_c))


def disc_lattice_scene(seed: int = 0, nx: int = 4, ny: int = 4, pitch: float = 2.2e-3,
                       rmin: float = 0.9e-3, rmax: float = 1.1e-3, n_border: int = 48,
                       n_interior: int = 100, min_sep: float = 0.1e-3, v_plate: float = 0.01,
                       nsteps: int = 10000, gap0: float = 5e-6, prox_every: int = 10,
                       mass_factor: float = 1.0, name: str = "lattice") -> Scene:
    """Config 0: 4x4 lattice of deformable discs between two rigid plates driven at +-v_plate."""
    rng = np.random.default_rng(seed)
    import random
    prng = random.Random(seed + 1)
    E, nu, rho = 1e8, 0.3, 2500.0
    mats = [("Grain", 0, [rho, 0.0, 0.0, E, nu, 1000.0]), ("Steel", 0, [7800.0, 0.0, 0.0, 2e11, 0.3, 500.0])]
    laws = [("Grain", "Grain", 2, 0, [1e10, 1e9, 0.3, 0.0, 0.0]),
            ("Grain", "Steel", 2, 0, [1e10, 1e9, 0.3, 0.0, 0.0])]
    bodies = []
    radii = rng.uniform(rmin, rmax, size=nx * ny)
    k = 0
    for j in range(ny):
        for i in range(nx):
            c = (0.5 * pitch + i * pitch, 0.5 * pitch + j * pitch)
            bodies.append(make_disc(prng, c, float(radii[k]), n_border, n_interior, min_sep, 0, rho,
                                    mass_factor=mass_factor))
            k += 1
    ymin = min(b.nodes[:, 1].min() for b in bodies)
    ymax = max(b.nodes[:, 1].max() for b in bodies)
    xmin = min(b.nodes[:, 0].min() for b in bodies)
    xmax = max(b.nodes[:, 0].max() for b in bodies)
    h_b = 2.0 * math.pi * rmin / n_border
    margin = 0.1 * (xmax - xmin)
    thick = 0.1 * (xmax - xmin)
    hist = lambda v: (np.array([0.0, T_HIST_END]), np.array([v, v]))
    bot = make_rect_rigid(xmin - margin, ymin - gap0 - thick, xmax + margin, ymin - gap0, h_b, 1, 7800.0,
                          (BC_DRIVEN, (0.0, 0.0), hist(0.0)), (BC_DRIVEN, (0.0, 0.0), hist(v_plate)),
                          0.5 * h_b, 0.5 * h_b)
    top = make_rect_rigid(xmin - margin, ymax + gap0, xmax + margin, ymax + gap0 + thick, h_b, 1, 7800.0,
                          (BC_DRIVEN, (0.0, 0.0), hist(0.0)), (BC_DRIVEN, (0.0, 0.0), hist(-v_plate)),
                          0.5 * h_b, 0.5 * h_b)
    bodies += [bot, top]
    mu = E / (2 * (1 + nu)); lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    dtc = min(critical_dt(b, mu, lam, 1e10) for b in bodies if b.kind == "deformable")
    dt = float("%.4g" % (0.5 * dtc))      # 4 significant digits: reproducible across BLAS builds
    return Scene(name=name, bodies=bodies, materials=mats, laws=laws, dt=dt, nsteps=nsteps,
                 contact_update_period=prox_every * dt,
                 meta=dict(config="lattice", seed=seed, dt_crit=dtc))


def periodic_strip_scene(seed: int = 2, nx: int = 3, ny: int = 2, pitch: float = 2.0e-3, rmin: float = 0.9e-3,
                         rmax: float = 1.1e-3, n_border: int = 32, n_interior: int = 60, min_sep: float = 0.1e-3,
                         v_plate: float = 0.05, nsteps: int = 300, gap0: float = -1e-6, x_shift: float = -0.3,
                         prox_every: int = 10, name: str = "periodic") -> Scene:
    """A lattice of deformable discs in an x-periodic domain of one row's width (period [0, nx*pitch],
    PERIODIC_BOUNDARIES), squeezed between two rigid "Periodic" strips driven at +-v_plate.  The
    lattice is offset by x_shift*pitch, so the first column straddles the periodic seam: its discs
    meet the last column's discs one period away (proximity shifts of -1 and +1), and their nodes
    slide over the strips' seams, where the contact segment walk changes the master shift."""
    rng = np.random.default_rng(seed)
    import random
    prng = random.Random(seed + 1)
    E, nu, rho = 1e8, 0.3, 2500.0
    mats = [("Grain", 0, [rho, 0.0, 0.0, E, nu, 1000.0]), ("Steel", 0, [7800.0, 0.0, 0.0, 2e11, 0.3, 500.0])]
    laws = [("Grain", "Grain", 2, 0, [1e10, 1e9, 0.3, 0.0, 0.0]),
            ("Grain", "Steel", 2, 0, [1e10, 1e9, 0.3, 0.0, 0.0])]
    W = nx * pitch
    radii = rng.uniform(rmin, rmax, size=nx * ny)
    bodies = []
    k = 0
    for j in range(ny):
        for i in range(nx):
            c = ((0.5 + i + x_shift) * pitch, 0.5 * pitch + j * pitch)
            bodies.append(make_disc(prng, c, float(radii[k]), n_border, n_interior, min_sep, 0, rho))
            k += 1
    ymin = min(b.nodes[:, 1].min() for b in bodies)
    ymax = max(b.nodes[:, 1].max() for b in bodies)
    h_b = 2.0 * math.pi * rmin / n_border
    thick = 0.25 * pitch
    hist = lambda v: (np.array([0.0, T_HIST_END]), np.array([v, v]))
    bot = make_periodic_strip_rigid(W, ymin - gap0 - thick, ymin - gap0, h_b, 1, 7800.0,
                                    (BC_DRIVEN, (0.0, 0.0), hist(0.0)), (BC_DRIVEN, (0.0, 0.0), hist(v_plate)),
                                    0.5 * h_b, 0.5 * h_b)
    top = make_periodic_strip_rigid(W, ymax + gap0, ymax + gap0 + thick, h_b, 1, 7800.0,
                                    (BC_DRIVEN, (0.0, 0.0), hist(0.0)), (BC_DRIVEN, (0.0, 0.0), hist(-v_plate)),
                                    0.5 * h_b, 0.5 * h_b)
    bodies += [bot, top]
    mu = E / (2 * (1 + nu)); lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    dtc = min(critical_dt(b, mu, lam, 1e10) for b in bodies if b.kind == "deformable")
    dt = float("%.4g" % (0.5 * dtc))
    return Scene(name=name, bodies=bodies, materials=mats, laws=laws, dt=dt, nsteps=nsteps,
                 contact_update_period=prox_every * dt, period=(0.0, W),
                 meta=dict(config="periodic", seed=seed, dt_crit=dtc))


def rotor_scene(seed: int = 0, omega: float = 200.0, nsteps: int = 300, n_rotor: int = 40, name: str = "rotor") -> Scene:
    """The pressed 3x3 lattice (pitch 2.0 mm, plates starting 1 um inside the outer discs) with its
    centre disc replaced by a free rigid steel disc of the same radius spinning at `omega` rad/s: its
    nodes turn through cos and sin of the body's rotation every step, and the contacts with its four
    neighbours load it with moments."""
    sc = disc_lattice_scene(seed=seed, nx=3, ny=3, pitch=2.0e-3, gap0=-1e-6, nsteps=nsteps, v_plate=0.05, name=name)
    d = sc.bodies[4]
    c = d.nodes[:len(d.borders[0]["nodes"]) - 1].mean(axis=0)
    R = float(np.mean(np.linalg.norm(d.nodes[:len(d.borders[0]["nodes"]) - 1] - c, axis=1)))
    h = 2.0 * math.pi * R / n_rotor
    sc.bodies[4] = make_rigid_disc(c, R, n_rotor, 1, 7800.0, 0.5 * h, 0.5 * h, angular_velocity=omega)
    sc.meta = dict(sc.meta, config="rotor", omega=omega)
    return sc


# --------------------------------------------------------------------------------------------
# Flattening (the arrays behind mel_model_desc)
# --------------------------------------------------------------------------------------------

def flatten(scene: Scene) -> Dict[str, np.ndarray]:
    """Structure-of-arrays view of the scene, field by field as in mel_model_desc (include/melgpu.h)."""
    f: Dict[str, object] = {}
    nb = len(scene.bodies)
    f["period"] = np.array(scene.period, dtype=np.float64)
    f["gravity"] = np.array(scene.gravity, dtype=np.float64)
    f["time"] = 0.0
    f["dt"] = float(scene.dt)
    f["tend"] = float(scene.dt * scene.nsteps)
    f["contact_update_period"] = float(scene.contact_update_period)
    f["next_contact_update"] = 0.0
    f["solver"] = int(scene.solver)
    sp_ = list(scene.solver_params)
    if scene.solver not in (2, 3):          # Code/IO.h:821-893 reads these only for mass scaling
        sp_[3:7] = [0.0, 0.0, 0.0, 0.0]
    if scene.solver == 4:
        sp_[0:3] = [0.0, 0.0, 0.0]
        sp_[7] = 0.0
    else:
        sp_[7] = 1.0 / sp_[0]
    f["solver_params"] = np.array(sp_, dtype=np.float64)
    flags = np.zeros(11, dtype=np.int32)
    flags[7] = 1                          # NO_LOG
    if not scene.self_contact:
        flags[8] = 1                      # NO_MONITORING (also disables self contact, Proximity.h:332)
    if scene.initialize_czm:
        flags[3] = 1                      # INITIALIZE_CZM
    for k, on in enumerate(scene.update_matrices):
        flags[4 + k] = int(bool(on))      # rebuilt by Body::Update_material (Code/Body.h:2708-2875)
    flags[1] = int(scene.monitor_energy)
    flags[2] = int(scene.monitor_boundaries)
    f["flags"] = flags
    names = [m[0] for m in scene.materials]
    f["material_type"] = np.array([m[1] for m in scene.materials], dtype=np.int32)
    f["material_params"] = np.array([material_params_stored(m[1], m[2]) for m in scene.materials],
                                    dtype=np.float64).reshape(-1)
    nl = len(scene.laws)
    f["law_type"] = np.array([l[2] for l in scene.laws], dtype=np.int32)
    f["law_length"] = np.array([l[3] for l in scene.laws], dtype=np.int32)
    lp = np.zeros((nl, 11))
    for i, l in enumerate(scene.laws):
        lp[i, :len(l[4])] = l[4]
    f["law_params"] = lp.reshape(-1)
    nm = len(names)
    table = -np.ones((nm, nm), dtype=np.int32)
    for i, l in enumerate(scene.laws):       # Code/IO.h:797-812 (last law wins)
        a = names.index(l[0]); b = names.index(l[1])
        table[a, b] = i; table[b, a] = i
    f["contacts_table"] = table.reshape(-1)
    f["body_type"] = np.array([0 if b.kind == "deformable" else 1 for b in scene.bodies], dtype=np.int32)
    f["body_material"] = np.array([b.material for b in scene.bodies], dtype=np.int32)
    f["body_periodic"] = np.array([b.periodic for b in scene.bodies], dtype=np.int32)
    f["body_status"] = np.array([b.status for b in scene.bodies], dtype=np.int32)
    f["body_dist"] = np.array([[b.nodal_distance, b.detection, b.contact] for b in scene.bodies]).reshape(-1)
    nn = np.array([b.nodes.shape[0] for b in scene.bodies])
    f["body_node_ptr"] = np.concatenate([[0], np.cumsum(nn)]).astype(np.int32)
    nbd = np.array([len(b.borders) for b in scene.bodies])
    f["body_border_ptr"] = np.concatenate([[0], np.cumsum(nbd)]).astype(np.int32)
    ng = np.array([0 if b.gp is None else b.gp[0].shape[0] - 1 for b in scene.bodies])
    f["body_gp_ptr"] = np.concatenate([[0], np.cumsum(ng)]).astype(np.int32)
    nc = np.array([b.cells.shape[0] for b in scene.bodies])
    f["body_cell_ptr"] = np.concatenate([[0], np.cumsum(nc)]).astype(np.int32)
    rigid = np.zeros((nb, 20))
    for i, b in enumerate(scene.bodies):
        if b.kind == "rigid":
            rigid[i, 0:2] = b.centre
            rigid[i, 3] = b.rigid_mass
            rigid[i, 4] = b.rigid_inertia
            rigid[i, 5] = 1.0 / b.rigid_mass
            rigid[i, 6] = 1.0 / b.rigid_inertia
            rigid[i, 13:15] = b.velocity
            rigid[i, 15] = b.angular_velocity
    f["rigid"] = rigid.reshape(-1)
    N = int(nn.sum())
    x0 = np.concatenate([b.nodes for b in scene.bodies])
    f["node_x0"] = x0.reshape(-1).astype(np.float64)
    mass = np.zeros((N, 2)); dom = np.zeros(N)
    o = 0
    for b in scene.bodies:
        n = b.nodes.shape[0]
        if b.kind == "deformable":
            mass[o:o + n] = b.mass
            dom[o:o + n] = b.domain
        o += n
    f["node_mass"] = mass.reshape(-1)
    with np.errstate(divide="ignore"):
        inv = np.where(mass > 0, 1.0 / np.where(mass > 0, mass, 1.0), 0.0)
    f["node_inv_mass"] = inv.reshape(-1)
    f["node_domain"] = dom
    sptr = [np.zeros(1, dtype=np.int64)]; sidx = []; sN = []
    base = 0
    for b in scene.bodies:
        n = b.nodes.shape[0]
        if b.kind == "deformable":
            p, ix, Nv, _, _ = b.sup
            sptr.append(base + p[1:]); sidx.append(ix); sN.append(Nv)
            base += int(p[-1])
        else:
            sptr.append(np.full(n, base, dtype=np.int64))
    f["node_sup_ptr"] = np.concatenate(sptr).astype(np.int32)
    f["node_sup_idx"] = (np.concatenate(sidx) if sidx else np.zeros(0)).astype(np.int32)
    f["node_sup_N"] = (np.concatenate(sN) if sN else np.zeros(0)).astype(np.float64)
    state = np.zeros((N, 12))
    o = 0
    for b in scene.bodies:
        n = b.nodes.shape[0]
        state[o:o + n, 2:4] = b.velocity      # nodal velocity
        state[o:o + n, 8:10] = b.velocity     # velocity parameters
        o += n
    f["node_state"] = state.reshape(-1)
    bb, bper, bint, bbef, baft, bptr, bnodes, bct, bcp, hptr, ht, hv = ([] for _ in range(12))
    bptr.append(0); hptr.append(0)
    for bi, b in enumerate(scene.bodies):
        for br in b.borders:
            bb.append(bi); bper.append(br["periodicity"]); bint.append(br["interpolant"])
            bbef.append(br["before"]); baft.append(br["after"])
            bnodes.extend(br["nodes"]); bptr.append(len(bnodes))
            for d in range(2):
                t, prm, hist = br["bc"][d]
                bct.append(t); bcp.extend(prm)
                if hist is not None:
                    ht.extend(hist[0]); hv.extend(hist[1])
                hptr.append(len(ht))
    f["border_body"] = np.array(bb, dtype=np.int32)
    f["border_periodicity"] = np.array(bper, dtype=np.int32)
    f["border_interpolant"] = np.array(bint, dtype=np.int32)
    f["border_before"] = np.array(bbef, dtype=np.int32)
    f["border_after"] = np.array(baft, dtype=np.int32)
    f["border_node_ptr"] = np.array(bptr, dtype=np.int32)
    f["border_nodes"] = np.array(bnodes, dtype=np.int32)
    f["border_bc_type"] = np.array(bct, dtype=np.int32)
    f["border_bc_param"] = np.array(bcp, dtype=np.float64)
    f["border_hist_ptr"] = np.array(hptr, dtype=np.int32)
    f["hist_time"] = np.array(ht, dtype=np.float64)
    f["hist_value"] = np.array(hv, dtype=np.float64)
    gptr = [np.zeros(1, dtype=np.int64)]; gidx = []; gN = []; gx = []; gy = []; gw = []; gJ = []
    base = 0
    for b in scene.bodies:
        if b.gp is None:
            continue
        p, ix, Nv, dx, dy = b.gp
        gptr.append(base + p[1:]); gidx.append(ix); gN.append(Nv); gx.append(dx); gy.append(dy)
        gw.append(b.gp_w); gJ.append(b.gp_J)
        base += int(p[-1])
    f["gp_sup_ptr"] = np.concatenate(gptr).astype(np.int32)
    f["gp_sup_idx"] = np.concatenate(gidx).astype(np.int32)
    f["gp_N"] = np.concatenate(gN).astype(np.float64)
    f["gp_dNdx"] = np.concatenate(gx).astype(np.float64)
    f["gp_dNdy"] = np.concatenate(gy).astype(np.float64)
    f["gp_weight"] = np.concatenate(gw).astype(np.float64)
    f["gp_jacobian"] = np.concatenate(gJ).astype(np.float64)
    f["cells"] = np.concatenate([b.cells for b in scene.bodies]).reshape(-1).astype(np.int32)
    mptr = [0]; mdofs = []; mk = []; mc = []
    for b in scene.bodies:
        if b.matrices is not None:
            mdofs.append(b.matrices[0].reshape(-1)); mk.append(b.matrices[1]); mc.append(b.matrices[2])
            mptr.append(mptr[-1] + b.matrices[1].shape[0])
        else:
            mptr.append(mptr[-1])
    f["body_matrix_ptr"] = np.array(mptr, dtype=np.int32)
    f["matrix_dofs"] = np.concatenate(mdofs).astype(np.int32) if mdofs else np.zeros(0, dtype=np.int32)
    f["matrix_stiffness"] = np.concatenate(mk).astype(np.float64) if mk else np.zeros(0, dtype=np.float64)
    f["matrix_damping"] = np.concatenate(mc).astype(np.float64) if mc else np.zeros(0, dtype=np.float64)
    f["deactivated"] = np.array([deactivation_vector(line) for line in scene.deactivation],
                                dtype=np.float64).reshape(-1, 8)
    if any(b.alid is not None for b in scene.bodies):
        aptr = [0]; at = []; av = []; ab = []
        for b in scene.bodies:
            for key in ("x_hist", "y_hist"):
                h = b.alid[key] if b.alid is not None else []
                at += [float(t) for t, _ in h]; av += [float(v) for _, v in h]
                aptr.append(len(at))
            ab.append(alid_coefficients(b) if b.kind == "deformable" else np.zeros((b.nodes.shape[0], 2)))
        f["body_alid_ptr"] = np.array(aptr, dtype=np.int32)
        f["alid_time"] = np.array(at, dtype=np.float64)
        f["alid_value"] = np.array(av, dtype=np.float64)
        f["node_alid"] = np.concatenate(ab).reshape(-1).astype(np.float64)
    f["material_names"] = names
    return f  # type: ignore[return-value]


# --------------------------------------------------------------------------------------------
# ASCII writer (Preprocessor/ExportStatic.m, Preprocessor/ExportDynamic.m layouts)
# --------------------------------------------------------------------------------------------

def _g(x: float) -> str:
    return repr(float(x)) if math.isfinite(x) else str(x)


def _bc_lines(axis: str, bc) -> List[str]:
    t, prm, hist = bc
    if t == BC_NONE:
        return [f"{axis} None"]
    out = []
    if t == BC_DRIVEN:
        out.append(f"{axis} Dirichlet Driven")
    elif t == BC_SOFT:
        out.append(f"{axis} Dirichlet Soft {_g(prm[0])} {_g(prm[1])}")
    elif t == BC_ORIENTED:
        out.append(f"{axis} Neumann Oriented")
    elif t == BC_FOLLOWING:
        out.append(f"{axis} Neumann Following")
    out.append(str(len(hist[0])))
    out += [f"{_g(a)} {_g(b)}" for a, b in zip(hist[0], hist[1])]
    return out


def write_asc(scene: Scene, directory: str, workers: int = 1) -> None:
    """Write STATIC_CONTROL.asc, STATIC_DATA.asc and DYNAMIC_00000.asc readable by Load_static /
    Load_dynamic (Code/IO.h).  Numbers use 17 significant digits so the files round-trip.  With
    workers > 1 the bodies' blocks are formatted in that many forked processes (a 2000-disc
    sample is 6 GB of text); fork only from a process that holds no CUDA context."""
    os.makedirs(directory, exist_ok=True)
    mats = scene.materials
    names = [m[0] for m in mats]
    per = ["Closed", "Simple", "Periodic"]
    itp = ["Linear", "Spline"]
    L: List[str] = [" ", "SIMULATION_NAME", scene.name, " ", "MATERIALS", str(len(mats)), " "]
    for name, t, p in mats:
        L += [name, MAT_NAMES[t], " ".join(_g(v) for v in p) + " ", " "]
    L += [" ", "CONTACT_LAWS", str(len(scene.laws)), " "]
    for m1, m2, t, le, p in scene.laws:
        L += [m1, m2, LAW_NAMES[t], ["Fixed", "Evolutive"][le],
              " ".join(_g(v) for v in p[:LAW_NPARAM_FILE[t]]) + " ", " "]
    tend = scene.dt * scene.nsteps
    sp_ = scene.solver_params
    L += [" ", "SOLVER", SOLVER_NAMES[scene.solver], f"{_g(0.0)} {_g(scene.dt)} {_g(tend)}"]
    if scene.solver != 4:
        L.append(f"{_g(sp_[0])} {_g(sp_[1])} {_g(sp_[2])}")
    if scene.solver in (2, 3):
        L.append(f"{_g(sp_[3])} {_g(sp_[4])} {_g(sp_[5])} {_g(sp_[6])}")
    save = scene.save_period if scene.save_period is not None else tend
    prnt = scene.print_period if scene.print_period is not None else tend
    L += [f"{_g(save)} {_g(prnt)} {_g(scene.contact_update_period)}", " ",
          "PERIODIC_BOUNDARIES", f"{_g(scene.period[0])} {_g(scene.period[1])}", " ",
          "GRAVITY", f"{_g(scene.gravity[0])} {_g(scene.gravity[1])}", " ",
          "NUMBER_BODIES", str(len(scene.bodies)), " ",
          "MONITORING", str(len(scene.monitored))] + list(scene.monitored) + [
          " ", "SPIES", "0", " ", "DEACTIVATION", str(len(scene.deactivation))] + list(scene.deactivation) + [" "]
    for bi, b in enumerate(scene.bodies):
        L += [" ", "DEFORMABLE" if b.kind == "deformable" else "RIGID", str(bi), names[b.material],
              "Periodic" if b.periodic else "Simple",
              f"{_g(b.nodal_distance)} {_g(b.detection)} {_g(b.contact)}", " ",
              "NODES", str(b.nodes.shape[0]), " ", "BORDERS", str(len(b.borders)), " "]
        for br in b.borders:
            L += [f"{per[br['periodicity']]} {itp[br['interpolant']]}", str(len(br["nodes"]))]
            L += _bc_lines("X", br["bc"][0])
            L += _bc_lines("Y", br["bc"][1])
            L += [" "]
        if b.kind == "deformable":
            L += ["INTEGRATION", f"{b.gp[0].shape[0] - 1} {b.n_regions}", " "]
        L += ["TRIANGULATION", str(b.cells.shape[0]), " ", " "]
        if b.alid is not None:
            # Load_static reads the twelve numbers, skips the rest of their line and one more line,
            # then the x history, one separating line when both exist, and the y history
            A = b.alid
            L += ["ALID", " ".join([str(len(A["x_hist"])), str(len(A["y_hist"]))] +
                                   [_g(A[k]) for k in ("xmin", "xmax", "ymin", "ymax", "range", "alphain",
                                                       "alphaout", "betain", "betaout", "exponent")]), " "]
            L += [f"{_g(t)} {_g(v)}" for t, v in A["x_hist"]]
            if A["x_hist"] and A["y_hist"]:
                L += [" "]
            L += [f"{_g(t)} {_g(v)}" for t, v in A["y_hist"]]
            L += [" "]
    with open(os.path.join(directory, "STATIC_CONTROL.asc"), "w") as fh:
        fh.write("\n".join(L) + "\n")

    parts = _write_body_parts(scene, workers)
    with open(os.path.join(directory, "STATIC_DATA.asc"), "w") as fh:
        fh.write(" \nSIMULATION_NAME\n%s\n \n \nNUMBER_BODIES\n%d\n \n \n" % (scene.name, len(scene.bodies)))
        for text in _collect(parts, 0):
            fh.write(text)
    with open(os.path.join(directory, "DYNAMIC_00000.asc"), "w") as fh:
        tend = scene.dt * scene.nsteps
        fh.write(" \nSIMULATION_NAME\n%s\n \nSOLVER\n%s\n0 0 0 0 \n%s\n%s %s %s \nNO_LOG\n" % (
            scene.name, SOLVER_NAMES[scene.solver], _g(scene.dt), _g(save), _g(prnt), _g(0.0)))
        if not scene.self_contact:
            fh.write("NO_MONITORING\n")
        if scene.monitor_energy:
            fh.write("MONITOR_ENERGY\n")
        if scene.monitor_boundaries:
            fh.write("MONITOR_BOUNDARIES\n")
        if scene.initialize_czm:
            fh.write("INITIALIZE_CZM\n")
        for on, kw in zip(scene.update_matrices, ("UPDATE_MASS_MATRIX", "UPDATE_STIFFNESS_MATRIX", "UPDATE_DAMPING_MATRIX")):
            if on:
                fh.write(kw + "\n")
        fh.write(" \n")
        for text in _collect(parts, 1):
            fh.write(text)
    for part in parts:
        if part[0] is not None:
            for path in part:
                os.unlink(path)
            tmp = os.path.dirname(part[0])
    if parts and parts[0][0] is not None:
        os.rmdir(tmp)


def _static_data_body(bi: int, b: Body) -> str:
    """The block of body bi in STATIC_DATA.asc (Preprocessor/ExportStatic.m layout)."""
    out: List[str] = []
    w = out.append
    n = b.nodes.shape[0]
    per = ["Closed", "Simple", "Periodic"]
    itp = ["Linear", "Spline"]
    if b.kind == "deformable":
        w(" \nDEFORMABLE\n%d\n \nNODES\n%d\n \n" % (bi, n))
        inv = 1.0 / b.mass
        for i in range(n):
            w("%d %s %s %s %s %s %s %s\n" % (i, _g(b.nodes[i, 0]), _g(b.nodes[i, 1]), _g(b.domain[i]),
                                             _g(b.mass[i, 0]), _g(b.mass[i, 1]), _g(inv[i, 0]), _g(inv[i, 1])))
    else:
        w(" \nRIGID\n%d\n%s %s\n%s %s %s %s\n \nNODES\n%d\n \n" % (
            bi, _g(b.centre[0]), _g(b.centre[1]), _g(b.rigid_mass), _g(b.rigid_inertia),
            _g(1.0 / b.rigid_mass), _g(1.0 / b.rigid_inertia), n))
        for i in range(n):
            w("%d %s %s\n" % (i, _g(b.nodes[i, 0]), _g(b.nodes[i, 1])))
    w(" \nBORDERS\n%d\n \n" % len(b.borders))
    for br in b.borders:
        w("%s %s\n%d %d %d\n" % (per[br["periodicity"]], itp[br["interpolant"]], len(br["nodes"]),
                                  br["before"], br["after"]))
        w("".join("%d\n" % k for k in br["nodes"]))
        w(" \n")
    if b.kind == "deformable":
        ptr, idx, Nv, dx, dy = b.gp
        w("INTEGRATION\nGauss\n%d %d\n \n" % (ptr.shape[0] - 1, b.n_regions))
        for g in range(ptr.shape[0] - 1):
            w("Gauss Point %d\n%s %s %s %s\n%d\n" % (g, _g(b.gp_xy[g, 0]), _g(b.gp_xy[g, 1]),
                                                      _g(b.gp_w[g]), _g(b.gp_J[g]), ptr[g + 1] - ptr[g]))
            for e in range(ptr[g], ptr[g + 1]):
                k = idx[e]
                w("%d %d %d %s %s %s\n" % (k, 2 * k, 2 * k + 1, _g(Nv[e]), _g(dx[e]), _g(dy[e])))
            w(" \n")
    w("TRIANGULATION\n%d\n" % b.cells.shape[0])
    for c, t in enumerate(b.cells):
        w("%d %d %d %d\n" % (c, t[0], t[1], t[2]))
    w(" \n")
    if b.kind == "deformable":
        ptr, idx, Nv, dx, dy = b.sup
        w("DOF_TO_DISP\n")
        for i in range(n):
            w(" \nNODE %d\n%d\n" % (i, ptr[i + 1] - ptr[i]))
            for e in range(ptr[i], ptr[i + 1]):
                w("%d %s %s %s\n" % (idx[e], _g(Nv[e]), _g(dx[e]), _g(dy[e])))
        if b.matrices is None:
            w(" \n \nMATRICES\n0\n \n \n \n \n")
        else:
            dofs, kv, cv = b.matrices
            w(" \n \nMATRICES\n%d\n \n" % kv.shape[0])
            for (d0, d1), k_, c_ in zip(dofs, kv, cv):
                w("%d %d %s %s\n" % (d0, d1, _g(k_), _g(c_)))
            w(" \n \n \n")
    return "".join(out)


def _dynamic_body(bi: int, b: Body) -> str:
    """The block of body bi in DYNAMIC_00000.asc (Preprocessor/ExportDynamic.m layout)."""
    out: List[str] = []
    w = out.append
    n = b.nodes.shape[0]
    vx, vy = b.velocity
    if b.kind == "deformable":
        w(" \nDEFORMABLE\nactive\n%d\n \nKINEMATICS\n%d\n" % (bi, n))
        for i in range(n):
            w("%d %s %s 0 0 %s %s 0 0 0 0 %s %s 0 0\n" % (i, _g(b.nodes[i, 0]), _g(b.nodes[i, 1]),
                                                        _g(vx), _g(vy), _g(vx), _g(vy)))
        w(" \nFORCES\n")
        for i in range(n):
            w("%d 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0 0\n" % i)
        w(" \nNEIGHBOURS\n0\n \nCONTACTS\n0\n \n")
    else:
        w(" \nRIGID\nactive\n%d\n \nKINEMATICS\n%s %s 0\n0 0 0\n%s %s %s\n \n" % (
            bi, _g(b.centre[0]), _g(b.centre[1]), _g(vx), _g(vy), _g(b.angular_velocity)))
        w("FORCES\n0 0 0\n0 0 0\n0 0 0\n0 0 0\n0 0 0\n0 0 0\n \nNEIGHBOURS\n0\n \nCONTACTS\n0\n \n")
    return "".join(out)


_WRITE_SCENE: Optional[Scene] = None


def _write_range(job):
    """Worker: the STATIC_DATA and DYNAMIC blocks of bodies [b0, b1) into two temporary files."""
    b0, b1, tmpdir = job
    paths = []
    for k, fn in enumerate((_static_data_body, _dynamic_body)):
        path = os.path.join(tmpdir, "part%07d_%d.asc" % (b0, k))
        with open(path, "w") as fh:
            for bi in range(b0, b1):
                fh.write(fn(bi, _WRITE_SCENE.bodies[bi]))
        paths.append(path)
    return tuple(paths)


def _write_body_parts(scene: Scene, workers: int):
    """Per-body text of both files: in this process (a list of string pairs), or, with workers > 1,
    in forked workers that each write a range of bodies to temporary files (a list of path pairs)."""
    global _WRITE_SCENE
    nb = len(scene.bodies)
    if workers <= 1 or nb < 2 * workers:
        return [(None, _static_data_body(bi, b), _dynamic_body(bi, b)) for bi, b in enumerate(scene.bodies)]
    import multiprocessing as mp
    import tempfile
    tmpdir = tempfile.mkdtemp(prefix="melasc")
    step = (nb + 4 * workers - 1) // (4 * workers)
    jobs = [(b0, min(nb, b0 + step), tmpdir) for b0 in range(0, nb, step)]
    _WRITE_SCENE = scene
    try:
        with mp.get_context("fork").Pool(workers) as pool:
            return list(pool.map(_write_range, jobs))
    finally:
        _WRITE_SCENE = None


def _collect(parts, k):
    for part in parts:
        if part[0] is None:
            yield part[1 + k]
        else:
            with open(part[k]) as fh:
                while True:
                    chunk = fh.read(1 << 24)
                    if not chunk:
                        break
                    yield chunk


# --------------------------------------------------------------------------------------------
# Biaxial grain packings (the 2000-disc workload and the batched sample distribution)
# --------------------------------------------------------------------------------------------

def _rsa_pack(rng, radii, width, height, gap, max_tries=2000):
    """Seeded random sequential addition, largest discs first, inside [0,width]x[0,height]."""
    order = np.argsort(-radii, kind="stable")
    cell = 2.0 * float(radii.max()) + gap
    grid: Dict[Tuple[int, int], List[int]] = {}
    centres = np.zeros((len(radii), 2))
    placed = np.zeros(len(radii), dtype=bool)
    for i in order:
        r = radii[i]
        for _ in range(max_tries):
            x = rng.uniform(r + gap, width - r - gap)
            y = rng.uniform(r + gap, height - r - gap)
            gx, gy = int(x // cell), int(y // cell)
            ok = True
            for ix in range(gx - 1, gx + 2):
                for iy in range(gy - 1, gy + 2):
                    for j in grid.get((ix, iy), ()):
                        dx = centres[j, 0] - x; dy = centres[j, 1] - y
                        if dx * dx + dy * dy < (r + radii[j] + gap) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                centres[i] = (x, y)
                placed[i] = True
                grid.setdefault((gx, gy), []).append(i)
                break
    return centres, placed


def _disc_worker(args):
    seed, centre, radius, n_border, n_interior, rho, mass_factor = args[:7]
    import random as _r
    prng = _r.Random(int(seed))
    area = math.pi * radius * radius
    h = math.sqrt(area / (n_border + n_interior))
    # with (mu, lambda, E): draws checked for their critical step, which the disc then carries
    return make_disc(prng, centre, radius, n_border, n_interior, 0.6 * h, 0, rho, mass_factor=mass_factor,
                     dt_check=args[7] if len(args) > 7 else None)


def make_discs_parallel(jobs, workers: Optional[int] = None):
    """Builds discs in a spawn-started process pool (no fork after CUDA initialisation)."""
    if workers is None:
        workers = max(1, min(32, (os.cpu_count() or 2)))
    if workers <= 1 or len(jobs) < 16:
        return [_disc_worker(j) for j in jobs]
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    ctx = mp.get_context("spawn")
    with ProcessPoolExecutor(max_workers=workers, mp_context=ctx) as ex:
        return list(ex.map(_disc_worker, jobs, chunksize=max(1, len(jobs) // (4 * workers))))


def contact_distance(sigma: float, radius: float, kn: float = 1e10, peak: float = 3.0, margin: float = 1.3) -> float:
    """Contact (and detection) distance a biaxial sample needs so that its contact elements survive
    the penetration its loading causes.  Update_proximity keeps a node-to-segment candidate only
    while its gap is above -contact_distance (Code/Proximity.h:269), and the penalty law
    Pn = -kn * gapn (Code/Model.h:123-128) balances a stress s with a penetration g: a disc of radius
    R pressed on a flat side carries kn (4/3) sqrt(2R) g^(3/2) per unit depth against s * 2R, so
    g = (3/4 s sqrt(2R) / kn)^(2/3).  With kn = 1e10 Pa/m and 100 kPa this is about 50 um for a
    1 mm disc, more than half the border-node spacing; a contact distance of half that spacing
    drops the contacts at every proximity update and the walls pass through the grains.  The
    distance is taken at `peak` times the confining stress (the axial stress of the compression),
    with a `margin`."""
    g = (0.75 * peak * sigma * math.sqrt(2.0 * radius) / kn) ** (2.0 / 3.0)
    return margin * g


def biaxial_scene(seed: int = 1, n_discs: int = 2000, rmin: float = 0.5e-3, rmax: float = 1.5e-3,
                  n_border: int = 64, n_interior: int = 340, aspect: float = 100.0 / 60.0, fill: float = 0.45,
                  gap: float = 0.02e-3, v_plate: float = 0.05, sigma: float = 100e3, mass_factor: float = 100.0,
                  mu_fric: float = 0.3, nsteps: int = 50000, prox_every: int = 10, workers: Optional[int] = None,
                  name: str = "biaxial") -> Scene:
    """Biaxial compression sample: polydisperse deformable discs packed by seeded random sequential
    addition, rigid top/bottom plates driven towards each other at v_plate, rigid lateral walls
    loaded by a constant confining pressure (Neumann, oriented) and fixed vertically.

    The box keeps the workload's 100:60 aspect ratio but is sized so the discs fill `fill` of it
    (2000 discs with radii in [0.5,1.5] mm cover 1.13x the area of a 100x60 mm box)."""
    rng = np.random.default_rng(seed)
    radii = rng.uniform(rmin, rmax, size=n_discs)
    area = float(np.sum(np.pi * radii ** 2))
    W = math.sqrt(area / fill * aspect)
    H = W / aspect
    centres, placed = _rsa_pack(rng, radii, W, H, gap)
    tries = 0
    while not placed.all() and tries < 5:      # enlarge slightly until every disc fits
        W *= 1.03; H *= 1.03; tries += 1
        centres, placed = _rsa_pack(rng, radii, W, H, gap)
    if not placed.all():
        raise RuntimeError("packing failed")
    E, nu, rho = 1e8, 0.3, 2500.0
    rho_steel = 7800.0 * mass_factor        # mass scaling applies to the rigid plates and walls too
    mats = [("Grain", 0, [rho, 0.0, 0.0, E, nu, 1000.0]), ("Steel", 0, [rho_steel, 0.0, 0.0, 2e11, 0.3, 500.0])]
    # plates and walls overlap at the corners; a zero-stiffness law makes rigid-rigid contact inert
    laws = [("Grain", "Grain", 2, 0, [1e10, 1e9, mu_fric, 0.0, 0.0]),
            ("Grain", "Steel", 2, 0, [1e10, 1e9, mu_fric, 0.0, 0.0]),
            ("Steel", "Steel", 0, 0, [0.0])]
    seeds = rng.integers(0, 2 ** 31 - 1, size=n_discs)
    mu = E / (2 * (1 + nu)); lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    jobs = [(int(seeds[i]), (float(centres[i, 0]), float(centres[i, 1])), float(radii[i]), n_border, n_interior,
             rho, mass_factor, (mu, lam, E)) for i in range(n_discs)]
    bodies = make_discs_parallel(jobs, workers)
    for b, r in zip(bodies, radii):
        b.detection = b.contact = max(b.contact, contact_distance(sigma, float(r)))
    h_min = 2.0 * math.pi * rmin / n_border
    bodies += _biaxial_frame(W, H, h_min, rho_steel, v_plate, sigma, contact_distance(sigma, rmax))
    # every disc's own critical step: a disc whose node layout leaves one node with a small lumped
    # mass can have a critical step below the smallest discs' (a 1.1 mm disc of the 2000-disc
    # sample at 0.97 us against 2.3 us), and runs unstable once a contact excites it
    kn = 1e10
    dtc = min(2.0 / math.sqrt(max(b.dt_terms[0], kn * b.dt_terms[1])) for b in bodies[:n_discs])
    dt = float("%.4g" % (0.5 * dtc))
    return Scene(name=name, bodies=bodies, materials=mats, laws=laws, dt=dt, nsteps=nsteps,
                 contact_update_period=prox_every * dt,
                 meta=dict(config="biaxial", seed=seed, dt_crit=dtc, box=(W, H), n_discs=n_discs,
                           radii=(rmin, rmax), sigma=sigma, v_plate=v_plate, mass_factor=mass_factor))


def _biaxial_frame(W: float, H: float, h_min: float, rho_steel: float, v_plate: float, sigma: float,
                   dist: float = 0.0) -> List[Body]:
    """Rigid plates (bottom, top) driven towards each other at v_plate and lateral walls (left,
    right) loaded by the confining pressure sigma, fixed vertically; detection and contact distance
    max(h_min / 2, dist)."""
    thick = 0.05 * H
    dd = max(0.5 * h_min, dist)
    hist = lambda v: (np.array([0.0, T_HIST_END]), np.array([v, v]))
    # plates span the box and the walls' inward travel; walls span the plates' full height, so no
    # grain can leave the sample through a corner
    bot = make_rect_rigid(-0.1 * W, -thick, 1.1 * W, 0.0, 2.0 * h_min, 1, rho_steel,
                          (BC_DRIVEN, (0.0, 0.0), hist(0.0)), (BC_DRIVEN, (0.0, 0.0), hist(v_plate)), dd, dd)
    top = make_rect_rigid(-0.1 * W, H, 1.1 * W, H + thick, 2.0 * h_min, 1, rho_steel,
                          (BC_DRIVEN, (0.0, 0.0), hist(0.0)), (BC_DRIVEN, (0.0, 0.0), hist(-v_plate)), dd, dd)
    wall_h = H + 2.0 * thick
    y0 = -thick
    perim = 2.0 * (wall_h + thick)
    p_eff = sigma * H / perim               # oriented load per unit border length, total = sigma * sample height
    left = make_rect_rigid(-thick, y0, 0.0, y0 + wall_h, 2.0 * h_min, 1, rho_steel,
                           (BC_ORIENTED, (0.0, 0.0), hist(p_eff)), (BC_DRIVEN, (0.0, 0.0), hist(0.0)), dd, dd)
    right = make_rect_rigid(W, y0, W + thick, y0 + wall_h, 2.0 * h_min, 1, rho_steel,
                            (BC_ORIENTED, (0.0, 0.0), hist(-p_eff)), (BC_DRIVEN, (0.0, 0.0), hist(0.0)), dd, dd)
    return [bot, top, left, right]


# --------------------------------------------------------------------------------------------
# batched workload: many independent biaxial samples whose grains are scaled disc templates
# --------------------------------------------------------------------------------------------
def _dt_terms(body: Body, mu: float, lam: float):
    """Largest eigenvalue of the lumped-mass elastic operator and the contact term kn*h/m per unit
    kn, the two parts of critical_dt, for the body as built."""
    lam_el = (2.0 / critical_dt(body, mu, lam, 0.0)) ** 2
    h_b = body.nodal_distance
    m_border = body.mass[: len(body.borders[0]["nodes"]) - 1, 0]
    return lam_el, float(np.max(h_b / m_border))


class DiscTemplates:
    """Unit-radius deformable discs, one per border-node count, with interior_factor x that many
    interior nodes (density 1, no mass scaling), and the two critical-time-step terms of each.
    A grain of radius r is a template scaled by r: N is unchanged, dN/dx and dN/dy scale by 1/r,
    weight x jacobian and masses by r^2 (times density and mass factor); the elastic eigenvalue
    scales by 1/r^2 and the contact term by 1/r (both divided by density x mass factor)."""

    def __init__(self, border_counts, interior_factor: int = 5, seed: int = 20240, workers: Optional[int] = None,
                 E: float = 1e8, nu: float = 0.3):
        counts = sorted(set(int(c) for c in border_counts))
        rng = np.random.default_rng(seed)
        seeds = rng.integers(0, 2 ** 31 - 1, size=len(counts))
        mu = E / (2 * (1 + nu)); lam = E * nu / ((1 + nu) * (1 - 2 * nu))
        jobs = [(int(s), (0.0, 0.0), 1.0, nb, interior_factor * nb, 1.0, 1.0, (mu, lam, E)) for s, nb in zip(seeds, counts)]
        bodies = make_discs_parallel(jobs, workers)
        self.E, self.nu = E, nu
        self.discs = dict(zip(counts, bodies))
        self.terms = {nb: _dt_terms(b, mu, lam) for nb, b in self.discs.items()}

    def grain(self, n_border: int, centre, radius: float, rho: float, mass_factor: float, material: int = 0) -> Body:
        t = self.discs[n_border]
        c = np.asarray(centre, dtype=np.float64)
        r = float(radius)
        s2 = r * r * rho * mass_factor
        gp = (t.gp[0], t.gp[1], t.gp[2], t.gp[3] / r, t.gp[4] / r)
        sup = (t.sup[0], t.sup[1], t.sup[2], t.sup[3] / r, t.sup[4] / r)
        borders = [dict(b, nodes=list(b["nodes"])) for b in t.borders]
        return Body(kind="deformable", material=material, nodes=c + r * t.nodes, borders=borders, cells=t.cells,
                    nodal_distance=r * t.nodal_distance, detection=r * t.detection, contact=r * t.contact,
                    domain=r * t.domain, mass=t.mass * s2, sup=sup, gp_xy=c + r * t.gp_xy, gp_w=t.gp_w,
                    gp_J=t.gp_J * (r * r), gp=gp, n_regions=t.n_regions)

    def critical_dt(self, n_border: int, radius: float, rho: float, mass_factor: float, kn: float) -> float:
        lam_el, lam_c = self.terms[n_border]
        m = rho * mass_factor
        return 2.0 / math.sqrt(max(lam_el / (radius * radius * m), kn * lam_c / (radius * m)))


def batch_sample_params(seed: int, grains=(50, 1000), border=(32, 96), sigma=(50e3, 400e3), mu_fric=(0.1, 0.5),
                        rmin: float = 0.5e-3, rmax: float = 1.5e-3):
    """Per-sample draws of the batched workload: grain count log-uniform, border nodes per grain
    uniform integers, confining pressure and friction uniform, radii uniform."""
    rng = np.random.default_rng(seed)
    n = int(round(math.exp(rng.uniform(math.log(grains[0]), math.log(grains[1])))))
    return dict(n_grains=n, radii=rng.uniform(rmin, rmax, size=n),
                n_border=rng.integers(border[0], border[1] + 1, size=n),
                sigma=float(rng.uniform(*sigma)), mu_fric=float(rng.uniform(*mu_fric)),
                rng_state=int(rng.integers(0, 2 ** 31 - 1)))


def batch_sample_scene(seed: int, templates: DiscTemplates, aspect: float = 100.0 / 60.0, fill: float = 0.45,
                       gap: float = 0.02e-3, v_plate: float = 0.05, mass_factor: float = 100.0,
                       nsteps: int = 20000, prox_every: int = 10, **draws) -> Scene:
    """One sample of the batched workload: the biaxial set-up (plates driven at v_plate, walls
    under the sample's confining pressure, mass scaling, proximity every prox_every steps) around
    grains built from `templates`."""
    p = batch_sample_params(seed, **draws)
    rng = np.random.default_rng(p["rng_state"])
    radii = p["radii"]
    area = float(np.sum(np.pi * radii ** 2))
    W = math.sqrt(area / fill * aspect)
    H = W / aspect
    centres, placed = _rsa_pack(rng, radii, W, H, gap)
    tries = 0
    while not placed.all() and tries < 5:
        W *= 1.03; H *= 1.03; tries += 1
        centres, placed = _rsa_pack(rng, radii, W, H, gap)
    if not placed.all():
        raise RuntimeError("packing failed")
    E, rho = templates.E, 2500.0
    rho_steel = 7800.0 * mass_factor
    mats = [("Grain", 0, [rho, 0.0, 0.0, E, templates.nu, 1000.0]), ("Steel", 0, [rho_steel, 0.0, 0.0, 2e11, 0.3, 500.0])]
    kn = 1e10
    laws = [("Grain", "Grain", 2, 0, [kn, 1e9, p["mu_fric"], 0.0, 0.0]),
            ("Grain", "Steel", 2, 0, [kn, 1e9, p["mu_fric"], 0.0, 0.0]),
            ("Steel", "Steel", 0, 0, [0.0])]
    bodies = [templates.grain(int(nb), c, r, rho, mass_factor) for nb, c, r in zip(p["n_border"], centres, radii)]
    for b, r in zip(bodies, radii):
        b.detection = b.contact = max(b.contact, contact_distance(p["sigma"], float(r), kn))
    h_min = float(np.min(2.0 * math.pi * radii / p["n_border"]))
    bodies += _biaxial_frame(W, H, h_min, rho_steel, v_plate, p["sigma"], contact_distance(p["sigma"], float(radii.max()), kn))
    dtc = min(templates.critical_dt(int(nb), float(r), rho, mass_factor, kn) for nb, r in zip(p["n_border"], radii))
    dt = float("%.4g" % (0.5 * dtc))
    return Scene(name=f"batch{seed}", bodies=bodies, materials=mats, laws=laws, dt=dt, nsteps=nsteps,
                 contact_update_period=prox_every * dt,
                 meta=dict(config="batch", seed=seed, dt_crit=dtc, box=(W, H), n_discs=p["n_grains"],
                           sigma=p["sigma"], mu_fric=p["mu_fric"], v_plate=v_plate, mass_factor=mass_factor))


# --------------------------------------------------------------------------------------------
# Moving flattened samples between processes without copying them through a pipe
# --------------------------------------------------------------------------------------------
# A batched-workload sample flattens to 250-700 MB of arrays (the Gauss-point shape-function
# columns dominate).  Returned from a spawned worker, it is pickled through a pipe and unpickled by
# the parent, one sample after another: for hundreds of samples that transfer, not the
# generation, bounds the admission path.  A worker instead copies each array into a named
# shared-memory block and returns only the names; the parent maps the blocks (no copy), creates
# its solver from them and releases them.  Where shared memory is unavailable or full, the arrays
# travel the ordinary way.

def share_flat(flat: Dict[str, np.ndarray]) -> dict:
    """Worker side: the arrays of `flat` in shared-memory blocks.  Returns a small picklable
    description for SharedFlat; the blocks live until SharedFlat.release() unlinks them."""
    from multiprocessing import shared_memory
    need = sum(v.nbytes for v in flat.values() if isinstance(v, np.ndarray) and v.nbytes >= 4096)
    try:
        st = os.statvfs("/dev/shm")
        free = st.f_bavail * st.f_frsize
    except OSError:
        free = 0
    # tmpfs pages are allocated on write, and a write into a full tmpfs kills the process (SIGBUS)
    # instead of raising: keep a wide margin for the other samples in flight
    if free < 4 * need:
        return {"__plain__": flat}
    blocks, desc = [], {}
    try:
        for k, v in flat.items():
            if isinstance(v, np.ndarray) and v.nbytes >= 4096:
                shm = shared_memory.SharedMemory(create=True, size=v.nbytes)
                blocks.append(shm)
                np.ndarray(v.shape, dtype=v.dtype, buffer=shm.buf)[...] = v
                desc[k] = ("shm", shm.name, v.dtype.str, v.shape)
            else:
                desc[k] = ("value", v)
    except OSError:
        for shm in blocks:
            shm.close()
            shm.unlink()
        return {"__plain__": flat}
    for shm in blocks:
        shm.close()
    return desc


class SharedFlat:
    """Parent side: `flat` maps the blocks described by share_flat() (or holds the plain arrays
    of the fallback).  release() drops the mapping and frees the blocks; the arrays must not be
    used afterwards."""

    def __init__(self, desc: dict):
        from multiprocessing import shared_memory
        self._blocks = []
        if "__plain__" in desc:
            self.flat = desc["__plain__"]
            return
        self.flat = {}
        for k, entry in desc.items():
            if entry[0] == "shm":
                _, name, dtype, shape = entry
                shm = shared_memory.SharedMemory(name=name)
                self._blocks.append(shm)
                self.flat[k] = np.ndarray(shape, dtype=np.dtype(dtype), buffer=shm.buf)
            else:
                self.flat[k] = entry[1]

    @property
    def nbytes(self) -> int:
        return sum(np.asarray(v).nbytes for k, v in self.flat.items() if k != "material_names")

    def release(self) -> None:
        self.flat = None
        for shm in self._blocks:
            try:
                shm.close()
            except BufferError:          # arrays still referenced elsewhere: the block is freed
                pass                     # when they go, its name is removed now
            try:
                shm.unlink()
            except FileNotFoundError:
                pass
        self._blocks = []


_templates_of_worker: Optional["DiscTemplates"] = None


def _init_template_worker(counts):
    global _templates_of_worker
    _templates_of_worker = DiscTemplates(counts, workers=1)


def _shared_sample(seed: int):
    sc = batch_sample_scene(seed, _templates_of_worker)
    return seed, share_flat(flatten(sc)), sc.meta, sc.dt


def build_batch_samples(seeds, create, workers: int, create_threads: int = 4, keep=(), counts=None):
    """Generates the batched workload's samples `seeds` in a spawn pool (each worker holds the disc
    templates) and calls create(flat) for each in a thread pool as soon as it arrives, with at most
    2 x workers samples generated ahead and 2 x create_threads creations in flight, so that shared
    memory holds a bounded number of samples.  Returns (created, kept, meta): created[i] =
    create(flat of seeds[i]); kept[i] the SharedFlat of the indices in `keep` (release them when
    done; the others are released after their creation); meta[i] = (scene meta, dt)."""
    import multiprocessing as mp
    from concurrent.futures import FIRST_COMPLETED, ProcessPoolExecutor, ThreadPoolExecutor, wait
    counts = list(range(32, 97)) if counts is None else list(counts)
    keep = set(keep)
    n = len(seeds)
    created, kept, meta = [None] * n, {}, [None] * n
    ctx = mp.get_context("spawn")
    with ProcessPoolExecutor(max_workers=workers, mp_context=ctx, initializer=_init_template_worker,
                             initargs=(counts,)) as ex, ThreadPoolExecutor(max_workers=create_threads) as cx:
        gen, mk = {}, {}
        nxt = 0
        finished = False
        try:
            while nxt < n or gen or mk:
                while nxt < n and len(gen) < 2 * workers and len(mk) < 2 * create_threads:
                    gen[ex.submit(_shared_sample, seeds[nxt])] = nxt
                    nxt += 1
                done, _ = wait(list(gen) + list(mk), return_when=FIRST_COMPLETED)
                for f in done:
                    if f in gen:
                        i = gen.pop(f)
                        _, desc, m, dt = f.result()
                        sf = SharedFlat(desc)
                        meta[i] = (m, dt)
                        mk[cx.submit(create, sf.flat)] = (i, sf)
                    else:
                        i, sf = mk.pop(f)
                        try:
                            created[i] = f.result()
                        except BaseException:
                            sf.release()
                            raise
                        if i in keep:
                            kept[i] = sf
                        else:
                            sf.release()
            finished = True
        finally:
            if not finished:                 # the caller gets nothing: free what it would have kept
                for sf in kept.values():
                    sf.release()
            for f, (i, sf) in list(mk.items()):
                if i not in kept:
                    f.cancel()
                    try:
                        f.result()
                    except Exception:
                        pass
                    sf.release()
            for f in list(gen):
                f.cancel()
            for f in list(gen):              # samples already being built: wait, then free them
                try:
                    SharedFlat(f.result()[1]).release()
                except BaseException:
                    pass
    return created, kept, meta
