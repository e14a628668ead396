"""Seeded synthetic tube geometries in the reference's input conventions.

The reference builds its inputs with an SWC/OBJ mesher and an unstructured
spline extractor (preprocessing/mesh, preprocessing/spline); this module is
the project's own generator for the benchmark tubes.  It produces the same
artefacts the solver consumes:

* a ``FlatMesh`` / ``.ntiga`` database: one element per hex cell, one basis
  function per control-mesh vertex, sparse Bezier extraction rows and 64
  Bezier points per element (Bezier points = extraction^T x vertices);
* ``controlmesh.vtk`` with 8-node hexes in element order and point labels
  (-1 interior, 0 wall, 1 inlet, 2.. outlets), as read by ReadLabeledHexMesh
  (solvers/cpu/include/BoundarySupport.hpp:25-73);
* ``initial_velocityfield.txt`` with a parabolic axial profile of peak 1, the
  reference mesher's inlet profile convention (preprocessing/mesh/src/MeshGenerator.cpp:176);
* ``simulation_config.json`` (schema v4 subset).

Cross-section: an O-grid of five patches -- an ``core x core`` square core
and four ring patches of ``core`` tangential x ``ring`` radial cells -- so a
4x4 core with one ring layer has 32 cells and 41 vertices per plane, and an
8x8 core with two ring layers has 128 cells and 145 vertices per plane.
Each patch carries uniform cubic B-splines whose phantom end points are
eliminated by linear extrapolation (v_-1 = 2 v_0 - v_1), which keeps C2
inside a patch, interpolates patch boundaries and gives C0 coupling across
patch interfaces.  Interior elements have 64 basis functions; elements next
to a patch boundary have 48 or fewer.
"""
from __future__ import annotations

import json
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .ntiga import FlatMesh, write as write_ntiga

_UNIFORM = np.array([[1.0, 0.0, 0.0, 0.0],
                     [4.0, 4.0, 2.0, 1.0],
                     [1.0, 2.0, 4.0, 4.0],
                     [0.0, 0.0, 0.0, 1.0]]) / 6.0


def natural_extraction_1d(ncells: int, cell: int):
    """(vertex indices, Bernstein coefficient rows) of one cell of a natural-end cubic spline."""
    acc: dict[int, np.ndarray] = {}
    for k, j in enumerate(range(cell - 1, cell + 3)):
        row = _UNIFORM[k]
        if j < 0:
            targets = ((0, 2.0), (1, -1.0))
        elif j > ncells:
            targets = ((ncells, 2.0), (ncells - 1, -1.0))
        else:
            targets = ((j, 1.0),)
        for v, s in targets:
            acc.setdefault(v, np.zeros(4))
            acc[v] = acc[v] + s * row
    verts = sorted(v for v in acc if np.any(np.abs(acc[v]) > 1e-15))
    return np.array(verts, np.int64), np.array([acc[v] for v in verts])


@dataclass
class Tube:
    mesh: FlatMesh
    points: np.ndarray        # [n, 3] control-mesh vertices (= spline control points)
    labels: np.ndarray        # [n] point labels
    cells: np.ndarray         # [E, 8] VTK hex connectivity
    profile: np.ndarray       # [n, 3] peak-1 inlet profile
    radius: float
    length: float
    planes: int
    per_plane: int


def ogrid_cross_section(radius: float, core: int, ring: int, core_half: float = 0.5, bulge: float = 0.2):
    """2D O-grid: vertex positions, patch vertex maps (patch -> [nu+1, nv+1] global ids), rim flags."""
    nc, nr = core, ring
    n_core = (nc + 1) ** 2
    n2d = n_core + 4 * nc * nr
    pos = np.zeros((n2d, 2))
    a = core_half * radius
    for j in range(nc + 1):
        for i in range(nc + 1):
            s, t = -1.0 + 2.0 * i / nc, -1.0 + 2.0 * j / nc
            pos[i + (nc + 1) * j] = (a * s * (1.0 + bulge * (1.0 - t * t)), a * t * (1.0 + bulge * (1.0 - s * s)))

    def core_boundary(k, m):
        if k == 0:
            i, j = nc, m
        elif k == 1:
            i, j = nc - m, nc
        elif k == 2:
            i, j = 0, nc - m
        else:
            i, j = m, 0
        return i + (nc + 1) * j

    patches = [np.array([[i + (nc + 1) * j for j in range(nc + 1)] for i in range(nc + 1)], np.int64)]
    rim = np.zeros(n2d, bool)
    for k in range(4):
        grid = np.zeros((nr + 1, nc + 1), np.int64)   # [radial u][tangential v]
        for m in range(nc + 1):
            inner = core_boundary(k, m)
            theta = -0.25 * math.pi + 0.5 * math.pi * k + 0.5 * math.pi * m / nc
            outer = radius * np.array([math.cos(theta), math.sin(theta)])
            grid[0, m] = inner
            for r in range(1, nr + 1):
                vid = n_core + (r - 1) * 4 * nc + (k * nc + m) % (4 * nc)
                grid[r, m] = vid
                rho = r / nr
                pos[vid] = (1.0 - rho) * pos[inner] + rho * outer
                if r == nr:
                    rim[vid] = True
        patches.append(grid)
    return pos, patches, rim


@dataclass
class SweptBlock:
    """A cross-section of 2D patches swept through ``planes`` vertex planes.

    ``patches[p]`` is a [nu+1, nv+1] grid of plane-local vertex ids (u radial for ring patches, rim at
    u = nu); ``ids[k, v]`` is the global vertex id of plane-local vertex v in plane k, so blocks that
    share a plane share its vertices (a C0 interface). ``wall[p]`` marks ring patches whose rim faces
    are no-slip walls (face label 0); ``bottom`` / ``top`` label the faces of the first / last layer."""
    patches: list
    ids: np.ndarray
    wall: list
    bottom: int | None = None
    top: int | None = None


def swept_mesh(points, blocks):
    """FlatMesh + VTK hex cells of swept blocks: one element per cell, natural-end cubic B-splines per
    patch and per block axis.  Elements are enumerated block by block, then layer, patch, v, u."""
    ext_cache: dict = {}

    def ext(nc_, c_):
        key = (nc_, c_)
        if key not in ext_cache:
            ext_cache[key] = natural_extraction_1d(nc_, c_)
        return ext_cache[key]

    conn_list, rows_list, labels_list, cells, groups = [], [], [], [], {}
    for blk in blocks:
        layers = blk.ids.shape[0] - 1
        for layer in range(layers):
            wv, wc = ext(layers, layer)
            plane_ids = blk.ids[wv]                                   # [nw_l, n_local]
            for p, grid in enumerate(blk.patches):
                nu, nv = grid.shape[0] - 1, grid.shape[1] - 1
                for jv in range(nv):
                    vv, vc = ext(nv, jv)
                    for iu in range(nu):
                        uv, uc = ext(nu, iu)
                        # local basis ordering: w outer, v, u inner
                        ids2 = grid[np.ix_(uv, vv)]                   # [nu_l, nv_l]
                        conn = plane_ids[:, ids2.T].reshape(-1)
                        key = (layers, layer, nu, iu, nv, jv)
                        if key not in groups:
                            # row (w,v,u) x Bernstein index c*16 + b*4 + a (u fastest)
                            rows = np.einsum("wc,vb,ua->wvucba", wc, vc, uc)
                            groups[key] = rows.reshape(len(wv) * len(vv) * len(uv), 64)
                        conn_list.append(conn.astype(np.int32))
                        rows_list.append(key)
                        lab = [-1] * 6
                        if layer == 0 and blk.bottom is not None:
                            lab[0] = blk.bottom
                        if layer == layers - 1 and blk.top is not None:
                            lab[5] = blk.top
                        if p > 0 and blk.wall[p] and iu == nu - 1:
                            lab[2] = 0
                        labels_list.append(lab)
                        c = [grid[iu, jv], grid[iu + 1, jv], grid[iu + 1, jv + 1], grid[iu, jv + 1]]
                        cells.append([blk.ids[layer, v] for v in c] + [blk.ids[layer + 1, v] for v in c])
    E = len(conn_list)
    nen = np.array([len(c) for c in conn_list], np.int64)
    element_offsets = np.zeros(E + 1, np.int64)
    element_offsets[1:] = np.cumsum(nen)
    connectivity = np.concatenate(conn_list)
    # Sparse extraction rows and Bezier points, grouped by extraction type.
    sparse = {}
    for key, rows in groups.items():
        cols = [np.nonzero(np.abs(r) > 0.0)[0].astype(np.uint8) for r in rows]
        sparse[key] = (np.concatenate(cols), np.concatenate([rows[i][cols[i]] for i in range(len(rows))]),
                       np.array([len(c) for c in cols], np.int64))
    xc = np.concatenate([sparse[k][0] for k in rows_list])
    xv = np.concatenate([sparse[k][1] for k in rows_list])
    xo = np.zeros(int(element_offsets[-1]) + 1, np.int64)
    xo[1:] = np.cumsum(np.concatenate([sparse[k][2] for k in rows_list]))
    bezier = np.zeros((E, 64, 3))
    by_key: dict = {}
    for e, key in enumerate(rows_list):
        by_key.setdefault(key, []).append(e)
    for key, es in by_key.items():
        es = np.array(es)
        Cm = groups[key]                                          # [nen, 64]
        conn = np.stack([conn_list[e] for e in es])               # [g, nen]
        bezier[es] = np.einsum("ap,gad->gpd", Cm, points[conn])
    mesh = FlatMesh(
        nodes=len(points),
        element_offsets=element_offsets.astype(np.int32),
        connectivity=connectivity.astype(np.int32),
        extraction_offsets=xo.astype(np.int32),
        extraction_columns=xc.astype(np.uint8),
        extraction_values=xv.astype(np.float64),
        bezier_points=bezier.ravel(),
        boundary_labels=np.array(labels_list, np.int32).ravel(),
    ).contiguous()
    return mesh, np.array(cells, np.int64)


def straight_tube(radius: float, length: float, core: int, ring: int, layers: int,
                  core_half: float = 0.5, bulge: float = 0.2) -> Tube:
    """Straight tube along +z: inlet face label 1 at z=0, outlet label 2 at z=length, wall label 0."""
    pos2, patches, rim = ogrid_cross_section(radius, core, ring, core_half, bulge)
    n2d = len(pos2)
    planes = layers + 1
    n = n2d * planes
    z = np.linspace(0.0, length, planes)
    points = np.zeros((n, 3))
    for k in range(planes):
        points[k * n2d:(k + 1) * n2d, :2] = pos2
        points[k * n2d:(k + 1) * n2d, 2] = z[k]
    labels = np.full(n, -1, np.int32)
    for k in range(planes):
        sl = slice(k * n2d, (k + 1) * n2d)
        lab = labels[sl]
        if k == 0:
            lab[:] = 1
        elif k == planes - 1:
            lab[:] = 2
        lab[rim] = 0
    r2 = (points[:, 0] ** 2 + points[:, 1] ** 2) / radius ** 2
    profile = np.zeros((n, 3))
    profile[:, 2] = np.maximum(0.0, 1.0 - r2)

    ids = np.arange(n, dtype=np.int64).reshape(planes, n2d)
    block = SweptBlock(patches=patches, ids=ids, wall=[False] + [True] * 4, bottom=1, top=2)
    mesh, cells = swept_mesh(points, [block])
    return Tube(mesh=mesh, points=points, labels=labels, cells=cells, profile=profile,
                radius=radius, length=length, planes=planes, per_plane=n2d)



def helical_tube(radius: float, length: float, curvature_radius: float, core: int, ring: int, layers: int,
                 handed: float = 1.0, core_half: float = 0.5, bulge: float = 0.2) -> Tube:
    """Tube of the straight tube's O-grid swept along a helix whose curvature radius is
    ``curvature_radius``: helix radius a and pitch parameter c equal (a 45 degree helix), so the
    curvature a / (a^2 + c^2) is 1 / curvature_radius for a = c = curvature_radius / 2.  Each vertex
    plane sits at arc length s_k = k length / layers and spans the Frenet normal and binormal there;
    the centreline starts at the origin with tangent (0, c, c) / |.| rotated onto +z, so the inlet
    face is the plane z = 0 as for the straight tube.  Labels and the peak-1 inlet profile (along the
    inlet tangent) follow ``straight_tube``.  ``handed`` = +1 or -1 picks the helix's sense."""
    if not curvature_radius > radius:
        raise ValueError("the curvature radius must exceed the tube radius")
    pos2, patches, rim = ogrid_cross_section(radius, core, ring, core_half, bulge)
    n2d = len(pos2)
    planes = layers + 1
    a = c = 0.5 * curvature_radius
    speed = math.hypot(a, c)
    s = np.linspace(0.0, length, planes)
    t = s / speed
    # helix along +y (local frame), starting at (a, 0, 0): P(t) = (a cos t, c t, handed a sin t)
    P = np.stack([a * np.cos(t), c * t, handed * a * np.sin(t)], axis=1)
    T = np.stack([-a * np.sin(t), np.full_like(t, c), handed * a * np.cos(t)], axis=1) / speed
    N = np.stack([-np.cos(t), np.zeros_like(t), -handed * np.sin(t)], axis=1)
    B = np.cross(T, N)
    # rigid motion taking P(0) to the origin and T(0) to +z, N(0) to +x
    frame0 = np.stack([N[0], B[0], T[0]])                 # rows: images of x, y, z
    P = (P - P[0]) @ frame0.T
    T, N, B = T @ frame0.T, N @ frame0.T, B @ frame0.T
    points = np.zeros((planes * n2d, 3))
    for k in range(planes):
        points[k * n2d:(k + 1) * n2d] = P[k] + pos2[:, :1] * N[k] + pos2[:, 1:2] * B[k]
    n = len(points)
    labels = np.full(n, -1, np.int32)
    for k in range(planes):
        lab = labels[k * n2d:(k + 1) * n2d]
        if k == 0:
            lab[:] = 1
        elif k == planes - 1:
            lab[:] = 2
        lab[rim] = 0
    r2 = (pos2[:, 0] ** 2 + pos2[:, 1] ** 2) / radius ** 2
    profile = np.zeros((n, 3))
    profile[:n2d] = np.maximum(0.0, 1.0 - r2)[:, None] * T[0]
    ids = np.arange(n, dtype=np.int64).reshape(planes, n2d)
    block = SweptBlock(patches=patches, ids=ids, wall=[False] + [True] * 4, bottom=1, top=2)
    mesh, cells = swept_mesh(points, [block])
    return Tube(mesh=mesh, points=points, labels=labels, cells=cells, profile=profile,
                radius=radius, length=length, planes=planes, per_plane=n2d)


def quad_ogrid(sides, center, ax: int, ay: int, ring: int, core_scale: float = 0.5, bulge: float = 0.2):
    """2D O-grid of a region bounded by four curves: an ``ax x ay`` core and four ring patches.

    ``sides[k](t)`` (t in [0, 1], arrays of t accepted) traces boundary side k counter-clockwise:
    k = 0 and 2 carry ``ay`` cells, k = 1 and 3 carry ``ax``; side k ends where side k+1 starts.
    The core corners are the boundary corners pulled toward ``center`` by ``core_scale``; each core
    side is the chord between its corners bent by ``bulge`` toward the pulled boundary side, and the
    core interior is their transfinite (Coons) interpolation.  Ring vertex r of a radial line lies
    at r / ring between the core side and the boundary.
    Returns (positions [n2d, 2], patches, rim) with ``rim[k]`` the plane-local ids of side k's
    boundary vertices in side order."""
    center = np.asarray(center, np.float64)
    counts = [ay, ax, ay, ax]
    corners = [np.asarray(sides[k](0.0), np.float64) for k in range(4)]

    def core_side(k, t):
        t = np.atleast_1d(np.asarray(t, np.float64))
        c0 = center + core_scale * (corners[k] - center)
        c1 = center + core_scale * (corners[(k + 1) % 4] - center)
        chord = (1.0 - t)[:, None] * c0 + t[:, None] * c1
        pulled = center + core_scale * (np.asarray(sides[k](t), np.float64).reshape(-1, 2) - center)
        return (1.0 - bulge) * chord + bulge * pulled

    n_core = (ax + 1) * (ay + 1)
    per_ring = 2 * (ax + ay)
    pos = np.zeros((n_core + ring * per_ring, 2))
    # core: Coons patch; i along sides 3 (bottom, i increasing) and 1 (top, i decreasing), j along 0 / 2
    s_ = np.linspace(0.0, 1.0, ax + 1)
    t_ = np.linspace(0.0, 1.0, ay + 1)
    bottom = core_side(3, s_)                 # (i, 0)
    right = core_side(0, t_)                  # (ax, j)
    top = core_side(1, 1.0 - s_)              # (i, ay): side 1 runs from i = ax to i = 0
    left = core_side(2, 1.0 - t_)             # (0, j): side 2 runs from j = ay to j = 0
    P00, P10, P11, P01 = bottom[0], bottom[-1], top[-1], top[0]
    for j in range(ay + 1):
        for i in range(ax + 1):
            u, v = s_[i], t_[j]
            pos[i + (ax + 1) * j] = ((1 - v) * bottom[i] + v * top[i] + (1 - u) * left[j] + u * right[j]
                                     - ((1 - u) * (1 - v) * P00 + u * (1 - v) * P10 + u * v * P11
                                        + (1 - u) * v * P01))

    def core_boundary(k, m):
        if k == 0:
            i, j = ax, m
        elif k == 1:
            i, j = ax - m, ay
        elif k == 2:
            i, j = 0, ay - m
        else:
            i, j = m, 0
        return i + (ax + 1) * j

    patches = [np.array([[i + (ax + 1) * j for j in range(ay + 1)] for i in range(ax + 1)], np.int64)]
    offsets = [0, ay, ay + ax, 2 * ay + ax]
    rim = []
    for k in range(4):
        nk = counts[k]
        grid = np.zeros((ring + 1, nk + 1), np.int64)       # [radial u][tangential v]
        outer = np.asarray(sides[k](np.linspace(0.0, 1.0, nk + 1)), np.float64).reshape(-1, 2)
        for m in range(nk + 1):
            inner = core_boundary(k, m)
            grid[0, m] = inner
            for r in range(1, ring + 1):
                vid = n_core + (r - 1) * per_ring + (offsets[k] + m) % per_ring
                grid[r, m] = vid
                rho = r / ring
                pos[vid] = (1.0 - rho) * pos[inner] + rho * outer[m]
        patches.append(grid)
        rim.append(grid[ring].copy())
    return pos, patches, rim


def _arc(cx, cy, radius, a0, a1):
    return lambda t: np.stack([cx + radius * np.cos(a0 + (a1 - a0) * np.asarray(t, np.float64)),
                               cy + radius * np.sin(a0 + (a1 - a0) * np.asarray(t, np.float64))], axis=-1)


def _segment(p0, p1):
    p0, p1 = np.asarray(p0, np.float64), np.asarray(p1, np.float64)
    return lambda t: p0 + np.asarray(t, np.float64)[..., None] * (p1 - p0)


def half_disc_section(radius: float, ax: int, ay: int, ring: int):
    """O-grid of the half disc {s >= 0, s^2 + y^2 <= R^2} in local (s, y): side 0 the arc from -45 to
    45 degrees, sides 1 / 3 the arcs up to +-90 degrees, side 2 the straight septum s = 0 (y from R to
    -R).  With ax = ay / 2 every arc cell spans the same angle."""
    q = 0.25 * math.pi
    sides = [_arc(0.0, 0.0, radius, -q, q), _arc(0.0, 0.0, radius, q, 2 * q),
             _segment((0.0, radius), (0.0, -radius)), _arc(0.0, 0.0, radius, -2 * q, -q)]
    return quad_ogrid(sides, (4.0 * radius / (3.0 * math.pi), 0.0), ax, ay, ring)


def disc_section_like_half(radius: float, ax: int, ay: int, ring: int):
    """O-grid of the disc of radius r centred at (r, 0) (touching s = 0 at the origin) with the
    topology of ``half_disc_section``: the boundary split in proportion to the cell counts."""
    per = 2.0 * math.pi / (2 * (ax + ay))
    a0 = -0.5 * ay * per
    a1 = a0 + ay * per
    a2 = a1 + ax * per
    a3 = a2 + ay * per
    sides = [_arc(radius, 0.0, radius, a0, a1), _arc(radius, 0.0, radius, a1, a2),
             _arc(radius, 0.0, radius, a2, a3), _arc(radius, 0.0, radius, a3, a0 + 2.0 * math.pi)]
    return quad_ogrid(sides, (radius, 0.0), ax, ay, ring)


def _smoothstep(x):
    x = np.clip(x, 0.0, 1.0)
    return x * x * (3.0 - 2.0 * x)


@dataclass
class Bifurcation:
    """Y-bifurcation: parent along +z from z = 0 (inlet, label 1), two daughters (outlets labels 2 and
    3) leaving the junction plane z = parent_length symmetrically about x = 0."""
    mesh: FlatMesh
    points: np.ndarray
    labels: np.ndarray
    cells: np.ndarray
    profile: np.ndarray
    radius: float             # parent radius
    daughter_radius: float
    parent_layers: int
    daughter_layers: int
    outlet_labels: tuple = (2, 3)


def y_bifurcation(parent_radius: float = 2.0e-3, parent_length: float = 20e-3,
                  daughter_radius: float = 1.59e-3, daughter_length: float = 16e-3,
                  half_angle_deg: float = 35.0, ax: int = 6, ay: int = 12, ring: int = 3,
                  parent_layers: int = 308, daughter_layers: int = 247,
                  bend_length: float | None = None, morph_length: float | None = None) -> Bifurcation:
    """Swept O-grid Y-bifurcation (all hexahedra, one element per cell, C2 inside each block, C0
    across block and patch interfaces).

    Each half of the parent is a half-disc O-grid (``half_disc_section``); the two halves share the
    septum vertices on the diameter x = 0, so the parent cross-section has 2 (ax ay + 2 (ax + ay)
    ring) cells.  At the junction plane each daughter starts from its half of the parent section;
    along the daughter (arc length t) the section blends into a disc of the daughter radius
    (``disc_section_like_half``) over ``morph_length`` and turns about the septum line by the
    half-angle over ``bend_length`` (smoothstep profiles).  The left daughter's control points all
    have x <= 0 and the right daughter is its mirror image, so the daughters never overlap (convex
    hull of the spline); the septum line in the junction plane is the carina edge, a wall.
    The defaults give 360 (parent_layers + daughter_layers) = 199,800 elements."""
    R, r = parent_radius, daughter_radius
    bend = bend_length if bend_length is not None else 0.5 * daughter_length
    morph = morph_length if morph_length is not None else 0.375 * daughter_length
    hpos, patches, rim = half_disc_section(R, ax, ay, ring)
    dpos, dpatches, drim = disc_section_like_half(r, ax, ay, ring)
    for a, b in zip(patches, dpatches):
        assert np.array_equal(a, b)
    nd = len(hpos)
    septum = rim[2]                                     # local ids, y from +R to -R (local)
    # Parent plane ids: left half = local ids; right half = new ids except its septum, which is the
    # left half's septum vertex at the same global y (the left half is rotated by 180 degrees).
    right_map = np.full(nd, -1, np.int64)
    right_map[septum] = septum[::-1]
    others = np.setdiff1d(np.arange(nd), septum)
    right_map[others] = nd + np.arange(len(others))
    n_parent = nd + len(others)
    # parent plane positions
    ppos = np.zeros((n_parent, 2))
    ppos[:nd] = -hpos                                   # left half: (s, y) -> (-s, -y)
    ppos[right_map[others]] = hpos[others]              # right half: (s, y) -> (s, y)
    planes_p = parent_layers + 1
    base_left = planes_p * n_parent
    base_right = base_left + daughter_layers * nd
    n = base_right + daughter_layers * nd
    points = np.zeros((n, 3))
    zp = np.linspace(0.0, parent_length, planes_p)
    for k in range(planes_p):
        points[k * n_parent:(k + 1) * n_parent, :2] = ppos
        points[k * n_parent:(k + 1) * n_parent, 2] = zp[k]
    # left daughter: pivot path P(t) on the septum line, frame e_s = (-cos th, 0, -sin th), e_y = -y
    theta_max = math.radians(half_angle_deg)
    t = np.linspace(0.0, daughter_length, daughter_layers + 1)
    fine = np.linspace(0.0, daughter_length, 64 * daughter_layers + 1)
    th_f = theta_max * _smoothstep(fine / bend)
    dx = np.concatenate([[0.0], np.cumsum(0.5 * (np.sin(th_f[1:]) + np.sin(th_f[:-1])) * np.diff(fine))])
    dz = np.concatenate([[0.0], np.cumsum(0.5 * (np.cos(th_f[1:]) + np.cos(th_f[:-1])) * np.diff(fine))])
    px = -np.interp(t, fine, dx)
    pz = parent_length + np.interp(t, fine, dz)
    th = theta_max * _smoothstep(t / bend)
    w = _smoothstep(t / morph)
    left_ids = np.zeros((daughter_layers + 1, nd), np.int64)
    right_ids = np.zeros((daughter_layers + 1, nd), np.int64)
    left_ids[0] = (planes_p - 1) * n_parent + np.arange(nd)
    right_ids[0] = (planes_p - 1) * n_parent + right_map
    for j in range(1, daughter_layers + 1):
        loc = (1.0 - w[j]) * hpos + w[j] * dpos          # [nd, 2] local (s, y)
        sl, yl = loc[:, 0], loc[:, 1]
        left = np.stack([px[j] - sl * math.cos(th[j]), -yl, pz[j] - sl * math.sin(th[j])], axis=1)
        # right daughter = mirror x of the left daughter evaluated at local (s, -y)
        right = np.stack([-(px[j] - sl * math.cos(th[j])), yl, pz[j] - sl * math.sin(th[j])], axis=1)
        left_ids[j] = base_left + (j - 1) * nd + np.arange(nd)
        right_ids[j] = base_right + (j - 1) * nd + np.arange(nd)
        points[left_ids[j]] = left
        points[right_ids[j]] = right
    parent_patches = [p.copy() for p in patches] + [right_map[p] for p in patches]
    arc_wall = [False, True, True, False, True]          # core, then ring sides 0..3 (2 = septum)
    blocks = [
        SweptBlock(patches=parent_patches, ids=np.arange(planes_p * n_parent).reshape(planes_p, n_parent),
                   wall=arc_wall + arc_wall, bottom=1, top=None),
        SweptBlock(patches=patches, ids=left_ids, wall=[False] + [True] * 4, bottom=None, top=2),
        SweptBlock(patches=patches, ids=right_ids, wall=[False] + [True] * 4, bottom=None, top=3),
    ]
    mesh, cells = swept_mesh(points, blocks)
    labels = np.full(n, -1, np.int32)
    labels[:n_parent] = 1                                        # inlet plane
    labels[left_ids[-1]] = 2
    labels[right_ids[-1]] = 3
    arc = np.unique(np.concatenate([rim[0], rim[1], rim[3]]))
    for k in range(planes_p):
        labels[k * n_parent + arc] = 0
        labels[k * n_parent + right_map[arc]] = 0
    all_rim = np.unique(np.concatenate(rim))
    labels[left_ids[:, all_rim].ravel()] = 0
    labels[right_ids[:, all_rim].ravel()] = 0
    profile = np.zeros((n, 3))
    r2 = (points[:n_parent, 0] ** 2 + points[:n_parent, 1] ** 2) / R ** 2
    profile[:n_parent, 2] = np.maximum(0.0, 1.0 - r2)
    return Bifurcation(mesh=mesh, points=points, labels=labels, cells=cells, profile=profile, radius=R,
                       daughter_radius=r, parent_layers=parent_layers, daughter_layers=daughter_layers)

# --- binary trees ---------------------------------------------------------------------------------
#
# A tree segment whose subtree ends in 2^m outlets has a cross-section of 2^m O-grid regions (each a
# ``quad_ogrid`` with an n x n core).  At its end the section is a disc split by a diameter (the
# septum) into two halves of 2^(m-1) regions each; each half is the start section of one daughter,
# which morphs it into its own disc of 2^(m-1) regions.  So no section changes topology along a
# segment, and every junction is conforming (the daughters share the parent's last vertex plane).
#
# Section layouts, in a segment's local frame (s away from the parent's septum, y along it):
#   half-disc layouts S_m(R), the half disc {s >= 0, s^2 + y^2 <= R^2} (a daughter's start):
#     S_0: one region (sides: arc -45..45 deg, arc 45..90, flat side, arc -90..-45);
#     S_1: two quarter discs split by the chord y = 0;
#     S_2: four regions around a hub H = (0.4 R, 0) with spokes to the flat side's midpoint, the arc's
#          midpoint and the arc points at +-acos(0.4) (the spokes to them are parallel to y);
#   disc layouts E_m(r) (a segment's end, centred on the disc's centre):
#     E_0: one region with corners at -45, 45, 135 and 225 deg;
#     E_m: S_{m-1}(r) rotated by +90 deg (the half y > 0, daughter 0) and by -90 deg (y < 0,
#          daughter 1); their flat sides meet on the septum y = 0.
# S_m and E_m list the same regions with the same side numbering and the same shared sides (checked
# when the layouts are built), so vertex positions morph linearly from one to the other.

_TREE_HUB = 0.4                     # S_2's hub on the s axis, in units of R


def _half_layout_sides(m: int, R: float):
    """Regions of S_m(R): per region its four side curves (counter-clockwise)."""
    q = 0.25 * math.pi
    o = (0.0, 0.0)
    if m == 0:
        return [[_arc(0.0, 0.0, R, -q, q), _arc(0.0, 0.0, R, q, 2 * q), _segment((0.0, R), (0.0, -R)),
                 _arc(0.0, 0.0, R, -2 * q, -q)]]
    if m == 1:
        return [[_arc(0.0, 0.0, R, q, 2 * q), _segment((0.0, R), o), _segment(o, (R, 0.0)), _arc(0.0, 0.0, R, 0.0, q)],
                [_arc(0.0, 0.0, R, -2 * q, -q), _arc(0.0, 0.0, R, -q, 0.0), _segment((R, 0.0), o),
                 _segment(o, (0.0, -R))]]
    if m == 2:
        phi = math.acos(_TREE_HUB)
        H, E = (_TREE_HUB * R, 0.0), (R, 0.0)
        N, S = (R * math.cos(phi), R * math.sin(phi)), (R * math.cos(phi), -R * math.sin(phi))
        return [[_segment((0.0, R), o), _segment(o, H), _segment(H, N), _arc(0.0, 0.0, R, phi, 2 * q)],
                [_arc(0.0, 0.0, R, 0.0, 0.5 * phi), _arc(0.0, 0.0, R, 0.5 * phi, phi), _segment(N, H), _segment(H, E)],
                [_arc(0.0, 0.0, R, -0.5 * phi, 0.0), _segment(E, H), _segment(H, S), _arc(0.0, 0.0, R, -phi, -0.5 * phi)],
                [_segment(o, (0.0, -R)), _arc(0.0, 0.0, R, -2 * q, -phi), _segment(S, H), _segment(H, o)]]
    raise ValueError("tree sections support at most 4 regions per half (depth <= 4)")


# shared sides (region, side) <-> (region, side) of S_m, and its flat-side sides from (0, R) to (0, -R)
_HALF_PAIRS = {0: [], 1: [((0, 2), (1, 2))],
               2: [((0, 2), (1, 2)), ((1, 3), (2, 1)), ((2, 2), (3, 2)), ((3, 3), (0, 1))]}
_HALF_FLAT = {0: [(0, 2)], 1: [(0, 1), (1, 3)], 2: [(0, 0), (3, 0)]}


def _disc_pairs(m: int):
    """Shared sides of E_m: each daughter half's own, plus the septum pairs (daughter 0's k-th flat side
    with daughter 1's flat side counted from the other end)."""
    if m == 0:
        return []
    k = 2 ** (m - 1)
    pairs = list(_HALF_PAIRS[m - 1]) + [((a + k, sa), (b + k, sb)) for (a, sa), (b, sb) in _HALF_PAIRS[m - 1]]
    flat = _HALF_FLAT[m - 1]
    for i, (a, sa) in enumerate(flat):
        b, sb = flat[len(flat) - 1 - i]
        pairs.append(((a, sa), (b + k, sb)))
    return pairs


def _region_centre(sides):
    """Area centroid of a region bounded by four side curves (polygon of 64 samples per side)."""
    t = np.linspace(0.0, 1.0, 65)[:-1]
    p = np.concatenate([np.asarray(s(t), np.float64).reshape(-1, 2) for s in sides])
    x, y = p[:, 0], p[:, 1]
    xn, yn = np.roll(x, -1), np.roll(y, -1)
    c = x * yn - xn * y
    a = 0.5 * c.sum()
    return np.array([((x + xn) * c).sum(), ((y + yn) * c).sum()]) / (6.0 * a)


def _layout_positions(sides_list, core: int, ring: int):
    out = []
    for sides in sides_list:
        pos, patches, rim = quad_ogrid(sides, _region_centre(sides), core, core, ring)
        out.append(pos)
    return out, patches, rim


def _rot90(pos, sign):
    """(s, y) -> (-y, s) for sign +1 (daughter 0's half), (y, -s) for sign -1 (daughter 1's)."""
    return np.stack([-sign * pos[:, 1], sign * pos[:, 0]], axis=1)


@dataclass
class TreeSection:
    """Plane layout of 2^m O-grid regions: region-local quad_ogrid vertex v of region i is plane-local
    vertex ``ids[i, v]``; ``start`` = S_m(1) and ``end`` = E_m(1) (centred) positions per plane-local
    vertex; ``patches[i]`` region i's patches in plane-local ids; ``wall[i]`` its patches' wall flags
    (core False, ring patch k True when side k is on the outer boundary); ``boundary`` the plane-local
    ids on the outer boundary."""
    m: int
    ids: np.ndarray
    start: np.ndarray
    end: np.ndarray
    patches: list
    wall: list
    boundary: np.ndarray


def tree_section(m: int, core: int, ring: int) -> TreeSection:
    """The layout of a segment with 2^m outlets below it (``start`` is None for m = 3, the root of a
    depth-4 tree, which starts at the inlet with its end layout)."""
    regions = 2 ** m
    if m == 0:
        disc, patches, rim = _layout_positions(
            [[_arc(0.0, 0.0, 1.0, a, a + 0.5 * math.pi) for a in
              (-0.25 * math.pi, 0.25 * math.pi, 0.75 * math.pi, 1.25 * math.pi)]], core, ring)
    else:
        sub, patches, rim = _layout_positions(_half_layout_sides(m - 1, 1.0), core, ring)
        disc = [_rot90(p, 1.0) for p in sub] + [_rot90(p, -1.0) for p in sub]
    half = _layout_positions(_half_layout_sides(m, 1.0), core, ring)[0] if m in _HALF_PAIRS else None
    pairs = _disc_pairs(m)
    if half is not None and sorted(map(sorted, _HALF_PAIRS[m])) != sorted(map(sorted, pairs)):
        raise AssertionError("half and disc layouts disagree on shared sides")
    nl = len(disc[0])
    parent = np.arange(regions * nl)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for (a, sa), (b, sb) in pairs:
        for u, v in zip(a * nl + rim[sa], b * nl + rim[sb][::-1]):
            fu, fv = find(int(u)), find(int(v))
            if fu != fv:
                parent[max(fu, fv)] = min(fu, fv)
    roots = np.array([find(x) for x in range(regions * nl)])
    _, ids = np.unique(roots, return_inverse=True)
    ids = ids.reshape(regions, nl)
    count = int(ids.max()) + 1
    layouts = []
    for src in (half, disc):
        if src is None:
            layouts.append(None)
            continue
        dst = np.full((count, 2), np.nan)
        for i in range(regions):
            seen = ~np.isnan(dst[ids[i], 0])
            if np.any(np.abs(dst[ids[i]][seen] - src[i][seen]).max(initial=0.0) > 1e-12):
                raise AssertionError("shared sides do not coincide")
            dst[ids[i]] = src[i]
        layouts.append(dst)
    shared = {rs for pr in pairs for rs in pr}
    wall = [[False] + [(i, k) not in shared for k in range(4)] for i in range(regions)]
    bnd = np.unique(np.concatenate([ids[i][rim[k]] for i in range(regions) for k in range(4)
                                    if (i, k) not in shared]))
    return TreeSection(m=m, ids=ids, start=layouts[0], end=layouts[1],
                       patches=[[ids[i][p] for p in patches] for i in range(regions)], wall=wall, boundary=bnd)


@dataclass
class TreeSegment:
    """One vessel of a binary tree, in pre-order.  ``side`` 0 / 1: the half of the parent's end
    section it starts from (+y / -y of the parent's end frame); ``outlet``: the outlet label of a
    terminal segment (2, 3, ... in pre-order), else -1."""
    level: int
    parent: int
    side: int
    radius: float
    length: float
    half_angle: float          # turn of the centreline away from the parent's septum (rad); 0 for the root
    layers: int = 0
    outlet: int = -1


def tree_segments(depth: int = 4, seed: int = 0, root_radius: float = 2.5e-3) -> list:
    """Seeded binary tree of ``depth`` generations (2^depth - 1 segments): each daughter's radius is the
    parent's over 2^(1/3) (Murray's law for equal daughters) times U(0.9, 1.1); each segment is
    U(8, 12) of its radii long; each bifurcation's branch angle (between the two daughters) is
    U(30, 80) degrees, half of it to each daughter."""
    if not 1 <= depth <= 4:
        raise ValueError("tree depth must be 1..4")
    rng = np.random.Generator(np.random.PCG64(seed))
    segs: list = []

    def grow(level, parent, side, radius, half_angle):
        index = len(segs)
        segs.append(TreeSegment(level, parent, side, radius, rng.uniform(8.0, 12.0) * radius, half_angle))
        if level + 1 == depth:
            return
        angle = math.radians(rng.uniform(30.0, 80.0))
        radii = [radius * 2.0 ** (-1.0 / 3.0) * rng.uniform(0.9, 1.1) for _ in range(2)]
        for c in range(2):
            grow(level + 1, index, c, radii[c], 0.5 * angle)

    grow(0, -1, 0, root_radius, 0.0)
    label = 2
    for s in segs:
        if s.level == depth - 1:
            s.outlet = label
            label += 1
    return segs


@dataclass
class Tree:
    """Binary tree of swept O-grid segments: inlet label 1 at the root's first plane (z = 0, flow along
    +z), one outlet label per terminal segment, wall 0.  ``element_offset[i]`` / ``plane_ids[i]``:
    segment i's first element and its vertex planes' global ids; ``frames[i]``: its end centre,
    axis, e_s, e_y."""
    mesh: FlatMesh
    points: np.ndarray
    labels: np.ndarray
    cells: np.ndarray
    profile: np.ndarray
    radius: float
    segments: list
    element_offset: np.ndarray
    plane_ids: list
    frames: list
    outlet_labels: tuple


def binary_tree(depth: int = 4, seed: int = 0, root_radius: float = 2.5e-3, elements: int = 600_000,
                core: int = 8, ring: int = 3, bend_fraction: float = 0.5, morph_fraction: float = 0.375) -> Tree:
    """Swept O-grid binary tree (all hexahedra, one element per cell, C2 inside each patch and segment,
    C0 across patch and junction interfaces) on ``tree_segments``' seeded skeleton.

    A segment with 2^m terminal segments below it has 2^m regions of ``core`` x ``core`` cores with
    ``ring`` ring layers each, so every generation has 2^(depth-1) (core^2 + 4 core ring) cells per
    plane (1,280 for the defaults); the axial spacing is chosen so that the tree has about ``elements``
    elements.  The root runs straight along +z with its disc layout.  A daughter starts from its half
    of the parent's last plane (shared vertices), turns its centreline by its half-angle away from the
    parent's septum over ``bend_fraction`` of its length (about the septum line, smoothstep profile),
    and morphs its half-disc layout into its own disc over ``morph_fraction`` of it; its points keep
    s >= 0 in its turning frame, so the two daughters stay on their own sides of the parent's septum
    plane.  Daughters' septa are perpendicular to their parent's, so successive bifurcation planes
    alternate."""
    segs = tree_segments(depth, seed, root_radius)
    sections = [tree_section(m, core, ring) for m in range(depth)]
    per_region = core * core + 4 * core * ring
    spacing = sum(per_region * 2 ** (depth - 1 - s.level) * s.length for s in segs) / elements
    for s in segs:
        s.layers = max(3, int(round(s.length / spacing)))
    counts = []
    for s in segs:
        sec = sections[depth - 1 - s.level]
        counts.append((s.layers + (1 if s.parent < 0 else 0)) * len(sec.end))
    n = int(sum(counts))
    points = np.zeros((n, 3))
    labels = np.full(n, -1, np.int32)
    plane_ids: list = []
    frames: list = []
    blocks = []
    base = 0
    fine_per_layer = 64
    for i, s in enumerate(segs):
        sec = sections[depth - 1 - s.level]
        nl = len(sec.end)
        ids = np.zeros((s.layers + 1, nl), np.int64)
        if s.parent < 0:
            d, es, ey = np.array([0.0, 0.0, 1.0]), np.array([1.0, 0.0, 0.0]), np.array([0.0, 1.0, 0.0])
            ids[:] = base + np.arange((s.layers + 1) * nl).reshape(s.layers + 1, nl)
            for k in range(s.layers + 1):
                z = s.length * k / s.layers
                points[ids[k]] = (z * d + s.radius * (sec.end[:, :1] * es + sec.end[:, 1:] * ey))
            base += (s.layers + 1) * nl
            centre = s.length * d
            labels[ids[0]] = 1
        else:
            p = segs[s.parent]
            pc, pd, pes, pey = frames[s.parent]
            psec = sections[depth - 1 - p.level]
            k_half = len(sec.ids)
            to_parent = np.full(nl, -1, np.int64)
            for r in range(k_half):
                to_parent[sec.ids[r]] = psec.ids[s.side * k_half + r]
            ids[0] = plane_ids[s.parent][-1][to_parent]
            ids[1:] = base + np.arange(s.layers * nl).reshape(s.layers, nl)
            base += s.layers * nl
            n0 = pey if s.side == 0 else -pey
            ey = np.cross(pd, n0)
            t = s.length * np.arange(s.layers + 1) / s.layers
            fine = np.linspace(0.0, s.length, fine_per_layer * s.layers + 1)
            bend = bend_fraction * s.length
            th_f = s.half_angle * _smoothstep(fine / bend)
            dirs = np.cos(th_f)[:, None] * pd + np.sin(th_f)[:, None] * n0
            path = np.concatenate([np.zeros((1, 3)), np.cumsum(0.5 * (dirs[1:] + dirs[:-1]) * np.diff(fine)[:, None],
                                                               axis=0)])
            pivot = pc + np.stack([np.interp(t, fine, path[:, a]) for a in range(3)], axis=1)
            th = s.half_angle * _smoothstep(t / bend)
            w = _smoothstep(t / (morph_fraction * s.length))
            target = s.radius * sec.end + np.array([s.radius, 0.0])
            for k in range(1, s.layers + 1):
                loc = (1.0 - w[k]) * p.radius * sec.start + w[k] * target
                e_s = math.cos(th[k]) * n0 - math.sin(th[k]) * pd
                points[ids[k]] = pivot[k] + loc[:, :1] * e_s + loc[:, 1:] * ey
            d = math.cos(th[-1]) * pd + math.sin(th[-1]) * n0
            es = math.cos(th[-1]) * n0 - math.sin(th[-1]) * pd
            centre = pivot[-1] + s.radius * es
        if s.outlet >= 0:
            labels[ids[-1]] = s.outlet
        plane_ids.append(ids)
        frames.append((centre, d, es, ey))
        blocks.append(SweptBlock(patches=[g for reg in sec.patches for g in reg], ids=ids,
                                 wall=[f for reg in sec.wall for f in reg],
                                 bottom=1 if s.parent < 0 else None, top=s.outlet if s.outlet >= 0 else None))
    for i, s in enumerate(segs):
        labels[plane_ids[i][:, sections[depth - 1 - s.level].boundary].ravel()] = 0
    mesh, cells = swept_mesh(points, blocks)
    per_plane = [len(sections[depth - 1 - s.level].ids) * per_region for s in segs]
    element_offset = np.zeros(len(segs) + 1, np.int64)
    element_offset[1:] = np.cumsum([per_plane[i] * s.layers for i, s in enumerate(segs)])
    profile = np.zeros((n, 3))
    inlet = plane_ids[0][0]
    r2 = (points[inlet, 0] ** 2 + points[inlet, 1] ** 2) / root_radius ** 2
    profile[inlet, 2] = np.maximum(0.0, 1.0 - r2)
    profile[labels != 1] = 0.0
    return Tree(mesh=mesh, points=points, labels=labels, cells=cells, profile=profile, radius=root_radius,
                segments=segs, element_offset=element_offset, plane_ids=plane_ids, frames=frames,
                outlet_labels=tuple(s.outlet for s in segs if s.outlet >= 0))


def write_vtk(path, tube: Tube) -> None:
    n, E = len(tube.points), len(tube.cells)
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.1\nTubularFlowIGA-B200 synthetic control mesh\nASCII\n"
                "DATASET UNSTRUCTURED_GRID\n")
        f.write(f"POINTS {n} double\n")
        np.savetxt(f, tube.points, fmt="%.17g")
        f.write(f"CELLS {E} {9 * E}\n")
        np.savetxt(f, np.hstack([np.full((E, 1), 8), tube.cells]), fmt="%d")
        f.write(f"CELL_TYPES {E}\n")
        np.savetxt(f, np.full(E, 12), fmt="%d")
        f.write(f"POINT_DATA {n}\nSCALARS label float 1\nLOOKUP_TABLE default\n")
        np.savetxt(f, tube.labels, fmt="%d")


def fourier_waveform(seed: int, mean: float = 0.15, harmonics: int = 4, amplitude: float = 0.05,
                     period: float = 1.0):
    """Seeded Fourier inflow: mean + sum_k c_k cos(k theta) + s_k sin(k theta), amplitudes U(0, amplitude)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cosine = rng.uniform(0.0, amplitude, harmonics).tolist()
    sine = rng.uniform(0.0, amplitude, harmonics).tolist()
    return {"name": "inflow", "kind": "fourier", "units": "m/s", "mean": mean, "period": period,
            "phase": 0.0, "cosine": cosine, "sine": sine}


def simulation_config(density: float, viscosity: float, dt: float, steps: int, inlet_scale: float,
                      transient: bool = True, waveform: dict | None = None, outlets: list | None = None) -> dict:
    inlet = {"field": "velocity", "type": "dirichlet", "profile": "initial_velocityfield.txt",
             "scale": inlet_scale}
    if waveform is not None:
        inlet["waveform"] = waveform["name"]
    boundaries = [
        {"label": 0, "name": "wall", "conditions": [{"field": "velocity", "type": "dirichlet",
                                                      "value": [0.0, 0.0, 0.0]}]},
        {"label": 1, "name": "inlet", "conditions": [inlet]},
    ]
    if outlets is None:
        outlets = [{"label": 2, "name": "outlet", "conditions": [
            {"field": "pressure", "type": "pressure_traction", "value": 0.0}]}]
    boundaries += outlets
    cfg = {
        "schema_version": 3,
        "dimension": "3d",
        "fields": [{"name": "velocity", "kind": "vector3"}, {"name": "pressure", "kind": "pressure"}],
        "time": {"dt": dt, "steps": steps},
        "equation_systems": [{"name": "blood_flow", "kind": "navier_stokes",
                              "unknowns": ["velocity", "pressure"], "viscosity": viscosity,
                              "density": density,
                              "time_integration": "backward_euler" if transient else "steady"}],
        "boundaries": boundaries,
    }
    if waveform is not None:
        cfg["temporal_functions"] = [waveform]
    return cfg


def write_case(directory, tube: Tube, config: dict, database_name: str = "tube-1.ntiga") -> Path:
    """Write database + case directory; returns the database path."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    write_vtk(d / "controlmesh.vtk", tube)
    np.savetxt(d / "initial_velocityfield.txt", tube.profile, fmt="%.17g")
    (d / "simulation_config.json").write_text(json.dumps(config, indent=1))
    db = d / database_name
    write_ntiga(db, tube.mesh)
    return db


# Keys of a legacy transport case's simulation_parameter.txt (iga::ReadTransportParameters).
TRANSPORT_PARAMETER_KEYS = {"diffusion": "D", "vplus": "vplus", "vminus": "vminus", "kplus": "kplus",
                            "kminus": "kminus", "detach_plus": "k'plus", "detach_minus": "k'minus", "dt": "dt",
                            "steps": "nstep", "n0_bc": "N0bc", "nplus_bc": "Nplusbc", "nminus_bc": "Nminusbc",
                            "artificial_diffusion": "artificial_diffusion"}


def transport_parameter_text(params: dict) -> str:
    """simulation_parameter.txt: one `key value` line per parameter (missing ones are 0)."""
    lines = []
    for name, key in TRANSPORT_PARAMETER_KEYS.items():
        v = params.get(name, 0)
        lines.append(f"{key} {int(v)}" if name == "steps" else f"{key} {float(v):.17g}")
    return "\n".join(lines) + "\n"


def write_transport_case(directory, tube: Tube, params: dict, velocity=None, case_config: dict | None = None,
                         database_name: str = "tube-1.ntiga") -> Path:
    """Legacy transport case (controlmesh.vtk, initial_velocityfield.txt, simulation_parameter.txt and an
    optional case_config.json) plus the database; returns the database path."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    write_vtk(d / "controlmesh.vtk", tube)
    np.savetxt(d / "initial_velocityfield.txt", tube.profile if velocity is None else velocity, fmt="%.17g")
    (d / "simulation_parameter.txt").write_text(transport_parameter_text(params))
    if case_config is not None:
        (d / "case_config.json").write_text(json.dumps(case_config, indent=1))
    db = d / database_name
    write_ntiga(db, tube.mesh)
    return db


# Benchmark configurations (SI units: m, kg/m^3, Pa s).
def straight_cylinder_1280() -> Tube:
    """1,280 elements: 4x4 core + one 16-cell ring layer (32 cells/layer) x 40 layers, R 1.5 mm, L 30 mm."""
    return straight_tube(1.5e-3, 30e-3, core=4, ring=1, layers=40)


def pulsatile_tube_51200() -> Tube:
    """51,200 elements: 8x8 core + two 32-cell ring layers (128 cells/layer) x 400 layers, R 1.5 mm."""
    return straight_tube(1.5e-3, 30e-3, core=8, ring=2, layers=400)


@dataclass
class TubeBatch:
    """Many independent tubes as one mesh with disjoint node sets (a block-diagonal system).

    Every tube keeps its own labels (wall 0, inlet 1, outlet 2) and peak-1 inlet profile; the
    union is solved by one Newton/FGMRES loop whose kernels cover all tubes in each launch."""
    mesh: FlatMesh
    tubes: list
    node_offset: np.ndarray        # [T+1] first node of each tube
    element_offset: np.ndarray     # [T+1] first element of each tube
    inlet_scale: np.ndarray        # [T] inlet peak velocity of each tube (m/s)
    labels: np.ndarray             # [n] point labels of the union
    profile: np.ndarray            # [n, 3] peak-1 inlet profiles of the union


def combine_tubes(tubes, inlet_scale, gap: float = 1e-3) -> TubeBatch:
    """Disjoint union of tubes; tube k is shifted along x so that no two tubes touch."""
    node_offset = np.zeros(len(tubes) + 1, np.int64)
    element_offset = np.zeros(len(tubes) + 1, np.int64)
    eo, conn, xo, xc, xv, bez, lab = [np.zeros(1, np.int64)], [], [np.zeros(1, np.int64)], [], [], [], []
    labels, profile = [], []
    x = 0.0
    for k, t in enumerate(tubes):
        m = t.mesh
        node_offset[k + 1] = node_offset[k] + m.nodes
        element_offset[k + 1] = element_offset[k] + m.elements
        eo.append(eo[-1][-1] + m.element_offsets[1:].astype(np.int64))
        conn.append(m.connectivity.astype(np.int64) + node_offset[k])
        xo.append(xo[-1][-1] + m.extraction_offsets[1:].astype(np.int64))
        xc.append(m.extraction_columns)
        xv.append(m.extraction_values)
        b = m.bezier_points.reshape(-1, 3).copy()
        b[:, 0] += x + t.radius
        bez.append(b.ravel())
        x += 2 * t.radius + gap
        lab.append(m.boundary_labels)
        labels.append(t.labels)
        profile.append(t.profile)
    mesh = FlatMesh(
        nodes=int(node_offset[-1]),
        element_offsets=np.concatenate(eo).astype(np.int32),
        connectivity=np.concatenate(conn).astype(np.int32),
        extraction_offsets=np.concatenate(xo).astype(np.int32),
        extraction_columns=np.concatenate(xc).astype(np.uint8),
        extraction_values=np.concatenate(xv).astype(np.float64),
        bezier_points=np.concatenate(bez),
        boundary_labels=np.concatenate(lab).astype(np.int32),
    ).contiguous()
    return TubeBatch(mesh=mesh, tubes=list(tubes), node_offset=node_offset, element_offset=element_offset,
                     inlet_scale=np.asarray(inlet_scale, np.float64), labels=np.concatenate(labels),
                     profile=np.concatenate(profile))


@dataclass
class TubeSpec:
    """Parameters of one tube of a batch (enough to build it, or to estimate its cost)."""
    radius: float
    length: float
    layers: int
    inlet_scale: float
    curvature_radius: float = 0.0      # 0: straight, else helical with this centreline curvature radius
    handed: float = 1.0

    @property
    def elements(self) -> int:
        return 32 * self.layers

    def build(self) -> Tube:
        if self.curvature_radius > 0.0:
            return helical_tube(self.radius, self.length, self.curvature_radius, core=4, ring=1, layers=self.layers,
                                handed=self.handed)
        return straight_tube(self.radius, self.length, core=4, ring=1, layers=self.layers)


def tube_batch_specs(count: int, seed: int = 0, min_elements: int = 1000, max_elements: int = 8000,
                     density: float = 1060.0, viscosity: float = 3.5e-3, helical: float = 0.0,
                     log_sizes: bool = False) -> list:
    """Seeded tube parameters: radius U(0.5, 3) mm, length U(10, 40) radii, 4x4-core O-grid (32 cells
    per layer) with layers giving an element count drawn U(min_elements, max_elements) (log-uniform with
    ``log_sizes``), Reynolds number U(50, 800) giving the inlet peak velocity Re mu / (rho 2R); with
    probability ``helical`` a tube is helically curved with centreline curvature radius U(10, 40) mm."""
    rng = np.random.Generator(np.random.PCG64(seed))
    specs = []
    for _ in range(count):
        radius = rng.uniform(0.5e-3, 3e-3)
        length = rng.uniform(10.0, 40.0) * radius
        if log_sizes:
            elements = int(math.exp(rng.uniform(math.log(min_elements), math.log(max_elements))))
        else:
            elements = int(rng.uniform(min_elements, max_elements))
        layers = max(4, elements // 32)
        reynolds = rng.uniform(50.0, 800.0)
        curved = rng.uniform() < helical
        curvature = rng.uniform(10e-3, 40e-3) if curved else 0.0
        handed = 1.0 if rng.uniform() < 0.5 else -1.0
        specs.append(TubeSpec(radius, length, layers, reynolds * viscosity / (density * 2.0 * radius),
                              curvature, handed))
    return specs


def tube_batch(count: int, seed: int = 0, min_elements: int = 1000, max_elements: int = 8000,
               density: float = 1060.0, viscosity: float = 3.5e-3, helical: float = 0.0,
               log_sizes: bool = False, indices=None) -> TubeBatch:
    """Seeded batch of tubes of uneven sizes (``tube_batch_specs``) as one disjoint-union mesh; with
    ``indices``, only those tubes of the seeded batch (in that order)."""
    specs = tube_batch_specs(count, seed, min_elements, max_elements, density, viscosity, helical, log_sizes)
    chosen = range(count) if indices is None else indices
    return combine_tubes([specs[k].build() for k in chosen], [specs[k].inlet_scale for k in chosen])


def tube_cost(spec: TubeSpec) -> float:
    """Work estimate of one tube for partitioning a batch: sum_e nen_e^2 (the element contraction)
    plus the 4x4 block nonzeros (SpMV and Krylov), with nen = 64 and about 216 blocks per node row
    (a cubic C2 node couples to a 6x6x6 neighbourhood) for 1.03 nodes per element."""
    return spec.elements * 64.0 * 64.0 + 1.03 * spec.elements * 216.0


def pack_tubes(costs, parts: int) -> list:
    """Greedy longest-processing-time bin packing: tubes in decreasing cost, each into the part with the
    smallest total so far (ties to the lower part); each part's tubes in increasing index.  The largest
    part is within 4/3 of the optimum."""
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    totals = [0.0] * parts
    members = [[] for _ in range(parts)]
    for k in order:
        p = min(range(parts), key=lambda j: (totals[j], j))
        totals[p] += costs[k]
        members[p].append(k)
    return [sorted(m) for m in members]
