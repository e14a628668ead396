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

    ext_cache: dict = {}

    def ext(nc_, c_):
        key = (nc_, c_)
        if key not in ext_cache:
            ext_cache[key] = natural_extraction_1d(nc_, c_)
        return ext_cache[key]

    # Element enumeration: axial layer outermost, then patch, then v, then u.
    conn_list, rows_list, labels_list, cells, groups = [], [], [], [], {}
    for layer in range(layers):
        wv, wc = ext(layers, layer)
        for p, grid in enumerate(patches):
            nu, nv = grid.shape[0] - 1, grid.shape[1] - 1
            for jv in range(nv):
                vv, vc = ext(nv, jv)
                for iu in range(nu):
                    uv, uc = ext(nu, iu)
                    # local basis ordering: w outer, v, u inner
                    ids2 = grid[np.ix_(uv, vv)]                       # [nu_l, nv_l]
                    ids = (wv[:, None, None] * n2d + ids2.T[None, :, :]).reshape(-1)
                    key = (layers, layer, nu, iu, nv, jv)
                    if key not in groups:
                        # row (w,v,u) x Bernstein index c*16 + b*4 + a (u fastest)
                        rows = np.einsum("wc,vb,ua->wvucba", wc, vc, uc)
                        groups[key] = rows.reshape(len(wv) * len(vv) * len(uv), 64)
                    conn_list.append(ids.astype(np.int32))
                    rows_list.append(key)
                    lab = [-1] * 6
                    if layer == 0:
                        lab[0] = 1
                    if layer == layers - 1:
                        lab[5] = 2
                    if p > 0 and iu == nu - 1:
                        lab[2] = 0
                    labels_list.append(lab)
                    c = [grid[iu, jv], grid[iu + 1, jv], grid[iu + 1, jv + 1], grid[iu, jv + 1]]
                    cells.append([layer * n2d + v for v in c] + [(layer + 1) * n2d + v for v in c])
    E = len(conn_list)
    nen = np.array([len(c) for c in conn_list], np.int64)
    element_offsets = np.zeros(E + 1, np.int64)
    element_offsets[1:] = np.cumsum(nen)
    connectivity = np.concatenate(conn_list)
    # Sparse extraction rows and Bezier points, grouped by extraction type.
    xo = [0]
    xc_parts, xv_parts = [], []
    sparse_cache = {}
    for key in groups:
        rows = groups[key]
        cols = [np.nonzero(np.abs(r) > 0.0)[0].astype(np.uint8) for r in rows]
        vals = [rows[i][cols[i]] for i in range(len(rows))]
        sparse_cache[key] = (cols, vals)
    bezier = np.zeros((E, 64, 3))
    for e in range(E):
        cols, vals = sparse_cache[rows_list[e]]
        for c, v in zip(cols, vals):
            xc_parts.append(c); xv_parts.append(v)
            xo.append(xo[-1] + len(c))
    by_key: dict = {}
    for e, key in enumerate(rows_list):
        by_key.setdefault(key, []).append(e)
    for key, es in by_key.items():
        es = np.array(es)
        Cm = groups[key]                                          # [nen, 64]
        conn = np.stack([conn_list[e] for e in es])               # [g, nen]
        bezier[es] = np.einsum("ap,gad->gpd", Cm, points[conn])
    mesh = FlatMesh(
        nodes=n,
        element_offsets=element_offsets.astype(np.int32),
        connectivity=connectivity.astype(np.int32),
        extraction_offsets=np.array(xo, np.int32),
        extraction_columns=np.concatenate(xc_parts).astype(np.uint8),
        extraction_values=np.concatenate(xv_parts).astype(np.float64),
        bezier_points=bezier.ravel(),
        boundary_labels=np.array(labels_list, np.int32).ravel(),
    ).contiguous()
    return Tube(mesh=mesh, points=points, labels=labels, cells=np.array(cells, np.int64), profile=profile,
                radius=radius, length=length, planes=planes, per_plane=n2d)


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
        "schema_version": 4,
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


def tube_batch(count: int, seed: int = 0, min_elements: int = 1000, max_elements: int = 8000,
               density: float = 1060.0, viscosity: float = 3.5e-3) -> TubeBatch:
    """Seeded batch of straight tubes of uneven sizes: radius U(0.5, 3) mm, length U(10, 40) radii,
    4x4-core O-grid (32 cells per layer) with layers chosen so that each tube has an element count
    drawn U(min_elements, max_elements), Reynolds number U(50, 800) giving the inlet peak velocity
    Re mu / (rho 2R)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    tubes, scales = [], []
    for _ in range(count):
        radius = rng.uniform(0.5e-3, 3e-3)
        length = rng.uniform(10.0, 40.0) * radius
        elements = int(rng.uniform(min_elements, max_elements))
        layers = max(4, elements // 32)
        tubes.append(straight_tube(radius, length, core=4, ring=1, layers=layers))
        reynolds = rng.uniform(50.0, 800.0)
        scales.append(reynolds * viscosity / (density * 2.0 * radius))
    return combine_tubes(tubes, scales)
