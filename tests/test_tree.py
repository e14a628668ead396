"""Binary-tree generator (the 600k-element learned-stage training workload).

CPU:
* the seeded skeleton follows its specification: 2^depth - 1 segments in pre-order, daughter radii
  Murray's law x U(0.9, 1.1), lengths U(8, 12) radii, branch angles U(30, 80) degrees;
* the section layouts: the half-disc and disc layouts of every size have the same shared sides, every
  2D cell is positively oriented in both, and they cover the half disc / disc;
* a small tree is a valid body-fitted mesh (positive Jacobian at every Gauss point and element corner),
  its daughters share their parent's last vertex plane, each daughter's points stay on its side of the
  parent's septum plane, non-adjacent segments keep apart, and labels / face labels / element counts
  follow the construction;
* at the default size the tree has about 600k elements.

GPU: FP64 assembly on a small tree equals the oracle's (1e-12 per field pair), and one mixed-precision
step with traction-free outlets converges.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from tests.test_bifurcation import gauss_and_corner_det


def small_tree(seed=0):
    from tubularflowiga_b200 import meshgen
    return meshgen.binary_tree(seed=seed, core=2, ring=1, elements=6000)


def test_tree_skeleton_follows_its_specification():
    from tubularflowiga_b200 import meshgen
    segs = meshgen.tree_segments(depth=4, seed=3, root_radius=2.5e-3)
    assert len(segs) == 15
    assert segs[0].parent == -1 and segs[0].radius == 2.5e-3 and segs[0].half_angle == 0.0
    children = {}
    for i, s in enumerate(segs):
        assert 8.0 * s.radius <= s.length <= 12.0 * s.radius
        if s.parent >= 0:
            p = segs[s.parent]
            assert s.parent < i and s.level == p.level + 1
            ratio = s.radius / (p.radius * 2.0 ** (-1.0 / 3.0))
            assert 0.9 <= ratio <= 1.1
            assert math.radians(15.0) <= s.half_angle <= math.radians(40.0)
            children.setdefault(s.parent, []).append(i)
    for p, cs in children.items():
        assert [segs[c].side for c in cs] == [0, 1]
        assert segs[cs[0]].half_angle == segs[cs[1]].half_angle
    outlets = [s.outlet for s in segs if s.level == 3]
    assert outlets == list(range(2, 10))
    assert all(s.outlet == -1 for s in segs if s.level < 3)
    with pytest.raises(ValueError):
        meshgen.tree_segments(depth=5)


def _cell_areas(pos, patches):
    out = []
    for reg in patches:
        for g in reg:
            a, b, c, d = pos[g[:-1, :-1]], pos[g[1:, :-1]], pos[g[1:, 1:]], pos[g[:-1, 1:]]
            cross = lambda p, q: p[..., 0] * q[..., 1] - q[..., 0] * p[..., 1]
            out.append((0.5 * (cross(a, b) + cross(b, c) + cross(c, d) + cross(d, a))).ravel())
    return np.concatenate(out)


@pytest.mark.parametrize("m", [0, 1, 2, 3])
def test_section_layouts(m):
    from tubularflowiga_b200 import meshgen
    sec = meshgen.tree_section(m, 4, 2)
    assert sec.ids.shape[0] == 2 ** m
    per_region = 4 * 4 + 4 * 4 * 2
    for name, pos, area in (("start", sec.start, 0.5 * np.pi), ("end", sec.end, np.pi)):
        if pos is None:
            assert m == 3 and name == "start"
            continue
        a = _cell_areas(pos, sec.patches)
        assert a.size == 2 ** m * per_region
        assert a.min() > 0.0
        # the polygonal cells cover the (half) disc up to the chords of its arcs (16 chords of the
        # 4x4-core disc: 1 - sin(2 pi / 16) / (2 pi / 16) = 2.6%)
        assert abs(a.sum() - area) < 0.03 * area
    # boundary vertices lie on the unit circle (end layout) or on the half disc's boundary (start layout)
    r = np.hypot(sec.end[sec.boundary, 0], sec.end[sec.boundary, 1])
    assert np.allclose(r, 1.0)
    if sec.start is not None:
        s, y = sec.start[sec.boundary, 0], sec.start[sec.boundary, 1]
        assert np.all(np.isclose(np.hypot(s, y), 1.0) | np.isclose(s, 0.0, atol=1e-15))


def test_small_tree_geometry_junctions_and_labels():
    tr = small_tree()
    m = tr.mesh
    g = np.polynomial.legendre.leggauss(4)[0] * 0.5 + 0.5
    mins, maxs = gauss_and_corner_det(m.bezier_points, np.concatenate([[0.0], g, [1.0]]))
    assert mins.min() > 0.0 and (mins / maxs).min() > 0.1
    segs = tr.segments
    per_region = 2 * 2 + 4 * 2 * 1
    counts = [per_region * 2 ** (3 - s.level) * s.layers for s in segs]
    assert m.elements == sum(counts)
    assert np.array_equal(np.diff(tr.element_offset), counts)
    P = tr.points
    for i, s in enumerate(segs):
        if s.parent < 0:
            continue
        parent_last = tr.plane_ids[s.parent][-1]
        assert np.all(np.isin(tr.plane_ids[i][0], parent_last))
        centre, d, es, ey = tr.frames[s.parent]
        n0 = ey if s.side == 0 else -ey
        beyond = tr.plane_ids[i][1:].ravel()
        assert np.all((P[beyond] - centre) @ n0 > 0.0)
        # no vertex of a later plane is shared with another segment
        others = np.concatenate([tr.plane_ids[j][1:].ravel() for j in range(len(segs)) if j != i])
        assert not np.any(np.isin(beyond, others))
    # labels: inlet plane (rim is wall), one outlet label per terminal segment, wall elsewhere on the rims
    lab = tr.labels
    assert set(np.unique(lab)) == {-1, 0, 1} | set(tr.outlet_labels)
    assert np.all(np.isin(lab[tr.plane_ids[0][0]], (0, 1)))
    for s, ids in zip(segs, tr.plane_ids):
        if s.outlet >= 0:
            assert np.all(np.isin(lab[ids[-1]], (0, s.outlet))) and np.any(lab[ids[-1]] == s.outlet)
    assert np.all(tr.profile[lab == 1, 2] > 0) and np.all(tr.profile[lab != 1] == 0)
    faces = m.boundary_labels.reshape(-1, 6)
    root_cells = per_region * 8
    assert (faces[:, 0] == 1).sum() == root_cells
    for s in segs:
        if s.outlet >= 0:
            assert (faces[:, 5] == s.outlet).sum() == per_region
    assert (faces[:, 2] == 0).sum() > 0


def test_tree_segments_keep_apart():
    """Every vertex of a segment lies farther than 2 radii from the centreline of any segment that is not
    its parent, daughter or sibling (centre of each vertex plane's rim, radius its largest rim distance)."""
    from tubularflowiga_b200 import meshgen
    from scipy.spatial import cKDTree
    tr = small_tree(seed=1)
    segs = tr.segments
    secs = [meshgen.tree_section(k, 2, 1) for k in range(4)]
    info = []
    for i, s in enumerate(segs):
        ids = tr.plane_ids[i]
        bnd = secs[3 - s.level].boundary
        rim = tr.points[ids[:, bnd]]
        c = rim.mean(axis=1)
        r = np.linalg.norm(rim - c[:, None, :], axis=2).max(axis=1)
        info.append((c, r, tr.points[ids[1:].ravel()]))
    for i in range(len(segs)):
        for j in range(len(segs)):
            si, sj = segs[i], segs[j]
            if i == j or si.parent == j or sj.parent == i or (si.parent == sj.parent and si.parent >= 0):
                continue
            c, r, _ = info[j]
            d, k = cKDTree(c).query(info[i][2])
            assert (d / r[k]).min() > 2.0, (i, j)


def test_default_tree_size():
    from tubularflowiga_b200 import meshgen
    segs = meshgen.tree_segments()
    per_region = 8 * 8 + 4 * 8 * 3
    spacing = sum(per_region * 2 ** (3 - s.level) * s.length for s in segs) / 600_000
    total = sum(per_region * 2 ** (3 - s.level) * max(3, int(round(s.length / spacing))) for s in segs)
    assert abs(total - 600_000) < 0.002 * 600_000


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.gpu
def test_tree_assembly_matches_oracle_and_steps():
    from tubularflowiga_b200 import api
    tr = small_tree()
    flat = tr.mesh
    P = O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity)
    rng = np.random.default_rng(5)
    st = (rng.normal(size=(flat.nodes, 4)) * [0.1, 0.1, 0.1, 10.0]).ravel()
    pv = (rng.normal(size=(flat.nodes, 4)) * [0.1, 0.1, 0.1, 10.0]).ravel()
    ov, orhs = O.assemble(flat, P, st, pv, 1060.0, 3.5e-3, 2e-3)
    mesh = api.Mesh(flat)
    ns = api.NavierStokes(mesh, density=1060.0, viscosity=3.5e-3, dt=2e-3)
    ns.set_state(st, pv)
    values, rhs = ns.assemble()
    v, r = values.reshape(-1, 4, 4), ov.reshape(-1, 4, 4)
    for i in range(4):
        for f in range(4):
            assert rel(v[:, i, f], r[:, i, f]) < 1e-12
    for f in range(4):
        assert rel(rhs[f::4], orhs[f::4]) < 1e-12
    ns.close()
    vmask, pmask, vel = api.tube_boundary_conditions(tr, 0.1)
    mixed = api.NavierStokes(mesh, density=1060.0, viscosity=3.5e-3, dt=2e-3, preconditioner=api.AMG,
                             precision=api.MIXED_BF16X3, nonlinear_rtol=1e-10, nonlinear_atol=1e-300)
    mixed.set_dirichlet(vmask, pmask, vel)
    mixed.set_tractions({label: 0.0 for label in tr.outlet_labels})
    s0 = api.initial_state(vmask, vel)
    mixed.set_state(s0, s0)
    report = mixed.step()
    assert report["converged"]
    flows = mixed.boundary_flows([1] + list(tr.outlet_labels))
    inflow, outflows = -flows[0], flows[1:]
    assert inflow > 0 and np.all(outflows > 0)
    assert abs(outflows.sum() - inflow) < 1e-3 * inflow
    mixed.close()
