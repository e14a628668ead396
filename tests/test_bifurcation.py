"""Y-bifurcation generator and outlet-coupled steps.

CPU: the swept O-grid Y is a valid body-fitted mesh (positive Jacobian at
every Gauss point and element corner, checked against the oracle's
determinant), its daughters share the junction plane with the parent, they
never overlap, and its labels and element counts follow the construction.

GPU (tolerances as in the straight-tube parity tests):
* FP64 assembly on a small Y equals the oracle's to 1e-12 relative per field
  pair (the junction's C0 connectivity goes through the same pattern);
* the tensor-core tangent on the Y is within 2e-2 per field pair (1e-4 in the
  split-BF16 mode);
* tfiga_ns_step_outlets with RCR outlets reproduces, to 1e-10, the coupling
  loop written out on the host with the oracle's outlet model
  (OutletModel.hpp:70-150 restated in C); an iteration cap that is too small
  ends with TFIGA_E_NOT_CONVERGED.
"""
import ctypes
from math import comb

import numpy as np
import pytest

from oracle import oracle as O

RHO, MU, DT = 1060.0, 3.5e-3, 2e-3


def small_y():
    from tubularflowiga_b200 import meshgen
    return meshgen.y_bifurcation(parent_layers=5, daughter_layers=4, ax=2, ay=4, ring=1,
                                 parent_length=6e-3, daughter_length=5e-3)


def gauss_and_corner_det(bezier, pts1d):
    """det J of the Bezier geometry map on [0,1]^3 at the tensor points pts1d^3 (per element: min, max)."""
    t = np.asarray(pts1d)
    B = np.stack([comb(3, i) * t ** i * (1 - t) ** (3 - i) for i in range(4)], -1)
    dB = np.stack([3 * ((comb(2, i - 1) * t ** (i - 1) * (1 - t) ** (3 - i)) if i > 0 else 0 * t)
                   - 3 * ((comb(2, i) * t ** i * (1 - t) ** (2 - i)) if i < 3 else 0 * t) for i in range(4)], -1)
    n = len(t)
    G = np.zeros((n ** 3, 64, 3))
    q = 0
    for k in range(n):
        for j in range(n):
            for i in range(n):
                G[q, :, 0] = np.einsum("c,b,a->cba", B[k], B[j], dB[i]).ravel()
                G[q, :, 1] = np.einsum("c,b,a->cba", B[k], dB[j], B[i]).ravel()
                G[q, :, 2] = np.einsum("c,b,a->cba", dB[k], B[j], B[i]).ravel()
                q += 1
    d = np.linalg.det(np.einsum("epi,qpj->eqij", bezier.reshape(-1, 64, 3), G))
    return d.min(1), d.max(1)


def test_y_bifurcation_counts_and_geometry():
    y = small_y()
    m = y.mesh
    per_half = 2 * 4 + 2 * (2 + 4) * 1                   # ax ay + 2 (ax + ay) ring
    assert m.elements == 2 * per_half * (5 + 4)
    half_vertices = 3 * 5 + 2 * (2 + 4) * 1
    parent_plane = 2 * half_vertices - (4 + 1)
    assert m.nodes == parent_plane * 6 + 2 * half_vertices * 4
    g = np.polynomial.legendre.leggauss(4)[0] * 0.5 + 0.5
    mins, maxs = gauss_and_corner_det(m.bezier_points, np.concatenate([[0.0], g, [1.0]]))
    assert mins.min() > 0.0 and (mins / maxs).min() > 0.1
    # the oracle's determinant is taken on the reference's [-1,1]^3 parametric domain (1/8 of ours)
    gm, _ = gauss_and_corner_det(m.bezier_points, g)
    bad = ctypes.c_int()
    for e in range(0, m.elements, 7):
        X = np.ascontiguousarray(m.bezier_points.reshape(-1, 64, 3)[e].ravel())
        assert abs(8.0 * O.lib().tfo_min_determinant(X, ctypes.byref(bad)) - gm[e]) <= 1e-12 * gm[e]
        assert bad.value == 0


def test_y_bifurcation_junction_symmetry_and_labels():
    y = small_y()
    P, lab = y.points, y.labels
    zj = 6e-3
    parent_plane = 2 * (3 * 5 + 2 * (2 + 4)) - (4 + 1)
    parent = np.isclose(P[:, 2], zj, rtol=0, atol=1e-12) & (np.arange(len(P)) < (y.parent_layers + 1) * parent_plane)
    # every element touching the junction plane uses parent-plane vertices there (shared, C0)
    conn = y.mesh.connectivity
    on_plane = np.isclose(P[conn, 2], zj, rtol=0, atol=1e-12)
    assert np.all(parent[conn[on_plane]])
    # beyond the junction: the daughters keep to their own side of x = 0 and mirror each other
    beyond = P[:, 2] > zj + 1e-12
    assert not np.any(np.abs(P[beyond, 0]) < 1e-9)
    left, right = P[beyond & (P[:, 0] < 0)], P[beyond & (P[:, 0] > 0)]
    assert len(left) == len(right)
    from scipy.spatial import cKDTree
    dist, match = cKDTree(left).query(right * [-1.0, 1.0, 1.0])
    assert dist.max() < 1e-15 and len(np.unique(match)) == len(left)
    # labels: inlet plane (rim is wall), two outlets, septum line of the junction is wall
    assert set(np.unique(lab)) == {-1, 0, 1, 2, 3}
    assert (lab == 2).sum() == (lab == 3).sum() > 0
    septum = parent & (np.abs(P[:, 0]) < 1e-15)
    assert septum.sum() == 5 and np.all(lab[septum] == 0)
    inlet = np.isclose(P[:, 2], 0.0)
    assert np.all(np.isin(lab[inlet], (0, 1)))
    assert np.all(y.profile[lab == 1, 2] > 0) and np.all(y.profile[lab != 1] == 0)
    # faces: inlet label 1 on the first parent layer, outlets 2 and 3 on the daughters' last layers
    faces = y.mesh.boundary_labels.reshape(-1, 6)
    assert (faces[:, 0] == 1).sum() == 2 * (2 * 4 + 2 * 6)
    assert (faces[:, 5] == 2).sum() == (faces[:, 5] == 3).sum() == 2 * 4 + 2 * 6


def test_outlet_struct_layout():
    from tubularflowiga_b200 import api
    assert ctypes.sizeof(api.Outlet) == 8 + 8 * 8
    o = api.Outlet.rcr(2, 1e8, 1e-10, 1e9)
    assert (o.kind, o.proximal_resistance, o.capacitance, o.distal_resistance) == (api.OUTLET_RCR, 1e8, 1e-10, 1e9)


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def random_state(nodes, seed, speed=0.2, pressure=20.0):
    rng = np.random.default_rng(seed)
    s = rng.normal(size=(nodes, 4))
    s[:, :3] *= speed
    s[:, 3] *= pressure
    return s.ravel()


@pytest.mark.gpu
def test_y_bifurcation_assembly_matches_oracle():
    from tubularflowiga_b200 import api
    flat = small_y().mesh
    P = O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity)
    st, pv = random_state(flat.nodes, 21), random_state(flat.nodes, 22)
    ov, orhs = O.assemble(flat, P, st, pv, RHO, MU, DT)
    mesh = api.Mesh(flat)
    ro, cols, _ = mesh.pattern()
    assert np.array_equal(ro, P.row_offsets) and np.array_equal(cols, P.columns)
    for precision, tol in ((api.FP64, 1e-12), (api.MIXED, 2e-2), (api.MIXED_BF16X3, 1e-4)):
        ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG, precision=precision)
        ns.set_state(st, pv)
        values, rhs = ns.assemble()
        v, r = values.reshape(-1, 4, 4), ov.reshape(-1, 4, 4)
        assert max(rel(v[:, i, f], r[:, i, f]) for i in range(4) for f in range(4)) < tol
        for f in range(4):
            assert rel(rhs[f::4], orhs[f::4]) < 1e-12


def _y_solver(api, y, **kw):
    from tubularflowiga_b200 import api as a
    vmask, pmask, vel = a.tube_boundary_conditions(y, 0.15)
    ns = a.NavierStokes(a.Mesh(y.mesh), density=RHO, viscosity=MU, dt=DT, preconditioner=a.AMG,
                        nonlinear_rtol=1e-10, nonlinear_atol=1e-16, gmres_rtol=1e-12,
                        gmres_max_iterations=20000, **kw)
    ns.set_dirichlet(vmask, pmask, vel)
    s0 = a.initial_state(vmask, vel)
    ns.set_state(s0, s0)
    return ns


@pytest.mark.gpu
def test_step_outlets_matches_host_coupling_loop():
    from tubularflowiga_b200 import api
    y = small_y()
    models = [api.Outlet.rcr(2, 1e8, 1e-10, 1e9), api.Outlet.rcr(3, 1e8, 1e-10, 1e9)]
    relaxation = 1.0
    # library loop
    ns = _y_solver(api, y)
    lib_outlets = [api.Outlet(**m.as_dict()) for m in models]
    history = []
    for step in range(2):
        ns.commit_step()
        rep = ns.step_outlets(lib_outlets, relaxation=relaxation, max_iterations=12)
        assert rep["converged"] and rep["outlet_iterations"] >= 2
        history.append([o.as_dict() for o in lib_outlets])
    lib_state = ns.get_state()
    # the same loop on the host (iga_cuda.cu:927-1086) with the oracle's outlet model
    ns2 = _y_solver(api, y)
    host = [m.as_dict() for m in models]
    for step in range(2):
        ns2.commit_step()
        previous = [h["capacitor_pressure"] for h in host]
        for it in range(12):
            ns2.set_tractions({h["label"]: h["pressure"] for h in host})
            assert ns2.step()["converged"]
            flows = ns2.boundary_flows([h["label"] for h in host])
            ev = [O.outlet_model(2, 0.0, h["proximal_resistance"], h["distal_resistance"], h["capacitance"],
                                 h["reference_pressure"], previous[i], flows[i], DT) for i, h in enumerate(host)]
            change = max(abs(ev[i][0] - h["pressure"]) for i, h in enumerate(host))
            scale = max([1.0] + [abs(e[0]) for e in ev])
            if change <= 1e-8 + 1e-6 * scale:
                for i, h in enumerate(host):
                    h.update(flow=flows[i], pressure=ev[i][0], capacitor_pressure=ev[i][1])
                break
            for i, h in enumerate(host):
                h.update(flow=flows[i], pressure=(1 - relaxation) * h["pressure"] + relaxation * ev[i][0])
        else:
            pytest.fail("host coupling loop did not converge")
        for i, h in enumerate(host):
            for k in ("flow", "pressure", "capacitor_pressure"):
                assert abs(history[step][i][k] - h[k]) <= 1e-10 * max(abs(h[k]), 1e-30), (step, i, k)
    assert history[-1][0]["flow"] > 0 and history[-1][1]["flow"] > 0
    # symmetric Y: the two outlets carry the same flow
    assert abs(history[-1][0]["flow"] - history[-1][1]["flow"]) <= 1e-6 * history[-1][0]["flow"]
    assert rel(lib_state, ns2.get_state()) < 1e-10


@pytest.mark.gpu
def test_step_outlets_reports_non_convergence():
    from tubularflowiga_b200 import api
    ns = _y_solver(api, small_y())
    outlets = [api.Outlet.rcr(2, 1e8, 1e-10, 1e9), api.Outlet.rcr(3, 1e8, 1e-10, 1e9)]
    ns.commit_step()
    with pytest.raises(api.TfigaError, match="outlet fixed-point iteration did not converge"):
        ns.step_outlets(outlets, relaxation=0.5, max_iterations=1)


@pytest.mark.gpu
def test_step_outlets_coupled_reaches_the_outer_loop_fixed_point():
    """Outlet pressures updated inside one Newton loop: the accepted pressures, flows and state agree with
    the reference's outer loop within the coupling tolerance (1e-6 relative on P), with fewer solves."""
    from tubularflowiga_b200 import api
    y = small_y()
    outer_ns, coupled_ns = _y_solver(api, y), _y_solver(api, y)
    outer = [api.Outlet.rcr(2, 1e8, 1e-10, 1e9), api.Outlet.rcr(3, 1e8, 1e-10, 1e9)]
    coupled = [api.Outlet(**o.as_dict()) for o in outer]
    solves = {"outer": 0, "coupled": 0}
    for step in range(3):
        outer_ns.commit_step()
        coupled_ns.commit_step()
        a = outer_ns.step_outlets(outer, relaxation=1.0, max_iterations=12)
        b = coupled_ns.step_outlets_coupled(coupled, relaxation=1.0, max_newton=20)
        assert a["converged"] and b["converged"]
        solves["outer"] += a["newton_iterations"]
        solves["coupled"] += b["newton_iterations"]
        for o, c in zip(outer, coupled):
            assert abs(o.pressure - c.pressure) <= 2e-6 * abs(o.pressure)
            assert abs(o.capacitor_pressure - c.capacitor_pressure) <= 2e-6 * abs(o.capacitor_pressure)
            assert abs(o.flow - c.flow) <= 1e-7 * abs(o.flow)
        assert rel(coupled_ns.get_state(), outer_ns.get_state()) < 1e-7
    assert solves["coupled"] < solves["outer"]
