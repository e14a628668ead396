"""Batched solve of independent tubes as one disjoint-union mesh (block-diagonal system).

CPU: the generator's union keeps every tube's nodes, elements, labels and
profiles in disjoint ranges.  GPU: Newton on the union (FP64, AMG-FGMRES to
tight tolerances) reproduces every tube solved on its own to 1e-8 relative L2
in velocity and 1e-6 in pressure.
"""
import numpy as np
import pytest


def test_tube_batch_union_is_disjoint():
    from tubularflowiga_b200 import meshgen
    batch = meshgen.tube_batch(3, seed=1, min_elements=150, max_elements=400)
    m = batch.mesh
    assert m.nodes == sum(t.mesh.nodes for t in batch.tubes)
    assert m.elements == sum(t.mesh.elements for t in batch.tubes)
    for k, t in enumerate(batch.tubes):
        e0, e1 = batch.element_offset[k], batch.element_offset[k + 1]
        c = m.connectivity[m.element_offsets[e0]:m.element_offsets[e1]]
        assert c.min() >= batch.node_offset[k] and c.max() < batch.node_offset[k + 1]
        assert np.array_equal(batch.labels[batch.node_offset[k]:batch.node_offset[k + 1]], t.labels)
    assert (batch.inlet_scale > 0).all()


@pytest.mark.gpu
def test_union_solve_matches_individual_tubes():
    from tubularflowiga_b200 import api, meshgen
    batch = meshgen.tube_batch(3, seed=2, min_elements=150, max_elements=400)
    # Newton stops at 1e-12 of its own initial residual or at an RMS of 1e-16, whichever is larger: a
    # small tube alone starts from a residual so small that 1e-12 of it lies below the FP64 floor.
    kw = dict(density=1060.0, viscosity=3.5e-3, dt=1e-3, preconditioner=api.AMG, nonlinear_rtol=1e-12,
              nonlinear_atol=1e-16, gmres_rtol=1e-12, gmres_max_iterations=20000, max_newton=20)
    vmask, pmask, vel = api.batch_boundary_conditions(batch)
    s0 = api.initial_state(vmask, vel)
    ns = api.NavierStokes(api.Mesh(batch.mesh), **kw)
    ns.set_dirichlet(vmask, pmask, vel)
    ns.set_tractions({2: 0.0})
    ns.set_state(s0, s0)
    assert ns.step()["converged"]
    union = ns.get_state().reshape(-1, 4)
    for k, tube in enumerate(batch.tubes):
        vm, pm, v = api.tube_boundary_conditions(tube, batch.inlet_scale[k])
        s = api.initial_state(vm, v)
        one = api.NavierStokes(api.Mesh(tube.mesh), **kw)
        one.set_dirichlet(vm, pm, v)
        one.set_tractions({2: 0.0})
        one.set_state(s, s)
        assert one.step()["converged"]
        ref = one.get_state().reshape(-1, 4)
        part = union[batch.node_offset[k]:batch.node_offset[k + 1]]
        assert np.linalg.norm(part[:, :3] - ref[:, :3]) <= 1e-8 * np.linalg.norm(ref[:, :3])
        assert np.linalg.norm(part[:, 3] - ref[:, 3]) <= 1e-6 * max(np.linalg.norm(ref[:, 3]), 1e-300)


@pytest.mark.gpu
def test_batch_mesh_through_the_c_abi_matches_the_union():
    """tfiga_batch_mesh_create gives the same mesh as the generator's disjoint union (pattern, sizes,
    geometry check) and the tube offsets."""
    from tubularflowiga_b200 import api, meshgen
    tubes = [meshgen.straight_tube(1e-3, 3e-3, 4, 1, k) for k in (2, 3)]
    union = meshgen.combine_tubes(tubes, [1.0, 1.0])
    a = api.Mesh([t.mesh for t in tubes])
    b = api.Mesh(union.mesh)
    assert list(a.node_offsets) == list(union.node_offset) and list(a.element_offsets) == list(union.element_offset)
    for key in ("nodes", "elements", "basis_entries", "extraction_nonzeros", "block_nonzeros", "bad_samples"):
        assert a.info[key] == b.info[key], key
    assert abs(a.info["min_detj"] - b.info["min_detj"]) <= 1e-12 * abs(b.info["min_detj"])
    for x, y in zip(a.pattern(), b.pattern()):
        assert np.array_equal(x, y)


def test_helical_tube_geometry():
    """The helical sweep: valid Jacobians at every Gauss point (oracle determinant), the inlet in z = 0
    with its profile along +z, and the centreline's curvature radius recovered from the plane centres."""
    import ctypes
    from oracle import oracle as O
    from tubularflowiga_b200 import meshgen
    R, Rc = 1.5e-3, 12e-3
    t = meshgen.helical_tube(R, 40e-3, Rc, core=4, ring=1, layers=40)
    bad = ctypes.c_int()
    for e in range(t.mesh.elements):
        O.lib().tfo_min_determinant(np.ascontiguousarray(t.mesh.element(e)[2].ravel()), ctypes.byref(bad))
        assert bad.value == 0
    assert np.abs(t.points[:t.per_plane, 2]).max() < 1e-15
    assert np.allclose(t.profile[t.labels == 1][:, :2], 0.0) and t.profile[:, 2].max() == pytest.approx(1.0)
    # centreline = mean of each plane's rim; curvature radius from three consecutive centres
    rim = t.labels[:t.per_plane] == 0
    c = np.stack([t.points[k * t.per_plane:(k + 1) * t.per_plane][rim].mean(axis=0) for k in range(t.planes)])
    a, b, d = c[19], c[20], c[21]
    ab, bd, ad = np.linalg.norm(b - a), np.linalg.norm(d - b), np.linalg.norm(d - a)
    area = 0.5 * np.linalg.norm(np.cross(b - a, d - a))
    assert ab * bd * ad / (4 * area) == pytest.approx(Rc, rel=2e-2)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["bf16x3", "fp64"])
def test_per_tube_newton_tests_match_individual_tubes(precision):
    """Per-tube Newton tests and per-tube FGMRES on a batch of straight and helical tubes
    (tfiga_ns_set_segments: each tube its own Newton test, and its own Arnoldi process, Hessenberg
    matrix and tolerance inside the union's linear solve): every tube passes its own relative test, and
    its part of the union equals the tube solved alone with the same test (1e-8 velocity, 1e-6 pressure
    relative L2); FP32 Krylov basis with the split-BF16 tangent, FP64 basis with the FP64 solver."""
    from tubularflowiga_b200 import api, meshgen
    batch = meshgen.tube_batch(4, seed=5, min_elements=150, max_elements=400, helical=0.5)
    specs = meshgen.tube_batch_specs(4, seed=5, min_elements=150, max_elements=400, helical=0.5)
    assert any(s.curvature_radius > 0 for s in specs) and any(s.curvature_radius == 0 for s in specs)
    mode = api.MIXED_BF16X3 if precision == "bf16x3" else api.FP64
    kw = dict(density=1060.0, viscosity=3.5e-3, dt=1e-3, preconditioner=api.AMG, precision=mode,
              nonlinear_rtol=1e-10, nonlinear_atol=1e-300, gmres_rtol=1e-10, gmres_max_iterations=20000,
              max_newton=25, gmres_restart=64)
    vmask, pmask, vel = api.batch_boundary_conditions(batch)
    s0 = api.initial_state(vmask, vel)
    ns = api.NavierStokes(api.Mesh(batch.mesh), **kw)
    ns.set_segments(batch.node_offset)
    ns.set_dirichlet(vmask, pmask, vel)
    ns.set_tractions({2: 0.0})
    ns.set_state(s0, s0)
    assert ns.step()["converged"]
    done, residuals = ns.segment_status()
    assert done.all() and np.isfinite(residuals).all()
    union = ns.get_state().reshape(-1, 4)
    for k, t in enumerate(batch.tubes):
        vm, pm, v = api.tube_boundary_conditions(t, batch.inlet_scale[k])
        s = api.initial_state(vm, v)
        one = api.NavierStokes(api.Mesh(t.mesh), **kw)
        one.set_dirichlet(vm, pm, v)
        one.set_tractions({2: 0.0})
        one.set_state(s, s)
        assert one.step()["converged"]
        ref = one.get_state().reshape(-1, 4)
        part = union[batch.node_offset[k]:batch.node_offset[k + 1]]
        assert np.linalg.norm(part[:, :3] - ref[:, :3]) <= 1e-8 * np.linalg.norm(ref[:, :3]), k
        assert np.linalg.norm(part[:, 3] - ref[:, 3]) <= 1e-6 * max(np.linalg.norm(ref[:, 3]), 1e-300), k
        one.close()
    ns.close()
