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
