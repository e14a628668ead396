"""Elements with 65..80 basis functions.

The reference's CUDA path accepts up to 80 basis functions per element
(solvers/cuda/include/DeviceMesh.hpp:55-56); its spline extraction produces them at the
extraordinary vertices of a bifurcation.  The fixture tests/golden/reference_bifurcation
is a Y-bifurcation made by the reference's own mesher, spline extractor and packer
(make_reference_bifurcation.sh): 2,688 elements with 36..80 basis functions, 60 of them
with 80.  The library moves those elements behind the others and assembles them with its
FP64 large-element kernels (80-wide tables); everything else takes the regular kernels.

* CPU: the oracle's restated element equals the reference's compiled element on the
  80-function elements (1e-12), so the oracle is pinned there too.
* GPU, against the oracle on the whole mesh: FP64 Jacobian blocks and residual 1e-12 per
  field pair; the split-BF16 mixed tangent 1e-4 per field pair (residual 1e-12); two
  Newton iterations with the reference's boundary set-up and wall trace 1e-10 on velocity
  and pressure (tight linear solves on both sides); the transport matrices 1e-12 of the
  largest entry.
"""
import lzma

import numpy as np
import pytest

from oracle import oracle as O
from tests.conftest import GOLDEN, requires_ref

RHO, MU, DT = 1.0, 1.0, 0.1          # the fixture's simulation_config.json physics


@pytest.fixture(scope="module")
def bifurcation(tmp_path_factory):
    d = tmp_path_factory.mktemp("reference_bifurcation")
    for f in (GOLDEN / "reference_bifurcation").glob("*.xz"):
        (d / f.name[:-3]).write_bytes(lzma.decompress(f.read_bytes()))
    return d


@pytest.fixture(scope="module")
def flat(bifurcation):
    from tubularflowiga_b200 import ntiga
    return ntiga.read(bifurcation / "bifurcation-1.ntiga")


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def random_state(nodes, seed, speed=0.01, pressure=1.0):
    rng = np.random.default_rng(seed)
    s = rng.normal(size=(nodes, 4))
    s[:, :3] *= speed
    s[:, 3] *= pressure
    return s.ravel()


def test_fixture_has_80_function_elements(flat):
    nen = np.diff(flat.element_offsets)
    assert nen.max() == 80 and (nen == 80).sum() >= 32 and nen.min() < 64


@requires_ref
def test_oracle_element_matches_reference_build_at_80_functions(flat):
    nen = np.diff(flat.element_offsets)
    large = np.nonzero(nen > 64)[0]
    st = random_state(flat.nodes, 3).reshape(-1, 4)
    pv = random_state(flat.nodes, 4).reshape(-1, 4)
    for e in large[::6]:
        conn, Cx, X, _ = flat.element(int(e))
        a_res, a_jac = O.ns_element(Cx, X, st[conn], pv[conn], RHO, MU, DT)
        b_res, b_jac = O.ns_element(Cx, X, st[conn], pv[conn], RHO, MU, DT, use_ref=True)
        assert rel(a_res, b_res) < 1e-12 and rel(a_jac, b_jac) < 1e-12


def field_pair_errors(values, reference):
    v, r = values.reshape(-1, 4, 4), reference.reshape(-1, 4, 4)
    return np.array([[rel(v[:, i, f], r[:, i, f]) for f in range(4)] for i in range(4)])


@pytest.mark.gpu
def test_assembly_with_80_function_elements_matches_oracle(flat):
    from tubularflowiga_b200 import api
    mesh = api.Mesh(flat)
    P = O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity)
    ro, cols, diag = mesh.pattern()
    assert np.array_equal(ro, P.row_offsets) and np.array_equal(cols, P.columns)
    st, pv = random_state(flat.nodes, 11), random_state(flat.nodes, 12)
    ov, orhs = O.assemble(flat, P, st, pv, RHO, MU, DT)
    ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT)
    ns.set_state(st, pv)
    values, rhs = ns.assemble()
    assert field_pair_errors(values, ov).max() < 1e-12
    for f in range(4):
        assert rel(rhs[f::4], orhs[f::4]) < 1e-12
    # the split-BF16 tensor-core path: regular elements on the tensor cores, the 80-function ones in FP64
    tc = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG,
                          precision=api.MIXED_BF16X3)
    tc.set_state(st, pv)
    tvalues, trhs = tc.assemble()
    assert field_pair_errors(tvalues, ov).max() < 1e-4
    for f in range(4):
        assert rel(trhs[f::4], orhs[f::4]) < 1e-12
    ns.close()
    tc.close()


@pytest.mark.gpu
def test_newton_iterations_on_the_reference_bifurcation(bifurcation, flat):
    """The reference's boundary set-up of the fixture's case (inlet profile x 0.01, no-slip wall plus
    the wall trace, traction-free outlets 2 and 3) and two Newton iterations of the first step, against
    the oracle's Newton with direct solves; GMRES to 1e-13 so that iterates, not tolerances, compare."""
    import ctypes
    import scipy.sparse.linalg as spla
    from tubularflowiga_b200 import api
    words = (bifurcation / "controlmesh.vtk").read_text().split()
    first = words.index("LOOKUP_TABLE") + 2
    labels = np.array(words[first:first + flat.nodes], np.int32)
    velocity = np.loadtxt(bifurcation / "initial_velocityfield.txt")
    bc = api.resolve_flow_boundaries(bifurcation / "simulation_config.json", labels, velocity, DT)
    wall = np.zeros(flat.nodes, np.int32)
    count = ctypes.c_int64()
    api.check(api.lib().tfiga_wall_trace_basis(str(bifurcation / "bifurcation-1.ntiga").encode(),
                                               str(bifurcation / "controlmesh.vtk").encode(),
                                               wall.ctypes.data_as(ctypes.c_void_p), flat.nodes,
                                               ctypes.byref(count)))
    vmask = bc["velocity_mask"].copy()
    vel = bc["velocity"].reshape(-1, 3).copy()
    vmask[wall[:count.value]] = 1
    vel[wall[:count.value]] = 0.0
    pmask, pressure = bc["pressure_mask"], bc["pressure"]
    assert vmask.sum() > 0
    mesh = api.Mesh(flat)
    ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG, gmres_rtol=1e-13,
                          gmres_max_iterations=20000, nonlinear_rtol=1e-30, nonlinear_atol=1e-300, mass_rtol=1e300)
    ns.set_dirichlet(vmask, pmask, vel, pressure)
    ns.set_tractions({2: 0.0, 3: 0.0})
    s0 = np.zeros(4 * flat.nodes)
    ns.set_state(s0, s0)
    P = O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity)
    state = s0.copy()
    for it in range(2):
        ns.newton_iteration(-1.0)
        values, rhs = O.assemble(flat, P, state, s0, RHO, MU, DT)
        O.apply_dirichlet(P, vmask, pmask, vel.ravel(), pressure, state, values, rhs)
        state = state + spla.spsolve(P.to_scipy(values).tocsc(), rhs)
        gpu = ns.get_state().reshape(-1, 4)
        ref = state.reshape(-1, 4)
        assert rel(gpu[:, :3], ref[:, :3]) < 1e-10, it
        assert rel(gpu[:, 3], ref[:, 3]) < 1e-10, it
    ns.close()


@pytest.mark.gpu
def test_transport_with_80_function_elements_matches_oracle(flat):
    from tubularflowiga_b200 import api
    mesh = api.Mesh(flat)
    rng = np.random.default_rng(8)
    velocity = rng.normal(size=(flat.nodes, 3)) * 0.1
    p = {"diffusion": 1e-2, "vplus": 0.8, "kplus": 0.5, "kminus": 0.1, "detach_plus": 0.2, "dt": 1e-2,
         "artificial_diffusion": 1e-3}
    params = api.transport_params(**p, n0_bc=1.0, nplus_bc=0.25, steps=1)
    mask = np.zeros(flat.nodes, np.int32)
    zeros = np.zeros(flat.nodes)
    t = api.Transport(mesh, params, velocity, mask, zeros, zeros)
    left, previous = t.matrices()
    P = O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity)
    ol, op = O.transport_assemble(flat, P, velocity, p, mask)
    for got, want in ((left, ol), (previous, op)):
        assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    t.close()
