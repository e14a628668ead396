"""Mixed-precision Newton path (TFIGA_PRECISION_MIXED): tensor-core tangent.

The tangent is contracted on the tcgen05 tensor cores with BF16 operands and
FP32 accumulation and stored in FP32; the residual stays FP64.  Tolerances:
* residual (rhs): 1e-12 relative per field, as the FP64 assembly;
* Jacobian: 2e-2 relative (Frobenius) per field pair (i, f) against the FP64
  oracle -- BF16 keeps 8 significant bits (unit roundoff 2^-9 ~ 2e-3 per
  operand), and the blocks whose terms cancel lose a few bits more;
* Newton: the mixed Newton iteration converges to the FP64 solution; after
  convergence to 1e-10 of the initial residual velocity and pressure agree to
  1e-8 relative L2 with the FP64 path (the accuracy bar of the mixed path; measured about
  2e-13 on the cylinder), and over several transient steps of the pulsatile
  section with the bench's solver settings every step stays within 1e-8
  (measured 3e-11 .. 7e-11).
Split-BF16 mode (TFIGA_PRECISION_MIXED_BF16X3, operands hi + lo, three
products): Jacobian within 1e-4 relative per field pair -- about 2^-16 per
product plus FP32 accumulation and the FP32 coefficients -- and Newton takes
no more iterations than with the FP64 tangent.
TF32 mode (TFIGA_PRECISION_MIXED_TF32, FP32 operands rounded to TF32, one
product): Jacobian within 5e-3 relative per field pair (2^-11 per operand,
eight times finer than BF16), and Newton converges to the FP64 solution.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

RHO, MU, DT = 1060.0, 3.5e-3, 1e-3
TANGENT_TOL = 2e-2
SPLIT_TOL = 1e-4
TF32_TOL = 5e-3


@pytest.fixture(scope="module")
def api():
    from tubularflowiga_b200 import api as a
    return a


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def random_state(nodes, seed, speed=0.2, pressure=20.0):
    rng = np.random.default_rng(seed)
    s = rng.normal(size=(nodes, 4))
    s[:, :3] *= speed
    s[:, 3] *= pressure
    return s.ravel()


def check_tensor_tangent(api, flat, rho, mu, dt, seed, precision=None, tol=TANGENT_TOL, kernel=0):
    mesh = api.Mesh(flat)
    ns = api.NavierStokes(mesh, density=rho, viscosity=mu, dt=dt, preconditioner=api.AMG,
                          precision=api.MIXED if precision is None else precision, tangent_kernel=kernel)
    st = random_state(flat.nodes, seed)
    pv = random_state(flat.nodes, seed + 1)
    ns.set_state(st, pv)
    values, rhs = ns.assemble()
    P = O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity)
    ov, orhs = O.assemble(flat, P, st, pv, rho, mu, dt)
    for f in range(4):
        assert rel(rhs[f::4], orhs[f::4]) < 1e-12
    v, r = values.reshape(-1, 4, 4), ov.reshape(-1, 4, 4)
    errors = np.array([[rel(v[:, i, f], r[:, i, f]) for f in range(4)] for i in range(4)])
    assert errors.max() < tol, errors
    return errors


def test_tensor_tangent_small_tube(api, small_tube):
    check_tensor_tangent(api, small_tube.mesh, RHO, MU, DT, 0)


def test_tensor_tangent_steady(api, small_tube):
    check_tensor_tangent(api, small_tube.mesh, RHO, MU, 0.0, 3)


def test_tensor_tangent_reference_tube_ragged(api, reference_tube):
    """Elements with 36..64 basis functions: padded rows and columns must not leak into the matrix."""
    from tubularflowiga_b200 import ntiga
    flat = ntiga.read(reference_tube / "tube-1.ntiga")
    check_tensor_tangent(api, flat, 1.0, 1.0, 0.1, 5)


# the tangent organisations: point coefficients stored by the point kernel and contracted per row-field
# pair (1) or per element (3), coefficients made in the tensor-core kernel from the stored point state
# with the basis staged from the FP64 tables (2)
KERNELS = [1, 2, 3]


@pytest.mark.parametrize("kernel", KERNELS)
def test_split_tangent_small_tube(api, small_tube, kernel):
    errors = check_tensor_tangent(api, small_tube.mesh, RHO, MU, DT, 0, api.MIXED_BF16X3, SPLIT_TOL, kernel)
    plain = check_tensor_tangent(api, small_tube.mesh, RHO, MU, DT, 0, kernel=kernel)
    assert errors.max() < 0.05 * plain.max()


@pytest.mark.parametrize("kernel", KERNELS)
def test_split_tangent_steady_and_ragged(api, small_tube, reference_tube, kernel):
    from tubularflowiga_b200 import ntiga
    check_tensor_tangent(api, small_tube.mesh, RHO, MU, 0.0, 3, api.MIXED_BF16X3, SPLIT_TOL, kernel)
    flat = ntiga.read(reference_tube / "tube-1.ntiga")
    check_tensor_tangent(api, flat, 1.0, 1.0, 0.1, 5, api.MIXED_BF16X3, SPLIT_TOL, kernel)


@pytest.mark.parametrize("kernel", KERNELS)
def test_tf32_tangent(api, small_tube, reference_tube, kernel):
    from tubularflowiga_b200 import ntiga
    errors = check_tensor_tangent(api, small_tube.mesh, RHO, MU, DT, 0, api.MIXED_TF32, TF32_TOL, kernel)
    plain = check_tensor_tangent(api, small_tube.mesh, RHO, MU, DT, 0, kernel=kernel)
    print(f"TF32 tangent error per field pair: max {errors.max():.2e} (BF16 {plain.max():.2e})")
    assert errors.max() < 0.5 * plain.max()
    check_tensor_tangent(api, small_tube.mesh, RHO, MU, 0.0, 3, api.MIXED_TF32, TF32_TOL, kernel)
    flat = ntiga.read(reference_tube / "tube-1.ntiga")
    check_tensor_tangent(api, flat, 1.0, 1.0, 0.1, 5, api.MIXED_TF32, TF32_TOL, kernel)


def test_tf32_newton_converges_to_fp64_solution(api, cylinder_1280):
    tube = cylinder_1280
    flat = tube.mesh
    vmask, pmask, vel = api.tube_boundary_conditions(tube, 0.2)
    s0 = api.initial_state(vmask, vel)
    mesh = api.Mesh(flat)
    states, reports = {}, {}
    for name, precision in (("fp64", api.FP64), ("tf32", api.MIXED_TF32)):
        ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG, precision=precision,
                              nonlinear_rtol=1e-10, nonlinear_atol=1e-30, gmres_rtol=1e-10, max_newton=20)
        ns.set_dirichlet(vmask, pmask, vel)
        ns.set_tractions({2: 0.0})
        ns.set_state(s0, s0)
        reports[name] = ns.step()
        states[name] = ns.get_state().reshape(-1, 4)
    print("Newton iterations: FP64", reports["fp64"]["newton_iterations"], "TF32", reports["tf32"]["newton_iterations"])
    assert reports["tf32"]["converged"]
    assert rel(states["tf32"][:, :3], states["fp64"][:, :3]) < 1e-8
    assert rel(states["tf32"][:, 3], states["fp64"][:, 3]) < 1e-8


def test_tangent_autotuner_picks_one_and_matches(api, small_tube):
    """TFIGA_TANGENT_AUTO: the first tangent times the three organisations (memory is plentiful here),
    keeps one, and every tangent it assembles agrees with the fixed organisations' to FP32 addition
    order."""
    flat = small_tube.mesh
    st, pv = random_state(flat.nodes, 21), random_state(flat.nodes, 22)
    got = {}
    for kernel in (0, 1, 2, 3):
        ns = api.NavierStokes(api.Mesh(flat), density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG,
                              precision=api.MIXED_BF16X3, tangent_kernel=kernel)
        ns.set_state(st, pv)
        got[kernel] = ns.assemble()[0]
        info = ns.tangent_kernel()
        if kernel == 0:
            assert info["kernel"] in ("coefficients", "fused", "element")
            assert info["coefficients_ms"] > 0 and info["fused_ms"] > 0 and info["element_ms"] > 0
            again = ns.assemble()[0]
            assert rel(again, got[0]) < 1e-6
        ns.close()
    assert rel(got[1], got[2]) < 1e-6 and rel(got[0], got[2]) < 1e-6 and rel(got[3], got[1]) < 1e-6


def test_split_newton_matches_fp64_iterations(api, cylinder_1280):
    tube = cylinder_1280
    flat = tube.mesh
    vmask, pmask, vel = api.tube_boundary_conditions(tube, 0.2)
    s0 = api.initial_state(vmask, vel)
    mesh = api.Mesh(flat)
    states, reports = {}, {}
    for name, precision in (("fp64", api.FP64), ("split", api.MIXED_BF16X3)):
        ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG, precision=precision,
                              nonlinear_rtol=1e-10, nonlinear_atol=1e-30, gmres_rtol=1e-10, max_newton=20)
        ns.set_dirichlet(vmask, pmask, vel)
        ns.set_tractions({2: 0.0})
        ns.set_state(s0, s0)
        reports[name] = ns.step()
        states[name] = ns.get_state().reshape(-1, 4)
    assert reports["split"]["converged"]
    assert reports["split"]["newton_iterations"] <= reports["fp64"]["newton_iterations"]
    assert rel(states["split"][:, :3], states["fp64"][:, :3]) < 1e-8
    assert rel(states["split"][:, 3], states["fp64"][:, 3]) < 1e-8


def test_tensor_tangent_is_repeatable_in_norm(api, small_tube):
    """Two assemblies of the same state agree to FP32 summation-order noise (atomic scatter order varies)."""
    flat = small_tube.mesh
    mesh = api.Mesh(flat)
    ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG, precision=api.MIXED)
    st = random_state(flat.nodes, 9)
    ns.set_state(st, st)
    v1, r1 = ns.assemble()
    v2, r2 = ns.assemble()
    assert rel(v1, v2) < 1e-6
    assert rel(r1, r2) < 1e-13


def test_mixed_newton_converges_to_fp64_solution(api, cylinder_1280):
    tube = cylinder_1280
    flat = tube.mesh
    vmask, pmask, vel = api.tube_boundary_conditions(tube, 0.2)
    s0 = api.initial_state(vmask, vel)
    mesh = api.Mesh(flat)
    states, reports = {}, {}
    for name, precision in (("fp64", api.FP64), ("mixed", api.MIXED)):
        ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG, precision=precision,
                              nonlinear_rtol=1e-10, nonlinear_atol=1e-30, gmres_rtol=1e-10, max_newton=20)
        ns.set_dirichlet(vmask, pmask, vel)
        ns.set_tractions({2: 0.0})
        ns.set_state(s0, s0)
        reports[name] = ns.step()
        states[name] = ns.get_state().reshape(-1, 4)
        ns.close()
    for name in ("mixed",):
        print(name, reports[name]["newton_iterations"], "Newton iterations; FP64", reports["fp64"]["newton_iterations"])
        assert reports[name]["converged"] and reports["fp64"]["converged"]
        assert reports[name]["newton_iterations"] <= reports["fp64"]["newton_iterations"] + 4
        assert rel(states[name][:, :3], states["fp64"][:, :3]) < 1e-8
        assert rel(states[name][:, 3], states["fp64"][:, 3]) < 1e-8


def test_mixed_transient_steps_match_fp64_on_the_pulsatile_section(api):
    """The 12,800-element section of the pulsatile tube (C2's cross-section and Fourier inflow, 100 layers),
    four backward-Euler steps at dt 2e-3 with the bench's solver settings (Newton rel.res 1e-10 on the FP64
    residual, Eisenstat-Walker linear tolerances, tangent reuse factor 100, AMG-FGMRES(64)): the split-BF16
    and the plain-BF16 mixed solvers and the FP64 solver from the same state with the same Dirichlet
    sequence agree within 1e-8 relative L2 on velocity and on pressure after every step."""
    import bench
    tube, _, wave = bench.workload("c2-100")
    mesh = api.Mesh(tube.mesh)
    vmask, pmask, velocity_at = bench.boundary(tube, wave)
    dt = 2e-3
    s0 = api.initial_state(vmask, velocity_at(0.0))
    trajectories = {}
    for name, precision in (("fp64", api.FP64), ("split", api.MIXED_BF16X3), ("bf16", api.MIXED)):
        ns = api.NavierStokes(mesh, precision=precision, density=1060.0, viscosity=3.5e-3, dt=dt,
                              nonlinear_rtol=1e-10, nonlinear_atol=1e-300, mass_rtol=1e-3, gmres_restart=64,
                              gmres_max_iterations=5000, gmres_rtol=1e-8, preconditioner=api.AMG,
                              amg_coarse_period=3, newton_forcing=1, tangent_reuse_factor=100.0)
        ns.set_dirichlet(vmask, pmask, velocity_at(0.0))
        ns.set_tractions({2: 0.0})
        ns.set_state(s0, s0)
        states = []
        for k in range(4):
            ns.set_dirichlet_values(velocity_at((k + 1) * dt).ravel())
            ns.commit_step()
            assert ns.step()["converged"]
            states.append(ns.get_state().reshape(-1, 4))
        ns.close()
        trajectories[name] = states
    for name in ("split", "bf16"):
        for k, (a, b) in enumerate(zip(trajectories[name], trajectories["fp64"])):
            ev, ep = rel(a[:, :3], b[:, :3]), rel(a[:, 3], b[:, 3])
            print(f"step {k + 1}: {name} vs FP64 velocity {ev:.3e} pressure {ep:.3e}")
            assert ev < 1e-8 and ep < 1e-8
