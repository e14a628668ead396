"""Inexact Newton (newton_forcing = 1): each Newton system is solved to an
Eisenstat-Walker forcing tolerance after the step's Dirichlet values are lifted
into the state.  On the 1,280-element cylinder a step converges to the same
solution as the fixed-tolerance step -- velocity within 1e-8 and pressure within
1e-6 relative L2, the tolerances of the mixed-vs-FP64 Newton test, both stopping
at rel.res 1e-10 -- with fewer FGMRES iterations, in FP64 and in the split-BF16
mode."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO, MU, DT = 1060.0, 3.5e-3, 1e-3


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.parametrize("precision_name", ["FP64", "MIXED_BF16X3"])
def test_forcing_step_matches_fixed_tolerance_step(cylinder_1280, precision_name):
    from tubularflowiga_b200 import api
    tube = cylinder_1280
    flat = tube.mesh
    vmask, pmask, vel = api.tube_boundary_conditions(tube, 0.2)
    s0 = api.initial_state(vmask, vel * 0.9)          # the step moves the inlet from 0.9 to 1.0 of its peak
    mesh = api.Mesh(flat)
    precision = getattr(api, precision_name)
    states, reports = {}, {}
    for forcing in (0, 1):
        ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG, precision=precision,
                              nonlinear_rtol=1e-10, nonlinear_atol=1e-30, gmres_rtol=1e-10, max_newton=20,
                              gmres_restart=64, newton_forcing=forcing)
        ns.set_dirichlet(vmask, pmask, vel)
        ns.set_tractions({2: 0.0})
        ns.set_state(s0, s0)
        reports[forcing] = ns.step()
        states[forcing] = ns.get_state().reshape(-1, 4)
        ns.close()
    assert reports[0]["converged"] and reports[1]["converged"]
    assert np.array_equal(states[1][vmask != 0, :3], vel[vmask != 0])
    assert rel(states[1][:, :3], states[0][:, :3]) < 1e-8
    assert rel(states[1][:, 3], states[0][:, 3]) < 1e-6
    assert reports[1]["linear_iterations"] < reports[0]["linear_iterations"]


def test_tangent_reuse_step_matches_fixed_tolerance_step(cylinder_1280):
    """Split-BF16 step with forcing and tangent reuse (factor 100): the same solution as the
    fixed-tolerance step within the same tolerances, and no more tensor-core tangent launches than
    the forcing step without reuse."""
    from tubularflowiga_b200 import api
    tube = cylinder_1280
    vmask, pmask, vel = api.tube_boundary_conditions(tube, 0.2)
    s0 = api.initial_state(vmask, vel * 0.9)
    mesh = api.Mesh(tube.mesh)
    states, tangents = {}, {}
    for name, kw in (("fixed", {}), ("forcing", dict(newton_forcing=1)),
                     ("reuse", dict(newton_forcing=1, tangent_reuse_factor=100.0))):
        ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG,
                              precision=api.MIXED_BF16X3, nonlinear_rtol=1e-10, nonlinear_atol=1e-30,
                              gmres_rtol=1e-10, max_newton=30, gmres_restart=64, **kw)
        ns.set_dirichlet(vmask, pmask, vel)
        ns.set_tractions({2: 0.0})
        ns.set_state(s0, s0)
        ns.set_profiling(True)
        ns.profile(reset=True)
        report = ns.step()
        assert report["converged"]
        tangents[name] = ns.profile()["assembly"][1]
        states[name] = ns.get_state().reshape(-1, 4)
        ns.close()
    for name in ("forcing", "reuse"):
        assert rel(states[name][:, :3], states["fixed"][:, :3]) < 1e-8
        assert rel(states[name][:, 3], states["fixed"][:, 3]) < 1e-6
    assert 1 <= tangents["reuse"] <= tangents["forcing"]
