"""Newton convergence diagnostics and the acceptance decision, with the mass test live.

The device computes, for every Newton iteration, the continuity L2 norm and sum of
the raw rhs (after the traction, before the Dirichlet rows), the boundary flow per
face label of the current state, their net and absolute sums and the relative mass
imbalance 2|net|/absolute, and accepts the iterate when
||r|| <= max(atol sqrt(4n), rtol ||r_0||) and the imbalance <= mass_rtol.  These
are checked against the oracle's restatement of the reference's
MeasureFlowConvergence and acceptance test (solvers/cuda/src/iga_cuda.cu:520-557,
989-996), evaluated on the oracle's own FP64 assembly of the same state:
* diagnostics: 1e-12 relative (continuity sum and net flow: 1e-12 of the sum of
  magnitudes, since both are signed sums that can cancel), with an absolute floor of
  1e-20 on the continuity norm and sum for converged states, whose rows cancel;
* the accept / reject decision of every Newton iteration of a step, including
  iterations that the mass test alone rejects (mass_rtol at the default 1e-3 and
  at a value the step-start imbalance exceeds).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

RHO, MU, DT = 1060.0, 3.5e-3, 1e-3
OUTLET_PRESSURE = 17.0


def traction_rhs(flat, label, pressure):
    """-p F_a over the faces of `label` (the oracle's face coefficients)."""
    trac = np.zeros((flat.nodes, 4))
    for e in range(flat.elements):
        conn, C, X, labels = flat.element(e)
        for face, lab in enumerate(labels):
            if lab == label:
                np.add.at(trac, (conn, slice(0, 3)), -pressure * O.face_coefficients(C, X, face))
    return trac.ravel()


def oracle_diagnostics(flat, pattern, state, previous, traction):
    _, rhs = O.assemble(flat, pattern, state, previous, RHO, MU, DT, jacobian=False)
    return O.measure_flow_convergence(flat, state, rhs + traction)


# Absolute floor of the continuity diagnostics: near a converged state the continuity rows are sums of
# element contributions of about 1e-7 that cancel to 1e-12, so the device's and the oracle's summation
# orders differ by a few roundings of those contributions (measured 3.4e-24 at a 1.75e-12 norm).
CONTINUITY_FLOOR = 1e-20


def check_report(report, expect):
    assert abs(report["continuity_l2"] - expect["continuity_l2"]) <= 1e-12 * expect["continuity_l2"] + CONTINUITY_FLOOR
    scale_c = expect["continuity_l2"] * 1e3
    assert abs(report["continuity_sum"] - expect["continuity_sum"]) <= 1e-12 * scale_c + CONTINUITY_FLOOR
    absolute = expect["absolute_boundary_flow"]
    assert abs(report["absolute_boundary_flow"] - absolute) <= 1e-12 * absolute
    assert abs(report["net_boundary_flow"] - expect["net_boundary_flow"]) <= 1e-12 * absolute
    assert abs(report["relative_mass_imbalance"] - expect["relative_mass_imbalance"]) <= 1e-11


@pytest.fixture(scope="module")
def c1(cylinder_1280):
    from tubularflowiga_b200 import api
    flat = cylinder_1280.mesh
    return (api, cylinder_1280, api.Mesh(flat), O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity),
            traction_rhs(flat, 2, OUTLET_PRESSURE))


def test_diagnostics_match_measure_flow_convergence(c1):
    """Three states: the step start (inlet values, interior at rest: imbalance 2), a random state, and
    the state after one Newton update.  The residual test is switched off by a huge atol so that no
    iteration solves, except the one that produces the third state."""
    api, tube, mesh, P, trac = c1
    flat = tube.mesh
    vmask, pmask, vel = api.tube_boundary_conditions(tube, 0.2)
    s0 = api.initial_state(vmask, vel)
    rng = np.random.default_rng(3)
    random = (rng.normal(size=(flat.nodes, 4)) * [0.2, 0.2, 0.2, 20.0]).ravel()
    look = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG,
                            nonlinear_atol=1e300, mass_rtol=1e300)
    look.set_dirichlet(vmask, pmask, vel)
    look.set_tractions({2: OUTLET_PRESSURE})
    solve = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG,
                             nonlinear_rtol=1e-30, nonlinear_atol=1e-300, mass_rtol=1e300, gmres_rtol=1e-10)
    solve.set_dirichlet(vmask, pmask, vel)
    solve.set_tractions({2: OUTLET_PRESSURE})
    solve.set_state(s0, s0)
    solve.newton_iteration(-1.0)
    updated = solve.get_state()
    solve.close()
    for name, state in (("start", s0), ("random", random), ("updated", updated)):
        look.set_state(state, s0)
        report = look.newton_iteration(-1.0)
        assert report["converged"] == 1, name
        expect = oracle_diagnostics(flat, P, state, s0, trac)
        if name == "start":
            assert expect["relative_mass_imbalance"] == pytest.approx(2.0)
        check_report(report, expect)
    look.close()


@pytest.mark.parametrize("mass_rtol", [1e-3, 2.5])
def test_acceptance_decisions_match_the_reference_rule(c1, mass_rtol):
    """Every Newton iteration of a C1 step from rest: the device's accept / reject decision and
    tolerance equal the reference rule applied to the oracle's diagnostics of the same state.  At the
    step start the imbalance is 2: with mass_rtol 1e-3 the mass test rejects every iterate until the
    outflow matches the inflow; with 2.5 it accepts as soon as the residual test holds.  The first
    iteration of each run is also made to pass the residual test (huge initial residual) so that its
    decision is the mass test's alone."""
    api, tube, mesh, P, trac = c1
    flat = tube.mesh
    vmask, pmask, vel = api.tube_boundary_conditions(tube, 0.2)
    s0 = api.initial_state(vmask, vel)
    ns = api.NavierStokes(mesh, density=RHO, viscosity=MU, dt=DT, preconditioner=api.AMG, nonlinear_rtol=1e-8,
                          nonlinear_atol=1e-300, mass_rtol=mass_rtol, gmres_rtol=1e-10, gmres_restart=64)
    ns.set_dirichlet(vmask, pmask, vel)
    ns.set_tractions({2: OUTLET_PRESSURE})
    ns.set_state(s0, s0)
    # iteration 0 with the residual test forced to pass: the decision is the mass test's
    report = ns.newton_iteration(1e300)
    expect = oracle_diagnostics(flat, P, s0, s0, trac)
    accepted, _ = O.newton_accepts(report["residual_l2"], 1e300, 4 * flat.nodes, 1e-300, 1e-8,
                                   expect["relative_mass_imbalance"], mass_rtol)
    assert bool(report["converged"]) == accepted == (mass_rtol > 2.0)
    if accepted:
        return
    # then the genuine iterations of the step, each state checked before the iteration runs
    ns.set_state(s0, s0)
    initial = -1.0
    decisions = []
    for _ in range(12):
        state = ns.get_state()
        report = ns.newton_iteration(initial)
        if initial < 0:
            initial = report["residual_l2"]
        expect = oracle_diagnostics(flat, P, state, s0, trac)
        check_report(report, expect)
        accepted, tolerance = O.newton_accepts(report["residual_l2"], initial, 4 * flat.nodes, 1e-300, 1e-8,
                                               expect["relative_mass_imbalance"], mass_rtol)
        assert abs(report["tolerance"] - tolerance) <= 1e-12 * tolerance
        assert bool(report["converged"]) == accepted
        decisions.append((report["residual_l2"] <= tolerance, expect["relative_mass_imbalance"] <= mass_rtol,
                          accepted))
        if accepted:
            break
    assert decisions[-1][2], decisions
    ns.close()
