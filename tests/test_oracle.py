"""Pins the CPU oracle (oracle/ns_oracle.c) before anything is checked against it.

* Known-answer checks restated from the reference's element test
  (solvers/cpu/tests/test_navier_stokes.cpp:244-358): FD tangent defect,
  backward-Euler mass sums, the off-centre single-point residual and the
  +-2 boundary flows of the unit element.
* Golden vectors produced by the reference's own element code
  (tests/golden/element_golden.npz, tests/golden/make_element_golden.py).
* Direct element-by-element comparison with the compiled reference
  (oracle/_ref) on the reference-generated tube and on the project's tubes.
"""
import ctypes

import numpy as np
import pytest

from tests.conftest import GOLDEN, requires_ref
from oracle import oracle as O
from tests.golden.make_element_golden import CASES, curved, previous, state, unit_element


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def test_golden_element_vectors():
    golden = np.load(GOLDEN / "element_golden.npz")
    C, X = unit_element()
    for name, (is_curved, rho, mu, dt) in CASES.items():
        XX = curved(X) if is_curved else X
        negres, jac = O.ns_element(C, XX, state(), previous() if dt > 0 else None, rho, mu, dt)
        assert rel(negres, golden[name + "_negres"]) < 1e-13, name
        assert rel(jac[::16], golden[name + "_jac_rows"]) < 1e-13, name


def test_fd_tangent_defect():
    # test_navier_stokes.cpp:244-271: central FD of -r along a fixed direction.
    C, X = unit_element()
    st, pv = state(), previous()
    direction = np.array([[1e-3 * (1.0 + ((7 * a + 3 * f) % 13)) for f in range(4)] for a in range(64)])
    eps = 1e-4
    _, jac = O.ns_element(C, X, st, pv, 2.5, 0.17, 0.2)
    rp, _ = O.ns_element(C, X, st + eps * direction, pv, 2.5, 0.17, 0.2, jacobian=False)
    rm, _ = O.ns_element(C, X, st - eps * direction, pv, 2.5, 0.17, 0.2, jacobian=False)
    action = jac @ direction.ravel()
    defect = action + (rp - rm) / (2 * eps)
    assert np.linalg.norm(defect) / np.linalg.norm(action) <= 1e-8


def test_backward_euler_mass_sums():
    # test_navier_stokes.cpp:311-332.
    C, X = unit_element()
    rho, dt = 2.5, 0.2
    cur, prv = np.array([1.0, -0.5, 0.25]), np.array([0.6, -0.1, 0.05])
    st = np.tile(np.r_[cur, 0.0], (64, 1))
    pv = np.tile(np.r_[prv, 0.0], (64, 1))
    negres, jac = O.ns_element(C, X, st, pv, rho, 0.17, dt)
    for c in range(3):
        assert abs(negres[c::4].sum() - (-rho * (cur[c] - prv[c]) / dt)) < 2e-11
        assert abs(jac[c::4, c::4].sum() - rho / dt) < 2e-11
    _, reduced = O.ns_element(C, X, st, pv, rho, 0.17, dt, points=np.array([[0.5, 0.5, 0.5]]),
                              weights=np.array([0.25]))
    assert abs(reduced[0::4, 0::4].sum() - 0.25 * rho / dt) < 2e-11


def test_off_centre_single_point_residual():
    # test_navier_stokes.cpp:333-356.
    C, X = unit_element()
    rho, dt, vel = 2.5, 0.2, 0.15
    pt = np.array([0.23, 0.61, 0.37])
    N, dN, H, inv, det = O.basis(C, X, *pt)
    # tau_m from the restated Stabilization at this point.
    G = inv.T @ inv
    g = inv.sum(axis=0)
    nu = 0.17 / rho
    tau_m = 1.0 / np.sqrt(4.0 / dt ** 2 + vel * G[0, 0] * vel + nu * nu * (G * G).sum() / 12.0)
    deriv = vel / tau_m
    st = np.tile([vel, 0.0, 0.0, 0.0], (64, 1))
    pv = np.tile([vel - dt * deriv, 0.0, 0.0, 0.0], (64, 1))
    negres, _ = O.ns_element(C, X, st, pv, rho, 0.17, dt, jacobian=False, points=pt[None, :],
                             weights=np.array([0.41]))
    expected = -rho * N * deriv * 0.41 * det
    assert np.abs(negres[0::4] - expected).max() < 2e-13
    assert g.shape == (3,)


def test_unit_boundary_flow():
    # test_navier_stokes.cpp:357-358.
    C, X = unit_element()
    st = np.tile([2.0, 0.0, 0.0, 0.0], (64, 1))
    assert abs(O.boundary_flow(C, X, 2, st) - 2.0) < 2e-13
    assert abs(O.boundary_flow(C, X, 4, st) + 2.0) < 2e-13


def test_outlet_and_waveform_closed_forms():
    # RCR closed form (OutletModel.hpp:70-90) and a Fourier waveform (TemporalFunction.hpp:97-112).
    R1, Cc, R2, dt, q, pc0 = 1e8, 1e-10, 1e9, 2e-3, 1e-6, 10.0
    p, pc = O.outlet_model(2, 0.0, R1, R2, Cc, 0.0, pc0, q, dt)
    pc_exp = (Cc * pc0 / dt + q) / (Cc / dt + 1.0 / R2)
    assert abs(pc - pc_exp) <= 1e-14 * abs(pc_exp) and abs(p - (pc_exp + R1 * q)) <= 1e-14 * abs(p)
    p, _ = O.outlet_model(0, 5.0, 0, 0, 0, 3.0, 0.0, 2.0, 0.0)
    assert p == 13.0
    v = O.temporal(2, mean=0.15, period=1.0, cosine=[0.01, 0.02], sine=[0.03, 0.0], time=1.25)
    th = 2 * np.pi * 0.25
    assert abs(v - (0.15 + 0.01 * np.cos(th) + 0.02 * np.cos(2 * th) + 0.03 * np.sin(th))) < 1e-15


@requires_ref
def test_restatement_matches_reference_build(reference_tube):
    """Element-by-element against the reference's own compiled element code (ragged nen)."""
    from tubularflowiga_b200 import ntiga
    mesh = ntiga.read(reference_tube / "tube-1.ntiga")
    rng = np.random.default_rng(0)
    nens = set()
    for e in rng.choice(mesh.elements, 24, replace=False):
        conn, C, X, _ = mesh.element(int(e))
        nen = len(conn)
        nens.add(nen)
        st = rng.normal(size=(nen, 4)) * [0.3, 0.3, 0.3, 1.0]
        pv = rng.normal(size=(nen, 4)) * 0.3
        a = O.ns_element(C, X, st, pv, 1.0, 1.0, 0.1)
        b = O.ns_element(C, X, st, pv, 1.0, 1.0, 0.1, use_ref=True)
        assert rel(a[0], b[0]) < 1e-12 and rel(a[1], b[1]) < 1e-12
        for face in range(6):
            assert abs(O.boundary_flow(C, X, face, st) - O.boundary_flow(C, X, face, st, use_ref=True)) \
                <= 1e-13 * max(1.0, abs(O.boundary_flow(C, X, face, st, use_ref=True)))
    assert len(nens) >= 3, nens


@requires_ref
def test_generator_database_reads_through_reference(tmp_path, small_tube):
    from tubularflowiga_b200 import meshgen
    db = meshgen.write_case(tmp_path, small_tube, meshgen.simulation_config(1060, 3.5e-3, 1e-3, 2, 0.2))
    R = O.ref()
    header = np.zeros(4, np.uint64)
    assert R.ref_ntiga_header(str(db).encode(), header) == 0
    assert list(header) == [5, 1, small_tube.mesh.elements, small_tube.mesh.nodes]
    for e in (0, small_tube.mesh.elements // 2, small_tube.mesh.elements - 1):
        nen = ctypes.c_int()
        lab = np.zeros(6, np.int32); conn = np.zeros(80, np.int32)
        ext = np.zeros(80 * 64); bz = np.zeros(192)
        assert R.ref_ntiga_element(str(db).encode(), e, ctypes.byref(nen), lab, conn, ext, bz) == 0
        c, Cx, X, lb = small_tube.mesh.element(e)
        assert np.array_equal(conn[:nen.value], c) and np.array_equal(ext[:64 * nen.value].reshape(-1, 64), Cx)
        assert np.array_equal(bz, X.ravel()) and np.array_equal(lab, lb)
    out = np.zeros(small_tube.mesh.nodes, np.int32)
    count = R.ref_wall_trace(str(db).encode(), str(tmp_path / "controlmesh.vtk").encode(), out, len(out))
    assert np.array_equal(np.sort(out[:count]), np.nonzero(small_tube.labels == 0)[0])


def test_generator_geometry(small_tube):
    m = small_tube.mesh
    bad = ctypes.c_int()
    for e in range(m.elements):
        _, C, X, _ = m.element(e)
        assert np.abs(C.sum(axis=0) - 1.0).max() < 1e-12      # partition of unity
        assert O.lib().tfo_min_determinant(np.ascontiguousarray(X.ravel()), ctypes.byref(bad)) > 0
        assert bad.value == 0
    assert small_tube.per_plane == 41 and m.elements == 32 * 3


def test_pattern_and_oracle_gmres(small_tube):
    m = small_tube.mesh
    P = O.Pattern(m.nodes, m.element_offsets, m.connectivity)
    rng = np.random.default_rng(1)
    st = rng.normal(size=(m.nodes, 4)) * 0.01
    values, rhs = O.assemble(m, P, st, st, 1060.0, 3.5e-3, 1e-3)
    vmask = (small_tube.labels >= 0) & (small_tube.labels <= 1)
    O.apply_dirichlet(P, vmask.astype(np.int32), np.zeros(m.nodes, np.int32), np.zeros(3 * m.nodes),
                      np.zeros(m.nodes), st, values, rhs)
    A = P.to_scipy(values)
    x, it, res, singular = O.gmres_bjacobi(P, values, rhs, rtol=1e-10)
    assert it > 0 and singular == 0
    assert np.linalg.norm(A @ x - rhs) <= 1e-7 * np.linalg.norm(rhs)
    assert np.allclose(O.spmv(P, values, x), A @ x, rtol=1e-13, atol=1e-20)


def test_ntiga_writer_reproduces_the_reference_pack_byte_for_byte(reference_tube, tmp_path):
    """The generator's .ntiga writer, given the content of the database the reference's own
    iga_pack wrote (tests/golden/reference_tube, solvers/cpu/src/iga_pack.cpp:278-417), writes
    the same bytes: header, ownership and rank indices, element records and their order."""
    from tubularflowiga_b200 import ntiga
    source = (reference_tube / "tube-1.ntiga").read_bytes()
    mesh = ntiga.read(reference_tube / "tube-1.ntiga")
    ntiga.write(tmp_path / "copy.ntiga", mesh)
    assert (tmp_path / "copy.ntiga").read_bytes() == source


@requires_ref
def test_vtu_snapshot_matches_the_reference_writer_byte_for_byte(tmp_path, small_tube, reference_tube):
    """tfiga_write_vtu (the navier-stokes command's VTU snapshots) against the reference's own WriteVtu
    with the arrays of WriteNavierStokesVtu: identical files, on a generated control mesh and on the
    reference-generated one."""
    from tubularflowiga_b200 import api, build, meshgen
    build.build()
    meshgen.write_vtk(tmp_path / "controlmesh.vtk", small_tube)
    rng = np.random.default_rng(4)
    for k, (mesh_vtk, nodes) in enumerate(((tmp_path / "controlmesh.vtk", small_tube.mesh.nodes),
                                           (reference_tube / "controlmesh.vtk", 725))):
        state = rng.normal(size=4 * nodes) * np.array([0.3, 0.3, 0.3, 40.0] * nodes)
        ours, theirs = tmp_path / f"ours{k}.vtu", tmp_path / f"ref{k}.vtu"
        api.check(api.lib().tfiga_write_vtu(str(mesh_vtk).encode(), str(ours).encode(),
                                            state.ctypes.data_as(ctypes.c_void_p), nodes, 0.125 * (k + 1)))
        assert O.ref().ref_write_vtu(str(mesh_vtk).encode(), str(theirs).encode(), state, nodes,
                                     0.125 * (k + 1)) == 0
        assert ours.read_bytes() == theirs.read_bytes()


@requires_ref
def test_flow_checkpoint_matches_the_reference_format(tmp_path):
    """tfiga_write_flow_checkpoint writes the metadata and state bytes the reference's own
    WriteFlowCheckpointMetadata + raw state write produce; each side restarts from the other's files
    (the reference through ReadFlowCheckpointMetadata + ValidateFlowCheckpoint)."""
    from tubularflowiga_b200 import api, build
    build.build()
    rng = np.random.default_rng(8)
    nodes = 57
    state = rng.normal(size=4 * nodes)
    outlets = (api.Outlet * 2)(api.Outlet.rcr(2, 1e8, 1e-10, 1e9), api.Outlet.resistance_model(3, 2e7, 5.0))
    outlets[0].flow, outlets[0].pressure, outlets[0].capacitor_pressure = 1.25e-6, 143.9, 74.2
    outlets[1].flow, outlets[1].pressure, outlets[1].capacitor_pressure = -3.5e-7, 12.5, 0.0
    args = (nodes, 7, 7 * 2e-3, 2e-3, 1060.0, 3.5e-3)
    ours, theirs = tmp_path / "ours", tmp_path / "theirs"
    api.check(api.lib().tfiga_write_flow_checkpoint(str(ours).encode(), *args, outlets, 2,
                                                    state.ctypes.data_as(ctypes.c_void_p)))
    ints = np.array([2, 2, 3, 0], np.int32)
    vals = np.array([1.25e-6, 143.9, 74.2, -3.5e-7, 12.5, 0.0])
    assert O.ref().ref_write_flow_checkpoint(str(theirs).encode(), *args, ints, vals, 2, state) == 0
    assert (tmp_path / "ours.json").read_text() == (tmp_path / "theirs.json").read_text().replace("theirs.state",
                                                                                                 "ours.state")
    assert (tmp_path / "ours.state").read_bytes() == (tmp_path / "theirs.state").read_bytes()
    # the reference restarts from our files
    back = np.zeros(4 * nodes)
    completed, time, count = ctypes.c_int(), ctypes.c_double(), ctypes.c_int(4)
    labels, values = np.zeros(4, np.int32), np.zeros(12)
    assert O.ref().ref_read_flow_checkpoint(str(ours).encode(), nodes, 10, 2e-3, 1060.0, 3.5e-3, back,
                                            ctypes.byref(completed), ctypes.byref(time), labels, values,
                                            ctypes.byref(count)) == 0
    assert np.array_equal(back, state) and completed.value == 7 and count.value == 2
    assert list(labels[:2]) == [2, 3] and np.array_equal(values[:6], vals)
    # we restart from the reference's files
    fresh = (api.Outlet * 2)(api.Outlet.rcr(2, 1e8, 1e-10, 1e9), api.Outlet.resistance_model(3, 2e7, 5.0))
    back2 = np.zeros(4 * nodes)
    step, t = ctypes.c_int32(), ctypes.c_double()
    api.check(api.lib().tfiga_read_flow_checkpoint(str(theirs).encode(), nodes, 2e-3, 1060.0, 3.5e-3, fresh, 2,
                                                   back2.ctypes.data_as(ctypes.c_void_p), ctypes.byref(step),
                                                   ctypes.byref(t)))
    assert np.array_equal(back2, state) and step.value == 7 and t.value == 7 * 2e-3
    assert (fresh[0].flow, fresh[0].pressure, fresh[0].capacitor_pressure) == (1.25e-6, 143.9, 74.2)
    # a mismatched configuration is refused by both
    assert api.lib().tfiga_read_flow_checkpoint(str(theirs).encode(), nodes, 1e-3, 1060.0, 3.5e-3, fresh, 2,
                                                back2.ctypes.data_as(ctypes.c_void_p), None, None) == -4
    assert O.ref().ref_read_flow_checkpoint(str(ours).encode(), nodes, 10, 1e-3, 1060.0, 3.5e-3, back,
                                            ctypes.byref(completed), ctypes.byref(time), labels, values,
                                            ctypes.byref(count)) == -1


@requires_ref
def test_wall_trace_and_ntiga_reader_match_the_reference(tmp_path, small_tube, reference_tube):
    """The command's no-slip basis set from this library's .ntiga reader (tfiga_wall_trace_basis)
    equals the reference's own WallTraceBasis over its own Database, on a generated case and on the
    reference-generated tube."""
    from tubularflowiga_b200 import api, build, meshgen
    build.build()
    db = meshgen.write_case(tmp_path, small_tube, meshgen.simulation_config(1060, 3.5e-3, 1e-3, 2, 0.2))
    for database, vtk, nodes in ((db, tmp_path / "controlmesh.vtk", small_tube.mesh.nodes),
                                 (reference_tube / "tube-1.ntiga", reference_tube / "controlmesh.vtk", 725)):
        want = np.zeros(nodes, np.int32)
        n_ref = O.ref().ref_wall_trace(str(database).encode(), str(vtk).encode(), want, nodes)
        got = np.zeros(nodes, np.int32)
        count = ctypes.c_int64()
        api.check(api.lib().tfiga_wall_trace_basis(str(database).encode(), str(vtk).encode(),
                                                   got.ctypes.data_as(ctypes.c_void_p), nodes, ctypes.byref(count)))
        assert count.value == n_ref > 0
        assert np.array_equal(got[:count.value], np.sort(want[:n_ref]))


def test_womersley_restatement_known_answers():
    """The reference's own known answers for its Womersley solution
    (solvers/cpu/tests/test_womersley_reference.cpp:8-57), on the oracle's restatement."""
    import scipy.special as sp
    # the reference sums in long double (1e-14 there); in double the alternating series at |z| = 10
    # cancels terms of size 1e3, so 1e-13 here
    for value in (1.0, 5.0, 10.0):
        assert abs(O.complex_bessel_j0(complex(value, 0.0)).real - sp.j0(value)) < 1e-13
    moderate = O.complex_bessel_j0(complex(10.0, -10.0))
    assert abs(moderate - complex(-2314.9753144452134, -411.5628570253805)) / abs(moderate) < 1e-13
    args = dict(radius=1.0, density=1.0, viscosity=1.0, period=2.0, mean_gradient=4.0, cosine=[2.0], sine=[])
    assert abs(O.womersley_axial_velocity(r=1.0, t=0.25, **args)) < 1e-14
    assert abs(O.womersley_axial_velocity(r=0.4, t=0.25, **args) - O.womersley_axial_velocity(r=0.4, t=2.25, **args)) \
        < 1e-13
    steady = dict(args, cosine=[], sine=[])
    assert abs(O.womersley_axial_velocity(r=0.5, t=17.0, **steady) - 0.75) < 1e-15
    quasi = dict(args, mean_gradient=0.0, period=1e7)
    assert abs(O.womersley_axial_velocity(r=0.0, t=0.0, **quasi) - 0.5) < 1e-7


@requires_ref
def test_womersley_restatement_matches_reference_build():
    """The restatement against the reference's compiled WomersleyAxialVelocity on the pulsatile test's
    pipe (R 1.5 mm, blood, 1 Hz, a mean and four harmonics): 1e-12 relative over radii and times."""
    rng = np.random.default_rng(1)
    g0 = 1866.7
    cosine, sine = rng.uniform(0, 600, 4), rng.uniform(0, 600, 4)
    for r in np.linspace(0.0, 1.5e-3, 7):
        for t in (0.0, 0.13, 0.5, 0.77):
            a = O.womersley_axial_velocity(1.5e-3, 1060.0, 3.5e-3, 1.0, g0, cosine, sine, r, t)
            b = O.womersley_axial_velocity(1.5e-3, 1060.0, 3.5e-3, 1.0, g0, cosine, sine, r, t, use_ref=True)
            assert abs(a - b) <= 1e-12 * max(abs(b), 1e-3)


@requires_ref
def test_flow_convergence_restatement_uses_the_reference_flow_integrals(small_tube):
    """measure_flow_convergence: per-label flows with the restated face integral equal those with the
    reference's compiled IntegrateBoundaryFlow; the imbalance of a state carrying only the inlet
    profile is 2; continuity norms are those of field 3 of the raw rhs."""
    flat = small_tube.mesh
    rng = np.random.default_rng(5)
    st = rng.normal(size=4 * flat.nodes)
    raw = rng.normal(size=4 * flat.nodes)
    a = O.measure_flow_convergence(flat, st, raw)
    b = O.measure_flow_convergence(flat, st, raw, use_ref=True)
    assert a["boundary_flow"].keys() == b["boundary_flow"].keys() == {0, 1, 2}
    for k in a["boundary_flow"]:
        assert abs(a["boundary_flow"][k] - b["boundary_flow"][k]) <= 1e-12 * b["absolute_boundary_flow"]
    assert a["continuity_l2"] == pytest.approx(np.linalg.norm(raw[3::4]), rel=1e-14)
    inlet_only = np.zeros((flat.nodes, 4))
    inlet_only[small_tube.labels == 1, :3] = small_tube.profile[small_tube.labels == 1]
    c = O.measure_flow_convergence(flat, inlet_only.ravel(), raw)
    assert c["relative_mass_imbalance"] == pytest.approx(2.0, rel=1e-14)
    assert O.newton_accepts(1.0, 1e9, 4 * flat.nodes, 1e-300, 1e-8, c["relative_mass_imbalance"], 1e-3)[0] is False
    assert O.newton_accepts(1.0, 1e9, 4 * flat.nodes, 1e-300, 1e-8, c["relative_mass_imbalance"], 2.5)[0] is True
