"""Two-species transport on the GPU against the oracle (the `iga_cuda transport` path,
solvers/cuda/src/iga_cuda.cu:621-732).

* assembly: both 2x2 block matrices after the boundary rows against the oracle's global
  assembly of the same restated element, FP64, max error <= 1e-12 of the largest entry;
* steps: the block-Jacobi GMRES(50) steps (rtol 1e-8) against an exact sparse LU of the
  oracle's system, relative L2 error <= 1e-6 per field, in FP64 and with the FP32 copy of L
  in the Arnoldi SpMV;
* the backward-Euler decay recurrence of the reference's own CUDA transport test
  (solvers/cuda/tests/test_transport_time_integration.py: c_n = 1/1.1^n for dc/dt = -c,
  dt 0.1, checked there to 1e-5), here to 1e-8 with the GMRES tolerance tightened to 1e-12 (at
  the default 1e-8 the tricubic mass matrix leaves a solution error of about 1e-5);
* the `transport` command: log lines, `node N0 N+` text output and VTK output, equal to the
  API run.
"""
import re
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT
from oracle import oracle as O

pytestmark = pytest.mark.gpu

COMMAND = ROOT / "tubularflowiga_b200" / "lib" / "iga_cuda_b200"

PARAMS = {"diffusion": 1e-5, "vplus": 0.8, "vminus": 0.0, "kplus": 0.5, "kminus": 0.1, "detach_plus": 0.2,
          "detach_minus": 0.0, "dt": 1e-3, "steps": 6, "n0_bc": 1.0, "nplus_bc": 0.25, "nminus_bc": 0.0,
          "artificial_diffusion": 1e-4}


def swirl_velocity(tube):
    """The inlet profile (peak 1 along the axis) plus a small swirl, so that all three components act."""
    v = tube.profile.copy()
    v[:, 0] += -0.1 * tube.points[:, 1] / tube.radius
    v[:, 1] += 0.1 * tube.points[:, 0] / tube.radius
    return v


@pytest.fixture(scope="module")
def setup():
    from tubularflowiga_b200 import api, meshgen
    tube = meshgen.straight_tube(1.5e-3, 6e-3, core=4, ring=1, layers=6)
    mesh = api.Mesh(tube.mesh)
    velocity = swirl_velocity(tube)
    params = api.transport_params(**{k: v for k, v in PARAMS.items()})
    mask, n0, nplus = api.resolve_transport_boundaries(tube.labels, velocity, params)
    pattern = O.Pattern(tube.mesh.nodes, tube.mesh.element_offsets, tube.mesh.connectivity)
    return api, tube, mesh, velocity, params, (mask, n0, nplus), pattern


def test_transport_assembly_matches_oracle(setup):
    api, tube, mesh, velocity, params, (mask, n0, nplus), pattern = setup
    t = api.Transport(mesh, params, velocity, mask, n0, nplus)
    left, previous = t.matrices()
    ro, cols, _ = mesh.pattern()
    assert np.array_equal(ro, pattern.row_offsets) and np.array_equal(cols, pattern.columns)
    ol, op = O.transport_assemble(tube.mesh, pattern, velocity, PARAMS, mask)
    for got, want in ((left, ol), (previous, op)):
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err <= 1e-12, err
    # the initial state carries the boundary values and nothing else
    c0 = t.get_state()
    assert np.array_equal(c0, O.transport_initial(tube.mesh.nodes, mask, n0, nplus))
    info = t.info()
    assert info["assembly_ms"] > 0 and info["steps"] == 0
    t.close()


def test_transport_reference_tube_ragged(reference_tube):
    """The reference-generated mesh (nen in {36, ..., 64}, its own labels and velocity file):
    assembly against the oracle, one step against the direct solve (GMRES tolerance tightened to
    1e-12 so that the step, not the stopping tolerance, is compared)."""
    from tubularflowiga_b200 import api, ntiga
    flat = ntiga.read(reference_tube / "tube-1.ntiga")
    assert len(set(np.diff(flat.element_offsets))) >= 4
    words = (reference_tube / "controlmesh.vtk").read_text().split()
    first = words.index("LOOKUP_TABLE") + 2
    labels = np.array([int(float(w)) for w in words[first:first + flat.nodes]], np.int32)
    velocity = np.loadtxt(reference_tube / "initial_velocityfield.txt").reshape(-1, 3)
    p = dict(PARAMS, dt=0.05, diffusion=1e-3)
    params = api.transport_params(**p, gmres_rtol=1e-12)
    mask, n0, nplus = api.resolve_transport_boundaries(labels, velocity, params)
    assert mask.sum() > 0
    mesh = api.Mesh(flat)
    t = api.Transport(mesh, params, velocity, mask, n0, nplus)
    left, previous = t.matrices()
    pattern = O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity)
    ol, op = O.transport_assemble(flat, pattern, velocity, p, mask)
    for got, want in ((left, ol), (previous, op)):
        assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))
    t.step(1)
    c = O.transport_steps(pattern, ol, op, O.transport_initial(flat.nodes, mask, n0, nplus), mask, n0, nplus, 1)
    got = t.get_state()
    for f in (0, 1):
        assert np.linalg.norm(got[f::2] - c[f::2]) <= 1e-8 * np.linalg.norm(c[f::2])
    t.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32_krylov"])
def test_transport_steps_match_direct_solve(setup, precision):
    """Both arithmetic modes stop on the FP64 true residual, so both meet the same bound."""
    api, tube, mesh, velocity, params, (mask, n0, nplus), pattern = setup
    p = api.transport_params(**PARAMS, precision=api.MIXED if precision == "fp32_krylov" else api.FP64)
    t = api.Transport(mesh, p, velocity, mask, n0, nplus)
    ol, op = O.transport_assemble(tube.mesh, pattern, velocity, PARAMS, mask)
    c = O.transport_initial(tube.mesh.nodes, mask, n0, nplus)
    for step in range(3):
        r = t.step(2)
        c = O.transport_steps(pattern, ol, op, c, mask, n0, nplus, 2)
        got = t.get_state()
        assert r["steps"] == 2 and r["total_iterations"] >= 2 and np.isfinite(r["last_residual"])
        assert abs(r["final_l2"] - np.linalg.norm(got)) <= 1e-12 * np.linalg.norm(got)
        for f in (0, 1):
            err = np.linalg.norm(got[f::2] - c[f::2]) / np.linalg.norm(c[f::2])
            assert err <= 1e-6, (step, f, err)
        # boundary values hold on constrained nodes (to the solver tolerance)
        m = mask != 0
        assert np.allclose(got[0::2][m], n0[m], rtol=1e-6, atol=0)
        assert np.allclose(got[1::2][m], nplus[m], rtol=1e-6, atol=0)
    assert t.info()["steps"] == 6
    t.close()


def test_transport_backward_euler_decay(setup):
    """dN0/dt = -N0 with dt 0.1 and no boundary nodes: N0_n = N0_0 / 1.1^n, N+ unchanged.  Solved to
    rtol 1e-12 so that the recurrence, not the stopping tolerance, is what is checked."""
    api, tube, mesh, *_ = setup
    n = tube.mesh.nodes
    params = api.transport_params(kminus=1.0, dt=0.1, gmres_rtol=1e-12)
    zeros = np.zeros(n)
    t = api.Transport(mesh, params, np.zeros((n, 3)), np.zeros(n, np.int32), zeros, zeros)
    t.set_state(np.ones(2 * n))
    r = t.step(2)
    c = t.get_state()
    assert np.max(np.abs(c[0::2] - 1 / 1.1 ** 2)) < 1e-8 and np.max(np.abs(c[1::2] - 1.0)) < 1e-8
    assert r["singular_blocks"] == 0
    t.close()


def test_transport_rejects_bad_input(setup):
    api, tube, mesh, velocity, params, (mask, n0, nplus), _ = setup
    bad = api.transport_params(**dict(PARAMS, dt=0.0))
    with pytest.raises(api.TfigaError) as err:
        api.Transport(mesh, bad, velocity, mask, n0, nplus)
    assert err.value.status == -1
    t = api.Transport(mesh, params, velocity, mask, n0, nplus)
    with pytest.raises(api.TfigaError):
        t.step(-1)
    t.close()


def run(*args):
    return subprocess.run([str(COMMAND), *map(str, args)], capture_output=True, text=True, timeout=600)


def test_transport_command(setup, tmp_path):
    from tubularflowiga_b200 import meshgen
    api, tube, mesh, velocity, params, (mask, n0, nplus), _ = setup
    db = meshgen.write_transport_case(tmp_path, tube, PARAMS, velocity=velocity)
    out = tmp_path / "result.txt"
    r = run("transport", db, tmp_path, 4, out)
    assert r.returncode == 0, r.stderr
    assert f"boundary_config=legacy-defaults transport_nodes={int(mask.sum())}" in r.stdout
    m = re.search(r"transport_cuda nodes=(\d+) elements=(\d+) steps=4 .* total_iterations=(\d+) "
                  r"final_l2=(\S+) singular_diagonal_blocks=0", r.stdout)
    assert m, r.stdout
    assert int(m.group(1)) == tube.mesh.nodes and int(m.group(2)) == tube.mesh.elements
    assert "transport step=4/4 iterations=" in r.stdout
    rows = [line.split() for line in out.read_text().splitlines()]
    assert len(rows) == tube.mesh.nodes and all(len(x) == 3 and int(x[0]) == i for i, x in enumerate(rows))
    got = np.array([[float(x[1]), float(x[2])] for x in rows]).ravel()
    assert abs(float(m.group(4)) - np.linalg.norm(got)) <= 1e-6 * np.linalg.norm(got)
    vtk = (tmp_path / "result.txt.vtk").read_text()
    assert vtk.startswith((tmp_path / "controlmesh.vtk").read_text())
    assert "SCALARS N0 double 1" in vtk and "SCALARS Nplus double 1" in vtk
    # the same run through the API
    t = api.Transport(mesh, params, velocity, mask, n0, nplus)
    t.step(4)
    want = t.get_state()
    t.close()
    # the assembly's atomic sums make the two runs differ in the last bits, which GMRES carries to the
    # level of its stopping tolerance
    assert np.max(np.abs(got - want)) <= 1e-6 * np.max(np.abs(want))
    # case_config.json overrides the inlet values
    (tmp_path / "case_config.json").write_text(
        '{"boundaries": {"conditions": [{"label": 1, "type": "inlet", "transport": {"N0": 2.0, "Nplus": 0.5}}]}}')
    r = run("transport", db, tmp_path, 1, out)
    assert r.returncode == 0 and "boundary_config=case_config.json" in r.stdout, r.stderr
    rows = np.loadtxt(out)
    inlet = mask != 0
    assert np.allclose(rows[inlet, 1], 2.0, rtol=1e-6) and np.allclose(rows[inlet, 2], 0.5, rtol=1e-6)
    # a missing parameter fails with the reference's message and exit code 1
    (tmp_path / "simulation_parameter.txt").write_text("D 1\n")
    r = run("transport", db, tmp_path)
    assert r.returncode == 1 and "missing transport parameter: vplus" in r.stderr


def test_flow_line_preconditioner_on_the_device(setup):
    """The flow-line preconditioner (TFIGA_TRANSPORT_FLOW_LINES): the device application
    (LineApplyKernel, one thread per line) equals the oracle's tfo_line_apply with the oracle's
    lines and factors of the same L within 1e-12; steps with it match the exact sparse LU of the
    oracle's system as the block-Jacobi steps do (1e-6 per field at rtol 1e-8) in no more GMRES
    iterations."""
    import scipy.sparse.linalg as spla
    api, tube, mesh, velocity, params, (mask, n0, nplus), pattern = setup
    lines_params = api.transport_params(**{k: v for k, v in PARAMS.items()}, preconditioner=api.TRANSPORT_FLOW_LINES)
    t = api.Transport(mesh, lines_params, velocity, mask, n0, nplus)
    left, previous = t.matrices()
    ro, cols, _ = mesh.pattern()
    oracle_lines = O.FlowLines(ro, cols, left)
    rng = np.random.default_rng(21)
    for _ in range(3):
        x = rng.normal(size=2 * tube.mesh.nodes)
        got = t.apply_preconditioner(x)
        want = oracle_lines.apply(x)
        assert np.linalg.norm(got - want) <= 1e-12 * np.linalg.norm(want)
    # steps against the direct solve, and the iteration count against block-Jacobi
    A = O.transport_scipy(pattern, left).tocsc()
    P = O.transport_scipy(pattern, previous)
    c = O.transport_initial(tube.mesh.nodes, mask, n0, nplus)
    constrained = np.nonzero(mask)[0]
    bj = api.Transport(mesh, params, velocity, mask, n0, nplus)
    its = {"lines": 0, "bj": 0}
    for _ in range(4):
        rhs = P @ c
        rhs[2 * constrained] = n0[constrained]
        rhs[2 * constrained + 1] = nplus[constrained]
        c = spla.spsolve(A, rhs)
        its["lines"] += t.step(1)["last_iterations"]
        its["bj"] += bj.step(1)["last_iterations"]
        got = t.get_state()
        for f in (0, 1):
            assert np.linalg.norm(got[f::2] - c[f::2]) <= 1e-6 * np.linalg.norm(c[f::2])
    assert its["lines"] <= its["bj"], its
    t.close()
    bj.close()
