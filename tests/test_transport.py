"""Two-species transport on the CPU: the oracle's transport element against the
reference's own element (golden vectors and, where the reference build exists,
element by element), closed-form identities of the element, and the host-side
case inputs of the `transport` command through the C ABI (no GPU needed).

Reference: BuildTransportElement (solvers/cpu/include/TransportElement.hpp:213-253),
ReadTransportParameters and ResolveBoundaryConditions
(solvers/cpu/include/CaseInput.hpp:85-118, 162-258), ParseCaseConfiguration
(include/CaseConfig.hpp:280-387).
"""
import ctypes
import json
import subprocess

import numpy as np
import pytest

from tests.conftest import GOLDEN, ROOT, requires_ref
from oracle import oracle as O
from tests.golden.make_element_golden import curved, unit_element
from tests.golden.make_transport_golden import PARAMS, cases


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def test_transport_golden_element_vectors():
    g = np.load(GOLDEN / "transport_golden.npz")
    for key, C, X, vel, p in cases():
        left, previous = O.transport_element(C, X, vel, p)
        assert rel(left, g[f"{key}_left"]) < 1e-13, key
        assert rel(previous, g[f"{key}_previous"]) < 1e-13, key


@requires_ref
def test_transport_restatement_matches_reference_build(reference_tube):
    """Element by element against the reference's compiled element (ragged nen, random velocity)."""
    from tubularflowiga_b200 import ntiga
    mesh = ntiga.read(reference_tube / "tube-1.ntiga")
    rng = np.random.default_rng(3)
    nens = set()
    for e in rng.choice(mesh.elements, 16, replace=False):
        conn, C, X, _ = mesh.element(int(e))
        nens.add(len(conn))
        vel = rng.normal(size=(len(conn), 3))
        for p in PARAMS.values():
            a = O.transport_element(C, X, vel, p)
            b = O.transport_element(C, X, vel, p, use_ref=True)
            assert rel(a[0], b[0]) < 1e-12 and rel(a[1], b[1]) < 1e-12
    assert len(nens) >= 3, nens


def test_transport_element_identities():
    """Partition of unity and the zero-velocity form of the blocks."""
    C, X = unit_element()
    X = curved(X)
    p = dict(PARAMS["reaction"])
    left, previous = O.transport_element(C, X, np.zeros((64, 3)), p)
    M = previous[0::2, 0::2]
    # sum_b M_ab = int N_a, sum_ab M_ab = volume (= sum of w over the rule)
    volume = M.sum()
    qp, qw = O.gauss_rule()
    dets = [O.basis(C, X, *qp[q], hessian=False)[4] for q in range(64)]
    assert abs(volume - float(np.dot(qw, dets))) < 1e-15
    assert np.allclose(previous[1::2, 1::2], M, rtol=0, atol=1e-18)     # T = N without velocity
    assert np.all(previous[0::2, 1::2] == 0) and np.all(previous[1::2, 0::2] == 0)
    dt, kp, km, det = p["dt"], p["kplus"], p["kminus"], p["detach_plus"]
    assert np.allclose(left[0::2, 1::2], -det * dt * M, rtol=1e-13, atol=1e-20)
    assert np.allclose(left[1::2, 0::2], -kp * dt * M, rtol=1e-13, atol=1e-20)
    K = (left[0::2, 0::2] - (1 + dt * (kp + km)) * M) / (dt * p["diffusion"])
    assert np.allclose(K.sum(axis=1), 0.0, atol=1e-12 * np.abs(K).max())   # stiffness annihilates constants
    assert np.allclose(K, K.T, atol=1e-12 * np.abs(K).max())


# ---- host-side case inputs through the C ABI ------------------------------------------------

@pytest.fixture(scope="module")
def api():
    from tubularflowiga_b200 import api, build
    build.build()
    return api


def test_read_transport_params(api, tmp_path):
    from tubularflowiga_b200 import meshgen
    want = {"diffusion": 1e-5, "vplus": 0.8, "vminus": 0.3, "kplus": 0.5, "kminus": 0.1, "detach_plus": 0.2,
            "detach_minus": 0.05, "dt": 1e-3, "steps": 7, "n0_bc": 1.0, "nplus_bc": 0.25, "nminus_bc": 0.5,
            "artificial_diffusion": 1e-4}
    path = tmp_path / "simulation_parameter.txt"
    path.write_text(meshgen.transport_parameter_text(want))
    got = api.read_transport_params(path).as_dict()
    for k, v in want.items():
        assert got[k] == v, k
    assert (got["restart"], got["gmres_rtol"], got["gmres_max_iterations"]) == (50, 1e-8, 10000)
    # artificial_diffusion is optional and may be spelled artificial_diffusion_weight
    path.write_text(path.read_text().replace("artificial_diffusion", "artificial_diffusion_weight"))
    assert api.read_transport_params(path).artificial_diffusion == 1e-4
    path.write_text("\n".join(l for l in path.read_text().splitlines() if not l.startswith("artificial")))
    assert api.read_transport_params(path).artificial_diffusion == 0.0
    path.write_text(path.read_text().replace("D 1", "X 1"))
    with pytest.raises(api.TfigaError) as err:
        api.read_transport_params(path)
    assert err.value.status == -4 and "missing transport parameter: D" in str(err.value)
    path.write_text(meshgen.transport_parameter_text(dict(want, dt=0.0)))
    with pytest.raises(api.TfigaError, match="dt and nstep must be positive"):
        api.read_transport_params(path)
    with pytest.raises(api.TfigaError) as err:
        api.read_transport_params(tmp_path / "missing.txt")
    assert err.value.status == -3


def test_resolve_transport_boundaries(api, tmp_path, small_tube):
    """Legacy labels, then case_config.json rules (inlet transport values, inherit_legacy false)."""
    t = small_tube
    p = api.transport_params(vplus=0.8, n0_bc=1.5, nplus_bc=0.25)
    mask, n0, nplus = api.resolve_transport_boundaries(t.labels, t.profile, p)
    inlet = t.labels == 1
    assert np.array_equal(mask, inlet.astype(np.int32))
    assert np.all(n0[inlet] == 1.5) and np.all(nplus[inlet] == 0.25)
    assert np.all(n0[~inlet] == 0) and np.all(nplus[~inlet] == 0)
    # an absent case_config.json is the legacy default
    same = api.resolve_transport_boundaries(t.labels, t.profile, p, tmp_path / "case_config.json")
    assert all(np.array_equal(a, b) for a, b in zip(same, (mask, n0, nplus)))

    cfg = tmp_path / "case_config.json"
    cfg.write_text(json.dumps({"schema_version": 1, "boundaries": {"conditions": [
        {"label": 1, "type": "inlet", "transport": {"N0": 2.0, "Nplus": 0.75}}]}}))
    mask2, n02, nplus2 = api.resolve_transport_boundaries(t.labels, t.profile, p, cfg)
    assert np.array_equal(mask2, mask) and np.all(n02[inlet] == 2.0) and np.all(nplus2[inlet] == 0.75)
    # the outlet label as an inlet adds its nodes to the constrained set
    cfg.write_text(json.dumps({"boundaries": {"inherit_legacy": True, "conditions": [
        {"label": 2, "type": "inlet"}]}}))
    with pytest.raises(api.TfigaError, match="no pressure boundary nodes"):
        api.resolve_transport_boundaries(t.labels, t.profile, p, cfg)
    cfg.write_text(json.dumps({"boundaries": {"inherit_legacy": False, "conditions": [
        {"label": 1, "type": "inlet"}, {"label": 2, "type": "outlet"}]}}))
    with pytest.raises(api.TfigaError, match="mesh boundary label 0 has no case_config.json rule"):
        api.resolve_transport_boundaries(t.labels, t.profile, p, cfg)
    for bad, message in (
            ({"boundaries": {"conditions": [{"label": 7, "type": "wall"}]}}, "label 7 is not present"),
            ({"boundaries": {"conditions": [{"label": 1, "type": "inlet", "colour": 1}]}}, "unknown"),
            ({"boundaries": {"conditions": [{"label": 1, "type": "inlet"}, {"label": 1, "type": "inlet"}]}},
             "duplicate boundary label 1"),
            ({"schema_version": 2, "boundaries": {"conditions": []}}, "only schema_version 1"),
            ({"boundaries": {"conditions": [{"label": 2, "type": "outlet", "transport": {"N0": 1, "Nplus": 1}}]}},
             "outlet rules only support an optional pressure"),
            ({"boundaries": {"conditions": [{"label": 1, "type": "inlet", "transport": {"N0": 1}}]}},
             "requires N0 and Nplus")):
        cfg.write_text(json.dumps(bad))
        with pytest.raises(api.TfigaError, match=message) as err:
            api.resolve_transport_boundaries(t.labels, t.profile, p, cfg)
        assert err.value.status == -4


STRUCTS = {"tfiga_mesh_desc": "MeshDesc", "tfiga_mesh_info": "MeshInfo", "tfiga_ns_params": "NsParams",
           "tfiga_amg_info": "AmgInfo", "tfiga_newton_report": "NewtonReport", "tfiga_step_report": "StepReport",
           "tfiga_outlet": "Outlet", "tfiga_transport_params": "TransportParams",
           "tfiga_transport_report": "TransportReport"}


def test_struct_layouts_match_the_header(api, tmp_path):
    """sizeof and every field offset of the header's structs, compiled with gcc, equal the ctypes mirror."""
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tfiga.h"', 'int main(void) {']
    for c_name, py_name in STRUCTS.items():
        lines.append(f'printf("{c_name} %zu\\n", sizeof({c_name}));')
        for field, _ in getattr(api, py_name)._fields_:
            lines.append(f'printf("{c_name}.{field} %zu\\n", offsetof({c_name}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for c_name, py_name in STRUCTS.items():
        cls = getattr(api, py_name)
        assert int(got[c_name]) == ctypes.sizeof(cls), c_name
        for field, _ in cls._fields_:
            assert int(got[f"{c_name}.{field}"]) == getattr(cls, field).offset, (c_name, field)


def test_transport_oracle_gmres_matches_direct_solve(small_tube):
    """The CPU restatement of the transport step's block-Jacobi GMRES(50) (the bench's CPU baseline)
    reaches the sparse-LU solution of the oracle's assembled system."""
    t = small_tube
    params = {"diffusion": 1e-5, "vplus": 0.8, "kplus": 0.5, "kminus": 0.1, "detach_plus": 0.2, "dt": 1e-3,
              "artificial_diffusion": 1e-4}
    velocity = t.profile + 0.05
    pattern = O.Pattern(t.mesh.nodes, t.mesh.element_offsets, t.mesh.connectivity)
    mask = (t.labels == 1).astype(np.int32)
    n0, nplus = mask * 1.0, mask * 0.25
    left, previous = O.transport_assemble(t.mesh, pattern, velocity, params, mask)
    c0 = O.transport_initial(t.mesh.nodes, mask, n0, nplus)
    want = O.transport_steps(pattern, left, previous, c0, mask, n0, nplus, 1)
    rhs = O.transport_spmv(pattern.row_offsets, pattern.columns, previous, c0)
    rhs[0::2][mask != 0] = n0[mask != 0]
    rhs[1::2][mask != 0] = nplus[mask != 0]
    x, iterations, residual = O.transport_gmres(pattern.row_offsets, pattern.columns, pattern.diagonal, left, rhs,
                                                np.zeros_like(rhs))
    assert iterations > 0
    for f in (0, 1):
        assert np.linalg.norm(x[f::2] - want[f::2]) <= 1e-6 * np.linalg.norm(want[f::2])


@requires_ref
def test_legacy_boundaries_match_the_reference_resolver(api, tmp_path, small_tube):
    """Every mask and value of a legacy case against the reference's own ParseCaseConfiguration +
    ResolveBoundaryConditions (compiled unmodified into oracle/_ref), for the legacy defaults and a
    set of case_config.json rule sets, including the ones the reference rejects (same message)."""
    t = small_tube
    rng = np.random.default_rng(5)
    velocity = rng.normal(size=(t.mesh.nodes, 3))
    p = api.transport_params(vplus=0.7, n0_bc=1.25, nplus_bc=0.375)
    configs = [None,
               {"boundaries": {"conditions": [{"label": 1, "type": "inlet", "transport": {"N0": 2.0, "Nplus": 0.5}}]}},
               {"boundaries": {"conditions": [{"label": 1, "type": "inlet", "velocity_scale": 3.0}]}},
               {"boundaries": {"conditions": [{"label": 1, "type": "inlet", "velocity": [0.1, 0.2, 0.3]},
                                              {"label": 0, "type": "wall", "velocity": [0.0, 0.0, 0.05]},
                                              {"label": 2, "type": "outlet", "pressure": 7.5}]}},
               {"schema_version": 1, "boundaries": {"inherit_legacy": False, "conditions": [
                   {"label": 0, "type": "wall"}, {"label": 1, "type": "inlet"}, {"label": 2, "type": "outlet"}]}},
               {"boundaries": {"conditions": [{"label": 2, "type": "interior"}]}},
               {"boundaries": {"inherit_legacy": False, "conditions": [{"label": 1, "type": "inlet"}]}},
               {"boundaries": {"conditions": [{"label": 9, "type": "wall"}]}},
               {"boundaries": {"conditions": [{"label": 1, "type": "inlet", "velocity": [1, 2, 3],
                                               "velocity_scale": 2.0}]}}]
    keys = ("velocity_mask", "velocity", "pressure_mask", "pressure", "transport_mask", "n0", "nplus", "counts")
    for cfg in configs:
        path = None
        if cfg is not None:
            path = tmp_path / "case_config.json"
            path.write_text(json.dumps(cfg))
        try:
            want = O.ref_resolve_boundaries(t.labels, velocity, 0.7, 1.25, 0.375,
                                            None if cfg is None else json.dumps(cfg))
        except RuntimeError as ref_error:
            with pytest.raises(api.TfigaError) as err:
                api.resolve_legacy_boundaries(t.labels, velocity, p, path)
            assert str(ref_error) in str(err.value), (cfg, str(ref_error), str(err.value))
            continue
        got = api.resolve_legacy_boundaries(t.labels, velocity, p, path)
        for k in keys:
            assert np.array_equal(got[k], want[k]), (cfg, k)


@requires_ref
def test_flow_boundaries_match_the_reference_set_up(api, tmp_path, small_tube):
    """The navier-stokes command's boundary set-up of simulation_config.json cases (schema 4:
    steady and transient, Fourier and sinusoid waveforms at several times, zero-traction, resistance,
    RC and RCR outlets, wall velocity) against the reference's own compiled ReadSimulationConfiguration
    ... ResolveFlowBoundaries chain (iga_cuda.cu:766-790): every mask, value, traction and the physics."""
    from tubularflowiga_b200 import meshgen
    t = small_tube
    rng = np.random.default_rng(9)
    velocity = t.profile + 0.1 * rng.normal(size=t.profile.shape)
    wave = meshgen.fourier_waveform(3)
    sine = {"name": "inflow", "kind": "sinusoid", "units": "m/s", "mean": 0.2, "amplitude": 0.05, "period": 0.8,
            "phase": 0.3}
    outlet = lambda cond: [{"label": 2, "name": "outlet", "conditions": [dict(field="pressure", **cond)]}]
    cases = [
        meshgen.simulation_config(1060.0, 3.5e-3, 2e-3, 3, 0.7, transient=False),
        meshgen.simulation_config(1060.0, 3.5e-3, 2e-3, 5, 1.3, transient=True, waveform=wave),
        meshgen.simulation_config(1.0, 0.01, 1e-2, 4, 2.0, transient=True, waveform=sine),
        meshgen.simulation_config(1060.0, 3.5e-3, 2e-3, 3, 1.0, transient=True, waveform=wave,
                                  outlets=outlet({"type": "resistance", "resistance": 2e7,
                                                  "reference_pressure": 10.0})),
        meshgen.simulation_config(1060.0, 3.5e-3, 2e-3, 3, 1.0, transient=True, waveform=wave,
                                  outlets=outlet({"type": "windkessel_rc", "resistance": 3e8, "capacitance": 2e-10,
                                                  "initial_pressure": 40.0})),
        meshgen.simulation_config(1060.0, 3.5e-3, 2e-3, 3, 1.0, transient=True, waveform=wave,
                                  outlets=outlet({"type": "windkessel_rcr", "proximal_resistance": 1e8,
                                                  "capacitance": 1e-10, "distal_resistance": 1e9,
                                                  "initial_pressure": 25.0})),
        meshgen.simulation_config(1060.0, 3.5e-3, 2e-3, 3, 1.0, transient=True,
                                  outlets=outlet({"type": "pressure_traction", "value": 133.0})),
    ]
    cases[1]["boundaries"][0]["conditions"][0]["value"] = [0.0, 0.0, 0.01]
    keys = ("velocity_mask", "velocity", "pressure_mask", "pressure", "counts")
    for k, cfg in enumerate(cases):
        path = tmp_path / f"case{k}" / "simulation_config.json"
        path.parent.mkdir()
        path.write_text(json.dumps(cfg))
        for time in (0.0, 0.37, 1.05):
            want = O.ref_flow_boundaries(path, t.labels, velocity, time)
            got = api.resolve_flow_boundaries(path, t.labels, velocity, time)
            for key in keys:
                assert np.allclose(got[key], want[key], rtol=1e-15, atol=0), (k, time, key)
            assert got["tractions"].keys() == want["tractions"].keys(), (k, time)
            for label, value in want["tractions"].items():
                assert got["tractions"][label] == pytest.approx(value, rel=1e-15, abs=0), (k, time)
            assert np.array_equal(got["physics"], want["physics"]), (k, time)


@requires_ref
def test_transport_params_match_the_reference_reader(api, tmp_path):
    """simulation_parameter.txt through tfiga_transport_read_params against the reference's own
    ReadTransportParameters: values, the optional artificial-diffusion spellings, and failures."""
    order = ("diffusion", "vplus", "vminus", "kplus", "kminus", "detach_plus", "detach_minus", "dt", "steps",
             "n0_bc", "nplus_bc", "nminus_bc", "artificial_diffusion")
    texts = ["D 1e-3\nvplus 0.5\nvminus 0.25\nkplus 2\nkminus 0.5\nk'plus 0.125\nk'minus 0.0625\ndt 0.01\n"
             "nstep 12\nN0bc 1\nNplusbc 0.5\nNminusbc 0.25\n",
             "nstep 3 dt 0.5 D 0 vplus 1 vminus 1 kplus 0 kminus 0 k'plus 0 k'minus 0 N0bc 0 Nplusbc 0 Nminusbc 0 "
             "artificial_diffusion_weight 0.75\n",
             "D 1\nD 2\nvplus 1\nvminus 1\nkplus 1\nkminus 1\nk'plus 1\nk'minus 1\ndt 1\nnstep 1\nN0bc 1\n"
             "Nplusbc 1\nNminusbc 1\nartificial_diffusion 3\nartificial_diffusion_weight 4\n",
             "D 1\nvplus 1\n",
             "D 1\nvplus 1\nvminus 1\nkplus 1\nkminus 1\nk'plus 1\nk'minus 1\ndt 0\nnstep 1\nN0bc 1\nNplusbc 1\n"
             "Nminusbc 1\n"]
    for k, text in enumerate(texts):
        path = tmp_path / f"p{k}.txt"
        path.write_text(text)
        try:
            want = O.ref_read_transport_parameters(path)
        except RuntimeError as ref_error:
            with pytest.raises(api.TfigaError) as err:
                api.read_transport_params(path)
            assert str(ref_error) in str(err.value), (k, str(ref_error), str(err.value))
            continue
        got = api.read_transport_params(path).as_dict()
        assert [float(got[name]) for name in order] == list(want), k


def test_flow_line_preconditioner_oracle(small_tube):
    """The flow-line preconditioner restated in the oracle (the checker of a device version): every
    node on exactly one line, the banded no-pivot line factors solve each line's 2x2-block system
    exactly, and GMRES(50) with them needs fewer iterations than block-Jacobi for the same solution."""
    from tubularflowiga_b200 import meshgen
    tube = meshgen.straight_tube(1.5e-3, 7.5e-3, core=8, ring=2, layers=25)
    flat = tube.mesh
    params = {"diffusion": 1e-9, "vplus": 1.0, "kplus": 1.0, "kminus": 0.1, "detach_plus": 0.5, "dt": 2e-3,
              "artificial_diffusion": 1e-6}
    pattern = O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity)
    mask = (tube.labels == 1).astype(np.int32)
    left, previous = O.transport_assemble(flat, pattern, 0.3 * tube.profile, params, mask)
    lines = O.FlowLines(pattern.row_offsets, pattern.columns, left)
    assert np.array_equal(np.sort(lines.line_nodes), np.arange(flat.nodes))
    assert lines.lines < flat.nodes // 2 and np.max(np.diff(lines.line_offsets)) >= 20
    # exact per-line solves
    A = O.transport_scipy(pattern, left).tocsr()
    rng = np.random.default_rng(2)
    r = rng.normal(size=2 * flat.nodes)
    z = lines.apply(r)
    longest = np.argsort(np.diff(lines.line_offsets))[-8:]
    for l in longest:
        nodes = lines.line_nodes[lines.line_offsets[l]:lines.line_offsets[l + 1]]
        dof = np.stack([2 * nodes, 2 * nodes + 1], axis=1).ravel()
        sub = A[dof][:, dof].toarray()
        assert np.allclose(sub @ z[dof], r[dof], rtol=0, atol=1e-9 * np.abs(r[dof]).max())
    # GMRES
    c0 = O.transport_initial(flat.nodes, mask, mask * 1.0, mask * 0.5)
    rhs = O.transport_spmv(pattern.row_offsets, pattern.columns, previous, c0)
    rhs[0::2][mask != 0] = 1.0
    rhs[1::2][mask != 0] = 0.5
    want = O.transport_steps(pattern, left, previous, c0, mask, mask * 1.0, mask * 0.5, 1)
    _, it_bj, _ = O.transport_gmres(pattern.row_offsets, pattern.columns, pattern.diagonal, left, rhs,
                                    np.zeros_like(rhs))
    _, it_ln, _ = lines.gmres(rhs, np.zeros_like(rhs))
    assert 0 < it_ln < 0.7 * it_bj, (it_ln, it_bj)
    # both converge to the direct solution (tightened tolerance: the two stopping tests measure the
    # residual through different preconditioners)
    for x in (O.transport_gmres(pattern.row_offsets, pattern.columns, pattern.diagonal, left, rhs,
                                np.zeros_like(rhs), rtol=1e-12)[0], lines.gmres(rhs, np.zeros_like(rhs), rtol=1e-12)[0]):
        for f in (0, 1):
            assert np.linalg.norm(x[f::2] - want[f::2]) <= 1e-9 * np.linalg.norm(want[f::2])


def test_flow_line_host_builder_matches_the_oracle(api, small_tube):
    """The library's host construction of the flow lines and their banded factors
    (tfiga_transport_flow_lines) equals the oracle's restatement."""
    from tubularflowiga_b200 import meshgen
    tube = meshgen.straight_tube(1.5e-3, 7.5e-3, core=8, ring=2, layers=12)
    flat = tube.mesh
    params = {"diffusion": 1e-9, "vplus": 1.0, "kplus": 1.0, "kminus": 0.1, "detach_plus": 0.5, "dt": 2e-3,
              "artificial_diffusion": 1e-6}
    pattern = O.Pattern(flat.nodes, flat.element_offsets, flat.connectivity)
    mask = (tube.labels == 1).astype(np.int32)
    left, _ = O.transport_assemble(flat, pattern, 0.3 * tube.profile + 0.01, params, mask)
    want = O.FlowLines(pattern.row_offsets, pattern.columns, left)
    got = api.transport_flow_lines(pattern.row_offsets, pattern.columns, left)
    for key in ("line_offsets", "line_nodes", "band_width", "band_offsets"):
        assert np.array_equal(got[key], getattr(want, key)), key
    assert np.allclose(got["factors"], want.factors, rtol=1e-14, atol=1e-14 * np.abs(want.factors).max())


@requires_ref
def test_simulation_config_errors_match_the_reference(api, tmp_path, small_tube):
    """Validation of simulation_config.json for the flow path (root keys and schema rules, fields, time,
    temporal functions, equation systems, boundaries and their conditions, outlet models): 39 invalid
    files fail here and in the reference's own ReadSimulationConfiguration chain with the reference's
    message, and the valid base file resolves in both."""
    from tubularflowiga_b200 import meshgen
    t = small_tube
    base = meshgen.simulation_config(1060.0, 3.5e-3, 2e-3, 3, 1.0, transient=True,
                                     waveform=meshgen.fourier_waveform(1))

    def variant(edit):
        cfg = json.loads(json.dumps(base))
        edit(cfg)
        return cfg

    rcr = {"label": 2, "name": "outlet", "conditions": [{"field": "pressure", "type": "windkessel_rcr",
                                                          "proximal_resistance": 1e8, "capacitance": 0.0,
                                                          "distal_resistance": 1e9}]}
    cond = lambda c, k: c["boundaries"][k]["conditions"][0]
    bad = [
        lambda c: c.pop("dimension"), lambda c: c.update(dimension="2d"), lambda c: c.update(schema_version=5),
        lambda c: c.update(schema_version=2), lambda c: c.update(schema_version=4), lambda c: c.update(colour=1),
        lambda c: c.update(geometry={"kind": "swc_network"}), lambda c: c.pop("schema_version"),
        lambda c: c.pop("fields"), lambda c: c.update(fields=[]), lambda c: c["fields"][0].update(kind="tensor"),
        lambda c: c["fields"].append(dict(c["fields"][0])), lambda c: c["fields"][0].update(colour=1),
        lambda c: c["time"].update(dt=0.0), lambda c: c["time"].update(steps=-1), lambda c: c["time"].update(colour=1),
        lambda c: c["temporal_functions"][0].pop("units"), lambda c: c["temporal_functions"][0].update(units=""),
        lambda c: c["temporal_functions"][0].update(kind="spline"),
        lambda c: c["temporal_functions"].append(dict(c["temporal_functions"][0])),
        lambda c: c["temporal_functions"][0].update(period=0.0), lambda c: c["temporal_functions"][0].update(colour=1),
        lambda c: c.pop("equation_systems"), lambda c: c["equation_systems"][0].update(kind="euler"),
        lambda c: c["equation_systems"][0].update(colour=1),
        lambda c: c["equation_systems"][0].update(unknowns=["velocity"]),
        lambda c: c["equation_systems"][0].update(viscosity=-1.0),
        lambda c: c["equation_systems"][0].update(time_integration="bdf2"),
        lambda c: c.pop("boundaries"), lambda c: c["boundaries"][0].update(colour=1),
        lambda c: c["boundaries"][0].pop("label"), lambda c: c["boundaries"].append(dict(c["boundaries"][0])),
        lambda c: cond(c, 0).update(type="magic"), lambda c: cond(c, 0).update(field="temperature"),
        lambda c: cond(c, 0).update(colour=1), lambda c: cond(c, 0).update(value=[0, 0]),
        lambda c: cond(c, 1).update(profile="nofile.txt"), lambda c: cond(c, 1).update(waveform="nothing"),
        lambda c: c["boundaries"].__setitem__(2, rcr),
    ]
    assert len(bad) == 39
    for k, edit in enumerate([lambda c: None] + bad):
        path = tmp_path / f"case{k}" / "simulation_config.json"
        path.parent.mkdir()
        path.write_text(json.dumps(variant(edit)))
        if k == 0:
            O.ref_flow_boundaries(path, t.labels, t.profile, 0.0)
            api.resolve_flow_boundaries(path, t.labels, t.profile, 0.0)
            continue
        with pytest.raises(RuntimeError) as ref_error:
            O.ref_flow_boundaries(path, t.labels, t.profile, 0.0)
        with pytest.raises(api.TfigaError) as err:
            api.resolve_flow_boundaries(path, t.labels, t.profile, 0.0)
        assert str(ref_error.value) in str(err.value), (k, str(ref_error.value), str(err.value))
    # a transport system beside the flow: its time integration and its terms
    transport = {"name": "species", "kind": "linear_transport", "unknowns": ["pressure"]}
    for k, system in enumerate([dict(transport, time_integration="steady",
                                     terms=[{"operator": "mass", "equation": "pressure"}]),
                                transport]):
        path = tmp_path / f"transport{k}" / "simulation_config.json"
        path.parent.mkdir()
        path.write_text(json.dumps(variant(lambda c: c["equation_systems"].append(system))))
        with pytest.raises(RuntimeError) as ref_error:
            O.ref_flow_boundaries(path, t.labels, t.profile, 0.0)
        with pytest.raises(api.TfigaError) as err:
            api.resolve_flow_boundaries(path, t.labels, t.profile, 0.0)
        assert str(ref_error.value) in str(err.value), (k, str(ref_error.value), str(err.value))
    # texts json.dumps cannot write: a repeated key, and two unknown keys in the opposite of sorted order
    text = json.dumps(base)
    raw = [text.replace('"time": {', '"time": {"dt": 0.004, ', 1),
           text.replace('"schema_version"', '"zeta": 1, "alpha": 2, "schema_version"', 1)]
    for k, body in enumerate(raw):
        path = tmp_path / f"raw{k}" / "simulation_config.json"
        path.parent.mkdir()
        path.write_text(body)
        with pytest.raises(RuntimeError) as ref_error:
            O.ref_flow_boundaries(path, t.labels, t.profile, 0.0)
        with pytest.raises(api.TfigaError) as err:
            api.resolve_flow_boundaries(path, t.labels, t.profile, 0.0)
        assert str(ref_error.value) in str(err.value), (k, str(ref_error.value), str(err.value))


@requires_ref
def test_periodic_table_waveforms_match_the_reference_set_up(api, small_tube, tmp_path):
    """periodic_table inflow waveforms (a CSV of time,value samples, linearly interpolated and wrapped at
    the period; TemporalFunction.hpp:45-134) through the flow boundary set-up against the reference's own
    compiled chain: the materialised inlet values at times inside, between and past the samples and
    across the wrap; and the CSV's validation messages."""
    from tubularflowiga_b200 import meshgen
    t = small_tube
    rng = np.random.default_rng(4)
    velocity = t.profile + 0.1 * rng.normal(size=t.profile.shape)
    table = {"name": "inflow", "kind": "periodic_table", "units": "m/s", "period": 0.8, "file": "inflow.csv",
             "interpolation": "linear"}
    cfg = meshgen.simulation_config(1060.0, 3.5e-3, 2e-3, 4, 1.0, transient=True, waveform=table)
    d = tmp_path / "table"
    d.mkdir()
    (d / "simulation_config.json").write_text(json.dumps(cfg))
    (d / "inflow.csv").write_text("# inflow factor\ntime,value\n0.0, 0.4\n0.1,1.3\n 0.25 ,0.9\n0.5,0.2\n0.7,0.55\n")
    keys = ("velocity_mask", "velocity", "pressure_mask", "pressure", "counts")
    for time in (0.0, 0.05, 0.1, 0.3, 0.69, 0.75, 0.8, 1.23, 2.4001):
        want = O.ref_flow_boundaries(d / "simulation_config.json", t.labels, velocity, time)
        got = api.resolve_flow_boundaries(d / "simulation_config.json", t.labels, velocity, time)
        for key in keys:
            assert np.allclose(got[key], want[key], rtol=1e-15, atol=0), (time, key)
    bad = {"one sample": "0.0,1.0\n", "not at zero": "0.1,1.0\n0.2,2.0\n", "decreasing": "0.0,1\n0.5,2\n0.3,3\n",
           "past the period": "0.0,1\n0.9,2\n", "three fields": "0.0,1,2\n0.5,2\n", "text": "0.0,a\n0.5,2\n"}
    for name, text in bad.items():
        (d / "inflow.csv").write_text(text)
        with pytest.raises(RuntimeError) as want:
            O.ref_flow_boundaries(d / "simulation_config.json", t.labels, velocity, 0.3)
        with pytest.raises(api.TfigaError) as got:
            api.resolve_flow_boundaries(d / "simulation_config.json", t.labels, velocity, 0.3)
        assert str(want.value) in str(got.value), (name, str(want.value), str(got.value))
