"""ctypes access to the CPU oracle (test infrastructure only).

Two libraries live here:

* ``liboracle.so`` -- the C restatement in ``ns_oracle.c`` of the reference's
  element arithmetic, block pattern, Dirichlet rows and block-Jacobi GMRES.
* ``_ref/libtfiga_ref.so`` -- the reference's own header-only element code
  compiled unmodified (``ref_shim.cpp``); present where it was built.

Only the tests, the smoke check and the bench's CPU-baseline leg import this
module, and only as the checker.  ``newton_step`` restates one iteration of
the reference Newton loop (solvers/cuda/src/iga_cuda.cu:956-1033) with a
direct sparse solve so the parity tests can use a linear solve far tighter
than the reference's GMRES tolerance.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def _load(path: Path):
    if not path.exists():
        raise FileNotFoundError(f"{path} is not built; run `make -C {HERE}`")
    return C.CDLL(str(path))


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load(HERE / "liboracle.so")
        L = _lib
        L.tfo_gauss_rule.argtypes = [_dp, _dp]
        L.tfo_basis.argtypes = [_dp, _dp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                _dp, _dp, _dp, _dp, C.POINTER(C.c_double)]
        L.tfo_ns_element.argtypes = [_dp, _dp, C.c_int, _dp, C.c_void_p, C.c_double, C.c_double,
                                     C.c_double, _dp, _dp, C.c_int, C.c_void_p, _dp]
        L.tfo_min_determinant.argtypes = [_dp, C.POINTER(C.c_int)]
        L.tfo_min_determinant.restype = C.c_double
        L.tfo_face_coefficients.argtypes = [_dp, _dp, C.c_int, C.c_int, _dp]
        L.tfo_boundary_flow.argtypes = [_dp, _dp, C.c_int, C.c_int, _dp]
        L.tfo_boundary_flow.restype = C.c_double
        L.tfo_outlet_model.argtypes = [C.c_int] + [C.c_double] * 8 + [C.POINTER(C.c_double)] * 2
        L.tfo_temporal.argtypes = [C.c_int] + [C.c_double] * 5 + [_dp, _dp, C.c_int, C.c_double]
        L.tfo_temporal.restype = C.c_double
        L.tfo_block_pattern.argtypes = [C.c_int, C.c_int, _ip, _ip, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_longlong)]
        L.tfo_assemble.argtypes = [C.c_int, C.c_int, _ip, _ip, _ip, _up, _dp, _dp, _ip, _ip, _dp, _dp,
                                   C.c_double, C.c_double, C.c_double, C.c_void_p, _dp, C.POINTER(C.c_int)]
        L.tfo_apply_dirichlet.argtypes = [C.c_int, _ip, _ip, _ip, _ip, _dp, _dp, _dp, C.c_void_p, _dp]
        L.tfo_spmv.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp]
        L.tfo_gmres_bjacobi.argtypes = [C.c_int, _ip, _ip, _ip, _dp, _dp, _dp, C.c_int, C.c_int, C.c_double,
                                        C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.tfo_max_threads.restype = C.c_int
        L.tfo_transport_element.argtypes = [_dp, _dp, C.c_int, _dp, _dp, _dp, _dp]
        L.tfo_transport_spmv.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp]
        _lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
        L.tfo_flow_lines.argtypes = [C.c_int, _ip, _ip, _dp, _ip, _ip]
        L.tfo_line_factors.argtypes = [C.c_int, _ip, _ip, _dp, C.c_int, _ip, _ip, _ip, _lp, C.c_void_p]
        L.tfo_line_factors.restype = C.c_longlong
        L.tfo_line_apply.argtypes = [C.c_int, _ip, _ip, _ip, _lp, _dp, _dp, _dp]
        L.tfo_transport_gmres_lines.argtypes = [C.c_int, _ip, _ip, _dp, C.c_int, _ip, _ip, _ip, _lp, _dp, _dp, _dp,
                                                C.c_int, C.c_int, C.c_double, C.POINTER(C.c_double)]
        L.tfo_transport_gmres.argtypes = [C.c_int, _ip, _ip, _ip, _dp, _dp, _dp, C.c_int, C.c_int, C.c_double,
                                          C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.tfo_transport_assemble.argtypes = [C.c_int, C.c_int, _ip, _ip, _ip, _up, _dp, _dp, _ip, _ip, _ip,
                                             _dp, _dp, C.c_void_p, _dp, _dp, C.POINTER(C.c_int)]
    return _lib


def ref_available() -> bool:
    return (HERE / "_ref" / "libtfiga_ref.so").exists()


def ref():
    global _ref
    if _ref is None:
        _ref = _load(HERE / "_ref" / "libtfiga_ref.so")
        R = _ref
        R.ref_last_error.restype = C.c_char_p
        R.ref_ns_element.argtypes = [_dp, _dp, C.c_int, _dp, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                     C.c_void_p, _dp]
        R.ref_ns_element_points.argtypes = [_dp, _dp, C.c_int, _dp, C.c_void_p, C.c_double, C.c_double,
                                            C.c_double, _dp, _dp, C.c_int, C.c_void_p, _dp]
        R.ref_basis.argtypes = [_dp, _dp, C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp, _dp,
                                C.POINTER(C.c_double)]
        R.ref_boundary_flow.argtypes = [_dp, _dp, C.c_int, C.c_int, _dp]
        R.ref_boundary_flow.restype = C.c_double
        R.ref_pressure_traction.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_double, _dp]
        R.ref_outlet_model.argtypes = [C.c_int] + [C.c_double] * 8 + [C.POINTER(C.c_double)] * 2
        R.ref_ntiga_header.argtypes = [C.c_char_p, np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")]
        R.ref_ntiga_element.argtypes = [C.c_char_p, C.c_uint64, C.POINTER(C.c_int), _ip, _ip, _dp, _dp]
        R.ref_wall_trace.argtypes = [C.c_char_p, C.c_char_p, _ip, C.c_longlong]
        R.ref_wall_trace.restype = C.c_longlong
        R.ref_assemble.argtypes = [C.c_int, C.c_int, _ip, _ip, _ip, _up, _dp, _dp, _ip, _ip, _dp, _dp,
                                   C.c_double, C.c_double, C.c_double, C.c_void_p, _dp]
        R.ref_max_threads.restype = C.c_int
        R.ref_transport_element.argtypes = [_dp, _dp, C.c_int, _dp, _dp, _dp, _dp]
        R.ref_read_transport_parameters.argtypes = [C.c_char_p, _dp]
        R.ref_write_flow_checkpoint.argtypes = [C.c_char_p, C.c_longlong, C.c_int, C.c_double, C.c_double, C.c_double,
                                                C.c_double, _ip, _dp, C.c_int, _dp]
        R.ref_read_flow_checkpoint.argtypes = [C.c_char_p, C.c_longlong, C.c_int, C.c_double, C.c_double, C.c_double,
                                               _dp, C.POINTER(C.c_int), C.POINTER(C.c_double), _ip, _dp,
                                               C.POINTER(C.c_int)]
        R.ref_write_vtu.argtypes = [C.c_char_p, C.c_char_p, _dp, C.c_longlong, C.c_double]
        R.ref_flow_boundaries.argtypes = [C.c_char_p, C.c_char_p, C.c_double, C.c_longlong, _ip, _dp, _ip, _dp, _ip,
                                          _dp, np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS"), _ip,
                                          _dp, C.POINTER(C.c_int), _dp]
        R.ref_resolve_boundaries.argtypes = [C.c_longlong, _ip, _dp, C.c_double, C.c_double, C.c_double, C.c_char_p,
                                             _ip, _ip, _ip, _dp, _dp, _dp, _dp,
                                             np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
        R.ref_womersley_axial_velocity.argtypes = [C.c_double] * 5 + [_dp, _dp, C.c_int, C.c_double, C.c_double,
                                                   C.POINTER(C.c_double)]
    return _ref


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def gauss_rule():
    p = np.zeros(64 * 3)
    w = np.zeros(64)
    lib().tfo_gauss_rule(p, w)
    return p.reshape(64, 3), w


# --------------------------------------------------------------------------
# Element level
# --------------------------------------------------------------------------

def basis(Cx, X, u, v, w, hessian=True, use_ref=False):
    Cx = np.ascontiguousarray(Cx, dtype=np.float64)
    X = np.ascontiguousarray(X, dtype=np.float64)
    nen = Cx.shape[0]
    N = np.zeros(nen); dN = np.zeros(nen * 3); H = np.zeros(nen * 9); inv = np.zeros(9)
    det = C.c_double()
    if use_ref:
        st = ref().ref_basis(Cx.ravel(), X.ravel(), nen, u, v, w, N, dN, H, inv, C.byref(det))
    else:
        st = lib().tfo_basis(Cx.ravel(), X.ravel(), nen, u, v, w, int(hessian), N, dN, H, inv, C.byref(det))
    if st != 0:
        raise RuntimeError(f"basis evaluation failed ({st})")
    return N, dN.reshape(nen, 3), H.reshape(nen, 3, 3), inv.reshape(3, 3), det.value


def ns_element(Cx, X, state, previous, density, viscosity, dt, jacobian=True, use_ref=False,
               points=None, weights=None):
    """Element (-r, dr/du) of the reference VMS formulation; jac is (4nen, 4nen)."""
    Cx = np.ascontiguousarray(Cx, dtype=np.float64)
    X = np.ascontiguousarray(X, dtype=np.float64)
    st = np.ascontiguousarray(state, dtype=np.float64)
    pv = None if previous is None else np.ascontiguousarray(previous, dtype=np.float64)
    nen = Cx.shape[0]
    negres = np.zeros(4 * nen)
    jac = np.zeros((4 * nen, 4 * nen)) if jacobian else None
    if points is None:
        points, weights = gauss_rule()
    points = np.ascontiguousarray(points, dtype=np.float64).ravel()
    weights = np.ascontiguousarray(weights, dtype=np.float64).ravel()
    if use_ref:
        R = ref()
        if len(weights) == 64 and np.allclose(points.reshape(-1, 3), gauss_rule()[0]):
            s = R.ref_ns_element(Cx.ravel(), X.ravel(), nen, st.ravel(), _ptr(pv), density, viscosity, dt,
                                 _ptr(jac), negres)
        else:
            s = R.ref_ns_element_points(Cx.ravel(), X.ravel(), nen, st.ravel(), _ptr(pv), density, viscosity,
                                        dt, points, weights, len(weights), _ptr(jac), negres)
        if s != 0:
            raise RuntimeError(R.ref_last_error().decode())
    else:
        s = lib().tfo_ns_element(Cx.ravel(), X.ravel(), nen, st.ravel(), _ptr(pv), density, viscosity, dt,
                                 points, weights, len(weights), _ptr(jac), negres)
        if s != 0:
            raise RuntimeError(f"oracle element failed ({s})")
    return negres, jac


def face_coefficients(Cx, X, face):
    Cx = np.ascontiguousarray(Cx, dtype=np.float64)
    nen = Cx.shape[0]
    F = np.zeros(nen * 3)
    if lib().tfo_face_coefficients(Cx.ravel(), np.ascontiguousarray(X, dtype=np.float64).ravel(), nen, face, F):
        raise RuntimeError("face coefficients failed")
    return F.reshape(nen, 3)


def boundary_flow(Cx, X, face, state, use_ref=False):
    Cx = np.ascontiguousarray(Cx, dtype=np.float64)
    X = np.ascontiguousarray(X, dtype=np.float64)
    st = np.ascontiguousarray(state, dtype=np.float64).ravel()
    f = ref().ref_boundary_flow if use_ref else lib().tfo_boundary_flow
    return f(Cx.ravel(), X.ravel(), Cx.shape[0], face, st)


def outlet_model(kind, resistance, proximal, distal, capacitance, reference_pressure, capacitor_pressure,
                 flow, dt, use_ref=False):
    p = C.c_double(); pc = C.c_double()
    f = ref().ref_outlet_model if use_ref else lib().tfo_outlet_model
    if f(kind, resistance, proximal, distal, capacitance, reference_pressure, capacitor_pressure, flow, dt,
         C.byref(p), C.byref(pc)):
        raise RuntimeError("outlet model rejected its input")
    return p.value, pc.value


def temporal(kind, value=0.0, mean=0.0, amplitude=0.0, period=1.0, phase=0.0, cosine=(), sine=(), time=0.0):
    c = np.ascontiguousarray(cosine, dtype=np.float64)
    s = np.ascontiguousarray(sine, dtype=np.float64)
    if c.size == 0:
        c = np.zeros(1); s = np.zeros(1); h = 0
    else:
        h = len(cosine)
    return lib().tfo_temporal(kind, value, mean, amplitude, period, phase, c, s, h, time)


# --------------------------------------------------------------------------
# Mesh level
# --------------------------------------------------------------------------

class Pattern:
    def __init__(self, nodes, element_offsets, connectivity):
        L = lib()
        eo = np.ascontiguousarray(element_offsets, dtype=np.int32)
        cn = np.ascontiguousarray(connectivity, dtype=np.int32)
        blocks = C.c_longlong()
        st = L.tfo_block_pattern(nodes, len(eo) - 1, eo, cn, None, None, None, C.byref(blocks))
        if st:
            raise RuntimeError("block pattern failed")
        self.nodes = nodes
        self.row_offsets = np.zeros(nodes + 1, np.int32)
        self.columns = np.zeros(blocks.value, np.int32)
        self.diagonal = np.zeros(nodes, np.int32)
        st = L.tfo_block_pattern(nodes, len(eo) - 1, eo, cn, _ptr(self.row_offsets), _ptr(self.columns),
                                 _ptr(self.diagonal), C.byref(blocks))
        if st:
            raise RuntimeError("block pattern failed (missing diagonal)")
        self.blocks = int(blocks.value)

    def to_scipy(self, values):
        import scipy.sparse as sp
        v = np.asarray(values).reshape(-1, 4, 4)
        return sp.bsr_matrix((v, self.columns, self.row_offsets),
                             shape=(4 * self.nodes, 4 * self.nodes)).tocsr()


def assemble(mesh, pattern, state, previous, density, viscosity, dt, jacobian=True):
    """Global assembly of (block-CSR values, rhs = -r) over a FlatMesh-like object."""
    L = lib()
    values = np.zeros(pattern.blocks * 16) if jacobian else None
    rhs = np.zeros(4 * mesh.nodes)
    failed = C.c_int(-1)
    prev = np.ascontiguousarray(previous if previous is not None else np.zeros(4 * mesh.nodes), np.float64)
    st = L.tfo_assemble(mesh.nodes, mesh.elements, mesh.element_offsets, mesh.connectivity,
                        mesh.extraction_offsets, mesh.extraction_columns, mesh.extraction_values,
                        mesh.bezier_points, pattern.row_offsets, pattern.columns,
                        np.ascontiguousarray(state, np.float64).ravel(), prev.ravel(),
                        density, viscosity, dt, _ptr(values), rhs, C.byref(failed))
    if st:
        raise RuntimeError(f"oracle assembly failed at element {failed.value} ({st})")
    return values, rhs


def ref_assemble(mesh, pattern, state, previous, density, viscosity, dt, first=0, last=None,
                 jacobian=True):
    """Assembly of elements [first, last) with the reference's own compiled element code."""
    R = ref()
    last = mesh.elements if last is None else last
    values = np.zeros(pattern.blocks * 16) if jacobian else None
    rhs = np.zeros(4 * mesh.nodes)
    prev = np.ascontiguousarray(previous if previous is not None else np.zeros(4 * mesh.nodes), np.float64)
    st = R.ref_assemble(first, last, mesh.element_offsets, mesh.connectivity, mesh.extraction_offsets,
                        mesh.extraction_columns, mesh.extraction_values, mesh.bezier_points,
                        pattern.row_offsets, pattern.columns, np.ascontiguousarray(state, np.float64).ravel(),
                        prev.ravel(), density, viscosity, dt, _ptr(values), rhs)
    if st:
        raise RuntimeError(R.ref_last_error().decode())
    return values, rhs


def apply_dirichlet(pattern, vmask, pmask, velocity, pressure, state, values, rhs):
    lib().tfo_apply_dirichlet(pattern.nodes, pattern.row_offsets, pattern.diagonal,
                              np.ascontiguousarray(vmask, np.int32), np.ascontiguousarray(pmask, np.int32),
                              np.ascontiguousarray(velocity, np.float64).ravel(),
                              np.ascontiguousarray(pressure, np.float64).ravel(),
                              np.ascontiguousarray(state, np.float64).ravel(), _ptr(values), rhs)


def spmv(pattern, values, x):
    y = np.zeros(4 * pattern.nodes)
    lib().tfo_spmv(pattern.nodes, pattern.row_offsets, pattern.columns, values,
                   np.ascontiguousarray(x, np.float64), y)
    return y


def gmres_bjacobi(pattern, values, rhs, x0=None, restart=200, maxit=5000, rtol=1e-8):
    x = np.zeros(4 * pattern.nodes) if x0 is None else np.array(x0, np.float64)
    res = C.c_double(); singular = C.c_int()
    it = lib().tfo_gmres_bjacobi(pattern.nodes, pattern.row_offsets, pattern.columns, pattern.diagonal,
                                 values, np.ascontiguousarray(rhs, np.float64), x, restart, maxit, rtol,
                                 C.byref(res), C.byref(singular))
    return x, it, res.value, singular.value


def newton_step(mesh, pattern, state, previous, density, viscosity, dt, vmask, pmask, velocity, pressure,
                traction_rhs=None):
    """One reference Newton iteration (iga_cuda.cu:959-1033) with a direct solve.

    Returns (new_state, residual_norm_after_bc, raw_rhs_before_bc)."""
    import scipy.sparse.linalg as spla
    values, rhs = assemble(mesh, pattern, state, previous, density, viscosity, dt)
    if traction_rhs is not None:
        rhs += traction_rhs
    raw = rhs.copy()
    apply_dirichlet(pattern, vmask, pmask, velocity, pressure, state, values, rhs)
    norm = float(np.linalg.norm(rhs))
    A = pattern.to_scipy(values)
    update = spla.spsolve(A.tocsc(), rhs)
    return np.asarray(state, np.float64).ravel() + update, norm, raw


# --------------------------------------------------------------------------
# Two-species transport (iga_cuda transport, iga_cuda.cu:621-732)
# --------------------------------------------------------------------------

# Element parameter vector of tfo_transport_element / ref_transport_element.
TRANSPORT_KEYS = ("diffusion", "vplus", "kplus", "kminus", "detach_plus", "dt", "artificial_diffusion")


def transport_vector(params):
    """params: a mapping with TRANSPORT_KEYS (missing ones are 0)."""
    return np.array([float(params.get(k, 0.0)) for k in TRANSPORT_KEYS], np.float64)


def transport_element(Cx, X, velocity, params, use_ref=False):
    """(left, previous), each (2 nen)^2 with dof 2a = N0, 2a + 1 = N+."""
    nen = Cx.shape[0]
    left = np.zeros((2 * nen) ** 2)
    previous = np.zeros((2 * nen) ** 2)
    f = ref().ref_transport_element if use_ref else lib().tfo_transport_element
    st = f(np.ascontiguousarray(Cx, np.float64).ravel(), np.ascontiguousarray(X, np.float64).ravel(), nen,
           np.ascontiguousarray(velocity, np.float64).ravel(), transport_vector(params), left, previous)
    if st:
        raise RuntimeError(f"transport element failed ({st})")
    return left.reshape(2 * nen, 2 * nen), previous.reshape(2 * nen, 2 * nen)


def transport_assemble(mesh, pattern, velocity, params, constrained=None):
    """Global 2x2 block-CSR (left, previous) with the boundary rows applied."""
    left = np.zeros(pattern.blocks * 4)
    previous = np.zeros(pattern.blocks * 4)
    failed = C.c_int(-1)
    mask = None if constrained is None else np.ascontiguousarray(constrained, np.int32)
    st = lib().tfo_transport_assemble(mesh.nodes, mesh.elements, mesh.element_offsets, mesh.connectivity,
                                      mesh.extraction_offsets, mesh.extraction_columns, mesh.extraction_values,
                                      mesh.bezier_points, pattern.row_offsets, pattern.columns, pattern.diagonal,
                                      np.ascontiguousarray(velocity, np.float64).ravel(), transport_vector(params),
                                      _ptr(mask), left, previous, C.byref(failed))
    if st:
        raise RuntimeError(f"oracle transport assembly failed at element {failed.value} ({st})")
    return left, previous


def ref_read_transport_parameters(path):
    """The reference's ReadTransportParameters: the 13 values in the order of its struct."""
    out = np.zeros(13)
    if ref().ref_read_transport_parameters(str(path).encode(), out):
        raise RuntimeError(ref().ref_last_error().decode())
    return out


def ref_flow_boundaries(config_path, labels, velocity, time=0.0, system=""):
    """The reference's own flow boundary set-up (iga_cuda.cu:766-790) of a simulation_config.json case."""
    labels = np.ascontiguousarray(labels, np.int32)
    n = labels.size
    out = {"velocity_mask": np.zeros(n, np.int32), "velocity": np.zeros(3 * n), "pressure_mask": np.zeros(n, np.int32),
           "pressure": np.zeros(n), "counts": np.zeros(2, np.int64)}
    tl, tv, count = np.zeros(64, np.int32), np.zeros(64), C.c_int(64)
    physics = np.zeros(5)
    st = ref().ref_flow_boundaries(str(config_path).encode(), system.encode(), time, n, labels,
                                   np.ascontiguousarray(velocity, np.float64).ravel(), out["velocity_mask"],
                                   out["velocity"], out["pressure_mask"], out["pressure"], out["counts"], tl, tv,
                                   C.byref(count), physics)
    if st:
        raise RuntimeError(ref().ref_last_error().decode())
    out["tractions"] = {int(tl[i]): float(tv[i]) for i in range(min(count.value, 64))}
    out["physics"] = physics
    return out


def ref_resolve_boundaries(labels, velocity, vplus, n0_bc, nplus_bc, case_config_text=None):
    """The reference's own ResolveBoundaryConditions (+ ParseCaseConfiguration) on the given inputs."""
    labels = np.ascontiguousarray(labels, np.int32)
    n = labels.size
    out = {"velocity_mask": np.zeros(n, np.int32), "pressure_mask": np.zeros(n, np.int32),
           "transport_mask": np.zeros(n, np.int32), "velocity": np.zeros(3 * n), "pressure": np.zeros(n),
           "n0": np.zeros(n), "nplus": np.zeros(n), "counts": np.zeros(3, np.int64)}
    st = ref().ref_resolve_boundaries(n, labels, np.ascontiguousarray(velocity, np.float64).ravel(), vplus, n0_bc,
                                      nplus_bc, None if case_config_text is None else case_config_text.encode(),
                                      out["velocity_mask"], out["pressure_mask"], out["transport_mask"],
                                      out["velocity"], out["pressure"], out["n0"], out["nplus"], out["counts"])
    if st:
        raise RuntimeError(ref().ref_last_error().decode())
    return out


def transport_scipy(pattern, values):
    import scipy.sparse as sp
    v = np.asarray(values).reshape(-1, 2, 2)
    return sp.bsr_matrix((v, pattern.columns, pattern.row_offsets),
                         shape=(2 * pattern.nodes, 2 * pattern.nodes)).tocsr()


def transport_initial(nodes, constrained, n0, nplus):
    """Zero state with the boundary values set (SetTransportBoundaryVectorKernel, IgaCudaKernels.cuh:426-434)."""
    c = np.zeros(2 * nodes)
    m = np.asarray(constrained) != 0
    c[0::2][m] = np.asarray(n0)[m]
    c[1::2][m] = np.asarray(nplus)[m]
    return c


def transport_steps(pattern, left, previous, current, constrained, n0, nplus, steps):
    """`steps` backward-Euler steps solved directly: rhs = P c, boundary values set in rhs, L c' = rhs
    (the loop of iga_cuda.cu:683-707 with an exact linear solve)."""
    import scipy.sparse.linalg as spla
    L = transport_scipy(pattern, left).tocsc()
    P = transport_scipy(pattern, previous)
    lu = spla.splu(L)
    m = np.asarray(constrained) != 0
    c = np.array(current, np.float64)
    for _ in range(steps):
        rhs = P @ c
        rhs[0::2][m] = np.asarray(n0)[m]
        rhs[1::2][m] = np.asarray(nplus)[m]
        c = lu.solve(rhs)
    return c


def transport_spmv(row_offsets, columns, values, x):
    nodes = len(row_offsets) - 1
    y = np.zeros(2 * nodes)
    lib().tfo_transport_spmv(nodes, np.ascontiguousarray(row_offsets, np.int32),
                             np.ascontiguousarray(columns, np.int32), values, np.ascontiguousarray(x, np.float64), y)
    return y


def transport_gmres(row_offsets, columns, diagonal, values, rhs, x0, restart=50, maxit=10000, rtol=1e-8):
    """Block-Jacobi GMRES(restart) on the 2x2 system (the CPU restatement); returns (x, iterations, residual)."""
    nodes = len(row_offsets) - 1
    x = np.array(x0, np.float64)
    res = C.c_double(); singular = C.c_int()
    it = lib().tfo_transport_gmres(nodes, np.ascontiguousarray(row_offsets, np.int32),
                                   np.ascontiguousarray(columns, np.int32), np.ascontiguousarray(diagonal, np.int32),
                                   values, np.ascontiguousarray(rhs, np.float64), x, restart, maxit, rtol,
                                   C.byref(res), C.byref(singular))
    return x, it, res.value


class FlowLines:
    """Flow-line preconditioner of the 2x2 transport matrix (tfo_flow_lines / tfo_line_factors)."""

    def __init__(self, row_offsets, columns, values):
        self.row_offsets = np.ascontiguousarray(row_offsets, np.int32)
        self.columns = np.ascontiguousarray(columns, np.int32)
        self.values = np.ascontiguousarray(values, np.float64)
        self.nodes = len(self.row_offsets) - 1
        self.line_offsets = np.zeros(self.nodes + 1, np.int32)
        self.line_nodes = np.zeros(self.nodes, np.int32)
        L = lib()
        self.lines = L.tfo_flow_lines(self.nodes, self.row_offsets, self.columns, self.values, self.line_offsets,
                                      self.line_nodes)
        if self.lines < 0:
            raise RuntimeError("flow lines failed")
        self.line_offsets = self.line_offsets[:self.lines + 1].copy()
        self.band_width = np.zeros(self.lines, np.int32)
        self.band_offsets = np.zeros(self.lines, np.int64)
        size = L.tfo_line_factors(self.nodes, self.row_offsets, self.columns, self.values, self.lines,
                                  self.line_offsets, self.line_nodes, self.band_width, self.band_offsets, None)
        self.factors = np.zeros(size)
        L.tfo_line_factors(self.nodes, self.row_offsets, self.columns, self.values, self.lines, self.line_offsets,
                           self.line_nodes, self.band_width, self.band_offsets, _ptr(self.factors))

    def apply(self, r):
        out = np.zeros(2 * self.nodes)
        lib().tfo_line_apply(self.lines, self.line_offsets, self.line_nodes, self.band_width, self.band_offsets,
                             self.factors, np.ascontiguousarray(r, np.float64), out)
        return out

    def gmres(self, rhs, x0, restart=50, maxit=10000, rtol=1e-8):
        x = np.array(x0, np.float64)
        res = C.c_double()
        it = lib().tfo_transport_gmres_lines(self.nodes, self.row_offsets, self.columns, self.values, self.lines,
                                             self.line_offsets, self.line_nodes, self.band_width, self.band_offsets,
                                             self.factors, np.ascontiguousarray(rhs, np.float64), x, restart, maxit,
                                             rtol, C.byref(res))
        return x, it, res.value


# --------------------------------------------------------------------------
# Convergence diagnostics of the Newton loop and closed-form pipe flows
# --------------------------------------------------------------------------

def measure_flow_convergence(mesh, state, raw_rhs, use_ref=False):
    """MeasureFlowConvergence (solvers/cuda/src/iga_cuda.cu:520-557): the continuity L2 norm and sum of
    the raw rhs (after the traction, before the Dirichlet rows; continuity is field 3 of every node),
    the boundary flow of the state per face label (IntegrateBoundaryFlow over every labelled face,
    labels >= 0), their net and absolute sums in label order, and the relative mass imbalance
    2 |net| / absolute (0 when no flow)."""
    raw = np.asarray(raw_rhs, np.float64).reshape(-1, 4)
    st = np.asarray(state, np.float64).reshape(-1, 4)
    continuity_sq = 0.0
    continuity_sum = 0.0
    for c in raw[:, 3]:
        continuity_sq += c * c
        continuity_sum += c
    flows = {}
    labels_all = np.asarray(mesh.boundary_labels).reshape(-1, 6)
    for e in np.nonzero((labels_all >= 0).any(axis=1))[0]:
        conn, Cx, X, labels = mesh.element(int(e))
        nodal = np.ascontiguousarray(st[conn])
        for face in range(6):
            if labels[face] >= 0:
                lab = int(labels[face])
                flows[lab] = flows.get(lab, 0.0) + boundary_flow(Cx, X, face, nodal, use_ref=use_ref)
    net = 0.0
    absolute = 0.0
    for lab in sorted(flows):
        net += flows[lab]
        absolute += abs(flows[lab])
    return {"continuity_l2": float(np.sqrt(continuity_sq)), "continuity_sum": float(continuity_sum),
            "boundary_flow": flows, "net_boundary_flow": net, "absolute_boundary_flow": absolute,
            "relative_mass_imbalance": 2.0 * abs(net) / absolute if absolute > 0.0 else 0.0}


def newton_accepts(residual_l2, initial_residual_l2, dofs, nonlinear_atol, nonlinear_rtol, imbalance, mass_rtol):
    """The Newton acceptance test of NavierStokes (solvers/cuda/src/iga_cuda.cu:989-996): accept when
    ||r|| <= max(atol sqrt(dofs), rtol ||r_0||) and the relative mass imbalance <= mass_rtol.
    Returns (accepted, tolerance)."""
    tolerance = max(nonlinear_atol * np.sqrt(dofs), nonlinear_rtol * initial_residual_l2)
    return bool(residual_l2 <= tolerance and imbalance <= mass_rtol), float(tolerance)


def complex_bessel_j0(z):
    """J0 of a complex argument by its power series sum_k (-z^2/4)^k / (k!)^2, summed until the term
    falls below 8 eps of the sum past k > |z| (the series and stopping rule of ComplexBesselJ0,
    solvers/cpu/include/WomersleyReference.hpp:131-148, in double precision)."""
    z = complex(z)
    factor = -z * z / 4.0
    term = 1.0 + 0.0j
    total = term
    for order in range(1, 10001):
        term *= factor / float(order * order)
        total += term
        if order > abs(z) and abs(term) <= 8.0 * np.finfo(float).eps * max(1.0, abs(total)):
            return total
    raise RuntimeError("complex Bessel J0 series did not converge")


def womersley_axial_velocity(radius, density, viscosity, period, mean_gradient, cosine, sine, r, t,
                             use_ref=False):
    """Axial velocity of fully developed pipe flow driven by the pressure gradient (along the flow)
    G(t) = mean + sum_k cosine[k] cos(k w t) + sine[k] sin(k w t), w = 2 pi / period
    (WomersleyAxialVelocity, solvers/cpu/include/WomersleyReference.hpp:150-189): the Poiseuille part
    mean (R^2 - r^2) / (4 mu) plus, for every harmonic k, Re[(cosine_k - i sine_k) / (i w_k rho)
    (1 - J0(a_k r/R) / J0(a_k)) e^{i w_k t}] with a_k = alpha_k e^{-i pi/4}, alpha_k = R sqrt(w_k rho / mu)."""
    cosine = np.asarray(cosine, np.float64)
    sine = np.asarray(sine, np.float64)
    h = max(len(cosine), len(sine))
    cosine = np.pad(cosine, (0, h - len(cosine)))
    sine = np.pad(sine, (0, h - len(sine)))
    if use_ref:
        out = C.c_double()
        c = np.ascontiguousarray(cosine if h else np.zeros(1))
        s = np.ascontiguousarray(sine if h else np.zeros(1))
        if ref().ref_womersley_axial_velocity(radius, density, viscosity, period, mean_gradient, c, s, h, r, t,
                                              C.byref(out)):
            raise RuntimeError(ref().ref_last_error().decode())
        return out.value
    fraction = min(r / radius, 1.0)
    velocity = mean_gradient * (radius * radius - r * r) / (4.0 * viscosity)
    fundamental = 2.0 * np.pi / period
    for k in range(h):
        omega = (k + 1) * fundamental
        alpha = radius * np.sqrt(omega * density / viscosity)
        wall = complex(alpha / np.sqrt(2.0), -alpha / np.sqrt(2.0))
        profile = 1.0 - complex_bessel_j0(wall * fraction) / complex_bessel_j0(wall)
        amplitude = complex(cosine[k], -sine[k]) / (1j * omega * density) * profile
        velocity += float((amplitude * np.exp(1j * omega * t)).real)
    return velocity


def evaluate_state(mesh, control_points, state, elements, points):
    """The state sum_a N_a(xi) state_a and the physical point sum_a N_a(xi) P_a (the spline geometry map
    through the control points P) at the parametric points `points` [m, 3] of every listed element.
    Returns (x [len(elements) m, 3], state [len(elements) m, 4], det [len(elements) m]) with det the
    Jacobian determinant of the map from the unit parametric cube (the volume weight of a unit-cube
    quadrature rule)."""
    st = np.asarray(state, np.float64).reshape(-1, 4)
    xs, us, ms = [], [], []
    for e in elements:
        conn, Cx, X, _ = mesh.element(int(e))
        for (u, v, w) in points:
            N, _, _, _, det = basis(Cx, X, u, v, w, hessian=False)
            xs.append(N @ control_points[conn])
            us.append(N @ st[conn])
            ms.append(det)
    return np.array(xs), np.array(us), np.array(ms)


def max_threads() -> int:
    return int(lib().tfo_max_threads())


os.environ.setdefault("OMP_PROC_BIND", "false")
