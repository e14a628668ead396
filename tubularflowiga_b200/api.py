"""Python binding of the C ABI in include/tfiga.h (ctypes, no torch types).

The product path is the CUDA library ``lib/libtfiga_b200.so``; there is no
CPU fallback: loading fails loudly when the library is missing, and the
create calls fail without an sm_100 device.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .ntiga import FlatMesh

LIBRARY = Path(__file__).resolve().parent / "lib" / "libtfiga_b200.so"


class TfigaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"tfiga error {status}: {message}")
        self.status = status


class MeshDesc(C.Structure):
    _fields_ = [("nodes", C.c_int64), ("elements", C.c_int64), ("element_offsets", C.c_void_p),
                ("connectivity", C.c_void_p), ("extraction_offsets", C.c_void_p),
                ("extraction_columns", C.c_void_p), ("extraction_values", C.c_void_p),
                ("bezier_points", C.c_void_p), ("boundary_labels", C.c_void_p)]


class MeshInfo(C.Structure):
    _fields_ = [("nodes", C.c_int64), ("elements", C.c_int64), ("max_basis", C.c_int32),
                ("basis_entries", C.c_int64), ("extraction_nonzeros", C.c_int64), ("block_nonzeros", C.c_int64),
                ("max_block_row", C.c_int32), ("min_detj", C.c_double), ("bad_samples", C.c_int64),
                ("device_bytes", C.c_int64)]


class NsParams(C.Structure):
    _fields_ = [("density", C.c_double), ("viscosity", C.c_double), ("dt", C.c_double),
                ("max_newton", C.c_int32), ("nonlinear_rtol", C.c_double), ("nonlinear_atol", C.c_double),
                ("mass_rtol", C.c_double), ("gmres_restart", C.c_int32), ("gmres_max_iterations", C.c_int32),
                ("gmres_rtol", C.c_double), ("preconditioner", C.c_int32), ("precision", C.c_int32),
                ("amg_coarse_nodes", C.c_int32), ("amg_coarse_period", C.c_int32),
                ("krylov_fp64_basis", C.c_int32), ("newton_forcing", C.c_int32),
                ("tangent_reuse_factor", C.c_double), ("tangent_kernel", C.c_int32)]


TANGENT_AUTO = 0
TANGENT_COEFFICIENTS = 1
TANGENT_FUSED = 2
TANGENT_ELEMENT = 3

FP64 = 0
MIXED = 1
FP32_JACOBIAN = 2
MIXED_BF16X3 = 3
MIXED_TF32 = 4


BLOCK_JACOBI = 0
AMG = 1


class AmgInfo(C.Structure):
    _fields_ = [("levels", C.c_int32), ("nodes", C.c_int32 * 8), ("blocks", C.c_int64 * 8),
                ("transfer_blocks", C.c_int64)]


class NewtonReport(C.Structure):
    _fields_ = [("converged", C.c_int32), ("linear_iterations", C.c_int32),
                ("singular_diagonal_blocks", C.c_int32), ("residual_l2", C.c_double), ("tolerance", C.c_double),
                ("continuity_l2", C.c_double), ("continuity_sum", C.c_double), ("net_boundary_flow", C.c_double),
                ("absolute_boundary_flow", C.c_double), ("relative_mass_imbalance", C.c_double),
                ("update_l2", C.c_double), ("linear_residual", C.c_double), ("assembly_ms", C.c_double),
                ("linear_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StepReport(C.Structure):
    _fields_ = [("converged", C.c_int32), ("newton_iterations", C.c_int32), ("linear_iterations", C.c_int32),
                ("residual_l2", C.c_double), ("initial_residual_l2", C.c_double),
                ("relative_mass_imbalance", C.c_double), ("assembly_ms", C.c_double), ("linear_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


OUTLET_RESISTANCE, OUTLET_RC, OUTLET_RCR = 0, 1, 2
_OUTLET_KINDS = {"resistance": OUTLET_RESISTANCE, "windkessel_rc": OUTLET_RC, "windkessel_rcr": OUTLET_RCR}


class Outlet(C.Structure):
    """tfiga_outlet: one labelled outlet model (OutletModelState, include/OutletModel.hpp:15-26)."""
    _fields_ = [("label", C.c_int32), ("kind", C.c_int32), ("resistance", C.c_double),
                ("proximal_resistance", C.c_double), ("distal_resistance", C.c_double),
                ("capacitance", C.c_double), ("reference_pressure", C.c_double),
                ("capacitor_pressure", C.c_double), ("flow", C.c_double), ("pressure", C.c_double)]

    @classmethod
    def rcr(cls, label, proximal, capacitance, distal, reference_pressure=0.0, initial_pressure=0.0):
        """RCR outlet starting at capacitor and outlet pressure = initial_pressure (InitializeOutletModels,
        OutletModel.hpp:41-68)."""
        return cls(label=label, kind=OUTLET_RCR, proximal_resistance=proximal, capacitance=capacitance,
                   distal_resistance=distal, reference_pressure=reference_pressure,
                   capacitor_pressure=initial_pressure, pressure=initial_pressure)

    @classmethod
    def resistance_model(cls, label, resistance, reference_pressure=0.0):
        return cls(label=label, kind=OUTLET_RESISTANCE, resistance=resistance,
                   reference_pressure=reference_pressure, pressure=reference_pressure)

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TransportParams(C.Structure):
    _fields_ = [("diffusion", C.c_double), ("vplus", C.c_double), ("vminus", C.c_double),
                ("kplus", C.c_double), ("kminus", C.c_double), ("detach_plus", C.c_double),
                ("detach_minus", C.c_double), ("dt", C.c_double), ("steps", C.c_int32), ("restart", C.c_int32),
                ("n0_bc", C.c_double), ("nplus_bc", C.c_double), ("nminus_bc", C.c_double),
                ("artificial_diffusion", C.c_double), ("gmres_rtol", C.c_double),
                ("gmres_max_iterations", C.c_int32), ("precision", C.c_int32), ("preconditioner", C.c_int32),
                ("reserved", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


TRANSPORT_BLOCK_JACOBI = 0
TRANSPORT_FLOW_LINES = 1


class TransportReport(C.Structure):
    _fields_ = [("steps", C.c_int32), ("last_iterations", C.c_int32), ("total_iterations", C.c_int64),
                ("last_residual", C.c_double), ("final_l2", C.c_double), ("singular_blocks", C.c_uint32),
                ("reserved", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


# Every exported symbol of include/tfiga.h with its signature.
SIGNATURES = {
    "tfiga_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "tfiga_version": (C.c_char_p, []),
    "tfiga_mesh_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(C.c_void_p)]),
    "tfiga_mesh_load_ntiga": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "tfiga_batch_mesh_create": (C.c_int, [C.POINTER(MeshDesc), C.c_int32, C.POINTER(C.c_void_p), C.c_void_p,
                                          C.c_void_p]),
    "tfiga_mesh_destroy": (C.c_int, [C.c_void_p]),
    "tfiga_mesh_info_get": (C.c_int, [C.c_void_p, C.POINTER(MeshInfo)]),
    "tfiga_mesh_pattern": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_ns_default_params": (None, [C.POINTER(NsParams)]),
    "tfiga_ns_create": (C.c_int, [C.c_void_p, C.POINTER(NsParams), C.POINTER(C.c_void_p)]),
    "tfiga_ns_destroy": (C.c_int, [C.c_void_p]),
    "tfiga_ns_set_dirichlet": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_ns_set_dirichlet_values": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_ns_set_tractions": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "tfiga_ns_set_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_ns_get_state": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_ns_commit_step": (C.c_int, [C.c_void_p]),
    "tfiga_ns_assemble": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_ns_apply_dirichlet": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_ns_solve_linear": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, C.c_void_p, C.POINTER(C.c_int32),
                                        C.POINTER(C.c_double)]),
    "tfiga_ns_newton_iteration": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(NewtonReport)]),
    "tfiga_ns_step": (C.c_int, [C.c_void_p, C.POINTER(StepReport)]),
    "tfiga_ns_step_outlets": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_double, C.c_int32,
                                        C.POINTER(StepReport), C.POINTER(C.c_int32)]),
    "tfiga_ns_step_outlets_coupled": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_double, C.c_int32,
                                                C.POINTER(StepReport), C.POINTER(C.c_int32)]),
    "tfiga_ns_amg_info": (C.c_int, [C.c_void_p, C.POINTER(AmgInfo)]),
    "tfiga_ns_tangent_kernel": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_ns_tangent_element_ms": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_ns_set_segments": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "tfiga_ns_segment_status": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_ns_boundary_flows": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "tfiga_ns_spmv_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_ns_device_buffers": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                          C.POINTER(C.c_void_p)]),
    "tfiga_ns_launch_count": (C.c_int64, [C.c_void_p]),
    "tfiga_ns_synchronize": (C.c_int, [C.c_void_p]),
    "tfiga_ns_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "tfiga_ns_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "tfiga_ns_profile": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "tfiga_ns_profile_bytes": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_block_residual_norm_static": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                   C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_learned_create": (C.c_int, [C.c_void_p, C.c_int32, C.c_uint64, C.c_int32, C.POINTER(C.c_void_p)]),
    "tfiga_learned_destroy": (C.c_int, [C.c_void_p]),
    "tfiga_learned_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int32)]),
    "tfiga_ns_set_learned": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32]),
    "tfiga_learned_fit_scales": (C.c_int, [C.c_void_p]),
    "tfiga_learned_set_loss": (C.c_int, [C.c_void_p, C.c_int32]),
    "tfiga_learned_set_capacity": (C.c_int, [C.c_void_p, C.c_int32]),
    "tfiga_ns_learned_fallbacks": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "tfiga_learned_train": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.POINTER(C.c_double)]),
    "tfiga_learned_evaluate": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "tfiga_learned_fit_gain": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "tfiga_learned_get_parameters": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_learned_set_parameters": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_learned_get_scales": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_learned_set_scales": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_learned_neighbours": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_learned_forward_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_learned_apply_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_learned_loss_gradient_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                                     C.c_void_p]),
    "tfiga_learned_save": (C.c_int, [C.c_void_p, C.c_char_p]),
    "tfiga_learned_load": (C.c_int, [C.c_void_p, C.c_char_p]),
    "tfiga_transport_default_params": (None, [C.POINTER(TransportParams)]),
    "tfiga_transport_read_params": (C.c_int, [C.c_char_p, C.POINTER(TransportParams)]),
    "tfiga_transport_resolve_boundaries": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.POINTER(TransportParams),
                                                     C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                     C.POINTER(C.c_int64)]),
    "tfiga_wall_trace_basis": (C.c_int, [C.c_char_p, C.c_char_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]),
    "tfiga_write_flow_checkpoint": (C.c_int, [C.c_char_p, C.c_int64, C.c_int32, C.c_double, C.c_double, C.c_double,
                                              C.c_double, C.c_void_p, C.c_int32, C.c_void_p]),
    "tfiga_read_flow_checkpoint": (C.c_int, [C.c_char_p, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_void_p,
                                             C.c_int32, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "tfiga_write_vtu": (C.c_int, [C.c_char_p, C.c_char_p, C.c_void_p, C.c_int64, C.c_double]),
    "tfiga_resolve_flow_boundaries": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double, C.c_int64, C.c_void_p,
                                                C.c_void_p] + [C.c_void_p] * 5 + [C.c_void_p, C.c_void_p,
                                                                                  C.POINTER(C.c_int32), C.c_void_p]),
    "tfiga_resolve_legacy_boundaries": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.POINTER(TransportParams),
                                                  C.c_char_p] + [C.c_void_p] * 8),
    "tfiga_transport_flow_lines": (C.c_int, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int64)]),
    "tfiga_transport_create": (C.c_int, [C.c_void_p, C.POINTER(TransportParams), C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "tfiga_transport_destroy": (C.c_int, [C.c_void_p]),
    "tfiga_transport_step": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(TransportReport)]),
    "tfiga_transport_set_state": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_transport_get_state": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tfiga_transport_matrices": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_transport_apply_preconditioner": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "tfiga_transport_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int64)]),
    "tfiga_transport_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "tfiga_transport_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "tfiga_transport_profile": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "tfiga_main": (C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise ImportError(f"{LIBRARY} is not built: run `python -m tubularflowiga_b200.build` "
                              "(there is no CPU fallback)")
        L = C.CDLL(str(LIBRARY))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib().tfiga_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(status: int):
    if status != 0:
        raise TfigaError(status, last_error())


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def default_params(**overrides) -> NsParams:
    p = NsParams()
    lib().tfiga_ns_default_params(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


class Mesh:
    """Device-resident mesh (tfiga_mesh)."""

    def __init__(self, source):
        """source: a .ntiga path, a FlatMesh, or a list of FlatMesh (batched tubes: their disjoint union,
        with self.node_offsets / self.element_offsets marking where each tube starts)."""
        L = lib()
        self._h = C.c_void_p()
        if isinstance(source, (str, Path)):
            check(L.tfiga_mesh_load_ntiga(str(source).encode(), C.byref(self._h)))
        elif isinstance(source, (list, tuple)):
            meshes = [m.contiguous() for m in source]
            self._keep = meshes
            descs = (MeshDesc * len(meshes))(*[
                MeshDesc(m.nodes, m.elements, _p(m.element_offsets), _p(m.connectivity), _p(m.extraction_offsets),
                         _p(m.extraction_columns), _p(m.extraction_values), _p(m.bezier_points),
                         _p(m.boundary_labels)) for m in meshes])
            self.node_offsets = np.zeros(len(meshes) + 1, np.int64)
            self.element_offsets = np.zeros(len(meshes) + 1, np.int64)
            check(L.tfiga_batch_mesh_create(descs, len(meshes), C.byref(self._h), _p(self.node_offsets),
                                            _p(self.element_offsets)))
        else:
            m: FlatMesh = source.contiguous()
            self._keep = m
            d = MeshDesc(m.nodes, m.elements, _p(m.element_offsets), _p(m.connectivity),
                         _p(m.extraction_offsets), _p(m.extraction_columns), _p(m.extraction_values),
                         _p(m.bezier_points), _p(m.boundary_labels))
            check(L.tfiga_mesh_create(C.byref(d), C.byref(self._h)))
        info = MeshInfo()
        check(L.tfiga_mesh_info_get(self._h, C.byref(info)))
        self.info = {k: getattr(info, k) for k, _ in MeshInfo._fields_}
        self.nodes = int(info.nodes)
        self.blocks = int(info.block_nonzeros)

    def pattern(self):
        ro = np.zeros(self.nodes + 1, np.int32)
        cols = np.zeros(self.blocks, np.int32)
        diag = np.zeros(self.nodes, np.int32)
        check(lib().tfiga_mesh_pattern(self._h, _p(ro), _p(cols), _p(diag)))
        return ro, cols, diag

    def close(self):
        if self._h:
            lib().tfiga_mesh_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NavierStokes:
    """Device-resident Navier-Stokes solver (tfiga_ns)."""

    def __init__(self, mesh: Mesh, **params):
        self.mesh = mesh
        self.params = default_params(**params)
        self._h = C.c_void_p()
        check(lib().tfiga_ns_create(mesh._h, C.byref(self.params), C.byref(self._h)))
        self.nodes = mesh.nodes

    def set_dirichlet(self, velocity_mask, pressure_mask, velocity, pressure=None):
        vm = np.ascontiguousarray(velocity_mask, np.int32)
        pm = np.ascontiguousarray(pressure_mask if pressure_mask is not None else np.zeros(self.nodes), np.int32)
        v = np.ascontiguousarray(velocity, np.float64).ravel()
        p = None if pressure is None else np.ascontiguousarray(pressure, np.float64)
        check(lib().tfiga_ns_set_dirichlet(self._h, _p(vm), _p(pm), _p(v), _p(p)))

    def set_dirichlet_values(self, velocity, pressure=None):
        v = np.ascontiguousarray(velocity, np.float64).ravel()
        p = None if pressure is None else np.ascontiguousarray(pressure, np.float64)
        check(lib().tfiga_ns_set_dirichlet_values(self._h, _p(v), _p(p)))

    def set_tractions(self, tractions: dict):
        labels = np.array(list(tractions.keys()), np.int32)
        pressures = np.array(list(tractions.values()), np.float64)
        check(lib().tfiga_ns_set_tractions(self._h, _p(labels), _p(pressures), len(labels)))

    def set_state(self, state, previous=None):
        s = np.ascontiguousarray(state, np.float64).ravel()
        p = None if previous is None else np.ascontiguousarray(previous, np.float64).ravel()
        check(lib().tfiga_ns_set_state(self._h, _p(s), _p(p)))

    def get_state(self, out=None):
        out = np.zeros(4 * self.nodes) if out is None else out
        check(lib().tfiga_ns_get_state(self._h, _p(out)))
        return out

    def commit_step(self):
        check(lib().tfiga_ns_commit_step(self._h))

    def assemble(self, values=True, rhs=True):
        v = np.zeros(self.mesh.blocks * 16) if values else None
        r = np.zeros(4 * self.nodes) if rhs else None
        check(lib().tfiga_ns_assemble(self._h, _p(v), _p(r)))
        return v, r

    def apply_dirichlet(self, values=True, rhs=True):
        v = np.zeros(self.mesh.blocks * 16) if values else None
        r = np.zeros(4 * self.nodes) if rhs else None
        check(lib().tfiga_ns_apply_dirichlet(self._h, _p(v), _p(r)))
        return v, r

    def solve_linear(self, rtol=1e-8, max_iterations=5000):
        u = np.zeros(4 * self.nodes)
        it = C.c_int32(); res = C.c_double()
        check(lib().tfiga_ns_solve_linear(self._h, rtol, max_iterations, _p(u), C.byref(it), C.byref(res)))
        return u, it.value, res.value

    def newton_iteration(self, initial_residual=-1.0) -> dict:
        r = NewtonReport()
        check(lib().tfiga_ns_newton_iteration(self._h, initial_residual, C.byref(r)))
        return r.as_dict()

    def step(self) -> dict:
        r = StepReport()
        check(lib().tfiga_ns_step(self._h, C.byref(r)))
        return r.as_dict()

    def step_outlets(self, outlets, relaxation=0.5, max_iterations=12):
        """One physical step coupled to outlet models (a list or ctypes array of Outlet, updated in place:
        accepted flow, pressure and capacitor pressure).  Returns the step report with the number of
        Newton loops as ``outlet_iterations``."""
        arr = outlets if isinstance(outlets, C.Array) else (Outlet * len(outlets))(*outlets)
        r = StepReport()
        it = C.c_int32()
        check(lib().tfiga_ns_step_outlets(self._h, C.cast(arr, C.c_void_p) if len(arr) else None, len(arr),
                                          relaxation, max_iterations, C.byref(r), C.byref(it)))
        if not isinstance(outlets, C.Array):
            for k in range(len(outlets)):
                outlets[k] = arr[k]
        d = r.as_dict()
        d["outlet_iterations"] = it.value
        return d

    def step_outlets_coupled(self, outlets, relaxation=1.0, max_newton=20):
        """One physical step with the outlet pressures updated inside the Newton loop (same fixed point and
        tolerances as step_outlets).  Returns the step report with ``pressure_updates``."""
        arr = outlets if isinstance(outlets, C.Array) else (Outlet * len(outlets))(*outlets)
        r = StepReport()
        it = C.c_int32()
        check(lib().tfiga_ns_step_outlets_coupled(self._h, C.cast(arr, C.c_void_p) if len(arr) else None, len(arr),
                                                  relaxation, max_newton, C.byref(r), C.byref(it)))
        if not isinstance(outlets, C.Array):
            for k in range(len(outlets)):
                outlets[k] = arr[k]
        d = r.as_dict()
        d["pressure_updates"] = it.value
        return d

    def boundary_flows(self, labels):
        lab = np.ascontiguousarray(labels, np.int32)
        out = np.zeros(len(lab))
        check(lib().tfiga_ns_boundary_flows(self._h, _p(lab), len(lab), _p(out)))
        return out

    def device_buffers(self):
        v, s, r = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib().tfiga_ns_device_buffers(self._h, C.byref(v), C.byref(s), C.byref(r)))
        return v.value, s.value, r.value

    def spmv_device(self, x_ptr: int, y_ptr: int):
        check(lib().tfiga_ns_spmv_device(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr)))

    def launches(self) -> int:
        return int(lib().tfiga_ns_launch_count(self._h))

    def synchronize(self):
        check(lib().tfiga_ns_synchronize(self._h))

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().tfiga_ns_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def set_profiling(self, enable: bool):
        check(lib().tfiga_ns_set_profiling(self._h, int(enable)))

    FAMILIES = ("assembly", "spmv", "krylov_orthogonalisation", "amg_vcycle", "residual", "amg_setup",
                "newton_vectors")

    def set_segments(self, node_offsets):
        """Per-tube Newton tests over the node ranges of a batch (tfiga_ns_set_segments); None removes them."""
        if node_offsets is None:
            self._segments = None
            check(lib().tfiga_ns_set_segments(self._h, None, 0))
            return
        self._segments = np.ascontiguousarray(node_offsets, np.int64)
        check(lib().tfiga_ns_set_segments(self._h, _p(self._segments), len(self._segments) - 1))

    def segment_status(self):
        """(done [T], residual norms [T]) after the last Newton iteration."""
        count = len(self._segments) - 1
        done = np.zeros(count, np.int32)
        res = np.zeros(count)
        check(lib().tfiga_ns_segment_status(self._h, _p(done), _p(res)))
        return done, res

    def tangent_kernel(self) -> dict:
        """The tensor-core tangent organisation in use and the autotuner's timings."""
        k = C.c_int32(); a = C.c_double(); b = C.c_double()
        check(lib().tfiga_ns_tangent_kernel(self._h, C.byref(k), C.byref(a), C.byref(b)))
        names = {TANGENT_AUTO: "auto", TANGENT_COEFFICIENTS: "coefficients", TANGENT_FUSED: "fused",
                 TANGENT_ELEMENT: "element"}
        el = C.c_double()
        check(lib().tfiga_ns_tangent_element_ms(self._h, C.byref(el)))
        return {"kernel": names.get(k.value, str(k.value)), "coefficients_ms": a.value, "fused_ms": b.value,
                "element_ms": el.value}

    def amg_info(self) -> dict:
        info = AmgInfo()
        check(lib().tfiga_ns_amg_info(self._h, C.byref(info)))
        return {"levels": info.levels, "nodes": list(info.nodes[:info.levels]),
                "blocks": list(info.blocks[:info.levels]), "transfer_blocks": int(info.transfer_blocks)}

    def profile_bytes(self) -> dict:
        """{family: (algorithmic bytes, moved bytes)} since the last profile reset."""
        n = len(self.FAMILIES)
        b = np.zeros(2 * n)
        check(lib().tfiga_ns_profile_bytes(self._h, _p(b)))
        return {f: (float(b[i]), float(b[n + i])) for i, f in enumerate(self.FAMILIES)}

    def profile(self, reset=False) -> dict:
        ms = np.zeros(len(self.FAMILIES))
        counts = np.zeros(len(self.FAMILIES), np.int64)
        check(lib().tfiga_ns_profile(self._h, _p(ms), _p(counts), int(reset)))
        return {f: (float(ms[i]), int(counts[i])) for i, f in enumerate(self.FAMILIES)}

    def close(self):
        if self._h:
            lib().tfiga_ns_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Learned:
    """Learned FGMRES preconditioner stage of a NavierStokes handle (AMG preconditioner); see tfiga.h."""

    def __init__(self, ns: "NavierStokes", layers: int = 3, seed: int = 0, linear: bool = False):
        self.ns = ns
        self.layers = layers
        self.linear = linear
        self._h = C.c_void_p()
        check(lib().tfiga_learned_create(ns._h, layers, seed, int(linear), C.byref(self._h)))
        p, e, q = C.c_int64(), C.c_int64(), C.c_int32()
        check(lib().tfiga_learned_info(self._h, C.byref(p), C.byref(e), C.byref(q)))
        self.parameter_count, self.elements = int(p.value), int(e.value)

    def pairs(self) -> int:
        p, e, q = C.c_int64(), C.c_int64(), C.c_int32()
        check(lib().tfiga_learned_info(self._h, C.byref(p), C.byref(e), C.byref(q)))
        return int(q.value)

    def attach(self, use=True, collect=False):
        check(lib().tfiga_ns_set_learned(self.ns._h, self._h, int(use), int(collect)))

    def detach(self):
        check(lib().tfiga_ns_set_learned(self.ns._h, None, 0, 0))

    def set_loss(self, error: bool):
        """Train on the FP64 error of the AMG (error=True) or on the residual it leaves (default)."""
        check(lib().tfiga_learned_set_loss(self._h, 1 if error else 0))

    def set_capacity(self, capacity: int):
        check(lib().tfiga_learned_set_capacity(self._h, int(capacity)))

    def fit_scales(self):
        check(lib().tfiga_learned_fit_scales(self._h))

    def fallbacks(self) -> int:
        c = C.c_int64()
        check(lib().tfiga_ns_learned_fallbacks(self.ns._h, C.byref(c)))
        return int(c.value)

    def train(self, steps: int, learning_rate: float = 1e-3) -> float:
        loss = C.c_double()
        check(lib().tfiga_learned_train(self._h, steps, learning_rate, C.byref(loss)))
        return loss.value

    def evaluate(self) -> float:
        loss = C.c_double()
        check(lib().tfiga_learned_evaluate(self._h, C.byref(loss)))
        return loss.value

    def fit_gain(self) -> float:
        g = C.c_double()
        check(lib().tfiga_learned_fit_gain(self._h, C.byref(g)))
        return g.value

    def parameters(self) -> np.ndarray:
        out = np.zeros(self.parameter_count, np.float32)
        check(lib().tfiga_learned_get_parameters(self._h, _p(out)))
        return out

    def set_parameters(self, theta):
        t = np.ascontiguousarray(theta, np.float32)
        assert t.size == self.parameter_count
        check(lib().tfiga_learned_set_parameters(self._h, _p(t)))

    def scales(self) -> np.ndarray:
        out = np.zeros(12)
        check(lib().tfiga_learned_get_scales(self._h, _p(out)))
        return out

    def set_scales(self, scales):
        s = np.ascontiguousarray(scales, np.float64)
        check(lib().tfiga_learned_set_scales(self._h, _p(s)))

    def neighbours(self) -> np.ndarray:
        out = np.zeros((self.elements, 6), np.int32)
        check(lib().tfiga_learned_neighbours(self._h, _p(out)))
        return out

    def forward_device(self, x_ptr: int, o_ptr: int):
        check(lib().tfiga_learned_forward_device(self._h, C.c_void_p(x_ptr), C.c_void_p(o_ptr)))

    def apply_device(self, x_ptr: int, z_ptr: int):
        check(lib().tfiga_learned_apply_device(self._h, C.c_void_p(x_ptr), C.c_void_p(z_ptr)))

    def loss_gradient_device(self, x_ptr: int, t_ptr: int):
        loss = C.c_double()
        grad = np.zeros(self.parameter_count, np.float32)
        check(lib().tfiga_learned_loss_gradient_device(self._h, C.c_void_p(x_ptr), C.c_void_p(t_ptr), C.byref(loss),
                                                        _p(grad)))
        return loss.value, grad

    def save(self, path):
        check(lib().tfiga_learned_save(self._h, str(path).encode()))

    def load(self, path):
        check(lib().tfiga_learned_load(self._h, str(path).encode()))

    def close(self):
        if self._h:
            lib().tfiga_learned_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 -- interpreter shutdown
            pass


def transport_params(**overrides) -> TransportParams:
    p = TransportParams()
    lib().tfiga_transport_default_params(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def read_transport_params(path, **overrides) -> TransportParams:
    """simulation_parameter.txt of a legacy transport case (ReadTransportParameters)."""
    p = transport_params()
    check(lib().tfiga_transport_read_params(str(path).encode(), C.byref(p)))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def resolve_transport_boundaries(labels, reference_velocity, params: TransportParams, case_config=None):
    """(constrained, n0, nplus) of a legacy case: controlmesh.vtk labels, the reference velocity and an
    optional case_config.json (ResolveBoundaryConditions)."""
    labels = np.ascontiguousarray(labels, np.int32)
    vel = np.ascontiguousarray(reference_velocity, np.float64).reshape(-1)
    n = labels.size
    mask = np.zeros(n, np.int32)
    n0 = np.zeros(n)
    nplus = np.zeros(n)
    count = C.c_int64()
    path = None if case_config is None else str(case_config).encode()
    check(lib().tfiga_transport_resolve_boundaries(n, _p(labels), _p(vel), C.byref(params), path, _p(mask),
                                                   _p(n0), _p(nplus), C.byref(count)))
    return mask, n0, nplus


def resolve_flow_boundaries(config_path, labels, reference_velocity, time=0.0, system=None) -> dict:
    """The navier-stokes command's boundary set-up of a simulation_config.json case at `time` (before
    the wall trace): masks, values, labelled pressure tractions and the flow physics."""
    labels = np.ascontiguousarray(labels, np.int32)
    vel = np.ascontiguousarray(reference_velocity, np.float64).reshape(-1)
    n = labels.size
    out = {"velocity_mask": np.zeros(n, np.int32), "velocity": np.zeros(3 * n), "pressure_mask": np.zeros(n, np.int32),
           "pressure": np.zeros(n), "counts": np.zeros(2, np.int64)}
    tl, tv, count = np.zeros(64, np.int32), np.zeros(64), C.c_int32(64)
    physics = np.zeros(5)
    check(lib().tfiga_resolve_flow_boundaries(str(config_path).encode(), None if system is None else system.encode(),
                                              time, n, _p(labels), _p(vel), _p(out["velocity_mask"]),
                                              _p(out["velocity"]), _p(out["pressure_mask"]), _p(out["pressure"]),
                                              _p(out["counts"]), _p(tl), _p(tv), C.byref(count), _p(physics)))
    out["tractions"] = {int(tl[i]): float(tv[i]) for i in range(min(count.value, 64))}
    out["physics"] = physics
    return out


def resolve_legacy_boundaries(labels, reference_velocity, params: TransportParams, case_config=None) -> dict:
    """Every mask and value of a legacy case (ResolveBoundaryConditions): velocity, pressure, transport."""
    labels = np.ascontiguousarray(labels, np.int32)
    vel = np.ascontiguousarray(reference_velocity, np.float64).reshape(-1)
    n = labels.size
    out = {"velocity_mask": np.zeros(n, np.int32), "velocity": np.zeros(3 * n), "pressure_mask": np.zeros(n, np.int32),
           "pressure": np.zeros(n), "transport_mask": np.zeros(n, np.int32), "n0": np.zeros(n),
           "nplus": np.zeros(n), "counts": np.zeros(3, np.int64)}
    path = None if case_config is None else str(case_config).encode()
    check(lib().tfiga_resolve_legacy_boundaries(n, _p(labels), _p(vel), C.byref(params), path,
                                                *[_p(out[k]) for k in ("velocity_mask", "velocity", "pressure_mask",
                                                                       "pressure", "transport_mask", "n0", "nplus",
                                                                       "counts")]))
    return out


def transport_flow_lines(row_offsets, columns, values) -> dict:
    """Host construction of the flow-line preconditioner of a 2x2 block system (tfiga_transport_flow_lines)."""
    ro = np.ascontiguousarray(row_offsets, np.int32)
    co = np.ascontiguousarray(columns, np.int32)
    va = np.ascontiguousarray(values, np.float64)
    n = len(ro) - 1
    lines, count = C.c_int32(), C.c_int64()
    L = lib()
    check(L.tfiga_transport_flow_lines(n, _p(ro), _p(co), _p(va), None, None, None, None, None, C.byref(lines),
                                       C.byref(count)))
    out = {"line_offsets": np.zeros(lines.value + 1, np.int32), "line_nodes": np.zeros(n, np.int32),
           "band_width": np.zeros(lines.value, np.int32), "band_offsets": np.zeros(lines.value, np.int64),
           "factors": np.zeros(count.value)}
    check(L.tfiga_transport_flow_lines(n, _p(ro), _p(co), _p(va), _p(out["line_offsets"]), _p(out["line_nodes"]),
                                       _p(out["band_width"]), _p(out["band_offsets"]), _p(out["factors"]),
                                       C.byref(lines), C.byref(count)))
    return out


class Transport:
    """Two-species transport solver (tfiga_transport): the `iga_cuda transport` path."""

    def __init__(self, mesh: Mesh, params: TransportParams, velocity, constrained, n0, nplus):
        self.mesh = mesh
        self.params = params
        n = mesh.nodes
        self._velocity = np.ascontiguousarray(velocity, np.float64).reshape(-1)
        self._mask = np.ascontiguousarray(constrained, np.int32).reshape(-1)
        self._n0 = np.ascontiguousarray(n0, np.float64).reshape(-1)
        self._nplus = np.ascontiguousarray(nplus, np.float64).reshape(-1)
        if (self._velocity.size != 3 * n or self._mask.size != n or self._n0.size != n
                or self._nplus.size != n):
            raise ValueError("transport inputs must have 3*nodes velocities and nodes mask/values")
        self._h = C.c_void_p()
        check(lib().tfiga_transport_create(mesh._h, C.byref(params), _p(self._velocity), _p(self._mask),
                                           _p(self._n0), _p(self._nplus), C.byref(self._h)))

    def step(self, steps: int = 1) -> dict:
        r = TransportReport()
        check(lib().tfiga_transport_step(self._h, steps, C.byref(r)))
        return r.as_dict()

    def set_state(self, state):
        s = np.ascontiguousarray(state, np.float64).reshape(-1)
        if s.size != 2 * self.mesh.nodes:
            raise ValueError("state must have 2*nodes entries")
        check(lib().tfiga_transport_set_state(self._h, _p(s)))

    def get_state(self, out=None):
        out = np.zeros(2 * self.mesh.nodes) if out is None else out
        check(lib().tfiga_transport_get_state(self._h, _p(out)))
        return out

    def matrices(self):
        left = np.zeros(4 * self.mesh.blocks)
        previous = np.zeros(4 * self.mesh.blocks)
        check(lib().tfiga_transport_matrices(self._h, _p(left), _p(previous)))
        return left, previous

    def apply_preconditioner(self, x):
        """y = M^{-1} x with the handle's flow-line factors (TRANSPORT_FLOW_LINES handles only)."""
        xs = np.ascontiguousarray(x, np.float64).reshape(-1)
        if xs.size != 2 * self.mesh.nodes:
            raise ValueError("x must have 2*nodes entries")
        y = np.zeros_like(xs)
        check(lib().tfiga_transport_apply_preconditioner(self._h, _p(xs), _p(y)))
        return y

    def info(self) -> dict:
        ms = C.c_double(); steps = C.c_int32(); launches = C.c_int64()
        check(lib().tfiga_transport_info(self._h, C.byref(ms), C.byref(steps), C.byref(launches)))
        return {"assembly_ms": ms.value, "steps": steps.value, "launches": launches.value}

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().tfiga_transport_stream(self._h, C.byref(s)))
        return s.value or 0

    def set_profiling(self, enable: bool):
        check(lib().tfiga_transport_set_profiling(self._h, 1 if enable else 0))

    def profile(self, reset=False) -> dict:
        families = NavierStokes.FAMILIES
        ms = np.zeros(len(families)); counts = np.zeros(len(families), np.int64)
        check(lib().tfiga_transport_profile(self._h, _p(ms), _p(counts), 1 if reset else 0))
        return {f: (float(ms[i]), int(counts[i])) for i, f in enumerate(families)}

    def close(self):
        if self._h:
            lib().tfiga_transport_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def block_residual_norm_static(nodes: int, row_offsets_ptr: int, columns_ptr: int, values_ptr: int, x_ptr: int,
                               b_ptr: int, norm_ptr: int, stream: int = 0):
    """Enqueue ||b - A x||_2 (4x4 block CSR, all device pointers) without allocating; see tfiga.h."""
    check(lib().tfiga_block_residual_norm_static(nodes, C.c_void_p(row_offsets_ptr), C.c_void_p(columns_ptr),
                                                  C.c_void_p(values_ptr), C.c_void_p(x_ptr), C.c_void_p(b_ptr),
                                                  C.c_void_p(norm_ptr), C.c_void_p(stream or None)))


def tube_boundary_conditions(tube, inlet_scale: float):
    """Dirichlet masks/values of a generated tube: wall (label 0) no-slip, inlet (label 1) scaled profile.

    Mirrors ResolveFlowBoundaries (solvers/cpu/include/GenericCaseInput.hpp:174-259) for the generator's
    simulation_config, plus the wall-trace basis, which for the generator tubes is exactly the label-0
    vertex set."""
    labels = tube.labels
    vmask = ((labels == 0) | (labels == 1)).astype(np.int32)
    vel = np.zeros((len(labels), 3))
    inlet = labels == 1
    vel[inlet] = inlet_scale * tube.profile[inlet]
    return vmask, np.zeros(len(labels), np.int32), vel


def batch_boundary_conditions(batch, factors=None):
    """Dirichlet masks/values of a meshgen.TubeBatch: every tube's wall no-slip and its inlet profile
    scaled by its own peak velocity (times factors[k] when given, e.g. a per-tube waveform value)."""
    labels = batch.labels
    vmask = ((labels == 0) | (labels == 1)).astype(np.int32)
    per_tube = batch.inlet_scale if factors is None else batch.inlet_scale * np.asarray(factors, np.float64)
    scale = np.repeat(per_tube, np.diff(batch.node_offset))
    vel = np.zeros((len(labels), 3))
    inlet = labels == 1
    vel[inlet] = scale[inlet, None] * batch.profile[inlet]
    return vmask, np.zeros(len(labels), np.int32), vel


def initial_state(vmask, velocity, pmask=None, pressure=None):
    """Initial state of a transient run (iga_cuda.cu:879-889): constrained values, zero elsewhere."""
    n = len(vmask)
    s = np.zeros((n, 4))
    s[vmask != 0, :3] = np.asarray(velocity).reshape(n, 3)[vmask != 0]
    if pmask is not None and pressure is not None:
        s[pmask != 0, 3] = np.asarray(pressure)[pmask != 0]
    return s.ravel()
