"""The C-ABI library loads and exports every symbol include/tfiga.h declares (no GPU needed)."""
import ctypes
import re
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT


def header_symbols():
    text = (ROOT / "include" / "tfiga.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tfiga_[a-z_0-9]+)\s*\(", text)))


@pytest.fixture(scope="module")
def library():
    from tubularflowiga_b200 import api, build
    build.build()
    return api.lib()


def test_header_symbols_exported(library):
    from tubularflowiga_b200 import api
    symbols = header_symbols()
    assert len(symbols) >= 25
    for name in symbols:
        assert hasattr(library, name), name
        assert name in api.SIGNATURES, name
    out = subprocess.run(["nm", "-D", "--defined-only", str(api.LIBRARY)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (tfiga_[a-z_0-9]+)", out))
    assert set(symbols) <= exported


def test_library_targets_sm100a(library):
    from tubularflowiga_b200 import api
    assert b"sm_100a" in library.tfiga_version()
    assert api.LIBRARY.stat().st_size > 100_000


def test_default_params(library):
    from tubularflowiga_b200 import api
    p = api.default_params()
    assert (p.max_newton, p.nonlinear_rtol, p.nonlinear_atol, p.mass_rtol) == (12, 1e-5, 1e-10, 1e-3)
    assert (p.gmres_restart, p.gmres_max_iterations, p.gmres_rtol) == (200, 5000, 1e-8)


def test_errors_cross_the_abi_as_status(library):
    from tubularflowiga_b200 import api
    h = ctypes.c_void_p()
    status = library.tfiga_mesh_load_ntiga(b"/nonexistent.ntiga", ctypes.byref(h))
    assert status in (-2, -3)          # no device here, or the file is missing
    assert api.last_error()
    assert library.tfiga_ns_step(None, None) == -1


def test_no_cpu_fallback_without_device(library):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from tubularflowiga_b200 import api, meshgen
    tube = meshgen.straight_tube(1e-3, 2e-3, 4, 1, 1)
    with pytest.raises(api.TfigaError) as err:
        api.Mesh(tube.mesh)
    assert err.value.status == -2 and "no CPU fallback" in str(err.value)
    assert np.all(np.isfinite(tube.mesh.bezier_points))


def test_batch_mesh_offsets_before_device(library):
    """tfiga_batch_mesh_create builds the union (and its offsets) on the host before it needs the
    device; without one it reports TFIGA_E_CUDA."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from tubularflowiga_b200 import api, meshgen
    tubes = [meshgen.straight_tube(1e-3, 2e-3, 4, 1, k) for k in (1, 2, 3)]
    meshes = [t.mesh.contiguous() for t in tubes]
    descs = (api.MeshDesc * 3)(*[api.MeshDesc(m.nodes, m.elements, api._p(m.element_offsets),
                                              api._p(m.connectivity), api._p(m.extraction_offsets),
                                              api._p(m.extraction_columns), api._p(m.extraction_values),
                                              api._p(m.bezier_points), api._p(m.boundary_labels)) for m in meshes])
    nodes = np.full(4, -1, np.int64)
    elements = np.full(4, -1, np.int64)
    h = ctypes.c_void_p()
    status = library.tfiga_batch_mesh_create(descs, 3, ctypes.byref(h), api._p(nodes), api._p(elements))
    assert status == -2 and "no CPU fallback" in api.last_error()
    assert list(nodes) == [0] + list(np.cumsum([m.nodes for m in meshes]))
    assert list(elements) == [0] + list(np.cumsum([m.elements for m in meshes]))
    assert library.tfiga_batch_mesh_create(descs, 0, ctypes.byref(h), None, None) == -1
