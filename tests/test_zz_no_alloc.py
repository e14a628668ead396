"""The allocation-free residual-norm entry point (tfiga_block_residual_norm_static).

Its result is checked against the library's allocating entry point
tfiga_ns_spmv_device (y = A x on the handle's assembled Jacobian) followed by
||b - y||_2, on two calls in a row; the two calls must agree bitwise (fixed
summation order, shared static scratch).  This file runs last so the static
scratch is exercised after every other test has used the device.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _assembled_handle():
    from tubularflowiga_b200 import api, meshgen
    tube = meshgen.straight_tube(1.5e-3, 6e-3, core=4, ring=1, layers=3)
    flat = tube.mesh
    mesh = api.Mesh(flat)
    ns = api.NavierStokes(mesh, density=1060.0, viscosity=3.5e-3, dt=1e-3)
    rng = np.random.default_rng(11)
    state = (rng.normal(size=(flat.nodes, 4)) * [0.2, 0.2, 0.2, 20.0]).ravel()
    ns.set_state(state, state)
    ns.assemble()
    return mesh, ns, flat.nodes


def test_static_residual_norm_matches_spmv_entry_point():
    import torch
    from tubularflowiga_b200 import api
    mesh, ns, nodes = _assembled_handle()
    values_ptr, _, _ = ns.device_buffers()
    ro, cols, _ = mesh.pattern()
    dev = torch.device("cuda", 0)
    ro_d = torch.from_numpy(ro).to(dev)
    cols_d = torch.from_numpy(cols).to(dev)
    g = torch.Generator(device=dev).manual_seed(5)
    x = torch.randn(4 * nodes, dtype=torch.float64, device=dev, generator=g)
    b = torch.randn(4 * nodes, dtype=torch.float64, device=dev, generator=g)
    y = torch.zeros_like(x)
    torch.cuda.synchronize()
    ns.spmv_device(x.data_ptr(), y.data_ptr())
    ns.synchronize()
    expected = torch.linalg.norm(b - y).item()

    norms = torch.full((2,), -1.0, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for k in range(2):
        api.block_residual_norm_static(nodes, ro_d.data_ptr(), cols_d.data_ptr(), values_ptr, x.data_ptr(),
                                       b.data_ptr(), norms[k:].data_ptr(), stream)
    torch.cuda.synchronize()
    got = norms.cpu().numpy()
    assert got[0] == got[1]
    assert abs(got[0] - expected) <= 1e-12 * expected


def test_static_residual_norm_rejects_oversize():
    from tubularflowiga_b200 import api
    with pytest.raises(api.TfigaError, match="262144"):
        api.block_residual_norm_static(262145, 16, 16, 16, 16, 16, 16, 0)
