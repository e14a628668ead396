"""Learned FGMRES preconditioner stage.

CPU: the numpy oracle's gradients against finite differences, and its face
adjacency on a generator tube.  GPU: the device forward, loss and parameter
gradients against the oracle (FP32 device arithmetic: 1e-5 on outputs and
loss, 1e-4 relative L2 on the gradient), the device adjacency against the
oracle's, a save/load round trip, and training on the solver's own Newton
pairs followed by the FGMRES iteration count with and without the stage.
"""
import numpy as np
import pytest

from oracle import learned_oracle as L


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def test_oracle_gradient_finite_differences():
    rng = np.random.default_rng(1)
    E, n, H, layers = 10, 30, 8, 2
    conn = rng.integers(0, n, size=(E, 64))
    conn[:, 48:] = -1
    nb = -np.ones((E, 6), int)
    for e in range(E - 1):
        nb[e, 0] = e + 1
        nb[e + 1, 1] = e
    g = L.Graph(conn, nb, n)
    _, total = L.layout(H, layers)
    theta = rng.normal(size=total) * 0.3
    x, t = rng.normal(size=(n, 4)), rng.normal(size=(n, 4))
    w, s = [1.0, 2.0, 0.5, 3.0], [0.7, 1.2, 1.0, 0.3]
    o, cache = L.forward(theta, g, x, s, H, layers)
    grad = L.backward(theta, g, cache, o, t, w, s, H, layers)
    eps = 1e-6
    for k in rng.choice(total, 30, replace=False):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += eps
        tm[k] -= eps
        fd = (L.loss(L.forward(tp, g, x, s, H, layers)[0], t, w) - L.loss(L.forward(tm, g, x, s, H, layers)[0], t, w))
        fd /= 2 * eps
        assert abs(fd - grad[k]) <= 1e-6 * max(abs(fd), abs(grad[k]), 1e-8)


def test_oracle_face_neighbours_on_generator_tube(small_tube):
    flat = small_tube.mesh
    nb = L.face_neighbours(np.asarray(flat.bezier_points).reshape(-1, 64, 3))
    E = flat.elements
    assert nb.shape == (E, 6)
    for e in range(E):
        for f in range(6):
            o = nb[e, f]
            if o >= 0:
                assert e in nb[o]
    counts = (nb >= 0).sum(1)
    # 3 layers: every element has its axial neighbour(s), and the cross-section is connected
    assert counts.min() >= 3 and counts.max() == 6


def _graph_of(flat):
    conn = -np.ones((flat.elements, 64), np.int64)
    for e in range(flat.elements):
        lo, hi = flat.element_offsets[e], flat.element_offsets[e + 1]
        conn[e, :hi - lo] = flat.connectivity[lo:hi]
    nb = L.face_neighbours(np.asarray(flat.bezier_points).reshape(-1, 64, 3))
    return L.Graph(conn, nb, flat.nodes)


@pytest.mark.gpu
def test_learned_forward_gradient_match_oracle(small_tube, tmp_path):
    import torch
    from tubularflowiga_b200 import api
    flat = small_tube.mesh
    mesh = api.Mesh(flat)
    ns = api.NavierStokes(mesh, density=1060.0, viscosity=3.5e-3, dt=1e-3, preconditioner=api.AMG)
    layers = 2
    net = api.Learned(ns, layers=layers, seed=3)
    g = _graph_of(flat)
    assert np.array_equal(net.neighbours(), g.nb)
    rng = np.random.default_rng(7)
    theta = (rng.normal(size=net.parameter_count) * 0.2).astype(np.float32)
    net.set_parameters(theta)
    s_in, s_out, w = np.array([1.3, 0.8, 1.1, 0.02]), np.array([0.5, 0.7, 0.6, 40.0]), np.array([1.0, 2.0, 1.5, 0.3])
    net.set_scales(np.concatenate([s_in, s_out, w]))
    x = rng.normal(size=(flat.nodes, 4))
    t = rng.normal(size=(flat.nodes, 4)) * s_out
    xd = torch.tensor(x.ravel(), dtype=torch.float64, device="cuda")
    td = torch.tensor(t.ravel(), dtype=torch.float64, device="cuda")
    od = torch.zeros_like(xd)
    torch.cuda.synchronize()
    net.forward_device(xd.data_ptr(), od.data_ptr())
    o_ref, cache = L.forward(theta.astype(np.float64), g, x * s_in, s_out, 64, layers)
    assert rel(od.cpu().numpy().reshape(-1, 4), o_ref) < 1e-5
    loss, grad = net.loss_gradient_device(xd.data_ptr(), td.data_ptr())
    loss_ref = L.loss(o_ref, t, w)
    grad_ref = L.backward(theta.astype(np.float64), g, cache, o_ref, t, w, s_out, 64, layers)
    assert abs(loss - loss_ref) <= 1e-5 * loss_ref
    assert rel(grad, grad_ref) < 1e-4
    # save / load round trip
    net.save(tmp_path / "stage.bin")
    other = api.Learned(ns, layers=layers, seed=99)
    other.load(tmp_path / "stage.bin")
    assert np.array_equal(other.parameters(), theta)
    assert np.allclose(other.scales(), np.concatenate([s_in, s_out, w]))


@pytest.mark.gpu
def test_learned_stage_training_and_iterations(cylinder_1280):
    """Train on the solver's own pairs, then count FGMRES iterations with and without the stage.

    The training (residual loss through the bound Jacobian) must lower the loss, the fitted output
    gain must be finite and non-negative, and a step with the stage attached must still converge to
    the same FP64 Newton tolerance (FGMRES's true residual decides; a solve that fails with the stage is redone
    with the AMG alone).  The iteration counts of both runs are reported: on these tubes the stage
    does not lower them."""
    from tubularflowiga_b200 import api
    tube = cylinder_1280
    vmask, pmask, vel = api.tube_boundary_conditions(tube, 0.2)
    s0 = api.initial_state(vmask, vel)
    mesh = api.Mesh(tube.mesh)
    ns = api.NavierStokes(mesh, density=1060.0, viscosity=3.5e-3, dt=1e-3, preconditioner=api.AMG,
                          nonlinear_rtol=1e-8, nonlinear_atol=1e-300, gmres_rtol=1e-8, gmres_max_iterations=1500)
    ns.set_dirichlet(vmask, pmask, vel)
    ns.set_tractions({2: 0.0})
    ns.set_state(s0, s0)
    net = api.Learned(ns, layers=3, seed=0, linear=True)
    net.attach(use=False, collect=True)
    for _ in range(4):
        ns.commit_step()
        ns.step()
    assert net.pairs() >= 8
    net.fit_scales()
    before = net.evaluate()
    net.train(800, 1e-3)
    after = net.evaluate()
    assert after < before
    gain = net.fit_gain()
    assert np.isfinite(gain) and gain >= 0.0
    state = ns.get_state()
    ns.commit_step()
    net.attach(use=False, collect=False)
    base = ns.step()
    ns.set_state(state, state)
    ns.commit_step()
    net.attach(use=True, collect=False)
    learned = ns.step()
    assert base["converged"] and learned["converged"]
    print(f"FGMRES iterations per step: AMG {base['linear_iterations']}, AMG + learned stage "
          f"{learned['linear_iterations']} (residual loss {before:.3e} -> {after:.3e}, gain {gain:.3f}, "
          f"fallbacks {net.fallbacks()})")


@pytest.mark.gpu
def test_learned_stage_on_held_out_steps():
    """The 12,800-element pulsatile section (C2's cross-section and inflow, 100 layers) with the split-BF16
    solver: training pairs from 40 steps (a 1,024-pair store of flexible-GMRES pairs w = A z and Newton
    pairs), the residual loss through the bound Jacobian, 3,000 Adam steps and the fitted output gain; then
    five held-out steps, from the same state and with the same Dirichlet sequence, with and without the
    stage.  Asserted: the trained loss and the output gain are finite, the gain non-negative, and every
    held-out step converges (a solve the stage does not converge is redone with the AMG alone; the
    fallbacks are reported).  Neither the loss reduction nor the iteration counts are asserted: the
    training is not reproducible (one run ended with a loss eight times its start) and the stage does
    not give a reliable gain.  Two runs of this protocol on a
    B200 gave 860, 841, 827, 815, 813 FGMRES iterations per step with the stage against 876, 855, 845,
    831, 831 without (2% fewer), and 1640, 1986, 2058, 2002, 2063 against 876, 858, 844, 831, 831 (2.3
    times more); the training is not deterministic (FP32 atomics in the gradient) and the fitted gain
    (0.068, 0.026) is small either way."""
    import bench
    from tubularflowiga_b200 import api
    tube, _, wave = bench.workload("c2-100")
    mesh = api.Mesh(tube.mesh)
    vmask, pmask, velocity_at = bench.boundary(tube, wave)
    dt = 2e-3
    ns = api.NavierStokes(mesh, precision=api.MIXED_BF16X3, density=1060.0, viscosity=3.5e-3, dt=dt,
                          nonlinear_rtol=1e-8, nonlinear_atol=1e-300, gmres_restart=64, gmres_max_iterations=5000,
                          gmres_rtol=1e-8, preconditioner=api.AMG, amg_coarse_period=3, newton_forcing=1,
                          tangent_reuse_factor=100.0)
    ns.set_dirichlet(vmask, pmask, velocity_at(0.0))
    ns.set_tractions({2: 0.0})
    s0 = api.initial_state(vmask, velocity_at(0.0))
    ns.set_state(s0, s0)
    net = api.Learned(ns, layers=3, seed=0, linear=False)
    net.set_capacity(1024)
    net.set_loss(False)
    net.attach(use=False, collect=True)

    def step(k):
        ns.set_dirichlet_values(velocity_at((k + 1) * dt).ravel())
        ns.commit_step()
        r = ns.step()
        assert r["converged"]
        return r["linear_iterations"]

    for k in range(40):
        step(k)
    net.fit_scales()
    before = net.evaluate()
    net.train(3000, 1e-3)
    after = net.evaluate()
    gain = net.fit_gain()
    # Adam on FP32 atomics is not reproducible and may end above its start on these pairs; the fitted
    # output gain (least squares over the stored pairs, at least 0) is what keeps the stage harmless
    assert np.isfinite(after) and np.isfinite(gain) and gain >= 0.0
    state = ns.get_state()
    counts = {}
    for use in (False, True):
        ns.set_state(state, state)
        net.attach(use=use, collect=False)
        counts[use] = [step(k) for k in range(40, 45)]
    print(f"held-out FGMRES iterations per step: AMG {counts[False]}, AMG + learned stage {counts[True]} "
          f"(residual loss {before:.3e} -> {after:.3e}, gain {gain:.3f}, fallbacks {net.fallbacks()})")
    # a held-out solve the stage does not converge is redone with the AMG alone (every step above
    # converged); the number of such fallbacks is reported with the counts
    net.detach()
    ns.close()
