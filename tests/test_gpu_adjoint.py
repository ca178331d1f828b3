"""Adjoint (dem_adj_forward / dem_adj_backward) against the oracle adjoint
(forward-mode tangent of the oracle step) and central finite differences of
the FP64 oracle; checkpoint-independence; the torch.autograd.Function.

Tolerances: against the FP32 tangent -- the same float trajectory the GPU
forward follows bit for bit -- 1e-3 relative on every checked derivative;
against FP64 central differences (h = 1e-4 relative) and the FP64 tangent,
1e-3 relative on windows short enough that the float and double
trajectories stay together."""
import math

import numpy as np
import pytest

from adjoint_harness import (AdjointLoss, central_fd, f64_loss, gpu_loss_and_grad,
                             tangent_grad)
from demso_b200 import scenes

pytestmark = pytest.mark.gpu

KN, ZETA, MU = 1e5, 0.3, 0.5


def slope_scene(n=480, seed=3):
    """Dense agitated disks under gravity rotated by 20 degrees: contacts
    with dashpot, stick and slip throughout, walls and floor active."""
    a = math.radians(20.0)
    return scenes.agitated_gas(n=n, seed=seed, pitch_factor=0.97, jitter=0.08, vel_std=0.05,
                               omega_std=20.0,
                               gravity=(9.81 * math.sin(a), -9.81 * math.cos(a)))


def gpu_directional(sc, steps, every, u):
    loss, (dkn, dz, dmu), dv, g = gpu_loss_and_grad(sc, KN, ZETA, MU, steps, every)
    return loss, (dkn, dz, dmu, float(np.sum(dv.astype(np.float64) * u))), dv, g


def rel(a, b):
    return abs(a - b) / abs(b)


def test_checkpointing_does_not_change_the_gradient():
    sc = slope_scene()
    a = gpu_loss_and_grad(sc, KN, ZETA, MU, 120, 120)
    b = gpu_loss_and_grad(sc, KN, ZETA, MU, 120, 25)
    c = gpu_loss_and_grad(sc, KN, ZETA, MU, 120, 7)
    assert a[0] == b[0] == c[0]
    assert a[3] == b[3] == c[3]
    assert np.array_equal(a[2], b[2]) and np.array_equal(a[2], c[2])


def test_gpu_loss_is_the_float_oracle_loss():
    sc = slope_scene()
    u = np.zeros((sc.n, 2))
    loss, _, _ = tangent_grad(sc, KN, ZETA, MU, 150, u, "f32")
    assert gpu_loss_and_grad(sc, KN, ZETA, MU, 150, 50)[0] == loss


@pytest.mark.parametrize("n,steps,every", [(480, 150, 50), (1024, 300, 100)])
def test_adjoint_matches_the_float_tangent(n, steps, every):
    sc = slope_scene(n)
    u = np.random.default_rng(7).normal(size=(sc.n, 2))
    _, d_gpu, _, g = gpu_directional(sc, steps, every, u)
    _, d_tan, _ = tangent_grad(sc, KN, ZETA, MU, steps, u, "f32")
    assert all(np.isfinite(g))
    for k in range(4):
        assert rel(d_gpu[k], d_tan[k]) < 1e-3, (k, d_gpu[k], d_tan[k])


def test_adjoint_matches_fp64_central_differences():
    sc = slope_scene(160, seed=4)
    steps = 60
    u = np.random.default_rng(3).normal(size=(sc.n, 2))
    _, d_gpu, _, _ = gpu_directional(sc, steps, 20, u)
    _, d64, _ = tangent_grad(sc, KN, ZETA, MU, steps, u, "f64")
    v0 = sc.vel.astype(np.float64)[np.argsort(sc.id)]
    funs = ((KN, lambda x: f64_loss(sc, x, ZETA, MU, steps)),
            (ZETA, lambda x: f64_loss(sc, KN, x, MU, steps)),
            (MU, lambda x: f64_loss(sc, KN, ZETA, x, steps)),
            (0.05, lambda e: f64_loss(sc, KN, ZETA, MU, steps,
                                      vel0=(v0 + (e - 0.05) * u)[sc.id])))
    for k, (x0, f) in enumerate(funs):
        fd, same = central_fd(f, x0, 1e-4 * x0)
        assert rel(d_gpu[k], d64[k]) < 1e-3, (k, d_gpu[k], d64[k])
        if same:
            assert rel(d_gpu[k], fd) < 1e-3, (k, d_gpu[k], fd)


def test_single_velocity_components():
    sc = slope_scene(480)
    steps = 150
    _, _, dv, _ = gpu_loss_and_grad(sc, KN, ZETA, MU, steps, 50)
    rng = np.random.default_rng(0)
    picks = rng.choice(sc.n, size=4, replace=False)
    scale = np.abs(dv).max()
    for p in picks:
        u = np.zeros((sc.n, 2))
        u[p, 0] = 1.0
        _, d, _ = tangent_grad(sc, KN, ZETA, MU, steps, u, "f32")
        assert abs(dv[p, 0] - d[3]) <= 1e-3 * max(abs(d[3]), 1e-2 * scale), (p, dv[p, 0], d[3])


def test_autograd_function_wraps_the_adjoint():
    import torch
    sc = slope_scene(n=300, seed=5)
    F = AdjointLoss.make(sc, 80, 40)
    kn = torch.tensor(KN, dtype=torch.float64, requires_grad=True)
    z = torch.tensor(ZETA, dtype=torch.float64, requires_grad=True)
    mu = torch.tensor(MU, dtype=torch.float64, requires_grad=True)
    order = np.argsort(sc.id)
    v0 = torch.from_numpy(sc.vel[order].copy()).requires_grad_(True)
    loss = F.apply(kn, z, mu, v0)
    loss.backward()
    ref = gpu_loss_and_grad(sc, KN, ZETA, MU, 80, 40)
    assert float(loss) == ref[0]
    assert float(kn.grad) == ref[1][0] and float(z.grad) == ref[1][1]
    assert float(mu.grad) == ref[1][2]
    assert np.array_equal(v0.grad.numpy(), ref[2])


def test_adjoint_rejects_what_it_does_not_differentiate():
    import torch
    import demso_b200 as D
    sc = scenes.agitated_gas(n=256, seed=1, attraction=10.0)
    sim = D.Simulation(sc.sys, capacity=sc.n)
    sim.set_state(*(torch.from_numpy(np.ascontiguousarray(a)) for a in
                    (sc.pos, sc.vel, sc.theta, sc.omega, sc.radius, sc.mass,
                     sc.id.view(np.int32))))
    L = D.load()
    stream = torch.cuda.current_stream().cuda_stream
    assert L.dem_adj_forward(sim.handle, 10, 5, stream) == 1  # DEM_ERR_INVALID_ARG
    sim.close()


def test_backward_refuses_particles_replaced_after_the_forward():
    """The backward restores the forward's checkpoints without re-deriving
    the culling bound, so a state with a larger radius set in between is
    refused; the same particles set again are not."""
    import torch
    import demso_b200 as D
    sc = scenes.agitated_gas(n=512, seed=3)
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_ACCEL)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).copy())
    state = lambda r: (t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(r), t(sc.mass),
                       t(sc.id.view(np.int32)))
    L = D.load()
    stream = torch.cuda.current_stream().cuda_stream
    lam = [torch.zeros(k, dtype=torch.float32, device="cuda") for k in (2 * sc.n, 2 * sc.n, sc.n)]
    sim.set_state(*state(sc.radius))
    sim.adjoint_forward(20, 7)
    sim.set_state(*state(sc.radius * np.float32(1.5)))
    with pytest.raises(D.DemError):
        sim.adjoint_backward(*lam)
    sim.set_state(*state(sc.radius))
    sim.adjoint_forward(20, 7)
    sim.set_state(*state(sc.radius))
    g = sim.adjoint_backward(*lam)
    assert np.all(np.isfinite(g))
    sim.close()


def test_batched_adjoint_equals_each_specimen_alone():
    """Three specimens of different sizes and contact parameters in one
    batch: the state cotangents equal each specimen's own adjoint bit for
    bit, and the per-specimen coefficient gradients agree to FP64 rounding
    (the double sums run over differently aligned warps)."""
    from adjoint_harness import batch_adjoint, single_adjoint, with_params
    items = []
    for n, seed, kn, zeta, mu in ((300, 11, 1e5, 0.3, 0.5), (450, 12, 2e5, 0.2, 0.7),
                                  (200, 13, 6e4, 0.4, 0.3)):
        sc = slope_scene(n, seed=seed)
        items.append((with_params(sc, kn, zeta, mu), sc))
    g, per = batch_adjoint(items, 90, 30)
    for s, (sys, sc) in enumerate(items):
        g1, (dp, dv, dw) = single_adjoint(sys, sc, 90, 30)
        assert np.array_equal(per[s][0], dp) and np.array_equal(per[s][1], dv)
        assert np.array_equal(per[s][2], dw)
        assert np.allclose(g[s], g1, rtol=1e-12, atol=0.0), (s, g[s], g1)
        assert np.any(g1 != 0.0)


def test_repeated_backward_calls_reuse_their_loops_exactly():
    """dem_adj_backward keeps its record, scratch and loops in the context:
    later calls (same cotangent buffers, other buffers, after a forward with
    another checkpoint interval) give the first call's gradients bit for
    bit."""
    import ctypes as C
    import torch
    import demso_b200 as D
    from adjoint_harness import NUM_COEF
    sc = slope_scene(480)
    steps = 90
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a))
    sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass),
                  t(sc.id))
    L = D.load()
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(5)
    seeds = [torch.from_numpy(rng.normal(size=s).astype(np.float32)).cuda()
             for s in ((sc.n, 2), (sc.n, 2), (sc.n,))]

    def backward(bufs):
        for b, s in zip(bufs, seeds):
            b.copy_(s)
        grad = (C.c_double * NUM_COEF)()
        D.check(L.dem_adj_backward(sim.handle, *(b.data_ptr() for b in bufs), grad, stream))
        torch.cuda.synchronize()
        return list(grad), [b.cpu().numpy() for b in bufs]

    def same_result(a, b):
        assert a[0] == b[0]
        for x, y in zip(a[1], b[1]):
            assert np.array_equal(x, y)

    def restart(every):
        sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius),
                      t(sc.mass), t(sc.id))
        D.check(L.dem_adj_forward(sim.handle, steps, every, stream))

    bufs_a = [torch.empty_like(s) for s in seeds]
    bufs_b = [torch.empty_like(s) for s in seeds]
    restart(30)
    first = backward(bufs_a)
    assert all(np.isfinite(first[0]))
    same_result(first, backward(bufs_a))
    same_result(first, backward(bufs_b))
    restart(20)
    same_result(first, backward(bufs_a))
    sim.check()
    sim.close()
