"""The oracle adjoint (forward-mode tangent of the oracle step, dem_tangent.cpp):
its trajectory equals the oracle's bit for bit, and its derivatives equal
central finite differences of the FP64 oracle where the differences cross
no branch change."""
import math

import numpy as np
import pytest

from adjoint_harness import central_fd, f64_loss, tangent_grad, with_params
from demso_b200 import scenes
from oracle.oracle import PortOracle, TangentOracle


def slope_scene(n, seed=3):
    a = math.radians(20.0)
    return scenes.agitated_gas(n=n, seed=seed, pitch_factor=0.97, jitter=0.08, vel_std=0.05,
                               omega_std=20.0,
                               gravity=(9.81 * math.sin(a), -9.81 * math.cos(a)))


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_tangent_trajectory_is_the_oracle_trajectory(prec):
    sc = slope_scene(300)
    sys = with_params(sc, 1e5, 0.3, 0.5)
    o = PortOracle(prec).run(sys, sc.state(), 40)
    t = TangentOracle(prec).run(sys, sc.state(), 40)
    assert o["signature"] == t["signature"]
    assert np.array_equal(o["id"], t["id"])
    for k in ("pos", "vel", "omega", "theta"):
        assert np.array_equal(o[k].astype(np.float64), t[k]), k


def test_tangent_refuses_attraction():
    sc = scenes.agitated_gas(n=64, seed=1, attraction=10.0)
    with pytest.raises(ValueError):
        TangentOracle("f64").run(sc.sys, sc.state(), 1)


def test_tangent_matches_fp64_central_differences():
    sc = slope_scene(120)
    steps = 60
    u = np.random.default_rng(1).normal(size=(sc.n, 2))
    loss, d, sig = tangent_grad(sc, 1e5, 0.3, 0.5, steps, u)
    assert loss == f64_loss(sc, 1e5, 0.3, 0.5, steps)[0]
    v0 = sc.vel.astype(np.float64)[np.argsort(sc.id)]
    funs = ((1e5, lambda x: f64_loss(sc, x, 0.3, 0.5, steps)),
            (0.3, lambda x: f64_loss(sc, 1e5, x, 0.5, steps)),
            (0.5, lambda x: f64_loss(sc, 1e5, 0.3, x, steps)),
            (0.0, lambda e: f64_loss(sc, 1e5, 0.3, 0.5, steps, vel0=(v0 + e * u)[sc.id])))
    checked = 0
    for k, (x0, f) in enumerate(funs):
        h = 1e-4 * x0 if x0 else 5e-6
        fd, same = central_fd(f, x0, h)
        if not same:
            continue
        checked += 1
        assert abs(d[k] - fd) <= 1e-6 * abs(fd), (k, d[k], fd)
    assert checked >= 3


def test_tangent_of_a_free_flight_is_exact():
    """No contact anywhere: x(T) = x0 + T v0 + g-terms, so dL/dv0 . u is the
    closed form sum over disks and the coefficient derivatives vanish."""
    sc = scenes.agitated_gas(n=16, seed=2, pitch_factor=3.0, jitter=0.0, vel_std=0.01,
                             omega_std=0.0, gravity=(0.0, 0.0))
    steps = 10
    u = np.zeros((sc.n, 2))
    u[:, 0] = 1.0
    loss, d, _ = tangent_grad(sc, 1e5, 0.3, 0.5, steps, u)
    assert d[0] == 0.0 and d[1] == 0.0 and d[2] == 0.0
    dt = sc.sys.dt
    m = sc.mass[np.argsort(sc.id)].astype(np.float64)
    v = sc.vel[np.argsort(sc.id)].astype(np.float64)
    expect = steps * dt + np.sum(m * v[:, 0])
    assert abs(d[3] - expect) <= 1e-9 * abs(expect)
