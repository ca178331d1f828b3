"""The control particle on the GPU (dem_set_control / dem_get_control)
against the oracle's restatement of the reference with USE_BIG_PARTICLE 1:
trajectories, the per-step reaction sums and the control particle's motion,
bit for bit; removing it restores the plain step."""
import math

import numpy as np
import pytest

from demso_b200 import scenes
from helpers import gpu_run, same
from oracle.oracle import PortOracle, orc_control

pytestmark = pytest.mark.gpu


def _sim(sc):
    import torch
    import demso_b200 as D
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a))
    st = sc.state()
    sim.set_state(t(st["pos"]), t(st["vel"]), t(st["theta"]), t(st["omega"]), t(st["radius"]),
                  t(st["mass"]), t(st["id"]), t(st["type"]) if st["type"] is not None else None)
    return sim


@pytest.mark.parametrize("kind", ["plain", "typed"])
def test_control_particle_matches_the_oracle(kind):
    if kind == "typed":
        sc = scenes.agitated_gas(n=3000, seed=71, n_mat=3, attraction=15.0, vel_std=0.3)
        mat = 2
    else:
        sc = scenes.agitated_gas(n=4000, seed=72, vel_std=0.3)
        mat = 0
    L = sc.sys.Lx
    c = dict(pos=(0.5 * L, 0.5 * sc.sys.Ly), vel=(0.0, 0.0), theta=0.0, omega=2.0,
             radius=5e-3, mat=mat, drift=(2e-5, -5e-5),
             wrap_y=(0.2 * sc.sys.Ly, 0.8 * sc.sys.Ly),
             wrap_x=(float(np.float32(L)) + 0.5, -0.5))
    steps = 120
    sim = _sim(sc)
    sim.set_control(c["pos"], c["radius"], material=mat, vel=c["vel"], theta=c["theta"],
                    omega=c["omega"], drift=c["drift"], wrap_y=c["wrap_y"], wrap_x=c["wrap_x"])
    reactions, positions = [], []
    for _ in range(steps):
        sim.step(1)
        p, r = sim.control()
        reactions.append(r)
        positions.append(p)
    st = {k: (None if v is None else (v.numpy().view(np.uint32) if k in ("id", "type", "loc")
                                      else v.numpy())) for k, v in sim.get_state("cpu").items()}
    sim.close()
    oc = orc_control(c)
    ref, reac = PortOracle("f32").run_control(sc.sys, sc.state(), steps, oc)
    for k in ("pos", "vel", "theta", "omega", "id"):
        assert same(st[k], ref[k]), k
    assert np.array_equal(np.array(reactions, np.float32), reac)
    assert np.count_nonzero(reac[:, 0]) > steps // 2
    assert positions[-1] == (np.float32(oc.pos[0]), np.float32(oc.pos[1]))


def test_removing_the_control_particle_restores_the_plain_step():
    sc = scenes.agitated_gas(n=2000, seed=73, vel_std=0.3)
    sim = _sim(sc)
    sim.set_control((0.5 * sc.sys.Lx, 0.5 * sc.sys.Ly), 4e-3)
    sim.step(5)
    sim.set_control(None, 0)
    sim.step(20)
    a = {k: v.numpy() for k, v in sim.get_state("cpu").items() if v is not None}
    sim.close()
    sim = _sim(sc)
    sim.set_control((0.5 * sc.sys.Lx, 0.5 * sc.sys.Ly), 4e-3)
    sim.step(5)
    st = {k: v for k, v in sim.get_state("cpu").items() if v is not None}
    sim.close()
    mid = {k: (v.numpy().view(np.uint32) if k in ("id",) else v.numpy()) for k, v in st.items()
           if k in ("pos", "vel", "theta", "omega", "radius", "mass", "id")}
    mid["type"] = None
    b = gpu_run(sc.sys, mid, 20)
    for k in ("pos", "vel", "theta", "omega"):
        assert same(a[k], b[k]), k


def test_control_particle_rejections():
    import demso_b200 as D
    sc = scenes.agitated_gas(n=500, seed=74)
    sim = _sim(sc)
    with pytest.raises(D.DemError):
        sim.set_control((0.01, 0.01), 4e-3, material=1)      # one material: only 0
    with pytest.raises(D.DemError):
        sim.set_control((0.01, 0.01), -1.0)
    with pytest.raises(D.DemError):
        sim.control()                                       # none set
    sim.close()


def test_set_control_is_ordered_on_the_callers_stream():
    """Steps queued on a side stream (torch streams are non-blocking), then a
    new control particle set on that stream while they may still run, then
    more steps: the result equals the same sequence on the default stream."""
    import torch
    sc = scenes.agitated_gas(n=200000, seed=73, vel_std=0.3)
    L = sc.sys.Lx
    first = dict(pos=(0.3 * L, 0.5 * sc.sys.Ly), radius=5e-3, material=0, omega=1.0)
    second = dict(pos=(0.7 * L, 0.4 * sc.sys.Ly), radius=8e-3, material=0, omega=-3.0)

    def run(stream):
        sim = _sim(sc)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            sim.set_control(**first)
            sim.step(1)
            sim.step(200)
            sim.set_control(**second)
            sim.step(20)
            p, r = sim.control()
        stream.synchronize()
        st = {k: (None if v is None else v.numpy()) for k, v in sim.get_state("cpu").items()}
        sim.close()
        return st, p, r

    a = run(torch.cuda.current_stream())
    b = run(torch.cuda.Stream())
    for k in ("pos", "vel", "theta", "omega", "id"):
        assert same(a[0][k], b[0][k]), k
    assert np.array_equal(np.asarray(a[1], np.float32), np.asarray(b[1], np.float32))
    assert np.array_equal(np.asarray(a[2], np.float32), np.asarray(b[2], np.float32))
