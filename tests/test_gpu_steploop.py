"""The device-side step loop: a multi-step dem_step runs its steps in pairs
inside one graph launch (a WHILE node over two captured steps).  It must give
the same bits as stepping one call at a time -- on a quiet pile, on a hot gas
whose movers overflow the incremental sort (the full sort then runs inside
the loop's body), for a batch, with odd step counts and from either parity."""
import numpy as np
import pytest

from demso_b200 import scenes
from helpers import same

pytestmark = pytest.mark.gpu

KEYS = ("pos", "vel", "theta", "omega", "radius", "mass", "id", "pressure", "acc", "alpha")


def _torch(a):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.int32).copy() if a.dtype == np.uint32 else a.copy())


def run(make, chunks, batch=None):
    import torch
    import demso_b200 as D
    flags = D.CTX_PRESSURE | D.CTX_ACCEL
    if batch is None:
        sc = make()
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=flags)
        st = sc.state()
    else:
        sim = D.Batch([(s.sys, s.n) for s in batch], flags=flags)
        st = scenes.concat_specimens(batch)
    sim.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]),
                  _torch(st["omega"]), _torch(st["radius"]), _torch(st["mass"]),
                  _torch(st["id"]), _torch(st["type"]) if st["type"] is not None else None)
    for c in chunks:
        sim.step(c)
    torch.cuda.synchronize()
    out = {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                       else v.numpy())) for k, v in sim.get_state("cpu").items()}
    sim.check()
    sim.close()
    return out


def _same_run(a, b):
    for k in KEYS:
        if a[k] is None:
            assert b[k] is None, k
        else:
            assert same(a[k], b[k]), k


@pytest.mark.parametrize("name,make,chunks", [
    ("pile", lambda: scenes.settling_pile(side=40, box=0.12, seed=4, vel_std=0.3), [61]),
    ("pile_odd_start", lambda: scenes.settling_pile(side=40, box=0.12, seed=4, vel_std=0.3),
     [1, 2, 27, 31]),
    ("hot_gas", lambda: scenes.agitated_gas(n=20000, seed=4, vel_std=300.0, omega_std=500.0),
     [40]),
    ("materials", lambda: scenes.agitated_gas(n=3000, seed=7, n_mat=3, attraction=25.0), [33]),
])
def test_loop_equals_single_steps(name, make, chunks):
    total = sum(chunks)
    _same_run(run(make, [1] * total), run(make, chunks))


def test_loop_equals_single_steps_for_a_batch():
    batch = scenes.specimen_batch(num=10, seed=8, nmin=64, nmax=2048)
    _same_run(run(None, [1] * 50, batch=batch), run(None, [3, 47], batch=batch))
