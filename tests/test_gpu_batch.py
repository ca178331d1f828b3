"""Batched form (dem_batch_create): every specimen of a batch evolves bit for
bit as it would alone -- checked against the CPU oracle run on each specimen
separately, and against the single-scene context on the GPU."""
import numpy as np
import pytest

from helpers import same
from oracle.oracle import PortOracle
from demso_b200 import scenes

pytestmark = pytest.mark.gpu

KEYS = ["pos", "vel", "theta", "omega", "pressure", "acc", "alpha"]


def _torch(a):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a.copy())


def run_batch(specimens, steps):
    import torch
    import demso_b200 as D
    b = D.Batch([(sc.sys, sc.n) for sc in specimens], flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    st = scenes.concat_specimens(specimens)
    b.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]), _torch(st["omega"]),
                _torch(st["radius"]), _torch(st["mass"]), _torch(st["id"]),
                _torch(st["type"]) if st["type"] is not None else None)
    b.step(steps)
    torch.cuda.synchronize()
    out = {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                       else v.numpy())) for k, v in b.get_state("cpu").items()}
    ranges = [b.slots(s) for s in range(len(specimens))]
    b.check()
    b.close()
    return out, ranges


def mixed_specimens():
    out = []
    out.append(scenes.agitated_gas(n=700, seed=51))
    out.append(scenes.agitated_gas(n=300, seed=52, grid="ref", vel_std=1.0))
    out.append(scenes.settling_pile(side=24, box=0.06, seed=53, vel_std=0.3))
    out.append(scenes.agitated_gas(n=1200, seed=54, dt=1e-6))
    out.append(scenes.agitated_gas(n=90, seed=55, grid=(2, 2)))
    sc = scenes.agitated_gas(n=500, seed=56, gravity=(1.5, -9.0))
    sc.sys.materials[0].frictionCoefficient = 0.9
    out.append(sc)
    return out


@pytest.mark.parametrize("steps", [1, 60])
def test_batch_specimens_match_oracle_alone(steps):
    specimens = mixed_specimens()
    out, ranges = run_batch(specimens, steps)
    po = PortOracle("f32")
    for sc, (a, b) in zip(specimens, ranges):
        assert b - a == sc.n
        ref = po.run(sc.sys, sc.state(), steps)
        for k in KEYS:
            assert same(out[k][a:b], ref[k]), (sc.name, k)
        assert np.array_equal(out["id"][a:b] - a, ref["id"]), sc.name
        assert np.array_equal(out["loc"][a:b] - a, ref["loc"]), sc.name


def test_batch_multi_material_matches_oracle():
    specimens = [scenes.agitated_gas(n=400, seed=61, n_mat=3),
                 scenes.agitated_gas(n=350, seed=62),
                 scenes.agitated_gas(n=500, seed=63, n_mat=2)]
    out, ranges = run_batch(specimens, 40)
    po = PortOracle("f32")
    for sc, (a, b) in zip(specimens, ranges):
        st = sc.state()
        if st["type"] is None:
            st["type"] = np.zeros(sc.n, np.uint32)
        ref = po.run(sc.sys, st, 40)
        for k in KEYS:
            assert same(out[k][a:b], ref[k]), (sc.name, k)


def test_generated_batch_matches_single_scene_contexts():
    from helpers import gpu_run
    specimens = scenes.specimen_batch(num=24, seed=3, nmin=64, nmax=2048)
    out, ranges = run_batch(specimens, 120)
    for sc, (a, b) in zip(specimens, ranges):
        ref = gpu_run(sc.sys, sc.state(), 120)
        for k in KEYS:
            assert same(out[k][a:b], ref[k]), (sc.name, k)


def test_set_systems_is_ordered_on_the_callers_stream():
    """Batch steps queued on a side stream, new specimen parameters set on
    that stream while they may still run, then more steps: the result equals
    the same sequence on the default stream, and differs from never changing
    the parameters."""
    import copy
    import torch
    import demso_b200 as D
    specimens = scenes.specimen_batch(num=64, seed=5, nmin=2048, nmax=8192)
    st = scenes.concat_specimens(specimens)
    changed = []
    for sc in specimens:
        s = copy.deepcopy(sc.sys)
        s.materials[0].normalStiffness *= 3.0
        s.gravity = (2.0, -9.81)
        changed.append(s)

    def run(stream, change=True):
        b = D.Batch([(sc.sys, sc.n) for sc in specimens], flags=D.CTX_PRESSURE)
        b.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]),
                    _torch(st["omega"]), _torch(st["radius"]), _torch(st["mass"]),
                    _torch(st["id"]))
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            b.step(1)
            b.step(300)
            if change:
                b.set_systems(changed)
            b.step(30)
        stream.synchronize()
        out = {k: (None if v is None else v.numpy()) for k, v in b.get_state("cpu").items()}
        b.close()
        return out

    a = run(torch.cuda.current_stream())
    c = run(torch.cuda.Stream())
    for k in KEYS:
        assert same(a[k], c[k]), k
    u = run(torch.cuda.current_stream(), change=False)
    assert not same(a["pos"], u["pos"])
