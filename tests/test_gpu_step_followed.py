"""dem_step_followed: steps with the reference's per-step followed-particle
rows gathered on the device inside the step loop.  One call must give, bit
for bit, the rows and the state of stepping one step at a time with
dem_get_followed after each: odd step counts, enough ids that the 64 MB row
ring is used in chunks, an autotuned context whose tuning steps fall inside
the calls (rows into pinned memory), and a batch."""
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


def _make(sc=None, batch=None, flags=0):
    import demso_b200 as D
    flags |= D.CTX_PRESSURE | D.CTX_ACCEL
    if batch is None:
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=flags)
        st = sc.state()
    else:
        sim = D.Batch([(s.sys, s.n) for s in batch], flags=flags)
        st = scenes.concat_specimens(batch)
    sim.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]),
                  _torch(st["omega"]), _torch(st["radius"]), _torch(st["mass"]),
                  _torch(st["id"]), _torch(st["type"]) if st["type"] is not None else None)
    return sim


def _host(sim):
    import torch
    torch.cuda.synchronize()
    return {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                        else v.numpy())) for k, v in sim.get_state("cpu").items()}


def _check(make, ids, chunks, pinned=False):
    import torch
    a, b = make(), make()
    got = []
    for c in chunks:
        if pinned:
            rows = torch.zeros(c * ids.size * 12, dtype=torch.float32).pin_memory()
            a.step_followed(c, ids, rows)
            torch.cuda.current_stream().synchronize()
            got.append(rows.numpy().reshape(c, ids.size, 12).copy())
        else:
            got.append(a.step_followed(c, ids))
    got = np.concatenate(got)
    want = []
    for _ in range(sum(chunks)):
        b.step(1)
        want.append(b.followed(ids))
    for k in range(sum(chunks)):
        assert same(got[k], want[k]), k
    sa, sb = _host(a), _host(b)
    for k in KEYS:
        if sa[k] is None:
            assert sb[k] is None, k
        else:
            assert same(sa[k], sb[k]), k
    a.check()
    a.close()
    b.close()


def test_rows_of_one_call_equal_per_step_rows():
    sc = scenes.agitated_gas(n=3000, seed=21, n_mat=3, attraction=25.0)
    ids = np.arange(0, 3000, 19, dtype=np.uint32)
    _check(lambda: _make(sc), ids, [37, 1, 2])


def test_rows_in_chunks_of_the_ring():
    # 100,000 ids: 4.8 MB of rows per step, so the 64 MB ring takes 13 steps
    sc = scenes.agitated_gas(n=120000, seed=5, vel_std=2.0)
    ids = np.random.default_rng(1).permutation(120000)[:100000].astype(np.uint32)
    _check(lambda: _make(sc), ids, [30])


def test_autotuned_context_into_pinned_rows():
    import demso_b200 as D
    sc = scenes.settling_pile(side=40, box=0.12, seed=4, vel_std=0.3)
    ids = np.array([0, 7, 99, 1599, 800], dtype=np.uint32)
    _check(lambda: _make(sc, flags=D.CTX_AUTOTUNE), ids, [1, 20, 9, 10], pinned=True)


def test_direct_launches():
    import demso_b200 as D
    sc = scenes.agitated_gas(n=2000, seed=9, vel_std=1.0)
    ids = np.arange(0, 2000, 7, dtype=np.uint32)
    _check(lambda: _make(sc, flags=D.CTX_DIRECT), ids, [12, 5])


def test_batch_rows():
    batch = scenes.specimen_batch(num=10, seed=8, nmin=64, nmax=2048)
    n = sum(s.n for s in batch)
    ids = np.arange(0, n, 37, dtype=np.uint32)
    _check(lambda: _make(batch=batch), ids, [25])


def test_rejects_an_id_out_of_range():
    import demso_b200 as D
    sc = scenes.agitated_gas(n=500, seed=2)
    sim = _make(sc)
    with pytest.raises(D.DemError):
        sim.step_followed(4, np.array([3, 500], dtype=np.uint32))
    sim.close()
