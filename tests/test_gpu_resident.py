"""Resident batched step (DEM_CTX_RESIDENT): a dem_step call of a batch run
as one persistent launch, each bin of specimens stepped inside one
multiprocessor's shared memory, gives the graph path's state bit for bit --
positions, velocities, angles, spins, the static fields in the same order,
loc, and the last step's pressure, acc and alpha -- including specimens that
change cell every step (a sort on every step), unsorted initial states,
consecutive calls, the full batched workload, and batches it declines."""
import numpy as np
import pytest

from demso_b200 import scenes
from helpers import same

pytestmark = pytest.mark.gpu

FIELDS = ["pos", "vel", "theta", "omega", "radius", "mass", "id", "loc", "pressure", "acc",
          "alpha"]


def _torch(a):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a.copy())


def run(specimens, calls, resident, shuffle_seed=None):
    """The batch stepped by dem_step calls of calls[k] steps; the state."""
    import torch
    import demso_b200 as D
    flags = D.CTX_PRESSURE | D.CTX_ACCEL | (D.CTX_RESIDENT if resident else 0)
    b = D.Batch([(sc.sys, sc.n) for sc in specimens], flags=flags)
    st = scenes.concat_specimens(specimens)
    if shuffle_seed is not None:
        # every specimen's particles in a random order within its slots
        rng = np.random.default_rng(shuffle_seed)
        order, start = [], 0
        for sc in specimens:
            order.append(start + rng.permutation(sc.n))
            start += sc.n
        order = np.concatenate(order)
        st = {k: (None if v is None else v[order]) for k, v in st.items()}
    b.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]), _torch(st["omega"]),
                _torch(st["radius"]), _torch(st["mass"]), _torch(st["id"]))
    for k in calls:
        b.step(k)
    torch.cuda.synchronize()
    out = {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                       else v.numpy())) for k, v in b.get_state("cpu").items()}
    b.check()
    b.close()
    return out


def assert_same_state(a, b):
    for k in FIELDS:
        assert same(a[k], b[k]), k


def mixed():
    out = [scenes.agitated_gas(n=700, seed=51),
           scenes.agitated_gas(n=300, seed=52, grid="ref", vel_std=1.0),
           scenes.settling_pile(side=24, box=0.06, seed=53, vel_std=0.3),
           scenes.agitated_gas(n=1200, seed=54, dt=1e-6),
           scenes.agitated_gas(n=90, seed=55, grid=(2, 2))]
    sc = scenes.agitated_gas(n=500, seed=56, gravity=(1.5, -9.0))
    sc.sys.materials[0].frictionCoefficient = 0.9
    out.append(sc)
    return out


@pytest.mark.parametrize("steps", [1, 2, 60])
def test_resident_equals_graph_path(steps):
    specimens = mixed()
    assert_same_state(run(specimens, [steps], True), run(specimens, [steps], False))


def test_resident_hot_specimens_sort_every_step():
    """Fast, dense gases: particles change cell on nearly every step, so the
    resident launch re-sorts its bins on nearly every step."""
    specimens = [scenes.agitated_gas(n=n, seed=70 + k, vel_std=4.0, omega_std=500.0)
                 for k, n in enumerate((400, 900, 1500, 2600))]
    assert_same_state(run(specimens, [80], True), run(specimens, [80], False))


def test_resident_few_movers_per_step():
    """Gases at a few m/s: a handful of particles change cell on most steps,
    so most steps re-sort incrementally (at most 32 movers in a bin) and the
    busier ones sort in full."""
    specimens = [scenes.agitated_gas(n=n, seed=90 + k, vel_std=v, omega_std=50.0)
                 for k, (n, v) in enumerate(((2000, 2.0), (3500, 1.0), (1200, 3.0), (800, 0.5),
                                             (5000, 0.3)))]
    assert_same_state(run(specimens, [150], True), run(specimens, [150], False))


def test_resident_from_unsorted_state_and_across_calls():
    specimens = scenes.specimen_batch(num=40, seed=11, nmin=64, nmax=3000)
    ref = run(specimens, [47], False, shuffle_seed=2)
    assert_same_state(run(specimens, [47], True, shuffle_seed=2), ref)
    assert_same_state(run(specimens, [1, 9, 20, 17], True, shuffle_seed=2), ref)


def test_resident_full_batched_workload():
    """All 4,096 specimens of the batched workload (256 to 8,192 disks,
    9.26M in all), 12 steps in one call."""
    specimens = scenes.specimen_batch()
    assert_same_state(run(specimens, [12], True), run(specimens, [12], False))


def test_resident_declines_a_specimen_larger_than_a_bin():
    """A specimen of more than 8,192 disks: the batch takes the graph path
    (same results)."""
    specimens = [scenes.agitated_gas(n=9000, seed=81), scenes.agitated_gas(n=500, seed=82)]
    assert_same_state(run(specimens, [10], True), run(specimens, [10], False))
