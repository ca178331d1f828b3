"""Single scenes stepped by a thread-block cluster (DEM_CTX_RESIDENT on a
context of at most 8,192 disks and cells): every block holds the whole scene
in shared memory, steps its share of the slots and broadcasts the new state
to the other blocks through distributed shared memory.  The state equals
the graph path's bit for bit -- positions, velocities, angles, spins, the
static fields in the same order, loc, and the last step's pressure, acc and
alpha -- on piles, gases that re-sort on most steps or every step, tiny
wrapping grids, both block sizes, unsorted starts, consecutive calls, and
scenes it declines."""
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


def run(sc, calls, resident, shuffle_seed=None):
    import torch
    import demso_b200 as D
    flags = D.CTX_PRESSURE | D.CTX_ACCEL | (D.CTX_RESIDENT if resident else 0)
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=flags)
    st = sc.state()
    if shuffle_seed is not None:
        order = np.random.default_rng(shuffle_seed).permutation(sc.n)
        st = {k: (None if v is None else np.asarray(v)[order]) for k, v in st.items()}
    sim.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]), _torch(st["omega"]),
                  _torch(st["radius"]), _torch(st["mass"]), _torch(st["id"]),
                  None if st.get("type") is None else _torch(st["type"]))
    for k in calls:
        sim.step(k)
    torch.cuda.synchronize()
    out = {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                       else v.numpy())) for k, v in sim.get_state("cpu").items()}
    sim.check()
    sim.close()
    return out


def assert_same(sc, calls, **kw):
    a = run(sc, calls, True, **kw)
    b = run(sc, calls, False, **kw)
    for k in FIELDS:
        assert same(a[k], b[k]), k


def test_cluster_settling_pile():
    """The 4,096-disk settling pile (64 x 64 cells), 400 steps."""
    assert_same(scenes.settling_pile(), [400])


@pytest.mark.parametrize("n,vel,steps", [(3000, 1.0, 120), (1500, 4.0, 60), (7000, 0.5, 60)])
def test_cluster_gases(n, vel, steps):
    """Gases whose disks change cell on most steps (incremental re-sorts) or
    on every step in numbers (full sorts); 7,000 disks take the 1,024-thread
    blocks."""
    assert_same(scenes.agitated_gas(n=n, seed=7 + n, vel_std=vel, omega_std=100.0), [steps])


def test_cluster_tiny_wrapping_grid():
    """90 disks on a 2 x 2 grid: no culling, cells visited more than once."""
    assert_same(scenes.agitated_gas(n=90, seed=55, grid=(2, 2)), [40])


def test_cluster_unsorted_start_and_consecutive_calls():
    sc = scenes.agitated_gas(n=2500, seed=31, vel_std=0.8)
    ref = run(sc, [33], False, shuffle_seed=4)
    out = run(sc, [1, 12, 20], True, shuffle_seed=4)
    for k in FIELDS:
        assert same(out[k], ref[k]), k


def test_cluster_declines_a_larger_scene():
    """More than 8,192 disks: the graph path steps the scene (same results)."""
    assert_same(scenes.agitated_gas(n=9000, seed=81), [10])


@pytest.mark.parametrize("n", [1, 2, 5, 33])
def test_cluster_tiny_scenes(n):
    """A handful of disks: most blocks of the cluster own no slot."""
    assert_same(scenes.agitated_gas(n=n, seed=100 + n, vel_std=1.0), [25])


def test_cluster_declines_types_and_attraction():
    """Several materials, or attraction: the graph path steps the scene."""
    assert_same(scenes.agitated_gas(n=600, seed=61, n_mat=3), [20])
    assert_same(scenes.agitated_gas(n=600, seed=62, attraction=0.05), [20])


def test_followed_rows_on_a_resident_context():
    """dem_step_followed steps a resident context on the graph path (its rows
    come from that path's buffers), then dem_step takes the cluster again:
    rows and state equal a plain context's."""
    import torch
    import demso_b200 as D
    sc = scenes.agitated_gas(n=1800, seed=44, vel_std=0.7)
    ids = np.array([0, 17, 900, 1799], dtype=np.uint32)

    def go(flags):
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=flags)
        st = sc.state()
        sim.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]),
                      _torch(st["omega"]), _torch(st["radius"]), _torch(st["mass"]),
                      _torch(st["id"]))
        sim.step(7)
        rows = sim.step_followed(15, ids)
        sim.step(9)
        torch.cuda.synchronize()
        out = {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                           else v.numpy()))
               for k, v in sim.get_state("cpu").items()}
        sim.check()
        sim.close()
        return rows, out

    base = D.CTX_PRESSURE | D.CTX_ACCEL
    rows_a, a = go(base | D.CTX_RESIDENT)
    rows_b, b = go(base)
    assert np.array_equal(rows_a.view(np.uint32), rows_b.view(np.uint32))
    for k in FIELDS:
        assert same(a[k], b[k]), k


@pytest.mark.parametrize("caller_state", [False, True])
def test_cluster_steps_in_adopted_sets(caller_state):
    """The cluster reads and writes the caller's two ping-pong sets
    (dem_adopt_state), with or without a context state of its own; the view
    then shows the graph path's state."""
    import torch
    import demso_b200 as D
    from helpers import gpu_run
    from test_gpu_adopt import FIELDS as ADOPT_FIELDS, _sets, _view_np
    sc = scenes.agitated_gas(n=2200, seed=57, vel_std=0.8)
    chunks = [1, 9, 30]
    ref = gpu_run(sc.sys, sc.state(), sum(chunks), chunks=chunks)
    flags = D.CTX_PRESSURE | D.CTX_ACCEL | D.CTX_RESIDENT | (D.CTX_CALLER_STATE if caller_state
                                                            else 0)
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=flags)
    first, second = _sets(sc.state(), False)
    sim.adopt_state(first, second, sc.n)
    for c in chunks:
        sim.step(c)
    torch.cuda.synchronize()
    sim.check()
    got = _view_np(sim.state_view())
    sim.close()
    for k in ADOPT_FIELDS:
        if k == "type":
            continue
        assert same(got[k], ref[k]), k


def test_nan_is_reported_on_the_resident_paths():
    """A NaN position: the cluster launch and the resident batch set the
    error word (dem_check: DEM_ERR_OOB) and carry the NaN exactly as the
    graph path does."""
    import torch
    import demso_b200 as D
    sc = scenes.agitated_gas(n=1000, seed=2)
    sc.pos[10] = [np.nan, 0.01]

    def state_after(flags):
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_PRESSURE | D.CTX_ACCEL | flags)
        st = sc.state()
        sim.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]),
                      _torch(st["omega"]), _torch(st["radius"]), _torch(st["mass"]),
                      _torch(st["id"]))
        sim.step(6)
        torch.cuda.synchronize()
        out = {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                           else v.numpy()))
               for k, v in sim.get_state("cpu").items()}
        with pytest.raises(D.DemError) as err:
            sim.check()
        sim.close()
        return out, err.value.code

    a, code_a = state_after(0)
    b, code_b = state_after(D.CTX_RESIDENT)
    assert code_a == code_b == 3
    for k in FIELDS:
        assert same(a[k], b[k]), k

    specimens = [sc, scenes.agitated_gas(n=500, seed=3)]
    bt = D.Batch([(s.sys, s.n) for s in specimens],
                 flags=D.CTX_PRESSURE | D.CTX_ACCEL | D.CTX_RESIDENT)
    st = scenes.concat_specimens(specimens)
    bt.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]),
                 _torch(st["omega"]), _torch(st["radius"]), _torch(st["mass"]), _torch(st["id"]))
    bt.step(6)
    torch.cuda.synchronize()
    with pytest.raises(D.DemError) as err:
        bt.check()
    assert err.value.code == 3
    bt.close()
