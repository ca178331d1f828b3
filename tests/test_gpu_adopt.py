"""Caller-owned state (dem_adopt_state, dem_state_view): the context steps in
two ping-pong sets of the caller's device buffers, the reference's own
arrangement (allocateVectors, functions.cu:68-149; the set switch of the
step loop, main.cu:395-430).  The trajectory is bit for bit the one of the
context's own buffers and of the oracle; the view aliases the adopted
buffers; bad sets are refused on the host before any launch."""
import ctypes as C

import numpy as np
import pytest

from demso_b200 import scenes
from helpers import gpu_run, same
from oracle.oracle import PortOracle

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "theta", "omega", "radius", "mass", "id", "type")


def _np(t):
    a = t.detach().cpu().numpy()
    return a.view(np.uint32) if a.dtype == np.int32 else a


def _sets(st, typed, fill=float("nan")):
    """Two sets on the GPU: the first holds the state (pos and radius padded
    by STATE_PAD rows), the second is scratch filled with `fill`."""
    import torch
    import demso_b200 as D
    n = st["pos"].shape[0]
    pad = D.STATE_PAD

    def make(k, src):
        shape = {"pos": (n + pad, 2), "vel": (n, 2), "radius": (n + pad,)}.get(k, (n,))
        ints = k in ("id", "type")
        t = torch.full(shape, 0 if ints else fill, dtype=torch.int32 if ints else torch.float32,
                       device="cuda")
        if src is not None:
            a = np.ascontiguousarray(src)
            t[:n] = torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).cuda()
        return t

    first = {k: make(k, st[k]) for k in FIELDS if k != "type" or typed}
    second = {k: make(k, None) for k in FIELDS if k != "type" or typed}
    return first, second


def _view_np(view):
    return {k: (None if view[k] is None else _np(view[k])) for k in FIELDS}


@pytest.mark.parametrize("kind", ["hot", "typed"])
@pytest.mark.parametrize("own", [True, False])
def test_adopted_sets_step_like_the_context_buffers(kind, own):
    import torch
    import demso_b200 as D
    if kind == "typed":
        sc = scenes.agitated_gas(n=3000, seed=81, n_mat=3, attraction=15.0, vel_std=0.3)
    else:
        # movers overflow the incremental sort: both sort paths run
        sc = scenes.agitated_gas(n=20000, seed=82, vel_std=300.0, omega_std=500.0)
    typed = sc.state()["type"] is not None
    steps, chunks = 60, [1, 9, 50]
    ref = gpu_run(sc.sys, sc.state(), steps, chunks=chunks)
    flags = D.CTX_PRESSURE | D.CTX_ACCEL | (0 if own else D.CTX_CALLER_STATE)
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=flags)
    first, second = _sets(sc.state(), typed)
    sim.adopt_state(first, second, sc.n)
    for c in chunks:
        sim.step(c)
    torch.cuda.synchronize()
    sim.check()
    view = sim.state_view()
    got = _view_np(view)
    for k in FIELDS:
        if k == "type" and not typed:
            assert got[k] is None
            continue
        assert same(got[k], ref[k]), k
    # the view is the adopted buffers themselves: positions in the first
    # set, every other field in the set it names
    which = (first, second)[view["set"]]
    assert view["pos"].data_ptr() == first["pos"].data_ptr()
    for k in FIELDS[1:]:
        if view[k] is not None:
            assert view[k].data_ptr() == which[k].data_ptr(), k
    # the copy-out reads the same buffers
    cp = sim.get_state(device="cpu")
    assert same(_np(cp["pos"]), ref["pos"]) and same(_np(cp["vel"]), ref["vel"])
    assert same(_np(cp["loc"]), ref["loc"])
    sim.close()


def test_adopted_trajectory_matches_the_oracle():
    import torch
    import demso_b200 as D
    sc = scenes.settling_pile(side=48, vel_std=0.2)
    steps = 40
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_CALLER_STATE)
    first, second = _sets(sc.state(), False)
    sim.adopt_state(first, second, sc.n)
    sim.step(steps)
    torch.cuda.synchronize()
    got = _view_np(sim.state_view())
    sim.close()
    ref = PortOracle("f32").run(sc.sys, sc.state(), steps)
    for k in ("pos", "vel", "theta", "omega", "id"):
        assert same(got[k], ref[k]), k


def test_readopting_a_copy_of_the_view_continues_the_run():
    """Halfway through, the caller moves the state into new buffers (a copy
    of the view, in the context's order) and hands those over: the run goes
    on bit for bit, through newly captured graphs."""
    import torch
    import demso_b200 as D
    sc = scenes.agitated_gas(n=12000, seed=83, vel_std=0.5)
    ref = gpu_run(sc.sys, sc.state(), 50)
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    first, second = _sets(sc.state(), False)
    sim.adopt_state(first, second, sc.n)
    sim.step(20)
    torch.cuda.synchronize()
    view = _view_np(sim.state_view())
    view["type"] = None
    first2, second2 = _sets(view, False, fill=1.0e30)
    sim.adopt_state(first2, second2, sc.n)
    sim.step(30)
    torch.cuda.synchronize()
    got = _view_np(sim.state_view())
    sim.close()
    for k in ("pos", "vel", "theta", "omega", "radius", "mass", "id"):
        assert same(got[k], ref[k]), k


def test_caller_state_context_takes_its_state_only_by_adoption():
    import torch
    import demso_b200 as D
    sc = scenes.settling_pile(side=16)
    st = sc.state()
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_CALLER_STATE)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a))
    args = [t(st[k]) for k in ("pos", "vel", "theta", "omega", "radius", "mass", "id")]
    with pytest.raises(D.DemError):
        sim.set_state(*args)
    with pytest.raises(D.DemError):
        sim.state_view()
    with pytest.raises(D.DemError):
        sim.get_state()
    sim.step(3)  # no particles: nothing to do
    first, second = _sets(st, False, fill=0.0)
    sim.adopt_state(first, second, sc.n)
    # dem_set_state now copies into the adopted buffers
    args[0] = args[0] + 1e-4
    sim.set_state(*args)
    torch.cuda.synchronize()
    assert same(_np(first["pos"][:sc.n]), st["pos"] + np.float32(1e-4))
    sim.close()


def test_caller_state_context_allocates_no_state():
    import torch
    import demso_b200 as D
    sc = scenes.settling_pile(side=16)
    n = 1 << 20
    D.Simulation(sc.sys, capacity=sc.n).close()  # the library's first context
    drops = []
    for flags in (0, D.CTX_CALLER_STATE):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        sim = D.Simulation(sc.sys, capacity=n, flags=flags)
        torch.cuda.synchronize()
        drops.append(free0 - torch.cuda.mem_get_info()[0])
        sim.close()
    # two dynamic sets (8 + 8 + 4 + 4 bytes) and two static sets
    # (4 + 4 + 4 bytes) per particle: 72 bytes
    saved = drops[0] - drops[1]
    assert 64 * n <= saved <= 80 * n, (drops, saved)


def test_bad_sets_are_refused_before_any_launch():
    import torch
    import demso_b200 as D
    from demso_b200 import _lib
    sc = scenes.settling_pile(side=16)
    st = sc.state()
    n = sc.n
    sim = D.Simulation(sc.sys, capacity=n, flags=D.CTX_CALLER_STATE)
    first, second = _sets(st, False)

    def refused(a, b, count=n):
        with pytest.raises(D.DemError):
            sim.adopt_state(a, b, count)

    refused(first, second, n + 1)          # over capacity
    refused(first, second, 0)              # nothing to adopt
    refused(first, dict(second, vel=first["vel"]))            # shared buffer
    refused(first, dict(second, mass=first["theta"][1:]))      # overlapping
    refused(dict(first, pos=first["pos"].view(-1)[1:]), second)  # misaligned float2
    refused(dict(first, omega=None), second)                  # missing field
    # host memory (through the C ABI directly: the binding takes CUDA tensors only)
    host = (C.c_float * (2 * (n + 8)))()
    a = _lib.DemStateSet(*[t.data_ptr() for t in (first[k] for k in FIELDS[:7])], None)
    b = _lib.DemStateSet(*[t.data_ptr() for t in (second[k] for k in FIELDS[:7])], None)
    a.pos = C.addressof(host)
    assert _lib.load().dem_adopt_state(sim.handle, n, C.byref(a), C.byref(b), None) == 1
    with pytest.raises(D.DemError):
        sim.state_view()
    sim.close()


@pytest.mark.parametrize("resident", [False, True])
def test_a_batch_steps_in_adopted_sets(resident):
    """The batched form in caller buffers, on the graph path or the resident
    launch: the concatenated specimens in the first set, every specimen bit
    for bit the oracle's run alone."""
    import torch
    import demso_b200 as D
    specimens = [scenes.agitated_gas(n=700, seed=84), scenes.settling_pile(side=20, box=0.05,
                                                                            seed=85, vel_std=0.3),
                 scenes.agitated_gas(n=400, seed=86, grid="ref", vel_std=1.0)]
    steps = 30
    b = D.Batch([(sc.sys, sc.n) for sc in specimens],
                flags=D.CTX_CALLER_STATE | (D.CTX_RESIDENT if resident else 0))
    st = scenes.concat_specimens(specimens)
    first, second = _sets(st, False)
    b.adopt_state(first, second, b.capacity)
    b.step(steps)
    torch.cuda.synchronize()
    b.check()
    got = _view_np(b.state_view())
    ranges = [b.slots(s) for s in range(len(specimens))]
    b.close()
    po = PortOracle("f32")
    for sc, (lo, hi) in zip(specimens, ranges):
        ref = po.run(sc.sys, sc.state(), steps)
        ids = got["id"][lo:hi] - np.uint32(lo)
        assert np.array_equal(ids, ref["id"])
        for k in ("pos", "vel", "theta", "omega"):
            assert same(got[k][lo:hi], ref[k]), k
