"""Failure detection without a GPU fault.

* A bounded wait runs out: the context's full sort is told to hold one tile's
  publication (dem_debug_sort_hold) with a short spin limit, so the tile
  after it waits on a flag that nothing sets.  Its wait gives up, the step
  completes with every access in bounds, dem_check reports DEM_ERR_TIMEOUT,
  later steps keep running (each sorting from scratch), and after
  dem_set_state the context steps bit for bit like the oracle again.
* An allocation fails: the k-th device allocation of dem_create /
  dem_batch_create / a lazily allocating call is made to fail on the host
  (dem_debug_fail_allocation).  The call returns DEM_ERR_NO_MEMORY and every
  allocation it had made is released (dem_debug_live_allocations).

Nothing here traps, asserts on the device or waits without a limit.
"""
import ctypes as C
import time

import numpy as np
import pytest

from helpers import same
from oracle.oracle import PortOracle
from demso_b200 import scenes

pytestmark = pytest.mark.gpu

NO_MEMORY, TIMEOUT = 5, 4
NO_HOLD = 0xFFFFFFFF


def _t(a):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a.copy())


def _set(sim, sc):
    sim.set_state(_t(sc.pos), _t(sc.vel), _t(sc.theta), _t(sc.omega), _t(sc.radius),
                  _t(sc.mass), _t(sc.id))


def test_bounded_sort_wait_runs_out_and_the_context_recovers():
    import torch
    import demso_b200 as D
    L = D.load()
    sc = scenes.agitated_gas(n=20000, seed=81)  # five sort tiles of 4,096 keys
    sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    D.check(L.dem_debug_sort_hold(sim.handle, 0, 2000))
    _set(sim, sc)
    t0 = time.perf_counter()
    sim.step(1)  # the first step after dem_set_state is a full sort
    torch.cuda.synchronize()
    waited = time.perf_counter() - t0
    with pytest.raises(D.DemError) as e:
        sim.check()
    assert e.value.code == TIMEOUT
    sim.step(3)  # the context keeps stepping, sorting from scratch each step
    torch.cuda.synchronize()
    with pytest.raises(D.DemError) as e:
        sim.check()
    assert e.value.code == TIMEOUT
    assert waited < 5.0
    # the hold lifted and the state set again: the error word is cleared and
    # the steps are the oracle's again
    D.check(L.dem_debug_sort_hold(sim.handle, NO_HOLD, 0))
    _set(sim, sc)
    sim.step(1)
    sim.step(9)
    torch.cuda.synchronize()
    sim.check()
    got = sim.get_state("cpu")
    sim.close()
    ref = PortOracle("f32").run(sc.sys, sc.state(), 10)
    for k in ("pos", "vel", "theta", "omega"):
        assert same(got[k].numpy(), ref[k]), k


def test_failed_allocations_return_no_memory_and_release_everything():
    import torch
    import demso_b200 as D
    L = D.load()
    sc = scenes.agitated_gas(n=200000, seed=82)
    base = L.dem_debug_live_allocations()
    free0 = torch.cuda.mem_get_info()[0]
    try:
        # dem_create makes three device allocations
        for k in (1, 2, 3):
            D.check(L.dem_debug_fail_allocation(k))
            h = C.c_void_p()
            rc = L.dem_create(sc.sys.to_c(0), sc.n, D.CTX_PRESSURE, C.byref(h))
            assert rc == NO_MEMORY and not h.value, k
            assert b"out of memory" in L.dem_last_error_string().lower()
            assert L.dem_debug_live_allocations() == base, k
        # a batch makes two more (its parameter table and slot map)
        specs = scenes.specimen_batch(num=8, seed=4, nmin=512, nmax=2048)
        arr = (D._lib.DemSystem * len(specs))()
        for i, s in enumerate(specs):
            arr[i] = s.sys.to_c(s.n)
        for k in (1, 2, 3, 4, 5):
            D.check(L.dem_debug_fail_allocation(k))
            h = C.c_void_p()
            rc = L.dem_batch_create(arr, len(specs), D.CTX_PRESSURE, C.byref(h))
            assert rc == NO_MEMORY and not h.value, k
            assert L.dem_debug_live_allocations() == base, k
        D.check(L.dem_debug_fail_allocation(0))
        # a call that allocates on first use fails cleanly and the context
        # keeps working
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_PRESSURE)
        _set(sim, sc)
        sim.step(2)
        D.check(L.dem_debug_fail_allocation(1))
        with pytest.raises(D.DemError) as e:
            sim.set_control((0.5 * sc.sys.Lx, 0.5 * sc.sys.Ly), 5e-3)
        assert e.value.code == NO_MEMORY
        D.check(L.dem_debug_fail_allocation(0))
        sim.step(3)
        sim.check()
        sim.close()
        assert L.dem_debug_live_allocations() == base
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] >= free0 - (8 << 20)
    finally:
        L.dem_debug_fail_allocation(0)
