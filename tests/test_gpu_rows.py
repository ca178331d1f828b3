"""Row windows (dem_create_rows): a context over a power-of-two block of a
tall grid's cell rows steps the particles inside those rows exactly as a
context over the whole grid does, whether the block starts at the band's
edge or wraps past the top of its rows; dem_row_slots answers in the
scene's rows; the slab decomposition's windows use row windows on tall
scenes and still equal the single-domain step."""
import ctypes as C

import numpy as np
import pytest

from demso_b200 import scenes
from helpers import gpu_run, same

pytestmark = pytest.mark.gpu


def _band(kind="gas", copy=2):
    """One copy of a four-copy stacked gas, alone in the tall box: its disks
    start in cell rows [32 copy, 32 copy + 32) of a 32 x 128 grid.  The gas's
    initial overlaps drive disks to about 70 m/s, so over 60 steps they
    spread a few rows beyond the band (rows 61..98 for the plain gas)."""
    if kind == "typed":
        base = scenes.agitated_gas(n=1200, seed=33, n_mat=3, attraction=20.0, vel_std=0.5)
    else:
        base = scenes.agitated_gas(n=1500, seed=31, vel_std=0.4)
    sc = scenes.stacked(base, 4)
    n = base.pos.shape[0]
    sl = slice(copy * n, (copy + 1) * n)
    st = {k: (None if v is None else np.ascontiguousarray(v[sl])) for k, v in sc.state().items()}
    st["id"] = np.arange(n, dtype=np.uint32)
    return sc.sys, st


def _compare(a, b):
    for k in ("pos", "vel", "theta", "omega", "radius", "mass", "id", "pressure"):
        if a.get(k) is not None:
            assert same(a[k], b[k]), k


def _inside(sys, st, rows):
    """Every disk of a whole-grid state is in the window's rows and one row
    clear of its edges (so are its neighbour rows): the premise under which
    a row window steps it exactly."""
    from demso_b200.slab import cell_rows
    r = cell_rows(sys, st["pos"])
    first, count = rows
    assert r.min() >= first + 1 and r.max() <= first + count - 2, (r.min(), r.max(), rows)


# Row windows holding every row each band visits: the plain gas (32 x 128
# cells, rows 61..98) in 64-row windows, the typed gas (16 x 64 cells, rows
# 29..49) in 32-row ones; the second of each wraps its cell rows inside the
# grid (at rows 104 and 56).
WINDOWS = {"gas": [(56, 64), (40, 64), (48, 64)], "typed": [(20, 32), (24, 32), (26, 32)]}


@pytest.mark.parametrize("kind", ["gas", "typed"])
@pytest.mark.parametrize("w", [0, 1, 2])
def test_row_window_steps_its_rows_as_the_whole_grid(kind, w):
    """60 steps with a full sort, the incremental sort and, for the typed
    gas, three materials and attraction (the per-cell collide)."""
    rows = WINDOWS[kind][w]
    sys, st = _band(kind)
    ref = gpu_run(sys, st, 60)
    _inside(sys, ref, rows)
    got = gpu_run(sys, st, 60, rows=rows)
    _compare(got, ref)


def test_row_window_chunks_equal_one_call():
    """The device-side step loop and single steps on a row window."""
    sys, st = _band()
    a = gpu_run(sys, st, 41, rows=(56, 64))
    _inside(sys, a, (56, 64))
    b = gpu_run(sys, st, 41, rows=(56, 64), chunks=[1, 7, 1, 32])
    _compare(a, b)


def _sim(sys, st, rows):
    import torch
    import demso_b200 as D
    sim = D.Simulation(sys, capacity=st["pos"].shape[0], flags=D.CTX_PRESSURE, rows=rows)
    to = (lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32).copy())
          if a.dtype == np.uint32 else torch.from_numpy(np.ascontiguousarray(a).copy()))
    sim.set_state(*(to(st[k]) for k in ("pos", "vel", "theta", "omega", "radius", "mass", "id")))
    return sim


def _row_slots(sim, lo, hi):
    from demso_b200._lib import check, load
    f, c = C.c_uint32(0), C.c_uint32(0)
    check(load().dem_row_slots(sim.handle, lo, hi, C.byref(f), C.byref(c), None))
    return f.value, c.value


def test_row_slots_take_the_scenes_rows():
    import torch
    from demso_b200 import DemError
    sys, st = _band()
    whole, win = _sim(sys, st, None), _sim(sys, st, (56, 64))
    try:
        whole.step(3)
        win.step(3)
        torch.cuda.synchronize()
        for lo, hi in [(56, 120), (64, 96), (70, 71), (64, 64), (90, 100)]:
            assert _row_slots(win, lo, hi) == _row_slots(whole, lo, hi), (lo, hi)
        for lo, hi in [(55, 70), (100, 121), (0, 128)]:
            with pytest.raises(DemError):
                _row_slots(win, lo, hi)
    finally:
        whole.close()
        win.close()


def test_row_slots_stop_at_the_grids_last_row():
    """A block of rows that runs past the grid's top (rows 96..159 of 128):
    dem_row_slots takes rows up to 128, not beyond."""
    import torch
    from demso_b200 import DemError
    sys, st = _band()
    win = _sim(sys, st, (96, 64))
    try:
        win.step(2)
        torch.cuda.synchronize()
        first, count = _row_slots(win, 96, 128)
        assert first + count <= st["pos"].shape[0]
        for lo, hi in [(96, 129), (95, 100), (120, 160)]:
            with pytest.raises(DemError):
                _row_slots(win, lo, hi)
    finally:
        win.close()


@pytest.mark.parametrize("first,count", [(0, 48), (0, 256), (128, 32), (10, 0)])
def test_bad_row_windows_are_refused(first, count):
    import demso_b200 as D
    from demso_b200 import DemError
    sys, st = _band()
    with pytest.raises(DemError):
        D.Simulation(sys, capacity=16, flags=D.CTX_PRESSURE, rows=(first, count))


def test_row_windows_decline_the_cluster_form():
    """CTX_RESIDENT on a row window: the graph path steps it (the cluster
    form takes whole grids), with the graph path's bits."""
    import demso_b200 as D
    sys, st = _band()
    ref = gpu_run(sys, st, 30, rows=(56, 64))
    got = gpu_run(sys, st, 30, rows=(56, 64), flags=D.CTX_PRESSURE | D.CTX_ACCEL | D.CTX_RESIDENT)
    _compare(got, ref)


def test_slab_windows_of_a_tall_scene_are_row_windows():
    """Four stacked 65,536-disk plain-at-scale scenes (128 x 512 cells) in
    four slabs, exchanging every 10 steps (22-row halos): every window's
    context holds 256 rows, not the scene's 512, and the slabs' own rows
    equal the single-domain context after 60 steps."""
    import torch
    from demso_b200.slab import ContextStepper, HaloSlab, run_group, scene_bounds, unpack
    sc = scenes.stacked_plain(65536, 4)
    bounds = scene_bounds(sc.sys, sc.pos, 4)
    rmax = float(sc.radius.max())
    slabs = [HaloSlab(sc.sys, r, 4, bounds, 10, ContextStepper(sc.sys, rmax)) for r in range(4)]
    for s in slabs:
        s.load(sc.state())
    rows = [s.stepper.rows for s in slabs]
    run_group(slabs, 60)
    torch.cuda.synchronize()
    g = unpack(torch.cat([s.own() for s in slabs]), False)
    g = {k: (None if v is None else v.cpu().numpy()) for k, v in g.items()}
    for s in slabs:
        s.stepper.sim.check()
        s.stepper.close()
    assert all(c == 256 for _, c in rows), rows
    assert [f for f, _ in rows] == [s.wlo for s in slabs]
    ref = gpu_run(sc.sys, sc.state(), 60)
    assert same(g["id"].view(np.uint32), ref["id"])
    for k in ("pos", "vel", "theta", "omega", "radius", "mass"):
        assert same(g[k], ref[k]), k
