"""The slab decomposition (demso_b200.slab) on the GPU: halo windows stepped
by the library's fused context (ContextStepper), several slabs held by one
process and exchanging bands through local copies -- the decomposition of a
multi-GPU run on one GPU -- equal the single-domain context bit for bit; so
does one slab in a one-rank NCCL group."""
import numpy as np
import pytest

from demso_b200 import scenes
from helpers import gpu_run, same
from slab_harness import make_scene

pytestmark = pytest.mark.gpu


def _slabs(sc, world, period):
    from demso_b200.slab import ContextStepper, HaloSlab, scene_bounds
    bounds = scene_bounds(sc.sys, sc.pos, world)
    rmax = float(sc.radius.max())
    slabs = [HaloSlab(sc.sys, r, world, bounds, period, ContextStepper(sc.sys, rmax))
             for r in range(world)]
    for s in slabs:
        s.load(sc.state())
    return slabs


def _gathered(slabs, typed):
    import torch
    from demso_b200.slab import unpack
    g = unpack(torch.cat([s.own() for s in slabs]), typed)
    return {k: (None if v is None else v.cpu().numpy()) for k, v in g.items()}


def _compare(g, ref):
    assert same(g["id"].view(np.uint32), ref["id"])
    for k in ("pos", "vel", "theta", "omega", "radius", "mass"):
        assert same(g[k], ref[k]), k
    if ref.get("type") is not None:
        assert same(g["type"].view(np.uint32), ref["type"])


@pytest.mark.parametrize("world,kind,steps,period", [(2, "gas", 40, 6), (3, "hot", 30, 2),
                                                     (2, "typed", 30, 4), (3, "pile", 60, 8),
                                                     (2, "hot", 40, 6)])
def test_slabs_on_one_gpu_equal_the_fused_step(world, kind, steps, period):
    import torch
    from demso_b200.slab import run_group
    sc = make_scene(kind)
    slabs = _slabs(sc, world, period)
    run_group(slabs, steps)
    torch.cuda.synchronize()
    g = _gathered(slabs, len(sc.sys.materials) > 1)
    caps = [s.stepper.capacity for s in slabs]
    rebuilt = [s.rebuilds for s in slabs]
    for s in slabs:
        s.stepper.sim.check()
        s.stepper.close()
    ref = gpu_run(sc.sys, sc.state(), steps)
    _compare(g, ref)
    assert rebuilt == [(steps - 1) // period] * world
    # the windows kept their contexts (padding absorbed the changing counts)
    assert all(c > 0 for c in caps)


def test_slabs_at_scale_equal_the_fused_step():
    """Two stacked 262,144-disk plain-at-scale scenes in two slabs of 256
    rows, 100 steps exchanging every 20: the single-domain context's state."""
    import torch
    from demso_b200.slab import run_group
    sc = scenes.stacked_plain(262144, 2)
    slabs = _slabs(sc, 2, 20)
    ctx_before = [id(s.stepper.sim) for s in slabs]
    run_group(slabs, 100)
    torch.cuda.synchronize()
    g = _gathered(slabs, False)
    same_ctx = [id(s.stepper.sim) for s in slabs] == ctx_before
    for s in slabs:
        s.stepper.close()
    ref = gpu_run(sc.sys, sc.state(), 100)
    _compare(g, ref)
    assert same_ctx  # no window outgrew its context


def test_too_thin_a_halo_is_detected():
    """A halo of 2 rows for 6-step periods lets the error at the window's
    cut reach the slab: the state differs (the exactness checks above can
    fail)."""
    import torch
    from demso_b200.slab import ContextStepper, HaloSlab, run_group, scene_bounds
    sc = make_scene("hot")
    bounds = scene_bounds(sc.sys, sc.pos, 2)
    slabs = [HaloSlab(sc.sys, r, 2, bounds, 6, ContextStepper(sc.sys, float(sc.radius.max())),
                      halo=2) for r in range(2)]
    for s in slabs:
        s.load(sc.state())
    run_group(slabs, 40)
    torch.cuda.synchronize()
    g = _gathered(slabs, False)
    for s in slabs:
        s.stepper.close()
    ref = gpu_run(sc.sys, sc.state(), 40)
    differs = g["pos"].shape != ref["pos"].shape or not (same(g["id"].view(np.uint32), ref["id"])
                                                         and same(g["pos"], ref["pos"]))
    assert differs


@pytest.fixture(scope="module")
def group():
    import datetime
    import socket
    import torch.distributed as dist
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                            world_size=1, timeout=datetime.timedelta(seconds=60))
    yield
    dist.destroy_process_group()


def test_one_rank_nccl_slab_is_the_fused_step(group):
    import torch
    from demso_b200.slab import ContextStepper, DistExchange, HaloSlab, run, unpack
    sc = scenes.agitated_gas(n=6000, seed=41, vel_std=2.0)
    slab = HaloSlab(sc.sys, 0, 1, [0, sc.sys.gy], 5,
                    ContextStepper(sc.sys, float(sc.radius.max())))
    slab.load(sc.state())
    ex = DistExchange(0, 1, torch.device("cuda"))
    run(slab, ex, 40)
    g = unpack(ex.gather(slab.own()), False)
    g = {k: (None if v is None else v.cpu().numpy()) for k, v in g.items()}
    slab.stepper.close()
    _compare(g, gpu_run(sc.sys, sc.state(), 40))


@pytest.mark.parametrize("world,kind,steps,period", [(2, "hot", 40, 6), (3, "gas", 40, 5)])
def test_rank_processes_equal_the_fused_step(world, kind, steps, period, tmp_path):
    """The decomposition as separate rank processes (run + DistExchange),
    each rank's window on the GPU, the bands through gloo."""
    import os
    import socket
    import torch.multiprocessing as mp
    from slab_harness import gpu_worker
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.start_processes(gpu_worker, args=(world, port, kind, steps, period, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    g = dict(np.load(os.path.join(tmp_path, "gathered.npz")))
    sc = make_scene(kind)
    _compare(g, gpu_run(sc.sys, sc.state(), steps))
