"""The slab decomposition's CUDA backend (the library's per-stage entry
points) through SlabStep, on one GPU as a one-rank NCCL group: the same
state as the fused context step, bit for bit."""
import numpy as np
import pytest

from demso_b200 import scenes
from helpers import gpu_run, same

pytestmark = pytest.mark.gpu


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


@pytest.mark.parametrize("kind", ["gas", "typed"])
def test_cuda_backend_slab_equals_the_fused_step(group, kind):
    from demso_b200.slab import CudaBackend, SlabStep
    if kind == "gas":
        sc = scenes.agitated_gas(n=6000, seed=41, vel_std=2.0)
    else:
        sc = scenes.agitated_gas(n=4000, seed=42, n_mat=3, attraction=20.0, vel_std=0.5)
    steps = 40
    s = SlabStep(sc.sys, sc.state(), 0, 1, CudaBackend())
    s.step(steps)
    g = {k: (None if v is None else v.cpu().numpy()) for k, v in s.gather().items()}
    ref = gpu_run(sc.sys, sc.state(), steps)
    assert same(g["id"].view(np.uint32), ref["id"])
    for k in ("pos", "vel", "theta", "omega", "radius", "mass"):
        assert same(g[k], ref[k]), k
