"""Direct-launch mode (DEM_CTX_DIRECT): the same kernels launched one by one
with the sort path chosen on the host give the same trajectory, bit for bit,
as the CUDA-graph step -- on a quiet scene (incremental sort every step) and
on a hot gas whose movers overflow the incremental sort (full-sort path)."""
import numpy as np
import pytest

from demso_b200 import scenes
from helpers import gpu_run, same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [
    lambda: scenes.settling_pile(),
    lambda: scenes.agitated_gas(n=20000, seed=4, vel_std=300.0, omega_std=500.0),
])
def test_direct_mode_equals_graph_mode(make):
    import demso_b200 as D
    sc = make()
    base = D.CTX_PRESSURE | D.CTX_ACCEL
    a = gpu_run(sc.sys, sc.state(), 60, flags=base)
    b = gpu_run(sc.sys, sc.state(), 60, flags=base | D.CTX_DIRECT, chunks=[1, 7, 52])
    for k in ("pos", "vel", "theta", "omega", "radius", "mass", "id", "pressure", "acc", "alpha"):
        assert same(a[k], b[k]), k
