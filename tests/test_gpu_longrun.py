"""A long run against the reference's own step functions built for the host:
a 1,000-disk column collapses for 30,000 steps (0.3 s, dt 1e-5 s, kn 2e4
N/m).  The GPU trajectory equals the reference's bit for bit, so its bulk
statistics (kinetic energy, coordination number, packing fraction, heap
angle) are the reference's exactly."""
import numpy as np
import pytest

from bulk_stats import bulk_stats
from demso_b200 import calibrate
from helpers import gpu_run, same
from oracle.oracle import RefHarness, ref_available

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not ref_available(), reason="reference host build absent")
def test_long_run_and_bulk_statistics_equal_the_reference():
    sc = calibrate.column_scene(1000, seed=1, kn=2e4, dt=1e-5)
    steps = 30000
    out = gpu_run(sc.sys, sc.state(), steps, chunks=[10000, 10000, 10000])
    h = RefHarness()
    h.setup(sc.sys, sc.radius, sc.mass, None)
    b = h.make_buffers(sc.state())
    h.run(b, steps)
    ref = dict(pos=b["pos1"], vel=b["vel1"], theta=b["theta1"], omega=b["omega1"], id=b["id1"])
    for k in ("pos", "vel", "theta", "omega", "id"):
        assert same(out[k], ref[k]), k
    ref["radius"] = sc.radius[ref["id"]]
    ref["mass"] = sc.mass[ref["id"]]
    a, r = bulk_stats(out), bulk_stats(ref)
    assert a == r
    assert a["z"] > 0.5 and 0.3 < a["phi"] < 0.9 and a["angle"] > 1.0
