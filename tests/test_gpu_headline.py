"""Parity at the benchmarked sizes themselves.

* The plain-at-scale scene that the headline figure is measured on
  (4,194,304 disks, 1024 x 1024 grid, seed 0): its first step (a full
  radix sort) and ten more steps issued as one dem_step call, which the
  library runs through its device-side step loop with the incremental sort,
  against the reference's own step functions built for the host
  (particles_kernel.cuh:114-233 hash/reorder, :459-549 collide, :580-627
  integrate, with a stable sort), bit for bit.
* The same scene with seeded random velocities, so that thousands of disks
  change cells every step (the incremental sort's movers at full scale) and
  pairs collide, against the reference again.
* The batched workload at its full size (4,096 specimens, 9.26M disks) for
  five steps, every 64th specimen against the CPU restatement run on that
  specimen alone.
"""
import numpy as np
import pytest

from helpers import gpu_run, same
from oracle.oracle import PortOracle, RefHarness, ref_available
from demso_b200 import scenes

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not ref_available(), reason="reference host build absent")
HEADLINE_N = 4194304


def _reference(sc, steps, st=None):
    h = RefHarness()
    h.setup(sc.sys, sc.radius, sc.mass, None)
    b = h.make_buffers(sc.state() if st is None else st)
    h.run(b, steps)
    return dict(pos=b["pos1"], vel=b["vel1"], theta=b["theta1"], omega=b["omega1"],
                id=b["id1"], loc=b["loc1"], pressure=b["pressure"])


def _compare(out, ref):
    for k in ("pos", "vel", "theta", "omega", "id", "loc", "pressure"):
        assert same(out[k], ref[k]), k


@needs_ref
def test_headline_scene_matches_reference():
    sc = scenes.plain_at_scale(HEADLINE_N, seed=0)
    assert (sc.sys.gx, sc.sys.gy) == (1024, 1024)
    out = gpu_run(sc.sys, sc.state(), 11, chunks=[1, 10])
    _compare(out, _reference(sc, 11))


@needs_ref
def test_headline_scene_with_movers_matches_reference():
    sc = scenes.plain_at_scale(HEADLINE_N, seed=0)
    rng = np.random.default_rng(11)
    st = sc.state()
    st["vel"] = rng.normal(0.0, 0.5, size=(sc.n, 2)).astype(np.float32)
    st["omega"] = rng.normal(0.0, 100.0, size=sc.n).astype(np.float32)
    out = gpu_run(sc.sys, st, 11, chunks=[1, 10])
    ref = _reference(sc, 11, st)
    _compare(out, ref)
    # the steps moved disks across cells and made contacts
    moved = np.count_nonzero(scenes.cell_hash(ref["pos"], sc.sys)
                             != scenes.cell_hash(st["pos"][ref["id"]], sc.sys))
    assert moved > 10000
    assert np.count_nonzero(ref["pressure"]) > 1000


def test_batched_workload_sampled_specimens_match_oracle():
    import torch
    import demso_b200 as D
    specimens = scenes.specimen_batch(num=4096, seed=0)
    steps = 5
    b = D.Batch([(sc.sys, sc.n) for sc in specimens], flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    st = scenes.concat_specimens(specimens)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a))
    b.set_state(t(st["pos"]), t(st["vel"]), t(st["theta"]), t(st["omega"]), t(st["radius"]),
                t(st["mass"]), t(st["id"]))
    b.step(1)
    b.step(steps - 1)
    torch.cuda.synchronize()
    out = {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                       else v.numpy())) for k, v in b.get_state("cpu").items()}
    ranges = [b.slots(s) for s in range(len(specimens))]
    b.check()
    b.close()
    po = PortOracle("f32")
    for s in range(0, len(specimens), 64):
        sc = specimens[s]
        a, e = ranges[s]
        assert e - a == sc.n
        ref = po.run(sc.sys, sc.state(), steps)
        for k in ("pos", "vel", "theta", "omega", "pressure", "acc", "alpha"):
            assert same(out[k][a:e], ref[k]), (s, k)
        assert np.array_equal(out["id"][a:e] - a, ref["id"]), s
