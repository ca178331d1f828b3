"""Launch shapes of the step kernel and the autotuner that picks one
(DEM_CTX_AUTOTUNE, dem_set_step_variant, dem_get_step_variant).

Every shape -- threads per block and register cap -- computes the same bits,
so a context fixed to any shape, and a context whose first steps rotate
through all of them while they are timed, follow the default context's
trajectory exactly: single scenes (one material, several materials with
attraction, neighbour culling on and off), a batch, and direct launches."""
import numpy as np
import pytest

from demso_b200 import scenes
from helpers import same

pytestmark = pytest.mark.gpu

KEYS = ("pos", "vel", "theta", "omega", "radius", "mass", "id", "pressure", "acc", "alpha")


def _torch(a):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.int32).copy() if a.dtype == np.uint32 else a.copy())


def _host(sim):
    import torch
    torch.cuda.synchronize()
    return {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                        else v.numpy())) for k, v in sim.get_state("cpu").items()}


def run(sc, steps, flags=0, variant=None, chunks=None, batch=None):
    import demso_b200 as D
    flags |= D.CTX_PRESSURE | D.CTX_ACCEL
    if batch is None:
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=flags)
        st = sc.state()
    else:
        sim = D.Batch([(s.sys, s.n) for s in batch], flags=flags)
        st = scenes.concat_specimens(batch)
    sim.set_state(_torch(st["pos"]), _torch(st["vel"]), _torch(st["theta"]),
                  _torch(st["omega"]), _torch(st["radius"]), _torch(st["mass"]),
                  _torch(st["id"]), _torch(st["type"]) if st["type"] is not None else None)
    if variant is not None:
        sim.set_step_variant(variant)
    for c in chunks or [steps]:
        sim.step(c)
    out = _host(sim)
    info = sim.step_variant()
    sim.check()
    sim.close()
    return out, info


def _same_run(a, b):
    for k in KEYS:
        if a[k] is None:
            assert b[k] is None, k
        else:
            assert same(a[k], b[k]), k


SCENES = {
    "pile": lambda: scenes.settling_pile(side=48, box=0.15, seed=2, vel_std=0.3),
    "gas_materials_attraction": lambda: scenes.agitated_gas(n=3000, seed=7, n_mat=3,
                                                            attraction=25.0),
    "gas_no_cull": lambda: scenes.agitated_gas(n=2000, seed=8, grid="ref", vel_std=1.0),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_every_shape_gives_the_default_bits(name):
    import demso_b200 as D
    sc = SCENES[name]()
    ref, info = run(sc, 40)
    assert info["variant"] == 0 and info["tuned"] == 0
    for v in range(1, D._lib.STEP_VARIANTS):
        out, info = run(sc, 40, variant=v)
        assert info["variant"] == v and info["tuned"] == 0
        _same_run(ref, out)


@pytest.mark.parametrize("direct", [False, True])
def test_autotuned_context_follows_the_default_trajectory(direct):
    import demso_b200 as D
    sc = SCENES["pile"]()
    ref, _ = run(sc, 60)
    flags = D.CTX_AUTOTUNE | (D.CTX_DIRECT if direct else 0)
    # the 24 tuning steps straddle the chunks
    out, info = run(sc, 60, flags=flags, chunks=[1, 10, 20, 29])
    _same_run(ref, out)
    assert info["tuned"] == 1
    assert 0 <= info["variant"] < D._lib.STEP_VARIANTS
    med = info["median_ms"]
    assert all(m > 0.0 for m in med)
    assert med[info["variant"]] == min(med)
    assert info["threads"] in (64, 128, 256)


def test_tuning_in_progress_and_fixed_shape():
    import demso_b200 as D
    sc = SCENES["pile"]()
    _, info = run(sc, 10, flags=D.CTX_AUTOTUNE)
    assert info["tuned"] == -1
    # fixing the shape ends the tuning
    out, info = run(sc, 30, flags=D.CTX_AUTOTUNE, variant=2)
    assert info["tuned"] == 0 and info["variant"] == 2 and info["threads"] == 256
    with pytest.raises(D.DemError):
        s = D.Simulation(sc.sys, capacity=sc.n)
        try:
            s.set_step_variant(D._lib.STEP_VARIANTS)
        finally:
            s.close()


def test_autotuned_batch_follows_the_default_trajectory():
    import demso_b200 as D
    batch = scenes.specimen_batch(num=12, seed=5, nmin=64, nmax=2048)
    ref, _ = run(None, 50, batch=batch)
    out, info = run(None, 50, flags=D.CTX_AUTOTUNE, batch=batch)
    _same_run(ref, out)
    assert info["tuned"] == 1
