"""Parity of the CUDA path (through the C ABI) with the reference.

Bit-exact, stage by stage and over whole trajectories, against:
* the golden fixtures made by the reference's own kernels (tests/golden/);
* the CPU restatement (oracle/dem_oracle.c, float) on fresh seeded scenes
  larger than the fixtures.
Also: stable radix sort against numpy's stable argsort, determinism, the
size-independent invariants at full size, and the FP64 trajectory tolerance.
"""
import numpy as np
import pytest

from helpers import (gpu_run, gpu_stages, golden_names, host, load_golden, dev, same,
                     state_of)
from oracle.oracle import PortOracle
from demso_b200 import scenes

pytestmark = pytest.mark.gpu

STAGE_KEYS = ["hash", "index", "sorted_hash", "sorted_index", "cellStart", "cellEnd",
              "sorted_pos", "sorted_vel", "sorted_theta", "sorted_omega", "sorted_id",
              "sorted_loc", "acc", "alpha", "pressure_collide", "int_pos", "int_vel",
              "int_theta", "int_omega", "int_pressure"]
FINAL_KEYS = ["pos", "vel", "theta", "omega", "id", "loc", "pressure", "acc", "alpha"]


@pytest.fixture(scope="module")
def f32():
    return PortOracle("f32")


@pytest.mark.parametrize("name", golden_names())
def test_stages_match_reference_golden(name):
    d = load_golden(name)
    out = gpu_stages(d["sys"], state_of(d))
    for k in STAGE_KEYS:
        assert same(out[k], d[k]), k


@pytest.mark.parametrize("name", golden_names())
def test_step_matches_reference_golden_trajectory(name):
    d = load_golden(name)
    out = gpu_run(d["sys"], state_of(d), d["steps"])
    for k in FINAL_KEYS:
        assert same(out[k], d["final_" + k]), k


@pytest.mark.parametrize("kind,steps", [("gas20k", 300), ("gas_ref", 200), ("gas_mat", 150),
                                        ("pile_c0", 500)])
def test_step_matches_oracle_fresh(f32, kind, steps):
    if kind == "gas20k":
        sc = scenes.agitated_gas(n=20000, seed=7)
    elif kind == "gas_ref":
        sc = scenes.agitated_gas(n=12000, seed=8, grid="ref", vel_std=1.0)
    elif kind == "gas_mat":
        sc = scenes.agitated_gas(n=8000, seed=9, n_mat=5, attraction=30.0)
    else:
        sc = scenes.settling_pile()   # 4,096 disks, the plain settling pile
    out = gpu_run(sc.sys, sc.state(), steps, chunks=[1, 2, steps - 3])
    ref = f32.run(sc.sys, sc.state(), steps)
    for k in FINAL_KEYS:
        assert same(out[k], ref[k]), k


def test_per_stage_equals_fused_step(f32):
    """The fused context step and the five separate entry points agree."""
    sc = scenes.agitated_gas(n=5000, seed=21)
    st = sc.state()
    a = gpu_run(sc.sys, st, 1)
    b = gpu_stages(sc.sys, st)
    assert same(a["pos"], b["int_pos"]) and same(a["vel"], b["int_vel"])
    assert same(a["omega"], b["int_omega"]) and same(a["theta"], b["int_theta"])
    assert same(a["pressure"], b["int_pressure"]) and same(a["acc"], b["acc"])


def test_deterministic_bitwise():
    sc = scenes.agitated_gas(n=30000, seed=5)
    a = gpu_run(sc.sys, sc.state(), 100)
    b = gpu_run(sc.sys, sc.state(), 100)
    for k in FINAL_KEYS:
        assert same(a[k], b[k]), k


# ---------------------------------------------------------------------------- sort
def _sort_gpu(keys, vals, bits):
    import torch
    import demso_b200 as D
    n = keys.shape[0]
    k, v = dev(keys), dev(vals)
    D.sortParticles(k, v, n, keyBits=bits)
    torch.cuda.synchronize()
    return host(k), host(v)


@pytest.mark.parametrize("n", [0, 1, 31, 4095, 4096, 4097, 100003, 1 << 20])
@pytest.mark.parametrize("bits", [1, 7, 10, 20, 22, 32])
def test_radix_sort_is_stable_and_exact(n, bits):
    rng = np.random.default_rng(n * 37 + bits)
    hi = (1 << bits) if bits < 32 else (1 << 32)
    keys = rng.integers(0, hi, size=n, dtype=np.uint64).astype(np.uint32)
    vals = rng.permutation(n).astype(np.uint32)
    k, v = _sort_gpu(keys, vals, bits)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order])
    assert np.array_equal(v, vals[order])


def test_radix_sort_nearly_sorted_and_degenerate():
    rng = np.random.default_rng(3)
    n = 1 << 20
    keys = np.sort(rng.integers(0, 1 << 20, size=n)).astype(np.uint32)
    swap = rng.integers(0, n, size=2000)
    keys[swap] = rng.integers(0, 1 << 20, size=swap.size).astype(np.uint32)
    for ks in (keys, np.zeros(n, np.uint32), np.full(n, (1 << 20) - 1, np.uint32),
               np.arange(n, dtype=np.uint32)[::-1].copy()):
        vals = np.arange(n, dtype=np.uint32)
        k, v = _sort_gpu(ks, vals, 20)
        order = np.argsort(ks, kind="stable")
        assert np.array_equal(k, ks[order]) and np.array_equal(v, vals[order])


def test_radix_sort_zero_bits_is_identity():
    keys = np.zeros(5000, np.uint32)
    vals = np.random.default_rng(0).permutation(5000).astype(np.uint32)
    k, v = _sort_gpu(keys, vals, 0)
    assert np.array_equal(v, vals) and np.array_equal(k, keys)


# ---------------------------------------------------------------- full-size invariants
def test_invariants_at_one_million():
    """Size-independent properties of one step at 1M disks: sorted keys,
    consistent cell ranges, loc inverts id, equal and opposite pair forces."""
    rng = np.random.default_rng(0)
    n = 1 << 20
    sc = scenes.agitated_gas(n=n, seed=31)
    out = gpu_stages(sc.sys, sc.state())
    h = out["sorted_hash"]
    assert np.all(h[1:] >= h[:-1])
    assert np.array_equal(np.sort(out["hash"], kind="stable"), h)
    cs, ce = out["cellStart"], out["cellEnd"]
    occ = cs != 0xFFFFFFFF
    assert int((ce[occ] - cs[occ]).sum()) == n
    assert np.array_equal(np.bincount(h, minlength=sc.sys.num_cells)[occ], (ce - cs)[occ])
    ids = out["sorted_id"]
    assert np.array_equal(out["sorted_loc"][ids], np.arange(n))
    # Newton's third law: sum of m*a over all particles ~ 0 relative to sum |m*a|
    m = out["sorted_mass"].astype(np.float64)
    f = out["acc"].astype(np.float64) * m[:, None]
    assert np.abs(f.sum(0)).max() < 1e-5 * np.abs(f).sum()
    del rng


def test_nan_is_reported_as_oob():
    import torch
    import demso_b200 as D
    sc = scenes.agitated_gas(n=1000, seed=2)
    sc.pos[10] = [np.nan, 0.01]
    sim = D.Simulation(sc.sys, capacity=sc.n)
    t = lambda a: torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a)
    sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass),
                  t(sc.id))
    sim.step(2)
    with pytest.raises(D.DemError) as e:
        sim.check()
    assert e.value.code == 3
    sim.close()


def test_trajectory_within_tolerance_of_fp64_oracle():
    """Positions after 1,000 steps of the plain settling pile (4,096 disks)
    stay within 1e-6 m (0.1 % of the mean radius) of the FP64 oracle."""
    sc = scenes.settling_pile()
    out = gpu_run(sc.sys, sc.state(), 1000)
    ref = PortOracle("f64").run(sc.sys, sc.state(), 1000)
    pa = out["pos"][np.argsort(out["id"])].astype(np.float64)
    pb = ref["pos"][np.argsort(ref["id"])]
    assert np.abs(pa - pb).max() < 1e-6


def _permuted(sc, seed):
    """The same scene with its particles stored in a random order (ids kept)."""
    perm = np.random.default_rng(seed).permutation(sc.n)
    st = sc.state()
    return {k: (None if v is None else np.ascontiguousarray(v[perm])) for k, v in st.items()}


def test_step_from_random_order_matches_oracle(f32):
    """First sort of the context step on a fully shuffled state (the look-back
    sort then sees random keys, not the nearly sorted keys of later steps)."""
    sc = scenes.agitated_gas(n=50000, seed=17)
    st = _permuted(sc, 3)
    out = gpu_run(sc.sys, st, 3)
    ref = f32.run(sc.sys, st, 3)
    for k in FINAL_KEYS:
        assert same(out[k], ref[k]), k


def test_step_scale_scene_matches_oracle(f32):
    """The plain-at-scale workload at 262,144 disks (log-normal radii, random
    sequential placement, neighbour culling active) for 50 steps."""
    sc = scenes.plain_at_scale(262144, seed=5)
    out = gpu_run(sc.sys, sc.state(), 50, chunks=[7, 43])
    ref = f32.run(sc.sys, sc.state(), 50)
    for k in FINAL_KEYS:
        assert same(out[k], ref[k]), k


def test_step_one_million_matches_oracle(f32):
    sc = scenes.agitated_gas(n=1 << 20, seed=41)
    out = gpu_run(sc.sys, sc.state(), 4)
    ref = f32.run(sc.sys, sc.state(), 4)
    for k in FINAL_KEYS:
        assert same(out[k], ref[k]), k


def test_step_with_sixteen_million_cells_matches_oracle(f32):
    """A 4096 x 4096 grid (16.8M cells, more than the cell scan's blocks
    cover at two cells per thread) with a slow gas, so that the incremental
    sort runs on such a grid: 30 steps against the oracle."""
    sc = scenes.agitated_gas(n=30000, seed=23, vel_std=0.2, omega_std=50.0, grid=(4096, 4096))
    out = gpu_run(sc.sys, sc.state(), 30, chunks=[1, 29])
    ref = f32.run(sc.sys, sc.state(), 30)
    for k in FINAL_KEYS:
        assert same(out[k], ref[k]), k
