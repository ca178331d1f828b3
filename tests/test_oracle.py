"""The CPU oracle is pinned before it is trusted.

* The float restatement (oracle/dem_oracle.c) reproduces every golden
  fixture bit for bit.  The fixtures were produced by the reference's own
  src/particles_kernel.cuh compiled for the host (tests/golden/make_golden.py).
* When the reference host build is present (oracle/_ref/libdemso_ref.so),
  restatement and reference also agree on fresh seeded scenes, stage by
  stage and over many steps.
* The double restatement obeys closed forms (free fall is exact for
  symplectic Euler) and tracks the float one.
"""
import math

import numpy as np
import pytest

from helpers import golden_names, load_golden, occupied_cell_end, same, state_of
from oracle.oracle import PortOracle, RefHarness, ref_available
from demso_b200 import scenes


@pytest.fixture(scope="module")
def f32():
    return PortOracle("f32")


@pytest.fixture(scope="module")
def f64():
    return PortOracle("f64")


def oracle_stages(po, sys, st):
    out = {}
    h, ix = po.calc_hash(sys, st["pos"])
    out["hash"], out["index"] = h, ix
    hs, ixs = po.sort(h, ix)
    out["sorted_hash"], out["sorted_index"] = hs, ixs
    cs, ce, o = po.reorder(sys, hs, ixs, st)
    out["cellStart"], out["cellEnd"] = cs, occupied_cell_end(cs, ce)
    for k in ("pos", "vel", "theta", "omega", "id", "loc"):
        out["sorted_" + k] = o[k]
    acc, alpha, pr = po.collide(sys, o, cs, ce)
    out["acc"], out["alpha"], out["pressure_collide"] = acc, alpha, pr
    p, v, th, om, pr2 = po.integrate(sys, o, acc, alpha, pr)
    out.update(int_pos=p, int_vel=v, int_theta=th, int_omega=om, int_pressure=pr2)
    return out


STAGE_KEYS = ["hash", "index", "sorted_hash", "sorted_index", "cellStart", "cellEnd",
              "sorted_pos", "sorted_vel", "sorted_theta", "sorted_omega", "sorted_id",
              "sorted_loc", "acc", "alpha", "pressure_collide", "int_pos", "int_vel",
              "int_theta", "int_omega", "int_pressure"]
FINAL_KEYS = ["pos", "vel", "theta", "omega", "id", "loc", "pressure", "acc", "alpha"]


def test_golden_fixtures_present():
    names = golden_names()
    assert len(names) >= 9
    for kat in ("kat_oblique_collision", "kat_rolling_on_floor", "kat_head_on"):
        assert kat in names


@pytest.mark.parametrize("name", golden_names())
def test_restatement_matches_reference_golden_one_step(f32, name):
    d = load_golden(name)
    out = oracle_stages(f32, d["sys"], state_of(d))
    for k in STAGE_KEYS:
        assert same(out[k], d[k]), k


@pytest.mark.parametrize("name", golden_names())
def test_restatement_matches_reference_golden_trajectory(f32, name):
    d = load_golden(name)
    out = f32.run(d["sys"], state_of(d), d["steps"])
    for k in FINAL_KEYS:
        assert same(out[k], d["final_" + k]), k


def test_fixtures_have_contacts_and_all_branches():
    """The fixtures exercise contacts, the floor and the Coulomb cap."""
    d = load_golden("gas_2r_1024")
    assert np.count_nonzero(d["acc"]) > 500
    assert np.count_nonzero(d["alpha"]) > 200
    assert np.count_nonzero(d["int_pressure"] != d["pressure_collide"]) > 0  # floor contacts
    d = load_golden("kat_oblique_collision")
    # the two disks met and separated: momentum exchanged along x and y
    assert abs(float(d["final_vel"][:, 1].sum())) < 1e-5
    assert np.all(np.abs(d["final_vel"][:, 1]) > 1e-3)


needs_ref = pytest.mark.skipif(not ref_available(), reason="reference host build not present")


@needs_ref
@pytest.mark.parametrize("seed", [101, 102])
@pytest.mark.parametrize("kind", ["gas", "gas_ref", "gas_mat", "pile"])
def test_restatement_matches_reference_fresh(f32, seed, kind):
    ref = RefHarness()
    if kind == "gas":
        sc = scenes.agitated_gas(n=2000, seed=seed)
    elif kind == "gas_ref":
        sc = scenes.agitated_gas(n=1500, seed=seed, grid="ref", vel_std=1.0)
    elif kind == "gas_mat":
        sc = scenes.agitated_gas(n=1200, seed=seed, n_mat=4, attraction=25.0)
    else:
        sc = scenes.settling_pile(side=40, box=0.125, seed=seed, vel_std=0.3)
    ref.setup(sc.sys, sc.radius, sc.mass, sc.type)
    b = ref.make_buffers(sc.state())
    ref.run(b, 60)
    out = f32.run(sc.sys, sc.state(), 60)
    for k in ("pos", "vel", "theta", "omega", "id", "loc"):
        assert same(out[k], b[k + "1"]), k
    assert same(out["pressure"], b["pressure"])


def test_free_fall_closed_form(f64):
    """Symplectic Euler free fall: p_k = p0 + v0 k dt + g dt^2 k (k+1) / 2."""
    sc = scenes.agitated_gas(n=4, seed=3, vel_std=0.0, omega_std=0.0, box=1.0)
    sc.pos[:] = [[0.2, 0.8], [0.4, 0.7], [0.6, 0.9], [0.8, 0.6]]
    sc.vel[:] = [[0.1, 0.0], [-0.1, 0.2], [0.0, 0.0], [0.05, -0.05]]
    k, dt, g = 500, sc.sys.dt, -9.81
    out = f64.run(sc.sys, sc.state(), k)
    order = np.argsort(out["id"])
    p = out["pos"][order]
    p0 = sc.pos.astype(np.float64)
    v0 = sc.vel.astype(np.float64)
    exp_x = p0[:, 0] + v0[:, 0] * k * dt
    exp_y = p0[:, 1] + v0[:, 1] * k * dt + g * dt * dt * k * (k + 1) / 2
    assert np.allclose(p[:, 0], exp_x, rtol=0, atol=1e-12)
    assert np.allclose(p[:, 1], exp_y, rtol=0, atol=1e-12)


def test_head_on_restitution_of_approach_only_dashpot(f64):
    """Two equal disks, head on, no gravity or spin: the dashpot acts only while
    approaching, so the restitution follows the damped half-period of the
    approach and the undamped rebound.  Check the FP64 oracle against that
    closed form (within 2 % for dt << contact time)."""
    from demso_b200 import Material, System
    kn, cn, m, r, v = 1000.0, 0.2, 1.0, 0.2, 1.0
    mat = Material(2 * kn, 0.0, 2 * cn, 1.0, 0.0)
    sys_ = System(Lx=10.0, Ly=10.0, gx=8, gy=8, dt=1e-4, gravity=(0.0, 0.0), materials=[mat])
    st = dict(pos=np.array([[4.7, 5.0], [5.3, 5.0]]), vel=np.array([[v, 0.0], [-v, 0.0]]),
              theta=np.zeros(2), omega=np.zeros(2), radius=np.full(2, r), mass=np.full(2, m),
              id=np.arange(2, dtype=np.uint32), type=None)
    out = f64.run(sys_, st, 20000)
    vf = out["vel"][np.argsort(out["id"])]
    e_sim = abs(vf[1, 0] - vf[0, 0]) / (2 * v)
    # relative motion: m_eff x'' + c x' + k x = 0 with m_eff = m/2 while approaching,
    # the compression phase ends at the velocity zero of the damped oscillator
    meff = m / 2
    w0 = math.sqrt(kn / meff)
    z = cn / (2 * math.sqrt(kn * meff))
    wd = w0 * math.sqrt(1 - z * z)
    t1 = math.atan2(wd, z * w0) / wd           # time of maximum compression
    xmax = (2 * v) / wd * math.exp(-z * w0 * t1) * math.sin(wd * t1)
    e_th = xmax * w0 / (2 * v)                 # undamped rebound from xmax
    assert abs(e_sim - e_th) < 0.02 * e_th


def test_f64_tracks_f32_short_window(f32, f64):
    d = load_golden("pile_1024")
    a = f32.run(d["sys"], state_of(d), 50)
    b = f64.run(d["sys"], state_of(d), 50)
    pa = a["pos"][np.argsort(a["id"])]
    pb = b["pos"][np.argsort(b["id"])]
    assert np.abs(pa - pb).max() < 1e-6
