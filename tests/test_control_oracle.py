"""The control particle in the oracle (orc_collide_control, orc_control_reduce,
orc_control_move): pinned bit for bit against the reference's own collideD
built with USE_BIG_PARTICLE 1 for the host (oracle/_ref), and the reduction's
and motion's own rules."""
import numpy as np
import pytest

from demso_b200 import scenes
from oracle.oracle import PortOracle, RefHarness, orc_control
import os
from oracle.oracle import OUT

need_ref = pytest.mark.skipif(not os.path.isfile(os.path.join(OUT, "libdemso_ref_ctrl.so")),
                              reason="reference host build absent")


def control_case(kind):
    if kind == "typed":
        sc = scenes.agitated_gas(n=1500, seed=61, n_mat=3, attraction=10.0, vel_std=0.3)
        mat = 1
    else:
        sc = scenes.agitated_gas(n=2000, seed=62, vel_std=0.3)
        mat = 0
    c = dict(pos=(0.45 * sc.sys.Lx, 0.55 * sc.sys.Ly), vel=(0.1, -0.2), theta=0.3, omega=3.0,
             radius=6e-3, mat=mat, mass=2e-4)
    return sc, c


@need_ref
@pytest.mark.parametrize("kind", ["plain", "typed"])
def test_collide_with_control_matches_the_reference(kind):
    sc, c = control_case(kind)
    st = sc.state()
    ref = RefHarness(control=True)
    typ = st["type"] if st["type"] is not None else np.zeros(sc.n, np.uint32)
    ref.setup(sc.sys, st["radius"], st["mass"], material=typ)
    ref.set_control(c["pos"], c["vel"], c["theta"], c["omega"], c["radius"], c["mass"],
                    sc.sys.materials[c["mat"]])
    h, ix = ref.calc_hash(st["pos"])
    h, ix = ref.sort(h, ix)
    cs, ce, srt = ref.reorder(h, ix, st["pos"], st["vel"], st["theta"], st["omega"],
                              np.arange(sc.n, dtype=np.uint32))
    acc, alpha, pr = ref.collide(srt["pos"], srt["vel"], srt["omega"], srt["id"], cs, ce)
    fx, fy, fm = ref.control_vectors()
    assert np.count_nonzero(fx) > 3            # the control particle touches some disks
    po = PortOracle("f32")
    cs2, ce2, s2 = po.reorder(sc.sys, h, ix, st)
    out = po.collide_control(sc.sys, s2, cs2, ce2, orc_control(c))
    for a, b, name in zip(out, (acc, alpha, pr, fx, fy, fm),
                          ("acc", "alpha", "pressure", "fx", "fy", "fm")):
        assert np.array_equal(a, b), name


def test_reduction_follows_the_reference_tree():
    """reduceVecD over blocks of min(512, n) threads: a tree that halves the
    block size, so entries beyond a power of two in a short block are left
    out (n = 3 sums only the first two), then the block sums in order."""
    po = PortOracle("f32")
    assert po.control_reduce(np.float32([1, 2, 4])) == np.float32(3)
    assert po.control_reduce(np.float32([1, 2, 4, 8])) == np.float32(15)
    v = np.random.default_rng(0).normal(size=1500).astype(np.float32)
    blocks = [v[i:i + 512] for i in range(0, 1536, 512)]
    want = np.float32(0)
    for b in blocks:
        c = np.zeros(512, np.float32)
        c[:b.size] = b
        i = 256
        while i:
            c[:i] = c[:i] + c[i:2 * i]
            i //= 2
        want = np.float32(want + c[0])
    assert po.control_reduce(v) == want


def test_control_motion_is_the_reference_motion():
    """main.cu:511-514: y += -0.005 each step (float += double), wrap to 10.5
    below -1, x wraps to -0.5 beyond Lx + 0.5."""
    po = PortOracle("f32")
    c = orc_control(dict(pos=(10.6, -0.998), radius=0.5, drift=(0.0, -0.005),
                         wrap_y=(-1.0, 10.5), wrap_x=(float(np.float32(10.0)) + 0.5, -0.5)))
    po.control_move(c)
    assert c.pos[1] == 10.5 and c.pos[0] == -0.5
    y = np.float32(5.0)
    c = orc_control(dict(pos=(1.0, 5.0), radius=0.5, drift=(0.0, -0.005)))
    for _ in range(3):
        po.control_move(c)
        y = np.float32(np.float64(y) - 0.005)
    assert c.pos[1] == float(y)
