"""Host-side logic of the calibration: the chain rule from the adjoint's
seven effective coefficients to (kn, friction), checked by finite
differences of the parameter mapping, and the column specimens."""
import numpy as np

from demso_b200 import calibrate as C


def effective(sys):
    """The seven coefficients the adjoint differentiates, as the step forms
    them from a single-material System: pair kn, kt, cn (series of the
    per-type values), pair friction (mean), floor dashpot (the material's),
    floor friction, floor shear stiffness (series with the wall's)."""
    m = sys.materials[0]
    ser = lambda a, b: a * b / (a + b)
    return np.array([ser(m.normalStiffness, m.normalStiffness),
                     ser(m.shearStiffness, m.shearStiffness),
                     ser(m.normalDamping, m.normalDamping),
                     m.frictionCoefficient, m.normalDamping, m.frictionCoefficient,
                     ser(m.shearStiffness, sys.ktWall)])


def test_param_gradient_is_the_chain_rule():
    sc = C.column_scene(300, seed=1)
    rng = np.random.default_rng(0)
    g = rng.normal(size=(3, 7))
    for kn, mu in ((1e5, 0.4), (2.5e5, 0.7)):
        dkn, dmu = C.param_gradient(g, kn)
        h = 1e-6
        jk = (effective(C.with_params(sc.sys, kn * (1 + h), mu))
              - effective(C.with_params(sc.sys, kn * (1 - h), mu))) / (2 * h * kn)
        jm = (effective(C.with_params(sc.sys, kn, mu + h))
              - effective(C.with_params(sc.sys, kn, mu - h))) / (2 * h)
        t = g.sum(axis=0)
        assert abs(dkn - t @ jk) <= 1e-6 * np.abs(t * jk).sum()
        assert abs(dmu - t @ jm) <= 1e-6 * np.abs(t * jm).sum()


def test_column_specimens():
    sp = C.column_specimens(20, seed=2)
    counts = [s.n for s in sp]
    assert min(counts) >= 1024 and max(counts) <= 4096
    for s in sp:
        w = s.pos[:, 0].max() - s.pos[:, 0].min()
        h = s.pos[:, 1].max() - s.pos[:, 1].min()
        assert 1.6 < h / w < 2.5
        # no initial overlaps, inside the box
        assert np.all(s.pos[:, 0] > s.radius) and np.all(s.pos[:, 1] > s.radius)
        d = np.linalg.norm(s.pos[:, None, :] - s.pos[None, :, :], axis=2)
        np.fill_diagonal(d, np.inf)
        assert np.all(d > s.radius[:, None] + s.radius[None, :])
        assert s.sys.gx >= 3 and s.sys.gy >= 3
        assert s.sys.Lx / s.sys.gx > 2 * 1.1e-3 and s.sys.Ly / s.sys.gy > 2 * 1.1e-3
