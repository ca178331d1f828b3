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


def test_profiles_conserve_area_and_differentiate():
    """The column-height profile: every disk's area lands in its specimen's
    bins (over bin width and packing, to the fixed-point resolution), the sums
    do not depend on the order of the disks, and dL/dx equals central
    differences of the loss (the binning is piecewise linear)."""
    import torch
    sp = C.column_specimens(3, seed=5, nmin=200, nmax=400)
    prof = C.Profiles(sp, "cpu")
    x = torch.tensor(np.concatenate([s.pos[:, 0] for s in sp]), dtype=torch.float64)
    n = x.shape[0]
    h = prof(x)
    r = np.concatenate([s.radius for s in sp]).astype(np.float64)
    tol = n / C.Profiles.FIXED * 2
    assert abs(float(h.sum()) * prof.bw * C.PACKING - np.pi * (r * r).sum()) < tol
    k = 0
    for s in sp:
        nb = int(np.ceil(s.sys.Lx / prof.bw))
        rs = s.radius.astype(np.float64)
        assert abs(float(h[k:k + nb].sum()) * prof.bw * C.PACKING - np.pi * (rs * rs).sum()) < tol
        k += nb
    rng = np.random.default_rng(1)
    xs = x + torch.tensor(rng.uniform(0, 5e-3, size=n))
    # the same positions in another order (scale and bins permuted alike) sum
    # to the same bits
    perm = torch.from_numpy(rng.permutation(n))
    prof2 = C.Profiles(sp, "cpu")
    prof2.first, prof2.last, prof2.scale = prof.first[perm], prof.last[perm], prof.scale[perm]
    assert torch.equal(prof(xs), prof2(xs[perm]))
    target = prof(xs) + torch.tensor(rng.normal(scale=1e-3, size=prof.nbins))
    g = prof.grad(xs, prof(xs), target)
    for i in rng.choice(n, size=8, replace=False):
        e = torch.zeros_like(xs)
        e[i] = 1e-7
        fd = (prof.loss(prof(xs + e), target) - prof.loss(prof(xs - e), target)) / 2e-7
        assert abs(fd - float(g[i])) <= 1e-5 * abs(fd) + 1e-9, (fd, float(g[i]))


def test_trimmed_total_resists_a_few_blown_up_specimens():
    rng = np.random.default_rng(2)
    per = rng.normal(loc=[1.0, -2.0], scale=0.1, size=(100, 2))
    clean = C.trimmed_total(per)
    per[:3] = [[1e9, 1e9], [-1e9, 5e8], [2e9, -3e9]]
    noisy = C.trimmed_total(per)
    assert np.allclose(clean, [100.0, -200.0], rtol=0.05)
    assert np.allclose(noisy, clean, rtol=0.05)
    assert np.array_equal(C.trimmed_total(np.zeros((7, 2))), np.zeros(2))
    assert np.allclose(C.trimmed_total(np.ones((3, 2))), [3.0, 3.0])
