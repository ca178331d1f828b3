"""Seeded disk-splat scenes shared by the renderer tests: particles inside a
unit box with a margin (so that no splat reaches below pixel 0, where the
reference converts negative floats to unsigned), three materials, spins of
either sign, pressures up to twice the colour bar's maximum."""
import numpy as np

COLORS = [(255, 40, 10), (20, 200, 90), (60, 80, 250)]


def splat_scene(seed, n=3000):
    rng = np.random.default_rng(seed)
    return dict(radius=rng.uniform(0.004, 0.02, size=n).astype(np.float32),
                pos=rng.uniform(0.03, 0.97, size=(n, 2)).astype(np.float32),
                theta=rng.uniform(-10.0, 10.0, size=n).astype(np.float32),
                type=rng.integers(0, 3, size=n).astype(np.uint32),
                pressure=rng.uniform(0.0, 2.0, size=n).astype(np.float32),
                height=400 + 37 * seed)


def reference_splat(sc, view_rotations, by_pressure, bg=9, max_pressure=1.5):
    """The reference's own plotSpheresD (host build) over the scene: image and
    the mask of pixels its output cannot class (see RefHarness.render)."""
    from demso_b200 import scenes
    from oracle.oracle import RefHarness
    n = sc["radius"].size
    sys = scenes.agitated_gas(n=64, seed=1, n_mat=3).sys
    sys.Lx = sys.Ly = 1.0
    h = RefHarness()
    h.setup(sys, sc["radius"], np.ones(n, np.float32), sc["type"])
    rgb = np.array([COLORS[t] for t in sc["type"]], np.float32)
    H = sc["height"]
    return h.render(H, H, bg, view_rotations, by_pressure, max_pressure, rgb, sc["pos"],
                    sc["theta"], sc["pressure"])
