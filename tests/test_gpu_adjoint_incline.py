"""The adjoint on the differentiable workload itself: 16,384 disks released
from a seeded heap onto a 20-degree incline, 2,000 steps, a checkpoint every
100 steps (the scene, step count and interval the adjoint is benchmarked on).

The oracle values come from tests/golden/adjoint_incline_16k.json, made on
host cores by tests/golden/make_adjoint_incline.py:

* the FP32 forward-mode tangent (oracle/dem_tangent.cpp in float), the exact
  derivative of the float trajectory that the GPU forward follows bit for
  bit.  The GPU adjoint must equal it within 1e-3 relative on dL/dkn,
  dL/dzeta, dL/dmu and two seeded random directions over the 16,384 x 2
  initial velocities, and the GPU loss must equal the oracle's bit for bit;
* the FP64 tangent and FP64 central differences (h = 1e-4 relative) with
  the branch signature of every run.  On this scene every perturbation
  crosses branches and float and double trajectories part, so these are
  reported (DEM_TEST_REPORT_DIR) but not asserted.

Contact law followed: particles_kernel.cuh:236-307 (pair), :388-456
(floor), :580-627 (integrate).
"""
import json
import os

import numpy as np
import pytest

from adjoint_harness import gpu_loss_and_grad
from demso_b200 import scenes

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                       "adjoint_incline_16k.json")


def fixture():
    with open(FIXTURE) as f:
        return json.load(f)


def directions(fx, n):
    return [np.random.default_rng(s).normal(size=(n, 2)) for s in fx["direction_seeds"]]


def test_fixture_scene_is_the_generated_scene():
    """The committed oracle values belong to the scene incline_heap makes."""
    import sys
    sys.path.insert(0, os.path.dirname(FIXTURE))
    from make_adjoint_incline import scene_checksum
    fx = fixture()
    sc = scenes.incline_heap(n=fx["n"], seed=0)
    assert scene_checksum(sc) == fx["scene_sha256"]
    assert len(fx["f32_tangent"]) == len(fx["names"]) == 5
    assert fx["f32_loss"] > 0.0


@pytest.mark.gpu
def test_adjoint_on_the_incline_workload_matches_the_float_tangent():
    fx = fixture()
    sc = scenes.incline_heap(n=fx["n"], seed=0)
    loss, (dkn, dz, dmu), dv, g = gpu_loss_and_grad(sc, fx["kn"], fx["zeta"], fx["mu"],
                                                    fx["steps"], fx["every"])
    us = directions(fx, sc.n)
    d_gpu = [dkn, dz, dmu] + [float(np.sum(dv.astype(np.float64) * u)) for u in us]
    rel = lambda a, b: abs(a - b) / abs(b)
    report = {
        "workload": fx["workload"], "names": fx["names"], "gpu": d_gpu, "gpu_loss": loss,
        "coefficient_gradients": list(g),
        "rel_vs_f32_tangent": [rel(a, b) for a, b in zip(d_gpu, fx["f32_tangent"])],
        "rel_vs_f64_tangent": [rel(a, b) for a, b in zip(d_gpu, fx["f64_tangent"])],
        "rel_vs_f64_central_difference": [rel(a, b) for a, b in
                                          zip(d_gpu, fx["f64_central_difference"])],
        "f64_fd_same_branches": fx["f64_fd_same_branches"],
        "loss_equals_f32_oracle": bool(loss == fx["f32_loss"]),
    }
    out_dir = os.environ.get("DEM_TEST_REPORT_DIR")
    if out_dir:
        os.makedirs(out_dir, exist_ok=True)
        with open(os.path.join(out_dir, "adjoint_incline_16k_check.json"), "w") as f:
            json.dump(report, f, indent=1)
    assert np.all(np.isfinite(g)) and np.all(np.isfinite(dv))
    assert loss == fx["f32_loss"]
    for k, name in enumerate(fx["names"]):
        assert report["rel_vs_f32_tangent"][k] < 1e-3, (name, d_gpu[k], fx["f32_tangent"][k])
