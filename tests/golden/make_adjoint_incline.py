"""Generate tests/golden/adjoint_incline_16k.json: the oracle derivatives of
the differentiable workload itself (16,384 disks released from a seeded heap
onto a 20-degree incline, 2,000 steps), against which the GPU adjoint is
checked by tests/test_gpu_adjoint_incline.py.

Everything here runs on host cores from the CPU oracles (oracle/):

* the FP32 forward-mode tangent (dem_tangent.cpp built in float): the exact
  derivative of the float trajectory that the GPU forward follows bit for
  bit, along kn, the damping ratio, friction and two seeded random
  directions over the 16,384 x 2 initial velocities;
* the same five derivatives from the FP64 tangent;
* FP64 central differences (h = 1e-4 relative) of the FP64 oracle loss, with
  the branch signature of every run (whether a perturbation crossed a
  contact, dashpot, slip, wall or floor branch of the unperturbed run), and
  the same differences at h = 1e-6, 1e-8 and 1e-10 relative.

The scene is fixed by its seed; its checksum is stored so that the test can
confirm it generated the same initial state.  Run from the repository root:

    python tests/golden/make_adjoint_incline.py

The runs are spread over a spawned process pool (about six minutes on eight
cores).
"""
from __future__ import annotations

import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.dirname(HERE)):
    if p not in sys.path:
        sys.path.insert(0, p)

N, STEPS, EVERY = 16384, 2000, 100
KN, ZETA, MU = 1e5, 0.3, 0.5
DIR_SEEDS = (7, 8)
H_REL = 1e-4
# smaller steps of the FP64 central difference, to show where it stops
# crossing branches and meets the FP64 tangent
H_STUDY = (1e-6, 1e-8, 1e-10)
OUT = os.path.join(HERE, "adjoint_incline_16k.json")


def scene():
    from demso_b200 import scenes
    return scenes.incline_heap(n=N, seed=0)


def scene_checksum(sc) -> str:
    h = hashlib.sha256()
    for a in (sc.pos, sc.vel, sc.theta, sc.omega, sc.radius, sc.mass, sc.id):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def directions(n):
    return [np.random.default_rng(s).normal(size=(n, 2)) for s in DIR_SEEDS]


def _tangent(args):
    precision, which = args
    from adjoint_harness import tangent_grad
    sc = scene()
    u = directions(sc.n)[which]
    loss, d, sig = tangent_grad(sc, KN, ZETA, MU, STEPS, u, precision)
    return precision, which, loss, [float(x) for x in d], sig


def _f64_loss(args):
    name, x = args
    from adjoint_harness import f64_loss
    sc = scene()
    if name == "kn":
        return name, x, f64_loss(sc, x, ZETA, MU, STEPS)
    if name == "zeta":
        return name, x, f64_loss(sc, KN, x, MU, STEPS)
    if name == "mu":
        return name, x, f64_loss(sc, KN, ZETA, x, STEPS)
    k = int(name[1:])
    u = directions(sc.n)[k]
    v0 = sc.vel.astype(np.float64)[np.argsort(sc.id)]
    return name, x, f64_loss(sc, KN, ZETA, MU, STEPS, vel0=(v0 + (x - 0.05) * u)[sc.id])


def main():
    t0 = time.time()
    sc = scene()
    base = {"kn": KN, "zeta": ZETA, "mu": MU, "u0": 0.05, "u1": 0.05}
    jobs_t = [(p, w) for p in ("f32", "f64") for w in (0, 1)]
    jobs_l = [("kn", KN)]
    for name, x in base.items():
        for hr in (H_REL,) + H_STUDY:
            h = hr * x
            jobs_l += [(name, x + h), (name, x - h)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(len(jobs_t) + len(jobs_l), os.cpu_count() or 1)) as pool:
        rt = pool.map_async(_tangent, jobs_t)
        rl = pool.map_async(_f64_loss, jobs_l)
        tangents, losses = rt.get(), rl.get()
    tan = {}
    for precision, which, loss, d, sig in tangents:
        tan.setdefault(precision, {})["loss"] = loss
        tan[precision]["signature"] = str(sig)
        t = tan[precision].setdefault("d", [None] * 5)
        t[0:3] = d[0:3]
        t[3 + which] = d[3]
    base_loss, base_sig = [v for n_, x, v in losses if n_ == "kn" and x == KN][0]
    def central(hr):
        fd, same = [], []
        for name, x in base.items():
            h = hr * x
            (lp, sp), = [v for n_, xx, v in losses if n_ == name and xx == x + h]
            (lm, sm), = [v for n_, xx, v in losses if n_ == name and xx == x - h]
            fd.append((lp - lm) / (2.0 * h))
            same.append(bool(sp == base_sig and sm == base_sig))
        return fd, same

    fd, same = central(H_REL)
    study = []
    for hr in H_STUDY:
        f, sm_ = central(hr)
        study.append({"h_rel": hr, "central_difference": f, "same_branches": sm_})
    out = {
        "workload": "differentiable: %d disks (radii U[0.9, 1.1] mm) released from a seeded "
                    "heap onto a 20-degree incline, %d steps, checkpoint every %d steps"
                    % (N, STEPS, EVERY),
        "scene_sha256": scene_checksum(sc), "n": N, "steps": STEPS, "every": EVERY,
        "kn": KN, "zeta": ZETA, "mu": MU, "direction_seeds": list(DIR_SEEDS), "h_rel": H_REL,
        "names": ["dL/dkn", "dL/dzeta", "dL/dmu", "dL/dv0 . u(seed 7)", "dL/dv0 . u(seed 8)"],
        "f32_tangent": tan["f32"]["d"], "f32_loss": tan["f32"]["loss"],
        "f32_signature": tan["f32"]["signature"],
        "f64_tangent": tan["f64"]["d"], "f64_loss": tan["f64"]["loss"],
        "f64_loss_oracle": base_loss, "f64_signature": str(base_sig),
        "f64_central_difference": fd, "f64_fd_same_branches": same,
        "f64_fd_step_study": study,
        "generated_s": round(time.time() - t0, 1),
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
