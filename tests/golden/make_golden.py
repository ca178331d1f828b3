"""Generate the golden fixtures in tests/golden/ from the reference itself.

The outputs come from the reference's own src/particles_kernel.cuh compiled
for the host (oracle/_ref/libdemso_ref.so, built by oracle/Makefile from the
reference tree), so they pin both the CPU restatement (oracle/dem_oracle.c)
and the CUDA library.  Run from the repository root:

    python tests/golden/make_golden.py

Each fixture ``<case>.npz`` holds the input scene, the scene parameters
(``sys_json``), every stage output of the first step, and the state after
``steps`` full steps.  The known-answer scenes restate the parameters of the
reference's example scenes (exemplos/colisao-elastica.dsml,
rolamento-sobre-plano.dsml, singleparticle.dsml) with per-particle values.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from demso_b200 import Material, System, scenes  # noqa: E402
from oracle.oracle import RefHarness, build  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def sys_to_json(s: System) -> str:
    return json.dumps(dict(Lx=s.Lx, Ly=s.Ly, gx=s.gx, gy=s.gy, dt=s.dt, gravity=list(s.gravity),
                           knWall=s.knWall, ktWall=s.ktWall,
                           materials=[m.row() for m in s.materials]))


def sys_from_json(txt: str) -> System:
    d = json.loads(txt)
    mats = [Material(*row) for row in d.pop("materials")]
    return System(materials=mats, **d)


def two_disk_scene(name, Lx, Ly, dt, grav, ktWall, mat, parts, grid):
    """Explicit particles (the reference's <particle> blocks) with one type."""
    n = len(parts)
    pos = np.array([p[0] for p in parts], np.float32)
    vel = np.array([p[1] for p in parts], np.float32)
    theta = np.array([p[2] for p in parts], np.float32)
    omega = np.array([p[3] for p in parts], np.float32)
    radius = np.full(n, mat["radius"], np.float32)
    mass = np.full(n, mat["mass"], np.float32)
    m = Material(mat["kn"], mat["kt"], mat["cn"], mat["eb"], mat["mu"], 0.0)
    s = System(Lx=Lx, Ly=Ly, gx=grid[0], gy=grid[1], dt=dt, gravity=grav, knWall=mat["kn"],
               ktWall=ktWall, materials=[m])
    return scenes.Scene(sys=s, pos=pos, vel=vel, theta=theta, omega=omega, radius=radius,
                        mass=mass, id=np.arange(n, dtype=np.uint32), type=None, name=name)


def known_answer_scenes():
    out = []
    # exemplos/colisao-elastica.dsml: oblique two-disk collision, g = 0, no dashpot
    mat = dict(radius=0.1, mass=0.1, kn=1000.0, kt=1000.0, cn=0.0, eb=0.5, mu=0.4)
    out.append((two_disk_scene("kat_oblique_collision", 5.0, 5.0, 1e-3, (0.0, 0.0), 1000.0, mat,
                               [((2.0, 2.55), (2.0, 0.0), 0.0, 0.0),
                                ((3.0, 2.45), (0.0, 0.0), 0.0, 0.0)],
                               scenes.reference_grid(5.0, 5.0, 0.1)), 1000))
    # exemplos/rolamento-sobre-plano.dsml: one disk on the floor, v = 1 m/s, w = -7.5 rad/s
    mat = dict(radius=0.1, mass=0.1, kn=1e5, kt=1e7, cn=0.0, eb=0.0, mu=0.4)
    out.append((two_disk_scene("kat_rolling_on_floor", 5.0, 5.0, 0.25e-4, (0.0, -9.81), 1e7, mat,
                               [((2.0, 0.1), (1.0, 0.0), 0.0, -7.5)],
                               scenes.reference_grid(5.0, 5.0, 0.1)), 2000))
    # exemplos/singleparticle.dsml: head-on collision with spin, g = 0
    mat = dict(radius=0.2, mass=1.0, kn=1000.0, kt=1e6, cn=0.2, eb=1.0, mu=0.4)
    out.append((two_disk_scene("kat_head_on", 10.0, 10.0, 1e-3, (0.0, 0.0), 100.0, mat,
                               [((1.0, 5.0), (3.0, 0.0), 0.0, 4.0),
                                ((9.0, 5.0), (-3.0, 0.0), 0.0, -4.0)],
                               scenes.reference_grid(10.0, 10.0, 0.2)), 2000))
    return out


def named(sc, name):
    sc.name = name
    return sc


def cases():
    return [
        (named(scenes.agitated_gas(n=1024, seed=11), "gas_2r_1024"), 100),
        (named(scenes.agitated_gas(n=1024, seed=12, grid="ref"), "gas_refgrid_1024"), 100),
        (named(scenes.agitated_gas(n=600, seed=13, n_mat=3, attraction=40.0),
               "gas_3mat_attract_600"), 50),
        (named(scenes.agitated_gas(n=96, seed=14, grid=(2, 2)), "gas_grid2x2_96"), 20),
        (named(scenes.agitated_gas(n=40, seed=15, grid=(1, 1), vel_std=0.05, omega_std=5.0),
               "gas_grid1x1_40"), 5),
        (named(scenes.settling_pile(side=32, box=0.1, seed=0, vel_std=0.2), "pile_1024"), 200),
    ] + known_answer_scenes()


def run_case(ref: RefHarness, sc, steps: int) -> dict:
    s = sc.sys
    material = sc.type
    ref.setup(s, sc.radius, sc.mass, material)
    d = dict(pos=sc.pos, vel=sc.vel, theta=sc.theta, omega=sc.omega, radius=sc.radius,
             mass=sc.mass, id=sc.id, steps=np.int64(steps), sys_json=np.array(sys_to_json(s)))
    if material is not None:
        d["type"] = material
    h, ix = ref.calc_hash(sc.pos)
    d["hash"], d["index"] = h, ix
    hs, ixs = ref.sort(h, ix)
    d["sorted_hash"], d["sorted_index"] = hs, ixs
    cs, ce, o = ref.reorder(hs, ixs, sc.pos, sc.vel, sc.theta, sc.omega, sc.id)
    d["cellStart"] = cs
    d["cellEnd"] = np.where(cs != 0xffffffff, ce, 0).astype(np.uint32)
    for k in ("pos", "vel", "theta", "omega", "id", "loc"):
        d["sorted_" + k] = o[k]
    acc, alpha, pr = ref.collide(o["pos"], o["vel"], o["omega"], o["type"], cs, ce)
    d["acc"], d["alpha"], d["pressure_collide"] = acc, alpha, pr
    p2, v2, th2, om2, pr2 = ref.integrate(o["pos"], o["vel"], acc, o["theta"], o["omega"], alpha,
                                          o["type"], pr)
    d.update(int_pos=p2, int_vel=v2, int_theta=th2, int_omega=om2, int_pressure=pr2)
    b = ref.make_buffers(sc.state())
    ref.run(b, steps)
    d.update(final_pos=b["pos1"], final_vel=b["vel1"], final_theta=b["theta1"],
             final_omega=b["omega1"], final_id=b["id1"], final_loc=b["loc1"],
             final_pressure=b["pressure"], final_acc=b["acc"], final_alpha=b["alpha"])
    return d


def main():
    build()
    ref = RefHarness()
    for sc, steps in cases():
        d = run_case(ref, sc, steps)
        path = os.path.join(OUT, sc.name + ".npz")
        np.savez_compressed(path, **d)
        print("%-28s n=%-5d steps=%-5d %7.1f KB" % (sc.name, sc.n, steps,
                                                     os.path.getsize(path) / 1024))


if __name__ == "__main__":
    main()
