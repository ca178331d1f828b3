"""Seeded synthetic scenes for the step and the reference's grid-sizing rule.

No dataset is involved anywhere: every scene is generated from a seed with
the sizes and distributions of the workload it names.  Contact parameters
are given as pair values (kn, kt = 0.5 kn, damping ratio, friction) and
mapped onto the reference's per-type coefficients, which combine in series
(particles_kernel.cuh:36-41): a per-type stiffness of 2 kn gives the pair
stiffness kn, and likewise for shear stiffness and the dashpot.  The damping
ratio zeta maps to the pair dashpot coefficient c = 2 zeta sqrt(m_eff kn)
with m_eff = m_ref / 2, m_ref the mass of a disk of the median radius.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import Material, System

RHO = 2650.0          # kg/m^3
THICK = 1e-3          # disk thickness, m


def disk_mass(r, rho=RHO, t=THICK):
    """Mass of a disk of radius r (float32 in, float32 out)."""
    r = np.asarray(r, dtype=np.float64)
    return (rho * math.pi * r * r * t).astype(np.float32)


def pair_material(kn=1e5, kt_ratio=0.5, zeta=0.3, mu=0.5, r_ref=1e-3, e_boundary=0.5,
                  attraction=0.0) -> Material:
    """Per-type coefficients whose series/mean combination gives the pair values."""
    kt = kt_ratio * kn
    m_ref = float(disk_mass(r_ref))
    cn = 2.0 * zeta * math.sqrt(0.5 * m_ref * kn)
    return Material(normalStiffness=2.0 * kn, shearStiffness=2.0 * kt, normalDamping=2.0 * cn,
                    boundaryDamping=e_boundary, frictionCoefficient=mu,
                    attractCoefficient=attraction)


def grid_2r(L: float, rmax: float) -> int:
    """Largest power-of-two cell count whose cell is at least 2 rmax."""
    g = int(math.floor(math.log2(L / (2.0 * rmax))))
    return 1 << max(g, 0)


def reference_grid(Lx: float, Ly: float, rmax: float):
    """The reference's grid-size rule (main.cu:218-236), replayed exactly.

    float32 arithmetic like the reference; log2 is its `log(x)/log(2)` macro
    (main.cu:38) in double; the y branch measures the cell with the box's x
    size, as the reference does."""
    f = np.float32
    Lx, Ly, rmax = f(Lx), f(Ly), f(rmax)

    def axis(num, cell_len):
        grid = int(np.uint32(num))
        temp = int(math.log(grid) / math.log(2)) if grid > 0 else 0
        upd = 1 << temp
        cell = f(cell_len / f(upd))
        if cell / f(2.0) <= f(1.2) * rmax:
            temp -= 1
        elif cell / f(2.0) >= f(3.0) * rmax:
            temp += 1
        return 1 << temp

    gx = axis(Lx / (f(4.0) * rmax), Lx)
    gy = axis(Ly / (f(4) * rmax), Lx)
    return gx, gy


@dataclass
class Scene:
    sys: System
    pos: np.ndarray      # (n, 2) float32
    vel: np.ndarray      # (n, 2) float32
    theta: np.ndarray    # (n,) float32
    omega: np.ndarray    # (n,) float32
    radius: np.ndarray   # (n,) float32
    mass: np.ndarray     # (n,) float32
    id: np.ndarray       # (n,) uint32
    type: np.ndarray = None   # (n,) uint32 material index, None = single material
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.pos.shape[0])

    def state(self) -> dict:
        return dict(pos=self.pos, vel=self.vel, theta=self.theta, omega=self.omega,
                    radius=self.radius, mass=self.mass, id=self.id, type=self.type)


def _finish(sys, pos, vel, radius, rng=None, omega=None, theta=None, type_=None, name=""):
    n = pos.shape[0]
    radius = radius.astype(np.float32)
    return Scene(sys=sys, pos=np.ascontiguousarray(pos, np.float32),
                 vel=np.ascontiguousarray(vel, np.float32),
                 theta=(np.zeros(n, np.float32) if theta is None else theta.astype(np.float32)),
                 omega=(np.zeros(n, np.float32) if omega is None else omega.astype(np.float32)),
                 radius=radius, mass=disk_mass(radius), id=np.arange(n, dtype=np.uint32),
                 type=type_, name=name)


def settling_pile(side=64, box=0.2, seed=0, grid="2r", dt=2e-6, vel_std=0.0) -> Scene:
    """Plain 2D settling pile (4,096 disks at side=64): jittered side x side
    lattice in a box x box walled box, radii U[0.9, 1.1] mm, jitter +-0.1 mm,
    zero velocity, kn 1e5, kt 0.5 kn, zeta 0.3, mu 0.5, dt 2e-6."""
    rng = np.random.default_rng(seed)
    n = side * side
    pitch = box / side
    ij = np.stack(np.meshgrid(np.arange(side), np.arange(side), indexing="xy"), -1).reshape(-1, 2)
    pos = (ij + 0.5) * pitch + rng.uniform(-1e-4, 1e-4, size=(n, 2))
    radius = rng.uniform(0.9e-3, 1.1e-3, size=n)
    vel = rng.normal(0.0, vel_std, size=(n, 2)) if vel_std > 0 else np.zeros((n, 2))
    rmax = 1.1e-3
    gx, gy = ((grid_2r(box, rmax), grid_2r(box, rmax)) if grid == "2r"
              else reference_grid(box, box, rmax))
    mat = pair_material()
    sys = System(Lx=box, Ly=box, gx=gx, gy=gy, dt=dt, gravity=(0.0, -9.81),
                 knWall=mat.normalStiffness, ktWall=mat.shearStiffness, materials=[mat])
    return _finish(sys, pos, vel, radius, name="settling_pile_%d" % n)


def agitated_gas(n=2048, seed=1, pitch_factor=0.95, jitter=0.25, vel_std=0.5, omega_std=200.0,
                 grid="2r", n_mat=1, attraction=0.0, gravity=(0.0, -9.81), dt=2e-6,
                 box=None) -> Scene:
    """Dense random disks with initial overlaps, random velocities and spins:
    every branch of the contact law fires (dashpot on/off, stick and slip,
    walls and floor).  Disks sit on a lattice of pitch `pitch_factor` mean
    diameters, shifted by up to `jitter` pitches, so most have several
    overlapping neighbours; the box is the lattice's extent (or `box`)."""
    rng = np.random.default_rng(seed)
    radius = rng.uniform(0.9e-3, 1.1e-3, size=n)
    side = int(math.ceil(math.sqrt(n)))
    pitch = 2e-3 * pitch_factor
    if box is None:
        box = side * pitch
    ij = np.stack(np.meshgrid(np.arange(side), np.arange(side), indexing="xy"), -1).reshape(-1, 2)[:n]
    pos = (ij + 0.5) * pitch + rng.uniform(-jitter, jitter, size=(n, 2)) * pitch
    pos = np.clip(pos, 1e-5, box - 1e-5)
    vel = rng.normal(0.0, vel_std, size=(n, 2))
    omega = rng.normal(0.0, omega_std, size=n)
    theta = rng.uniform(0.0, 2 * math.pi, size=n)
    rmax = 1.1e-3
    gx, gy = ((grid_2r(box, rmax), grid_2r(box, rmax)) if grid == "2r"
              else reference_grid(box, box, rmax) if grid == "ref" else grid)
    mats = []
    for m in range(n_mat):
        mats.append(pair_material(kn=1e5 * (1 + m), mu=0.5 - 0.1 * m, zeta=0.3 + 0.05 * m,
                                  e_boundary=0.5 + 0.1 * m, attraction=attraction * (m + 1)))
    type_ = rng.integers(0, n_mat, size=n).astype(np.uint32) if n_mat > 1 else None
    sys = System(Lx=box, Ly=box, gx=gx, gy=gy, dt=dt, gravity=gravity,
                 knWall=mats[0].normalStiffness, ktWall=mats[0].shearStiffness, materials=mats)
    return _finish(sys, pos, vel, radius, omega=omega, theta=theta, type_=type_,
                   name="agitated_gas_%d" % n)


def lognormal_radii(n, rng, median=1e-3, sigma=0.15, lo=0.6e-3, hi=1.6e-3):
    return np.clip(median * np.exp(sigma * rng.standard_normal(n)), lo, hi)


def scale_box(n, width_4m=4.1, phi=0.55, er2=None, n_ref=4194304):
    """Box (W, H) for n disks of the plain-at-scale workload: width scales
    with sqrt(n / 4M), height gives area fraction phi."""
    if er2 is None:
        er2 = 1.0458e-6
    W = width_4m * math.sqrt(n / n_ref)
    H = n * math.pi * er2 / (phi * W)
    return W, H


def rsa_positions(radius, W, H, seed=0, strips=None, trials=200):
    """Seeded random sequential placement through the native generator
    (dem_scene_rsa); returns (n, 2) float32 positions."""
    import ctypes as C
    from ._lib import check, load
    radius = np.ascontiguousarray(radius, dtype=np.float32)
    n = radius.shape[0]
    rmax = float(radius.max())
    if strips is None:
        strips = max(1, min(256, int(H / (16 * rmax))))
    pos = np.empty((n, 2), np.float32)
    placed = C.c_uint32(0)
    check(load().dem_scene_rsa(n, radius.ctypes.data, W, H, int(seed), strips, trials,
                               pos.ctypes.data, C.byref(placed)))
    return pos


def plain_at_scale(n=4194304, seed=0, grid="2r", dt=2e-6, phi=0.55) -> Scene:
    """Plain at scale: n disks (4,194,304 by default) with log-normal radii
    (median 1 mm, sigma 0.15, clipped to [0.6, 1.6] mm) in a walled box 4.1 m
    wide at 4M (width scaled by sqrt(n / 4M)), packed to area fraction `phi`
    by seeded random sequential placement; zero initial velocity; the contact
    parameters of the settling pile."""
    rng = np.random.default_rng(seed)
    radius = lognormal_radii(n, rng).astype(np.float32)
    er2 = float(np.mean(radius.astype(np.float64) ** 2))
    W, H = scale_box(n, phi=phi, er2=er2)
    pos = rsa_positions(radius, W, H, seed=seed)
    rmax = 1.6e-3
    gx, gy = ((grid_2r(W, rmax), grid_2r(H, rmax)) if grid == "2r"
              else reference_grid(W, H, rmax))
    mat = pair_material()
    sys = System(Lx=W, Ly=H, gx=gx, gy=gy, dt=dt, gravity=(0.0, -9.81),
                 knWall=mat.normalStiffness, ktWall=mat.shearStiffness, materials=[mat])
    # number the disks in cell order, as the reference's block generators
    # number theirs lattice row by lattice row (createRectanglesD,
    # particles_kernel.cuh:61-71)
    order = np.argsort(cell_hash(pos, sys), kind="stable")
    return _finish(sys, pos[order], np.zeros((n, 2)), radius[order],
                   name="plain_at_scale_%d" % n)


def stacked(scene: Scene, copies: int, by_cell: bool = False) -> Scene:
    """`copies` of a scene stacked upward in one box of the same width and
    `copies` times the height, on one grid of the same cells (copies a power
    of two).  Disks are numbered copy by copy, or in cell order with
    `by_cell`."""
    if copies == 1:
        return scene
    if copies < 1 or copies & (copies - 1):
        raise ValueError("copies must be a power of two (the grid's rows are)")
    b = scene.sys
    sys = System(Lx=b.Lx, Ly=b.Ly * copies, gx=b.gx, gy=b.gy * copies, dt=b.dt,
                 gravity=b.gravity, knWall=b.knWall, ktWall=b.ktWall, materials=b.materials)
    pos = np.concatenate([scene.pos.astype(np.float64) + np.array([0.0, c * b.Ly])
                          for c in range(copies)]).astype(np.float32)
    tile = lambda a: None if a is None else np.concatenate([a] * copies)
    vel, radius = tile(scene.vel), tile(scene.radius)
    omega, theta, type_ = tile(scene.omega), tile(scene.theta), tile(scene.type)
    if by_cell:
        order = np.argsort(cell_hash(pos, sys), kind="stable")
        pos, vel, radius, omega, theta = (a[order] for a in (pos, vel, radius, omega, theta))
        type_ = None if type_ is None else type_[order]
    return _finish(sys, pos, vel, radius, omega=omega, theta=theta, type_=type_,
                   name="%s_x%d" % (scene.name, copies))


def stacked_plain(n=4194304, copies=1, seed=0, dt=2e-6) -> Scene:
    """The workload of a slab decomposition over `copies` GPUs: `copies`
    plain-at-scale scenes of n disks (n per GPU) stacked upward, numbered
    in cell order.  Copies do not overlap: each copy's disks lie inside its
    own walls."""
    return stacked(plain_at_scale(n, seed=seed, dt=dt), copies, by_cell=True)


def cell_hash(pos, sys: System) -> np.ndarray:
    """The reference's cell index of each position (particles_kernel.cuh:114-130),
    with the same float32 operations."""
    p = np.asarray(pos, dtype=np.float32)
    gxf, gyf = np.float32(sys.gx), np.float32(sys.gy)
    cx = np.floor((p[:, 0] * gxf) / np.float32(sys.Lx)).astype(np.int64)
    cy = np.floor((p[:, 1] * gyf) / np.float32(sys.Ly)).astype(np.int64)
    cx &= sys.gx - 1
    cy &= sys.gy - 1
    return (cy * sys.gx + cx).astype(np.uint32)


def specimen_batch(num=4096, seed=0, nmin=256, nmax=8192, phi=0.5, dt=2e-6):
    """Batched workload: `num` independent specimens with particle counts
    log-uniform in [nmin, nmax]; each has its own square walled box at area
    fraction `phi`, radii uniform in [0.9, 1.1] mm, kn log-uniform in
    [5e4, 5e5] N/m, friction uniform in [0.2, 0.8] and damping ratio uniform
    in [0.1, 0.5]; seeded random sequential placement, zero velocity.
    Returns a list of Scenes (one per specimen)."""
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=num)).astype(np.int64)
    kns = np.exp(rng.uniform(np.log(5e4), np.log(5e5), size=num))
    mus = rng.uniform(0.2, 0.8, size=num)
    zetas = rng.uniform(0.1, 0.5, size=num)
    out = []
    rmax = 1.1e-3
    radii = [rng.uniform(0.9e-3, 1.1e-3, size=int(counts[k])).astype(np.float32)
             for k in range(num)]
    boxes = [math.sqrt(r.size * math.pi * float(np.mean(r.astype(np.float64) ** 2)) / phi)
             for r in radii]
    # the native placement releases the GIL: place the specimens in parallel
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=16) as ex:
        placed = list(ex.map(lambda k: rsa_positions(radii[k], boxes[k], boxes[k],
                                                     seed=seed * 100003 + k, strips=1),
                             range(num)))
    for k in range(num):
        n = int(counts[k])
        r, L, pos = radii[k], boxes[k], placed[k]
        g = grid_2r(L, rmax)
        mat = pair_material(kn=float(kns[k]), zeta=float(zetas[k]), mu=float(mus[k]))
        sys = System(Lx=L, Ly=L, gx=g, gy=g, dt=dt, gravity=(0.0, -9.81),
                     knWall=mat.normalStiffness, ktWall=mat.shearStiffness, materials=[mat])
        order = np.argsort(cell_hash(pos, sys), kind="stable")
        out.append(_finish(sys, pos[order], np.zeros((n, 2)), r[order],
                           name="specimen_%d" % k))
    return out


def concat_specimens(specimens):
    """Concatenated state arrays of a batch (ids renumbered 0..N-1)."""
    n = sum(sc.n for sc in specimens)
    cat = lambda k: np.concatenate([getattr(sc, k) for sc in specimens])
    st = dict(pos=cat("pos"), vel=cat("vel"), theta=cat("theta"), omega=cat("omega"),
              radius=cat("radius"), mass=cat("mass"), id=np.arange(n, dtype=np.uint32))
    types = [sc.type for sc in specimens]
    st["type"] = (None if all(t is None for t in types) else
                  np.concatenate([t if t is not None else np.zeros(sc.n, np.uint32)
                                  for t, sc in zip(types, specimens)]))
    return st


def incline_heap(n=16384, seed=0, slope_deg=20.0, vel_std=0.05, phi=0.5, dt=2e-6,
                 kn=1e5, zeta=0.3, mu=0.5):
    """Differentiable workload: n disks (radii U[0.9, 1.1] mm) in a seeded
    heap -- random sequential placement at area fraction `phi` in a
    rectangle twice as wide as high at the bottom-left of a walled box three
    times as wide and twice as high -- with initial velocities N(0, vel_std^2)
    and gravity rotated by `slope_deg`, so that the floor is a wall inclined
    at that angle in the frame of gravity."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.9e-3, 1.1e-3, size=n).astype(np.float32)
    area = n * math.pi * float(np.mean(r.astype(np.float64) ** 2)) / phi
    h = math.sqrt(area / 2.0)
    w = 2.0 * h
    pos = rsa_positions(r, w, h, seed=seed + 7, strips=max(1, int(h / 0.02)))
    Lx, Ly = 3.0 * w, 2.0 * h
    vel = rng.normal(0.0, vel_std, size=(n, 2))
    a = math.radians(slope_deg)
    rmax = 1.1e-3
    mat = pair_material(kn=kn, zeta=zeta, mu=mu)
    sys = System(Lx=Lx, Ly=Ly, gx=grid_2r(Lx, rmax), gy=grid_2r(Ly, rmax), dt=dt,
                 gravity=(9.81 * math.sin(a), -9.81 * math.cos(a)),
                 knWall=mat.normalStiffness, ktWall=mat.shearStiffness, materials=[mat])
    order = np.argsort(cell_hash(pos, sys), kind="stable")
    return _finish(sys, pos[order], vel[order], r[order], name="incline_heap_%d" % n)
