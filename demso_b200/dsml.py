"""The reference's .dsml scene files, read by the library's loader (dem_dsml_*).

``load(path)`` returns the scene's System (box, gravity, time step, wall
stiffnesses, one material per particle type, the reference's grid rule), its
initial state (single particles, then rectangles, then triangles, as the
reference builds them), the followed particle ids and the particle types.
Rectangle lattices are jittered from `seed` (the reference seeds its
generator with the wall clock); ``jitter=False`` gives the unjittered
formula.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import Material, System
from ._lib import DSML_NO_JITTER, DemDsmlInfo, DemDsmlType, DemSystem, check, load as _load


@dataclass
class DsmlScene:
    system: System
    pos: np.ndarray
    vel: np.ndarray
    theta: np.ndarray
    omega: np.ndarray
    radius: np.ndarray
    mass: np.ndarray
    id: np.ndarray
    type: np.ndarray
    followed: np.ndarray
    time_step: float
    sim_duration: float          # seconds; -1 = run forever
    image_height: int
    controlled_type: int         # -1 without a <controlled> tag
    types: list = field(default_factory=list)   # dicts: id, name, mass, radius, color

    @property
    def n(self) -> int:
        return int(self.id.size)

    def state(self) -> dict:
        """State arrays as Scene.state() gives them (type None for one material)."""
        return dict(pos=self.pos, vel=self.vel, theta=self.theta, omega=self.omega,
                    radius=self.radius, mass=self.mass, id=self.id,
                    type=self.type if len(self.system.materials) > 1 else None)


def _system_from_c(s: DemSystem) -> System:
    mats = [Material(m.normalStiffness, m.shearStiffness, m.normalDamping, m.boundaryDamping,
                     m.frictionCoefficient, m.attractCoefficient)
            for m in s.materials[:s.numMaterials]]
    return System(Lx=s.cubeDimension[0], Ly=s.cubeDimension[1], gx=s.gridSize[0],
                  gy=s.gridSize[1], dt=s.timeStep, gravity=(s.gravity[0], s.gravity[1]),
                  knWall=s.boundaryNormalStiffness, ktWall=s.boundaryShearStiffness,
                  materials=mats)


def _scene(handle) -> DsmlScene:
    L = _load()
    info = DemDsmlInfo()
    check(L.dem_dsml_info(handle, C.byref(info)))
    sysc = DemSystem()
    check(L.dem_dsml_system(handle, C.byref(sysc)))
    n = info.numParticles
    arr = {k: np.zeros(shape, dt) for k, shape, dt in (
        ("pos", (n, 2), np.float32), ("vel", (n, 2), np.float32), ("theta", n, np.float32),
        ("omega", n, np.float32), ("radius", n, np.float32), ("mass", n, np.float32),
        ("id", n, np.uint32), ("type", n, np.uint32))}
    check(L.dem_dsml_state(handle, *(arr[k].ctypes.data for k in (
        "pos", "vel", "theta", "omega", "radius", "mass", "id", "type"))))
    followed = np.zeros(info.numFollowed, np.uint32)
    if info.numFollowed:
        check(L.dem_dsml_followed(handle, followed.ctypes.data))
    types = []
    for t in range(info.numTypes):
        d = DemDsmlType()
        check(L.dem_dsml_type(handle, t, C.byref(d)))
        types.append(dict(id=d.id.decode(), name=d.name.decode(errors="replace"),
                          mass=d.mass, radius=d.radius, color=tuple(d.color)))
    return DsmlScene(system=_system_from_c(sysc), followed=followed,
                     time_step=info.timeStep, sim_duration=info.simDuration,
                     image_height=info.imageHeight, controlled_type=info.controlledType,
                     types=types, **arr)


def _with(handle_fn) -> DsmlScene:
    L = _load()
    h = C.c_void_p()
    check(handle_fn(L, C.byref(h)))
    try:
        return _scene(h)
    finally:
        L.dem_dsml_free(h)


def load(path: str, seed: int = 0, jitter: bool = True) -> DsmlScene:
    flags = 0 if jitter else DSML_NO_JITTER
    return _with(lambda L, h: L.dem_dsml_load(str(path).encode(), seed, flags, h))


def parse(text, seed: int = 0, jitter: bool = True) -> DsmlScene:
    data = text.encode() if isinstance(text, str) else bytes(text)
    flags = 0 if jitter else DSML_NO_JITTER
    return _with(lambda L, h: L.dem_dsml_parse(data, len(data), seed, flags, h))
