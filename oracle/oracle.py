"""Test infrastructure (oracle only): ctypes wrappers for the CPU oracles.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference arms import this module, and only as the checker or the timed CPU
baseline.  The product path (the ``demso_b200`` package and its CUDA
library) never imports or calls anything here.

Four oracles are wrapped:

* ``PortOracle`` -- ``dem_oracle.c``, our CPU restatement of the reference's
  step (particles_kernel.cuh / functions.cu / main.cu), in float
  (``libdem_oracle_f32.so``) or double (``libdem_oracle_f64.so``).
* ``TangentOracle`` -- ``dem_tangent.cpp``, the forward-mode derivative of
  the same step (the FP64 oracle of the adjoint).
* ``RefDsml`` -- ``_ref/libdsml_ref.so``, the reference's own scene-file
  parser, with the block generators of ``_ref/libdemso_ref.so``.
* ``RefHarness`` -- ``_ref/libdemso_ref.so``, the reference's own
  ``src/particles_kernel.cuh`` compiled for the host by oracle/Makefile (only
  when the reference tree was present at build time).

Both take arrays in the reference layout: ``pos``/``vel``/``acc`` are
(n, 2) float arrays, everything else (n,).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
MAX_MATERIALS = 10

_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


@dataclass
class Material:
    """Per-type contact coefficients (reference ParticleProperties, main.cuh:39-54)."""
    normalStiffness: float
    shearStiffness: float
    normalDamping: float
    boundaryDamping: float
    frictionCoefficient: float
    attractCoefficient: float = 0.0

    def row(self):
        return [self.normalStiffness, self.shearStiffness, self.normalDamping,
                self.boundaryDamping, self.frictionCoefficient, self.attractCoefficient]


@dataclass
class System:
    """Scene-wide parameters (reference SystemProperties, main.cuh:108-122)."""
    Lx: float
    Ly: float
    gx: int
    gy: int
    dt: float
    gravity: Sequence[float] = (0.0, -9.81)
    knWall: float = 0.0
    ktWall: float = 0.0
    materials: list = field(default_factory=list)

    @property
    def num_cells(self) -> int:
        return self.gx * self.gy


class _OrcSystem(C.Structure):
    _fields_ = [("Lx", C.c_double), ("Ly", C.c_double), ("gx", C.c_uint32), ("gy", C.c_uint32),
                ("dt", C.c_double), ("gravx", C.c_double), ("gravy", C.c_double),
                ("knWall", C.c_double), ("ktWall", C.c_double), ("nmat", C.c_uint32),
                ("reserved", C.c_uint32), ("mat", (C.c_double * 6) * MAX_MATERIALS)]


def _orc_system(s: System) -> _OrcSystem:
    o = _OrcSystem()
    o.Lx, o.Ly, o.gx, o.gy, o.dt = s.Lx, s.Ly, s.gx, s.gy, s.dt
    o.gravx, o.gravy = float(s.gravity[0]), float(s.gravity[1])
    o.knWall, o.ktWall = s.knWall, s.ktWall
    if not 1 <= len(s.materials) <= MAX_MATERIALS:
        raise ValueError("need 1..%d materials" % MAX_MATERIALS)
    o.nmat = len(s.materials)
    for m, mat in enumerate(s.materials):
        for k, v in enumerate(mat.row()):
            o.mat[m][k] = v
    return o


class OrcControl(C.Structure):
    """The control particle (dem_oracle.h)."""
    _fields_ = [("pos", C.c_double * 2), ("vel", C.c_double * 2), ("theta", C.c_double),
                ("omega", C.c_double), ("radius", C.c_double), ("mat", C.c_uint32),
                ("reserved", C.c_uint32), ("drift", C.c_double * 2), ("wrapYBelow", C.c_double),
                ("wrapYTo", C.c_double), ("wrapXAbove", C.c_double), ("wrapXTo", C.c_double)]


def orc_control(ctl: dict) -> OrcControl:
    """dict keys: pos, vel, theta, omega, radius, mat, drift, wrap_y (below, to) and
    wrap_x (above, to); missing wraps are off."""
    c = OrcControl()
    c.pos[0], c.pos[1] = ctl["pos"]
    c.vel[0], c.vel[1] = ctl.get("vel", (0.0, 0.0))
    c.theta, c.omega = ctl.get("theta", 0.0), ctl.get("omega", 0.0)
    c.radius, c.mat = ctl["radius"], int(ctl.get("mat", 0))
    c.drift[0], c.drift[1] = ctl.get("drift", (0.0, 0.0))
    nan = float("nan")
    c.wrapYBelow, c.wrapYTo = ctl.get("wrap_y", (nan, nan))
    c.wrapXAbove, c.wrapXTo = ctl.get("wrap_x", (nan, nan))
    return c


# Where this build container mounts the reference checkout; the REF_ROOT
# environment variable overrides it.
_DEFAULT_REF_ROOT = "/root/reference"


def ref_root() -> Optional[str]:
    """The reference checkout: $REF_ROOT, else the container's mount point;
    None when neither holds the reference's sources."""
    root = os.environ.get("REF_ROOT") or _DEFAULT_REF_ROOT
    return root if os.path.isfile(os.path.join(root, "src", "particles_kernel.cuh")) else None


def build(ref_root_dir: Optional[str] = None, quiet: bool = True) -> None:
    """Compile the oracles (and the reference host build when its tree exists)."""
    targets = ["all"]
    root = ref_root_dir or ref_root()
    args = []
    if root:
        targets.append("ref")
        args.append("REF_ROOT=" + root)
    subprocess.run(["make", "-C", HERE] + args + targets, check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def ref_available() -> bool:
    return os.path.isfile(os.path.join(OUT, "libdemso_ref.so"))


# ---------------------------------------------------------------------------
# CPU restatement
# ---------------------------------------------------------------------------
class PortOracle:
    """The C restatement (dem_oracle.c) at float or double precision."""

    def __init__(self, precision: str = "f32"):
        if precision not in ("f32", "f64"):
            raise ValueError(precision)
        path = os.path.join(OUT, "libdem_oracle_%s.so" % precision)
        if not os.path.isfile(path):
            build()
        self.lib = C.CDLL(path)
        self.dt = np.float32 if precision == "f32" else np.float64
        rp = _f32p if precision == "f32" else _f64p
        L = self.lib
        sp = C.POINTER(_OrcSystem)
        u32 = C.c_uint32
        L.orc_calc_hash.argtypes = [sp, u32, rp, _u32p, _u32p]
        L.orc_sort.argtypes = [u32, _u32p, _u32p]
        L.orc_reorder.argtypes = [sp, u32, _u32p, _u32p] + [rp] * 6 + [_u32p, _u32p, C.c_void_p] + \
            [_u32p, _u32p] + [rp] * 6 + [_u32p, C.c_void_p]
        L.orc_collide.argtypes = [sp, u32, rp, rp, rp, rp, rp, C.c_void_p, _u32p, _u32p,
                                  rp, rp, _f32p]
        L.orc_integrate.argtypes = [sp, u32, rp, rp, rp, rp, rp, rp, rp, rp, C.c_void_p, _f32p]
        L.orc_signature.restype = C.c_uint64
        L.orc_collide_control.argtypes = [sp, u32, rp, rp, rp, rp, rp, C.c_void_p, _u32p, _u32p,
                                          rp, rp, _f32p, C.POINTER(OrcControl), rp, rp, rp]
        L.orc_control_reduce.argtypes = [u32, _f32p]
        L.orc_control_reduce.restype = C.c_float
        L.orc_control_move.argtypes = [C.POINTER(OrcControl)]
        L.orc_step.argtypes = [sp, u32] + [rp] * 6 + [_u32p, C.c_void_p] + [rp] * 6 + \
            [_u32p, _u32p, C.c_void_p] + [rp, rp, _f32p, _u32p, _u32p, _u32p, _u32p]

    def _r(self, a, shape=None):
        a = np.ascontiguousarray(a, dtype=self.dt)
        return a if shape is None else a.reshape(shape)

    @staticmethod
    def _tp(t):
        if t is None:
            return None
        t = np.ascontiguousarray(t, dtype=np.uint32)
        return t

    def calc_hash(self, sys: System, pos):
        pos = self._r(pos)
        n = pos.shape[0]
        h = np.empty(n, np.uint32)
        ix = np.empty(n, np.uint32)
        self.lib.orc_calc_hash(C.byref(_orc_system(sys)), n, pos.reshape(-1), h, ix)
        return h, ix

    def sort(self, hash_, index):
        h = np.ascontiguousarray(hash_, dtype=np.uint32).copy()
        ix = np.ascontiguousarray(index, dtype=np.uint32).copy()
        self.lib.orc_sort(h.shape[0], h, ix)
        return h, ix

    def reorder(self, sys: System, hash_, index, st: dict, cell_end_init=None):
        n = len(hash_)
        cs = np.empty(sys.num_cells, np.uint32)
        ce = (np.zeros(sys.num_cells, np.uint32) if cell_end_init is None
              else np.array(cell_end_init, dtype=np.uint32))
        out = {k: np.empty_like(self._r(st[k])) for k in ("pos", "vel", "theta", "omega",
                                                          "radius", "mass")}
        out["id"] = np.empty(n, np.uint32)
        out["loc"] = np.zeros(n, np.uint32)
        typ = self._tp(st.get("type"))
        out["type"] = np.empty(n, np.uint32) if typ is not None else None
        src = {k: self._r(st[k]) for k in ("pos", "vel", "theta", "omega", "radius", "mass")}
        self.lib.orc_reorder(
            C.byref(_orc_system(sys)), n, cs, ce,
            out["pos"].reshape(-1), out["vel"].reshape(-1), out["theta"], out["omega"],
            out["radius"], out["mass"], out["id"], out["loc"],
            out["type"].ctypes.data if typ is not None else None,
            np.ascontiguousarray(hash_, dtype=np.uint32), np.ascontiguousarray(index, dtype=np.uint32),
            src["pos"].reshape(-1), src["vel"].reshape(-1), src["theta"], src["omega"],
            src["radius"], src["mass"], np.ascontiguousarray(st["id"], dtype=np.uint32),
            typ.ctypes.data if typ is not None else None)
        if typ is None:
            out["type"] = None
        return cs, ce, out

    def collide(self, sys: System, st: dict, cell_start, cell_end):
        pos = self._r(st["pos"])
        n = pos.shape[0]
        acc = np.empty((n, 2), self.dt)
        alpha = np.empty(n, self.dt)
        pr = np.empty(n, np.float32)
        typ = self._tp(st.get("type"))
        self.lib.orc_collide(C.byref(_orc_system(sys)), n, pos.reshape(-1),
                             self._r(st["vel"]).reshape(-1), self._r(st["omega"]),
                             self._r(st["radius"]), self._r(st["mass"]),
                             typ.ctypes.data if typ is not None else None,
                             np.ascontiguousarray(cell_start, dtype=np.uint32),
                             np.ascontiguousarray(cell_end, dtype=np.uint32),
                             acc.reshape(-1), alpha, pr)
        return acc, alpha, pr

    def collide_control(self, sys: System, st: dict, cell_start, cell_end, ctl: OrcControl):
        """collide with the control particle: acc, alpha, pressure and the
        reaction vectors fx, fy, fm."""
        pos = self._r(st["pos"])
        n = pos.shape[0]
        acc = np.empty((n, 2), self.dt)
        alpha = np.empty(n, self.dt)
        pr = np.empty(n, np.float32)
        fx, fy, fm = (np.zeros(n, self.dt) for _ in range(3))
        typ = self._tp(st.get("type"))
        self.lib.orc_collide_control(C.byref(_orc_system(sys)), n, pos.reshape(-1),
                                     self._r(st["vel"]).reshape(-1), self._r(st["omega"]),
                                     self._r(st["radius"]), self._r(st["mass"]),
                                     typ.ctypes.data if typ is not None else None,
                                     np.ascontiguousarray(cell_start, dtype=np.uint32),
                                     np.ascontiguousarray(cell_end, dtype=np.uint32),
                                     acc.reshape(-1), alpha, pr, C.byref(ctl), fx, fy, fm)
        return acc, alpha, pr, fx, fy, fm

    def control_reduce(self, v) -> np.float32:
        v = np.ascontiguousarray(v, dtype=np.float32)
        return np.float32(self.lib.orc_control_reduce(v.size, v))

    def control_move(self, ctl: OrcControl) -> None:
        self.lib.orc_control_move(C.byref(ctl))

    def run_control(self, sys: System, st: dict, nsteps: int, ctl: OrcControl):
        """`nsteps` steps with the control particle, each as the reference's
        SimLooping takes it (main.cu:431-514): hash, sort, reorder, collide
        with the control particle and its reaction sums, integrate, then the
        control particle's move.  Returns the final state and the reaction
        (fx, fy, moment) of every step."""
        cur = {k: (None if v is None else np.array(v)) for k, v in st.items()}
        reac = []
        for _ in range(nsteps):
            h, ix = self.calc_hash(sys, cur["pos"])
            h, ix = self.sort(h, ix)
            cs, ce, srt = self.reorder(sys, h, ix, cur)
            acc, alpha, pr, fx, fy, fm = self.collide_control(sys, srt, cs, ce, ctl)
            reac.append((self.control_reduce(fx), self.control_reduce(fy),
                         self.control_reduce(fm)))
            pos, vel, th, om, pr = self.integrate(sys, srt, acc, alpha, pr)
            cur = dict(srt)
            cur.update(pos=pos, vel=vel, theta=th, omega=om, pressure=pr)
            self.control_move(ctl)
        return cur, np.array(reac, np.float32)

    def integrate(self, sys: System, st: dict, acc, alpha, pressure):
        """Returns new (pos, vel, theta, omega, pressure); inputs are not modified."""
        pos = self._r(st["pos"]).copy()
        vel = self._r(st["vel"]).copy()
        th = self._r(st["theta"]).copy()
        om = self._r(st["omega"]).copy()
        pr = np.array(pressure, dtype=np.float32)
        typ = self._tp(st.get("type"))
        n = pos.shape[0]
        self.lib.orc_integrate(C.byref(_orc_system(sys)), n, pos.reshape(-1), vel.reshape(-1),
                               self._r(acc).reshape(-1), th, om, self._r(alpha),
                               self._r(st["radius"]), self._r(st["mass"]),
                               typ.ctypes.data if typ is not None else None, pr)
        return pos, vel, th, om, pr

    def run(self, sys: System, st: dict, nsteps: int):
        """`nsteps` full steps; returns the final sorted state dict plus
        acc/alpha/pressure/cellStart/cellEnd/hash/index of the last step, and
        `signature`, a hash of every branch the contact law and the
        integrator took."""
        self.lib.orc_signature_reset()
        a = {k: self._r(st[k]).copy() for k in ("pos", "vel", "theta", "omega", "radius", "mass")}
        n = a["pos"].shape[0]
        a["id"] = np.ascontiguousarray(st["id"], dtype=np.uint32).copy()
        typ = self._tp(st.get("type"))
        a["type"] = typ.copy() if typ is not None else None
        b = {k: np.empty_like(v) for k, v in a.items() if v is not None}
        b["type"] = np.empty(n, np.uint32) if typ is not None else None
        b["loc"] = np.zeros(n, np.uint32)
        a["loc"] = np.zeros(n, np.uint32)
        acc = np.zeros((n, 2), self.dt)
        alpha = np.zeros(n, self.dt)
        pr = np.zeros(n, np.float32)
        h = np.zeros(n, np.uint32)
        ix = np.zeros(n, np.uint32)
        cs = np.zeros(sys.num_cells, np.uint32)
        ce = np.zeros(sys.num_cells, np.uint32)
        osys = _orc_system(sys)
        for _ in range(nsteps):
            self.lib.orc_step(
                C.byref(osys), n, a["pos"].reshape(-1), a["vel"].reshape(-1), a["theta"],
                a["omega"], a["radius"], a["mass"], a["id"],
                a["type"].ctypes.data if a["type"] is not None else None,
                b["pos"].reshape(-1), b["vel"].reshape(-1), b["theta"], b["omega"], b["radius"],
                b["mass"], b["id"], b["loc"],
                b["type"].ctypes.data if b["type"] is not None else None,
                acc.reshape(-1), alpha, pr, h, ix, cs, ce)
            a, b = b, a
        out = dict(a)
        out.update(acc=acc, alpha=alpha, pressure=pr, cellStart=cs, cellEnd=ce, hash=h, index=ix,
                   signature=int(self.lib.orc_signature()))
        return out


class TangentOracle:
    """Forward-mode tangent of the oracle step (dem_tangent.cpp) in float or
    double: the oracle's trajectory, bit-identical to ``PortOracle`` at the
    same precision, plus its exact derivatives along up to four seeded
    directions (the derivative with every branch held as taken)."""

    DIRECTIONS = 4

    def __init__(self, precision: str = "f64"):
        if precision not in ("f32", "f64"):
            raise ValueError(precision)
        path = os.path.join(OUT, "libdem_tangent_%s.so" % precision)
        if not os.path.isfile(path):
            build()
        self.lib = C.CDLL(path)
        u32 = C.c_uint32
        self.lib.tan_run.argtypes = [C.POINTER(_OrcSystem), u32, u32] + [_f64p] * 6 + [_u32p] + \
            [_f64p] * 5 + [C.POINTER(C.c_uint64)]
        self.lib.tan_run.restype = C.c_int

    def run(self, sys: System, st: dict, nsteps: int, dmat=None, dwall=None, dpos=None,
            dvel=None, domega=None):
        """`nsteps` steps from ``st`` with the given tangents (direction-major:
        dmat (4, 6) over the material row of ``Material.row()``, dwall (4, 2)
        over (knWall, ktWall), dpos/dvel (4, n, 2), domega (4, n)).  Returns
        the final sorted state with ``dpos``/``dvel``/``domega`` (final
        tangents, sorted order) and ``signature``."""
        K = self.DIRECTIONS
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64).copy()
        out = {k: f(st[k]) for k in ("pos", "vel", "theta", "omega", "radius", "mass")}
        n = out["pos"].shape[0]
        out["id"] = np.ascontiguousarray(st["id"], dtype=np.uint32).copy()
        z = lambda shape, a: np.zeros(shape) if a is None else f(np.broadcast_to(a, shape))
        dmat, dwall = z((K, 6), dmat), z((K, 2), dwall)
        dpos, dvel, domega = z((K, n, 2), dpos), z((K, n, 2), dvel), z((K, n), domega)
        sig = C.c_uint64(0)
        rc = self.lib.tan_run(C.byref(_orc_system(sys)), n, nsteps, out["pos"].reshape(-1),
                              out["vel"].reshape(-1), out["theta"], out["omega"], out["radius"],
                              out["mass"], out["id"], dmat.reshape(-1), dwall.reshape(-1),
                              dpos.reshape(-1), dvel.reshape(-1), domega.reshape(-1),
                              C.byref(sig))
        if rc != 0:
            raise ValueError("the tangent oracle takes one material without attraction")
        out.update(dpos=dpos, dvel=dvel, domega=domega, signature=int(sig.value))
        return out


# ---------------------------------------------------------------------------
# Reference host build
# ---------------------------------------------------------------------------
class RefHarness:
    """The reference's own kernels (src/particles_kernel.cuh) run on host cores.

    Particle i is given its own reference "type" i carrying radius[i],
    mass[i] and the coefficients of material[i]; the reference's ``type``
    arrays therefore hold particle ids.  Global state lives in the library
    (the reference's constant-memory symbols), so one harness per process.
    """

    def __init__(self, threads: Optional[int] = None, control: bool = False):
        path = os.path.join(OUT, "libdemso_ref_ctrl.so" if control else "libdemso_ref.so")
        if not os.path.isfile(path):
            raise FileNotFoundError("reference host build missing: " + path)
        self.lib = C.CDLL(path)
        L = self.lib
        u32 = C.c_uint32
        f = C.c_float
        L.ref_setup.argtypes = [u32, f, f, u32, u32, f, f, f, f, f, _f32p, _f32p, C.c_void_p,
                                _f32p, u32]
        L.ref_setup.restype = C.c_int
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_set_threads.restype = C.c_int
        L.ref_calc_hash.argtypes = [_f32p, _u32p, _u32p]
        L.ref_sort.argtypes = [_u32p, _u32p]
        L.ref_reorder.argtypes = [_u32p, _u32p, _f32p, _f32p, _f32p, _f32p, _u32p, _u32p, _u32p,
                                  _u32p, _u32p, _f32p, _f32p, _f32p, _f32p, _u32p, _u32p]
        L.ref_collide.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _u32p, _u32p, _u32p, _f32p]
        L.ref_integrate.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _f32p, _u32p, _f32p]
        L.ref_run.argtypes = [u32] + [_f32p] * 4 + [_u32p] * 3 + [_f32p] * 4 + [_u32p] * 3 + \
            [_f32p, _f32p, _f32p, _u32p, _u32p, _u32p, _u32p]
        L.ref_max_particles.restype = C.c_int
        L.ref_render.argtypes = [np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS"),
                                 C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, _f32p,
                                 _f32p, _f32p, C.c_void_p,
                                 np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")]
        L.ref_render.restype = C.c_int
        if control:
            f = C.c_float
            L.ref_set_control.argtypes = [f, f, f, f, f, f, f, f, _f32p]
            L.ref_set_control.restype = C.c_int
            L.ref_control_vectors.argtypes = [_f32p, _f32p, _f32p]
        self.threads = L.ref_set_threads(int(threads or 0))
        self.sys = None
        self.n = 0

    def setup(self, sys: System, radius, mass, material=None):
        radius = np.ascontiguousarray(radius, dtype=np.float32)
        mass = np.ascontiguousarray(mass, dtype=np.float32)
        n = radius.shape[0]
        tab = np.zeros((MAX_MATERIALS, 6), np.float32)
        for m, mat in enumerate(sys.materials):
            tab[m] = mat.row()
        mt = None if material is None else np.ascontiguousarray(material, dtype=np.uint32)
        rc = self.lib.ref_setup(n, sys.Lx, sys.Ly, sys.gx, sys.gy, sys.dt, float(sys.gravity[0]),
                                float(sys.gravity[1]), sys.knWall, sys.ktWall, radius, mass,
                                mt.ctypes.data if mt is not None else None, tab.reshape(-1),
                                len(sys.materials))
        if rc != 0:
            raise ValueError("ref_setup failed: %d" % rc)
        self.sys, self.n = sys, n

    def set_control(self, pos, vel, theta, omega, radius, mass, material):
        """The control particle (control build only), of reference type n."""
        row = np.ascontiguousarray(material.row(), dtype=np.float32)
        rc = self.lib.ref_set_control(pos[0], pos[1], vel[0], vel[1], theta, omega, radius, mass,
                                      row)
        if rc != 0:
            raise ValueError("ref_set_control failed")

    def control_vectors(self):
        fx, fy, fm = (np.empty(self.n, np.float32) for _ in range(3))
        self.lib.ref_control_vectors(fx, fy, fm)
        return fx, fy, fm

    def calc_hash(self, pos):
        pos = np.ascontiguousarray(pos, dtype=np.float32)
        h = np.empty(self.n, np.uint32)
        ix = np.empty(self.n, np.uint32)
        self.lib.ref_calc_hash(pos.reshape(-1), h, ix)
        return h, ix

    def sort(self, hash_, index):
        h = np.array(hash_, dtype=np.uint32)
        ix = np.array(index, dtype=np.uint32)
        self.lib.ref_sort(h, ix)
        return h, ix

    def reorder(self, hash_, index, pos, vel, theta, omega, ids, cell_end_init=None):
        n = self.n
        cs = np.empty(self.sys.num_cells, np.uint32)
        ce = (np.zeros(self.sys.num_cells, np.uint32) if cell_end_init is None
              else np.array(cell_end_init, dtype=np.uint32))
        sp = np.empty((n, 2), np.float32)
        sv = np.empty((n, 2), np.float32)
        sth = np.empty(n, np.float32)
        som = np.empty(n, np.float32)
        sid = np.empty(n, np.uint32)
        sloc = np.zeros(n, np.uint32)
        styp = np.empty(n, np.uint32)
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        self.lib.ref_reorder(cs, ce, sp.reshape(-1), sv.reshape(-1), sth, som, sid, sloc, styp,
                             np.ascontiguousarray(hash_, dtype=np.uint32),
                             np.ascontiguousarray(index, dtype=np.uint32),
                             np.ascontiguousarray(pos, dtype=np.float32).reshape(-1),
                             np.ascontiguousarray(vel, dtype=np.float32).reshape(-1),
                             np.ascontiguousarray(theta, dtype=np.float32),
                             np.ascontiguousarray(omega, dtype=np.float32), ids, ids.copy())
        return cs, ce, dict(pos=sp, vel=sv, theta=sth, omega=som, id=sid, loc=sloc, type=styp)

    def collide(self, pos, vel, omega, ids, cell_start, cell_end):
        n = self.n
        acc = np.empty((n, 2), np.float32)
        alpha = np.empty(n, np.float32)
        pr = np.empty(n, np.float32)
        self.lib.ref_collide(np.ascontiguousarray(pos, dtype=np.float32).reshape(-1),
                             np.ascontiguousarray(vel, dtype=np.float32).reshape(-1),
                             acc.reshape(-1), np.ascontiguousarray(omega, dtype=np.float32), alpha,
                             np.ascontiguousarray(ids, dtype=np.uint32),
                             np.ascontiguousarray(cell_start, dtype=np.uint32),
                             np.ascontiguousarray(cell_end, dtype=np.uint32), pr)
        return acc, alpha, pr

    def integrate(self, pos, vel, acc, theta, omega, alpha, ids, pressure):
        pos = np.array(pos, dtype=np.float32)
        vel = np.array(vel, dtype=np.float32)
        th = np.array(theta, dtype=np.float32)
        om = np.array(omega, dtype=np.float32)
        pr = np.array(pressure, dtype=np.float32)
        self.lib.ref_integrate(pos.reshape(-1), vel.reshape(-1),
                               np.ascontiguousarray(acc, dtype=np.float32).reshape(-1), th, om,
                               np.ascontiguousarray(alpha, dtype=np.float32),
                               np.ascontiguousarray(ids, dtype=np.uint32), pr)
        return pos, vel, th, om, pr

    def render(self, dimx, dimy, bg, view_rotations, by_pressure, max_pressure, rgb, pos, theta,
               pressure=None):
        """The reference's plotSpheresD over the particles of the last setup,
        in index order, disks first and orientation lines after every disk;
        rgb: (n, 3) colour of each particle.  Returns (image (dimy, dimx, 4)
        uint8, mask (dimy, dimx) of the pixels whose line/disk class the
        reference's output cannot decide: disk pixels of shade 0 under a
        possible line)."""
        img = np.zeros((dimy, dimx, 4), np.uint8)
        amb = np.zeros((dimy, dimx), np.uint8)
        pr = None if pressure is None else np.ascontiguousarray(pressure, dtype=np.float32)
        k = self.lib.ref_render(img.reshape(-1), int(dimx), int(dimy), int(bg),
                                int(bool(view_rotations)), int(bool(by_pressure)),
                                float(max_pressure),
                                np.ascontiguousarray(pos, dtype=np.float32).reshape(-1),
                                np.ascontiguousarray(theta, dtype=np.float32),
                                np.ascontiguousarray(rgb, dtype=np.float32).reshape(-1),
                                pr.ctypes.data if pr is not None else None, amb.reshape(-1))
        if k < 0:
            raise ValueError("a particle's square reaches below pixel 0")
        return img, amb.astype(bool)

    def make_buffers(self, st: dict):
        """Allocate the two state sets and scratch for ``run`` (kept out of timing)."""
        n = self.n
        b = {}
        b["pos1"] = np.ascontiguousarray(st["pos"], dtype=np.float32).copy()
        b["vel1"] = np.ascontiguousarray(st["vel"], dtype=np.float32).copy()
        b["theta1"] = np.ascontiguousarray(st["theta"], dtype=np.float32).copy()
        b["omega1"] = np.ascontiguousarray(st["omega"], dtype=np.float32).copy()
        b["id1"] = np.ascontiguousarray(st["id"], dtype=np.uint32).copy()
        b["type1"] = b["id1"].copy()
        b["loc1"] = np.zeros(n, np.uint32)
        for k in ("pos", "vel"):
            b[k + "2"] = np.zeros((n, 2), np.float32)
        for k in ("theta", "omega"):
            b[k + "2"] = np.zeros(n, np.float32)
        for k in ("id", "type", "loc"):
            b[k + "2"] = np.zeros(n, np.uint32)
        b["acc"] = np.zeros((n, 2), np.float32)
        b["alpha"] = np.zeros(n, np.float32)
        b["pressure"] = np.zeros(n, np.float32)
        b["hash"] = np.zeros(n, np.uint32)
        b["index"] = np.zeros(n, np.uint32)
        b["cellStart"] = np.zeros(self.sys.num_cells, np.uint32)
        b["cellEnd"] = np.zeros(self.sys.num_cells, np.uint32)
        return b

    def run(self, b: dict, nsteps: int):
        """`nsteps` full reference steps in place on buffers from ``make_buffers``."""
        self.lib.ref_run(nsteps, b["pos1"].reshape(-1), b["vel1"].reshape(-1), b["theta1"],
                         b["omega1"], b["id1"], b["type1"], b["loc1"], b["pos2"].reshape(-1),
                         b["vel2"].reshape(-1), b["theta2"], b["omega2"], b["id2"], b["type2"],
                         b["loc2"], b["acc"].reshape(-1), b["alpha"], b["pressure"], b["hash"],
                         b["index"], b["cellStart"], b["cellEnd"])
        return b


# ---------------------------------------------------------------------------
# Reference scene parser and block generators (host builds)
# ---------------------------------------------------------------------------
def dsml_ref_available() -> bool:
    return (os.path.isfile(os.path.join(OUT, "libdsml_ref.so"))
            and os.path.isfile(os.path.join(OUT, "libdemso_ref.so")))


class RefDsml:
    """The reference's own .dsml parser (src/parser.cpp, src/DEMSimulation.cpp)
    and block generator kernels (createRectanglesD with a zero normal deviate,
    createTrianglesD), built for the host by oracle/Makefile.  ``load``
    returns the parsed scene and the particles the reference would create,
    in PrepareSim's order (main.cu:246-325): single particles, rectangles,
    triangles.  The parser is handed a copy without color attributes (it
    overflows its colour buffers, parser.cpp:120-134)."""

    def __init__(self):
        self.p = C.CDLL(os.path.join(OUT, "libdsml_ref.so"))
        self.k = C.CDLL(os.path.join(OUT, "libdemso_ref.so"))
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        self.p.ref_dsml_load.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        self.p.ref_dsml_counts.argtypes = [ip]
        self.p.ref_dsml_params.argtypes = [dp]
        self.p.ref_dsml_type.argtypes = [C.c_int, dp, C.c_char_p, C.c_int]
        self.p.ref_dsml_rect.argtypes = [C.c_int, dp, ip]
        self.p.ref_dsml_tri.argtypes = [C.c_int, dp, ip]
        self.p.ref_dsml_single.argtypes = [C.c_int, dp]
        self.p.ref_dsml_followed.argtypes = [ip, ip]
        u = C.c_uint32
        f = C.c_float
        self.k.ref_create_rectangles.argtypes = [_f32p, _u32p, _u32p, _u32p, f, f, f, f, u, u, u,
                                                 u, _u32p]
        self.k.ref_create_triangles.argtypes = [_f32p, _u32p, _u32p, _u32p, f, f, f, u, u, u,
                                                _u32p]

    def load(self, path: str, tmpdir: str):
        import re
        text = open(path, "rb").read()
        text = re.sub(rb"\scolor=\"[^\"]*\"", b"", text)
        tmp = os.path.join(tmpdir, "ref_nocolor.dsml")
        open(tmp, "wb").write(text)
        err = C.create_string_buffer(512)
        if self.p.ref_dsml_load(tmp.encode(), err, 512):
            return {"error": err.value.decode()}
        c = (C.c_int * 7)()
        self.p.ref_dsml_counts(c)
        nt, nr, ntri, ns, nfs, nfp, _ = list(c)
        par = (C.c_double * 9)()
        self.p.ref_dsml_params(par)
        out = {"params": list(par), "types": [], "followed": []}
        for t in range(nt):
            v = (C.c_double * 11)()
            name = C.create_string_buffer(128)
            self.p.ref_dsml_type(t, v, name, 128)
            out["types"].append({"id": name.value.decode(), "values": list(v)[:8]})
        fs = (C.c_int * max(nfs, 1))()
        fp = (C.c_int * max(nfp, 1))()
        self.p.ref_dsml_followed(fs, fp)
        out["followed"] = list(fs)[:nfs] + list(fp)[:nfp]
        pos, ids, types = [], [], []
        start = 0
        for i in range(ns):
            v = (C.c_double * 7)()
            self.p.ref_dsml_single(i, v)
            pos.append(np.array([[v[0], v[1]]], np.float32))
            types.append(np.array([int(v[6])], np.uint32))
            ids.append(np.array([start], np.uint32))
            start += 1
        for i in range(nr):
            v = (C.c_double * 6)()
            tv = (C.c_int * 16)()
            k = self.p.ref_dsml_rect(i, v, tv)
            nx, ny = int(v[4]), int(v[5])
            m = nx * ny
            p = np.zeros(2 * m, np.float32)
            idv = np.zeros(m, np.uint32)
            loc = np.zeros(m, np.uint32)
            ty = np.zeros(m, np.uint32)
            vec = np.array(list(tv)[:k], np.uint32)
            self.k.ref_create_rectangles(p, idv, loc, ty, v[0], v[1], v[2], v[3], nx, ny, start,
                                         k, vec)
            pos.append(p.reshape(-1, 2)); ids.append(idv); types.append(ty)
            start += m
        for i in range(ntri):
            v = (C.c_double * 4)()
            tv = (C.c_int * 16)()
            k = self.p.ref_dsml_tri(i, v, tv)
            N = int(v[3])
            m = N * (N + 1) // 2
            p = np.zeros(2 * m, np.float32)
            idv = np.zeros(m, np.uint32)
            loc = np.zeros(m, np.uint32)
            ty = np.zeros(m, np.uint32)
            vec = np.array(list(tv)[:k], np.uint32)
            self.k.ref_create_triangles(p, idv, loc, ty, v[0], v[1], v[2], N, start, k, vec)
            pos.append(p.reshape(-1, 2)); ids.append(idv); types.append(ty)
            start += m
        cat = lambda a, dt: np.concatenate(a) if a else np.zeros(0, dt)
        out["pos"] = cat(pos, np.float32).reshape(-1, 2)
        out["id"] = cat(ids, np.uint32)
        out["type"] = cat(types, np.uint32)
        return out


# ---------------------------------------------------------------------------
# Headless outputs (dem_render.c)
# ---------------------------------------------------------------------------
class RenderOracle:
    """CPU disk splat (orc_render) and the output.csv line (orc_followed_line)."""

    def __init__(self):
        path = os.path.join(OUT, "libdem_render.so")
        if not os.path.isfile(path):
            build()
        self.lib = C.CDLL(path)
        u = C.c_uint32
        f = C.c_float
        self.lib.orc_render.argtypes = [u, u, u, C.c_int, C.c_int, f, _f32p, f, f, _f32p,
                                        _f32p, C.c_void_p, _f32p, C.c_void_p, u,
                                        np.ctypeslib.ndpointer(dtype=np.uint8,
                                                               flags="C_CONTIGUOUS")]
        self.lib.orc_followed_line.argtypes = [f, _f32p, u, C.c_char_p, C.c_size_t]
        self.lib.orc_followed_line.restype = C.c_size_t

    def render(self, dimx, dimy, bg, view_rotations, by_pressure, max_pressure, colors, Lx, Ly,
               pos, theta, type_, radius, pressure):
        n = int(np.asarray(radius).size)
        img = np.zeros((dimy, dimx, 4), np.uint8)
        col = np.ascontiguousarray(colors, dtype=np.float32).reshape(-1)
        t = None if type_ is None else np.ascontiguousarray(type_, dtype=np.uint32)
        pr = None if pressure is None else np.ascontiguousarray(pressure, dtype=np.float32)
        self.lib.orc_render(dimx, dimy, bg, int(view_rotations), int(by_pressure), max_pressure,
                            col, Lx, Ly, np.ascontiguousarray(pos, dtype=np.float32).reshape(-1),
                            np.ascontiguousarray(theta, dtype=np.float32),
                            t.ctypes.data if t is not None else None,
                            np.ascontiguousarray(radius, dtype=np.float32),
                            pr.ctypes.data if pr is not None else None, n, img.reshape(-1))
        return img

    def followed_line(self, elapsed, rows) -> str:
        rows = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1)
        buf = C.create_string_buffer(64 + 256 * (rows.size // 12 + 1))
        k = self.lib.orc_followed_line(np.float32(elapsed), rows, rows.size // 12, buf,
                                       len(buf))
        return buf.raw[:k].decode()
