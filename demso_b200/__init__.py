"""demso_b200 -- B200-native DEM step of DemSo (blumberg/DemSo).

Python binding of the native library (include/demso_b200.h).  The compute
path is the CUDA library only; this module converts arguments, passes torch
device pointers and the current torch stream through the C ABI, and raises
``DemError`` on any non-zero status.

Two levels mirror the reference's host layer (src/functions.cuh):

* per-stage functions with the reference's names and argument order --
  ``calcHash``, ``sortParticles``, ``reorderDataAndFindCellStart``,
  ``collide``, ``integrateSystem`` -- writing into caller-owned tensors;
* ``Simulation``, the whole step loop of ``SimLooping`` (main.cu:396-507)
  on library-owned buffers (fused kernels, CUDA-graph replay).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Sequence

from . import _lib
from ._lib import (CTX_ACCEL, CTX_AUTOTUNE, CTX_CALLER_STATE, CTX_DIRECT, CTX_PRESSURE,
                   CTX_RESIDENT,
                   DEM_MAX_MATERIALS, STATE_PAD, DemError, check, load)

__all__ = ["Material", "System", "DemError", "calcHash", "sortParticles",
           "reorderDataAndFindCellStart", "collide", "integrateSystem", "Simulation", "Batch",
           "sort_scratch_bytes", "load", "CTX_PRESSURE", "CTX_ACCEL", "CTX_DIRECT",
           "CTX_AUTOTUNE", "CTX_CALLER_STATE", "CTX_RESIDENT", "STATE_PAD"]


@dataclass
class Material:
    """Contact coefficients of one particle type (main.cuh:39-54)."""
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
    """Scene-wide parameters (SystemProperties, main.cuh:108-122) + materials."""
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

    @property
    def key_bits(self) -> int:
        return max(0, (self.num_cells - 1).bit_length())

    def to_c(self, n: int = 0) -> "_lib.DemSystem":
        s = _lib.DemSystem()
        s.numParticles = n
        s.cubeDimension[0], s.cubeDimension[1] = self.Lx, self.Ly
        s.gridSize[0], s.gridSize[1] = self.gx, self.gy
        s.timeStep = self.dt
        s.gravity[0], s.gravity[1] = float(self.gravity[0]), float(self.gravity[1])
        s.boundaryNormalStiffness = self.knWall
        s.boundaryShearStiffness = self.ktWall
        if not 1 <= len(self.materials) <= DEM_MAX_MATERIALS:
            raise ValueError("need 1..%d materials" % DEM_MAX_MATERIALS)
        s.numMaterials = len(self.materials)
        for i, m in enumerate(self.materials):
            (s.materials[i].normalStiffness, s.materials[i].shearStiffness,
             s.materials[i].normalDamping, s.materials[i].boundaryDamping,
             s.materials[i].frictionCoefficient, s.materials[i].attractCoefficient) = m.row()
        return s


def _ptr(t) -> Optional[int]:
    """Device pointer of a torch CUDA tensor (None passes NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


class _DeviceSpan:
    """A device array the library owns, exposed through
    ``__cuda_array_interface__`` so that ``torch.as_tensor`` wraps it without
    a copy."""

    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


def _stream(stream=None) -> Optional[int]:
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream or None


# ---------------------------------------------------------------------------
# per-stage entry points (functions.cuh:50-72)
# ---------------------------------------------------------------------------
def calcHash(sys: System, pos, gridParticleIndex, gridParticleHash, numParticles: int,
             stream=None) -> None:
    """calcHash (functions.cu:315-327)."""
    s = sys.to_c(numParticles)
    check(load().dem_calc_hash(s, _ptr(pos), _ptr(gridParticleIndex), _ptr(gridParticleHash),
                               numParticles, _stream(stream)))


def sort_scratch_bytes(numParticles: int, keyBits: int) -> int:
    return int(load().dem_sort_scratch_bytes(numParticles, keyBits))


def sortParticles(gridParticleHash, gridParticleIndex, numParticles: int, keyBits: int = 32,
                  scratch=None, stream=None) -> None:
    """sortParticles (functions.cu:336-341): stable in-place sort by hash.

    ``scratch`` is a uint8 CUDA tensor of ``sort_scratch_bytes`` bytes; one
    is allocated when omitted."""
    import torch
    need = sort_scratch_bytes(numParticles, keyBits)
    if scratch is None:
        scratch = torch.empty(max(need, 1), dtype=torch.uint8, device=gridParticleHash.device)
    check(load().dem_sort_particles(_ptr(gridParticleHash), _ptr(gridParticleIndex), numParticles,
                                    keyBits, _ptr(scratch), scratch.numel(), _stream(stream)))


def reorderDataAndFindCellStart(sys: System, cellStart, cellEnd, sortedPos, sortedVel,
                                sortedTheta, sortedOmega, sortedRadius, sortedMass, sortedID,
                                sortedLoc, sortedType, gridParticleHash, gridParticleIndex,
                                oldPos, oldVel, oldTheta, oldOmega, oldRadius, oldMass, oldID,
                                oldType, numParticles: int, numCells: int, stream=None) -> None:
    """reorderDataAndFindCellStart (functions.cu:347-393) + radius/mass."""
    s = sys.to_c(numParticles)
    check(load().dem_reorder_data_and_find_cell_start(
        s, _ptr(cellStart), _ptr(cellEnd), _ptr(sortedPos), _ptr(sortedVel), _ptr(sortedTheta),
        _ptr(sortedOmega), _ptr(sortedRadius), _ptr(sortedMass), _ptr(sortedID), _ptr(sortedLoc),
        _ptr(sortedType), _ptr(gridParticleHash), _ptr(gridParticleIndex), _ptr(oldPos),
        _ptr(oldVel), _ptr(oldTheta), _ptr(oldOmega), _ptr(oldRadius), _ptr(oldMass),
        _ptr(oldID), _ptr(oldType), numParticles, numCells, _stream(stream)))


def collide(sys: System, oldPos, oldVel, newAcc, oldOmega, newAlpha, oldType, oldRadius, oldMass,
            cellStart, cellEnd, numParticles: int, numCells: int, pressure=None,
            stream=None) -> None:
    """collide (functions.cu:398-467), without the control particle."""
    s = sys.to_c(numParticles)
    check(load().dem_collide(s, _ptr(oldPos), _ptr(oldVel), _ptr(newAcc), _ptr(oldOmega),
                             _ptr(newAlpha), _ptr(oldType), _ptr(oldRadius), _ptr(oldMass),
                             _ptr(cellStart), _ptr(cellEnd), numParticles, numCells,
                             _ptr(pressure), _stream(stream)))


def integrateSystem(sys: System, pos, vel, acc, theta, omega, alpha, type_, radius, mass,
                    pressure, numParticles: int, stream=None) -> None:
    """integrateSystem (functions.cu:529-551), in place."""
    s = sys.to_c(numParticles)
    check(load().dem_integrate_system(s, _ptr(pos), _ptr(vel), _ptr(acc), _ptr(theta),
                                      _ptr(omega), _ptr(alpha), _ptr(type_), _ptr(radius),
                                      _ptr(mass), _ptr(pressure), numParticles, _stream(stream)))


# ---------------------------------------------------------------------------
# context
# ---------------------------------------------------------------------------
class Simulation:
    """Library-owned state and the fused, graph-captured step (dem_step)."""

    def __init__(self, sys: System, capacity: int, flags: int = CTX_PRESSURE, _handle=None,
                 rows=None):
        """`rows` = (first, count): a context over those cell rows of the
        grid only (dem_create_rows); None for the whole grid."""
        import ctypes as C
        self.sys = sys
        self.capacity = int(capacity)
        self.flags = flags
        self.rows = None if rows is None else (int(rows[0]), int(rows[1]))
        if _handle is None:
            self._h = C.c_void_p()
            if self.rows is None:
                check(load().dem_create(sys.to_c(0), self.capacity, flags, C.byref(self._h)))
            else:
                check(load().dem_create_rows(sys.to_c(0), self.capacity, flags, self.rows[0],
                                             self.rows[1], C.byref(self._h)))
        else:
            self._h = _handle
        self.n = 0
        self._adopted = None

    def close(self) -> None:
        if self._h:
            load().dem_destroy(self._h)
            self._h = None
        self._adopted = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_system(self, sys: System) -> None:
        check(load().dem_set_system(self._h, sys.to_c(self.n)))
        self.sys = sys

    def set_state(self, pos, vel, theta, omega, radius, mass, ids, type_=None, stream=None):
        """Tensors on the GPU (device copy) or on the CPU (host copy)."""
        host = not pos.is_cuda
        ptr = (lambda t: None if t is None else t.data_ptr())
        n = pos.shape[0]
        for t in (pos, vel, theta, omega, radius, mass, ids):
            if not t.is_contiguous() or t.is_cuda == host:
                raise ValueError("state tensors must be contiguous and on one device")
        check(load().dem_set_state(self._h, n, ptr(pos), ptr(vel), ptr(theta), ptr(omega),
                                   ptr(radius), ptr(mass), ptr(ids), ptr(type_), int(host),
                                   _stream(stream)))
        self.n = n

    def get_state(self, device="cuda", stream=None) -> dict:
        """Current state (cell-sorted order) as a dict of tensors."""
        import torch
        n = self.n
        host = str(device) == "cpu"
        kw = dict(device=device, pin_memory=host) if host else dict(device=device)
        out = dict(pos=torch.empty((n, 2), dtype=torch.float32, **kw),
                   vel=torch.empty((n, 2), dtype=torch.float32, **kw),
                   theta=torch.empty(n, dtype=torch.float32, **kw),
                   omega=torch.empty(n, dtype=torch.float32, **kw),
                   radius=torch.empty(n, dtype=torch.float32, **kw),
                   mass=torch.empty(n, dtype=torch.float32, **kw),
                   id=torch.empty(n, dtype=torch.int32, **kw),
                   loc=torch.empty(n, dtype=torch.int32, **kw),
                   pressure=torch.empty(n, dtype=torch.float32, **kw),
                   acc=torch.empty((n, 2), dtype=torch.float32, **kw),
                   alpha=torch.empty(n, dtype=torch.float32, **kw))
        typed = len(self.sys.materials) > 1
        out["type"] = torch.empty(n, dtype=torch.int32, **kw) if typed else None
        p = (lambda k: None if out[k] is None else out[k].data_ptr())
        st = _stream(stream)
        check(load().dem_get_state(self._h, p("pos"), p("vel"), p("theta"), p("omega"),
                                   p("radius"), p("mass"), p("id"), p("type"), p("loc"),
                                   p("pressure") if self.flags & CTX_PRESSURE else None,
                                   p("acc") if self.flags & CTX_ACCEL else None,
                                   p("alpha") if self.flags & CTX_ACCEL else None,
                                   int(host), st))
        if host:
            torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
        return out

    _SET_FIELDS = ("pos", "vel", "theta", "omega", "radius", "mass", "id", "type")

    def adopt_state(self, first: dict, second: dict, n: int, stream=None) -> None:
        """Steps in caller-owned CUDA tensors (dem_adopt_state): the
        reference's two ping-pong sets of ParticlesValues (functions.cu:68-149)
        as dicts of ``_SET_FIELDS``.  ``first`` holds the initial state of n
        particles; ``pos`` and ``radius`` hold n + STATE_PAD rows.  This object
        keeps the tensors alive until the next adopt_state or close."""
        import ctypes as C
        sets = []
        for d in (first, second):
            ss = _lib.DemStateSet()
            for k in self._SET_FIELDS:
                setattr(ss, k, _ptr(d.get(k)))
            sets.append(ss)
        check(load().dem_adopt_state(self._h, int(n), C.byref(sets[0]), C.byref(sets[1]),
                                     _stream(stream)))
        self._adopted = (first, second)
        self.n = int(n)

    def state_view(self) -> dict:
        """The current state without a copy (dem_state_view): tensors over the
        buffers that hold it, valid until the next step, set_state or
        adopt_state, plus ``set`` (0 or 1), the set that holds every field but
        the positions."""
        import ctypes as C
        import torch
        v = _lib.DemStateSet()
        which = C.c_int(0)
        check(load().dem_state_view(self._h, C.byref(v), C.byref(which)))
        n = self.n
        shapes = {"pos": ((n, 2), "<f4"), "vel": ((n, 2), "<f4"), "theta": ((n,), "<f4"),
                  "omega": ((n,), "<f4"), "radius": ((n,), "<f4"), "mass": ((n,), "<f4"),
                  "id": ((n,), "<i4"), "type": ((n,), "<i4")}
        out = {}
        for k, (shape, ts) in shapes.items():
            ptr = getattr(v, k)
            out[k] = None if ptr is None else torch.as_tensor(_DeviceSpan(ptr, shape, ts),
                                                              device="cuda")
        out["set"] = which.value
        return out

    def step(self, nsteps: int = 1, stream=None) -> None:
        check(load().dem_step(self._h, int(nsteps), _stream(stream)))

    def check(self, stream=None) -> None:
        check(load().dem_check(self._h, _stream(stream)))

    def kernels_per_step(self) -> int:
        return int(load().dem_kernels_per_step(self._h))

    def step_variant(self) -> dict:
        """The step kernel's launch shape (dem_get_step_variant): variant,
        threads, blocks_per_sm, tuned (1 by the autotuner, 0 fixed, -1 still
        timing) and the tuner's median ms per variant."""
        from ._lib import DemStepVariant
        import ctypes as C
        v = DemStepVariant()
        check(load().dem_get_step_variant(self._h, C.byref(v)))
        return {"variant": v.variant, "threads": v.threads, "blocks_per_sm": v.blocksPerSm,
                "tuned": v.tuned, "median_ms": [float(x) for x in v.medianMs]}

    def set_step_variant(self, variant: int) -> None:
        check(load().dem_set_step_variant(self._h, int(variant)))

    def set_control(self, pos, radius, material=0, vel=(0.0, 0.0), theta=0.0, omega=0.0,
                    drift=(0.0, 0.0), wrap_y=None, wrap_x=None, stream=None) -> None:
        """The control particle (dem_set_control); ``wrap_y`` = (below, to) and
        ``wrap_x`` = (above, to), None for no wrap.  ``set_control(None, 0)``
        removes it."""
        import ctypes as C
        if pos is None:
            check(load().dem_set_control(self._h, None, _stream(stream)))
            return
        c = _lib.DemControl()
        c.pos[0], c.pos[1] = pos
        c.vel[0], c.vel[1] = vel
        c.theta, c.omega, c.radius, c.material = theta, omega, radius, material
        c.drift[0], c.drift[1] = drift
        nan = float("nan")
        c.wrapYBelow, c.wrapYTo = wrap_y if wrap_y is not None else (nan, nan)
        c.wrapXAbove, c.wrapXTo = wrap_x if wrap_x is not None else (nan, nan)
        check(load().dem_set_control(self._h, C.byref(c), _stream(stream)))

    def control(self, stream=None):
        """(position (x, y), reaction (fx, fy, moment) of the last step)."""
        import ctypes as C
        c = _lib.DemControl()
        r = (C.c_float * 3)()
        check(load().dem_get_control(self._h, C.byref(c), r, _stream(stream)))
        return (c.pos[0], c.pos[1]), (r[0], r[1], r[2])

    def render(self, params, image=None, stream=None):
        """The disk splat of the current state (dem_render) into a CUDA uint8
        tensor of shape (imageDIMy, imageDIMx, 4), row 0 at the bottom."""
        import ctypes as C
        import torch
        if image is None:
            image = torch.empty((params.imageDIMy, params.imageDIMx, 4), dtype=torch.uint8,
                                device="cuda")
        check(load().dem_render(self._h, C.byref(params), image.data_ptr(), _stream(stream)))
        return image

    def followed(self, ids, stream=None):
        """Rows of dem_get_followed for the given particle ids: an (n, 12)
        float32 array (id and type as integer bits)."""
        import numpy as np
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        rows = np.zeros((ids.size, 12), np.float32)
        if ids.size:
            check(load().dem_get_followed(self._h, ids.ctypes.data, ids.size, rows.ctypes.data,
                                          _stream(stream)))
        return rows

    def followed_async(self, ids, rows, stream=None) -> None:
        """dem_get_followed_async: enqueues the rows of `ids` into `rows`, an
        (n, 12) float32 tensor in pinned host memory (or on the GPU), and
        returns without waiting.  Synchronise `stream`, or an event recorded
        on it after this call, before reading `rows`."""
        import numpy as np
        import torch
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        if rows.dtype != torch.float32 or not rows.is_contiguous() or rows.numel() < 12 * ids.size:
            raise ValueError("rows must be a contiguous float32 tensor of 12 * len(ids) values")
        if ids.size:
            check(load().dem_get_followed_async(self._h, ids.ctypes.data, ids.size,
                                                rows.data_ptr(), _stream(stream)))

    def step_followed(self, nsteps: int, ids, rows=None, stream=None):
        """dem_step_followed: `nsteps` steps with the followed rows of `ids`
        after each, into `rows`, a contiguous float32 tensor of
        nsteps * len(ids) * 12 values in pinned host memory or on the GPU
        (returned without waiting: synchronise `stream` before reading it), or,
        when None, a new (nsteps, len(ids), 12) numpy array (filled on
        return)."""
        import numpy as np
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        need = int(nsteps) * ids.size * 12
        if rows is None:
            out = np.zeros((int(nsteps), ids.size, 12), np.float32)
            ptr = out.ctypes.data
        else:
            import torch
            if rows.dtype != torch.float32 or not rows.is_contiguous() or rows.numel() < need:
                raise ValueError("rows must be a contiguous float32 tensor of "
                                 "nsteps * 12 * len(ids) values")
            out, ptr = rows, rows.data_ptr()
        check(load().dem_step_followed(self._h, int(nsteps), ids.ctypes.data if ids.size else None,
                                       ids.size, ptr if ids.size else None, _stream(stream)))
        if rows is None:
            import torch
            (stream or torch.cuda.current_stream()).synchronize()
        return out

    # -- adjoint (dem_adj_forward / dem_adj_backward) ------------------------
    def adjoint_forward(self, nsteps: int, every: int, stream=None) -> None:
        """`nsteps` steps as ``step``, keeping a checkpoint every `every` steps
        (needs flags with CTX_ACCEL)."""
        check(load().dem_adj_forward(self._h, int(nsteps), int(every), _stream(stream)))

    def adjoint_backward(self, lam_pos, lam_vel, lam_omega, stream=None):
        """Reverse pass of the last ``adjoint_forward``.  lam_* are contiguous
        float32 CUDA tensors in particle-id order holding the cotangents of
        the final pos (n, 2), vel (n, 2) and omega (n,); on return they hold
        those of the initial state.  Returns the coefficient gradients as a
        (specimens, 7) float64 array: pair normal stiffness, pair shear
        stiffness, pair dashpot, pair friction, floor dashpot, floor friction,
        floor shear stiffness."""
        import ctypes as C
        ns = getattr(self, "num_specimens", 1)
        for t in (lam_pos, lam_vel, lam_omega):
            if not (t.is_cuda and t.is_contiguous() and t.dtype.itemsize == 4):
                raise ValueError("cotangents must be contiguous float32 CUDA tensors")
        grad = (C.c_double * (_lib.ADJ_NUM_COEF * ns))()
        check(load().dem_adj_backward(self._h, lam_pos.data_ptr(), lam_vel.data_ptr(),
                                      lam_omega.data_ptr(), grad, _stream(stream)))
        import numpy as np
        return np.array(list(grad)).reshape(ns, _lib.ADJ_NUM_COEF)

    def cells(self, stream=None):
        """(cellStart, cellEnd) of the last step's reorder as int32 CUDA tensors."""
        import torch
        nc = self.sys.num_cells
        cs = torch.empty(nc, dtype=torch.int32, device="cuda")
        ce = torch.empty(nc, dtype=torch.int32, device="cuda")
        check(load().dem_get_cells(self._h, cs.data_ptr(), ce.data_ptr(), _stream(stream)))
        return cs, ce


class Batch(Simulation):
    """Many independent scenes stepped together (dem_batch_create).

    ``specs`` is a list of (System, particle count).  State arrays are the
    concatenation of the specimens in order; ``slots(s)`` gives the slot range
    of specimen s, which never changes."""

    def __init__(self, specs, flags: int = CTX_PRESSURE):
        import ctypes as C
        arr = (_lib.DemSystem * len(specs))()
        total = 0
        for k, (sys, n) in enumerate(specs):
            arr[k] = sys.to_c(int(n))
            total += int(n)
        h = C.c_void_p()
        check(load().dem_batch_create(arr, len(specs), flags, C.byref(h)))
        super().__init__(specs[0][0], total, flags, _handle=h)
        self.specs = specs
        self.num_specimens = len(specs)
        self.materials_max = max(len(sys.materials) for sys, _ in specs)

    def set_systems(self, systems, stream=None) -> None:
        """New parameters for every specimen (same grids and counts), copied
        on `stream` (default: torch's current stream) after the steps already
        queued there."""
        arr = (_lib.DemSystem * len(systems))()
        for k, sys in enumerate(systems):
            arr[k] = sys.to_c(int(self.specs[k][1]))
        check(load().dem_batch_set_systems(self._h, arr, len(systems), _stream(stream)))
        self.specs = [(sys, n) for sys, (_, n) in zip(systems, self.specs)]

    def slots(self, s: int):
        import ctypes as C
        a, b = C.c_uint32(), C.c_uint32()
        check(load().dem_batch_specimen(self._h, s, C.byref(a), C.byref(b)))
        return a.value, a.value + b.value

    def get_state(self, device="cuda", stream=None) -> dict:
        # the typed layout follows the largest material count in the batch
        saved = self.sys
        if self.materials_max > 1 and len(self.sys.materials) == 1:
            self.sys = self.specs[[len(sp.materials) for sp, _ in self.specs].index(
                self.materials_max)][0]
        try:
            return super().get_state(device, stream)
        finally:
            self.sys = saved
