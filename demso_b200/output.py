"""Headless outputs: the reference's particle image (as a device buffer and
a PPM file) and its followed-particle file output.csv.

``render_params`` builds the renderer's parameters as the reference sets them
up (main.cu:172-177): image height from the scene (800 by default), width
Lx / Ly times the height, black background, orientation lines on, colour by
particle type.  ``ppm_bytes`` turns an RGBA image (row 0 at the bottom of the
box, as the reference's GL buffer) into a binary PPM with row 0 at the top.
``followed_line`` formats one line of output.csv exactly as the reference's
writeOutputFile does (functions.cu:608-661).
"""
from __future__ import annotations

import numpy as np

from . import _lib


def render_params(Lx: float, Ly: float, colors, image_height: int = 800, bg: int = 0,
                  view_rotations: bool = True, color_by_pressure: bool = False,
                  max_pressure: float = 1.0) -> "_lib.DemRenderParams":
    """colors: one (r, g, b) per material, 0..255."""
    p = _lib.DemRenderParams()
    p.imageDIMy = int(image_height)
    # renderPar->imageDIMx = cubeDimension.x / cubeDimension.y * imageDIMy (float, truncated)
    p.imageDIMx = int(np.float32(np.float32(Lx) / np.float32(Ly)) * np.float32(image_height))
    p.bgColor = int(bg) & 0xFF
    p.viewRotations = int(bool(view_rotations))
    p.colorByPressure = int(bool(color_by_pressure))
    p.maxPressure = float(max_pressure)
    if len(colors) > _lib.DEM_MAX_MATERIALS:
        raise ValueError("at most %d colours" % _lib.DEM_MAX_MATERIALS)
    for m, c in enumerate(colors):
        for k in range(3):
            p.color[m][k] = float(c[k])
    return p


def ppm_bytes(image_rgba: np.ndarray) -> bytes:
    """Binary PPM (P6) of an (H, W, 4) uint8 image whose row 0 is the bottom."""
    img = np.ascontiguousarray(image_rgba[::-1, :, :3])
    h, w = img.shape[:2]
    return b"P6\n%d %d\n255\n" % (w, h) + img.tobytes()


def followed_line(elapsed: float, rows: np.ndarray) -> str:
    """One output.csv line: the elapsed time (the float product time step x
    step count), then for each followed particle id, type, x, y, vx, vy, ax,
    ay, theta, omega, alpha, pressure; rows as dem_get_followed returns them
    (12 float32 words per particle, id and type as integer bits)."""
    rows = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1, 12)
    bits = rows.view(np.uint32)
    parts = []
    for r, b in zip(rows, bits):
        parts.append("%u,%u,%s" % (b[0], b[1], ",".join("%f" % float(v) for v in r[2:])))
    return "%f," % float(np.float32(elapsed)) + ",".join(parts) + "\n"


def elapsed_time(dt: float, step: int) -> np.float32:
    """sisProps->timeStep * timeCtrl->tempo as the reference forms it (float)."""
    return np.float32(np.float32(dt) * np.float32(step))
