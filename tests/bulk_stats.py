"""Bulk statistics of a disk packing: kinetic energy (translational and
rotational), coordination number (contacts per disk, contact when the centre
distance is below the sum of radii), packing fraction of the lower half of
the heap, and the heap's surface angle (a line fitted to the tops of columns
one mean diameter wide, between 20 % and 80 % of the heap's height)."""
import math

import numpy as np


def bulk_stats(st) -> dict:
    from scipy.spatial import cKDTree
    p = np.asarray(st["pos"], np.float64)
    v = np.asarray(st["vel"], np.float64)
    r = np.asarray(st["radius"], np.float64)
    m = np.asarray(st["mass"], np.float64)
    w = np.asarray(st["omega"], np.float64)
    ke = 0.5 * np.sum(m * np.sum(v * v, 1)) + 0.5 * np.sum(0.4 * m * r * r * w * w)
    pairs = cKDTree(p).query_pairs(2 * r.max(), output_type="ndarray")
    d = np.linalg.norm(p[pairs[:, 0]] - p[pairs[:, 1]], axis=1)
    z = 2.0 * np.sum(d < r[pairs[:, 0]] + r[pairs[:, 1]]) / len(r)
    bw = 2 * r.mean()
    xb = np.floor(p[:, 0] / bw).astype(int)
    tops = {}
    for i in range(len(r)):
        tops[xb[i]] = max(tops.get(xb[i], 0.0), p[i, 1] + r[i])
    xs = np.array(sorted(tops))
    hs = np.array([tops[k] for k in xs])
    xc = (xs + 0.5) * bw
    top = hs.max()
    sel = (hs > 0.2 * top) & (hs < 0.8 * top)
    angle = (math.degrees(math.atan(-np.polyfit(xc[sel], hs[sel], 1)[0]))
             if sel.sum() > 3 else float("nan"))
    inside = p[:, 1] < 0.5 * top
    phi = np.sum(np.pi * r[inside] ** 2) / (p[inside, 0].max() * 0.5 * top)
    return dict(ke=ke, z=z, phi=phi, angle=angle)
