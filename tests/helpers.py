"""Shared test helpers: golden fixtures, device transfer, the GPU stage runner."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

from demso_b200 import Material, System

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EMPTY = np.uint32(0xFFFFFFFF)


def golden_names():
    return sorted(os.path.splitext(os.path.basename(p))[0]
                  for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def sys_from_json(txt: str) -> System:
    d = json.loads(str(txt))
    mats = [Material(*row) for row in d.pop("materials")]
    d["gravity"] = tuple(d["gravity"])
    return System(materials=mats, **d)


def load_golden(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["sys"] = sys_from_json(d.pop("sys_json"))
    d["steps"] = int(d["steps"])
    d.setdefault("type", None)
    return d


def state_of(d: dict) -> dict:
    return dict(pos=d["pos"], vel=d["vel"], theta=d["theta"], omega=d["omega"],
                radius=d["radius"], mass=d["mass"], id=d["id"], type=d.get("type"))


def same(a, b) -> bool:
    """Bit-exact equality up to the sign of zero; NaN equals NaN."""
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=a.dtype.kind == "f")


def occupied_cell_end(cs, ce):
    return np.where(np.asarray(cs) != EMPTY, ce, 0).astype(np.uint32)


# --------------------------------------------------------------------------- GPU
def dev(a, dtype=None):
    import torch
    a = np.ascontiguousarray(a)
    if a.dtype == np.uint32:
        a = a.view(np.int32)
    t = torch.from_numpy(a.copy())
    return t.cuda()


def host(t, dtype=None):
    a = t.detach().cpu().numpy()
    if dtype == np.uint32 or (dtype is None and a.dtype == np.int32):
        a = a.view(np.uint32)
    return a


def empty_like_dev(a):
    import torch
    a = np.asarray(a)
    dt = {np.float32: torch.float32, np.uint32: torch.int32}[a.dtype.type]
    return torch.empty(a.shape, dtype=dt, device="cuda")


def gpu_stages(sys: System, st: dict) -> dict:
    """One step through the per-stage C-ABI entry points; returns every stage
    output with the golden fixtures' keys."""
    import torch
    import demso_b200 as D
    n = st["pos"].shape[0]
    nc = sys.num_cells
    typed = st.get("type") is not None
    pos, vel = dev(st["pos"]), dev(st["vel"])
    theta, omega = dev(st["theta"]), dev(st["omega"])
    radius, mass, ids = dev(st["radius"]), dev(st["mass"]), dev(st["id"])
    typ = dev(st["type"]) if typed else None
    h = torch.empty(n, dtype=torch.int32, device="cuda")
    ix = torch.empty(n, dtype=torch.int32, device="cuda")
    D.calcHash(sys, pos, ix, h, n)
    out = dict(hash=host(h).copy(), index=host(ix).copy())
    D.sortParticles(h, ix, n, keyBits=sys.key_bits)
    out["sorted_hash"], out["sorted_index"] = host(h), host(ix)
    cs = torch.empty(nc, dtype=torch.int32, device="cuda")
    ce = torch.zeros(nc, dtype=torch.int32, device="cuda")
    sp, sv = torch.empty_like(pos), torch.empty_like(vel)
    sth, som = torch.empty_like(theta), torch.empty_like(omega)
    sr, sm = torch.empty_like(radius), torch.empty_like(mass)
    sid, sloc = torch.empty_like(ids), torch.zeros_like(ids)
    styp = torch.empty_like(typ) if typed else None
    D.reorderDataAndFindCellStart(sys, cs, ce, sp, sv, sth, som, sr, sm, sid, sloc, styp, h, ix,
                                  pos, vel, theta, omega, radius, mass, ids, typ, n, nc)
    out["cellStart"] = host(cs)
    out["cellEnd"] = occupied_cell_end(out["cellStart"], host(ce))
    for k, t in (("pos", sp), ("vel", sv), ("theta", sth), ("omega", som), ("id", sid),
                 ("loc", sloc), ("radius", sr), ("mass", sm)):
        out["sorted_" + k] = host(t)
    acc = torch.empty_like(sp)
    alpha = torch.empty_like(som)
    pr = torch.empty_like(som)
    D.collide(sys, sp, sv, acc, som, alpha, styp, sr, sm, cs, ce, n, nc, pr)
    out["acc"], out["alpha"], out["pressure_collide"] = host(acc), host(alpha), host(pr)
    D.integrateSystem(sys, sp, sv, acc, sth, som, alpha, styp, sr, sm, pr, n)
    torch.cuda.synchronize()
    out.update(int_pos=host(sp), int_vel=host(sv), int_theta=host(sth), int_omega=host(som),
               int_pressure=host(pr))
    return out


def gpu_run(sys: System, st: dict, steps: int, flags=None, chunks=None, rows=None) -> dict:
    """`steps` full steps through the context API (fused kernels, graphs);
    `rows` = (first, count) steps a row window (dem_create_rows)."""
    import torch
    import demso_b200 as D
    if flags is None:
        flags = D.CTX_PRESSURE | D.CTX_ACCEL
    n = st["pos"].shape[0]
    sim = D.Simulation(sys, capacity=max(n, 1), flags=flags, rows=rows)
    typed = st.get("type") is not None
    to = (lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32).copy())
          if a.dtype == np.uint32 else torch.from_numpy(np.ascontiguousarray(a).copy()))
    sim.set_state(to(st["pos"]), to(st["vel"]), to(st["theta"]), to(st["omega"]),
                  to(st["radius"]), to(st["mass"]), to(st["id"]),
                  to(st["type"]) if typed else None)
    if chunks:
        done = 0
        for c in chunks:
            sim.step(c)
            done += c
        assert done == steps
    else:
        sim.step(steps)
    torch.cuda.synchronize()
    s = sim.get_state(device="cpu")
    out = {k: (None if v is None else (v.numpy().view(np.uint32) if v.dtype == torch.int32
                                       else v.numpy())) for k, v in s.items()}
    out["kernels_per_step"] = sim.kernels_per_step()
    sim.check()
    sim.close()
    return out
