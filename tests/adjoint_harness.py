"""Adjoint test harness: the loss of the differentiable workload, its gradient
through the C ABI (dem_adj_forward / dem_adj_backward), central finite
differences on the FP64 oracle, and a torch.autograd.Function around the
adjoint.

Loss = mean x-displacement of the disks + final kinetic energy
(translational and rotational).  Parameters: pair normal stiffness kn,
damping ratio zeta, friction mu (mapped onto the per-type coefficients by
scenes.pair_material) and the initial velocities.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from demso_b200 import scenes

NUM_COEF = 7


def with_params(sc, kn, zeta, mu):
    """The scene's System with the contact coefficients of (kn, zeta, mu)."""
    import copy
    sys = copy.deepcopy(sc.sys)
    mat = scenes.pair_material(kn=kn, zeta=zeta, mu=mu,
                               e_boundary=sc.sys.materials[0].boundaryDamping)
    sys.materials = [mat]
    sys.knWall = mat.normalStiffness
    sys.ktWall = mat.shearStiffness
    return sys


def inertia(m, r):
    m = np.float32(m)
    r = np.float32(r)
    return (np.float32(2.0) * m * r * r) / np.float32(5.0)


def loss_of(final, x0_by_id, mass_by_id, radius_by_id):
    """Loss from a final state (any order; mapped by id), in double."""
    order = np.argsort(final["id"])
    pos = np.asarray(final["pos"], np.float64)[order]
    vel = np.asarray(final["vel"], np.float64)[order]
    om = np.asarray(final["omega"], np.float64)[order]
    m = mass_by_id.astype(np.float64)
    I = inertia(mass_by_id, radius_by_id).astype(np.float64)
    disp = np.mean(pos[:, 0] - x0_by_id[:, 0].astype(np.float64))
    ke = 0.5 * np.sum(m * np.sum(vel * vel, axis=1)) + 0.5 * np.sum(I * om * om)
    return disp + ke


def coef_chain(kn, zeta, g):
    """dL/d(kn, zeta, mu) from the 7 coefficient gradients of dem_adj_backward."""
    m_ref = float(scenes.disk_mass(1e-3))
    cn = 2.0 * zeta * math.sqrt(0.5 * m_ref * kn)
    dcn_dkn = cn / (2.0 * kn)
    dcn_dz = cn / zeta
    dkn = g[0] + 0.5 * g[1] + g[2] * dcn_dkn + 2.0 * g[4] * dcn_dkn + 0.5 * g[6]
    dz = g[2] * dcn_dz + 2.0 * g[4] * dcn_dz
    dmu = g[3] + g[5]
    return dkn, dz, dmu


def gpu_loss_and_grad(sc, kn, zeta, mu, steps, every, vel0=None):
    """Loss (GPU forward) and its gradient (GPU adjoint) with respect to
    (kn, zeta, mu) and the initial velocities (by id)."""
    import torch
    import demso_b200 as D
    sys = with_params(sc, kn, zeta, mu)
    n = sc.n
    vel = sc.vel if vel0 is None else np.asarray(vel0, np.float32)
    sim = D.Simulation(sys, capacity=n, flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a))
    sim.set_state(t(sc.pos), t(vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass), t(sc.id))
    L = D.load()
    stream = torch.cuda.current_stream().cuda_stream
    D.check(L.dem_adj_forward(sim.handle, steps, every, stream))
    final = {k: v.numpy() for k, v in sim.get_state("cpu").items() if v is not None}
    final["id"] = final["id"].view(np.uint32)
    order_ids = np.argsort(sc.id)
    x0 = sc.pos[order_ids]
    m_by_id = sc.mass[order_ids]
    r_by_id = sc.radius[order_ids]
    loss = loss_of(final, x0, m_by_id, r_by_id)
    # cotangents of the final state, in id order
    order = np.argsort(final["id"])
    vel_f = final["vel"][order].astype(np.float32)
    om_f = final["omega"][order].astype(np.float32)
    lam_pos = np.zeros((n, 2), np.float32)
    lam_pos[:, 0] = np.float32(1.0 / n)
    lam_vel = (m_by_id[:, None] * vel_f).astype(np.float32)
    lam_om = (inertia(m_by_id, r_by_id) * om_f).astype(np.float32)
    dp, dv, dw = (torch.from_numpy(a).cuda() for a in (lam_pos, lam_vel, lam_om))
    grad = (C.c_double * NUM_COEF)()
    D.check(L.dem_adj_backward(sim.handle, dp.data_ptr(), dv.data_ptr(), dw.data_ptr(), grad,
                               stream))
    torch.cuda.synchronize()
    sim.close()
    g = list(grad)
    return loss, coef_chain(kn, zeta, g), dv.cpu().numpy(), g


def f64_loss(sc, kn, zeta, mu, steps, vel0=None):
    """Loss of the FP64 oracle run, and its branch signature."""
    from oracle.oracle import PortOracle
    sys = with_params(sc, kn, zeta, mu)
    st = sc.state()
    if vel0 is not None:
        st = dict(st)
        st["vel"] = vel0
    out = PortOracle("f64").run(sys, st, steps)
    order_ids = np.argsort(sc.id)
    return (loss_of(out, sc.pos[order_ids], sc.mass[order_ids], sc.radius[order_ids]),
            out["signature"])


def coef_tangents(kn, zeta):
    """Tangents of the material row (kn, kt, cn, eb, mu, at) and of the wall
    stiffnesses (knWall, ktWall) along kn, zeta and mu, for the material
    that scenes.pair_material makes (kt = kn / 2, cn = 2 zeta sqrt(m kn / 2),
    each per-type value twice the pair value)."""
    m_ref = float(scenes.disk_mass(1e-3))
    cn = 2.0 * zeta * math.sqrt(0.5 * m_ref * kn)
    dmat = np.zeros((4, 6))
    dwall = np.zeros((4, 2))
    dmat[0, 0], dmat[0, 1], dmat[0, 2] = 2.0, 1.0, 2.0 * cn / (2.0 * kn)
    dwall[0] = (2.0, 1.0)
    dmat[1, 2] = 2.0 * cn / zeta
    dmat[2, 4] = 1.0
    return dmat, dwall


def tangent_grad(sc, kn, zeta, mu, steps, u_by_id, precision="f64"):
    """The FP64 (or FP32) oracle adjoint, by forward mode: loss, (dL/dkn,
    dL/dzeta, dL/dmu, dL/dv0 . u) and the branch signature, where u is an
    (n, 2) direction over the initial velocities in id order."""
    from oracle.oracle import TangentOracle
    sys = with_params(sc, kn, zeta, mu)
    n = sc.n
    dmat, dwall = coef_tangents(kn, zeta)
    dvel = np.zeros((4, n, 2))
    dvel[3] = np.asarray(u_by_id, np.float64)[sc.id]
    out = TangentOracle(precision).run(sys, sc.state(), steps, dmat=dmat, dwall=dwall, dvel=dvel)
    order_ids = np.argsort(sc.id)
    loss = loss_of({k: out[k] for k in ("pos", "vel", "omega", "id")}, sc.pos[order_ids],
                   sc.mass[order_ids], sc.radius[order_ids])
    m = out["mass"].astype(np.float32)
    I = inertia(m, out["radius"].astype(np.float32)).astype(np.float64)
    m = m.astype(np.float64)
    d = []
    for k in range(4):
        d.append(np.mean(out["dpos"][k, :, 0])
                 + np.sum(m * np.sum(out["vel"] * out["dvel"][k], axis=1))
                 + np.sum(I * out["omega"] * out["domega"][k]))
    return loss, tuple(d), out["signature"]


def central_fd(fun, x, h):
    """(f(x + h) - f(x - h)) / 2h and whether both sides took the branches of
    the base run."""
    l0, s0 = fun(x)
    lp, sp = fun(x + h)
    lm, sm = fun(x - h)
    return (lp - lm) / (2.0 * h), (sp == s0 and sm == s0)


class AdjointLoss:
    """torch.autograd.Function over (kn, zeta, mu, v0) -> loss, backed by the
    C-ABI forward/adjoint; v0 is the (n, 2) initial velocity in id order."""

    @staticmethod
    def make(sc, steps, every):
        import torch

        class F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, kn, zeta, mu, v0):
                # v0 is indexed by particle id, like the velocity gradient
                vel0 = v0.detach().cpu().numpy()[sc.id]
                loss, dcoef, dv, _ = gpu_loss_and_grad(sc, float(kn), float(zeta), float(mu),
                                                       steps, every, vel0)
                ctx.save_for_backward(torch.tensor(dcoef, dtype=torch.float64),
                                      torch.from_numpy(dv))
                return torch.tensor(loss, dtype=torch.float64)

            @staticmethod
            def backward(ctx, gout):
                dcoef, dv = ctx.saved_tensors
                return (gout * dcoef[0], gout * dcoef[1], gout * dcoef[2],
                        (gout * dv.to(torch.float64)).to(torch.float32))

        return F


def batch_adjoint(systems_and_scenes, steps, every):
    """Batched adjoint over specimens [(System, Scene)]: the per-specimen
    loss of ``loss_of`` (mean x-displacement of the specimen + its kinetic
    energy), summed.  Returns (per-specimen coefficient gradients (S, 7),
    per-specimen (dpos, dvel, domega) cotangents of the initial state in each
    specimen's own particle order)."""
    import torch
    import demso_b200 as D
    specs = [sc for _, sc in systems_and_scenes]
    b = D.Batch([(sys, sc.n) for sys, sc in systems_and_scenes],
                flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    st = scenes.concat_specimens(specs)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a).copy())
    b.set_state(t(st["pos"]), t(st["vel"]), t(st["theta"]), t(st["omega"]), t(st["radius"]),
                t(st["mass"]), t(st["id"]))
    L = D.load()
    stream = torch.cuda.current_stream().cuda_stream
    D.check(L.dem_adj_forward(b.handle, steps, every, stream))
    final = {k: v.numpy() for k, v in b.get_state("cpu").items() if v is not None}
    order = np.argsort(final["id"].view(np.uint32))
    n = st["pos"].shape[0]
    m = st["mass"]
    r = st["radius"]
    offs = np.cumsum([0] + [sc.n for sc in specs])
    lam_pos = np.zeros((n, 2), np.float32)
    for s in range(len(specs)):
        lam_pos[offs[s]:offs[s + 1], 0] = np.float32(1.0 / specs[s].n)
    lam_vel = (m[:, None] * final["vel"][order]).astype(np.float32)
    lam_om = (inertia(m, r) * final["omega"][order]).astype(np.float32)
    dp, dv, dw = (torch.from_numpy(a).cuda() for a in (lam_pos, lam_vel, lam_om))
    grad = (C.c_double * (NUM_COEF * len(specs)))()
    D.check(L.dem_adj_backward(b.handle, dp.data_ptr(), dv.data_ptr(), dw.data_ptr(), grad, stream))
    torch.cuda.synchronize()
    b.close()
    g = np.array(list(grad)).reshape(len(specs), NUM_COEF)
    dp, dv, dw = dp.cpu().numpy(), dv.cpu().numpy(), dw.cpu().numpy()
    per = [(dp[offs[s]:offs[s + 1]], dv[offs[s]:offs[s + 1]], dw[offs[s]:offs[s + 1]])
           for s in range(len(specs))]
    return g, per


def single_adjoint(sys, sc, steps, every):
    """The same loss and cotangents as batch_adjoint for one specimen in its
    own context, in the specimen's particle (array) order."""
    import torch
    import demso_b200 as D
    n = sc.n
    ids = np.arange(n, dtype=np.uint32)
    sim = D.Simulation(sys, capacity=n, flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a).copy())
    sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass), t(ids))
    L = D.load()
    stream = torch.cuda.current_stream().cuda_stream
    D.check(L.dem_adj_forward(sim.handle, steps, every, stream))
    final = {k: v.numpy() for k, v in sim.get_state("cpu").items() if v is not None}
    order = np.argsort(final["id"].view(np.uint32))
    lam_pos = np.zeros((n, 2), np.float32)
    lam_pos[:, 0] = np.float32(1.0 / n)
    lam_vel = (sc.mass[:, None] * final["vel"][order]).astype(np.float32)
    lam_om = (inertia(sc.mass, sc.radius) * final["omega"][order]).astype(np.float32)
    dp, dv, dw = (torch.from_numpy(a).cuda() for a in (lam_pos, lam_vel, lam_om))
    grad = (C.c_double * NUM_COEF)()
    D.check(L.dem_adj_backward(sim.handle, dp.data_ptr(), dv.data_ptr(), dw.data_ptr(), grad,
                               stream))
    torch.cuda.synchronize()
    sim.close()
    return np.array(list(grad)), (dp.cpu().numpy(), dv.cpu().numpy(), dw.cpu().numpy())
