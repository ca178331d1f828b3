"""Batched, differentiable calibration of the contact law on collapsing columns.

Workload: `num` specimens (512 by default) of 1,024 to 4,096 disks
(log-uniform counts), radii uniform in [0.9, 1.1] mm, each a rectangular
column twice as high as wide, released at rest at the left wall of its own
walled box.  The target trajectory is the plain step run with hidden
parameters (kn = 2e5 N/m, friction 0.55; damping ratio 0.3, kt = kn / 2).
Calibration walks the collapse in windows of `window_steps` steps; iteration
i takes one Adam step on (log kn, friction) down the gradient of window
i's loss.  A window is cut into shots of `shot_steps` steps (multiple
shooting): each shot starts every specimen from the target state at its
start, runs with the current (kn, friction) through the batched adjoint
(checkpoint every `every` steps) and adds

    L = sum over specimens s of (1 / n_s) sum_i |x_i(end) - x*_i(end)|^2 / r^2

(r = 1 mm).  Shots keep the gradient meaningful: the dense contact flow is
chaotic, and the derivative of a single 3,000-step trajectory overflows
(measured: 1e18 and more, then NaN), while over 300 steps it agrees with
finite differences.  At the hidden parameters L is exactly zero: the step is
deterministic bit for bit.

Nothing here is on the stepping path; it drives the library through its
public API (Batch, adjoint_forward / adjoint_backward, set_systems).
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import Batch, CTX_ACCEL, CTX_PRESSURE, Simulation, System
from . import scenes

R_REF = 1e-3
HIDDEN = (2e5, 0.55)
ZETA = 0.3


def column_scene(n: int, seed: int, kn: float = HIDDEN[0], zeta: float = ZETA,
                 mu: float = HIDDEN[1], dt: float = 2e-6, aspect: float = 2.0) -> scenes.Scene:
    """n disks on a jittered square lattice (pitch 2.35 mm, no overlaps) forming a column
    `aspect` times as high as wide at the bottom-left of a walled box 6
    column widths wide and 1.25 column heights high."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.9e-3, 1.1e-3, size=n).astype(np.float32)
    pitch = 2.35e-3
    cols = max(1, int(round(math.sqrt(n / aspect))))
    rows = (n + cols - 1) // cols
    ij = np.stack(np.meshgrid(np.arange(cols), np.arange(rows), indexing="xy"), -1).reshape(-1, 2)[:n]
    pos = (ij + 0.5) * pitch + 0.1e-3 + rng.uniform(-0.05e-3, 0.05e-3, size=(n, 2))
    w, h = cols * pitch + 0.2e-3, rows * pitch + 0.2e-3
    Lx, Ly = 6.0 * w, 1.25 * h
    mat = scenes.pair_material(kn=kn, zeta=zeta, mu=mu)
    rmax = 1.1e-3
    sys = System(Lx=Lx, Ly=Ly, gx=max(4, scenes.grid_2r(Lx, rmax)),
                 gy=max(4, scenes.grid_2r(Ly, rmax)), dt=dt, gravity=(0.0, -9.81),
                 knWall=mat.normalStiffness, ktWall=mat.shearStiffness, materials=[mat])
    return scenes._finish(sys, pos, np.zeros((n, 2)), r, name="column_%d" % n)


def column_specimens(num: int = 512, seed: int = 0, nmin: int = 1024, nmax: int = 4096):
    rng = np.random.default_rng(seed)
    counts = np.exp(rng.uniform(np.log(nmin), np.log(nmax), size=num)).astype(np.int64)
    return [column_scene(int(c), seed * 100003 + k) for k, c in enumerate(counts)]


def with_params(sys: System, kn: float, mu: float, zeta: float = ZETA) -> System:
    import copy
    out = copy.deepcopy(sys)
    mat = scenes.pair_material(kn=kn, zeta=zeta, mu=mu,
                               e_boundary=sys.materials[0].boundaryDamping)
    out.materials = [mat]
    out.knWall, out.ktWall = mat.normalStiffness, mat.shearStiffness
    return out


def param_gradient(g: np.ndarray, kn: float, zeta: float = ZETA):
    """dL/d(kn, friction) from per-specimen coefficient gradients (S, 7) of
    the material made by scenes.pair_material: pair kn, kt = kn/2, pair
    dashpot cn = 2 zeta sqrt(m kn / 2), friction; floor dashpot 2 cn,
    friction, floor shear stiffness kn/2 (series of kn and the wall's kn)."""
    m_ref = float(scenes.disk_mass(1e-3))
    cn = 2.0 * zeta * math.sqrt(0.5 * m_ref * kn)
    dcn = cn / (2.0 * kn)
    t = g.sum(axis=0)
    dkn = t[0] + 0.5 * t[1] + t[2] * dcn + 2.0 * t[4] * dcn + 0.5 * t[6]
    dmu = t[3] + t[5]
    return dkn, dmu


class Calibration:
    """Targets and the windowed gradient descent over one batch context."""

    def __init__(self, specimens, windows: int = 50, window_steps: int = 3000,
                 shot_steps: int = 300, every: int = 100):
        import torch
        if window_steps % shot_steps:
            raise ValueError("window_steps must be a multiple of shot_steps")
        self.specimens = specimens
        self.windows, self.window_steps, self.every = windows, window_steps, every
        self.shot_steps = shot_steps
        self.shots = window_steps // shot_steps
        self.n = sum(sc.n for sc in specimens)
        st = scenes.concat_specimens(specimens)
        self.initial = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda()
                        for k, v in st.items() if k != "type" and v is not None}
        self.initial["id"] = self.initial["id"].view(torch.int32)
        self.batch = Batch([(sc.sys, sc.n) for sc in specimens], flags=CTX_PRESSURE | CTX_ACCEL)
        counts = torch.tensor([sc.n for sc in specimens], dtype=torch.float32, device="cuda")
        spec_of = torch.repeat_interleave(torch.arange(len(specimens), device="cuda"),
                                          counts.to(torch.int64))
        self.weight = (2.0 / (counts[spec_of] * R_REF * R_REF)).unsqueeze(1)  # by id
        self.snapshots = []

    def _set(self, state):
        s = state
        self.batch.set_state(s["pos"], s["vel"], s["theta"], s["omega"], s["radius"], s["mass"],
                             s["id"])

    def _by_id(self):
        """The current state scattered into id order (a dict of CUDA tensors)."""
        import torch
        st = self.batch.get_state("cuda")
        idx = st["id"].to(torch.int64)
        out = {}
        for k in ("pos", "vel", "theta", "omega", "radius", "mass"):
            v = torch.empty_like(st[k])
            v[idx] = st[k]
            out[k] = v
        out["id"] = self.initial["id"]
        return out

    def _systems(self, kn, mu):
        return [with_params(sc.sys, kn, mu) for sc in self.specimens]

    def make_targets(self, kn=HIDDEN[0], mu=HIDDEN[1]):
        """Target states at every shot boundary (run with the hidden
        parameters)."""
        import torch
        self.batch.set_systems(self._systems(kn, mu))
        self._set(self.initial)
        self.snapshots = [self._by_id()]
        for _ in range(self.windows * self.shots):
            self.batch.step(self.shot_steps)
            self.snapshots.append(self._by_id())
        torch.cuda.synchronize()
        self.batch.check()

    def shot_loss_and_grad(self, q: int, kn: float, mu: float):
        """Loss of shot q at (kn, mu) and dL/d(kn, friction)."""
        import torch
        self._set(self.snapshots[q])
        self.batch.adjoint_forward(self.shot_steps, min(self.every, self.shot_steps))
        fin = self._by_id()
        diff = fin["pos"] - self.snapshots[q + 1]["pos"]
        loss = float((0.5 * self.weight * diff * diff).sum().item())
        lam_pos = (self.weight * diff).contiguous()
        lam_vel = torch.zeros_like(lam_pos)
        lam_om = torch.zeros(self.n, dtype=torch.float32, device="cuda")
        g = self.batch.adjoint_backward(lam_pos, lam_vel, lam_om)
        return loss, param_gradient(g, kn)

    def loss_and_grad(self, w: int, kn: float, mu: float):
        """Loss of window w (the sum over its shots) and its gradient."""
        self.batch.set_systems(self._systems(kn, mu))
        loss, dkn, dmu = 0.0, 0.0, 0.0
        for j in range(self.shots):
            l, (a, b) = self.shot_loss_and_grad(w * self.shots + j, kn, mu)
            loss, dkn, dmu = loss + l, dkn + a, dmu + b
        return loss, (dkn, dmu)

    def run(self, kn0=1e5, mu0=0.4, iters=50, lr=(0.25, 0.04), betas=(0.5, 0.9)):
        """Adam on (log kn, friction); iteration i uses window i mod windows."""
        x = np.array([math.log(kn0), mu0])
        m = np.zeros(2)
        v = np.zeros(2)
        hist = []
        for it in range(iters):
            kn, mu = math.exp(x[0]), float(x[1])
            loss, (dkn, dmu) = self.loss_and_grad(it % self.windows, kn, mu)
            g = np.array([dkn * kn, dmu])
            if not np.all(np.isfinite(g)):
                g = np.zeros(2)
            m = betas[0] * m + (1 - betas[0]) * g
            v = betas[1] * v + (1 - betas[1]) * g * g
            mh = m / (1 - betas[0] ** (it + 1))
            vh = v / (1 - betas[1] ** (it + 1))
            step = np.array(lr) * (0.5 + 0.5 * math.cos(math.pi * it / iters))
            x = x - step * mh / (np.sqrt(vh) + 1e-30)
            x[1] = min(max(x[1], 0.01), 2.0)
            hist.append(dict(iter=it, kn=kn, mu=mu, loss=loss))
        return math.exp(x[0]), float(x[1]), hist

    def close(self):
        self.batch.close()


def looped_window_seconds(specimens, steps: int, sample: int = 16) -> float:
    """Seconds for one window of `steps` steps of every specimen with the
    plain single-scene step looped over the specimens, extrapolated from an
    evenly spaced sample."""
    import torch
    picks = specimens[:: max(1, len(specimens) // sample)][:sample]
    sims = []
    for sc in picks:
        sim = Simulation(sc.sys, capacity=sc.n, flags=CTX_PRESSURE)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)
                                       if a.dtype == np.uint32 else np.ascontiguousarray(a))
        sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass),
                      t(sc.id))
        sim.step(3)
        sims.append(sim)
    torch.cuda.synchronize()
    k = max(3, min(steps, 200))
    t0 = time.perf_counter()
    for sim in sims:
        sim.step(k)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    for sim in sims:
        sim.close()
    per_particle_step = dt / (k * sum(sc.n for sc in picks))
    per_step_launch = dt / (k * len(picks))
    # launch-bound at these sizes: scale by specimen count and steps
    return per_step_launch * len(specimens) * steps, per_particle_step


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--num", type=int, default=512)
    ap.add_argument("--windows", type=int, default=50)
    ap.add_argument("--window-steps", type=int, default=3000)
    ap.add_argument("--shot-steps", type=int, default=300)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--iters", type=int, default=50)
    ap.add_argument("--kn0", type=float, default=1e5)
    ap.add_argument("--mu0", type=float, default=0.4)
    args = ap.parse_args(argv)
    import torch
    t0 = time.perf_counter()
    specimens = column_specimens(args.num)
    cal = Calibration(specimens, args.windows, args.window_steps, args.shot_steps, args.every)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    cal.make_targets()
    t2 = time.perf_counter()
    kn, mu, hist = cal.run(args.kn0, args.mu0, args.iters)
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    cal.close()
    window_s, _ = looped_window_seconds(specimens, args.window_steps)
    fd_s = args.iters * 5 * window_s  # loss + central differences in kn and friction
    print(json.dumps({
        "workload": "calibration: %d column specimens of 1,024..4,096 disks, %d windows of %d "
                    "steps in shots of %d (checkpoint every %d), hidden kn %.0f N/m, "
                    "friction %.2f" % (args.num, args.windows, args.window_steps,
                                       args.shot_steps, args.every, *HIDDEN),
        "particles": cal.n, "start": {"kn": args.kn0, "friction": args.mu0},
        "result": {"kn": kn, "friction": mu},
        "rel_error": {"kn": abs(kn - HIDDEN[0]) / HIDDEN[0], "friction": abs(mu - HIDDEN[1]) / HIDDEN[1]},
        "seconds": {"setup": t1 - t0, "targets": t2 - t1, "gradient_descent": t3 - t2},
        "fd_looped_plain_seconds_estimate": fd_s,
        "history": hist[:: max(1, len(hist) // 10)] + hist[-1:]}), flush=True)


if __name__ == "__main__":
    main()
