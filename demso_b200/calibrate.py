"""Batched, differentiable calibration of the contact law on collapsing columns.

Workload: `num` specimens (512 by default) of 1,024 to 4,096 disks
(log-uniform counts), radii uniform in [0.9, 1.1] mm, each a rectangular
column twice as high as wide, released at rest at the left wall of its own
walled box.  The targets are pile profiles only: the plain step is run with
hidden parameters (kn = 2e5 N/m, friction 0.55; damping ratio 0.3,
kt = kn / 2) and, every `shot_steps` steps, each specimen's column-height
profile h(x) is kept -- the disks' area binned along x (bins of
`bin_width`, 4 mm by default, each disk shared between its two nearest bin
centres in proportion to its distance from them) and divided by the bin
width and the columns' initial packing fraction.  Nothing else of the
hidden run is kept.

Calibration walks the collapse with the model's own trajectory: iteration i
takes window i (`window_steps` steps) from the state where the model's own
run, with the parameters of the iterations before, left it -- the state in
the context's order, so that the run continues bit for bit as if it had not
stopped -- and takes one Adam step on (log kn, friction) down the gradient
of

    L = sum over specimens s, shots q of the window:
        (1 / B_s) sum_b (h_s(x_b; q) - h*_s(x_b; q))^2 / H_s^2

(B_s bins, H_s the column's initial height); the gradient is each
specimen's gradient summed over the window, combined over the specimens by
a trimmed mean (trimmed_total).  The window is cut into shots
of `shot_steps` steps: each shot runs through the batched adjoint
(checkpoint every `every` steps) from the model's state at its start, and
its gradient is taken over that shot alone (the start state held fixed),
which keeps the derivative of the dense, chaotic flow bounded: over a whole
3,000-step window it overflows (measured: 1e18 and more, then NaN), while
over 300 steps it agrees with finite differences.  The binning is piecewise
linear in the positions; its derivative dL/dx enters the adjoint as the
position cotangent.  The profiles are summed in fixed point, so at the hidden
parameters -- where the model's run is the hidden run bit for bit, the step
being deterministic -- L and its gradient are exactly zero.

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


def specimen_gradients(g: np.ndarray, kn: float, zeta: float = ZETA) -> np.ndarray:
    """Each specimen's dL/d(kn, friction), (S, 2), from its coefficient
    gradients (S, 7) -- param_gradient row by row."""
    return np.array([param_gradient(g[s:s + 1], kn, zeta) for s in range(g.shape[0])])


def trimmed_total(per: np.ndarray, trim: float = 0.1) -> np.ndarray:
    """The sum over specimens of per-specimen gradients (S, 2), estimated as
    S times the mean of each column with the `trim` fraction of the largest
    and of the smallest values left out.  A few specimens whose 300-step
    derivative the chaotic flow has blown up would otherwise outweigh the
    rest; the estimate is zero when every specimen's gradient is."""
    S = per.shape[0]
    k = int(math.floor(trim * S))
    srt = np.sort(per, axis=0)
    kept = srt[k:S - k] if S - 2 * k > 0 else srt
    return S * kept.mean(axis=0)


PROFILE_BIN = 4e-3   # m, bin width of the column-height profiles
PACKING = 0.57       # area fraction of the initial lattice (radii U[0.9, 1.1] mm, pitch 2.35 mm)


class Profiles:
    """Column-height profiles h(x) of every specimen of a batch, from the
    disks' positions in id order (the concatenation order of the specimens).
    Bin b of specimen s is centred at (b + 1/2) * bin_width; a disk at x adds
    its area to bins floor(u) and floor(u) + 1 (u = x / bin_width - 1/2) in
    proportion 1 - f and f (f = u - floor(u)), clamped to the box's bins; the
    sums are divided by bin_width and PACKING.  The sums are taken in 64-bit
    fixed point (2^-40 m), so they do not depend on the order the GPU adds
    them in; dL/dx is the derivative of the piecewise-linear binning."""

    FIXED = float(2 ** 40)

    def __init__(self, specimens, device, bin_width: float = PROFILE_BIN):
        import torch
        self.bw = bin_width
        nb = [max(2, int(math.ceil(sc.sys.Lx / bin_width))) for sc in specimens]
        off = np.concatenate([[0], np.cumsum(nb)])
        counts = np.array([sc.n for sc in specimens])
        spec = np.repeat(np.arange(len(specimens)), counts)
        self.nbins = int(off[-1])
        self.first = torch.tensor(off[:-1][spec], dtype=torch.int64, device=device)
        self.last = torch.tensor((off[1:] - 1)[spec], dtype=torch.int64, device=device)
        r = np.concatenate([sc.radius for sc in specimens]).astype(np.float64)
        self.scale = torch.tensor(np.pi * r * r / (bin_width * PACKING), dtype=torch.float64,
                                  device=device)
        # loss weight of each bin: 1 / (B_s H_s^2), H_s the column's height
        h = np.array([sc.pos[:, 1].max() + sc.radius.max() for sc in specimens], np.float64)
        wb = np.repeat(1.0 / (np.array(nb) * h * h), nb)
        self.weight = torch.tensor(wb, dtype=torch.float64, device=device)

    def _bins(self, x):
        import torch
        u = x.to(torch.float64) / self.bw - 0.5
        k = torch.floor(u)
        f = u - k
        k = k.to(torch.int64)
        b0 = torch.clamp(self.first + k, self.first, self.last)
        b1 = torch.clamp(self.first + k + 1, self.first, self.last)
        return f, b0, b1

    def __call__(self, x):
        """Profiles (all bins of all specimens, float64) from x (n,), by id."""
        import torch
        f, b0, b1 = self._bins(x)
        c0 = torch.round(self.scale * (1.0 - f) * self.FIXED).to(torch.int64)
        c1 = torch.round(self.scale * f * self.FIXED).to(torch.int64)
        h = torch.zeros(self.nbins, dtype=torch.int64, device=x.device)
        h.index_add_(0, b0, c0)
        h.index_add_(0, b1, c1)
        return h.to(torch.float64) / self.FIXED

    def loss(self, h, target):
        d = h - target
        return float((self.weight * d * d).sum().item())

    def grad(self, x, h, target):
        """dL/dx (n,) of loss(profiles(x), target) (zero where a disk's two
        bins are clamped into one)."""
        f, b0, b1 = self._bins(x)
        r = 2.0 * self.weight * (h - target)
        return self.scale / self.bw * (r[b1] - r[b0])


class Calibration:
    """Profile targets and the windowed gradient descent over one batch
    context."""

    def __init__(self, specimens, windows: int = 50, window_steps: int = 3000,
                 shot_steps: int = 300, every: int = 100, bin_width: float = PROFILE_BIN):
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
        self.profiles = Profiles(specimens, "cuda", bin_width)
        self.targets = []

    def _set(self, state):
        s = state
        self.batch.set_state(s["pos"], s["vel"], s["theta"], s["omega"], s["radius"], s["mass"],
                             s["id"])

    def _current(self):
        """The current state in the context's order: the sorted order of the
        last step, which a following step's stable sort breaks ties by.  A run
        continued from it with dem_set_state is the uninterrupted run bit for
        bit (a state re-set in another order, such as by id, is not)."""
        st = self.batch.get_state("cuda")
        return {k: st[k] for k in ("pos", "vel", "theta", "omega", "radius", "mass", "id")}

    def _x_by_id(self, state):
        """The x-coordinates of a context-order state, in id order."""
        import torch
        x = torch.empty_like(state["pos"][:, 0])
        x[state["id"].to(torch.int64)] = state["pos"][:, 0]
        return x

    def _systems(self, kn, mu):
        return [with_params(sc.sys, kn, mu) for sc in self.specimens]

    def make_targets(self, kn=HIDDEN[0], mu=HIDDEN[1]):
        """The target profiles at the end of every shot of the collapse, from
        the plain step run with the hidden parameters (only the profiles are
        kept)."""
        import torch
        self.batch.set_systems(self._systems(kn, mu))
        self._set(self.initial)
        self.targets = [self.profiles(self._x_by_id(self.initial))]
        for _ in range(self.windows * self.shots):
            self.batch.step(self.shot_steps)
            self.targets.append(self.profiles(self._x_by_id(self._current())))
        torch.cuda.synchronize()
        self.batch.check()

    def state_at(self, w: int, kn: float, mu: float):
        """The model's own state at the start of window w, run from the
        initial columns with (kn, mu)."""
        self.batch.set_systems(self._systems(kn, mu))
        self._set(self.initial)
        if w:
            self.batch.step(w * self.window_steps)
        return self._current()

    def shot_loss_and_grad(self, q: int, state, kn: float, mu: float):
        """Shot q (ending at target q + 1) from `state`: its loss at (kn, mu),
        dL/d(kn, friction) over the shot, and the model's state at its end."""
        import torch
        self._set(state)
        self.batch.adjoint_forward(self.shot_steps, min(self.every, self.shot_steps))
        fin = self._current()  # before the backward, which restores checkpoints
        x = self._x_by_id(fin)
        h = self.profiles(x)
        loss = self.profiles.loss(h, self.targets[q + 1])
        lam_pos = torch.zeros((self.n, 2), dtype=torch.float32, device="cuda")
        lam_pos[:, 0] = self.profiles.grad(x, h, self.targets[q + 1]).to(torch.float32)
        lam_vel = torch.zeros_like(lam_pos)
        lam_om = torch.zeros(self.n, dtype=torch.float32, device="cuda")
        g = self.batch.adjoint_backward(lam_pos.contiguous(), lam_vel, lam_om)
        return loss, specimen_gradients(np.asarray(g).reshape(-1, 7), kn), fin

    def loss_and_grad(self, w: int, kn: float, mu: float, state):
        """Loss of window w from the model's state `state` at its start (the
        sum over its shots), its gradient (each specimen's summed over the
        shots, then combined by trimmed_total), and the model's state at its
        end."""
        self.batch.set_systems(self._systems(kn, mu))
        loss = 0.0
        per = np.zeros((len(self.specimens), 2))
        for j in range(self.shots):
            l, g, state = self.shot_loss_and_grad(w * self.shots + j, state, kn, mu)
            loss += l
            per += g
        dkn, dmu = trimmed_total(per)
        return loss, (float(dkn), float(dmu)), state

    def run(self, kn0=1e5, mu0=0.4, iters=50, lr=(0.25, 0.04), betas=(0.5, 0.9)):
        """Adam on (log kn, friction); iteration i takes window i mod windows,
        continuing the model's own run where window i - 1 left it (from the
        initial columns at window 0)."""
        x = np.array([math.log(kn0), mu0])
        m = np.zeros(2)
        v = np.zeros(2)
        hist = []
        state = self.initial
        for it in range(iters):
            w = it % self.windows
            if w == 0:
                state = self.initial
            kn, mu = math.exp(x[0]), float(x[1])
            loss, (dkn, dmu), state = self.loss_and_grad(w, kn, mu, state)
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
    evenly spaced sample, in the faster of its two forms: the graph path and
    the cluster launch (CTX_RESIDENT, for specimens of up to 8,192 disks)."""
    import torch
    from . import CTX_RESIDENT
    picks = specimens[:: max(1, len(specimens) // sample)][:sample]
    k = max(3, min(steps, 200))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)
                                   if a.dtype == np.uint32 else np.ascontiguousarray(a))

    def timed(flags):
        sims = []
        for sc in picks:
            sim = Simulation(sc.sys, capacity=sc.n, flags=flags)
            sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius),
                          t(sc.mass), t(sc.id))
            sim.step(3)
            sims.append(sim)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for sim in sims:
            sim.step(k)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        for sim in sims:
            sim.close()
        return dt

    dt = min(timed(CTX_PRESSURE), timed(CTX_PRESSURE | CTX_RESIDENT))
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
    ap.add_argument("--bin-width", type=float, default=PROFILE_BIN)
    ap.add_argument("--out", default=None, help="also write the result as JSON to this path")
    args = ap.parse_args(argv)
    import torch
    t0 = time.perf_counter()
    specimens = column_specimens(args.num)
    cal = Calibration(specimens, args.windows, args.window_steps, args.shot_steps, args.every,
                      args.bin_width)
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
    res = {
        "workload": "calibration: %d column specimens of 1,024..4,096 disks (aspect 2), %d "
                    "windows of %d steps in shots of %d (checkpoint every %d); targets: "
                    "column-height profiles h(x) in %.0f mm bins every %d steps of the run "
                    "with hidden kn %.0f N/m, friction %.2f; the model follows its own run"
                    % (args.num, args.windows, args.window_steps, args.shot_steps, args.every,
                       1e3 * args.bin_width, args.shot_steps, *HIDDEN),
        "particles": cal.n, "start": {"kn": args.kn0, "friction": args.mu0},
        "result": {"kn": kn, "friction": mu},
        "rel_error": {"kn": abs(kn - HIDDEN[0]) / HIDDEN[0],
                      "friction": abs(mu - HIDDEN[1]) / HIDDEN[1]},
        "seconds": {"setup": t1 - t0, "targets": t2 - t1, "gradient_descent": t3 - t2},
        "fd_looped_plain_seconds_estimate": fd_s,
        "fd_over_adjoint_wall_time": fd_s / (t3 - t2),
        "history": hist}
    print(json.dumps(res), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
