"""Multi-GPU slab decomposition of the plain step, one process per GPU.

The cell grid is cut into slabs of whole cell rows, one per rank, balanced by
particle count at the start (``partition_rows``).  Cells are numbered row by
row, so the particles of rank r's rows [y0, y1) are one contiguous range of
the global sorted order, and the global order is the concatenation of the
ranks' ranges.

Each rank steps a *window*: its own rows plus ``halo`` rows on either side,
with the library's fused context (incremental sort, collide, integrate and
next hash on the GPU, replayed as CUDA graphs) -- the single-GPU hot path,
unchanged.  The window is the single-domain scene cut at its edges, so a
particle near a cut misses its neighbours beyond it and drifts from the
single-domain result.  That error reaches at most two more rows a step: one
through the 3 x 3 cell neighbourhood and one through the particle's own
displacement, which is below one cell per step (the reference's own 3 x 3
search rests on the same bound).  With ``halo = 2 * period + 2`` rows every
own row is still exact after ``period`` steps.  The ranks then exchange bands:
each sends its ``halo`` lowest own rows to rank r - 1 and its ``halo`` highest
own rows to rank r + 1 (NCCL send/recv over NVLink on GPUs), and rebuilds its
window as [rows from below] + [own rows] + [rows from above].

Rows are cut by the keys of the last sort, which ordered every window, so each
part is a contiguous slot range (``dem_row_slots``), in the global order
restricted to it, and the rebuilt window is the global sorted state
restricted to the window.  Its next sort, a stable sort of that order, is the
global stable sort restricted: the decomposition reproduces the
single-domain step bit for bit.

A window's particle count changes with every rebuild (particles cross slab
boundaries).  The context keeps a fixed count, so that its captured graphs
stay valid: the window is padded with parked particles, one per cell in rows
two or more rows away from the window (no window particle ever visits their
cells), at rest; one of them has the scene's largest radius, so the
context's largest radius never changes either.  Particles carry window-local
ids (the context indexes loc by id) and a table back to the global ids.

``run`` drives one rank over ``torch.distributed`` (``DistExchange``);
``run_group`` drives several slabs in one process, exchanging through local
copies (``LocalExchange``), which tests the decomposition on one GPU.  The
stepping is behind a small interface (``ContextStepper`` on the GPU; the tests
add one over the CPU oracle and run the same code over gloo).
"""
from __future__ import annotations

import numpy as np

FIELDS = ("pos", "vel", "theta", "omega", "radius", "mass", "id", "type")
ROW_WIDTH = 10  # packed row: pos(2) vel(2) theta omega radius mass, id and type bits


def partition_rows(row_counts, world: int):
    """Row boundaries y[0] = 0 < y[1] < ... < y[world] = gy splitting the
    particle count per row as evenly as whole rows allow (each slab at least
    one row)."""
    gy = len(row_counts)
    if world > gy:
        raise ValueError("more ranks (%d) than cell rows (%d)" % (world, gy))
    cum = np.concatenate([[0], np.cumsum(np.asarray(row_counts, np.int64))])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        y = int(np.searchsorted(cum, total * r / world, side="left"))
        y = max(y, bounds[-1] + 1)
        y = min(y, gy - (world - r))
        bounds.append(y)
    bounds.append(gy)
    return bounds


def halo_rows(period: int) -> int:
    """Rows a window holds on either side of its slab for `period` steps
    between exchanges."""
    return 2 * int(period) + 2


def check_bounds(bounds, halo: int):
    """Every slab needs 2 * halo + 3 rows: its two bands are disjoint and a
    window leaves rows free for the parked particles."""
    for r in range(len(bounds) - 1):
        if bounds[r + 1] - bounds[r] < 2 * halo + 3 and len(bounds) > 2:
            raise ValueError("slab %d has %d rows; the halo of %d rows needs %d" %
                             (r, bounds[r + 1] - bounds[r], halo, 2 * halo + 3))


def pack(st: dict):
    """(m, ROW_WIDTH) float32 rows of a state dict of torch tensors."""
    import torch
    m = st["pos"].shape[0]
    typ = st.get("type")
    if typ is None:
        typ = torch.zeros(m, dtype=torch.int32, device=st["pos"].device)
    cols = [st["pos"].reshape(m, 2), st["vel"].reshape(m, 2), st["theta"][:, None],
            st["omega"][:, None], st["radius"][:, None], st["mass"][:, None],
            st["id"].view(torch.float32)[:, None], typ.view(torch.float32)[:, None]]
    return torch.cat(cols, dim=1).contiguous()


def unpack(rows, typed: bool) -> dict:
    import torch
    return {"pos": rows[:, 0:2].contiguous(), "vel": rows[:, 2:4].contiguous(),
            "theta": rows[:, 4].contiguous(), "omega": rows[:, 5].contiguous(),
            "radius": rows[:, 6].contiguous(), "mass": rows[:, 7].contiguous(),
            "id": rows[:, 8].contiguous().view(torch.int32),
            "type": rows[:, 9].contiguous().view(torch.int32) if typed else None}


def fields(part, typed: bool) -> dict:
    """A window part as a dict of per-field tensors: packed rows (a band
    received from a neighbour) are unpacked, dicts pass through."""
    return part if isinstance(part, dict) else unpack(part, typed)


def concat(parts, typed: bool) -> dict:
    """Parts (packed rows or field dicts) joined field by field."""
    import torch
    fs = [fields(p, typed) for p in parts if p is not None]
    out = {}
    for k in FIELDS:
        if k == "type" and not typed:
            out[k] = None
            continue
        out[k] = torch.cat([f[k] for f in fs])  # a new tensor, even from one part
    return out


def cell_rows(sys, pos) -> np.ndarray:
    """Grid row of each position (the reference's calcGridPos, as
    scenes.cell_hash computes it)."""
    from .scenes import cell_hash
    return (cell_hash(np.asarray(pos, np.float32), sys) >> np.uint32(sys.gx.bit_length() - 1)
            ).astype(np.int64)


class HaloSlab:
    """Rank `rank`'s slab: own rows bounds[rank] .. bounds[rank + 1] and a
    window of `halo` more rows on either side, stepped by `stepper`."""

    def __init__(self, sys, rank: int, world: int, bounds, period: int, stepper, halo=None):
        self.sys, self.rank, self.world = sys, rank, world
        self.bounds = list(bounds)
        self.period = int(period)
        if world == 1:
            self.halo = 0
        else:
            self.halo = halo_rows(period) if halo is None else int(halo)
        check_bounds(self.bounds, self.halo)
        self.y0, self.y1 = self.bounds[rank], self.bounds[rank + 1]
        self.wlo = max(0, self.y0 - self.halo)
        self.whi = min(sys.gy, self.y1 + self.halo)
        self.stepper = stepper
        self.rebuilds = 0
        self.moved_rows = 0  # rows received from the neighbours, all exchanges

    def load(self, state_all: dict):
        """The window's particles of a global state (host arrays, any
        order), in that order."""
        rows = cell_rows(self.sys, state_all["pos"])
        keep = np.nonzero((rows >= self.wlo) & (rows < self.whi))[0]
        part = {k: (None if v is None else np.ascontiguousarray(np.asarray(v)[keep]))
                for k, v in state_all.items() if k in FIELDS}
        self.stepper.set_window([self.stepper.from_host(part)], (self.wlo, self.whi))

    def advance(self, k: int):
        self.stepper.step(int(k))

    def _rows(self, lo: int, hi: int, packed: bool = True):
        first, count = self.stepper.slots(lo, hi)
        return self.stepper.take(first, count, packed)

    def bands(self):
        """(rows for rank - 1, rows for rank + 1): the slab's `halo` lowest and
        highest rows, by the keys of the last sort."""
        down = self._rows(self.y0, self.y0 + self.halo) if self.rank > 0 else None
        up = self._rows(self.y1 - self.halo, self.y1) if self.rank < self.world - 1 else None
        return down, up

    def own(self, packed: bool = True):
        """The slab's own rows in the global order restricted to them:
        packed rows, or a dict of per-field tensors."""
        return self._rows(self.y0, self.y1, packed)

    def rebuild(self, below, above):
        """New window: rows from rank - 1, own rows, rows from rank + 1."""
        self.moved_rows += sum(int(p.shape[0]) for p in (below, above) if p is not None)
        self.stepper.set_window([below, self.own(packed=False), above], (self.wlo, self.whi))
        self.rebuilds += 1


class LocalExchange:
    """Bands between slabs held by one process (tests the decomposition on
    one device)."""

    @staticmethod
    def exchange(outgoing):
        """outgoing[r] = (down, up) of slab r; returns (below, above) per slab."""
        n = len(outgoing)
        return [(outgoing[r - 1][1] if r > 0 else None,
                 outgoing[r + 1][0] if r < n - 1 else None) for r in range(n)]


class DistExchange:
    """Bands between neighbouring ranks over torch.distributed (NCCL on GPUs,
    gloo on CPU): the counts first, then the rows, each as one batch of
    point-to-point operations."""

    def __init__(self, rank: int, world: int, device):
        self.rank, self.world, self.device = rank, world, device

    def _swap(self, send, recv_shapes=None):
        import torch
        import torch.distributed as dist
        ops, got = [], {}
        for peer, t in send.items():
            ops.append(dist.P2POp(dist.isend, t, peer))
        for peer, shape in (recv_shapes or {}).items():
            buf = torch.empty(shape, dtype=torch.float32 if len(shape) == 2 else torch.int64,
                              device=self.device)
            got[peer] = buf
            ops.append(dist.P2POp(dist.irecv, buf, peer))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return got

    def exchange(self, down, up):
        import torch
        peers = {}
        if self.rank > 0:
            peers[self.rank - 1] = down
        if self.rank < self.world - 1:
            peers[self.rank + 1] = up
        counts = {p: torch.tensor([int(t.shape[0])], dtype=torch.int64, device=self.device)
                  for p, t in peers.items()}
        got = self._swap(counts, {p: (1,) for p in peers})
        sizes = {p: int(t.item()) for p, t in got.items()}
        send = {p: t.to(self.device).contiguous() for p, t in peers.items() if t.shape[0]}
        rows = self._swap(send, {p: (m, ROW_WIDTH) for p, m in sizes.items() if m})
        empty = lambda: torch.empty((0, ROW_WIDTH), dtype=torch.float32, device=self.device)
        below = rows.get(self.rank - 1, empty()) if self.rank > 0 else None
        above = rows.get(self.rank + 1, empty()) if self.rank < self.world - 1 else None
        return below, above

    def gather(self, rows):
        """Every rank's rows, concatenated in rank order, on rank 0 (None
        elsewhere)."""
        import torch
        import torch.distributed as dist
        n = torch.tensor([int(rows.shape[0])], dtype=torch.int64, device=self.device)
        table = [torch.empty_like(n) for _ in range(self.world)]
        dist.all_gather(table, n)
        sizes = [int(t.item()) for t in table]
        if self.rank != 0:
            if sizes[self.rank]:
                dist.send(rows.to(self.device).contiguous(), 0)
            return None
        out = [rows.to(self.device)]
        for src in range(1, self.world):
            buf = torch.empty((sizes[src], ROW_WIDTH), dtype=torch.float32, device=self.device)
            if sizes[src]:
                dist.recv(buf, src)
            out.append(buf)
        return torch.cat(out)


def _rounds(steps: int, period: int):
    done = 0
    while done < steps:
        k = min(period, steps - done)
        done += k
        yield k, done < steps


def run(slab: HaloSlab, ex: DistExchange, steps: int):
    """`steps` steps of one rank's slab, exchanging bands every slab.period
    steps (every rank calls this with the same arguments)."""
    for k, more in _rounds(steps, slab.period):
        slab.advance(k)
        if more and slab.world > 1:
            below, above = ex.exchange(*slab.bands())
            slab.rebuild(below, above)


def run_group(slabs, steps: int):
    """`steps` steps of all slabs of a decomposition held by this process."""
    period = slabs[0].period
    for k, more in _rounds(steps, period):
        for s in slabs:
            s.advance(k)
        if more and len(slabs) > 1:
            got = LocalExchange.exchange([s.bands() for s in slabs])
            for s, (below, above) in zip(slabs, got):
                s.rebuild(below, above)


class ContextStepper:
    """A window stepped by the library's context (``Simulation``) on the GPU.

    The window is padded to a fixed particle count (parked particles, see the
    module docstring) so that the context's graphs survive rebuilds; a window
    that outgrows the count gets a new context with room to spare."""

    SPARE = 0.01  # capacity above the first window's particle count

    def __init__(self, sys, rmax: float, flags=None, device="cuda"):
        import torch
        from . import CTX_PRESSURE
        self.sys = sys
        self.rmax = float(rmax)
        self.flags = CTX_PRESSURE if flags is None else flags
        self.device = torch.device(device)
        self.typed = len(sys.materials) > 1
        self.sim = None
        self.capacity = 0
        self.rows = (0, sys.gy)  # the context's cell rows (first, count)
        self.gid = None     # global id of every window-local id (-1: parked)
        self.m = 0          # real particles of the window
        self._park = None

    def from_host(self, part: dict) -> dict:
        import torch
        t = {}
        for k in FIELDS:
            v = part.get(k)
            if v is None:
                t[k] = None
                continue
            a = np.ascontiguousarray(v)
            if a.dtype == np.uint32:
                a = a.view(np.int32)
            t[k] = torch.from_numpy(a).to(self.device)
        return t

    def _context_rows(self, window, parked: int):
        """(first, count) cell rows for a window's context: the window's rows,
        a row clear of them on either side and rows for `parked` parked
        particles, rounded up to a power of two (dem_create_rows); the whole
        grid when that reaches it.  A window of a tall scene then sorts and
        scans its own cells only."""
        wlo, whi = window
        gx, gy = self.sys.gx, self.sys.gy
        need = (whi - wlo) + 2 + -(-int(parked) // gx)
        count = 1
        while count < need:
            count <<= 1
        return (0, gy) if count >= gy else (wlo, count)

    def _free_rows(self, window, rows=None):
        """Scene rows for parked particles: rows whose cell row in the
        context (rows = (first, count); (R - wlo) mod count relative to the
        window) is at least one row clear of the window's on either side,
        each cell row once.  They are two or more rows from the window in the
        scene too, so no window particle ever visits their cells."""
        rows = rows or self.rows
        key = (tuple(window), tuple(rows))
        cache = self.__dict__.setdefault("_free_cache", {})
        if key not in cache:
            wlo, whi = window
            count, m = rows[1], whi - wlo
            y = np.arange(self.sys.gy, dtype=np.int64)
            lr = (y - wlo) % count
            ok = (lr >= m + 1) & (lr < count - 1)
            # the first scene row of each cell row
            _, first = np.unique(lr[ok], return_index=True)
            cache[key] = np.sort(y[ok][first]).tolist()
        return cache[key]

    def _parked(self, count: int, window) -> dict:
        """`count` parked particles in the cells of the free rows, one per
        cell (built once per window and count bound, then sliced)."""
        import torch
        key = (window, self.rows)
        if self._park is None or self._park[0] != key or self._park[1] < count:
            sys = self.sys
            free = self._free_rows(window)
            cells = len(free) * sys.gx
            size = min(cells, max(count, self.capacity))
            if count > size:
                raise ValueError("no room for %d parked particles (%d free cells)" %
                                 (count, cells))
            k = np.arange(size)
            ys = np.asarray(free, np.int64)[k // sys.gx]
            xs = k % sys.gx
            cw, ch = sys.Lx / sys.gx, sys.Ly / sys.gy
            pos = np.stack([(xs + 0.5) * cw, (ys + 0.5) * ch], axis=1).astype(np.float32)
            radius = np.full(size, min(0.25 * min(cw, ch), self.rmax), np.float32)
            radius[0] = np.float32(self.rmax)  # keeps the context's largest radius fixed
            from .scenes import disk_mass
            dev = self.device
            st = {"pos": torch.from_numpy(pos).to(dev),
                  "vel": torch.zeros((size, 2), device=dev),
                  "theta": torch.zeros(size, device=dev), "omega": torch.zeros(size, device=dev),
                  "radius": torch.from_numpy(radius).to(dev),
                  "mass": torch.from_numpy(disk_mass(radius).astype(np.float32)).to(dev),
                  "id": torch.full((size,), -1, dtype=torch.int32, device=dev),
                  "type": torch.zeros(size, dtype=torch.int32, device=dev)}
            self._park = (key, size, st)
        st = self._park[2]
        return {k: v[:count] for k, v in st.items()}

    def set_window(self, parts, window):
        import torch
        from . import Simulation
        # bands that crossed through host memory (a gloo transport) come back
        parts = [p.to(self.device) if torch.is_tensor(p) else p for p in parts]
        st = concat(parts, self.typed)
        m = int(st["pos"].shape[0])
        # without free rows (one slab) the window is the whole scene: no padding
        parking = bool(self._free_rows(window, (0, self.sys.gy)))
        want = int(m * (1.0 + self.SPARE)) + 64 if parking else m
        room = len(self._free_rows(window)) * self.sys.gx if self.sim is not None else 0
        if self.sim is None or m + (1 if parking else 0) > self.capacity or \
                (not parking and m != self.capacity) or \
                (parking and self.capacity - m > room):
            if self.sim is not None:
                self.sim.close()
            self.capacity = want
            # rows for four times the first window's parked particles
            self.rows = self._context_rows(window, 4 * (want - m) if parking else 0)
            whole = self.rows == (0, self.sys.gy)
            self.sim = Simulation(self.sys, capacity=self.capacity, flags=self.flags,
                                  rows=None if whole else self.rows)
        if parking:
            st = concat([st, self._parked(self.capacity - m, window)], self.typed)
        self.gid = st["id"]
        self.m = m
        ids = torch.arange(self.capacity, dtype=torch.int32, device=self.device)
        self.sim.set_state(st["pos"], st["vel"], st["theta"], st["omega"], st["radius"],
                           st["mass"], ids, st["type"] if self.typed else None)

    def step(self, k: int):
        self.sim.step(k)

    def slots(self, lo: int, hi: int):
        import ctypes as C
        from ._lib import check, load
        f, c = C.c_uint32(0), C.c_uint32(0)
        check(load().dem_row_slots(self.sim.handle, lo, hi, C.byref(f), C.byref(c), None))
        return f.value, c.value

    def take(self, first: int, count: int, packed: bool = True):
        """Slots [first, first + count) of the current state with their
        global ids: packed rows, or a dict of tensors (views of the state
        but the ids; valid until the next step or set_window copies them)."""
        v = self.sim.state_view()
        sl = slice(first, first + count)
        st = {k: (None if v.get(k) is None else v[k][sl]) for k in FIELDS}
        st["id"] = self.gid[st["id"].long()]
        return pack(st) if packed else st

    def close(self):
        if self.sim is not None:
            self.sim.close()
            self.sim = None


def scene_bounds(sys, pos, world: int):
    """Slab boundaries balancing the particle counts of a global state."""
    rows = cell_rows(sys, pos)
    return partition_rows(np.bincount(rows, minlength=sys.gy), world)


def local_main(args):
    """The decomposition of `args.local` ranks held by one process on one
    GPU (slabs stepped one after another, bands exchanged by local copies),
    timed against the single-domain context on the same scene: the compute
    cost a rank adds by stepping a halo window and rebuilding it every
    `period` steps, without the transfers between GPUs.  Prints one JSON
    line."""
    import json
    import torch
    from . import CTX_PRESSURE, Simulation, scenes
    world = int(args.local)
    torch.cuda.set_device(0)
    sc = scenes.stacked_plain(args.n, world)
    bounds = scene_bounds(sc.sys, sc.pos, world)
    rmax = float(sc.radius.max())
    slabs = [HaloSlab(sc.sys, r, world, bounds, args.period, ContextStepper(sc.sys, rmax))
             for r in range(world)]
    for s in slabs:
        s.load(sc.state())
    ev = lambda: torch.cuda.Event(enable_timing=True)
    # warm-up: every window's graphs and two exchanges
    run_group(slabs, 2 * args.period + 3)
    torch.cuda.synchronize()
    # timed: `steps` steps in rounds of `period`; the windows' steps and the
    # rebuilds (band cut, exchange by copies, new window state) timed apart
    step_ms, rebuild_ms = 0.0, 0.0
    for k, more in _rounds(args.steps, args.period):
        a, b, c = ev(), ev(), ev()
        a.record()
        for s in slabs:
            s.advance(k)
        b.record()
        if more and world > 1:
            got = LocalExchange.exchange([s.bands() for s in slabs])
            for s, (below, above) in zip(slabs, got):
                s.rebuild(below, above)
        c.record()
        torch.cuda.synchronize()
        step_ms += a.elapsed_time(b)
        rebuild_ms += b.elapsed_time(c)
    caps = [s.stepper.capacity for s in slabs]
    moved = sum(s.moved_rows for s in slabs)
    for s in slabs:
        s.stepper.sim.check()
        s.stepper.close()
    # the single domain: the fused context on the whole scene
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x).view(np.int32) if x.dtype == np.uint32
                                   else np.ascontiguousarray(x))
    sim = Simulation(sc.sys, capacity=sc.n, flags=CTX_PRESSURE)
    sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass),
                  t(sc.id))
    sim.step(2 * args.period + 3)
    sim.step(2)
    sim.step(1)
    sim.step(2)
    torch.cuda.synchronize()
    a, b = ev(), ev()
    a.record()
    sim.step(args.steps)
    b.record()
    torch.cuda.synchronize()
    single_ms = a.elapsed_time(b)
    sim.check()
    sim.close()
    rounds = -(-args.steps // args.period)
    print(json.dumps({
        "workload": "%d stacked copies of the %d-disk plain-at-scale scene (%d disks, %d x %d "
                    "grid), %d slabs on one GPU" % (world, args.n, sc.n, sc.sys.gx, sc.sys.gy,
                                                    world),
        "steps": args.steps, "period": args.period, "halo_rows": slabs[0].halo,
        "slab_rows": bounds, "window_capacity": caps,
        "single_domain_ms_per_step": single_ms / args.steps,
        "windows_ms_per_step": step_ms / args.steps,
        "rebuilds_ms_per_step": rebuild_ms / args.steps,
        "rebuild_ms_each": rebuild_ms / max(1, rounds - 1),
        "per_rank_ms_per_step": (step_ms + rebuild_ms) / args.steps / world,
        "per_rank_over_single_share": (step_ms + rebuild_ms) / single_ms,
        "rows_exchanged_per_round": moved / max(1, rounds - 1)}), flush=True)


def main(argv=None):
    """A tall plain-at-scale scene (`ranks` copies of the n-disk scene stacked
    upward) decomposed over the ranks of a torchrun launch:

        torchrun --nproc-per-node N --master-addr 127.0.0.1 -m demso_b200.slab --n 4194304

    With ``--local N`` the N slabs run in this one process on one GPU
    (``local_main``)."""
    import argparse
    import datetime
    import json
    import os
    import torch
    import torch.distributed as dist
    from . import scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--period", type=int, default=20)
    ap.add_argument("--local", type=int, default=0,
                    help="hold this many slabs in one process on one GPU (no torchrun)")
    args = ap.parse_args(argv)
    if args.local:
        return local_main(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        sc = scenes.stacked_plain(args.n, world)
        bounds = scene_bounds(sc.sys, sc.pos, world)
        slab = HaloSlab(sc.sys, rank, world, bounds, args.period,
                        ContextStepper(sc.sys, float(sc.radius.max())))
        slab.load(sc.state())
        ex = DistExchange(rank, world, torch.device("cuda"))
        run(slab, ex, 2 * args.period)
        torch.cuda.synchronize()
        dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run(slab, ex, args.steps)
        e1.record()
        torch.cuda.synchronize()
        dt = torch.tensor([e0.elapsed_time(e1)], device="cuda")
        dist.all_reduce(dt, op=dist.ReduceOp.MAX)
        if rank == 0:
            print(json.dumps({"particles": sc.n, "ranks": world, "steps": args.steps,
                              "period": args.period, "halo_rows": slab.halo,
                              "particle_steps_per_s": sc.n * args.steps / (float(dt.item()) * 1e-3),
                              "bounds": bounds}))
        slab.stepper.close()
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
