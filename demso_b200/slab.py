"""Multi-GPU slab decomposition of the plain step, one process per GPU.

The cell grid is cut into slabs of whole cell rows, one per rank, balanced
by particle count at the start.  Cells are numbered row by row, so rank r's
cells are one contiguous range of cell keys, and the global sorted order of
the reference's step (a stable sort by cell key) is the concatenation of the
ranks' own sorted orders.  Each step, on every rank:

1. the cell key of every particle is computed; particles whose row now
   belongs to another rank are sent there (torch.distributed send/recv, NCCL
   over NVLink on GPUs);
2. the particles received from every rank are concatenated in rank order --
   the order they hold in the global sorted order of the previous step --
   with the rank's own staying particles in their place, and stably sorted
   by key: exactly the global stable sort restricted to the slab;
3. the slab's bottom row goes to rank r - 1 and its top row to rank r + 1 as
   ghosts; [ghosts below] + [slab] + [ghosts above] is then a contiguous
   window of the global sorted state, and the collide over it gives every
   slab particle the forces of the single-domain step, in the same order
   (the 3x3 neighbourhood of a slab cell lies in the window; cells beyond it
   are more than one row away and, across the grid's periodic wrap, a box
   height away, so they hold no contact);
4. the slab's particles are integrated.

The result is the single-domain step bit for bit.  The compute runs through
a backend with four operations (cell keys, stable order, cell ranges +
collide, integrate): ``CudaBackend`` uses the library's per-stage entry
points on CUDA tensors; the tests also drive the same decomposition with the
CPU oracle over gloo.
"""
from __future__ import annotations

import numpy as np

FIELDS = ("pos", "vel", "theta", "omega", "radius", "mass", "id", "type")


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


def pack(st: dict):
    """(m, 10) float32 rows: pos, vel, theta, omega, radius, mass, then the
    id and type words as raw bits."""
    import torch
    m = st["pos"].shape[0]
    typ = st["type"] if st.get("type") is not None else torch.zeros(m, dtype=torch.int32,
                                                                     device=st["pos"].device)
    cols = [st["pos"], st["vel"], st["theta"][:, None], st["omega"][:, None],
            st["radius"][:, None], st["mass"][:, None], st["id"].view(torch.float32)[:, None],
            typ.view(torch.float32)[:, None]]
    return torch.cat(cols, dim=1).contiguous()


def unpack(rows, typed: bool) -> dict:
    import torch
    rows = rows.contiguous()
    st = {"pos": rows[:, 0:2].contiguous(), "vel": rows[:, 2:4].contiguous(),
          "theta": rows[:, 4].contiguous(), "omega": rows[:, 5].contiguous(),
          "radius": rows[:, 6].contiguous(), "mass": rows[:, 7].contiguous(),
          "id": rows[:, 8].contiguous().view(torch.int32),
          "type": rows[:, 9].contiguous().view(torch.int32) if typed else None}
    return st


def take(st: dict, idx) -> dict:
    return {k: (None if v is None else v[idx].contiguous()) for k, v in st.items()}


class Exchange:
    """Variable-size row exchange between ranks (torch.distributed)."""

    def __init__(self, rank: int, world: int, device):
        self.rank, self.world, self.device = rank, world, device

    def all_to_all(self, outgoing):
        """outgoing[d]: (m_d, 10) rows for rank d (own entry kept locally);
        returns the rows received from every rank, in rank order."""
        import torch
        import torch.distributed as dist
        counts = torch.tensor([o.shape[0] for o in outgoing], dtype=torch.int64,
                              device=self.device)
        table = [torch.empty_like(counts) for _ in range(self.world)]
        dist.all_gather(table, counts)
        table = torch.stack(table).cpu().numpy()     # table[src, dst]
        ops, incoming = [], []
        for src in range(self.world):
            if src == self.rank:
                incoming.append(outgoing[src])
                continue
            n = int(table[src, self.rank])
            buf = torch.empty((n, 10), dtype=torch.float32, device=self.device)
            incoming.append(buf)
            if n:
                ops.append(dist.P2POp(dist.irecv, buf, src))
        for dst in range(self.world):
            if dst != self.rank and outgoing[dst].shape[0]:
                ops.append(dist.P2POp(dist.isend, outgoing[dst].contiguous(), dst))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return incoming

    def neighbours(self, down, up):
        """Send `down` to rank - 1 and `up` to rank + 1; returns the rows
        received from rank - 1 and rank + 1 (empty at the ends)."""
        import torch
        empty = lambda: torch.empty((0, 10), dtype=torch.float32, device=self.device)
        out = [empty() for _ in range(self.world)]
        if self.rank > 0:
            out[self.rank - 1] = down
        if self.rank < self.world - 1:
            out[self.rank + 1] = up
        got = self.all_to_all(out)
        below = got[self.rank - 1] if self.rank > 0 else empty()
        above = got[self.rank + 1] if self.rank < self.world - 1 else empty()
        return below, above


class SlabStep:
    """One rank's slab of a decomposed scene.  ``state`` holds the rank's
    particles (torch tensors on the backend's device) in their order of the
    last step; ``step(k)`` advances k steps; ``gather()`` returns the global
    sorted state on rank 0 (None elsewhere)."""

    def __init__(self, sys, state_all: dict, rank: int, world: int, backend, bounds=None):
        import torch
        self.sys, self.rank, self.world, self.be = sys, rank, world, backend
        self.typed = state_all.get("type") is not None and len(sys.materials) > 1
        full = {k: (None if (k == "type" and not self.typed) else
                    backend.tensor(state_all[k], k)) for k in FIELDS}
        keys = backend.keys(sys, full).to(torch.int64)
        rows = keys // sys.gx
        if bounds is None:
            counts = torch.bincount(rows.cpu(), minlength=sys.gy).numpy()
            bounds = partition_rows(counts, world)
        self.bounds = bounds
        owner = np.zeros(sys.gy, np.int64)
        for r in range(world):
            owner[bounds[r]:bounds[r + 1]] = r
        self.owner = torch.from_numpy(owner).to(full["pos"].device)
        self.state = take(full, torch.nonzero(self.owner[rows] == rank).flatten())
        self.ex = Exchange(rank, world, backend.comm_device)
        self.migrated = 0
        self.ghosts = 0

    def _step(self):
        import torch
        be, sys = self.be, self.sys
        st = self.state
        rows = be.keys(sys, st).to(torch.int64) // sys.gx
        dest = self.owner[rows]
        rowsets = pack(st)
        outgoing = [rowsets[dest == d].to(be.comm_device) for d in range(self.world)]
        incoming = self.ex.all_to_all(outgoing)
        self.migrated += sum(int(incoming[s].shape[0]) for s in range(self.world)
                             if s != self.rank)
        seq = unpack(torch.cat([t.to(st["pos"].device) for t in incoming]), self.typed)
        keys = be.keys(sys, seq)
        perm = be.stable_order(sys, keys)
        owned = take(seq, perm)
        krow = keys[perm].to(torch.int64) // sys.gx
        y0, y1 = self.bounds[self.rank], self.bounds[self.rank + 1]
        packed = pack(owned)
        bottom = packed[krow == y0].to(be.comm_device)
        top = packed[krow == y1 - 1].to(be.comm_device)
        below, above = self.ex.neighbours(bottom, top)
        dev = owned["pos"].device
        lo, m = int(below.shape[0]), int(packed.shape[0])
        self.ghosts += lo + int(above.shape[0])
        window = unpack(torch.cat([below.to(dev), packed, above.to(dev)]), self.typed)
        acc, alpha, pressure = be.collide(sys, window)
        sl = slice(lo, lo + m)
        self.state = be.integrate(sys, owned, acc[sl], alpha[sl], pressure[sl])

    def step(self, k: int = 1):
        for _ in range(int(k)):
            self._step()

    def gather(self):
        """The global state in the single-domain sorted order, on rank 0."""
        import torch
        import torch.distributed as dist
        rows = pack(self.state).to(self.be.comm_device)
        empty = lambda: torch.empty((0, 10), dtype=torch.float32, device=self.be.comm_device)
        out = [empty() for _ in range(self.world)]
        out[0] = rows
        got = self.ex.all_to_all(out) if self.world > 1 else [rows]
        if self.rank != 0:
            return None
        return unpack(torch.cat(got), self.typed)


class CudaBackend:
    """The library's per-stage entry points (calcHash, sortParticles,
    reorderDataAndFindCellStart, collide, integrateSystem) on CUDA tensors;
    collectives over NCCL."""

    def __init__(self, device="cuda"):
        import torch
        self.device = torch.device(device)
        self.comm_device = self.device

    def tensor(self, a, field):
        import torch
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        return torch.from_numpy(a).to(self.device)

    def keys(self, sys, st):
        import torch
        from . import calcHash
        m = st["pos"].shape[0]
        h = torch.empty(m, dtype=torch.int32, device=self.device)
        ix = torch.empty(m, dtype=torch.int32, device=self.device)
        if m:
            calcHash(sys, st["pos"], ix, h, m)
        return h

    def stable_order(self, sys, keys):
        import torch
        from . import sortParticles
        m = keys.shape[0]
        h = keys.clone()
        ix = torch.arange(m, dtype=torch.int32, device=self.device)
        if m:
            sortParticles(h, ix, m, max(1, sys.key_bits))
        return ix.to(torch.int64)

    def collide(self, sys, w):
        import torch
        from . import collide, reorderDataAndFindCellStart
        m = w["pos"].shape[0]
        nc = sys.num_cells
        dev = self.device
        f = lambda *s: torch.empty(*s, dtype=torch.float32, device=dev)
        i = lambda *s: torch.empty(*s, dtype=torch.int32, device=dev)
        acc, alpha, pr = f((m, 2)), f(m), f(m)
        if m == 0:
            return acc, alpha, pr
        keys = self.keys(sys, w)
        ident = torch.arange(m, dtype=torch.int32, device=dev)
        cs, ce = i(nc), torch.zeros(nc, dtype=torch.int32, device=dev)
        s = {k: torch.empty_like(v) for k, v in w.items() if v is not None}
        loc = i(m)  # sortedLoc[id]: the window's particles get local ids here
        typed = w.get("type") is not None
        reorderDataAndFindCellStart(sys, cs, ce, s["pos"], s["vel"], s["theta"], s["omega"],
                                    s["radius"], s["mass"], s["id"], loc,
                                    s["type"] if typed else None, keys, ident, w["pos"],
                                    w["vel"], w["theta"], w["omega"], w["radius"], w["mass"],
                                    ident, w["type"] if typed else None, m, nc)
        collide(sys, s["pos"], s["vel"], acc, s["omega"], alpha, s["type"] if typed else None,
                s["radius"], s["mass"], cs, ce, m, nc, pressure=pr)
        return acc, alpha, pr

    def integrate(self, sys, st, acc, alpha, pressure):
        from . import integrateSystem
        out = {k: (None if v is None else v.clone()) for k, v in st.items()}
        m = out["pos"].shape[0]
        if m:
            integrateSystem(sys, out["pos"], out["vel"], acc.contiguous(), out["theta"],
                            out["omega"], alpha.contiguous(), out["type"], out["radius"],
                            out["mass"], pressure.contiguous(), m)
        return out


def main(argv=None):
    """Plain-at-scale scene decomposed over the ranks of a torchrun launch:

        torchrun --nproc-per-node N --master-addr 127.0.0.1 -m demso_b200.slab --n 4194304
    """
    import argparse
    import json
    import os
    import time
    import torch
    import torch.distributed as dist
    from . import scenes
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--steps", type=int, default=100)
    args = ap.parse_args(argv)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    import datetime
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        sc = scenes.plain_at_scale(args.n)
        s = SlabStep(sc.sys, sc.state(), rank, world, CudaBackend())
        s.step(2)
        torch.cuda.synchronize()
        dist.barrier()
        t0 = time.perf_counter()
        s.step(args.steps)
        torch.cuda.synchronize()
        dt = torch.tensor([time.perf_counter() - t0], device="cuda")
        dist.all_reduce(dt, op=dist.ReduceOp.MAX)
        if rank == 0:
            print(json.dumps({"particles": sc.n, "ranks": world, "steps": args.steps,
                              "particle_steps_per_s": sc.n * args.steps / float(dt.item()),
                              "bounds": s.bounds}))
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
