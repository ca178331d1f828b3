"""Slab decomposition (demso_b200.slab) driven by the CPU oracle: the same
HaloSlab host logic as on GPUs, with the oracle stepping each window and
gloo as the transport.  Each worker process runs one rank."""
import os

import numpy as np


class OracleStepper:
    """A window stepped by PortOracle (f32) on CPU tensors; the window's
    particles carry window-local ids (the oracle's reorder indexes loc by
    id) and a table back to the global ids."""

    def __init__(self, sys):
        from oracle.oracle import PortOracle
        self.po = PortOracle("f32")
        self.sys = sys
        self.typed = len(sys.materials) > 1
        self.log2gx = sys.gx.bit_length() - 1

    def from_host(self, part):
        import torch
        t = {}
        for k, v in part.items():
            if v is None:
                t[k] = None
                continue
            a = np.ascontiguousarray(v)
            t[k] = torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a.copy())
        return t

    def set_window(self, parts, window):
        from demso_b200.slab import concat
        st = concat(parts, self.typed)
        self.gid = st["id"].numpy().copy()
        m = self.gid.shape[0]
        self.state = {k: (None if v is None else v.numpy().copy()) for k, v in st.items()}
        self.state["id"] = np.arange(m, dtype=np.uint32)
        if self.typed:
            self.state["type"] = self.state["type"].view(np.uint32)
        self.skeys = None

    def step(self, k):
        out = self.po.run(self.sys, self.state, k)
        self.state = {f: (None if out.get(f) is None else out[f])
                      for f in ("pos", "vel", "theta", "omega", "radius", "mass", "id", "type")}
        self.skeys = out["hash"]

    def slots(self, lo, hi):
        rows = (self.skeys >> np.uint32(self.log2gx)).astype(np.int64)
        a = int(np.searchsorted(rows, lo, side="left"))
        b = int(np.searchsorted(rows, hi, side="left"))
        return a, b - a

    def take(self, first, count, packed=True):
        import torch
        from demso_b200.slab import pack
        sl = slice(first, first + count)
        t = {}
        for k, v in self.state.items():
            if v is None:
                t[k] = None
                continue
            a = np.ascontiguousarray(v[sl])
            if k == "id":
                a = self.gid[a.astype(np.int64)]
            t[k] = torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a.copy())
        return pack(t) if packed else t


def make_scene(kind):
    """Tall scenes (copies stacked upward) with room for slabs and halos."""
    from demso_b200 import scenes
    if kind == "gas":
        return scenes.stacked(scenes.agitated_gas(n=1500, seed=31, vel_std=0.4), 4)
    if kind == "hot":  # disks cross slab boundaries every few steps
        return scenes.stacked(scenes.agitated_gas(n=1000, seed=32, vel_std=300.0,
                                                  omega_std=300.0), 4)
    if kind == "typed":
        return scenes.stacked(scenes.agitated_gas(n=1200, seed=33, n_mat=3, attraction=20.0,
                                                  vel_std=0.5), 4)
    return scenes.stacked(scenes.settling_pile(), 2)


def worker(rank, world, port, kind, steps, period, outdir):
    import torch
    import torch.distributed as dist
    from demso_b200.slab import DistExchange, HaloSlab, run, scene_bounds, unpack
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    try:
        sc = make_scene(kind)
        bounds = scene_bounds(sc.sys, sc.pos, world)
        slab = HaloSlab(sc.sys, rank, world, bounds, period, OracleStepper(sc.sys))
        slab.load(sc.state())
        ex = DistExchange(rank, world, torch.device("cpu"))
        run(slab, ex, steps)
        g = ex.gather(slab.own())
        stats = np.array([slab.rebuilds, slab.moved_rows, int(slab.own().shape[0])], np.int64)
        np.save(os.path.join(outdir, "stats_%d.npy" % rank), stats)
        if rank == 0:
            typed = len(sc.sys.materials) > 1
            out = {k: v.numpy() for k, v in unpack(g, typed).items() if v is not None}
            np.savez(os.path.join(outdir, "gathered.npz"), bounds=np.array(bounds), **out)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def gpu_worker(rank, world, port, kind, steps, period, outdir):
    """One rank of a decomposition on a GPU (every rank on device 0), the
    bands through gloo in host memory: no rank's kernels wait on another's."""
    import torch
    import torch.distributed as dist
    from demso_b200.slab import (ContextStepper, DistExchange, HaloSlab, run, scene_bounds,
                                 unpack)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    try:
        sc = make_scene(kind)
        bounds = scene_bounds(sc.sys, sc.pos, world)
        slab = HaloSlab(sc.sys, rank, world, bounds, period,
                        ContextStepper(sc.sys, float(sc.radius.max())))
        slab.load(sc.state())
        ex = DistExchange(rank, world, torch.device("cpu"))
        run(slab, ex, steps)
        g = ex.gather(slab.own().cpu())
        slab.stepper.sim.check()
        slab.stepper.close()
        if rank == 0:
            typed = len(sc.sys.materials) > 1
            out = {k: v.numpy() for k, v in unpack(g, typed).items() if v is not None}
            np.savez(os.path.join(outdir, "gathered.npz"), **out)
    finally:
        dist.barrier()
        dist.destroy_process_group()
