"""Slab decomposition (demso_b200.slab) driven by the CPU oracle: the same
SlabStep host logic as on GPUs, with the oracle's per-stage functions as the
backend and gloo as the transport.  Each worker process runs one rank."""
import os

import numpy as np


class OracleBackend:
    """PortOracle (f32) stages on torch CPU tensors."""

    def __init__(self):
        import torch
        from oracle.oracle import PortOracle
        self.po = PortOracle("f32")
        self.comm_device = torch.device("cpu")

    def tensor(self, a, field):
        import torch
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint32:
            a = a.view(np.int32)
        return torch.from_numpy(a.copy())

    @staticmethod
    def _np(st):
        out = {}
        for k, v in st.items():
            if v is None:
                out[k] = None
            elif k in ("id", "type"):
                out[k] = v.numpy().view(np.uint32)
            else:
                out[k] = v.numpy()
        return out

    def keys(self, sys, st):
        import torch
        h, _ = self.po.calc_hash(sys, st["pos"].numpy())
        return torch.from_numpy(h.view(np.int32).copy())

    def stable_order(self, sys, keys):
        import torch
        m = keys.shape[0]
        h, ix = self.po.sort(keys.numpy().view(np.uint32), np.arange(m, dtype=np.uint32))
        return torch.from_numpy(ix.astype(np.int64))

    def collide(self, sys, w):
        import torch
        wn = self._np(w)
        m = wn["pos"].shape[0]
        if m == 0:
            return (torch.zeros((0, 2)), torch.zeros(0), torch.zeros(0))
        h, _ = self.po.calc_hash(sys, wn["pos"])
        # the reorder scatters loc[id]: give the window local ids (the
        # collide does not read ids)
        wn["id"] = np.arange(m, dtype=np.uint32)
        cs, ce, s = self.po.reorder(sys, h, np.arange(m, dtype=np.uint32), wn)
        acc, alpha, pr = self.po.collide(sys, s, cs, ce)
        return torch.from_numpy(acc), torch.from_numpy(alpha), torch.from_numpy(pr)

    def integrate(self, sys, st, acc, alpha, pressure):
        import torch
        sn = self._np(st)
        out = dict(st)
        if sn["pos"].shape[0] == 0:
            return out
        pos, vel, th, om, _ = self.po.integrate(sys, sn, acc.numpy(), alpha.numpy(),
                                                pressure.numpy())
        out.update(pos=torch.from_numpy(pos), vel=torch.from_numpy(vel),
                   theta=torch.from_numpy(th), omega=torch.from_numpy(om))
        return out


def make_scene(kind):
    from demso_b200 import scenes
    if kind == "gas":
        return scenes.agitated_gas(n=3000, seed=31, vel_std=0.4)
    if kind == "hot":  # particles cross slab boundaries every few steps
        return scenes.agitated_gas(n=2000, seed=32, vel_std=30.0, omega_std=300.0)
    if kind == "typed":
        return scenes.agitated_gas(n=2500, seed=33, n_mat=3, attraction=20.0, vel_std=0.5)
    return scenes.settling_pile()


def worker(rank, world, port, kind, steps, outdir):
    import torch.distributed as dist
    from demso_b200.slab import SlabStep
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    try:
        sc = make_scene(kind)
        s = SlabStep(sc.sys, sc.state(), rank, world, OracleBackend())
        s.step(steps)
        g = s.gather()
        stats = np.array([s.migrated, s.ghosts, s.state["pos"].shape[0]], np.int64)
        np.save(os.path.join(outdir, "stats_%d.npy" % rank), stats)
        if rank == 0:
            out = {k: (v.numpy() if v is not None else None) for k, v in g.items()}
            np.savez(os.path.join(outdir, "gathered.npz"),
                     **{k: v for k, v in out.items() if v is not None},
                     bounds=np.array(s.bounds))
    finally:
        dist.barrier()
        dist.destroy_process_group()
