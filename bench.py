"""Benchmark of the plain FP32 DEM step at 4M disks on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one DEM time step (sort, reorder, collide + integrate) of the
4,194,304-disk "plain at scale" scene: log-normal radii (median 1 mm,
sigma 0.15, clipped [0.6, 1.6] mm), seeded random sequential placement to
area fraction 0.55 in a 4.1 m x 6.11 m walled box, 1024 x 1024 grid, dt 2e-6.
With N > 1 (torchrun, one rank per GPU) the ranks step ONE scene of N x 4M
disks (the 4M scene stacked N times upward) cut into slabs of cell rows: each
rank steps its slab's halo window with the fused context and the ranks
exchange bands over NCCL every --period steps (demso_b200.slab), the same
bits as one domain; --replicas instead steps an independent 4M-disk scene
per rank.  Weak scaling either way (4M disks per GPU).

`value` is whole-job particle-steps/s over K timed steps issued as one
dem_step call (device time, CUDA events, max over ranks); the library runs
them as one graph launch of its device-side step loop.  `e2e` is the same
workload through the C ABI with host buffers: the state uploaded from pinned
host memory, K steps with the reference's per-step followed-particle output
(writeOutputFile) of every step gathered on the device and copied to pinned
host memory (dem_step_followed), and the state downloaded, all inside the
timed region.  `roofline` is for the dominant kernel, timed by
CUDA events recorded around each stage's graph launch in a second pass of K
steps launched one step at a time (events cannot sit inside the device-side
loop); that pass's whole-step time is `ms_per_step_stage_timed`.
`cpu_baseline` times the reference's own step functions built for the host
(oracle/_ref) on a bounded sample of the same workload.

`--impl reference` times only that CPU reference on the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at 4M disks"
UNIT = "particle-steps/s"
N_DEFAULT = 4194304
# Algorithmic bytes of the step kernel, counted per stage of the reference step
# as the reference moves them, for the stages (or parts of them) it does:
#   collide: reads own pos/vel/omega/radius/mass 28, writes force 8 + torque 4
#     (neighbours are cache hits) = 40 per particle + 8 per cell (cell ranges);
#   integrate: reads pos, vel, omega, theta, radius, mass, acc, alpha 44, writes
#     pos, vel, omega, theta 24 = 68 per particle;
#   the gather half of the reorder (84 per particle in all): the step kernel
#     reads vel, theta, omega, mass, id at each particle's previous slot 24 and
#     writes them in sorted order 24, with loc 4 = 52; the sort phase moves the
#     positions and radii and writes the keys and slots (the other 32).
# The fused kernel keeps force, torque and the sorted fields in registers, so
# its own minimum is 88 per particle (reads 44, writes 44; reported beside).
STEP_KERNEL_STAGE_BYTES = {"collide": 40, "integrate": 68, "reorder_gather": 52}
STEP_KERNEL_BYTES_PER_PARTICLE = sum(STEP_KERNEL_STAGE_BYTES.values())
STEP_KERNEL_BYTES_PER_CELL = 8
FUSED_MIN_BYTES_PER_PARTICLE = 88
# Whole step, per particle: hash 16 + sort 52 + reorder 84 + collide 40 +
# integrate 68 = 260, plus 20 per cell (reorder 12, collide 8).
WHOLE_STEP_BYTES = lambda n, c: 260.0 * n + 20.0 * c  # whole-step model, per step
# the plain-at-scale sizes of the roofline curve (the same workload scaled)
DEFAULT_SWEEP = "65536,262144,1048576,4194304,16777216"
# the timed K-step call is repeated until this much device time is under load
MIN_TIMED_S = 1.0
MIN_REPEATS, MAX_REPEATS = 3, 5000
BACKWARD_REPEATS = 3  # timed adjoint backward calls (after an untimed first call)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.isfile(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index),
                                          "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU reference
def cpu_reference_rate(target_s: float, n_hint: int = 262144, seed: int = 0):
    """Particle-steps/s of the reference's step functions built for the host
    (oracle/_ref), or of the CPU restatement when that build is absent, on a
    bounded sample of the plain-at-scale workload."""
    from demso_b200 import scenes
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    sc = scenes.plain_at_scale(n_hint, seed=seed + 1000)
    if O.ref_available():
        h = O.RefHarness(threads=threads)
        h.setup(sc.sys, sc.radius, sc.mass, None)
        b = h.make_buffers(sc.state())
        h.run(b, 1)
        t0 = time.perf_counter()
        h.run(b, 1)
        t1 = time.perf_counter() - t0
        steps = max(1, min(1000, int(target_s / max(t1, 1e-6))))
        t0 = time.perf_counter()
        h.run(b, steps)
        dt = time.perf_counter() - t0
        kind, cores = "reference", h.threads
    else:
        po = O.PortOracle("f32")
        st = sc.state()
        t0 = time.perf_counter()
        po.run(sc.sys, st, 1)
        t1 = time.perf_counter() - t0
        steps = max(1, min(1000, int(target_s / max(t1, 1e-6))))
        t0 = time.perf_counter()
        po.run(sc.sys, st, steps)
        dt = time.perf_counter() - t0
        kind, cores = "port", 1
    rate = sc.n * steps / dt
    sample = ("%d steps of a %d-disk instance of the plain-at-scale workload (same radii, "
              "density and parameters; %dx%d grid) on %d host threads"
              % (steps, sc.n, sc.sys.gx, sc.sys.gy, cores))
    return dict(value=rate, unit=UNIT, cores=cores, kind=kind, sample=sample), dt


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # each of the K + W steps is a bounded sample sized so the run ends in minutes
    per_step = max(0.02, 150.0 / max(1, args.steps + args.warmup))
    from demso_b200 import scenes
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    sc = scenes.plain_at_scale(65536, seed=1000)
    if O.ref_available():
        h = O.RefHarness(threads=threads)
        h.setup(sc.sys, sc.radius, sc.mass, None)
        b = h.make_buffers(sc.state())
        h.run(b, 2)
        t0 = time.perf_counter()
        h.run(b, 2)
        rate = sc.n * 2 / (time.perf_counter() - t0)
        n_s = int(min(N_DEFAULT, max(4096, rate * per_step)))
        sc = scenes.plain_at_scale(n_s, seed=1000)
        h.setup(sc.sys, sc.radius, sc.mass, None)
        b = h.make_buffers(sc.state())
        h.run(b, args.warmup)
        t0 = time.perf_counter()
        h.run(b, args.steps)
        dt = time.perf_counter() - t0
        kind, cores = "reference", h.threads
    else:
        po = O.PortOracle("f32")
        n_s = 16384
        sc = scenes.plain_at_scale(n_s, seed=1000)
        st = po.run(sc.sys, sc.state(), args.warmup)
        t0 = time.perf_counter()
        po.run(sc.sys, st, args.steps)
        dt = time.perf_counter() - t0
        kind, cores = "port", 1
    value = sc.n * args.steps / dt
    sample = ("each step is one step of a %d-disk instance of the plain-at-scale workload "
              "(same radii, density and parameters, %dx%d grid) on %d host threads"
              % (sc.n, sc.sys.gx, sc.sys.gy, cores))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(args.n, None),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def config_dict(n, sc):
    d = {"workload": "plain at scale: %d disks, log-normal radii (median 1 mm, sigma 0.15, "
                     "clipped [0.6, 1.6] mm), seeded random sequential placement to area "
                     "fraction 0.55 in a walled box (4.1 m wide at 4M), zero initial velocity, "
                     "kn 1e5 N/m, kt 0.5 kn, damping ratio 0.3, friction 0.5, dt 2e-6 s, "
                     "grid cell >= 2 rmax" % n,
         "n_particles": n, "precision": "fp32 state and contact law (pressure sum in fp64)",
         "l2": "inputs larger than L2: the state read each step is >= 150 MB at 4M disks"}
    if sc is not None:
        d.update(grid=[sc.sys.gx, sc.sys.gy], box_m=[round(sc.sys.Lx, 4), round(sc.sys.Ly, 4)],
                 parallelism="replicas" if int(os.environ.get("WORLD_SIZE", "1")) > 1
                 else "single")
    return d


# ------------------------------------------------------------------ batched form
def measure_batched(steps: int, warmup: int, num: int = 4096, loop_sample: int = 256):
    """Batched form on the batched workload (4,096 specimens of 256..8,192
    disks, own boxes/parameters; 5,000 steps issued as one dem_step call) in
    its two forms -- one persistent launch of the resident step, and one
    graph launch of the device-side step loop -- against looping the plain
    single-scene step over an evenly spaced sample of the same specimens, in
    the faster of its two forms (graph path, cluster launch).  `value` is
    the faster batched form."""
    import torch
    import demso_b200 as D
    from demso_b200 import scenes
    specimens = scenes.specimen_batch(num=num, seed=0)
    total = sum(sc.n for sc in specimens)
    b = D.Batch([(sc.sys, sc.n) for sc in specimens], flags=D.CTX_PRESSURE | D.CTX_AUTOTUNE)
    st = scenes.concat_specimens(specimens)
    t = lambda a: torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a)
    b.set_state(t(st["pos"]), t(st["vel"]), t(st["theta"]), t(st["omega"]), t(st["radius"]),
                t(st["mass"]), t(st["id"]))
    b.step(max(3, warmup))
    while b.step_variant()["tuned"] < 0:
        b.step(1)
    b.step(2)  # instantiates the step-loop graph for this parity outside the timed region
    shape = b.step_variant()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.step(steps)
    e1.record()
    torch.cuda.synchronize()
    b.check()
    graph_path = total * steps / (e0.elapsed_time(e1) * 1e-3)
    kernels = b.kernels_per_step()
    b.close()
    # the resident form (DEM_CTX_RESIDENT): the call's steps as one persistent
    # launch, every bin of specimens stepped in one multiprocessor's shared
    # memory; its first call packs the bins and is untimed
    r = D.Batch([(sc.sys, sc.n) for sc in specimens], flags=D.CTX_PRESSURE | D.CTX_RESIDENT)
    r.set_state(t(st["pos"]), t(st["vel"]), t(st["theta"]), t(st["omega"]), t(st["radius"]),
                t(st["mass"]), t(st["id"]))
    r.step(max(3, warmup))
    torch.cuda.synchronize()
    e0.record()
    r.step(steps)
    e1.record()
    torch.cuda.synchronize()
    r.check()
    r.close()
    resident = total * steps / (e0.elapsed_time(e1) * 1e-3)
    batched = max(resident, graph_path)
    # looped plain step, in its strongest form: one single-scene context per
    # specimen, each stepping its `lsteps` steps as one dem_step call (one
    # graph launch of the device-side step loop), specimens one after another
    sample = specimens[::max(1, num // loop_sample)]
    sims = []
    for sc in sample:
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_PRESSURE)
        sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass),
                      t(sc.id))
        sim.step(3)
        sim.step(2)  # the step loop's graphs of both parities, captured untimed
        sim.step(1)
        sim.step(2)
        sims.append(sim)
    torch.cuda.synchronize()
    lsteps = max(4, min(steps, 500))
    e0.record()
    for sim in sims:
        sim.step(lsteps)
    e1.record()
    torch.cuda.synchronize()
    sample_n = sum(sc.n for sc in sample)
    looped_graph = sample_n * lsteps / (e0.elapsed_time(e1) * 1e-3)
    # the same, each specimen's context stepped as one thread-block cluster
    # launch (DEM_CTX_RESIDENT on a single scene of at most 8,192 disks)
    csims = []
    for sc in sample:
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_PRESSURE | D.CTX_RESIDENT)
        sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass),
                      t(sc.id))
        sim.step(3)
        csims.append(sim)
    torch.cuda.synchronize()
    e0.record()
    for sim in csims:
        sim.step(lsteps)
    e1.record()
    torch.cuda.synchronize()
    for sim in csims:
        sim.check()
        sim.close()
    looped_cluster = sample_n * lsteps / (e0.elapsed_time(e1) * 1e-3)
    # the looped plain step in its faster form is the baseline of the ratios
    looped = max(looped_graph, looped_cluster)
    # the weaker form measured before: single-step calls interleaved across
    # the contexts (two graph launches per specimen-step)
    isteps = 20
    e0.record()
    for _ in range(isteps):
        for sim in sims:
            sim.step(1)
    e1.record()
    torch.cuda.synchronize()
    interleaved = sample_n * isteps / (e0.elapsed_time(e1) * 1e-3)
    for sim in sims:
        sim.close()
    return {"metric": "aggregate particle-steps/s, batched vs looped plain",
            "value": batched, "looped_plain": looped, "ratio": batched / looped,
            "path": "resident" if resident >= graph_path else "graph",
            "resident": {"value": resident, "ratio": resident / looped, "launches": 1,
                         "form": "the %d steps as one persistent kernel launch; specimens in "
                                 "bins of up to 8,192 disks, each bin stepped inside one "
                                 "multiprocessor's shared memory" % steps},
            "graph_path": {"value": graph_path, "ratio": graph_path / looped,
                           "kernels_per_step": kernels,
                           "graph_launches": 1 if steps % 2 == 0 else 2,
                           "step_kernel_shape": [shape["threads"], shape["blocks_per_sm"]],
                           "form": "the %d steps as one graph launch of the device-side step "
                                   "loop, %d kernels per step" % (steps, kernels)},
            "looped_plain_forms": {"graph_path": looped_graph, "cluster": looped_cluster},
            "looped_plain_interleaved_single_steps": interleaved,
            "ratio_vs_interleaved": batched / interleaved,
            "unit": UNIT, "specimens": num, "particles": total, "steps": steps,
            "looped_sample": "%d of the %d specimens (every %d-th), each its own context "
                             "stepping %d steps as one dem_step call, one specimen after "
                             "another; the faster of the graph path (device-side step "
                             "loop) and the cluster launch"
                             % (len(sample), num, max(1, num // loop_sample), lsteps),
            "workload": "batched: specimens with counts log-uniform in [256, 8192], square "
                        "walled boxes at area fraction 0.5, radii U[0.9, 1.1] mm, kn "
                        "log-uniform [5e4, 5e5] N/m, friction U[0.2, 0.8], damping ratio "
                        "U[0.1, 0.5], dt 2e-6 s"}


# ------------------------------------------------------------------ adjoint
def measure_adjoint(n: int = 16384, steps: int = 2000, every: int = 100):
    """Cost of the adjoint on the differentiable workload (n disks released
    from a seeded heap onto a 20-degree incline, `steps` steps, a checkpoint
    every `every` steps): the plain forward, the checkpointing forward and the
    backward (recompute of each window plus the reverse steps), per step."""
    import ctypes as C
    import torch
    import demso_b200 as D
    from demso_b200 import scenes
    sc = scenes.incline_heap(n=n, seed=0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a))
    L = D.load()
    sim = D.Simulation(sc.sys, capacity=n, flags=D.CTX_PRESSURE | D.CTX_ACCEL)
    stream = torch.cuda.current_stream().cuda_stream
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def reset():
        sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass),
                      t(sc.id))

    reset()
    sim.step(50)
    reset()
    torch.cuda.synchronize()
    e0, e1, e2, e3 = ev(), ev(), ev(), ev()
    e0.record()
    sim.step(steps)
    e1.record()
    torch.cuda.synchronize()
    plain = e0.elapsed_time(e1) / steps
    reset()
    torch.cuda.synchronize()
    e0.record()
    D.check(L.dem_adj_forward(sim.handle, steps, every, stream))
    e1.record()
    torch.cuda.synchronize()
    fwd = e0.elapsed_time(e1) / steps
    # cotangents of loss = mean x-displacement + kinetic energy, by id
    st = {k: v.numpy() for k, v in sim.get_state("cpu").items() if v is not None}
    order = np.argsort(st["id"].view(np.uint32))
    m = st["mass"][order]
    r = st["radius"][order]
    inertia = (np.float32(2.0) * m * r * r) / np.float32(5.0)
    lam_pos = np.zeros((n, 2), np.float32)
    lam_pos[:, 0] = np.float32(1.0 / n)
    lam_vel = (m[:, None] * st["vel"][order]).astype(np.float32)
    lam_om = (inertia * st["omega"][order]).astype(np.float32)
    seeds = [torch.from_numpy(a).cuda() for a in (lam_pos, lam_vel, lam_om)]
    dp, dv, dw = (t0.clone() for t0 in seeds)
    grad = (C.c_double * 7)()
    # the first call allocates the context's record and scratch and captures
    # its loops (both kept for later calls): untimed; then the median of
    # BACKWARD_REPEATS calls, each from the same cotangent seeds
    bwds = []
    for rep in range(1 + BACKWARD_REPEATS):
        for dst, src in zip((dp, dv, dw), seeds):
            dst.copy_(src)
        torch.cuda.synchronize()
        e2.record()
        D.check(L.dem_adj_backward(sim.handle, dp.data_ptr(), dv.data_ptr(), dw.data_ptr(), grad,
                                   stream))
        e3.record()
        torch.cuda.synchronize()
        if rep:
            bwds.append(e2.elapsed_time(e3) / steps)
    bwd = float(np.median(bwds))
    sim.check()
    sim.close()
    return {"workload": "differentiable: %d disks (radii U[0.9, 1.1] mm) released from a seeded "
                        "heap onto a 20-degree incline, %d steps, checkpoint every %d steps"
                        % (n, steps, every),
            "plain_forward_ms_per_step": plain, "checkpointing_forward_ms_per_step": fwd,
            "backward_ms_per_step": bwd, "backward_over_forward": bwd / plain,
            "backward_repeats": {"count": len(bwds), "statistic": "median",
                                 "ms_per_step_min": float(np.min(bwds)),
                                 "ms_per_step_max": float(np.max(bwds)),
                                 "first_call": "untimed (allocates the record, captures the loops)"},
            "forward_plus_backward_over_forward": (fwd + bwd) / plain,
            "coefficient_gradients": list(grad),
            "finite": bool(np.all(np.isfinite(list(grad))) and
                           torch.isfinite(dv).all().item())}


# ------------------------------------------------------------------ config 0
def measure_settling_pile(steps: int = 20000):
    """The plain 2D settling pile (4,096 disks, 20,000 steps): wall time of
    the whole run on the GPU as one dem_step call, for the context stepped
    by a thread-block cluster (DEM_CTX_RESIDENT) and on the graph path; the
    faster gives gpu_seconds (settling_pile_cpu adds the host build's)."""
    import torch
    import demso_b200 as D
    from demso_b200 import scenes
    sc = scenes.settling_pile()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a))
    st = sc.state()

    def run(flags):
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=flags)
        sim.set_state(t(st["pos"]), t(st["vel"]), t(st["theta"]), t(st["omega"]), t(st["radius"]),
                      t(st["mass"]), t(st["id"]))
        sim.step(10)
        sim.set_state(t(st["pos"]), t(st["vel"]), t(st["theta"]), t(st["omega"]), t(st["radius"]),
                      t(st["mass"]), t(st["id"]))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sim.step(steps)
        e1.record()
        torch.cuda.synchronize()
        sim.check()
        sim.close()
        return e0.elapsed_time(e1) * 1e-3

    cluster_s = run(D.CTX_PRESSURE | D.CTX_RESIDENT)
    graph_s = run(D.CTX_PRESSURE)
    gpu_s = min(cluster_s, graph_s)
    out = {"workload": "plain 2D settling pile: 4096 disks, radii U[0.9, 1.1] mm, 64x64 "
                       "jittered lattice in a 0.2 x 0.2 m box, dt 2e-6 s, %d steps" % steps,
           "gpu_seconds": gpu_s, "gpu_steps_per_s": steps / gpu_s,
           "gpu_particle_steps_per_s": sc.n * steps / gpu_s,
           "path": "cluster" if cluster_s <= graph_s else "graph",
           "cluster_seconds": cluster_s, "graph_path_seconds": graph_s,
           "cluster_form": "one launch of a cluster of 8 blocks, each holding the scene in "
                           "shared memory and stepping an eighth of the disks",
           "graph_path_form": "one graph launch of the device-side step loop"}
    return out


def settling_pile_cpu(out: dict, steps: int = 20000, cpu_sample: int = 2000) -> dict:
    """The reference's step functions built for the host on the settling pile
    (timed on `cpu_sample` of the steps, all host threads), beside the GPU
    run of measure_settling_pile."""
    from demso_b200 import scenes
    from oracle import oracle as O
    sc = scenes.settling_pile()
    gpu_s = out["gpu_seconds"]
    if O.ref_available():
        h = O.RefHarness(threads=os.cpu_count() or 1)
        h.setup(sc.sys, sc.radius, sc.mass, None)
        b = h.make_buffers(sc.state())
        h.run(b, 10)
        t0 = time.perf_counter()
        h.run(b, cpu_sample)
        cpu_s = (time.perf_counter() - t0) * steps / cpu_sample
        out.update(cpu_reference_seconds_estimate=cpu_s, cpu_threads=h.threads,
                   cpu_sample="%d of the %d steps, scaled" % (cpu_sample, steps),
                   gpu_over_cpu=cpu_s / gpu_s)
    return out


def measure_sweep(sizes, steps: int = 200, warmup: int = 50):
    """The plain-at-scale workload at several sizes: particle-steps/s and the
    roofline fractions of the step kernel and of the whole step."""
    import ctypes as C
    import torch
    import demso_b200 as D
    from demso_b200 import scenes
    hbm, _ = peaks()
    rows = []
    for n in sizes:
        sc = scenes.plain_at_scale(n)
        sim = D.Simulation(sc.sys, capacity=sc.n, flags=D.CTX_PRESSURE | D.CTX_AUTOTUNE)
        t = lambda a: torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a)
        sim.set_state(t(sc.pos), t(sc.vel), t(sc.theta), t(sc.omega), t(sc.radius), t(sc.mass),
                      t(sc.id))
        sim.step(warmup)
        while sim.step_variant()["tuned"] < 0:
            sim.step(1)
        shape = sim.step_variant()
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record()
        sim.step(steps)  # one call: the device-side step loop
        e[1].record()
        torch.cuda.synchronize()
        D.check(D.load().dem_profile_begin(sim.handle, steps))
        e[2].record()
        sim.step(steps)  # stage timing, one step at a time
        e[3].record()
        torch.cuda.synchronize()
        ms = (C.c_float * D._lib.NUM_STAGES)()
        k = C.c_uint32(0)
        D.check(D.load().dem_profile_end(sim.handle, ms, C.byref(k)))
        sim.check()
        sim.close()
        step_ms = e[0].elapsed_time(e[1]) / steps
        cells = sc.sys.num_cells
        kern_ms = ms[2] / max(1, k.value)
        kb = STEP_KERNEL_BYTES_PER_PARTICLE * sc.n + STEP_KERNEL_BYTES_PER_CELL * cells
        rows.append({"n": sc.n, "grid": [sc.sys.gx, sc.sys.gy], "ms_per_step": step_ms,
                     "ms_per_step_stage_timed": e[2].elapsed_time(e[3]) / steps,
                     "step_kernel_shape": [shape["threads"], shape["blocks_per_sm"]],
                     "value": sc.n / (step_ms * 1e-3),
                     "sort_ms": ms[0] / max(1, k.value), "step_kernel_ms": kern_ms,
                     "step_kernel_frac": kb / (kern_ms * 1e-3) / 1e9 / hbm,
                     "whole_step_frac": WHOLE_STEP_BYTES(sc.n, cells) / (step_ms * 1e-3) / 1e9
                                        / hbm})
        del sc
    return rows


# ------------------------------------------------------------------ slabs
def main_slabs(args, world, rank, local, dist):
    """N > 1: one scene of N x n disks (the n-disk plain-at-scale scene
    stacked N times upward, n disks per GPU) cut into N slabs of cell rows
    (demso_b200.slab): every rank steps its slab's halo window with the fused
    context and the ranks exchange bands over NCCL every `period` steps.
    `value` counts the scene's N x n disks (not the windows' halo and parked
    particles) over the device time of K steps, max over ranks."""
    import ctypes as C
    import torch
    import demso_b200 as D
    from demso_b200 import scenes
    from demso_b200.slab import ContextStepper, DistExchange, HaloSlab, run, scene_bounds

    sc = scenes.stacked_plain(args.n, world)
    total = sc.n
    bounds = scene_bounds(sc.sys, sc.pos, world)
    stepper = ContextStepper(sc.sys, float(sc.radius.max()))
    slab = HaloSlab(sc.sys, rank, world, bounds, args.period, stepper)
    # this rank's window of the initial state, in pinned host memory (the
    # end-to-end pass uploads it from there)
    from demso_b200.slab import cell_rows
    rows = cell_rows(sc.sys, sc.pos)
    keep = np.nonzero((rows >= slab.wlo) & (rows < slab.whi))[0]
    host = {}
    for k in ("pos", "vel", "theta", "omega", "radius", "mass", "id"):
        a = np.ascontiguousarray(getattr(sc, k)[keep])
        host[k] = torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).pin_memory()
    host["type"] = None
    del sc, rows, keep
    comm = torch.device("cuda" if args.comm_backend == "nccl" else "cpu")
    ex = DistExchange(rank, world, comm)

    def reduce_max(values):
        t = torch.tensor(values, device=comm, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return t.cpu().numpy()

    def load():
        dev = {k: (None if v is None else v.to("cuda", non_blocking=True))
               for k, v in host.items()}
        stepper.set_window([dev], (slab.wlo, slab.whi))

    load()
    # warm-up: every graph of the window's context (both parities, the step
    # loop) and at least two band exchanges, untimed
    run(slab, ex, max(args.warmup, 2 * args.period + 3))
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    clocks = Clocks(local)
    clocks.start()
    reps, target = [], None
    while target is None or len(reps) < target:
        dist.barrier()
        torch.cuda.synchronize()
        ev[0].record(stream)
        run(slab, ex, args.steps)
        ev[1].record(stream)
        torch.cuda.synchronize()
        reps.append(ev[0].elapsed_time(ev[1]))
        if target is None:
            first = float(reduce_max([reps[0]])[0])
            target = int(min(MAX_REPEATS, max(MIN_REPEATS,
                                              np.ceil(1e3 * args.min_timed_s / first))))
    clk = clocks.stop()
    reps = reduce_max(reps)
    elapsed = float(np.median(reps))
    value = total * args.steps / (elapsed * 1e-3)
    stepper.sim.check()
    sim = stepper.sim
    kernels_per_step = sim.kernels_per_step()

    # the window's stage times (one step per launch, events around the
    # stages) for the step kernel's roofline; no exchange in this pass
    D.check(D.load().dem_profile_begin(sim.handle, args.period))
    sim.step(args.period)
    torch.cuda.synchronize()
    ms = (C.c_float * D._lib.NUM_STAGES)()
    nprof = C.c_uint32(0)
    D.check(D.load().dem_profile_end(sim.handle, ms, C.byref(nprof)))
    stage_ms = [ms[i] / max(1, nprof.value) for i in range(3)]
    hbm, kind = peaks()
    cells = stepper.sys.num_cells
    cap = stepper.capacity
    bytes_launch = STEP_KERNEL_BYTES_PER_PARTICLE * cap + STEP_KERNEL_BYTES_PER_CELL * cells
    achieved = bytes_launch / (stage_ms[2] * 1e-3) / 1e9

    # end to end: the window uploaded from pinned host memory, K steps with
    # their exchanges, the slab's own rows downloaded
    e2e = None
    if not args.no_e2e:
        times, target = [], None
        down = 0
        while target is None or len(times) < target:
            dist.barrier()
            t0 = time.perf_counter()
            load()
            run(slab, ex, args.steps)
            own = slab.own().cpu()
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            down = own.numel() * own.element_size()
            if target is None:
                first = float(reduce_max([times[0]])[0])
                target = int(min(MAX_REPEATS, max(MIN_REPEATS,
                                                  np.ceil(args.min_timed_s / first))))
        times = reduce_max(times)
        up = sum(v.numel() * v.element_size() for v in host.values() if v is not None)
        e2e = {"value": total * args.steps / float(np.median(times)), "unit": UNIT,
               "h2d_bytes_per_step": up / args.steps, "d2h_bytes_per_step": down / args.steps,
               "path": "each rank: its window set from pinned host memory, K steps with "
                       "the band exchanges, its own rows downloaded",
               "repeats": int(len(times)), "statistic": "median (host wall clock), max over ranks"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": elapsed / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(config_dict(args.n, None),
                               workload="%d stacked copies of the plain-at-scale scene of %d "
                                        "disks (%d disks in one box %.4g m x %.4g m, %d x %d "
                                        "grid)" % (world, args.n, total, stepper.sys.Lx,
                                                   stepper.sys.Ly, stepper.sys.gx,
                                                   stepper.sys.gy),
                               n_particles=total,
                               parallelism="slab decomposition over %d ranks: halo windows of "
                                           "%d rows, bands exchanged every %d steps over %s"
                                           % (world, slab.halo, args.period,
                                              "NCCL" if args.comm_backend == "nccl" else "gloo"),
                               slab_rows=bounds, window_capacity=cap),
                "timed_repeats": {"count": int(len(reps)), "statistic": "median",
                                  "timed_s": float(np.sum(reps)) * 1e-3},
                "roofline": {"bound": "hbm", "kernel": "step_kernel of rank 0's window",
                             "achieved": achieved, "peak": hbm, "unit": "GB/s",
                             "frac": achieved / hbm, "peak_kind": kind, "traffic": None,
                             "bytes_per_launch": bytes_launch},
                "stage_ms_per_step": {"sort_reorder": stage_ms[0],
                                      "collide_integrate": stage_ms[2]},
                "cpu_baseline": None, "e2e": e2e, "clocks": clk,
                "gpu_launches": kernels_per_step * args.steps,
                "kernels_per_step": kernels_per_step}
        print(json.dumps(line), flush=True)
    stepper.close()
    dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=500)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--particles", dest="n", type=int, default=N_DEFAULT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-specimens", type=int, default=4096,
                    help="specimens of the batched leg (a smaller batch for profiling)")
    ap.add_argument("--batched-steps", type=int, default=5000,
                    help="steps of the batched leg's timed call")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-pile", action="store_true")
    ap.add_argument("--sweep", default=DEFAULT_SWEEP,
                    help="comma-separated sizes of the plain-at-scale sweep, 200 steps each "
                         "(default: %s; empty for none)" % DEFAULT_SWEEP)
    ap.add_argument("--min-timed-s", type=float, default=MIN_TIMED_S,
                    help="repeat the timed K-step call until this much device time is timed "
                         "(at least %d repeats)" % MIN_REPEATS)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the step kernel's default launch shape (128 threads x 8 "
                         "blocks per SM) instead of timing the shapes on the first steps")
    ap.add_argument("--direct", action="store_true",
                    help="launch each kernel directly instead of through CUDA graphs "
                         "(for per-kernel profilers; one host read-back per step)")
    ap.add_argument("--period", type=int, default=40,
                    help="N > 1: steps between the slabs' band exchanges")
    ap.add_argument("--comm-backend", default="nccl", choices=["nccl", "gloo"],
                    help="N > 1: process-group backend; gloo moves the bands through host "
                         "memory (for running several ranks on one GPU in tests)")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: every rank steps its own n-disk scene instead of one slab "
                         "of a shared N x n-disk scene")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import demso_b200 as D
    from demso_b200 import scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local % torch.cuda.device_count())
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(args.comm_backend, timeout=datetime.timedelta(seconds=120))

    if world > 1 and not args.replicas:
        return main_slabs(args, world, rank, local, dist)

    def barrier():
        if dist is not None:
            dist.barrier()

    sc = scenes.plain_at_scale(args.n, seed=rank)
    n = sc.n
    sim = D.Simulation(sc.sys, capacity=n,
                       flags=D.CTX_PRESSURE | (D.CTX_DIRECT if args.direct else 0)
                       | (0 if args.no_autotune else D.CTX_AUTOTUNE))
    pin = lambda a: torch.from_numpy(a.view(np.int32) if a.dtype == np.uint32 else a).pin_memory()
    host = {k: pin(getattr(sc, k)) for k in ("pos", "vel", "theta", "omega", "radius", "mass",
                                              "id")}
    stream = torch.cuda.current_stream()
    sim.set_state(host["pos"], host["vel"], host["theta"], host["omega"], host["radius"],
                  host["mass"], host["id"])
    sim.step(args.warmup)
    # the launch-shape tuner times its variants on the first 24 steps; any it
    # still needs run here, untimed
    while sim.step_variant()["tuned"] < 0:
        sim.step(1)
    # the device-side step loop's graphs of both parities (a multi-step call
    # starting on an even and on an odd step) are captured here, untimed
    sim.step(2)
    sim.step(1)
    sim.step(2)
    torch.cuda.synchronize()
    sim.check()
    kernels_per_step = sim.kernels_per_step()
    shape = sim.step_variant()

    # ---- timed region (device-resident state): the K steps as one dem_step
    # call, which the library runs as one graph launch of its device-side
    # step loop.  The K-step call is repeated, each repeat bracketed by a
    # barrier and a synchronize, until at least MIN_TIMED_S of device time is
    # under load; `value` is from the median repeat (max over ranks).
    clocks = Clocks(local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    clocks.start()
    reps = []
    target = None
    while target is None or len(reps) < target:
        barrier()
        torch.cuda.synchronize()
        ev[0].record(stream)
        sim.step(args.steps)
        ev[1].record(stream)
        torch.cuda.synchronize()
        reps.append(ev[0].elapsed_time(ev[1]))
        if target is None:
            first = torch.tensor([reps[0]], device="cuda")
            if dist is not None:
                dist.all_reduce(first, op=dist.ReduceOp.MAX)
            target = int(min(MAX_REPEATS, max(MIN_REPEATS,
                                              np.ceil(1e3 * args.min_timed_s / float(first.item())))))
    # ---- stage timing: K more steps, launched one step at a time with CUDA
    # events around each stage (events cannot sit inside the device-side
    # loop); the roofline's kernel duration comes from this pass
    D.check(D.load().dem_profile_begin(sim.handle, args.steps))
    ev[2].record(stream)
    sim.step(args.steps)
    ev[3].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    import ctypes as C
    ms = (C.c_float * D._lib.NUM_STAGES)()
    nprof = C.c_uint32(0)
    D.check(D.load().dem_profile_end(sim.handle, ms, C.byref(nprof)))
    elapsed_staged = ev[2].elapsed_time(ev[3])
    barrier()
    t = torch.tensor(reps + [elapsed_staged], device="cuda", dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    t = t.cpu().numpy()
    reps, elapsed_staged = t[:-1], float(t[-1])
    elapsed = float(np.median(reps))
    sim.check()
    value = n * world * args.steps / (elapsed * 1e-3)
    # kernels of the timed call: every step's, plus the loop's init kernel and
    # one count-down kernel per pair of steps (none on direct launches)
    loop_kernels = 0 if args.direct or args.steps < 2 else 1 + args.steps // 2

    stage_ms = [ms[i] / max(1, nprof.value) for i in range(3)]
    stage_names = ["sort_reorder", "reorder_separate", "collide_integrate"]
    dom = 2 if stage_ms[2] >= stage_ms[0] else 0
    hbm, kind = peaks()
    cells = sc.sys.num_cells
    if dom == 2:
        bytes_launch = STEP_KERNEL_BYTES_PER_PARTICLE * n + STEP_KERNEL_BYTES_PER_CELL * cells
        kname = "step_kernel (collide + integrate + next hash + gather into sorted order)"
    else:
        # counted as its share of the reorder alone (positions and radii 12 B
        # in and out, key and slot 8 B per particle, 12 B per cell); the sort
        # work is not counted
        bytes_launch = 32 * n + 12 * cells
        kname = "sort phase (incremental sort + positions and radii into sorted order)"
    achieved = bytes_launch / (stage_ms[dom] * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.txt")
    if os.path.isfile(tf):
        for ln in open(tf):
            f = ln.split()
            if len(f) >= 3 and f[0] == stage_names[dom] and f[1] == "bytes_per_particle":
                traffic = float(f[2]) * n
    whole_bytes = WHOLE_STEP_BYTES(n, cells)
    step_ms = elapsed / args.steps

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        sim2 = D.Simulation(sc.sys, capacity=n, flags=D.CTX_PRESSURE | D.CTX_ACCEL)
        sim2.set_step_variant(shape["variant"])
        out_host = {k: torch.empty_like(v).pin_memory() for k, v in host.items()}
        follow = np.array([n // 3, (2 * n) // 3], dtype=np.uint32)
        # every step's followed rows (the reference's per-step output) are
        # gathered on the device inside the step loop and reach this pinned
        # buffer by one copy (dem_step_followed)
        rows = torch.zeros(args.steps * follow.size * 12, dtype=torch.float32).pin_memory()
        L = D.load()
        p = lambda k: out_host[k].data_ptr()

        def e2e_pass():
            sim2.set_state(host["pos"], host["vel"], host["theta"], host["omega"],
                           host["radius"], host["mass"], host["id"])
            sim2.step_followed(args.steps, follow, rows)
            D.check(L.dem_get_state(sim2.handle, p("pos"), p("vel"), p("theta"), p("omega"),
                                    p("radius"), p("mass"), p("id"), None, None, None, None,
                                    None, 1, D._stream()))
            torch.cuda.synchronize()

        # warm-up outside the timed region: the step loop's graphs of both
        # parities, and one whole pass of K steps (the followed-row ring grows
        # to K steps and its loop graphs are captured)
        sim2.set_state(host["pos"], host["vel"], host["theta"], host["omega"], host["radius"],
                       host["mass"], host["id"])
        sim2.step_followed(3, follow, rows)
        sim2.step(1)
        sim2.step_followed(2, follow, rows)
        e2e_pass()
        # timed: the pass repeated (each one the state up, K steps with their
        # rows, the state down) until MIN_TIMED_S, the median kept
        times = []
        target = None
        while target is None or len(times) < target:
            barrier()
            t0 = time.perf_counter()
            e2e_pass()
            times.append(time.perf_counter() - t0)
            if target is None:
                # every rank makes the same number of passes
                first = torch.tensor([times[0]], device="cuda", dtype=torch.float64)
                if dist is not None:
                    dist.all_reduce(first, op=dist.ReduceOp.MAX)
                target = int(min(MAX_REPEATS, max(MIN_REPEATS,
                                                  np.ceil(args.min_timed_s / float(first.item())))))
        last = rows.numpy().reshape(args.steps, follow.size, 12)[-1]
        if not np.array_equal(last[:, 0].view(np.uint32), follow):
            raise RuntimeError("the last step's followed rows were not written")
        t = torch.tensor(times, device="cuda", dtype=torch.float64)
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        times = t.cpu().numpy()
        e2e_s = float(np.median(times))
        state_bytes = sum(v.numel() * v.element_size() for v in host.values())
        e2e = {"value": n * world * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": state_bytes / args.steps + 48 * follow.size,
               "path": "dem_set_state from pinned host memory, dem_step_followed (the "
                       "followed rows of every step), dem_get_state to pinned host memory",
               "repeats": int(len(times)), "statistic": "median (host wall clock)",
               "ms_min": 1e3 * float(times.min()), "ms_max": 1e3 * float(times.max())}
        sim2.close()

    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        try:
            batched = measure_batched(args.batched_steps, args.warmup,
                                      num=args.batched_specimens)
        except Exception as e:  # reported beside the headline, never instead of it
            batched = {"error": str(e)}

    pile = None
    if rank == 0 and world == 1 and not args.no_pile:
        try:
            pile = measure_settling_pile()
        except Exception as e:  # reported beside the headline, never instead of it
            pile = {"error": str(e)}
    sweep = None
    if rank == 0 and world == 1 and args.sweep:
        sweep = measure_sweep([int(v) for v in args.sweep.split(",") if v])

    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        try:
            adjoint = measure_adjoint()
        except Exception as e:  # reported beside the headline, never instead of it
            adjoint = {"error": str(e)}

    # ---- host-core measurements, after every GPU leg: the reference's host
    # build leaves its OpenMP threads busy on every core for a while after it
    # returns, which would slow the host-side work of a GPU leg run after it
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu, _ = cpu_reference_rate(12.0)
        except Exception as e:  # the baseline is reported, never the target
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "unavailable",
                   "sample": "failed: %s" % e}
    if pile is not None and "error" not in pile:
        try:
            pile = settling_pile_cpu(pile)
        except Exception as e:  # reported beside the GPU time, never instead of it
            pile["cpu_error"] = str(e)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": dict(config_dict(n, sc),
                               launch="direct, no graphs" if args.direct
                               else "one graph launch of the device-side step loop for the "
                                    "K steps (stage timing: a second pass of K steps, two "
                                    "graph launches per step)"),
                "ms_per_step_stage_timed": elapsed_staged / args.steps,
                "timed_repeats": {"count": int(len(reps)), "statistic": "median",
                                  "timed_s": float(np.sum(reps)) * 1e-3,
                                  "ms_per_step_min": float(np.min(reps)) / args.steps,
                                  "ms_per_step_max": float(np.max(reps)) / args.steps},
                "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved,
                             "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                             "peak_kind": kind, "traffic": traffic,
                             "bytes_per_launch": bytes_launch,
                             "stage_bytes_per_particle": (STEP_KERNEL_STAGE_BYTES if dom == 2
                                                          else {"reorder_move": 32}),
                             "fused_minimum_frac": (FUSED_MIN_BYTES_PER_PARTICLE * n
                                                    / (stage_ms[dom] * 1e-3) / 1e9 / hbm
                                                    if dom == 2 else None)},
                "stage_ms_per_step": {"sort_reorder": stage_ms[0],
                                      "collide_integrate": stage_ms[2]},
                "whole_step": {"model_bytes_per_step": whole_bytes,
                               "achieved_gbs": whole_bytes / (step_ms * 1e-3) / 1e9,
                               "frac": whole_bytes / (step_ms * 1e-3) / 1e9 / hbm},
                "cpu_baseline": cpu, "e2e": e2e, "clocks": clk, "batched": batched,
                "adjoint": adjoint, "settling_pile": pile,
                "gpu_launches": kernels_per_step * args.steps + loop_kernels,
                "kernels_per_step": kernels_per_step,
                "step_kernel_shape": {"threads": shape["threads"],
                                      "blocks_per_sm": shape["blocks_per_sm"],
                                      "tuned": shape["tuned"] == 1,
                                      "tuner_median_ms": shape["median_ms"]}}
        if sweep is not None:
            line["sweep"] = sweep
        print(json.dumps(line), flush=True)
    sim.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
