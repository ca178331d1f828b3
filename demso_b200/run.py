"""Run a .dsml scene headless: the reference's program (main.cu) without its
GL window.

Loads the scene (demso_b200.dsml), steps it on the GPU, writes the
followed-particle file in the reference's format (output.csv: one line per
step, writeOutputFile, functions.cu:608-661) and, on request, an image of
the particles every `--frame-every` steps as binary PPM (the reference's
plotParticles drawn into a device buffer).  The number of steps is
`--steps`, else the scene's <simduration> / <timestep>.

    python -m demso_b200.run scene.dsml --csv output.csv --frames frames/ --frame-every 100
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np


def run(path: str, steps: int = None, seed: int = 0, csv: str = None, frames: str = None,
        frame_every: int = 0, color_by_pressure: bool = False, chunk: int = 256) -> dict:
    import torch
    from . import CTX_ACCEL, CTX_PRESSURE, Simulation, dsml
    from .output import elapsed_time, followed_line, ppm_bytes, render_params

    sc = dsml.load(path, seed=seed)
    if steps is None:
        if sc.sim_duration == -1:
            raise ValueError("the scene runs forever (no <simduration>); give --steps")
        # timeCtrl->simDuration = simDuration / timeStep (main.cu:158), in float
        steps = int(np.float32(np.float32(sc.sim_duration) / np.float32(sc.time_step)))
    followed = [int(i) for i in sc.followed if int(i) < sc.n]
    dropped = [int(i) for i in sc.followed if int(i) >= sc.n]
    sim = Simulation(sc.system, capacity=max(sc.n, 1), flags=CTX_PRESSURE | CTX_ACCEL)
    st = sc.state()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32) if a.dtype == np.uint32
                                   else np.ascontiguousarray(a))
    sim.set_state(t(st["pos"]), t(st["vel"]), t(st["theta"]), t(st["omega"]), t(st["radius"]),
                  t(st["mass"]), t(st["id"]), t(st["type"]) if st["type"] is not None else None)
    out = open(csv, "w") if csv and followed else None
    if frames:
        os.makedirs(frames, exist_ok=True)
    colors = [t_["color"] for t_ in sc.types]

    def frame(k):
        pr = 1.0
        if color_by_pressure:
            # updatePressureScale (functions.cu:684-693): the largest pressure, or 1
            m = float(sim.get_state("cuda")["pressure"].max().item()) if sc.n else 0.0
            pr = m if m > 0.0 else 1.0
        p = render_params(sc.system.Lx, sc.system.Ly, colors, sc.image_height,
                          color_by_pressure=color_by_pressure, max_pressure=pr)
        img = sim.render(p).cpu().numpy()
        with open(os.path.join(frames, "frame_%07d.ppm" % k), "wb") as f:
            f.write(ppm_bytes(img))

    t0 = time.perf_counter()
    if frames:
        frame(0)
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        if frames and frame_every:
            k = min(k, frame_every - done % frame_every)
        if out is not None:
            # k steps with every step's rows gathered on the device (dem_step_followed)
            rows = sim.step_followed(k, followed)
            for j in range(k):
                out.write(followed_line(elapsed_time(sc.time_step, done + j + 1), rows[j]))
        else:
            sim.step(k)
        done += k
        if frames and frame_every and done % frame_every == 0:
            frame(done)
    torch.cuda.synchronize()
    sim.check()
    secs = time.perf_counter() - t0
    if out is not None:
        out.close()
    sim.close()
    return {"scene": os.path.basename(path), "particles": sc.n, "steps": steps,
            "seconds": secs, "particle_steps_per_s": sc.n * steps / secs if secs > 0 else None,
            "followed": followed, "followed_out_of_range": dropped,
            "grid": [sc.system.gx, sc.system.gy]}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("scene")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--csv", default="output.csv")
    ap.add_argument("--frames", default=None)
    ap.add_argument("--frame-every", type=int, default=0)
    ap.add_argument("--color-by-pressure", action="store_true")
    args = ap.parse_args(argv)
    res = run(args.scene, args.steps, args.seed, args.csv, args.frames, args.frame_every,
              args.color_by_pressure)
    if res["followed_out_of_range"]:
        print("followed ids beyond the %d particles were skipped: %s"
              % (res["particles"], res["followed_out_of_range"]), file=sys.stderr)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
