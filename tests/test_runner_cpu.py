"""The headless runner's stepping plan, on the CPU: a stand-in for the GPU
context records every call, so the runner must issue exactly the scene's
steps, in chunks that never cross a frame, write one output.csv line per
step in order (each from its own step's rows, with that step's elapsed
time), and draw the frames at their steps."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "dsml", "blocks.dsml")


class _Image:
    def __init__(self, h, w):
        self.a = np.zeros((h, w, 4), np.uint8)

    def cpu(self):
        return self

    def numpy(self):
        return self.a


class _Sim:
    """Context stand-in: rows of step k carry x = k for every followed id."""
    made = []

    def __init__(self, sys, capacity, flags):
        self.steps = 0
        self.calls = []
        _Sim.made.append(self)

    def set_state(self, *args):
        pass

    def step(self, k):
        self.calls.append(("step", k))
        self.steps += k

    def step_followed(self, k, ids):
        self.calls.append(("followed", k))
        rows = np.zeros((k, len(ids), 12), np.float32)
        rows[..., 0] = np.asarray(ids, np.uint32).view(np.float32)[None, :]
        rows[..., 2] = (self.steps + 1 + np.arange(k, dtype=np.float32))[:, None]
        self.steps += k
        return rows

    def render(self, p):
        self.calls.append(("frame", self.steps))
        return _Image(p.imageDIMy, p.imageDIMx)

    def check(self):
        pass

    def close(self):
        pass


@pytest.mark.parametrize("steps,frame_every,chunk", [(75, 30, 16), (64, 0, 16), (7, 3, 256),
                                                     (40, 40, 256)])
def test_runner_plan(tmp_path, monkeypatch, steps, frame_every, chunk):
    import torch
    import demso_b200 as D
    from demso_b200 import dsml, run as R
    from demso_b200.output import elapsed_time
    monkeypatch.setattr(D, "Simulation", _Sim)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    _Sim.made.clear()
    csv = tmp_path / "output.csv"
    frames = tmp_path / "frames" if frame_every else None
    res = R.run(FIXTURE, steps=steps, seed=3, csv=str(csv),
                frames=str(frames) if frames else None, frame_every=frame_every, chunk=chunk)
    sim = _Sim.made[-1]
    assert sim.steps == steps and res["steps"] == steps
    followed = res["followed"]
    lines = csv.read_text().splitlines()
    assert len(lines) == steps
    dt = dsml.load(FIXTURE, seed=3).time_step
    for k, ln in enumerate(lines, start=1):
        f = ln.split(",")
        assert f[0] == "%f" % float(elapsed_time(dt, k))
        assert int(f[1]) == followed[0] and float(f[3]) == float(k)  # id, then x = step
    sizes = [k for what, k in sim.calls if what == "followed"]
    assert all(0 < k <= chunk for k in sizes) and sum(sizes) == steps
    drawn = [k for what, k in sim.calls if what == "frame"]
    if frame_every:
        assert drawn == list(range(0, steps + 1, frame_every))
        names = sorted(os.listdir(frames))
        assert names == ["frame_%07d.ppm" % k for k in drawn]
    else:
        assert drawn == []
    # no chunk crosses a frame
    done = 0
    for k in sizes:
        if frame_every:
            assert (done // frame_every) == ((done + k - 1) // frame_every)
        done += k
