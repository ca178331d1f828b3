"""Batched differentiable calibration (demso_b200.calibrate) on a few small
column specimens, with column-height profiles as the only targets and the
model following its own run: the loss and its gradient vanish at the hidden
parameters, and the friction gradient does not point away from the hidden
value."""
import math

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cal():
    from demso_b200 import calibrate as C
    specimens = C.column_specimens(6, seed=3, nmin=300, nmax=700)
    # the columns fall freely for the first few milliseconds: window 1
    # (steps 3,000 to 6,000) is the first with contacts throughout
    c = C.Calibration(specimens, windows=2, window_steps=3000, shot_steps=300, every=100,
                      bin_width=2e-3)
    c.make_targets()
    yield c
    c.close()


def _window1(cal, kn, mu):
    return cal.loss_and_grad(1, kn, mu, cal.state_at(1, kn, mu))


def test_loss_and_gradient_vanish_at_hidden_parameters(cal):
    from demso_b200 import calibrate as C
    loss, (dkn, dmu), _ = _window1(cal, *C.HIDDEN)
    assert loss == 0.0 and dkn == 0.0 and dmu == 0.0


def test_friction_gradient_points_toward_hidden_value(cal):
    from demso_b200 import calibrate as C
    kn = C.HIDDEN[0]
    low = _window1(cal, kn, 0.35)
    high = _window1(cal, kn, 0.80)
    assert low[0] > 0.0 and high[0] > 0.0
    assert math.isfinite(low[1][0]) and math.isfinite(high[1][0])
    # below the hidden value friction must rise; above it the gradient is
    # zero once every contact sticks (the stick force does not depend on
    # friction), else positive
    assert low[1][1] < 0.0 <= high[1][1]


def test_adam_steps_follow_the_models_own_run(cal):
    kn, mu, hist = cal.run(kn0=1.5e5, mu0=0.45, iters=3)
    assert len(hist) == 3 and all(math.isfinite(h["loss"]) for h in hist)
    assert math.isfinite(kn) and math.isfinite(mu)
