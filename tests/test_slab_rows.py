"""Host logic of the slab windows' row windows (no GPU): the cell rows a
window's context spans and the scene rows its parked particles use."""
import pytest

from demso_b200 import scenes


def _stepper(sys):
    from demso_b200.slab import ContextStepper
    return ContextStepper(sys, 1e-3, device="cpu")


@pytest.mark.parametrize("window,parked,expect", [
    ((0, 150), 3320, (0, 256)),        # bottom slab: 150 rows + 2 + 26 parked rows
    ((106, 278), 3840, (106, 256)),     # middle slab
    ((362, 512), 3320, (362, 256)),     # top slab
    ((0, 300), 3320, (0, 512)),         # rounds up to the whole grid
    ((100, 200), 0, (100, 128)),
])
def test_context_rows(window, parked, expect):
    sys = scenes.stacked_plain(65536, 4).sys  # 128 x 512 cells
    assert _stepper(sys)._context_rows(window, parked) == expect


@pytest.mark.parametrize("window,rows", [((0, 150), (0, 256)), ((106, 278), (106, 256)),
                                         ((362, 512), (362, 256)), ((200, 330), (0, 512))])
def test_parking_rows_clear_the_window(window, rows):
    """Every parking row is in the scene, two or more rows from the window,
    and on its own cell row of the context, at least one cell row clear of
    the window's rows on either side."""
    sys = scenes.stacked_plain(65536, 4).sys
    st = _stepper(sys)
    st.rows = rows
    wlo, whi = window
    free = st._free_rows(window)
    count = rows[1]
    local = [(y - wlo) % count for y in free]
    assert len(set(local)) == len(local)
    assert len(free) == min(count - (whi - wlo) - 2, sum(1 for y in range(sys.gy)
                                                          if y <= wlo - 2 or y >= whi + 1))
    for y, lr in zip(free, local):
        assert 0 <= y < sys.gy
        assert y <= wlo - 2 or y >= whi + 1
        assert whi - wlo + 1 <= lr < count - 1


def test_one_slab_parks_nothing():
    sys = scenes.stacked_plain(65536, 4).sys
    assert _stepper(sys)._free_rows((0, sys.gy), (0, sys.gy)) == []
