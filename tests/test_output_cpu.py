"""Headless output host logic: output.csv lines against the C printf
restatement of the reference's writeOutputFile, the reference's elapsed-time
and image-width arithmetic, the PPM layout, and the CPU disk splat against
the reference's own plotSpheresD built for the host."""
import numpy as np
import pytest

from demso_b200 import output
from oracle.oracle import RenderOracle, ref_available
from render_scenes import COLORS, reference_splat, splat_scene


def test_followed_line_is_the_reference_format():
    rng = np.random.default_rng(1)
    ro = RenderOracle()
    for count in (0, 1, 3, 17):
        rows = rng.normal(scale=10.0 ** rng.integers(-8, 6), size=(count, 12)).astype(np.float32)
        rows.view(np.uint32)[:, 0] = rng.integers(0, 2**32 - 1, size=count, dtype=np.uint64)
        rows.view(np.uint32)[:, 1] = rng.integers(0, 10, size=count)
        rows[:, 5] = np.float32(-0.0) if count else rows[:, 5]
        for step in (1, 7, 123457):
            el = output.elapsed_time(2e-6, step)
            assert output.followed_line(el, rows) == ro.followed_line(el, rows)


def test_elapsed_time_and_image_width_use_float_arithmetic():
    assert output.elapsed_time(1e-3, 3) == np.float32(np.float32(1e-3) * np.float32(3))
    p = output.render_params(10.0, 7.0, [(255, 0, 0)], image_height=800)
    assert (p.imageDIMx, p.imageDIMy) == (int(np.float32(10 / np.float32(7)) * 800), 800)
    assert p.viewRotations == 1 and p.colorByPressure == 0 and p.bgColor == 0


def test_ppm_puts_the_top_of_the_box_first():
    img = np.zeros((2, 3, 4), np.uint8)
    img[0, :, 0] = 10   # bottom row
    img[1, :, 1] = 20   # top row
    b = output.ppm_bytes(img)
    head = b"P6\n3 2\n255\n"
    assert b.startswith(head)
    px = np.frombuffer(b[len(head):], np.uint8).reshape(2, 3, 3)
    assert np.all(px[0, :, 1] == 20) and np.all(px[1, :, 0] == 10)


def test_render_oracle_draws_disks_and_lines():
    """A lone disk: its pixels, shading and the orientation line."""
    ro = RenderOracle()
    img = ro.render(40, 40, 0, True, False, 1.0, [(200, 100, 50)], 1.0, 1.0,
                    np.float32([[0.5, 0.5]]), np.float32([0.0]), None, np.float32([0.1]), None)
    f = np.sqrt(np.float32((np.float32(16.0) - np.float32(9.0)) / np.float32(16.0)))
    expect = tuple(int(np.float32(c) * f) for c in (200, 100, 50, 255))
    assert tuple(img[20, 17]) == expect and tuple(img[23, 20]) == expect
    assert np.all(img[20, 20:24] == 0)          # the line along +x from the centre
    assert np.all(img[20, 15] == 0) and np.all(img[0, 0] == 0)
    covered = np.count_nonzero(img[..., 3])
    assert abs(covered + 4 - np.pi * 16) < 8


@pytest.mark.skipif(not ref_available(), reason="reference host build absent")
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
@pytest.mark.parametrize("lines,by_pressure", [(False, False), (True, False), (True, True)])
def test_cpu_splat_is_the_reference_plotspheres(seed, lines, by_pressure):
    """The restatement (oracle/dem_render.c) against the reference's own
    plotSpheresD (particles_kernel.cuh:656-734) built for the host and run
    in index order: equal everywhere except the few pixels whose disk/line
    class the reference's output cannot decide (none without lines)."""
    sc = splat_scene(seed)
    ref, amb = reference_splat(sc, lines, by_pressure)
    H = sc["height"]
    mine = RenderOracle().render(H, H, 9, lines, by_pressure, 1.5, COLORS, 1.0, 1.0, sc["pos"],
                                 sc["theta"], sc["type"], sc["radius"], sc["pressure"])
    assert not lines or np.count_nonzero(np.all(ref == 0, axis=2)) > 5000
    assert amb.sum() < 1e-4 * H * H and (lines or amb.sum() == 0)
    assert np.array_equal(ref[~amb], mine[~amb])
