"""Host-side pieces of bench.py's measurement contract that need no GPU: the pyramid's
algorithmic bytes (the roofline numerator: 1 B per input pixel + 44 B per octave pixel, 5 DoG
planes and 3 gradient magnitude / angle pairs of float32), on the bench image and the smaller
configuration, with the octave count of the reference's _pyramid (gsift.py:158-179)."""
import pytest


def _octave_pixels(h, w):
    import math
    n = max(1, int(round(math.log2(min(h, w)) - 2)) + 1)
    R, C, tot = 2 * h, 2 * w, 0
    for _ in range(n):
        if min(R, C) < 14:
            break
        tot += R * C
        R, C = (R + 1) // 2, (C + 1) // 2
    return tot


@pytest.mark.parametrize("h, w, octave_px", [(1978, 2640, 27.85e6), (989, 1320, 6.96e6)])
def test_pyramid_algorithmic_bytes(h, w, octave_px):
    import bench
    px = _octave_pixels(h, w)
    assert px == pytest.approx(octave_px, rel=2e-3)
    assert bench.pyramid_bytes(h, w) == h * w + 44 * px


def test_bench_image_figure():
    import bench
    assert bench.pyramid_bytes(1978, 2640) == pytest.approx(1.23e9, rel=1e-3)
