"""The device pyramid (DoG, gradient magnitude and angle atlases) against the oracle's, octave by
octave. With FSB_SIFT_EXACT_BLUR the DoG and magnitude atlases are bit-identical to the
reference's NumPy/SciPy path; the float32 FMA path (fused streaming kernel for wide octaves,
per-layer kernels for narrow ones) stays within a few float32 ulps."""
import numpy as np
import pytest

from sift_compare import paired_fraction

pytestmark = pytest.mark.gpu

SIZES = [(240, 320, 11), (495, 660, 77), (989, 1320, 5)]


@pytest.fixture(scope="module")
def oracle_pyr():
    from fieldstitch_b200 import synth
    from oracle import gsift_ref
    out = {}
    for h, w, seed in SIZES:
        img = synth.synth_image(h, w, seed)
        octs = gsift_ref.build_pyramid(img)
        out[(h, w)] = (img, [o["dog"] for o in octs], [gsift_ref.gradients(o) for o in octs])
    return out


def _ang_diff(a, b):
    d = np.abs(a.astype(np.float64) - b.astype(np.float64)) % 360.0
    return np.minimum(d, 360.0 - d)


@pytest.mark.parametrize("hw", [(h, w) for h, w, _ in SIZES])
def test_atlas_exact_is_bit_identical(oracle_pyr, hw):
    import fieldstitch_b200 as f
    img, dogs, grads = oracle_pyr[hw]
    _, st = f.gsift.detect(img, exact=True)
    shapes, dog, mag, ang = st.atlas()
    assert shapes == [d.shape[1:] for d in dogs]
    for o in range(len(shapes)):
        np.testing.assert_array_equal(dog[o], dogs[o], err_msg="DoG octave %d" % o)
        np.testing.assert_array_equal(mag[o], grads[o][0], err_msg="magnitude octave %d" % o)
        assert _ang_diff(ang[o], grads[o][1]).max() < 1e-3


@pytest.mark.parametrize("hw", [(h, w) for h, w, _ in SIZES])
def test_atlas_fast_within_ulps(oracle_pyr, hw):
    import fieldstitch_b200 as f
    img, dogs, grads = oracle_pyr[hw]
    _, st = f.gsift.detect(img)
    shapes, dog, mag, ang = st.atlas()
    for o in range(len(shapes)):
        ddog = np.abs(dog[o] - dogs[o])
        assert ddog.max() < 2e-6, (o, ddog.max())
        assert ddog.mean() < 1e-7, (o, ddog.mean())
        assert np.abs(mag[o] - grads[o][0]).max() < 4e-6
        # the angle error scales like (float32 error of dx, dy) / magnitude
        for floor, tol in ((1e-3, 0.05), (1e-2, 0.01)):
            strong = grads[o][0] > floor
            assert _ang_diff(ang[o][strong], grads[o][1][strong]).max() < tol, (o, floor)


def test_detect_fast_wide_image_matches_oracle():
    """1320 x 989 (config-1 size; octave 0 is 2640 wide and takes the fused kernel)."""
    import fieldstitch_b200 as f
    from fieldstitch_b200 import synth
    from oracle import gsift_ref
    img = synth.synth_image(989, 1320, 5)
    ref, _ = gsift_ref.detect(img, max_kp=100000, contrast=0.04, edge=10.0)
    got, _ = f.gsift.detect(img, max_kp=100000, contrast=0.04, edge=10.0)
    frac, _ = paired_fraction(ref, got)
    assert frac >= 0.97, frac
    back, _ = paired_fraction(got, ref)
    assert back >= 0.97, back


def test_autotuned_tile_heights_are_bit_identical(monkeypatch):
    """The per-layer kernel's tile heights (16, 32, 64) compute the same values: a pyramid whose
    launches the autotuner times and picks equals the untuned one bit for bit, and the tuner
    records one choice per (layer, octave size)."""
    import fieldstitch_b200 as f
    from fieldstitch_b200 import _lib, synth
    img = synth.synth_image(700, 900, 31)
    monkeypatch.setenv("FSB_PYRAMID", "layer")
    monkeypatch.setenv("FSB_AUTOTUNE", "0")
    _, st0 = f.gsift.detect(img)
    ref = st0.atlas()
    monkeypatch.delenv("FSB_AUTOTUNE")
    _, st1 = f.gsift.detect(img)   # first call with this geometry: every variant runs
    got = st1.atlas()
    _, st2 = f.gsift.detect(img)   # cached choices
    again = st2.atlas()
    for o in range(len(ref[0])):
        for k in (1, 2, 3):
            np.testing.assert_array_equal(got[k][o], ref[k][o])
            np.testing.assert_array_equal(again[k][o], ref[k][o])
    table = _lib.autotune_table()
    assert any("k_layer5_1400x1800" in k for k in table), table
    assert all(v in (0, 1, 2) for v in table.values())


@pytest.mark.parametrize("engine", ["group", "strip"])
@pytest.mark.parametrize("hw", [(37, 53), (240, 320), (495, 661), (610, 830), (989, 1320), (1978, 2640),
                                (1001, 1111)])
def test_octave_engine_bit_identical_to_per_layer(monkeypatch, hw, engine):
    """The fused layer-group kernels (L1..L3 and L4, L5 per launch, halos recomputed in shared
    memory) and the strip engine (the whole octave in one launch, layers in shared-memory row
    rings, L0 rows by TMA where the row pitch allows) give the per-layer kernels' DoG, magnitude
    and angle atlases bit for bit, including odd and tiny octaves whose halos reflect more than
    once, (610 x 830) octaves whose atlas planes start off a 16-byte boundary and (1001 x 1111)
    octave widths that are not a multiple of four, and the same keypoints."""
    import fieldstitch_b200 as f
    from fieldstitch_b200 import synth
    h, w = hw
    img = synth.synth_image(h, w, 3 + h)
    monkeypatch.setenv("FSB_PYRAMID", "layer")
    k0, st0 = f.gsift.detect(img)
    ref = st0.atlas()
    monkeypatch.setenv("FSB_PYRAMID", engine)
    k1, st1 = f.gsift.detect(img)
    got = st1.atlas()
    assert got[0] == ref[0] and len(ref[0]) >= 3
    for o in range(len(ref[0])):
        for k, name in ((1, "dog"), (2, "mag"), (3, "ang")):
            np.testing.assert_array_equal(got[k][o], ref[k][o], err_msg="%s octave %d" % (name, o))
    for key in ("x", "y", "size", "angle", "response"):
        np.testing.assert_array_equal(k1[key], k0[key])


def test_autotuned_octave_engines_are_bit_identical(monkeypatch):
    """With no engine forced, the autotuner times the per-layer kernels, the fused layer groups and
    the strip engine per octave size and keeps the fastest; the atlases (first call, tuning; second call, cached
    choices) equal the untuned per-layer ones bit for bit, and each octave size has a choice."""
    import fieldstitch_b200 as f
    from fieldstitch_b200 import _lib, synth
    img = synth.synth_image(610, 830, 41)
    monkeypatch.setenv("FSB_PYRAMID", "layer")
    monkeypatch.setenv("FSB_AUTOTUNE", "0")
    _, st0 = f.gsift.detect(img)
    ref = st0.atlas()
    monkeypatch.delenv("FSB_PYRAMID")
    monkeypatch.delenv("FSB_AUTOTUNE")
    for _ in range(2):
        _, st = f.gsift.detect(img)
        got = st.atlas()
        for o in range(len(ref[0])):
            for k in (1, 2, 3):
                np.testing.assert_array_equal(got[k][o], ref[k][o])
    table = _lib.autotune_table()
    for r, c in ref[0]:
        assert any(k.endswith("k_octave3_%dx%d" % (r, c)) for k in table), (r, c, table)


@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("hw", [(37, 53), (240, 320), (610, 830), (1001, 1111), (1978, 2640)])
def test_layer_tile_height_variants_bit_identical(monkeypatch, hw, variant):
    """Each tile height of the per-layer kernel, forced for every layer (16 and 64 rows against
    32), gives the same DoG, magnitude and angle atlases bit for bit - interior tiles by tensor
    copy, border tiles by cp.async with reflected rows and columns - on tiny octaves, planes off a
    16-byte boundary and widths that are not a multiple of four, and the same keypoints."""
    import fieldstitch_b200 as f
    from fieldstitch_b200 import synth
    h, w = hw
    img = synth.synth_image(h, w, 11 + w)
    monkeypatch.setenv("FSB_PYRAMID", "layer")
    monkeypatch.setenv("FSB_LAYER_VARIANT", "0")
    k0, st0 = f.gsift.detect(img)
    ref = st0.atlas()
    monkeypatch.setenv("FSB_LAYER_VARIANT", str(variant))
    k1, st1 = f.gsift.detect(img)
    got = st1.atlas()
    assert got[0] == ref[0]
    for o in range(len(ref[0])):
        for k, name in ((1, "dog"), (2, "mag"), (3, "ang")):
            np.testing.assert_array_equal(got[k][o], ref[k][o], err_msg="%s octave %d" % (name, o))
    for key in ("x", "y", "size", "angle", "response"):
        np.testing.assert_array_equal(k1[key], k0[key])
