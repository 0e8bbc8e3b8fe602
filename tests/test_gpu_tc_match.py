"""The tcgen05 dense matcher (BF16 and E4M3 precisions) through the C ABI: match lists identical to
the reference fixtures, the oracle and the CUDA-core FP32 path (integer/index work, bit-exact bar),
for single pairs and for ragged batches in one persistent launch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRECS = ["bf16", "fp8"]


@pytest.fixture(scope="module")
def m():
    import fieldstitch_b200 as f
    f.context(0)
    return f.matching


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("case", ["bf_400x380", "bf_257x300", "bf_2x2"])
def test_tc_matches_reference_fixture(m, golden, case, prec):
    g = golden["match_ref"]
    q, t = m._ratio_match_bf(g[case + "/a"].astype(np.float32), g[case + "/b"].astype(np.float32),
                             float(g[case + "/ratio"]), precision=prec)
    np.testing.assert_array_equal(q, g[case + "/q"])
    np.testing.assert_array_equal(t, g[case + "/t"])


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("na,nb,seed,ratio", [(3000, 2500, 1, 0.8), (1000, 4097, 2, 0.85), (129, 131, 3, 0.7),
                                              (2, 5000, 4, 0.9), (5000, 2, 5, 0.8), (300, 33, 6, 0.8),
                                              (700, 64, 7, 0.95)])
def test_tc_matches_oracle(m, na, nb, seed, ratio, prec):
    from fieldstitch_b200 import synth
    from oracle import matching_ref
    a, b, _ = synth.synth_descriptors(na, nb, seed)
    q, t = m._ratio_match_bf(a, b, ratio, precision=prec)
    q2, t2 = matching_ref.ratio_match_bf(a.astype(np.float32), b.astype(np.float32), ratio)
    np.testing.assert_array_equal(q, q2)
    np.testing.assert_array_equal(t, t2)


@pytest.mark.parametrize("prec", PRECS)
def test_tc_ties_duplicates_and_zero_rows(m, prec):
    """Duplicate B rows tie the best distance (rejected by the ratio test); all-zero rows and
    rows at the uint8 maximum exercise the extremes of the norm slots and the E4M3 scale."""
    from oracle import matching_ref
    rng = np.random.default_rng(9)
    a = rng.integers(0, 40, (300, 128)).astype(np.uint8)
    a[5] = 0
    a[6] = 255
    b = np.concatenate([a[:100], a[:100], rng.integers(0, 40, (50, 128)).astype(np.uint8),
                        np.zeros((3, 128), np.uint8), np.full((2, 128), 255, np.uint8)])
    for ratio in (0.8, 0.99):
        q, t = m._ratio_match_bf(a, b, ratio, precision=prec)
        q2, t2 = matching_ref.ratio_match_bf(a.astype(np.float32), b.astype(np.float32), ratio)
        np.testing.assert_array_equal(q, q2)
        np.testing.assert_array_equal(t, t2)


def test_bf16_exact_distances_no_fallback(m):
    """BF16 products of uint8 values with FP32 accumulation are exact: the approximate best
    distance equals the exact one on every row and no row needs the exact fallback."""
    from fieldstitch_b200 import synth
    a, b, _ = synth.synth_descriptors(6000, 7000, 11)
    q, t = m._ratio_match_bf(a, b, 0.8, precision="bf16")
    st = m.tc_stats()
    assert st["rows"] == 6000
    assert st["fallback_rows"] == 0
    assert st["max_abs_err"] == 0.0
    q2, t2 = m._ratio_match_bf(a, b, 0.8, precision="fp32")
    np.testing.assert_array_equal(q, q2)
    np.testing.assert_array_equal(t, t2)


def test_fp8_large_equals_fp32(m):
    from fieldstitch_b200 import synth
    a, b, _ = synth.synth_descriptors(8192, 8192, 12)
    q, t = m._ratio_match_bf(a, b, 0.8, precision="fp8")
    st = m.tc_stats()
    assert st["rows"] == 8192
    assert st["max_abs_err"] > 0.0        # E4M3 rounding is visible in the approximate distances
    q2, t2 = m._ratio_match_bf(a, b, 0.8, precision="fp32")
    np.testing.assert_array_equal(q, q2)
    np.testing.assert_array_equal(t, t2)


@pytest.mark.parametrize("prec", PRECS)
def test_tc_batch_ragged_equals_single(m, prec):
    import torch
    from fieldstitch_b200 import synth
    sizes = [(2000, 16000), (16000, 2000), (257, 300), (2, 2), (1, 50), (4096, 4096), (513, 129)]
    A, B, ref = [], [], []
    for i, (na, nb) in enumerate(sizes):
        a, b, _ = synth.synth_descriptors(na, nb, 100 + i)
        A.append(torch.from_numpy(a).cuda())
        B.append(torch.from_numpy(b).cuda())
        ref.append(m._ratio_match_bf(a, b, 0.8, precision="fp32") if na >= 2 else (np.zeros(0), np.zeros(0)))
    out = m.ratio_match_bf_batch_d(A, B, 0.8, precision=prec)
    for (q, t), (q2, t2) in zip(out, ref):
        np.testing.assert_array_equal(q.cpu().numpy(), q2)
        np.testing.assert_array_equal(t.cpu().numpy(), t2)
