"""Batched guided matching (one set of launches for all pairs, issued as a CUDA graph) through the
C ABI: every pair's match list is identical to the per-pair guided matcher's, on the first call
(capture), on replays, after the data behind the same pointers change (replay reads the new data)
and after the pair table changes (new capture)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H = 1320.0, 989.0


def _problem(na, nb, seed):
    from fieldstitch_b200 import synth
    rng = np.random.default_rng(seed)
    a, b, truth = synth.synth_descriptors(max(na, 1), max(nb, 1), seed)
    a, b, truth = a[:na], b[:nb], truth[:nb]
    bxy = np.c_[rng.uniform(0, W, nb), rng.uniform(0, H, nb)]
    pred = np.c_[rng.uniform(-50, W + 50, na), rng.uniform(-50, H + 50, na)]
    for j in np.flatnonzero((truth >= 0) & (truth < na)):
        pred[truth[j]] = bxy[j] + rng.normal(0, 10, 2)
    return pred, a, bxy, b


def _dev(torch, p):
    pred, a, bxy, b = p
    return (torch.from_numpy(np.ascontiguousarray(pred)).cuda(), torch.from_numpy(np.ascontiguousarray(a)).cuda(),
            torch.from_numpy(np.ascontiguousarray(bxy)).cuda(), torch.from_numpy(np.ascontiguousarray(b)).cuda(),
            (W, H))


def _check(m, probs, got, kc):
    for (pred, a, bxy, b), (q, t) in zip(probs, got):
        if len(a) == 0 or len(b) == 0:
            assert len(q) == 0
            continue
        q2, t2 = m.guided_from_pred(pred, a, bxy, b, (W, H), 40.0, kc, 0.85)
        np.testing.assert_array_equal(q.cpu().numpy(), q2)
        np.testing.assert_array_equal(t.cpu().numpy(), t2)


@pytest.mark.parametrize("kc", [16, None])
def test_batch_equals_per_pair(kc):
    import torch

    import fieldstitch_b200 as F
    m = F.matching
    sizes = [(2000, 1500), (300, 4000), (0, 50), (40, 0), (1, 1), (5000, 5000), (777, 333)]
    probs = [_problem(na, nb, 10 + i) for i, (na, nb) in enumerate(sizes)]
    dev = [_dev(torch, p) for p in probs]
    out = [(torch.empty(max(len(p[1]), 1), dtype=torch.int64, device="cuda"),
            torch.empty(max(len(p[1]), 1), dtype=torch.int64, device="cuda")) for p in probs]
    for _ in range(2):   # capture, then replay
        _check(m, probs, m.guided_from_pred_batch_d(dev, 40.0, kc, 0.85, out=out), kc)
    # new data behind the same pointers: the replayed graph reads it
    p0 = _problem(2000, 1500, 99)
    dev[0][0].copy_(torch.from_numpy(p0[0]))
    dev[0][1].copy_(torch.from_numpy(p0[1]))
    probs[0] = (p0[0], p0[1], probs[0][2], probs[0][3])
    _check(m, probs, m.guided_from_pred_batch_d(dev, 40.0, kc, 0.85, out=out), kc)
    # a different table (one pair fewer): a new capture
    _check(m, probs[1:], m.guided_from_pred_batch_d(dev[1:], 40.0, kc, 0.85, out=out[1:]), kc)


@pytest.mark.parametrize("kc", [16, None])
def test_host_batch_entry_equals_per_pair(kc):
    """matching.match_guided_batch (host arrays in and out) returns each pair's guided_from_pred
    result, with float32 RootSIFT-valued descriptors accepted like the per-pair call."""
    import fieldstitch_b200 as F
    m = F.matching
    sizes = [(900, 700), (0, 30), (50, 0), (3000, 2500)]
    probs = [_problem(na, nb, 40 + i) for i, (na, nb) in enumerate(sizes)]
    got = m.match_guided_batch([(p, a.astype(np.float32), bxy, b, (W, H)) for p, a, bxy, b in probs], 40.0, kc,
                               0.85)
    for (pred, a, bxy, b), (q, t) in zip(probs, got):
        if len(a) == 0 or len(b) == 0:
            assert len(q) == 0
            continue
        q2, t2 = m.guided_from_pred(pred, a, bxy, b, (W, H), 40.0, kc, 0.85)
        np.testing.assert_array_equal(q, q2)
        np.testing.assert_array_equal(t, t2)
