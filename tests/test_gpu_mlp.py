"""The learned match filter's kernels (through the C ABI) against the float64 oracle, GPU training,
the ratio-test fallback's parity with the plain guided matcher, and what the trained network gains
over the plain ratio test on held-out synthetic pairs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, 8)) * np.array([0.3, 0.5, 1.0, 0.4, 0.6, 0.02, 0.02, 2.0]) + 0.5
    y = ((x[:, 0] < 0.5) & (x[:, 4] < 0.7)).astype(np.float32)
    return x.astype(np.float32), y


@pytest.fixture(scope="module")
def mods():
    import torch

    import fieldstitch_b200 as F  # noqa: F401
    from fieldstitch_b200 import match_filter as MF
    from oracle import mlp_ref as M
    return torch, MF, M


def test_gradient_matches_oracle(mods):
    torch, MF, M = mods
    x, y = _data(1000, 1)
    p = M.init_params(x.mean(0), x.std(0), seed=2)
    mf = MF.MatchFilter(p)
    loss, g = mf.grad(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda())
    l_ref, g_ref = M.grad(p.astype(np.float64), x.astype(np.float64), y)
    assert abs(loss - l_ref) < 1e-5 * max(1.0, abs(l_ref))
    np.testing.assert_allclose(g.cpu().numpy(), g_ref, rtol=1e-3, atol=1e-5 * np.abs(g_ref).max())


def test_inference_fp32_and_bf16_match_oracle(mods):
    torch, MF, M = mods
    x, y = _data(5000, 3)
    p = M.init_params(x.mean(0), x.std(0), seed=4)
    mf = MF.MatchFilter(p)
    xt = torch.from_numpy(x).cuda()
    z, _ = M.forward(p.astype(np.float64), x.astype(np.float64))
    np.testing.assert_allclose(mf.predict(xt, bf16=False).cpu().numpy(), M.sigmoid(z), atol=2e-6)
    np.testing.assert_allclose(mf.predict(xt, bf16=True).cpu().numpy(), M.forward_bf16(p, x), atol=5e-3)


def test_first_adam_step_matches_oracle(mods):
    torch, MF, M = mods
    x, y = _data(512, 5)
    p = M.init_params(x.mean(0), x.std(0), seed=6)
    mf = MF.MatchFilter(p)
    lr = 1e-3
    mf.fit(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), epochs=1, batch=4096, lr=lr, seed=1)
    _, g = M.grad(p.astype(np.float64), x.astype(np.float64), y)
    p1, _, _ = M.adam(p.astype(np.float64), np.zeros(M.N_TRAIN), np.zeros(M.N_TRAIN), g, 1, lr)
    got = mf.params.cpu().numpy().astype(np.float64)
    sel = np.abs(g) > 1e-6   # Adam's first step is lr * sign(g) away from tiny gradients
    np.testing.assert_allclose(got[:M.N_TRAIN][sel], p1[:M.N_TRAIN][sel], rtol=0, atol=lr * 1e-3)
    np.testing.assert_array_equal(got[M.N_TRAIN:], p[M.N_TRAIN:])   # normalisation is not trained


def test_training_converges_and_is_deterministic(mods):
    torch, MF, M = mods
    x, y = _data(60000, 7)
    xt, yt = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    p0 = M.init_params(x.mean(0), x.std(0), seed=8)
    a, b = MF.MatchFilter(p0), MF.MatchFilter(p0)
    la = a.fit(xt, yt, epochs=8, batch=4096, lr=3e-3, seed=11)
    lb = b.fit(xt, yt, epochs=8, batch=4096, lr=3e-3, seed=11)
    assert la[-1] < 0.5 * la[0], la
    assert torch.equal(a.params, b.params)
    np.testing.assert_array_equal(la, lb)
    acc = ((a.predict(xt).cpu().numpy() > 0.5) == (y > 0.5)).mean()
    assert acc > 0.97, acc


@pytest.fixture(scope="module")
def one_pair(mods):
    torch, MF, M = mods
    from fieldstitch_b200 import synth
    a, b, H = synth.synth_pair(495, 660, 21)
    noise = synth.prior_noise(4000, 21)
    return a, b, H, noise


def test_features_match_numpy(mods, one_pair):
    torch, MF, M = mods
    a, b, H, noise = one_pair
    A = MF.extract(torch.from_numpy(a).cuda(), 1500)
    B = MF.extract(torch.from_numpy(b).cuda(), 1500)
    xa = A["xy"].cpu().numpy().astype(np.float64)
    src = np.c_[xa, np.ones(len(xa))] @ H.T
    pred = src[:, :2] / src[:, 2:3] + noise[:len(xa)]
    pt = torch.from_numpy(pred).cuda()
    t1, b12 = MF.candidates(pt, A, B, (660, 495), 40.0, 16)
    f = MF.features(t1, b12, pt, A, B, 40.0).cpu().numpy()
    t1h, bh = t1.cpu().numpy(), b12.cpu().numpy()
    ok = t1h >= 0
    assert ok.sum() > 100
    h = {k: v.cpu().numpy() for k, v in list(A.items())}
    g = {k: v.cpu().numpy() for k, v in list(B.items())}
    t = t1h[ok]
    b1, b2 = bh[ok, 0].astype(np.float64), bh[ok, 1].astype(np.float64)
    want = np.zeros((ok.sum(), 8))
    want[:, 0] = np.where(np.isinf(b2), 0.0, np.sqrt(b1) / np.sqrt(np.where(np.isinf(b2), 1.0, b2)))
    want[:, 1] = np.sqrt(b1) / 512.0
    want[:, 2] = np.log2(g["size"][t] / h["size"][ok])
    da = g["angle"][t].astype(np.float64) - h["angle"][ok]
    want[:, 3] = (da - 360.0 * np.floor((da + 180.0) / 360.0)) / 180.0
    want[:, 4] = np.linalg.norm(pred[ok] - g["xy"][t].astype(np.float64), axis=1) / 40.0
    want[:, 5] = h["resp"][ok]
    want[:, 6] = g["resp"][t]
    want[:, 7] = h["octave"][ok]
    np.testing.assert_allclose(f[ok], want, rtol=1e-5, atol=1e-5)
    assert np.all(f[~ok] == 0.0)


def test_fallback_equals_plain_guided_matcher(mods, one_pair):
    """Without a network the filter is the plain ratio test: identical to matching._guided."""
    torch, MF, M = mods
    import fieldstitch_b200 as F
    a, b, H, noise = one_pair
    A = MF.extract(torch.from_numpy(a).cuda(), 1500)
    B = MF.extract(torch.from_numpy(b).cuda(), 1500)
    xa = A["xy"].cpu().numpy().astype(np.float64)
    src = np.c_[xa, np.ones(len(xa))] @ H.T
    pred = src[:, :2] / src[:, 2:3] + noise[:len(xa)]
    t1, b12 = MF.candidates(torch.from_numpy(pred).cuda(), A, B, (660, 495), 40.0, 16)
    q, t = MF.MatchFilter().matches(t1, b12, len(B["xy"]), ratio=0.85)
    q2, t2 = F.matching.guided_from_pred(pred, A["u8"].cpu().numpy(), B["xy"].cpu().numpy().astype(np.float64),
                                         B["u8"].cpu().numpy(), (660, 495), 40.0, 16, 0.85)
    np.testing.assert_array_equal(q.cpu().numpy(), q2)
    np.testing.assert_array_equal(t.cpu().numpy(), t2)


def test_trained_filter_gains_over_ratio_test(mods):
    """Train on 24 synthetic pairs (labels from the plain pipeline's RANSAC verification), evaluate
    on 10 held-out pairs: the filter's F1 against the same verification beats the ratio test's."""
    torch, MF, M = mods
    from fieldstitch_b200 import synth
    sets = []
    for i in range(34):
        a, b, H = synth.synth_pair(989, 1320, 300 + i)
        sets.append(MF.label_pair(a, b, H, 4000, 4000, synth.prior_noise(4000, 300 + i), ratio=0.85))
    train, test = sets[:24], sets[24:]
    feat = torch.cat([s["feat"][torch.from_numpy(s["has_cand"]).cuda()] for s in train])
    lab = torch.cat([s["label"][torch.from_numpy(s["has_cand"]).cuda()] for s in train])
    mf = MF.MatchFilter()
    losses = mf.fit(feat, lab, epochs=30, batch=4096, lr=2e-3, seed=3)
    assert losses[-1] < losses[0]
    tp_p = n_p = tp_m = n_m = pos = 0.0
    for s in test:
        lab_h = s["label_host"]
        if lab_h.sum() == 0:
            continue
        qm, _ = mf.matches(s["t1"], s["b12"], s["nb"], s["feat"])
        qm = qm.cpu().numpy()
        pos += lab_h.sum()
        tp_p += lab_h[s["q_plain"]].sum()
        n_p += len(s["q_plain"])
        tp_m += lab_h[qm].sum()
        n_m += len(qm)
    f1 = lambda tp, n: 2 * tp / (n + pos)   # noqa: E731
    prec_p, rec_p, prec_m, rec_m = tp_p / n_p, tp_p / pos, tp_m / n_m, tp_m / pos
    print("plain P=%.4f R=%.4f F1=%.4f | filter P=%.4f R=%.4f F1=%.4f" % (prec_p, rec_p, f1(tp_p, n_p), prec_m,
                                                                          rec_m, f1(tp_m, n_m)))
    assert f1(tp_m, n_m) > f1(tp_p, n_p) + 0.01
