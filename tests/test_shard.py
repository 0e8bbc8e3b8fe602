"""Sharding by source image over ranks (fieldstitch_b200.shard): the plan, and the driver loop end to
end on two gloo ranks on CPU (spawned processes). Each rank extracts only the images it owns,
receives the features of the other images its pairs need, and matches its pairs; the union of the
ranks' match lists equals a single-rank run, and every image is extracted exactly once. The
"extraction" and the matcher here are CPU stand-ins (seeded feature sets, the oracle's exhaustive
ratio matcher), so the test exercises the host logic and the exchange, not the kernels."""
import socket

import numpy as np

from fieldstitch_b200 import shard, synth


def _pairs():
    poses = synth.lawnmower(3, lines=4, per_line=6)
    return synth.gnss_pairs(poses, sigma=15.0, seed=2), len(poses)


def _extract(i):
    """Seeded features of image i: 300 keypoints whose descriptors overlap image i+1's (shared pool)."""
    pool, _, _ = synth.synth_descriptors(24 * 100 + 400, 1, 77)
    rng = np.random.default_rng(1000 + i)
    desc = pool[100 * i:100 * i + 300].copy()
    jit = rng.integers(-2, 3, desc.shape)
    desc = np.clip(desc.astype(np.int32) + jit, 0, 255).astype(np.uint8)
    xy = rng.uniform(0, 1000, (300, 2)).astype(np.float32)
    resp = np.sort(rng.uniform(0, 1, 300).astype(np.float32))[::-1].copy()
    return shard.pack(xy, resp, desc)


def _match(k, A, B):
    from oracle import matching_ref
    q, t = matching_ref.ratio_match_bf(A[2].astype(np.float32), B[2].astype(np.float32), 0.8)
    return np.asarray(q).tolist(), np.asarray(t).tolist()


def test_plan_assigns_every_pair_once_and_balances():
    pairs, n = _pairs()
    for world in (1, 2, 3, 5):
        p = shard.plan(pairs, n, world)
        got = sorted(k for r in range(world) for k in p["pairs_of"][r])
        assert got == list(range(len(pairs)))
        assert sorted(i for r in range(world) for i in p["own"][r]) == list(range(n))
        for r in range(world):
            for k in p["pairs_of"][r]:
                i, j = pairs[k]
                assert p["owner"][i] == r and (p["owner"][j] == r or j in p["need"][r])
            # what r receives is exactly what the owners send to r
            assert sorted(j for s in range(world) for j, d in p["send"][s] if d == r) == p["need"][r]
        # contiguous image ranges: a rank exceeds the even share by at most one image's pairs
        counts = [len(p["pairs_of"][r]) for r in range(world)]
        heaviest = max(np.bincount([i for i, _ in pairs], minlength=n))
        assert max(counts) <= len(pairs) / world + heaviest + 1, counts


def test_pack_roundtrip():
    buf = _extract(3)
    xy, resp, desc = shard.unpack(buf)
    assert xy.shape == (300, 2) and resp.shape == (300,) and desc.shape == (300, 128)
    np.testing.assert_array_equal(shard.pack(xy, resp, desc), buf)
    e = shard.unpack(shard.pack(np.zeros((0, 2)), np.zeros(0), np.zeros((0, 128), np.uint8)))
    assert e[0].shape == (0, 2) and e[2].shape == (0, 128)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        pairs, n = _pairs()
        extracted = []

        def extract(i):
            extracted.append(i)
            return _extract(i)

        out = shard.run(pairs, n, extract, _match, rank=rank, world=world)
        q.put((rank, extracted, out))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_sharded_run_on_two_gloo_ranks_equals_one_rank():
    import torch.multiprocessing as mp
    pairs, n = _pairs()
    single = shard.run(pairs, n, _extract, _match)
    assert sorted(single) == list(range(len(pairs)))
    assert sum(len(v[0]) for v in single.values()) > 0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted((q.get(timeout=240) for _ in range(2)), key=lambda r: r[0])
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    # every image extracted exactly once over the two ranks
    assert sorted(res[0][1] + res[1][1]) == list(range(n))
    merged = {}
    for _, _, out in res:
        assert not set(out) & set(merged)
        merged.update(out)
    assert merged == single
    # the ranks really share images (the exchange was exercised)
    p = shard.plan(pairs, n, 2)
    assert p["need"][0] or p["need"][1]
