"""Sharding the feature front end over ranks (one process per GPU) by source image.

The reference parallelises over independent units with process pools: photos through a spawn
queue (app/planesite/pipeline.py:922-931), pairs through ``pool.imap(match_pair, pairs)``
(pipeline.py:535-536). Across GPUs the same independence holds, with one twist: a pair needs the
features of both of its images, and extracting an image twice on two GPUs wastes the dominant
stage. So:

* ``plan(pairs, n_images, world)`` gives every image one owner rank (contiguous runs of images in
  flight order, balanced by the number of pairs they start) and every pair the owner of its first
  image. A rank extracts only the images it owns; for each pair whose second image another rank
  owns, that image's features are sent by the owner once per receiving rank.
* ``exchange(plan, rank, feats, group)`` moves those features point to point (torch.distributed
  isend / irecv; NCCL over NVLink on GPUs, gloo on CPU), after every rank has extracted its own
  images: one exchange step per job, no per-step collective.
* ``run(...)`` is the driver loop of one rank: extract the owned images, exchange, match the
  assigned pairs; the union of the ranks' results is the single-rank result.

Features travel as one flat uint8 buffer per image (keypoint count, float32 coordinates and
responses, uint8 RootSIFT rows), so the exchange is a byte copy and needs no type handling.
"""
import numpy as np


def plan(pairs, n_images, world):
    """Shard plan for `pairs` (sorted (i, j), i < j) over `world` ranks.

    Returns a dict: owner (n_images,) int rank of each image; pairs_of[r] the indices of the pairs
    rank r matches; own[r] the images rank r extracts; need[r] the images rank r receives (owned
    elsewhere); send[r] a list of (image, destination rank) rank r sends, in a fixed order."""
    pairs = [(int(i), int(j)) for i, j in pairs]
    world = max(1, int(world))
    starts = np.zeros(n_images, np.int64)
    for i, _ in pairs:
        starts[i] += 1
    # contiguous image ranges with about equal pair counts (each image weighted by 1 + its pairs,
    # so that images without pairs still spread the extraction)
    w = starts + 1
    cum = np.cumsum(w)
    total = cum[-1] if n_images else 0
    owner = np.minimum((world * (cum - w)) // max(total, 1), world - 1).astype(np.int64) if n_images else \
        np.zeros(0, np.int64)
    pairs_of = [[] for _ in range(world)]
    need = [set() for _ in range(world)]
    for k, (i, j) in enumerate(pairs):
        r = int(owner[i])
        pairs_of[r].append(k)
        if owner[j] != r:
            need[r].add(j)
    own = [np.flatnonzero(owner == r).tolist() for r in range(world)]
    send = [[] for _ in range(world)]
    for r in range(world):
        for j in sorted(need[r]):
            send[int(owner[j])].append((j, r))
    for r in range(world):
        send[r].sort()
    return {"owner": owner, "pairs_of": pairs_of, "own": own, "need": [sorted(s) for s in need], "send": send,
            "world": world}


def pack(xy, resp, desc):
    """One image's features as a flat uint8 array: int64 count, float32 xy (n,2), float32 resp (n,),
    uint8 desc (n,128)."""
    xy = np.ascontiguousarray(xy, np.float32).reshape(-1, 2)
    n = len(xy)
    head = np.array([n], np.int64).view(np.uint8)
    return np.concatenate([head, xy.view(np.uint8).ravel(),
                           np.ascontiguousarray(resp, np.float32).reshape(n).view(np.uint8),
                           np.ascontiguousarray(desc, np.uint8).reshape(n, 128).ravel()])


def unpack(buf):
    """Inverse of pack: (xy float32 (n,2), resp float32 (n,), desc uint8 (n,128))."""
    buf = np.asarray(buf, np.uint8)
    n = int(buf[:8].view(np.int64)[0])
    o = 8
    xy = buf[o:o + 8 * n].view(np.float32).reshape(n, 2)
    o += 8 * n
    resp = buf[o:o + 4 * n].view(np.float32)
    o += 4 * n
    desc = buf[o:o + 128 * n].reshape(n, 128)
    return xy, resp, desc


def exchange(p, rank, feats, group=None, device=None):
    """Sends the features of owned images other ranks need and receives those this rank needs.
    feats: {image: packed uint8 numpy array} of this rank's own images (extended in place with the
    received ones). Sizes go first (one int64 per transfer), then the bytes; every transfer is a
    matched isend / irecv, so the ranks need no common step count. device: a torch device for the
    transfer buffers (CUDA for NCCL), None for CPU (gloo)."""
    import torch
    import torch.distributed as dist
    dev = torch.device("cpu") if device is None else torch.device(device)
    recv_from = [(j, int(p["owner"][j])) for j in p["need"][rank]]
    ops, sizes = [], {}
    for j, dst in p["send"][rank]:
        ops.append(dist.P2POp(dist.isend, torch.tensor([len(feats[j])], dtype=torch.int64, device=dev), dst,
                              group=group))
    for j, src in recv_from:
        sizes[j] = torch.zeros(1, dtype=torch.int64, device=dev)
        ops.append(dist.P2POp(dist.irecv, sizes[j], src, group=group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    ops, bufs = [], {}
    for j, dst in p["send"][rank]:
        ops.append(dist.P2POp(dist.isend, torch.from_numpy(feats[j]).to(dev), dst, group=group))
    for j, src in recv_from:
        bufs[j] = torch.empty(int(sizes[j].item()), dtype=torch.uint8, device=dev)
        ops.append(dist.P2POp(dist.irecv, bufs[j], src, group=group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    for j, b in bufs.items():
        feats[j] = b.cpu().numpy()
    return feats


def run(pairs, n_images, extract, match, rank=0, world=1, group=None, device=None):
    """The driver loop of one rank: extract(i) -> packed features of image i for the owned images,
    exchange, then match(k, feats_i, feats_j) for the assigned pairs (feats as unpack returns).
    Returns {pair index: match result} of this rank's pairs."""
    p = plan(pairs, n_images, world)
    feats = {i: extract(i) for i in p["own"][rank]}
    if world > 1:
        exchange(p, rank, feats, group, device)
    out = {}
    for k in p["pairs_of"][rank]:
        i, j = pairs[k]
        out[k] = match(k, unpack(feats[i]), unpack(feats[j]))
    return out
