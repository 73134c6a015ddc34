"""Frame-sharded orchestration (fuse_sharded) on world_size 2 over gloo, on
CPU: a stand-in stack with the library's phase interface (pass-1 weight sum
and union, pass-2 accumulators normalised by the global weight sum, collapse)
must give, split over two ranks, what one stack over all frames gives."""
import os
import socket

import numpy as np
import pytest

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from __graft_entry__ import load_package

fsb = load_package()

W, H, P, F = 13, 9, 16, 7  # valid width, height, pitch, frames


def frame(k):
    rng = np.random.default_rng(100 + k)
    img = rng.uniform(0, 255, (H, W)).astype(np.float32)
    w = rng.uniform(0, 1, (H, W)).astype(np.float32) * (rng.uniform(0, 1, (H, W)) > 0.2)
    return img, w.astype(np.float32)


class FakeStack:
    """Phase interface of PyramidContrastStack over CPU tensors: the weight
    sum and union of its frames, acc = sum_k img_k * w_k / global weight sum
    (1/N where it is 0), collapse = rounded acc."""

    def __init__(self, frames):
        self.frames = frames
        self.out_width, self.out_height = W, H
        self.norm = torch.zeros((H, P), dtype=torch.float32)
        self.uni = torch.zeros((H, P), dtype=torch.uint8)
        self.acc = [torch.zeros((3, H, P), dtype=torch.float32) for _ in range(fsb.sharded.level_count(W, H))]
        self.total = len(frames)

    def set_frame_total(self, n):
        self.total = n

    def end_pass1(self):
        for _, w in self.frames:
            self.norm[:, :W] += torch.from_numpy(w)
            self.uni[:, :W] = torch.maximum(self.uni[:, :W], torch.from_numpy((w > 0).astype(np.uint8)))

    def buffer(self, which, level=0):
        return {fsb.BUFFER_WEIGHT_SUM: self.norm, fsb.BUFFER_UNION: self.uni}.get(which, self.acc[level])

    def blend(self):
        nv = self.norm[:, :W]
        for img, w in self.frames:
            m = torch.where(nv > 1e-12, torch.from_numpy(w) / nv, torch.full_like(nv, 1.0 / self.total))
            for c in range(3):
                self.acc[0][c, :, :W] += torch.from_numpy(img) * m * self.uni[:, :W]
        for lvl in range(1, len(self.acc)):
            self.acc[lvl][:, 0, 0] += float(len(self.frames))  # frame count summed over shards

    def collapse(self):
        return np.rint(self.acc[0][:, :, :W].numpy()), self.acc[-1][:, 0, 0].numpy().copy()


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b, e = fsb.sharded.shard_range(F, world, rank)
    st = FakeStack([frame(k) for k in range(b, e)])
    out = fsb.sharded.fuse_sharded(st, F, dist, as_tensor=lambda x: x)
    q.put((rank, out))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_ranges_cover_the_stack():
    for n in (1, 2, 7, 30, 143):
        for world in (1, 2, 3, 8):
            r = [fsb.sharded.shard_range(n, world, k) for k in range(world)]
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [e - b for b, e in r]
            assert max(sizes) - min(sizes) <= 1


def test_two_ranks_match_one_stack():
    single = FakeStack([frame(k) for k in range(F)])
    single.end_pass1()
    single.blend()
    want, want_count = single.collapse()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[1] is None
    out, count = got[0]
    assert np.abs(out - want).max() <= 1e-3
    assert np.array_equal(count, want_count)  # every shard's contribution reached the root
