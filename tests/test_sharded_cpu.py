"""Frame-sharded orchestration (fuse_sharded) on world_size 2 over gloo, on
CPU.  Each rank holds an oracle-backed stack with the library's phase
interface: pass 1 gives the shard's weight sum and union (the oracle's
weight maps), pass 2 blends the shard's frames into an FP32 accumulator
pyramid with masks normalised by the weight sum of the whole stack (the
oracle's accumulateImage), and the root collapses the summed pyramids.  Split
over two ranks, the fused image must be the oracle's fusion of all frames in
one stack, to the rounding that the changed order of FP32 sums allows."""
import os
import socket

import numpy as np
import pytest

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from __graft_entry__ import load_package

fsb = load_package()

W, H, F = 96, 64, 7  # aligned frame size, frames


def aligned_frames():
    """Aligned RGBA frames: the oracle's remap of a small synthetic stack."""
    poses = [oracle.synth_pose(5, oracle.SCENE_SMALL, 120, 90, k, F) for k in range(F)]
    frames = [oracle.synth_frame(5, oracle.SCENE_SMALL, 120, 90, k, F) for k in range(F)]
    return [oracle.remap(f, p, (10, 12, 10 + W, 12 + H)) for f, p in zip(frames, poses)]


class OracleShardStack:
    """The phase interface of PyramidContrastStack (end_pass1, buffer, blend,
    collapse) over the oracle's stages, for a shard of a stack's frames."""

    def __init__(self, frames):
        self.frames = frames
        self.out_width, self.out_height = W, H
        self.total = len(frames)
        self.norm = torch.zeros((H, W), dtype=torch.float32)
        self.uni = torch.zeros((H, W), dtype=torch.uint8)
        self.acc = torch.zeros(oracle.pyramid_floats(W, H), dtype=torch.float32)
        self.weights = []
        self.levels = []
        w, h, off = W, H, 0
        for _ in range(fsb.sharded.level_count(W, H)):
            self.levels.append(self.acc[off:off + w * h * 3])
            off += w * h * 3
            w, h = oracle.next_level_size(w), oracle.next_level_size(h)

    def set_frame_total(self, n):
        self.total = n

    def end_pass1(self):
        for f in self.frames:
            w = oracle.weight_map(f)
            self.weights.append(w)
            self.norm += torch.from_numpy(w)
            self.uni = torch.maximum(self.uni, torch.from_numpy((f[..., 3] > 0).astype(np.uint8)))

    def buffer(self, which, level=0):
        if which == fsb.BUFFER_WEIGHT_SUM:
            return self.norm
        if which == fsb.BUFFER_UNION:
            return self.uni
        return self.levels[level]

    def blend(self):
        norm = self.norm.numpy()
        uni = self.uni.numpy().astype(np.float32)
        acc = self.acc.numpy()  # shares memory with the tensor the collectives use
        for f, w in zip(self.frames, self.weights):
            m = oracle.normalize_weights(w, norm, self.total)
            oracle.pyramid_accumulate(f, m, uni, acc)

    def collapse(self):
        return oracle.pyramid_collapse(self.acc.numpy(), W, H)


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    b, e = fsb.sharded.shard_range(F, world, rank)
    st = OracleShardStack(aligned_frames()[b:e])
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


def test_oracle_shard_stack_alone_is_the_oracle_fusion():
    frames = aligned_frames()
    st = OracleShardStack(frames)
    st.end_pass1()
    st.blend()
    out, base = st.collapse()
    ref, ref_base = oracle.fuse_aligned(frames, want_base=True)
    assert np.array_equal(out, ref) and np.array_equal(base, ref_base)


def test_two_ranks_match_one_stack():
    frames = aligned_frames()
    want, want_base = oracle.fuse_aligned(frames, want_base=True)
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
    out, base = got[0]
    assert np.abs(base - want_base).max() <= 1e-3
    assert np.abs(out.astype(np.int16) - want.astype(np.int16)).max() <= 1
