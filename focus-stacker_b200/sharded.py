"""Frame-sharded fusion of one stack over several GPUs, one process per GPU.

Each rank fuses a contiguous shard of the stack's frames (frame order kept
across ranks) in its own stack.  Pass 1 gives each rank the weight sum and
the union support of its shard; those are summed and maxed over all ranks in
place (all-reduce), so that every rank normalises its masks by the weight
sum of the whole stack.  Pass 2 then blends each shard into that rank's
accumulator pyramid; the pyramids are summed onto the root rank (reduce),
which collapses them into the fused image.  Two exchanges per stack, plain
collectives (NCCL between GPUs; anything with the torch.distributed
interface works, gloo included).

The sums over ranks change the order of FP32 additions against a single
stack, so results agree to rounding, not bit for bit; remap and alpha are
per frame and do not change.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

from . import api


def shard_range(frames: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous frames [begin, end) of `rank` (earlier ranks get the
    remainder, one frame each)."""
    base, extra = divmod(frames, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def level_count(w: int, h: int) -> int:
    """Pyramid depth of a w x h level 0 (src/fuse/pyramid.zig:163-176)."""
    n = 1
    while w > 1 or h > 1:
        w = (w + 1) // 2 if w > 1 else 1
        h = (h + 1) // 2 if h > 1 else 1
        n += 1
    return n


def fuse_sharded(stack, frame_total: int, dist, as_tensor: Callable, group=None, root: int = 0,
                 sync: Optional[Callable[[], None]] = None, rank: Optional[int] = None):
    """Finish a stack that holds this rank's shard (all its frames added):
    pass 1, the weight-sum / union all-reduce, pass 2, the accumulator reduce
    onto `root`, and the collapse there.  `as_tensor` turns the stack's device
    buffers into tensors the collectives take (torch.as_tensor for CUDA
    buffers); `sync` waits for the collectives before the library reads their
    results (torch.cuda.synchronize on GPUs).  Returns the fused image on the
    root rank, None elsewhere."""
    rank = dist.get_rank(group) if rank is None else rank
    stack.set_frame_total(frame_total)
    stack.end_pass1()
    norm = as_tensor(stack.buffer(api.BUFFER_WEIGHT_SUM))
    uni = as_tensor(stack.buffer(api.BUFFER_UNION))
    dist.all_reduce(norm, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(uni, op=dist.ReduceOp.MAX, group=group)
    if sync:
        sync()
    stack.blend()
    for level in range(level_count(stack.out_width, stack.out_height)):
        acc = as_tensor(stack.buffer(api.BUFFER_ACCUMULATOR, level))
        dist.reduce(acc, dst=root, op=dist.ReduceOp.SUM, group=group)
    if sync:
        sync()
    return stack.collapse() if rank == root else None
