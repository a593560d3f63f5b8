"""Multi-GPU synthesis: time steps sharded over ranks, one image reduction per run.

Time steps are independent until the image sum, so each rank (one process per GPU)
runs the batched pipeline on its own contiguous block of steps and the level images
are summed once (NCCL over NVLink on GPUs, gloo on CPU), then normalised by the total
number of steps. This is the reference's MPI scheme (sample split
src/image_synthesis.cpp:75-80, MPI_Reduce(SUM) of the float images :140-147,
normalisation :336-347) with torch.distributed as the transport. There is no
per-step collective.
"""
from __future__ import annotations

from typing import Tuple

import numpy as np


def sample_split(n_total: int, rank: int, size: int) -> Tuple[int, int]:
    """(begin, count) of the contiguous block of steps of `rank`: ceil(n/size) steps per
    rank, the last ranks possibly fewer or none (src/image_synthesis.cpp:77-80)."""
    per = (n_total + size - 1) // size
    begin = rank * per
    count = min(per, max(n_total - begin, 0))
    return min(begin, n_total), count


def reduce_images(images, dst: int = 0, group=None):
    """Sum a rank's level images (torch tensor [L, P], float32) into rank `dst`."""
    import torch.distributed as dist

    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.reduce(images, dst=dst, op=dist.ReduceOp.SUM, group=group)
    return images


def distributed_synthesis(pipeline, s, xyz, wl, n_total: int, rank: int, size: int, group=None,
                          normalize: bool = True):
    """Run `pipeline` (a bipp_b200.Pipeline) on this rank's block of the steps given by
    s [T, N, N], xyz [T, N, 3], wl [T] (host arrays of all steps; only the block is
    used) and return the reduced images on rank 0 (None elsewhere)."""
    import torch

    begin, count = sample_split(n_total, rank, size)
    if count:
        pipeline.process(s[begin:begin + count], xyz[begin:begin + count], wl[begin:begin + count])
    img = torch.from_numpy(pipeline.images(normalize=False).copy())
    if torch.distributed.is_initialized() and torch.distributed.get_backend(group) == "nccl":
        img = img.cuda()
    reduce_images(img, dst=0, group=group)
    if rank != 0:
        return None
    out = img.cpu().numpy().astype(np.float64)
    if normalize and n_total:
        out /= n_total
    return out
