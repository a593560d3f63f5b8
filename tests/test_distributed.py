"""CPU, world_size 2 over gloo: step sharding and the single image reduction reproduce
the single-process result (the reference's MPI split + MPI_Reduce semantics,
src/image_synthesis.cpp:75-80, 140-163). The per-rank synthesis is stood in for by the
FP64 oracle so that the host logic is tested without a GPU."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from bipp_b200.distributed import reduce_images, sample_split


def test_sample_split_matches_reference_rule():
    for n in (0, 1, 5, 16, 17, 2048):
        for size in (1, 2, 3, 4, 8):
            blocks = [sample_split(n, r, size) for r in range(size)]
            covered = []
            for b, c in blocks:
                covered += list(range(b, b + c))
            assert covered == list(range(n))
            per = (n + size - 1) // size
            assert all(c <= per for _, c in blocks)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, size, port, steps, lmn, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    from oracle import bluebild as bb

    begin, count = sample_split(len(steps), rank, size)
    img = np.zeros((lmn.shape[0], 1))
    if count:
        img = bb.image_synthesis(steps[begin:begin + count], np.array([[0.0, np.inf]]), lmn, normalize=False)
    t = torch.from_numpy(img.T.astype(np.float32).copy())
    reduce_images(t, dst=0)
    if rank == 0:
        out_q.put(t.numpy() / len(steps))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("size", [2])
def test_gloo_sharded_synthesis_equals_single_process(size):
    from bipp_b200 import simulate as sim
    from oracle import bluebild as bb

    cfg = sim.config_c1(n_antenna=12, n_steps=5, image_size=8)
    obs = sim.observation(cfg)
    s, xyz = sim.visibilities(obs, list(range(5)))
    steps = []
    for k in range(5):
        v, d, nr, sc = bb.eigh_gram(cfg.wl, s[k].numpy(), np.eye(12), xyz[k].numpy())
        steps.append(dict(uvw=sim.baseline_uvw(obs, xyz[k].numpy()), v=v, d=d, scale=sc, wl=cfg.wl))
    full = bb.image_synthesis(steps, np.array([[0.0, np.inf]]), obs.lmn).T
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, size, port, steps, obs.lmn, q)) for r in range(size)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert np.abs(got - full).max() <= 1e-5 * np.abs(full).max()


def _levels_worker(rank, size, port, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    import bench

    # each rank calibrated its own levels; all must use rank 0's
    mine = np.array([[0.0, 1.0 + rank], [1.0 + rank, np.inf]])
    shared = bench.share_levels(mine, torch.device("cpu"))
    out_q.put((rank, shared))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_bench_levels_are_rank0s():
    """bench.py on N GPUs: every rank images with rank 0's energy levels (inf included)."""
    size = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_levels_worker, args=(r, size, port, q)) for r in range(size)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(size)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for _, lv in got:
        assert np.array_equal(lv, np.array([[0.0, 1.0], [1.0, np.inf]]))
