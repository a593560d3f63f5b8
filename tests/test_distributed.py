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


def test_split_selection_rules():
    """Checks over the whole selection before the split, then contiguous blocks of the
    id-sorted samples (src/image_synthesis.cpp:44-105)."""
    import bipp_b200 as bipp

    ev = np.ones(3, np.float32)
    sel = {"a": {7: ev, 2: 2 * ev, 5: 3 * ev, 0: 4 * ev, 9: 5 * ev}, "b": {0: ev, 2: ev, 5: ev, 7: ev, 9: ev}}
    blocks = [bipp.split_selection(sel, 10, r, 2) for r in range(2)]
    assert [sorted(b[0]["a"]) for b in blocks] == [[0, 2, 5], [7, 9]]
    assert all(b[1] == 5 for b in blocks)
    assert np.array_equal(blocks[1][0]["a"][7], ev) and np.array_equal(blocks[0][0]["a"][0], 4 * ev)
    assert [sorted(b[0]["b"]) for b in blocks] == [[0, 2, 5], [7, 9]]
    assert sorted(bipp.split_selection(sel, 10, 2, 3)[0]["a"]) == [9]
    assert sorted(bipp.split_selection(sel, 10, 3, 4)[0]["a"]) == []
    for bad, msg in (({"a": {0: ev, 12: ev}}, "exceeds"), ({"a": {0: ev, 1: ev}, "b": {0: ev, 2: ev}}, "same sample"),
                     ({"a": {}}, "Empty")):
        with pytest.raises(bipp.InvalidParameterError, match=msg):
            bipp.split_selection(bad, 10, 0, 2)


def test_communicator():
    import bipp_b200 as bipp

    assert (bipp.communicator.local().rank, bipp.communicator.local().size) == (0, 1)
    os.environ["RANK"], os.environ["WORLD_SIZE"] = "1", "3"
    try:
        w = bipp.communicator.world()
        assert (w.rank, w.size) == (1, 3)
    finally:
        del os.environ["RANK"], os.environ["WORLD_SIZE"]
    with pytest.raises(bipp.InvalidParameterError):
        bipp.communicator(2, 2)
    assert bipp.config.cuda and not bipp.config.mpi


def test_rank_device_choice():
    """Under a multi-rank communicator a rank's GPU is rank % device count, as the
    reference's context (src/context_internal.cpp:59-66); the image reduction runs on it."""
    from bipp_b200.api import pick_device

    import bipp_b200 as bipp

    for size, n_dev in ((2, 1), (4, 2), (8, 8), (3, 8)):
        for rank in range(size):
            assert pick_device(bipp.communicator(rank, size), n_dev) == rank % n_dev
    assert pick_device(bipp.communicator(1, 2), 0) is None


def _oracle_synthesize(ctx, opt, dataset, selection, tags, lmn, normalize):
    """The per-rank GPU synthesis call stood in by the FP64 oracle: VV = V diag(scale ev)
    V^H per image and sample, exact sum over the baselines, 1/nSamples if normalize."""
    from oracle import bluebild as bb

    lmn = np.asarray(lmn, np.float64)
    out = np.zeros((len(tags), lmn.shape[0]))
    for ti, tag in enumerate(tags):
        for sid, ev in selection[tag].items():
            uvw = dataset.uvw(sid).astype(np.float64) * (2 * np.pi / dataset.wl(sid))
            vv = bb.virtual_vis(dataset.scale(sid), np.asarray(ev, np.float64), dataset.eig_vec(sid))
            out[ti] += bb.nuft_sum(1.0, vv.reshape(-1, order="F"), uvw[:, 0], uvw[:, 1], uvw[:, 2],
                                   lmn[:, 0], lmn[:, 1], lmn[:, 2])
        if normalize:
            out[ti] /= len(selection[tag])
    return out.astype(np.float32)


def _dataset_case():
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim
    from oracle import bluebild as bb

    cfg = sim.config_c1(n_antenna=10, n_steps=5, image_size=6)
    obs = sim.observation(cfg)
    s, xyz = sim.visibilities(obs, list(range(5)))
    ds = bipp.InMemoryDataset(10, 10)
    sel = {"lvl0": {}, "lvl1": {}}
    for k in range(5):
        v, d, nr, sc = bb.eigh_gram(cfg.wl, s[k].numpy(), np.eye(10), xyz[k].numpy())
        ds.write(k, cfg.wl, sc, v, d, sim.baseline_uvw(obs, xyz[k].numpy()))
        sel["lvl0"][k] = (d * (d > 0)).astype(np.float32)
        sel["lvl1"][k] = (d * (d <= 0)).astype(np.float32)
    return ds, sel, obs.lmn


def _synthesis_worker(rank, size, port, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size)
    import types

    import bipp_b200 as bipp
    from bipp_b200 import api

    api._synthesize = _oracle_synthesize
    ds, sel, lmn = _dataset_case()
    ctx = types.SimpleNamespace(communicator=bipp.communicator(rank, size))
    out = bipp.image_synthesis(ctx, bipp.NufftSynthesisOptions(), ds, sel, lmn)
    out_q.put((rank, out))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_image_synthesis_over_two_ranks():
    """image_synthesis with a context of two ranks: sample blocks per rank, one SUM
    reduction into rank 0, normalisation by the total there; equal to one process over
    all samples (the per-rank synthesis is the oracle, so this tests the host logic)."""
    import types

    import bipp_b200 as bipp
    from bipp_b200 import api

    ds, sel, lmn = _dataset_case()
    saved = api._synthesize
    api._synthesize = _oracle_synthesize
    try:
        full = bipp.image_synthesis(types.SimpleNamespace(communicator=bipp.communicator.local()),
                                    bipp.NufftSynthesisOptions(), ds, sel, lmn)
    finally:
        api._synthesize = saved
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_synthesis_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert got[1] == {}
    for tag in ("lvl0", "lvl1"):
        assert np.abs(got[0][tag] - full[tag]).max() <= 1e-5 * np.abs(full[tag]).max()


def test_split_selection_property():
    """For any set of sample ids and rank count: the ranks' blocks partition the sorted
    ids in rank order, no block is longer than ceil(n / size), and every image's block
    carries its own eigenvalues."""
    from hypothesis import given, settings, strategies as st

    import bipp_b200 as bipp

    @settings(max_examples=200, deadline=None, database=None)
    @given(st.sets(st.integers(0, 999), min_size=1, max_size=60), st.integers(1, 9))
    def check(ids, size):
        sel = {"a": {i: np.full(2, i, np.float32) for i in ids}, "b": {i: np.full(2, -i, np.float32) for i in ids}}
        got = []
        for r in range(size):
            local, n = bipp.split_selection(sel, 1000, r, size)
            assert n == len(ids)
            assert list(local["a"]) == list(local["b"])
            assert len(local["a"]) <= -(-len(ids) // size)
            for i in local["a"]:
                assert local["a"][i][0] == i and local["b"][i][0] == -i
            got += list(local["a"])
        assert got == sorted(ids)

    check()
