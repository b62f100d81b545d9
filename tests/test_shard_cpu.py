"""Multi-rank sharding of one J/K build, on CPU.

The plan splits every class pair's work items into contiguous, cost-balanced
blocks per rank (b200jk_partition_items, the host function the GPU plan uses)
and the ranks' partial J/K are summed by one all-reduce
(gradscf_b200.jk.allreduce_partial).  Here two gloo ranks each evaluate the
canonical shell quartets (i>=j, k>=l, ij>=kl; the reference's unique set,
csrc/coulomb_shells.h:80-128) that the partition gives them -- from the
oracle's ERI tensor -- and the all-reduced sum must equal the full J/K.
"""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from gradscf_b200 import _capi  # noqa: E402
from gradscf_b200 import basis as B  # noqa: E402
from tests.gpu_util import WATER  # noqa: E402


def test_partition_contiguous_balanced_complete():
    rng = np.random.default_rng(5)
    for n, world in ((1, 1), (7, 2), (1000, 4), (333, 8), (5, 8)):
        cost = rng.integers(0, 5000, size=n)
        owner = _capi.partition_items(cost, world)
        assert owner.shape == (n,) and owner.min() >= 0 and owner.max() < world
        assert np.all(np.diff(owner) >= 0)                      # contiguous blocks
        load = np.bincount(owner, weights=cost, minlength=world)
        assert load.sum() == cost.sum()
        assert load.max() <= cost.sum() / world + cost.max() + 1e-9
    assert np.all(_capi.partition_items(np.zeros(6, np.int64), 3) == [0, 0, 1, 1, 2, 2])
    with pytest.raises(_capi.InvalidArgument):
        _capi.partition_items(np.ones(3, np.int64), 0)
    with pytest.raises(_capi.InvalidArgument):
        _capi.partition_items(np.array([1, -1]), 2)


def _quartets(bas):
    """Canonical shell quartets in the reference's loop order with their
    primitive-quartet costs."""
    nb = bas.shape[0]
    quart, cost = [], []
    for i in range(nb):
        for j in range(i + 1):
            for k in range(i + 1):
                for l in range(k + 1):
                    if (i, j) < (k, l):
                        continue
                    quart.append((i, j, k, l))
                    cost.append(int(np.prod([bas[s, 2] for s in (i, j, k, l)])))
    return quart, np.asarray(cost, dtype=np.int64)


def _partial_jk(rank, world):
    top, par, _ = B.prepare_basis(WATER, "6-31g*", cart=False)
    atm, bas, env = B.pack(top, par)
    eri = oracle.eri_s1(atm, bas, env, cart=False)
    n = eri.shape[0]
    ao = np.concatenate([[0], np.cumsum([(2 * bas[s, 1] + 1) * bas[s, 3] for s in range(bas.shape[0])])])
    quart, cost = _quartets(bas)
    owner = _capi.partition_items(cost, world)
    mask = np.zeros_like(eri)
    for (i, j, k, l), r in zip(quart, owner):
        if r != rank:
            continue
        si, sj, sk, sl = (slice(ao[s], ao[s + 1]) for s in (i, j, k, l))
        for a, b, c, d in ((si, sj, sk, sl), (sj, si, sk, sl), (si, sj, sl, sk), (sj, si, sl, sk),
                           (sk, sl, si, sj), (sl, sk, si, sj), (sk, sl, sj, si), (sl, sk, sj, si)):
            mask[a, b, c, d] = 1.0
    rng = np.random.default_rng(11)
    dm = rng.normal(size=(n, n))
    v = eri * mask
    j = np.einsum("abcd,cd->ab", v, dm)
    k = np.einsum("acbd,cd->ab", v, dm)
    return j, k, eri, dm


def _worker(rank, world, port, queue):
    import torch.distributed as dist
    from gradscf_b200.jk import allreduce_partial
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        j, k, _, _ = _partial_jk(rank, world)
        out = torch.tensor(np.stack([j, k]))
        allreduce_partial(out)
        queue.put((rank, out.numpy()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_sum_to_full_jk():
    world = 2
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(queue.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    _, _, eri, dm = _partial_jk(0, 1)
    jref, kref = oracle.full_jk(eri, dm)
    for r in range(world):
        np.testing.assert_allclose(got[r][0], jref, atol=1e-12)
        np.testing.assert_allclose(got[r][1], kref, atol=1e-12)
    # each rank alone holds only part of the result
    j0, _, _, _ = _partial_jk(0, world)
    assert np.abs(j0 - jref).max() > 1e-3


def _replica_worker(rank, world, port, queue):
    import torch.distributed as dist
    from gradscf_b200 import scf as S
    from gradscf_b200 import workloads as Wl
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = Wl.batch_sizes(256, 3)
        cost = (24 * sizes.astype(np.int64)) ** 3
        mine = S.replica_shard(cost, rank, world)
        # stand-in per-molecule results: any function of the molecule id
        vals = [1.5 * sizes[m] + 1e-3 * m for m in mine]
        got = S.gather_replicas(mine, vals, len(sizes))
        queue.put((rank, mine, got, int(cost[mine].sum())))
    finally:
        dist.destroy_process_group()


def test_batch_replicas_on_two_gloo_ranks():
    # the 256-cluster batch as replicas: each rank a contiguous cost-balanced
    # share of the clusters, per-cluster results gathered on every rank
    world = 2
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica_worker, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, mine, got, load = queue.get(timeout=240)
        res[r] = (mine, got, load)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from gradscf_b200 import workloads as Wl
    sizes = Wl.batch_sizes(256, 3)
    want = 1.5 * sizes + 1e-3 * np.arange(256)
    ids = np.concatenate([res[r][0] for r in range(world)])
    assert np.array_equal(np.sort(ids), np.arange(256))           # every cluster exactly once
    for r in range(world):
        np.testing.assert_allclose(res[r][1], want)                # gathered on every rank
    loads = [res[r][2] for r in range(world)]
    cost = (24 * sizes.astype(np.int64)) ** 3
    assert max(loads) <= cost.sum() / world + cost.max()           # balanced shares
