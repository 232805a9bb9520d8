"""The sharded reduction of column-sharded runs: the host restatement of the
device tree against the oracle's tree, and the exchange over 2 and 3 gloo
ranks giving every rank the single-device value bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import pyoracle
from parallellocallyoptimalapproximatesparsematrixinverses_b200 import sharding


def _values(count, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(count) * 10.0 ** rng.integers(-6, 6, count)


@pytest.mark.parametrize("count", [0, 1, 255, 4095, 4096, 4097, 3 * 4096 + 17, 70_000])
def test_host_tree_is_the_device_tree(count):
    v = _values(count, count)
    assert sharding.tree_sum(v) == pyoracle.tree_sum(v)
    assert sharding.tree_sum(v * v) == pyoracle.tree_sum(v * v)


@pytest.mark.parametrize("n,world", [(0, 2), (10, 4), (4096, 2), (4097, 2), (70_000, 3), (262_144, 8)])
def test_shards_cover_the_columns_at_chunk_boundaries(n, world):
    ranges = sharding.shard_columns(n, world)
    assert len(ranges) == world
    assert ranges[0][0] == 0 and ranges[-1][1] == n
    for (a, b), (c, d) in zip(ranges, ranges[1:]):
        assert b == c and a <= b
    for a, _ in ranges:
        assert a % sharding.TREE_CHUNK == 0 or a == n
    sizes = [b - a for a, b in ranges]
    assert max(sizes) - min(sizes) <= sharding.TREE_CHUNK or n < world * sharding.TREE_CHUNK


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    a, b = sharding.shard_columns(n, world)[rank]
    # three per-column partial arrays (e.g. <Z, PrAZ>, ||PrAZ||^2, ||R||^2): this rank's columns only
    local = np.stack([sharding.tree_chunk_sums(_values(n, seed)[a:b]) if b > a else np.zeros(0)
                      for seed in (1, 2, 3)])
    out[rank] = sharding.sharded_tree_sums(local)
    dist.destroy_process_group()


@pytest.mark.parametrize("n,world", [(70_000, 2), (20_000, 3), (5_000, 3)])
def test_sharded_sums_equal_the_single_device_tree(n, world):
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    want = [pyoracle.tree_sum(_values(n, seed)) for seed in (1, 2, 3)]
    for r in range(world):
        assert list(out[r]) == want, f"rank {r}"


def _transpose_worker(rank, world, port, n, out):
    import torch
    import torch.distributed as dist
    from scipy import sparse
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    m = sparse.random(n, n, density=0.01, random_state=np.random.default_rng(4), format="csc")
    m = sparse.csc_matrix(m + sparse.identity(n))
    m.sort_indices()
    ranges = sharding.shard_columns(n, world, align=64)
    a, b = ranges[rank]
    local = m[:, a:b]
    ptr, rows, vals = sharding.sharded_transpose(torch.tensor(local.indptr, dtype=torch.int64),
                                                 torch.tensor(local.indices, dtype=torch.int64),
                                                 torch.tensor(local.data, dtype=torch.float64), ranges, rank)
    out[rank] = (ptr.numpy(), rows.numpy(), vals.numpy())
    dist.destroy_process_group()


@pytest.mark.parametrize("n,world", [(700, 2), (1000, 3)])
def test_sharded_transpose_gives_each_rank_its_columns_of_the_transpose(n, world):
    from scipy import sparse
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_transpose_worker, args=(r, world, port, n, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    m = sparse.random(n, n, density=0.01, random_state=np.random.default_rng(4), format="csc")
    m = sparse.csc_matrix(m + sparse.identity(n))
    mt = sparse.csc_matrix(m.T)
    mt.sort_indices()
    for r, (a, b) in enumerate(sharding.shard_columns(n, world, align=64)):
        want = mt[:, a:b]
        ptr, rows, vals = out[r]
        assert np.array_equal(ptr, want.indptr) and np.array_equal(rows, want.indices)
        assert np.array_equal(vals, want.data)


def _scores(total, seed):
    rng = np.random.default_rng(seed)
    s = rng.standard_normal(total) * 10.0 ** rng.integers(-3, 3, total)
    s[rng.integers(0, total, total // 10)] = 0.0          # ties at zero
    s[rng.integers(0, total, total // 20)] = -0.0
    s[rng.integers(0, total, total // 50)] = -np.inf      # non-finite scores map to -inf
    s[rng.integers(0, total, total // 10)] = 1.5           # more ties
    return s


def _select_worker(rank, world, port, total, drop, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bounds = [total * r // world for r in range(world + 1)]
    scores = _scores(total, 9)[bounds[rank]:bounds[rank + 1]]
    out[rank] = sharding.sharded_drop_cutoff(sharding.ordered_bits(scores), bounds[rank], drop)
    dist.destroy_process_group()


@pytest.mark.parametrize("total,drop,world", [(5_000, 1, 2), (5_000, 2_500, 3), (20_011, 19_000, 2),
                                              (20_011, 20_011, 3)])
def test_sharded_drop_cutoff_is_the_single_device_select(total, drop, world):
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_select_worker, args=(r, world, port, total, drop, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    bits = sharding.ordered_bits(_scores(total, 9))
    order = np.lexsort((np.arange(total), bits))  # by (bits, offset)
    want = (int(bits[order[drop - 1]]), int(order[drop - 1]))
    for r in range(world):
        assert tuple(out[r]) == want, f"rank {r}"
    # exactly `drop` candidates lie at or below the cutoff
    keys = [(int(b), i) for i, b in enumerate(bits)]
    assert sum(1 for k in keys if k <= want) == drop


def _bad_drop_worker(rank, world, port, total, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bounds = [total * r // world for r in range(world + 1)]
    bits = sharding.ordered_bits(_scores(total, 9)[bounds[rank]:bounds[rank + 1]])
    messages = []
    for drop in (0, -3, total + 1):
        try:
            sharding.sharded_drop_cutoff(bits, bounds[rank], drop)
            messages.append(None)
        except ValueError as err:
            messages.append(str(err))
    # the group is still usable: a valid select afterwards agrees on every rank
    messages.append(sharding.sharded_drop_cutoff(bits, bounds[rank], total))
    out[rank] = messages
    dist.destroy_process_group()


def test_sharded_drop_cutoff_rejects_drop_counts_outside_the_candidates():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    total, world = 3_001, 2
    procs = [ctx.Process(target=_bad_drop_worker, args=(r, world, port, total, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    for r in range(world):
        bad = out[r][:3]
        assert all(m is not None and "[1, 3001]" in m for m in bad), bad
    assert out[0][3] == out[1][3]


def test_ordered_bits_preserve_the_order():
    v = np.array([-np.inf, -1e300, -2.0, -1e-300, -0.0, 0.0, 1e-300, 3.0, 1e300, np.inf])
    bits = sharding.ordered_bits(v)
    assert all(bits[i] <= bits[i + 1] for i in range(len(v) - 1))
    assert bits[4] == bits[5]
