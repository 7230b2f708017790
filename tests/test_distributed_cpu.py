"""The multi-process plumbing of bench.py on CPU: world size 2 over gloo (127.0.0.1)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from v3dsfmtoolkit_b200.distributed import shard_range


def test_shard_range_partitions():
    for n in (0, 1, 5, 4096, 4097):
        for world in (1, 2, 3, 8):
            covered = []
            for r in range(world):
                lo, hi = shard_range(n, r, world)
                assert hi >= lo
                covered.extend(range(lo, hi))
            assert covered == list(range(n))
            sizes = [shard_range(n, r, world)[1] - shard_range(n, r, world)[0] for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from v3dsfmtoolkit_b200 import distributed
    dist = distributed.init("gloo", timeout_s=60)
    lo, hi = shard_range(4096, rank, world)
    # each rank "processes" its shard and reports the time it took (rank-dependent)
    done = distributed.reduce_scalar(dist, hi - lo, "sum")
    tmax = distributed.reduce_scalar(dist, 1.0 + rank, "max")
    dist.barrier()
    out[rank] = (done, tmax)
    dist.destroy_process_group()


def test_two_ranks_over_gloo():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == (4096.0, 2.0)


def _solve_worker(rank, world, port, n, out):
    """One rank of a sharded triplet job: solves its contiguous shard with the CPU restatement of
    the reference optimizer and gathers every rank's results."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from oracle.bindings import Restatement
    from v3dsfmtoolkit_b200 import distributed, scenes
    dist = distributed.init("gloo", timeout_s=60)
    trips = scenes.triplet_batch(n_triplets=n, min_points=20, max_points=60, seed=11)
    lo, hi = shard_range(n, rank, world)
    eng = Restatement()
    local = []
    for sc in trips[lo:hi]:
        (K, R, T, d, X), info = eng.minimize(sc, max_iterations=5)
        local.append((info["status"], info["iterations"], R.tobytes(), T.tobytes(), X.tobytes()))
    allres = distributed.gather_shards(dist, local)
    dist.barrier()
    out[rank] = allres
    dist.destroy_process_group()


def test_sharded_solve_equals_single_process():
    """The union of the shards solved on two gloo ranks is the single-process result, item by
    item in the job's order."""
    from oracle.bindings import Restatement
    from v3dsfmtoolkit_b200 import scenes
    n, world = 9, 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_solve_worker, args=(r, world, port, n, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    trips = scenes.triplet_batch(n_triplets=n, min_points=20, max_points=60, seed=11)
    eng = Restatement()
    single = []
    for sc in trips:
        (K, R, T, d, X), info = eng.minimize(sc, max_iterations=5)
        single.append((info["status"], info["iterations"], R.tobytes(), T.tobytes(), X.tobytes()))
    assert out[0] == out[1] == single
