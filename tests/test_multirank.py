"""The N > 1 host logic on CPU: two ranks over gloo (127.0.0.1) -- the
max-over-ranks timing bench.py uses for every multi-GPU number, and the
communication-free sharding (fg_shard_plan through the C ABI) of a ragged
batch and of a served request stream across GPUs."""
import datetime
import json
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _ragged_dims():
    rng = np.random.default_rng(42)
    return np.rint(np.exp(rng.uniform(np.log(8), np.log(512), (4096, 3)))).astype(int)


def _stream():
    """A served stream in arrival order with per-request cost estimates
    (f64 requests weighted 4x: the FP64 pipe is slower per flop)."""
    import bench_serving
    reqs = bench_serving.workload(3000)
    dims = [(m, n, k) for m, n, k, _ in reqs]
    weights = [2.0 * m * n * k * (4.0 if dt == np.float64 else 1.0) for m, n, k, dt in reqs]
    return dims, weights


def _online_py(weights, world):
    """FG_SHARD_ONLINE restated: arrival order, least-loaded rank, ties low."""
    load, owner = [0.0] * world, []
    for w in weights:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += w
        owner.append(r)
    return owner


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import ferray_b200 as fg
        slowest = bench.max_over_ranks(dist, torch, 1.5 + rank, device="cpu")
        mine = fg.shard_problems(_ragged_dims(), world, rank)
        shards = [None] * world
        dist.all_gather_object(shards, mine)
        reqs, weights = _stream()
        routed = fg.shard_requests(reqs, world, rank, weights)
        streams = [None] * world
        dist.all_gather_object(streams, routed)
        with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
            json.dump({"max": slowest, "shards": shards, "streams": streams}, f)
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(world)]
    assert all(r["max"] == 2.5 for r in res)  # every rank sees the slowest rank's time
    shards = res[0]["shards"]
    assert res[1]["shards"] == shards  # both ranks agree without a data-path exchange
    dims = _ragged_dims()
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(dims)))  # disjoint and complete
    work = 2 * dims[:, 0] * dims[:, 1] * dims[:, 2]
    loads = [int(work[s].sum()) for s in shards]
    assert max(loads) - min(loads) <= int(work.max())
    # served stream: every request routed to exactly one rank, the same on
    # both ranks, and to the rank the online rule picks
    streams = res[0]["streams"]
    assert res[1]["streams"] == streams
    _, weights = _stream()
    assert sorted(i for s in streams for i in s) == list(range(len(weights)))
    owner = _online_py(weights, world)
    for r, idx in enumerate(streams):
        assert all(owner[i] == r for i in idx)


def test_shard_problems_single_rank_and_errors():
    import ferray_b200 as fg
    dims = _ragged_dims()[:10]
    assert fg.shard_problems(dims, 1, 0) == list(range(10))
    for bad in ((2, 2), (0, 0), (2, -1)):
        try:
            fg.shard_problems(dims, *bad)
        except fg.InvalidValue:
            continue
        raise AssertionError("accepted world=%d rank=%d" % bad)


def test_shard_lpt_matches_restated_rule():
    import ferray_b200 as fg
    dims = _ragged_dims()[:500]
    work = 2 * dims[:, 0] * dims[:, 1] * dims[:, 2]
    order = np.argsort(-work, kind="stable")
    for world in (1, 2, 3, 8):
        load, owner = [0] * world, {}
        for i in order:
            r = min(range(world), key=lambda q: (load[q], q))
            load[r] += int(work[i])
            owner[int(i)] = r
        for rank in range(world):
            assert fg.shard_problems(dims, world, rank) == sorted(i for i, r in owner.items() if r == rank)
