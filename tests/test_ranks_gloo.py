"""The N>1 plumbing on CPU: two gloo ranks deal a batch ensemble and a request
stream between them (every problem exactly once, sizes balanced) and reduce
their timings (max) and work (sum) the way bench.py does on the GPU box."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from ramses2_b200.batch import ensemble_octs, riemann_blast_ensemble
    from ramses2_b200.ranks import max_over_ranks, shard, sum_over_ranks
    from ramses2_b200.serve import make_requests

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        ens = riemann_blast_ensemble(64, seed=5)
        mine = shard(list(enumerate(ens)), rank, world)
        ids = [i for i, _ in mine]
        octs = ensemble_octs([e for _, e in mine])
        reqs = shard(make_requests(10, rate_hz=4.0, seed=9), rank, world)
        t_local = 1.0 + rank  # stand-in for a per-rank device time
        tmax = max_over_ranks([t_local, 10.0 * t_local], dist, device="cpu")
        tot = sum_over_ranks([octs, len(reqs)], dist, device="cpu")
        q.put((rank, ids, octs, [r.rid for r in reqs], tmax, tot))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_shard_and_reduce():
    from ramses2_b200.batch import ensemble_octs, riemann_blast_ensemble

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=150) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    ids = sorted(out[0][1] + out[1][1])
    assert ids == list(range(64))
    total = ensemble_octs(riemann_blast_ensemble(64, seed=5))
    assert out[0][2] + out[1][2] == total
    assert 0.25 < out[0][2] / total < 0.75
    assert sorted(out[0][3] + out[1][3]) == list(range(10))
    for r in out:
        assert r[4] == [2.0, 20.0]
        assert r[5] == [float(total), 10.0]
