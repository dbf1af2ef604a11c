"""Instance sharding over ranks: gloo, world size 2, on CPU."""
import os
import socket

import torch.multiprocessing as mp

from pscf_b200.parallel import shard


def test_shard_covers_everything():
    for n in (0, 1, 5, 12, 257):
        for world in (1, 2, 3, 8):
            parts = [shard(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [e - b for b, e in parts]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _lamellae():
    from tests.cases import diblock, lamellar_guess
    out = []
    for i in range(5):
        s = diblock(1, [32], "lamellar", [1.5 + 0.05 * i], fA=0.5, chiN=14.0 + i)
        out.append((s, lamellar_guess(s)))
    return out


def _solve(items):
    from oracle import oracle as O
    res = []
    for s, w in items:
        _, _, r = O.Oracle(s).iterate_am(w, error_max=1e-10, max_itr=500)
        res.append({"f": r["f_helmholtz"], "itr": r["itr"], "converged": r["converged"]})
    return res


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from pscf_b200.parallel import solve_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = solve_sharded(_lamellae(), _solve)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_solve_sharded_gloo_matches_serial():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    serial = _solve(_lamellae())
    for r in range(2):
        assert [x["f"] for x in outs[r]] == [x["f"] for x in serial]
        assert all(x["converged"] for x in outs[r])


def _reduce_worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # per-rank seconds (max over ranks) and MDE steps (sum over ranks)
        q.put((rank, bench.reduce_max_sum([0.5 + rank, 1000 * (rank + 1)], ["max", "sum"], "cpu", world)))
    finally:
        dist.destroy_process_group()


def test_bench_reduction_over_ranks_gloo():
    """The bench's whole-job figures over ranks: the time is the slowest
    rank's, the work the sum of all ranks' (world size 2, gloo)."""
    import bench
    assert bench.reduce_max_sum([1.5, 7], ["max", "sum"], "cpu", 1) == [1.5, 7.0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_reduce_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert outs[0] == outs[1] == [1.5, 3000.0]
