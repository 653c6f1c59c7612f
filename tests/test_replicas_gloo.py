"""Multi-GPU form (independent replicas, weak scaling): the rank plumbing
that bench.py uses -- barrier, max over ranks of a timing, whole-job
throughput = units of all ranks / slowest rank's time -- run as two gloo
ranks on the CPU (one process each, rendezvous on 127.0.0.1)."""
import multiprocessing as mp
import os
import socket


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from compmatmul_b200.replicas import Replicas
    r = Replicas(backend="gloo", timeout_s=60)
    r.barrier()
    res = {"max": r.max(1.5 + rank), "sum": r.sum(10.0 * (rank + 1)),
           "throughput": r.throughput(10, 1.0 + rank), "world": r.world, "rank": r.rank}
    r.barrier()
    r.close()
    out.put(res)


def test_replicas_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, out)) for k in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in res:
        assert r["world"] == 2
        assert r["max"] == 2.5           # the slower rank's value
        assert r["sum"] == 30.0
        assert r["throughput"] == 10.0   # 2 x 10 units over the slowest rank's 2 s


def test_replicas_single_process_is_identity():
    from compmatmul_b200.replicas import Replicas
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    r = Replicas(backend="gloo")
    assert r.world == 1 and r.max(3.0) == 3.0 and r.throughput(4, 2.0) == 2.0
    r.close()
