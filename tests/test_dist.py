"""The bench's multi-process plumbing (replicas, no data-path collective) on
CPU: two gloo ranks, as ``torchrun --nproc-per-node 2 bench.py`` starts
them, agree on the max-over-ranks time and pass the barriers."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    try:
        d.barrier()
        v = d.max(10.0 + rank)  # per-rank step time; the job's time is the max
        d.barrier()
        q.put((rank, d.world, v))
    finally:
        d.close()


def test_two_rank_max_and_barrier():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 11.0), (1, 2, 11.0)]


def test_single_process_is_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("WORLD_SIZE", "RANK"):
        os.environ.pop(k, None)
    d = bench.Dist()
    assert d.world == 1 and d.max(3.5) == 3.5
    d.barrier()
    d.close()
