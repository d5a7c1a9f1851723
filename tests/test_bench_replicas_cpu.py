"""The multi-process plumbing of bench.py --gpus N (independent replicas, one process per
device): two gloo ranks on the host agree on the barrier and take the maximum over ranks of
their step times, as the bench does for its device-timed value. No GPU is used."""
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    run = bench.Run()
    run.barrier()
    worst = run.max_over_ranks(10.0 + rank)  # this rank's step time
    run.barrier()
    run.close()
    q.put((rank, run.device, worst))


def test_two_gloo_ranks_take_the_max_step_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(out) == [(0, "cpu", 11.0), (1, "cpu", 11.0)]
