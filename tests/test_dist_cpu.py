"""The multi-process host logic of bench.py on CPU: two gloo ranks, set up as
torchrun sets them up (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR / MASTER_PORT),
join one process group through bench._dist() and agree on the largest per-rank
time (the timing rule of the replicated benchmark: every rank runs the whole
workload, the slowest rank's device time counts)."""
import os
import socket


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(ws), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import bench
    dist, r, w, local = bench._dist()
    try:
        assert (r, w, local) == (rank, ws, rank)
        got = bench.max_over_ranks(10.0 + 3.5 * rank, dist, device="cpu")
        dist.barrier()
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = dict(q.get(timeout=180) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    assert got == {0: 13.5, 1: 13.5}


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(4.25, None) == 4.25
    if "WORLD_SIZE" not in os.environ:
        assert bench._dist() == (None, 0, 1, 0)
