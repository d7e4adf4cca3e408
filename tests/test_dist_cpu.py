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


def _sweep_cfgs(max_steps=50_000):
    import bench
    return bench.sweep_configs(max_steps=max_steps)


def test_partition_covers_every_case_once_and_balances():
    """The sweep's 72 cases split over 1..8 ranks: every case on exactly one
    rank, the same split on every call, and the largest load above the
    smallest by at most one case's cost (longest-processing-time rule)."""
    from iblbm_b200.batch import case_cost, partition_cases
    cfgs = _sweep_cfgs()
    cost = [case_cost(c) for c in cfgs]
    for world in range(1, 9):
        parts = partition_cases(cfgs, world)
        assert parts == partition_cases(cfgs, world)
        assert len(parts) == world
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(cfgs)))
        loads = [sum(cost[k] for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(cost)
        if world > 1:  # balanced to within 5 % of the mean on this sweep
            assert max(loads) <= 1.05 * sum(loads) / world


def _small_cfgs():
    from iblbm_b200.config import SimConfig
    out = []
    for k, (method, delta, coll) in enumerate([("DF", "hat", "BGK"), ("MDF", "peskin4pt", "TRT"),
                                              ("DFC", "peskin4pt", "CM_MRT"), ("DF", "peskin4pt", "TRT"),
                                              ("MDF", "hat", "BGK")]):
        out.append(SimConfig(Re=20 + 10 * k, NN=33 + 8 * k, xmax=2, ymax=1, cylinder_center=(0.45, 0.5),
                             cylinder_D_ratio=0.25, lattice_u=0.05, inflow_u=0.05, bc_type="dirichlet_neumann",
                             delta_type=delta, ibm_method=method, collision_model=coll, trt_magic_param=0.1875,
                             mdf_iterations=10, mdf_min_iterations=3, mdf_tolerance=1e-6,
                             marker_spacing_factor=1.0, max_steps=40, use_convergence=False, check_interval=20))
    return out


def _partition_worker(rank, ws, port, out):
    """One rank of a partitioned sweep: its share of the cases (run here on
    the CPU oracle), then the host-side gather of every case's Cd / Cl."""
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(ws), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), OMP_NUM_THREADS="1")
    import bench
    from iblbm_b200.batch import gather_case_results, partition_cases
    from oracle import harness as H
    dist, r, w, _ = bench._dist()
    try:
        cfgs = _small_cfgs()
        mine = partition_cases(cfgs, w)[r]
        local = {}
        for k in mine:
            res = H.run(cfgs[k])
            local[k] = (list(res["Cd_history"]), list(res["Cl_history"]))
        allres = gather_case_results(local, dist)
        dist.barrier()
        out.put((rank, mine, allres))
    finally:
        dist.destroy_process_group()


def test_partitioned_sweep_gathers_every_case_on_two_gloo_ranks():
    """Two gloo ranks split a small sweep, run their own cases and gather the
    Cd / Cl histories on the host: both ranks end with every case exactly
    once, each equal to the single-process run of that case."""
    import torch.multiprocessing as mp
    from oracle import harness as H
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_partition_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = {r: (mine, res) for r, mine, res in (q.get(timeout=300) for _ in procs)}
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    cfgs = _small_cfgs()
    assert sorted(got[0][0] + got[1][0]) == list(range(len(cfgs)))
    assert got[0][0] and got[1][0]
    assert got[0][1] == got[1][1]
    for k, cfg in enumerate(cfgs):
        res = H.run(cfg)
        assert got[0][1][k] == (list(res["Cd_history"]), list(res["Cl_history"]))


def test_gather_without_group_is_identity():
    from iblbm_b200.batch import gather_case_results
    assert gather_case_results({3: "c", 1: "a"}) == {1: "a", 3: "c"}
