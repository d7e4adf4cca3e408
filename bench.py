#!/usr/bin/env python
"""Benchmark of the IB-LBM per-timestep hot path on B200.

Two forms of the hot path are timed on one GPU:

plain   the FP64 form (the reference's arithmetic, bit for bit) on the
        reference's single-case benchmark: fixed cylinder at Re = 100 on a
        1601 x 641 D2Q9 lattice, D = 40, 126 Lagrangian markers, inflow
        u = 0.04, TRT (magic Lambda = 3/16), multi-direct forcing with the
        Peskin 4-point kernel (5 to 20 iterations until the slip residual
        < 1e-6), Dirichlet/Neumann channel.  One step = the band kernel (all MDF
        iterations) and the fused collide-stream pass; L2 flushed between steps.
chosen  the FP32 shifted-population form (FP64 force sums and MDF residual
        norm) run batched: the 72-case sweep Re {20, 40, 100, 200} x
        {DF, MDF, DFC} x {hat, Peskin-4} x {BGK, TRT, CM-MRT} of fixed cylinders
        on 401x161 to 1921x961 lattices, all cases stepped together (one
        batched band launch, one collide-stream launch per kind of case).  The
        same workload as the plain form is also timed in the FP32 form, one
        case alone (chosen_single_case).

Reported (one JSON line on rank 0):
  value       aggregate MLUPS of the chosen form (device time, CUDA events);
              plain.mlups is the plain form's.
  e2e         the same through the public API with host buffers: every step
              uploads all cases' markers from pinned host memory and reads all
              marker forces back.
  roofline    the collide-stream launches of a step against the measured HBM
              copy bandwidth: 72 algorithmic bytes per lattice update in FP32
              (9 populations read + 9 written), 144 in FP64.
  sweep       Cd/Cl of every batched case against the FP64 plain form of the
              same case after the same steps (target: within 0.1 %).
  cpu_baseline  the CPU oracle (a C + OpenMP restatement of the reference's
              CPU path) on a bounded sample of the single-case workload.

Inputs are deterministic initial states (no dataset).  --form plain times the
plain form alone.  --impl reference times the CPU restatement of the
reference's own path (the reference is a Python package whose CPU path cannot
travel to the GPU box).  Multi-GPU: cases do not shard; N ranks run N
independent replicas (weak scaling), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_LU_F64 = 144
BYTES_PER_LU_F32 = 72
# DRAM bytes per updated node measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum within the kernel window, caches flushed before the
# launch): FP32 batched bulk pass of one collision model on the Re 20/40 part of
# the sweep (71.63 MB read + 28.31 MB written for the 1 930 092 nodes of its 12
# lattices, exclusion boxes included), FP64 single-case bulk pass (73.81 MB read
# + 25.93 MB written for 1 023 949 nodes).  Part of the population writes stays
# in L2 until after the kernel, so the write share is a lower bound.
TRAFFIC_PER_NODE_F32 = (71.63e6 + 28.31e6) / 1930092
TRAFFIC_PER_NODE_F64 = (73.81e6 + 25.93e6) / 1023949
METRIC = "MLUPS and HBM GB/s (1 B200), chosen vs plain form at Cd within 0.1% of FP64"


def workload_config(collision="TRT", max_steps=1_000_000):
    from iblbm_b200 import SimConfig
    return SimConfig(Re=100, NN=641, xmax=2.5, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.0625,
                     lattice_u=0.04, inflow_u=0.04, bc_type="dirichlet_neumann", delta_type="peskin4pt",
                     ibm_method="MDF", collision_model=collision, trt_magic_param=0.1875, mdf_iterations=20,
                     mdf_min_iterations=5, mdf_tolerance=1e-6, marker_spacing_factor=1.0, max_steps=max_steps,
                     use_convergence=False, check_interval=100)


WORKLOAD = {"workload": "fixed cylinder Re=100, 1601x641 D2Q9, D=40, 126 markers, MDF(5-20 it, tol 1e-6)+P4, "
                        "TRT Lambda=3/16, Dirichlet/Neumann channel", "lattice": [1601, 641], "markers": 126,
            "collision": "TRT", "ibm": "MDF", "delta": "peskin4pt", "form": "FP64 plain",
            "l2": "evicted between timed steps (256 MB read); the flushed steps replay from one CUDA graph"}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.fh = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.fh.flush()
        rows = []
        with open(self.fh.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.fh.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        import statistics
        mhz = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(mhz) if mhz else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def _dist():
    """One process per GPU, launched by torchrun (RANK / LOCAL_RANK / WORLD_SIZE /
    MASTER_* in the environment): NCCL on GPUs, gloo on a host without one.
    Returns (torch.distributed or None, rank, world size, local rank)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        cuda = torch.cuda.is_available()
        if cuda:
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if cuda else "gloo", timeout=datetime.timedelta(seconds=120))
        return dist, int(os.environ.get("RANK", "0")), ws, local
    return None, 0, 1, 0


def max_over_ranks(x, dist, device="cuda"):
    """The largest of x over all ranks (every rank calls it at the same point);
    x itself without a process group."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def oracle_sweep_sample(per_case, threads=None):
    """The CPU oracle on the sweep: every case in turn (one in memory at a time),
    one warm-up step and `per_case` timed steps each, so the mix of lattices and
    band methods per step is the sweep's.  MLUPS over the timed steps."""
    threads = threads or os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import harness as H
    cfgs = sweep_configs(max_steps=per_case + 2)
    lu, dt = 0, 0.0
    for cfg in cfgs:
        sim = H.OracleSim(cfg)
        sim.step()
        t0 = time.perf_counter()
        for _ in range(per_case):
            sim.step()
        dt += time.perf_counter() - t0
        lu += sim.s.nx * sim.s.ny * per_case
        del sim
    return {"value": lu / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port", "timed_s": dt,
            "cases": len(cfgs), "sample": f"{per_case} timed steps of each of the {len(cfgs)} sweep cases after one "
                                          f"warm-up step each ({dt:.1f} s timed)"}


def cpu_baseline(seconds=20.0, threads=None):
    """Time the CPU oracle on a bounded sample of the workload (whole timesteps)."""
    threads = threads or os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import harness as H
    sim = H.OracleSim(workload_config())
    sim.step()  # warm-up (first touch, library load)
    n, t0 = 0, time.perf_counter()
    while True:
        sim.step()
        n += 1
        dt = time.perf_counter() - t0
        if dt > seconds or n >= 400:
            break
    N = sim.s.nx * sim.s.ny
    return {"value": N * n / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{n} timesteps of the workload after 1 warm-up step ({dt:.1f} s)"}


def run_reference(args):
    dist, rank, ws, _ = _dist()
    if rank != 0:
        return
    per_case = max(1, min(args.steps, 2))
    base = oracle_sweep_sample(per_case)
    v, dt, threads, cfgs = base["value"], base["timed_s"], base["cores"], base["cases"]
    line = {"metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus, "steps": per_case,
            "warmup": 1, "ms_per_step": dt / per_case * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (deterministic initial state)",
            "config": {"workload": SWEEP_WORKLOAD, "cases": cfgs, "form": "reference CPU path (C + OpenMP "
                       "restatement of the reference's numba/numpy path), FP64"}, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": threads, "kind": "port", "sample": base["sample"]},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _flushed_steps_graph(eng, K, flush, sink):
    """K overlapped steps of one engine, each followed by a 256 MB read that evicts
    the populations from L2, captured as one CUDA graph so that the host's launch
    rate does not enter the per-step times; the timing events are graph nodes
    (start, bulk start, bulk end, end of each step)."""
    import torch
    E = lambda: torch.cuda.Event(enable_timing=True, external=True)
    ev = [[E() for _ in range(4)] for _ in range(K)]
    cap = torch.cuda.Stream(eng.dev)
    cap.wait_stream(torch.cuda.current_stream(eng.dev))
    cap.wait_stream(eng.side)
    g = torch.cuda.CUDAGraph()
    p0 = eng.parity
    with torch.cuda.stream(cap):
        with torch.cuda.graph(g, stream=cap):
            eng.fence()  # fork: the side stream's first wait is on captured work
            for k in range(K):
                ev[k][0].record(cap)
                eng._step_overlapped(False, bulk_events=(ev[k][1], ev[k][2]))
                eng.join()
                ev[k][3].record(cap)
                torch.sum(flush, dim=0, out=sink)
                eng.fence()
    torch.cuda.current_stream(eng.dev).wait_stream(cap)
    eng.parity = p0  # capture does not execute
    return g, ev


def measure(eng, args, dist, ws):
    """Time one engine on the workload: per-step (L2 flushed) overlapped steps,
    the band kernel alone, graph-replayed steady state and the host-buffer e2e
    loop.  Returns a dict of the numbers (all ranks)."""
    import torch
    N = eng.N
    # warm-up: graph chunks and eager steps; tile choice of the FP32 pass
    eng.advance(max(args.warmup, 3), outputs_last=True)
    torch.cuda.synchronize()
    from iblbm_b200.autotune import tune_dense
    tile_ms, tile = tune_dense(eng)
    eng.advance(3, outputs_last=True)
    torch.cuda.synchronize()
    flush = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    sink = torch.zeros((), dtype=torch.float32, device="cuda")
    K = args.steps
    E = lambda: torch.cuda.Event(enable_timing=True)
    excl = eng.d_excl[eng.parity].tolist()
    box_nodes = excl[2] * excl[3]
    graph, ev = _flushed_steps_graph(eng, K, flush, sink)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(torch.cuda.current_device()) as clk:
        t_wall = time.perf_counter()
        graph.replay()
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    eng.parity ^= K & 1
    step_ms = [ev[k][0].elapsed_time(ev[k][3]) for k in range(K)]
    dense_ms = [ev[k][1].elapsed_time(ev[k][2]) for k in range(K)]
    tot_ms = max_over_ranks(sum(step_ms), dist)
    dense_avg = sum(dense_ms) / K
    bpl = BYTES_PER_LU_F32 if eng.f32 else BYTES_PER_LU_F64

    # band kernel alone (serial step: band kernel then the whole lattice), for the breakdown
    sev = [[E() for _ in range(3)] for _ in range(8)]
    for k in range(8):
        eng._step_serial(False, events=sev[k])
        eng.fence()
    torch.cuda.synchronize()
    ibm_ms = sum(sev[k][0].elapsed_time(sev[k][1]) for k in range(8)) / 8
    full_ms = sum(sev[k][1].elapsed_time(sev[k][2]) for k in range(8)) / 8

    # steady state: CUDA-graph replay, no flush (L2-warm; reported, not the headline)
    torch.cuda.synchronize()
    e0, e1 = E(), E()
    eng.advance(K, outputs_last=False)  # capture
    torch.cuda.synchronize()
    e0.record()
    eng.advance(K, outputs_last=False)
    e1.record()
    torch.cuda.synchronize()
    steady = N * K / (e0.elapsed_time(e1) / 1e3) / 1e6

    # end to end through the engine with host buffers
    Lb = eng.Lb
    host_in = torch.empty(4 * Lb, dtype=torch.float64).pin_memory()
    host_in[:Lb] = torch.as_tensor(eng.st.Lx)
    host_in[Lb:2 * Lb] = torch.as_tensor(eng.st.Ly)
    host_in[2 * Lb:] = torch.as_tensor(eng.st.desired_velocity.reshape(-1))
    host_out = torch.empty(2, dtype=torch.float64).pin_memory()
    Ke = max(10, K // 2)
    # a host program one step ahead, two pinned buffer pairs alternating (as for the batch)
    ins = [host_in, torch.empty_like(host_in).pin_memory()]
    ins[1].copy_(host_in)
    outs = [host_out, torch.empty_like(host_out).pin_memory()]
    for k in range(2):  # capture the two (parity, buffer) graphs
        eng.step_io(ins[k], outs[k])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prev = None
    for k in range(Ke):
        ev = eng.step_io(ins[k % 2], outs[k % 2], wait=False)
        if prev is not None:
            prev.synchronize()  # the previous step's band force is in outs[(k - 1) % 2]
        prev = ev
    prev.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)  # the slowest rank
    # one output step so both forms can be compared at the same step
    eng.advance(1, outputs_last=True)
    torch.cuda.synchronize()
    cd, cl = eng.cd_cl()
    return {"value": N * K * ws / (tot_ms / 1e3) / 1e6, "ms_per_step": tot_ms / K, "dense_ms": dense_avg,
            "box_nodes": box_nodes, "bytes_per_lu": bpl,
            "achieved": bpl * (N - box_nodes) / (dense_avg / 1e3) / 1e9, "band_ms": ibm_ms, "full_ms": full_ms,
            "steady": steady, "e2e": N * Ke * ws / e2e_s / 1e6, "e2e_h2d": 4 * Lb * 8, "e2e_d2h": 16,
            "clocks": clk.summary(), "wall_s_timed": t_wall, "status": eng.status(), "mdf": eng.mdf_stats(),
            "cd": cd, "cl": cl, "steps_done": eng.ttt - 1,
            "tile": tile, "tile_ms": tile_ms}


# Batched sweep: fixed cylinders, Re x band method x delta kernel x collision
# model on uneven lattices (Re -> NN, xmax, D/(NN-1), inflow u).
SWEEP_SIZES = {20: (161, 2.5, 0.125, 0.05), 40: (321, 2.5, 0.1, 0.05), 100: (641, 2.5, 0.0625, 0.04),
               200: (961, 2.0, 0.05, 0.04)}


SWEEP_WORKLOAD = ("chosen form: batched sweep of 72 fixed-cylinder cases, Re {20,40,100,200} x {DF,MDF,DFC} x "
                  "{hat,P4} x {BGK,TRT,CM-MRT} on 401x161 (D=20), 801x321 (D=32), 1601x641 (D=40), 1921x961 "
                  "(D=48) lattices")


def sweep_configs(max_steps):
    from iblbm_b200 import SimConfig
    out = []
    for Re, (NN, xmax, Dr, u) in SWEEP_SIZES.items():
        for method in ("DF", "MDF", "DFC"):
            for delta in ("hat", "peskin4pt"):
                for coll in ("BGK", "TRT", "CM_MRT"):
                    out.append(SimConfig(Re=Re, NN=NN, xmax=xmax, ymax=1, cylinder_center=(0.5, 0.5),
                                         cylinder_D_ratio=Dr, lattice_u=u, inflow_u=u, bc_type="dirichlet_neumann",
                                         delta_type=delta, ibm_method=method, collision_model=coll,
                                         trt_magic_param=0.1875, mdf_iterations=20, mdf_min_iterations=5,
                                         mdf_tolerance=1e-6, marker_spacing_factor=1.0, max_steps=max_steps,
                                         use_convergence=False, check_interval=100))
    return out


def measure_batch(b, K, W, dist, ws):
    """Time the batched sweep: per-group tile tuning, K overlapped steps (every
    step streams the whole sweep, ~4 GB, far above L2), graph-replayed steady
    state, and the host-buffer loop (all markers in, all marker forces out)."""
    import torch
    E = lambda: torch.cuda.Event(enable_timing=True)
    b.advance(max(W, 3), outputs_last=False)
    torch.cuda.synchronize()
    # tile choice per bulk group (cases of one collision, closure and compressibility):
    # the bulk pass is side-effect free when repeated without a parity flip
    tiles = {}
    main = torch.cuda.current_stream()
    for g in range(len(b.bulk_groups)):
        best = None
        for tile in ("node", "rows2", "rows4"):
            b.set_bulk_tile(g, tile)
            b._bulk(g, main.cuda_stream)
            ev = [(E(), E()) for _ in range(3)]
            for e0, e1 in ev:
                e0.record()
                b._bulk(g, main.cuda_stream)
                e1.record()
            torch.cuda.synchronize()
            ms = min(e0.elapsed_time(e1) for e0, e1 in ev)
            if best is None or ms < best[1]:
                best = (tile, ms)
        b.set_bulk_tile(g, best[0])
        tiles[g] = best
    # one bulk launch over every case against one launch per group
    per_group_ms = sum(ms for _, ms in tiles.values())
    merged = {}
    if b.C <= 72 and len(b.bulk_groups) > 1:
        for tile in ("node", "rows2", "rows4"):
            b.set_tile_all(tile, merged=True)
            b._dense("all", "bulk", main.cuda_stream)
            ev = [(E(), E()) for _ in range(3)]
            for e0, e1 in ev:
                e0.record()
                b._dense("all", "bulk", main.cuda_stream)
                e1.record()
            torch.cuda.synchronize()
            merged[tile] = min(e0.elapsed_time(e1) for e0, e1 in ev)
        best_tile = min(merged, key=merged.get)
        # in the timed schedule the single launch also competes with the band and
        # box kernels of the side stream, which slip in between per-group launches:
        # take it only on a clear win in isolation
        b.set_tile_all(best_tile, merged=merged[best_tile] < 0.95 * per_group_ms)
    b.fence()
    ev = [[E() for _ in range(4)] for _ in range(K)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(torch.cuda.current_device()) as clk:
        t_wall = time.perf_counter()
        for k in range(K):
            ev[k][0].record(main)
            b._step(bulk_events=(ev[k][1], ev[k][2]))
            b.join()
            ev[k][3].record(main)
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    b._bump(K)
    tot_ms = sum(ev[k][0].elapsed_time(ev[k][3]) for k in range(K))
    bulk_ms = sum(ev[k][1].elapsed_time(ev[k][2]) for k in range(K)) / K
    tot_ms = max_over_ranks(tot_ms, dist)
    box_nodes = sum(int(x[2]) * int(x[3]) for e in b.engines for x in [e.d_excl[b.parity].tolist()])
    achieved = BYTES_PER_LU_F32 * (b.N - box_nodes) / (bulk_ms / 1e3) / 1e9
    # steady state through one captured graph
    e0, e1 = E(), E()
    b.advance(K, outputs_last=False)
    torch.cuda.synchronize()
    e0.record()
    b.advance(K, outputs_last=False)
    e1.record()
    torch.cuda.synchronize()
    steady = b.N * K / (e0.elapsed_time(e1) / 1e3) / 1e6
    # host buffers: every step uploads all cases' markers and reads all marker forces back
    nin = b.marker_in.numel()
    host_in = torch.empty(nin, dtype=torch.float64).pin_memory()
    host_in.copy_(b.marker_in.cpu())
    host_out = torch.empty(b.marker_out.numel(), dtype=torch.float64).pin_memory()
    Ke = max(10, K // 2)
    # a host program one step ahead: step k runs while the host reads step k-1's
    # forces; two pinned buffer pairs alternate (each step still copies all its
    # markers in and all its forces out)
    ins = [host_in, torch.empty_like(host_in).pin_memory()]
    ins[1].copy_(host_in)
    outs = [host_out, torch.empty_like(host_out).pin_memory()]
    for k in range(2):  # capture the two (parity, buffer) graphs
        b.step_io(ins[k], outs[k])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    prev = None
    for k in range(Ke):
        ev = b.step_io(ins[k % 2], outs[k % 2], wait=False)
        if prev is not None:
            prev.synchronize()  # the previous step's forces are in outs[(k - 1) % 2]
        prev = ev
    prev.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)  # the slowest rank
    b.advance(1, outputs_last=True)
    torch.cuda.synchronize()
    return {"value": b.N * K * ws / (tot_ms / 1e3) / 1e6, "ms_per_step": tot_ms / K, "bulk_ms": bulk_ms,
            "achieved": achieved, "box_nodes": box_nodes, "steady": steady,
            "e2e": b.N * Ke * ws / e2e_s / 1e6, "h2d": nin * 8, "d2h": host_out.numel() * 8,
            "clocks": clk.summary(), "wall_s_timed": t_wall, "status": b.status(),
            "tiles": {str(g): {"tile": t, "bulk_ms": ms, "cases": len(b.bulk_groups[g])}
                      for g, (t, ms) in tiles.items()},
            "bulk_one_launch_ms": merged, "bulk_per_group_ms_sum": per_group_ms, "bulk_merged": b.merged,
            "tile_merged": b.tile_all,
            "launches_per_step": 1 + len(b.kinds) + (1 if b.merged else len(b.bulk_groups)),
            "steps_done": b.engines[0].ttt - 1}


def measure_learned(args, n_train=200, K=200):
    """The learned MDF warm start on the single-case workload (FP32 form).

    Plain MDF (the workload's 20 iterations per step) records n_train steps of
    (features, accumulated force) pairs and its final slip residual; the
    network is trained on them (GPU kernels); then two copies of that state
    continue K steps, warm-started and plain, both iterating until the slip residual is
    below the level plain MDF reached in 20 iterations (median over the last
    50 training steps).  Reports both forms' step rate, mean iterations and
    residual, and Cd against the FP64 form at the same step."""
    import statistics
    import torch
    from iblbm_b200.autotune import tune_dense
    from iblbm_b200.engine import Engine
    from iblbm_b200.learned import MdfNet, collect
    total = n_train + K + 8
    cfg = workload_config(max_steps=total + 8)
    cfg.mdf_min_iterations = 20
    engs = {}
    for name in ("warm", "plain"):
        e = Engine(cfg, precision="f32")
        tune_dense(e)
        engs[name] = e
    X, T, _ = collect(engs["warm"], n_train)
    res = []
    for _ in range(n_train):
        engs["plain"].advance(1, outputs_last=False, use_graph=False)
        res.append(float(engs["plain"].d_dstats[0].item()))
    tol = statistics.median(res[-50:])
    net = MdfNet(seed=0)
    hist = net.fit(X, T, epochs=80, batch=512, lr=2e-3)
    engs["warm"].set_mlp(mode=2, net=net)
    out = {"train_pairs": int(X.shape[0]), "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1],
           "tolerance": tol}
    E = lambda: torch.cuda.Event(enable_timing=True)
    for name, e in engs.items():
        for a in e.ibm_args:
            a.mdf_min_iterations = 1
            a.mdf_tol = tol
        e.graphs = {}
        its, resid = [], []
        ev = [(E(), E()) for _ in range(K)]
        for k in range(K):
            ev[k][0].record()
            e._launch(False)
            e.join()
            ev[k][1].record()
            its.append(e.d_stats[0].clone())
            resid.append(e.d_dstats[0].clone())
        torch.cuda.synchronize()
        e.ttt += K
        ms = sum(a.elapsed_time(b) for a, b in ev) / K
        e.advance(1, outputs_last=True, use_graph=False)
        torch.cuda.synchronize()
        its = [int(x.item()) for x in its]
        resid = [float(x.item()) for x in resid]
        out[name] = {"mlups": e.N / (ms / 1e3) / 1e6, "ms_per_step": ms, "mean_iterations": statistics.mean(its),
                     "max_residual": max(resid), "steps_at_tolerance": sum(r < tol for r in resid),
                     "Cd": e.cd_cl()[0], "step": e.ttt - 1}
    ref = Engine(cfg, precision="f64")
    ref.advance(engs["warm"].ttt - 1, outputs_last=True)
    torch.cuda.synchronize()
    cd64 = ref.cd_cl()[0]
    for name in ("warm", "plain"):
        out[name]["cd_rel_err_vs_f64"] = abs(out[name]["Cd"] - cd64) / abs(cd64)
    out["iterations_saved"] = out["plain"]["mean_iterations"] - out["warm"]["mean_iterations"]
    out["speedup_vs_plain_fp32"] = out["warm"]["mlups"] / out["plain"]["mlups"]
    return out


def sweep_cd_check(cfgs, batch, steps):
    """Cd/Cl of every batched case against the FP64 plain form of the same case
    after the same number of steps (one case at a time), and for DF / MDF cases
    the interpolated marker velocities (so the marker slip) over U."""
    import torch
    from iblbm_b200.engine import Engine
    worst_cd, worst_cl, worst_u, rows = 0.0, 0.0, 0.0, []
    for cfg, eb in zip(cfgs, batch.engines):
        e = Engine(cfg, precision="f64")
        e.advance(steps, outputs_last=True)
        torch.cuda.synchronize()
        cd64, cl64 = e.cd_cl()
        cd32, cl32 = eb.cd_cl()
        rc = abs(cd32 - cd64) / abs(cd64)
        rl = abs(cl32 - cl64) / abs(cd64)
        worst_cd, worst_cl = max(worst_cd, rc), max(worst_cl, rl)
        if cfg.ibm_method in ("DF", "MDF"):
            for k in ("d_Lux", "d_Luy"):
                du = (getattr(eb, k)[: eb.Lb] - getattr(e, k)[: e.Lb]).abs().max().item()
                worst_u = max(worst_u, du / cfg.inflow_u)
        rows.append((cfg.Re, cfg.ibm_method, cfg.delta_type, cfg.collision_model, cd64, rc))
        del e
    torch.cuda.empty_cache()
    return worst_cd, worst_cl, worst_u, rows


def run_b200(args):
    import torch
    dist, rank, ws, local = _dist()
    torch.cuda.set_device(local)
    from iblbm_b200.batch import Batch
    from iblbm_b200.engine import Engine
    cfg = workload_config(max_steps=args.warmup + 4 * args.steps + 16)
    peak, peak_kind = _peaks()
    plain = measure(Engine(cfg, precision="f64"), args, dist, ws)
    single = measure(Engine(cfg, precision="f32"), args, dist, ws)
    bres, sweep = None, None
    if args.form == "chosen":
        Kb = max(20, args.steps)
        cfgs = sweep_configs(max_steps=args.warmup + 4 * Kb + 16)
        batch = Batch(cfgs)
        bres = measure_batch(batch, Kb, args.warmup, dist, ws)
        worst_cd, worst_cl, worst_u, rows = sweep_cd_check(cfgs, batch, bres["steps_done"])
        sweep = {"cases": len(cfgs), "lattice_nodes": batch.N, "max_cd_rel_err_vs_f64": worst_cd,
                 "max_cl_err_vs_f64_rel_cd": worst_cl, "max_marker_velocity_err_vs_f64_rel_u": worst_u,
                 "worst_case": max(rows, key=lambda r: r[5])[:4]}
        del batch
    learned = measure_learned(args) if args.form == "chosen" else None
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    N = 1601 * 641
    cpu = None
    if ws == 1:  # the oracle on a bounded sample of the line's own workload
        if bres:
            cpu = {k: v for k, v in oracle_sweep_sample(2).items() if k not in ("timed_s", "cases")}
        else:
            cpu = cpu_baseline(seconds=float(os.environ.get("IBLBM_CPU_SECONDS", "20")))

    def summary(m):
        return {"mlups": m["value"], "ms_per_step": m["ms_per_step"], "bulk_kernel_ms": m["dense_ms"],
                "hbm_gbs_bulk": m["achieved"], "bytes_per_lu": m["bytes_per_lu"], "band_kernel_ms": m["band_ms"],
                "whole_lattice_kernel_ms_serial": m["full_ms"], "steady_state_mlups_graph_l2_warm": m["steady"],
                "e2e_mlups": m["e2e"], "mdf_last_iterations": m["mdf"]["iter_count"], "status": m["status"],
                "Cd": m["cd"], "Cl": m["cl"], "step": m["steps_done"], "tile": m["tile"],
                "tile_ms_whole_lattice": m["tile_ms"]}

    line = {"metric": METRIC, "unit": "MLUPS", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "data": "synthetic (deterministic initial states of the workloads)"}
    single_s = summary(single)
    single_s["cd_rel_err_vs_f64"] = abs(single["cd"] - plain["cd"]) / abs(plain["cd"])
    single_s["cl_err_vs_f64_rel_cd"] = abs(single["cl"] - plain["cl"]) / abs(plain["cd"])
    if bres:
        line.update({
            "value": bres["value"], "ms_per_step": bres["ms_per_step"], "dtype": "f32",
            "config": {"workload": SWEEP_WORKLOAD + ", FP32 shifted populations with FP64 force sums; plain form: "
                                   + WORKLOAD["workload"] + ", FP64",
                       "cases": sweep["cases"], "lattice_nodes_per_step": bres and sweep["lattice_nodes"],
                       "l2": "per-step traffic ~4 GB (inputs far larger than L2), no flush",
                       "parallelism": f"replicas x{ws}"},
            "steps_batch": max(20, args.steps),
            "schedule": "one batched band launch + box passes (side stream) concurrent with one bulk launch per "
                        "collision model (cases of every band method together); CUDA graph between outputs",
            "roofline": {"bound": "hbm", "achieved": bres["achieved"], "peak": peak, "unit": "GB/s",
                         "frac": bres["achieved"] / peak,
                         "traffic": TRAFFIC_PER_NODE_F32 * (sweep["lattice_nodes"] - bres["box_nodes"]),
                         "traffic_unit": "bytes per step (all bulk launches), scaled from an ncu capture of the "
                                         "36-case part of the sweep", "peak_kind": peak_kind,
                         "kernel": "dense32_batch_kernel bulk passes of all groups (fused pull-stream+BC+macro+"
                                   "collide, FP32 shifted)", "bytes_per_lu": BYTES_PER_LU_F32,
                         "lattice_updates_per_step": bres and (sweep["lattice_nodes"] - bres["box_nodes"])},
            "e2e": {"value": bres["e2e"], "unit": "MLUPS", "h2d_bytes_per_step": bres["h2d"],
                    "d2h_bytes_per_step": bres["d2h"]},
            "gpu_launches": bres["launches_per_step"] * max(20, args.steps),
            "clocks": bres["clocks"], "wall_s_timed": bres["wall_s_timed"],
            "chosen_vs_plain": bres["value"] / plain["value"],
            "sweep": dict(sweep, steady_state_mlups_graph=bres["steady"], status_nonzero=[
                k for k, st in enumerate(bres["status"]) if st], tiles=bres["tiles"],
                bulk_ms_per_step=bres["bulk_ms"], bulk_one_launch_ms=bres["bulk_one_launch_ms"],
                bulk_per_group_ms_sum=bres["bulk_per_group_ms_sum"], bulk_merged=bres["bulk_merged"],
                tile_merged=bres["tile_merged"])})
    else:
        line.update({"value": plain["value"], "ms_per_step": plain["ms_per_step"], "dtype": "f64",
                     "config": dict(WORKLOAD, form="FP64 plain", parallelism=f"replicas x{ws}"),
                     "roofline": {"bound": "hbm", "achieved": plain["achieved"], "peak": peak, "unit": "GB/s",
                                  "frac": plain["achieved"] / peak,
                                  "traffic": TRAFFIC_PER_NODE_F64 * (N - plain["box_nodes"]),
                                  "peak_kind": peak_kind,
                                  "kernel": "dense_step_kernel bulk pass (FP64)", "bytes_per_lu": BYTES_PER_LU_F64,
                                  "lattice_updates_per_launch": N - plain["box_nodes"]},
                     "e2e": {"value": plain["e2e"], "unit": "MLUPS", "h2d_bytes_per_step": plain["e2e_h2d"],
                             "d2h_bytes_per_step": plain["e2e_d2h"]},
                     "gpu_launches": 3 * args.steps, "clocks": plain["clocks"],
                     "wall_s_timed": plain["wall_s_timed"]})
    line["cpu_baseline"] = cpu
    line["plain"] = summary(plain)
    line["plain"]["roofline_frac_bulk"] = plain["achieved"] / peak
    line["chosen_single_case"] = single_s
    if learned:
        line["learned_mdf_single_case"] = learned
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def run_profile(args):
    """A short eager run for ncu captures: warm-up steps, then args.steps timesteps
    (two kernel launches each), no graphs, no baseline, no clock sampling."""
    import torch
    from iblbm_b200.engine import Engine
    eng = Engine(workload_config(collision=args.collision, max_steps=args.warmup + args.steps + 8),
                 precision=args.precision)
    for _ in range(args.warmup + args.steps):
        eng._launch(False)
    eng.join()
    torch.cuda.synchronize()
    print(json.dumps({"profile_steps": args.steps, "status": eng.status(), "mdf": eng.mdf_stats()}))


def run_profile_batch(args):
    """A short eager batched run for ncu captures: the Re 20 and 40 part of the
    sweep (36 cases, ~1.5 GB on the device), warm-up steps then args.steps."""
    import torch
    from iblbm_b200.batch import Batch
    cfgs = [c for c in sweep_configs(max_steps=args.warmup + args.steps + 8) if c.Re in (20, 40)]
    b = Batch(cfgs)
    b.advance(1, outputs_last=False)
    for _ in range(args.warmup + args.steps):
        b._step()
    b.join()
    torch.cuda.synchronize()
    print(json.dumps({"profile_batch_steps": args.steps, "cases": len(cfgs), "nodes": b.N,
                      "status_nonzero": [k for k, st in enumerate(b.status()) if st]}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--profile", action="store_true", help="short eager run for ncu captures")
    ap.add_argument("--profile-batch", action="store_true", help="short eager batched run for ncu captures")
    ap.add_argument("--collision", default="TRT", choices=["BGK", "TRT", "CM_MRT"])
    ap.add_argument("--form", default="chosen", choices=["chosen", "plain"],
                    help="chosen: time the FP32 shifted form and the FP64 plain form; plain: FP64 only")
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"], help="form used by --profile")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_batch:
        run_profile_batch(args)
    elif args.profile:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
