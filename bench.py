#!/usr/bin/env python
"""Benchmark of the IB-LBM per-timestep hot path on B200.

Two forms of the hot path are timed on one GPU:

plain   the FP64 form (the reference's arithmetic, bit for bit).
chosen  the FP32 shifted-population form (FP64 force sums and MDF residual
        norm) run batched.

Workloads:

sweep   the 72-case sweep Re {20, 40, 100, 200} x {DF, MDF, DFC} x {hat,
        Peskin-4} x {BGK, TRT, CM-MRT} of fixed cylinders on 401x161 to
        1921x961 lattices, all cases stepped together (one batched band
        launch, box passes, one collide-stream launch per collision model).
        Timed in both forms: `value` is the chosen form, `plain_sweep` the
        FP64 form on the same workload (the reference arm's workload), so the
        GPU/CPU ratio exists at equal precision.  `sweep` compares the two
        forms' Cd / Cl tail statistics after the configuration's 50 000 steps.
C2      the reference's single-case benchmark: fixed cylinder at Re = 100 on a
        1601 x 641 lattice, D = 40, 126 markers, TRT (Lambda = 3/16), MDF with
        Peskin-4 (5 to 20 iterations to a 1e-6 slip residual); `plain` (FP64)
        and `chosen_single_case` (FP32), L2 evicted between steps.
C3      oscillating cylinder, Re 100, KC 5, 1281 x 1281, DFC + Peskin-4, BGK,
        open boundary (`config3`, both forms).
C5      two settling discs, 321 x 1281, coupled MDF + Peskin-4, CM-MRT,
        Velocity-Verlet (`config5`, both forms).

Reported (one JSON line on rank 0):
  value       aggregate MLUPS of the chosen form on the sweep (device time,
              CUDA events, at least one second of timed steps); `windows` has
              the median and spread of 20-step windows.
  e2e         the same through the public API with host buffers: every step
              uploads all cases' markers from pinned host memory and reads all
              marker forces back (at least one second).
  roofline    the collide-stream launches of a step against the measured HBM
              copy bandwidth: 72 algorithmic bytes per lattice update in FP32
              (9 populations read + 9 written), 144 in FP64.
  cpu_baseline  the CPU oracle (a C + OpenMP restatement of the reference's
              CPU path) on a bounded sample of the sweep, in a fresh process.

Inputs are deterministic initial states (no dataset).  --impl reference times
the CPU restatement of the reference's own path (the reference is a Python
package whose CPU path cannot travel to the GPU box).  Multi-GPU: the sweep's
cases are partitioned over the ranks by estimated cost (no collective on the
data path; results gathered on the host), so total work is fixed (strong
scaling); the single-case workloads run as replicas.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
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
MIN_TIMED_S = 1.0     # every headline number rests on at least this much device time
CPU_PER_CASE = 4      # timed oracle steps per sweep case (both arms)
SWEEP_STEPS = 50_000  # configuration 4: steps per case


def workload_config(collision="TRT", max_steps=1_000_000):
    from iblbm_b200 import SimConfig
    return SimConfig(Re=100, NN=641, xmax=2.5, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.0625,
                     lattice_u=0.04, inflow_u=0.04, bc_type="dirichlet_neumann", delta_type="peskin4pt",
                     ibm_method="MDF", collision_model=collision, trt_magic_param=0.1875, mdf_iterations=20,
                     mdf_min_iterations=5, mdf_tolerance=1e-6, marker_spacing_factor=1.0, max_steps=max_steps,
                     use_convergence=False, check_interval=100)


def config3(max_steps=100_000, method="DFC"):
    """Oscillating cylinder, Re 100, KC 5: D = 40 on 1281 x 1281, x_c = -A sin(2 pi t / T),
    T = KC D / U = 10 000 steps, DFC + Peskin-4, BGK, open boundary (scenarios/oscillating.py:12-44)."""
    from iblbm_b200 import SimConfig
    return SimConfig(Re=100, NN=1281, xmax=1, ymax=1, cylinder_center=(0.5, 0.5), cylinder_D_ratio=0.03125,
                     lattice_u=0.02, inflow_u=0.0, bc_type="open_boundary", delta_type="peskin4pt",
                     ibm_method=method, collision_model="BGK", motion_type="oscillating", KC=5.0,
                     nx_formula="simple", marker_spacing_factor=1.0, mdf_iterations=20, mdf_min_iterations=5,
                     mdf_tolerance=1e-6, max_steps=max_steps, use_convergence=False, check_interval=100)


def config5(max_steps=300_000, rho_ratio=1.5):
    """Two settling discs (drafting, kissing, tumbling): D = 40 in a 321 x 1281 walled channel,
    centres (160, 1100) and (162, 1020) lattice units, coupled MDF + Peskin-4, CM-MRT,
    Velocity-Verlet (runtime/scenarios/sedimentation_multi.py:199-323)."""
    from iblbm_b200 import SimConfig
    return SimConfig(Re=20, NN=321, xmax=1, ymax=4, cylinder_center=(0.5, 3.4375), cylinder_D_ratio=0.125,
                     lattice_u=0.05, inflow_u=0.0, bc_type="settling_channel", delta_type="peskin4pt",
                     ibm_method="MDF", collision_model="CM_MRT", motion_type="sedimentation",
                     rho_ratio=rho_ratio, gravity=1e-5,
                     particles_config=[{"center": (0.5, 1100 / 320), "rho_ratio": rho_ratio},
                                       {"center": (0.5 + 2 / 320, 1020 / 320), "rho_ratio": rho_ratio}],
                     settling_inertia_model="explicit_history", marker_spacing_factor=1.0, max_steps=max_steps,
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
    """SM clock and throttle reasons sampled during a timed region: a thread
    runs one read-only nvidia-smi query every 200 ms (each query's output is
    complete when it exits, so no sample is lost to buffering) for this
    process's GPU, selected by UUID."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.sel = str(index)
        try:
            import torch
            u = str(torch.cuda.get_device_properties(index).uuid)
            if u:
                self.sel = u if u.startswith("GPU-") else "GPU-" + u
        except Exception:
            pass
        self.rows, self.err = [], None
        self._stop = threading.Event()
        self._t = None

    def _query(self):
        try:
            out = subprocess.run(["nvidia-smi", "-i", self.sel, f"--query-gpu={self.Q}",
                                  "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=10)
        except Exception as exc:  # no nvidia-smi on this host
            self.err = type(exc).__name__
            return
        for line in out.stdout.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)
        if out.returncode != 0 and not self.rows:
            self.err = (out.stderr.strip() or f"rc {out.returncode}")[:120]

    def _run(self):
        while not self._stop.is_set():
            self._query()
            if self.err and not self.rows:
                return
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=15)

    def summary(self):
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "error": self.err}
        mhz = [v for v in (num(r[0]) for r in self.rows) if v is not None]
        reasons = sorted({n for r in self.rows for n, v in zip(self.NAMES, r[3:7]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": num(self.rows[0][1]),
                "power_w_max": max((num(r[2]) or 0.0) for r in self.rows), "reasons": reasons,
                "samples": len(self.rows), "gpu": self.sel}


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
        dist.init_process_group("nccl" if cuda else "gloo", timeout=datetime.timedelta(seconds=300))
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


# ---- CPU baseline -------------------------------------------------------------------
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


def cpu_baseline_subprocess(per_case=CPU_PER_CASE):
    """oracle_sweep_sample in a fresh interpreter (no CUDA context, no torch
    thread pool beside the oracle's OpenMP threads), as the reference arm runs."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--cpu-sample", str(per_case)],
                         capture_output=True, text=True, timeout=1800)
    if out.returncode != 0:
        raise RuntimeError(f"CPU baseline failed: {out.stderr[-400:]}")
    return json.loads(out.stdout.strip().splitlines()[-1])


def run_reference(args):
    dist, rank, ws, _ = _dist()
    if rank != 0:
        return
    base = oracle_sweep_sample(CPU_PER_CASE)
    v, dt, threads, cfgs = base["value"], base["timed_s"], base["cores"], base["cases"]
    line = {"metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus, "steps": CPU_PER_CASE,
            "warmup": 1, "ms_per_step": dt / CPU_PER_CASE * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (deterministic initial state)",
            "config": {"workload": SWEEP_WORKLOAD, "cases": cfgs, "form": "reference CPU path (C + OpenMP "
                       "restatement of the reference's numba/numpy path), FP64"}, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": threads, "kind": "port", "sample": base["sample"]},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---- single case ---------------------------------------------------------------------
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


def _timed_flushed(eng, K, flush, sink, clk=None):
    """Per-step times (ms) of at least K overlapped steps and at least
    MIN_TIMED_S of device time: a flushed graph of up to 100 steps replayed as
    often as needed.  Returns (step_ms list, bulk_ms list, wall seconds)."""
    import torch
    Kg = min(max(K, 1), 100)
    graph, ev = _flushed_steps_graph(eng, Kg, flush, sink)
    graph.replay()  # first replay uploads the graph
    eng.parity ^= Kg & 1
    eng.ttt += Kg
    torch.cuda.synchronize()
    step_ms, dense_ms = [], []
    t_wall = time.perf_counter()
    while len(step_ms) < K or sum(step_ms) < MIN_TIMED_S * 1e3:
        graph.replay()
        eng.parity ^= Kg & 1
        eng.ttt += Kg
        torch.cuda.synchronize()
        step_ms += [ev[k][0].elapsed_time(ev[k][3]) for k in range(Kg)]
        dense_ms += [ev[k][1].elapsed_time(ev[k][2]) for k in range(Kg)]
    return step_ms, dense_ms, time.perf_counter() - t_wall


def measure(eng, args, dist, ws):
    """Time one fixed-body engine: per-step (L2 flushed) overlapped steps, the
    band kernel alone, graph-replayed steady state and the host-buffer e2e loop.
    Returns a dict of the numbers (all ranks)."""
    import torch
    N = eng.N
    eng.advance(max(args.warmup, 3), outputs_last=True)
    torch.cuda.synchronize()
    from iblbm_b200.autotune import tune_dense
    tile_ms, tile = tune_dense(eng)
    eng.advance(3, outputs_last=True)
    torch.cuda.synchronize()
    flush = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    sink = torch.zeros((), dtype=torch.float32, device="cuda")
    E = lambda: torch.cuda.Event(enable_timing=True)
    excl = eng.d_excl[eng.parity].tolist()
    box_nodes = excl[2] * excl[3]
    if dist:
        dist.barrier()
    with Clocks(torch.cuda.current_device()) as clk:
        step_ms, dense_ms, t_wall = _timed_flushed(eng, args.steps, flush, sink)
    K = len(step_ms)
    tot_ms = max_over_ranks(sum(step_ms), dist)
    dense_avg = sum(dense_ms) / K
    bpl = BYTES_PER_LU_F32 if eng.f32 else BYTES_PER_LU_F64

    # band kernel alone (serial step: band kernel then the whole lattice), for the breakdown
    sev = [[E() for _ in range(3)] for _ in range(8)]
    for k in range(8):
        eng._step_serial(False, events=sev[k])
        eng.fence()
    eng.ttt += 8
    torch.cuda.synchronize()
    ibm_ms = sum(sev[k][0].elapsed_time(sev[k][1]) for k in range(8)) / 8
    full_ms = sum(sev[k][1].elapsed_time(sev[k][2]) for k in range(8)) / 8

    # steady state: CUDA-graph replay, no flush (L2-warm; reported, not the headline)
    e0, e1 = E(), E()
    eng.advance(200, outputs_last=False)  # capture
    torch.cuda.synchronize()
    e0.record()
    eng.advance(200, outputs_last=False)
    e1.record()
    torch.cuda.synchronize()
    steady = N * 200 / (e0.elapsed_time(e1) / 1e3) / 1e6

    # end to end through the engine with host buffers, at least MIN_TIMED_S
    Lb = eng.Lb
    host_in = torch.empty(4 * Lb, dtype=torch.float64).pin_memory()
    host_in[:Lb] = torch.as_tensor(eng.st.Lx)
    host_in[Lb:2 * Lb] = torch.as_tensor(eng.st.Ly)
    host_in[2 * Lb:] = torch.as_tensor(eng.st.desired_velocity.reshape(-1))
    host_out = torch.empty(2, dtype=torch.float64).pin_memory()
    # a host program one step ahead, two pinned buffer pairs alternating (as for the batch)
    ins = [host_in, torch.empty_like(host_in).pin_memory()]
    ins[1].copy_(host_in)
    outs = [host_out, torch.empty_like(host_out).pin_memory()]
    for k in range(2):  # capture the two (parity, buffer) graphs
        eng.step_io(ins[k], outs[k])
    torch.cuda.synchronize()
    Ke = max(10, int(math.ceil(MIN_TIMED_S * 1e3 / (sum(step_ms) / K))))
    t0 = time.perf_counter()
    prev = None
    for k in range(Ke):
        ev = eng.step_io(ins[k % 2], outs[k % 2], wait=False)
        if prev is not None:
            prev.synchronize()  # the previous step's band force is in outs[(k - 1) % 2]
        prev = ev
    prev.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)  # the slowest rank
    eng.advance(1, outputs_last=True)
    torch.cuda.synchronize()
    cd, cl = eng.cd_cl()
    return {"value": N * K * ws / (tot_ms / 1e3) / 1e6, "ms_per_step": tot_ms / K, "steps": K, "dense_ms": dense_avg,
            "box_nodes": box_nodes, "bytes_per_lu": bpl,
            "achieved": bpl * (N - box_nodes) / (dense_avg / 1e3) / 1e9, "band_ms": ibm_ms, "full_ms": full_ms,
            "steady": steady, "e2e": N * Ke * ws / e2e_s / 1e6, "e2e_steps": Ke, "e2e_s": e2e_s,
            "e2e_h2d": 4 * Lb * 8, "e2e_d2h": 16, "clocks": clk.summary(), "wall_s_timed": t_wall,
            "status": eng.status(), "mdf": eng.mdf_stats(), "cd": cd, "cl": cl, "steps_done": eng.ttt - 1,
            "tile": tile, "tile_ms": tile_ms}


# ---- the sweep -------------------------------------------------------------------------
# Fixed cylinders, Re x band method x delta kernel x collision model on uneven
# lattices (Re -> NN, xmax, D/(NN-1), inflow u).
SWEEP_SIZES = {20: (161, 2.5, 0.125, 0.05), 40: (321, 2.5, 0.1, 0.05), 100: (641, 2.5, 0.0625, 0.04),
               200: (961, 2.0, 0.05, 0.04)}


SWEEP_WORKLOAD = ("batched sweep of 72 fixed-cylinder cases, Re {20,40,100,200} x {DF,MDF,DFC} x "
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


def _tune_batch(b):
    """Tile of each bulk group of an FP32 batch (the bulk pass is side-effect
    free when repeated without a parity flip), and whether one merged bulk
    launch over every case beats the per-group launches."""
    import torch
    E = lambda: torch.cuda.Event(enable_timing=True)
    main = torch.cuda.current_stream()
    tiles = {}
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
        # box kernels of the side stream: take it only on a clear win in isolation
        b.set_tile_all(best_tile, merged=merged[best_tile] < 0.95 * per_group_ms)
    b.fence()
    return tiles, merged, per_group_ms


def measure_batch(b, K, W, dist, n_total):
    """Time a batch: at least K overlapped steps and MIN_TIMED_S of device time
    (every step streams the whole sweep, several GB, far above L2, so no flush),
    per-step events around the bulk passes, graph-replayed steady state, and
    the host-buffer loop (all markers in, all marker forces out) for at least
    MIN_TIMED_S.  `n_total`: lattice nodes per step over all ranks."""
    import torch
    E = lambda: torch.cuda.Event(enable_timing=True)
    b.advance(max(W, 3), outputs_last=False)
    torch.cuda.synchronize()
    tiles, merged, per_group_ms = _tune_batch(b) if b.f32 else ({}, {}, None)
    main = torch.cuda.current_stream()
    # a probe of 10 steps sizes the timed region
    b._step()
    b.join()
    e0, e1 = E(), E()
    e0.record(main)
    for _ in range(10):
        b._step()
    b.join()
    e1.record(main)
    torch.cuda.synchronize()
    b._bump(11)
    K = max(K, int(math.ceil(MIN_TIMED_S * 1e3 / (e0.elapsed_time(e1) / 10))))
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
    step_ms = [ev[k][0].elapsed_time(ev[k][3]) for k in range(K)]
    bulk_ms = sum(ev[k][1].elapsed_time(ev[k][2]) for k in range(K)) / K
    tot_ms = max_over_ranks(sum(step_ms), dist)
    win = [sum(step_ms[s:s + 20]) for s in range(0, K - 19, 20)]
    win_mlups = sorted(b.N * 20 / (w / 1e3) / 1e6 for w in win)
    box_nodes = sum(int(x[2]) * int(x[3]) for e in b.engines for x in [e.d_excl[b.parity].tolist()])
    bpl = BYTES_PER_LU_F32 if b.f32 else BYTES_PER_LU_F64
    achieved = bpl * (b.N - box_nodes) / (bulk_ms / 1e3) / 1e9
    # steady state through one captured graph of 200 steps
    b.advance(200, outputs_last=False)
    torch.cuda.synchronize()
    e0.record()
    b.advance(200, outputs_last=False)
    e1.record()
    torch.cuda.synchronize()
    steady = b.N * 200 / (e0.elapsed_time(e1) / 1e3) / 1e6
    # host buffers: every step uploads all cases' markers and reads all marker forces back
    nin = b.marker_in.numel()
    host_in = torch.empty(nin, dtype=torch.float64).pin_memory()
    host_in.copy_(b.marker_in.cpu())
    host_out = torch.empty(b.marker_out.numel(), dtype=torch.float64).pin_memory()
    Ke = max(10, int(math.ceil(MIN_TIMED_S * 1e3 / (sum(step_ms) / K))))
    # a host program one step ahead: step k runs while the host reads step k-1's
    # forces; two pinned buffer pairs alternate (each step still copies all its
    # markers in and all its forces out)
    ins = [host_in, torch.empty_like(host_in).pin_memory()]
    ins[1].copy_(host_in)
    outs = [host_out, torch.empty_like(host_out).pin_memory()]
    for k in range(2):  # capture the two (parity, buffer) graphs
        b.step_io(ins[k], outs[k])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    prev = None
    for k in range(Ke):
        evk = b.step_io(ins[k % 2], outs[k % 2], wait=False)
        if prev is not None:
            prev.synchronize()  # the previous step's forces are in outs[(k - 1) % 2]
        prev = evk
    prev.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)  # the slowest rank
    b.advance(1, outputs_last=True)
    torch.cuda.synchronize()
    return {"value": n_total * K / (tot_ms / 1e3) / 1e6, "ms_per_step": tot_ms / K, "steps": K, "bulk_ms": bulk_ms,
            "achieved": achieved, "box_nodes": box_nodes, "steady": steady, "bytes_per_lu": bpl,
            "windows": {"size_steps": 20, "count": len(win_mlups), "median_mlups": statistics.median(win_mlups),
                        "min_mlups": win_mlups[0], "max_mlups": win_mlups[-1]},
            "e2e": n_total * Ke / e2e_s / 1e6, "e2e_steps": Ke, "e2e_s": e2e_s, "h2d": nin * 8,
            "d2h": host_out.numel() * 8, "clocks": clk.summary(), "wall_s_timed": t_wall, "status": b.status(),
            "tiles": {str(g): {"tile": t, "bulk_ms": ms, "cases": len(b.bulk_groups[g])}
                      for g, (t, ms) in tiles.items()},
            "bulk_one_launch_ms": merged, "bulk_per_group_ms_sum": per_group_ms, "bulk_merged": b.merged,
            "launches_per_step": 1 + len(b.kinds) + (1 if b.merged else len(b.bulk_groups)),
            "steps_done": b.engines[0].ttt - 1}


def sweep_accuracy(b32, b64, steps, every=500, tail=0.2):
    """Both forms of every case of the batch advanced to `steps` (the
    configuration's step count), Cd / Cl sampled every `every` steps; per case
    the FP32 form's error against the FP64 form (oracle-exact) in the tail
    statistics over the last `tail` of the run (mean Cd, mean Cl, Cl standard
    deviation, largest pointwise Cd difference), at the last step, and for DF /
    MDF the interpolated marker velocities (so the slip) at the last step.
    Returns {local case index: dict}."""
    import torch
    import numpy as np
    done = [b.engines[0].ttt - 1 for b in (b32, b64)]
    first = (max(done) // every + 1) * every
    targets = list(range(first, steps + 1, every))
    if not targets or targets[-1] != steps:
        targets.append(steps)
    hist = {"f32": [[] for _ in b32.engines], "f64": [[] for _ in b64.engines]}

    def slip_rms(e):
        """RMS over the markers of |interpolated - desired velocity| / U (DF / MDF)."""
        if e.method not in ("DF", "MDF"):
            return float("nan")
        Lb = e.Lb
        ux, uy = e.d_Lux[:Lb], e.d_Luy[:Lb]
        dv = e.d_dv[: 2 * Lb].reshape(Lb, 2)
        return float((((ux - dv[:, 0]) ** 2 + (uy - dv[:, 1]) ** 2).mean().sqrt() / e.cfg.inflow_u).item())

    for t in targets:
        for name, b in (("f32", b32), ("f64", b64)):
            b.advance(t - (b.engines[0].ttt - 1), outputs_last=True)
            torch.cuda.synchronize()
            for k, e in enumerate(b.engines):
                hist[name][k].append((t,) + e.cd_cl() + (slip_rms(e),))
    out = {}
    t_tail = steps - tail * steps
    for k, (e32, e64) in enumerate(zip(b32.engines, b64.engines)):
        h32, h64 = np.array(hist["f32"][k]), np.array(hist["f64"][k])
        bad = {n: [int(h[i, 0]) for i in range(len(h)) if not np.all(np.isfinite(h[i, 1:3]))]
               for n, h in (("f32", h32), ("f64", h64))}
        r = {"case": [e64.cfg.Re, e64.cfg.ibm_method, e64.cfg.delta_type, e64.cfg.collision_model],
             "finite": not (bad["f32"] or bad["f64"]),
             "first_nonfinite_sample_step": {n: (v[0] if v else None) for n, v in bad.items()}}
        if r["finite"]:
            m = h64[:, 0] >= t_tail
            cd32, cd64, cl32, cl64 = h32[m, 1], h64[m, 1], h32[m, 2], h64[m, 2]
            ref = abs(float(np.mean(cd64)))
            r.update({"cd_tail_mean_f64": float(np.mean(cd64)), "cl_tail_std_f64": float(np.std(cl64)),
                      "cd_tail_mean_rel_err": abs(float(np.mean(cd32) - np.mean(cd64))) / ref,
                      "cl_tail_mean_err_rel_cd": abs(float(np.mean(cl32) - np.mean(cl64))) / ref,
                      "cl_tail_std_err_rel_cd": abs(float(np.std(cl32) - np.std(cl64))) / ref,
                      "cd_tail_max_pointwise_rel_err": float(np.max(np.abs(cd32 - cd64))) / ref,
                      "cd_last_rel_err": abs(float(h32[-1, 1] - h64[-1, 1])) / abs(float(h64[-1, 1])),
                      "samples_tail": int(m.sum())})
            if e64.method in ("DF", "MDF"):
                u = float(e64.cfg.inflow_u)
                du = max((getattr(e32, a)[: e32.Lb] - getattr(e64, a)[: e64.Lb]).abs().max().item()
                         for a in ("d_Lux", "d_Luy"))
                r["marker_velocity_last_err_rel_u"] = du / u
                r["slip_rms_tail_mean_f64_rel_u"] = float(np.mean(h64[m, 3]))
                r["slip_rms_tail_mean_err_rel_u"] = abs(float(np.mean(h32[m, 3]) - np.mean(h64[m, 3])))
        out[k] = r
    return out


def _accuracy_summary(acc):
    keys = ["cd_tail_mean_rel_err", "cl_tail_mean_err_rel_cd", "cl_tail_std_err_rel_cd",
            "cd_tail_max_pointwise_rel_err", "cd_last_rel_err", "slip_rms_tail_mean_err_rel_u",
            "marker_velocity_last_err_rel_u"]
    s = {}
    for key in keys:
        vals = [(r[key], k) for k, r in acc.items() if key in r]
        if vals:
            v, k = max(vals)
            s["max_" + key] = v
            s["worst_case_" + key] = acc[k]["case"]
    s["cases_not_finite"] = [dict(case=r["case"], first_nonfinite_sample_step=r["first_nonfinite_sample_step"])
                             for r in acc.values() if not r["finite"]]
    s["cases_within_0p1pct_tail_cd"] = sum(r.get("cd_tail_mean_rel_err", 1.0) <= 1e-3 for r in acc.values())
    s["cases"] = len(acc)
    return s


# ---- configurations 3 and 5 ----------------------------------------------------------
def measure_case(cfg_fn, precision, K, W, flush, sink, e2e_steps):
    """One moving-body case in one form: device MLUPS over at least MIN_TIMED_S
    (L2 evicted between steps when the step can be graph-captured, i.e. the
    markers move on the device; otherwise eager steps, each with the host
    Newton-Euler update, wall-clock), the bulk pass's HBM rate, and e2e through
    the public run() with its per-check host outputs."""
    import torch
    from iblbm_b200 import run
    from iblbm_b200.autotune import tune_dense
    from iblbm_b200.engine import Engine
    E = lambda: torch.cuda.Event(enable_timing=True)
    eng = Engine(cfg_fn(max_steps=1_000_000), precision=precision)
    N = eng.N
    host_step = eng.st.particles is not None and not eng.dev_particles
    eng.advance(max(W, 3), outputs_last=True)
    torch.cuda.synchronize()
    tile_ms, tile = tune_dense(eng)
    eng.advance(2, outputs_last=False)
    torch.cuda.synchronize()
    bpl = BYTES_PER_LU_F32 if eng.f32 else BYTES_PER_LU_F64
    out = {"form": "FP32 shifted" if eng.f32 else "FP64 plain", "lattice_nodes": N, "bytes_per_lu": bpl,
           "tile": tile}
    if not host_step:
        step_ms, dense_ms, _ = _timed_flushed(eng, K, flush, sink)
        n = len(step_ms)
        excl = eng.d_excl[eng.parity].tolist()
        dense = sum(dense_ms) / n
        out.update({"mlups": N * n / (sum(step_ms) / 1e3) / 1e6, "ms_per_step": sum(step_ms) / n, "steps": n,
                    "bulk_kernel_ms": dense, "hbm_gbs_bulk": bpl * (N - excl[2] * excl[3]) / (dense / 1e3) / 1e9,
                    "timing": "device, one CUDA graph of overlapped steps, L2 evicted between steps"})
    else:
        ev = [(E(), E()) for _ in range(50)]
        for e0, e1 in ev:  # probe
            e0.record()
            eng._sedimentation_step(False)
            e1.record()
        torch.cuda.synchronize()
        per = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
        n = max(K, int(math.ceil(MIN_TIMED_S * 1e3 / per)))
        t0 = time.perf_counter()
        for _ in range(n):
            eng._sedimentation_step(False)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        out.update({"mlups": N * n / wall / 1e6, "ms_per_step": wall / n * 1e3, "steps": n,
                    "timing": "wall clock of eager steps: every step waits for the band kernel's particle "
                              "forces on the host (host Newton-Euler, the FP64 form's default)"})
    # serial step breakdown: band kernel, then the whole lattice
    sev = [[E() for _ in range(3)] for _ in range(8)]
    if not host_step:
        for k in range(8):
            eng._step_serial(False, events=sev[k])
            eng.fence()
        eng.ttt += 8
        torch.cuda.synchronize()
        out["band_kernel_ms"] = sum(sev[k][0].elapsed_time(sev[k][1]) for k in range(8)) / 8
        out["whole_lattice_kernel_ms_serial"] = sum(sev[k][1].elapsed_time(sev[k][2]) for k in range(8)) / 8
    out["status"] = eng.status()
    del eng
    # end to end: the public run() on a fresh engine (its first run captures the graphs, the second is timed)
    cfg = cfg_fn(max_steps=e2e_steps)
    eng = Engine(cfg_fn(max_steps=2 * e2e_steps + 16), precision=precision)
    run(cfg, verbose=False, engine=eng)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = run(cfg, verbose=False, engine=eng)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    nb = int(eng.d_count.item())
    ci = int(cfg.check_interval)
    if eng.st.particles is not None:
        h2d = 0 if eng.dev_particles else eng.Lb * 4 * 8  # markers + desired velocities of every step
        d2h = (96 * eng.P / ci) if eng.dev_particles else (nb * 4 + eng.P * nb * 2 * (4 if eng.f32 else 8))
    else:
        h2d, d2h = 0, 24 / ci  # the markers move on the device; Cd / Cl read at every check
    out["e2e"] = {"value": N * e2e_steps / wall / 1e6, "unit": "MLUPS", "steps": e2e_steps, "seconds": wall,
                  "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                  "how": "iblbm_b200.run(cfg) (the public API) with its per-check host outputs, graphs captured by "
                         "a first run on the same engine"}
    out["final_step"] = res["final_step"]
    del eng
    torch.cuda.empty_cache()
    return out


# ---- learned warm start -------------------------------------------------------------------
def measure_learned(cfg, n_train, K):
    """The learned MDF warm start (FP32 form) against plain MDF at the same
    residual, step by step.

    Plain MDF at 20 iterations per step records n_train steps of (features,
    accumulated force) pairs; the network is trained on them (GPU kernels).
    A second engine, in the same state, then steps alongside the warm-started
    one for K steps: at each step the warm-started loop iterates until its slip
    residual is down to what plain MDF reached in its 20 iterations at that
    step (20 at most).  Reports both step times (CUDA events around each
    engine's whole step), the mean iterations and the steps that reached the
    residual."""
    import torch
    from iblbm_b200.autotune import tune_dense
    from iblbm_b200.engine import Engine
    from iblbm_b200.learned import MdfNet, collect
    cfg.mdf_iterations, cfg.mdf_min_iterations, cfg.mdf_tolerance = 20, 20, 1e-12
    cfg.max_steps = n_train + K + 16
    plain, warm = Engine(cfg, precision="f32"), Engine(cfg, precision="f32")
    for e in (plain, warm):
        tune_dense(e)
    X, T, _ = collect(warm, n_train)
    for _ in range(n_train):
        plain.advance(1, outputs_last=False, use_graph=False)
    torch.cuda.synchronize()
    net = MdfNet(seed=0)
    t0 = time.perf_counter()
    hist = net.fit(X, T, epochs=40, batch=512, lr=2e-3)
    train_s = time.perf_counter() - t0
    E = lambda: torch.cuda.Event(enable_timing=True)
    # the network alone (iblbm_mlp_infer, tensor-core layers) on one body's markers
    xb = X[: warm.Lb].contiguous()
    for _ in range(10):
        net.predict(xb)
    i0, i1 = E(), E()
    i0.record()
    for _ in range(100):
        net.predict(xb)
    i1.record()
    torch.cuda.synchronize()
    infer_us = i0.elapsed_time(i1) / 100 * 1e3
    warm.set_mlp(mode=2, net=net)
    for a in warm.ibm_args:
        a.mdf_min_iterations = 1
    ms = {"plain": [], "warm": []}
    its, conv = [], []
    for k in range(K):
        for name, e in (("plain", plain), ("warm", warm)):
            if name == "warm":
                r = float(plain.d_dstats[0].item())
                for a in e.ibm_args:
                    a.mdf_tol = r * (1.0 + 1e-6)
            e0, e1 = E(), E()
            e0.record()
            e._launch(False)
            e.join()
            e1.record()
            e.ttt += 1
            torch.cuda.synchronize()
            ms[name].append(e0.elapsed_time(e1))
        its.append(int(warm.d_stats[0].item()))
        conv.append(int(warm.d_stats[2].item()))
    for e in (plain, warm):
        e.advance(1, outputs_last=True, use_graph=False)
    torch.cuda.synchronize()
    cdp, cdw = plain.cd_cl()[0], warm.cd_cl()[0]
    mp, mw = statistics.median(ms["plain"]), statistics.median(ms["warm"])
    return {"train_pairs": int(X.shape[0]), "train_epochs": 40, "train_s": train_s,
            "infer_us_per_body": infer_us, "markers": warm.Lb, "loss_first_epoch": hist[0],
            "loss_last_epoch": hist[-1], "steps_train": n_train, "steps_eval": K,
            "plain": {"iterations": 20, "ms_per_step_median": mp, "mlups": plain.N / (mp / 1e3) / 1e6},
            "warm": {"mean_iterations": statistics.mean(its), "ms_per_step_median": mw,
                     "mlups": warm.N / (mw / 1e3) / 1e6, "steps_at_plain_residual": sum(conv)},
            "iterations_saved": 20 - statistics.mean(its), "speedup_vs_plain_fp32": mp / mw,
            "cd_rel_diff_warm_vs_plain": abs(cdw - cdp) / abs(cdp),
            "how": "per-step residual matching: the warm-started loop iterates to the residual plain MDF reached "
                   "in 20 iterations at the same step"}


# ---- the run ---------------------------------------------------------------------------------
def run_b200(args):
    import torch
    dist, rank, ws, local = _dist()
    torch.cuda.set_device(local)
    from iblbm_b200.batch import Batch, gather_case_results, partition_cases
    from iblbm_b200.engine import Engine
    from iblbm_b200.state import grid_shape
    peak, peak_kind = _peaks()
    flush = torch.ones(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    sink = torch.zeros((), dtype=torch.float32, device="cuda")

    # single case, configuration 2 (replicas)
    cfg = workload_config(max_steps=10_000_000)
    e64, e32 = Engine(cfg, precision="f64"), Engine(cfg, precision="f32")
    plain = measure(e64, args, dist, ws)
    single = measure(e32, args, dist, ws)
    # both forms at the same step for the Cd / Cl comparison
    for m, e in ((plain, e64), (single, e32)):
        e.advance(max(e64.ttt, e32.ttt) - e.ttt + 1, outputs_last=True)
        torch.cuda.synchronize()
        m["cd"], m["cl"] = e.cd_cl()
        m["steps_done"] = e.ttt - 1
    del e64, e32
    torch.cuda.empty_cache()

    # the sweep, this rank's share of its cases
    acc_steps = args.accuracy_steps
    cfgs_all = sweep_configs(max_steps=max(acc_steps, 1) + 400_000)
    mine = partition_cases(cfgs_all, ws)[rank]
    n_total = sum(grid_shape(c)[0] * grid_shape(c)[1] for c in cfgs_all)
    cfgs = [cfgs_all[k] for k in mine]
    b32 = Batch(cfgs, precision="f32")
    bres = measure_batch(b32, args.steps, args.warmup, dist, n_total)
    b64 = Batch(cfgs, precision="f64")
    pres = measure_batch(b64, args.steps, args.warmup, dist, n_total)
    acc = {}
    if acc_steps > 0:
        acc_local = sweep_accuracy(b32, b64, acc_steps)
        acc = gather_case_results({mine[k]: v for k, v in acc_local.items()}, dist)
    nodes_local = b32.N
    del b32, b64
    torch.cuda.empty_cache()

    # configurations 3 and 5, both forms (replicas)
    c35 = {}
    if not args.skip_c35:
        for name, fn in (("config3", config3), ("config5", config5)):
            c35[name] = {p: measure_case(fn, p, args.steps, args.warmup, flush, sink, args.e2e_case_steps)
                         for p in ("f64", "f32")}
            f64, f32 = c35[name]["f64"], c35[name]["f32"]
            c35[name]["chosen_vs_plain"] = f32["mlups"] / f64["mlups"]
            for f in (f64, f32):
                if "hbm_gbs_bulk" in f:
                    f["roofline_frac_bulk"] = f["hbm_gbs_bulk"] / peak
    learned = None
    if args.form == "chosen" and not args.skip_learned:
        # config 3's motion sets the markers' desired velocity to their displacement (up to 32
        # lattice units per step), so its flow stays meaningful only for its first ~100 steps
        learned = {"config3_mdf": measure_learned(config3(method="MDF"), 60, 40),
                   "config2": measure_learned(workload_config(), 200, 200)}
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    cpu = cpu_baseline_subprocess() if ws == 1 else None

    def summary(m):
        return {"mlups": m["value"], "ms_per_step": m["ms_per_step"], "steps_timed": m["steps"],
                "bulk_kernel_ms": m["dense_ms"], "hbm_gbs_bulk": m["achieved"], "bytes_per_lu": m["bytes_per_lu"],
                "band_kernel_ms": m["band_ms"], "whole_lattice_kernel_ms_serial": m["full_ms"],
                "steady_state_mlups_graph_l2_warm": m["steady"], "e2e_mlups": m["e2e"], "e2e_steps": m["e2e_steps"],
                "mdf_last_iterations": m["mdf"]["iter_count"], "status": m["status"], "Cd": m["cd"], "Cl": m["cl"],
                "step": m["steps_done"], "tile": m["tile"], "tile_ms_whole_lattice": m["tile_ms"],
                "roofline_frac_bulk": m["achieved"] / peak, "clocks": m["clocks"]}

    line = {"metric": METRIC, "unit": "MLUPS", "n_gpus": ws, "steps": bres["steps"], "steps_requested": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "data": "synthetic (deterministic initial states of the workloads)"}
    single_s = summary(single)
    single_s["cd_rel_err_vs_f64"] = abs(single["cd"] - plain["cd"]) / abs(plain["cd"])
    single_s["cl_err_vs_f64_rel_cd"] = abs(single["cl"] - plain["cl"]) / abs(plain["cd"])
    line.update({
        "value": bres["value"], "ms_per_step": bres["ms_per_step"], "dtype": "f32",
        "config": {"workload": "chosen form: " + SWEEP_WORKLOAD + ", FP32 shifted populations with FP64 force sums",
                   "cases": len(cfgs_all), "lattice_nodes_per_step": n_total,
                   "l2": "per-step traffic ~4 GB (inputs far larger than L2), no flush",
                   "parallelism": f"cases partitioned over {ws} rank(s) by bytes x steps"},
        "windows": bres["windows"],
        "schedule": "one batched band launch + box passes (side stream) concurrent with one bulk launch per "
                    "collision model (cases of every band method together); eager launches in the timed region, "
                    "CUDA graphs between outputs otherwise",
        "roofline": {"bound": "hbm", "achieved": bres["achieved"], "peak": peak, "unit": "GB/s",
                     "frac": bres["achieved"] / peak,
                     "traffic": TRAFFIC_PER_NODE_F32 * (nodes_local - bres["box_nodes"]),
                     "traffic_unit": "bytes per step (all bulk launches), scaled from an ncu capture of the "
                                     "36-case part of the sweep; writes leaving L2 after a launch are not counted",
                     "peak_kind": peak_kind,
                     "kernel": "dense32_batch_kernel bulk passes of all groups (fused pull-stream+BC+macro+"
                               "collide, FP32 shifted)", "bytes_per_lu": BYTES_PER_LU_F32,
                     "lattice_updates_per_step": nodes_local - bres["box_nodes"]},
        "e2e": {"value": bres["e2e"], "unit": "MLUPS", "h2d_bytes_per_step": bres["h2d"],
                "d2h_bytes_per_step": bres["d2h"], "steps": bres["e2e_steps"], "seconds": bres["e2e_s"]},
        "gpu_launches": bres["launches_per_step"] * bres["steps"],
        "clocks": bres["clocks"], "wall_s_timed": bres["wall_s_timed"],
        "chosen_vs_plain": bres["value"] / plain["value"],
        "chosen_vs_plain_sweep": bres["value"] / pres["value"],
        "plain_sweep": {"mlups": pres["value"], "ms_per_step": pres["ms_per_step"], "steps_timed": pres["steps"],
                        "windows": pres["windows"], "bulk_ms_per_step": pres["bulk_ms"],
                        "hbm_gbs_bulk": pres["achieved"], "roofline_frac_bulk": pres["achieved"] / peak,
                        "bytes_per_lu": BYTES_PER_LU_F64, "steady_state_mlups_graph": pres["steady"],
                        "e2e": {"value": pres["e2e"], "unit": "MLUPS", "h2d_bytes_per_step": pres["h2d"],
                                "d2h_bytes_per_step": pres["d2h"], "steps": pres["e2e_steps"],
                                "seconds": pres["e2e_s"]},
                        "status_nonzero": [k for k, st in enumerate(pres["status"]) if st],
                        "launches_per_step": pres["launches_per_step"], "clocks": pres["clocks"],
                        "form": "FP64 plain (the reference's arithmetic, bit for bit per case), batched"},
        "sweep": {"steady_state_mlups_graph": bres["steady"],
                  "status_nonzero": [k for k, st in enumerate(bres["status"]) if st], "tiles": bres["tiles"],
                  "bulk_ms_per_step": bres["bulk_ms"], "bulk_one_launch_ms": bres["bulk_one_launch_ms"],
                  "bulk_per_group_ms_sum": bres["bulk_per_group_ms_sum"], "bulk_merged": bres["bulk_merged"],
                  "accuracy_vs_f64": dict(_accuracy_summary(acc), steps=acc_steps, sample_every=500,
                                          tail="last 20 % of the run") if acc else None}})
    line["cpu_baseline"] = cpu
    line["plain"] = summary(plain)
    line["chosen_single_case"] = single_s
    line.update(c35)
    if learned:
        line["learned_mdf"] = learned
    print(json.dumps(line))
    if args.accuracy_out and acc:
        with open(args.accuracy_out, "w") as fh:
            json.dump({str(k): v for k, v in acc.items()}, fh, indent=1)
    if dist:
        dist.destroy_process_group()


def run_profile(args):
    """A short eager run for ncu captures: warm-up steps, then args.steps timesteps
    of configuration 2 (or 3, 5: --profile-config), no graphs, no baseline, no
    clock sampling."""
    import torch
    from iblbm_b200.engine import Engine
    n = args.warmup + args.steps + 8
    cfg = {2: lambda: workload_config(collision=args.collision, max_steps=n), 3: lambda: config3(max_steps=n),
           5: lambda: config5(max_steps=n)}[args.profile_config]()
    eng = Engine(cfg, precision=args.precision, cluster=args.cluster)
    for _ in range(args.warmup + args.steps):
        eng._launch(False)
    eng.join()
    torch.cuda.synchronize()
    print(json.dumps({"profile_steps": args.steps, "status": eng.status(), "mdf": eng.mdf_stats()}))


def run_profile_batch(args):
    """A short eager batched run for ncu captures: the Re 20 and 40 part of the
    sweep (36 cases, ~1.5 GB on the device in FP32), warm-up steps then
    args.steps."""
    import torch
    from iblbm_b200.batch import Batch
    cfgs = [c for c in sweep_configs(max_steps=args.warmup + args.steps + 8) if c.Re in (20, 40)]
    b = Batch(cfgs, precision=args.precision if args.precision_set else "f32")
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
    ap.add_argument("--profile-config", type=int, default=2, choices=[2, 3, 5],
                    help="profile runs: configuration 2 (fixed cylinder), 3 (oscillating DFC) or 5 (two settling discs)")
    ap.add_argument("--collision", default="TRT", choices=["BGK", "TRT", "CM_MRT"])
    ap.add_argument("--form", default="chosen", choices=["chosen", "plain"])
    ap.add_argument("--precision", default=None, choices=["f64", "f32"], help="form used by the profile runs")
    ap.add_argument("--cluster", type=int, default=None, choices=[0, 2, 4, 8],
                    help="profile runs: CTAs of the FP64 MDF band step's cluster (0: one CTA; default: 8)")
    ap.add_argument("--accuracy-steps", type=int, default=SWEEP_STEPS,
                    help="steps of the sweep's FP32-vs-FP64 accuracy run (0: skip)")
    ap.add_argument("--accuracy-out", default=None, help="write the per-case accuracy table here (JSON)")
    ap.add_argument("--e2e-case-steps", type=int, default=10000, help="steps of the run() e2e of configs 3 and 5")
    ap.add_argument("--skip-c35", action="store_true")
    ap.add_argument("--skip-learned", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    args.precision_set = args.precision is not None
    if args.precision is None:
        args.precision = "f64"
    if args.warmup < 3:
        args.warmup = 3
    if args.cpu_sample is not None:
        base = oracle_sweep_sample(args.cpu_sample)
        print(json.dumps({k: v for k, v in base.items() if k not in ("timed_s", "cases")}))
    elif args.profile_batch:
        run_profile_batch(args)
    elif args.profile:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
