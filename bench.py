#!/usr/bin/env python
"""Benchmark of the IB-LBM per-timestep hot path on B200.

Workload (the reference's config-2 case, the largest single-case benchmark
configuration): fixed cylinder at Re = 100 on a 1601 x 641 D2Q9 lattice,
D = 40, 126 Lagrangian markers, inflow u = 0.04, TRT collision (magic
Lambda = 3/16), multi-direct forcing with the Peskin 4-point kernel (5 to 20
iterations until the slip residual < 1e-6), Dirichlet/Neumann channel
boundaries.  Inputs are the deterministic initial state of that case (no
dataset).  One "step" is one full lattice timestep: the IBM band kernel (all MDF
iterations) plus the fused collide-stream kernel.

Reported (one JSON line on rank 0):
  value       MLUPS of whole timesteps, inputs resident in HBM, L2 flushed
              between timed steps (the 150 MB population working set is close
              to the 126 MB L2, so each step is timed cold), CUDA events.
  e2e         MLUPS through the public engine with host buffers: every step
              uploads the marker positions / desired velocities from pinned
              host memory and reads the drag/lift force sums back.
  roofline    the fused collide-stream kernel against the measured HBM copy
              bandwidth: 144 algorithmic bytes per lattice update (9 FP64
              populations read + 9 written).
  cpu_baseline  the CPU oracle (a C + OpenMP restatement of the reference's
              CPU path) on a bounded sample of the same workload.

--impl reference times that CPU restatement of the reference's own path (the
reference is a Python package whose CPU path cannot travel to the GPU box).
Multi-GPU: a single case does not shard; N ranks run N independent replicas
(weak scaling), timed as the max over ranks.
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
            "l2": "flushed between timed steps (256 MB write)"}


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
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
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
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        return dist, int(os.environ.get("RANK", "0")), ws, local
    return None, 0, 1, 0


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
    threads = os.cpu_count()
    budget = float(os.environ.get("IBLBM_REF_SECONDS", "60"))
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import harness as H
    sim = H.OracleSim(workload_config())
    for _ in range(max(1, min(args.warmup, 3))):
        sim.step()
    n, t0 = 0, time.perf_counter()
    while n < args.steps:
        sim.step()
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    dt = time.perf_counter() - t0
    N = sim.s.nx * sim.s.ny
    v = N * n / dt / 1e6
    line = {"metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus, "steps": n,
            "warmup": max(1, min(args.warmup, 3)), "ms_per_step": dt / n * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (deterministic initial state)",
            "config": dict(WORKLOAD, form="reference CPU path (C + OpenMP restatement)"), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": threads, "kind": "port",
                             "sample": f"{n} timesteps of the workload ({dt:.1f} s, step cap {args.steps})"},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


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
    ev = [[E() for _ in range(4)] for _ in range(K)]
    excl = eng.d_excl[eng.parity].tolist()
    box_nodes = excl[2] * excl[3]
    main = torch.cuda.current_stream()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(torch.cuda.current_device()) as clk:
        t_wall = time.perf_counter()
        for k in range(K):
            ev[k][0].record(main)
            eng._step_overlapped(False, bulk_events=(ev[k][1], ev[k][2]))
            eng.join()
            ev[k][3].record(main)
            torch.sum(flush, dim=0, out=sink)  # read 256 MB: evict the populations from L2 (clean lines)
            eng.fence()
        torch.cuda.synchronize()
        t_wall = time.perf_counter() - t_wall
    step_ms = [ev[k][0].elapsed_time(ev[k][3]) for k in range(K)]
    dense_ms = [ev[k][1].elapsed_time(ev[k][2]) for k in range(K)]
    tot_ms = sum(step_ms)
    if dist:
        t = torch.tensor([tot_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
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
    nb = int(eng.d_count.item())
    Ke = max(10, K // 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(Ke):
        eng.d_Lx.copy_(host_in[:Lb], non_blocking=True)
        eng.d_Ly.copy_(host_in[Lb:2 * Lb], non_blocking=True)
        eng.d_dv.copy_(host_in[2 * Lb:], non_blocking=True)
        eng._launch(False)
        eng.join()
        host_out.copy_(eng.d_fib[: 2 * nb].view(nb, 2).double().sum(0), non_blocking=True)
        torch.cuda.current_stream().synchronize()
    e2e_s = time.perf_counter() - t0
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


def run_b200(args):
    import torch
    dist, rank, ws, local = _dist()
    torch.cuda.set_device(local)
    from iblbm_b200.engine import Engine
    cfg = workload_config(max_steps=args.warmup + 4 * args.steps + 16)
    peak, peak_kind = _peaks()
    plain = measure(Engine(cfg, precision="f64"), args, dist, ws)
    chosen = measure(Engine(cfg, precision="f32"), args, dist, ws) if args.form == "chosen" else None
    head = chosen or plain
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    N = 1601 * 641
    cpu = cpu_baseline(seconds=float(os.environ.get("IBLBM_CPU_SECONDS", "20"))) if ws == 1 else None
    form = "FP32 shifted populations (FP64 force sums, MDF residual norm)" if chosen else "FP64 plain"

    def summary(m):
        return {"mlups": m["value"], "ms_per_step": m["ms_per_step"], "bulk_kernel_ms": m["dense_ms"],
                "hbm_gbs_bulk": m["achieved"], "bytes_per_lu": m["bytes_per_lu"], "band_kernel_ms": m["band_ms"],
                "whole_lattice_kernel_ms_serial": m["full_ms"], "steady_state_mlups_graph_l2_warm": m["steady"],
                "e2e_mlups": m["e2e"], "mdf_last_iterations": m["mdf"]["iter_count"], "status": m["status"],
                "Cd": m["cd"], "Cl": m["cl"], "step": m["steps_done"], "tile": m["tile"],
                "tile_ms_whole_lattice": m["tile_ms"]}

    line = {"metric": METRIC, "value": head["value"], "unit": "MLUPS", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if chosen else "f64",
            "data": "synthetic (deterministic initial state of the workload)",
            "config": dict(WORKLOAD, form=form, parallelism=f"replicas x{ws}"),
            "hbm_gbs_dense": head["achieved"],
            "schedule": "band kernel + box pass (side stream) concurrent with the bulk pass",
            "roofline": {"bound": "hbm", "achieved": head["achieved"], "peak": peak, "unit": "GB/s",
                         "frac": head["achieved"] / peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": ("dense32_kernel" if chosen else "dense_step_kernel") +
                                   " bulk pass (fused pull-stream+BC+macro+collide)",
                         "bytes_per_lu": head["bytes_per_lu"], "lattice_updates_per_launch": N - head["box_nodes"]},
            "cpu_baseline": cpu,
            "e2e": {"value": head["e2e"], "unit": "MLUPS", "h2d_bytes_per_step": head["e2e_h2d"],
                    "d2h_bytes_per_step": head["e2e_d2h"]},
            "gpu_launches": 3 * args.steps,
            "clocks": head["clocks"], "wall_s_timed": head["wall_s_timed"],
            "plain": summary(plain)}
    if chosen:
        line["chosen"] = summary(chosen)
        line["chosen_vs_plain"] = chosen["value"] / plain["value"]
        line["cd_rel_err_vs_f64"] = abs(chosen["cd"] - plain["cd"]) / abs(plain["cd"])
        line["cl_err_vs_f64_rel_cd"] = abs(chosen["cl"] - plain["cl"]) / abs(plain["cd"])
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--profile", action="store_true", help="short eager run for ncu captures")
    ap.add_argument("--collision", default="TRT", choices=["BGK", "TRT", "CM_MRT"])
    ap.add_argument("--form", default="chosen", choices=["chosen", "plain"],
                    help="chosen: time the FP32 shifted form and the FP64 plain form; plain: FP64 only")
    ap.add_argument("--precision", default="f64", choices=["f64", "f32"], help="form used by --profile")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
