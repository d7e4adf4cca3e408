"""Many independent cases advancing together on one GPU (shifted FP32 form,
or the FP64 plain form with ``precision="f64"``).

A parameter sweep (Reynolds number x band method x delta kernel x collision
model, lattices of uneven size) is a set of independent cases.  Run one at a
time, each timestep of a small case is two short launches whose fixed costs
dominate, and the band kernel (one CTA, latency-bound) leaves most of the GPU
idle.  ``Batch`` advances all cases in lockstep with, per timestep:

* one launch of the batched band kernel (``iblbm_ibm_step_f32_batch``): one CTA
  per case, every case's DF / MDF / DFC on the GPU at once;
* per kind of case (collision, closure, compressibility, band method) one
  launch of the batched collide-stream pass (``iblbm_dense_step_f32_batch``)
  over the lattices of all cases of that kind.

From the second step on the schedule is the single-case overlapped one: the
band kernels and the box passes run on a high-priority side stream while the
bulk passes of all cases stream the lattices; steps between outputs are
captured once into a CUDA graph and replayed.  Each case keeps its own
``Engine`` (device buffers, host-side state, diagnostics); the batch only
drives their kernels together.  Output steps (rho, u, Cd, Cl) run through each
case's own engine.

The FP64 batch (``iblbm_ibm_step_f64_batch`` / ``iblbm_dense_step_f64_batch``)
runs the single-case FP64 device functions per case, so each case's results
are bit for bit those of its own engine; it has one tile shape (one node per
thread) and no merged bulk launch.
"""
from __future__ import annotations

from ._lib import IBM_IDS, TILES, Dense32Args, DenseArgs, Ibm32Args, IbmArgs, check
from .engine import Engine
from .state import grid_shape

MAX_KIND = 72  # cases per batched collide-stream launch (iblbm_dense_step_f32_batch)
BYTES_PER_LU = {"f32": 72, "f64": 144}  # populations read + written per lattice update


def case_cost(cfg, precision="f32", steps=None):
    """Estimated cost of a case: the population bytes its lattice streams per
    step (the bound of a batched step) times its steps (cfg.max_steps unless
    given)."""
    nx, ny, _, _ = grid_shape(cfg)
    return nx * ny * BYTES_PER_LU[precision] * int(cfg.max_steps if steps is None else steps)


def partition_cases(cfgs, world, precision="f32", steps=None):
    """Case indices of each of `world` ranks for a sweep of independent cases
    sharded over GPUs.  The cases, largest estimated cost first (ties by
    index), each go to the rank with the least cost so far (ties to the lower
    rank): the longest-processing-time rule, whose largest load exceeds the
    smallest by at most one case's cost.  Every rank computes the same
    partition from the same list, so no communication is needed; the cases
    exchange nothing, so the data path has no collective.  (The reference
    packs its sweep's cases onto GPUs by memory, scripts/experiments/
    _runner_common.py:83-152; here they are balanced by the bytes each step
    streams, which bounds a batched step's time.)  Returns a list of `world`
    sorted index lists."""
    if world < 1:
        raise ValueError(f"world={world}")
    cost = [case_cost(c, precision, steps) for c in cfgs]
    order = sorted(range(len(cfgs)), key=lambda k: (-cost[k], k))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += cost[k]
    return [sorted(p) for p in parts]


def gather_case_results(local, dist=None):
    """Per-case results of all ranks on every rank: `local` maps this rank's
    case indices to its results (any picklable value); returns the union as
    one dict ordered by case index.  Host-side, after the run (one object
    all-gather; the identity without a process group)."""
    if not dist:
        return dict(sorted(local.items()))
    got = [None] * dist.get_world_size()
    dist.all_gather_object(got, dict(local))
    out = {}
    for part in got:
        for k, v in part.items():
            if k in out:
                raise RuntimeError(f"case {k} reported by two ranks")
            out[k] = v
    return dict(sorted(out.items()))


def _copy(struct):
    return type(struct).from_buffer_copy(bytes(struct))


class Batch:
    """Independent cases on one GPU, stepped together (FP32 shifted form, or
    the FP64 plain form)."""

    def __init__(self, cfgs, device=None, tile="rows2", precision="f32"):
        if not cfgs:
            raise ValueError("empty batch")
        if precision not in ("f32", "f64"):
            raise ValueError(f"precision='{precision}' (f32 or f64)")
        if any(cfg.scenario_type == "taylor_green" for cfg in cfgs):
            raise NotImplementedError("Taylor-Green cases (a per-step closure factor) are stepped one at a time")
        self.precision = precision
        self.f32 = precision == "f32"
        self._IA, self._DA = (Ibm32Args, Dense32Args) if self.f32 else (IbmArgs, DenseArgs)
        self.engines = [Engine(cfg, device, precision=precision) for cfg in cfgs]
        for e in self.engines:
            if e.st.particles is not None:
                raise NotImplementedError("free particles (host Newton-Euler) are stepped one case at a time")
        e0 = self.engines[0]
        self.torch, self.dev, self.L = e0.torch, e0.dev, e0.L
        torch = self.torch
        self._pool_marker_arrays()
        self.C = len(self.engines)
        self.N = sum(e.N for e in self.engines)
        self.parity = 0
        self.started = False
        kinds = {}
        for k, e in enumerate(self.engines):
            c = e.case
            key = (c.collision, c.bc, c.incompressible, IBM_IDS[e.method])
            kinds.setdefault(key, []).append(k)
        self.kinds = []
        for key, idx in sorted(kinds.items()):
            for s in range(0, len(idx), MAX_KIND):
                self.kinds.append(idx[s:s + MAX_KIND])
        self.tiles = [tile] * len(self.kinds)
        # bulk passes run without the band (the box is left to the box passes),
        # so cases that differ only in band method share one bulk launch
        groups = {}
        for key, idx in sorted(kinds.items()):
            groups.setdefault(key[:3], []).extend(idx)
        self.bulk_groups = []
        for key, idx in sorted(groups.items()):
            for s in range(0, len(idx), MAX_KIND):
                self.bulk_groups.append(idx[s:s + MAX_KIND])
        self.bulk_tiles = [tile] * len(self.bulk_groups)
        # bulk passes: one launch per kind, or one launch over every case
        # (CTAs dispatch on their case's kind) when `merged`
        self.merged = False
        self.tile_all = tile
        # band argument blocks: [first step | later steps][parity], host and device copies
        self.ibm_host = {}
        self.ibm_dev = {}
        for first in (True, False):
            for p in (0, 1):
                arr = (self._IA * self.C)()
                for k, e in enumerate(self.engines):
                    a = _copy(e.ibm_args[p])
                    a.rebuild = 1 if (first or e.moving) else 0
                    a.excl_cur = 0 if first else int(e.d_excl[p].data_ptr())
                    arr[k] = a
                self.ibm_host[first, p] = arr
                raw = bytearray(bytes(arr))
                self.ibm_dev[first, p] = torch.frombuffer(raw, dtype=torch.uint8).to(self.dev)
        self._make_dense_arrays()
        self.side = torch.cuda.Stream(self.dev, priority=-1)
        self.ev_bulk = torch.cuda.Event()
        self.ev_side = torch.cuda.Event()
        self.graphs = {}

    def _pool_marker_arrays(self):
        """Place every case's marker inputs (x, y, desired velocity) in one device
        array and its per-marker outputs (IB force, DFC force) in another, so a
        host program moves all cases' markers with one copy each way."""
        torch = self.torch
        tot = sum(e.Lb for e in self.engines)
        self.marker_in = torch.zeros(4 * tot, dtype=torch.float64, device=self.dev)
        self.marker_out = torch.zeros(4 * tot, dtype=torch.float64, device=self.dev)
        o = 0
        self.marker_slices = []
        for e in self.engines:
            Lb = e.Lb
            xin, yin = self.marker_in[o:o + Lb], self.marker_in[tot + o:tot + o + Lb]
            dvin = self.marker_in[2 * tot + 2 * o:2 * tot + 2 * o + 2 * Lb]
            xin.copy_(e.d_Lx[:Lb]); yin.copy_(e.d_Ly[:Lb]); dvin.copy_(e.d_dv[:2 * Lb])
            e.d_Lx, e.d_Ly, e.d_dv = xin, yin, dvin
            e.d_Lfx = self.marker_out[o:o + Lb]
            e.d_Lfy = self.marker_out[tot + o:tot + o + Lb]
            e.d_dfc_force = self.marker_out[2 * tot + 2 * o:2 * tot + 2 * o + 2 * Lb]
            e.ibm_args = [e._make_ibm_args(p) for p in (0, 1)]
            self.marker_slices.append((o, Lb))
            o += Lb
        self.markers_total = tot

    def _make_dense_arrays(self):
        """Per kind and parity, the argument arrays of the whole-lattice and
        box passes (tile of the kind set on every entry); per bulk group and
        parity, those of the bulk passes."""
        self.dense = {}
        DA = self._DA
        for g, idx in enumerate(self.kinds):
            for p in (0, 1):
                for mode in ("full", "box"):
                    arr = (DA * len(idx))()
                    for n, k in enumerate(idx):
                        e = self.engines[k]
                        src = {"full": e.dense_full, "box": e.dense_box}[mode][p][0]
                        a = _copy(src)
                        if self.f32:
                            a.tile = TILES[self.tiles[g]]
                        a.box_blocks = 8
                        arr[n] = a
                    self.dense[g, p, mode] = arr
        for g, idx in enumerate(self.bulk_groups):
            for p in (0, 1):
                arr = (DA * len(idx))()
                for n, k in enumerate(idx):
                    a = _copy(self.engines[k].dense_bulk[p][0])
                    if self.f32:
                        a.tile = TILES[self.bulk_tiles[g]]
                    arr[n] = a
                self.dense["bulk", g, p] = arr
        if self.f32 and self.C <= MAX_KIND:
            order = [k for idx in self.kinds for k in idx]
            for p in (0, 1):
                arr = (Dense32Args * len(order))()
                for n, k in enumerate(order):
                    a = _copy(self.engines[k].dense_bulk[p][0])
                    a.tile = TILES[self.tile_all]
                    arr[n] = a
                self.dense["all", p, "bulk"] = arr

    def _need_f32(self, what):
        if not self.f32:
            raise NotImplementedError(f"{what}: the FP64 batch has one tile shape and no merged launch")

    def set_tile_all(self, tile, merged=True):
        """Tile of the single bulk launch over all cases (and whether to use it)."""
        self._need_f32("set_tile_all")
        if tile not in ("node", "rows2", "rows4"):
            raise ValueError(f"batched tile {tile!r} (node, rows2, rows4)")
        self.tile_all = tile
        self.merged = bool(merged) and self.C <= MAX_KIND
        self._make_dense_arrays()
        self.graphs = {}

    def set_tile(self, kind, tile):
        """Tile of the whole-lattice passes of one kind (the first step's)."""
        self._need_f32("set_tile")
        if tile not in ("node", "rows2", "rows4"):
            raise ValueError(f"batched tile {tile!r} (node, rows2, rows4)")
        self.tiles[kind] = tile
        self._make_dense_arrays()
        self.graphs = {}

    def set_bulk_tile(self, group, tile):
        """Tile of the bulk launch of one group (cases of one collision,
        closure and compressibility)."""
        self._need_f32("set_bulk_tile")
        if tile not in ("node", "rows2", "rows4"):
            raise ValueError(f"batched tile {tile!r} (node, rows2, rows4)")
        self.bulk_tiles[group] = tile
        self._make_dense_arrays()
        self.graphs = {}

    # ---------------------------------------------------------------------------------
    def _band(self, first, stream):
        p = self.parity
        if self.f32:
            rc = self.L.iblbm_ibm_step_f32_batch(self.ibm_host[first, p], self.ibm_dev[first, p].data_ptr(), self.C,
                                                 stream)
        else:
            rc = self.L.iblbm_ibm_step_f64_batch(self.ibm_host[first, p], self.ibm_dev[first, p].data_ptr(), self.C,
                                                 stream)
        check(rc, "batched band step")

    def _dense_call(self, arr, stream):
        if self.f32:
            check(self.L.iblbm_dense_step_f32_batch(arr, len(arr), stream), "iblbm_dense_step_f32_batch")
        else:
            check(self.L.iblbm_dense_step_f64_batch(arr, len(arr), stream), "iblbm_dense_step_f64_batch")

    def _dense(self, g, mode, stream):
        self._dense_call(self.dense[g, self.parity, mode], stream)

    def _bulk(self, g, stream):
        self._dense_call(self.dense["bulk", g, self.parity], stream)

    def _sync_engines(self):
        for e in self.engines:
            e.parity = self.parity
            e.rebuild_next = False

    def _step_first(self):
        """Serial step with band rebuild: band kernels, then every whole lattice."""
        torch = self.torch
        main = torch.cuda.current_stream(self.dev)
        s = main.cuda_stream
        self._band(True, s)
        for g in range(len(self.kinds)):
            self._dense(g, "full", s)
        self.parity ^= 1
        self.ev_bulk.record(main)
        self.ev_side.record(main)
        self.started = True

    def _step(self, bulk_events=None):
        """Overlapped step: band kernels and box passes on the side stream,
        bulk passes of every group on the current stream (bulk_events: two
        events recorded around the bulk passes)."""
        torch = self.torch
        main = torch.cuda.current_stream(self.dev)
        side = self.side
        side.wait_event(self.ev_bulk)
        self._band(False, side.cuda_stream)
        for g in range(len(self.kinds)):
            self._dense(g, "box", side.cuda_stream)
        main.wait_event(self.ev_side)
        self.ev_side.record(side)
        if bulk_events:
            bulk_events[0].record(main)
        if self.merged:
            self._dense("all", "bulk", main.cuda_stream)
        else:
            for g in range(len(self.bulk_groups)):
                self._bulk(g, main.cuda_stream)
        if bulk_events:
            bulk_events[1].record(main)
        self.ev_bulk.record(main)
        self.parity ^= 1

    def join(self):
        self.torch.cuda.current_stream(self.dev).wait_event(self.ev_side)

    def fence(self):
        main = self.torch.cuda.current_stream(self.dev)
        self.ev_bulk.record(main)
        self.ev_side.record(main)

    def _graph(self, length):
        key = (self.parity, length)
        g = self.graphs.get(key)
        if g is None:
            torch = self.torch
            cap = torch.cuda.Stream(self.dev)
            cap.wait_stream(torch.cuda.current_stream(self.dev))
            cap.wait_stream(self.side)
            g = torch.cuda.CUDAGraph()
            p0 = self.parity
            with torch.cuda.stream(cap):
                with torch.cuda.graph(g, stream=cap):
                    self.ev_bulk.record(cap)
                    self.ev_side.record(cap)
                    for _ in range(length):
                        self._step()
                    self.join()
            torch.cuda.current_stream(self.dev).wait_stream(cap)
            self.parity = p0
            self.graphs[key] = g
        return g

    def step_io(self, host_in, host_out, wait=True):
        """One timestep with its host I/O, as a host program drives the batch:
        every case's markers (the pooled marker_in layout) from pinned host
        memory host_in, the step, and every case's per-marker forces (marker_out)
        into pinned host memory host_out.  Replayed from one CUDA graph per
        parity and buffer pair (copies included).  With wait, returns when
        host_out holds this step's forces; otherwise returns at once with an
        event that completes then, so a host program can run one step ahead
        (alternating two buffer pairs, as step k+1's copy-in may run while the
        host still reads step k's forces)."""
        torch = self.torch
        if not self.started:
            self.advance(1, outputs_last=False)
        self.join()  # before a capture: events recorded inside one cannot be waited on outside
        main = torch.cuda.current_stream(self.dev)
        key = ("io", self.parity, host_in.data_ptr(), host_out.data_ptr())
        g = self.graphs.get(key)
        if g is None:
            cap = torch.cuda.Stream(self.dev)
            cap.wait_stream(main)
            cap.wait_stream(self.side)
            g = torch.cuda.CUDAGraph()
            p0 = self.parity
            with torch.cuda.stream(cap):
                with torch.cuda.graph(g, stream=cap):
                    self.ev_bulk.record(cap)
                    self.ev_side.record(cap)  # the bulk passes need no marker data: they start at once
                    self.side.wait_event(self.ev_bulk)
                    with torch.cuda.stream(self.side):  # markers in ahead of the band kernels (same stream)
                        self.marker_in.copy_(host_in, non_blocking=True)
                    self._step()
                    self.join()
                    host_out.copy_(self.marker_out, non_blocking=True)
            main.wait_stream(cap)
            self.parity = p0
            self.graphs[key] = g
        g.replay()
        self.parity ^= 1
        self._bump(1)
        self.fence()
        self._sync_engines()
        if wait:
            main.synchronize()
            return None
        done = torch.cuda.Event()
        done.record(main)
        return done

    def advance(self, nsteps, outputs_last=True, use_graph=True):
        """Advance every case nsteps timesteps; with outputs_last the last step
        writes each case's rho / u / f* (read with its engine's cd_cl, read_state)."""
        if nsteps <= 0:
            return
        if not self.started:
            self._step_first()
            nsteps -= 1
            self._bump(1)
        body = nsteps - 1 if (outputs_last and nsteps > 0) else nsteps
        if body > 0:
            if use_graph and body >= 4:
                self.join()
                self._graph(body).replay()
                self.parity ^= (body & 1)
                self.fence()
            else:
                for _ in range(body):
                    self._step()
                self.join()
            self._bump(body)
        if outputs_last and nsteps > 0:
            self.join()
            self._sync_engines()
            for e in self.engines:
                e._step_serial(outputs=True)
            self.parity ^= 1
            self.fence()
            self._bump(1)
            for e in self.engines:
                e.last_out_step = e.ttt - 1
        self._sync_engines()

    def _bump(self, n):
        for e in self.engines:
            e.ttt += n

    def status(self):
        return [e.status() for e in self.engines]

    def cd_cl(self):
        return [e.cd_cl() for e in self.engines]
