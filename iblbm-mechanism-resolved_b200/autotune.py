"""Tile autotuner for the FP32 collide-stream pass.

The pass has two tile parameters: nodes per thread (4 = one 16-byte load per
population plane and warp-shuffled x-neighbours, 1 = one node per thread) and
lattice rows per CTA (1, 2, 4, 8).  Which is fastest depends on the lattice
width (row segments of 128 nodes waste the tail of the last segment), on the
collision model (register count, hence resident CTAs) and on the band
variant, so the engine times each candidate on its own lattice and keeps the
fastest.

Timing is side-effect free: a whole-lattice pass reads f[parity] and writes
f[1 - parity] (plus the velocity ring), so launching it repeatedly without
flipping the parity recomputes the same output.  Each timed launch follows a
read of a buffer larger than L2, so every candidate is timed with the
populations coming from HBM.
"""
from __future__ import annotations

CANDIDATES = [(4, 1), (4, 2), (4, 4), (4, 8), (1, 1)]


def tune_dense(engine, candidates=None, reps=5, flush_mb=256):
    """Time the whole-lattice pass of `engine` for each (nodes, rows) tile and
    apply the fastest.  Returns {tile: mean ms} and the chosen tile."""
    if not engine.f32:
        return {}, None
    torch = engine.torch
    cands = list(candidates or CANDIDATES)
    flush = torch.ones(flush_mb * 1024 * 1024 // 4, dtype=torch.float32, device=engine.dev)
    sink = torch.zeros((), dtype=torch.float32, device=engine.dev)
    engine.join()
    s = engine.stream()
    times = {}
    for tile in cands:
        engine.set_tile(*tile)
        for _ in range(2):
            engine._dense(engine.dense_full, False, s)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for e0, e1 in ev:
            torch.sum(flush, dim=0, out=sink)
            e0.record()
            engine._dense(engine.dense_full, False, s)
            e1.record()
        torch.cuda.synchronize()
        times[tile] = sum(e0.elapsed_time(e1) for e0, e1 in ev) / reps
    best = min(times, key=times.get)
    engine.set_tile(*best)
    engine.fence()
    return times, best
