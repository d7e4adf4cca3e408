"""Tile autotuner for the FP32 collide-stream pass.

The pass comes in five tile shapes (iblbm_b200._lib.TILES): one thread per
node; one thread per 2 or 4 nodes stacked in y with all their loads issued
before the first collision; persistent pipelined CTAs with 4 or 8 rows x 128
columns per tile staged two tiles ahead in shared memory by bulk copies.
Which is fastest depends on the lattice (tiles per SM, the ragged last column
of tiles), on the collision model (register count, hence resident CTAs) and
on the band variant, so the engine times each candidate on its own lattice
and keeps the fastest.

Timing is side-effect free: a whole-lattice pass reads f[parity] and writes
f[1 - parity] (plus the velocity ring), so launching it repeatedly without
flipping the parity recomputes the same output.  Each timed launch follows a
read of a buffer larger than L2, so every candidate is timed with the
populations coming from HBM.
"""
from __future__ import annotations

CANDIDATES = ["node", "rows2", "rows4", "pipe4x2", "pipe8x2"]


def tune_dense(engine, candidates=None, reps=5, flush_mb=256):
    """Time the whole-lattice pass of `engine` for each tile shape and apply the
    fastest.  Returns {tile: mean ms} and the chosen tile."""
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
        engine.set_tile(tile)
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
    engine.set_tile(best)
    engine.fence()
    return times, best
