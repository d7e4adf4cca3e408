"""B200-native IB-LBM hot path (D2Q9 collide-stream + Guo forcing + boundary
closures + immersed-boundary marker loop) behind the reference solver's API.

Public names mirror the reference package ``iblbm``: ``SimConfig`` and
``run(cfg, verbose, callback, save_dir)``.  The compute path is hand-written
sm_100a CUDA in ``csrc/`` behind a C ABI (``include/iblbm_b200.h``), loaded with
ctypes; PyTorch CUDA tensors hold the device buffers.
"""
from .config import SimConfig


def run(cfg, verbose=True, callback=None, save_dir=None, engine=None):
    """iblbm.run drop-in: see loop.run."""
    from .loop import run as _run
    return _run(cfg, verbose=verbose, callback=callback, save_dir=save_dir, engine=engine)


__all__ = ["SimConfig", "run"]
