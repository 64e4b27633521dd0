"""Batched propagation of independent GPU_Wigner4D instances.

Not part of the reference's interface (GPU_Wigner4D.Run(), GPU_Wigner4D.py:431-541,
advances one instance per call).  ``WignerBatch(frames).Run()`` advances
every frame by its own ``timeSteps + 1`` iterations, which must be equal,
through ``wig4d_run_batch``: each step is one CUDA graph launch whose branches
are the frames' iterations, so instances of different grid sizes, dtypes and
physical parameters share the GPU concurrently.  Each frame ends with exactly
the state and result attributes its own ``Run()`` would give it.
"""
import ctypes

import torch

from . import _lib
from .device import stream_ptr


class WignerBatch:
    def __init__(self, frames):
        self.frames = list(frames)
        if len({id(f) for f in self.frames}) != len(self.frames):
            raise ValueError("WignerBatch: a frame appears twice")

    def run_device(self, iterations, histories):
        """``iterations`` Run() iterations of every frame; ``histories`` is a
        list of float64 CUDA tensors of shape (iterations, 11), one per frame
        (no host synchronisation)."""
        n = len(self.frames)
        if len(histories) != n:
            raise ValueError("WignerBatch: one history per frame")
        plans = (ctypes.c_void_p * n)(*[f._plan for f in self.frames])
        states = (ctypes.c_void_p * n)(*[f._check(f.W_init_gpu) for f in self.frames])
        hists = (ctypes.c_void_p * n)(*[h.data_ptr() for h in histories])
        _lib.call("wig4d_run_batch", plans, states, n, int(iterations), hists, stream_ptr())

    def Run(self):
        steps = {f.timeSteps for f in self.frames}
        if len(steps) > 1:
            raise ValueError("WignerBatch.Run(): frames need the same timeSteps")
        if not self.frames:
            return
        iterations = steps.pop() + 1
        hists = [torch.empty((max(iterations, 1), _lib.WIG4D_NOBS), dtype=torch.float64, device="cuda")
                 for _ in self.frames]
        self.run_device(iterations, hists)
        for f, h in zip(self.frames, hists):
            f._store_history(h.cpu().numpy()[:iterations])
