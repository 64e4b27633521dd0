"""Build reference-style frames (subclass sets attributes, then base __init__)."""
import numpy as np


def make_frame(cls, params, **extra):
    class Frame(cls):
        def __init__(self):
            for k, v in params.items():
                setattr(self, k, v)
            for k, v in extra.items():
                setattr(self, k, v)
            cls.__init__(self)
    return Frame()


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
