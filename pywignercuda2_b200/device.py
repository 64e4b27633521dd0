"""Device arrays with the small PyCUDA ``gpuarray`` surface the reference's
users touch (``.get()``, ``.gpudata``, ``.size``, in-place ``/=`` and ``*=``).

The storage is a PyTorch CUDA tensor (device memory and the current stream
are all PyTorch provides here); every arithmetic operation runs a kernel of
libwigner_b200.so.
"""
import numpy as np
import torch

from . import _lib


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("pywignercuda2_b200 needs a CUDA device (sm_100a); none is visible")
    _lib.load()


def stream_ptr():
    """The current PyTorch CUDA stream as a void* for the C ABI."""
    return torch.cuda.current_stream().cuda_stream


_DT = {np.dtype(np.complex128): (torch.complex128, _lib.C128),
       np.dtype(np.complex64): (torch.complex64, _lib.C64)}


class GPUArray:
    """A complex device array: ``tensor`` holds the storage."""

    def __init__(self, tensor):
        if tensor.dtype not in (torch.complex128, torch.complex64) or not tensor.is_cuda:
            raise TypeError("GPUArray needs a complex CUDA tensor")
        self.tensor = tensor

    @classmethod
    def zeros(cls, shape, dtype=np.complex128):
        tdt, _ = _DT[np.dtype(dtype)]
        return cls(torch.zeros(tuple(shape), dtype=tdt, device="cuda"))

    @classmethod
    def to_gpu(cls, arr):
        arr = np.ascontiguousarray(arr)
        return cls(torch.from_numpy(arr).cuda())

    # --- gpuarray surface -----------------------------------------------------
    @property
    def shape(self):
        return tuple(self.tensor.shape)

    @property
    def size(self):
        return self.tensor.numel()

    @property
    def dtype(self):
        return np.dtype(np.complex128 if self.tensor.dtype == torch.complex128 else np.complex64)

    @property
    def wig_dtype(self):
        return _lib.C128 if self.tensor.dtype == torch.complex128 else _lib.C64

    @property
    def gpudata(self):
        return self.tensor.data_ptr()

    @property
    def ptr(self):
        return self.tensor.data_ptr()

    def get(self):
        return self.tensor.cpu().numpy()

    def set(self, arr):
        self.tensor.copy_(torch.from_numpy(np.ascontiguousarray(arr, dtype=self.dtype)))
        return self

    def copy(self):
        return GPUArray(self.tensor.clone())

    def _scale(self, s):
        s = complex(s)
        _lib.call("wig_scale", self.ptr, self.size, self.wig_dtype, s.real, s.imag, stream_ptr())
        return self

    def __imul__(self, s):
        return self._scale(s)

    def __itruediv__(self, s):
        return self._scale(1.0 / complex(s))

    def __repr__(self):
        return "GPUArray(shape=%s, dtype=%s)" % (self.shape, self.dtype)


class DeviceScalar:
    """A reduction result; ``.get()`` returns it (as PyCUDA's ReductionKernel)."""

    def __init__(self, value):
        self._v = value

    def get(self):
        return self._v

    def __float__(self):
        return float(np.real(self._v))

    def __repr__(self):
        return repr(self._v)


def as_tensor(W):
    return W.tensor if isinstance(W, GPUArray) else W


def ptr_of(W):
    t = as_tensor(W)
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("state must be a contiguous CUDA tensor")
    return t.data_ptr()


def wdtype_of(W):
    t = as_tensor(W)
    if t.dtype == torch.complex128:
        return _lib.C128
    if t.dtype == torch.complex64:
        return _lib.C64
    raise TypeError("state must be complex128 or complex64")
