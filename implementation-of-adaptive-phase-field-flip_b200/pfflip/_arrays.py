"""Device arrays with the surface reference callers use.

The reference hands out ``warp.array`` objects; its tests and scripts call
``.numpy()``, ``.assign(ndarray)``, ``.zero_()``, ``.fill_()`` and ``.shape``
on them (e.g. tests/test_pfflip.py:182, :264-265; pfflip/io.py:22-26).
``DeviceArray`` offers that surface over a torch CUDA tensor; ``copy`` stands
in for ``wp.copy``.
"""

from __future__ import annotations

import numpy as np
import torch

_NP = {torch.float32: np.float32, torch.float64: np.float64, torch.int32: np.int32, torch.float16: np.float16,
       torch.uint8: np.uint8, torch.int64: np.int64}


class DeviceArray:
    __slots__ = ("tensor",)

    def __init__(self, tensor: torch.Tensor):
        self.tensor = tensor

    @classmethod
    def zeros(cls, shape, dtype=torch.float32, device="cuda"):
        return cls(torch.zeros(tuple(shape), dtype=dtype, device=device))

    @property
    def shape(self):
        return tuple(self.tensor.shape)

    @property
    def dtype(self):
        return _NP.get(self.tensor.dtype, None)

    @property
    def size(self):
        return self.tensor.numel()

    @property
    def device(self):
        return self.tensor.device

    def data_ptr(self):
        return self.tensor.data_ptr()

    def numpy(self) -> np.ndarray:
        return self.tensor.detach().cpu().numpy()

    def assign(self, a):
        src = torch.as_tensor(np.ascontiguousarray(np.asarray(a)).reshape(self.shape))
        self.tensor.copy_(src.to(self.tensor.dtype))
        return self

    def zero_(self):
        self.tensor.zero_()
        return self

    def fill_(self, value):
        self.tensor.fill_(value)
        return self

    def __array__(self, dtype=None, copy=None):
        a = self.numpy()
        return a if dtype is None else a.astype(dtype)

    def __repr__(self):
        return f"DeviceArray(shape={self.shape}, dtype={self.tensor.dtype}, device={self.tensor.device})"


def as_tensor(a) -> torch.Tensor:
    return a.tensor if isinstance(a, DeviceArray) else a


def copy(dst, src):
    """``dst <- src`` on the device (the reference's ``wp.copy``)."""
    as_tensor(dst).copy_(as_tensor(src))
    return dst


def to_device(a, device, dtype=torch.float32) -> DeviceArray:
    if isinstance(a, DeviceArray):
        return a
    if isinstance(a, torch.Tensor):
        return DeviceArray(a.to(device=device, dtype=dtype).contiguous())
    return DeviceArray(torch.as_tensor(np.ascontiguousarray(a)).to(device=device, dtype=dtype).contiguous())
