"""Device polynomial handles mirroring the runtime's ScalarArray (runtime/src/scalar.rs:150-445).

A ScalarArray is a view (len, rotate, slice offset / whole_len) over a torch tensor of shape
(whole_len, 8) int32 holding 32-byte Fr elements.  `poly_ptr()` produces the C-ABI PolyPtr
exactly as `PolyPtr::from(&ScalarArray)` does (core/src/poly_ptr.rs:45-86).  torch is used only
for device memory and streams.
"""
from __future__ import annotations

import numpy as np
import torch

from .native import PolyPtr


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("zkpoly_b200 kernels need a CUDA device; there is no CPU fallback")


class ScalarArray:
    def __init__(self, values: torch.Tensor, length: int | None = None, rotate: int = 0,
                 slice_info: tuple[int, int] | None = None):
        assert values.dtype == torch.int32 and values.dim() == 2 and values.shape[1] == 8
        assert values.is_contiguous()
        self.values = values
        self.len = values.shape[0] if length is None else length
        self._rotate = rotate
        self.slice_info = slice_info  # (offset, whole_len) or None

    # ---- construction
    @staticmethod
    def alloc(n: int, device="cuda") -> "ScalarArray":
        return ScalarArray(torch.empty((n, 8), dtype=torch.int32, device=device))

    @staticmethod
    def zeros(n: int, device="cuda") -> "ScalarArray":
        return ScalarArray(torch.zeros((n, 8), dtype=torch.int32, device=device))

    @staticmethod
    def from_numpy(a: np.ndarray, device="cuda") -> "ScalarArray":
        a = np.ascontiguousarray(a)
        if a.dtype == np.uint64:
            a = a.view(np.uint32).reshape(-1, 8)
        t = torch.from_numpy(np.ascontiguousarray(a.astype(np.uint32)).view(np.int32)).reshape(-1, 8)
        return ScalarArray(t.to(device).contiguous())

    # ---- view operations (scalar.rs:300-445)
    def get_rotation(self) -> int:
        return self._rotate

    def rotate(self, shift: int) -> None:
        assert self.slice_info is None
        self._rotate = (self._rotate + shift) % self.len

    def slice(self, start: int, end: int) -> "ScalarArray":
        assert 0 <= start <= end <= self.len and self.slice_info is None
        actual = (self.len + start - self._rotate) % self.len
        return ScalarArray(self.values, end - start, 0, (actual, self.len))

    def set_slice_raw(self, offset: int, length: int) -> "ScalarArray":
        whole = self.len if self.slice_info is None else self.slice_info[1]
        offset %= whole
        assert length <= whole
        info = None if (length == whole and offset == 0) else (offset, whole)
        return ScalarArray(self.values, length, 0, info)

    def whole_len(self) -> int:
        return self.len if self.slice_info is None else self.slice_info[1]

    def poly_ptr(self) -> PolyPtr:
        offset, whole = (0, self.len) if self.slice_info is None else self.slice_info
        return PolyPtr(self.values.data_ptr(), self.len, self._rotate, offset, whole)

    def index_map(self) -> np.ndarray:
        offset, whole = (0, self.len) if self.slice_info is None else self.slice_info
        return (np.arange(self.len) + whole + offset - self._rotate) % whole

    def numpy_u32(self) -> np.ndarray:
        """The view's elements in order, as (len, 8) uint32 on the host."""
        base = self.values.cpu().numpy().view(np.uint32)
        return base[self.index_map()]

    def numpy_u64(self) -> np.ndarray:
        return np.ascontiguousarray(self.numpy_u32()).view(np.uint64).reshape(-1, 4)


def stream_handle(stream=None) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


def device_words(a: np.ndarray, device="cuda") -> torch.Tensor:
    """Upload a (k, 8) uint32 / (k, 4) uint64 host array as an int32 device tensor."""
    return ScalarArray.from_numpy(a, device).values
