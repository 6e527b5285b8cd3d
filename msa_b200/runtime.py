"""Device contexts: one msa_ctx (one CUDA stream, its device buffers) per device."""
from __future__ import annotations

import ctypes
import threading

from ._lib import check, lib


class Context:
    """Owns an msa_ctx on one device (the reference's -d/--device, src/museqa.cpp:34)."""

    def __init__(self, device: int = 0):
        self.device = device
        h = ctypes.c_void_p()
        check(lib().msa_create(device, ctypes.byref(h)))
        self.handle = h

    def close(self) -> None:
        if self.handle:
            lib().msa_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(lib().msa_launch_count(self.handle))

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib().msa_set_stream(self.handle, ctypes.c_void_p(stream_ptr or 0)), self.handle)

    def stream(self) -> int:
        return int(lib().msa_get_stream(self.handle) or 0)


_contexts: dict[int, Context] = {}
_lock = threading.Lock()
_default_device = 0


def select_device(device: int) -> None:
    """Device used by module-level calls (cuda::device::select, src/cuda.cuh)."""
    global _default_device
    _default_device = int(device)


def context(device: int | None = None) -> Context:
    dev = _default_device if device is None else int(device)
    with _lock:
        ctx = _contexts.get(dev)
        if ctx is None:
            ctx = Context(dev)
            _contexts[dev] = ctx
        return ctx
