"""The device handle: `sims_field::Gpu` (crates/sims-field/src/gpu.rs:36-41) for the CUDA engine."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from ._lib import lib
from .fdtd import ERRLEN, FdtdError


@dataclass
class Options:
    """gpu.rs:16-34. Only `device` matters here; the wgpu fields have no CUDA counterpart."""

    label: str = "sims-field"
    device: int = 0


class Gpu:
    """One CUDA device and the stream runs launch on."""

    def __init__(self, handle, name):
        self._h = handle
        self.name = name

    @staticmethod
    def open(options: Options | None = None) -> "Gpu":
        """Gpu::open (gpu.rs:86-103). Raises FdtdError when no CUDA device can be opened."""
        opts = options or Options()
        L = lib()
        out = C.c_void_p()
        err = C.create_string_buffer(ERRLEN)
        code = L.fg_gpu_open(opts.device, C.byref(out), err, ERRLEN)
        if code:
            raise FdtdError(err.value.decode(), code)
        buf = C.create_string_buffer(256)
        L.fg_gpu_name(out, buf, 256)
        return Gpu(out, buf.value.decode())

    open_blocking = open

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().fg_gpu_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
