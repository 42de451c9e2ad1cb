"""Device context (one CUDA stream and its scratch memory) of libipg."""
from __future__ import annotations

import ctypes as C
import threading
import weakref

from ._lib import check, lib


class Context:
    """Wraps an ``ipg_ctx`` (include/ipg.h: ipg_create / ipg_destroy)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().ipg_create(int(device), C.byref(h)))
        self._h = h
        self.device = device
        # handles created on this context (SNAP objects): closed before the context itself, so
        # that finalizers running in any order (a reference cycle collected at exit) never
        # reach a destroyed context
        self._dependents = weakref.WeakSet()

    def _register(self, obj):
        self._dependents.add(obj)

    @property
    def handle(self):
        return self._h

    def check(self, status):
        check(status, self._h)

    def set_stream(self, stream_ptr: int | None):
        """Runs *_dev calls on a CUDA stream given as an integer handle (e.g. torch's)."""
        self.check(lib().ipg_set_stream(self._h, C.c_void_p(stream_ptr or 0)))

    def launch_count(self) -> int:
        v = C.c_int64()
        self.check(lib().ipg_launch_count(self._h, C.byref(v)))
        return v.value

    def timing(self, on: bool):
        """Enables per-kernel device timing (CUDA events around the dominant kernels)."""
        self.check(lib().ipg_timing_enable(self._h, int(bool(on))))

    def timing_read(self, kernel: str):
        """(total milliseconds, launches) recorded for `kernel` since the last read."""
        ms = C.c_double()
        n = C.c_int64()
        self.check(lib().ipg_timing_read(self._h, kernel.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def close(self):
        if getattr(self, "_h", None):
            for d in list(getattr(self, "_dependents", ())):
                d.close()
            lib().ipg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = {}
_lock = threading.Lock()


def default_context(device: int = 0) -> Context:
    """One shared context per (thread, device)."""
    key = (threading.get_ident(), device)
    with _lock:
        ctx = _default.get(key)
        if ctx is None:
            ctx = Context(device)
            _default[key] = ctx
        return ctx
