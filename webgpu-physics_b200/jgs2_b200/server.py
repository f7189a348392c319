"""Continuous-batching request loop over the JGS2 step (include/jgs2_server.h).

The loop itself is native (two threads in libjgs2.so); this wrapper only
submits requests and collects results."""
from __future__ import annotations

from ctypes import byref, c_uint64, c_void_p
from typing import Optional

import numpy as np

from . import _ffi
from .solver import _raise, settings_struct


def estimate_device_bytes(scene_input) -> int:
    """Device bytes the scene occupies once packed (the admission estimate)."""
    rec = scene_input.as_ctypes()
    return int(_ffi.step_lib().jgs2_estimate_device_bytes(byref(rec)))


class JGS2Server:
    def __init__(self, memoryBudgetBytes: int, device: int = 0, maxScenesPerWave: int = 0, maxWaves: int = 0):
        self._L = _ffi.step_lib()
        opts = _ffi.ServerOptions(device, int(memoryBudgetBytes), int(maxScenesPerWave), int(maxWaves))
        h = c_void_p()
        st = self._L.jgs2_server_create(byref(opts), byref(h))
        if st != 0:
            _raise(st, "jgs2_server_create failed (the memory budget must be positive).")
        self._h = h
        self._sizes = {}

    def destroy(self):
        if getattr(self, "_h", None):
            self._L.jgs2_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _error(self) -> str:
        return self._L.jgs2_server_last_error(self._h).decode() if self._h else "destroyed"

    def submit(self, scene_input, settings: Optional[dict] = None, frames: int = 1, exactIterations: int = 0) -> int:
        rec = scene_input.as_ctypes()
        s, m = settings_struct(settings)
        rid = c_uint64()
        st = self._L.jgs2_server_submit(self._h, byref(rec), byref(s), m, int(frames), int(exactIterations),
                                        byref(rid))
        if st != 0:
            _raise(st, self._error())
        self._sizes[rid.value] = scene_input.vertex_count
        return int(rid.value)

    def wait(self, request_id: int) -> dict:
        n = 4 * self._sizes.pop(request_id)
        pos = np.empty(n, dtype=np.float32)
        vel = np.empty(n, dtype=np.float32)
        res = _ffi.RequestResult()
        st = self._L.jgs2_server_wait(self._h, int(request_id), _ffi.fptr(pos), n, _ffi.fptr(vel), n, byref(res))
        if st != 0:
            _raise(st, self._error())
        out = {name: getattr(res, name) for name, _t in _ffi.RequestResult._fields_}
        out.update(positions=pos, velocities=vel)
        return out

    def drain(self):
        self._L.jgs2_server_drain(self._h)

    def stats(self) -> dict:
        out = _ffi.ServerStats()
        self._L.jgs2_server_get_stats(self._h, byref(out))
        return {name: getattr(out, name) for name, _t in _ffi.ServerStats._fields_}
