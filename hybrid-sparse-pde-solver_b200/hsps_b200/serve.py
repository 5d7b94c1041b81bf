"""The continuous-batching request loop (hamlss_server_*).

The reference solves one system per synchronous ``AdaptiveSelector::solve`` call
(src/adaptive/adaptive_selector.cpp:298-394).  ``Server`` accepts many requests at once:
it admits them against an HBM budget, runs large ones concurrently on several solve
lanes (one CUDA stream each) and coalesces small ones into single batched launches.
Every request still runs the adaptive ladder to its own tolerance.
"""
from __future__ import annotations

import ctypes as C
import threading
from typing import Optional

import numpy as np

from . import _abi
from ._abi import Params, ServerConfig, ServerReport, Stats, default_params, lib


def default_config(**over) -> ServerConfig:
    c = ServerConfig()
    lib().hamlss_server_config_default(C.byref(c))
    for k, v in over.items():
        if not hasattr(c, k):
            raise AttributeError(f"hamlss_server_config has no field {k!r}")
        setattr(c, k, v)
    return c


class Request:
    """One submitted solve.  Holds its host arrays until the result is collected."""

    def __init__(self, server: "Server", rid: int, arrays: tuple, x: np.ndarray):
        self.server = server
        self.id = rid
        self._arrays = arrays          # keep the CSR and b alive while the engine reads them
        self.x = x
        self.stats: Optional[Stats] = None
        self.status: Optional[int] = None

    def done(self) -> bool:
        from . import _check

        if self.status is not None:
            return True
        d = C.c_int32()
        _check(lib().hamlss_server_test(self.server.h, self.id, C.byref(d)))
        return bool(d.value)

    def wait(self, timeout: Optional[float] = None):
        """Block until the request finishes; returns (x, stats).  Raises on failure."""
        from . import HamlssError

        if self.status is None:
            st = Stats()
            rc = lib().hamlss_server_wait(self.server.h, self.id,
                                          -1.0 if timeout is None else float(timeout),
                                          C.byref(st))
            if rc == _abi.ERR_TIMEOUT:
                raise TimeoutError(f"request {self.id} still in flight")
            self.status = rc
            self.stats = st
            self._arrays = None
            self.server._forget(self.id)
            if rc != _abi.OK:
                self._error = lib().hamlss_last_error().decode(errors="replace")
        if self.status != _abi.OK:
            raise HamlssError(self.status, getattr(self, "_error", "request failed"))
        return self.x, self.stats

    def cancel(self) -> None:
        from . import _check

        _check(lib().hamlss_server_cancel(self.server.h, self.id))


class Server:
    """hamlss_server: admission by HBM footprint, concurrent solve lanes, coalescing."""

    def __init__(self, config: Optional[ServerConfig] = None, **over):
        from . import _check

        self.config = config or default_config(**over)
        h = C.c_void_p()
        _check(lib().hamlss_server_create(C.byref(self.config), C.byref(h)))
        self.h = h
        self._live = {}
        self._mu = threading.Lock()

    def submit(self, row_ptr, col_idx, values, b, x0=None,
               params: Optional[Params] = None) -> Request:
        """Queue A x = b (host CSR).  Returns a Request; x0 (default zeros) is copied."""
        from . import _check

        rp = np.ascontiguousarray(row_ptr, np.int32)
        ci = np.ascontiguousarray(col_idx, np.int32)
        v = np.ascontiguousarray(values, np.float64)
        bb = np.ascontiguousarray(b, np.float64)
        n = len(rp) - 1
        if len(bb) != n:
            raise ValueError("b does not match the matrix size")
        x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
        p = params or default_params()
        rid = C.c_int64()
        _check(lib().hamlss_server_submit(self.h, n, len(v), rp.ctypes.data, ci.ctypes.data,
                                          v.ctypes.data, bb.ctypes.data, x.ctypes.data,
                                          C.byref(p), C.byref(rid)))
        req = Request(self, rid.value, (rp, ci, v, bb, p), x)
        with self._mu:
            self._live[rid.value] = req
        return req

    def _forget(self, rid: int) -> None:
        with self._mu:
            self._live.pop(rid, None)

    def report(self) -> dict:
        from . import _check

        r = ServerReport()
        _check(lib().hamlss_server_get_report(self.h, C.byref(r)))
        return r.as_dict()

    def reset_report(self) -> None:
        from . import _check

        _check(lib().hamlss_server_reset_report(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().hamlss_server_destroy(self.h)
            self.h = None
            with self._mu:
                self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Router:
    """Requests spread over one Server per GPU: replicas, no traffic between GPUs.

    Each request goes to the server with the fewest requests queued or running (ties to
    the lowest index), so one GPU's long solves do not hold up the others."""

    def __init__(self, servers):
        self.servers = list(servers)
        if not self.servers:
            raise ValueError("a router needs at least one server")
        self.routed = [0] * len(self.servers)

    @classmethod
    def on_devices(cls, devices, **config):
        return cls([Server(device=d, **config) for d in devices])

    def _load(self, k: int) -> int:
        r = self.servers[k].report()
        return int(r["queued"]) + int(r["running"])

    def pick(self) -> int:
        return min(range(len(self.servers)), key=lambda k: (self._load(k), k))

    def submit(self, row_ptr, col_idx, values, b, x0=None, params=None):
        k = self.pick()
        req = self.servers[k].submit(row_ptr, col_idx, values, b, x0=x0, params=params)
        self.routed[k] += 1
        return req

    def report(self) -> list:
        return [s.report() for s in self.servers]

    def close(self) -> None:
        for s in self.servers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
