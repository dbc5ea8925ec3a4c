"""Python handle on the batched / served solve loop of the C ABI (dsmc_server_* in
include/dsmc_cuda.h).

A server owns one GPU: resident particle slots, one device work queue and a device-memory budget.
`submit` admits a whole problem (raising BudgetExceeded when it does not fit), `poll` advances the
queue and returns the tickets that completed, `fetch` returns a completed request's grids,
statistics and timing and frees its device memory. A batch is a set of submits before the first
poll. Every solve runs in the CUDA library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

ERR_BUDGET = -6
ERR_STATE = -5


class BudgetExceeded(N.DsmcError):
    """Admission refused: the request does not fit the memory budget or the queue is full."""


class Server:
    def __init__(self, device: int = 0, hbm_budget: int = 80 * 10**9, max_requests: int = 16384):
        self._lib = N.lib()
        h = C.c_void_p()
        st = self._lib.dsmc_server_create(device, int(hbm_budget), int(max_requests), C.byref(h))
        if st != 0:
            msg = self._lib.dsmc_server_last_error(None)
            raise N.DsmcError(st, "dsmc_server_create", msg.decode() if msg else "")
        self.h = h
        self._shapes: dict[int, tuple[int, int]] = {}
        self._done = np.zeros(4096, dtype=np.int64)

    def close(self) -> None:
        if self.h:
            self._lib.dsmc_server_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int, where: str) -> None:
        if status != 0:
            msg = self._lib.dsmc_server_last_error(self.h)
            cls = BudgetExceeded if status == ERR_BUDGET else N.DsmcError
            raise cls(status, where, msg.decode() if msg else "")

    def set_shape(self, block: int, blocks_per_sm: int, steps_per_launch: int,
                  launches_per_graph: int) -> None:
        self._check(self._lib.dsmc_server_set_shape(self.h, block, blocks_per_sm, steps_per_launch,
                                                     launches_per_graph), "set_shape")

    def submit(self, params: N.Params, surface: N.SurfaceInputs, n: int,
               collision: N.CollisionInputs | None = None) -> int:
        t = C.c_int64()
        col = C.byref(collision.struct) if collision is not None else None
        self._check(self._lib.dsmc_server_submit(self.h, C.byref(params), C.byref(surface.struct),
                                                 col, int(n), C.byref(t)), "submit")
        self._shapes[t.value] = ((params.hd, params.ftd, params.ffd), (params.ftd, params.ffd))
        return t.value

    def poll(self) -> list[int]:
        nd = C.c_int()
        self._check(self._lib.dsmc_server_poll(self.h, N.ptr(self._done, C.c_int64),
                                               self._done.size, C.byref(nd)), "poll")
        return [int(x) for x in self._done[:nd.value]]

    def fetch(self, ticket: int, grids: bool = True) -> dict:
        shape = self._shapes.get(ticket)
        grids = grids and shape is not None     # unknown tickets: the library reports the error
        den = np.zeros(shape[0], dtype=np.uint64) if grids else None     # [hd][ftd][ffd]
        hor = np.zeros(shape[1], dtype=np.uint64) if grids else None     # [ftd][ffd]
        st = N.Stats()
        info = N.RequestInfo()
        self._check(self._lib.dsmc_server_fetch(self.h, ticket, N.ptr(den, C.c_uint64),
                                                N.ptr(hor, C.c_uint64), C.byref(st), C.byref(info)),
                    "fetch")
        self._shapes.pop(ticket, None)
        return {"density": den, "horizon": hor, "stats": st.as_dict(), "n": info.n,
                "t_submit": info.t_submit, "t_done": info.t_done,
                "latency": info.t_done - info.t_submit}

    def info(self) -> dict:
        i = N.ServerInfo()
        self._check(self._lib.dsmc_server_info_get(self.h, C.byref(i)), "info")
        return i.as_dict()

    def now(self) -> float:
        return float(self._lib.dsmc_server_now(self.h))

    def run_all(self, tickets: list[int] | None = None, grids: bool = True) -> dict[int, dict]:
        """Poll until every active request has completed; fetch and return them by ticket."""
        out: dict[int, dict] = {}
        want = None if tickets is None else set(tickets)
        while True:
            for t in self.poll():
                out[t] = self.fetch(t, grids)
            inf = self.info()
            if inf["active"] == 0 and inf["completed"] == inf["fetched"]:
                break
        return out if want is None else {t: out[t] for t in want if t in out}
