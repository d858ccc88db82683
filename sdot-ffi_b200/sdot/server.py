"""Continuous batching of SDOT solves: a thin wrapper of the C ABI's server (sdot_server_*).

    srv = Server()
    t = srv.submit(positions, target=SumOfGaussians(...), settings=Iterative(...))
    plan = srv.result(t)            # dict: weights, masses, barycentres, cost, stats, history, clusters

Requests are copied at submission; the server's worker thread admits them between two Newton steps of the
solves already running (memory budget and `max_active` permitting) and returns each as soon as it is done.
"""
import ctypes

import numpy as np

from . import _lib
from .OtProblem import Iterative
from .SdotPlanNd import solver_options


class Server:
    def __init__(self, device=None, memory_budget=0, max_active=0):
        L = _lib.load()
        cfg = _lib.ServerConfig()
        cfg.device = _lib.device_index() if device is None else int(device)
        cfg.memory_budget = int(memory_budget)
        cfg.max_active = int(max_active)
        h = ctypes.c_void_p()
        st = _lib.Status()
        _lib.raise_for(L.sdot_server_create(ctypes.byref(cfg), ctypes.byref(h), ctypes.byref(st)), st, "sdot_server_create")
        self._h = h
        self._meta = {}

    def submit(self, positions, target, nu=None, weights0=None, settings=None):
        """queue one solve; returns its ticket (never waits on the GPU)"""
        settings = settings or Iterative()
        pos = _lib.f64(positions)
        n, d = pos.shape
        t = target.normalized_version(nb_dims=d)
        from .PowerDiagram import _domain_box
        lo, hi = _domain_box(t.bounding_half_spaces(), d)
        keep = []
        sd = _lib.solve_desc(pos, nu, weights0, lo, hi, t._sdot_density(), solver_options(settings, n, d), keep)
        ticket = ctypes.c_int64()
        st = _lib.Status()
        _lib.raise_for(_lib.load().sdot_server_submit(self._h, ctypes.byref(sd), ctypes.byref(ticket), ctypes.byref(st)), st, "sdot_server_submit")
        self._meta[ticket.value] = (n, d, settings)
        return ticket.value

    def poll(self, ticket, wait_ms=0):
        """the result dict when the solve is done, else None (`wait_ms` < 0 waits)"""
        n, d, settings = self._meta[ticket]
        keep = []
        so, res = _lib.solve_out(n, d, 1024, keep)
        st = _lib.Status()
        r = _lib.load().sdot_server_poll(self._h, ticket, ctypes.byref(so), int(wait_ms), ctypes.byref(st))
        if r == 0:
            return None
        del self._meta[ticket]
        if r < 0 or st.code != _lib.SDOT_OK:
            _lib.raise_for(st.code or _lib.SDOT_ERR_ARGS, st, "sdot_server_poll")
        res["stats"] = np.array(so.stats[:])
        res["history"] = res["history"][: so.nb_history].copy()
        res["cost"] = float(res["cost"][0])
        return res

    def result(self, ticket):
        return self.poll(ticket, wait_ms=-1)

    def counters(self):
        c = (ctypes.c_int64 * 8)()
        _lib.load().sdot_server_counters(self._h, c)
        names = ["admitted", "finished", "active", "max_active", "steps", "kernel_launches", "refused_for_memory", "reserved"]
        return dict(zip(names, list(c)))

    def close(self):
        if self._h:
            _lib.load().sdot_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:          # noqa: BLE001 - interpreter shutdown
            pass
