"""Serving loop binding (gf_srv_* in include/gf_b200.h).

A :class:`Server` owns one GPU through the library's worker thread.  Requests
are ``filter`` calls (Kalman, square-root Kalman, particle filter, RBPF) that
run concurrently: Kalman requests as persistent batched launches, particle
filters continuously batched into shared per-step launches.  Every request
returns what the standalone ``filter`` returns for the same model, algorithm,
observations and seed.

    srv = Server(hbm_budget_bytes=8 << 30)
    rid = srv.submit(model, KF(), ys, want_mean=True)
    for res in srv.poll(wait_ms=100): ...
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .algorithms import KalmanFilter, ParticleFilter, RBPF, SRKalmanFilter
from .filtering import _pf_config
from .models import HierarchicalSSM, StateSpaceModel

_KIND_NAMES = {L.GF_REQ_KF: "kf", L.GF_REQ_SRKF: "srkf", L.GF_REQ_PF: "pf", L.GF_REQ_RBPF: "rbpf"}


class Server:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, host_budget_bytes: int = 0,
                 max_pending: int = 0, pf_chunk: int = 0, kf_streams: int = 0,
                 max_active_pf: int = 0):
        cfg = L.SrvConfigC(device, hbm_budget_bytes, host_budget_bytes, max_pending, pf_chunk,
                           kf_streams, max_active_pf)
        h = C.c_void_p()
        code = L.load().gf_srv_create(C.byref(cfg), C.byref(h))
        if code != L.GF_OK:
            raise L.GFError(code, "gf_srv_create failed")
        self.h = h
        self._live = {}  # id -> output buffers kept alive until the result arrives

    def _error(self, code):
        msg = L.load().gf_srv_last_error(self.h)
        msg = msg.decode() if msg else ""
        if code == L.GF_ERR_NOT_PD:
            return L.PosDefException(code, msg)
        return L.GFError(code, msg)

    def submit(self, model, algo, observations, *, seed: int = 0, tag: int = 0,
               want_steps: bool = False, want_mean: bool = False, want_cov: bool = False,
               schedule=None) -> int:
        """Queues filter(model, algo, observations) and returns the request id.

        GF_ERR_BUSY (queue full) raises GFError with that code; the caller may retry."""
        ys = L.f64(observations)
        keep = {"ys": ys}
        req = L.SrvRequestC()
        req.tag = tag
        if isinstance(algo, (KalmanFilter, SRKalmanFilter)):
            if not isinstance(model, StateSpaceModel):
                raise TypeError("Kalman filters need a linear-Gaussian StateSpaceModel")
            req.kind = L.GF_REQ_KF if isinstance(algo, KalmanFilter) else L.GF_REQ_SRKF
            mc = model._c_struct()
            keep["mc"] = mc
            req.lg = C.pointer(mc)
            req.param_steps = model.param_steps() if model.is_time_varying() else 1
            req.jitter = float(algo.jitter or 0.0)
            req.use_jitter = int(algo.jitter is not None)
            dx, dy, mdim = model.dx, model.dy, model.dx
        elif isinstance(algo, RBPF):
            if not isinstance(model, HierarchicalSSM):
                raise TypeError("RBPF needs a HierarchicalSSM")
            req.kind = L.GF_REQ_RBPF
            mc = model._c_struct()
            keep["mc"] = mc
            req.rb = C.pointer(mc)
            dy, mdim = model.dy, model.dxo + model.dz
            T = ys.size // dy
            cfg, sched, _ = _pf_config(algo.pf, T, seed, schedule)
            keep["cfg"], keep["sched"] = cfg, sched
            req.pf = C.pointer(cfg)
        elif isinstance(algo, ParticleFilter):
            if not isinstance(model, StateSpaceModel):
                raise TypeError("this particle filter needs a linear-Gaussian StateSpaceModel")
            req.kind = L.GF_REQ_PF
            mc = model._c_struct()
            keep["mc"] = mc
            req.lg = C.pointer(mc)
            req.param_steps = model.param_steps() if model.is_time_varying() else 1
            dy, mdim = model.dy, model.dx
            T = ys.size // dy
            cfg, sched, _ = _pf_config(algo, T, seed, schedule)
            keep["cfg"], keep["sched"] = cfg, sched
            req.pf = C.pointer(cfg)
        else:
            raise TypeError(f"unsupported algorithm {type(algo).__name__}")
        T = ys.size // dy
        req.T = T
        req.ys = ys.ctypes.data_as(C.POINTER(C.c_double))
        out = {}
        if want_steps:
            out["ll_steps"] = np.zeros(T)
            req.ll_steps = out["ll_steps"].ctypes.data_as(C.POINTER(C.c_double))
        if want_mean:
            out["mean"] = np.zeros(mdim)
            req.mean = out["mean"].ctypes.data_as(C.POINTER(C.c_double))
        if want_cov and req.kind in (L.GF_REQ_KF, L.GF_REQ_SRKF):
            out["cov"] = np.zeros(model.dx * model.dx)
            req.cov = out["cov"].ctypes.data_as(C.POINTER(C.c_double))
        rid = C.c_uint64()
        code = L.load().gf_srv_submit(self.h, C.byref(req), C.byref(rid))
        if code != L.GF_OK:
            raise self._error(code)
        self._live[rid.value] = out
        return rid.value

    def poll(self, max_results: int = 1024, wait_ms: int = 0):
        """Finished requests as dicts (id, tag, status, kind, ll, times, outputs)."""
        buf = (L.SrvResultC * max_results)()
        n = L.load().gf_srv_poll(self.h, buf, max_results, int(wait_ms))
        res = []
        for i in range(n):
            r = buf[i]
            out = self._live.pop(r.id, {})
            cov = out.get("cov")
            if cov is not None:
                d = int(round(np.sqrt(cov.size)))
                cov = cov.reshape(d, d, order="F")
            res.append(dict(id=r.id, tag=r.tag, status=r.status, kind=_KIND_NAMES.get(r.kind),
                            ll=r.ll, submit_ms=r.submit_ms, start_ms=r.start_ms,
                            done_ms=r.done_ms, latency_ms=r.done_ms - r.submit_ms,
                            ll_steps=out.get("ll_steps"), mean=out.get("mean"), cov=cov))
        return res

    def drain(self, timeout_ms: int = -1):
        code = L.load().gf_srv_drain(self.h, int(timeout_ms))
        if code != L.GF_OK:
            raise self._error(code)

    def stats(self) -> dict:
        m = L.SrvMetricsC()
        L.load().gf_srv_stats(self.h, C.byref(m))
        return {k: getattr(m, k) for k, _ in L.SrvMetricsC._fields_}

    def reset_stats(self):
        L.load().gf_srv_reset_stats(self.h)

    def close(self):
        if getattr(self, "h", None):
            L.load().gf_srv_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
