"""Reusable device-resident plans (gf_pf_plan / gf_kf_plan) for repeated runs.

A plan uploads the model once, keeps particle / covariance buffers resident in
HBM and (unless profiling) replays one captured CUDA graph per run.  Inputs and
outputs are torch CUDA tensors (plumbing only; all compute is libgfb200).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .filtering import _pf_config


class PfPlan:
    def __init__(self, model, algo, T, *, seed=0, ctx=None, graph=True, want_steps=True,
                 simt=False, fuse=True, staged_gather=False, units=None):
        """units: True = the unit-grid tensor-core propagation, False = one block per
        tile, None = the library's default (the unit grid for Dx > 32)."""
        import torch
        self.ctx = ctx or L.default_context()
        self.model, self.algo, self.T = model, algo, int(T)
        self._mc = model._c_struct()
        self._cfg, self._sched, prec = _pf_config(algo, self.T, seed)
        h = C.c_void_p()
        flags = ((0 if graph else L.GF_PLAN_NO_GRAPH) | (L.GF_PLAN_SIMT if simt else 0)
                 | (0 if fuse else L.GF_PLAN_NO_FUSE)
                 | (L.GF_PLAN_STAGED_GATHER if staged_gather else 0) | (L.GF_PLAN_UNITS if units else 0)
                 | (L.GF_PLAN_TILES if units is False else 0))
        L.check(self.ctx.h, L.load().gf_pf_plan_create(self.ctx.h, C.byref(self._mc),
                                                       C.byref(self._cfg), self.T, flags,
                                                       C.byref(h)))
        self.h = h
        dev = f"cuda:{self.ctx.device}"
        self.ll = torch.zeros(1, dtype=torch.float64, device=dev)
        self.ll_steps = torch.zeros(self.T, dtype=torch.float64, device=dev) if want_steps else None
        self.ess = torch.zeros(self.T, dtype=torch.float64, device=dev) if want_steps else None
        self.resampled = torch.zeros(self.T, dtype=torch.int8, device=dev) if want_steps else None

    def run(self, ys_dev, noise_dev=None, unif_dev=None, states=None, log_weights=None,
            ancestors=None, means=None, paths=None):
        """paths: optional device buffer [T+1, dx, N] for every final particle's
        trajectory (device path storage; runs eagerly)."""
        o = L.PFOutC(L.ptr(self.ll), L.ptr(self.ll_steps), L.ptr(self.ess), L.ptr(self.resampled),
                     L.ptr(ancestors), L.ptr(means), L.ptr(states), L.ptr(log_weights), None,
                     L.ptr(paths))
        L.check(self.ctx.h, L.load().gf_pf_plan_run(self.h, L.ptr(ys_dev), L.ptr(noise_dev),
                                                    L.ptr(unif_dev), C.byref(o)))

    def close(self):
        if self.h:
            L.load().gf_pf_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KfPlan:
    """Batched persistent KF / SRKF plan over many uneven filters."""

    def __init__(self, models, algo, Ts, *, ctx=None, flags=0):
        import torch
        self.ctx = ctx or L.default_context()
        B = len(models)
        self.B = B
        self._mcs = (L.LGModelC * B)(*[m._c_struct() for m in models])
        self._keep = models
        self.T = np.asarray(Ts, dtype=np.int32)
        h = C.c_void_p()
        jit = algo.jitter
        L.check(self.ctx.h, L.load().gf_kf_plan_create(
            self.ctx.h, algo.algo, self._mcs, B, self.T.ctypes.data_as(C.POINTER(C.c_int32)),
            float(jit or 0.0), int(jit is not None), int(flags), C.byref(h)))
        self.h = h
        dx = np.array([m.dx for m in models])
        self.n_steps = int(self.T.sum())
        self.n_means = int((self.T * dx).sum())
        self.n_covs = int((self.T * dx * dx).sum())
        self.n_y = int(sum(int(t) * m.dy for t, m in zip(self.T, models)))
        dev = f"cuda:{self.ctx.device}"
        self.ll = torch.zeros(B, dtype=torch.float64, device=dev)
        self.status = torch.zeros(B, dtype=torch.int32, device=dev)

    def run(self, ys_dev, ll_steps=None, means=None, covs=None):
        o = L.KFOutC(L.ptr(self.ll), L.ptr(ll_steps), L.ptr(means), L.ptr(covs),
                     L.ptr(self.status))
        L.check(self.ctx.h, L.load().gf_kf_plan_run(self.h, L.ptr(ys_dev), C.byref(o)))

    def smooth(self, ys_dev, means, covs, ll_steps=None):
        """Forward run and RTS pass: means / covs receive the smoothed moments."""
        o = L.KFOutC(L.ptr(self.ll), L.ptr(ll_steps), L.ptr(means), L.ptr(covs),
                     L.ptr(self.status))
        L.check(self.ctx.h, L.load().gf_kf_plan_smooth(self.h, L.ptr(ys_dev), C.byref(o)))

    def close(self):
        if self.h:
            L.load().gf_kf_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
