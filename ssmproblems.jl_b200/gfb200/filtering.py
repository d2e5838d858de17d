"""``filter(model, algo, ys)`` and friends on the B200 library.

Mirrors GeneralisedFilters.filter (GeneralisedFilters.jl:58-84): returns
``(state, log_likelihood)`` with ``state`` an ``MvNormal`` (KF / SRKF) or a
``ParticleDistribution`` (PF / RBPF).  Every call goes through the C ABI of
libgfb200.so; unsupported models or options raise instead of falling back.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .algorithms import (AlternatingResampler, AuxiliaryParticleFilter, ESSResampler, KalmanFilter,
                         KalmanSmoother, ParticleFilter, RBPF, SRKalmanFilter)
from .models import HierarchicalSSM, StateSpaceModel


class MvNormal:
    """Filtered Gaussian N(mu, Sigma) (Distributions.MvNormal stand-in)."""

    def __init__(self, mu, Sigma):
        self.mu = np.asarray(mu)
        self.Sigma = np.asarray(Sigma)

    def mean(self):
        return self.mu

    def cov(self):
        return self.Sigma


class ParticleDistribution:
    """containers.jl:125-141: particles with normalised log-weights (and the
    per-step diagnostics of the run)."""

    def __init__(self, particles, log_weights, **info):
        self.particles = particles
        self.log_weights = log_weights
        for k, v in info.items():
            setattr(self, k, v)

    def weights(self):
        """StatsBase.weights(state) -> softmax(log_weights) (containers.jl:140-144)."""
        lw = np.asarray(self.log_weights, dtype=np.float64)
        w = np.exp(lw - lw.max())
        return w / w.sum()

    def __len__(self):
        return len(self.log_weights)


def _resolve_ctx(ctx):
    return ctx if ctx is not None else L.default_context()


def _rs_params(algo: ParticleFilter, T: int):
    rs = algo.resampler
    sched = None
    if isinstance(rs, AlternatingResampler):
        sched = np.asarray(rs.schedule(T), dtype=np.int8)
        threshold, base = 1.0, rs.resampler
    elif isinstance(rs, ESSResampler):
        threshold, base = rs.threshold, rs.resampler
    else:
        threshold, base = 1.0, rs
    return threshold, base.kind, sched


def _pf_config(algo: ParticleFilter, T: int, seed: int, schedule=None, lookahead=0):
    threshold, kind, sched = _rs_params(algo, T)
    if schedule is not None:
        sched = np.asarray(schedule, dtype=np.int8)
    prec = L.GF_PREC_F64 if algo.precision in ("f64", np.float64, "float64") else L.GF_PREC_F32
    conv = L.GF_CONV_CUDAEXT if algo.convention == "cudaext" else L.GF_CONV_CPU
    cfg = L.PFConfigC(algo.N, kind, conv, threshold, prec, algo.proposal.kind,
                      float(getattr(algo.proposal, "k", 1.0)), int(seed) & (2**64 - 1),
                      None if sched is None else sched.ctypes.data_as(C.POINTER(C.c_int8)),
                      int(lookahead))
    return cfg, sched, prec


class AncestorCallback:
    """AncestorCallback (callbacks.jl:83-111): pass as filter(..., callback=cb); the
    device path storage fills cb.tree, whose get_ancestry gives every final
    particle's trajectory."""

    def __init__(self, tree=None):
        self.tree = tree


class DenseAncestorCallback:
    """DenseAncestorCallback (callbacks.jl:47-81): pass as filter(..., callback=cb);
    cb.container is the DenseParticleContainer of the run."""

    def __init__(self, container=None):
        self.container = container


class ParticleTree:
    """The trajectories kept by the device path storage: paths [T+1, N, dx]."""

    def __init__(self, paths):
        self.paths = paths

    def __len__(self):
        return self.paths.shape[1]


class DenseParticleContainer:
    """DenseParticleContainer (containers.jl:296-419): initial_states [N, dx],
    states [T, N, dx] (times 1..T), weights [T, N] (normalised log-weights after
    each update), ancestors [T, N] (1-based)."""

    def __init__(self, history, log_weights, ancestors, ctx=None):
        self._hist = history  # [T+1, dx, N], the library's layout
        self.weights = log_weights
        self.ancestors = ancestors
        self._ctx = ctx

    @property
    def initial_states(self):
        return self._hist[0].T

    @property
    def states(self):
        return self._hist[1:].transpose(0, 2, 1)


def get_ancestry(container, i=None, *, ctx=None):
    """get_ancestry(container, i) (containers.jl:421-440, 587-631): the trajectory
    [T+1, dx] of final particle i (1-based), or of every final particle
    ([N, T+1, dx]) when i is None.  A ParticleTree already holds them all."""
    if isinstance(container, ParticleTree):
        paths = container.paths.transpose(1, 0, 2)
        return paths if i is None else paths[i - 1]
    if not isinstance(container, DenseParticleContainer):
        raise TypeError("get_ancestry takes a DenseParticleContainer or a ParticleTree")
    ctx = _resolve_ctx(ctx if ctx is not None else container._ctx)
    hist = container._hist
    T1, dx, N = hist.shape
    prec = L.GF_PREC_F64 if hist.dtype == np.float64 else L.GF_PREC_F32
    idx = None if i is None else np.atleast_1d(np.asarray(i, dtype=np.int32))
    M = N if idx is None else idx.size
    out = np.empty((T1, dx, M), hist.dtype)
    anc = np.ascontiguousarray(container.ancestors, dtype=np.int32)
    L.check(ctx.h, L.load().gf_pf_dense_ancestry(ctx.h, T1 - 1, N, dx, prec, L.ptr(np.ascontiguousarray(hist)),
                                                 L.ptr(anc), M, L.ptr(idx), L.GF_MEM_HOST, L.ptr(out)))
    paths = out.transpose(2, 0, 1)  # [M, T+1, dx]
    return paths if i is None or np.ndim(i) > 0 else paths[0]


def filter(model, algo, observations, *, seed: int = 0, noise=None, uniforms=None,
           ctx=None, want_ancestors=False, want_means=False, schedule=None, want_paths=False,
           callback=None):
    """filter([rng,] model, algo, observations) -> (state, ll).

    seed     : Philox key of the in-kernel noise and uniforms (the reference's rng)
    noise    : optional injected standard normals [(T+1), dx, N] (step 0 = prior)
    uniforms : optional injected resampling uniforms ([T] systematic, else [T, N])
    want_paths: keep the ancestry on the device (AncestorCallback / ParticleTree) and
                return every final particle's trajectory as state.paths [T+1, N, dx]
    callback : AncestorCallback() (fills cb.tree) or DenseAncestorCallback() (fills
               cb.container); particle filters only
    """
    ctx = _resolve_ctx(ctx)
    ys = L.f64(observations)
    if isinstance(algo, AuxiliaryParticleFilter) and isinstance(algo.pf, RBPF):
        # AuxiliaryParticleFilter(RBPF(pf, KalmanFilter()), pp) (rbpf.jl:86-124)
        la = algo.weight_strategy.pp.lookahead
        if callback is not None:
            if not isinstance(callback, (AncestorCallback, DenseAncestorCallback)):
                raise TypeError(f"unsupported callback {type(callback).__name__}")
            dense = isinstance(callback, DenseAncestorCallback)
            st, ll = _rbpf(model, algo.pf, ys, seed, noise, uniforms, ctx, True, want_means, schedule,
                           want_paths=not dense, want_history=dense, lookahead=la)
            if dense:
                callback.container = DenseParticleContainer(st._history, st._lw_history, st.ancestors, ctx)
            else:
                callback.tree = ParticleTree(st.paths)
            return st, ll
        return _rbpf(model, algo.pf, ys, seed, noise, uniforms, ctx, want_ancestors, want_means,
                     schedule, lookahead=la)
    if callback is not None and isinstance(algo, RBPF):
        if not isinstance(callback, (AncestorCallback, DenseAncestorCallback)):
            raise TypeError(f"unsupported callback {type(callback).__name__}")
        dense = isinstance(callback, DenseAncestorCallback)
        st, ll = _rbpf(model, algo, ys, seed, noise, uniforms, ctx, True, want_means, schedule,
                       want_paths=not dense, want_history=dense)
        if dense:
            callback.container = DenseParticleContainer(st._history, st._lw_history, st.ancestors, ctx)
        else:
            callback.tree = ParticleTree(st.paths)
        return st, ll
    if callback is not None:
        if not isinstance(algo, (ParticleFilter, AuxiliaryParticleFilter)):
            raise TypeError("ancestry callbacks are built for the particle filters")
        if isinstance(callback, AncestorCallback):
            st, ll = filter(model, algo, observations, seed=seed, noise=noise, uniforms=uniforms, ctx=ctx,
                            want_ancestors=want_ancestors, want_means=want_means, schedule=schedule,
                            want_paths=True)
            callback.tree = ParticleTree(st.paths)
            return st, ll
        if isinstance(callback, DenseAncestorCallback):
            pf = algo.pf if isinstance(algo, AuxiliaryParticleFilter) else algo
            la = algo.weight_strategy.pp.lookahead if isinstance(algo, AuxiliaryParticleFilter) else 0
            st, ll = _pf(model, pf, ys, seed, noise, uniforms, ctx, True, want_means, schedule,
                         want_paths, lookahead=la, want_history=True)
            callback.container = DenseParticleContainer(st._history, st._lw_history, st.ancestors, ctx)
            return st, ll
        raise TypeError(f"unsupported callback {type(callback).__name__}")
    if isinstance(algo, (KalmanFilter, SRKalmanFilter)):
        if not isinstance(model, StateSpaceModel):
            raise TypeError("Kalman filters need a linear-Gaussian StateSpaceModel")
        res = filter_batch([model], algo, [ys], ctx=ctx)
        return res[0]
    if isinstance(algo, RBPF):
        return _rbpf(model, algo, ys, seed, noise, uniforms, ctx, want_ancestors, want_means,
                     schedule)
    if isinstance(algo, ParticleFilter):
        return _pf(model, algo, ys, seed, noise, uniforms, ctx, want_ancestors, want_means,
                   schedule, want_paths)
    if isinstance(algo, AuxiliaryParticleFilter):
        return _pf(model, algo.pf, ys, seed, noise, uniforms, ctx, want_ancestors, want_means,
                   schedule, want_paths, lookahead=algo.weight_strategy.pp.lookahead)
    raise TypeError(f"unsupported algorithm {type(algo).__name__}")


def _pf(model, algo, ys, seed, noise, uniforms, ctx, want_anc, want_means, schedule,
        want_paths=False, lookahead=0, want_history=False):
    if not isinstance(model, StateSpaceModel):
        raise TypeError("particle filter needs a linear-Gaussian StateSpaceModel")
    mc = model._c_struct()
    ys = ys.reshape(-1, model.dy)
    T = ys.shape[0]
    cfg, sched, prec = _pf_config(algo, T, seed, schedule, lookahead)
    N, dx = algo.N, model.dx
    rdt = np.float64 if prec == L.GF_PREC_F64 else np.float32
    out = dict(ll=np.zeros(1), ll_steps=np.zeros(T), ess_steps=np.zeros(T),
               resampled=np.zeros(T, np.int8), states=np.zeros((dx, N), rdt),
               log_weights=np.zeros(N), clamps=np.zeros(1, np.int32))
    out["ancestors"] = np.zeros((T, N), np.int32) if want_anc else None
    out["means"] = np.zeros((T, dx)) if want_means else None
    out["paths"] = np.zeros((T + 1, dx, N), rdt) if want_paths else None
    out["history"] = np.zeros((T + 1, dx, N), rdt) if want_history else None
    out["log_weight_history"] = np.zeros((T, N)) if want_history else None
    o = L.PFOutC(*[L.ptr(out[k]) for k in ("ll", "ll_steps", "ess_steps", "resampled",
                                           "ancestors", "means", "states", "log_weights",
                                           "clamps", "paths", "history", "log_weight_history")])
    nz = None if noise is None else np.ascontiguousarray(noise, dtype=rdt)
    un = None if uniforms is None else L.f64(uniforms)
    if model.is_time_varying():
        ps = model.param_steps()
        if ps < T:
            raise ValueError(f"{ps} parameter steps for {T} observations")
        L.check(ctx.h, L.load().gf_pf_run_tv(ctx.h, C.byref(mc), ps, C.byref(cfg), T, L.ptr(ys),
                                             L.ptr(nz), L.ptr(un), L.GF_MEM_HOST, C.byref(o)))
    else:
        L.check(ctx.h, L.load().gf_pf_run(ctx.h, C.byref(mc), C.byref(cfg), T, L.ptr(ys),
                                          L.ptr(nz), L.ptr(un), L.GF_MEM_HOST, C.byref(o)))
    state = ParticleDistribution(out["states"].T, out["log_weights"], ll_steps=out["ll_steps"],
                                 ess_steps=out["ess_steps"], resampled=out["resampled"],
                                 ancestors=out["ancestors"], means=out["means"],
                                 clamps=int(out["clamps"][0]),
                                 paths=None if out["paths"] is None else out["paths"].transpose(0, 2, 1))
    state._history, state._lw_history = out["history"], out["log_weight_history"]
    return state, float(out["ll"][0])


def _rbpf(model, algo, ys, seed, noise, uniforms, ctx, want_anc, want_means, schedule,
          want_paths=False, want_history=False, lookahead=0):
    """RBPF run; paths and history hold the packed device state per particle
    [x (dxo) | mu (dz) | Sigma upper triangle by rows (dz (dz + 1) / 2)]."""
    if not isinstance(model, HierarchicalSSM):
        raise TypeError("RBPF needs a HierarchicalSSM")
    mc = model._c_struct()
    ys = ys.reshape(-1, model.dy)
    T = ys.shape[0]
    pf = algo.pf
    cfg, sched, prec = _pf_config(pf, T, seed, schedule, lookahead)
    N, dxo, dz = pf.N, model.dxo, model.dz
    width = dxo + dz + dz * dz
    out = dict(ll=np.zeros(1), ll_steps=np.zeros(T), ess_steps=np.zeros(T),
               resampled=np.zeros(T, np.int8), states=np.zeros((width, N), np.float32),
               log_weights=np.zeros(N), clamps=np.zeros(1, np.int32))
    out["ancestors"] = np.zeros((T, N), np.int32) if want_anc else None
    out["means"] = np.zeros((T, dxo)) if want_means else None
    zmeans = np.zeros((T, dz)) if want_means else None
    pw = dxo + dz + dz * (dz + 1) // 2
    out["paths"] = np.zeros((T + 1, pw, N), np.float32) if want_paths else None
    out["history"] = np.zeros((T + 1, pw, N), np.float32) if want_history else None
    out["log_weight_history"] = np.zeros((T, N)) if want_history else None
    o = L.PFOutC(*[L.ptr(out[k]) for k in ("ll", "ll_steps", "ess_steps", "resampled",
                                           "ancestors", "means", "states", "log_weights",
                                           "clamps", "paths", "history", "log_weight_history")])
    nz = None if noise is None else np.ascontiguousarray(noise, dtype=np.float32)
    un = None if uniforms is None else L.f64(uniforms)
    if model.is_time_varying():
        ps = model.param_steps()
        if ps < T:
            raise ValueError(f"{ps} parameter steps for {T} observations")
        L.check(ctx.h, L.load().gf_rbpf_run_tv(ctx.h, C.byref(mc), ps, C.byref(cfg), T, L.ptr(ys),
                                               L.ptr(nz), L.ptr(un), L.GF_MEM_HOST, C.byref(o),
                                               L.ptr(zmeans)))
    else:
        L.check(ctx.h, L.load().gf_rbpf_run(ctx.h, C.byref(mc), C.byref(cfg), T, L.ptr(ys),
                                            L.ptr(nz), L.ptr(un), L.GF_MEM_HOST, C.byref(o),
                                            L.ptr(zmeans)))
    S = out["states"]
    x = S[:dxo].T
    mu = S[dxo:dxo + dz].T
    Sig = S[dxo + dz:].T.reshape(N, dz, dz).transpose(0, 2, 1)  # column-major per particle
    state = ParticleDistribution(dict(x=x, mu=mu, Sigma=Sig), out["log_weights"],
                                 ll_steps=out["ll_steps"], ess_steps=out["ess_steps"],
                                 resampled=out["resampled"], ancestors=out["ancestors"],
                                 means=out["means"], zmeans=zmeans,
                                 clamps=int(out["clamps"][0]),
                                 paths=None if out["paths"] is None else out["paths"].transpose(0, 2, 1))
    state._history, state._lw_history = out["history"], out["log_weight_history"]
    return state, float(out["ll"][0])


def _param_steps(models, T):
    """Per-model parameter blocks for the time-varying entry points, or None
    when every model is homogeneous.  A time-varying model needs a block for
    every observed step (calc_params(dyn, t) for t = 1..T)."""
    if not any(m.is_time_varying() for m in models):
        return None
    ps = np.array([m.param_steps() for m in models], dtype=np.int32)
    for f, m in enumerate(models):
        if m.is_time_varying() and ps[f] < T[f]:
            raise ValueError(f"model {f}: {ps[f]} parameter steps for {T[f]} observations")
    return ps


def filter_batch(models, algo, observations, *, ctx=None, want_steps=True, want_covs=True):
    """Many independent Kalman / square-root Kalman filters in one batched launch.
    Returns a list of (MvNormal(final mu, Sigma), ll) with per-step outputs
    attached as .ll_steps, .means, .covs."""
    ctx = _resolve_ctx(ctx)
    if not isinstance(algo, (KalmanFilter, SRKalmanFilter)):
        raise TypeError("filter_batch supports KalmanFilter / SRKF")
    B = len(models)
    mcs = (L.LGModelC * B)(*[m._c_struct() for m in models])
    ys_list = [L.f64(y).reshape(-1, m.dy) for y, m in zip(observations, models)]
    T = np.array([y.shape[0] for y in ys_list], dtype=np.int32)
    psteps = _param_steps(models, T)
    ys = np.concatenate([y.ravel() for y in ys_list]) if B else np.zeros(0)
    dxs = np.array([m.dx for m in models])
    tot_steps = int(T.sum())
    out = dict(ll=np.zeros(B), ll_steps=np.zeros(tot_steps) if want_steps else None,
               means=np.zeros(int((T * dxs).sum()), np.float32),
               covs=np.zeros(int((T * dxs * dxs).sum()), np.float32) if want_covs else None,
               status=np.zeros(B, np.int32))
    o = L.KFOutC(*[L.ptr(out[k]) for k in ("ll", "ll_steps", "means", "covs", "status")])
    jit = algo.jitter
    i32 = C.POINTER(C.c_int32)
    if psteps is None:
        L.check(ctx.h, L.load().gf_kf_batch(ctx.h, algo.algo, mcs,  B, T.ctypes.data_as(i32),
                                            L.ptr(ys), float(jit or 0.0), int(jit is not None),
                                            L.GF_MEM_HOST, C.byref(o)))
    else:
        L.check(ctx.h, L.load().gf_kf_batch_tv(ctx.h, algo.algo, mcs, B, T.ctypes.data_as(i32),
                                               psteps.ctypes.data_as(i32), L.ptr(ys),
                                               float(jit or 0.0), int(jit is not None),
                                               L.GF_MEM_HOST, C.byref(o)))
    res = []
    so = mo = co = 0
    for f, m in enumerate(models):
        dx, t = m.dx, int(T[f])
        means = out["means"][mo:mo + t * dx].reshape(t, dx)
        covs = None
        if want_covs:
            covs = out["covs"][co:co + t * dx * dx].reshape(t, dx, dx).transpose(0, 2, 1)
        st = MvNormal(means[-1], covs[-1] if covs is not None else None)
        st.means, st.covs = means, covs
        st.ll_steps = out["ll_steps"][so:so + t] if want_steps else None
        res.append((st, float(out["ll"][f])))
        so += t
        mo += t * dx
        co += t * dx * dx
    return res


def smooth_batch(models, observations, *, ctx=None):
    """smooth(model, KalmanSmoother(), ys) for many models in one batched launch
    set (kalman.jl:206-234).  Returns a list of (means [T, dx], covs [T, dx, dx],
    ll): the smoothed p(x_t | y_1:T) of every step and the forward log-likelihood."""
    ctx = _resolve_ctx(ctx)
    B = len(models)
    mcs = (L.LGModelC * B)(*[m._c_struct() for m in models])
    ys_list = [L.f64(y).reshape(-1, m.dy) for y, m in zip(observations, models)]
    T = np.array([y.shape[0] for y in ys_list], dtype=np.int32)
    psteps = _param_steps(models, T)
    ys = np.concatenate([y.ravel() for y in ys_list]) if B else np.zeros(0)
    dxs = np.array([m.dx for m in models])
    out = dict(ll=np.zeros(B), ll_steps=None,
               means=np.zeros(int((T * dxs).sum()), np.float32),
               covs=np.zeros(int((T * dxs * dxs).sum()), np.float32),
               status=np.zeros(B, np.int32))
    o = L.KFOutC(*[L.ptr(out[k]) for k in ("ll", "ll_steps", "means", "covs", "status")])
    i32 = C.POINTER(C.c_int32)
    if psteps is None:
        L.check(ctx.h, L.load().gf_kf_smooth(ctx.h, mcs, B, T.ctypes.data_as(i32),
                                             L.ptr(ys), L.GF_MEM_HOST, C.byref(o)))
    else:
        L.check(ctx.h, L.load().gf_kf_smooth_tv(ctx.h, mcs, B, T.ctypes.data_as(i32),
                                                psteps.ctypes.data_as(i32), L.ptr(ys),
                                                L.GF_MEM_HOST, C.byref(o)))
    res = []
    mo = co = 0
    for f, m in enumerate(models):
        dx, t = m.dx, int(T[f])
        means = out["means"][mo:mo + t * dx].reshape(t, dx)
        covs = out["covs"][co:co + t * dx * dx].reshape(t, dx, dx).transpose(0, 2, 1)
        res.append((means, covs, float(out["ll"][f])))
        mo += t * dx
        co += t * dx * dx
    return res


def smooth(model, algo, observations, *, t_smooth=1, ctx=None):
    """smooth([rng,] model, KalmanSmoother(), observations; t_smooth=1) -> (MvNormal, ll)
    (kalman.jl:206-234): the smoothed p(x_t | y_1:T) at t = t_smooth (1-based)."""
    if not isinstance(algo, KalmanSmoother):
        raise TypeError("smooth supports KalmanSmoother()")
    means, covs, ll = smooth_batch([model], [observations], ctx=ctx)[0]
    T = means.shape[0]
    if not 1 <= t_smooth <= T:
        raise ValueError(f"t_smooth must be in 1..{T}")
    st = MvNormal(means[t_smooth - 1], covs[t_smooth - 1])
    st.means, st.covs = means, covs
    return st, ll


# ------------------------------------------------------------ resampling API
def _dev_i64(n, device):
    import torch
    return torch.zeros(n, dtype=torch.int64, device=f"cuda:{device}")


def sample_ancestors(resampler, weights, uniforms, *, convention="cpu", ctx=None):
    """sample_ancestors(rng, resampler, weights) on device tensors (torch CUDA
    float64 weights and uniforms); returns 1-based int64 ancestors (device)."""
    ctx = _resolve_ctx(ctx)
    n = weights.numel()
    out = _dev_i64(n, ctx.device)
    conv = L.GF_CONV_CUDAEXT if convention == "cudaext" else L.GF_CONV_CPU
    L.check(ctx.h, L.load().gf_sample_ancestors(ctx.h, resampler.kind, conv, n, L.ptr(weights),
                                                L.ptr(uniforms), L.ptr(out)))
    return out


def offspring_to_ancestors(offspring, *, ctx=None):
    """ext/CUDAExt.jl:105-117 on a device int64 tensor."""
    ctx = _resolve_ctx(ctx)
    out = _dev_i64(offspring.numel(), ctx.device)
    L.check(ctx.h, L.load().gf_offspring_to_ancestors(ctx.h, offspring.numel(), L.ptr(offspring),
                                                      L.ptr(out)))
    return out


def ancestors_to_offspring(ancestors, *, ctx=None):
    """ext/CUDAExt.jl:130-142 on a device int64 tensor."""
    ctx = _resolve_ctx(ctx)
    out = _dev_i64(ancestors.numel(), ctx.device)
    L.check(ctx.h, L.load().gf_ancestors_to_offspring(ctx.h, ancestors.numel(), L.ptr(ancestors),
                                                      L.ptr(out)))
    return out


def rng_normals(seed, t, dx, n, precision="f32", *, ctx=None):
    """The standard normals the PF kernels draw in-kernel at step t, as [dx, n]."""
    import torch
    ctx = _resolve_ctx(ctx)
    dt = torch.float64 if precision == "f64" else torch.float32
    out = torch.empty((dx, n), dtype=dt, device=f"cuda:{ctx.device}")
    prec = L.GF_PREC_F64 if precision == "f64" else L.GF_PREC_F32
    L.check(ctx.h, L.load().gf_rng_normals(ctx.h, int(seed), int(t), int(dx), int(n), prec,
                                           L.ptr(out)))
    return out


# --------------------------------------------------- log-likelihood gradients
GRAD_KEYS = ("mu0", "Sigma0", "A", "b", "Q", "H", "c", "R")


def kf_loglikelihood_grad_batch(models, observations, *, jitter=None, ctx=None):
    """kf_loglikelihood and its pullback (integrations/logdensity.jl:136-161,
    integrations/kalman_rrule.jl:22-107) for many homogeneous models at once.
    Returns a list of (ll, grads): grads maps mu0, Sigma0, A, b, Q, H, c, R to
    the gradient of ll (summed over time for the dynamics and observation
    parameters)."""
    ctx = _resolve_ctx(ctx)
    B = len(models)
    if B != len(observations):
        raise ValueError("one observation sequence per model")
    mcs = (L.LGModelC * B)(*[m._c_struct() for m in models])
    Ts = np.array([np.asarray(y).reshape(-1, m.dy).shape[0] for m, y in zip(models, observations)], np.int32)
    ys = L.f64(np.concatenate([np.asarray(y, np.float64).ravel() for y in observations]))
    dxs = np.array([m.dx for m in models])
    dys = np.array([m.dy for m in models])
    sizes = dict(mu0=dxs, Sigma0=dxs * dxs, A=dxs * dxs, b=dxs, Q=dxs * dxs, H=dys * dxs, c=dys, R=dys * dys)
    bufs = {k: np.zeros(int(v.sum())) for k, v in sizes.items()}
    ll = np.zeros(B)
    status = np.zeros(B, np.int32)
    out = L.KFGradOutC(L.ptr(ll), *[L.ptr(bufs[k]) for k in GRAD_KEYS], L.ptr(status))
    L.check(ctx.h, L.load().gf_kf_loglikelihood_grad(
        ctx.h, mcs, B, Ts.ctypes.data_as(C.POINTER(C.c_int32)), L.ptr(ys),
        float(jitter or 0.0), int(jitter is not None), L.GF_MEM_HOST, C.byref(out)))
    res = []
    off = {k: 0 for k in GRAD_KEYS}
    for f, m in enumerate(models):
        g = {}
        shapes = dict(mu0=(m.dx,), Sigma0=(m.dx, m.dx), A=(m.dx, m.dx), b=(m.dx,), Q=(m.dx, m.dx),
                      H=(m.dy, m.dx), c=(m.dy,), R=(m.dy, m.dy))
        for k in GRAD_KEYS:
            n = int(np.prod(shapes[k]))
            g[k] = bufs[k][off[k]:off[k] + n].reshape(shapes[k][::-1]).T  # column-major
            off[k] += n
        res.append((float(ll[f]), g))
    return res


def kf_loglikelihood_grad(model, observations, *, jitter=None, ctx=None):
    """(ll, grads) of kf_loglikelihood for one homogeneous model."""
    return kf_loglikelihood_grad_batch([model], [observations], jitter=jitter, ctx=ctx)[0]


# ------------------------------------------------- backward information filter
class InformationLikelihood:
    """InformationLikelihood (containers.jl): exp(lam'x - x'Om x / 2) up to a constant."""

    def __init__(self, lam, Om):
        self.lam, self.Om = lam, Om

    def natural_params(self):
        return self.lam, self.Om


def backward_information_batch(models, observations, *, initial_jitter=None, jitter=None, smooth=True,
                               ctx=None):
    """BackwardInformationPredictor(; initial_jitter, jitter) (kalman.jl:236-334) run
    backward over every model, and with smooth=True two_filter_smooth (kalman.jl:
    336-370) at every time.  Returns one dict per model: lam_pred [T, dx], Om_pred
    [T, dx, dx] (p(y_{t+1:T} | x_t)), lam_upd, Om_upd (p(y_{t:T} | x_t)), and
    mu_smooth [T, dx], Sigma_smooth [T, dx, dx] (p(x_t | y_1:T))."""
    ctx = _resolve_ctx(ctx)
    B = len(models)
    mcs = (L.LGModelC * B)(*[m._c_struct() for m in models])
    Ts = np.array([np.asarray(y).reshape(-1, m.dy).shape[0] for m, y in zip(models, observations)], np.int32)
    ys = L.f64(np.concatenate([np.asarray(y, np.float64).ravel() for y in observations]))
    dxs = np.array([m.dx for m in models])
    nv, nm = int(np.sum(Ts * dxs)), int(np.sum(Ts * dxs * dxs))
    names = ("lam_pred", "Om_pred", "lam_upd", "Om_upd", "mu_smooth", "Sigma_smooth")
    bufs = {k: np.zeros(nm if k.startswith(("Om", "Sigma")) else nv) for k in names}
    if not smooth:
        bufs["mu_smooth"] = bufs["Sigma_smooth"] = None
    status = np.zeros(B, np.int32)
    out = L.KFBackOutC(*[L.ptr(bufs[k]) for k in names], L.ptr(status))
    jit = (float(initial_jitter or 0.0), int(initial_jitter is not None), float(jitter or 0.0),
           int(jitter is not None), L.GF_MEM_HOST, C.byref(out))
    ps = _param_steps(models, Ts)
    if ps is None:
        L.check(ctx.h, L.load().gf_kf_backward_information(
            ctx.h, mcs, B, Ts.ctypes.data_as(C.POINTER(C.c_int32)), L.ptr(ys), *jit))
    else:
        L.check(ctx.h, L.load().gf_kf_backward_information_tv(
            ctx.h, mcs, B, Ts.ctypes.data_as(C.POINTER(C.c_int32)),
            ps.ctypes.data_as(C.POINTER(C.c_int32)), L.ptr(ys), *jit))
    res, ov, om = [], 0, 0
    for f, m in enumerate(models):
        T, d = int(Ts[f]), m.dx
        r = {}
        for k in names:
            if bufs[k] is None:
                continue
            if k.startswith(("Om", "Sigma")):
                r[k] = bufs[k][om:om + T * d * d].reshape(T, d, d).transpose(0, 2, 1)  # column-major
            else:
                r[k] = bufs[k][ov:ov + T * d].reshape(T, d)
        ov += T * d
        om += T * d * d
        res.append(r)
    return res


def two_filter_smooth_all(model, observations, *, initial_jitter=None, jitter=None, ctx=None):
    """p(x_t | y_1:T) at every t by the two-filter smoother: (means [T, dx], covs [T, dx, dx])."""
    r = backward_information_batch([model], [observations], initial_jitter=initial_jitter, jitter=jitter,
                                   ctx=ctx)[0]
    return r["mu_smooth"], r["Sigma_smooth"]
