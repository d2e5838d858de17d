"""TEST INFRASTRUCTURE ONLY -- ctypes front end of the FP64 CPU oracle.

The oracle restates GeneralisedFilters' filtering path (KF, SRKF, bootstrap and
guided PF, systematic/stratified/multinomial resampling, RBPF) in plain C
(``gf_oracle.c``) plus the numpy pieces below.  Only ``tests/``, the smoke
check in ``__graft_entry__`` and the CPU-baseline leg of ``bench.py`` import
this module; the product never does.

numpy helpers restated here:
* ``compute_joint`` -- the joint-Gaussian construction of
  GFTest/models/linear_gaussian.jl:171-215 used by test/algorithms/kalman.jl:5-43;
* ``rand_cov`` -- GFTest/utils.jl:15-36;
* ``create_linear_gaussian_model`` -- GFTest/models/linear_gaussian.jl:6-38
  (numpy-seeded: Julia's StableRNG streams cannot be reproduced here);
* ``sample`` -- SSMProblems/src/utils/forward_simulation.jl:14-26.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD, "libgforacle.so")

SYSTEMATIC, STRATIFIED, MULTINOMIAL = 0, 1, 2
CONV_CPU, CONV_CUDAEXT = 0, 1
PROP_BOOTSTRAP, PROP_OPTIMAL, PROP_OVERDISPERSED = 0, 1, 2


def build(force: bool = False) -> str:
    """Compile gf_oracle.c into oracle/_build/libgforacle.so."""
    src = os.path.join(HERE, "gf_oracle.c")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)):
        return LIB_PATH
    os.makedirs(BUILD, exist_ok=True)
    subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-o",
                           LIB_PATH, src, "-lm"])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
        _lib.or_logsumexp.restype = C.c_double
        _lib.or_philox_uniform.restype = C.c_double
    return _lib


_dp = C.POINTER(C.c_double)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _fortran(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


class _LG(C.Structure):
    _fields_ = [("dx", C.c_int), ("dy", C.c_int)] + [
        (n, _dp) for n in ("mu0", "Sigma0", "A", "b", "Q", "H", "c", "R")] + [("tv", C.c_int)]


class _RC(C.Structure):
    _fields_ = [("kind", C.c_int), ("conv", C.c_int), ("threshold", C.c_double),
                ("schedule", C.POINTER(C.c_int8))]


class _Prop(C.Structure):
    _fields_ = [("kind", C.c_int), ("k", C.c_double), ("lookahead", C.c_int)]


class _PFOut(C.Structure):
    _fields_ = [("ll_steps", _dp), ("ess", _dp), ("resampled", C.POINTER(C.c_int8)),
                ("ancestors", C.POINTER(C.c_int32)), ("margins", _dp), ("means", _dp),
                ("x_final", _dp), ("logw_final", _dp), ("clamps", C.POINTER(C.c_long)),
                ("x_all", _dp), ("logw_all", _dp)]


class _RB(C.Structure):
    _fields_ = ([("dxo", C.c_int), ("dz", C.c_int), ("dy", C.c_int)]
                + [(n, _dp) for n in ("mu_o", "Sigma_o", "A_o", "b_o", "Q_o",
                                      "mu_z", "Sigma_z", "A_z", "b_z", "C_z", "Q_z")]
                + [("q_gamma", C.c_double), ("q_index", C.c_int)]
                + [(n, _dp) for n in ("H", "c", "R")]
                + [("tv", C.c_int)])


class LGModel:
    """Plain FP64 container of a homogeneous linear-Gaussian SSM
    (models/linear_gaussian.jl:96-131): mu0, Sigma0, A, b, Q, H, c, R."""

    def __init__(self, mu0, Sigma0, A, b, Q, H, c, R):
        self.mu0, self.b, self.c = _f64(mu0).ravel(), _f64(b).ravel(), _f64(c).ravel()
        self.Sigma0, self.A, self.Q = _fortran(Sigma0), _fortran(A), _fortran(Q)
        self.H, self.R = _fortran(np.atleast_2d(H)), _fortran(np.atleast_2d(R))
        self.dx, self.dy = self.A.shape[0], self.H.shape[0]
        self.tv = False

    @classmethod
    def time_varying(cls, mu0, Sigma0, As, bs, Qs, Hs, cs, Rs):
        """Non-homogeneous model (GFTest/models/linear_gaussian.jl:42-95): the
        parameters of steps 1..T as sequences; params(t) returns step t's."""
        m = cls(mu0, Sigma0, As[0], bs[0], Qs[0], Hs[0], cs[0], Rs[0])
        m.tv = True
        m.steps = len(As)
        m.As = [_fortran(a) for a in As]
        m.bs = [_f64(v).ravel() for v in bs]
        m.Qs = [_fortran(q) for q in Qs]
        m.Hs = [_fortran(np.atleast_2d(h)) for h in Hs]
        m.cs = [_f64(v).ravel() for v in cs]
        m.Rs = [_fortran(np.atleast_2d(r)) for r in Rs]
        # step-major blocks, each column-major (the C oracle's tv layout)
        m._stk = {n: np.ascontiguousarray(np.concatenate([np.asarray(x).ravel(order="F")
                                                          for x in getattr(m, n + "s")]))
                  for n in ("A", "b", "Q", "H", "c", "R")}
        return m

    def params(self, t):
        """(A, b, Q, H, c, R) of 1-based step t (calc_params(dyn, t), calc_params(obs, t))."""
        if not self.tv:
            return self.A, self.b, self.Q, self.H, self.c, self.R
        k = t - 1
        return self.As[k], self.bs[k], self.Qs[k], self.Hs[k], self.cs[k], self.Rs[k]

    def _struct(self):
        if self.tv:
            arrs = [self.mu0, self.Sigma0] + [self._stk[n] for n in ("A", "b", "Q", "H", "c", "R")]
            return _LG(self.dx, self.dy, *[_p(a) for a in arrs], 1)
        s = _LG(self.dx, self.dy, *[_p(getattr(self, n)) for n in
                                    ("mu0", "Sigma0", "A", "b", "Q", "H", "c", "R")], 0)
        return s


def kf_filter(m: LGModel, ys, jitter=None, algo="kf"):
    """filter(model, KF()/SRKF(), ys) -> (ll, ll_steps, mus[T,dx], Sigmas[T,dx,dx])."""
    ys = _f64(ys).reshape(-1, m.dy)
    T = ys.shape[0]
    ll = C.c_double()
    lls = np.zeros(T)
    mus = np.zeros((T, m.dx))
    sig = np.zeros((T, m.dx, m.dx))
    f = lib().or_kf_filter if algo == "kf" else lib().or_srkf_filter
    st = f(C.byref(m._struct()), T, _p(ys), C.c_double(jitter or 0.0),
           int(jitter is not None), C.byref(ll), _p(lls), _p(mus), _p(sig))
    if st:
        raise np.linalg.LinAlgError(f"oracle KF status {st}")
    # Sigmas are column-major per step; transpose to row-major numpy
    return ll.value, lls, mus, np.ascontiguousarray(sig.transpose(0, 2, 1))


def rts_smooth(m: LGModel, ys):
    """smooth(model, KalmanSmoother(), ys) for every t -> (ll, mus[T,dx], Sigmas[T,dx,dx])
    (kalman.jl:89-126,206-234)."""
    ys = _f64(ys).reshape(-1, m.dy)
    T = ys.shape[0]
    ll = C.c_double()
    mus = np.zeros((T, m.dx))
    sig = np.zeros((T, m.dx, m.dx))
    st = lib().or_rts_smooth(C.byref(m._struct()), T, _p(ys), C.byref(ll), _p(mus), _p(sig))
    if st:
        raise np.linalg.LinAlgError(f"oracle RTS status {st}")
    return ll.value, mus, np.ascontiguousarray(sig.transpose(0, 2, 1))


def joint_smooth_truth(m: LGModel, ys):
    """Exact smoothed means/covariances of X_1..X_T given y_1:T by Gaussian
    conditioning of the joint of compute_joint (the analytic counterpart of the
    RTS pass)."""
    ys = np.asarray(ys, np.float64).reshape(-1, m.dy)
    T = ys.shape[0]
    mu_Z, S_Z = compute_joint(m, T)
    Dx, Dy = m.dx, m.dy
    Iy = slice(Dx * (T + 1), Dx * (T + 1) + T * Dy)
    Syy = S_Z[Iy, Iy]
    Syy = (Syy + Syy.T) / 2
    d = ys.ravel() - mu_Z[Iy]
    w = np.linalg.solve(Syy, d)
    mus, Ss = [], []
    for t in range(1, T + 1):
        Ix = slice(t * Dx, (t + 1) * Dx)
        mus.append(mu_Z[Ix] + S_Z[Ix, Iy] @ w)
        Ss.append(S_Z[Ix, Ix] - S_Z[Ix, Iy] @ np.linalg.solve(Syy, S_Z[Iy, Ix]))
    return np.array(mus), np.array(Ss)


def pf_run(m: LGModel, N, ys, *, resampler=SYSTEMATIC, conv=CONV_CPU, threshold=0.5,
           schedule=None, noise=None, uniforms=None, seed=0, proposal=PROP_BOOTSTRAP,
           k=1.0, want_ancestors=False, want_margins=False, want_states=False, threads=1,
           lookahead=0):
    """filter(rng, model, ParticleFilter(N, proposal; threshold, resampler), ys), or with
    lookahead=1 filter(rng, model, AuxiliaryParticleFilter(pf, MeanPredictive()), ys) and
    lookahead=2 the same with DrawPredictive() (its draw from the Philox stream tagged
    0x4C4B4844, counters (i, t, q), key seed).

    noise: [(T+1), dx, N] standard normals (step 0 = prior draw) or None for the
    shared Philox stream with ``seed``; uniforms: systematic [T], else [T, N].
    Returns a dict of outputs (ll, ll_steps, ess, resampled, ancestors (1-based),
    margins, means, x_final [N,dx], logw_final, clamps)."""
    ys = _f64(ys).reshape(-1, m.dy)
    T = ys.shape[0]
    out = dict(ll_steps=np.zeros(T), ess=np.zeros(T), resampled=np.zeros(T, np.int8),
               means=np.zeros((T, m.dx)), x_final=np.zeros((N, m.dx)),
               logw_final=np.zeros(N))
    anc = np.zeros((T, N), np.int32) if want_ancestors else None
    mar = np.zeros((T, N)) if want_margins else None
    clamps = C.c_long(0)
    o = _PFOut(_p(out["ll_steps"]), _p(out["ess"]),
               out["resampled"].ctypes.data_as(C.POINTER(C.c_int8)),
               None if anc is None else anc.ctypes.data_as(C.POINTER(C.c_int32)),
               _p(mar), _p(out["means"]), _p(out["x_final"]), _p(out["logw_final"]),
               C.pointer(clamps))
    xall = np.zeros((T + 1, N, m.dx)) if want_states else None
    o.x_all = _p(xall)
    lwall = np.zeros((T, N)) if want_states else None
    o.logw_all = _p(lwall)
    sched = None if schedule is None else np.ascontiguousarray(schedule, np.int8)
    rc = _RC(resampler, conv, threshold,
             None if sched is None else sched.ctypes.data_as(C.POINTER(C.c_int8)))
    nz = None if noise is None else _f64(noise)
    un = None if uniforms is None else _f64(uniforms)
    ll = C.c_double()
    lib().or_set_threads(int(threads))
    st = lib().or_pf_run(C.byref(m._struct()), C.byref(_Prop(proposal, k, int(lookahead))), C.byref(rc),
                         C.c_long(N), T, _p(ys), _p(nz), _p(un), C.c_uint64(seed),
                         C.byref(ll), C.byref(o))
    lib().or_set_threads(1)
    if st:
        raise np.linalg.LinAlgError(f"oracle PF status {st}")
    out["ll"] = ll.value
    out["ancestors"] = anc
    out["margins"] = mar
    out["clamps"] = clamps.value
    out["states"] = xall
    out["log_weights_all"] = lwall
    return out


def ancestry_paths(ancestors, states):
    """get_ancestry (containers.jl:587-611): the trajectory of every final particle,
    rebuilt densely from the 1-based ancestors [T, N] and the states [(T+1), N, dx];
    returns paths [(T+1), N, dx] with paths[T] = states[T]."""
    T, N = ancestors.shape
    paths = np.empty_like(states)
    idx = np.arange(N)
    for t in range(T, 0, -1):
        paths[t] = states[t][idx]
        idx = ancestors[t - 1][idx] - 1
    paths[0] = states[0][idx]
    return paths


def pf_step(m: LGModel, x, logw, y, noise_t, u, *, uniform=False, resampler=SYSTEMATIC,
            conv=CONV_CPU, threshold=0.5, decision=-1):
    """One bootstrap PF step from a given state (teacher forcing).  x: [N, dx]
    FP64, logw: [N] normalised; noise_t: [dx, N]; u: this step's uniforms."""
    N = x.shape[0]
    x = np.ascontiguousarray(x, np.float64).copy()
    logw = np.ascontiguousarray(logw, np.float64).copy()
    anc = np.zeros(N, np.int32)
    mar = np.zeros(N)
    ess = C.c_double()
    res = C.c_int8()
    inc = C.c_double()
    sched = np.array([decision], np.int8)
    rc = _RC(resampler, conv, threshold, sched.ctypes.data_as(C.POINTER(C.c_int8)))
    un = _f64(np.atleast_1d(u))
    st = lib().or_pf_step(C.byref(m._struct()), C.byref(rc), C.c_long(N), 1,
                          _p(_f64(y).ravel()), _p(_f64(noise_t)), _p(un), int(uniform),
                          _p(x), _p(logw), anc.ctypes.data_as(C.POINTER(C.c_int32)),
                          _p(mar), C.byref(ess), C.byref(res), C.byref(inc))
    if st:
        raise np.linalg.LinAlgError(f"oracle PF step status {st}")
    return dict(x=x, logw=logw, ancestors=anc, margins=mar, ess=ess.value,
                resampled=bool(res.value), ll_inc=inc.value)


def sample_ancestors(kind, weights, u, conv=CONV_CPU):
    """sample_ancestors(rng, resampler, weights) with injected uniforms.
    Returns (ancestors 1-based int32, margins, clamps)."""
    w = _f64(weights)
    n = w.shape[0]
    anc = np.zeros(n, np.int32)
    mar = np.zeros(n)
    un = _f64(np.atleast_1d(u))
    cl = lib().or_sample_ancestors(kind, conv, C.c_long(n), _p(w), _p(un),
                                   anc.ctypes.data_as(C.POINTER(C.c_int32)), _p(mar))
    return anc, mar, cl


def offspring_to_ancestors(offspring):
    o = np.ascontiguousarray(offspring, np.int64)
    a = np.zeros_like(o)
    lib().or_offspring_to_ancestors(C.c_long(o.size), o.ctypes.data_as(C.POINTER(C.c_int64)),
                                    a.ctypes.data_as(C.POINTER(C.c_int64)))
    return a


def ancestors_to_offspring(ancestors):
    a = np.ascontiguousarray(ancestors, np.int64)
    o = np.zeros_like(a)
    lib().or_ancestors_to_offspring(C.c_long(a.size), a.ctypes.data_as(C.POINTER(C.c_int64)),
                                    o.ctypes.data_as(C.POINTER(C.c_int64)))
    return o


def philox_normals(seed, N, dx, t):
    """[dx, N] normals of step t from the shared Philox stream (FP64 Box-Muller).
    A one-dimensional state takes normal i % 4 of the call (i // 4, t, 0)."""
    out = np.zeros((dx, N))
    buf = (C.c_double * 4)()
    if dx == 1:
        for g in range((N + 3) // 4):
            lib().or_philox_normals4(C.c_uint64(seed), g, t, 0, buf)
            for r in range(4):
                if 4 * g + r < N:
                    out[0, 4 * g + r] = buf[r]
        return out
    for i in range(N):
        for q in range((dx + 3) // 4):
            lib().or_philox_normals4(C.c_uint64(seed), i, t, q, buf)
            for r in range(4):
                if 4 * q + r < dx:
                    out[4 * q + r, i] = buf[r]
    return out


def philox_uniform(seed, j, t):
    return lib().or_philox_uniform(C.c_uint64(seed), j, t)


class RBModel:
    """Conditionally linear-Gaussian HierarchicalSSM (models/hierarchical.jl:4-50):
    outer LG state x, inner LG state z with b_t = b_z + C_z x_prev and
    Q_t = Q_z * exp(q_gamma * x_new[q_index]); y = H z + c + N(0, R)."""

    def __init__(self, mu_o, Sigma_o, A_o, b_o, Q_o, mu_z, Sigma_z, A_z, b_z, C_z, Q_z,
                 H, c, R, q_gamma=0.0, q_index=0):
        f = _fortran
        self.mu_o, self.b_o = _f64(mu_o).ravel(), _f64(b_o).ravel()
        self.Sigma_o, self.A_o, self.Q_o = f(Sigma_o), f(A_o), f(Q_o)
        self.mu_z, self.b_z = _f64(mu_z).ravel(), _f64(b_z).ravel()
        self.Sigma_z, self.A_z, self.Q_z = f(Sigma_z), f(A_z), f(Q_z)
        self.C_z = f(np.atleast_2d(C_z).reshape(self.mu_z.size, self.mu_o.size))
        self.H, self.c, self.R = f(np.atleast_2d(H)), _f64(c).ravel(), f(np.atleast_2d(R))
        self.q_gamma, self.q_index = float(q_gamma), int(q_index)
        self.dxo, self.dz, self.dy = self.mu_o.size, self.mu_z.size, self.H.shape[0]

    STEP_NAMES = ("A_o", "b_o", "Q_o", "A_z", "b_z", "C_z", "Q_z", "H", "c", "R")

    @classmethod
    def time_varying(cls, mu_o, Sigma_o, mu_z, Sigma_z, steps, q_gamma=0.0, q_index=0):
        """Non-homogeneous hierarchical model: `steps` is a list over t = 1..T of
        dicts with the STEP_NAMES parameters of step t (calc_params(., t))."""
        s0 = steps[0]
        m = cls(mu_o, Sigma_o, s0["A_o"], s0["b_o"], s0["Q_o"], mu_z, Sigma_z, s0["A_z"], s0["b_z"],
                s0["C_z"], s0["Q_z"], s0["H"], s0["c"], s0["R"], q_gamma, q_index)
        m.tv = True
        m.steps = [cls(mu_o, Sigma_o, d["A_o"], d["b_o"], d["Q_o"], mu_z, Sigma_z, d["A_z"], d["b_z"],
                       d["C_z"], d["Q_z"], d["H"], d["c"], d["R"], q_gamma, q_index) for d in steps]
        # step-major blocks, each column-major (the C oracle's tv layout)
        m._stk = {n: np.concatenate([np.asarray(getattr(k, n)).ravel(order="F") for k in m.steps])
                  for n in cls.STEP_NAMES}
        return m

    def step(self, t):
        """The homogeneous model of 1-based step t."""
        return self.steps[t - 1] if getattr(self, "tv", False) else self

    def _struct(self):
        names = ("mu_o", "Sigma_o", "A_o", "b_o", "Q_o", "mu_z", "Sigma_z", "A_z", "b_z",
                 "C_z", "Q_z")
        tv = getattr(self, "tv", False)
        get = (lambda n: self._stk[n] if n in self._stk else getattr(self, n)) if tv else \
            (lambda n: getattr(self, n))
        return _RB(self.dxo, self.dz, self.dy, *[_p(get(n)) for n in names],
                   self.q_gamma, self.q_index, _p(get("H")), _p(get("c")), _p(get("R")), int(tv))


def rbpf_run(m: RBModel, N, ys, *, resampler=SYSTEMATIC, conv=CONV_CPU, threshold=0.5,
             schedule=None, noise=None, uniforms=None, seed=0, proposal=PROP_BOOTSTRAP,
             k=1.0, want_ancestors=False, want_margins=False, threads=1, lookahead=0):
    """filter(rng, hier_model, RBPF(PF(N, ...), KalmanFilter()), ys); lookahead=1
    (MeanPredictive) or 2 (DrawPredictive) runs AuxiliaryParticleFilter(RBPF(...),
    pp) (rbpf.jl:86-124)."""
    ys = _f64(ys).reshape(-1, m.dy)
    T = ys.shape[0]
    width = m.dxo + m.dz + m.dz * m.dz
    out = dict(ll_steps=np.zeros(T), ess=np.zeros(T), resampled=np.zeros(T, np.int8),
               means=np.zeros((T, m.dxo)), x_final=np.zeros((N, width)),
               logw_final=np.zeros(N))
    zmeans = np.zeros((T, m.dz))
    anc = np.zeros((T, N), np.int32) if want_ancestors else None
    mar = np.zeros((T, N)) if want_margins else None
    clamps = C.c_long(0)
    o = _PFOut(_p(out["ll_steps"]), _p(out["ess"]),
               out["resampled"].ctypes.data_as(C.POINTER(C.c_int8)),
               None if anc is None else anc.ctypes.data_as(C.POINTER(C.c_int32)),
               _p(mar), _p(out["means"]), _p(out["x_final"]), _p(out["logw_final"]),
               C.pointer(clamps))
    sched = None if schedule is None else np.ascontiguousarray(schedule, np.int8)
    rc = _RC(resampler, conv, threshold,
             None if sched is None else sched.ctypes.data_as(C.POINTER(C.c_int8)))
    nz = None if noise is None else _f64(noise)
    un = None if uniforms is None else _f64(uniforms)
    ll = C.c_double()
    lib().or_set_threads(int(threads))
    st = lib().or_rbpf_run(C.byref(m._struct()), C.byref(_Prop(proposal, k, int(lookahead))), C.byref(rc),
                           C.c_long(N), T, _p(ys), _p(nz), _p(un), C.c_uint64(seed),
                           C.byref(ll), C.byref(o), _p(zmeans))
    lib().or_set_threads(1)
    if st:
        raise np.linalg.LinAlgError(f"oracle RBPF status {st}")
    out.update(ll=ll.value, ancestors=anc, margins=mar, zmeans=zmeans, clamps=clamps.value)
    return out


def rbpf_step(m: RBModel, x, mu, Sigma, logw, y, noise_t, u, *, uniform=False,
              resampler=SYSTEMATIC, conv=CONV_CPU, threshold=0.5, decision=-1):
    """One bootstrap RBPF step from a given state (teacher forcing).  x [N, dxo],
    mu [N, dz], Sigma [N, dz, dz]; logw [N] normalised; noise_t [dxo, N]; u this
    step's uniforms.  Returns the new x, mu, Sigma, logw and the step's
    ancestors (1-based), margins, ESS, decision and ll increment."""
    N, dxo, dz = x.shape[0], m.dxo, m.dz
    w_in = dxo + dz + dz * dz
    S = np.empty((N, w_in))
    S[:, :dxo] = x
    S[:, dxo:dxo + dz] = mu
    S[:, dxo + dz:] = np.asarray(Sigma, np.float64).transpose(0, 2, 1).reshape(N, dz * dz)
    S = np.ascontiguousarray(S)
    logw = np.ascontiguousarray(logw, np.float64).copy()
    anc = np.zeros(N, np.int32)
    mar = np.zeros(N)
    ess, res, inc = C.c_double(), C.c_int8(), C.c_double()
    sched = np.array([decision], np.int8)
    rc = _RC(resampler, conv, threshold, sched.ctypes.data_as(C.POINTER(C.c_int8)))
    un = _f64(np.atleast_1d(u))
    st = lib().or_rbpf_step(C.byref(m._struct()), C.byref(rc), C.c_long(N),
                            _p(_f64(y).ravel()), _p(_f64(noise_t)), _p(un), int(uniform), _p(S),
                            _p(logw), anc.ctypes.data_as(C.POINTER(C.c_int32)), _p(mar),
                            C.byref(ess), C.byref(res), C.byref(inc))
    if st:
        raise np.linalg.LinAlgError(f"oracle RBPF step status {st}")
    Sig = S[:, dxo + dz:].reshape(N, dz, dz).transpose(0, 2, 1)
    return dict(x=S[:, :dxo].copy(), mu=S[:, dxo:dxo + dz].copy(), Sigma=Sig.copy(), logw=logw,
                ancestors=anc, margins=mar, ess=ess.value, resampled=bool(res.value),
                ll_inc=inc.value)


# --------------------------------------------------------------------------- #
# numpy restatements of the reference's test fixtures                          #
# --------------------------------------------------------------------------- #
CSMC_NONE, CSMC_ANCESTOR, CSMC_BACKWARD = 0, 1, 2


def csmc_run(m: LGModel, N, ys, *, threshold=0.6, resampler=SYSTEMATIC, refresh=CSMC_NONE,
             chains=1, iters=1, burnin=0, ref=None, noise=None, uniforms=None, seed=0, threads=1):
    """`iters` ConditionalSMC sweeps per chain (csmc.jl:231-450) with the
    randomness injected (layouts of gf_csmc_run) or drawn from the CUDA
    library's Philox counters.  Returns (trajectories [chains, iters-burnin,
    T+1, dx], lls [chains, iters-burnin], last [chains, T+1, dx])."""
    ys = _f64(ys).reshape(-1, m.dy)
    T, dx = ys.shape[0], m.dx
    keep = iters - burnin
    trajs = np.zeros((chains, keep, T + 1, dx))
    lls = np.zeros((chains, keep))
    refs = np.zeros((chains, T + 1, dx))
    if ref is not None:
        refs[:] = _f64(ref).reshape(-1, T + 1, dx)
    nz = None if noise is None else _f64(noise)
    un = None if uniforms is None else _f64(uniforms)
    lib().or_set_threads(int(threads))
    f = lib().or_csmc_run
    f.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, _dp, C.c_int, C.c_int,
                  C.c_int, C.c_int, _dp, _dp, C.c_uint64, _dp, _dp, _dp]
    st = f(C.byref(m._struct()), int(N), float(threshold), int(resampler), int(refresh), T, _p(ys),
           int(chains), int(iters), int(burnin), int(ref is not None),
           None if nz is None else _p(nz), None if un is None else _p(un),
           C.c_uint64(int(seed) & (2**64 - 1)), _p(refs), _p(trajs), _p(lls))
    lib().or_set_threads(1)
    if st:
        raise FloatingPointError(f"oracle CSMC status {st}")
    return trajs, lls, refs


def rand_cov(rng, d, scale=1.0, var_range=(0.8, 1.2)):
    """GFTest/utils.jl:15-36: random correlation matrix rescaled by variances."""
    A = rng.random((d, d))
    S = A @ A.T
    Dis = np.diag(1.0 / np.sqrt(np.diag(S)))
    S = Dis @ S @ Dis
    var = (rng.random(d) * (var_range[1] - var_range[0]) + var_range[0]) * scale
    Ds = np.diag(np.sqrt(var))
    S = Ds @ S @ Ds
    return (S + S.T) / 2


def create_linear_gaussian_model(rng, Dx, Dy, process_noise_scale=0.1, obs_noise_scale=1.0):
    """GFTest/models/linear_gaussian.jl:6-38 (numpy RNG)."""
    mu0 = rng.random(Dx)
    S0 = rand_cov(rng, Dx)
    A = rng.random((Dx, Dx))
    b = rng.random(Dx)
    Q = rand_cov(rng, Dx, scale=process_noise_scale)
    H = rng.random((Dy, Dx))
    c = rng.random(Dy)
    R = rand_cov(rng, Dy, scale=obs_noise_scale)
    return LGModel(mu0, S0, A, b, Q, H, c, R)


def create_nonhomogeneous_linear_gaussian_model(rng, Dx, Dy, T_max, process_noise_scale=0.1,
                                                obs_noise_scale=1.0):
    """GFTest/models/linear_gaussian.jl:97-119 (numpy RNG): a prior and one
    (A, b, Q, H, c, R) per step t = 1..T_max."""
    mu0 = rng.random(Dx)
    S0 = rand_cov(rng, Dx)
    As = [rng.random((Dx, Dx)) for _ in range(T_max)]
    bs = [rng.random(Dx) for _ in range(T_max)]
    Qs = [rand_cov(rng, Dx, scale=process_noise_scale) for _ in range(T_max)]
    Hs = [rng.random((Dy, Dx)) for _ in range(T_max)]
    cs = [rng.random(Dy) for _ in range(T_max)]
    Rs = [rand_cov(rng, Dy, scale=obs_noise_scale) for _ in range(T_max)]
    return LGModel.time_varying(mu0, S0, As, bs, Qs, Hs, cs, Rs)


def sample(rng, m: LGModel, T):
    """SSMProblems forward simulation (utils/forward_simulation.jl:14-26)."""
    x = rng.multivariate_normal(m.mu0, m.Sigma0)
    xs, ys = [], []
    for t in range(1, T + 1):
        A, b, Q, H, c, R = m.params(t)
        x = A @ x + b + rng.multivariate_normal(np.zeros(m.dx), Q)
        xs.append(x)
        ys.append(H @ x + c + rng.multivariate_normal(np.zeros(m.dy), R))
    return np.array(xs), np.array(ys).reshape(T, m.dy)


def compute_joint(m: LGModel, T):
    """GFTest/models/linear_gaussian.jl:171-215 (and :121-169,
    _compute_joint_nonhomogeneous, for time-varying models): Z = [X0..XT, Y1..YT]
    ~ N(mu_Z, Sigma_Z) from (I - P) Z = eps."""
    Dx, Dy = m.dx, m.dy
    n = Dx + T * (Dx + Dy)
    P = np.zeros((n, n))
    mu_e = np.zeros(n)
    S_e = np.zeros((n, n))
    mu_e[:Dx] = m.mu0
    S_e[:Dx, :Dx] = m.Sigma0
    for t in range(1, T + 1):
        A, b, Q, H, c, R = m.params(t)   # _compute_joint_nonhomogeneous for tv models
        iA, jA = t * Dx, (t - 1) * Dx
        P[iA:iA + Dx, jA:jA + Dx] = A
        iH, jH = Dx * (T + 1) + (t - 1) * Dy, Dx * t
        P[iH:iH + Dy, jH:jH + Dx] = H
        mu_e[iA:iA + Dx] = b
        mu_e[iH:iH + Dy] = c
        S_e[iA:iA + Dx, iA:iA + Dx] = Q
        S_e[iH:iH + Dy, iH:iH + Dy] = R
    IP = np.eye(n) - P
    mu_Z = np.linalg.solve(IP, mu_e)
    Sigma_Z = np.linalg.solve(IP, np.linalg.solve(IP, S_e).T).T
    return mu_Z, Sigma_Z


def joint_filter_truth(m: LGModel, ys):
    """Exact filtered mean/cov of X_T and log p(y_1:T) by Gaussian conditioning
    (test/algorithms/kalman.jl:5-43, generalised to T steps)."""
    ys = np.asarray(ys, np.float64).reshape(-1, m.dy)
    T = ys.shape[0]
    mu_Z, S_Z = compute_joint(m, T)
    Dx, Dy = m.dx, m.dy
    Ix = slice(T * Dx, (T + 1) * Dx)
    Iy = slice(Dx * (T + 1), Dx * (T + 1) + T * Dy)
    y = ys.ravel()
    Syy = S_Z[Iy, Iy]
    Syy = (Syy + Syy.T) / 2
    d = y - mu_Z[Iy]
    mu_x = mu_Z[Ix] + S_Z[Ix, Iy] @ np.linalg.solve(Syy, d)
    S_x = S_Z[Ix, Ix] - S_Z[Ix, Iy] @ np.linalg.solve(Syy, S_Z[Iy, Ix])
    sign, logdet = np.linalg.slogdet(Syy)
    ll = -0.5 * (d @ np.linalg.solve(Syy, d) + logdet + y.size * np.log(2 * np.pi))
    return mu_x, S_x, ll


def random_orthogonal(rng, d):
    """Haar-random orthogonal matrix (QR of a Gaussian with sign fix)."""
    Z = rng.standard_normal((d, d))
    Qm, Rm = np.linalg.qr(Z)
    return Qm * np.sign(np.diag(Rm))


def kf_loglikelihood_grad(m: LGModel, ys, jitter=None):
    """kf_loglikelihood and its pullback for a homogeneous model (kalman_rrule.jl:
    22-107 with the step rules of kalman_gradient.jl:12-263), FP64 numpy.

    Forward: kalman_predict (kalman.jl:42-49) and _kalman_update_cached (Joseph
    form).  Backward, per step t = T..1, in the NLL convention of the reference:
    gradient_c/H/R (:172-263), backward_gradient_update (:97-120, eqs 8-9),
    gradient_b/A/Q (:150-205), backward_gradient_predict (:138-143, eqs 10-11).
    Returns (ll, grads) with grads the gradients of ll (the pullback with
    Delta ll = 1: minus the NLL gradients), summed over t for A, b, Q, H, c, R."""
    ys = _f64(ys).reshape(-1, m.dy)
    T = ys.shape[0]
    A, b, Q, H, c, R = (np.asarray(v, np.float64) for v in (m.A, m.b, m.Q, m.H, m.c, m.R))
    mu, S0 = np.asarray(m.mu0, np.float64).copy(), np.asarray(m.Sigma0, np.float64).copy()
    dx, dy = A.shape[0], H.shape[0]
    prev, caches, ll = [], [], 0.0
    Sig = S0
    for t in range(T):
        prev.append((mu, Sig))
        mp = A @ mu + b
        Sp = A @ Sig @ A.T + Q
        z = ys[t] - H @ mp - c
        S = H @ Sp @ H.T + R
        S = (S + S.T) / 2
        K = Sp @ H.T @ np.linalg.inv(S)
        IKH = np.eye(dx) - K @ H
        Sf = IKH @ Sp @ IKH.T + K @ R @ K.T
        if jitter is not None:
            Sf = Sf + jitter * np.eye(dx)
        mf = mp + K @ z
        sign, logdet = np.linalg.slogdet(S)
        ll += -0.5 * (dy * np.log(2 * np.pi) + logdet + z @ np.linalg.solve(S, z))
        caches.append(dict(mp=mp, Sp=Sp, mf=mf, S=S, K=K, z=z, IKH=IKH))
        mu, Sig = mf, Sf
    dmu, dS = np.zeros(dx), np.zeros((dx, dx))
    g = {k: np.zeros_like(v) for k, v in (("A", A), ("b", b), ("Q", Q), ("H", H), ("c", c), ("R", R))}
    Rinv = np.linalg.inv(R)
    for t in range(T - 1, -1, -1):
        C_ = caches[t]
        mp, Sp, mf, S, K, z, IKH = (C_[k] for k in ("mp", "Sp", "mf", "S", "K", "z", "IKH"))
        Si = np.linalg.inv(S)
        Siz = np.linalg.solve(S, z)
        g["c"] += -Siz - K.T @ dmu
        Pf = IKH @ Sp
        g["H"] += (Si @ H @ Sp - np.outer(Siz, mp) - np.outer(Siz, Siz) @ H @ Sp
                   + np.outer(Siz, dmu) @ Pf - K.T @ np.outer(dmu, mf) - 2 * K.T @ dS @ Pf)
        g["R"] += K.T @ dS @ K - 0.5 * (K.T @ np.outer(dmu, Siz) + np.outer(Siz, dmu) @ K) \
            + 0.5 * (Si - np.outer(Siz, Siz))
        dmp = IKH.T @ dmu - H.T @ Siz
        Riz = Rinv @ z
        cross = 0.5 * (np.outer(dmu, Riz @ H) + np.outer(H.T @ Riz, dmu))
        dSp = IKH.T @ (dS + cross) @ IKH + 0.5 * (H.T @ Si @ H - H.T @ np.outer(Siz, Siz) @ H)
        mu_prev, S_prev = prev[t]
        g["b"] += dmp
        g["A"] += np.outer(dmp, mu_prev) + 2 * dSp @ A @ S_prev
        g["Q"] += dSp
        dmu, dS = A.T @ dmp, A.T @ dSp @ A
    g["mu0"], g["Sigma0"] = dmu, dS
    return ll, {k: -v for k, v in g.items()}


def backward_information(m: LGModel, ys, initial_jitter=None, jitter=None):
    """BackwardInformationPredictor (kalman.jl:236-334), FP64 numpy: the backward
    predictive likelihoods in information form, exp(lam'x - x'Om x / 2).
    Returns (lam_pred [T, dx], Om_pred [T, dx, dx], lam_upd, Om_upd): row t
    (0-based, time t+1) of *_pred is p(y_{t+2:T} | x_{t+1}) after backward_predict
    (zero at the last time), of *_upd is p(y_{t+1:T} | x_{t+1}) after
    backward_initialise / backward_update."""
    ys = _f64(ys).reshape(-1, m.dy)
    T = ys.shape[0]
    dx = m.dx
    lp, Op = np.zeros((T, dx)), np.zeros((T, dx, dx))
    lu, Ou = np.zeros((T, dx)), np.zeros((T, dx, dx))

    def step(k):  # calc_params(dyn, k), calc_params(obs, k) (1-based), FP64
        return tuple(np.asarray(v, np.float64) for v in m.params(k))

    def sym(M):  # PDMat(Symmetric(M)): the upper triangle mirrored
        return np.triu(M) + np.triu(M, 1).T

    _, _, _, H, c, R = step(T)
    Ri = np.linalg.inv(R)
    lam = H.T @ Ri @ (ys[T - 1] - c)
    Om = H.T @ Ri @ H
    if initial_jitter is not None:
        Om = Om + initial_jitter * np.eye(dx)
    Om = sym(Om)
    lu[T - 1], Ou[T - 1] = lam, Om
    for t in range(T - 2, -1, -1):
        # backward_predict at iter t+1 uses calc_params(dyn, iter + 1) (kalman.jl:294-320)
        A, b, Q, _, _, _ = step(t + 2)
        F = np.linalg.cholesky(Q)
        mvec = lam - Om @ b
        Lam = F.T @ Om @ F + np.eye(dx)
        FLF = F @ np.linalg.solve(Lam, F.T)
        Im = np.eye(dx) - Om @ FLF
        Om_h = A.T @ Im @ Om @ A
        lam_h = A.T @ Im @ mvec
        if jitter is not None:
            Om_h = Om_h + jitter * np.eye(dx)
        Om_h = sym(Om_h)
        lp[t], Op[t] = lam_h, Om_h
        _, _, _, H, c, R = step(t + 1)  # backward_update at iter t+1
        Ri = np.linalg.inv(R)
        lam = lam_h + H.T @ Ri @ (ys[t] - c)
        Om = sym(Om_h + H.T @ Ri @ H)
        lu[t], Ou[t] = lam, Om
    return lp, Op, lu, Ou


def two_filter_smooth(m: LGModel, ys, initial_jitter=None, jitter=None):
    """two_filter_smooth (kalman.jl:336-370) at every time: the forward filtered
    N(mu_t, Sigma_t) (the KF of kf_filter) combined with p(y_{t+1:T} | x_t) from
    backward_information.  Returns (mus [T, dx], Sigmas [T, dx, dx])."""
    _, _, mus_f, Sf = kf_filter(m, ys)
    lp, Op, _, _ = backward_information(m, ys, initial_jitter, jitter)
    T, dx = mus_f.shape
    mus, Ss = np.zeros((T, dx)), np.zeros((T, dx, dx))
    for t in range(T):
        Si = np.linalg.inv(Sf[t])
        Om_s = Si + Op[t]
        S_s = np.linalg.inv(Om_s)
        mus[t] = S_s @ (Si @ mus_f[t] + lp[t])
        Ss[t] = S_s
    return mus, Ss
