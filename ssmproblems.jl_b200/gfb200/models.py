"""Model layer mirroring SSMProblems / GeneralisedFilters' model types.

* ``StatePrior``, ``LatentDynamics``, ``ObservationProcess``, ``StateSpaceModel``
  -- the abstract interface of SSMProblems/src/SSMProblems.jl:25,40,55,264-272.
* ``HomogeneousGaussianPrior``, ``HomogeneousLinearGaussianLatentDynamics``,
  ``HomogeneousLinearGaussianObservationProcess`` and
  ``create_homogeneous_linear_gaussian_model`` -- models/linear_gaussian.jl:96-131.
* ``HierarchicalSSM`` with a conditionally linear-Gaussian inner model --
  models/hierarchical.jl:4-50 with GFTest's InnerDynamics
  (GFTest/models/dummy_linear_gaussian.jl:25-46).

Only the model families the CUDA kernels implement are accepted by ``filter``;
anything else raises (there is no CPU fallback).
"""
from __future__ import annotations

import numpy as np

from ._lib import LGModelC, RBModelC, f64, fortran64


class StatePrior:
    """SSMProblems.StatePrior (SSMProblems.jl:25)."""


class LatentDynamics:
    """SSMProblems.LatentDynamics (SSMProblems.jl:40)."""


class ObservationProcess:
    """SSMProblems.ObservationProcess (SSMProblems.jl:55)."""


class HomogeneousGaussianPrior(StatePrior):
    def __init__(self, mu0, Sigma0):
        self.mu0 = f64(mu0).ravel()
        self.Sigma0 = fortran64(np.atleast_2d(Sigma0))


class HomogeneousLinearGaussianLatentDynamics(LatentDynamics):
    def __init__(self, A, b, Q):
        self.A = fortran64(np.atleast_2d(A))
        self.b = f64(b).ravel()
        self.Q = fortran64(np.atleast_2d(Q))


class HomogeneousLinearGaussianObservationProcess(ObservationProcess):
    def __init__(self, H, c, R):
        self.H = fortran64(np.atleast_2d(H))
        self.c = f64(c).ravel()
        self.R = fortran64(np.atleast_2d(R))


class NonHomogeneousLinearGaussianLatentDynamics(LatentDynamics):
    """Time-varying linear-Gaussian dynamics: calc_params(dyn, t) = (As[t], bs[t],
    Qs[t]) for 1-based step t (models/linear_gaussian.jl:44-52; GFTest's
    NonHomogeneousLinearGaussianLatentDynamics, GFTest/models/linear_gaussian.jl:42-66)."""

    def __init__(self, As, bs, Qs):
        if not (len(As) == len(bs) == len(Qs)) or len(As) < 1:
            raise ValueError("As, bs, Qs need one entry per step")
        self.As = [fortran64(np.atleast_2d(a)) for a in As]
        self.bs = [f64(v).ravel() for v in bs]
        self.Qs = [fortran64(np.atleast_2d(q)) for q in Qs]
        self.A = self.As[0]


class NonHomogeneousLinearGaussianObservationProcess(ObservationProcess):
    """Time-varying observations: calc_params(obs, t) = (Hs[t], cs[t], Rs[t])
    (models/linear_gaussian.jl:54-63; GFTest/models/linear_gaussian.jl:68-95)."""

    def __init__(self, Hs, cs, Rs):
        if not (len(Hs) == len(cs) == len(Rs)) or len(Hs) < 1:
            raise ValueError("Hs, cs, Rs need one entry per step")
        self.Hs = [fortran64(np.atleast_2d(h)) for h in Hs]
        self.cs = [f64(v).ravel() for v in cs]
        self.Rs = [fortran64(np.atleast_2d(r)) for r in Rs]
        self.H = self.Hs[0]


class StateSpaceModel:
    """SSMProblems.StateSpaceModel{PT,LD,OP} (SSMProblems.jl:264-272)."""

    def __init__(self, prior: StatePrior, dyn: LatentDynamics, obs: ObservationProcess):
        self.prior, self.dyn, self.obs = prior, dyn, obs

    # calc_* accessors of models/linear_gaussian.jl:33-63 (homogeneous: step ignored)
    def is_linear_gaussian(self):
        return (isinstance(self.prior, HomogeneousGaussianPrior)
                and isinstance(self.dyn, HomogeneousLinearGaussianLatentDynamics)
                and isinstance(self.obs, HomogeneousLinearGaussianObservationProcess))

    def is_time_varying(self):
        """A linear-Gaussian model whose dynamics or observations vary with t."""
        return (isinstance(self.prior, HomogeneousGaussianPrior)
                and isinstance(self.dyn, (HomogeneousLinearGaussianLatentDynamics,
                                          NonHomogeneousLinearGaussianLatentDynamics))
                and isinstance(self.obs, (HomogeneousLinearGaussianObservationProcess,
                                          NonHomogeneousLinearGaussianObservationProcess))
                and not self.is_linear_gaussian())

    def param_steps(self):
        """Per-step parameter blocks the model carries (1 if homogeneous)."""
        if not self.is_time_varying():
            return 1
        n = [len(x.As) for x in (self.dyn,) if hasattr(x, "As")] + \
            [len(x.Hs) for x in (self.obs,) if hasattr(x, "Hs")]
        return min(n)

    @property
    def dx(self):
        return self.dyn.A.shape[0]

    @property
    def dy(self):
        return self.obs.H.shape[0]

    def _c_struct(self):
        """gf_lg_model view; keeps references to the arrays alive on self.  For a
        time-varying model the A, b, Q, H, c, R pointers hold param_steps()
        step-major blocks (each column-major)."""
        import ctypes as C
        dp = C.POINTER(C.c_double)
        p, d, o = self.prior, self.dyn, self.obs
        dx, dy = self.dx, self.dy
        if self.is_time_varying():
            n = self.param_steps()
            dl = [(getattr(d, "As", None), d.A), (getattr(d, "bs", None), getattr(d, "b", None)),
                  (getattr(d, "Qs", None), getattr(d, "Q", None))]
            ol = [(getattr(o, "Hs", None), o.H), (getattr(o, "cs", None), getattr(o, "c", None)),
                  (getattr(o, "Rs", None), getattr(o, "R", None))]
            shapes = [(dx, dx), (dx,), (dx, dx), (dy, dx), (dy,), (dy, dy)]
            stk = []
            for (seq, one), shp in zip(dl + ol, shapes):
                blocks = seq[:n] if seq is not None else [one] * n
                for blk in blocks:
                    if blk.shape != shp:
                        raise ValueError(f"DimensionMismatch: expected {shp}, got {blk.shape}")
                stk.append(np.ascontiguousarray(np.concatenate([np.asarray(b).ravel(order="F")
                                                                for b in blocks])))
            arrs = [p.mu0, p.Sigma0] + stk
            for a, s in zip(arrs[:2], [(dx,), (dx, dx)]):
                if a.shape != s:
                    raise ValueError(f"DimensionMismatch: expected {s}, got {a.shape}")
            self._keep = arrs
            return LGModelC(dx, dy, *[a.ctypes.data_as(dp) for a in arrs])
        if not self.is_linear_gaussian():
            raise TypeError("filter on the GPU needs a linear-Gaussian model")
        arrs = [p.mu0, p.Sigma0, d.A, d.b, d.Q, o.H, o.c, o.R]
        self._keep = arrs
        shapes = [(dx,), (dx, dx), (dx, dx), (dx,), (dx, dx), (dy, dx), (dy,), (dy, dy)]
        for a, s in zip(arrs, shapes):
            if a.shape != s:
                raise ValueError(f"DimensionMismatch: expected {s}, got {a.shape}")
        return LGModelC(dx, dy, *[a.ctypes.data_as(dp) for a in arrs])


def create_homogeneous_linear_gaussian_model(mu0, Sigma0, A, b, Q, H, c, R):
    """models/linear_gaussian.jl:125-131."""
    return StateSpaceModel(HomogeneousGaussianPrior(mu0, Sigma0),
                           HomogeneousLinearGaussianLatentDynamics(A, b, Q),
                           HomogeneousLinearGaussianObservationProcess(H, c, R))


def create_nonhomogeneous_linear_gaussian_model(mu0, Sigma0, As, bs, Qs, Hs, cs, Rs):
    """A time-varying linear-Gaussian model from per-step parameter sequences
    (entry t-1 = step t), the model of GFTest's
    create_nonhomogeneous_linear_gaussian_model (GFTest/models/linear_gaussian.jl:97-119)."""
    return StateSpaceModel(HomogeneousGaussianPrior(mu0, Sigma0),
                           NonHomogeneousLinearGaussianLatentDynamics(As, bs, Qs),
                           NonHomogeneousLinearGaussianObservationProcess(Hs, cs, Rs))


class InnerDynamics(LatentDynamics):
    """Conditionally linear-Gaussian inner dynamics given the outer state:
    z_t = A z_{t-1} + b + C x_{t-1} + N(0, Q * exp(q_gamma * x_t[q_index])).
    C follows GFTest's InnerDynamics (dummy_linear_gaussian.jl:25-46, calc_b
    with prev_outer); the exp scale on Q is the stochastic-volatility form of
    examples/trend-inflation/script.jl (calc_Q with new_outer)."""

    def __init__(self, A, b, C, Q, q_gamma=0.0, q_index=0):
        self.A = fortran64(np.atleast_2d(A))
        self.b = f64(b).ravel()
        self.C = fortran64(np.atleast_2d(C).reshape(self.b.size, -1))
        self.Q = fortran64(np.atleast_2d(Q))
        self.q_gamma = float(q_gamma)
        self.q_index = int(q_index)


class NonHomogeneousInnerDynamics(LatentDynamics):
    """InnerDynamics with step-dependent parameters: calc_params(inner_dyn, t) =
    (As[t], bs[t] + Cs[t] x_{t-1}, Qs[t] exp(q_gamma x_t[q_index])) for 1-based
    step t (models/hierarchical.jl:96-137 with a time-varying inner model)."""

    def __init__(self, As, bs, Cs, Qs, q_gamma=0.0, q_index=0):
        if not (len(As) == len(bs) == len(Cs) == len(Qs)) or len(As) < 1:
            raise ValueError("As, bs, Cs, Qs need one entry per step")
        self.As = [fortran64(np.atleast_2d(a)) for a in As]
        self.bs = [f64(v).ravel() for v in bs]
        self.Cs = [fortran64(np.atleast_2d(c).reshape(self.bs[0].size, -1)) for c in Cs]
        self.Qs = [fortran64(np.atleast_2d(q)) for q in Qs]
        self.A, self.b = self.As[0], self.bs[0]
        self.q_gamma = float(q_gamma)
        self.q_index = int(q_index)


class HierarchicalSSM:
    """models/hierarchical.jl:4-45: outer prior + outer dynamics + inner model."""

    def __init__(self, outer_prior, outer_dyn, inner_prior, inner_dyn, obs):
        self.outer_prior, self.outer_dyn = outer_prior, outer_dyn
        self.inner_model = StateSpaceModel(inner_prior, inner_dyn, obs)

    _TV = (NonHomogeneousLinearGaussianLatentDynamics, NonHomogeneousInnerDynamics,
           NonHomogeneousLinearGaussianObservationProcess)

    def is_time_varying(self):
        """Outer dynamics, inner dynamics or observations vary with t."""
        return any(isinstance(x, self._TV) for x in (self.outer_dyn, self.inner_model.dyn,
                                                     self.inner_model.obs))

    def param_steps(self):
        """Per-step parameter blocks the model carries (1 if homogeneous)."""
        n = [len(getattr(x, a)) for x, a in ((self.outer_dyn, "As"), (self.inner_model.dyn, "As"),
                                             (self.inner_model.obs, "Hs")) if hasattr(x, a)]
        return min(n) if n else 1

    def _c_struct(self):
        """gf_rb_model view; for a time-varying model the step parameters hold
        param_steps() step-major blocks (each column-major)."""
        import ctypes as C
        op, od = self.outer_prior, self.outer_dyn
        ip, idyn, ob = self.inner_model.prior, self.inner_model.dyn, self.inner_model.obs
        lgd = (HomogeneousLinearGaussianLatentDynamics, NonHomogeneousLinearGaussianLatentDynamics)
        lgo = (HomogeneousLinearGaussianObservationProcess, NonHomogeneousLinearGaussianObservationProcess)
        if not (isinstance(op, HomogeneousGaussianPrior) and isinstance(od, lgd)
                and isinstance(ip, HomogeneousGaussianPrior) and isinstance(ob, lgo)):
            raise TypeError("RBPF on the GPU needs Gaussian priors, LG outer dynamics and LG obs")
        dxo = od.A.shape[0]
        if isinstance(idyn, HomogeneousLinearGaussianLatentDynamics):
            idyn = InnerDynamics(idyn.A, idyn.b, np.zeros((idyn.b.size, dxo)), idyn.Q)
        elif isinstance(idyn, NonHomogeneousLinearGaussianLatentDynamics):
            idyn = NonHomogeneousInnerDynamics(idyn.As, idyn.bs, [np.zeros((idyn.bs[0].size, dxo))] *
                                               len(idyn.As), idyn.Qs)
        n = self.param_steps()

        def stk(x, seq, one):  # the step parameter: n stacked blocks, or the single one
            if not self.is_time_varying():
                return getattr(x, one)
            blocks = getattr(x, seq)[:n] if hasattr(x, seq) else [getattr(x, one)] * n
            return np.concatenate([np.asarray(b, np.float64).ravel(order="F") for b in blocks])

        arrs = [op.mu0, op.Sigma0, stk(od, "As", "A"), stk(od, "bs", "b"), stk(od, "Qs", "Q"),
                ip.mu0, ip.Sigma0, stk(idyn, "As", "A"), stk(idyn, "bs", "b"), stk(idyn, "Cs", "C"),
                stk(idyn, "Qs", "Q"), stk(ob, "Hs", "H"), stk(ob, "cs", "c"), stk(ob, "Rs", "R")]
        self._keep = arrs
        dp = C.POINTER(C.c_double)
        P = [a.ctypes.data_as(dp) for a in arrs]
        return RBModelC(dxo, idyn.b.size, ob.H.shape[0], *P[:11], idyn.q_gamma, idyn.q_index,
                        *P[11:])

    @property
    def dxo(self):
        return self.outer_dyn.A.shape[0]

    @property
    def dz(self):
        return self.inner_model.dyn.A.shape[0]

    @property
    def dy(self):
        return self.inner_model.obs.H.shape[0]
