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


class StateSpaceModel:
    """SSMProblems.StateSpaceModel{PT,LD,OP} (SSMProblems.jl:264-272)."""

    def __init__(self, prior: StatePrior, dyn: LatentDynamics, obs: ObservationProcess):
        self.prior, self.dyn, self.obs = prior, dyn, obs

    # calc_* accessors of models/linear_gaussian.jl:33-63 (homogeneous: step ignored)
    def is_linear_gaussian(self):
        return (isinstance(self.prior, HomogeneousGaussianPrior)
                and isinstance(self.dyn, HomogeneousLinearGaussianLatentDynamics)
                and isinstance(self.obs, HomogeneousLinearGaussianObservationProcess))

    @property
    def dx(self):
        return self.dyn.A.shape[0]

    @property
    def dy(self):
        return self.obs.H.shape[0]

    def _c_struct(self):
        """gf_lg_model view; keeps references to the arrays alive on self."""
        if not self.is_linear_gaussian():
            raise TypeError("filter on the GPU needs a homogeneous linear-Gaussian model")
        p, d, o = self.prior, self.dyn, self.obs
        arrs = [p.mu0, p.Sigma0, d.A, d.b, d.Q, o.H, o.c, o.R]
        self._keep = arrs
        dx, dy = self.dx, self.dy
        shapes = [(dx,), (dx, dx), (dx, dx), (dx,), (dx, dx), (dy, dx), (dy,), (dy, dy)]
        for a, s in zip(arrs, shapes):
            if a.shape != s:
                raise ValueError(f"DimensionMismatch: expected {s}, got {a.shape}")
        import ctypes as C
        dp = C.POINTER(C.c_double)
        return LGModelC(dx, dy, *[a.ctypes.data_as(dp) for a in arrs])


def create_homogeneous_linear_gaussian_model(mu0, Sigma0, A, b, Q, H, c, R):
    """models/linear_gaussian.jl:125-131."""
    return StateSpaceModel(HomogeneousGaussianPrior(mu0, Sigma0),
                           HomogeneousLinearGaussianLatentDynamics(A, b, Q),
                           HomogeneousLinearGaussianObservationProcess(H, c, R))


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


class HierarchicalSSM:
    """models/hierarchical.jl:4-45: outer prior + outer dynamics + inner model."""

    def __init__(self, outer_prior, outer_dyn, inner_prior, inner_dyn, obs):
        self.outer_prior, self.outer_dyn = outer_prior, outer_dyn
        self.inner_model = StateSpaceModel(inner_prior, inner_dyn, obs)

    def _c_struct(self):
        import ctypes as C
        op, od = self.outer_prior, self.outer_dyn
        ip, idyn, ob = self.inner_model.prior, self.inner_model.dyn, self.inner_model.obs
        if not (isinstance(op, HomogeneousGaussianPrior)
                and isinstance(od, HomogeneousLinearGaussianLatentDynamics)
                and isinstance(ip, HomogeneousGaussianPrior)
                and isinstance(ob, HomogeneousLinearGaussianObservationProcess)):
            raise TypeError("RBPF on the GPU needs Gaussian priors, LG outer dynamics and LG obs")
        if isinstance(idyn, HomogeneousLinearGaussianLatentDynamics):
            idyn = InnerDynamics(idyn.A, idyn.b, np.zeros((idyn.b.size, od.b.size)), idyn.Q)
        arrs = [op.mu0, op.Sigma0, od.A, od.b, od.Q, ip.mu0, ip.Sigma0, idyn.A, idyn.b, idyn.C,
                idyn.Q, ob.H, ob.c, ob.R]
        self._keep = arrs
        dp = C.POINTER(C.c_double)
        P = [a.ctypes.data_as(dp) for a in arrs]
        return RBModelC(od.b.size, idyn.b.size, ob.c.size, *P[:11], idyn.q_gamma, idyn.q_index,
                        *P[11:])

    @property
    def dxo(self):
        return self.outer_dyn.b.size

    @property
    def dz(self):
        return self.inner_model.dyn.b.size

    @property
    def dy(self):
        return self.inner_model.obs.c.size
