"""Algorithm descriptors mirroring GeneralisedFilters' constructors.

* ``KalmanFilter(jitter=None)`` / ``KF()`` -- algorithms/kalman.jl:16-21
* ``SRKalmanFilter(jitter=None)`` / ``SRKF()`` -- algorithms/srkf.jl:34-39
* ``KalmanSmoother()`` / ``KS`` -- algorithms/kalman.jl:83-85
* ``ParticleFilter(N, proposal; threshold=1.0, resampler=Systematic())`` and
  ``BootstrapFilter(N; ...)`` / ``BF`` -- algorithms/particles.jl:92-108,197-201
* ``RBPF(pf, af)`` -- algorithms/rbpf.jl:8-14
* ``Multinomial``, ``Systematic``, ``Stratified``, ``ESSResampler`` --
  resamplers.jl:171-240
* ``OptimalProposal``, ``OverdispersedProposal``, ``AlternatingResampler`` --
  GFTest/proposals.jl:11-50, GFTest/resamplers.jl:11-39
"""
from __future__ import annotations

from . import _lib as L


class AbstractResampler:
    kind = None


class Multinomial(AbstractResampler):
    kind = L.GF_RS_MULTINOMIAL


class Systematic(AbstractResampler):
    kind = L.GF_RS_SYSTEMATIC


class Stratified(AbstractResampler):
    kind = L.GF_RS_STRATIFIED


class ESSResampler(AbstractResampler):
    """Resample iff threshold * N >= ESS (resamplers.jl:171-183)."""

    def __init__(self, threshold, resampler=None):
        self.threshold = float(threshold)
        self.resampler = resampler if resampler is not None else Systematic()

    def schedule(self, T):
        return None


class AlternatingResampler(AbstractResampler):
    """GFTest/resamplers.jl:11-39.  Its will_resample returns `resample_next`,
    which only resample() flips, so the reference resamples at step 1 and then
    never again; schedule() reproduces that decision sequence."""

    def __init__(self, resampler=None):
        self.resampler = resampler if resampler is not None else Systematic()
        self.threshold = 1.0

    def schedule(self, T):
        return [1] + [0] * (T - 1)


class AbstractProposal:
    pass


class LatentProposal(AbstractProposal):
    """Bootstrap proposal (particles.jl:197-245)."""
    kind = L.GF_PROP_BOOTSTRAP
    k = 1.0


class OptimalProposal(AbstractProposal):
    """p(x_t | x_{t-1}, y_t) for LG models (GFTest/proposals.jl:11-31)."""
    kind = L.GF_PROP_OPTIMAL

    def __init__(self, dyn=None, obs=None):
        self.dyn, self.obs = dyn, obs
        self.k = 1.0


class OverdispersedProposal(AbstractProposal):
    """MvNormal(A x + b, k Q) (GFTest/proposals.jl:33-50)."""
    kind = L.GF_PROP_OVERDISPERSED

    def __init__(self, dyn=None, k=1.0):
        self.dyn, self.k = dyn, float(k)


class AbstractFilter:
    pass


class KalmanFilter(AbstractFilter):
    algo = L.GF_ALGO_KF

    def __init__(self, jitter=None):
        self.jitter = jitter


def KF():
    return KalmanFilter()


class KalmanSmoother(AbstractFilter):
    """KalmanSmoother() (kalman.jl:83-85): Rauch-Tung-Striebel smoothing after a
    KalmanFilter() forward pass."""


KS = KalmanSmoother()


class SRKalmanFilter(AbstractFilter):
    algo = L.GF_ALGO_SRKF

    def __init__(self, jitter=None):
        self.jitter = jitter


def SRKF():
    return SRKalmanFilter()


class ParticleFilter(AbstractFilter):
    """ParticleFilter(N, proposal; threshold=1.0, resampler=Systematic()).

    Extra keyword arguments of the B200 build: ``precision`` ("f32" state with
    FP64 normaliser, or "f64"), ``convention`` ("cpu" = resamplers.jl rule,
    "cudaext" = ext/CUDAExt.jl rule)."""

    def __init__(self, N, proposal, threshold=1.0, resampler=None, precision="f32",
                 convention="cpu"):
        self.N = int(N)
        self.proposal = proposal
        rs = resampler if resampler is not None else Systematic()
        if isinstance(rs, (ESSResampler, AlternatingResampler)):
            self.resampler = rs
        else:
            self.resampler = ESSResampler(threshold, rs)
        self.precision = precision
        self.convention = convention


PF = ParticleFilter


def BootstrapFilter(N, **kw):
    return ParticleFilter(N, LatentProposal(), **kw)


BF = BootstrapFilter


class PredictiveStatistic:
    """How AuxiliaryParticleFilter picks a particle's representative next state
    (particles.jl:359-384)."""
    lookahead = -1


class MeanPredictive(PredictiveStatistic):
    """mean(transition) = A x + b."""
    lookahead = 1


class ModePredictive(PredictiveStatistic):
    """mode(transition) = A x + b for the Gaussian transition (same scores as MeanPredictive)."""
    lookahead = 1


class DrawPredictive(PredictiveStatistic):
    """A draw from the transition, A x + b + chol(Q) e' (the linear-Gaussian PF with the
    bootstrap proposal, or the outer transition of an RBPF; e' from its own in-kernel
    Philox stream)."""
    lookahead = 2


class RepresentativeStateLookAhead:
    def __init__(self, pp: PredictiveStatistic):
        self.pp = pp


class AuxiliaryParticleFilter(AbstractFilter):
    """AuxiliaryParticleFilter(pf, pp) (particles.jl:270-357): first-stage weights
    log p(y_t | x*) with x* the predictive statistic `pp` of each particle's
    transition, resampling on softmax(logw + log eta) (AuxiliaryResampler,
    resamplers.jl:85-143), second-stage weights corrected by -log eta[a].  ``pf`` is a
    ParticleFilter on a linear-Gaussian model, or an RBPF on a HierarchicalSSM, whose
    x* is the outer predictive statistic and log eta the inner Kalman update's
    log-likelihood after predicting to x* (rbpf.jl:86-124)."""

    def __init__(self, pf, pp):
        if isinstance(pp, RepresentativeStateLookAhead):
            pp = pp.pp
        if not isinstance(pp, PredictiveStatistic):
            raise TypeError("AuxiliaryParticleFilter(pf, MeanPredictive() | ModePredictive())")
        if pp.lookahead < 0:
            raise NotImplementedError(f"{type(pp).__name__} lookahead is not built")
        self.pf = pf
        self.weight_strategy = RepresentativeStateLookAhead(pp)


APF = AuxiliaryParticleFilter


class RBPF(AbstractFilter):
    """RBPF(pf, af) (rbpf.jl:8-14); af must be a KalmanFilter."""

    def __init__(self, pf: ParticleFilter, af: AbstractFilter):
        if not isinstance(af, KalmanFilter):
            raise TypeError("RBPF inner filter must be KalmanFilter()")
        self.pf, self.af = pf, af
