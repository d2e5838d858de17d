"""Conditional SMC / particle Gibbs (csmc.jl) on the B200 library.

Mirrors the reference's API:

* ``ConditionalSMC(pf, refreshment=NoRefreshment())`` with ``NoRefreshment``,
  ``AncestorSampling`` and ``BackwardSimulation`` (csmc.jl:10-67);
* ``CSMCModel(ssm, observations)`` and ``CSMCState(trajectory)`` (:69-96);
* ``_csmc_sample(model, csmc, observations, ref_traj)`` -> (trajectory, ll),
  one sweep (:231-434);
* ``sample(CSMCModel, csmc, n_samples; burnin, chains)``: the AbstractMCMC
  chain of sweeps (:438-450), every chain of sweeps in one CTA of
  ``gf_csmc_run`` and all chains at once.

Trajectories are numpy arrays [T+1, dx]; row 0 is the time-0 state (the
reference's ``ReferenceTrajectory`` is indexed 0..T the same way).  The
particle filter must be a bootstrap ``BF(N; threshold, resampler)`` on a
homogeneous linear-Gaussian model, N <= ``gf_csmc_max_particles()``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .algorithms import ESSResampler, LatentProposal, ParticleFilter


class AbstractTrajectoryRefreshment:
    kind = -1


class NoRefreshment(AbstractTrajectoryRefreshment):
    """Vanilla conditional SMC: the reference pinned to particle 1 (csmc.jl:12-18)."""
    kind = L.GF_CSMC_NONE


class AncestorSampling(AbstractTrajectoryRefreshment):
    """CSMC-AS / PGAS: the reference particle's ancestor is redrawn from
    logw_i + log p(ref_t | x_i) at every step (csmc.jl:20-28, 240-278)."""
    kind = L.GF_CSMC_ANCESTOR


class BackwardSimulation(AbstractTrajectoryRefreshment):
    """CSMC-BS: a backward pass over the stored history (csmc.jl:30-40, 378-434)."""
    kind = L.GF_CSMC_BACKWARD


class ConditionalSMC:
    def __init__(self, pf: ParticleFilter, refreshment: AbstractTrajectoryRefreshment | None = None):
        if not isinstance(pf, ParticleFilter) or not isinstance(pf.proposal, LatentProposal):
            raise TypeError("ConditionalSMC runs a bootstrap filter BF(N; ...)")
        if not isinstance(pf.resampler, ESSResampler):
            raise TypeError("ConditionalSMC needs an ESS-conditioned resampler")
        self.pf = pf
        self.refreshment = refreshment if refreshment is not None else NoRefreshment()


class CSMCState:
    def __init__(self, trajectory):
        self.trajectory = trajectory


class CSMCModel:
    def __init__(self, ssm, observations):
        self.ssm = ssm
        self.observations = observations


def max_particles() -> int:
    return int(L.load().gf_csmc_max_particles())


def _run(ssm, csmc: ConditionalSMC, observations, *, chains, iters, burnin, ref, seed,
         noise, uniforms, ctx):
    ctx = ctx if ctx is not None else L.default_context()
    ys = L.f64(np.asarray(observations, dtype=np.float64).reshape(len(observations), -1))
    T, dx = ys.shape[0], ssm.dx
    rs = csmc.pf.resampler
    cfg = L.CsmcConfigC(csmc.pf.N, float(rs.threshold), rs.resampler.kind, csmc.refreshment.kind,
                        int(seed) & (2**64 - 1))
    keep = iters - burnin
    trajs = np.empty((chains, keep, T + 1, dx))
    lls = np.empty((chains, keep))
    refs = np.zeros((chains, T + 1, dx))
    if ref is not None:
        refs[:] = np.asarray(ref, dtype=np.float64).reshape(-1, T + 1, dx)
    status = np.zeros(chains, np.int32)
    nz = L.f64(noise) if noise is not None else None
    un = L.f64(uniforms) if uniforms is not None else None
    if nz is not None and nz.size != chains * iters * (T + 1) * csmc.pf.N * dx:
        raise ValueError("noise must hold [chains][iters][T+1][N][dx] normals")
    if un is not None and un.size != chains * iters * (T + 1) * (csmc.pf.N + 1):
        raise ValueError("uniforms must hold [chains][iters][T+1][N+1] values")
    out = L.CsmcOutC(L.ptr(trajs), L.ptr(lls), L.ptr(refs), L.ptr(status))
    mc = ssm._c_struct()
    rest = (chains, iters, burnin, int(ref is not None), L.ptr(nz), L.ptr(un), L.GF_MEM_HOST, C.byref(out))
    if ssm.is_time_varying():
        ps = ssm.param_steps()
        if ps < T:
            raise ValueError(f"{ps} parameter steps for {T} observations")
        L.check(ctx.h, L.load().gf_csmc_run_tv(ctx.h, C.byref(mc), ps, C.byref(cfg), T, L.ptr(ys), *rest))
    else:
        L.check(ctx.h, L.load().gf_csmc_run(ctx.h, C.byref(mc), C.byref(cfg), T, L.ptr(ys), *rest))
    return trajs, lls, refs


def _csmc_sample(model, csmc: ConditionalSMC, observations, ref_traj=None, *, seed: int = 0,
                 noise=None, uniforms=None, ctx=None):
    """One conditional SMC sweep (csmc.jl:231-434) -> (trajectory [T+1, dx], ll)."""
    trajs, lls, _ = _run(model, csmc, observations, chains=1, iters=1, burnin=0, ref=ref_traj,
                         seed=seed, noise=noise, uniforms=uniforms, ctx=ctx)
    return trajs[0, 0], float(lls[0, 0])


def sample(model: CSMCModel, csmc: ConditionalSMC, n_samples: int, *, burnin: int = 0,
           chains: int = 1, seed: int = 0, initial=None, noise=None, uniforms=None, ctx=None):
    """AbstractMCMC.sample(rng, CSMCModel, csmc, n_samples) after `burnin`
    discarded sweeps, for `chains` independent chains.

    Returns (trajectories [chains, n_samples, T+1, dx], lls [chains, n_samples],
    last [chains, T+1, dx]); pass `last` back as `initial` to continue the
    chains (the first sweep is then conditioned on it)."""
    if n_samples < 1:
        raise ValueError("n_samples must be >= 1")
    return _run(model.ssm, csmc, model.observations, chains=int(chains), iters=int(burnin + n_samples),
                burnin=int(burnin), ref=initial, seed=seed, noise=noise, uniforms=uniforms, ctx=ctx)
