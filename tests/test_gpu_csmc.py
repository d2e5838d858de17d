"""GPU conditional SMC (csmc.jl) against the FP64 oracle restatement.

* Injected randomness: the CUDA sweeps and the oracle consume the same
  normals and uniforms, so trajectories, log-likelihoods and the final
  references agree to FP64 rounding (rtol 1e-9) for every refreshment and
  resampler.
* In-kernel Philox: the oracle regenerates the same streams.
* Convergence (test/algorithms/csmc.jl:5-98): the mean of the sampled
  trajectories at t_smooth matches the Kalman smoother within rtol 1e-3, and
  logsumexp(-ll) - log(n) (1/Z-hat is unbiased for 1/Z) matches -ll_KF within
  rtol 1e-3.  These use multinomial resampling: with systematic or stratified
  resampling, overwriting the reference slot of a correlated draw (the
  reference's _set_ref_index!) leaves a small bias, which the oracle shows
  too (about 0.4% under ancestor sampling on this model).
"""
import numpy as np
import pytest

import gfb200 as G
import oracle as O
from gfb200 import csmc as CS
from helpers import random_lg, simulate, to_oracle

pytestmark = pytest.mark.gpu

RS = {"systematic": (G.Systematic(), O.SYSTEMATIC), "stratified": (G.Stratified(), O.STRATIFIED),
      "multinomial": (G.Multinomial(), O.MULTINOMIAL)}
REFRESH = {"none": G.NoRefreshment(), "ancestor": G.AncestorSampling(), "backward": G.BackwardSimulation()}


def _inputs(rng, chains, iters, T, N, dx):
    noise = rng.standard_normal((chains, iters, T + 1, N, dx))
    unif = rng.random((chains, iters, T + 1, N + 1))
    return noise, unif


@pytest.mark.parametrize("refresh", list(REFRESH))
@pytest.mark.parametrize("rs", list(RS))
@pytest.mark.parametrize("dims", [(1, 1), (3, 2)])
def test_csmc_matches_oracle_injected(ctx, refresh, rs, dims):
    dx, dy = dims
    rng = np.random.default_rng(100 + dx)
    m = random_lg(rng, dx, dy)
    T, N, chains, iters, burnin = 8, 13, 3, 6, 2
    _, ys = simulate(rng, m, T)
    noise, unif = _inputs(rng, chains, iters, T, N, dx)
    ref0 = rng.standard_normal((chains, T + 1, dx)) if refresh != "backward" else None
    csmc = G.ConditionalSMC(G.BF(N, threshold=0.6, resampler=RS[rs][0]), REFRESH[refresh])
    tr, lls, last = CS.sample(G.CSMCModel(m, ys), csmc, iters - burnin, burnin=burnin, chains=chains,
                              initial=ref0, noise=noise, uniforms=unif, ctx=ctx)
    otr, olls, olast = O.csmc_run(to_oracle(m), N, ys, threshold=0.6, resampler=RS[rs][1],
                                  refresh=REFRESH[refresh].kind,
                                  chains=chains, iters=iters, burnin=burnin, ref=ref0,
                                  noise=noise, uniforms=unif)
    np.testing.assert_allclose(tr, otr, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(lls, olls, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(last, olast, rtol=1e-9, atol=1e-9)


def test_csmc_wide_state_matches_oracle(ctx):
    """dx = 16 (the widest kernel instance), dy = 8, N = 40 (two warps)."""
    rng = np.random.default_rng(7)
    m = random_lg(rng, 16, 8)
    T, N, chains, iters = 5, 40, 2, 3
    _, ys = simulate(rng, m, T)
    noise, unif = _inputs(rng, chains, iters, T, N, 16)
    for refresh in REFRESH.values():
        csmc = G.ConditionalSMC(G.BF(N, threshold=0.6, resampler=G.Multinomial()), refresh)
        tr, lls, _ = CS.sample(G.CSMCModel(m, ys), csmc, iters, chains=chains, noise=noise,
                               uniforms=unif, ctx=ctx)
        otr, olls, _ = O.csmc_run(to_oracle(m), N, ys, threshold=0.6, resampler=O.MULTINOMIAL,
                                  refresh=refresh.kind, chains=chains, iters=iters, noise=noise,
                                  uniforms=unif)
        np.testing.assert_allclose(tr, otr, rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(lls, olls, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("refresh", list(REFRESH))
def test_csmc_philox_streams_match_oracle(ctx, refresh):
    """In-kernel Philox draws (sweep, chain, t<<12 | slot) regenerated by the oracle."""
    rng = np.random.default_rng(11)
    m = random_lg(rng, 2, 1)
    T, N = 6, 300  # N > 256: several particles per thread
    _, ys = simulate(rng, m, T)
    csmc = G.ConditionalSMC(G.BF(N, threshold=0.6), REFRESH[refresh])
    tr, lls, _ = CS.sample(G.CSMCModel(m, ys), csmc, 4, chains=2, seed=99, ctx=ctx)
    otr, olls, _ = O.csmc_run(to_oracle(m), N, ys, threshold=0.6, refresh=REFRESH[refresh].kind,
                              chains=2, iters=4, seed=99)
    np.testing.assert_allclose(tr, otr, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(lls, olls, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("refresh", list(REFRESH))
def test_csmc_converges_to_kalman_smoother(ctx, refresh):
    """test/algorithms/csmc.jl:5-98: Dx = Dy = 1, K = 10, N = 10, threshold 0.6,
    t_smooth = 2; 1184 chains x 1000 kept sweeps."""
    rng = np.random.default_rng(1234)
    m = random_lg(rng, 1, 1)
    K, t_smooth = 10, 2
    _, ys = simulate(rng, m, K)
    ks, ks_ll = G.smooth(m, G.KalmanSmoother(), ys, t_smooth=t_smooth, ctx=ctx)
    kf_ll = O.kf_filter(to_oracle(m), ys)[0]
    csmc = G.ConditionalSMC(G.BF(10, threshold=0.6, resampler=G.Multinomial()), REFRESH[refresh])
    tr, lls, _ = CS.sample(G.CSMCModel(m, ys), csmc, 1000, burnin=100, chains=1184, seed=2024, ctx=ctx)
    mean = tr[:, :, t_smooth, 0].mean()
    np.testing.assert_allclose(mean, ks.mu[0], rtol=1e-3)
    l = -lls.ravel()
    log_recip = l.max() + np.log(np.mean(np.exp(l - l.max())))
    np.testing.assert_allclose(log_recip, -kf_ll, rtol=1e-3)


def test_csmc_single_sweep_and_errors(ctx):
    rng = np.random.default_rng(5)
    m = random_lg(rng, 2, 2)
    _, ys = simulate(rng, m, 4)
    csmc = G.ConditionalSMC(G.BF(8, threshold=0.5))
    traj, ll = CS._csmc_sample(m, csmc, ys, None, seed=1, ctx=ctx)
    assert traj.shape == (5, 2) and np.isfinite(ll)
    # conditioned on traj, the next sweep still returns a (T+1, dx) trajectory
    traj2, ll2 = CS._csmc_sample(m, csmc, ys, traj, seed=2, ctx=ctx)
    assert traj2.shape == (5, 2) and np.isfinite(ll2)
    big = G.ConditionalSMC(G.BF(CS.max_particles() + 1))
    with pytest.raises(G.GFError):
        CS._csmc_sample(m, big, ys, None, ctx=ctx)
    wide = random_lg(rng, 17, 1)
    _, ys17 = simulate(rng, wide, 3)
    with pytest.raises(G.GFError):
        CS._csmc_sample(wide, csmc, ys17, None, ctx=ctx)


@pytest.mark.parametrize("refresh", list(REFRESH))
def test_nonhomogeneous_csmc_matches_oracle(ctx, refresh):
    """A time-varying model: every step's transition (in the propagation, the
    ancestor-sampling and the backward-simulation weights) and observation model
    are that step's; GPU = FP64 oracle on the same injected randomness."""
    rng = np.random.default_rng(300 + len(refresh))
    T, N, chains, iters, burnin, dx, dy = 9, 17, 3, 5, 1, 3, 2
    om = O.create_nonhomogeneous_linear_gaussian_model(rng, dx, dy, T)
    As = [O.random_orthogonal(rng, dx) * rng.uniform(0.5, 0.95) for _ in range(T)]
    om = O.LGModel.time_varying(om.mu0, om.Sigma0, As, om.bs, om.Qs, om.Hs, om.cs, om.Rs)
    gm = G.create_nonhomogeneous_linear_gaussian_model(om.mu0, om.Sigma0, om.As, om.bs, om.Qs, om.Hs,
                                                       om.cs, om.Rs)
    _, ys = O.sample(rng, om, T)
    noise, unif = _inputs(rng, chains, iters, T, N, dx)
    ref0 = rng.standard_normal((chains, T + 1, dx)) if refresh != "backward" else None
    csmc = G.ConditionalSMC(G.BF(N, threshold=0.6, resampler=G.Stratified()), REFRESH[refresh])
    tr, lls, last = CS.sample(G.CSMCModel(gm, ys), csmc, iters - burnin, burnin=burnin, chains=chains,
                              initial=ref0, noise=noise, uniforms=unif, ctx=ctx)
    otr, olls, olast = O.csmc_run(om, N, ys, threshold=0.6, resampler=O.STRATIFIED,
                                  refresh=REFRESH[refresh].kind, chains=chains, iters=iters,
                                  burnin=burnin, ref=ref0, noise=noise, uniforms=unif)
    np.testing.assert_allclose(tr, otr, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(lls, olls, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(last, olast, rtol=1e-9, atol=1e-9)
