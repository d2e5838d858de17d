"""Particle filters on time-varying linear-Gaussian models (calc_params(dyn, t),
calc_params(obs, t) of models/linear_gaussian.jl:44-63; GFTest's non-homogeneous
model, GFTest/models/linear_gaussian.jl:42-119).

Bars: FP64 runs equal the FP64 oracle on the same injected randomness (per-step
ll within 1e-9, ancestors exact); FP32 runs without resampling keep states within
2e-5 of the oracle's scale; the bootstrap log-likelihood converges to the exact
time-varying Kalman value."""
import numpy as np
import pytest

import gfb200 as G
import oracle as O

pytestmark = pytest.mark.gpu


def _tv(rng, Dx, Dy, T, rho=(0.5, 0.95)):
    om = O.create_nonhomogeneous_linear_gaussian_model(rng, Dx, Dy, T)
    As = [O.random_orthogonal(rng, Dx) * rng.uniform(*rho) for _ in range(T)]
    om = O.LGModel.time_varying(om.mu0, om.Sigma0, As, om.bs, om.Qs, om.Hs, om.cs, om.Rs)
    gm = G.create_nonhomogeneous_linear_gaussian_model(om.mu0, om.Sigma0, om.As, om.bs, om.Qs,
                                                       om.Hs, om.cs, om.Rs)
    _, ys = O.sample(rng, om, T)
    return om, gm, ys


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.STRATIFIED, O.MULTINOMIAL])
@pytest.mark.parametrize("lookahead", [0, 1])
def test_tv_pf_f64_matches_oracle(ctx, kind, lookahead):
    rng = np.random.default_rng(20 + kind + 3 * lookahead)
    om, gm, ys = _tv(rng, 3, 2, 15)
    N, T = 2000, 15
    noise = rng.standard_normal((T + 1, 3, N))
    unif = rng.random(T) if kind == O.SYSTEMATIC else rng.random((T, N))
    rs = {O.SYSTEMATIC: G.Systematic(), O.STRATIFIED: G.Stratified(), O.MULTINOMIAL: G.Multinomial()}[kind]
    pf = G.BF(N, threshold=0.6, resampler=rs, precision="f64")
    algo = G.AuxiliaryParticleFilter(pf, G.MeanPredictive()) if lookahead else pf
    st, ll = G.filter(gm, algo, ys, noise=noise, uniforms=unif, want_ancestors=True, ctx=ctx)
    ref = O.pf_run(om, N, ys, resampler=kind, threshold=0.6, noise=noise, uniforms=unif,
                   want_ancestors=True, lookahead=lookahead)
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], rtol=0, atol=1e-9)
    np.testing.assert_array_equal(st.ancestors, ref["ancestors"])
    assert st.resampled.sum() >= 2


@pytest.mark.parametrize("prop", ["optimal", "overdispersed"])
@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.MULTINOMIAL])
def test_tv_guided_pf_f64_matches_oracle(ctx, prop, kind):
    """Guided proposals (GFTest/proposals.jl:11-50) on a time-varying model: each
    step's proposal factors and log-normaliser difference are that step's."""
    rng = np.random.default_rng(40 + kind + (prop == "optimal"))
    om, gm, ys = _tv(rng, 3, 2, 12)
    N, T = 2000, 12
    noise = rng.standard_normal((T + 1, 3, N))
    unif = rng.random(T) if kind == O.SYSTEMATIC else rng.random((T, N))
    rs = {O.SYSTEMATIC: G.Systematic(), O.MULTINOMIAL: G.Multinomial()}[kind]
    q = G.OptimalProposal() if prop == "optimal" else G.OverdispersedProposal(k=1.6)
    algo = G.PF(N, q, threshold=0.6, resampler=rs, precision="f64")
    st, ll = G.filter(gm, algo, ys, noise=noise, uniforms=unif, want_ancestors=True, ctx=ctx)
    ref = O.pf_run(om, N, ys, resampler=kind, threshold=0.6, noise=noise, uniforms=unif,
                   want_ancestors=True,
                   proposal=O.PROP_OPTIMAL if prop == "optimal" else O.PROP_OVERDISPERSED,
                   k=1.0 if prop == "optimal" else 1.6)
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], rtol=0, atol=1e-9)
    np.testing.assert_array_equal(st.ancestors, ref["ancestors"])
    assert st.resampled.sum() >= 2


@pytest.mark.parametrize("dx,dy", [(4, 3), (16, 8)])
def test_tv_pf_f32_matches_oracle_without_resampling(ctx, dx, dy):
    """FP32 state (the tensor-core path at Dx = 16): every step's parameters reach
    the kernels; no resampling keeps the particles aligned with the oracle's."""
    rng = np.random.default_rng(30 + dx)
    om, gm, ys = _tv(rng, dx, dy, 10)
    N, T = 3000, 10
    noise = rng.standard_normal((T + 1, dx, N)).astype(np.float32)
    st, ll = G.filter(gm, G.BF(N, threshold=0.0), ys, noise=noise, ctx=ctx)
    ref = O.pf_run(om, N, ys, threshold=0.0, noise=noise.astype(np.float64))
    scale = np.abs(ref["x_final"]).max()
    np.testing.assert_allclose(st.particles, ref["x_final"], rtol=0, atol=2e-5 * max(1.0, scale))
    # FP32 log-weights without resampling grow to hundreds: 5e-4 relative
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], rtol=5e-4, atol=1e-3)


def test_tv_bootstrap_converges_to_tv_kalman(ctx):
    """The bootstrap ll of a time-varying model against the exact time-varying KF
    (as test/algorithms/particles.jl:5-27 checks for homogeneous models)."""
    rng = np.random.default_rng(41)
    om, gm, ys = _tv(rng, 2, 2, 6)
    lls = [G.filter(gm, G.BF(2 ** 20, threshold=0.5, precision="f64"), ys, seed=s, ctx=ctx)[1]
           for s in range(3)]
    llkf = O.kf_filter(om, ys)[0]
    assert abs(np.mean(lls) - llkf) < 1e-2, (lls, llkf)
    (kst, kll), = G.filter_batch([gm], G.KalmanFilter(), [ys], ctx=ctx)
    assert abs(kll - llkf) <= 1e-4 * max(1.0, abs(llkf))
