"""GPU auxiliary particle filter (AuxiliaryParticleFilter(pf, MeanPredictive()),
particles.jl:247-394; AuxiliaryResampler, resamplers.jl:85-143) against the
FP64 oracle restatement.

Tolerances as for the bootstrap filter: FP64 runs match per-step ll increments
to 1e-9 (absolute), ESS values to 1e-9 (relative) and ancestors bit-exactly
outside a 1e-9 band around cumulative-weight boundaries; the convergence test
repeats test/algorithms/particles.jl:57-82 (ll within 1e-3 of the Kalman
filter, final mean within rtol 1e-2)."""
import numpy as np
import pytest

import gfb200 as G
import oracle as O
from helpers import ancestors_match, injected, random_lg, simulate, to_oracle

pytestmark = pytest.mark.gpu

RS = {O.SYSTEMATIC: G.Systematic(), O.STRATIFIED: G.Stratified(), O.MULTINOMIAL: G.Multinomial()}


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.STRATIFIED, O.MULTINOMIAL])
@pytest.mark.parametrize("mode", ["always", "mixed"])
@pytest.mark.parametrize("dims", [(1, 1), (4, 2)])
def test_apf_f64_injected_matches_oracle(ctx, kind, mode, dims):
    """threshold 1.0 resamples at every step; the "mixed" thresholds (0.97 for the
    1-D model, 0.3 for the 4-D one) alternate resampled and preserved steps."""
    dx, dy = dims
    threshold = 1.0 if mode == "always" else {1: 0.97, 4: 0.3}[dx]
    rng = np.random.default_rng(40 + dx + kind)
    m = random_lg(rng, dx, dy)
    T, N = 8, 1500
    _, ys = simulate(rng, m, T)
    noise, unif = injected(rng, T, dx, N, kind)
    algo = G.AuxiliaryParticleFilter(G.BF(N, threshold=threshold, resampler=RS[kind], precision="f64"),
                                     G.MeanPredictive())
    st, ll = G.filter(m, algo, ys, noise=noise, uniforms=unif, want_ancestors=True, ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, resampler=kind, threshold=threshold, noise=noise,
                   uniforms=unif, want_ancestors=True, want_margins=True, lookahead=1)
    assert st.resampled.sum() >= 1, "workload must exercise the auxiliary resample"
    np.testing.assert_array_equal(st.resampled, ref["resampled"])
    np.testing.assert_allclose(st.ess_steps, ref["ess"], rtol=1e-9)
    bad, boundary = ancestors_match(st.ancestors, ref["ancestors"], ref["margins"], 1e-9)
    assert bad == 0 and boundary == 0
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], atol=1e-9, rtol=0)
    assert abs(ll - ref["ll"]) < 1e-8
    np.testing.assert_allclose(st.particles, ref["x_final"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(st.log_weights, ref["logw_final"], atol=1e-9)


def test_apf_differs_from_bf_only_on_resampling_steps(ctx):
    """Without a resample the first-stage scores are unused (preserve_sample keeps the
    weights), so threshold 0 gives the bootstrap filter's run bit for bit."""
    rng = np.random.default_rng(8)
    m = random_lg(rng, 2, 2)
    T, N = 6, 4096
    _, ys = simulate(rng, m, T)
    bf = G.BF(N, threshold=0.0, precision="f64")
    s0, l0 = G.filter(m, bf, ys, seed=5, ctx=ctx)
    s1, l1 = G.filter(m, G.APF(bf, G.ModePredictive()), ys, seed=5, ctx=ctx)
    assert l0 == l1
    np.testing.assert_array_equal(s0.particles, s1.particles)


@pytest.mark.parametrize("dims", [(16, 8), (32, 16)])
def test_apf_f32_tensor_core_path(ctx, dims):
    """FP32 with the tcgen05 propagation: the per-step ll increments stay within 1e-4 of
    the FP64 oracle on the same injected noise, resampling at both steps (step 1 scores
    the initial uniform weights; step 2 gathers -log eta of the ancestors and shifts
    the baseline).  Longer FP32 runs leave the FP64 particle set: FP32 log-weights move
    a few slots across cumulative-weight boundaries, which is why the bootstrap FP32
    checks are teacher-forced."""
    from gfb200 import workloads as W
    dx, dy = dims
    m, ys = W.lgssm_rot(seed=dx, dx=dx, dy=dy, T=2)
    T, N = 2, 8192
    rng = np.random.default_rng(2)
    noise, unif = injected(rng, T, dx, N, O.SYSTEMATIC, dtype=np.float32)
    algo = G.APF(G.BF(N, threshold=1.0), G.MeanPredictive())
    st, ll = G.filter(m, algo, ys, noise=noise, uniforms=unif, ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, threshold=1.0, noise=noise.astype(np.float64),
                   uniforms=unif, lookahead=1)
    np.testing.assert_array_equal(st.resampled, ref["resampled"])
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], atol=1e-4 * max(1.0, abs(ref["ll"])) / T)


@pytest.mark.parametrize("threshold", [1.0, 0.8])
def test_apf_converges_to_kf(ctx, threshold):
    """test/algorithms/particles.jl:57-82: AuxiliaryParticleFilter(BF(10^6;
    ESSResampler(0.8)), MeanPredictive()) on a 1-D model, T = 4: ll within 1e-3 of
    the Kalman filter, final weighted mean within rtol 1e-2 (threshold 1.0 makes
    every step take the auxiliary resample)."""
    rng = np.random.default_rng(1234)
    m = random_lg(rng, 1, 1)
    _, ys = simulate(rng, m, 4)
    algo = G.APF(G.BF(10**6, threshold=threshold), G.MeanPredictive())
    st, ll = G.filter(m, algo, ys, seed=21, ctx=ctx)
    kll, _, mus, _ = O.kf_filter(to_oracle(m), ys)
    assert abs(ll - kll) <= 1e-3
    w = st.weights()
    np.testing.assert_allclose(np.sum(st.particles[:, 0] * w), mus[-1, 0], rtol=1e-2)
    if threshold == 1.0:
        assert st.resampled.all()


def test_apf_with_path_storage(ctx):
    """The path storage follows the auxiliary filter's ancestors."""
    rng = np.random.default_rng(17)
    m = random_lg(rng, 2, 1)
    T, N = 6, 700
    _, ys = simulate(rng, m, T)
    noise, unif = injected(rng, T, 2, N, O.MULTINOMIAL)
    algo = G.APF(G.BF(N, threshold=0.9, resampler=G.Multinomial(), precision="f64"), G.MeanPredictive())
    st, _ = G.filter(m, algo, ys, noise=noise, uniforms=unif, want_ancestors=True, want_paths=True,
                     ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, resampler=O.MULTINOMIAL, threshold=0.9, noise=noise,
                   uniforms=unif, want_ancestors=True, want_states=True, lookahead=1)
    np.testing.assert_array_equal(st.ancestors, ref["ancestors"])
    np.testing.assert_allclose(st.paths, O.ancestry_paths(ref["ancestors"], ref["states"]),
                               rtol=1e-10, atol=1e-12)



@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.STRATIFIED])
def test_apf_draw_predictive_matches_oracle(ctx, kind):
    """DrawPredictive (particles.jl:377-384): the lookahead point is one draw from the
    transition, from its own Philox stream (regenerated by the oracle); in-kernel
    Philox propagation noise and uniforms, FP64."""
    rng = np.random.default_rng(90 + kind)
    m = random_lg(rng, 3, 2)
    T, N = 8, 2048
    _, ys = simulate(rng, m, T)
    algo = G.APF(G.BF(N, threshold=1.0, resampler=RS[kind], precision="f64"), G.DrawPredictive())
    st, ll = G.filter(m, algo, ys, seed=77, want_ancestors=True, ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, resampler=kind, threshold=1.0, seed=77, want_ancestors=True,
                   want_margins=True, lookahead=2)
    np.testing.assert_array_equal(st.resampled, ref["resampled"])
    bad, boundary = ancestors_match(st.ancestors, ref["ancestors"], ref["margins"], 1e-9)
    assert bad == 0
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], atol=1e-9, rtol=0)


def test_apf_draw_predictive_converges_to_kf(ctx):
    rng = np.random.default_rng(1234)
    m = random_lg(rng, 1, 1)
    _, ys = simulate(rng, m, 4)
    st, ll = G.filter(m, G.APF(G.BF(10**6, threshold=1.0), G.DrawPredictive()), ys, seed=5, ctx=ctx)
    kll = O.kf_filter(to_oracle(m), ys)[0]
    assert abs(ll - kll) <= 1e-3


def test_apf_draw_predictive_needs_bootstrap_proposal(ctx):
    """The lookahead draw uses the transition covariance; other proposals are refused."""
    rng = np.random.default_rng(3)
    m = random_lg(rng, 2, 1)
    _, ys = simulate(rng, m, 3)
    pf = G.ParticleFilter(256, G.OverdispersedProposal(k=2.0), precision="f64")
    with pytest.raises(G.GFError):
        G.filter(m, G.APF(pf, G.DrawPredictive()), ys, seed=1, ctx=ctx)
