"""GPU parity of the Rao-Blackwellised PF (per-particle Kalman banks).

FP32 bank with FP64 innovation Cholesky: per-step ll increments within 1e-4
relative of the FP64 oracle fed the same injected noise and uniforms (one
resample at step 1, as GFTest's AlternatingResampler does); convergence to the
exact KF of the joint model within the reference's 1e-3 (test/algorithms/rbpf.jl:5-34)."""
import numpy as np
import pytest

import gfb200 as G
import oracle as O
from gfb200 import workloads as W
from helpers import dummy_rb_model, simulate, to_oracle, to_oracle_rb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 4, 2), (2, 8, 4)])
def test_rbpf_matches_oracle(ctx, dims):
    rng = np.random.default_rng(sum(dims))
    full, hier = dummy_rb_model(rng, *dims)
    _, ys = simulate(rng, full, 10)
    N, T = 2048, 10
    noise = rng.standard_normal((T + 1, dims[0], N)).astype(np.float32)
    unif = rng.random(T)
    algo = G.RBPF(G.BF(N, resampler=G.AlternatingResampler()), G.KalmanFilter())
    st, ll = G.filter(hier, algo, ys, noise=noise, uniforms=unif, want_ancestors=True,
                      want_means=True, ctx=ctx)
    ref = O.rbpf_run(to_oracle_rb(hier), N, ys, schedule=[1] + [0] * (T - 1),
                     noise=noise.astype(np.float64), uniforms=unif, want_ancestors=True)
    np.testing.assert_array_equal(st.ancestors, ref["ancestors"])
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(st.means, ref["means"], rtol=1e-3, atol=1e-4)
    np.testing.assert_allclose(st.zmeans, ref["zmeans"], rtol=1e-3, atol=1e-4)


def test_rbpf_converges_to_kf(ctx):
    """Reference tolerances (ll 1e-3 absolute, means 1e-3 relative) at N = 2^22."""
    rng = np.random.default_rng(1234)
    full, hier = dummy_rb_model(rng, 1, 1, 1)
    _, ys = simulate(rng, full, 4)
    algo = G.RBPF(G.BF(2**22, resampler=G.AlternatingResampler()), G.KalmanFilter())
    st, ll = G.filter(hier, algo, ys, seed=31, ctx=ctx)
    llkf, _, mus, _ = O.kf_filter(to_oracle(full), ys)
    w = st.weights()
    assert abs(ll - llkf) <= 1e-3
    assert abs(np.sum(st.particles["x"][:, 0] * w) - mus[-1, 0]) <= 1e-3 * abs(mus[-1, 0])
    assert abs(np.sum(st.particles["mu"][:, 0] * w) - mus[-1, 1]) <= 1e-3 * abs(mus[-1, 1])


def test_guided_rbpf_matches_oracle(ctx):
    rng = np.random.default_rng(77)
    full, hier = dummy_rb_model(rng, 1, 1, 1)
    _, ys = simulate(rng, full, 8)
    N, T = 1024, 8
    noise = rng.standard_normal((T + 1, 1, N)).astype(np.float32)
    unif = rng.random(T)
    prop = G.OverdispersedProposal(hier.outer_dyn, 1.5)
    algo = G.RBPF(G.PF(N, prop, resampler=G.AlternatingResampler()), G.KalmanFilter())
    st, ll = G.filter(hier, algo, ys, noise=noise, uniforms=unif, ctx=ctx)
    ref = O.rbpf_run(to_oracle_rb(hier), N, ys, schedule=[1] + [0] * (T - 1),
                     noise=noise.astype(np.float64), uniforms=unif,
                     proposal=O.PROP_OVERDISPERSED, k=1.5)
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], rtol=1e-4, atol=1e-4)


def test_trend_model_full_size(ctx):
    """N = 65536, T = 500 stochastic-volatility RBPF: invariants of the full run."""
    model, ys = W.rb_trend(seed=1)
    algo = G.RBPF(G.BF(65536, threshold=0.5), G.KalmanFilter())
    st, ll = G.filter(model, algo, ys, seed=2, ctx=ctx)
    assert np.isfinite(ll)
    assert st.resampled.sum() > 0 and st.clamps == 0
    assert np.all(st.ess_steps > 0) and np.all(st.ess_steps <= 65536 * (1 + 1e-9))
    S = st.particles["Sigma"]
    assert np.all(np.linalg.eigvalsh(S[:1000].astype(np.float64)) > 0)


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.MULTINOMIAL])
def test_rbpf_ancestry_callbacks(ctx, kind):
    """test/algorithms/rbpf.jl:211-234 (AncestorCallback on an RBPF gives one path per
    particle) and the dense container of the same run: the device path storage's
    trajectories equal the walk through the recorded per-step states (packed
    [x | mu | Sigma upper] states), and the last recorded states are the final ones."""
    rng = np.random.default_rng(21 + kind)
    full, hier = dummy_rb_model(rng, 1, 2, 1)
    T, N = 6, 3000
    _, ys = simulate(rng, full, T)
    rs = {O.SYSTEMATIC: G.Systematic(), O.MULTINOMIAL: G.Multinomial()}[kind]
    algo = G.RBPF(G.BF(N, threshold=0.8, resampler=rs), G.KalmanFilter())
    cb = G.AncestorCallback()
    st, ll = G.filter(hier, algo, ys, seed=3, callback=cb, ctx=ctx)
    paths = G.get_ancestry(cb.tree)
    assert len(paths) == N and paths.shape[1] == T + 1
    dcb = G.DenseAncestorCallback()
    st2, ll2 = G.filter(hier, algo, ys, seed=3, callback=dcb, ctx=ctx)
    assert ll2 == ll
    dense = G.get_ancestry(dcb.container, ctx=ctx)
    np.testing.assert_array_equal(paths, dense)
    last = dcb.container.states[-1]  # [N, width]: x (1), mu (2), Sigma packed (3)
    np.testing.assert_array_equal(last[:, :1], np.asarray(st2.particles["x"]).reshape(N, 1))
    np.testing.assert_array_equal(last[:, 1:3], np.asarray(st2.particles["mu"]).reshape(N, 2))


@pytest.mark.parametrize("pp", ["mean", "draw"])
@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.MULTINOMIAL])
def test_auxiliary_rbpf_matches_oracle(ctx, pp, kind):
    """AuxiliaryParticleFilter(RBPF(BF(N), KalmanFilter()), pp) (rbpf.jl:86-124) on the
    stochastic-volatility model, whose inner Q scales with exp(x*[1]), so the mean and
    the draw of the outer transition give different first-stage scores.  Resamples are
    forced at steps 1 and 4 (the second on non-uniform weights); the FP32 bank against
    the FP64 oracle on the same injected noise, uniforms and lookahead seed: ESS of
    softmax(logw + log eta) within 1e-4, ancestors exact outside a 1e-6 band around
    the cumulative-weight boundaries (band cases counted), per-step ll within 1e-4."""
    from helpers import ancestors_match
    model, ys = W.rb_trend(seed=9, T=8, dz=4, dy=2)
    T, N = 8, 2048
    rng = np.random.default_rng(31 + kind)
    noise = rng.standard_normal((T + 1, 2, N)).astype(np.float32)
    unif = rng.random(T) if kind == O.SYSTEMATIC else rng.random((T, N))
    sched = [1, 0, 0, 1, 0, 0, 0, 0]
    rs = {O.SYSTEMATIC: G.Systematic(), O.MULTINOMIAL: G.Multinomial()}[kind]
    p = G.MeanPredictive() if pp == "mean" else G.DrawPredictive()
    algo = G.APF(G.RBPF(G.BF(N, resampler=rs), G.KalmanFilter()), p)
    st, ll = G.filter(model, algo, ys, noise=noise, uniforms=unif, schedule=sched, seed=17,
                      want_ancestors=True, want_means=True, ctx=ctx)
    la = 1 if pp == "mean" else 2
    om = to_oracle_rb(model)
    ref = O.rbpf_run(om, N, ys, resampler=kind, schedule=sched, noise=noise.astype(np.float64),
                     uniforms=unif, seed=17, want_ancestors=True, want_margins=True, lookahead=la)
    plain = O.rbpf_run(om, N, ys, resampler=kind, schedule=sched, noise=noise.astype(np.float64),
                       uniforms=unif, seed=17, lookahead=0)
    assert abs(ref["ll"] - plain["ll"]) > 1e-6, "the first stage must change the estimate"
    np.testing.assert_array_equal(st.resampled, ref["resampled"])
    np.testing.assert_allclose(st.ess_steps, ref["ess"], rtol=1e-4)
    bad, boundary = ancestors_match(st.ancestors, ref["ancestors"], ref["margins"], 1e-6)
    print(f"auxiliary RBPF ({pp}, resampler {kind}): ancestor boundary cases {boundary}")
    assert bad == 0
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(st.means, ref["means"], rtol=1e-3, atol=1e-4)


def test_auxiliary_rbpf_converges_to_kf(ctx):
    """The auxiliary RBPF's log-evidence at N = 2^22, resampling at every step, within
    the reference's 1e-3 of the joint Kalman filter (test/algorithms/rbpf.jl:5-34)."""
    rng = np.random.default_rng(1234)
    full, hier = dummy_rb_model(rng, 1, 1, 1)
    _, ys = simulate(rng, full, 4)
    algo = G.APF(G.RBPF(G.BF(2**22, threshold=1.0), G.KalmanFilter()), G.MeanPredictive())
    st, ll = G.filter(hier, algo, ys, seed=31, ctx=ctx)
    llkf = O.kf_filter(to_oracle(full), ys)[0]
    assert st.resampled.all()
    assert abs(ll - llkf) <= 1e-3


def test_auxiliary_rbpf_without_resampling_is_the_rbpf(ctx):
    """threshold 0: the first-stage scores are computed but never used, so the run is
    the plain RBPF's bit for bit."""
    model, ys = W.rb_trend(seed=5, T=6, dz=4, dy=2)
    bf = G.BF(4096, threshold=0.0)
    s0, l0 = G.filter(model, G.RBPF(bf, G.KalmanFilter()), ys, seed=5, ctx=ctx)
    s1, l1 = G.filter(model, G.APF(G.RBPF(bf, G.KalmanFilter()), G.DrawPredictive()), ys, seed=5,
                      ctx=ctx)
    assert l0 == l1
    np.testing.assert_array_equal(s0.particles["x"], s1.particles["x"])


@pytest.mark.parametrize("apf", [False, True])
def test_nonhomogeneous_rbpf_matches_oracle(ctx, apf):
    """A time-varying hierarchical model (every outer, inner and observation
    parameter of step t its own): the FP32 bank against the FP64 oracle on the
    same injected noise and uniforms, resampling at steps 1 and 4 (plain RBPF and
    AuxiliaryParticleFilter(RBPF, MeanPredictive())).  Bars as the homogeneous
    parity test."""
    from helpers import ancestors_match, tv_rb_model, tv_rb_oracle_pair
    rng = np.random.default_rng(41 + apf)
    T, N = 8, 2048
    joint, rb = tv_rb_oracle_pair(rng, T, 2, 4, 2)
    _, ys = O.sample(rng, joint, T)
    hier = tv_rb_model(rb)
    noise = rng.standard_normal((T + 1, 2, N)).astype(np.float32)
    unif = rng.random(T)
    sched = [1, 0, 0, 1, 0, 0, 0, 0]
    algo = G.RBPF(G.BF(N), G.KalmanFilter())
    if apf:
        algo = G.APF(algo, G.MeanPredictive())
    st, ll = G.filter(hier, algo, ys, noise=noise, uniforms=unif, schedule=sched, seed=9,
                      want_ancestors=True, want_means=True, ctx=ctx)
    ref = O.rbpf_run(rb, N, ys, schedule=sched, noise=noise.astype(np.float64), uniforms=unif, seed=9,
                     want_ancestors=True, want_margins=True, lookahead=int(apf))
    bad, boundary = ancestors_match(st.ancestors, ref["ancestors"], ref["margins"], 1e-6)
    print(f"time-varying RBPF (apf={apf}): ancestor boundary cases {boundary}")
    assert bad == 0
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(st.means, ref["means"], rtol=1e-3, atol=1e-4)
    np.testing.assert_allclose(st.zmeans, ref["zmeans"], rtol=1e-3, atol=1e-4)


def test_nonhomogeneous_rbpf_converges_to_kf(ctx):
    """N = 2^22 on a time-varying hierarchical model that is jointly linear-Gaussian:
    the log-evidence within the reference's 1e-3 of the joint time-varying KF."""
    from helpers import tv_rb_model, tv_rb_oracle_pair
    rng = np.random.default_rng(1234)
    T = 4
    joint, rb = tv_rb_oracle_pair(rng, T, 1, 1, 1)
    _, ys = O.sample(rng, joint, T)
    algo = G.RBPF(G.BF(2**22, resampler=G.AlternatingResampler()), G.KalmanFilter())
    st, ll = G.filter(tv_rb_model(rb), algo, ys, seed=31, ctx=ctx)
    assert abs(ll - O.kf_filter(joint, ys)[0]) <= 1e-3

