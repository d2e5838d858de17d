"""Time-varying (non-homogeneous) linear-Gaussian models on the GPU: the
parameter layer calc_params(dyn, t) / calc_params(obs, t) of
models/linear_gaussian.jl:44-63, with GFTest's
create_nonhomogeneous_linear_gaussian_model (GFTest/models/linear_gaussian.jl:97-119).

Bars: |d ll| / max(1, |ll|) <= 1e-4 against the FP64 oracle; per-step means
and covariances within 1e-3 of their scale (FP32 storage); the oracle itself is
pinned to joint-Gaussian conditioning (tests/test_oracle.py)."""
import numpy as np
import pytest

import gfb200 as G
import oracle as O

pytestmark = pytest.mark.gpu


def _tv_pair(rng, Dx, Dy, T, stable=False):
    """GFTest's generator, or (stable) the same with each A_t a random orthogonal
    matrix scaled to spectral radius in [0.5, 0.95], so long runs stay bounded
    in FP32 (GFTest's A ~ U(0,1)^{Dx x Dx} grows like (Dx/2)^t)."""
    om = O.create_nonhomogeneous_linear_gaussian_model(rng, Dx, Dy, T)
    if stable:
        As = [O.random_orthogonal(rng, Dx) * rng.uniform(0.5, 0.95) for _ in range(T)]
        om = O.LGModel.time_varying(om.mu0, om.Sigma0, As, om.bs, om.Qs, om.Hs, om.cs, om.Rs)
    gm = G.create_nonhomogeneous_linear_gaussian_model(om.mu0, om.Sigma0, om.As, om.bs, om.Qs,
                                                       om.Hs, om.cs, om.Rs)
    _, ys = O.sample(rng, om, T)
    return om, gm, ys


def test_nonhomogeneous_kf_matches_oracle_and_joint_gaussian(ctx):
    """Uneven batch of time-varying models (and one homogeneous model in the same
    launch): every step's ll, mean and covariance equal the oracle's; the final
    filtered moments equal Gaussian conditioning of the joint."""
    rng = np.random.default_rng(11)
    oms, gms, yss = [], [], []
    for Dx, Dy, T in [(2, 2, 4), (3, 1, 30), (5, 3, 64), (12, 7, 40), (20, 9, 25), (32, 16, 50)]:
        om, gm, ys = _tv_pair(rng, Dx, Dy, T, stable=(Dx, T) != (2, 4))
        oms.append(om)
        gms.append(gm)
        yss.append(ys)
    h = O.create_linear_gaussian_model(rng, 4, 2)
    h = O.LGModel(h.mu0, h.Sigma0, O.random_orthogonal(rng, 4) * 0.9, h.b, h.Q, h.H, h.c, h.R)
    oms.append(h)
    gms.append(G.create_homogeneous_linear_gaussian_model(h.mu0, h.Sigma0, h.A, h.b, h.Q, h.H, h.c, h.R))
    yss.append(O.sample(rng, h, 17)[1])
    res = G.filter_batch(gms, G.KalmanFilter(), yss, ctx=ctx)
    for (st, ll), om, ys in zip(res, oms, yss):
        rll, rsteps, rmus, rsig = O.kf_filter(om, ys)
        assert abs(ll - rll) <= 1e-4 * max(1.0, abs(rll)), (ll, rll)
        scale_mu = np.abs(rmus).max(axis=1, keepdims=True) + 1e-3
        assert np.all(np.abs(st.means - rmus) <= 1e-3 * scale_mu + 1e-5)
        scale_s = np.abs(rsig).reshape(len(ys), -1).max(axis=1)[:, None, None]
        assert np.all(np.abs(st.covs - rsig) <= 1e-3 * scale_s + 1e-6)
        # per step: 1e-3 of the step's own size -- GFTest's random A has entries
        # in U(0, 1), so these models grow like rho(A)^t and FP32 storage loses
        # digits over the run (the total ll still meets the 1e-4 bar above)
        np.testing.assert_allclose(st.ll_steps, rsteps, rtol=1e-3, atol=1e-4)
    # the reference test's shape (test/algorithms/kalman.jl:263-300): Dx = Dy = 2, T = 4
    mu, S, lt = O.joint_filter_truth(oms[0], yss[0])
    st, ll = res[0]
    assert abs(ll - lt) <= 1e-4 * max(1.0, abs(lt))
    np.testing.assert_allclose(st.mu, mu, rtol=1e-3, atol=1e-4)
    np.testing.assert_allclose(st.Sigma, S, rtol=1e-3, atol=1e-4)


def test_nonhomogeneous_smoother_matches_joint_gaussian(ctx):
    """The RTS smoother of a time-varying model (kalman.jl:89-126,206-234; the
    predictions from t to t+1 use step t+1's parameters) against the oracle and
    the joint-Gaussian smoothed marginals of every step."""
    rng = np.random.default_rng(12)
    oms, gms, yss = [], [], []
    for Dx, Dy, T in [(2, 2, 3), (4, 2, 12), (9, 5, 20), (16, 8, 30)]:
        om, gm, ys = _tv_pair(rng, Dx, Dy, T, stable=(Dx, T) != (2, 3))
        oms.append(om)
        gms.append(gm)
        yss.append(ys)
    res = G.smooth_batch(gms, yss, ctx=ctx)
    for (means, covs, ll), om, ys in zip(res, oms, yss):
        _, rm, rS = O.rts_smooth(om, ys)
        sm = np.abs(rm).max() + 1e-3
        np.testing.assert_allclose(means, rm, atol=2e-3 * sm)
        ss = np.abs(rS).max()
        np.testing.assert_allclose(covs, rS, atol=2e-3 * ss)
    mj, Sj = O.joint_smooth_truth(oms[0], yss[0])
    np.testing.assert_allclose(res[0][0], mj, rtol=1e-3, atol=1e-4)
    np.testing.assert_allclose(res[0][1], Sj, rtol=1e-3, atol=1e-4)


def test_nonhomogeneous_needs_a_block_per_step(ctx):
    """Fewer parameter steps than observations is an argument error, not a read
    past the model."""
    rng = np.random.default_rng(13)
    om, gm, ys = _tv_pair(rng, 3, 2, 5)
    with pytest.raises(ValueError):
        G.filter_batch([gm], G.KalmanFilter(), [np.vstack([ys, ys])], ctx=ctx)
    with pytest.raises(ValueError):
        G.filter_batch([gm], G.SRKF(), [np.vstack([ys, ys])], ctx=ctx)


def test_nonhomogeneous_srkf_matches_oracle(ctx):
    """The square-root filter (srkf.jl:93-176) on time-varying models: each step's
    A, b, H, c and the Cholesky factors of Q_t and R_t are that step's.  Uneven
    batch with a homogeneous model mixed in; every step's ll, mean and covariance
    against the FP64 oracle KF, at the bars of the time-varying KF test."""
    rng = np.random.default_rng(29)
    oms, gms, yss = [], [], []
    for Dx, Dy, T in [(2, 2, 4), (3, 1, 30), (6, 3, 40), (16, 8, 25), (32, 16, 20)]:
        om, gm, ys = _tv_pair(rng, Dx, Dy, T, stable=(Dx, T) != (2, 4))
        oms.append(om)
        gms.append(gm)
        yss.append(ys)
    h = O.create_linear_gaussian_model(rng, 4, 2)
    h = O.LGModel(h.mu0, h.Sigma0, O.random_orthogonal(rng, 4) * 0.9, h.b, h.Q, h.H, h.c, h.R)
    oms.append(h)
    gms.append(G.create_homogeneous_linear_gaussian_model(h.mu0, h.Sigma0, h.A, h.b, h.Q, h.H, h.c, h.R))
    yss.append(O.sample(rng, h, 17)[1])
    res = G.filter_batch(gms, G.SRKF(), yss, ctx=ctx)
    for (st, ll), om, ys in zip(res, oms, yss):
        rll, rsteps, rmus, rsig = O.kf_filter(om, ys)
        assert abs(ll - rll) <= 1e-4 * max(1.0, abs(rll)), (ll, rll)
        scale_mu = np.abs(rmus).max(axis=1, keepdims=True) + 1e-3
        assert np.all(np.abs(st.means - rmus) <= 1e-3 * scale_mu + 1e-5)
        scale_s = np.abs(rsig).reshape(len(ys), -1).max(axis=1)[:, None, None]
        assert np.all(np.abs(st.covs - rsig) <= 1e-3 * scale_s + 1e-6)
        np.testing.assert_allclose(st.ll_steps, rsteps, rtol=1e-3, atol=1e-4)
