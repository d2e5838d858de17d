"""GPU parity of the batched Kalman / square-root Kalman filters.

Tolerance (north_star): |d ll| / |ll| <= 1e-4 per filter against the FP64
oracle; per-step means and covariances within 1e-3 relative to their norm
(FP32 storage)."""
import numpy as np
import pytest

import gfb200 as G
import oracle as O
from gfb200 import workloads as W
from helpers import random_lg, simulate, to_oracle

pytestmark = pytest.mark.gpu


def _check(res, models, yss, algo_name, ll_rtol=1e-4, mat_rtol=1e-3):
    worst = 0.0
    for (st, ll), m, ys in zip(res, models, yss):
        rll, rsteps, rmus, rsig = O.kf_filter(to_oracle(m), ys, algo=algo_name)
        rel = abs(ll - rll) / max(1.0, abs(rll))
        worst = max(worst, rel)
        assert rel <= ll_rtol, (rel, ll, rll)
        scale_mu = np.abs(rmus).max(axis=1, keepdims=True) + 1e-3
        assert np.all(np.abs(st.means - rmus) <= mat_rtol * scale_mu + 1e-5)
        scale_s = np.abs(rsig).reshape(len(ys), -1).max(axis=1)[:, None, None]
        assert np.all(np.abs(st.covs - rsig) <= mat_rtol * scale_s + 1e-6)
        np.testing.assert_allclose(st.ll_steps, rsteps, atol=1e-4 * max(1.0, abs(rll)) / len(ys) + 1e-5)
    return worst


@pytest.mark.parametrize("algo", ["kf", "srkf"])
def test_reference_shaped_models(ctx, algo):
    """test/algorithms/kalman.jl:5-43 and srkf.jl:3-26 shapes: Dx=3, Dy in {2,3,4}, T=5."""
    rng = np.random.default_rng(1234)
    models, yss = [], []
    for Dy in (2, 3, 4):
        m = random_lg(rng, 3, Dy)
        _, ys = simulate(rng, m, 5)
        models.append(m)
        yss.append(ys)
    A = G.KalmanFilter() if algo == "kf" else G.SRKF()
    res = G.filter_batch(models, A, yss, ctx=ctx)
    _check(res, models, yss, algo)


def test_kf_matches_joint_gaussian(ctx):
    rng = np.random.default_rng(42)
    for Dy in (2, 3, 4):
        m = random_lg(rng, 3, Dy)
        _, ys = simulate(rng, m, 3)
        (st, ll), = G.filter_batch([m], G.KalmanFilter(), [ys], ctx=ctx)
        mu, S, lt = O.joint_filter_truth(to_oracle(m), ys)
        assert abs(ll - lt) <= 1e-4 * abs(lt)
        np.testing.assert_allclose(st.mu, mu, rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(st.Sigma, S, rtol=1e-3, atol=1e-5)


@pytest.mark.parametrize("algo", ["kf", "srkf"])
def test_uneven_bank(ctx, algo):
    """Batched bank of uneven filters (Dx 2..32, Dy 1..Dx, uneven T)."""
    models, Ts, yss = W.kf_bank(96, seed=5, T_range=(64, 200), simulate=True)
    A = G.KalmanFilter() if algo == "kf" else G.SRKF()
    res = G.filter_batch(models, A, yss, ctx=ctx)
    _check(res, models, yss, algo)


def test_srkf_equals_kf(ctx):
    models, Ts, yss = W.kf_bank(32, seed=6, T_range=(64, 128), simulate=True)
    a = G.filter_batch(models, G.KalmanFilter(), yss, ctx=ctx)
    b = G.filter_batch(models, G.SRKF(), yss, ctx=ctx)
    for (sa, la), (sb, lb) in zip(a, b):
        assert abs(la - lb) <= 1e-4 * max(1.0, abs(la))


def test_jitter_is_applied(ctx):
    rng = np.random.default_rng(3)
    m = random_lg(rng, 4, 2)
    _, ys = simulate(rng, m, 10)
    (st, ll), = G.filter_batch([m], G.KalmanFilter(jitter=1e-2), [ys], ctx=ctx)
    rll, _, rmus, rsig = O.kf_filter(to_oracle(m), ys, jitter=1e-2)
    assert abs(ll - rll) <= 1e-4 * abs(rll)
    np.testing.assert_allclose(st.Sigma, rsig[-1], rtol=1e-3, atol=1e-6)


def test_not_pd_is_reported_per_filter(ctx):
    """An indefinite R makes S non-PD (PosDefException in the reference); the batch
    reports it for that filter only."""
    rng = np.random.default_rng(9)
    good = random_lg(rng, 3, 2)
    bad = random_lg(rng, 3, 2)
    bad.obs.R[:] = -np.eye(2) * 50.0
    _, ys = simulate(rng, good, 5)
    with pytest.raises(G.PosDefException):
        G.filter_batch([good, bad], G.KalmanFilter(), [ys, ys], ctx=ctx)


def test_plan_graph_matches_one_shot(ctx):
    """The graph-captured persistent plan gives the same numbers as gf_kf_batch."""
    import ctypes as C
    import torch
    from gfb200 import _lib as L
    models, Ts, yss = W.kf_bank(200, seed=8, T_range=(64, 300))
    one = G.filter_batch(models, G.KalmanFilter(), yss, ctx=ctx)
    B = len(models)
    mcs = (L.LGModelC * B)(*[m._c_struct() for m in models])
    T = np.array(Ts, np.int32)
    plan = C.c_void_p()
    L.check(ctx.h, L.load().gf_kf_plan_create(ctx.h, 0, mcs, B, T.ctypes.data_as(C.POINTER(C.c_int32)),
                                              0.0, 0, 0, C.byref(plan)))
    try:
        dev = "cuda:0"
        ys = torch.tensor(np.concatenate([y.ravel() for y in yss]), device=dev)
        ll = torch.zeros(B, dtype=torch.float64, device=dev)
        st = torch.zeros(B, dtype=torch.int32, device=dev)
        steps = torch.zeros(int(T.sum()), dtype=torch.float64, device=dev)
        out = L.KFOutC(ll.data_ptr(), steps.data_ptr(), None, None, st.data_ptr())
        for _ in range(2):
            L.check(ctx.h, L.load().gf_kf_plan_run(plan, ys.data_ptr(), C.byref(out)))
        ctx.synchronize()
        np.testing.assert_array_equal(ll.cpu().numpy(), np.array([l for _, l in one]))
        assert int(st.abs().sum()) == 0
    finally:
        L.load().gf_kf_plan_destroy(plan)


def _check_smooth(res, models, yss, mat_rtol=1e-3):
    for (means, covs, ll), m, ys in zip(res, models, yss):
        rll, rmus, rsig = O.rts_smooth(to_oracle(m), ys)
        assert abs(ll - rll) <= 1e-4 * max(1.0, abs(rll)), (ll, rll)
        scale_mu = np.abs(rmus).max(axis=1, keepdims=True) + 1e-3
        assert np.all(np.abs(means - rmus) <= mat_rtol * scale_mu + 1e-5), np.abs(means - rmus).max()
        scale_s = np.abs(rsig).reshape(len(ys), -1).max(axis=1)[:, None, None]
        assert np.all(np.abs(covs - rsig) <= mat_rtol * scale_s + 1e-6), np.abs(covs - rsig).max()


def test_rts_smoother_bank_matches_oracle(ctx):
    """smooth(model, KalmanSmoother(), ys) (kalman.jl:89-126,206-234) for a bank of
    uneven stable models covering every dimension bucket, against the FP64 oracle
    (same tolerances as the filter)."""
    models, Ts, _ = W.kf_bank(40, seed=3, dx_range=(2, 32), T_range=(2, 120), make_ys=False)
    rng = np.random.default_rng(8)
    yss = [simulate(rng, m, T)[1] for m, T in zip(models, Ts)]
    res = G.smooth_batch(models, yss, ctx=ctx)
    _check_smooth(res, models, yss)


def test_rts_smoother_matches_joint_gaussian(ctx):
    """Every smoothed marginal against Gaussian conditioning of the joint."""
    rng = np.random.default_rng(17)
    for Dy in (1, 2, 3):
        m = random_lg(rng, 3, Dy)
        _, ys = simulate(rng, m, 4)
        means, covs, ll = G.smooth_batch([m], [ys], ctx=ctx)[0]
        mt, St = O.joint_smooth_truth(to_oracle(m), ys)
        np.testing.assert_allclose(means, mt, rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(covs, St, rtol=1e-3, atol=1e-5)


def test_smooth_api_t_smooth(ctx):
    """smooth(...; t_smooth) returns that step; at t_smooth = T it is the filtered one."""
    rng = np.random.default_rng(23)
    m = random_lg(rng, 4, 2)
    _, ys = simulate(rng, m, 12)
    st1, ll = G.smooth(m, G.KalmanSmoother(), ys, ctx=ctx)
    stT, _ = G.smooth(m, G.KS, ys, t_smooth=12, ctx=ctx)
    fst, fll = G.filter(m, G.KalmanFilter(), ys, ctx=ctx)
    assert ll == fll
    np.testing.assert_array_equal(stT.mu, fst.mu)
    np.testing.assert_array_equal(stT.Sigma, fst.Sigma)
    np.testing.assert_array_equal(st1.mu, st1.means[0])


def test_plan_smooth_matches_one_shot(ctx):
    """gf_kf_plan_smooth on a resident plan returns exactly what gf_kf_smooth returns."""
    import torch
    from gfb200.plans import KfPlan
    models, Ts, _ = W.kf_bank(12, seed=5, dx_range=(2, 32), T_range=(3, 40), make_ys=False)
    rng = np.random.default_rng(2)
    yss = [simulate(rng, m, T)[1] for m, T in zip(models, Ts)]
    ref = G.smooth_batch(models, yss, ctx=ctx)
    plan = KfPlan(models, G.KalmanFilter(), Ts, ctx=ctx)
    ys = torch.tensor(np.concatenate([y.ravel() for y in yss]), device="cuda:0")
    means = torch.zeros(plan.n_means, dtype=torch.float32, device="cuda:0")
    covs = torch.zeros(plan.n_covs, dtype=torch.float32, device="cuda:0")
    plan.smooth(ys, means, covs)
    ctx.synchronize()
    m_all = np.concatenate([r[0].ravel() for r in ref])
    c_all = np.concatenate([r[1].transpose(0, 2, 1).ravel() for r in ref])
    np.testing.assert_array_equal(means.cpu().numpy(), m_all)
    np.testing.assert_array_equal(covs.cpu().numpy(), c_all)
    np.testing.assert_array_equal(plan.ll.cpu().numpy(), [r[2] for r in ref])
    plan.close()
