"""GPU backward information filter and two-filter smoother (kalman.jl:236-370)
against the FP64 oracle restatement (pinned to the joint-Gaussian information and
to the RTS smoother in tests/test_oracle.py).  Both sides are FP64: natural
parameters and smoothed moments agree to 1e-9 of each array's largest entry."""
import numpy as np
import pytest

import gfb200 as G
import oracle as O
from helpers import random_lg, simulate, to_oracle

pytestmark = pytest.mark.gpu


def _stable_lg(rng, dx, dy):
    om = O.create_linear_gaussian_model(rng, dx, dy)
    A = np.asarray(om.A) * (0.9 / max(np.abs(np.linalg.eigvals(om.A)).max(), 0.9))
    return G.create_homogeneous_linear_gaussian_model(om.mu0, om.Sigma0, A, om.b, om.Q, om.H, om.c, om.R)


def _close(a, b, name):
    scale = np.abs(b).max() + 1e-12
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-9 * scale, err_msg=name)


@pytest.mark.parametrize("dims", [(3, 2), (3, 4), (1, 1), (6, 3), (16, 16)])
def test_backward_information_matches_oracle(ctx, dims):
    dx, dy = dims
    rng = np.random.default_rng(7 * dx + dy)
    m = random_lg(rng, dx, dy) if dx <= 3 else _stable_lg(rng, dx, dy)
    _, ys = simulate(rng, m, 9)
    r = G.backward_information_batch([m], [ys], initial_jitter=1e-8, ctx=ctx)[0]
    lp, Op, lu, Ou = O.backward_information(to_oracle(m), ys, initial_jitter=1e-8)
    _close(r["lam_pred"], lp, "lam_pred")
    _close(r["Om_pred"], Op, "Om_pred")
    _close(r["lam_upd"], lu, "lam_upd")
    _close(r["Om_upd"], Ou, "Om_upd")
    mus, Ss = O.two_filter_smooth(to_oracle(m), ys, initial_jitter=1e-8)
    _close(r["mu_smooth"], mus, "mu_smooth")
    _close(r["Sigma_smooth"], Ss, "Sigma_smooth")


def test_two_filter_smoother_equals_rts_on_gpu(ctx):
    """test/algorithms/kalman.jl:363-412: two-filter smoothed moments equal the
    RTS smoother's (gf_kf_smooth) at every time."""
    rng = np.random.default_rng(5)
    m = _stable_lg(rng, 4, 2)
    _, ys = simulate(rng, m, 12)
    mus, covs = G.two_filter_smooth_all(m, ys, initial_jitter=1e-10, ctx=ctx)
    _, mr, Sr = O.rts_smooth(to_oracle(m), ys)
    np.testing.assert_allclose(mus, mr, rtol=1e-7, atol=1e-9)
    np.testing.assert_allclose(covs, Sr, rtol=1e-7, atol=1e-9)


def test_backward_information_uneven_batch(ctx):
    rng = np.random.default_rng(11)
    models, yss = [], []
    for _ in range(30):
        dx = int(rng.integers(1, 8))
        dy = int(rng.integers(1, dx + 2))
        m = _stable_lg(rng, dx, dy)
        _, ys = simulate(rng, m, int(rng.integers(1, 25)))
        models.append(m)
        yss.append(ys)
    res = G.backward_information_batch(models, yss, initial_jitter=1e-8, jitter=1e-12, ctx=ctx)
    for r, m, ys in zip(res, models, yss):
        lp, Op, lu, Ou = O.backward_information(to_oracle(m), ys, initial_jitter=1e-8, jitter=1e-12)
        _close(r["Om_upd"], Ou, "Om_upd")
        _close(r["lam_upd"], lu, "lam_upd")
        mus, Ss = O.two_filter_smooth(to_oracle(m), ys, initial_jitter=1e-8, jitter=1e-12)
        _close(r["mu_smooth"], mus, "mu_smooth")


def test_nonhomogeneous_backward_information_matches_oracle(ctx):
    """Time-varying models (test/algorithms/kalman.jl:139-190 runs the backward
    predictor on one): each step's dynamics and observation blocks are used where
    the reference's calc_params(dyn, iter + 1) / calc_params(obs, iter) put them.
    An uneven batch with a homogeneous model in the same launch; FP64 both sides."""
    rng = np.random.default_rng(23)
    oms, gms, yss = [], [], []
    for dx, dy, T in [(2, 2, 4), (3, 1, 9), (5, 3, 12), (8, 8, 7)]:
        om = O.create_nonhomogeneous_linear_gaussian_model(rng, dx, dy, T)
        As = [O.random_orthogonal(rng, dx) * rng.uniform(0.5, 0.95) for _ in range(T)]
        om = O.LGModel.time_varying(om.mu0, om.Sigma0, As, om.bs, om.Qs, om.Hs, om.cs, om.Rs)
        gm = G.create_nonhomogeneous_linear_gaussian_model(om.mu0, om.Sigma0, om.As, om.bs, om.Qs,
                                                           om.Hs, om.cs, om.Rs)
        oms.append(om)
        gms.append(gm)
        yss.append(O.sample(rng, om, T)[1])
    h = _stable_lg(rng, 4, 2)
    oms.append(to_oracle(h))
    gms.append(h)
    yss.append(simulate(rng, h, 10)[1])
    res = G.backward_information_batch(gms, yss, initial_jitter=1e-8, ctx=ctx)
    for r, om, ys in zip(res, oms, yss):
        lp, Op, lu, Ou = O.backward_information(om, ys, initial_jitter=1e-8)
        _close(r["lam_pred"], lp, "lam_pred")
        _close(r["Om_pred"], Op, "Om_pred")
        _close(r["lam_upd"], lu, "lam_upd")
        _close(r["Om_upd"], Ou, "Om_upd")
        mus, Ss = O.two_filter_smooth(om, ys, initial_jitter=1e-8)
        _close(r["mu_smooth"], mus, "mu_smooth")
        _close(r["Sigma_smooth"], Ss, "Sigma_smooth")
