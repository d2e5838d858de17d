"""GPU gradients of kf_loglikelihood (integrations/kalman_rrule.jl:22-107,
algorithms/kalman_gradient.jl:89-263) against the FP64 oracle restatement,
which is pinned by finite differences of the Kalman log-likelihood as the
reference's own tests do (test/components/kalman_gradient.jl: symmetrised
perturbations of Q, R and Sigma0).  Both sides are FP64: gradients agree to
1e-9 relative to their largest entry."""
import numpy as np
import pytest

import gfb200 as G
import oracle as O
from helpers import random_lg, simulate, to_oracle

pytestmark = pytest.mark.gpu


def _stable_lg(rng, dx, dy):
    """GFTest's model with A rescaled to spectral radius 0.9 (its U(0,1) entries make
    larger A explosive, and the FP64 comparison then measures conditioning)."""
    om = O.create_linear_gaussian_model(rng, dx, dy)
    A = np.asarray(om.A) * (0.9 / max(np.abs(np.linalg.eigvals(om.A)).max(), 0.9))
    return G.create_homogeneous_linear_gaussian_model(om.mu0, om.Sigma0, A, om.b, om.Q, om.H, om.c, om.R)


def _check(g, r):
    for k in ("mu0", "Sigma0", "A", "b", "Q", "H", "c", "R"):
        scale = np.abs(r[k]).max() + 1e-12
        np.testing.assert_allclose(g[k], r[k], rtol=0, atol=1e-9 * scale, err_msg=k)


@pytest.mark.parametrize("dims", [(2, 2), (1, 1), (3, 2), (5, 4), (16, 16), (8, 3)])
def test_kf_gradient_matches_oracle(ctx, dims):
    dx, dy = dims
    rng = np.random.default_rng(10 * dx + dy)
    m = random_lg(rng, dx, dy) if dx <= 3 else _stable_lg(rng, dx, dy)
    _, ys = simulate(rng, m, 12)
    ll, g = G.kf_loglikelihood_grad(m, ys, ctx=ctx)
    rll, r = O.kf_loglikelihood_grad(to_oracle(m), ys)
    assert abs(ll - rll) <= 1e-10 * abs(rll)
    _check(g, r)


def test_kf_gradient_batch_uneven(ctx):
    """A batch of models of different sizes and lengths equals the per-model results."""
    rng = np.random.default_rng(3)
    models, yss = [], []
    for f in range(40):
        dx = int(rng.integers(1, 9))
        dy = int(rng.integers(1, dx + 1))
        m = _stable_lg(rng, dx, dy)
        _, ys = simulate(rng, m, int(rng.integers(1, 40)))
        models.append(m)
        yss.append(ys)
    res = G.kf_loglikelihood_grad_batch(models, yss, ctx=ctx)
    for (ll, g), m, ys in zip(res, models, yss):
        rll, r = O.kf_loglikelihood_grad(to_oracle(m), ys)
        assert abs(ll - rll) <= 1e-10 * max(1.0, abs(rll))
        _check(g, r)


def test_kf_gradient_ll_equals_kalman_filter(ctx):
    rng = np.random.default_rng(9)
    m = _stable_lg(rng, 4, 3)
    _, ys = simulate(rng, m, 30)
    ll, _ = G.kf_loglikelihood_grad(m, ys, ctx=ctx)
    assert abs(ll - O.kf_filter(to_oracle(m), ys)[0]) <= 1e-10 * abs(ll)
