"""GPU resampling primitives: sample_ancestors, offspring <-> ancestors.

Known answers from test/components/resamplers.jl:76-92; the importance-weight
workload of :5-74 (N = 10^6) checked against the FP64 oracle bit-exactly
outside a 1e-9 boundary band, and statistically (resampled mean, rtol 0.1)."""
import numpy as np
import pytest

import gfb200 as G
import oracle as O
from helpers import ancestors_match

pytestmark = pytest.mark.gpu

KINDS = [(O.SYSTEMATIC, G.Systematic()), (O.STRATIFIED, G.Stratified()),
         (O.MULTINOMIAL, G.Multinomial())]


def _tensor(a, dtype=None):
    import torch
    return torch.tensor(a, dtype=dtype, device="cuda:0")


def test_offspring_to_ancestors_known_answer(ctx):
    import torch
    out = G.offspring_to_ancestors(_tensor([0, 2, 2, 3, 5], torch.int64), ctx=ctx)
    assert out.cpu().tolist() == [2, 2, 4, 5, 5]


def test_ancestors_to_offspring_known_answer(ctx):
    import torch
    out = G.ancestors_to_offspring(_tensor([4, 2, 2, 3, 1], torch.int64), ctx=ctx)
    assert out.cpu().tolist() == [1, 2, 1, 1, 0]


def _importance_weights(n, seed=1234):
    rng = np.random.default_rng(seed)
    xs = rng.standard_normal(n)
    ws = np.exp(-0.5 * (xs - 1) ** 2) / np.exp(-0.5 * xs ** 2)
    return xs, ws / ws.sum(), rng


@pytest.mark.parametrize("kind,rs", KINDS)
@pytest.mark.parametrize("conv", ["cpu", "cudaext"])
def test_sample_ancestors_matches_oracle(ctx, kind, rs, conv):
    import torch
    n = 10**6
    xs, ws, rng = _importance_weights(n)
    u = rng.random(1 if kind == O.SYSTEMATIC else n)
    anc = G.sample_ancestors(rs, _tensor(ws, torch.float64), _tensor(u, torch.float64),
                             convention=conv, ctx=ctx).cpu().numpy()
    ref, mar, cl = O.sample_ancestors(kind, ws, u, conv=O.CONV_CUDAEXT if conv == "cudaext" else O.CONV_CPU)
    bad, boundary = ancestors_match(anc, ref, mar, 1e-9)
    assert bad == 0, (bad, boundary)
    mu0 = np.sum(ws * xs)
    mu1 = xs[anc - 1].mean()
    assert abs(mu1 - mu0) <= 0.1 * abs(mu0)


def test_sample_ancestors_edge_cases(ctx):
    import torch
    # one particle
    a = G.sample_ancestors(G.Systematic(), _tensor([3.0], torch.float64), _tensor([0.3], torch.float64), ctx=ctx)
    assert a.cpu().tolist() == [1]
    # all mass on one particle
    w = np.zeros(1000)
    w[417] = 1.0
    a = G.sample_ancestors(G.Systematic(), _tensor(w, torch.float64), _tensor([0.5], torch.float64), ctx=ctx)
    assert set(a.cpu().tolist()) == {418}
    # unnormalised weights give the same ancestors as normalised ones
    xs, ws, rng = _importance_weights(5000, seed=3)
    u = _tensor([0.25], torch.float64)
    a1 = G.sample_ancestors(G.Systematic(), _tensor(ws, torch.float64), u, ctx=ctx).cpu().numpy()
    a2 = G.sample_ancestors(G.Systematic(), _tensor(ws * 8.0, torch.float64), u, ctx=ctx).cpu().numpy()
    np.testing.assert_array_equal(a1, a2)
    # all-zero weights are an error, not a silent result
    with pytest.raises(G.GFError):
        G.sample_ancestors(G.Systematic(), _tensor(np.zeros(10), torch.float64), u, ctx=ctx)


def test_ragged_sizes(ctx):
    """Sizes around the scan tile (4096) and odd sizes exercise partial tiles."""
    import torch
    for n in (1, 7, 4095, 4096, 4097, 12289, 100003):
        rng = np.random.default_rng(n)
        w = rng.random(n)
        u = rng.random(n)
        anc = G.sample_ancestors(G.Stratified(), _tensor(w, torch.float64), _tensor(u, torch.float64),
                                 ctx=ctx).cpu().numpy()
        ref, mar, _ = O.sample_ancestors(O.STRATIFIED, w / w.sum(), u)
        bad, _ = ancestors_match(anc, ref, mar, 1e-9)
        assert bad == 0, n
