"""GPU parity at the benchmark configurations, against the FP64 oracle.

* Large bootstrap PF (Dx=16/Dy=8 and Dx=64/Dy=32, FP32 state on the
  tensor-core propagation, FP64 normaliser): one GPU run records every step's
  states, normalised log-weights and ancestors; each step is then re-done by
  the oracle from the GPU's own previous state with the same injected noise and
  uniforms (teacher forcing), for the systematic, stratified and multinomial
  resamplers.  Bars: resampling decisions equal; ancestors bit-exact except
  where a slot's threshold lies within 1e-8 of a cumulative-weight boundary
  (those boundary cases are counted and printed); states within 2e-5; ll
  increments within 1e-4 + 2e-6 |ll_inc| (FP32 log-weights: at Dx=64/Dy=32 a
  particle's log-weight is a sum of 32 squared residuals of size ~1e2, whose
  FP32 rounding alone is ~1e-4).
* Rao-Blackwellised PF (config-4 model: outer 2-D, inner Dx=8, Dy=4) with
  ESS-triggered systematic resampling over 60 steps, teacher-forced the same
  way through the oracle's RBPF step: decisions equal, ancestors exact outside
  the band, outer states within 2e-5, inner means and covariances within 1e-4
  of their scale, ll increments within 1e-4 relative.
* Batched Kalman and square-root Kalman filters over a 260-filter bank of the
  config-3 distribution with simulated observations, including T = 2048 at
  spectral radius 0.99: |d ll| / max(1, |ll|) <= 1e-4 per filter, per-step means
  and covariances within 1e-3 of their scale (FP32 storage).
"""
import numpy as np
import pytest

import gfb200 as G
import oracle as O
from gfb200 import workloads as W
from helpers import ancestors_match, to_oracle, to_oracle_rb

pytestmark = pytest.mark.gpu

RS = {O.SYSTEMATIC: G.Systematic(), O.STRATIFIED: G.Stratified(), O.MULTINOMIAL: G.Multinomial()}
NAMES = {O.SYSTEMATIC: "systematic", O.STRATIFIED: "stratified", O.MULTINOMIAL: "multinomial"}


def _uniforms(rng, kind, T, N):
    return rng.random(T) if kind == O.SYSTEMATIC else rng.random((T, N))


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.STRATIFIED, O.MULTINOMIAL])
@pytest.mark.parametrize("dims", [(16, 8, 16384, 16), (64, 32, 4096, 8)], ids=["dx16", "dx64"])
def test_large_pf_teacher_forced(ctx, kind, dims, record_property):
    dx, dy, N, T = dims
    m, ys = W.lgssm_rot(seed=dx + kind, dx=dx, dy=dy, T=T)
    rng = np.random.default_rng(100 + dx + kind)
    noise = rng.standard_normal((T + 1, dx, N)).astype(np.float32)
    unif = _uniforms(rng, kind, T, N)
    thr = 0.9
    cb = G.DenseAncestorCallback()
    st, ll = G.filter(m, G.BF(N, threshold=thr, resampler=RS[kind]), ys, noise=noise,
                      uniforms=unif, callback=cb, ctx=ctx)
    hist, lwh, anc = cb.container._hist, cb.container.weights, cb.container.ancestors
    om = to_oracle(m)
    n_res = n_boundary = 0
    for t in range(1, T + 1):
        x_prev = hist[t - 1].T.astype(np.float64)
        lw_prev = np.zeros(N) if t == 1 else lwh[t - 2]
        ref = O.pf_step(om, x_prev, lw_prev, ys[t - 1], noise[t].astype(np.float64), unif[t - 1],
                        uniform=t == 1, resampler=kind, threshold=thr)
        assert bool(st.resampled[t - 1]) == ref["resampled"], t
        n_res += ref["resampled"]
        bad, boundary = ancestors_match(anc[t - 1], ref["ancestors"], ref["margins"], 1e-8)
        assert bad == 0, (t, bad, boundary)
        n_boundary += boundary
        if boundary == 0:  # a boundary case moves one particle; compare the rest only then
            np.testing.assert_allclose(hist[t].T, ref["x"], rtol=2e-5, atol=2e-5)
            np.testing.assert_allclose(lwh[t - 1], ref["logw"], rtol=1e-4, atol=2e-4)
        assert abs(st.ll_steps[t - 1] - ref["ll_inc"]) < 1e-4 + 2e-6 * abs(ref["ll_inc"]), t
    assert n_res >= 3
    print(f"\nPF Dx={dx} {NAMES[kind]}: {n_res} resampling steps, "
          f"{n_boundary} ancestor boundary cases of {n_res * N} slots")
    record_property("ancestor_boundary_cases", n_boundary)


def _unpack_rb(hist_t, dxo, dz):
    """Packed RBPF state [x | mu | Sigma upper triangle by rows] ([pw, N]) ->
    x [N, dxo], mu [N, dz], Sigma [N, dz, dz]."""
    N = hist_t.shape[1]
    x = hist_t[:dxo].T.astype(np.float64)
    mu = hist_t[dxo:dxo + dz].T.astype(np.float64)
    Sig = np.zeros((N, dz, dz))
    k = dxo + dz
    for i in range(dz):
        for j in range(i, dz):
            Sig[:, i, j] = Sig[:, j, i] = hist_t[k]
            k += 1
    return x, mu, Sig


def test_rbpf_teacher_forced_ess_triggered(ctx, record_property):
    hier, ys = W.rb_trend(seed=5, T=60)
    om = to_oracle_rb(hier)
    N, T, dxo, dz = 4096, 60, om.dxo, om.dz
    rng = np.random.default_rng(6)
    noise = rng.standard_normal((T + 1, dxo, N)).astype(np.float32)
    unif = rng.random(T)
    cb = G.DenseAncestorCallback()
    algo = G.RBPF(G.BF(N, threshold=0.5), G.KalmanFilter())
    st, ll = G.filter(hier, algo, ys, noise=noise, uniforms=unif, callback=cb, ctx=ctx)
    hist, lwh, anc = cb.container._hist, cb.container.weights, cb.container.ancestors
    # the packed history's last entry is the run's final state
    xf, muf, Sf = _unpack_rb(hist[T], dxo, dz)
    np.testing.assert_array_equal(xf, np.asarray(st.particles["x"], np.float64).reshape(N, dxo))
    np.testing.assert_allclose(Sf, st.particles["Sigma"], rtol=0, atol=0)
    n_res = n_boundary = 0
    for t in range(1, T + 1):
        x, mu, Sig = _unpack_rb(hist[t - 1], dxo, dz)
        lw_prev = np.zeros(N) if t == 1 else lwh[t - 2]
        ref = O.rbpf_step(om, x, mu, Sig, lw_prev, ys[t - 1], noise[t].astype(np.float64),
                          unif[t - 1], uniform=t == 1, threshold=0.5)
        assert bool(st.resampled[t - 1]) == ref["resampled"], t
        n_res += ref["resampled"]
        bad, boundary = ancestors_match(anc[t - 1], ref["ancestors"], ref["margins"], 1e-8)
        assert bad == 0, (t, bad, boundary)
        n_boundary += boundary
        xg, mug, Sg = _unpack_rb(hist[t], dxo, dz)
        if boundary == 0:
            np.testing.assert_allclose(xg, ref["x"], rtol=2e-5, atol=2e-5)
            np.testing.assert_allclose(mug, ref["mu"], rtol=0, atol=1e-4 * (np.abs(ref["mu"]).max() + 1))
            np.testing.assert_allclose(Sg, ref["Sigma"], rtol=0,
                                       atol=1e-4 * np.abs(ref["Sigma"]).max())
        assert abs(st.ll_steps[t - 1] - ref["ll_inc"]) <= 1e-4 * max(1.0, abs(ref["ll_inc"])), t
    assert n_res >= 5, n_res
    print(f"\nRBPF (2,8,4) ESS-triggered: {n_res} resampling steps over {T}, "
          f"{n_boundary} ancestor boundary cases")
    record_property("ancestor_boundary_cases", n_boundary)


def _config3_bank():
    models, Ts, yss = W.kf_bank(256, seed=31, simulate=True)
    rng = np.random.default_rng(32)
    # the hardest corners of the distribution: longest T, largest spectral radius,
    # smallest and largest state dimensions, tight and loose noise
    for dx, dy, q, r in ((32, 32, 1e-3, 1e-2), (32, 1, 1.0, 1.0), (2, 2, 1e-3, 1e-2),
                         (17, 9, 1e-2, 1e-1)):
        A = W.random_orthogonal(rng, dx) * 0.99
        H = rng.standard_normal((dy, dx)) / np.sqrt(dx)
        m = G.create_homogeneous_linear_gaussian_model(np.zeros(dx), np.eye(dx), A, np.zeros(dx),
                                                       q * np.eye(dx), H, np.zeros(dy),
                                                       r * np.eye(dy))
        _, ys = W.simulate_lg(rng, m, 2048)
        models.append(m)
        Ts.append(2048)
        yss.append(ys)
    return models, Ts, yss


@pytest.mark.parametrize("algo", ["kf", "srkf"])
def test_kf_bank_config3_full_lengths(ctx, algo, record_property):
    models, Ts, yss = _config3_bank()
    assert max(Ts) == 2048 and len(models) >= 256
    A = G.KalmanFilter() if algo == "kf" else G.SRKF()
    res = G.filter_batch(models, A, yss, ctx=ctx)
    worst_ll = worst_mu = worst_sig = 0.0
    for (st, ll), m, ys in zip(res, models, yss):
        rll, rsteps, rmus, rsig = O.kf_filter(to_oracle(m), ys, algo=algo)
        rel = abs(ll - rll) / max(1.0, abs(rll))
        worst_ll = max(worst_ll, rel)
        assert rel <= 1e-4, (rel, ll, rll, m.dx, len(ys))
        scale_mu = np.abs(rmus).max() + 1e-3
        emu = np.abs(st.means - rmus).max() / scale_mu
        scale_s = np.abs(rsig).max()
        esig = np.abs(st.covs - rsig).max() / scale_s
        worst_mu, worst_sig = max(worst_mu, emu), max(worst_sig, esig)
        assert emu <= 1e-3 and esig <= 1e-3, (emu, esig, m.dx, len(ys))
        np.testing.assert_allclose(st.ll_steps, rsteps, atol=1e-4 * max(1.0, abs(rll)) / len(ys) + 1e-5)
    print(f"\n{algo} bank of {len(models)} (T up to 2048): worst |dll|/|ll| {worst_ll:.2e}, "
          f"mu {worst_mu:.2e}, Sigma {worst_sig:.2e} of scale")
    record_property("worst_ll_rel", worst_ll)
