"""GPU parity of the particle-filter path against the FP64 oracle.

Tolerances: FP64 runs match the oracle's per-step log-likelihood increments to
1e-9 (absolute) and ancestors bit-exactly except where a slot's threshold lies
within 1e-9 of a cumulative-weight boundary (counted, expected 0).  FP32 runs
are checked step by step from the GPU's own state (teacher forcing): ancestors
exact outside a 1e-8 band, states to 2e-5 relative, ll increments to 1e-4.
"""
import numpy as np
import pytest

import gfb200 as G
import oracle as O
from gfb200 import workloads as W
from helpers import ancestors_match, injected, random_lg, simulate, to_oracle

pytestmark = pytest.mark.gpu

RS = {O.SYSTEMATIC: G.Systematic(), O.STRATIFIED: G.Stratified(), O.MULTINOMIAL: G.Multinomial()}


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.STRATIFIED, O.MULTINOMIAL])
@pytest.mark.parametrize("conv", ["cpu", "cudaext"])
def test_bf_f64_injected_matches_oracle(ctx, kind, conv):
    """Config-1 model (1-D, N=1024, T=100, ESS < 0.5N, FP64) with injected noise."""
    m, ys = W.lgssm_1d(seed=3, T=100)
    N, T = 1024, 100
    rng = np.random.default_rng(11)
    noise, unif = injected(rng, T, 1, N, kind)
    algo = G.BF(N, threshold=0.5, resampler=RS[kind], precision="f64", convention=conv)
    st, ll = G.filter(m, algo, ys, noise=noise, uniforms=unif, want_ancestors=True, ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, resampler=kind,
                   conv=O.CONV_CUDAEXT if conv == "cudaext" else O.CONV_CPU, threshold=0.5,
                   noise=noise, uniforms=unif, want_ancestors=True, want_margins=True)
    assert st.resampled.sum() > 3, "workload must exercise resampling"
    np.testing.assert_array_equal(st.resampled, ref["resampled"])
    bad, boundary = ancestors_match(st.ancestors, ref["ancestors"], ref["margins"], 1e-9)
    assert bad == 0 and boundary == 0
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], atol=1e-9, rtol=0)
    np.testing.assert_allclose(st.ess_steps, ref["ess"], rtol=1e-9)
    assert abs(ll - ref["ll"]) < 1e-8
    np.testing.assert_allclose(st.particles[:, 0], ref["x_final"][:, 0], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(st.log_weights, ref["logw_final"], atol=1e-9)
    assert st.clamps == ref["clamps"] == 0


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.STRATIFIED])
@pytest.mark.parametrize("conv", ["cpu", "cudaext"])
def test_degenerate_weights_ancestors_match_oracle(ctx, kind, conv):
    """An observation far more precise than the prior piles the weight on a few
    particles, so one tile of 1024 particles owns more than 8192 of the slots: the
    merge-path fill still gives every block the same number of items, and the
    ancestors stay bit-exact with the FP64 oracle on the same injected noise."""
    from gfb200 import create_homogeneous_linear_gaussian_model
    dx = 2
    m = create_homogeneous_linear_gaussian_model(np.zeros(dx), 4.0 * np.eye(dx), 0.9 * np.eye(dx),
                                                 np.zeros(dx), np.eye(dx), np.eye(dx), np.zeros(dx),
                                                 1e-4 * np.eye(dx))
    rng = np.random.default_rng(19)
    T, N = 4, 32768
    _, ys = simulate(rng, m, T)
    noise, unif = injected(rng, T, dx, N, kind)
    algo = G.BF(N, threshold=0.5, resampler=RS[kind], precision="f64", convention=conv)
    st, ll = G.filter(m, algo, ys, noise=noise, uniforms=unif, want_ancestors=True, ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, resampler=kind,
                   conv=O.CONV_CUDAEXT if conv == "cudaext" else O.CONV_CPU, threshold=0.5,
                   noise=noise, uniforms=unif, want_ancestors=True, want_margins=True)
    np.testing.assert_array_equal(st.resampled, ref["resampled"])
    res = np.flatnonzero(st.resampled)
    # slots owned by the busiest tile of 1024 particles on a resampling step
    busiest = max(np.bincount((st.ancestors[t] - 1) // 1024).max() for t in res)
    assert busiest > 8192, "workload must pile the offspring on one tile"
    bad, boundary = ancestors_match(st.ancestors, ref["ancestors"], ref["margins"], 1e-9)
    assert bad == 0 and boundary == 0
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], atol=1e-7, rtol=1e-9)


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.STRATIFIED, O.MULTINOMIAL])
def test_bf_f64_in_kernel_philox_matches_oracle(ctx, kind):
    """In-kernel Philox noise and uniforms: the oracle regenerates the same stream."""
    rng = np.random.default_rng(5)
    m = random_lg(rng, 2, 2)
    _, ys = simulate(rng, m, 30)
    N = 2048
    algo = G.BF(N, threshold=0.6, resampler=RS[kind], precision="f64")
    st, ll = G.filter(m, algo, ys, seed=1234, want_ancestors=True, ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, resampler=kind, threshold=0.6, seed=1234,
                   want_ancestors=True, want_margins=True)
    assert st.resampled.sum() >= 2
    np.testing.assert_array_equal(st.resampled, ref["resampled"])
    bad, boundary = ancestors_match(st.ancestors, ref["ancestors"], ref["margins"], 1e-9)
    assert bad == 0
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], atol=1e-9, rtol=0)


@pytest.mark.parametrize("prop", ["optimal", "overdispersed"])
def test_guided_pf_f64_matches_oracle(ctx, prop):
    rng = np.random.default_rng(21)
    m = random_lg(rng, 3, 2)
    _, ys = simulate(rng, m, 25)
    N, T = 1024, 25
    noise, unif = injected(rng, T, 3, N, O.SYSTEMATIC)
    p = G.OptimalProposal(m.dyn, m.obs) if prop == "optimal" else G.OverdispersedProposal(m.dyn, 1.5)
    algo = G.PF(N, p, threshold=0.5, precision="f64")
    st, ll = G.filter(m, algo, ys, noise=noise, uniforms=unif, want_ancestors=True, ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, threshold=0.5, noise=noise, uniforms=unif,
                   proposal=O.PROP_OPTIMAL if prop == "optimal" else O.PROP_OVERDISPERSED,
                   k=1.5, want_ancestors=True, want_margins=True)
    np.testing.assert_array_equal(st.resampled, ref["resampled"])
    bad, _ = ancestors_match(st.ancestors, ref["ancestors"], ref["margins"], 1e-9)
    assert bad == 0
    np.testing.assert_allclose(st.ll_steps, ref["ll_steps"], atol=1e-8, rtol=0)


def test_bf_f32_teacher_forced_steps(ctx):
    """FP32 state, Dx=16/Dy=8 (large-PF model shape): every step of the GPU run is
    re-done by the FP64 oracle from the GPU's own previous state."""
    m, ys = W.lgssm_rot(seed=7, dx=16, dy=8, T=12)
    N, T = 4096, 12
    rng = np.random.default_rng(8)
    noise = rng.standard_normal((T + 1, 16, N)).astype(np.float32)
    unif = rng.random(T)
    om = to_oracle(m)
    runs = {}
    for t in range(1, T + 1):
        algo = G.BF(N, threshold=0.9)
        runs[t] = G.filter(m, algo, ys[:t], noise=noise[:t + 1], uniforms=unif[:t],
                           want_ancestors=True, ctx=ctx)
    n_res = 0
    for t in range(2, T + 1):
        prev, _ = runs[t - 1]
        cur, _ = runs[t]
        ref = O.pf_step(om, prev.particles.astype(np.float64), prev.log_weights, ys[t - 1],
                        noise[t].astype(np.float64), unif[t - 1], threshold=0.9)
        assert bool(cur.resampled[t - 1]) == ref["resampled"]
        n_res += ref["resampled"]
        bad, _ = ancestors_match(cur.ancestors[t - 1], ref["ancestors"], ref["margins"], 1e-8)
        assert bad == 0
        np.testing.assert_allclose(cur.particles, ref["x"], rtol=2e-5, atol=2e-5)
        assert abs(cur.ll_steps[t - 1] - ref["ll_inc"]) < 1e-4
    assert n_res >= 3


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("dx,N", [(4, 3000), (1, 3001), (1, 1000)])
def test_fused_rng_equals_exported_noise(ctx, prec, dx, N):
    """Noise drawn in-kernel == the same stream exported by gf_rng_normals and injected
    (the 1-D layout shares one Philox call between four particles; N = 1000 runs
    the whole filter in one block)."""
    m, ys = W.lgssm_rot(seed=2, dx=dx, dy=dx, T=20)
    T, seed = 20, 99
    a, lla = G.filter(m, G.BF(N, threshold=0.7, precision=prec), ys, seed=seed, ctx=ctx,
                      want_ancestors=True)
    noise = np.stack([G.rng_normals(seed, t, dx, N, prec, ctx=ctx).cpu().numpy()
                      for t in range(T + 1)])
    if dx == 1:
        np.testing.assert_allclose(noise[3], O.philox_normals(seed, N, 1, 3),
                                   rtol=0, atol=1e-5 if prec == "f32" else 1e-12)
    unif = np.array([O.philox_uniform(seed, 0, t) for t in range(1, T + 1)])
    b, llb = G.filter(m, G.BF(N, threshold=0.7, precision=prec), ys, noise=noise, uniforms=unif,
                      ctx=ctx, want_ancestors=True)
    assert lla == llb
    np.testing.assert_array_equal(a.ancestors, b.ancestors)
    np.testing.assert_array_equal(a.particles, b.particles)


def test_kept_plans_take_each_calls_seed_and_inputs(ctx):
    """gf_pf_run keeps its plan for calls with the same model and configuration:
    a later call with another seed or other observations must still see them
    (and give what a fresh context gives)."""
    m, ys = W.lgssm_rot(seed=3, dx=16, dy=8, T=30)
    algo = G.BF(50000, threshold=0.5)
    a = G.filter(m, algo, ys, seed=1, ctx=ctx)[1]
    b = G.filter(m, algo, ys, seed=2, ctx=ctx)[1]
    c = G.filter(m, algo, ys, seed=1, ctx=ctx)[1]
    d = G.filter(m, algo, ys[::-1].copy(), seed=1, ctx=ctx)[1]
    fresh = G.Context(0)
    e = G.filter(m, algo, ys[::-1].copy(), seed=1, ctx=fresh)[1]
    fresh.close()
    assert a == c and a != b and d != a and d == e


def test_runs_are_deterministic(ctx):
    m, ys = W.lgssm_rot(seed=4, dx=16, dy=8, T=40)
    algo = G.BF(200_000, threshold=0.5)
    a, lla = G.filter(m, algo, ys, seed=5, ctx=ctx)
    b, llb = G.filter(m, algo, ys, seed=5, ctx=ctx)
    assert lla == llb
    np.testing.assert_array_equal(a.ll_steps, b.ll_steps)
    np.testing.assert_array_equal(a.particles, b.particles)


def _kf_ll(m, ys):
    ll, _, mus, _ = O.kf_filter(to_oracle(m), ys)
    return ll, mus


def test_bf_converges_to_kf(ctx):
    """test/algorithms/particles.jl:5-27 shape: 1-D random model, T=4, N=10^6,
    AlternatingResampler: |ll_BF - ll_KF| <= 1e-3, filtered mean rtol 1e-3."""
    rng = np.random.default_rng(1234)
    m = random_lg(rng, 1, 1)
    _, ys = simulate(rng, m, 4)
    algo = G.BF(10**6, resampler=G.AlternatingResampler())
    st, ll = G.filter(m, algo, ys, seed=77, ctx=ctx)
    llkf, mus = _kf_ll(m, ys)
    w = st.weights()
    assert abs(ll - llkf) <= 1e-3
    assert abs(np.sum(st.particles[:, 0] * w) - mus[-1, 0]) <= 1e-3 * abs(mus[-1, 0])


def test_guided_converges_to_kf(ctx):
    """test/algorithms/particles.jl:31-53 shape with OptimalProposal."""
    rng = np.random.default_rng(1234)
    m = random_lg(rng, 1, 1)
    _, ys = simulate(rng, m, 4)
    algo = G.PF(10**6, G.OptimalProposal(m.dyn, m.obs), resampler=G.AlternatingResampler())
    st, ll = G.filter(m, algo, ys, seed=78, ctx=ctx)
    llkf, mus = _kf_ll(m, ys)
    assert abs(ll - llkf) <= 1e-3
    assert abs(np.sum(st.particles[:, 0] * st.weights()) - mus[-1, 0]) <= 1e-3 * abs(mus[-1, 0])


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.STRATIFIED, O.MULTINOMIAL])
def test_large_pf_properties(ctx, kind):
    """N = 2^20, Dx=16, Dy=8: size-independent invariants of the full-size run."""
    m, ys = W.lgssm_rot(seed=1, dx=16, dy=8, T=30)
    N = 2**20
    st, ll = G.filter(m, G.BF(N, threshold=0.5, resampler=RS[kind]), ys, seed=3,
                      want_ancestors=True, ctx=ctx)
    assert np.isfinite(ll) and abs(ll - st.ll_steps.sum()) < 1e-6 * max(1, abs(ll))
    assert st.clamps == 0
    assert st.resampled[1:].sum() >= 1
    for t in range(30):
        a = st.ancestors[t]
        assert a.min() >= 1 and a.max() <= N
        if not st.resampled[t]:
            np.testing.assert_array_equal(a, np.arange(1, N + 1))
        else:
            assert st.ess_steps[t] <= 0.5 * N + 1e-6 or t == 0
            if kind != O.MULTINOMIAL:
                assert np.all(np.diff(a) >= 0)
    np.testing.assert_allclose(st.weights().sum(), 1.0, rtol=1e-12)


def test_large_pf_converges_to_kf_ll(ctx):
    """The PF log-likelihood estimate at N = 2^20 (Dx=16, T=50) agrees with the exact
    KF value within its Monte-Carlo spread (6 independent seeds)."""
    m, ys = W.lgssm_rot(seed=9, dx=16, dy=8, T=50)
    lls = np.array([G.filter(m, G.BF(2**20, threshold=0.5), ys, seed=s, ctx=ctx)[1]
                    for s in range(6)])
    llkf, _ = _kf_ll(m, ys)
    sd = lls.std(ddof=1)
    assert sd < 5.0
    assert abs(np.median(lls) - llkf) < 2.0 + 3 * sd


@pytest.mark.parametrize("dims", [(16, 8), (32, 16), (20, 5), (64, 32), (40, 20)])
def test_tensor_core_path_matches_simt(ctx, dims):
    """The tcgen05 propagation (3xTF32) and the CUDA-core propagation agree to FP32
    accuracy on the same injected noise (no resampling, so particles stay aligned)."""
    import torch
    from gfb200.plans import PfPlan
    dx, dy = dims
    m, ys = W.lgssm_rot(seed=dx, dx=dx, dy=dy, T=4)
    N, T = 5000, 4
    rng = np.random.default_rng(3)
    noise = torch.tensor(rng.standard_normal((T + 1, dx, N)).astype(np.float32), device="cuda:0")
    ysd = torch.tensor(ys, device="cuda:0")
    algo = G.BF(N, resampler=G.AlternatingResampler())
    out = {}
    for simt in (False, True):
        plan = PfPlan(m, algo, T, ctx=ctx, graph=False, simt=simt)
        plan._cfg.schedule = None
        states = torch.zeros((dx, N), dtype=torch.float32, device="cuda:0")
        lw = torch.zeros(N, dtype=torch.float64, device="cuda:0")
        plan.run(ysd, noise_dev=noise, unif_dev=torch.zeros(T, dtype=torch.float64, device="cuda:0"),
                 states=states, log_weights=lw)
        ctx.synchronize()
        out[simt] = (states.cpu().numpy(), lw.cpu().numpy(), plan.ll_steps.cpu().numpy())
        plan.close()
    (s0, w0, l0), (s1, w1, l1) = out[False], out[True]
    np.testing.assert_allclose(s0, s1, rtol=2e-5, atol=2e-5)
    np.testing.assert_allclose(w0, w1, rtol=1e-5, atol=2e-4)
    # per-step ll is a log-sum-exp of the log-weights: its error is bounded by
    # theirs (FP32 sums of up to 32 squared residuals per particle)
    np.testing.assert_allclose(l0, l1, rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("kind,N,threshold", [(O.SYSTEMATIC, 2 ** 16, 0.5), (O.STRATIFIED, 5000, 0.7),
                                              (O.SYSTEMATIC, 5001, 0.5), (O.MULTINOMIAL, 4096, 0.5),
                                              (O.SYSTEMATIC, 3000, 0.0)])
def test_staged_gather_equals_per_thread_gather(ctx, kind, N, threshold):
    """The bulk-copy (TMA-engine) staged ancestor gather reads the same states as
    the per-thread gather: identical ll, ancestors and final states.  Covers
    resampling and non-resampling steps (threshold 0), ragged N, N % 4 != 0 and
    the multinomial search (both of which take the per-thread path)."""
    import torch
    from gfb200.plans import PfPlan
    m, ys = W.lgssm_rot(seed=5, dx=16, dy=8, T=12)
    T = 12
    ysd = torch.tensor(ys, device="cuda:0")
    algo = G.BF(N, threshold=threshold, resampler={O.SYSTEMATIC: G.Systematic(), O.STRATIFIED: G.Stratified(),
                                                  O.MULTINOMIAL: G.Multinomial()}[kind])
    out = {}
    for staged in (False, True):
        plan = PfPlan(m, algo, T, seed=9, ctx=ctx, graph=False, staged_gather=staged)
        states = torch.zeros((16, N), dtype=torch.float32, device="cuda:0")
        anc = torch.zeros((T, N), dtype=torch.int32, device="cuda:0")
        plan.run(ysd, states=states, ancestors=anc)
        ctx.synchronize()
        out[staged] = (plan.ll.item(), states.cpu().numpy(), anc.cpu().numpy(),
                       plan.resampled.cpu().numpy())
        plan.close()
    assert out[False][0] == out[True][0]
    np.testing.assert_array_equal(out[False][1], out[True][1])
    np.testing.assert_array_equal(out[False][2], out[True][2])
    np.testing.assert_array_equal(out[False][3], out[True][3])
    if threshold > 0:
        assert out[True][3].sum() >= 3


@pytest.mark.parametrize("dims,N", [((16, 8), 5000), ((16, 16), 2 ** 16 + 77), ((32, 16), 3000),
                                    ((64, 32), 2 ** 14 + 5)])
def test_unit_grid_propagation_matches_tile_blocks(ctx, dims, N):
    """The unit-grid tensor-core propagation (resident blocks striding over
    128-particle units, one log-sum-exp partial per unit) computes the same MMA
    chain as one block per tile: identical states on the same injected noise; the
    log-weights and ll differ only through the fold order of the partials."""
    import torch
    from gfb200.plans import PfPlan
    dx, dy = dims
    m, ys = W.lgssm_rot(seed=dx + dy, dx=dx, dy=dy, T=5)
    T = 5
    rng = np.random.default_rng(4)
    noise = torch.tensor(rng.standard_normal((T + 1, dx, N)).astype(np.float32), device="cuda:0")
    ysd = torch.tensor(ys, device="cuda:0")
    out = {}
    for units in (False, True):
        plan = PfPlan(m, G.BF(N, threshold=0.0), T, ctx=ctx, graph=False, units=units)
        states = torch.zeros((dx, N), dtype=torch.float32, device="cuda:0")
        lw = torch.zeros(N, dtype=torch.float64, device="cuda:0")
        plan.run(ysd, noise_dev=noise, states=states, log_weights=lw)
        ctx.synchronize()
        out[units] = (states.cpu().numpy(), lw.cpu().numpy(), plan.ll_steps.cpu().numpy())
        plan.close()
    (s0, w0, l0), (s1, w1, l1) = out[False], out[True]
    np.testing.assert_array_equal(s0, s1)
    np.testing.assert_allclose(w0, w1, rtol=0, atol=1e-5)
    np.testing.assert_allclose(l0, l1, rtol=0, atol=1e-9)


def test_unit_grid_resampling_run_matches_oracle_steps(ctx):
    """Unit-grid propagation with ESS-triggered systematic resampling, teacher-forced
    against the FP64 oracle step by step (as test_bf_f32_teacher_forced_steps)."""
    from gfb200.plans import PfPlan
    import torch
    m, ys = W.lgssm_rot(seed=7, dx=16, dy=8, T=8)
    N, T = 4096, 8
    rng = np.random.default_rng(8)
    noise = rng.standard_normal((T + 1, 16, N)).astype(np.float32)
    unif = rng.random(T)
    om = to_oracle(m)
    prev = None
    n_res = 0
    for t in range(1, T + 1):
        plan = PfPlan(m, G.BF(N, threshold=0.9), t, ctx=ctx, graph=False, units=True)
        states = torch.zeros((16, N), dtype=torch.float32, device="cuda:0")
        lw = torch.zeros(N, dtype=torch.float64, device="cuda:0")
        anc = torch.zeros((t, N), dtype=torch.int32, device="cuda:0")
        plan.run(torch.tensor(ys[:t], device="cuda:0"), noise_dev=torch.tensor(noise[:t + 1], device="cuda:0"),
                 unif_dev=torch.tensor(unif[:t], device="cuda:0"), states=states, log_weights=lw,
                 ancestors=anc)
        ctx.synchronize()
        cur = (states.cpu().numpy().T.copy(), lw.cpu().numpy(), anc.cpu().numpy(),
               plan.resampled.cpu().numpy(), plan.ll_steps.cpu().numpy())
        plan.close()
        if prev is not None:
            ref = O.pf_step(om, prev[0].astype(np.float64), prev[1], ys[t - 1],
                            noise[t].astype(np.float64), unif[t - 1], threshold=0.9)
            assert bool(cur[3][t - 1]) == ref["resampled"]
            n_res += ref["resampled"]
            bad, _ = ancestors_match(cur[2][t - 1], ref["ancestors"], ref["margins"], 1e-8)
            assert bad == 0
            np.testing.assert_allclose(cur[0], ref["x"], rtol=2e-5, atol=2e-5)
            assert abs(cur[4][t - 1] - ref["ll_inc"]) < 1e-4
        prev = cur
    assert n_res >= 3


@pytest.mark.parametrize("kind,threshold,T", [(O.SYSTEMATIC, 0.5, 6), (O.STRATIFIED, 1.0, 5),
                                              (O.MULTINOMIAL, 0.7, 5), (O.SYSTEMATIC, 0.0, 70)])
def test_path_storage_matches_dense_ancestry(ctx, kind, threshold, T):
    """AncestorCallback / ParticleTree (callbacks.jl:90-111, containers.jl:466-631):
    the device path storage returns every final particle's trajectory, equal to the
    dense reconstruction from the oracle's ancestors and per-step states (FP64,
    injected noise and uniforms).  threshold 0 never resamples, so no lineage is
    pruned and the pool must grow past its default size."""
    rng = np.random.default_rng(T + kind)
    m = random_lg(rng, 2, 2)
    _, ys = simulate(rng, m, T)
    N = 1000
    noise, unif = injected(rng, T, 2, N, kind)
    rs = {O.SYSTEMATIC: G.Systematic(), O.STRATIFIED: G.Stratified(), O.MULTINOMIAL: G.Multinomial()}[kind]
    algo = G.BF(N, threshold=threshold, resampler=rs, precision="f64")
    st, ll = G.filter(m, algo, ys, noise=noise, uniforms=unif, want_ancestors=True, want_paths=True,
                      ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, resampler=kind, threshold=threshold, noise=noise,
                   uniforms=unif, want_ancestors=True, want_states=True)
    np.testing.assert_array_equal(st.ancestors, ref["ancestors"])
    dense = O.ancestry_paths(ref["ancestors"], ref["states"])
    np.testing.assert_allclose(st.paths, dense, rtol=1e-10, atol=1e-12)
    # the plan reuses (and keeps) its grown pool on a second run
    assert st.paths.shape == (T + 1, N, 2)


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.MULTINOMIAL])
@pytest.mark.parametrize("apf", [False, True])
def test_dense_ancestry_container_matches_oracle(ctx, kind, apf):
    """DenseAncestorCallback / DenseParticleContainer (callbacks.jl:47-81,
    containers.jl:296-440): the per-step states and normalised PostUpdate
    log-weights equal the oracle's (FP64, injected noise), and get_ancestry over
    the container equals the oracle's dense reconstruction and the device path
    storage."""
    rng = np.random.default_rng(60 + kind)
    m = random_lg(rng, 3, 2)
    T, N = 7, 900
    _, ys = simulate(rng, m, T)
    noise, unif = injected(rng, T, 3, N, kind)
    bf = G.BF(N, threshold=0.8, resampler=RS[kind], precision="f64")
    algo = G.APF(bf, G.MeanPredictive()) if apf else bf
    cb = G.DenseAncestorCallback()
    st, ll = G.filter(m, algo, ys, noise=noise, uniforms=unif, callback=cb, ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, resampler=kind, threshold=0.8, noise=noise, uniforms=unif,
                   want_ancestors=True, want_states=True, lookahead=int(apf))
    c = cb.container
    np.testing.assert_array_equal(c.ancestors, ref["ancestors"])
    np.testing.assert_allclose(c.initial_states, ref["states"][0], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(c.states, ref["states"][1:], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(c.weights, ref["log_weights_all"], atol=1e-9)
    dense = O.ancestry_paths(ref["ancestors"], ref["states"])  # [T+1, N, dx]
    paths = G.get_ancestry(c, ctx=ctx)                          # [N, T+1, dx]
    np.testing.assert_allclose(paths, dense.transpose(1, 0, 2), rtol=1e-10, atol=1e-12)
    one = G.get_ancestry(c, 5, ctx=ctx)
    np.testing.assert_array_equal(one, paths[4])
    tcb = G.AncestorCallback()
    G.filter(m, algo, ys, noise=noise, uniforms=unif, callback=tcb, ctx=ctx)
    np.testing.assert_array_equal(G.get_ancestry(tcb.tree), paths)


def test_dense_ancestry_walk_with_shifting_ancestors(ctx):
    """test/algorithms/rbpf.jl:236-277 pattern: with ancestors a_i = mod1(i - 1, N)
    at every step, the trajectory of final particle N is x0 = initial_states[N - K]
    and x_t = states[t][N - K + t] (the walk through the container alone)."""
    K, N, dx = 5, 10, 2
    rng = np.random.default_rng(0)
    hist = rng.standard_normal((K + 1, dx, N))
    anc = np.tile(np.array([((a - 2) % N) + 1 for a in range(1, N + 1)], np.int32), (K, 1))
    c = G.DenseParticleContainer(hist, np.zeros((K, N)), anc, ctx)
    traj = G.get_ancestry(c, N, ctx=ctx)
    np.testing.assert_array_equal(traj[0], c.initial_states[N - K - 1])
    for t in range(1, K + 1):
        np.testing.assert_array_equal(traj[t], c.states[t - 1][N - K + t - 1])
    with pytest.raises(G.GFError):
        G.get_ancestry(c, N + 1, ctx=ctx)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("kind,conv", [(O.SYSTEMATIC, "cpu"), (O.STRATIFIED, "cpu"), (O.SYSTEMATIC, "cudaext"),
                                       (O.STRATIFIED, "cudaext")])
@pytest.mark.parametrize("N,guided", [(1024, False), (777, False), (1000, True), (5, False)])
def test_small_filter_in_one_block_equals_step_kernels(ctx, prec, kind, conv, N, guided):
    """Filters of N <= 1024 run as one block for the whole filter; the result equals
    the per-step kernels' run bit for bit (ll, per-step outputs, ancestors, weighted
    means, final states and log-weights), in-kernel Philox noise and uniforms."""
    import torch
    from gfb200.plans import PfPlan
    rng = np.random.default_rng(N + kind)
    m = random_lg(rng, 3, 2)
    T = 40
    _, ys = simulate(rng, m, T)
    yd = torch.tensor(ys, device="cuda:0")
    prop = G.OptimalProposal() if guided else G.LatentProposal()
    algo = G.PF(N, prop, threshold=0.7, resampler=RS[kind], precision=prec, convention=conv)
    dt = torch.float64 if prec == "f64" else torch.float32
    res = []
    for fuse in (True, False):
        plan = PfPlan(m, algo, T, seed=31, ctx=ctx, fuse=fuse)
        st = torch.zeros((3, N), dtype=dt, device="cuda:0")
        lw = torch.zeros(N, dtype=torch.float64, device="cuda:0")
        anc = torch.zeros((T, N), dtype=torch.int32, device="cuda:0")
        means = torch.zeros((T, 3), dtype=torch.float64, device="cuda:0")
        plan.run(yd, states=st, log_weights=lw, ancestors=anc, means=means)
        ctx.synchronize()
        res.append([x.cpu().numpy() for x in (plan.ll, plan.ll_steps, plan.ess, plan.resampled, st, lw, anc,
                                              means)])
        plan.close()
    assert res[0][3].sum() >= 1
    for a, b in zip(*res):
        np.testing.assert_array_equal(a, b)
