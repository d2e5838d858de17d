"""CPU pins of the FP64 oracle: analytic truths, the reference's known answers,
the committed golden fixtures and Monte-Carlo convergence (no GPU needed)."""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


@pytest.mark.parametrize("Dy", [2, 3, 4])
@pytest.mark.parametrize("T", [1, 5])
def test_kf_matches_joint_gaussian(Dy, T):
    """test/algorithms/kalman.jl:5-43 (the reference's analytic oracle)."""
    rng = np.random.default_rng(1234 + Dy + 10 * T)
    m = O.create_linear_gaussian_model(rng, 3, Dy)
    _, ys = O.sample(rng, m, T)
    ll, _, mus, S = O.kf_filter(m, ys)
    mu, St, lt = O.joint_filter_truth(m, ys)
    assert abs(ll - lt) <= 1e-10 * abs(lt)
    np.testing.assert_allclose(mus[-1], mu, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(S[-1], St, rtol=1e-8, atol=1e-12)


@pytest.mark.parametrize("Dy", [1, 2, 3])
@pytest.mark.parametrize("T", [1, 4])
def test_nonhomogeneous_kf_and_smoother_match_joint_gaussian(Dy, T):
    """Time-varying parameters (calc_params(dyn, t), models/linear_gaussian.jl:44-63):
    the filter and the RTS smoother of a non-homogeneous model equal Gaussian
    conditioning of _compute_joint_nonhomogeneous (GFTest/models/linear_gaussian.jl:
    121-169), as test/algorithms/kalman.jl:263-300 checks for the smoother."""
    rng = np.random.default_rng(77 + Dy + 10 * T)
    m = O.create_nonhomogeneous_linear_gaussian_model(rng, 2, Dy, T)
    _, ys = O.sample(rng, m, T)
    ll, _, mus, S = O.kf_filter(m, ys)
    mu, St, lt = O.joint_filter_truth(m, ys)
    assert abs(ll - lt) <= 1e-10 * max(1.0, abs(lt))
    np.testing.assert_allclose(mus[-1], mu, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(S[-1], St, rtol=1e-8, atol=1e-12)
    _, ms, Ss = O.rts_smooth(m, ys)
    mj, Sj = O.joint_smooth_truth(m, ys)
    np.testing.assert_allclose(ms, mj, rtol=1e-8, atol=1e-11)
    np.testing.assert_allclose(Ss, Sj, rtol=1e-8, atol=1e-11)
    # a homogeneous model written as per-step copies is the homogeneous model
    h = O.create_linear_gaussian_model(rng, 2, Dy)
    hv = O.LGModel.time_varying(h.mu0, h.Sigma0, *[[x] * T for x in (h.A, h.b, h.Q, h.H, h.c, h.R)])
    np.testing.assert_array_equal(O.kf_filter(h, ys)[2], O.kf_filter(hv, ys)[2])


def test_nonhomogeneous_pf_oracle_converges_to_kf():
    """The oracle's bootstrap PF on a time-varying model uses step t's
    parameters: its ll converges to the exact time-varying KF (N = 2e5)."""
    rng = np.random.default_rng(5)
    m = O.create_nonhomogeneous_linear_gaussian_model(rng, 2, 2, 5)
    m = O.LGModel.time_varying(m.mu0, m.Sigma0, [O.random_orthogonal(rng, 2) * 0.8 for _ in range(5)],
                               m.bs, m.Qs, m.Hs, m.cs, m.Rs)
    _, ys = O.sample(rng, m, 5)
    lls = [O.pf_run(m, 200000, ys, threshold=0.5, seed=s, threads=4)["ll"] for s in range(2)]
    assert abs(np.mean(lls) - O.kf_filter(m, ys)[0]) < 2e-2


@pytest.mark.parametrize("proposal,k", [(O.PROP_OPTIMAL, 1.0), (O.PROP_OVERDISPERSED, 1.7)])
def test_nonhomogeneous_guided_pf_oracle_converges_to_kf(proposal, k):
    """Guided proposals on a time-varying model take step t's factors (the
    optimal proposal's gain and covariance from Q_t, H_t, R_t; k Q_t for the
    overdispersed one): the log-evidence converges to the exact time-varying KF."""
    rng = np.random.default_rng(6)
    m = O.create_nonhomogeneous_linear_gaussian_model(rng, 2, 2, 5)
    m = O.LGModel.time_varying(m.mu0, m.Sigma0, [O.random_orthogonal(rng, 2) * 0.8 for _ in range(5)],
                               m.bs, m.Qs, m.Hs, m.cs, m.Rs)
    _, ys = O.sample(rng, m, 5)
    lls = [O.pf_run(m, 200000, ys, threshold=0.5, seed=s, threads=4, proposal=proposal, k=k)["ll"]
           for s in range(2)]
    assert abs(np.mean(lls) - O.kf_filter(m, ys)[0]) < 2e-2


@pytest.mark.parametrize("Dy", [1, 2, 3])
@pytest.mark.parametrize("T", [1, 5])
def test_rts_smoother_matches_joint_gaussian(Dy, T):
    """smooth(model, KalmanSmoother(), ys) (kalman.jl:89-126,206-234): every
    smoothed marginal p(x_t | y_1:T) equals Gaussian conditioning of the joint."""
    rng = np.random.default_rng(77 + Dy + 10 * T)
    m = O.create_linear_gaussian_model(rng, 3, Dy)
    _, ys = O.sample(rng, m, T)
    ll, mus, S = O.rts_smooth(m, ys)
    mt, St = O.joint_smooth_truth(m, ys)
    assert ll == O.kf_filter(m, ys)[0]
    np.testing.assert_allclose(mus, mt, rtol=1e-9, atol=1e-11)
    np.testing.assert_allclose(S, St, rtol=1e-8, atol=1e-11)


@pytest.mark.parametrize("refresh", [O.CSMC_NONE, O.CSMC_ANCESTOR, O.CSMC_BACKWARD])
def test_csmc_oracle_targets_the_smoothing_distribution(refresh):
    """test/algorithms/csmc.jl:5-98 on the oracle restatement (smaller run):
    the sampled trajectories' mean at t_smooth = 2 matches the RTS smoother and
    1/Z-hat is unbiased for 1/Z (multinomial resampling)."""
    rng = np.random.default_rng(1234)
    m = O.create_linear_gaussian_model(rng, 1, 1)
    _, ys = O.sample(rng, m, 10)
    _, mus, _ = O.rts_smooth(m, ys)
    kf_ll = O.kf_filter(m, ys)[0]
    tr, lls, _ = O.csmc_run(m, 10, ys, threshold=0.6, resampler=O.MULTINOMIAL, refresh=refresh,
                            chains=64, iters=1600, burnin=100, seed=31 + refresh, threads=4)
    np.testing.assert_allclose(tr[:, :, 2, 0].mean(), mus[1, 0], rtol=6e-3)
    l = -lls.ravel()
    np.testing.assert_allclose(l.max() + np.log(np.mean(np.exp(l - l.max()))), -kf_ll, rtol=1e-3)


@pytest.mark.parametrize("refresh", [O.CSMC_ANCESTOR, O.CSMC_BACKWARD])
def test_nonhomogeneous_csmc_oracle_targets_the_smoothing_distribution(refresh):
    """CSMC on a time-varying model: each step's transition (also in the ancestor
    and backward-simulation weights) and observation model are that step's, so the
    sampled trajectories' mean matches the time-varying RTS smoother."""
    rng = np.random.default_rng(77)
    T = 8
    m = O.create_nonhomogeneous_linear_gaussian_model(rng, 1, 1, T)
    m = O.LGModel.time_varying(m.mu0, m.Sigma0, [np.array([[rng.uniform(0.5, 0.95)]]) for _ in range(T)],
                               m.bs, m.Qs, m.Hs, m.cs, m.Rs)
    _, ys = O.sample(rng, m, T)
    _, mus, _ = O.rts_smooth(m, ys)
    tr, _, _ = O.csmc_run(m, 10, ys, threshold=0.6, resampler=O.MULTINOMIAL, refresh=refresh,
                          chains=64, iters=1600, burnin=100, seed=5 + refresh, threads=4)
    for t in (1, 4, 7):
        np.testing.assert_allclose(tr[:, :, t + 1, 0].mean(), mus[t, 0], rtol=1e-2, atol=5e-3)


def test_csmc_oracle_pins_reference_particle():
    """With NoRefreshment and threshold 0 (no resampling) every particle keeps
    its own lineage, so the sampled trajectory is one particle's path and, when
    the final draw lands on particle 1, the reference itself."""
    rng = np.random.default_rng(3)
    m = O.create_linear_gaussian_model(rng, 2, 1)
    T, N = 5, 6
    _, ys = O.sample(rng, m, T)
    ref = rng.standard_normal((1, T + 1, 2))
    unif = rng.random((1, 1, T + 1, N + 1))
    unif[0, 0, 0, N] = 0.0  # final draw: the first particle with nonzero weight, particle 1
    noise = rng.standard_normal((1, 1, T + 1, N, 2))
    tr, _, last = O.csmc_run(m, N, ys, threshold=0.0, refresh=O.CSMC_NONE, ref=ref,
                             noise=noise, uniforms=unif)
    np.testing.assert_array_equal(tr[0, 0], ref[0])
    np.testing.assert_array_equal(last[0], ref[0])


@pytest.mark.parametrize("Dy", [2, 3, 4])
def test_srkf_equals_kf(Dy):
    """test/algorithms/srkf.jl:3-26."""
    rng = np.random.default_rng(99 + Dy)
    m = O.create_linear_gaussian_model(rng, 3, Dy)
    _, ys = O.sample(rng, m, 5)
    a = O.kf_filter(m, ys)
    b = O.kf_filter(m, ys, algo="srkf")
    assert abs(a[0] - b[0]) <= 1e-10 * abs(a[0])
    np.testing.assert_allclose(a[2], b[2], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(a[3], b[3], rtol=1e-9, atol=1e-12)


def test_known_answer_offspring_ancestors():
    g = GOLD["offspring_to_ancestors"]
    assert O.offspring_to_ancestors(g["offspring"]).tolist() == g["ancestors"]
    g = GOLD["ancestors_to_offspring"]
    assert O.ancestors_to_offspring(g["ancestors"]).tolist() == g["offspring"]


def test_golden_kalman():
    for case in GOLD["kalman"]:
        m = O.LGModel(*[np.array(case["model"][k]) for k in
                        ("mu0", "Sigma0", "A", "b", "Q", "H", "c", "R")])
        ys = np.array(case["ys"])
        ll, lls, mus, S = O.kf_filter(m, ys)
        assert ll == pytest.approx(case["ll"], rel=1e-13)
        np.testing.assert_allclose(lls, case["ll_steps"], rtol=1e-12)
        np.testing.assert_allclose(S[-1], case["Sigma_T"], rtol=1e-12)
        ll2 = O.kf_filter(m, ys, algo="srkf")[0]
        assert ll2 == pytest.approx(case["ll_srkf"], rel=1e-13)


def test_golden_bootstrap_pf():
    m = O.LGModel([0.0], [[1.0]], [[1.0]], [0.0], [[0.01]], [[1.0]], [0.0], [[0.04]])
    for case in GOLD["bootstrap_pf"]:
        N = case["N"]
        ys = np.array(case["ys"]).reshape(-1, 1)
        T = ys.shape[0]
        noise = np.array(case["noise"]).reshape(T + 1, 1, N)
        unif = np.array(case["uniforms"])
        if case["kind"] != O.SYSTEMATIC:
            unif = unif.reshape(T, N)
        r = O.pf_run(m, N, ys, resampler=case["kind"], threshold=0.5, noise=noise, uniforms=unif,
                     want_ancestors=True)
        assert r["ll"] == pytest.approx(case["ll"], rel=1e-12)
        np.testing.assert_array_equal(r["ancestors"], np.array(case["ancestors"]))
        np.testing.assert_array_equal(r["resampled"], case["resampled"])


def test_systematic_rule_small_case():
    """resamplers.jl:216-238 by hand: vs = n*cumsum(w), a_i = min{k : vs_k > u0 + i - 1}."""
    w = np.array([0.1, 0.4, 0.0, 0.3, 0.2])
    a, mar, cl = O.sample_ancestors(O.SYSTEMATIC, w, [0.5])
    # vs = [0.5, 2.5, 2.5, 4.0, 5.0]; thresholds 0.5,1.5,2.5,3.5,4.5
    assert a.tolist() == [2, 2, 4, 4, 5]
    assert cl == 0


def test_cudaext_systematic_rule_small_case():
    """CUDAExt.jl:49-58 + offspring_to_ancestors: O_k = min(n, floor(n W_k/W_n + u0))."""
    w = np.array([0.1, 0.4, 0.0, 0.3, 0.2])
    a, _, _ = O.sample_ancestors(O.SYSTEMATIC, w, [0.5], conv=O.CONV_CUDAEXT)
    # r = [0.5, 2.5, 2.5, 4, 5] -> O = [1, 3, 3, 4, 5]
    assert a.tolist() == [1, 2, 2, 4, 5]


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.STRATIFIED, O.MULTINOMIAL])
def test_resampled_mean(kind):
    """test/components/resamplers.jl:5-34: N = 10^6 importance weights, rtol 0.1."""
    rng = np.random.default_rng(1234)
    n = 10**6
    xs = rng.standard_normal(n)
    ws = np.exp(-0.5 * (xs - 1) ** 2 + 0.5 * xs ** 2)
    ws /= ws.sum()
    u = rng.random(1 if kind == O.SYSTEMATIC else n)
    a, _, cl = O.sample_ancestors(kind, ws, u)
    mu0 = np.sum(ws * xs)
    assert abs(xs[a - 1].mean() - mu0) <= 0.1 * abs(mu0)


def test_pf_converges_to_kf():
    """test/algorithms/particles.jl:5-27 shape (N = 10^6, T = 4, resample at step 1)."""
    rng = np.random.default_rng(1234)
    m = O.create_linear_gaussian_model(rng, 1, 1)
    _, ys = O.sample(rng, m, 4)
    ll, _, mus, _ = O.kf_filter(m, ys)
    r = O.pf_run(m, 10**6, ys, schedule=[1, 0, 0, 0], seed=3, threads=os.cpu_count())
    assert abs(r["ll"] - ll) <= 1e-3
    w = np.exp(r["logw_final"])
    assert abs(np.sum(w * r["x_final"][:, 0]) - mus[-1, 0]) <= 1e-3 * abs(mus[-1, 0])


def test_philox_known_answer():
    """Philox4x32-10 against the published Random123 known-answer vectors; the CUDA
    kernels use the same round function (checked on the GPU by the fused-RNG tests)."""
    import ctypes as C
    lib = O.lib()

    def ph(ctr, k):
        c = (C.c_uint32 * 4)(*ctr)
        o = (C.c_uint32 * 4)()
        lib.or_philox4x32_10(c, C.c_uint32(k[0]), C.c_uint32(k[1]), o)
        return [int(v) for v in o]

    assert ph([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert ph([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert ph([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]
    vals = np.array([O.philox_uniform(12345, j, 3) for j in range(20000)])
    assert abs(vals.mean() - 0.5) < 0.01 and abs(vals.var() - 1 / 12) < 0.005
    z = O.philox_normals(7, 4000, 4, 1)
    assert abs(z.mean()) < 0.03 and abs(z.var() - 1) < 0.05


def test_apf_oracle_without_resampling_is_the_bootstrap_filter():
    """preserve_sample keeps the weights, so the auxiliary scores only act through
    a resample: with threshold 0 the APF run equals the BF run exactly."""
    rng = np.random.default_rng(12)
    m = O.create_linear_gaussian_model(rng, 2, 2)
    _, ys = O.sample(rng, m, 5)
    a = O.pf_run(m, 500, ys, threshold=0.0, seed=4, lookahead=1)
    b = O.pf_run(m, 500, ys, threshold=0.0, seed=4, lookahead=0)
    assert a["ll"] == b["ll"]


def test_apf_oracle_converges_to_kf():
    """test/algorithms/particles.jl:57-82 with every step resampling (threshold 1.0):
    the APF log-evidence estimate is unbiased for the Kalman filter's."""
    rng = np.random.default_rng(1234)
    m = O.create_linear_gaussian_model(rng, 1, 1)
    _, ys = O.sample(rng, m, 4)
    kll = O.kf_filter(m, ys)[0]
    r = O.pf_run(m, 200_000, ys, threshold=1.0, seed=2, lookahead=1, threads=4)
    assert r["resampled"].all()
    assert abs(r["ll"] - kll) < 3e-3


@pytest.mark.parametrize("seed,D,T", [(1234, 2, 3), (7, 3, 6)])
def test_kf_gradient_oracle_matches_finite_differences(seed, D, T):
    """test/components/kalman_gradient.jl: the pullback of kf_loglikelihood equals
    central differences of the Kalman log-likelihood (5-point stencil; Q, R and
    Sigma0 perturbed symmetrically, as make_nll_func's make_pd does)."""
    rng = np.random.default_rng(seed)
    m = O.create_linear_gaussian_model(rng, D, D)
    _, ys = O.sample(rng, m, T)
    ll, g = O.kf_loglikelihood_grad(m, ys)
    assert abs(ll - O.kf_filter(m, ys)[0]) <= 1e-12 * abs(ll)

    def kfll(p):
        A, b, Q, H, c, R, mu, S = (np.asarray(p[k], float) for k in ("A", "b", "Q", "H", "c", "R", "mu0", "Sigma0"))
        tot = 0.0
        for y in ys:
            mp, Sp = A @ mu + b, A @ S @ A.T + Q
            z, Sy = y - H @ mp - c, H @ Sp @ H.T + R
            K = Sp @ H.T @ np.linalg.inv(Sy)
            IKH = np.eye(len(mu)) - K @ H
            S, mu = IKH @ Sp @ IKH.T + K @ R @ K.T, mp + K @ z
            tot += -0.5 * (len(y) * np.log(2 * np.pi) + np.linalg.slogdet(Sy)[1] + z @ np.linalg.solve(Sy, z))
        return tot

    P = {n: np.array(getattr(m, n), float) for n in ("mu0", "Sigma0", "A", "b", "Q", "H", "c", "R")}
    h = 1e-5
    for name, base in P.items():
        fd = np.zeros(base.size)
        for k in range(base.size):
            vals = []
            for s in (-2, -1, 1, 2):
                q = dict(P)
                p = base.copy().ravel()
                p[k] += s * h
                p = p.reshape(base.shape)
                if name in ("Sigma0", "Q", "R"):
                    p = (p + p.T) / 2
                q[name] = p
                vals.append(kfll(q))
            fd[k] = (vals[0] - 8 * vals[1] + 8 * vals[2] - vals[3]) / (12 * h)
        fd = fd.reshape(base.shape)
        np.testing.assert_allclose(g[name], fd, rtol=0, atol=1e-6 * (np.abs(fd).max() + 1e-12), err_msg=name)


@pytest.mark.parametrize("Dy", [2, 3, 4])
def test_backward_information_matches_joint_gaussian(Dy):
    """test/algorithms/kalman.jl:83-137: after backward_initialise at T and two
    backward predict/update steps, the natural parameters of p(y_{T-2:T} | x_{T-2})
    equal F' S^-1 (y - g) and F' S^-1 F of the joint of (y_{T-2}, y_{T-1}, y_T)
    given x_{T-2} (F = [H; HA; HA^2])."""
    rng = np.random.default_rng(1234 + Dy)
    m = O.create_linear_gaussian_model(rng, 3, Dy)
    T = 4
    _, ys = O.sample(rng, m, T)
    _, _, lu, Ou = O.backward_information(m, ys, initial_jitter=1e-8)
    A, b, Q, H, c, R = (np.asarray(v) for v in (m.A, m.b, m.Q, m.H, m.c, m.R))
    Z = np.zeros((Dy, Dy))
    F = np.vstack([H, H @ A, H @ A @ A])
    g = np.concatenate([c, H @ b + c, H @ (A @ b + b) + c])
    S = np.block([[R, Z, Z],
                  [Z, H @ Q @ H.T + R, H @ Q @ A.T @ H.T],
                  [Z, H @ A @ Q @ H.T, H @ (A @ Q @ A.T + Q) @ H.T + R]])
    y = np.concatenate([ys[T - 3], ys[T - 2], ys[T - 1]])
    lam_t = F.T @ np.linalg.solve(S, y - g)
    Om_t = F.T @ np.linalg.solve(S, F)
    np.testing.assert_allclose(lu[T - 3], lam_t, rtol=1e-7)
    np.testing.assert_allclose(Ou[T - 3], Om_t, atol=1e-6)


@pytest.mark.parametrize("Dy", [1, 2, 3])
def test_nonhomogeneous_backward_information_matches_joint_gaussian(Dy):
    """test/algorithms/kalman.jl:139-190 (T = 4, a non-homogeneous model): after
    backward_initialise at T and two backward predict/update steps with each step's
    own parameters (backward_predict at iter uses calc_params(dyn, iter + 1)), the
    natural parameters of p(y_{T-2:T} | x_{T-2}) equal F' S^-1 (y - g) and
    F' S^-1 F of the joint of (y_{T-2}, y_{T-1}, y_T) given x_{T-2}."""
    rng = np.random.default_rng(1234 + Dy)
    T = 4
    m = O.create_nonhomogeneous_linear_gaussian_model(rng, 2, Dy, T)
    _, ys = O.sample(rng, m, T)
    _, _, lu, Ou = O.backward_information(m, ys, initial_jitter=1e-8)
    _, _, _, H2, c2, R2 = m.params(T - 2)
    A3, b3, Q3, H3, c3, R3 = m.params(T - 1)
    A4, b4, Q4, H4, c4, R4 = m.params(T)
    Z = np.zeros((Dy, Dy))
    F = np.vstack([H2, H3 @ A3, H4 @ A4 @ A3])
    g = np.concatenate([c2, H3 @ b3 + c3, H4 @ (A4 @ b3 + b4) + c4])
    S = np.block([[R2, Z, Z],
                  [Z, H3 @ Q3 @ H3.T + R3, H3 @ Q3 @ A4.T @ H4.T],
                  [Z, H4 @ A4 @ Q3 @ H3.T, H4 @ (A4 @ Q3 @ A4.T + Q4) @ H4.T + R4]])
    y = np.concatenate([ys[T - 3], ys[T - 2], ys[T - 1]])
    lam_t = F.T @ np.linalg.solve(S, y - g)
    Om_t = F.T @ np.linalg.solve(S, F)
    np.testing.assert_allclose(lu[T - 3], lam_t, rtol=1e-7)
    np.testing.assert_allclose(Ou[T - 3], Om_t, atol=1e-6)
    # and the two-filter smoother of the time-varying model is the RTS smoother's
    mus, Ss = O.two_filter_smooth(m, ys, initial_jitter=1e-10)
    _, mr, Sr = O.rts_smooth(m, ys)
    np.testing.assert_allclose(mus, mr, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(Ss, Sr, rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("Dy", [1, 2, 3])
def test_two_filter_smoother_equals_rts(Dy):
    """test/algorithms/kalman.jl:363-412: the two-filter smoother (forward filter x
    backward predictive likelihood) equals the RTS smoother at every time."""
    rng = np.random.default_rng(50 + Dy)
    m = O.create_linear_gaussian_model(rng, 3, Dy)
    _, ys = O.sample(rng, m, 6)
    mus, Ss = O.two_filter_smooth(m, ys, initial_jitter=1e-10)
    _, mr, Sr = O.rts_smooth(m, ys)
    np.testing.assert_allclose(mus, mr, rtol=1e-7, atol=1e-9)
    np.testing.assert_allclose(Ss, Sr, rtol=1e-7, atol=1e-9)


@pytest.mark.parametrize("kind", [O.SYSTEMATIC, O.MULTINOMIAL])
def test_rbpf_step_chain_equals_rbpf_run(kind):
    """The teacher-forcing step (or_rbpf_step) chained from the prior draw
    reproduces the full oracle RBPF run (or_rbpf_run) with ESS-triggered
    resampling: same decisions, ancestors, ll increments and final state."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "ssmproblems.jl_b200"))
    from gfb200 import workloads as W
    from helpers import to_oracle_rb
    hier, ys = W.rb_trend(seed=4, T=25, dz=4, dy=2)
    om = to_oracle_rb(hier)
    N, T = 400, 25
    rng = np.random.default_rng(3)
    noise = rng.standard_normal((T + 1, om.dxo, N))
    unif = rng.random(T) if kind == O.SYSTEMATIC else rng.random((T, N))
    ref = O.rbpf_run(om, N, ys, resampler=kind, threshold=0.9, noise=noise, uniforms=unif,
                     want_ancestors=True)
    x = (om.mu_o[:, None] + np.linalg.cholesky(om.Sigma_o) @ noise[0]).T
    mu = np.tile(om.mu_z, (N, 1))
    Sig = np.tile(om.Sigma_z, (N, 1, 1))
    logw = np.zeros(N)
    for t in range(1, T + 1):
        r = O.rbpf_step(om, x, mu, Sig, logw, ys[t - 1], noise[t], unif[t - 1], uniform=t == 1,
                        resampler=kind, threshold=0.9)
        assert r["resampled"] == bool(ref["resampled"][t - 1])
        np.testing.assert_array_equal(r["ancestors"], ref["ancestors"][t - 1])
        assert abs(r["ll_inc"] - ref["ll_steps"][t - 1]) < 1e-10
        x, mu, Sig, logw = r["x"], r["mu"], r["Sigma"], r["logw"]
    assert ref["resampled"].sum() >= 3
    dz = om.dz
    xf = ref["x_final"]
    np.testing.assert_allclose(x, xf[:, :om.dxo], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(mu, xf[:, om.dxo:om.dxo + dz], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(logw, ref["logw_final"], atol=1e-10)


def _rb_helpers():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "ssmproblems.jl_b200"))
    from helpers import dummy_rb_model, to_oracle, to_oracle_rb
    return dummy_rb_model, to_oracle, to_oracle_rb


@pytest.mark.parametrize("lookahead", [1, 2])
def test_rbpf_apf_oracle_without_resampling_is_the_rbpf(lookahead):
    """AuxiliaryParticleFilter(RBPF(...), pp): the first-stage scores only act through
    a resample, so with threshold 0 the run equals the plain RBPF's exactly."""
    dummy_rb_model, _, to_oracle_rb = _rb_helpers()
    rng = np.random.default_rng(13)
    full, hier = dummy_rb_model(rng, 1, 2, 1)
    ys = rng.standard_normal((5, 1))
    om = to_oracle_rb(hier)
    a = O.rbpf_run(om, 500, ys, threshold=0.0, seed=4, lookahead=lookahead)
    b = O.rbpf_run(om, 500, ys, threshold=0.0, seed=4, lookahead=0)
    assert a["ll"] == b["ll"]
    assert not a["resampled"].any()


@pytest.mark.parametrize("lookahead", [1, 2])
def test_rbpf_apf_oracle_converges_to_kf(lookahead):
    """test/algorithms/rbpf.jl:5-34 with the auxiliary first stage and a resample at
    every step: the log-evidence estimate is unbiased for the joint Kalman filter's
    (the dummy hierarchical model is jointly linear-Gaussian)."""
    dummy_rb_model, to_oracle, to_oracle_rb = _rb_helpers()
    rng = np.random.default_rng(1234)
    full, hier = dummy_rb_model(rng, 1, 1, 1)
    from helpers import simulate
    _, ys = simulate(rng, full, 4)
    kll = O.kf_filter(to_oracle(full), ys)[0]
    r = O.rbpf_run(to_oracle_rb(hier), 100_000, ys, threshold=1.0, seed=2, lookahead=lookahead,
                   threads=4)
    assert r["resampled"].all()
    assert abs(r["ll"] - kll) < 2e-3


@pytest.mark.parametrize("lookahead", [0, 1])
def test_nonhomogeneous_rbpf_oracle_converges_to_kf(lookahead):
    """An RBPF on a time-varying hierarchical model (every outer, inner and
    observation parameter of step t its own, calc_params(., t)) uses step t's
    parameters: its log-evidence converges to the exact Kalman filter of the
    time-varying joint model, plain and auxiliary."""
    _, _, _ = _rb_helpers()
    from helpers import tv_rb_oracle_pair
    rng = np.random.default_rng(321)
    T = 5
    joint, rb = tv_rb_oracle_pair(rng, T, 1, 2, 1)
    _, ys = O.sample(rng, joint, T)
    kll = O.kf_filter(joint, ys)[0]
    runs = [O.rbpf_run(rb, 100_000, ys, threshold=1.0, seed=s, lookahead=lookahead, threads=4)
            for s in (3, 4)]
    assert all(r["resampled"][1:].all() for r in runs)
    # Monte-Carlo SD of one run's ll here is about 3e-3
    assert abs(np.mean([r["ll"] for r in runs]) - kll) < 6e-3
    # a homogeneous model written as per-step copies runs as the homogeneous one
    h = O.RBModel.time_varying(rb.mu_o, rb.Sigma_o, rb.mu_z, rb.Sigma_z,
                               [{n: getattr(rb.steps[0], n) for n in O.RBModel.STEP_NAMES}] * T)
    a = O.rbpf_run(h, 500, ys, threshold=0.5, seed=4)
    b = O.rbpf_run(rb.steps[0], 500, ys, threshold=0.5, seed=4)
    assert a["ll"] == b["ll"]

