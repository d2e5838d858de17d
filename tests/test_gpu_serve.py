"""GPU tests of the serving loop (gf_srv_*): a request served in a mix of
concurrent Kalman, particle-filter and RBPF requests returns bit for bit what
the standalone entry point returns for the same inputs; admission respects the
HBM budget; a full queue answers GF_ERR_BUSY; a failing filter fails alone."""
import time

import numpy as np
import pytest

import gfb200 as G
from gfb200 import _lib as L
from gfb200 import workloads as W

pytestmark = pytest.mark.gpu


def _kf_model(rng, dx, dy):
    A = W.random_orthogonal(rng, dx) * rng.uniform(0.8, 0.99)
    H = rng.standard_normal((dy, dx)) / np.sqrt(dx)
    return G.create_homogeneous_linear_gaussian_model(
        np.zeros(dx), np.eye(dx), A, np.zeros(dx), 0.1 * np.eye(dx), H, np.zeros(dy),
        0.2 * np.eye(dy))


def _mix(seed=7):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(14):
        dx = int(rng.integers(2, 33))
        dy = int(rng.integers(1, dx + 1))
        m = _kf_model(rng, dx, dy)
        T = int(rng.integers(20, 300))
        ys = rng.standard_normal((T, dy))
        algo = G.SRKF() if i % 4 == 3 else G.KF()
        reqs.append(("kf", m, algo, ys, 0))
    m1, _ = W.lgssm_1d(seed=1, T=10)
    rss = [G.Systematic(), G.Stratified(), G.Multinomial()]
    for i, N in enumerate([3000, 4096, 20000, 1 << 17, 777, 50000]):
        _, ys = W.lgssm_1d(seed=10 + i, T=int(rng.integers(30, 200)))
        algo = G.BF(N, threshold=0.5, resampler=rss[i % 3])
        reqs.append(("pf", m1, algo, ys, 100 + i))
    m16, ys16 = W.lgssm_rot(seed=3, dx=16, dy=8, T=60)
    reqs.append(("pf", m16, G.BF(20000, threshold=0.5), ys16, 200))        # tensor-core path
    reqs.append(("pf", m16, G.BF(5000, threshold=0.5, precision="f64"), ys16, 201))
    for i, N in enumerate([4096, 10000]):
        hm, ys = W.rb_trend(seed=20 + i, T=80)
        algo = G.RBPF(G.BF(N, threshold=0.5), G.KalmanFilter())
        reqs.append(("rbpf", hm, algo, ys, 300 + i))
    return reqs


def _standalone(ctx, kind, model, algo, ys, seed):
    if kind == "kf":
        st, ll = G.filter(model, algo, ys, ctx=ctx)
        return ll, None, np.asarray(st.mu), np.asarray(st.Sigma)
    st, ll = G.filter(model, algo, ys, seed=seed, want_means=True, ctx=ctx)
    mean = st.means[-1]
    if kind == "rbpf":
        mean = np.concatenate([st.means[-1], st.zmeans[-1]])
    return ll, st.ll_steps, mean, None


def test_served_mix_matches_standalone(ctx):
    reqs = _mix()
    with G.Server(hbm_budget_bytes=2 << 30, host_budget_bytes=256 << 20, pf_chunk=8) as srv:
        ids = {}
        order = np.random.default_rng(0).permutation(len(reqs))
        for j, k in enumerate(order):
            kind, m, algo, ys, seed = reqs[k]
            rid = srv.submit(m, algo, ys, seed=seed, tag=int(k), want_steps=True, want_mean=True,
                             want_cov=(kind == "kf"))
            ids[rid] = k
            if j % 5 == 4:
                time.sleep(0.002)  # later requests join batches already running
        srv.drain(timeout_ms=120000)
        got = {r["tag"]: r for r in srv.poll(max_results=4096)}
        stats = srv.stats()
    assert len(got) == len(reqs)
    assert stats["completed"] == len(reqs) and stats["failed"] == 0
    for k, (kind, m, algo, ys, seed) in enumerate(reqs):
        r = got[k]
        assert r["status"] == 0, (k, kind, r)
        ll, steps, mean, cov = _standalone(ctx, kind, m, algo, ys, seed)
        assert r["ll"] == ll, (k, kind, r["ll"], ll)
        if steps is not None:
            np.testing.assert_array_equal(r["ll_steps"], steps)
        else:
            assert np.isclose(r["ll_steps"].sum(), ll, rtol=1e-12, atol=1e-9)
        np.testing.assert_array_equal(r["mean"], mean)
        if cov is not None:
            np.testing.assert_array_equal(r["cov"], cov)


def test_admission_respects_hbm_budget(ctx):
    m1, _ = W.lgssm_1d(seed=1, T=10)
    budget = 48 << 20
    # each FP64 job (N = 2^18) holds about 10 MB: at most four fit at once
    with G.Server(hbm_budget_bytes=budget, host_budget_bytes=64 << 20) as srv:
        for i in range(10):
            _, ys = W.lgssm_1d(seed=i, T=300)
            srv.submit(m1, G.BF(1 << 18, threshold=0.5, precision="f64"), ys, seed=i, tag=i)
        # larger than the whole arena: rejected, not queued forever
        _, ys = W.lgssm_1d(seed=99, T=10)
        srv.submit(m1, G.BF(1 << 21, precision="f64"), ys, tag=99)
        srv.drain(timeout_ms=120000)
        res = {r["tag"]: r for r in srv.poll(max_results=64)}
        st = srv.stats()
    assert res[99]["status"] == L.GF_ERR_OOM_BUDGET and res[99]["start_ms"] < 0
    assert all(res[i]["status"] == 0 for i in range(10))
    assert st["rejected"] == 1 and st["completed"] == 10
    assert 0 < st["hbm_peak"] <= budget
    # queued requests started only after earlier ones released their memory
    starts = sorted(res[i]["start_ms"] for i in range(10))
    firsts = sorted(res[i]["done_ms"] for i in range(10))
    assert starts[-1] >= firsts[0]


def test_queue_full_returns_busy(ctx):
    m1, _ = W.lgssm_1d(seed=1, T=10)
    # one FP64 job of N = 2^19 (about 20 MB) fills the 40 MB arena (which also
    # holds the job tables), so later requests wait in the pending queue
    with G.Server(hbm_budget_bytes=40 << 20, host_budget_bytes=64 << 20, max_pending=2) as srv:
        _, ys = W.lgssm_1d(seed=0, T=5000)
        srv.submit(m1, G.BF(1 << 19, precision="f64"), ys, tag=0)
        time.sleep(0.005)
        busy = 0
        for i in range(1, 8):
            try:
                srv.submit(m1, G.BF(1 << 19, precision="f64"), ys, tag=i)
            except G.GFError as e:
                assert e.code == L.GF_ERR_BUSY
                busy += 1
        srv.drain(timeout_ms=120000)
        done = srv.poll(max_results=64)
    assert busy >= 1
    assert len(done) == 8 - busy and all(r["status"] == 0 for r in done)


def test_failing_filter_fails_alone(ctx):
    rng = np.random.default_rng(5)
    good = _kf_model(rng, 4, 2)
    bad = _kf_model(rng, 4, 2)
    bad.obs.R[:] = -np.eye(2)  # innovation covariance not positive definite
    ys = rng.standard_normal((30, 2))
    with G.Server(hbm_budget_bytes=64 << 20, host_budget_bytes=64 << 20) as srv:
        srv.submit(good, G.KF(), ys, tag=0)
        srv.submit(bad, G.KF(), ys, tag=1)
        srv.submit(good, G.KF(), ys, tag=2)
        srv.drain(timeout_ms=60000)
        res = {r["tag"]: r for r in srv.poll()}
        st = srv.stats()
    _, ll = G.filter(good, G.KF(), ys, ctx=ctx)
    assert res[1]["status"] == L.GF_ERR_NOT_PD
    assert res[0]["status"] == 0 and res[0]["ll"] == ll and res[2]["ll"] == ll
    assert st["failed"] == 1 and st["completed"] == 2


def test_invalid_request_rejected_at_submit(ctx):
    rng = np.random.default_rng(2)
    m = _kf_model(rng, 40, 2)  # beyond the 32-wide Kalman buckets
    with G.Server(hbm_budget_bytes=16 << 20, host_budget_bytes=16 << 20) as srv:
        with pytest.raises(G.GFError) as e:
            srv.submit(m, G.KF(), rng.standard_normal((5, 2)))
        assert e.value.code == L.GF_ERR_DIM


def test_served_time_varying_pf_matches_standalone(ctx):
    """A particle filter on a time-varying model, served in a mix with homogeneous
    ones, returns exactly what the standalone gf_pf_run_tv call returns; a
    time-varying Kalman request is refused at submit (homogeneous only)."""
    import oracle as O
    rng = np.random.default_rng(8)
    reqs = []
    for dx, dy, T, N in [(2, 2, 30, 5000), (4, 3, 50, 3000), (16, 8, 20, 8192)]:
        om = O.create_nonhomogeneous_linear_gaussian_model(rng, dx, dy, T)
        As = [O.random_orthogonal(rng, dx) * rng.uniform(0.5, 0.95) for _ in range(T)]
        om = O.LGModel.time_varying(om.mu0, om.Sigma0, As, om.bs, om.Qs, om.Hs, om.cs, om.Rs)
        gm = G.create_nonhomogeneous_linear_gaussian_model(om.mu0, om.Sigma0, om.As, om.bs, om.Qs,
                                                           om.Hs, om.cs, om.Rs)
        reqs.append((gm, G.BF(N, threshold=0.6), O.sample(rng, om, T)[1], 40 + dx))
    m, ys = W.lgssm_1d(seed=5, T=40)
    reqs.append((m, G.BF(4096, threshold=0.5), ys, 9))
    with G.Server(hbm_budget_bytes=1 << 30, host_budget_bytes=128 << 20, pf_chunk=8) as srv:
        for k, (gm, algo, ys, seed) in enumerate(reqs):
            srv.submit(gm, algo, ys, seed=seed, tag=k, want_steps=True, want_mean=True)
        with pytest.raises(Exception):
            srv.submit(reqs[0][0], G.KalmanFilter(), reqs[0][2])
        srv.drain(timeout_ms=60000)
        got = {r["tag"]: r for r in srv.poll(max_results=64)}
    assert len(got) == len(reqs)
    for k, (gm, algo, ys, seed) in enumerate(reqs):
        r = got[k]
        assert r["status"] == 0, (k, r)
        ll, steps, mean, _ = _standalone(ctx, "bf", gm, algo, ys, seed)
        assert r["ll"] == ll, (k, r["ll"], ll)
        np.testing.assert_array_equal(r["ll_steps"], steps)
        np.testing.assert_array_equal(r["mean"], mean)
