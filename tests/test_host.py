"""Host-side logic of the Python mirror (no GPU calls)."""
import numpy as np
import pytest

import gfb200 as G
from gfb200 import _lib as L
from gfb200 import workloads as W
from gfb200.filtering import _pf_config


def test_alternating_resampler_schedule():
    """GFTest AlternatingResampler: resample_next is only flipped by resample(),
    so the reference resamples at step 1 and never again."""
    assert G.AlternatingResampler().schedule(5) == [1, 0, 0, 0, 0]


def test_pf_config_mapping():
    algo = G.BF(1000, threshold=0.5, resampler=G.Stratified(), precision="f64",
                convention="cudaext")
    cfg, sched, prec = _pf_config(algo, 10, seed=7)
    assert cfg.n_particles == 1000 and cfg.resampler == L.GF_RS_STRATIFIED
    assert cfg.threshold == 0.5 and cfg.precision == L.GF_PREC_F64
    assert cfg.convention == L.GF_CONV_CUDAEXT and cfg.seed == 7 and sched is None
    algo = G.PF(10, G.OverdispersedProposal(None, 2.5), resampler=G.AlternatingResampler())
    cfg, sched, _ = _pf_config(algo, 3, seed=1)
    assert cfg.proposal == L.GF_PROP_OVERDISPERSED and cfg.proposal_k == 2.5
    assert sched.tolist() == [1, 0, 0]


def test_default_threshold_is_reference_default():
    """ParticleFilter(N, proposal; threshold=1.0) (particles.jl:100-105)."""
    algo = G.BF(10)
    assert algo.resampler.threshold == 1.0 and isinstance(algo.resampler.resampler, G.Systematic)


def test_model_dimension_checks():
    m = G.create_homogeneous_linear_gaussian_model(np.zeros(2), np.eye(2), np.eye(2), np.zeros(2),
                                                   np.eye(2), np.ones((1, 2)), np.zeros(1),
                                                   np.eye(1))
    m._c_struct()
    bad = G.create_homogeneous_linear_gaussian_model(np.zeros(2), np.eye(3), np.eye(2),
                                                     np.zeros(2), np.eye(2), np.ones((1, 2)),
                                                     np.zeros(1), np.eye(1))
    with pytest.raises(ValueError):
        bad._c_struct()


def test_rbpf_requires_kalman_inner():
    with pytest.raises(TypeError):
        G.RBPF(G.BF(10), G.SRKF())


def test_workloads_shapes():
    m, ys = W.lgssm_rot(seed=1, dx=16, dy=8, T=10)
    assert m.dx == 16 and m.dy == 8 and ys.shape == (10, 8)
    assert abs(np.max(np.abs(np.linalg.eigvals(m.dyn.A))) - 0.95) < 1e-12
    models, Ts, yss = W.kf_bank(50, seed=2)
    assert all(1 <= mm.dy <= mm.dx <= 32 for mm in models)
    assert all(64 <= t <= 2048 for t in Ts)
    h, ys = W.rb_trend(seed=0, T=20)
    assert (h.dxo, h.dz, h.dy) == (2, 8, 4) and ys.shape == (20, 4)
    reqs = W.serving_mix(200, rate=1000.0, seed=0)
    kinds = [k for _, k, _ in reqs]
    assert kinds.count("kf") > kinds.count("bf") > kinds.count("rbpf")


def test_apf_config_and_unbuilt_lookahead():
    """AuxiliaryParticleFilter(pf, MeanPredictive()/ModePredictive()) maps to
    GF_LOOKAHEAD_MEAN, DrawPredictive() to GF_LOOKAHEAD_DRAW."""
    apf = G.APF(G.BF(100, threshold=0.7), G.MeanPredictive())
    cfg, _, _ = _pf_config(apf.pf, 5, 1, lookahead=apf.weight_strategy.pp.lookahead)
    assert cfg.lookahead == L.GF_LOOKAHEAD_MEAN and cfg.threshold == 0.7
    assert G.APF(G.BF(10), G.ModePredictive()).weight_strategy.pp.lookahead == L.GF_LOOKAHEAD_MEAN
    assert G.APF(G.BF(10), G.DrawPredictive()).weight_strategy.pp.lookahead == L.GF_LOOKAHEAD_DRAW
