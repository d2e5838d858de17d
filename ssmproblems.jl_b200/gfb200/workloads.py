"""Seeded synthetic workloads of the filtering benchmarks (numpy, FP64).

There are no public datasets for this path; each workload is generated from a
seed with the shapes and distributions of the benchmark configurations:

* ``lgssm_1d``     -- x0 ~ N(0,1), x_t = x_{t-1} + N(0, 0.1^2), y_t = x_t + N(0, 0.2^2)
                      (the SSMProblems README model), T = 100.
* ``lgssm_rot``    -- Dx-dim LGSSM with A a random orthogonal matrix scaled to
                      spectral radius 0.95, Q = 0.1 I, H_ij ~ N(0, 1/Dx), R = 0.2 I,
                      x0 ~ N(0, I); default Dx=16, Dy=8, T=1000.
* ``kf_bank``      -- B independent LGSSMs: Dx ~ U{2..32}, Dy ~ U{1..Dx}, A random
                      orthogonal scaled to rho ~ U(0.8, 0.99), Q = q I with
                      q ~ LogU(1e-3, 1), H Gaussian, R = r I with r ~ LogU(1e-2, 1),
                      T ~ U{64..2048}.
* ``rb_trend``     -- conditionally linear-Gaussian HierarchicalSSM: outer 2-D
                      z_t = 0.9 z_{t-1} + N(0, 0.3^2 I); inner Dx=8, A orthogonal*0.95,
                      Q = exp(z_t[1]) 0.05 I, H 4x8 Gaussian, R = 0.1 I; T = 500.
* ``serving_mix``  -- Poisson request stream: 70% KF (Dx 2..32, T 100..5000),
                      25% BF on the 1-D model (N 4096..262144, T 100..2000),
                      5% RBPF as rb_trend (N 4096..32768).
"""
from __future__ import annotations

import numpy as np

from .models import (HierarchicalSSM, HomogeneousGaussianPrior,
                     HomogeneousLinearGaussianLatentDynamics,
                     HomogeneousLinearGaussianObservationProcess, InnerDynamics,
                     create_homogeneous_linear_gaussian_model)


def random_orthogonal(rng, d):
    Z = rng.standard_normal((d, d))
    Qm, Rm = np.linalg.qr(Z)
    return Qm * np.sign(np.diag(Rm))


def simulate_lg(rng, model, T):
    """Forward simulation (SSMProblems utils/forward_simulation.jl:14-26)."""
    p, d, o = model.prior, model.dyn, model.obs
    dx, dy = d.A.shape[0], o.H.shape[0]
    Lq = np.linalg.cholesky(d.Q)
    Lr = np.linalg.cholesky(o.R)
    x = p.mu0 + np.linalg.cholesky(p.Sigma0) @ rng.standard_normal(dx)
    ys = np.empty((T, dy))
    xs = np.empty((T, dx))
    for t in range(T):
        x = d.A @ x + d.b + Lq @ rng.standard_normal(dx)
        xs[t] = x
        ys[t] = o.H @ x + o.c + Lr @ rng.standard_normal(dy)
    return xs, ys


def lgssm_1d(seed=0, T=100):
    rng = np.random.default_rng(seed)
    m = create_homogeneous_linear_gaussian_model([0.0], [[1.0]], [[1.0]], [0.0], [[0.01]],
                                                 [[1.0]], [0.0], [[0.04]])
    _, ys = simulate_lg(rng, m, T)
    return m, ys


def lgssm_rot(seed=0, dx=16, dy=8, T=1000, rho=0.95, q=0.1, r=0.2):
    rng = np.random.default_rng(seed)
    A = random_orthogonal(rng, dx) * rho
    H = rng.standard_normal((dy, dx)) / np.sqrt(dx)
    m = create_homogeneous_linear_gaussian_model(np.zeros(dx), np.eye(dx), A, np.zeros(dx),
                                                 q * np.eye(dx), H, np.zeros(dy), r * np.eye(dy))
    _, ys = simulate_lg(rng, m, T)
    return m, ys


def kf_bank(B, seed=0, dx_range=(2, 32), T_range=(64, 2048), simulate=False, make_ys=True):
    """Returns (models, T list, ys list).  With simulate=False the observations are
    N(0,1) draws: the KF's arithmetic does not depend on their values, and the
    bank stays cheap to build at B = 65536 (parameters are drawn in batches per
    state dimension)."""
    rng = np.random.default_rng(seed)
    dxs = rng.integers(dx_range[0], dx_range[1] + 1, size=B)
    dys = np.array([rng.integers(1, d + 1) for d in dxs])
    rhos = rng.uniform(0.8, 0.99, size=B)
    qs = np.exp(rng.uniform(np.log(1e-3), np.log(1.0), size=B))
    rs = np.exp(rng.uniform(np.log(1e-2), np.log(1.0), size=B))
    Ts = rng.integers(T_range[0], T_range[1] + 1, size=B)
    As = [None] * B
    for d in np.unique(dxs):
        idx = np.nonzero(dxs == d)[0]
        Z = rng.standard_normal((idx.size, d, d))
        Qm, Rm = np.linalg.qr(Z)
        sgn = np.sign(np.diagonal(Rm, axis1=1, axis2=2))
        Orth = Qm * sgn[:, None, :]
        for j, f in enumerate(idx):
            As[f] = Orth[j] * rhos[f]
    models, yss = [], []
    for f in range(B):
        dx, dy = int(dxs[f]), int(dys[f])
        H = rng.standard_normal((dy, dx)) / np.sqrt(dx)
        m = create_homogeneous_linear_gaussian_model(np.zeros(dx), np.eye(dx), As[f], np.zeros(dx),
                                                     qs[f] * np.eye(dx), H, np.zeros(dy),
                                                     rs[f] * np.eye(dy))
        T = int(Ts[f])
        if simulate:
            _, ys = simulate_lg(rng, m, T)
        elif make_ys:
            ys = rng.standard_normal((T, dy))
        else:
            ys = None
        models.append(m)
        yss.append(ys)
    return models, [int(t) for t in Ts], yss


def rb_trend(seed=0, T=500, dz=8, dy=4, q_gamma=1.0):
    rng = np.random.default_rng(seed)
    dxo = 2
    Az = random_orthogonal(rng, dz) * 0.95
    H = rng.standard_normal((dy, dz)) / np.sqrt(dz)
    model = HierarchicalSSM(
        HomogeneousGaussianPrior(np.zeros(dxo), np.eye(dxo)),
        HomogeneousLinearGaussianLatentDynamics(0.9 * np.eye(dxo), np.zeros(dxo), 0.09 * np.eye(dxo)),
        HomogeneousGaussianPrior(np.zeros(dz), np.eye(dz)),
        InnerDynamics(Az, np.zeros(dz), np.zeros((dz, dxo)), 0.05 * np.eye(dz), q_gamma=q_gamma,
                      q_index=0),
        HomogeneousLinearGaussianObservationProcess(H, np.zeros(dy), 0.1 * np.eye(dy)))
    # simulate (models/hierarchical.jl:57-86)
    x = rng.standard_normal(dxo)
    z = rng.standard_normal(dz)
    Lr = np.linalg.cholesky(0.1 * np.eye(dy))
    ys = np.empty((T, dy))
    for t in range(T):
        xn = 0.9 * x + 0.3 * rng.standard_normal(dxo)
        qz = 0.05 * np.exp(q_gamma * xn[0])
        z = Az @ z + np.sqrt(qz) * rng.standard_normal(dz)
        x = xn
        ys[t] = H @ z + Lr @ rng.standard_normal(dy)
    return model, ys


def serving_mix(n_requests, rate, seed=0):
    """List of (arrival_s, kind, params) with Poisson arrivals at `rate` req/s."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n_requests):
        t += rng.exponential(1.0 / rate)
        u = rng.random()
        if u < 0.70:
            dx = int(rng.integers(2, 33))
            out.append((t, "kf", dict(dx=dx, dy=int(rng.integers(1, dx + 1)),
                                      T=int(rng.integers(100, 5001)),
                                      seed=int(rng.integers(2**31)))))
        elif u < 0.95:
            out.append((t, "bf", dict(N=int(rng.integers(4096, 262145)),
                                      T=int(rng.integers(100, 2001)),
                                      seed=int(rng.integers(2**31)))))
        else:
            out.append((t, "rbpf", dict(N=int(rng.integers(4096, 32769)), T=500,
                                        seed=int(rng.integers(2**31)))))
    return out
