"""Shared helpers for the tests (model conversion, noise, tolerances)."""
import numpy as np

import oracle as O
from gfb200 import workloads as W


def to_oracle(m):
    p, d, o = m.prior, m.dyn, m.obs
    return O.LGModel(p.mu0, p.Sigma0, d.A, d.b, d.Q, o.H, o.c, o.R)


def to_oracle_rb(h):
    op, od = h.outer_prior, h.outer_dyn
    ip, idn, ob = h.inner_model.prior, h.inner_model.dyn, h.inner_model.obs
    return O.RBModel(op.mu0, op.Sigma0, od.A, od.b, od.Q, ip.mu0, ip.Sigma0, idn.A, idn.b, idn.C,
                     idn.Q, ob.H, ob.c, ob.R, q_gamma=idn.q_gamma, q_index=idn.q_index)


def random_lg(rng, dx, dy, process_noise_scale=0.1, obs_noise_scale=1.0):
    """GFTest create_linear_gaussian_model with a numpy RNG, as a gfb200 model."""
    from gfb200 import create_homogeneous_linear_gaussian_model
    om = O.create_linear_gaussian_model(rng, dx, dy, process_noise_scale, obs_noise_scale)
    return create_homogeneous_linear_gaussian_model(om.mu0, om.Sigma0, om.A, om.b, om.Q, om.H,
                                                    om.c, om.R)


def dummy_rb_model(rng, d_outer=1, d_inner=1, dy=1):
    """GFTest create_dummy_linear_gaussian_model (dummy_linear_gaussian.jl:48-154):
    returns (full LG model, HierarchicalSSM) sharing the same parameters."""
    from gfb200 import (HierarchicalSSM, HomogeneousGaussianPrior,
                        HomogeneousLinearGaussianLatentDynamics,
                        HomogeneousLinearGaussianObservationProcess, InnerDynamics,
                        create_homogeneous_linear_gaussian_model)
    D = d_outer + d_inner
    mu0 = rng.random(D)
    S0 = np.zeros((D, D))
    S0[:d_outer, :d_outer] = O.rand_cov(rng, d_outer)
    S0[d_outer:, d_outer:] = O.rand_cov(rng, d_inner)
    A = np.zeros((D, D))
    A[:d_outer, :d_outer] = rng.random((d_outer, d_outer))
    A[d_outer:, :d_outer] = rng.random((d_inner, d_outer))
    A[d_outer:, d_outer:] = rng.random((d_inner, d_inner))
    rho = np.max(np.abs(np.linalg.eigvals(A)))
    if D > 2 and rho > 0.9:  # GFTest draws U(0,1) entries; keep the larger test models stable
        A *= 0.9 / rho
    b = rng.random(D)
    Q = np.zeros((D, D))
    Q[:d_outer, :d_outer] = O.rand_cov(rng, d_outer, scale=0.1)
    Q[d_outer:, d_outer:] = O.rand_cov(rng, d_inner, scale=0.1)
    H = np.zeros((dy, D))
    H[:, d_outer:] = rng.random((dy, d_inner))
    c = rng.random(dy)
    R = O.rand_cov(rng, dy, scale=1.0)
    full = create_homogeneous_linear_gaussian_model(mu0, S0, A, b, Q, H, c, R)
    o, i = slice(0, d_outer), slice(d_outer, D)
    hier = HierarchicalSSM(
        HomogeneousGaussianPrior(mu0[o], S0[o, o]),
        HomogeneousLinearGaussianLatentDynamics(A[o, o], b[o], Q[o, o]),
        HomogeneousGaussianPrior(mu0[i], S0[i, i]),
        InnerDynamics(A[i, i], b[i], A[i, o], Q[i, i]),
        HomogeneousLinearGaussianObservationProcess(H[:, i], c, R))
    return full, hier


def tv_rb_oracle_pair(rng, T, d_outer=1, d_inner=1, dy=1):
    """A time-varying hierarchical model built from T GFTest dummy models sharing
    the first one's prior: (joint TV LGModel, TV RBModel), both oracle models."""
    pairs = [dummy_rb_model(rng, d_outer, d_inner, dy) for _ in range(T)]
    fulls = [to_oracle(f) for f, _ in pairs]
    rbs = [to_oracle_rb(h) for _, h in pairs]
    f0, r0 = fulls[0], rbs[0]
    joint = O.LGModel.time_varying(f0.mu0, f0.Sigma0, *[[getattr(f, n) for f in fulls]
                                                         for n in ("A", "b", "Q", "H", "c", "R")])
    steps = [{n: getattr(r, n) for n in O.RBModel.STEP_NAMES} for r in rbs]
    rb = O.RBModel.time_varying(r0.mu_o, r0.Sigma_o, r0.mu_z, r0.Sigma_z, steps)
    return joint, rb


def tv_rb_model(rb):
    """The gfb200 HierarchicalSSM of a time-varying oracle RBModel."""
    from gfb200 import (HierarchicalSSM, HomogeneousGaussianPrior, NonHomogeneousInnerDynamics,
                        NonHomogeneousLinearGaussianLatentDynamics,
                        NonHomogeneousLinearGaussianObservationProcess)
    st = rb.steps
    return HierarchicalSSM(
        HomogeneousGaussianPrior(rb.mu_o, rb.Sigma_o),
        NonHomogeneousLinearGaussianLatentDynamics([k.A_o for k in st], [k.b_o for k in st],
                                                   [k.Q_o for k in st]),
        HomogeneousGaussianPrior(rb.mu_z, rb.Sigma_z),
        NonHomogeneousInnerDynamics([k.A_z for k in st], [k.b_z for k in st], [k.C_z for k in st],
                                    [k.Q_z for k in st], rb.q_gamma, rb.q_index),
        NonHomogeneousLinearGaussianObservationProcess([k.H for k in st], [k.c for k in st],
                                                       [k.R for k in st]))


def simulate(rng, m, T):
    return W.simulate_lg(rng, m, T)


def injected(rng, T, dx, N, kind, dtype=np.float64):
    noise = rng.standard_normal((T + 1, dx, N)).astype(dtype)
    if kind == O.SYSTEMATIC:
        unif = rng.random(T)
    else:
        unif = rng.random((T, N))
    return noise, unif


def ancestors_match(gpu_anc, or_anc, margins, band):
    """Return the number of slots that differ outside the boundary band (must be
    0) and the number of differing slots inside it (reported)."""
    diff = gpu_anc != or_anc
    inside = margins <= band
    return int(np.sum(diff & ~inside)), int(np.sum(diff & inside))
