"""Generate the golden fixtures in tests/golden/ from the FP64 oracle.

The reference (pure Julia) cannot run in this environment, so the fixtures
are (a) the reference's own known-answer vectors, copied from
test/components/resamplers.jl:76-92, and (b) oracle outputs for small seeded
inputs -- the oracle itself is pinned by analytic checks in tests/test_oracle.py.
Run:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402


def main():
    out = {}
    # (a) known answers of ext/CUDAExt.jl offspring <-> ancestors
    out["offspring_to_ancestors"] = {"offspring": [0, 2, 2, 3, 5], "ancestors": [2, 2, 4, 5, 5]}
    out["ancestors_to_offspring"] = {"ancestors": [4, 2, 2, 3, 1], "offspring": [1, 2, 1, 1, 0]}
    # (b) KF / SRKF on GFTest-shaped models
    rng = np.random.default_rng(2024)
    kf = []
    for dy in (2, 3, 4):
        m = O.create_linear_gaussian_model(rng, 3, dy)
        _, ys = O.sample(rng, m, 5)
        ll, lls, mus, S = O.kf_filter(m, ys)
        ll2, _, _, _ = O.kf_filter(m, ys, algo="srkf")
        kf.append(dict(model={k: getattr(m, k).tolist() for k in
                              ("mu0", "Sigma0", "A", "b", "Q", "H", "c", "R")},
                       ys=ys.tolist(), ll=ll, ll_srkf=ll2, ll_steps=lls.tolist(),
                       mu_T=mus[-1].tolist(), Sigma_T=S[-1].tolist()))
    out["kalman"] = kf
    # (c) FP64 bootstrap PF with injected noise / uniforms, 3 resamplers
    pf = []
    m = O.LGModel([0.0], [[1.0]], [[1.0]], [0.0], [[0.01]], [[1.0]], [0.0], [[0.04]])
    rng = np.random.default_rng(7)
    x = rng.standard_normal() * 1.0
    ys = []
    for _ in range(20):
        x = x + 0.1 * rng.standard_normal()
        ys.append(x + 0.2 * rng.standard_normal())
    ys = np.array(ys).reshape(20, 1)
    N = 64
    noise = rng.standard_normal((21, 1, N))
    for kind in (O.SYSTEMATIC, O.STRATIFIED, O.MULTINOMIAL):
        unif = rng.random(20) if kind == O.SYSTEMATIC else rng.random((20, N))
        r = O.pf_run(m, N, ys, resampler=kind, threshold=0.5, noise=noise, uniforms=unif,
                     want_ancestors=True)
        pf.append(dict(kind=kind, N=N, ys=ys.ravel().tolist(), noise=noise.ravel().tolist(),
                       uniforms=np.asarray(unif).ravel().tolist(), ll=r["ll"],
                       ll_steps=r["ll_steps"].tolist(), resampled=r["resampled"].tolist(),
                       ancestors=r["ancestors"].tolist()))
    out["bootstrap_pf"] = pf
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
