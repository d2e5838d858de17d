"""Bounded device waits run out cleanly: the lookback scan's wait on a
predecessor's flag and the tensor-core propagate's mbarrier wait, each run
against a flag that nothing sets with a short poll limit, record
GF_ERR_TIMEOUT, and the context keeps working (a filter run afterwards still
matches the FP64 oracle).  With the flag published the same routines succeed."""
import ctypes as C

import numpy as np
import pytest

import gfb200 as G
import oracle as O
from gfb200 import workloads as W
from helpers import to_oracle

pytestmark = pytest.mark.gpu


def _selftest(which, publish, limit):
    from gfb200 import _lib as L
    lib = L.load()
    f = lib.gfx_wait_selftest
    f.argtypes = [C.c_int, C.c_int, C.c_longlong, C.POINTER(C.c_int),
                  C.POINTER(C.c_ulonglong)]
    st, ex = C.c_int(-1), C.c_ulonglong(0)
    assert f(which, publish, limit, C.byref(st), C.byref(ex)) == L.GF_OK
    return st.value, ex.value


@pytest.mark.parametrize("which", [0, 1], ids=["lookback", "mbarrier"])
def test_wait_on_unset_flag_times_out(ctx, which):
    from gfb200 import _lib as L
    st, _ = _selftest(which, 0, 64)
    assert st == L.GF_ERR_TIMEOUT
    st, ex = _selftest(which, 1, 1 << 20)
    assert st == L.GF_OK
    if which == 0:
        assert ex == 5  # tile 0's published inclusive prefix
    # the context is still usable after the timeouts
    m, ys = W.lgssm_1d(seed=3, T=20)
    rng = np.random.default_rng(1)
    N, T = 512, 20
    noise = rng.standard_normal((T + 1, 1, N))
    unif = rng.random(T)
    _, ll = G.filter(m, G.BF(N, threshold=0.5, precision="f64"), ys, noise=noise,
                     uniforms=unif, ctx=ctx)
    ref = O.pf_run(to_oracle(m), N, ys, threshold=0.5, noise=noise, uniforms=unif)
    assert abs(ll - ref["ll"]) < 1e-8
