"""gf_sample_ancestors_noalloc, the allocation-free variant for callers that
cannot call cudaMalloc while resampling: through the C ABI, its ancestors must
equal those of gf_sample_ancestors (exact integers) on two calls in a row,
which also checks that the shared fixed scratch is reset between calls; the
smaller call is also checked against the FP64 oracle directly, and repeated
calls must leave the device's free memory unchanged (nothing allocated).
Collected last so a stop-at-first-failure run has already run everything else."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_noalloc(lib, kind, conv, w, u, stream):
    import torch
    out = torch.zeros(w.numel(), dtype=torch.int64, device=w.device)
    st = lib.gf_sample_ancestors_noalloc(kind, conv, w.numel(), w.data_ptr(), u.data_ptr(),
                                         out.data_ptr(), stream)
    assert st == 0, st
    return out.cpu().numpy()


def _run_alloc(lib, ctx, kind, conv, w, u):
    import torch
    out = torch.zeros(w.numel(), dtype=torch.int64, device=w.device)
    st = lib.gf_sample_ancestors(ctx.h, kind, conv, w.numel(), w.data_ptr(), u.data_ptr(),
                                 out.data_ptr())
    assert st == 0, st
    return out.cpu().numpy()


@pytest.mark.parametrize("kind,conv", [(0, 0), (1, 0), (2, 0), (0, 1), (1, 1), (2, 1)])
def test_noalloc_matches_allocating_entry_point(kind, conv):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import gfb200
    from gfb200 import _lib as L
    lib = L.load()
    ctx = gfb200.default_context(0)
    n_max = lib.gf_sample_ancestors_noalloc_max_n()
    assert n_max == 1 << 18
    rng = np.random.default_rng(17 + kind + 10 * conv)
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row with different sizes and weights
    for n in (n_max, 5000):
        w = torch.tensor(rng.random(n) ** 4, dtype=torch.float64, device="cuda:0")
        u = torch.tensor(rng.random(1 if kind == 0 else n), dtype=torch.float64, device="cuda:0")
        a_noalloc = _run_noalloc(lib, kind, conv, w, u, stream)
        a_ref = _run_alloc(lib, ctx, kind, conv, w, u)
        np.testing.assert_array_equal(a_noalloc, a_ref)
        assert a_noalloc.min() >= 1 and a_noalloc.max() <= n
    # the last (n = 5000) call against the FP64 oracle: exact outside a 1e-9
    # band around the cumulative-weight boundaries
    import oracle as O
    from helpers import ancestors_match
    wh = w.cpu().numpy()
    ref, mar, _ = O.sample_ancestors(kind, wh / wh.sum(), u.cpu().numpy(),
                                     conv=O.CONV_CUDAEXT if conv else O.CONV_CPU)
    bad, _ = ancestors_match(a_noalloc, ref, mar, 1e-9)
    assert bad == 0
    # repeated calls allocate nothing: the device's free memory stays the same
    out = torch.zeros(n, dtype=torch.int64, device="cuda:0")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for _ in range(4):
        assert lib.gf_sample_ancestors_noalloc(kind, conv, n, w.data_ptr(), u.data_ptr(),
                                               out.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_noalloc_rejects_sizes_beyond_the_limit():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gfb200 import _lib as L
    lib = L.load()
    n = lib.gf_sample_ancestors_noalloc_max_n() + 1
    w = torch.ones(n, dtype=torch.float64, device="cuda:0")
    u = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    out = torch.zeros(n, dtype=torch.int64, device="cuda:0")
    st = lib.gf_sample_ancestors_noalloc(0, 0, n, w.data_ptr(), u.data_ptr(), out.data_ptr(), None)
    assert st == L.GF_ERR_DIM
