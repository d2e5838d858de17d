"""ctypes binding of libgfb200.so (the C ABI declared in include/gf_b200.h).

Loading fails loudly when the shared library is missing: there is no CPU
fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_PKG), "lib", "libgfb200.so")

# status codes
GF_OK, GF_ERR_NOT_PD, GF_ERR_DIM, GF_ERR_OOM_BUDGET, GF_ERR_TIMEOUT = 0, 1, 2, 3, 4
GF_ERR_CUDA, GF_ERR_ARG, GF_ERR_UNSUPPORTED, GF_ERR_BUSY = 5, 6, 7, 8
GF_MEM_HOST, GF_MEM_DEVICE = 0, 1
GF_RS_SYSTEMATIC, GF_RS_STRATIFIED, GF_RS_MULTINOMIAL = 0, 1, 2
GF_CONV_CPU, GF_CONV_CUDAEXT = 0, 1
GF_PREC_F32, GF_PREC_F64 = 0, 1
GF_PROP_BOOTSTRAP, GF_PROP_OPTIMAL, GF_PROP_OVERDISPERSED = 0, 1, 2
GF_ALGO_KF, GF_ALGO_SRKF = 0, 1
GF_PLAN_AUTOTUNE, GF_PLAN_NO_GRAPH, GF_PLAN_PLAIN, GF_PLAN_SIMT, GF_PLAN_NO_FUSE = 1, 2, 4, 8, 16
GF_PLAN_STAGED_GATHER, GF_PLAN_UNITS, GF_PLAN_TILES = 32, 64, 128
GF_REQ_KF, GF_REQ_SRKF, GF_REQ_PF, GF_REQ_RBPF = 0, 1, 2, 3
GF_CSMC_NONE, GF_CSMC_ANCESTOR, GF_CSMC_BACKWARD = 0, 1, 2
GF_LOOKAHEAD_NONE, GF_LOOKAHEAD_MEAN, GF_LOOKAHEAD_DRAW = 0, 1, 2

EXPORTED = [
    "gf_ctx_create", "gf_ctx_destroy", "gf_last_error", "gf_ctx_set_stream", "gf_ctx_get_stream",
    "gf_ctx_synchronize", "gf_ctx_memory", "gf_ctx_profile", "gf_ctx_profile_read", "gf_version",
    "gf_kf_batch", "gf_kf_smooth", "gf_kf_batch_tv", "gf_kf_smooth_tv", "gf_kf_plan_create_tv",
    "gf_kf_plan_create", "gf_kf_plan_run", "gf_kf_plan_smooth", "gf_kf_plan_destroy",
    "gf_pf_run", "gf_pf_run_tv", "gf_pf_plan_create_tv", "gf_pf_plan_create", "gf_pf_plan_run", "gf_pf_plan_destroy", "gf_rbpf_run",
    "gf_rbpf_run_tv",
    "gf_sample_ancestors", "gf_offspring_to_ancestors", "gf_ancestors_to_offspring",
    "gf_rng_normals", "gf_sample_ancestors_noalloc", "gf_sample_ancestors_noalloc_max_n",
    "gf_srv_create", "gf_srv_submit", "gf_srv_poll", "gf_srv_drain", "gf_srv_stats",
    "gf_srv_reset_stats", "gf_srv_last_error", "gf_srv_destroy",
    "gf_csmc_run", "gf_csmc_run_tv", "gf_csmc_max_particles", "gf_pf_dense_ancestry", "gf_kf_loglikelihood_grad",
    "gf_kf_backward_information", "gf_kf_backward_information_tv",
]

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p


class LGModelC(C.Structure):
    _fields_ = [("dx", C.c_int32), ("dy", C.c_int32)] + [
        (n, _dp) for n in ("mu0", "Sigma0", "A", "b", "Q", "H", "c", "R")]


class RBModelC(C.Structure):
    _fields_ = ([("dxo", C.c_int32), ("dz", C.c_int32), ("dy", C.c_int32)]
                + [(n, _dp) for n in ("mu_o", "Sigma_o", "A_o", "b_o", "Q_o",
                                      "mu_z", "Sigma_z", "A_z", "b_z", "C_z", "Q_z")]
                + [("q_gamma", C.c_double), ("q_index", C.c_int32)]
                + [(n, _dp) for n in ("H", "c", "R")])


class PFConfigC(C.Structure):
    _fields_ = [("n_particles", C.c_int64), ("resampler", C.c_int32), ("convention", C.c_int32),
                ("threshold", C.c_double), ("precision", C.c_int32), ("proposal", C.c_int32),
                ("proposal_k", C.c_double), ("seed", C.c_uint64),
                ("schedule", C.POINTER(C.c_int8)), ("lookahead", C.c_int32)]


class PFOutC(C.Structure):
    _fields_ = [("ll", _vp), ("ll_steps", _vp), ("ess_steps", _vp), ("resampled", _vp),
                ("ancestors", _vp), ("means", _vp), ("states", _vp), ("log_weights", _vp),
                ("clamps", _vp), ("paths", _vp), ("history", _vp), ("log_weight_history", _vp)]


class CsmcConfigC(C.Structure):
    _fields_ = [("N", C.c_int32), ("threshold", C.c_double), ("resampler", C.c_int32),
                ("refresh", C.c_int32), ("seed", C.c_uint64)]


class CsmcOutC(C.Structure):
    _fields_ = [("trajectories", _vp), ("ll", _vp), ("ref", _vp), ("status", _vp)]


class KFGradOutC(C.Structure):
    _fields_ = [(n, _vp) for n in ("ll", "d_mu0", "d_Sigma0", "d_A", "d_b", "d_Q", "d_H", "d_c", "d_R",
                                   "status")]


class KFBackOutC(C.Structure):
    _fields_ = [(n, _vp) for n in ("lam_pred", "Om_pred", "lam_upd", "Om_upd", "mu_smooth", "Sigma_smooth",
                                   "status")]


class KFOutC(C.Structure):
    _fields_ = [("ll", _vp), ("ll_steps", _vp), ("means", _vp), ("covs", _vp), ("status", _vp)]


class SrvConfigC(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_size_t),
                ("host_budget_bytes", C.c_size_t), ("max_pending", C.c_int32),
                ("pf_chunk", C.c_int32), ("kf_streams", C.c_int32), ("max_active_pf", C.c_int32)]


class SrvRequestC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("T", C.c_int32), ("lg", C.POINTER(LGModelC)),
                ("rb", C.POINTER(RBModelC)), ("pf", C.POINTER(PFConfigC)), ("ys", _dp),
                ("jitter", C.c_double), ("use_jitter", C.c_int32), ("param_steps", C.c_int32),
                ("ll_steps", _dp), ("mean", _dp), ("cov", _dp), ("tag", C.c_uint64)]


class SrvResultC(C.Structure):
    _fields_ = [("id", C.c_uint64), ("tag", C.c_uint64), ("status", C.c_int32),
                ("kind", C.c_int32), ("ll", C.c_double), ("submit_ms", C.c_double),
                ("start_ms", C.c_double), ("done_ms", C.c_double)]


class SrvMetricsC(C.Structure):
    _fields_ = ([(n, C.c_int64) for n in ("submitted", "completed", "failed", "rejected",
                                          "pending", "running")]
                + [(n, C.c_double) for n in ("p50_ms", "p99_ms", "mean_ms", "max_ms", "kf_steps",
                                             "particle_steps", "elapsed_ms")]
                + [(n, C.c_size_t) for n in ("hbm_budget", "hbm_used", "hbm_peak")]
                + [(n, C.c_int64) for n in ("pf_iterations", "kf_batches", "launches")])


class GFError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[gf status {code}] {msg}")
        self.code = code


class PosDefException(GFError):
    """Raised for GF_ERR_NOT_PD, mirroring LinearAlgebra.PosDefException."""


_lib = None


def load(path: str | None = None):
    """Load libgfb200.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"libgfb200.so not found at {p}; build it with "
                          f"`python ssmproblems.jl_b200/build.py`")
    lib = C.CDLL(p)
    i32, i64, u64, dbl, sz = C.c_int32, C.c_int64, C.c_uint64, C.c_double, C.c_size_t
    ctxp = C.c_void_p
    sig = {
        "gf_ctx_create": (i32, [i32, sz, C.POINTER(ctxp)]),
        "gf_ctx_destroy": (i32, [ctxp]),
        "gf_last_error": (C.c_char_p, [ctxp]),
        "gf_ctx_set_stream": (i32, [ctxp, _vp]),
        "gf_ctx_get_stream": (_vp, [ctxp]),
        "gf_ctx_synchronize": (i32, [ctxp]),
        "gf_ctx_memory": (i32, [ctxp, C.POINTER(sz), C.POINTER(sz)]),
        "gf_ctx_profile": (i32, [ctxp, i32]),
        "gf_ctx_profile_read": (i32, [ctxp, i32, C.POINTER(dbl), C.POINTER(i64)]),
        "gf_version": (i32, []),
        "gf_kf_batch": (i32, [ctxp, i32, C.POINTER(LGModelC), i32, C.POINTER(i32), _vp, dbl,
                              i32, i32, C.POINTER(KFOutC)]),
        "gf_kf_smooth": (i32, [ctxp, C.POINTER(LGModelC), i32, C.POINTER(i32), _vp, i32,
                               C.POINTER(KFOutC)]),
        "gf_kf_plan_create": (i32, [ctxp, i32, C.POINTER(LGModelC), i32, C.POINTER(i32), dbl,
                                    i32, i32, C.POINTER(_vp)]),
        "gf_kf_batch_tv": (i32, [ctxp, i32, C.POINTER(LGModelC), i32, C.POINTER(i32), C.POINTER(i32),
                                 _vp, dbl, i32, i32, C.POINTER(KFOutC)]),
        "gf_kf_smooth_tv": (i32, [ctxp, C.POINTER(LGModelC), i32, C.POINTER(i32), C.POINTER(i32), _vp,
                                  i32, C.POINTER(KFOutC)]),
        "gf_kf_plan_create_tv": (i32, [ctxp, i32, C.POINTER(LGModelC), i32, C.POINTER(i32),
                                       C.POINTER(i32), dbl, i32, i32, C.POINTER(_vp)]),
        "gf_kf_plan_run": (i32, [_vp, _vp, C.POINTER(KFOutC)]),
        "gf_kf_plan_smooth": (i32, [_vp, _vp, C.POINTER(KFOutC)]),
        "gf_kf_plan_destroy": (i32, [_vp]),
        "gf_pf_run": (i32, [ctxp, C.POINTER(LGModelC), C.POINTER(PFConfigC), i32, _vp, _vp,
                            _vp, i32, C.POINTER(PFOutC)]),
        "gf_pf_plan_create": (i32, [ctxp, C.POINTER(LGModelC), C.POINTER(PFConfigC), i32, i32,
                                    C.POINTER(_vp)]),
        "gf_pf_run_tv": (i32, [ctxp, C.POINTER(LGModelC), i32, C.POINTER(PFConfigC), i32, _vp, _vp,
                               _vp, i32, C.POINTER(PFOutC)]),
        "gf_pf_plan_create_tv": (i32, [ctxp, C.POINTER(LGModelC), i32, C.POINTER(PFConfigC), i32, i32,
                                       C.POINTER(_vp)]),
        "gf_pf_plan_run": (i32, [_vp, _vp, _vp, _vp, C.POINTER(PFOutC)]),
        "gf_pf_plan_destroy": (i32, [_vp]),
        "gf_rbpf_run": (i32, [ctxp, C.POINTER(RBModelC), C.POINTER(PFConfigC), i32, _vp, _vp,
                              _vp, i32, C.POINTER(PFOutC), _vp]),
        "gf_rbpf_run_tv": (i32, [ctxp, C.POINTER(RBModelC), i32, C.POINTER(PFConfigC), i32, _vp, _vp,
                                 _vp, i32, C.POINTER(PFOutC), _vp]),
        "gf_sample_ancestors": (i32, [ctxp, i32, i32, i64, _vp, _vp, _vp]),
        "gf_offspring_to_ancestors": (i32, [ctxp, i64, _vp, _vp]),
        "gf_ancestors_to_offspring": (i32, [ctxp, i64, _vp, _vp]),
        "gf_rng_normals": (i32, [ctxp, u64, i32, i32, i64, i32, _vp]),
        "gf_sample_ancestors_noalloc": (i32, [i32, i32, i64, _vp, _vp, _vp, _vp]),
        "gf_sample_ancestors_noalloc_max_n": (i64, []),
        "gf_srv_create": (i32, [C.POINTER(SrvConfigC), C.POINTER(_vp)]),
        "gf_srv_submit": (i32, [_vp, C.POINTER(SrvRequestC), C.POINTER(u64)]),
        "gf_srv_poll": (i32, [_vp, C.POINTER(SrvResultC), i32, i32]),
        "gf_srv_drain": (i32, [_vp, i32]),
        "gf_srv_stats": (i32, [_vp, C.POINTER(SrvMetricsC)]),
        "gf_srv_reset_stats": (i32, [_vp]),
        "gf_srv_last_error": (C.c_char_p, [_vp]),
        "gf_srv_destroy": (i32, [_vp]),
        "gf_csmc_run": (i32, [ctxp, C.POINTER(LGModelC), C.POINTER(CsmcConfigC), i32, _vp, i32,
                              i32, i32, i32, _vp, _vp, i32, C.POINTER(CsmcOutC)]),
        "gf_csmc_run_tv": (i32, [ctxp, C.POINTER(LGModelC), i32, C.POINTER(CsmcConfigC), i32, _vp, i32,
                              i32, i32, i32, _vp, _vp, i32, C.POINTER(CsmcOutC)]),
        "gf_csmc_max_particles": (i32, []),
        "gf_pf_dense_ancestry": (i32, [ctxp, i32, i64, i32, i32, _vp, _vp, i64, _vp, i32, _vp]),
        "gf_kf_loglikelihood_grad": (i32, [ctxp, C.POINTER(LGModelC), i32, C.POINTER(i32), _vp, dbl, i32,
                                           i32, C.POINTER(KFGradOutC)]),
        "gf_kf_backward_information": (i32, [ctxp, C.POINTER(LGModelC), i32, C.POINTER(i32), _vp, dbl, i32,
                                             dbl, i32, i32, C.POINTER(KFBackOutC)]),
        "gf_kf_backward_information_tv": (i32, [ctxp, C.POINTER(LGModelC), i32, C.POINTER(i32),
                                                C.POINTER(i32), _vp, dbl, i32, dbl, i32, i32,
                                                C.POINTER(KFBackOutC)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(ctx, code):
    """Raise the Python mirror of the reference's exception for a status."""
    if code == GF_OK:
        return
    msg = load().gf_last_error(ctx).decode() if ctx else ""
    if code == GF_ERR_NOT_PD:
        raise PosDefException(code, msg)
    if code in (GF_ERR_ARG, GF_ERR_DIM):
        raise GFError(code, "ArgumentError: " + msg)
    raise GFError(code, msg)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def fortran64(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def ptr(a):
    """Address of a numpy array or torch tensor (None for None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


class Context:
    """Owns a gf_ctx (device, stream, HBM budget)."""

    def __init__(self, device: int = 0, budget_bytes: int = 0):
        lib = load()
        h = C.c_void_p()
        check(None, lib.gf_ctx_create(device, budget_bytes, C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            load().gf_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        check(self.h, load().gf_ctx_set_stream(self.h, stream_ptr))

    @property
    def stream(self):
        return load().gf_ctx_get_stream(self.h)

    def synchronize(self):
        check(self.h, load().gf_ctx_synchronize(self.h))

    def memory(self):
        u, b = C.c_size_t(), C.c_size_t()
        check(self.h, load().gf_ctx_memory(self.h, C.byref(u), C.byref(b)))
        return u.value, b.value

    def profile(self, enable: bool):
        check(self.h, load().gf_ctx_profile(self.h, int(enable)))

    def profile_read(self, cls: int):
        ms, n = C.c_double(), C.c_int64()
        check(self.h, load().gf_ctx_profile_read(self.h, cls, C.byref(ms), C.byref(n)))
        return ms.value, n.value


_default_ctx = {}


def default_context(device: int = 0) -> Context:
    if device not in _default_ctx:
        _default_ctx[device] = Context(device)
    return _default_ctx[device]
