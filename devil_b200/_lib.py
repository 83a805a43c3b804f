"""ctypes binding of libdevil_b200.so (the C ABI in include/devil_b200.h).

The shared library is built in-tree (``devil_b200/libdevil_b200.so``) by
``devil_b200/csrc/Makefile``.  Importing this module never falls back to a
CPU implementation: if the library is missing or fails to load, the error
is raised.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdevil_b200.so")

# status codes (include/devil_b200.h)
(OK, ERR_ARG, ERR_CUDA, ERR_ZERO_COLUMN, ERR_SINGULAR, ERR_UNSORTED, ERR_NOMEM, ERR_UNSUPPORTED,
 ERR_NUMERIC) = range(9)
COUNTS_DENSE_F64, COUNTS_DENSE_F32, COUNTS_CSR_U16, COUNTS_CSR_F32, COUNTS_CSC_F64 = range(5)
DENSE_GENE_MAJOR, DENSE_CELL_MAJOR = 0, 1
SF_NONE, SF_NORMED_SUM, SF_PSINORM, SF_GIVEN = range(4)
OD_NONE, OD_MOM, OD_MLE, OD_NEW = range(4)
FORM_CHOSEN, FORM_PLAIN = 0, 1
PREC_FP32, PREC_TC_TF32, PREC_TC_BF16X3 = 0, 1, 2
ADJ_NONE, ADJ_BH, ADJ_BONFERRONI, ADJ_HOLM, ADJ_HOCHBERG, ADJ_BY, ADJ_HOMMEL = range(7)
GENE_CONVERGED, GENE_MAX_ITER, GENE_NAN = range(3)
NA_INT = -(2 ** 31)

# every exported entry point of include/devil_b200.h
EXPORTS = (
    "devil_version", "devil_fit_opts_default", "devil_ctx_create", "devil_ctx_destroy",
    "devil_last_error", "devil_ctx_stream", "devil_ctx_synchronize", "devil_ctx_launch_count",
    "devil_fit", "devil_fit_device", "devil_fit_async", "devil_test_de", "devil_test_de_device", "devil_p_adjust",
    "devil_calculate_sf", "devil_estimate_dispersion", "devil_init_beta", "devil_beta_fit",
    "devil_estimate_mom_dispersion", "devil_fit_dispersion", "devil_compute_hessian",
    "devil_compute_clustered_meat", "devil_nb_adjoint", "devil_cluster_blocks",
    "devil_group_order", "devil_ctx_set_profiling", "devil_ctx_profile", "devil_ctx_engine",
    "devil_p_adjust_device_static", "devil_fit_overdispersion_new", "devil_fit_batch",
    "devil_p_adjust_device", "devil_ctx_profile_tc", "devil_ctx_irls_rescued",
)


class DevilError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class Counts(C.Structure):
    _fields_ = [("format", C.c_int), ("dense_layout", C.c_int), ("n_genes", C.c_int64),
                ("n_cells", C.c_int64), ("nnz", C.c_int64), ("values", C.c_void_p),
                ("ptr", C.c_void_p), ("idx", C.c_void_p)]


class FitOpts(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("tolerance", C.c_double), ("overdispersion", C.c_int),
                ("init_beta_rough", C.c_int), ("size_factors", C.c_int),
                ("size_factor_values", C.c_void_p), ("offset", C.c_double),
                ("has_init_overdispersion", C.c_int), ("init_overdispersion", C.c_double),
                ("compute_theta_mom", C.c_int), ("form", C.c_int), ("precision", C.c_int)]


class Problem(C.Structure):
    _fields_ = [("counts", Counts), ("X", C.c_void_p), ("p", C.c_int),
                ("cluster_ends", C.c_void_p), ("n_clusters", C.c_int)]


class FitResult(C.Structure):
    _fields_ = [("beta", C.c_void_p), ("theta", C.c_void_p), ("beta_iters", C.c_void_p),
                ("theta_iters", C.c_void_p), ("bread", C.c_void_p), ("sandwich", C.c_void_p),
                ("theta_mom", C.c_void_p), ("status", C.c_void_p), ("size_factors", C.c_void_p),
                ("offset_vector", C.c_void_p), ("meat", C.c_void_p)]


_lib = None
_lock = threading.Lock()


def load():
    """Load the library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with "
                              "`make -C devil_b200/csrc` (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        vp, i64, i32, dbl, i = C.c_void_p, C.c_int64, C.c_int32, C.c_double, C.c_int
        L.devil_version.restype = C.c_char_p
        L.devil_fit_opts_default.argtypes = [C.POINTER(FitOpts)]
        L.devil_fit_opts_default.restype = None
        L.devil_ctx_create.argtypes = [i, C.POINTER(vp)]
        L.devil_ctx_destroy.argtypes = [vp]
        L.devil_last_error.argtypes = [vp]
        L.devil_last_error.restype = C.c_char_p
        L.devil_ctx_stream.argtypes = [vp]
        L.devil_ctx_stream.restype = vp
        L.devil_ctx_synchronize.argtypes = [vp]
        L.devil_ctx_launch_count.argtypes = [vp]
        L.devil_ctx_launch_count.restype = i64
        L.devil_fit.argtypes = [vp, C.POINTER(Counts), vp, i, vp, i, C.POINTER(FitOpts),
                                C.POINTER(FitResult)]
        L.devil_fit_device.argtypes = L.devil_fit.argtypes
        L.devil_fit_async.argtypes = [vp, vp] + list(L.devil_fit.argtypes[1:])
        L.devil_fit_async.restype = i
        L.devil_test_de.argtypes = [vp, i64, i, vp, vp, vp, i64, vp, i, dbl, vp, vp, vp]
        L.devil_test_de_device.argtypes = L.devil_test_de.argtypes
        L.devil_p_adjust.argtypes = [vp, i64, vp, i, vp]
        L.devil_p_adjust_device.argtypes = [vp, i64, vp, i, vp]
        L.devil_calculate_sf.argtypes = [vp, C.POINTER(Counts), i, vp]
        L.devil_estimate_dispersion.argtypes = [vp, C.POINTER(Counts), vp, vp]
        L.devil_init_beta.argtypes = [vp, C.POINTER(Counts), vp, i, vp, i, vp]
        L.devil_beta_fit.argtypes = [vp, C.POINTER(Counts), vp, i, vp, vp, vp, i, dbl, i, vp, vp]
        L.devil_estimate_mom_dispersion.argtypes = [vp, C.POINTER(Counts), vp, i, vp, vp, vp]
        L.devil_fit_dispersion.argtypes = [vp, C.POINTER(Counts), vp, i, vp, vp, i, i, vp, vp]
        L.devil_fit_overdispersion_new.argtypes = [vp, C.POINTER(Counts), vp, i, vp, vp, i, dbl, vp,
                                                   vp]
        L.devil_compute_hessian.argtypes = [vp, C.POINTER(Counts), vp, i, vp, vp, vp, vp]
        L.devil_compute_clustered_meat.argtypes = [vp, C.POINTER(Counts), vp, i, vp, vp, vp, vp,
                                                   i, vp]
        L.devil_nb_adjoint.argtypes = [vp, i64, vp, vp, dbl, vp, vp, vp]
        L.devil_cluster_blocks.argtypes = [i64, vp, vp, vp, C.POINTER(C.c_int)]
        L.devil_group_order.argtypes = [i64, vp, vp]
        L.devil_ctx_set_profiling.argtypes = [vp, i]
        L.devil_ctx_profile.argtypes = [vp, i, C.POINTER(i64), C.POINTER(dbl), C.POINTER(dbl)]
        L.devil_fit_batch.argtypes = [vp, i, C.POINTER(Problem), C.POINTER(FitOpts),
                                      C.POINTER(FitResult), i]
        L.devil_ctx_profile_tc.argtypes = [vp, i, C.POINTER(dbl)]
        L.devil_ctx_irls_rescued.argtypes = [vp]
        L.devil_ctx_irls_rescued.restype = i64
        L.devil_ctx_engine.argtypes = [vp, i]
        L.devil_ctx_engine.restype = i
        L.devil_p_adjust_device_static.argtypes = [i64, vp, i, vp, vp, C.c_char_p, C.c_size_t]
        _lib = L
    return _lib


class Context:
    """One devil_ctx (a CUDA stream plus device workspace) on one GPU."""

    def __init__(self, device: int = 0):
        L = load()
        h = C.c_void_p()
        rc = L.devil_ctx_create(int(device), C.byref(h))
        if rc != OK:
            raise DevilError(rc, f"devil_ctx_create failed with status {rc}")
        self.h = h
        self.device = device

    def check(self, rc):
        if rc != OK:
            msg = load().devil_last_error(self.h).decode()
            raise DevilError(rc, msg)

    @property
    def launches(self) -> int:
        return int(load().devil_ctx_launch_count(self.h))

    @property
    def stream(self) -> int:
        return int(load().devil_ctx_stream(self.h) or 0)

    def set_profiling(self, enable: bool):
        self.check(load().devil_ctx_set_profiling(self.h, int(bool(enable))))

    def profile(self, kind: int):
        """(launches, total ms, algorithmic bytes) of pass kind 0 IRLS, 1 MOM,
        2 MLE, 3 bread/meat since profiling was enabled."""
        n, ms, b = C.c_int64(0), C.c_double(0), C.c_double(0)
        self.check(load().devil_ctx_profile(self.h, int(kind), C.byref(n), C.byref(ms),
                                            C.byref(b)))
        return n.value, ms.value, b.value

    @property
    def irls_rescued(self) -> int:
        """Genes of the last fit that the tensor-core engine of p = 5..32
        handed back to the CUDA-core engine (a coefficient beyond +-8, or
        more steps than DEVIL_TCW_RESCUE)."""
        return int(load().devil_ctx_irls_rescued(self.h))

    def profile_tc_flops(self, kind: int) -> float:
        """Tensor-core FLOPs the profiled launches of a pass kind issued."""
        f = C.c_double(0)
        self.check(load().devil_ctx_profile_tc(self.h, int(kind), C.byref(f)))
        return f.value

    def engine(self, kind: int) -> str:
        """Engine of the last launch of pass kind 0 IRLS, 1 MOM, 2 MLE,
        3 bread/meat: "register", "shared", "groups", "tensor" (p <= 4),
        "tensor_wide" (IRLS, p = 5..32) or "none"."""
        e = load().devil_ctx_engine(self.h, int(kind))
        return {0: "register", 1: "shared", 2: "groups", 3: "tensor", 4: "tensor_wide"}.get(e, "none")

    def synchronize(self):
        self.check(load().devil_ctx_synchronize(self.h))

    def close(self):
        if getattr(self, "h", None):
            load().devil_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts: dict[int, Context] = {}


def context(device: int = 0) -> Context:
    ctx = _contexts.get(device)
    if ctx is None:
        ctx = _contexts[device] = Context(device)
    return ctx
