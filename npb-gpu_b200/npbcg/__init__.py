"""npbcg -- Python binding of libcgb.so, the B200 CG inverse-power-iteration library.

Mirrors the reference's CG call surface (GMAP/NPB-GPU CUDA/CG/cg.cu):

* ``makea(n, nonzer, rcond, shift, seed)`` -> ``(rowstr, colidx, a)``, the
  reference makea()+sparse() (cg.cu:1303-1368, :1611-1785) seeded as main()
  does (cg.cu:404-408);
* ``Session(rowstr, colidx, a)`` holds the matrix on the GPU (setup_gpu,
  cg.cu:1390-1603);
* ``Session.conj_grad(x)`` -> ``(z, p, q, r, rnorm)``, the reference
  conj_grad (cg.cu:653-801);
* ``Session.power_iterate(niter, shift, ...)`` runs the timed outer loop
  (cg.cu:491-522) and returns the zeta / rnorm traces.

Errors raise ``CgbError`` carrying the library's status code and message;
there is no CPU fallback: without libcgb.so or a usable sm_100 GPU the
solver calls raise.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libcgb.so")

# status codes (include/cgb.h)
OK = 0
ERR_INVALID = 1
ERR_NOMEM = 2
ERR_CAPACITY = 3
ERR_CUDA = 4
ERR_TIMEOUT = 5
ERR_NO_DEVICE = 6
ERR_STATE = 7
ERR_NUMERIC = 8
ERR_BAD_MATRIX = 9

MODE_FP64 = 0
MODE_FP64_TOL = 1
MODE_MIXED = 2
MODE_MIXED_LEARNED = 3

# NPB classes (setparams.cpp:751-785) and their verification zetas (cg.cu:373-396)
CLASSES = {
    "S": dict(n=1400, nonzer=7, niter=15, shift=10.0, zeta=8.5971775078648),
    "W": dict(n=7000, nonzer=8, niter=15, shift=12.0, zeta=10.362595087124),
    "A": dict(n=14000, nonzer=11, niter=15, shift=20.0, zeta=17.130235054029),
    "B": dict(n=75000, nonzer=13, niter=75, shift=60.0, zeta=22.712745482631),
    "C": dict(n=150000, nonzer=15, niter=75, shift=110.0, zeta=28.973605592845),
    # D and E: beyond what one CSR of this library holds in E's case (6.3e9
    # entries); the row-partitioned solver (Part) runs both
    "D": dict(n=1500000, nonzer=21, niter=100, shift=500.0, zeta=52.514532105794),
    "E": dict(n=9000000, nonzer=26, niter=100, shift=1500.0, zeta=77.522164599383),
}
RCOND = 0.1
SEED = 314159265.0
VERIFY_EPSILON = 1.0e-10


class CgbError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


class Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("lanes_per_row", ctypes.c_int),
                ("block_threads", ctypes.c_int), ("wait_limit_ns", ctypes.c_longlong),
                ("use_graph", ctypes.c_int), ("keep_fp32_copy", ctypes.c_int),
                ("spmv_kernel", ctypes.c_int), ("panel_rows", ctypes.c_int)]


class SolveParams(ctypes.Structure):
    _fields_ = [("niter", ctypes.c_int), ("shift", ctypes.c_double), ("mode", ctypes.c_int),
                ("cgitmax", ctypes.c_int), ("tol", ctypes.c_double),
                ("refresh_every", ctypes.c_int), ("recycle", ctypes.c_int)]


class BatchParams(ctypes.Structure):
    _fields_ = [("niter", ctypes.c_int), ("mode", ctypes.c_int), ("cgitmax", ctypes.c_int),
                ("tol", ctypes.c_double), ("refresh_every", ctypes.c_int),
                ("recycle", ctypes.c_int)]


class SolveResult(ctypes.Structure):
    _fields_ = [("zeta", ctypes.c_double), ("rnorm", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("total_inner", ctypes.c_int),
                ("fallbacks", ctypes.c_int), ("refreshes", ctypes.c_int)]


_I32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_F64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_F32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_lib = None

# every symbol include/cgb.h declares, with its ctypes signature
_SIGNATURES = {
    "cgb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "cgb_last_error": (ctypes.c_char_p, []),
    "cgb_version": (ctypes.c_int, []),
    "cgb_nz_bound": (ctypes.c_longlong, [ctypes.c_int, ctypes.c_int]),
    "cgb_makea": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, _I32, _I32, _F64, ctypes.c_longlong,
                                 ctypes.POINTER(ctypes.c_longlong)]),
    "cgb_makea_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, _I32, _I32, _F64,
                                        ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]),
    "cgb_create_generated": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_default_options": (None, [ctypes.POINTER(Options)]),
    "cgb_create": (ctypes.c_int, [ctypes.c_int, _I32, _I32, _F64, ctypes.POINTER(Options),
                                  ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_upload": (ctypes.c_int, [ctypes.c_void_p, _I32, _I32, _F64]),
    "cgb_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_conj_grad": (ctypes.c_int, [ctypes.c_void_p, _I32, _I32, _F64, _F64, _F64, _F64, _F64,
                                     _F64, ctypes.POINTER(ctypes.c_double)]),
    "cgb_matrix_changed": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_default_solve_params": (None, [ctypes.POINTER(SolveParams)]),
    "cgb_power_iterate": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SolveParams),
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.POINTER(SolveResult)]),
    "cgb_time_spmv": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double)]),
    "cgb_time_outer_steps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                            ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double)]),
    "cgb_plan_info": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 4 +
                      [ctypes.POINTER(ctypes.c_longlong)] * 2),
    "cgb_selftest_wait_timeout": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong,
                                                 ctypes.POINTER(ctypes.c_int)]),
    "cgb_conj_grad_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong] +
                              [ctypes.c_void_p] * 8),
    "cgb_set_preconditioner": (ctypes.c_int, [ctypes.c_void_p, _I32, _I32, _F64]),
    "cgb_gnn_param_count": (ctypes.c_int, []),
    "cgb_gnn_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint, ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_gnn_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_gnn_get_params": (ctypes.c_int, [ctypes.c_void_p, _F32, ctypes.c_int]),
    "cgb_gnn_set_params": (ctypes.c_int, [ctypes.c_void_p, _F32, ctypes.c_int]),
    "cgb_gnn_graph_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _I32, _I32, _F64,
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_gnn_graph_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_gnn_graph_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_longlong), ctypes.c_void_p]),
    "cgb_gnn_loss_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_uint, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_float), ctypes.c_void_p]),
    "cgb_gnn_train_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint,
                                          ctypes.c_int, ctypes.c_float,
                                          ctypes.POINTER(ctypes.c_float)]),
    "cgb_gnn_infer": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "cgb_gnn_attach": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "cgb_default_batch_params": (None, [ctypes.POINTER(BatchParams)]),
    "cgb_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _I32, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, _F64,
                                        ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_batch_solve": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchParams), _F64, _F64,
                                       _I32, _I32, ctypes.POINTER(ctypes.c_double)]),
    "cgb_batch_tune": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchParams),
                                      ctypes.POINTER(ctypes.c_int)] +
                       [ctypes.POINTER(ctypes.c_double)] * 4),
    "cgb_plan_l2_keep": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "cgb_plan_panels": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    "cgb_check_status": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    "cgb_time_barrier": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_double)]),
    "cgb_set_l2_keep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "cgb_batch_policy": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_int)]),
    "cgb_batch_set_team_frac": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "cgb_batch_set_preconditioner": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _I32, _I32,
                                                    _F64]),
    "cgb_batch_fallbacks": (ctypes.c_int, [ctypes.c_void_p, _I32]),
    "cgb_gnn_attach_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_int]),
    "cgb_part_rows": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "cgb_nccl_unique_id": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_part_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _I32,
                                       _I32, _F64, ctypes.c_void_p,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_part_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_part_join": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "cgb_part_set_wait_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "cgb_part_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)]),
    "cgb_part_create_generated": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                 ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_part_power_iterate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_double)]),
    "cgb_part_group_power_iterate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                    ctypes.c_double, ctypes.c_int,
                                                    ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.POINTER(ctypes.c_double)]),
    "cgb_mg_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_mg_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_mg_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    "cgb_mg_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _F64, ctypes.c_longlong]),
    "cgb_mg_points": (ctypes.c_int, [ctypes.c_void_p, _I32, _I32]),
    "cgb_mg_apply": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_void_p, _F64]),
    "cgb_ep_run": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                  ctypes.POINTER(ctypes.c_double), _F64,
                                  ctypes.POINTER(ctypes.c_double)]),
    "cgb_is_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_char, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_is_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_is_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                  ctypes.POINTER(ctypes.c_double)]),
    "cgb_is_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong]),
    "cgb_ft_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]),
    "cgb_ft_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_ft_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _F64, ctypes.POINTER(ctypes.c_double)]),
    "cgb_ft_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _F64, ctypes.c_longlong]),
    "cgb_host_alloc": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_longlong]),
    "cgb_host_free": (ctypes.c_int, [ctypes.c_void_p]),
    "cgb_device_info": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_longlong)]),
}


def lib():
    """Load libcgb.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CgbError(ERR_STATE, f"{LIB_PATH} is missing: run npb-gpu_b200/build.py")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def _check(status):
    if status != OK:
        msg = lib().cgb_last_error().decode(errors="replace")
        raise CgbError(status, msg or lib().cgb_status_string(status).decode())


def _ptr(arr):
    return None if arr is None else arr.ctypes.data_as(ctypes.c_void_p)


def nz_bound(n, nonzer):
    return int(lib().cgb_nz_bound(n, nonzer))


def makea(n, nonzer, rcond=RCOND, shift=10.0, seed=SEED):
    """The reference matrix: returns (rowstr int32[n+1], colidx int32[nnz], a float64[nnz])."""
    cap = nz_bound(n, nonzer)
    rowstr = np.zeros(n + 1, np.int32)
    colidx = np.zeros(max(cap, 1), np.int32)
    a = np.zeros(max(cap, 1), np.float64)
    nnz = ctypes.c_longlong(0)
    _check(lib().cgb_makea(n, nonzer, rcond, shift, seed, rowstr, colidx, a, cap,
                           ctypes.byref(nnz)))
    k = nnz.value
    return rowstr, colidx[:k].copy(), a[:k].copy()


def makea_device(n, nonzer, rcond=RCOND, shift=10.0, seed=SEED, device=0):
    """makea with the assembly on the GPU (bit-identical to makea)."""
    cap = nz_bound(n, nonzer)
    rowstr = np.zeros(n + 1, np.int32)
    colidx = np.zeros(max(cap, 1), np.int32)
    a = np.zeros(max(cap, 1), np.float64)
    nnz = ctypes.c_longlong(0)
    _check(lib().cgb_makea_device(device, n, nonzer, rcond, shift, seed, rowstr, colidx, a, cap,
                                  ctypes.byref(nnz)))
    k = nnz.value
    return rowstr, colidx[:k].copy(), a[:k].copy()


def device_info(device=0):
    sm, ma, mi, mem = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
    _check(lib().cgb_device_info(device, ctypes.byref(sm), ctypes.byref(ma), ctypes.byref(mi),
                                 ctypes.byref(mem)))
    return dict(sm_count=sm.value, cc=(ma.value, mi.value), global_mem=mem.value)


def default_options(**kw):
    o = Options()
    lib().cgb_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Session:
    """A matrix resident on one GPU (the reference's setup_gpu state)."""

    def __init__(self, rowstr, colidx, a, **options):
        self.n = int(len(rowstr) - 1)
        self._keep = (np.ascontiguousarray(rowstr, np.int32),
                      np.ascontiguousarray(colidx, np.int32),
                      np.ascontiguousarray(a, np.float64))
        opts = default_options(**options)
        h = ctypes.c_void_p()
        _check(lib().cgb_create(self.n, *self._keep, ctypes.byref(opts), ctypes.byref(h)))
        self._h = h

    @classmethod
    def generated(cls, n, nonzer, shift, seed=SEED, rcond=RCOND, **options):
        """A session on the generator's matrix built on the device, never
        copied to the host (the same matrix as Session(*makea(...)))."""
        self = cls.__new__(cls)
        self.n = int(n)
        self._keep = None
        opts = default_options(**options)
        h = ctypes.c_void_p()
        _check(lib().cgb_create_generated(int(n), int(nonzer), float(rcond), float(shift),
                                          float(seed), ctypes.byref(opts), ctypes.byref(h)))
        self._h = h
        return self

    def close(self):
        if getattr(self, "_h", None):
            lib().cgb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, rowstr, colidx, a):
        self._keep = (np.ascontiguousarray(rowstr, np.int32),
                      np.ascontiguousarray(colidx, np.int32),
                      np.ascontiguousarray(a, np.float64))
        _check(lib().cgb_upload(self._h, *self._keep))

    def conj_grad(self, x, matrix=None):
        """One reference conj_grad from z = 0; returns (z, p, q, r, rnorm), n+1 entries each.
        `matrix` (rowstr, colidx, a): the CSR to pass, as the reference's call does
        (uploaded when it is not the session's); default the arrays the session
        was created or last uploaded with."""
        n = self.n
        xv = np.ones(n + 1, np.float64)
        xv[: min(len(x), n + 1)] = np.asarray(x, np.float64)[: n + 1]
        z, p, q, r = (np.zeros(n + 1) for _ in range(4))
        rn = ctypes.c_double()
        if matrix is not None:
            self._keep = (np.ascontiguousarray(matrix[0], np.int32),
                          np.ascontiguousarray(matrix[1], np.int32),
                          np.ascontiguousarray(matrix[2], np.float64))
        if self._keep is None:
            raise ValueError("this session's matrix has no host arrays: pass matrix=")
        rowstr, colidx, a = self._keep
        _check(lib().cgb_conj_grad(self._h, colidx, rowstr, xv, z, a, p, q, r, ctypes.byref(rn)))
        return z, p, q, r, rn.value

    def matrix_changed(self):
        """The host arrays the session holds were edited in place: the next
        conj_grad uploads them again (cgb_matrix_changed)."""
        _check(lib().cgb_matrix_changed(self._h))

    def power_iterate(self, niter, shift, mode=MODE_FP64, cgitmax=25, tol=1e-12,
                      refresh_every=10, want_x=False, recycle=4):
        """The outer loop of cg.cu:500-520; returns a dict with traces and timings.
        `recycle`: Galerkin start on that many previous iterates (tolerance modes)."""
        P = SolveParams()
        lib().cgb_default_solve_params(ctypes.byref(P))
        P.niter, P.shift, P.mode, P.cgitmax = niter, shift, mode, cgitmax
        P.tol, P.refresh_every, P.recycle = tol, refresh_every, recycle
        zt, rt = np.zeros(niter), np.zeros(niter)
        it = np.zeros(niter, np.int32)
        x = np.zeros(self.n) if want_x else None
        res = SolveResult()
        _check(lib().cgb_power_iterate(self._h, ctypes.byref(P), _ptr(zt), _ptr(rt), _ptr(it),
                                       _ptr(x), ctypes.byref(res)))
        out = dict(zeta=zt, rnorm=rt, iters=it, device_ms=res.device_ms,
                   total_inner=res.total_inner, fallbacks=res.fallbacks,
                   refreshes=res.refreshes)
        if want_x:
            out["x"] = x
        return out

    def set_preconditioner(self, fptr, fcol, fval):
        """M = F^T F for the preconditioned mode; F lower CSR with a positive diagonal."""
        _check(lib().cgb_set_preconditioner(self._h, np.ascontiguousarray(fptr, np.int32),
                                            np.ascontiguousarray(fcol, np.int32),
                                            np.ascontiguousarray(fval, np.float64)))

    def time_spmv(self, reps=50, fp32=False):
        ms = ctypes.c_double()
        _check(lib().cgb_time_spmv(self._h, reps, int(fp32), ctypes.byref(ms)))
        return ms.value

    def time_outer_steps(self, niter, shift):
        k, g = ctypes.c_double(), ctypes.c_double()
        _check(lib().cgb_time_outer_steps(self._h, niter, shift, ctypes.byref(k), ctypes.byref(g)))
        return k.value, g.value

    def plan(self):
        """The kernel configuration chosen for this matrix."""
        v = [ctypes.c_int() for _ in range(4)]
        smem, entries = ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().cgb_plan_info(self._h, *[ctypes.byref(x) for x in v], ctypes.byref(smem),
                                   ctypes.byref(entries)))
        kind, lpr, grid, block = (x.value for x in v)
        keep = ctypes.c_double()
        _check(lib().cgb_plan_l2_keep(self._h, ctypes.byref(keep)))
        pa, pf = ctypes.c_int(), ctypes.c_int()
        _check(lib().cgb_plan_panels(self._h, ctypes.byref(pa), ctypes.byref(pf)))
        return dict(kind={1: "row", 2: "sliced", 3: "sliced"}.get(kind, kind), l2_prefetch=kind == 3,
                    l2_keep_mb=keep.value / 1e6, lanes_per_row=lpr, grid=grid, block=block,
                    smem=smem.value, layout_entries=entries.value, panels=pa.value,
                    prec_panels=pf.value)

    def set_l2_keep(self, nbytes):
        """Bytes of the sliced matrix stream kept in L2 across products
        (overrides the autotuner; 0 = pure stream; results unchanged)."""
        _check(lib().cgb_set_l2_keep(self._h, float(nbytes)))

    def time_barrier(self, iters=20000):
        """Device microseconds per grid barrier of the session's plan."""
        us = ctypes.c_double()
        _check(lib().cgb_time_barrier(self._h, int(iters), ctypes.byref(us)))
        return us.value

    def selftest_wait_timeout(self, limit_ns):
        """Returns (status, device_status) of the bounded-wait self-test."""
        dev = ctypes.c_int()
        st = lib().cgb_selftest_wait_timeout(self._h, limit_ns, ctypes.byref(dev))
        return st, dev.value


# the sources of the single-system solver's kernels and of the host code that
# plans and launches them
SOLVER_SOURCES = ("cg_kernels.cuh", "spmv_policies.cuh", "device_common.cuh", "galerkin.cuh",
                  "session.cu")


def source_fingerprint(names=SOLVER_SOURCES):
    """A hash of the single-system solver's sources (csrc/): names a build of
    those kernels, so a profile captured on one build is not read as
    another's."""
    import hashlib
    h = hashlib.sha256()
    csrc = os.path.join(os.path.dirname(_HERE), "csrc")
    for name in sorted(names):
        h.update(name.encode())
        with open(os.path.join(csrc, name), "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def spmv_bytes_fp64(n, nnz):
    """Algorithmic bytes of one FP64 CSR SpMV: values + indices + row pointers + p + q."""
    return 12 * nnz + 4 * (n + 1) + 8 * n + 8 * n


def spmv_bytes_fp32(n, nnz):
    return 8 * nnz + 4 * (n + 1) + 4 * n + 4 * n


# ------------------------------------------------------------ learned preconditioner
WEIGHTS_PATH = os.path.join(_HERE, "lp_weights.f32")


class GnnGraph:
    """A matrix prepared for the network (device resident)."""

    def __init__(self, model, rowstr, colidx, a):
        self.n = int(len(rowstr) - 1)
        self._model = model
        h = ctypes.c_void_p()
        _check(lib().cgb_gnn_graph_create(model._h, self.n, np.ascontiguousarray(rowstr, np.int32),
                                          np.ascontiguousarray(colidx, np.int32),
                                          np.ascontiguousarray(a, np.float64), ctypes.byref(h)))
        self._h = h
        n_, nl = ctypes.c_int(), ctypes.c_longlong()
        self.dscale = np.zeros(self.n)
        _check(lib().cgb_gnn_graph_info(h, ctypes.byref(n_), ctypes.byref(nl), _ptr(self.dscale)))
        self.nnz_low = nl.value

    def close(self):
        if getattr(self, "_h", None):
            lib().cgb_gnn_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Gnn:
    """The learned-preconditioner network (weights on one GPU)."""

    def __init__(self, device=0, seed=20241203):
        h = ctypes.c_void_p()
        _check(lib().cgb_gnn_create(device, seed, ctypes.byref(h)))
        self._h = h
        self.n_params = int(lib().cgb_gnn_param_count())

    def close(self):
        if getattr(self, "_h", None):
            lib().cgb_gnn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self):
        out = np.zeros(self.n_params, np.float32)
        _check(lib().cgb_gnn_get_params(self._h, out, self.n_params))
        return out

    @params.setter
    def params(self, values):
        v = np.ascontiguousarray(values, np.float32)
        if v.size != self.n_params:
            raise CgbError(ERR_INVALID, f"expected {self.n_params} weights, got {v.size}")
        _check(lib().cgb_gnn_set_params(self._h, v, self.n_params))

    def save(self, path=WEIGHTS_PATH):
        self.params.astype("<f4").tofile(path)

    def load(self, path=WEIGHTS_PATH):
        self.params = np.fromfile(path, dtype="<f4")

    def graph(self, rowstr, colidx, a):
        return GnnGraph(self, rowstr, colidx, a)

    def loss_grad(self, graph, probes=None, seed=0, cg_steps=0):
        loss = ctypes.c_float()
        grad = np.zeros(self.n_params, np.float32)
        pr = None
        if probes is not None:
            pr = np.ascontiguousarray(probes, np.float32)
            if pr.shape != (graph.n, 32):
                raise CgbError(ERR_INVALID, "probes must be n x 32")
        _check(lib().cgb_gnn_loss_grad(self._h, graph._h, _ptr(pr), seed, cg_steps,
                                       ctypes.byref(loss), _ptr(grad)))
        return float(loss.value), grad

    def train_step(self, graph, seed, cg_steps=0, lr=1e-3):
        loss = ctypes.c_float()
        _check(lib().cgb_gnn_train_step(self._h, graph._h, seed, cg_steps, lr, ctypes.byref(loss)))
        return float(loss.value)

    def infer(self, graph):
        goff = np.zeros(graph.nnz_low, np.float32)
        gdiag = np.zeros(graph.n, np.float32)
        _check(lib().cgb_gnn_infer(self._h, graph._h, _ptr(goff), _ptr(gdiag)))
        return goff, gdiag

    def attach(self, graph, session):
        """Installs F = G / sqrt(delta) as the session's preconditioner."""
        _check(lib().cgb_gnn_attach(self._h, graph._h, session._h))


def strict_lower_pattern(rowstr, colidx):
    """(ptr, col) of the entries with col < row, in CSR order (the graph's order)."""
    n = len(rowstr) - 1
    rows = np.repeat(np.arange(n), np.diff(rowstr))
    keep = colidx < rows
    ptr = np.zeros(n + 1, np.int64)
    np.add.at(ptr, rows[keep] + 1, 1)
    return np.cumsum(ptr).astype(np.int32), colidx[keep].astype(np.int32)


def factor_from_g(rowstr, colidx, goff, gdiag, dscale):
    """F = G diag(dscale) as lower CSR (strict lower entries, then the diagonal)."""
    n = len(rowstr) - 1
    lptr, lcol = strict_lower_pattern(rowstr, colidx)
    cnt = np.diff(lptr) + 1
    fptr = np.zeros(n + 1, np.int64)
    fptr[1:] = np.cumsum(cnt)
    fcol = np.empty(fptr[-1], np.int32)
    fval = np.empty(fptr[-1], np.float64)
    lrows = np.repeat(np.arange(n), np.diff(lptr))
    pos = fptr[lrows] + (np.arange(len(lcol)) - lptr[lrows])
    fcol[pos] = lcol
    fval[pos] = goff.astype(np.float64) * dscale[lcol]
    fcol[fptr[1:] - 1] = np.arange(n)
    fval[fptr[1:] - 1] = gdiag.astype(np.float64) * dscale
    return fptr.astype(np.int32), fcol, fval


def identity_factor(n):
    """F = I: the preconditioned solver then is plain CG (the method without the network)."""
    return np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.ones(n)


def jacobi_factor(rowstr, colidx, a):
    """F = diag(-A)^-1/2: M = diag(-A)^-1 (Jacobi)."""
    n = len(rowstr) - 1
    rows = np.repeat(np.arange(n), np.diff(rowstr))
    d = -a[colidx == rows]
    return (np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), 1.0 / np.sqrt(d))


# ------------------------------------------------------------------------ batches
def uneven_batch_specs(nsys=512, seed=20241203, n_range=(1400, 20000), nonzer_range=(7, 13)):
    """The batched workload: per system n log-uniform in n_range, nonzer
    uniform in nonzer_range, shift = 10 + n/1000, rcond 0.1, its own odd LCG
    seed; all drawn from a fixed host PRNG.  Returns [(n, nonzer, shift, seed)]."""
    rng = np.random.RandomState(seed)
    lo, hi = np.log(n_range[0]), np.log(n_range[1])
    out = []
    for s in range(nsys):
        n = int(round(np.exp(rng.uniform(lo, hi))))
        nonzer = int(rng.randint(nonzer_range[0], nonzer_range[1] + 1))
        lcg_seed = float(2 * rng.randint(1 << 20, 1 << 40) + 1)
        out.append((n, nonzer, 10.0 + n / 1000.0, lcg_seed))
    return out


def shard_systems(weights, world):
    """Greedy split of systems over `world` ranks by weight (largest first to
    the least loaded rank); returns the system indices of each rank."""
    order = sorted(range(len(weights)), key=lambda i: -weights[i])
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += weights[i]
    return [sorted(p) for p in parts]


def batch_shard(specs, rank, world):
    """The systems (indices into `specs`, [(n, nonzer, shift, seed)]) that rank
    `rank` of `world` solves: a greedy split by the CSR size bound
    n (nonzer + 1)^2, largest first to the least loaded rank.  Independent
    systems need no exchange: each rank builds and solves its own Batch."""
    weights = [n * (nz + 1) ** 2 for n, nz, _, _ in specs]
    return shard_systems(weights, world)[rank]


def gather_shards(local, index, nsys, dist, rank):
    """Rank 0 assembles the per-system arrays of every rank's shard
    (`local`: dict of equal-length arrays for the systems `index`) into
    arrays over all `nsys` systems, plus each rank's device_ms; other ranks
    get None.  `dist` is torch.distributed (gloo or NCCL)."""
    payload = {k: np.asarray(v).tolist() for k, v in local.items() if k != "device_ms"}
    payload["index"] = list(index)
    payload["device_ms"] = float(local.get("device_ms", 0.0))
    parts = [None] * dist.get_world_size() if rank == 0 else None
    dist.gather_object(payload, parts, dst=0)
    if rank != 0:
        return None
    out = {"device_ms_per_rank": [p["device_ms"] for p in parts]}
    for key in parts[0]:
        if key in ("index", "device_ms"):
            continue
        sample = np.asarray(parts[0][key])
        arr = np.zeros(nsys, dtype=sample.dtype if sample.size else np.float64)
        for p in parts:
            arr[np.asarray(p["index"], dtype=np.int64)] = np.asarray(p[key])
        out[key] = arr
    return out


class Batch:
    """Many independent systems on one GPU (cgb_batch)."""

    def __init__(self, systems, shifts, device=0):
        """systems: [(rowstr, colidx, a)], shifts: per system."""
        self.nsys = len(systems)
        self._keep = [(np.ascontiguousarray(r, np.int32), np.ascontiguousarray(c, np.int32),
                       np.ascontiguousarray(v, np.float64)) for r, c, v in systems]
        n = np.array([len(r) - 1 for r, _, _ in self._keep], np.int32)
        P = ctypes.c_void_p * self.nsys
        rp = P(*[r.ctypes.data for r, _, _ in self._keep])
        cp = P(*[c.ctypes.data for _, c, _ in self._keep])
        ap = P(*[v.ctypes.data for _, _, v in self._keep])
        self.shifts = np.ascontiguousarray(shifts, np.float64)
        h = ctypes.c_void_p()
        _check(lib().cgb_batch_create(device, self.nsys, n, rp, cp, ap, self.shifts, ctypes.byref(h)))
        self._h = h
        self.nnz = np.array([len(v) for _, _, v in self._keep], np.int64)

    def close(self):
        if getattr(self, "_h", None):
            lib().cgb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _params(self, niter, mode, cgitmax, tol, refresh_every, recycle=4):
        P = BatchParams()
        lib().cgb_default_batch_params(ctypes.byref(P))
        P.niter, P.mode, P.cgitmax, P.tol, P.refresh_every = niter, mode, cgitmax, tol, refresh_every
        P.recycle = recycle
        return P

    def solve(self, niter=15, mode=MODE_FP64, cgitmax=25, tol=1e-12, refresh_every=10,
              recycle=4):
        """`recycle`: Galerkin start on that many previous iterates (MIXED)."""
        P = self._params(niter, mode, cgitmax, tol, refresh_every, recycle)
        z, rn = np.zeros(self.nsys), np.zeros(self.nsys)
        it, st = np.zeros(self.nsys, np.int32), np.zeros(self.nsys, np.int32)
        ms = ctypes.c_double()
        _check(lib().cgb_batch_solve(self._h, ctypes.byref(P), z, rn, it, st, ctypes.byref(ms)))
        return dict(zeta=z, rnorm=rn, iters=it, status=st, device_ms=ms.value)

    def tune(self, niter=1, mode=MODE_FP64, cgitmax=25, tol=1e-12, refresh_every=10):
        P = self._params(niter, mode, cgitmax, tol, refresh_every)
        block = ctypes.c_int()
        t = [ctypes.c_double() for _ in range(4)]
        _check(lib().cgb_batch_tune(self._h, ctypes.byref(P), ctypes.byref(block),
                                    *[ctypes.byref(x) for x in t]))
        return dict(block=block.value, thresholds=(t[0].value, t[1].value, t[2].value),
                    best_ms=t[3].value, **self.policy())

    def policy(self):
        """Entries a lane loads ahead, the team fraction, and how many systems
        the last launch solved with a team of CTAs."""
        u, f, t = ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
        _check(lib().cgb_batch_policy(self._h, ctypes.byref(u), ctypes.byref(f), ctypes.byref(t)))
        return dict(unroll=u.value, team_frac=f.value, teams=t.value)

    def set_preconditioner(self, sys, fptr, fcol, fval):
        """M = F^T F for system `sys` in the learned mode (F lower CSR with a
        positive diagonal; stored with BF16 values)."""
        _check(lib().cgb_batch_set_preconditioner(self._h, int(sys),
                                                  np.ascontiguousarray(fptr, np.int32),
                                                  np.ascontiguousarray(fcol, np.int32),
                                                  np.ascontiguousarray(fval, np.float64)))

    def attach_learned(self, model):
        """The network's factor F = G / sqrt(delta) for every system (one
        inference per system matrix)."""
        for i, (rs, ci, a) in enumerate(self._keep):
            with model.graph(rs, ci, a) as g:
                _check(lib().cgb_gnn_attach_batch(model._h, g._h, self._h, i))

    def attach_identity(self):
        """F = I for every system: the learned mode's kernel without the
        network (plain CG in the preconditioned solver)."""
        for i, (rs, _, _) in enumerate(self._keep):
            self.set_preconditioner(i, *identity_factor(len(rs) - 1))

    def fallbacks(self):
        """Per system: outer steps of the last learned solve that fell back to plain CG."""
        out = np.zeros(self.nsys, np.int32)
        _check(lib().cgb_batch_fallbacks(self._h, out))
        return out

    def set_team_frac(self, frac):
        """0: every system on one CTA; larger systems get teams of CTAs below
        their work per CTA > frac x the batch's work per resident CTA."""
        _check(lib().cgb_batch_set_team_frac(self._h, float(frac)))


NCCL_ID_BYTES = 128


def part_rows(n, world, rank):
    """Rows [row0, row1) that rank `rank` of `world` owns of an n-row matrix
    (blocks of ceil(n / world) rows)."""
    r0, r1 = ctypes.c_int(), ctypes.c_int()
    _check(lib().cgb_part_rows(int(n), int(world), int(rank), ctypes.byref(r0), ctypes.byref(r1)))
    return r0.value, r1.value


def row_block(rowstr, colidx, a, row0, row1):
    """Rows row0..row1-1 of a CSR, column indices kept global:
    (rowstr rebased to 0, colidx, a)."""
    k0, k1 = int(rowstr[row0]), int(rowstr[row1])
    rs = (np.asarray(rowstr[row0:row1 + 1], np.int64) - k0).astype(np.int32)
    return rs, np.ascontiguousarray(colidx[k0:k1], np.int32), np.ascontiguousarray(a[k0:k1], np.float64)


def _choose_nccl():
    """Point libcgb at the NCCL that torch is built against (the pip
    nvidia-nccl package), when there is one and no choice was made: a
    process can hold only one libnccl.so.2, and whichever loads first binds
    every later user, so libcgb and torch must agree."""
    if os.environ.get("CGB_NCCL_LIBRARY"):
        return
    import importlib.util
    spec = importlib.util.find_spec("nvidia")
    for base in (spec.submodule_search_locations or []) if spec else []:
        cand = os.path.join(base, "nccl", "lib", "libnccl.so.2")
        if os.path.exists(cand):
            os.environ["CGB_NCCL_LIBRARY"] = cand
            return


def nccl_unique_id():
    """A new NCCL unique id (bytes) for rank 0 to broadcast to the others."""
    _choose_nccl()
    buf = ctypes.create_string_buffer(NCCL_ID_BYTES)
    _check(lib().cgb_nccl_unique_id(buf))
    return buf.raw


def _id_buffer(nccl_id):
    if nccl_id is None:
        return None
    _choose_nccl()
    if len(nccl_id) != NCCL_ID_BYTES:
        raise CgbError(ERR_INVALID, f"nccl_id must be {NCCL_ID_BYTES} bytes")
    return ctypes.create_string_buffer(bytes(nccl_id), NCCL_ID_BYTES)


class Part:
    """One rank's row block of a system split over GPUs (cgb_part).

    `rowstr, colidx, a` are the WHOLE matrix's CSR; the rank keeps its own
    rows (part_rows).  With `nccl_id` (the same bytes on every rank) the
    constructor joins the world's NCCL communicator -- every rank must make
    it -- and power_iterate is a collective call.  Without it, a world of
    one solves alone and a larger world is driven from one process by
    group_power_iterate."""

    def __init__(self, rowstr, colidx, a, world=1, rank=0, nccl_id=None, device=0):
        self.n = int(len(rowstr) - 1)
        self.world, self.rank = int(world), int(rank)
        self.rows = part_rows(self.n, world, rank)
        self._keep = row_block(rowstr, colidx, a, *self.rows)
        h = ctypes.c_void_p()
        _check(lib().cgb_part_create(device, self.n, self.world, self.rank, *self._keep,
                                     _id_buffer(nccl_id), ctypes.byref(h)))
        self._h = h

    @classmethod
    def generated(cls, n, nonzer, shift, seed=SEED, rcond=RCOND, world=1, rank=0, nccl_id=None,
                  device=0):
        """This rank's rows of makea(n, nonzer, rcond, shift, seed), assembled
        on the device (the whole matrix is never built)."""
        self = cls.__new__(cls)
        self.n, self.world, self.rank = int(n), int(world), int(rank)
        self.rows = part_rows(n, world, rank)
        self._keep = None
        h = ctypes.c_void_p()
        _check(lib().cgb_part_create_generated(device, n, nonzer, rcond, shift, seed, self.world,
                                               self.rank, _id_buffer(nccl_id), ctypes.byref(h)))
        self._h = h
        return self

    def close(self):
        if getattr(self, "_h", None):
            lib().cgb_part_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def join(self, nccl_id):
        """Joins the world's NCCL communicator (collective: every rank, same id)."""
        _check(lib().cgb_part_join(self._h, _id_buffer(nccl_id)))

    def set_wait_limit(self, seconds):
        """Longest wait for the peers' collectives before the communicator is aborted."""
        _check(lib().cgb_part_set_wait_limit(self._h, float(seconds)))

    @property
    def nnz(self):
        """Stored entries of this rank's rows."""
        k = ctypes.c_longlong()
        _check(lib().cgb_part_info(self._h, None, None, ctypes.byref(k)))
        return k.value

    def power_iterate(self, niter, shift, cgitmax=25):
        """The reference outer loop over this world; every rank calls it."""
        z, r = np.zeros(niter), np.zeros(niter)
        ms = ctypes.c_double()
        _check(lib().cgb_part_power_iterate(self._h, niter, shift, cgitmax, _ptr(z), _ptr(r),
                                            ctypes.byref(ms)))
        return dict(zeta=z, rnorm=r, device_ms=ms.value)


def group_power_iterate(parts, niter, shift, cgitmax=25):
    """All ranks of one world (Part objects without an NCCL id, on one
    device, in rank order) solved from this process."""
    P = ctypes.c_void_p * len(parts)
    hs = P(*[p._h.value for p in parts])
    z, r = np.zeros(niter), np.zeros(niter)
    ms = ctypes.c_double()
    _check(lib().cgb_part_group_power_iterate(ctypes.cast(hs, ctypes.c_void_p), len(parts), niter,
                                              shift, cgitmax, _ptr(z), _ptr(r), ctypes.byref(ms)))
    return dict(zeta=z, rnorm=r, device_ms=ms.value)


# NPB MG classes (the reference's mg.cu main :388-410, verification norms
# :528-543): lt (grid 2^lt a side), nit, smoother set, rnm2
MG_CLASSES = {
    "S": dict(lt=5, nit=4, smoother=0, rnm2=0.5307707005734e-04),
    "W": dict(lt=7, nit=4, smoother=0, rnm2=0.6467329375339e-05),
    "A": dict(lt=8, nit=4, smoother=0, rnm2=0.2433365309069e-05),
    "B": dict(lt=8, nit=20, smoother=1, rnm2=0.1800564401355e-05),
    "C": dict(lt=9, nit=20, smoother=1, rnm2=0.5706732285740e-06),
    "D": dict(lt=10, nit=50, smoother=1, rnm2=0.1583275060440e-09),
}
MG_VERIFY_EPSILON = 1.0e-8


class Mg:
    """The NPB MG benchmark's grids on one GPU (cgb_mg): v generated on the
    device, u and r for every level of the V-cycle."""

    def __init__(self, lt, smoother, device=0):
        self.lt, self.smoother = int(lt), int(smoother)
        self.m = (1 << self.lt) + 2
        h = ctypes.c_void_p()
        _check(lib().cgb_mg_create(device, self.lt, self.smoother, ctypes.byref(h)))
        self._h = h

    @classmethod
    def for_class(cls, name, device=0):
        c = MG_CLASSES[name]
        return cls(c["lt"], c["smoother"], device)

    def close(self):
        if getattr(self, "_h", None):
            lib().cgb_mg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, nit):
        """The reference's timed region from u = 0: {rnm2, rnmu, device_ms}."""
        a, b, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(lib().cgb_mg_run(self._h, int(nit), ctypes.byref(a), ctypes.byref(b), ctypes.byref(t)))
        return dict(rnm2=a.value, rnmu=b.value, device_ms=t.value)

    def grid(self, which):
        """The finest level's 'u', 'v' or 'r' as a flat float64 array."""
        out = np.zeros(self.m ** 3)
        _check(lib().cgb_mg_read(self._h, {"u": 0, "v": 1, "r": 2}[which], out, out.size))
        return out

    def points(self):
        """zran3's (i1, i2, i3) of the +1 and -1 points, the reference's list order."""
        plus, minus = np.zeros(30, np.int32), np.zeros(30, np.int32)
        _check(lib().cgb_mg_points(self._h, plus, minus))
        return plus.reshape(10, 3), minus.reshape(10, 3)


def mg_apply(op, m, in1, in2=None, out=None, smoother=0, device=0):
    """One MG operator on host grids (0 resid, 1 psinv, 2 rprj3, 3 interp
    adding, 4 interp assigning); returns the output grid."""
    mo = m // 2 + 1 if op == 2 else 2 * m - 2 if op >= 3 else m
    res = np.zeros(mo ** 3) if out is None else np.array(out, dtype=np.float64)
    a = np.ascontiguousarray(in1, np.float64)
    b = None if in2 is None else np.ascontiguousarray(in2, np.float64)
    _check(lib().cgb_mg_apply(device, op, m, smoother, a.ctypes.data_as(ctypes.c_void_p),
                              None if b is None else b.ctypes.data_as(ctypes.c_void_p), res))
    return res


def mg_region_bytes(lt, nit):
    """Algorithmic bytes of the MG timed region (resid, norm, nit x (V-cycle,
    resid), norm): every grid an operator reads or writes, counted once per
    operator, ghost layers included; a level-k grid is (2^k + 2)^3 doubles."""
    c = {k: 8.0 * ((1 << k) + 2) ** 3 for k in range(1, lt + 1)}
    cycle = sum(c[k] + c[k - 1] for k in range(2, lt + 1))          # rprj3
    cycle += c[1] + 3 * c[1]                                          # zero, psinv
    cycle += sum(c[k - 1] + c[k] + 3 * c[k] + 3 * c[k] for k in range(2, lt))  # interp, resid, psinv
    cycle += c[lt - 1] + 2 * c[lt] + 3 * c[lt] + 3 * c[lt]            # interp (adding), resid, psinv
    cycle += 3 * c[lt]                                                # the main loop's resid
    return 3 * c[lt] + 2 * c[lt] + nit * cycle


# NPB EP classes: m (2^m pairs; setparams.cpp:826-845) and the verification
# sums (ep.cu:189-212)
EP_CLASSES = {
    "S": dict(m=24, sx=-3.247834652034740e+3, sy=-6.958407078382297e+3),
    "W": dict(m=25, sx=-2.863319731645753e+3, sy=-6.320053679109499e+3),
    "A": dict(m=28, sx=-4.295875165629892e+3, sy=-1.580732573678431e+4),
    "B": dict(m=30, sx=4.033815542441498e+4, sy=-2.660669192809235e+4),
    "C": dict(m=32, sx=4.764367927995374e+4, sy=-8.084072988043731e+4),
    "D": dict(m=36, sx=1.982481200946593e+5, sy=-1.020596636361769e+5),
    "E": dict(m=40, sx=-5.319717441530e+05, sy=-3.688834557731e+05),
}
EP_VERIFY_EPSILON = 1.0e-8


def ep_run(m, device=0):
    """NPB EP with 2^m pairs on the GPU: {sx, sy, q (10 counts), device_ms}."""
    sx, sy, ms = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    q = np.zeros(10)
    _check(lib().cgb_ep_run(device, int(m), ctypes.byref(sx), ctypes.byref(sy), q, ctypes.byref(ms)))
    return dict(sx=sx.value, sy=sy.value, q=q, device_ms=ms.value)


# NPB IS classes (is.cu:86-140): (TOTAL_KEYS_LOG_2, MAX_KEY_LOG_2)
IS_CLASSES = {"S": (16, 11), "W": (20, 16), "A": (23, 19), "B": (25, 21), "C": (27, 23), "D": (31, 27)}
IS_PASSED = 51  # 5 test keys x 10 iterations + the full check


class IntSort:
    """The NPB IS benchmark's keys on one GPU (cgb_is)."""

    def __init__(self, cls="U", total_log2=None, max_log2=None, device=0):
        if cls != "U":
            total_log2, max_log2 = IS_CLASSES[cls]
        self.cls, self.total_log2, self.max_log2 = cls, int(total_log2), int(max_log2)
        h = ctypes.c_void_p()
        _check(lib().cgb_is_create(device, cls.encode(), self.total_log2, self.max_log2, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().cgb_is_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self):
        """main's sequence: {passed (51 verifies), device_ms (the ten timed passes)}."""
        p, t = ctypes.c_longlong(), ctypes.c_double()
        _check(lib().cgb_is_run(self._h, ctypes.byref(p), ctypes.byref(t)))
        return dict(passed=p.value, device_ms=t.value)

    def read(self, which):
        """'keys', 'below' (per value: keys below it) or 'sorted'."""
        w = {"keys": 0, "below": 1, "sorted": 2}[which]
        n = 1 << (self.max_log2 if w == 1 else self.total_log2)
        out = np.zeros(n, np.uint32 if w == 1 else np.int32)
        _check(lib().cgb_is_read(self._h, w, out.ctypes.data_as(ctypes.c_void_p), n))
        return out


# NPB FT: (nx, ny, nz, niter) per class (setparams.cpp:797-803) and the
# reference's checksums (real, imaginary) per iteration (ft.cu:1655-1810)
FT_CLASSES = {"S": (64, 64, 64, 6), "W": (128, 128, 32, 6), "A": (256, 256, 128, 6),
              "B": (512, 256, 256, 20), "C": (512, 512, 512, 20), "D": (2048, 1024, 1024, 25)}
FT_VERIFY_EPSILON = 1.0e-12
FT_CHECKSUMS = {
    "S": [(5.546087004964E+02, 4.845363331978E+02), (5.546385409189E+02, 4.865304269511E+02),
          (5.546148406171E+02, 4.883910722336E+02), (5.545423607415E+02, 4.901273169046E+02),
          (5.544255039624E+02, 4.917475857993E+02), (5.542683411902E+02, 4.932597244941E+02)],
    "W": [(5.673612178944E+02, 5.293246849175E+02), (5.631436885271E+02, 5.282149986629E+02),
          (5.594024089970E+02, 5.270996558037E+02), (5.560698047020E+02, 5.260027904925E+02),
          (5.530898991250E+02, 5.249400845633E+02), (5.504159734538E+02, 5.239212247086E+02)],
    "A": [(5.046735008193E+02, 5.114047905510E+02), (5.059412319734E+02, 5.098809666433E+02),
          (5.069376896287E+02, 5.098144042213E+02), (5.077892868474E+02, 5.101336130759E+02),
          (5.085233095391E+02, 5.104914655194E+02), (5.091487099959E+02, 5.107917842803E+02)],
    "B": [(5.177643571579E+02, 5.077803458597E+02), (5.154521291263E+02, 5.088249431599E+02),
          (5.146409228649E+02, 5.096208912659E+02), (5.142378756213E+02, 5.101023387619E+02),
          (5.139626667737E+02, 5.103976610617E+02), (5.137423460082E+02, 5.105948019802E+02),
          (5.135547056878E+02, 5.107404165783E+02), (5.133910925466E+02, 5.108576573661E+02),
          (5.132470705390E+02, 5.109577278523E+02), (5.131197729984E+02, 5.110460304483E+02),
          (5.130070319283E+02, 5.111252433800E+02), (5.129070537032E+02, 5.111968077718E+02),
          (5.128182883502E+02, 5.112616233064E+02), (5.127393733383E+02, 5.113203605551E+02),
          (5.126691062020E+02, 5.113735928093E+02), (5.126064276004E+02, 5.114218460548E+02),
          (5.125504076570E+02, 5.114656139760E+02), (5.125002331720E+02, 5.115053595966E+02),
          (5.124551951846E+02, 5.115415130407E+02), (5.124146770029E+02, 5.115744692211E+02)],
    "C": [(5.195078707457E+02, 5.149019699238E+02), (5.155422171134E+02, 5.127578201997E+02),
          (5.144678022222E+02, 5.122251847514E+02), (5.140150594328E+02, 5.121090289018E+02),
          (5.137550426810E+02, 5.121143685824E+02), (5.135811056728E+02, 5.121496764568E+02),
          (5.134569343165E+02, 5.121870921893E+02), (5.133651975661E+02, 5.122193250322E+02),
          (5.132955192805E+02, 5.122454735794E+02), (5.132410471738E+02, 5.122663649603E+02),
          (5.131971141679E+02, 5.122830879827E+02), (5.131605205716E+02, 5.122965869718E+02),
          (5.131290734194E+02, 5.123075927445E+02), (5.131012720314E+02, 5.123166486553E+02),
          (5.130760908195E+02, 5.123241541685E+02), (5.130528295923E+02, 5.123304037599E+02),
          (5.130310107773E+02, 5.123356167976E+02), (5.130103090133E+02, 5.123399592211E+02),
          (5.129905029333E+02, 5.123435588985E+02), (5.129714421109E+02, 5.123465164008E+02)],
    "D": [(5.122230065252E+02, 5.118534037109E+02), (5.120463975765E+02, 5.117061181082E+02),
          (5.119865766760E+02, 5.117096364601E+02), (5.119518799488E+02, 5.117373863950E+02),
          (5.119269088223E+02, 5.117680347632E+02), (5.119082416858E+02, 5.117967875532E+02),
          (5.118943814638E+02, 5.118225281841E+02), (5.118842385057E+02, 5.118451629348E+02),
          (5.118769435632E+02, 5.118649119387E+02), (5.118718203448E+02, 5.118820803844E+02),
          (5.118683569061E+02, 5.118969781011E+02), (5.118661708593E+02, 5.119098918835E+02),
          (5.118649768950E+02, 5.119210777066E+02), (5.118645605626E+02, 5.119307604484E+02),
          (5.118647586618E+02, 5.119391362671E+02), (5.118654451572E+02, 5.119463757241E+02),
          (5.118665212451E+02, 5.119526269238E+02), (5.118679083821E+02, 5.119580184108E+02),
          (5.118695433664E+02, 5.119626617538E+02), (5.118713748264E+02, 5.119666538138E+02),
          (5.118733606701E+02, 5.119700787219E+02), (5.118754661974E+02, 5.119730095953E+02),
          (5.118776626738E+02, 5.119755100241E+02), (5.118799262314E+02, 5.119776353561E+02),
          (5.118822370068E+02, 5.119794338060E+02)],
}


def ft_verify(cls, sums):
    """The largest relative error of a run's checksums against the class's
    (ft.cu:1811-1822: |(sum - ref) / ref| per iteration)."""
    ref = FT_CHECKSUMS[cls]
    return max(abs(complex(*s) - complex(*r)) / abs(complex(*r)) for s, r in zip(sums, ref))


class Ft:
    """The NPB FT benchmark's arrays on one GPU (cgb_ft)."""

    def __init__(self, nx, ny, nz, device=0):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        h = ctypes.c_void_p()
        _check(lib().cgb_ft_create(device, self.nx, self.ny, self.nz, ctypes.byref(h)))
        self._h = h

    @classmethod
    def for_class(cls, name, device=0):
        nx, ny, nz, _ = FT_CLASSES[name]
        return cls(nx, ny, nz, device)

    def close(self):
        if getattr(self, "_h", None):
            lib().cgb_ft_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, niter):
        """main's timed region: {sums: [(re, im)] * niter, device_ms}."""
        sums = np.zeros(2 * niter)
        t = ctypes.c_double()
        _check(lib().cgb_ft_run(self._h, int(niter), sums, ctypes.byref(t)))
        return dict(sums=[(sums[2 * i], sums[2 * i + 1]) for i in range(niter)], device_ms=t.value)

    def read(self, which):
        """'u0' or 'u1' (complex, shape (nz, ny, nx)) or 'twiddle' (float, same shape)."""
        w = {"u0": 0, "u1": 1, "twiddle": 2}[which]
        nt = self.nx * self.ny * self.nz
        out = np.zeros(nt if w == 2 else 2 * nt)
        _check(lib().cgb_ft_read(self._h, w, out, out.size))
        if w == 2:
            return out.reshape(self.nz, self.ny, self.nx)
        return out.view(np.complex128).reshape(self.nz, self.ny, self.nx)
