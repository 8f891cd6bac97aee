"""ctypes handle on the CPU oracle (oracle/liboracle.so) and the reference
libraries (oracle/_ref/libref_<class>.so).  Test infrastructure only."""
import ctypes
import os

import numpy as np

I32 = np.ctypeslib.ndpointer(np.int32, flags="C")
F64 = np.ctypeslib.ndpointer(np.float64, flags="C")


class Oracle:
    def __init__(self, path):
        lib = ctypes.CDLL(path)
        lib.orc_randlc.restype = ctypes.c_double
        lib.orc_randlc.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_double]
        lib.orc_nz_bound.restype = ctypes.c_longlong
        lib.orc_nz_bound.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.orc_makea.restype = ctypes.c_int
        lib.orc_makea.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, I32, I32, F64, ctypes.c_longlong,
                                  ctypes.POINTER(ctypes.c_longlong)]
        lib.orc_csr_hash.restype = ctypes.c_uint64
        lib.orc_csr_hash.argtypes = [ctypes.c_int, I32, I32, F64]
        lib.orc_spmv.restype = None
        lib.orc_spmv.argtypes = [ctypes.c_int, I32, I32, F64, F64, F64]
        lib.orc_conj_grad.restype = None
        lib.orc_conj_grad.argtypes = [ctypes.c_int, I32, I32, F64, F64, F64, F64, F64, F64,
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        lib.orc_power_iterate.restype = ctypes.c_int
        lib.orc_power_iterate.argtypes = [ctypes.c_int, I32, I32, F64, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.POINTER(ctypes.c_double)]
        lib.orc_max_threads.restype = ctypes.c_int
        # MG (mg_oracle.c)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.orc_mg_run.restype = ctypes.c_int
        lib.orc_mg_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp,
                                   ctypes.c_void_p, ctypes.c_void_p, dp]
        lib.orc_mg_zran3.restype = None
        lib.orc_mg_zran3.argtypes = [ctypes.c_int, F64, ctypes.c_void_p, ctypes.c_void_p]
        lib.orc_mg_resid.restype = None
        lib.orc_mg_resid.argtypes = [ctypes.c_int, F64, F64, F64, F64]
        lib.orc_mg_psinv.restype = None
        lib.orc_mg_psinv.argtypes = [ctypes.c_int, F64, F64, F64]
        lib.orc_mg_rprj3.restype = None
        lib.orc_mg_rprj3.argtypes = [ctypes.c_int, F64, ctypes.c_int, F64]
        lib.orc_mg_interp.restype = None
        lib.orc_mg_interp.argtypes = [ctypes.c_int, F64, ctypes.c_int, F64]
        I64 = np.ctypeslib.ndpointer(np.int64, flags="C")
        lib.orc_is_keys.restype = ctypes.c_int
        lib.orc_is_keys.argtypes = [ctypes.c_int, ctypes.c_int, I32]
        lib.orc_is_run.restype = ctypes.c_longlong
        lib.orc_is_run.argtypes = [ctypes.c_char, ctypes.c_int, ctypes.c_int, I64, I64, ctypes.c_void_p]
        lib.orc_ep_run.restype = ctypes.c_int
        lib.orc_ep_run.argtypes = [ctypes.c_int, dp, dp, F64, dp]
        lib.orc_mg_norm2u3.restype = None
        lib.orc_mg_norm2u3.argtypes = [ctypes.c_int, F64, dp, dp]
        lib.orc_ft_run.restype = ctypes.c_int
        lib.orc_ft_run.argtypes = [ctypes.c_int] * 4 + [F64, ctypes.c_void_p]
        lib.orc_ft_fft3d.restype = None
        lib.orc_ft_fft3d.argtypes = [ctypes.c_int] * 4 + [F64]
        lib.orc_ft_initial.restype = None
        lib.orc_ft_initial.argtypes = [ctypes.c_int] * 3 + [F64]
        lib.orc_ft_indexmap.restype = None
        lib.orc_ft_indexmap.argtypes = [ctypes.c_int] * 3 + [F64]
        self.lib = lib

    # ---- MG: grids are float64 cubes of side m, index (i3 * m + i2) * m + i1
    MG_A = np.array([-8.0 / 3.0, 0.0, 1.0 / 6.0, 1.0 / 12.0])
    MG_C = (np.array([-3.0 / 8.0, 1.0 / 32.0, -1.0 / 64.0, 0.0]),
            np.array([-3.0 / 17.0, 1.0 / 33.0, -1.0 / 61.0, 0.0]))

    def mg_run(self, lt, nit, smoother, grids=False):
        m = (1 << lt) + 2
        a, b, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        u = np.zeros(m ** 3) if grids else None
        r = np.zeros(m ** 3) if grids else None
        rc = self.lib.orc_mg_run(lt, nit, smoother, ctypes.byref(a), ctypes.byref(b),
                                 None if u is None else u.ctypes.data,
                                 None if r is None else r.ctypes.data, ctypes.byref(t))
        if rc != 0:
            raise RuntimeError(f"orc_mg_run failed: {rc}")
        out = dict(rnm2=a.value, rnmu=b.value, seconds=t.value)
        if grids:
            out.update(u=u, r=r)
        return out

    def mg_zran3(self, m):
        v = np.zeros(m ** 3)
        plus, minus = np.zeros(30, np.int32), np.zeros(30, np.int32)
        self.lib.orc_mg_zran3(m, v, plus.ctypes.data, minus.ctypes.data)
        return v, plus.reshape(10, 3), minus.reshape(10, 3)

    def mg_resid(self, m, u, v):
        r = np.zeros(m ** 3)
        self.lib.orc_mg_resid(m, np.ascontiguousarray(u), np.ascontiguousarray(v), r, self.MG_A)
        return r

    def mg_psinv(self, m, r, u, smoother):
        u = np.array(u, dtype=np.float64)
        self.lib.orc_mg_psinv(m, np.ascontiguousarray(r), u, self.MG_C[smoother])
        return u

    def mg_rprj3(self, mk, r):
        mj = mk // 2 + 1
        s = np.zeros(mj ** 3)
        self.lib.orc_mg_rprj3(mk, np.ascontiguousarray(r), mj, s)
        return s

    def mg_interp(self, mj, z, u):
        mk = 2 * mj - 2
        u = np.array(u, dtype=np.float64)
        self.lib.orc_mg_interp(mj, np.ascontiguousarray(z), mk, u)
        return u

    def is_keys(self, total_log2, max_log2):
        keys = np.zeros(1 << total_log2, np.int32)
        self.lib.orc_is_keys(total_log2, max_log2, keys)
        return keys

    def is_run(self, cls, total_log2, max_log2, test_index, test_rank, counts=False):
        """NPB IS (is_oracle.c): the passed count (51 verifies) and, with
        counts, the last iteration's running sums of the key counts."""
        c = np.zeros(1 << max_log2, np.int64) if counts else None
        passed = self.lib.orc_is_run(cls.encode(), total_log2, max_log2,
                                     np.ascontiguousarray(test_index, np.int64),
                                     np.ascontiguousarray(test_rank, np.int64),
                                     None if c is None else c.ctypes.data)
        return (passed, c) if counts else passed

    def ep_run(self, m):
        """NPB EP with 2^m pairs (ep_oracle.c): {sx, sy, q, seconds}."""
        sx, sy, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        q = np.zeros(10)
        rc = self.lib.orc_ep_run(m, ctypes.byref(sx), ctypes.byref(sy), q, ctypes.byref(t))
        if rc != 0:
            raise RuntimeError(f"orc_ep_run failed: {rc}")
        return dict(sx=sx.value, sy=sy.value, q=q, seconds=t.value)

    # ---- FT: fields are complex arrays of shape (nz, ny, nx)
    def ft_run(self, nx, ny, nz, niter, field=False):
        """NPB FT (ft_oracle.c): the checksums [(re, im)] * niter and, with
        field, the last inverse transform u1."""
        sums = np.zeros(2 * niter)
        u1 = np.zeros(2 * nx * ny * nz) if field else None
        rc = self.lib.orc_ft_run(nx, ny, nz, niter, sums, None if u1 is None else u1.ctypes.data)
        if rc != 0:
            raise RuntimeError("orc_ft_run: out of memory")
        out = [(sums[2 * i], sums[2 * i + 1]) for i in range(niter)]
        return (out, u1.view(np.complex128).reshape(nz, ny, nx)) if field else out

    def ft_fft3d(self, direction, a):
        """The reference's 3-D transform of a complex (nz, ny, nx) array."""
        nz, ny, nx = a.shape
        buf = np.ascontiguousarray(a, np.complex128).view(np.float64).ravel().copy()
        self.lib.orc_ft_fft3d(direction, nx, ny, nz, buf)
        return buf.view(np.complex128).reshape(nz, ny, nx)

    def ft_initial(self, nx, ny, nz):
        buf = np.zeros(2 * nx * ny * nz)
        self.lib.orc_ft_initial(nx, ny, nz, buf)
        return buf.view(np.complex128).reshape(nz, ny, nx)

    def ft_indexmap(self, nx, ny, nz):
        buf = np.zeros(nx * ny * nz)
        self.lib.orc_ft_indexmap(nx, ny, nz, buf)
        return buf.reshape(nz, ny, nx)

    def mg_norm(self, m, r):
        a, b = ctypes.c_double(), ctypes.c_double()
        self.lib.orc_mg_norm2u3(m, np.ascontiguousarray(r), ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def makea(self, n, nonzer, rcond, shift, seed=314159265.0):
        cap = self.lib.orc_nz_bound(n, nonzer)
        rs = np.zeros(n + 1, np.int32)
        ci = np.zeros(cap, np.int32)
        a = np.zeros(cap)
        nnz = ctypes.c_longlong()
        rc = self.lib.orc_makea(n, nonzer, rcond, shift, seed, rs, ci, a, cap, ctypes.byref(nnz))
        if rc != 0:
            raise RuntimeError(f"orc_makea failed: {rc}")
        k = nnz.value
        return rs, ci[:k].copy(), a[:k].copy()

    def csr_hash(self, rowstr, colidx, a):
        n = len(rowstr) - 1
        return "%016x" % self.lib.orc_csr_hash(n, np.ascontiguousarray(rowstr, np.int32),
                                                np.ascontiguousarray(colidx, np.int32),
                                                np.ascontiguousarray(a, np.float64))

    def spmv(self, rowstr, colidx, a, x):
        n = len(rowstr) - 1
        y = np.zeros(n)
        self.lib.orc_spmv(n, rowstr, colidx, a, np.ascontiguousarray(x, np.float64), y)
        return y

    def conj_grad(self, rowstr, colidx, a, x, cgitmax=25):
        n = len(rowstr) - 1
        xv = np.ones(n + 2)
        xv[:n] = x[:n]
        z, p, q, r = (np.zeros(n + 2) for _ in range(4))
        rn = ctypes.c_double()
        self.lib.orc_conj_grad(n, rowstr, colidx, a, xv, z, p, q, r, cgitmax, ctypes.byref(rn))
        return z[: n + 1], p[: n + 1], q[: n + 1], r[: n + 1], rn.value

    def power_iterate(self, rowstr, colidx, a, shift, niter, cgitmax=25, threads=1):
        n = len(rowstr) - 1
        zt, rt, x = np.zeros(niter), np.zeros(niter), np.zeros(n)
        secs = ctypes.c_double()
        rc = self.lib.orc_power_iterate(n, rowstr, colidx, a, shift, niter, cgitmax, threads,
                                        zt.ctypes.data, rt.ctypes.data, x.ctypes.data,
                                        ctypes.byref(secs))
        if rc != 0:
            raise RuntimeError(f"orc_power_iterate failed: {rc}")
        return dict(zeta=zt, rnorm=rt, x=x, seconds=secs.value)


class RefLib:
    """The reference's own CG code for one NPB class (oracle/_ref)."""

    def __init__(self, path):
        lib = ctypes.CDLL(path)
        lib.ref_info.argtypes = [ctypes.POINTER(ctypes.c_int)] * 3 + [
            ctypes.POINTER(ctypes.c_double)] * 2 + [ctypes.POINTER(ctypes.c_longlong)]
        lib.ref_makea.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p]
        lib.ref_makea.restype = ctypes.c_int
        lib.ref_power.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_power.restype = ctypes.c_double
        lib.ref_power_gpu.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_power_gpu.restype = ctypes.c_double
        lib.ref_set_matrix.argtypes = [ctypes.c_void_p] * 3
        lib.ref_set_matrix.restype = ctypes.c_int
        lib.ref_conj_grad.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_void_p]
        lib.ref_conj_grad.restype = ctypes.c_int
        na, nz, ni = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        sh, rc, bound = ctypes.c_double(), ctypes.c_double(), ctypes.c_longlong()
        lib.ref_info(ctypes.byref(na), ctypes.byref(nz), ctypes.byref(ni), ctypes.byref(sh),
                     ctypes.byref(rc), ctypes.byref(bound))
        self.n, self.nonzer, self.niter = na.value, nz.value, ni.value
        self.shift, self.rcond, self.nz_bound = sh.value, rc.value, bound.value
        self.lib = lib

    def makea(self, seed=314159265.0, copy_out=True):
        if not copy_out:
            return self.lib.ref_makea(seed, None, None, None)
        rs = np.zeros(self.n + 1, np.int32)
        ci = np.zeros(self.nz_bound, np.int32)
        a = np.zeros(self.nz_bound)
        nnz = self.lib.ref_makea(seed, rs.ctypes.data, ci.ctypes.data, a.ctypes.data)
        return rs, ci[:nnz].copy(), a[:nnz].copy()

    def power(self, niter):
        zt, rt = np.zeros(niter), np.zeros(niter)
        secs = self.lib.ref_power(niter, zt.ctypes.data, rt.ctypes.data)
        return dict(zeta=zt, rnorm=rt, seconds=secs)

    def set_matrix(self, rowstr, colidx, a):
        """Loads a CSR into the reference's arrays (in place of makea)."""
        rs = np.ascontiguousarray(rowstr, np.int32)
        ci = np.ascontiguousarray(colidx, np.int32)
        av = np.ascontiguousarray(a, np.float64)
        nnz = self.lib.ref_set_matrix(rs.ctypes.data, ci.ctypes.data, av.ctypes.data)
        if nnz < 0:
            raise ValueError("matrix larger than the reference's NZ")
        return nnz

    def power_gpu(self, niter):
        """The reference's own GPU loop (conj_grad_gpu, cg.cu:803-846) on
        the last generated matrix: traces and the loop's wall seconds."""
        zt, rt = np.zeros(niter), np.zeros(niter)
        secs = self.lib.ref_power_gpu(niter, zt.ctypes.data, rt.ctypes.data)
        return dict(zeta=zt, rnorm=rt, seconds=secs)

    def conj_grad(self, x):
        n = self.n
        z, r, p, q = (np.zeros(n) for _ in range(4))
        rn = np.zeros(1)
        self.lib.ref_conj_grad(np.ascontiguousarray(x, np.float64).ctypes.data, z.ctypes.data,
                               r.ctypes.data, p.ctypes.data, q.ctypes.data, rn.ctypes.data)
        return z, p, q, r, float(rn[0])


class RefMgLib:
    """The reference's own MG code for one NPB class (oracle/_ref/libref_mg_<class>.so)."""

    def __init__(self, path):
        lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        lib.ref_mg_info.restype = None
        lib.ref_mg_info.argtypes = [ip, ip]
        lib.ref_mg_cpu.restype = ctypes.c_int
        lib.ref_mg_cpu.argtypes = [dp, dp, dp, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_mg_gpu.restype = ctypes.c_int
        lib.ref_mg_gpu.argtypes = [dp, dp, dp]
        self.lib = lib
        lt, nit = ctypes.c_int(), ctypes.c_int()
        lib.ref_mg_info(ctypes.byref(lt), ctypes.byref(nit))
        self.lt, self.nit = lt.value, nit.value
        self.m = (1 << self.lt) + 2

    def cpu(self, grids=False):
        a, b, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        u = np.zeros(self.m ** 3) if grids else None
        r = np.zeros(self.m ** 3) if grids else None
        self.lib.ref_mg_cpu(ctypes.byref(a), ctypes.byref(b), ctypes.byref(t),
                            None if u is None else u.ctypes.data, None if r is None else r.ctypes.data)
        out = dict(rnm2=a.value, rnmu=b.value, seconds=t.value)
        if grids:
            out.update(u=u, r=r)
        return out

    def gpu(self):
        a, b, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        rc = self.lib.ref_mg_gpu(ctypes.byref(a), ctypes.byref(b), ctypes.byref(t))
        if rc != 0:
            raise RuntimeError("ref_mg_gpu failed")
        return dict(rnm2=a.value, rnmu=b.value, seconds=t.value)


class RefEpLib:
    """The reference's own EP GPU code for one NPB class (oracle/_ref/libref_ep_<class>.so)."""

    def __init__(self, path):
        lib = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.ref_ep_m.restype = ctypes.c_int
        lib.ref_ep_gpu.restype = ctypes.c_int
        lib.ref_ep_gpu.argtypes = [dp, dp, F64, dp, dp]
        self.lib = lib
        self.m = lib.ref_ep_m()

    def gpu(self):
        sx, sy, tl, tw = (ctypes.c_double() for _ in range(4))
        q = np.zeros(10)
        rc = self.lib.ref_ep_gpu(ctypes.byref(sx), ctypes.byref(sy), q, ctypes.byref(tl), ctypes.byref(tw))
        if rc != 0:
            raise RuntimeError("ref_ep_gpu failed")
        return dict(sx=sx.value, sy=sy.value, q=q, seconds_launch=tl.value, seconds_wall=tw.value)


class RefIsLib:
    """The reference's own IS GPU code for one NPB class (oracle/_ref/libref_is_<class>.so)."""

    def __init__(self, path):
        lib = ctypes.CDLL(path)
        lib.ref_is_gpu.restype = ctypes.c_longlong
        lib.ref_is_gpu.argtypes = [ctypes.POINTER(ctypes.c_double)]
        self.lib = lib

    def gpu(self):
        """main's sequence: {passed (51 verifies), seconds (the ten timed passes, wall)}."""
        t = ctypes.c_double()
        passed = self.lib.ref_is_gpu(ctypes.byref(t))
        return dict(passed=int(passed), seconds=t.value)


class RefFtLib:
    """The reference's own FT GPU code for one NPB class (oracle/_ref/libref_ft_<class>.so)."""

    def __init__(self, path):
        lib = ctypes.CDLL(path)
        lib.ref_ft_niter.restype = ctypes.c_int
        lib.ref_ft_gpu.restype = ctypes.c_int
        lib.ref_ft_gpu.argtypes = [F64, ctypes.POINTER(ctypes.c_double)]
        self.lib = lib
        self.niter = lib.ref_ft_niter()

    def gpu(self):
        """main's sequence: {sums: [(re, im)] * niter, seconds (the timed region, wall)}."""
        sums = np.zeros(2 * self.niter)
        t = ctypes.c_double()
        if self.lib.ref_ft_gpu(sums, ctypes.byref(t)) != self.niter:
            raise RuntimeError("ref_ft_gpu failed")
        return dict(sums=[(sums[2 * i], sums[2 * i + 1]) for i in range(self.niter)], seconds=t.value)
