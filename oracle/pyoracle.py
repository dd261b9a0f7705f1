"""ctypes view of the CPU oracle library (TEST INFRASTRUCTURE ONLY).

Loaded only by tests/, by ``__graft_entry__.smoke()`` and by bench.py's
CPU-baseline leg, always as the checker.  The product never imports this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libfsoracle.so")
_lib = None

VEC = {"Un": 0, "Unp1": 1, "Unp1_prev": 2, "UnpHalf": 3, "UnpHalf_prev": 4, "Acc": 5, "Acc_prev": 6,
       "Pn": 7, "Pnp1": 8, "Pnp1_prev": 9, "Pdot": 10, "Md": 11, "MdOrig": 12, "MdInv": 13,
       "MdOrigInv": 14, "KtimesAcc_prev": 15, "R1": 16, "R2": 17, "R3": 18}


def build(force: bool = False) -> str:
    if force or not os.path.exists(_LIB_PATH) or \
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "fs_oracle.cpp")):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, ip, dp, lp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_long)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.c_char_p, C.c_int, C.c_int, ip]
        L.orc_destroy.argtypes = [vp]
        L.orc_sizes.argtypes = [vp, lp]
        L.orc_params.argtypes = [vp, dp]
        L.orc_set_cg.argtypes = [vp, C.c_double, C.c_int, C.c_int]
        L.orc_set_print.argtypes = [vp, C.c_int]
        L.orc_set_maxiter.argtypes = [vp, C.c_int]
        L.orc_get_ltog.argtypes = [vp, ip]
        L.orc_get_coord.argtypes = [vp, dp]
        L.orc_get_bcnodes.argtypes = [vp, ip]
        L.orc_get_colors.argtypes = [vp, ip]
        L.orc_get_basis.argtypes = [vp, dp, dp, dp, dp, dp, dp]
        L.orc_get_detj.argtypes = [vp, dp]
        L.orc_get_slotmaps.argtypes = [vp, ip, ip]
        L.orc_step0.argtypes = [vp]
        L.orc_get_pattern.argtypes = [vp, C.c_int, ip, ip]
        L.orc_get_values.argtypes = [vp, C.c_int, dp]
        L.orc_get_vec.restype = C.c_long
        L.orc_get_vec.argtypes = [vp, C.c_int, dp]
        L.orc_set_vec.restype = C.c_long
        L.orc_set_vec.argtypes = [vp, C.c_int, dp]
        L.orc_begin_step.argtypes = [vp]
        L.orc_convect.argtypes = [vp, dp]
        L.orc_step1.argtypes = [vp, C.c_int]
        L.orc_step2.argtypes = [vp, C.c_int, dp]
        L.orc_step3.argtypes = [vp, C.c_int]
        L.orc_check_iter.restype = C.c_int
        L.orc_check_iter.argtypes = [vp, dp]
        L.orc_rotate.argtypes = [vp]
        L.orc_end_step.restype = C.c_int
        L.orc_end_step.argtypes = [vp, dp]
        L.orc_cg.argtypes = [vp, dp, dp, dp]
        L.orc_run.restype = C.c_int
        L.orc_run.argtypes = [vp, C.c_int, dp]
        L.orc_time.argtypes = [vp, ip, dp]
        L.orc_logs.argtypes = [vp, lp, ip, dp, C.c_int]
        L.orc_write_tecplot.restype = C.c_int
        L.orc_write_tecplot.argtypes = [vp, C.c_char_p, C.c_char_p]
        L.orc_read_restart.restype = C.c_int
        L.orc_read_restart.argtypes = [vp, C.c_char_p]
        L.orc_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Oracle:
    """One oracle solver instance built from an ``.inp`` deck."""

    def __init__(self, inp_path: str, ngp: int = 0, threads: int = 0):
        L = lib()
        rc = C.c_int(0)
        self.h = L.orc_create(inp_path.encode(), ngp, threads, C.byref(rc))
        if not self.h:
            raise RuntimeError(f"oracle setup failed for {inp_path}: rc={rc.value}")
        self.L = L
        self._refresh_sizes()

    def _refresh_sizes(self):
        s = np.zeros(13, dtype=np.int64)
        self.L.orc_sizes(self.h, _p(s, C.c_long))
        (self.NE, self.NCN, self.NN, self.NNp, self.nnzK, self.nnzG, self.nnzZ, self.nbc, self.mon,
         self.zero_p, self.NGP, self.max_iter, self.ncolors) = [int(x) for x in s]
        pr = np.zeros(7)
        self.L.orc_params(self.h, _p(pr, C.c_double))
        (self.dt, self.t_ini, self.t_final, self.tol, self.converge, self.density, self.viscosity) = pr.tolist()

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- setup products ----
    def ltog(self):
        a = np.zeros(self.NE * 27, dtype=np.int32)
        self.L.orc_get_ltog(self.h, _p(a, C.c_int))
        return a.reshape(self.NE, 27)

    def coord(self):
        a = np.zeros(self.NN * 3)
        self.L.orc_get_coord(self.h, _p(a, C.c_double))
        return a.reshape(self.NN, 3)

    def bcnodes(self):
        a = np.zeros(self.nbc * 2, dtype=np.int32)
        self.L.orc_get_bcnodes(self.h, _p(a, C.c_int))
        return a.reshape(self.nbc, 2)

    def colors(self):
        a = np.zeros(self.NE, dtype=np.int32)
        self.L.orc_get_colors(self.h, _p(a, C.c_int))
        return a

    def basis(self):
        n = self.NGP
        gqp, gqw = np.zeros(n * 3), np.zeros(n)
        sv, dsv, sp, dsp = np.zeros(n * 27), np.zeros(3 * 27 * n), np.zeros(n * 8), np.zeros(3 * 8 * n)
        self.L.orc_get_basis(self.h, *[_p(a, C.c_double) for a in (gqp, gqw, sv, dsv, sp, dsp)])
        return dict(gqp=gqp.reshape(n, 3), gqw=gqw, Sv=sv.reshape(n, 27), dSv=dsv.reshape(3, 27, n),
                    Sp=sp.reshape(n, 8), dSp=dsp.reshape(3, 8, n))

    def detj(self):
        a = np.zeros(self.NE * self.NGP)
        self.L.orc_get_detj(self.h, _p(a, C.c_double))
        return a.reshape(self.NE, self.NGP)

    def slotmaps(self):
        m = np.zeros(self.NE * 729, dtype=np.int32)
        g = np.zeros(self.NE * 216, dtype=np.int32)
        self.L.orc_get_slotmaps(self.h, _p(m, C.c_int), _p(g, C.c_int))
        return m.reshape(self.NE, 27, 27), g.reshape(self.NE, 27, 8)

    def step0(self):
        self.L.orc_step0(self.h)
        self._refresh_sizes()

    def pattern(self, which: str):
        w = {"K": 0, "G": 1, "Z": 2}[which]
        nrows = self.NNp if which == "Z" else self.NN
        nnz = {"K": self.nnzK, "G": self.nnzG, "Z": self.nnzZ}[which]
        rs = np.zeros(nrows + 1, dtype=np.int32)
        col = np.zeros(nnz, dtype=np.int32)
        self.L.orc_get_pattern(self.h, w, _p(rs, C.c_int), _p(col, C.c_int))
        return rs, col

    def values(self, which: str):
        w = {"K": 0, "G1": 1, "G2": 2, "G3": 3, "Z": 4}[which]
        nnz = {"K": self.nnzK, "Z": self.nnzZ}.get(which, self.nnzG)
        a = np.zeros(nnz)
        self.L.orc_get_values(self.h, w, _p(a, C.c_double))
        return a

    def csr(self, which: str):
        """scipy CSR of K, G1, G2, G3 or Z."""
        import scipy.sparse as sp
        pat = "G" if which.startswith("G") else which
        rs, col = self.pattern(pat)
        ncols = self.NNp if pat in ("G", "Z") else self.NN
        return sp.csr_matrix((self.values(which), col, rs), shape=(len(rs) - 1, ncols))

    # ---- state ----
    def vec(self, name: str):
        n = self.L.orc_get_vec(self.h, VEC[name], None)
        a = np.zeros(n)
        self.L.orc_get_vec(self.h, VEC[name], _p(a, C.c_double))
        return a

    def set_vec(self, name: str, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.L.orc_set_vec(self.h, VEC[name], _p(a, C.c_double))

    def set_cg(self, rtol=1e-8, maxit=1000, warm=0):
        self.L.orc_set_cg(self.h, rtol, maxit, warm)

    def set_print(self, on=True):
        self.L.orc_set_print(self.h, 1 if on else 0)

    def set_maxiter(self, m):
        self.L.orc_set_maxiter(self.h, m)

    # ---- stages ----
    def begin_step(self):
        self.L.orc_begin_step(self.h)

    def convect(self):
        r = np.zeros(3 * self.NN)
        self.L.orc_convect(self.h, _p(r, C.c_double))
        return r

    def step1(self, it):
        self.L.orc_step1(self.h, it)

    def step2(self, it):
        st = np.zeros(3)
        self.L.orc_step2(self.h, it, _p(st, C.c_double))
        return st

    def step3(self, it):
        self.L.orc_step3(self.h, it)

    def check_iter(self):
        nr = np.zeros(2)
        c = self.L.orc_check_iter(self.h, _p(nr, C.c_double))
        return bool(c), nr

    def rotate(self):
        self.L.orc_rotate(self.h)

    def end_step(self):
        m = C.c_double(0)
        s = self.L.orc_end_step(self.h, C.byref(m))
        return bool(s), m.value

    def cg(self, b, x0=None):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.NNp) if x0 is None else np.array(x0, dtype=np.float64)
        st = np.zeros(3)
        self.L.orc_cg(self.h, _p(b, C.c_double), _p(x, C.c_double), _p(st, C.c_double))
        return x, st

    def run(self, nsteps: int = -1):
        info = np.zeros(5)
        self.L.orc_run(self.h, nsteps, _p(info, C.c_double))
        return dict(steps=int(info[0]), cg_its=int(info[1]), subits=int(info[2]), steady=bool(info[3]),
                    max_acc=float(info[4]))

    def logs(self, clear: bool = False):
        """(CG iterations of every pressure solve, monitor rows per time
        step [timeN, iter, timeT, u, v, w, p, maxAcc]) since the last clear."""
        n = np.zeros(2, dtype=np.int64)
        self.L.orc_logs(self.h, _p(n, C.c_long), None, None, 0)
        cg = np.zeros(int(n[0]), dtype=np.int32)
        mon = np.zeros((int(n[1]), 8))
        self.L.orc_logs(self.h, None, _p(cg, C.c_int), _p(mon, C.c_double), 1 if clear else 0)
        return cg, mon

    def time(self):
        n, t = C.c_int(0), C.c_double(0)
        self.L.orc_time(self.h, C.byref(n), C.byref(t))
        return n.value, t.value

    def write_tecplot(self, path: str, title: str):
        return self.L.orc_write_tecplot(self.h, path.encode(), title.encode())

    def read_restart(self, path: str):
        return self.L.orc_read_restart(self.h, path.encode())


def threads() -> int:
    return int(lib().orc_threads())
