"""Python binding of libcfdfs (the B200 fractional-step solver's C ABI).

The solver itself is C++ host code plus sm_100a CUDA kernels inside
``lib/libcfdfs.so``; this module only declares the C prototypes (ctypes) and
offers a ``Solver`` class whose methods carry the names of the reference's
device seam (fractionalStep/Cpp/blascoCodinaHuerta.cpp:365-377):
``selectCUDAdevice``, ``initializeAndAllocateGPU``, ``calculateZ_CUSP``,
``calculateMatrixAGPU``, ``step1GPUpart``, ``step2GPU``, ``step3GPU``,
``calculate_KtimesAcc_prevGPU``, ``checkConvergenceGPU``,
``checkConvergenceInTimeGPU`` and ``printMonitorDataGPU``.  Where the
reference prints "ErrorNN" and waits on std::cin, these raise ``CfdError``.

There is no CPU fallback: if the library cannot be loaded, or no GPU is
present, construction fails.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(_PKG_DIR)
LIB_PATH = os.path.join(ROOT, "lib", "libcfdfs.so")
HEADER = os.path.join(os.path.dirname(ROOT), "include", "cfdfs.h")

CFD_OK, CFD_E_CUDA, CFD_E_NOCONV, CFD_E_NONFINITE, CFD_E_TIMEOUT, CFD_E_BADARG, CFD_E_BADINPUT, CFD_E_IO, \
    CFD_E_NOMEM = 0, -1, -2, -3, -4, -5, -6, -7, -8
FP64, MIXED = 0, 1
PC_JACOBI, PC_LEARNED, PC_TWOLEVEL = 0, 1, 2

VEC = dict(Un=0, Unp1=1, Unp1_prev=2, UnpHalf=3, UnpHalf_prev=4, Acc=5, Acc_prev=6, Pn=7, Pnp1=8,
           Pnp1_prev=9, Pdot=10, MdInv=11, MdOrigInv=12, KtimesAcc_prev=13, R1=14, R2=15, R3=16, DIV=17)
PRESSURE_SIZED = {"Pn", "Pnp1", "Pnp1_prev", "Pdot", "R2", "DIV"}
MAT = dict(K=0, G=1, GT=2, Z=3)


class CfdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cfdfs error {code}: {msg}")
        self.code = code


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("precond", C.c_int), ("cg_rtol", C.c_double), ("cg_maxit", C.c_int),
                ("cg_warm", C.c_int), ("ngp_override", C.c_int), ("inner_rtol", C.c_double),
                ("max_outer", C.c_int), ("fcg_m", C.c_int), ("fcg_net_iters", C.c_int),
                ("deterministic", C.c_int)]


class ProblemInfo(C.Structure):
    _fields_ = [("NE", C.c_int), ("NCN", C.c_int), ("NN", C.c_int), ("NNp", C.c_int), ("NGP", C.c_int),
                ("maxIter", C.c_int), ("nnzK", C.c_longlong), ("nnzG", C.c_longlong), ("nnzZ", C.c_longlong),
                ("nBCnodes", C.c_int), ("monPoint", C.c_int), ("zeroPressureNode", C.c_int),
                ("dt", C.c_double), ("t_ini", C.c_double), ("t_final", C.c_double), ("tolerance", C.c_double),
                ("convergence", C.c_double), ("density", C.c_double), ("viscosity", C.c_double),
                ("timeN", C.c_int), ("timeT", C.c_double)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("outer", C.c_int), ("relres", C.c_double), ("status", C.c_int),
                ("fallback", C.c_int)]


class RunStats(C.Structure):
    _fields_ = [("steps", C.c_int), ("subiters", C.c_longlong), ("cg_iters", C.c_longlong), ("steady", C.c_int),
                ("maxAcc", C.c_double), ("last_iter", C.c_int), ("fallbacks", C.c_int)]


_lib = None
_vp, _ip, _dp, _cp, _llp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_char_p, C.POINTER(C.c_longlong)
_fp = C.POINTER(C.c_float)

_PROTOS = {
    "cfd_abi_version": (C.c_int, []),
    "cfd_default_options": (None, [C.POINTER(Options)]),
    "cfd_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "cfd_destroy": (None, [_vp]),
    "cfd_last_error": (C.c_char_p, [_vp]),
    "cfd_set_options": (C.c_int, [_vp, C.POINTER(Options)]),
    "cfd_load_inp": (C.c_int, [_vp, _cp]),
    "cfd_load_mesh": (C.c_int, [_vp, C.POINTER(ProblemInfo), _dp, _ip, C.c_int, _dp, C.c_int, _ip, _dp]),
    "cfd_info": (C.c_int, [_vp, C.POINTER(ProblemInfo)]),
    "cfd_step0": (C.c_int, [_vp]),
    "cfd_begin_step": (C.c_int, [_vp]),
    "cfd_convect": (C.c_int, [_vp]),
    "cfd_step1": (C.c_int, [_vp, C.c_int]),
    "cfd_step2": (C.c_int, [_vp, C.c_int, C.POINTER(SolveStats)]),
    "cfd_step3": (C.c_int, [_vp, C.c_int]),
    "cfd_check_iter": (C.c_int, [_vp, C.c_double, _ip, _dp]),
    "cfd_rotate": (C.c_int, [_vp]),
    "cfd_k_times_acc": (C.c_int, [_vp]),
    "cfd_check_steady": (C.c_int, [_vp, C.c_double, _dp, _ip]),
    "cfd_end_step": (C.c_int, [_vp]),
    "cfd_run": (C.c_int, [_vp, C.c_int, C.POINTER(RunStats)]),
    "cfd_get_monitor": (C.c_int, [_vp, C.c_int, _dp]),
    "cfd_download_state": (C.c_int, [_vp, _dp, _dp]),
    "cfd_upload_state": (C.c_int, [_vp, _dp, _dp]),
    "cfd_download_vector": (C.c_int, [_vp, C.c_int, _dp]),
    "cfd_download_matrix": (C.c_int, [_vp, C.c_int, _llp, _ip, _ip, _dp]),
    "cfd_pressure_solve": (C.c_int, [_vp, _dp, _dp, C.POINTER(SolveStats)]),
    "cfd_write_tecplot": (C.c_int, [_vp, _cp, _cp]),
    "cfd_read_restart": (C.c_int, [_vp, _cp]),
    "cfd_set_bc_values": (C.c_int, [_vp, C.c_int, _ip, _dp]),
    "cfd_unet_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_ulonglong]),
    "cfd_unet_destroy": (None, [_vp]),
    "cfd_unet_last_error": (C.c_char_p, [_vp]),
    "cfd_unet_param_count": (C.c_longlong, []),
    "cfd_unet_get_params": (C.c_int, [_vp, _fp, C.c_longlong]),
    "cfd_unet_set_params": (C.c_int, [_vp, _fp, C.c_longlong]),
    "cfd_unet_save": (C.c_int, [_vp, _cp]),
    "cfd_unet_read": (C.c_int, [_vp, _cp]),
    "cfd_unet_forward": (C.c_int, [_vp, _ip, _vp, _vp, C.c_int]),
    "cfd_unet_gradient": (C.c_int, [_vp, _ip, _vp, _vp, C.c_int, _fp, _fp]),
    "cfd_unet_train_batch": (C.c_int, [_vp, _ip, C.c_int, _vp, _vp, C.c_int, C.c_float, _fp]),
    "cfd_unet_set_loss": (C.c_int, [_vp, C.c_float, C.c_float]),
    "cfd_unet_tensor": (C.c_int, [_vp, C.c_int, _fp, C.c_longlong]),
    "cfd_unet_set_tensor_cores": (C.c_int, [_vp, C.c_int]),
    "cfd_unet_status": (C.c_int, [_vp]),
    "cfd_unet_attach": (C.c_int, [_vp, _vp, _ip, _ip]),
    "cfd_unet_load": (C.c_int, [_vp, _cp, _ip]),
    "cfd_pressure_residual": (C.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "cfd_set_pressure_grid": (C.c_int, [_vp, _ip, _ip]),
    "cfd_precond_apply": (C.c_int, [_vp, _dp, _dp]),
    "cfd_stream": (C.c_void_p, [_vp]),
    "cfd_launch_count": (C.c_longlong, [_vp]),
    "cfd_profile": (C.c_int, [_vp, C.c_int]),
    "cfd_profile_read": (C.c_int, [_vp, _dp]),
    "cfd_profile_fcg2l": (C.c_int, [_vp, _dp]),
    "cfd_spd_inverse": (C.c_int, [C.c_int, _dp, C.c_int, _dp]),
    "cfd_coarse_matrix": (C.c_int, [C.c_int, _ip, _ip, _ip, _dp, C.c_double, _ip, _dp]),
    "cfd_selftest_wait_timeout": (C.c_int, [_vp, C.c_int]),
    "cfd_pcg_solve_noalloc": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, C.c_int, C.c_double, C.c_int, _vp, _dp,
                                        C.c_char_p, C.c_int]),
    "cfdh_load": (C.c_int, [C.POINTER(C.c_void_p), _cp, C.c_char_p, C.c_int]),
    "cfdh_free": (None, [_vp]),
    "cfdh_sizes": (C.c_int, [_vp, _llp]),
    "cfdh_get_ltog": (C.c_int, [_vp, _ip]),
    "cfdh_get_coord": (C.c_int, [_vp, _dp]),
    "cfdh_get_bcnodes": (C.c_int, [_vp, _ip]),
    "cfdh_get_pattern": (C.c_int, [_vp, C.c_int, _ip, _ip]),
    "cfdh_write_tecplot": (C.c_int, [_vp, _dp, _dp, _cp, _cp]),
    "cfdh_coarse_inverse": (C.c_int, [_ip, _ip, _ip, _dp, _ip, _dp]),
    "cfdh_coarse_matrix": (C.c_int, [_ip, _ip, _ip, _dp, C.c_double, _ip, _dp]),
    "cfdh_element_colors": (C.c_int, [_vp, _ip, _ip]),
}


def header_functions(path: str = HEADER) -> list[str]:
    """Names of every function the public header declares."""
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cfdh?_[a-z0-9_]+)\s*\(", txt)))


def lib():
    """Loads libcfdfs.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CfdError(CFD_E_CUDA, f"{LIB_PATH} is missing; build it with __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def default_options() -> Options:
    o = Options()
    lib().cfd_default_options(C.byref(o))
    return o


class HostMesh:
    """Deck + preprocessing on the host only (no GPU): cfdh_* entry points."""

    def __init__(self, path: str):
        L = lib()
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = L.cfdh_load(C.byref(h), path.encode(), err, 512)
        if rc != CFD_OK:
            raise CfdError(rc, err.value.decode())
        self.h, self.L = h, L
        s = np.zeros(12, dtype=np.int64)
        L.cfdh_sizes(h, _p(s, C.c_longlong))
        (self.NE, self.NCN, self.NN, self.NNp, self.nnzK, self.nnzG, self.nnzZ, self.nbc, self.mon, self.zero_p,
         self.NGP, self.max_iter) = [int(x) for x in s]

    def close(self):
        if getattr(self, "h", None):
            self.L.cfdh_free(self.h)
            self.h = None

    __del__ = close

    def ltog(self):
        a = np.zeros(self.NE * 27, dtype=np.int32)
        self.L.cfdh_get_ltog(self.h, _p(a, C.c_int))
        return a.reshape(self.NE, 27)

    def coord(self):
        a = np.zeros(self.NN * 3)
        self.L.cfdh_get_coord(self.h, _p(a, C.c_double))
        return a.reshape(self.NN, 3)

    def bcnodes(self):
        a = np.zeros(self.nbc * 2, dtype=np.int32)
        self.L.cfdh_get_bcnodes(self.h, _p(a, C.c_int))
        return a.reshape(self.nbc, 2)

    def pattern(self, which: str):
        w = {"K": 0, "G": 1, "GT": 2, "Z": 3}[which]
        nrows = self.NNp if which in ("GT", "Z") else self.NN
        nnz = {"K": self.nnzK, "G": self.nnzG, "GT": self.nnzG, "Z": self.nnzZ}[which]
        rp = np.zeros(nrows + 1, dtype=np.int32)
        col = np.zeros(nnz, dtype=np.int32)
        self.L.cfdh_get_pattern(self.h, w, _p(rp, C.c_int), _p(col, C.c_int))
        return rp, col

    def element_colors(self):
        """(order, off): the deterministic mode's element colouring, colour c
        owning order[off[c]:off[c+1]]."""
        nc = self.L.cfdh_element_colors(self.h, None, None)
        if nc < 0:
            raise CfdError(nc, "more than 64 element colours")
        order = np.zeros(self.NE, dtype=np.int32)
        off = np.zeros(nc + 1, dtype=np.int32)
        self.L.cfdh_element_colors(self.h, _p(order, C.c_int), _p(off, C.c_int))
        return order, off

    def write_tecplot(self, U, P, path: str, title: str):
        U = np.ascontiguousarray(U, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        rc = self.L.cfdh_write_tecplot(self.h, _p(U, C.c_double), _p(P, C.c_double), path.encode(), title.encode())
        if rc != CFD_OK:
            raise CfdError(rc, "tecplot write failed")


class Solver:
    """One GPU solver context (cfd_ctx)."""

    def __init__(self, device: int = 0, precision: int = FP64, cg_rtol: float = 1e-8, cg_maxit: int = 1000,
                 cg_warm: int = 0, ngp: int = 0, inner_rtol: float = 1e-4, max_outer: int = 12,
                 precond: int = PC_JACOBI, fcg_m: int = 4, fcg_net_iters: int = 0, deterministic: int = 0):
        L = lib()
        h = C.c_void_p()
        rc = L.cfd_create(C.byref(h), device)
        if rc != CFD_OK:
            raise CfdError(rc, "cfd_create failed (no usable CUDA device?)")
        self.h, self.L = h, L
        o = default_options()
        o.precision, o.precond, o.cg_rtol, o.cg_maxit, o.cg_warm = precision, precond, cg_rtol, cg_maxit, cg_warm
        o.ngp_override, o.inner_rtol, o.max_outer, o.fcg_m = ngp, inner_rtol, max_outer, fcg_m
        o.fcg_net_iters, o.deterministic = fcg_net_iters, deterministic
        self._check(L.cfd_set_options(h, C.byref(o)))
        self.opts = o
        self.info = None
        self._unet = None

    def set_options(self, **kw):
        """Changes options of a live context (precision and ngp only before
        load): precond, cg_rtol, cg_maxit, cg_warm, inner_rtol, max_outer, fcg_m,
        fcg_net_iters, deterministic."""
        o = Options()
        C.memmove(C.byref(o), C.byref(self.opts), C.sizeof(Options))
        for k, v in kw.items():
            if k == "ngp":
                k = "ngp_override"
            setattr(o, k, v)
        self._check(self.L.cfd_set_options(self.h, C.byref(o)))
        self.opts = o

    # ---- plumbing ----
    def _check(self, rc: int):
        if rc != CFD_OK:
            raise CfdError(rc, self.L.cfd_last_error(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.cfd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def refresh(self) -> ProblemInfo:
        i = ProblemInfo()
        self._check(self.L.cfd_info(self.h, C.byref(i)))
        self.info = i
        return i

    # ---- set-up ----
    def load(self, path: str):
        """readInputFile + preprocessing + initializeAndAllocateGPU."""
        self._check(self.L.cfd_load_inp(self.h, path.encode()))
        return self.refresh()

    def step0(self):
        """step0 + calculateZ_CUSP on the device."""
        self._check(self.L.cfd_step0(self.h))

    # ---- reference-named stage calls ----
    def begin_step(self):
        self._check(self.L.cfd_begin_step(self.h))

    def calculateMatrixAGPU(self):
        self._check(self.L.cfd_convect(self.h))

    def step1GPUpart(self, it: int):
        self._check(self.L.cfd_step1(self.h, it))

    def step2GPU(self, it: int) -> SolveStats:
        st = SolveStats()
        self._check(self.L.cfd_step2(self.h, it, C.byref(st)))
        return st

    def step3GPU(self, it: int):
        self._check(self.L.cfd_step3(self.h, it))

    def checkConvergenceGPU(self, tol: float | None = None):
        tol = self.refresh().tolerance if tol is None else tol
        conv = C.c_int(0)
        norms = np.zeros(2)
        self._check(self.L.cfd_check_iter(self.h, tol, C.byref(conv), _p(norms, C.c_double)))
        return bool(conv.value), norms

    def rotate(self):
        self._check(self.L.cfd_rotate(self.h))

    def calculate_KtimesAcc_prevGPU(self):
        self._check(self.L.cfd_k_times_acc(self.h))

    def checkConvergenceInTimeGPU(self, crit: float | None = None):
        crit = self.refresh().convergence if crit is None else crit
        m, s = C.c_double(0), C.c_int(0)
        self._check(self.L.cfd_check_steady(self.h, crit, C.byref(m), C.byref(s)))
        return bool(s.value), m.value

    def end_step(self):
        self._check(self.L.cfd_end_step(self.h))

    def printMonitorDataGPU(self, it: int) -> str:
        i = self.refresh()
        m = self.monitor()
        return "%6d  %6d  %10.5f  %12.5f  %12.5f  %12.5f  %12.5f" % (i.timeN, it, i.timeT, m[0], m[1], m[2], m[3])

    # aliases with the reference's set-up names
    def initializeAndAllocateGPU(self, path: str):
        return self.load(path)

    def calculateZ_CUSP(self):
        return self.step0()

    def run(self, nsteps: int = -1) -> RunStats:
        st = RunStats()
        self._check(self.L.cfd_run(self.h, nsteps, C.byref(st)))
        return st

    def time_step(self, after_step2=None):
        """One time step through the stage calls (timeLoop body);
        ``after_step2(it)`` is called after each pressure solve."""
        i = self.refresh()
        self.begin_step()
        cg = []
        it = 1
        while it <= i.maxIter:
            self.calculateMatrixAGPU()
            self.step1GPUpart(it)
            cg.append(self.step2GPU(it).iterations)
            if after_step2 is not None:
                after_step2(it)
            self.step3GPU(it)
            conv, _ = self.checkConvergenceGPU(i.tolerance)
            if conv:
                break
            self.rotate()
            self.calculate_KtimesAcc_prevGPU()
            it += 1
        steady, max_acc = self.checkConvergenceInTimeGPU(i.convergence)
        self.end_step()
        return dict(iter=it, cg=cg, steady=steady, max_acc=max_acc)

    # ---- state ----
    def monitor(self, node: int = -1):
        out = np.zeros(4)
        self._check(self.L.cfd_get_monitor(self.h, node, _p(out, C.c_double)))
        return out

    def state(self, out=None):
        """(U, P) in the reference layout; out = (U, P) writes into the
        caller's arrays (e.g. pinned host buffers) instead of new ones."""
        i = self.info or self.refresh()
        if out is None:
            U, P = np.zeros(3 * i.NN), np.zeros(i.NNp)
        else:
            U, P = out
            assert U.dtype == np.float64 and P.dtype == np.float64 and U.flags.c_contiguous and P.flags.c_contiguous
            assert U.size == 3 * i.NN and P.size == i.NNp
        self._check(self.L.cfd_download_state(self.h, _p(U, C.c_double), _p(P, C.c_double)))
        return U, P

    def set_state(self, U, P):
        U = np.ascontiguousarray(U, dtype=np.float64)
        P = np.ascontiguousarray(P, dtype=np.float64)
        self._check(self.L.cfd_upload_state(self.h, _p(U, C.c_double), _p(P, C.c_double)))

    def vector(self, name: str):
        i = self.info or self.refresh()
        n = i.NNp if name in PRESSURE_SIZED else 3 * i.NN
        out = np.zeros(n)
        self._check(self.L.cfd_download_vector(self.h, VEC[name], _p(out, C.c_double)))
        return out

    def matrix(self, which: str):
        """(rowptr, col, val); val is (nnz, 3) for G and GT."""
        w = MAT[which]
        i = self.info or self.refresh()
        nnz = C.c_longlong(0)
        self._check(self.L.cfd_download_matrix(self.h, w, C.byref(nnz), None, None, None))
        nrows = i.NNp if which in ("GT", "Z") else i.NN
        rp = np.zeros(nrows + 1, dtype=np.int32)
        col = np.zeros(nnz.value, dtype=np.int32)
        nv = 3 if which in ("G", "GT") else 1
        val = np.zeros(nnz.value * nv)
        self._check(self.L.cfd_download_matrix(self.h, w, C.byref(nnz), _p(rp, C.c_int), _p(col, C.c_int),
                                               _p(val, C.c_double)))
        return rp, col, (val.reshape(-1, 3) if nv == 3 else val)

    def pressure_solve(self, rhs, x0=None):
        i = self.info or self.refresh()
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros(i.NNp) if x0 is None else np.array(x0, dtype=np.float64)
        st = SolveStats()
        rc = self.L.cfd_pressure_solve(self.h, _p(rhs, C.c_double), _p(x, C.c_double), C.byref(st))
        if rc not in (CFD_OK, CFD_E_NOCONV):
            self._check(rc)
        return x, st

    def pressure_residual(self, rhs, x):
        """r = rhs - Z x in FP64 on the device; returns (r, ||r||)."""
        i = self.info or self.refresh()
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.ascontiguousarray(x, dtype=np.float64)
        r = np.zeros(i.NNp)
        nrm = C.c_double()
        self._check(self.L.cfd_pressure_residual(self.h, _p(rhs, C.c_double), _p(x, C.c_double),
                                                 _p(r, C.c_double), C.byref(nrm)))
        return r, nrm.value

    # ---- preconditioners ----
    def set_pressure_grid(self, dims, p_of_vox=None):
        """Structured grid of the pressure nodes for the coarse space and the
        network (dims = (nx, ny, nz); p_of_vox: pressure node of each voxel)."""
        d = np.ascontiguousarray(dims, dtype=np.int32)
        pm = None if p_of_vox is None else np.ascontiguousarray(p_of_vox, dtype=np.int32)
        self._check(self.L.cfd_set_pressure_grid(self.h, _p(d, C.c_int), None if pm is None else _p(pm, C.c_int)))

    def precond_apply(self, r):
        """Linear part of the configured preconditioner applied to r (FP64)."""
        i = self.info or self.refresh()
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros(i.NNp)
        self._check(self.L.cfd_precond_apply(self.h, _p(r, C.c_double), _p(z, C.c_double)))
        return z

    def attach_unet(self, net, dims=None, p_of_vox=None):
        """Use ``net`` (a ``UNet``) as the learned preconditioner on the
        pressure grid ``dims`` (default: a cube); None detaches."""
        if net is None:
            self._check(self.L.cfd_unet_attach(self.h, None, None, None))
            self._unet = None
            return
        i = self.info or self.refresh()
        if dims is None:
            m = round(i.NNp ** (1 / 3))
            dims = (m, m, m)
        d = np.ascontiguousarray(dims, dtype=np.int32)
        pm = None if p_of_vox is None else np.ascontiguousarray(p_of_vox, dtype=np.int32)
        self._check(self.L.cfd_unet_attach(self.h, net.h, _p(d, C.c_int), None if pm is None else _p(pm, C.c_int)))
        self._unet = net  # keep it alive while attached

    def load_unet(self, path: str, dims=None):
        d = None if dims is None else np.ascontiguousarray(dims, dtype=np.int32)
        self._check(self.L.cfd_unet_load(self.h, path.encode(), None if d is None else _p(d, C.c_int)))

    # ---- timing / counters ----
    KCLASS = ["convect", "step1", "gt", "pcg64", "pcg32", "resid64", "step3", "spmv_k3", "pupdate", "other",
              "unet", "fcg", "coarse", "spmv_z", "fcg2l"]

    @property
    def stream_ptr(self) -> int:
        return int(self.L.cfd_stream(self.h) or 0)

    def launch_count(self) -> int:
        return int(self.L.cfd_launch_count(self.h))

    def profile(self, on: bool):
        self._check(self.L.cfd_profile(self.h, 1 if on else 0))

    def profile_read(self) -> dict:
        out = np.zeros(3 * len(self.KCLASS))
        self._check(self.L.cfd_profile_read(self.h, _p(out, C.c_double)))
        return {k: dict(launches=int(out[3 * i]), ms=float(out[3 * i + 1]), iters=int(out[3 * i + 2]))
                for i, k in enumerate(self.KCLASS)}


    FCG2L_PHASES = ["restrict", "coarse", "zphase", "nbwait", "spmv", "dotwait", "update", "spmv_block_min",
                    "spmv_block_mean", "spmv_block_max"]

    def profile_fcg2l(self) -> dict:
        """Phase times (ms, first block, summed) of the persistent two-level
        iteration while profiling was on."""
        out = np.zeros(10)
        self._check(self.L.cfd_profile_fcg2l(self.h, _p(out, C.c_double)))
        return dict(zip(self.FCG2L_PHASES, out.tolist()))
    def selftest_wait_timeout(self, ms: int) -> int:
        return int(self.L.cfd_selftest_wait_timeout(self.h, ms))

    def write_tecplot(self, path: str, title: str):
        self._check(self.L.cfd_write_tecplot(self.h, path.encode(), title.encode()))

    def read_restart(self, path: str):
        self._check(self.L.cfd_read_restart(self.h, path.encode()))

    def set_bc_values(self, nodes, uvw):
        nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        uvw = np.ascontiguousarray(uvw, dtype=np.float64)
        self._check(self.L.cfd_set_bc_values(self.h, len(nodes), _p(nodes, C.c_int), _p(uvw, C.c_double)))


class UNet:
    """The learned pressure preconditioner's network (cfd_unet): a 3-level 3D
    conv U-Net with BF16 weights / activations and FP32 accumulation, trained
    by the library's own forward and backward kernels."""

    def __init__(self, device: int = -1, seed: int = 0, path: str | None = None):
        L = lib()
        h = C.c_void_p()
        rc = L.cfd_unet_create(C.byref(h), device, seed)
        if rc != CFD_OK:
            raise CfdError(rc, "cfd_unet_create failed (no usable CUDA device?)")
        self.h, self.L = h, L
        self.nparam = int(L.cfd_unet_param_count())
        if path:
            self.read(path)

    def _check(self, rc: int):
        if rc != CFD_OK:
            raise CfdError(rc, self.L.cfd_unet_last_error(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.cfd_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def param_count() -> int:
        return int(lib().cfd_unet_param_count())

    def params(self) -> np.ndarray:
        out = np.zeros(self.nparam, dtype=np.float32)
        self._check(self.L.cfd_unet_get_params(self.h, _p(out, C.c_float), self.nparam))
        return out

    def set_params(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(self.L.cfd_unet_set_params(self.h, _p(w, C.c_float), len(w)))

    def save(self, path: str):
        self._check(self.L.cfd_unet_save(self.h, path.encode()))

    def read(self, path: str):
        self._check(self.L.cfd_unet_read(self.h, path.encode()))

    def set_tensor_cores(self, on: bool):
        """Forward convolutions on tcgen05 tensor cores (default) or CUDA cores."""
        self._check(self.L.cfd_unet_set_tensor_cores(self.h, 1 if on else 0))

    def status(self):
        """Raises if a bounded wait in a tensor-core launch gave up."""
        self._check(self.L.cfd_unet_status(self.h))

    def set_loss(self, w_l2: float = 1.0, w_h1: float = 0.0):
        """Training loss weights (mean squared error, neighbour-difference term)."""
        self._check(self.L.cfd_unet_set_loss(self.h, w_l2, w_h1))

    @staticmethod
    def _dims(dims):
        return np.ascontiguousarray(dims, dtype=np.int32)

    def forward(self, x, dims=None):
        """f(x) for one grid; x is a (nz, ny, nx) float array (host)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        d = self._dims(dims if dims is not None else x.shape[::-1])
        y = np.zeros_like(x)
        self._check(self.L.cfd_unet_forward(self.h, _p(d, C.c_int), x.ctypes.data, y.ctypes.data, 0))
        return y

    TENSOR_CH = (1, 16, 32, 32, 64, 64, 64, 32, 32, 32, 16, 16, 16, 1)
    TENSOR_LEVEL = (0, 0, 1, 1, 2, 2, 2, 2, 1, 1, 1, 0, 0, 0)

    def tensor(self, t: int, dims):
        """Stored tensor t of the last forward pass on grid dims, shaped
        (nz, ny, nx, ch) at its level."""
        d = [int(v) for v in dims]
        for _ in range(self.TENSOR_LEVEL[t]):
            d = [(v - 1) // 2 + 1 for v in d]
        n = d[0] * d[1] * d[2] * self.TENSOR_CH[t]
        out = np.zeros(n, dtype=np.float32)
        self._check(self.L.cfd_unet_tensor(self.h, t, _p(out, C.c_float), n))
        return out.reshape(d[2], d[1], d[0], self.TENSOR_CH[t])

    def forward_device(self, x_ptr: int, y_ptr: int, dims):
        d = self._dims(dims)
        self._check(self.L.cfd_unet_forward(self.h, _p(d, C.c_int), x_ptr, y_ptr, 1))

    def gradient(self, x, t, dims=None):
        """(loss, dloss/dparams) of one host sample."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        d = self._dims(dims if dims is not None else x.shape[::-1])
        g = np.zeros(self.nparam, dtype=np.float32)
        loss = C.c_float()
        self._check(self.L.cfd_unet_gradient(self.h, _p(d, C.c_int), x.ctypes.data, t.ctypes.data, 0,
                                             C.byref(loss), _p(g, C.c_float)))
        return float(loss.value), g

    def train_batch(self, x, t, dims, lr: float, on_device: bool = False, nb: int | None = None) -> float:
        """One Adam step on nb samples.  Host arrays (nb, nz, ny, nx), or with
        on_device=True integer device addresses of nb consecutive grids."""
        d = self._dims(dims)
        loss = C.c_float()
        if on_device:
            self._check(self.L.cfd_unet_train_batch(self.h, _p(d, C.c_int), int(nb), x, t, 1, lr, C.byref(loss)))
        else:
            x = np.ascontiguousarray(x, dtype=np.float32)
            t = np.ascontiguousarray(t, dtype=np.float32)
            self._check(self.L.cfd_unet_train_batch(self.h, _p(d, C.c_int), x.shape[0], x.ctypes.data,
                                                    t.ctypes.data, 0, lr, C.byref(loss)))
        return float(loss.value)


def coarse_inverse(dims, rowptr, col, val):
    """Host-only coarse space of the two-level preconditioner for the CSR
    matrix Z on the grid dims: (coarse nodes per axis, inverse of P^T Z P)."""
    L = lib()
    d = np.ascontiguousarray(dims, dtype=np.int32)
    rp = np.ascontiguousarray(rowptr, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    vl = np.ascontiguousarray(val, dtype=np.float64)
    cd = np.zeros(3, dtype=np.int32)
    rc = L.cfdh_coarse_inverse(_p(d, C.c_int), _p(rp, C.c_int), _p(cl, C.c_int), _p(vl, C.c_double),
                               _p(cd, C.c_int), None)
    if rc != CFD_OK:
        raise CfdError(rc, "cfdh_coarse_inverse: bad arguments")
    nc = int(np.prod(cd))
    inv = np.zeros((nc, nc))
    rc = L.cfdh_coarse_inverse(_p(d, C.c_int), _p(rp, C.c_int), _p(cl, C.c_int), _p(vl, C.c_double),
                               _p(cd, C.c_int), _p(inv, C.c_double))
    if rc != CFD_OK:
        raise CfdError(rc, "cfdh_coarse_inverse: the coarse matrix is not positive definite")
    return tuple(int(v) for v in cd), inv


def coarse_matrix(dims, rowptr, col, val, spacing: float = 4.0, device=None):
    """Galerkin coarse matrix P^T Z P of the two-level preconditioner for the
    CSR matrix Z on the grid dims, dense: (coarse nodes per axis, Zc).  Built
    on the host, or on the given device (the solver's build, bit-identical
    to the host's)."""
    L = lib()
    d = np.ascontiguousarray(dims, dtype=np.int32)
    rp = np.ascontiguousarray(rowptr, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    vl = np.ascontiguousarray(val, dtype=np.float64)
    cd = np.zeros(3, dtype=np.int32)

    def call(out):
        ptr = None if out is None else _p(out, C.c_double)
        if device is None:
            return L.cfdh_coarse_matrix(_p(d, C.c_int), _p(rp, C.c_int), _p(cl, C.c_int), _p(vl, C.c_double),
                                        float(spacing), _p(cd, C.c_int), ptr)
        return L.cfd_coarse_matrix(int(device), _p(d, C.c_int), _p(rp, C.c_int), _p(cl, C.c_int),
                                   _p(vl, C.c_double), float(spacing), _p(cd, C.c_int), ptr)

    rc = call(None)
    if rc != CFD_OK:
        raise CfdError(rc, "coarse_matrix: bad arguments")
    nc = int(np.prod(cd))
    zc = np.zeros((nc, nc))
    rc = call(zc)
    if rc != CFD_OK:
        raise CfdError(rc, "coarse_matrix: a row of Z reaches more than 3 coarse nodes per axis"
                       if rc == CFD_E_BADINPUT else "coarse_matrix failed")
    return tuple(int(v) for v in cd), zc


NOALLOC_MAX_N = 524288


def spd_inverse(a, device: int = 0):
    """Inverse of a dense SPD matrix, factored and inverted on the device."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    inv = np.zeros_like(a)
    rc = lib().cfd_spd_inverse(device, _p(a, C.c_double), a.shape[0], _p(inv, C.c_double))
    if rc != CFD_OK:
        raise CfdError(rc, "cfd_spd_inverse failed")
    return inv


def pcg_solve_noalloc(rowptr, col, val, dinv, b, x, n, rtol=1e-8, maxit=1000, stream=0):
    """cfd_pcg_solve_noalloc on caller-owned device buffers (integer device
    addresses).  Returns (status, info[3], message)."""
    info = np.zeros(3)
    err = C.create_string_buffer(256)
    rc = lib().cfd_pcg_solve_noalloc(rowptr, col, val, dinv, b, x, n, rtol, maxit, stream or None,
                                     _p(info, C.c_double), err, 256)
    return rc, info, err.value.decode()


def selectCUDAdevice(device: int = -1) -> Solver:
    """selectCUDAdevice (CUDAcodes.cu:126-154): a solver on the given device
    (-1 = the last one, as the reference)."""
    return Solver(device=device)
