"""ctypes binding of oracle/libnsxref.so (the C restatement of the reference;
test infrastructure and host-core baseline only)."""
import ctypes as C
import os
import numpy as np

from .build_ref import build, LIB

_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_void_p]
        L.ref_dim.restype = C.c_int64
        L.ref_dim.argtypes = [C.c_void_p]
        L.ref_nthreads.restype = C.c_int
        L.ref_nthreads.argtypes = [C.c_void_p]
        L.ref_matvec.restype = None
        L.ref_matvec.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.ref_lanczos.restype = C.c_double
        L.ref_lanczos.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ref_solve.restype = C.c_double
        L.ref_solve.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint64,
                                C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.ref_destroy.restype = None
        L.ref_destroy.argtypes = [C.c_void_p]
        _lib = L
    return _lib


class RefSolver:
    """The reference algorithm (FP32 storage, axpy order, OpenMP) on a generated problem."""

    def __init__(self, P, variant=None):
        """variant: optional (op_vals, a_seg_vals, b_seg_vals) of an interaction variant in the
        order of P's operator keys and segments (InteractionFamily.arrays), used instead of
        P's own interaction."""
        from nushellx_b200.nsx import build_problem_struct
        self._prob, self._keep = build_problem_struct(P)
        if variant is not None:
            op, av, bv = (np.ascontiguousarray(v, dtype=np.float64) for v in variant)
            assert len(op) == self._prob.nop
            self._keep.append((op, av, bv))
            self._prob.op_vals = op.ctypes.data_as(C.POINTER(C.c_double))
            self._prob.a.seg_vals = av.ctypes.data_as(C.POINTER(C.c_double))
            self._prob.b.seg_vals = bv.ctypes.data_as(C.POINTER(C.c_double))
        self._h = lib().ref_create(C.byref(self._prob))
        self.dim = int(lib().ref_dim(self._h))
        self.threads = int(lib().ref_nthreads(self._h))

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty_like(x)
        lib().ref_matvec(self._h, x.ctypes.data_as(C.POINTER(C.c_float)), y.ctypes.data_as(C.POINTER(C.c_float)))
        return y

    def lanczos(self, npre, nsteps, seed=5):
        """(seconds of the steps, seconds of the pre-iterations, seconds of the steps spent in
        Gram-Schmidt against the stored vectors, alpha, beta)."""
        a = np.zeros(max(nsteps, 1))
        b = np.zeros(max(nsteps, 1))
        pre = C.c_double(0)
        cgs = C.c_double(0)
        t = lib().ref_lanczos(self._h, npre, nsteps, seed, a.ctypes.data_as(C.POINTER(C.c_double)),
                              b.ctypes.data_as(C.POINTER(C.c_double)), C.byref(pre), C.byref(cgs))
        return t, pre.value, cgs.value, a[:nsteps], b[:nsteps]

    def solve(self, nlev=10, npre=2, first_iter=90, inc_iter=3, noiter=300, level_limit=5e-4, seed=5):
        """A complete solve by the reference's standard Lanczos and its own stopping rule
        (src/NuLnz/NuCoreX.f90:595-751; parameters from src/NuCommon/NuCommon.f90:101-124 and
        src/NuCommonX/NuCommonX.f90:23-27).  Returns (lowest nlev Ritz values, steps, seconds)."""
        ev = np.zeros(nlev)
        it = C.c_int(0)
        t = lib().ref_solve(self._h, npre, nlev, first_iter, inc_iter, noiter, level_limit, seed,
                            ev.ctypes.data_as(C.POINTER(C.c_double)), C.byref(it))
        return ev, it.value, t

    def close(self):
        if self._h:
            lib().ref_destroy(self._h)
            self._h = None
