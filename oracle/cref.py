"""ctypes binding of `cg_ref.c`, the C restatement of the reference column loop.

TEST INFRASTRUCTURE: the oracle. Used by tests (as a faster checker) and by
bench.py's CPU-baseline leg (as the timed CPU restatement).
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libeqdref.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.eqdref_stiffness_columns.restype = C.c_int
        _lib.eqdref_max_threads.restype = C.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _csr(M):
    M = M.tocsr()
    M.sort_indices()
    return (np.ascontiguousarray(M.indptr, dtype=np.int64),
            np.ascontiguousarray(M.indices, dtype=np.int32),
            np.ascontiguousarray(M.data, dtype=np.float64))


class CRefStiffness:
    """Holds the CSR arrays of one `oracle.fault.FaultElasticity`."""

    def __init__(self, fe):
        self.fe = fe
        self.A = _csr(fe.sys.A)
        self.B = _csr(fe.HP_DSAT)
        self.P = _csr(fe.P)
        self.T2 = _csr(fe.T2)
        self.T3 = _csr(fe.T3)
        self.chi_rows = np.ascontiguousarray(fe.chi_rows, dtype=np.int64)
        self.chi_rows_plus = np.ascontiguousarray(fe.chi_rows_plus, dtype=np.int64)
        self.omega = np.ascontiguousarray(fe.omega, dtype=np.int64)

    def columns(self, cols, rtol=1e-10, atol=0.0, itmax=0, nthreads=0):
        fe = self.fe
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        n = len(cols)
        out = np.zeros((n, 2 * fe.nf))
        iters = np.zeros(n, dtype=np.int64)
        solved = np.zeros(n, dtype=np.int8)
        args = [C.c_int64(fe.Ntot)]
        for m in (self.A, self.B, self.P):
            args += [_p(m[0]), _p(m[1]), _p(m[2])]
        args += [C.c_int64(self.T2[0].shape[0] - 1)]
        for m in (self.T2, self.T3):
            args += [_p(m[0]), _p(m[1]), _p(m[2])]
        args += [C.c_int32(fe.nf), _p(self.chi_rows), _p(self.chi_rows_plus), _p(self.omega),
                 C.c_int32(n), _p(cols), C.c_double(rtol), C.c_double(atol),
                 C.c_int64(itmax), C.c_int32(nthreads), _p(out), _p(iters), _p(solved)]
        rc = lib().eqdref_stiffness_columns(*args)
        if rc != 0:
            raise MemoryError("eqdref_stiffness_columns: allocation failed")
        return out.T.copy(), iters, solved.astype(bool)


def max_threads():
    return lib().eqdref_max_threads()
