"""ctypes view of oracle/_build/libcsuoracle.so (csu_oracle.c, the plain-C restatement).
Test infrastructure only; the product never imports this module."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libcsuoracle.so")


def available():
    return os.path.exists(LIB)


def build():
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    _lib = None

    def __init__(self, case):
        """case: a csu_b200.Case (mesh arrays in reference order, verified integer-exact against the reference)."""
        if Oracle._lib is None:
            L = C.CDLL(LIB)
            L.orc_create.restype = C.c_void_p
            L.orc_create.argtypes = [C.c_void_p, C.c_void_p]
            for fn in ("orc_free", "orc_residual"):
                getattr(L, fn).argtypes = [C.c_void_p]
            L.orc_set_U.argtypes = [C.c_void_p, C.c_void_p]
            L.orc_get_U.argtypes = [C.c_void_p, C.c_void_p]
            L.orc_get.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
            L.orc_iterate.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
            L.orc_tube.argtypes = [C.c_void_p, C.c_double, C.POINTER(C.c_double)]
            L.orc_tube.restype = C.c_int
            Oracle._lib = L
        self.L = Oracle._lib
        self.case = case
        self.nc, self.nv, self.nf, self.nb = case.n_cells, case.nvar, case.n_faces, case.n_bfaces
        self.h = self.L.orc_create(C.byref(case.desc), C.byref(case.config))
        self.set_U(case.initial_state())

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_free(self.h)
            self.h = None

    def set_U(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        self.L.orc_set_U(self.h, _p(U))

    def get_U(self):
        U = np.zeros((self.nv, self.nc))
        self.L.orc_get_U(self.h, _p(U))
        return U

    def residual(self):
        self.L.orc_residual(self.h)
        return self.get("R")

    def get(self, what):
        nc, nv, nf, nb = self.nc, self.nv, self.nf, self.nb
        spec = {"P": (1, (nc, nv + 1)), "GHOST_P": (2, (nb, nv + 1)), "GRAD": (3, (2, nv, nc)), "PHI": (4, (nv, nc)),
                "FACEFLUX": (5, (nv, nf)), "R": (6, (nv, nc)), "D": (7, (nc,)), "DTL": (8, (nc,)), "DW": (9, (nv, nc)),
                "BLOCKS": (10, (nc, 4, 4, 4))}
        code, shape = spec[what]
        out = np.zeros(shape)
        self.L.orc_get(self.h, code, _p(out))
        return out

    def iterate(self, n, it0=0):
        hist = np.zeros((n, self.nv + 4))
        self.L.orc_iterate(self.h, n, it0, _p(hist))
        return hist

    def tube(self, tmax):
        t = C.c_double()
        steps = self.L.orc_tube(self.h, tmax, C.byref(t))
        return steps, t.value
