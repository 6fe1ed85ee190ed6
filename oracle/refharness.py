"""ctypes view of oracle/_ref/libcsuref.so: the reference solver built from its own C sources plus
ref_harness.c. Test infrastructure only; the product never imports this module."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libcsuref.so")
EXE = os.path.join(HERE, "_ref", "csu_ref")


def available():
    return os.path.exists(LIB)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Ref:
    """One reference solver instance (the harness holds a single global SOLVER*, so one at a time)."""
    _lib = None

    def __init__(self, wd, quiet=True):
        if Ref._lib is None:
            Ref._lib = C.CDLL(LIB)
            Ref._lib.ref_calc_dt.restype = C.c_double
            Ref._lib.ref_tube_run.restype = C.c_int
            Ref._lib.ref_tube_run.argtypes = [C.c_double, C.POINTER(C.c_double)]
        L = self.L = Ref._lib
        if not wd.endswith("/"):
            wd += "/"
        if len(wd) > 30:
            raise ValueError("reference case paths must be short (char[50] buffers): %s" % wd)
        if L.ref_open(wd.encode(), 1 if quiet else 0) != 0:
            raise RuntimeError("reference solverInit failed for %s" % wd)
        s = (C.c_int * 16)()
        L.ref_sizes(s)
        (self.nc, self.np, self.nf, self.nmark, self.nvar, self.nb, self.time_scheme, self.stages,
         self.order, self.flux, self.laminar, self.sa, self.sst, self.axi, self.dt_local, self.n_linear) = list(s)

    def mesh(self):
        nc, nf, nb = self.nc, self.nf, self.nb
        out = dict(con=np.zeros(4 * nf, np.int32), nodes=np.zeros(4 * nc, np.int32), npts=np.zeros(nc, np.int32),
                   f=np.zeros(4 * nc, np.int32), nint=np.zeros(nc, np.int32), nei=np.zeros(4 * nc, np.int32),
                   omega=np.zeros(nc), marker_nbf=np.zeros(self.nmark, np.int32),
                   marker_flag=np.zeros(self.nmark, np.int32), bface=np.zeros(3 * nb, np.int32),
                   xy=np.zeros(2 * self.np))
        self.L.ref_con(_p(out["con"]))
        self.L.ref_cells(_p(out["nodes"]), _p(out["npts"]), _p(out["f"]), _p(out["nint"]), _p(out["nei"]),
                         _p(out["omega"]))
        self.L.ref_bc(_p(out["marker_nbf"]), _p(out["marker_flag"]), _p(out["bface"]))
        self.L.ref_points(_p(out["xy"]))
        if self.sa or self.sst:
            out["wall_dist"] = np.zeros(nc)
            self.L.ref_wall_distance(_p(out["wall_dist"]))
        return out

    def get_U(self):
        U = np.zeros(self.nvar * self.nc)
        self.L.ref_get_U(_p(U))
        return U.reshape(self.nvar, self.nc)

    def set_U(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64)
        self.L.ref_set_U(_p(U))

    def calc_R(self):
        self.L.ref_calc_R()
        R = np.zeros(self.nvar * self.nc)
        self.L.ref_get_R(_p(R))
        return R.reshape(self.nvar, self.nc)

    def P(self):
        P = np.zeros(self.nc * (self.nvar + 1))
        self.L.ref_get_P(_p(P))
        return P.reshape(self.nc, self.nvar + 1)

    def ghost_P(self):
        P = np.zeros(self.nb * (self.nvar + 1))
        self.L.ref_get_ghostP(_p(P))
        return P.reshape(self.nb, self.nvar + 1)

    def grad(self):
        gx, gy = np.zeros(self.nvar * self.nc), np.zeros(self.nvar * self.nc)
        self.L.ref_get_grad(_p(gx), _p(gy))
        return np.stack([gx.reshape(self.nvar, self.nc), gy.reshape(self.nvar, self.nc)])

    def phi(self):
        a = np.zeros(self.nvar * self.nc)
        self.L.ref_get_phi(_p(a))
        return a.reshape(self.nvar, self.nc)

    def faceflux(self):
        a = np.zeros(self.nvar * self.nf)
        self.L.ref_get_faceflux(_p(a))
        return a.reshape(self.nvar, self.nf)

    def calc_dt(self):
        dtl = np.zeros(self.nc)
        dt = self.L.ref_calc_dt(_p(dtl))
        return dt, dtl

    def sst_jac(self):
        """SST source Jacobians of the last calc_R, [6][cell]."""
        J = np.zeros(6 * self.nc)
        self.L.ref_sst_jac(_p(J))
        return J.reshape(6, self.nc)

    def miT(self):
        """Face eddy viscosity of the last calc_R (SA, SST), per face in mesh->con order."""
        a = np.zeros(self.nf)
        self.L.ref_get_miT(_p(a))
        return a

    def implicit_D(self):
        D, dtl = np.zeros(self.nc), np.zeros(self.nc)
        self.L.ref_implicit_D(_p(D), _p(dtl))
        return D, dtl

    def implicit_A(self):
        A = np.zeros(self.nc * 4 * self.nvar * self.nvar)
        self.L.ref_implicit_A(_p(A))
        return A.reshape(self.nc, 4, self.nvar, self.nvar)

    def implicit_dplur(self):
        dW = np.zeros(self.nvar * self.nc)
        self.L.ref_implicit_dplur(_p(dW))
        return dW.reshape(self.nvar, self.nc)

    def iterate(self, n, it0=0):
        hist = np.zeros(n * (self.nvar + 4))
        self.L.ref_iterate(n, it0, _p(hist))
        return hist.reshape(n, self.nvar + 4)

    def tube_run(self, tmax):
        t = C.c_double()
        steps = self.L.ref_tube_run(tmax, C.byref(t))
        return steps, t.value

    def solve(self):
        self.L.ref_solve()
