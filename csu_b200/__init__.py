"""csu_b200 -- B200 engine for the residual-and-update path of CSU (2D unstructured finite volumes).

Python view of the C ABI declared in include/csu_gpu.h. The native library is required: importing
works without it (so the CPU-side tests can check the build), but every call that needs it raises
`NativeLibraryMissing` instead of falling back to anything else.

    case = Case.load("/tmp/wedge/")            # input.dat + mesh.su2 (+ restart.csv), like solverInit
    eng = Engine(case)                          # device layout + state, like solverMalloc/InitDomain
    hist = eng.iterate(100)                     # solverSolve iterations: res[Nvar], Cx_p, Cx_v, Cy_p, Cy_v
    U = eng.get_state()                         # [Nvar, Nelem] in the reference's cell order
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libcsu_b200.so")

CSU_OK = 0
ERRORS = {
    1: "CSU_ERR_INPUT", 2: "CSU_ERR_IO", 3: "CSU_ERR_OOM", 4: "CSU_ERR_NONFINITE", 5: "CSU_ERR_DIVERGED",
    6: "CSU_ERR_CANCELLED", 7: "CSU_ERR_CUDA", 8: "CSU_ERR_UNSUPPORTED", 9: "CSU_ERR_STATE",
    10: "CSU_ERR_NO_DEVICE",
}
DUMP = {"P": 1, "GHOST_P": 2, "GRAD": 3, "PHI": 4, "FACEFLUX": 5, "R": 6, "D": 7, "DTL": 8, "DW": 9, "BLOCKS": 10, "LSQ_X87": 11, "SST_JAC": 12, "BVISC": 13}
FLUX = {"ROE": 0, "AUSM": 1, "AUSMDV": 2, "AUSMpup": 3, "AUSMpup2": 4}
BC = {"symmetry": 0, "inlet": 1, "outlet": 2, "wall": 3, "wallT": 4}


class NativeLibraryMissing(RuntimeError):
    pass


class CsuError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (ERRORS.get(status, status), msg))
        self.status = status


class Config(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "nvar", "order", "flux", "stages", "time_scheme", "n_linear", "dt_local", "dt_local_n", "laminar", "sa",
        "sa_cc", "sst", "sst_trans", "axisymmetric", "turb1order", "visc_blazek", "tp", "limiter_type", "tube")] + [
        (n, C.c_double) for n in ("limiter_k", "cfl", "w_imp", "r_lim", "p_out", "t_wall", "sref", "turb_ratio",
                                  "e_fix", "pr", "pr_t", "gamma", "gas_r")] + [
        ("pin", C.c_double * 7), ("uin", C.c_double * 6), ("mach_inf", C.c_double), ("inlet_p", C.c_double),
        ("inlet_t", C.c_double), ("sst_l", C.c_double), ("k_factor", C.c_double), ("o_factor", C.c_double),
        ("o_wall_factor", C.c_double), ("implicit_fp32", C.c_int), ("implicit_local_dt", C.c_int),
        ("cfl_ramp_iters", C.c_int), ("cfl_max", C.c_double), ("conv_drop", C.c_double),
                ("iter_cap", C.c_int), ("limiter_func", C.c_int), ("gradient", C.c_int),
                ("sa_implicit_source", C.c_int)]


class MeshDesc(C.Structure):
    _fields_ = [("n_points", C.c_int), ("xy", C.c_void_p), ("n_cells", C.c_int), ("cell_npts", C.c_void_p),
                ("cell_nodes", C.c_void_p), ("n_faces", C.c_int), ("con", C.c_void_p), ("cell_nint", C.c_void_p),
                ("cell_faces", C.c_void_p), ("cell_nei", C.c_void_p), ("n_markers", C.c_int),
                ("marker_nbf", C.c_void_p), ("marker_flag", C.c_void_p), ("n_bfaces", C.c_int),
                ("bface", C.c_void_p), ("wall_dist", C.c_void_p)]


_lib = None


def lib():
    """The loaded native library (raises NativeLibraryMissing when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise NativeLibraryMissing("%s is missing: run `python csu_b200/build.py`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
        L.csu_last_error.restype = C.c_char_p
        L.csu_strerror.restype = C.c_char_p
        L.csu_case_load.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.csu_case_load_mem.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(vp)]
        L.csu_case_mesh.argtypes = [vp, C.POINTER(MeshDesc)]
        L.csu_case_config.argtypes = [vp, C.POINTER(Config)]
        L.csu_case_initial_state.argtypes = [vp, vp]
        L.csu_case_get_int.argtypes = [vp, C.c_char_p, ip]
        L.csu_case_get_double.argtypes = [vp, C.c_char_p, dp]
        L.csu_case_marker_name.argtypes = [vp, C.c_int, C.c_char_p, C.c_int]
        L.csu_case_free.argtypes = [vp]
        L.csu_case_free.restype = None
        L.csu_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(Config), C.POINTER(vp)]
        L.csu_destroy.argtypes = [vp]
        L.csu_destroy.restype = None
        L.csu_set_state.argtypes = [vp, vp]
        L.csu_get_state.argtypes = [vp, vp]
        L.csu_residual.argtypes = [vp, vp]
        L.csu_iterate.argtypes = [vp, C.c_int, C.c_int, vp]
        L.csu_iterate_ex.argtypes = [vp, C.c_int, C.c_int, vp, ip]
        L.csu_tube_run.argtypes = [vp, C.c_double, ip, dp]
        L.csu_dump.argtypes = [vp, C.c_int, vp]
        L.csu_wall_data.argtypes = [vp]
        L.csu_autotune.argtypes = [vp, ip, ip]
        L.csu_iterate_views.argtypes = [vp, C.c_int, vp, vp, vp]
        L.csu_stats.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.csu_set_stream.argtypes = [vp, vp]
        L.csu_time_kernels.argtypes = [vp, C.c_int, dp, ip]
        L.csu_residual_norms_noalloc.argtypes = [vp, C.c_int, C.c_int, vp, vp]
        L.csu_prep_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(Config), C.POINTER(vp)]
        L.csu_prep_bytes.argtypes = [vp]
        L.csu_prep_bytes.restype = C.c_longlong
        L.csu_prep_cells.argtypes = [vp]
        L.csu_prep_destroy.argtypes = [vp]
        L.csu_prep_destroy.restype = None
        L.csu_pack_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(vp)]
        L.csu_pack_size.argtypes = [vp]
        L.csu_pack_set_state.argtypes = [vp, C.c_int, vp]
        L.csu_pack_get_state.argtypes = [vp, C.c_int, vp]
        L.csu_pack_info.argtypes = [vp, C.c_int, C.POINTER(SolveInfo)]
        L.csu_pack_history.argtypes = [vp, C.c_int, vp, C.c_int, ip]
        L.csu_pack_transfer.argtypes = [vp, C.c_int, vp, C.c_int]
        L.csu_pack_rebuild.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(vp), C.c_int, C.POINTER(vp)]
        L.csu_srv_create.argtypes = [C.POINTER(SrvConfig), C.POINTER(vp)]
        L.csu_srv_submit.argtypes = [vp, C.POINTER(MeshDesc), C.POINTER(Config), vp, C.c_int,
                                     C.POINTER(C.c_longlong)]
        L.csu_srv_step.argtypes = [vp, ip, ip]
        L.csu_srv_info.argtypes = [vp, C.c_longlong, C.POINTER(SrvInfo)]
        L.csu_srv_take.argtypes = [vp, C.c_longlong, vp]
        L.csu_srv_cancel.argtypes = [vp, C.c_longlong]
        L.csu_srv_poll.argtypes = [vp, C.POINTER(C.c_longlong), C.c_int, ip]
        L.csu_srv_message.argtypes = [vp, C.c_longlong, C.c_char_p, C.c_int]
        L.csu_pack_stop.argtypes = [vp, C.c_int]
        L.csu_srv_totals.argtypes = [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.csu_srv_times.argtypes = [vp, dp, dp, dp, ip]
        L.csu_srv_destroy.argtypes = [vp]
        L.csu_srv_destroy.restype = None
        _lib = L
    return _lib


class SolveInfo(C.Structure):
    _fields_ = [("iter", C.c_int), ("status", C.c_int), ("done", C.c_int), ("hist_rows", C.c_int),
                ("have_res0", C.c_int), ("res0", C.c_double * 6), ("res", C.c_double * 6), ("coef", C.c_double * 4)]


class SrvConfig(C.Structure):
    _fields_ = [("budget_bytes", C.c_longlong), ("iters_per_step", C.c_int), ("max_pack", C.c_int),
                ("rebuild_steps", C.c_int), ("prep_threads", C.c_int)]


class SrvInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("iters", C.c_int), ("n_cells", C.c_int), ("drop", C.c_double),
                ("t_submit", C.c_double), ("t_start", C.c_double), ("t_end", C.c_double), ("status", C.c_int),
                ("coef", C.c_double * 4)]


SRV_STATES = {0: "queued", 1: "running", 2: "converged", 3: "failed", 4: "maxiter", 5: "cancelled"}


def _check(st):
    if st != CSU_OK:
        raise CsuError(st, lib().csu_last_error().decode(errors="replace"))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _arr(ptr, n, ctype, dtype):
    if not ptr or n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(n,)).astype(dtype, copy=True)


class Case:
    """A case folder read by the host C front end (input.dat keywords, SU2 mesh, initial state)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        d = MeshDesc()
        _check(lib().csu_case_mesh(self._h, C.byref(d)))
        self.desc = d
        cfg = Config()
        _check(lib().csu_case_config(self._h, C.byref(cfg)))
        self.config = cfg
        nc, nf, nb = d.n_cells, d.n_faces, d.n_bfaces
        self.n_cells, self.n_faces, self.n_bfaces, self.n_points = nc, nf, nb, d.n_points
        self.nvar = cfg.nvar
        self.xy = _arr(d.xy, 2 * d.n_points, C.c_double, np.float64).reshape(-1, 2)
        self.cell_npts = _arr(d.cell_npts, nc, C.c_int, np.int32)
        self.cell_nodes = _arr(d.cell_nodes, 4 * nc, C.c_int, np.int32).reshape(-1, 4)
        self.con = _arr(d.con, 4 * nf, C.c_int, np.int32).reshape(-1, 4)
        self.cell_nint = _arr(d.cell_nint, nc, C.c_int, np.int32)
        self.cell_faces = _arr(d.cell_faces, 4 * nc, C.c_int, np.int32).reshape(-1, 4)
        self.cell_nei = _arr(d.cell_nei, 4 * nc, C.c_int, np.int32).reshape(-1, 4)
        self.marker_nbf = _arr(d.marker_nbf, d.n_markers, C.c_int, np.int32)
        self.marker_flag = _arr(d.marker_flag, d.n_markers, C.c_int, np.int32)
        self.bface = _arr(d.bface, 3 * nb, C.c_int, np.int32).reshape(-1, 3)
        self.wall_dist = _arr(d.wall_dist, nc, C.c_double, np.float64) if d.wall_dist else None

    @classmethod
    def load(cls, wd):
        if not wd.endswith("/"):
            wd += "/"
        h = C.c_void_p()
        _check(lib().csu_case_load(wd.encode(), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_text(cls, input_dat, mesh_su2, restart_csv=None):
        h = C.c_void_p()
        _check(lib().csu_case_load_mem(input_dat.encode(), mesh_su2.encode(),
                                       restart_csv.encode() if restart_csv else None, C.byref(h)))
        return cls(h.value)

    def initial_state(self):
        U = np.zeros(self.nvar * self.n_cells)
        _check(lib().csu_case_initial_state(self._h, _ptr(U)))
        return U.reshape(self.nvar, self.n_cells)

    def get_int(self, key):
        v = C.c_int()
        _check(lib().csu_case_get_int(self._h, key.encode(), C.byref(v)))
        return v.value

    def get_double(self, key):
        v = C.c_double()
        _check(lib().csu_case_get_double(self._h, key.encode(), C.byref(v)))
        return v.value

    def marker_name(self, m):
        buf = C.create_string_buffer(64)
        _check(lib().csu_case_marker_name(self._h, m, buf, 64))
        return buf.value.decode()

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.csu_case_free(self._h)
            self._h = None


class Engine:
    """Device engine of one solve (a csu_ctx)."""

    def __init__(self, case, config=None, state=None):
        self.case = case
        self.config = config if config is not None else case.config
        self.nvar = self.config.nvar
        self.n_cells = case.n_cells
        h = C.c_void_p()
        _check(lib().csu_create(C.byref(case.desc), C.byref(self.config), C.byref(h)))
        self._h = h
        self.set_state(case.initial_state() if state is None else state)

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.nvar, self.n_cells)
        _check(lib().csu_set_state(self._h, _ptr(U)))

    def get_state(self, out=None):
        """The conserved state [var][cell] in reference order. `out`: a C-contiguous float64 array of that
        shape to fill (e.g. pinned host memory, which the device then writes by DMA) instead of a new one."""
        if out is None:
            out = np.empty((self.nvar, self.n_cells))
        elif (out.dtype != np.float64 or not out.flags.c_contiguous or out.size != self.nvar * self.n_cells):
            raise ValueError("get_state: out must be a C-contiguous float64 array of %d x %d"
                             % (self.nvar, self.n_cells))
        _check(lib().csu_get_state(self._h, _ptr(out)))
        return out

    def residual(self):
        R = np.zeros((self.nvar, self.n_cells))
        _check(lib().csu_residual(self._h, _ptr(R)))
        return R

    def iterate(self, n, it0=0):
        hist = np.zeros((max(n, 1), self.nvar + 4))
        _check(lib().csu_iterate(self._h, n, it0, _ptr(hist)))
        return hist[:n]

    def iterate_until(self, n, it0=0):
        """Up to n iterations, stopping at the convergence criterion; returns the history rows run."""
        hist = np.zeros((max(n, 1), self.nvar + 4))
        done = C.c_int()
        _check(lib().csu_iterate_ex(self._h, n, it0, _ptr(hist), C.byref(done)))
        return hist[:done.value]

    def tube_run(self, tmax):
        steps, t = C.c_int(), C.c_double()
        _check(lib().csu_tube_run(self._h, tmax, C.byref(steps), C.byref(t)))
        return steps.value, t.value

    def dump(self, what):
        nc, nv, nf, nb = self.n_cells, self.nvar, self.case.n_faces, self.case.n_bfaces
        shapes = {"P": (nc, nv + 1), "GHOST_P": (nb, nv + 1), "GRAD": (2, nv, nc), "PHI": (nv, nc),
                  "FACEFLUX": (nv, nf), "R": (nv, nc), "D": (nc,), "DTL": (nc,), "DW": (nv, nc),
                  "BLOCKS": (nc, 4, nv, nv), "LSQ_X87": (1,), "SST_JAC": (6, nc), "BVISC": (nb, 4)}
        out = np.zeros(shapes[what])
        _check(lib().csu_dump(self._h, DUMP[what], _ptr(out)))
        return out

    def set_stream(self, stream):
        """Run on a caller's cudaStream_t (an int handle, e.g. torch.cuda.Stream().cuda_stream); None resets."""
        _check(lib().csu_set_stream(self._h, C.c_void_p(stream) if stream else None))

    def time_kernels(self, iters):
        """Device time per kernel kind over `iters` iterations (the state advances)."""
        ms = (C.c_double * 9)()
        cnt = (C.c_int * 9)()
        _check(lib().csu_time_kernels(self._h, iters, ms, cnt))
        return {"ms": list(ms), "count": list(cnt)}

    def stats(self):
        a, b = C.c_longlong(), C.c_longlong()
        _check(lib().csu_stats(self._h, C.byref(a), C.byref(b)))
        return {"kernel_launches": a.value, "device_bytes": b.value}

    def autotune(self):
        """Times the launch shapes on this solve and keeps the fastest: (faces per flux block, cells per
        sweep block)."""
        fb, sb = C.c_int(), C.c_int()
        _check(lib().csu_autotune(self._h, C.byref(fb), C.byref(sb)))
        return fb.value, sb.value

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.csu_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Prep:
    """A solve prepared on the host for packing (device layout and byte count; no device memory)."""

    def __init__(self, case, config=None, state=None):
        self.case = case
        self.config = config if config is not None else case.config
        self.nvar = self.config.nvar
        self.n_cells = case.n_cells
        self.state = np.ascontiguousarray(case.initial_state() if state is None else state, dtype=np.float64)
        h = C.c_void_p()
        _check(lib().csu_prep_create(C.byref(case.desc), C.byref(self.config), C.byref(h)))
        self._h = h

    @property
    def bytes(self):
        return lib().csu_prep_bytes(self._h)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.csu_prep_destroy(self._h)
            self._h = None


class Pack:
    """Several steady solves advanced together: one launch of each kernel per iteration for all of them."""

    def __init__(self, preps, states=True):
        self.preps = list(preps)
        arr = (C.c_void_p * len(self.preps))(*[p._h.value for p in self.preps])
        h = C.c_void_p()
        _check(lib().csu_pack_create(arr, len(self.preps), C.byref(h)))
        self._h = h
        if states:
            for k, p in enumerate(self.preps):
                self.set_state(k, p.state)

    def __len__(self):
        return len(self.preps)

    def set_state(self, k, U):
        p = self.preps[k]
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(p.nvar, p.n_cells)
        _check(lib().csu_pack_set_state(self._h, k, _ptr(U)))

    def get_state(self, k):
        p = self.preps[k]
        U = np.zeros((p.nvar, p.n_cells))
        _check(lib().csu_pack_get_state(self._h, k, _ptr(U)))
        return U

    def iterate(self, n):
        """n iterations of every solve (converged or failed solves stay frozen)."""
        _check(lib().csu_iterate(self._h, n, 0, None))

    def info(self, k):
        i = SolveInfo()
        _check(lib().csu_pack_info(self._h, k, C.byref(i)))
        nv = self.preps[k].nvar
        return {"iter": i.iter, "status": i.status, "done": i.done, "hist_rows": i.hist_rows,
                "res0": np.array(i.res0[:nv]), "res": np.array(i.res[:nv]), "coef": np.array(i.coef[:]),
                "have_res0": i.have_res0}

    def history(self, k, max_rows=1 << 20):
        nv = self.preps[k].nvar
        rows = self.info(k)["hist_rows"]
        out = np.zeros((max(min(rows, max_rows), 1), nv + 4))
        n = C.c_int()
        _check(lib().csu_pack_history(self._h, k, _ptr(out), min(rows, max_rows), C.byref(n)))
        return out[:n.value]

    def rebuilt(self, keep, preps):
        """A new pack of `preps`; member k is member keep[k] of this pack (mesh and iteration state moved on
        the device) when keep[k] >= 0, else starts from its prep's state."""
        new = Pack.__new__(Pack)
        new.preps = list(preps)
        km = (C.c_int * len(new.preps))(*[int(v) for v in keep])
        arr = (C.c_void_p * len(new.preps))(*[p._h.value for p in new.preps])
        h = C.c_void_p()
        _check(lib().csu_pack_rebuild(self._h, km, arr, len(new.preps), C.byref(h)))
        new._h = h
        for k, p in enumerate(new.preps):
            if keep[k] < 0:
                new.set_state(k, p.state)
        return new

    def stop(self, k):
        """Freezes solve k where it stands; the others go on."""
        _check(lib().csu_pack_stop(self._h, k))

    def transfer_from(self, other, k_other, k):
        _check(lib().csu_pack_transfer(other._h, k_other, self._h, k))

    def stats(self):
        a, b = C.c_longlong(), C.c_longlong()
        _check(lib().csu_stats(self._h, C.byref(a), C.byref(b)))
        return {"kernel_launches": a.value, "device_bytes": b.value}

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.csu_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Server:
    """Continuous batching of steady solves (csu_srv_*): submit requests as they arrive, call step() in a loop."""

    def __init__(self, budget_bytes, iters_per_step=16, max_pack=0, rebuild_steps=1, prep_threads=0):
        cfg = SrvConfig(int(budget_bytes), int(iters_per_step), int(max_pack), int(rebuild_steps), int(prep_threads))
        h = C.c_void_p()
        _check(lib().csu_srv_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._shape = {}

    def submit(self, case, config=None, state=None, max_iters=100000):
        cfg = config if config is not None else case.config
        U = np.ascontiguousarray(case.initial_state() if state is None else state, dtype=np.float64)
        i = C.c_longlong()
        _check(lib().csu_srv_submit(self._h, C.byref(case.desc), C.byref(cfg), _ptr(U), int(max_iters),
                                    C.byref(i)))
        self._shape[i.value] = (cfg.nvar, case.n_cells)
        return i.value

    def step(self):
        r, q = C.c_int(), C.c_int()
        _check(lib().csu_srv_step(self._h, C.byref(r), C.byref(q)))
        return r.value, q.value

    def info(self, rid):
        i = SrvInfo()
        _check(lib().csu_srv_info(self._h, rid, C.byref(i)))
        return {"state": SRV_STATES[i.state], "iters": i.iters, "n_cells": i.n_cells, "drop": i.drop,
                "t_submit": i.t_submit, "t_start": i.t_start, "t_end": i.t_end, "status": i.status,
                "coef": list(i.coef)}

    def poll(self, cap=4096):
        """Ids of the requests that reached a final state since the last poll, in that order."""
        buf = (C.c_longlong * cap)()
        n = C.c_int()
        _check(lib().csu_srv_poll(self._h, buf, cap, C.byref(n)))
        return list(buf[:n.value])

    def cancel(self, rid):
        _check(lib().csu_srv_cancel(self._h, rid))

    def message(self, rid):
        buf = C.create_string_buffer(256)
        _check(lib().csu_srv_message(self._h, rid, buf, 256))
        return buf.value.decode(errors="replace")

    def take(self, rid):
        U = np.zeros(self._shape[rid])
        _check(lib().csu_srv_take(self._h, rid, _ptr(U)))
        del self._shape[rid]
        return U

    def totals(self):
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        _check(lib().csu_srv_totals(self._h, C.byref(a), C.byref(b), C.byref(c)))
        r, i, p, n = C.c_double(), C.c_double(), C.c_double(), C.c_int()
        _check(lib().csu_srv_times(self._h, C.byref(r), C.byref(i), C.byref(p), C.byref(n)))
        return {"solve_iterations": a.value, "cell_updates": b.value, "used_bytes": c.value,
                "rebuild_s": r.value, "iterate_s": i.value, "poll_s": p.value, "rebuilds": n.value}

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.csu_srv_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
