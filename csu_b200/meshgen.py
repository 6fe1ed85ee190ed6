"""Synthetic SU2 meshes and case folders for the benchmark configurations (gmsh is not available).

Every generator returns (su2_text, input_dat_text). Marker lines carry the trailing space that the SU2
reader of the reference requires (mesh.c:102-107 reads four tokens per boundary line). Inputs are
seeded and deterministic.

    ramp(...)      15 deg compression ramp, structured quads split in triangles, jittered interior nodes
    sod_tube(...)  1000 x 2 quads split in triangles, Sod initial states (dimensional, see below)
"""
import math
import os

import numpy as np

R_GAS = 287.0530  # solverSetData (solver.c:1425)


def _su2(points, cells, markers):
    """points: (Np,2); cells: list of int arrays (3 or 4 nodes, counter-clockwise); markers: {name: (Ne,2)}."""
    out = ["NDIME= 2", "NELEM= %d" % len(cells)]
    for i, c in enumerate(cells):
        out.append("%d %s %d" % (5 if len(c) == 3 else 9, " ".join(str(int(v)) for v in c), i))
    out.append("NPOIN= %d" % len(points))
    for i, (x, y) in enumerate(points):
        out.append("%.17g %.17g %d" % (x, y, i))
    out.append("NMARK= %d" % len(markers))
    for name, edges in markers.items():
        out.append("MARKER_TAG= %s" % name)
        out.append("MARKER_ELEMS= %d" % len(edges))
        for a, b in edges:
            out.append("3 %d %d " % (a, b))
    return "\n".join(out) + "\n"


def _input(kv):
    return "\n" + "".join("%s, %s\n" % (k, v) for k, v in kv.items())


def _structured_tris(X, Y, diag=0):
    """Nodes (nj+1, ni+1) -> triangles of every quad (i, j); node id = j*(ni+1) + i."""
    nj, ni = X.shape[0] - 1, X.shape[1] - 1
    idx = np.arange((ni + 1) * (nj + 1)).reshape(nj + 1, ni + 1)
    a, b = idx[:-1, :-1], idx[:-1, 1:]
    c, d = idx[1:, 1:], idx[1:, :-1]
    t1 = np.stack([a, b, c], axis=-1).reshape(-1, 3)
    t2 = np.stack([a, c, d], axis=-1).reshape(-1, 3)
    tris = np.empty((t1.shape[0] * 2, 3), dtype=np.int64)
    tris[0::2] = t1
    tris[1::2] = t2
    pts = np.stack([X.ravel(), Y.ravel()], axis=1)
    return pts, tris, idx


def ramp(ni=400, nj=200, length=1.5, x_ramp=0.5, angle_deg=15.0, height=1.0, jitter=0.1, seed=0, mach=2.5,
         pressure=1e5, temperature=300.0, flux="AUSM", lim_k=5.0, n_linear=4, cfl=10.0, nmax=1000, threads=8,
         scheme="DPLUR", order=2):
    """Supersonic flow over a 15 degree compression ramp: x in [0, length], the wall rises from x_ramp,
    top at `height`. ni x nj quads split into two triangles each; interior nodes jittered by U(-jitter, jitter)
    of the local spacing with numpy default_rng(seed)."""
    t = math.tan(math.radians(angle_deg))
    x = np.linspace(0.0, length, ni + 1)
    yb = np.where(x > x_ramp, (x - x_ramp) * t, 0.0)
    s = np.linspace(0.0, 1.0, nj + 1)
    X = np.repeat(x[None, :], nj + 1, axis=0)
    Y = yb[None, :] + (height - yb[None, :]) * s[:, None]
    rng = np.random.default_rng(seed)
    hx = length / ni
    hy = (height - yb[None, :]) / nj
    jx = rng.uniform(-jitter, jitter, size=X.shape) * hx
    jy = rng.uniform(-jitter, jitter, size=X.shape) * hy
    inner = np.zeros(X.shape, dtype=bool)
    inner[1:-1, 1:-1] = True
    X = np.where(inner, X + jx, X)
    Y = np.where(inner, Y + jy, Y)
    pts, tris, idx = _structured_tris(X, Y)
    markers = {
        "inlet": np.stack([idx[1:, 0], idx[:-1, 0]], axis=1),
        "outlet": np.stack([idx[:-1, -1], idx[1:, -1]], axis=1),
        "top": np.stack([idx[-1, 1:], idx[-1, :-1]], axis=1),
        "wall": np.stack([idx[0, :-1], idx[0, 1:]], axis=1),
    }
    su2 = _su2(pts, list(tris), markers)
    kv = {"pressure": "%.17g" % pressure, "temperature": "%.17g" % temperature, "mach": "%.17g" % mach,
          "nx": "1.", "ny": "0.", "BC:inlet": "inlet", "BC:outlet": "outlet", "BC:top": "symmetry",
          "BC:wall": "wall", "Nmax": str(nmax), "order": str(order), "stages": "5", "threads": str(threads),
          "flux": flux, "tube": "0", "axisymmetric": "0", "CFL": "%g" % cfl, "timeScheme": scheme,
          "Nlinear": str(n_linear), "limK": "%g" % lim_k}
    return su2, _input(kv)


def sod_tube(ni=1000, nj=2, length=1.0, height=0.01, flux="ROE", order=2, stages=3, cfl=0.5, threads=8,
             rho_l=1.0, p_l=1e5, rho_r=0.125, p_r=1e4, x_m=0.5):
    """Sod shock tube on 1000 x 2 quads split into triangles (4,000 cells). The reference takes p, T and
    Mach (solver.c:1709-1719) and clamps T < 1 K, so the classic rho = 1, p = 1 / rho = 0.125, p = 0.1 states
    are run dimensionally: p scaled by 1e5, T = p / (rho R); the nondimensional end time 0.2 becomes
    0.2 / sqrt(1e5) s. All four sides are slip walls (the waves do not reach the ends by t_end)."""
    x = np.linspace(0.0, length, ni + 1)
    y = np.linspace(0.0, height, nj + 1)
    X, Y = np.meshgrid(x, y)
    pts, tris, idx = _structured_tris(X, Y)
    markers = {
        "left": np.stack([idx[1:, 0], idx[:-1, 0]], axis=1),
        "right": np.stack([idx[:-1, -1], idx[1:, -1]], axis=1),
        "top": np.stack([idx[-1, 1:], idx[-1, :-1]], axis=1),
        "bottom": np.stack([idx[0, :-1], idx[0, 1:]], axis=1),
    }
    su2 = _su2(pts, list(tris), markers)
    scale = math.sqrt(p_l / rho_l)
    kv = {"pressure1": "%.17g" % p_l, "temperature1": "%.17g" % (p_l / (rho_l * R_GAS)), "mach1": "0.",
          "nx1": "1.", "ny1": "0.", "pressure2": "%.17g" % p_r, "temperature2": "%.17g" % (p_r / (rho_r * R_GAS)),
          "mach2": "0.", "nx2": "1.", "ny2": "0.", "BC:left": "symmetry", "BC:right": "symmetry",
          "BC:top": "symmetry", "BC:bottom": "symmetry", "xm": "%.17g" % x_m, "tmax": "%.17g" % (0.2 / scale),
          "order": str(order), "stages": str(stages), "threads": str(threads), "flux": flux, "tube": "1",
          "axisymmetric": "0", "CFL": "%g" % cfl}
    return su2, _input(kv)


def write_case(wd, su2, inp):
    """Writes mesh.su2 and input.dat into wd (created); returns wd with a trailing slash."""
    if not wd.endswith("/"):
        wd += "/"
    os.makedirs(wd, exist_ok=True)
    with open(wd + "mesh.su2", "w") as f:
        f.write(su2)
    with open(wd + "input.dat", "w") as f:
        f.write(inp)
    return wd
