"""Synthetic SU2 meshes and case folders for the benchmark configurations (gmsh is not available).

Every generator returns (su2_text, input_dat_text). Marker lines carry the trailing space that the SU2
reader of the reference requires (mesh.c:102-107 reads four tokens per boundary line). Inputs are
seeded and deterministic.

    ramp(...)      15 deg compression ramp, structured quads split in triangles, jittered interior nodes
    sod_tube(...)  1000 x 2 quads split in triangles, Sod initial states (dimensional, see below)
    bump(...)      channel with a 10 %-height circular bump, mixed triangles and quads
    cylinder(...)  cylinder (r = 0.5) in a 40-diameter box, O-grid
    airfoil(...)   NACA 0012 (closed trailing edge) C-mesh with wake cut, first cell y1
    plate(...)     turbulent flat plate: tanh clustering at the leading edge, geometric wall spacing
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


def _structured_quads(X, Y):
    """Nodes (nj+1, ni+1) -> one quad per cell (counter-clockwise for increasing i then j)."""
    nj, ni = X.shape[0] - 1, X.shape[1] - 1
    idx = np.arange((ni + 1) * (nj + 1)).reshape(nj + 1, ni + 1)
    q = np.stack([idx[:-1, :-1], idx[:-1, 1:], idx[1:, 1:], idx[1:, :-1]], axis=-1).reshape(-1, 4)
    pts = np.stack([X.ravel(), Y.ravel()], axis=1)
    return pts, q, idx


def _mixed(q, tri_fraction, rng):
    """Splits a seeded random share of the quads into two triangles: a mixed tri/quad mesh."""
    cells = []
    split = rng.random(len(q)) < tri_fraction
    for k, c in enumerate(q):
        if split[k]:
            cells.append(c[[0, 1, 2]])
            cells.append(c[[0, 2, 3]])
        else:
            cells.append(c)
    return cells


def _ccw(points, cells):
    """Orders every cell counter-clockwise (the reference reverses clockwise cells too, mesh.c:222-242)."""
    out = []
    for c in cells:
        x, y = points[c, 0], points[c, 1]
        a = np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y)
        out.append(c if a > 0 else c[::-1])
    return out


def _flow_kv(mach, pressure, temperature, alpha_deg=0.0):
    """Free stream; the outlet back pressure `pout` is the free-stream pressure (the reference's default,
    1e5 Pa, solver.c:1558-1565, would impose a wrong back pressure on cases run at another pressure, such
    as the low-Reynolds ones whose pressure is set by the Reynolds number)."""
    a = math.radians(alpha_deg)
    return {"pressure": "%.17g" % pressure, "temperature": "%.17g" % temperature, "mach": "%.17g" % mach,
            "nx": "%.17g" % math.cos(a), "ny": "%.17g" % math.sin(a), "pout": "%.17g" % pressure}


def _solver_kv(flux="AUSMDV", order=1, scheme="DPLUR", n_linear=4, cfl=5.0, nmax=1000, viscous=None):
    kv = {"Nmax": str(nmax), "order": str(order), "stages": "5", "threads": "8", "flux": flux, "tube": "0",
          "axisymmetric": "0", "CFL": "%g" % cfl, "timeScheme": scheme, "Nlinear": str(n_linear)}
    if viscous == "laminar":
        kv["laminar"] = "1"
    elif viscous == "sa":
        kv["sa"] = "1"
        kv["turbRatio"] = "3"
    elif viscous == "sst":
        kv["sst"] = "1"
    return kv


def _pressure_for_re(re, mach, temperature, length):
    """Pressure giving Re = rho U L / mu (Sutherland mu at T, sutherland() of solver.c:1222-1225)."""
    mu = 1.458e-6 * temperature ** 1.5 / (temperature + 110.4)
    c = math.sqrt(1.4 * R_GAS * temperature)
    rho = re * mu / (mach * c * length)
    return rho * R_GAS * temperature


def bump(ncells=20000, mach=0.5, height=0.1, tri_fraction=0.5, seed=0, viscous=None, re=None, temperature=300.0,
         **solver):
    """Channel [0, 3] x [0, 1] with a circular-arc bump of `height` (chord 1) on the lower wall from x = 1
    to 2; structured, a seeded share of the quads split into triangles (mixed tri/quad). About `ncells`
    cells. Inlet left, outlet right, upper symmetry, lower wall."""
    nj = max(4, int(round(math.sqrt(ncells / 3.0 / (1 + tri_fraction)))))
    ni = 3 * nj
    x = np.linspace(0.0, 3.0, ni + 1)
    r = (0.25 + height * height) / (2 * height)
    yb = np.where((x > 1) & (x < 2), np.sqrt(np.maximum(r * r - (x - 1.5) ** 2, 0.0)) - (r - height), 0.0)
    s = np.linspace(0.0, 1.0, nj + 1)
    X = np.repeat(x[None, :], nj + 1, axis=0)
    Y = yb[None, :] + (1.0 - yb[None, :]) * s[:, None]
    pts, q, idx = _structured_quads(X, Y)
    cells = _mixed(q, tri_fraction, np.random.default_rng(seed))
    markers = {
        "inlet": np.stack([idx[1:, 0], idx[:-1, 0]], axis=1),
        "outlet": np.stack([idx[:-1, -1], idx[1:, -1]], axis=1),
        "top": np.stack([idx[-1, 1:], idx[-1, :-1]], axis=1),
        "wall": np.stack([idx[0, :-1], idx[0, 1:]], axis=1),
    }
    p = _pressure_for_re(re, mach, temperature, 1.0) if re else 1e5
    kv = _flow_kv(mach, p, temperature)
    kv.update({"BC:inlet": "inlet", "BC:outlet": "outlet", "BC:top": "symmetry", "BC:wall": "wall"})
    kv.update(_solver_kv(viscous=viscous, **solver))
    return _su2(pts, cells, markers), _input(kv)


def cylinder(ncells=20000, mach=2.0, radius=0.5, box=40.0, tri_fraction=0.0, seed=0, viscous=None, re=None,
             temperature=300.0, **solver):
    """Cylinder of radius 0.5 in a square box of side 40 diameters: an O-grid from the circle to the box
    (points on rays blended from the circle to the square), geometric radial spacing. Upstream half of the
    box is an inlet, downstream half an outlet; the cylinder a wall."""
    nr = max(4, int(round(math.sqrt(ncells / 4.0))))
    nt = 4 * nr
    t = np.linspace(0.0, 2 * math.pi, nt + 1)[:-1]
    cx, cy = np.cos(t), np.sin(t)
    half = box * 2 * radius / 2
    m = np.maximum(np.abs(cx), np.abs(cy))
    sx, sy = half * cx / m, half * cy / m
    g = 1.0 + 6.0 / nr
    w = (g ** np.arange(nr + 1) - 1) / (g ** nr - 1)
    X = radius * cx[None, :] * (1 - w[:, None]) + sx[None, :] * w[:, None]
    Y = radius * cy[None, :] * (1 - w[:, None]) + sy[None, :] * w[:, None]
    idx = np.arange((nr + 1) * nt).reshape(nr + 1, nt)
    ip = np.roll(idx, -1, axis=1)
    q = np.stack([idx[:-1], ip[:-1], ip[1:], idx[1:]], axis=-1).reshape(-1, 4)
    pts = np.stack([X.ravel(), Y.ravel()], axis=1)
    cells = _ccw(pts, _mixed(q, tri_fraction, np.random.default_rng(seed)))
    wall = np.stack([idx[0], ip[0]], axis=1)[:, ::-1]
    outer = np.stack([idx[-1], ip[-1]], axis=1)
    up = cx < 0
    markers = {"wall": wall, "farin": outer[up], "farout": outer[~up]}
    p = _pressure_for_re(re, mach, temperature, 2 * radius) if re else 1e5
    kv = _flow_kv(mach, p, temperature)
    kv.update({"BC:wall": "wall", "BC:farin": "inlet", "BC:farout": "outlet"})
    kv.update(_solver_kv(viscous=viscous, **solver))
    return _su2(pts, cells, markers), _input(kv)


def plate(ni=545, nj=385, x0=-0.33, x1=2.0, height=1.0, y1=1e-6, growth=1.07, beta=3.0, mach=0.2, re=5e6,
          temperature=300.0, viscous="sa", **solver):
    """Flat plate: [x0, x1] x [0, height] m, no-slip adiabatic wall on x in [0, x1] and symmetry upstream.
    ni x nj quads; x clustered at the leading edge with tanh stretching (factor `beta`) on both sides; y with
    first spacing y1 growing geometrically by `growth` until the spacing that fills the height evenly is
    reached. Re based on the plate length x1. Inlet left, outlet right, characteristic far field on top."""
    n_up = max(2, int(round(ni * (-x0) / (x1 - x0))))
    n_dn = ni - n_up
    su = np.tanh(beta * np.linspace(0.0, 1.0, n_up + 1)) / np.tanh(beta)
    sd = np.tanh(beta * np.linspace(0.0, 1.0, n_dn + 1)) / np.tanh(beta)
    x = np.concatenate([x0 * su[::-1], x1 * sd[1:]])
    ys = [0.0]
    dy = y1
    for k in range(nj):
        rest = nj - k
        even = (height - ys[-1]) / rest
        if dy >= even:
            ys.extend(list(ys[-1] + even * np.arange(1, rest + 1)))
            break
        ys.append(ys[-1] + dy)
        dy *= growth
    y = np.array(ys[:nj + 1])
    y[-1] = height
    X, Y = np.meshgrid(x, y)
    pts, q, idx = _structured_quads(X, Y)
    i_le = n_up
    bottom = np.stack([idx[0, :-1], idx[0, 1:]], axis=1)
    markers = {
        "inlet": np.stack([idx[1:, 0], idx[:-1, 0]], axis=1),
        "outlet": np.stack([idx[:-1, -1], idx[1:, -1]], axis=1),
        "top": np.stack([idx[-1, 1:], idx[-1, :-1]], axis=1),
        "sym": bottom[:i_le],
        "plate": bottom[i_le:],
    }
    p = _pressure_for_re(re, mach, temperature, x1)
    kv = _flow_kv(mach, p, temperature)
    kv.update({"BC:inlet": "inlet", "BC:outlet": "outlet", "BC:top": "inlet", "BC:sym": "symmetry",
               "BC:plate": "wall"})
    kv.update(_solver_kv(viscous=viscous, **solver))
    return _su2(pts, list(q), markers), _input(kv)


def naca0012(x):
    """Closed-trailing-edge NACA 0012 half thickness at chord fraction x (four-digit series with the last
    coefficient -0.1036 so that y(1) = 0)."""
    return 0.6 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)


def airfoil(ncells=65536, mach=0.7, alpha_deg=2.0, y1=1e-6, far=100.0, tri_fraction=0.0, seed=0, viscous=None,
            re=None, temperature=300.0, **solver):
    """C-mesh around a NACA 0012 (chord 1, closed trailing edge): ni x nj quads with ni = 4 nj, wake to the
    far field, first cell height y1 with geometric growth, outer boundary a C of radius `far` around the
    leading edge. The wake cut shares nodes. Far field: characteristic inlet; airfoil: wall."""
    nj = max(4, int(round(math.sqrt(ncells / 4.0))))
    ni = 4 * nj
    nw = ni // 4                       # wake points per side
    na = ni - 2 * nw                   # airfoil intervals (even)
    # airfoil: cosine spacing, lower TE -> LE -> upper TE
    b = 0.5 * (1 - np.cos(np.linspace(0.0, math.pi, na // 2 + 1)))
    xl, xu = b[::-1], b[1:]
    ax = np.concatenate([xl, xu])
    ay = np.concatenate([-naca0012(xl), naca0012(xu)])
    # wake: geometric from the TE to x = 1 + far
    gw = np.geomspace(1e-3, far, nw)
    wx = 1.0 + gw
    inner_x = np.concatenate([wx[::-1], ax, wx])
    inner_y = np.concatenate([np.zeros(nw), ay, np.zeros(nw)])
    # outer C: lines y = -far and y = +far downstream of the trailing edge, joined by a half circle of
    # radius `far` around the trailing edge
    ang = np.linspace(-math.pi / 2, -3 * math.pi / 2, na + 1)
    outer_x = np.concatenate([wx[::-1], 1.0 + far * np.cos(ang), wx])
    outer_y = np.concatenate([-far * np.ones(nw), far * np.sin(ang), far * np.ones(nw)])
    n_in = inner_x.size
    # radial: geometric growth r with first spacing y1 over the distance `far` (bisection on r)
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if y1 * (r ** nj - 1) / (r - 1) > far:
            hi = r
        else:
            lo = r
    w = (r ** np.arange(nj + 1) - 1) / (r ** nj - 1)
    X = inner_x[None, :] + (outer_x - inner_x)[None, :] * w[:, None]
    Y = inner_y[None, :] + (outer_y - inner_y)[None, :] * w[:, None]
    pts, q, idx = _structured_quads(X, Y)
    # merge the wake cut and the trailing edge: node (j=0, i) and (j=0, n_in-1-i) coincide for i <= nw
    remap = np.arange(pts.shape[0])
    for i in range(nw + 1):
        remap[idx[0, n_in - 1 - i]] = idx[0, i]
    q = remap[q]
    used = np.unique(q)
    new = -np.ones(pts.shape[0], dtype=np.int64)
    new[used] = np.arange(used.size)
    q = new[q]
    pts = pts[used]
    cells = _ccw(pts, _mixed(q, tri_fraction, np.random.default_rng(seed)))
    ii = np.arange(nw, nw + na)
    wall = np.stack([new[remap[idx[0, ii + 1]]], new[remap[idx[0, ii]]]], axis=1)
    jo = nj
    nid = new[remap]
    far_edges = np.stack([nid[idx[jo, :-1]], nid[idx[jo, 1:]]], axis=1)
    left = np.stack([nid[idx[1:, 0]], nid[idx[:-1, 0]]], axis=1)
    right = np.stack([nid[idx[:-1, -1]], nid[idx[1:, -1]]], axis=1)
    markers = {"airfoil": wall, "far": np.concatenate([far_edges, left, right])}
    p = _pressure_for_re(re, mach, temperature, 1.0) if re else 1e5
    kv = _flow_kv(mach, p, temperature, alpha_deg)
    kv.update({"BC:airfoil": "wall", "BC:far": "inlet"})
    kv.update(_solver_kv(viscous=viscous, **solver))
    return _su2(pts, cells, markers), _input(kv)


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
    if pressure != 1e5:
        kv["pout"] = "%.17g" % pressure  # the outlet back pressure at the free stream's (default 1e5 Pa)
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
