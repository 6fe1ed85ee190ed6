"""More extensions (not in the reference; off by default): 2-stage RK, the Barth-Jespersen (minmod) limiter
function, Green-Gauss gradients. The 2-stage RK is checked bit for bit against the CPU restatement
(oracle/csu_oracle.c, which restates it the same way); the Sod configuration (Roe, minmod, 2-stage RK,
CFL 0.5) against the exact Riemann solution; Green-Gauss against the exact gradient of a linear field on a
rectangular grid."""
import math

import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu

GAMMA = 1.4


def _exact_sod(x, t, rl=1.0, pl=1.0, rr=0.125, pr=0.1, x0=0.5):
    """Exact solution of the Riemann problem with zero initial velocities (pressure from Newton iterations on
    the star-region pressure function; rarefaction, contact, shock)."""
    g = GAMMA
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)

    def f(p, rk, pk, ck):
        if p > pk:
            a, b = 2 / ((g + 1) * rk), (g - 1) / (g + 1) * pk
            return (p - pk) * math.sqrt(a / (p + b)), math.sqrt(a / (b + p)) * (1 - (p - pk) / (2 * (b + p)))
        r = p / pk
        return 2 * ck / (g - 1) * (r ** ((g - 1) / (2 * g)) - 1), r ** (-(g + 1) / (2 * g)) / (rk * ck)

    p = 0.5 * (pl + pr)
    for _ in range(100):
        fl, dl = f(p, rl, pl, cl)
        fr, dr = f(p, rr, pr, cr)
        dp = (fl + fr) / (dl + dr)
        p = max(p - dp, 1e-12)
        if abs(dp) < 1e-14 * p:
            break
    u = 0.5 * (f(p, rr, pr, cr)[0] - f(p, rl, pl, cl)[0])
    rsl = rl * (p / pl) ** (1 / g)                             # left rarefaction
    rsr = rr * ((p / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * p / pr + 1))  # right shock
    s = math.sqrt(pr * g / rr) * math.sqrt((g + 1) / (2 * g) * p / pr + (g - 1) / (2 * g))
    csl = cl * (p / pl) ** ((g - 1) / (2 * g))
    out = np.empty_like(x)
    for i, xi in enumerate(x):
        w = (xi - x0) / t
        if w < -cl:
            out[i] = rl
        elif w < u - csl:
            out[i] = rl * (2 / (g + 1) + (g - 1) / ((g + 1) * cl) * (-w)) ** (2 / (g - 1))
        elif w < u:
            out[i] = rsl
        elif w < s:
            out[i] = rsr
        else:
            out[i] = rr
    return out


def test_rk2_matches_restatement(native):
    import csu_b200
    from oracle.restated import Oracle, available
    if not available():
        pytest.skip("oracle not built")
    for name, kv, tube in [("caseSod", {"stages": "2"}, True), ("caseWedge", {"stages": "2", "timeScheme": "RK",
                                                                                "CFL": "0.5"}, False)]:
        wd = casekit.materialize(name, kv)
        case = csu_b200.Case.load(wd)
        eng, orc = csu_b200.Engine(case), Oracle(case)
        if tube:
            s1, t1 = eng.tube_run(0.002)
            s2, t2 = orc.tube(0.002)
            assert s1 == s2 and t1 == t2
        else:
            h1, h2 = eng.iterate(20), orc.iterate(20)
            assert np.max(np.abs(h1[:, 0] - h2[:, 0]) / h2[:, 0]) < 1e-13
        U1, U2 = eng.get_state(), orc.get_U()
        assert np.array_equal(U1, U2), "%s: %d state entries differ" % (name, np.count_nonzero(U1 != U2))
        eng.close()


def test_sod_roe_minmod_rk2(native):
    """The Sod configuration: 1000 x 2 quads split into 4,000 triangles, Roe, minmod (Barth-Jespersen
    limiter function), 2-stage RK, CFL 0.5, t = 0.2 (run dimensionally: p scaled by 1e5)."""
    import csu_b200
    from csu_b200 import meshgen
    su2, inp = meshgen.sod_tube(flux="ROE", order=2, stages=2, cfl=0.5)
    inp += "limiterFunc, 1\n"
    case = csu_b200.Case.from_text(inp, su2)
    eng = csu_b200.Engine(case)
    tmax = case.get_double("tmax")
    steps, t = eng.tube_run(tmax)
    U = eng.get_state()
    xc = case.xy[case.cell_nodes[:, :3], 0].mean(axis=1)
    rho = U[0]
    t_nd = t * math.sqrt(1e5)   # nondimensional time (p scaled by 1e5, rho by 1)
    exact = _exact_sod(xc, t_nd)
    l1 = np.mean(np.abs(rho - exact))
    print("\nSod: %d steps to t = %.6g (nondimensional %.4f); L1(rho) = %.4e, rho in [%.6f, %.6f]"
          % (steps, t, t_nd, l1, rho.min(), rho.max()))
    assert abs(t_nd - 0.2) < 1e-9
    assert l1 < 5e-3
    assert rho.min() > 0.125 - 1e-3 and rho.max() < 1.0 + 1e-3
    eng.close()


def test_green_gauss_linear_field(native):
    """On a rectangular grid the Green-Gauss gradient of a linear field is exact in interior cells."""
    import csu_b200
    from csu_b200 import meshgen
    ni, nj = 60, 20
    X, Y = np.meshgrid(np.linspace(0.0, 3.0, ni + 1), np.linspace(0.0, 1.0, nj + 1))
    pts, q, idx = meshgen._structured_quads(X, Y)
    markers = {"inlet": np.stack([idx[1:, 0], idx[:-1, 0]], axis=1),
               "outlet": np.stack([idx[:-1, -1], idx[1:, -1]], axis=1),
               "top": np.stack([idx[-1, 1:], idx[-1, :-1]], axis=1),
               "wall": np.stack([idx[0, :-1], idx[0, 1:]], axis=1)}
    su2 = meshgen._su2(pts, list(q), markers)
    kv = meshgen._flow_kv(0.5, 1e5, 300.0)
    kv.update({"BC:inlet": "inlet", "BC:outlet": "outlet", "BC:top": "symmetry", "BC:wall": "wall"})
    kv.update(meshgen._solver_kv(order=2))
    inp = meshgen._input(kv) + "gradient, 1\n"
    case = csu_b200.Case.from_text(inp, su2)
    nodes = case.cell_nodes
    xc = case.xy[nodes, 0].mean(axis=1)
    yc = case.xy[nodes, 1].mean(axis=1)
    rho = 1.0 + 0.1 * xc + 0.05 * yc
    u = 100.0 + 20.0 * xc - 10.0 * yc
    v = 5.0 + 3.0 * xc + 7.0 * yc
    p = 1e5 * (1.0 + 0.02 * xc - 0.03 * yc)
    U = np.stack([rho, rho * u, rho * v, p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v)])
    eng = csu_b200.Engine(case, state=U)
    eng.residual()
    G = eng.dump("GRAD")
    inner = (xc > 0.1) & (xc < 2.9) & (yc > 0.1) & (yc < 0.9)
    for k, (gx, gy) in enumerate([(0.1, 0.05), (20.0, -10.0), (3.0, 7.0), (2e3, -3e3)]):
        ex = np.max(np.abs(G[0, k, inner] - gx)) / (abs(gx) + abs(gy))
        ey = np.max(np.abs(G[1, k, inner] - gy)) / (abs(gx) + abs(gy))
        assert ex < 1e-8 and ey < 1e-8, (k, ex, ey)
    eng.close()
