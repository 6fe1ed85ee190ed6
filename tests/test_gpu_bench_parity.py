"""The benchmarked configuration against the reference solver (oracle/_ref) at its full size.

Case: the 15 degree compression ramp, 400 x 200 quads split into 160,000 triangles, interior nodes jittered
+-10 % (numpy default_rng(0)), M 2.5, p 1e5 Pa, T 300 K, AUSM, order 2, Venkatakrishnan K = 5, DPLUR with
4 sweeps, CFL 5, FP64 -- the case `bench.py` times, built by the same `bench.make_case`.

Bars: one residual evaluation bit-identical (and within 1e-12 of each cell's flux scale); 100 DPLUR
iterations (solverSolve, solver.c:1864-1906; implicitCalcDPLUR, implicit.c:990-1034) with the state bit-
identical to the reference's, the RMS residual history within 1e-13 relative (the device sums the squares
in another order than solverCalcRes, solver.c:867-892) and Cx/Cy within 1e-9 of their scale.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_ITER = 100


def _ref(wd):
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing")
    return Ref(wd)


@pytest.fixture(scope="module")
def bench_case(native):
    import bench
    return bench.make_case(os.cpu_count() or 1, "par")


def test_bench_residual_bit_identical(bench_case):
    import csu_b200
    case = csu_b200.Case.load(bench_case)
    assert case.n_cells == 160000
    eng = csu_b200.Engine(case)
    ref = _ref(bench_case)
    R_ref = ref.calc_R()
    R = eng.residual()
    assert np.array_equal(R, R_ref)
    assert np.array_equal(eng.dump("P"), ref.P())
    ff, ff_ref = eng.dump("FACEFLUX"), ref.faceflux()
    assert np.array_equal(ff, ff_ref)
    eng.close()


def test_bench_history_100_iterations(bench_case):
    import csu_b200
    case = csu_b200.Case.load(bench_case)
    eng = csu_b200.Engine(case)
    ref = _ref(bench_case)
    h_ref = ref.iterate(N_ITER)
    h = eng.iterate(N_ITER)
    nv = case.nvar
    assert np.isfinite(h).all() and np.isfinite(h_ref).all()
    # the run moves: the residual changes from the start (the shock system forms over these iterations)
    assert h_ref[-1, 0] < h_ref[0, 0]
    assert np.array_equal(eng.get_state(), ref.get_U())
    rel = np.max(np.abs(h[:, :nv] - h_ref[:, :nv]) / np.abs(h_ref[:, :nv]))
    assert rel < 1e-13, rel
    cs = np.abs(h_ref[:, nv:]).max() + 1e-300
    assert np.max(np.abs(h[:, nv:] - h_ref[:, nv:])) / cs < 1e-9
    eng.close()
