"""The turbulent flat plate at full size (545 x 385 quads, first wall spacing 1e-6 m, growth 1.07, M 0.2,
Re_L 5e6, SA with nu_tilde_inf = 3 nu) against the reference solver, on the settings the reference supports
(AUSMDV, second order, Venkatakrishnan limiter, DPLUR 4 sweeps, FP64): 100 iterations of solverSolve
(solver.c:1864-1906) with the state within 1e-9 of each variable's scale and the residual history within
1e-9 relative (SA's pow/exp evaluations may differ in the last bit between CUDA and glibc)."""
import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu


def test_sa_plate_full_size_100_iterations(native):
    import csu_b200
    from csu_b200 import meshgen
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing")
    su2, inp = meshgen.plate(flux="AUSMDV", order=2, n_linear=4, cfl=1.0)
    wd = casekit.write_case(inp, su2, "saplate")
    case = csu_b200.Case.load(wd)
    assert case.n_cells == 545 * 385 and case.config.sa == 1
    eng = csu_b200.Engine(case)
    ref = Ref(wd)
    n = 100
    h_ref = ref.iterate(n)
    h = eng.iterate(n)
    nv = case.nvar
    assert np.isfinite(h).all() and np.isfinite(h_ref).all()
    rel = np.max(np.abs(h[:, :nv] - h_ref[:, :nv]) / np.abs(h_ref[:, :nv]))
    assert rel < 1e-9, rel
    U, U_ref = eng.get_state(), ref.get_U()
    us = np.abs(U_ref).max(axis=1, keepdims=True)
    assert np.max(np.abs(U - U_ref) / us) < 1e-9
    eng.close()
