"""LU-SGS (implicit.c:274-482) as a multicolour Gauss-Seidel, checked at convergence: the reference sweeps
cells in index order, the device sweeps colour groups, so the paths differ but the converged first-order
solutions must agree."""
import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,kv", [("caseWedge", {"order": "1"}),
                                     ("caseWedgeQuad", {"order": "1", "timeScheme": "LUSGS", "CFL": "50.0"})])
def test_lusgs_converged_solution(native, name, kv):
    import csu_b200
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing")
    wd = casekit.materialize(name, kv)
    case = csu_b200.Case.load(wd)
    eng = csu_b200.Engine(case)
    ref = Ref(wd)
    n = 1200
    h_ref = ref.iterate(n)
    h = eng.iterate(n)
    nv = case.nvar
    drop = h[-1, :nv] / h[0, :nv]
    drop_ref = h_ref[-1, :nv] / h_ref[0, :nv]
    U, U_ref = eng.get_state(), ref.get_U()
    us = np.abs(U_ref).max(axis=1, keepdims=True)
    err = np.max(np.abs(U - U_ref) / us)
    print("%s: residual drop %s (reference %s), converged state max rel diff %.3e" % (name, drop, drop_ref, err))
    assert np.all(drop < 1e-11) and np.all(drop_ref < 1e-11)
    assert err < 1e-10
