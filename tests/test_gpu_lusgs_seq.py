"""LU-SGS against the reference's own sweeps (implicit.c:274-482): with CSU_LUSGS_ORDER=sequential the
engine colours one cell per colour in the reference's cell order, so its multicolour forward and backward
sweeps visit the cells exactly as implicitLUSGS_L / _U do, and a few iterations from the same state must
give the reference's state (Euler and laminar bit for bit; SA and SST within the last bits their
updates carry elsewhere too). Also the SST source Jacobians of the LU-SGS diagonal (sstInterSource, sst.c:643-680) against the
reference's arrays."""
import os

import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu

CASES = [
    ("caseWedge", {"order": "1", "timeScheme": "LUSGS", "CFL": "20.0"}, 0.0),
    ("caseWedgeQuad", {"order": "2", "timeScheme": "LUSGS", "CFL": "5.0"}, 0.0),
    ("caseBL", {"restart": "0", "timeScheme": "LUSGS", "CFL": "20.0"}, 0.0),
    ("caseBL_turb", {"restart": "0", "timeScheme": "LUSGS", "CFL": "20.0"}, 1e-14),
    ("caseBL_turb", {"restart": "0", "sa": "0", "sst": "1", "timeScheme": "LUSGS", "CFL": "20.0"}, 1e-14),
]


def _engine(wd, sequential):
    import csu_b200
    old = os.environ.get("CSU_LUSGS_ORDER")
    if sequential:
        os.environ["CSU_LUSGS_ORDER"] = "sequential"
    try:
        return csu_b200.Engine(csu_b200.Case.load(wd))
    finally:
        if old is None:
            os.environ.pop("CSU_LUSGS_ORDER", None)
        else:
            os.environ["CSU_LUSGS_ORDER"] = old


def _ref(wd):
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing")
    return Ref(wd)


@pytest.mark.parametrize("name,kv,tol", CASES,
                         ids=["wedge1", "wedgequad2", "bl", "bl_sa", "bl_sst"])
def test_lusgs_sequential_matches_reference(native, name, kv, tol):
    wd = casekit.materialize(name, kv)
    ref = _ref(wd)
    ref.iterate(10)
    U0 = ref.get_U()
    eng = _engine(wd, True)
    eng.set_state(U0)
    n = 3
    ref.iterate(n, 10)
    eng.iterate(n, it0=10)
    U, U_ref = eng.get_state(), ref.get_U()
    us = np.abs(U_ref).max(axis=1, keepdims=True) + 1e-300
    err = np.max(np.abs(U - U_ref) / us)
    print("\n%s: %d of %d state entries differ, max rel %.3e" % (name, np.count_nonzero(U != U_ref), U.size, err))
    if tol == 0.0:
        assert np.array_equal(U, U_ref)
    else:
        assert err < tol
    eng.close()


def test_sst_source_jacobians(native):
    wd = casekit.materialize("caseBL_turb", {"restart": "0", "sa": "0", "sst": "1", "timeScheme": "LUSGS",
                                             "CFL": "20.0"})
    ref = _ref(wd)
    ref.iterate(10)
    U0 = ref.get_U()
    ref.calc_R()
    J_ref = ref.sst_jac()
    eng = _engine(wd, False)
    eng.set_state(U0)
    eng.iterate(1)
    J = eng.dump("SST_JAC")
    scale = np.abs(J_ref).max(axis=1, keepdims=True) + 1e-300
    err = np.abs(J - J_ref) / scale
    print("\nSST Jacobians: max rel (to each row's scale) %s, %d nonzero rows entries" % (err.max(axis=1),
                                                                                    np.count_nonzero(J_ref)))
    assert np.count_nonzero(J_ref) > 0
    assert err.max() < 1e-8
    eng.close()
