"""Spalart-Allmaras path (sa.c) vs the reference on its SA flat-plate case (caseBL_turb)."""
import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu


def _setup(kv=None):
    import csu_b200
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing")
    kv = dict(casekit.GOLDEN_OVERRIDES["caseBL_turb"], **(kv or {}))
    wd = casekit.materialize("caseBL_turb", kv)
    case = csu_b200.Case.load(wd)
    return csu_b200.Engine(case), case, Ref(wd)


@pytest.mark.parametrize("blazek", ["0", "1"])
def test_sa_residual(native, blazek):
    eng, case, ref = _setup({"viscBlazek": blazek})
    ref.iterate(3)
    U = ref.get_U()
    eng.set_state(U)
    R_ref = ref.calc_R()
    R = eng.residual()
    S = np.abs(R_ref) + np.abs(R_ref).max(axis=1, keepdims=True) * 1e-3
    err = np.max(np.abs(R - R_ref) / S)
    diff = [np.count_nonzero(R[k] != R_ref[k]) for k in range(case.nvar)]
    print("SA blazek=%s: differing entries per variable %s, max scaled err %.3e" % (blazek, diff, err))
    assert err < 1e-12
    assert sum(diff[:4]) == 0


@pytest.mark.parametrize("scheme", ["RK", "DPLUR"])
def test_sa_history(native, scheme):
    kv = {"timeScheme": scheme}
    if scheme == "DPLUR":
        kv.update({"Nlinear": "4", "CFL": "1.0"})
    eng, case, ref = _setup(kv)
    n = 10
    h_ref = ref.iterate(n)
    h = eng.iterate(n)
    nv = case.nvar
    rel = np.max(np.abs(h[:, :nv] - h_ref[:, :nv]) / (np.abs(h_ref[:, :nv]) + 1e-300))
    U, U_ref = eng.get_state(), ref.get_U()
    same = np.count_nonzero(U != U_ref)
    print("SA %s: history max rel %.3e, state entries differing %d/%d" % (scheme, rel, same, U.size))
    assert rel < 1e-9
