"""Spalart-Allmaras path (sa.c) and its saCC variant (saCC.c: the density-gradient terms) vs the reference
on its SA flat-plate case (caseBL_turb)."""
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


@pytest.mark.parametrize("blazek,cc", [("0", "0"), ("1", "0"), ("0", "1")], ids=["sa", "sa_blazek", "saCC"])
def test_sa_residual(native, blazek, cc):
    eng, case, ref = _setup({"viscBlazek": blazek, "saCC": cc})
    ref.iterate(3)
    U = ref.get_U()
    eng.set_state(U)
    R_ref = ref.calc_R()
    R = eng.residual()
    S = np.abs(R_ref) + np.abs(R_ref).max(axis=1, keepdims=True) * 1e-3
    err = np.max(np.abs(R - R_ref) / S)
    diff = [np.count_nonzero(R[k] != R_ref[k]) for k in range(case.nvar)]
    print("SA blazek=%s saCC=%s: differing entries per variable %s, max scaled err %.3e" % (blazek, cc, diff, err))
    assert err < 1e-12
    assert sum(diff[:4]) == 0
    if cc == "1":
        # the variant's diffusion and source differ from the plain model's on the same state
        eng0, _, _ = _setup({"viscBlazek": blazek})
        eng0.set_state(U)
        assert not np.array_equal(eng0.residual()[4], R[4])
        eng0.close()


@pytest.mark.parametrize("scheme,cc", [("RK", "0"), ("DPLUR", "0"), ("RK", "1"), ("DPLUR", "1")],
                         ids=["rk", "dplur", "rk_saCC", "dplur_saCC"])
def test_sa_history(native, scheme, cc):
    kv = {"timeScheme": scheme, "saCC": cc}
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
