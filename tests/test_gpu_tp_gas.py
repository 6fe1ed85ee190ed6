"""Thermally perfect gas (`TP, 1`): the polynomial e(T) of gasprop.c:47-112 with its Newton inversion
(gasprop_e2T, gasprop.c:114-136) in every primitive recovery, speed of sound and gamma(T), against the
reference on its own cases: one residual bit for bit (primitives included) and 20 iterations with the state
bit for bit (RK on the wedge, DPLUR on the cylinder)."""
import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu


def _setup(name, kv):
    import csu_b200
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing")
    wd = casekit.materialize(name, dict(kv, TP="1"))
    case = csu_b200.Case.load(wd)
    assert case.config.tp == 1
    return csu_b200.Engine(case), case, Ref(wd)


@pytest.mark.parametrize("name,kv", [
    ("caseWedgeQuad", {}),
    ("caseCylinder", {"timeScheme": "DPLUR", "Nlinear": "4", "CFL": "4.0", "mach": "2.5"}),
])
def test_tp_gas_parity(native, name, kv):
    eng, case, ref = _setup(name, kv)
    # one residual at a non-uniform state
    ref.iterate(3)
    U = ref.get_U()
    eng.set_state(U)
    R_ref = ref.calc_R()
    R = eng.residual()
    assert np.array_equal(eng.dump("P"), ref.P())
    assert np.array_equal(R, R_ref)
    eng.close()
    # 20 iterations of both from the initial state (DPLUR warm-starts from its previous increment, so both
    # start fresh)
    eng, case, ref = _setup(name, kv)
    n = 20
    h_ref = ref.iterate(n)
    h = eng.iterate(n)
    assert np.array_equal(eng.get_state(), ref.get_U())
    nv = case.nvar
    assert np.max(np.abs(h[:, :nv] - h_ref[:, :nv]) / np.abs(h_ref[:, :nv])) < 1e-13
    eng.close()
