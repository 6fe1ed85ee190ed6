"""DPLUR pieces of one iteration, CUDA vs the reference, compared bit for bit where the arithmetic is the
same (residual, Omega/Lc, diagonal, finite-difference blocks) and to 1e-12 for the increment."""
import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu


def _setup(name, kv):
    import csu_b200
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing")
    wd = casekit.materialize(name, kv)
    case = csu_b200.Case.load(wd)
    return csu_b200.Engine(case), case, Ref(wd)


def _report(tag, a, b):
    d = np.abs(a - b)
    s = np.abs(b) + 1e-300
    bad = np.count_nonzero(a != b)
    return "%s: %d/%d differ, max rel %.3e" % (tag, bad, a.size, np.max(d / s) if bad else 0.0)


@pytest.mark.parametrize("name", ["caseWedge", "caseCylinder"])
def test_dplur_first_iteration(native, name):
    eng, case, ref = _setup(name, {"timeScheme": "DPLUR", "Nlinear": "4", "CFL": "10.0"})
    R_ref = ref.calc_R()
    D_ref, dtl_ref = ref.implicit_D()
    A_ref = ref.implicit_A()
    eng.iterate(1)
    msgs = []
    R = eng.dump("R")
    msgs.append(_report("R", R, R_ref))
    msgs.append(_report("DTL", eng.dump("DTL"), dtl_ref))
    msgs.append(_report("D", eng.dump("D"), D_ref))
    A = eng.dump("BLOCKS")
    mask = np.arange(4)[None, :] < case.cell_nint[:, None]
    msgs.append(_report("BLOCKS", A[mask], A_ref[mask]))
    # the reference increment of the same iteration (fresh instance: dW starts at zero)
    from oracle.refharness import Ref
    ref2 = Ref(casekit.materialize(name, {"timeScheme": "DPLUR", "Nlinear": "4", "CFL": "10.0"}))
    ref2.calc_R()
    dW_ref = ref2.implicit_dplur()
    dW = eng.dump("DW")
    msgs.append(_report("DW", dW, dW_ref))
    print("\n".join(msgs))
    sc = np.abs(dW_ref).max(axis=1, keepdims=True)
    assert np.max(np.abs(dW - dW_ref) / sc) < 1e-12, "\n".join(msgs)
    assert np.array_equal(A[mask], A_ref[mask]), "\n".join(msgs)
