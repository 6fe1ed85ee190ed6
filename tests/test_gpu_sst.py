"""Menter SST path (sst.c) vs the reference, and its sstTrans variant (sstTrans.c). The reference ships no
SST case; its SA flat plate (caseBL_turb) is run with `sst, 1` instead (RK here; LU-SGS in
test_gpu_lusgs_seq.py; the reference's SST DPLUR multiplies 4x4 blocks into 6 variables,
implicit.c:993-1000 with 938-972, so it has no defined results)."""
import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu


def _setup(kv=None):
    import csu_b200
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing")
    kv = dict(casekit.GOLDEN_OVERRIDES["caseBL_turb"], sa="0", sst="1", **(kv or {}))
    wd = casekit.materialize("caseBL_turb", kv)
    case = csu_b200.Case.load(wd)
    return csu_b200.Engine(case), case, Ref(wd)


@pytest.mark.parametrize("trans", ["0", "1"], ids=["sst", "sstTrans"])
def test_sst_residual(native, trans):
    eng, case, ref = _setup({"sstTrans": trans})
    ref.iterate(3)
    U = ref.get_U()
    eng.set_state(U)
    R_ref = ref.calc_R()
    R = eng.residual()
    S = np.abs(R_ref) + np.abs(R_ref).max(axis=1, keepdims=True) * 1e-3
    err = np.max(np.abs(R - R_ref) / S)
    diff = [int(np.count_nonzero(R[k] != R_ref[k])) for k in range(case.nvar)]
    print("SST: differing entries per variable %s of %d, max scaled err %.3e" % (diff, case.n_cells, err))
    assert err < 1e-12
    if trans == "1":
        # the variant's sources and diffusion differ from the standard model's on the same state
        eng0, _, _ = _setup({"sstTrans": "0"})
        eng0.set_state(U)
        R0 = eng0.residual()
        assert not np.array_equal(R0[4:], R[4:])
        eng0.close()


@pytest.mark.parametrize("trans", ["0", "1"], ids=["sst", "sstTrans"])
def test_sst_history(native, trans):
    eng, case, ref = _setup({"sstTrans": trans})
    n = 10
    h_ref = ref.iterate(n)
    h = eng.iterate(n)
    nv = case.nvar
    rel = np.max(np.abs(h[:, :nv] - h_ref[:, :nv]) / (np.abs(h_ref[:, :nv]) + 1e-300))
    print("SST RK: history max rel %.3e" % rel)
    assert rel < 1e-9
