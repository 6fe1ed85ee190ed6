"""Pins the plain-C restatement (oracle/csu_oracle.c) against the reference solver compiled from its own
sources (oracle/_ref), on the reference's example cases. CPU only."""
import numpy as np
import pytest

import casekit


@pytest.fixture(scope="module")
def oracle_lib():
    from oracle import restated
    restated.build()
    return restated


def _ref(wd):
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing (needs the reference tree)")
    return Ref(wd)


def _case(native, wd):
    import csu_b200
    return csu_b200.Case.load(wd)


@pytest.mark.parametrize("name", casekit.INVISCID)
def test_oracle_residual_bitexact(native, oracle_lib, name):
    wd = casekit.materialize(name, casekit.GOLDEN_OVERRIDES.get(name, {}))
    case = _case(native, wd)
    orc = oracle_lib.Oracle(case)
    ref = _ref(wd)
    R_ref = ref.calc_R()
    R = orc.residual()
    assert np.array_equal(orc.get("P"), ref.P())
    assert np.array_equal(orc.get("GHOST_P"), ref.ghost_P())
    assert np.array_equal(orc.get("GRAD"), ref.grad())
    if ref.order == 2:
        assert np.array_equal(orc.get("PHI"), ref.phi())
    assert np.array_equal(orc.get("FACEFLUX"), ref.faceflux())
    assert np.array_equal(R, R_ref)


@pytest.mark.parametrize("flux", ["ROE", "AUSM", "AUSMDV", "AUSMpup", "AUSMpup2"])
def test_oracle_fluxes(native, oracle_lib, flux):
    wd = casekit.materialize("caseCylinder", {"flux": flux})
    case = _case(native, wd)
    ref = _ref(wd)
    ref.iterate(2)
    U = ref.get_U()
    orc = oracle_lib.Oracle(case)
    orc.set_U(U)
    assert np.array_equal(orc.residual(), ref.calc_R())


@pytest.mark.parametrize("name", ["caseCylinder", "caseWedge", "caseWedgeQuad", "caseCylinderAxi"])
def test_oracle_history(native, oracle_lib, name):
    wd = casekit.materialize(name, casekit.GOLDEN_OVERRIDES.get(name, {}))
    case = _case(native, wd)
    orc = oracle_lib.Oracle(case)
    ref = _ref(wd)
    h_ref = ref.iterate(8)
    h = orc.iterate(8)
    nv = case.nvar
    assert np.array_equal(h[:, :nv], h_ref[:, :nv])
    assert np.allclose(h[:, nv:], h_ref[:, nv:], rtol=1e-13, atol=1e-300)
    assert np.array_equal(orc.get_U(), ref.get_U())


def test_oracle_tube(native, oracle_lib):
    wd = casekit.materialize("caseSod", {})
    case = _case(native, wd)
    orc = oracle_lib.Oracle(case)
    ref = _ref(wd)
    assert orc.tube(0.002) == ref.tube_run(0.002)
    assert np.array_equal(orc.get_U(), ref.get_U())


def test_oracle_golden(native, oracle_lib):
    """Against the committed reference vectors (usable where the reference tree is absent)."""
    import os
    for name in casekit.INVISCID:
        g = np.load(os.path.join(casekit.GOLDEN, "ref_%s.npz" % name))
        wd = casekit.materialize(name, casekit.GOLDEN_OVERRIDES.get(name, {}))
        case = _case(native, wd)
        orc = oracle_lib.Oracle(case)
        R = orc.residual()
        assert np.array_equal(R[:, g["sample"]], g["R_sample"])
        if len(g["hist"]):
            orc2 = oracle_lib.Oracle(case)
            h = orc2.iterate(len(g["hist"]))
            nv = case.nvar
            assert np.allclose(h[:, :nv], g["hist"][:, :nv], rtol=1e-12, atol=0)
