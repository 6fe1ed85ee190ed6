"""CUDA path vs the reference solver (oracle/_ref) on the synthetic meshes of csu_b200.meshgen (the
serving workload's families: mixed tri/quad bump channel, cylinder O-grid, NACA 0012 C-mesh with wake cut,
jittered ramp), inviscid and laminar, DPLUR: one residual evaluation, the first iteration's DPLUR pieces,
and the state after 20 iterations."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = {
    "bump_inv": ("bump", dict(ncells=3000, mach=0.5)),
    "bump_lam": ("bump", dict(ncells=3000, mach=1.9, viscous="laminar", re=2e4)),
    "cyl_inv": ("cylinder", dict(ncells=2500, mach=2.2)),
    "cyl_lam": ("cylinder", dict(ncells=2500, mach=1.6, viscous="laminar", re=5e3)),
    "naca_inv": ("airfoil", dict(ncells=3000, mach=0.7, alpha_deg=2.0, y1=1e-4)),
    "naca_lam": ("airfoil", dict(ncells=3000, mach=0.5, alpha_deg=-1.0, y1=1e-4, viscous="laminar", re=1e4)),
}


def _wd(name):
    from csu_b200 import meshgen
    fn, kw = CASES[name]
    su2, inp = getattr(meshgen, fn)(order=1, flux="AUSMDV", cfl=5.0, **kw)
    wd = "/tmp/csu_gen_%s/" % name
    return meshgen.write_case(wd, su2, inp)


def _ref(wd):
    from oracle.refharness import Ref, available
    if not available():
        pytest.skip("reference build oracle/_ref missing")
    return Ref(wd)


@pytest.mark.parametrize("name", sorted(CASES))
def test_generated_residual_and_dplur(native, name):
    import csu_b200
    wd = _wd(name)
    ref = _ref(wd)
    case = csu_b200.Case.load(wd)
    eng = csu_b200.Engine(case)
    R_ref = ref.calc_R()
    R = eng.residual()
    scale = np.abs(R_ref).max(axis=1, keepdims=True) + 1e-300
    err_r = np.max(np.abs(R - R_ref) / scale)
    eng.iterate(1)
    ref2 = _ref(wd)
    ref2.calc_R()
    D_ref, _ = ref2.implicit_D()
    dW_ref = ref2.implicit_dplur()
    D, dW = eng.dump("D"), eng.dump("DW")
    err_d = np.max(np.abs(D - D_ref) / np.abs(D_ref))
    err_w = np.max(np.abs(dW - dW_ref) / (np.abs(dW_ref).max(axis=1, keepdims=True) + 1e-300))
    print("\n%s: R %.2e, D %.2e, dW %.2e" % (name, err_r, err_d, err_w))
    assert err_r < 1e-12 and err_d < 1e-12 and err_w < 1e-10
    eng.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_generated_history(native, name):
    import csu_b200
    wd = _wd(name)
    ref = _ref(wd)
    eng = csu_b200.Engine(csu_b200.Case.load(wd))
    h = eng.iterate(20)
    U = eng.get_state()
    h_ref = np.asarray(ref.iterate(20, 0))
    U_ref = ref.get_U()
    scale = np.abs(U_ref).max(axis=1, keepdims=True)
    err = np.max(np.abs(U - U_ref) / scale)
    print("\n%s: state after 20 iterations %.2e, rho residual %s vs %s" % (name, err, h[-1, 0], h_ref[-1, 0]))
    assert np.all(np.isfinite(U))
    assert err < 1e-9
    eng.close()
