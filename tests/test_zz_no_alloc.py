"""csu_residual_norms_noalloc: residual RMS norms for callers that cannot let the library allocate device
memory (their device memory is a fixed budget under their own allocator, or cudaMalloc/cudaFree would
synchronize the device under their other work). Checked through the C ABI against the norms the engine
itself records for the same residual (csu_iterate's history row) and against a plain FP64 numpy sum of
solverCalcRes's quantity (solver.c:867-892) on seeded residuals up to the 8,388,608-cell limit, each on two
calls in a row. This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu


def test_no_alloc_norms_match_engine(native):
    import torch
    import csu_b200
    wd = casekit.materialize("caseWedge", casekit.GOLDEN_OVERRIDES["caseWedge"])
    case = csu_b200.Case.load(wd)
    eng = csu_b200.Engine(case)
    hist = eng.iterate(1)
    want = hist[0, :case.nvar]
    R = eng.dump("R")
    R_dev = torch.from_numpy(np.ascontiguousarray(R)).to("cuda")
    res_dev = torch.empty(case.nvar, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    L = csu_b200.lib()
    for _ in range(2):
        res_dev.fill_(float("nan"))
        st = L.csu_residual_norms_noalloc(C.c_void_p(R_dev.data_ptr()), case.nvar, case.n_cells,
                                          C.c_void_p(res_dev.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == 0, L.csu_last_error()
        torch.cuda.synchronize()
        got = res_dev.cpu().numpy()
        assert np.allclose(got, want, rtol=1e-12, atol=0), (got, want)


@pytest.mark.parametrize("ncells", [600000, 8388608])
@pytest.mark.parametrize("nvar", [4, 6])
def test_no_alloc_norms_match_numpy(native, ncells, nvar):
    """Sizes where the final kernel's threads each sum several partials (more than 256 partial blocks), up to
    exactly the largest size the fixed scratch holds (4,096 partial blocks)."""
    import torch
    import csu_b200
    rng = np.random.default_rng(ncells + nvar)
    R = rng.standard_normal((nvar, ncells)) * np.logspace(-8, 2, nvar)[:, None]
    want = np.sqrt((R ** 2).sum(axis=1) / ncells)
    R_dev = torch.from_numpy(R).to("cuda")
    res_dev = torch.empty(nvar, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    L = csu_b200.lib()
    for _ in range(2):
        res_dev.fill_(float("nan"))
        st = L.csu_residual_norms_noalloc(C.c_void_p(R_dev.data_ptr()), nvar, ncells,
                                          C.c_void_p(res_dev.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == 0, L.csu_last_error()
        torch.cuda.synchronize()
        got = res_dev.cpu().numpy()
        assert np.allclose(got, want, rtol=1e-12, atol=0), (got, want)


def test_no_alloc_rejects_oversize(native):
    import torch
    import csu_b200
    R_dev = torch.zeros(8, dtype=torch.float64, device="cuda")
    res_dev = torch.zeros(4, dtype=torch.float64, device="cuda")
    L = csu_b200.lib()
    st = L.csu_residual_norms_noalloc(C.c_void_p(R_dev.data_ptr()), 4, 8388608 + 1, C.c_void_p(res_dev.data_ptr()),
                                      None)
    assert st == 1
    assert b"exceed" in L.csu_last_error()
    st = L.csu_residual_norms_noalloc(C.c_void_p(R_dev.data_ptr()), 7, 8, C.c_void_p(res_dev.data_ptr()), None)
    assert st == 1
