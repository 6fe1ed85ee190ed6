"""The certified double-double least squares (default) against the x87 model on every component
(CSU_LSQ=x87): gradients, limiters and states bit-identical over several iterations, on inviscid,
laminar, SA and SST cases; and how many slots the FP64 path leaves to the integer x87 model."""
import os

import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu

CASES = [
    ("caseWedge", {}),
    ("caseCylinder", {}),
    ("caseWedgeQuad", {"order": "2"}),
    ("caseBL", {"restart": "0"}),
    ("caseNACA0012", {"restart": "0"}),
    ("caseBL_turb", {"restart": "0"}),
    ("caseBL_turb", {"restart": "0", "sa": "0", "sst": "1"}),
]


def _run(name, kv, mode, iters):
    import csu_b200
    old = os.environ.get("CSU_LSQ")
    if mode:
        os.environ["CSU_LSQ"] = mode
    else:
        os.environ.pop("CSU_LSQ", None)
    try:
        eng = csu_b200.Engine(csu_b200.Case.load(casekit.materialize(name, kv)))
    finally:
        if old is None:
            os.environ.pop("CSU_LSQ", None)
        else:
            os.environ["CSU_LSQ"] = old
    out = {"R0": eng.residual()}
    out["GRAD0"], out["PHI0"] = eng.dump("GRAD"), eng.dump("PHI")
    eng.iterate(iters)
    out["GRAD"], out["PHI"], out["U"] = eng.dump("GRAD"), eng.dump("PHI"), eng.get_state()
    out["x87"] = eng.dump("LSQ_X87")[0]
    out["ncomp"] = 2 * eng.nvar * eng.n_cells  # per gradient evaluation (upper bound with T)
    eng.close()
    return out


@pytest.mark.parametrize("name,kv", CASES, ids=["%s%s" % (n, "_sst" if k.get("sst") else "") for n, k in CASES])
def test_certified_lsq_equals_x87_model(native, name, kv):
    ref = _run(name, kv, "x87", 10)
    got = _run(name, kv, None, 10)
    for k in ("R0", "GRAD0", "PHI0", "GRAD", "PHI", "U"):
        a, b = got[k], ref[k]
        same = np.array_equal(a, b) or np.array_equal(np.nan_to_num(a), np.nan_to_num(b))
        assert same, "%s: %d entries differ" % (k, np.count_nonzero(a != b))
    print("\n%s: %d (cell, variable) gradients left to the integer x87 model over the residual and 10 "
          "iterations (%d cells x %d variables)" % (name, got["x87"], got["ncomp"] // (2 * len(got["R0"])),
                                                      len(got["R0"])))
