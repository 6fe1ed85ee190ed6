"""State upload and read-back through the C ABI for one-solve contexts: one copy of the caller's array each
way and the renumbering on the device. A round trip returns the caller's array bit for bit, into a new
array or into a buffer the caller passes (pinned host memory here, written by DMA)."""
import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,kv", [("caseWedgeQuad", {}), ("caseBL_turb", {"restart": "0"})])
def test_state_roundtrip(native, name, kv):
    import torch

    import csu_b200
    eng = csu_b200.Engine(csu_b200.Case.load(casekit.materialize(name, kv)))
    U0 = eng.get_state()
    rng = np.random.default_rng(1)
    U = U0 * (1.0 + 0.01 * rng.standard_normal(U0.shape))
    eng.set_state(U)
    assert np.array_equal(eng.get_state(), U)
    pin = torch.empty(U.shape, dtype=torch.float64).pin_memory().numpy()
    assert eng.get_state(out=pin) is pin
    assert np.array_equal(pin, U)
    # the state set from a pinned buffer iterates like the one set from pageable memory
    eng.set_state(pin)
    h1 = eng.iterate(3)
    eng.set_state(U)
    h2 = eng.iterate(3)
    assert np.array_equal(h1, h2)
    with pytest.raises(ValueError):
        eng.get_state(out=np.empty((1, 1)))
    eng.close()
