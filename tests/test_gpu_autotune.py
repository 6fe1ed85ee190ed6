"""Launch-shape autotuner (csu_autotune): the face-chunk size of the flux kernel and the cell-block size of
the DPLUR sweeps are picked by timing on the solve itself; whatever it picks, every result bit is the same
as with the default shapes (fluxes are per face, sweeps per cell, partial norms one row per warp)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case():
    import csu_b200
    from csu_b200 import meshgen
    su2, inp = meshgen.ramp(ni=160, nj=80, n_linear=4, cfl=5.0)  # 25,600 cells: above the tuning threshold
    return csu_b200.Case.from_text(inp, su2)


def test_autotuned_shapes_change_no_bit(native):
    import csu_b200
    case = _case()
    n = 24
    os.environ["CSU_AUTOTUNE"] = "0"
    try:
        ref = csu_b200.Engine(case)
        h_ref = ref.iterate(n)
        U_ref = ref.get_state()
        ref.close()
    finally:
        del os.environ["CSU_AUTOTUNE"]
    eng = csu_b200.Engine(case)
    h1 = eng.iterate(n // 2)          # tunes itself on its first iteration
    fb, sb = eng.autotune()           # and once more, explicitly, in the middle of the run
    assert fb in (32, 64, 128) and sb in (64, 128, 256)
    h2 = eng.iterate(n - n // 2, it0=n // 2)
    assert np.array_equal(np.vstack([h1, h2]), h_ref)
    assert np.array_equal(eng.get_state(), U_ref)
    eng.close()


def test_retuning_between_calls_same_bits(native):
    """Re-timing between calls (which may switch shapes and recapture the iteration graphs) leaves every
    continuation bit-identical to an engine that keeps its first choice."""
    import csu_b200
    case = _case()
    eng_a = csu_b200.Engine(case)
    eng_b = csu_b200.Engine(case)
    for k in range(3):
        eng_a.iterate(8, it0=8 * k)
        eng_b.autotune()
        eng_b.iterate(8, it0=8 * k)
        assert np.array_equal(eng_a.get_state(), eng_b.get_state())
    eng_a.close()
    eng_b.close()
