"""Failure paths, injected on the host (nothing here faults or hangs a GPU): a non-finite value written into
the caller's state before upload, one poisoned solve in a pack, a request over the memory budget, a
cancelled request. Each failure must be reported with its status (include/csu_gpu.h) while the rest of the
work goes on exactly as it would without it."""
import time

import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu

STRUCT = {"timeScheme": "DPLUR", "Nlinear": "4", "order": "1", "flux": "AUSMDV", "restart": "0"}
# flow conditions the first-order DPLUR runs stably with (as in the serving tests)
FLOW = {"caseWedge": {"CFL": "10.0"}, "caseCylinder": {"CFL": "4.0", "mach": "2.5"},
        "caseWedgeQuad": {"CFL": "8.0", "mach": "2.2"}, "caseDiamond": {"CFL": "5.0"}}


def _case(name, kv=None):
    import csu_b200
    return csu_b200.Case.load(casekit.materialize(name, dict(STRUCT, **FLOW[name], **(kv or {}))))


def test_nonfinite_state_before_upload(native):
    """NaN in one cell's x momentum of the uploaded state: the first iteration after it reports
    CSU_ERR_NONFINITE (status 4) with its iteration number, and no later iteration runs. (A NaN density or
    energy would not do: the write-back clamps of solverCalcPrimitive, solver.c:1163-1202, are fmax calls,
    which return rLim or the energy floor for a NaN operand, in the reference and here alike.)"""
    import csu_b200
    case = _case("caseWedge")
    eng = csu_b200.Engine(case)
    eng.iterate(3)
    U = eng.get_state()
    U[1, case.n_cells // 2] = np.nan
    eng.set_state(U)
    with pytest.raises(csu_b200.CsuError) as e:
        eng.iterate(5, it0=3)
    assert e.value.status == 4
    assert "iteration 4" in str(e.value)
    # the device halted the solve: asking again changes nothing and reports the same status
    with pytest.raises(csu_b200.CsuError) as e2:
        eng.iterate(2, it0=4)
    assert e2.value.status == 4
    eng.close()


def test_nonfinite_solve_frozen_in_pack(native):
    """One solve of a pack starts from a state with an infinite energy: it is frozen with its status set at
    its first iteration, while the other solves' iterations are bit-identical to their runs alone."""
    import csu_b200
    names = ["caseWedge", "caseCylinder", "caseWedgeQuad"]
    preps = [csu_b200.Prep(_case(nm)) for nm in names]
    pack = csu_b200.Pack(preps)
    bad = preps[1].state.copy()
    bad[3, 7] = np.inf
    pack.set_state(1, bad)
    n = 24
    pack.iterate(n)
    info = pack.info(1)
    assert info["status"] == 4 and info["iter"] == 1
    for k in (0, 2):
        eng = csu_b200.Engine(_case(names[k]))
        eng.iterate(n)
        assert pack.info(k)["status"] == 0 and pack.info(k)["iter"] == n
        assert np.array_equal(pack.get_state(k), eng.get_state())
        eng.close()
    pack.close()


@pytest.mark.parametrize("prep_threads", [0, 2])
def test_request_over_budget(native, prep_threads):
    """A request whose device bytes exceed the server's whole budget: refused at submission
    (CSU_ERR_OOM) when the caller's thread prepares it, or ended CSU_SRV_FAILED with status CSU_ERR_OOM and
    a message when a preparation thread found it."""
    import csu_b200
    srv = csu_b200.Server(1 << 20, iters_per_step=8, prep_threads=prep_threads)
    case = _case("caseDiamond")
    if prep_threads == 0:
        with pytest.raises(csu_b200.CsuError) as e:
            srv.submit(case, max_iters=16)
        assert e.value.status == 3
    else:
        rid = srv.submit(case, max_iters=16)
        t0 = time.time()
        while srv.info(rid)["state"] == "queued" and time.time() - t0 < 60.0:
            srv.step()
            time.sleep(0.01)
        info = srv.info(rid)
        assert info["state"] == "failed" and info["status"] == 3
        assert "budget" in srv.message(rid)
    srv.close()


def test_cancel_running_and_queued(native):
    """Cancelling a running request stops it where it stands and its pack is rebuilt without it; a queued
    request never starts; the other requests end exactly as they would alone."""
    import csu_b200
    kv = {"convDrop": "1e-4"}
    names = ["caseWedge", "caseCylinder", "caseWedgeQuad"]
    srv = csu_b200.Server(4096 << 20, iters_per_step=8, max_pack=3)
    ids = [srv.submit(_case(nm, kv), max_iters=400) for nm in names]
    late = srv.submit(_case("caseDiamond", kv), max_iters=400)  # queued: the pack is full
    srv.step()
    srv.step()
    assert srv.info(ids[1])["state"] == "running" and srv.info(late)["state"] == "queued"
    srv.cancel(ids[1])
    srv.cancel(late)
    info = srv.info(ids[1])
    assert info["state"] == "cancelled" and info["status"] == 6 and info["iters"] == 16
    assert srv.info(late)["state"] == "cancelled"
    with pytest.raises(csu_b200.CsuError):
        srv.cancel(ids[1])
    U_cancelled = srv.take(ids[1])
    srv.take(late)
    for _ in range(1000):
        running, queued = srv.step()
        if running == 0 and queued == 0:
            break
    for k in (0, 2):
        info = srv.info(ids[k])
        U = srv.take(ids[k])
        eng = csu_b200.Engine(_case(names[k], kv))
        h = eng.iterate_until(400)
        assert info["iters"] == len(h)
        assert np.array_equal(U, eng.get_state())
        eng.close()
    # the cancelled solve's state is its state after the 16 iterations it ran
    eng = csu_b200.Engine(_case(names[1], kv))
    eng.iterate(16)
    assert np.array_equal(U_cancelled, eng.get_state())
    eng.close()
    srv.close()
