"""Serving layer: requests arriving over time are admitted, packed with the running solves (which move
between packs as membership changes), retired at their residual drop; each result equals the solve run
alone, bit for bit. Requests of two classes (different orders) run in separate packs; a tight budget
makes requests wait for admission."""
import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu

BASE = {"timeScheme": "DPLUR", "Nlinear": "4", "flux": "AUSMDV", "restart": "0", "convDrop": "1e-5"}
REQUESTS = [
    ("caseWedge", {"order": "1", "CFL": "10.0"}),
    ("caseCylinder", {"order": "1", "CFL": "4.0", "mach": "2.5"}),
    ("caseWedgeQuad", {"order": "1", "CFL": "8.0", "mach": "2.2"}),
    ("caseDiamond", {"order": "2", "CFL": "5.0", "convDrop": "1e-3"}),
    ("caseWedge", {"order": "1", "CFL": "6.0", "mach": "2.4"}),
]
MAX_IT = 1500


def _case(name, kv):
    import csu_b200
    return csu_b200.Case.load(casekit.materialize(name, dict(BASE, **kv)))


def _alone(name, kv):
    import csu_b200
    eng = csu_b200.Engine(_case(name, kv))
    h = eng.iterate_until(MAX_IT)
    U = eng.get_state()
    eng.close()
    return len(h), U


@pytest.mark.parametrize("budget_mb,prep_threads", [(4096, 0), (18, 0), (4096, 2), (18, 2)])
def test_served_results_equal_alone(native, budget_mb, prep_threads):
    """prep_threads 2: the meshes are prepared on background threads while the packs iterate"""
    import csu_b200
    srv = csu_b200.Server(budget_mb << 20, iters_per_step=16, prep_threads=prep_threads)
    ids = []
    for k, (nm, kv) in enumerate(REQUESTS):
        ids.append(srv.submit(_case(nm, kv), max_iters=MAX_IT))
        if k % 2 == 1:
            srv.step()  # arrivals spread over steps: later requests join running packs
    for _ in range(10000):
        running, queued = srv.step()
        if running == 0 and queued == 0:
            break
    for rid, (nm, kv) in zip(ids, REQUESTS):
        info = srv.info(rid)
        assert info["state"] in ("converged", "maxiter"), info
        U = srv.take(rid)
        n, Ua = _alone(nm, kv)
        print("\n%s %s: %s after %d iterations (alone %d), waited %.3f s, ran %.3f s"
              % (nm, kv, info["state"], info["iters"], n, info["t_start"] - info["t_submit"],
                 info["t_end"] - info["t_start"]))
        assert info["iters"] == n
        assert np.array_equal(U, Ua), "%s: %d entries differ" % (nm, np.count_nonzero(U != Ua))
    srv.close()
