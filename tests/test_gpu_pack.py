"""Packs: several steady solves (different meshes and flow conditions) advanced by one launch of each kernel.
Every reduction is per solve and each solve's cells are block aligned, so each solve's iterations are
bit-identical alone and in the pack; a solve that converges (convDrop) freezes while the others run; a
solve moved into another pack (as the serving layer does on admission) continues unchanged."""
import numpy as np
import pytest

import casekit

pytestmark = pytest.mark.gpu

# one structure (AUSMDV, order 2, DPLUR 4 sweeps), different meshes and flow conditions
STRUCT = {"timeScheme": "DPLUR", "Nlinear": "4", "order": "2", "flux": "AUSMDV", "restart": "0"}
MEMBERS = [
    ("caseWedge", {"CFL": "5.0"}),
    ("caseCylinder", {"CFL": "3.0", "mach": "2.5"}),
    ("caseWedgeQuad", {"CFL": "8.0", "mach": "2.2", "temperature": "280."}),
    ("caseDiamond", {"CFL": "5.0"}),
]


def _case(name, kv):
    import csu_b200
    return csu_b200.Case.load(casekit.materialize(name, dict(STRUCT, **kv)))


def _alone(name, kv, n):
    import csu_b200
    eng = csu_b200.Engine(_case(name, kv))
    hist = eng.iterate(n)
    U = eng.get_state()
    eng.close()
    return hist, U


def test_pack_equals_alone(native):
    import csu_b200
    n = 30
    preps = [csu_b200.Prep(_case(nm, kv)) for nm, kv in MEMBERS]
    pack = csu_b200.Pack(preps)
    pack.iterate(n)
    for k, (nm, kv) in enumerate(MEMBERS):
        hist, U = _alone(nm, kv, n)
        Up = pack.get_state(k)
        hp = pack.history(k)
        info = pack.info(k)
        assert info["iter"] == n and info["status"] == 0
        assert np.array_equal(Up, U), "%s: %d state entries differ" % (nm, np.count_nonzero(Up != U))
        assert np.array_equal(hp, hist), "%s: history differs" % nm
    pack.close()


def test_pack_convergence_freezes_one_solve(native):
    """A solve whose residual drop is reached stops; the other continues, both as they would alone."""
    import csu_b200
    fast = ("caseWedge", {"CFL": "10.0", "order": "1", "convDrop": "1e-6"})
    slow = ("caseCylinder", {"CFL": "3.0", "order": "1"})
    pack = csu_b200.Pack([csu_b200.Prep(_case(*fast)), csu_b200.Prep(_case(*slow))])
    n = 1200
    pack.iterate(n)
    i0, i1 = pack.info(0), pack.info(1)
    assert i0["done"] == 1 and i0["iter"] < n
    assert i1["done"] == 0 and i1["iter"] == n
    eng = csu_b200.Engine(_case(*fast))
    h = eng.iterate_until(n)
    assert len(h) == i0["iter"]
    assert np.array_equal(eng.get_state(), pack.get_state(0))
    eng.close()
    pack.close()


def test_pack_transfer_continues_solve(native):
    """Solve moved between packs mid-run (admission of a new member) continues bit-identically."""
    import csu_b200
    a, b = MEMBERS[0], MEMBERS[1]
    pa, pb = csu_b200.Prep(_case(*a)), csu_b200.Prep(_case(*b))
    first = csu_b200.Pack([pa])
    first.iterate(12)
    second = csu_b200.Pack([pb, pa])
    second.transfer_from(first, 0, 1)
    first.close()
    second.iterate(18)
    hist, U = _alone(a[0], a[1], 30)
    assert second.info(1)["iter"] == 30
    assert np.array_equal(second.get_state(1), U)
    assert np.array_equal(second.history(1), hist[12:])
    hb, Ub = _alone(b[0], b[1], 18)
    assert np.array_equal(second.get_state(0), Ub)
    second.close()


def test_pack_rebuild_moves_solves_on_device(native):
    """A rebuilt pack (new member first, kept members reordered) continues the kept solves bit-identically
    and runs the new one as it would alone."""
    import csu_b200
    a, b, c = MEMBERS[0], MEMBERS[1], MEMBERS[2]
    pa, pb, pc = (csu_b200.Prep(_case(*m)) for m in (a, b, c))
    first = csu_b200.Pack([pa, pb])
    first.iterate(10)
    second = first.rebuilt([-1, 1, 0], [pc, pb, pa])
    first.close()
    second.iterate(20)
    for k, (m, n, skip) in enumerate([(c, 20, 0), (b, 30, 10), (a, 30, 10)]):
        hist, U = _alone(m[0], m[1], n)
        assert second.info(k)["iter"] == n
        assert np.array_equal(second.get_state(k), U), m[0]
        assert np.array_equal(second.history(k), hist[skip:]), m[0]
    second.close()
