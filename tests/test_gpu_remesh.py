"""sw2gpu_remesh on the B200: after an adaption the remeshed context keeps the kept nodes' time
levels and steps bit for bit like a context made from scratch for the adapted mesh."""
import numpy as np
import pytest

from adhv8_kraken_b200.sw2 import SW2GPU
from helpers import basin_model, centroid_refine

pytestmark = pytest.mark.gpu


def test_step_after_remesh_equals_a_fresh_context():
    m0 = basin_model()
    g = SW2GPU(m0)
    for _ in range(2):
        assert g.step()["status"] == 0
    levels0 = [g.get_state(l) for l in range(3)]
    rng = np.random.Generator(np.random.PCG64(5))
    m1 = centroid_refine(m0, sorted(rng.choice(m0.nelems2d, 40, replace=False).tolist()))
    t = g.t
    g.remesh(m1)
    V0 = m0.nnodes
    for l in range(3):   # kept nodes keep their levels, new nodes start at 0
        got = g.get_state(l)
        for a, b in zip(got, levels0[l]):
            assert np.array_equal(a[:V0], b) and not a[V0:].any()
    # new nodes take the mean of their triangle's vertices on every level, in both contexts
    new = [np.concatenate([lv[k], np.zeros(m1.nnodes - V0)]) for lv in levels0 for k in range(3)]
    tri = m1.tri
    for n in range(V0, m1.nnodes):
        vs = sorted({int(q) for t2 in tri[(tri == n).any(axis=1)] for q in t2 if q != n})
        for a in new:
            a[n] = np.mean(a[vs])
    fresh = SW2GPU(m1)
    for s in (g, fresh):
        for l in range(3):
            s.set_state(l, *new[3 * l:3 * l + 3])
        s.t = t
    dt = m1.dt
    for _ in range(2):
        a, b = g.step(dt=dt, t=g.t), fresh.step(dt=dt, t=fresh.t)
        assert a["status"] == 0 and b["status"] == 0
        assert (a["newton_its"], a["linear_its"]) == (b["newton_its"], b["linear_its"])
        for x, y in zip(g.get_state(0), fresh.get_state(0)):
            assert np.array_equal(x, y)
        assert np.array_equal(g.get_wd(), fresh.get_wd())
    g.close()
    fresh.close()
