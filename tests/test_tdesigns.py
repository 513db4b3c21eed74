"""The shipped spherical t-designs are exact: for the full antipodal set
{p} U {-p} of degree t, the mean of P_l(p_i . p_j) over all pairs vanishes
for 1 <= l <= t (addition theorem), i.e. every spherical harmonic of degree
<= t integrates exactly with equal weights (the property the reference's
cubature relies on, src/cubature.cu:461-523)."""
import numpy as np
import pytest

from oracle import planner


def _store_degrees(store):
    return sorted(store._cache)


def test_store_covers_consecutive_odd_degrees(store):
    ts = _store_degrees(store)
    assert ts[0] == 1
    assert ts == list(range(1, ts[-1] + 1, 2))
    assert ts[-1] >= 91


@pytest.mark.parametrize("t", [3, 15, 33, 51, 65])
def test_design_exactness(store, t):
    p = store.get(t)
    assert np.allclose(np.linalg.norm(p, axis=1), 1.0, atol=1e-14)
    full = np.concatenate([p, -p])
    G = np.clip(full @ full.T, -1.0, 1.0)
    n2 = full.shape[0] ** 2
    p_prev, p_cur = np.ones_like(G), G.copy()  # P_0, P_1 by the 3-term recurrence
    assert abs(p_cur.sum() / n2) < 1e-13
    for l in range(2, t + 1):
        p_prev, p_cur = p_cur, ((2 * l - 1) * G * p_cur - (l - 1) * p_prev) / l
        assert abs(p_cur.sum() / n2) < 1e-13, (t, l)
