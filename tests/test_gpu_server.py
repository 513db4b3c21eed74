"""Request server (glst_server_*): continuous batching of independent solves.

Each request's result must be the same whether it is solved alone or in the
mix with other requests in flight (bitwise: the same kernels on the same
inputs), also when the memory budget forces queueing and eviction of
resident systems.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _alone(pkg, r):
    with pkg.GlstForce(len(r["x"]), r["tol"], *r["box"], rcut=r["rcut"]) as f:
        f.calc_ener_force(*[torch.tensor(r[k], dtype=torch.float64, device="cuda:0") for k in ("x", "y", "z", "q")])
        return f.get_ef(), f.energy()


def _serve(pkg, reqs, budget, nslots):
    with pkg.GlstServer(budget, nslots=nslots) as s:
        tickets = [s.submit(r["key"], r["x"], r["y"], r["z"], r["q"], r["tol"], r["box"], r["rcut"]) for r in reqs]
        res = [s.wait(t, timeout_ms=120000) for t in tickets]
        return res, s.stats()


def test_results_alone_equal_results_in_the_mix(pkg):
    from glst_b200 import systems as S
    reqs = S.request_stream(14, seed=4, atom_min=600, atom_max=12000)
    res, st = _serve(pkg, reqs, budget=16 << 30, nslots=4)
    assert st.completed == len(reqs) and st.in_flight == 0
    assert st.systems_created < len(reqs)  # resident systems were reused
    for r, got in zip(reqs, res):
        (fx, fy, fz, en), e = _alone(pkg, r)
        for a, b in zip((fx, fy, fz, en), got[:4]):
            assert np.array_equal(a, b)
        assert got[4] == e and got[5] > 0


def test_tight_budget_queues_and_evicts(pkg):
    from glst_b200 import systems as S
    reqs = S.request_stream(10, seed=5, atom_min=3000, atom_max=9000, p_continue=0.3)
    res, st = _serve(pkg, reqs, budget=700 << 20, nslots=4)
    assert st.completed == len(reqs)
    assert st.peak_resident_bytes <= 700 << 20
    assert st.evictions > 0
    for r, got in zip(reqs, res):
        (fx, fy, fz, en), e = _alone(pkg, r)
        assert np.array_equal(fx, got[0]) and np.array_equal(en, got[3]) and e == got[4]


def test_request_over_budget_is_rejected(pkg):
    from glst_b200 import systems as S
    r = S.request_stream(1, seed=6, atom_min=30000, atom_max=30001)[0]
    with pkg.GlstServer(1 << 20, nslots=2) as s:
        t = s.submit(r["key"], r["x"], r["y"], r["z"], r["q"], r["tol"], r["box"], r["rcut"])
        with pytest.raises(pkg.GlstError) as e:
            s.wait(t, timeout_ms=60000)
        assert e.value.status == 6
