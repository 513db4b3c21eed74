"""Batched solves (glst_batch_*): many uneven systems in one CUDA graph.

Each system's result in the batch must be the same as the system solved
alone (bitwise: the same kernels on the same inputs, only scheduled together),
in graph mode and in the one-system-at-a-time plain mode, and on a replay of
the captured graph.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _cat(systems, key):
    return torch.tensor(np.concatenate([s[key] for s in systems]), dtype=torch.float64, device="cuda:0")


def test_batch_equals_individual_solves(pkg):
    """Ten uneven systems (a few without far field): the branch graph, its
    replay, the plain sequence and the work-list graph all give every system
    bit for bit its result alone."""
    from glst_b200 import systems as S
    sy = S.batch_uneven(10, seed=3, mol_min=100, mol_max=2500)
    ins = [_cat(sy, k) for k in ("x", "y", "z", "q")]
    n = ins[0].numel()
    outs = [torch.empty(n, dtype=torch.float64, device="cuda:0") for _ in range(4)]
    with pkg.GlstBatch(sy, nstreams=4) as b:
        b.compute(*ins, *outs)
        torch.cuda.synchronize()
        graph = [o.cpu().numpy().copy() for o in outs]
        e_graph = b.energies()
        b.compute(*ins, *outs)                 # replay of the captured graph
        torch.cuda.synchronize()
        replay = [o.cpu().numpy().copy() for o in outs]
        b.compute(*ins, *outs, plain=True)     # one system after another
        torch.cuda.synchronize()
        plain = [o.cpu().numpy().copy() for o in outs]
        b.compute(*ins, *outs, mode="worklist")  # one launch per phase over the work list
        torch.cuda.synchronize()
        branches = [o.cpu().numpy().copy() for o in outs]
        e_branches = b.energies()
        off = b.offsets
    for a, r, p, br in zip(graph, replay, plain, branches):
        assert np.array_equal(a, r) and np.array_equal(a, p) and np.array_equal(a, br)
    assert np.array_equal(e_graph, e_branches)
    for i, s in enumerate(sy):
        with pkg.GlstForce(s["natom"], s["tol"], *s["box"], rcut=s["rcut"]) as f:
            f.calc_ener_force(*[torch.tensor(s[k], dtype=torch.float64, device="cuda:0") for k in ("x", "y", "z", "q")])
            alone = f.get_ef()
            e = f.energy()
        for a, g in zip(alone, graph):
            assert np.array_equal(a, g[off[i]:off[i + 1]]), i
        assert e == e_graph[i]


def test_batch256_energies_match_reference(pkg):
    """The 256-system uneven batch (300-30,000 atoms, two cubature orders),
    solved in one captured graph, against the reference library run on the
    same systems one after another: every system's total energy within 1e-7
    relative.  Fixture: tests/golden/batch256_double.npz (make_golden.py)."""
    import os
    from glst_b200 import systems as S
    path = os.path.join(os.path.dirname(__file__), "golden", "batch256_double.npz")
    if not os.path.exists(path):
        pytest.skip("batch256 fixture not generated")
    gold = np.load(path)
    sy = S.batch_uneven(256, seed=0)
    import hashlib
    digest = hashlib.sha256(b"".join(np.ascontiguousarray(np.concatenate([s[k] for s in sy]), dtype="<f8").tobytes()
                                     for k in ("x", "y", "z", "q"))).hexdigest()
    assert str(gold["input_sha256"]) == digest
    ins = [_cat(sy, k) for k in ("x", "y", "z", "q")]
    n = ins[0].numel()
    outs = [torch.empty(n, dtype=torch.float64, device="cuda:0") for _ in range(4)]
    with pkg.GlstBatch(sy, nstreams=16) as b:
        b.compute(*ins, *outs)
        e = b.energies()
        off = b.offsets
        got = [o.cpu().numpy() for o in outs]
    ref = gold["energy"]
    assert np.array_equal(gold["natom"], [s["natom"] for s in sy])
    rel = np.abs(e - ref) / np.abs(ref)
    assert rel.max() <= 1e-7, (int(rel.argmax()), float(rel.max()))
    # per-atom forces and energies of every 16th system against the
    # reference's own outputs: <= 1e-5 relative force RMS per system
    if "forces_systems" not in gold:
        pytest.skip("batch256 fixture has no per-atom outputs")
    from oracle import oracle
    at = 0
    worst = 0.0
    for i in gold["forces_systems"]:
        n_i = int(gold["natom"][i])
        ref_i = [gold[k][at:at + n_i] for k in ("fx", "fy", "fz", "en")]
        got_i = [a[off[i]:off[i + 1]] for a in got]
        rep = oracle.error_report(got_i, ref_i)
        assert rep["force_rms_rel"] <= 1e-5 and rep["energy_rel"] <= 1e-7, (int(i), rep)
        worst = max(worst, rep["force_rms_rel"])
        at += n_i
    assert at == len(gold["fx"])
    print("batch256: %d systems' forces, worst relative force RMS %.3g" % (len(gold["forces_systems"]), worst))
