"""Generate the golden fixtures of this directory from the UNMODIFIED reference.

Runs ``oracle/_ref/glst_ref_harness`` (the reference library compiled from its
own sources by ``oracle/Makefile``; needs a CUDA GPU) on seeded synthetic water
boxes and stores, per case, the inputs' recipe and the reference's outputs:
per-atom fx, fy, fz, en in input order (glst_force<CT>::get_ef) and the cell
assignment (sorted_idx_, cell_atom_count_, cell_atom_point_).

The reference reads spherical t-designs from ``SS31-Mar-2016/`` in its working
directory (src/cubature.cu:490); this script renders the project's store there
(gauss-legendre-spherical-t_b200/data/tdesigns.bin) so both sides use the same
nodes.

    python tests/golden/make_golden.py [case ...]

Output: tests/golden/<case>_<ct>.npz, plus a timing summary on stdout.  The
case ``batch256`` runs the 256-system uneven batch through the reference one
system after another and keeps per-system energies and solve times, and the
per-atom outputs of every 16th system.
"""
import json
import math
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402

# case: (molecules, box A, rcut A, tol, seed); tol = erfc(alpha rcut)/rcut for
# the named configurations
CASES = {
    "water216": (216, 18.63, 9.0, math.erfc(0.34 * 9.0) / 9.0, 0),
    "w1000_tol1e-4": (1000, 31.04, 8.0, 1e-4, 3),
    "w2000_tol1e-5": (2000, 39.1, 10.0, 1e-5, 5),
    "water10k": (10000, 66.9, 10.0, math.erfc(0.31 * 10.0) / 10.0, 0),
    # water333k: one million atoms; stored as a seeded subset of atoms plus
    # digests of the full assignment (the full arrays would be 36 MB)
    "water333k": (333333, 215.3, 10.0, math.erfc(0.31 * 10.0) / 10.0, 0),
    # water10k at the next higher cubature order (tol / 10)
    "water10k_next": (10000, 66.9, 10.0, math.erfc(0.31 * 10.0) / 100.0, 0),
}
SUBSET = {"water333k": 20000}
CASE_CTS = {"water333k": ("double",), "water10k_next": ("double",)}
CTS = ("double", "float")


def input_sha256(x, y, z, q):
    """Digest of the FP64 inputs, so a test can tell that it regenerated the
    same positions and charges the fixture was made from."""
    import hashlib
    return hashlib.sha256(b"".join(np.ascontiguousarray(a, dtype="<f8").tobytes() for a in (x, y, z, q))).hexdigest()


def assignment_sha256(sorted_idx, cell_count, cell_point):
    """Digest of a cell assignment (u32 arrays, little endian)."""
    import hashlib
    return hashlib.sha256(b"".join(np.ascontiguousarray(a, dtype="<u4").tobytes()
                                   for a in (sorted_idx, cell_count, cell_point))).hexdigest()


def harness():
    return os.path.join(ROOT, "oracle", "_ref", "glst_ref_harness")


def write_input(path, x, y, z, q, tol, L, rcut):
    with open(path, "wb") as f:
        f.write(struct.pack("<I", len(x)))
        f.write(struct.pack("<d", tol))
        f.write(struct.pack("<ddd", L, L, L))
        f.write(struct.pack("<d", rcut))
        for a in (x, y, z, q):
            f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())


def read_output(path):
    with open(path, "rb") as f:
        data = f.read()
    natom, K, nx, ny, nz, iters = struct.unpack_from("<6I", data, 0)
    off = 24
    ms = np.frombuffer(data, dtype="<f8", count=8, offset=off)
    off += 64
    arrs = []
    for _ in range(4):
        arrs.append(np.frombuffer(data, dtype="<f8", count=natom, offset=off).copy())
        off += 8 * natom
    sidx = np.frombuffer(data, dtype="<u4", count=natom, offset=off).copy()
    off += 4 * natom
    C = nx * ny * nz
    cnt = np.frombuffer(data, dtype="<u4", count=C, offset=off).copy()
    off += 4 * C
    pnt = np.frombuffer(data, dtype="<u4", count=C, offset=off).copy()
    return dict(natom=natom, K=K, ncell=(nx, ny, nz), iters=iters, ms=ms, fx=arrs[0], fy=arrs[1],
                fz=arrs[2], en=arrs[3], sorted_idx=sidx, cell_count=cnt, cell_point=pnt)


def render_tdesigns(dst):
    g = __graft_entry__.load_package()
    sys.path.insert(0, os.path.join(os.path.dirname(g.TDESIGN_STORE)))
    import make_tdesigns
    make_tdesigns.write_reference_dir(g.TDESIGN_STORE, os.path.join(dst, "SS31-Mar-2016"))


# The uneven batch: 256 independent water boxes (300-30,000 atoms, two cubature
# orders, seed 0), run by the reference one system after another (its plain
# path).  The fixture keeps each system's total energy and solve time, and
# the per-atom forces and energies of every BATCH_FORCES_EVERY-th system.
BATCH_CASE = "batch256"
BATCH_FORCES_EVERY = 16


def batch_inputs_sha256(sy):
    return input_sha256(*[np.concatenate([s[k] for s in sy]) for k in ("x", "y", "z", "q")])


def make_batch(work, iters=2):
    from glst_b200 import systems
    sy = systems.batch_uneven(256, seed=0)
    lst = os.path.join(work, "batch.in")
    with open(lst, "wb") as f:
        f.write(struct.pack("<I", len(sy)))
    for s in sy:
        rec = lst + ".one"
        write_input(rec, s["x"], s["y"], s["z"], s["q"], s["tol"], s["box"][0], s["rcut"])
        with open(lst, "ab") as f, open(rec, "rb") as g:
            f.write(g.read())
    out = os.path.join(work, "batch.out")
    fout = os.path.join(work, "batch.forces")
    r = subprocess.run([harness(), "--batch", lst, out, "double", str(iters), fout, str(BATCH_FORCES_EVERY)],
                       cwd=work, capture_output=True, text=True)
    if r.returncode != 0:
        print(r.stdout[-2000:], r.stderr[-2000:])
        raise SystemExit("reference harness failed on the batch (%d)" % r.returncode)
    with open(out, "rb") as f:
        data = f.read()
    (nsys,) = struct.unpack_from("<I", data, 0)
    rec = np.dtype([("natom", "<u4"), ("K", "<u4"), ("ms_host", "<f8"), ("ms_events", "<f8"), ("energy", "<f8")])
    o = np.frombuffer(data, dtype=rec, count=nsys, offset=4)
    # forces of the sampled systems, concatenated in system order
    with open(fout, "rb") as f:
        fdata = f.read()
    idx, parts, off = [], [[], [], [], []], 0
    while off < len(fdata):
        s_i, n_i = struct.unpack_from("<II", fdata, off)
        off += 8
        idx.append(s_i)
        for k in range(4):
            parts[k].append(np.frombuffer(fdata, dtype="<f8", count=n_i, offset=off).copy())
            off += 8 * n_i
    np.savez_compressed(os.path.join(HERE, BATCH_CASE + "_double.npz"), natom=o["natom"].copy(), K=o["K"].copy(),
                        ms_host=o["ms_host"].copy(), ms_events=o["ms_events"].copy(), energy=o["energy"].copy(),
                        tol=np.array([s["tol"] for s in sy]), input_sha256=np.array(batch_inputs_sha256(sy)),
                        forces_systems=np.array(idx, dtype=np.uint32),
                        fx=np.concatenate(parts[0]), fy=np.concatenate(parts[1]), fz=np.concatenate(parts[2]),
                        en=np.concatenate(parts[3]))
    summary = dict(systems=int(nsys), atoms=int(o["natom"].sum()), sequential_ms_host=float(o["ms_host"].sum()),
                   sequential_ms_events=float(o["ms_events"].sum()))
    print(json.dumps({BATCH_CASE + "_double": summary}), flush=True)
    return summary


def main(cases, iters=3):
    g = __graft_entry__.load_package()
    from glst_b200 import systems
    if not os.path.exists(harness()):
        raise SystemExit("build the reference first: make -C oracle ref")
    summary = {}
    with tempfile.TemporaryDirectory() as work:
        render_tdesigns(work)
        for case in cases:
            if case == BATCH_CASE:
                summary[case] = make_batch(work)
                continue
            n_mol, L, rcut, tol, seed = CASES[case]
            x, y, z, q = systems.water_box(n_mol, L, seed=seed)
            digest = input_sha256(x, y, z, q)
            inp = os.path.join(work, case + ".in")
            write_input(inp, x, y, z, q, tol, L, rcut)
            for ct in CASE_CTS.get(case, CTS):
                out = os.path.join(work, "%s_%s.out" % (case, ct))
                r = subprocess.run([harness(), inp, out, ct, str(iters)], cwd=work, capture_output=True,
                                   text=True)
                if r.returncode != 0:
                    print(r.stdout[-2000:], r.stderr[-2000:])
                    raise SystemExit("reference harness failed on %s/%s (%d)" % (case, ct, r.returncode))
                o = read_output(out)
                path = os.path.join(HERE, "%s_%s.npz" % (case, ct))
                if case in SUBSET:
                    sel = np.sort(np.random.default_rng(1234).choice(o["natom"], SUBSET[case], replace=False))
                    np.savez_compressed(path, n_mol=n_mol, box=L, rcut=rcut, tol=tol, seed=seed, K=o["K"],
                                        ncell=np.array(o["ncell"]), subset=sel, fx=o["fx"][sel], fy=o["fy"][sel],
                                        fz=o["fz"][sel], en=o["en"][sel], energy_total=0.5 * float(np.sum(o["en"])),
                                        force_rms=float(np.sqrt(np.mean(o["fx"] ** 2 + o["fy"] ** 2 + o["fz"] ** 2))),
                                        assignment_sha256=np.array(assignment_sha256(
                                            o["sorted_idx"], o["cell_count"], o["cell_point"])),
                                        ref_ms=o["ms"], input_sha256=np.array(digest))
                else:
                    np.savez_compressed(path, n_mol=n_mol, box=L, rcut=rcut, tol=tol, seed=seed, K=o["K"],
                                        ncell=np.array(o["ncell"]), fx=o["fx"], fy=o["fy"], fz=o["fz"], en=o["en"],
                                        sorted_idx=o["sorted_idx"], cell_count=o["cell_count"],
                                        cell_point=o["cell_point"], ref_ms=o["ms"], input_sha256=np.array(digest))
                summary["%s_%s" % (case, ct)] = dict(
                    natom=o["natom"], K=o["K"], ncell=o["ncell"],
                    ms=dict(zip(["assign", "sf", "sum_rmt", "lr", "sr", "comm", "total_host", "total_events"],
                                [round(float(v), 4) for v in o["ms"]])))
                print(json.dumps({case + "_" + ct: summary["%s_%s" % (case, ct)]}), flush=True)
    return summary


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES) + [BATCH_CASE])
