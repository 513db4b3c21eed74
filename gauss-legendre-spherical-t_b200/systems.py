"""Seeded synthetic TIP3P-like water boxes (the inputs of every benchmark).

Rigid water: O -0.834 e, H +0.417 e, O-H 0.9572 A, H-O-H 104.52 degrees.
Oxygens sit on an m x m x m lattice of spacing L/m (m = ceil(n^(1/3)); when
n < m^3 a seeded random subset of sites is used), jittered by U(-0.3, 0.3) A
per axis; each molecule gets a uniformly random orientation (random unit
quaternion).  Coordinates are FP64 and finally shifted so that the minimum
coordinate on each axis is 0, as the reference's driver does before calling
the library (utils/utils.cpp:35-58).  Atom order: O, H, H per molecule.
"""
import math

import numpy as np

Q_O, Q_H = -0.834, 0.417
R_OH = 0.9572
THETA_HOH = math.radians(104.52)

# Standard configurations of the GLST benchmarks: (molecules, box edge A,
# cutoff A, splitting alpha 1/A).  tol = erfc(alpha rcut) / rcut.
CONFIGS = {
    "water216": dict(n_mol=216, box=18.63, rcut=9.0, alpha=0.34),
    "water10k": dict(n_mol=10000, box=66.9, rcut=10.0, alpha=0.31),
    "water333k": dict(n_mol=333333, box=215.3, rcut=10.0, alpha=0.31),
    # the water333k atoms and 22^3 grid at a coarse tolerance (K ~ 1,500
    # nodes, ~3 GB on the device): small enough for multi-pass profiler
    # captures of the same kernels, which the full order (44 GB) is not
    "water333k_coarse": dict(n_mol=333333, box=215.3, rcut=10.0, alpha=0.31, tol=1e-3),
}


def tol_from_alpha(alpha, rcut):
    return math.erfc(alpha * rcut) / rcut


def _random_rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def water_box(n_mol, box, seed=0, recenter=True):
    """Returns (x, y, z, q) FP64 arrays of 3*n_mol atoms."""
    rng = np.random.default_rng(seed)
    m = int(round(n_mol ** (1.0 / 3.0)))
    while m ** 3 < n_mol:
        m += 1
    s = box / m
    sites = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    if sites.shape[0] > n_mol:
        sites = sites[np.sort(rng.choice(sites.shape[0], n_mol, replace=False))]
    O = (sites + 0.5) * s + rng.uniform(-0.3, 0.3, size=(n_mol, 3))
    half = 0.5 * THETA_HOH
    local = np.array([[R_OH * math.sin(half), 0.0, R_OH * math.cos(half)],
                      [-R_OH * math.sin(half), 0.0, R_OH * math.cos(half)]])
    Rm = _random_rotations(rng, n_mol)
    H = O[:, None, :] + np.einsum("nij,kj->nki", Rm, local)
    pos = np.concatenate([O[:, None, :], H], axis=1).reshape(-1, 3)
    q = np.tile(np.array([Q_O, Q_H, Q_H]), n_mol)
    if recenter:
        pos = pos - pos.min(axis=0)
    return (np.ascontiguousarray(pos[:, 0]), np.ascontiguousarray(pos[:, 1]),
            np.ascontiguousarray(pos[:, 2]), q)


def config_system(name, seed=0):
    c = CONFIGS[name]
    x, y, z, q = water_box(c["n_mol"], c["box"], seed=seed)
    return dict(x=x, y=y, z=z, q=q, box=(c["box"],) * 3, rcut=c["rcut"],
                tol=c.get("tol", tol_from_alpha(c["alpha"], c["rcut"])))


# ----------------------------------------------------------------- CHARMM IO
# The reference's driver reads CHARMM extended-format files
# (utils/io.cpp:35-117): the .psf header line holds natom in columns 0-9 and
# "!NATOM" at column 11; each atom line holds the charge in columns 50-63.
# The .cor file has '*' title lines, natom in columns 0-9, then x, y, z in
# columns 40-59, 60-79 and 80-99.

def write_charmm(prefix, x, y, z, q):
    """Write <prefix>.psf and <prefix>.cor readable by the reference driver."""
    n = len(x)
    with open(prefix + ".psf", "w") as f:
        f.write("PSF EXT\n\n         1 !NTITLE\n* synthetic TIP3P-like water\n\n")
        f.write("%10d !NATOM\n" % n)
        for i in range(n):
            name = "OH2" if i % 3 == 0 else ("H1" if i % 3 == 1 else "H2")
            head = "%10d WAT      %-8d TIP3     %-8s" % (i + 1, i // 3 + 1, name)
            f.write(head.ljust(50)[:50] + "%14.6f" % q[i] + "%14.4f%12d\n" % (16.0 if i % 3 == 0 else 1.008, 0))
    with open(prefix + ".cor", "w") as f:
        f.write("* synthetic TIP3P-like water\n*\n")
        f.write("%10d  EXT\n" % n)
        for i in range(n):
            name = "OH2" if i % 3 == 0 else ("H1" if i % 3 == 1 else "H2")
            head = "%10d%10d  %-8s  %-8s" % (i + 1, i // 3 + 1, "TIP3", name)
            f.write(head.ljust(40)[:40] + "%20.10f%20.10f%20.10f" % (x[i], y[i], z[i]) + "  WAT      %-8d  0.0000000000\n" % (i // 3 + 1))


def read_charmm(prefix):
    """(x, y, z, q) from <prefix>.psf/.cor, the columns the reference reads."""
    natom = None
    q = []
    with open(prefix + ".psf") as f:
        lines = f.read().split("\n")
    it = iter(lines)
    for line in it:
        if len(line) >= 17 and line[11:17] == "!NATOM":
            natom = int(line[0:11])
            break
    for _ in range(natom):
        q.append(float(next(it)[50:64]))
    with open(prefix + ".cor") as f:
        lines = [ln for ln in f.read().split("\n")]
    k = 0
    while lines[k][:1] == "*" or not lines[k].strip():
        k += 1
    if int(lines[k][0:10]) != natom:
        raise ValueError("atom count differs between .psf and .cor")
    xyz = np.array([[float(ln[40:60]), float(ln[60:80]), float(ln[80:100])] for ln in lines[k + 1:k + 1 + natom]])
    return (np.ascontiguousarray(xyz[:, 0]), np.ascontiguousarray(xyz[:, 1]),
            np.ascontiguousarray(xyz[:, 2]), np.array(q))


def recenter(x, y, z):
    """Shift so the minimum coordinate on each axis is 0 (utils/utils.cpp:35-58)."""
    return x - x.min(), y - y.min(), z - z.min()


# ----------------------------------------------------------------- batches
WATER_DENSITY = 0.0334  # molecules / A^3


def batch_uneven(n_sys=256, seed=0, mol_min=100, mol_max=10000, rcut=10.0, alpha=0.31):
    """Independent water boxes of uneven size: molecule counts log-uniform in
    [mol_min, mol_max], box edge (n / 0.0334)^(1/3), cutoff rcut, and per
    system one of two cubature orders, tol = erfc(alpha rcut)/rcut or a
    tenth of it, drawn uniformly.  Returns a list of system dicts."""
    rng = np.random.default_rng(seed)
    t0 = tol_from_alpha(alpha, rcut)
    out = []
    for i in range(n_sys):
        n_mol = int(round(math.exp(rng.uniform(math.log(mol_min), math.log(mol_max)))))
        L = (n_mol / WATER_DENSITY) ** (1.0 / 3.0)
        tol = t0 if rng.uniform() < 0.5 else 0.1 * t0
        x, y, z, q = water_box(n_mol, L, seed=seed * 100003 + i)
        out.append(dict(x=x, y=y, z=z, q=q, box=(L, L, L), rcut=rcut, tol=tol, natom=len(x)))
    return out


def request_stream(n_requests, seed=0, atom_min=1000, atom_max=200000, p_continue=0.6, sigma=0.01,
                   rcut=10.0, alpha=0.31):
    """Energy+force requests of a served MD-like workload.  With probability
    p_continue a request continues a resident system (same key, every atom
    displaced by N(0, sigma) A); otherwise it opens a new water box with an
    atom count log-uniform in [atom_min, atom_max].  Returns a list of dicts
    (key, x, y, z, q, box, rcut, tol)."""
    rng = np.random.default_rng(seed)
    tol = tol_from_alpha(alpha, rcut)
    live = {}
    out = []
    next_key = 1
    for _ in range(n_requests):
        if live and rng.uniform() < p_continue:
            key = int(rng.choice(list(live)))
            st = live[key]
            st["x"] = st["x"] + rng.normal(0.0, sigma, st["x"].size)
            st["y"] = st["y"] + rng.normal(0.0, sigma, st["y"].size)
            st["z"] = st["z"] + rng.normal(0.0, sigma, st["z"].size)
        else:
            n_atom = math.exp(rng.uniform(math.log(atom_min), math.log(atom_max)))
            n_mol = max(1, int(round(n_atom / 3.0)))
            L = (n_mol / WATER_DENSITY) ** (1.0 / 3.0)
            x, y, z, q = water_box(n_mol, L, seed=int(rng.integers(1 << 30)))
            key = next_key
            next_key += 1
            st = live[key] = dict(x=x, y=y, z=z, q=q, box=(L, L, L))
        out.append(dict(key=key, x=st["x"].copy(), y=st["y"].copy(), z=st["z"].copy(), q=st["q"],
                        box=st["box"], rcut=rcut, tol=tol))
    return out
