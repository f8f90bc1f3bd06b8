"""Seeded synthetic molecules for the benchmark workloads and the parity tests.

* ``water_cluster``: oxygens on a regular grid with 3.1 A spacing, sites taken in fixed
  (x-major) order, uniform +-0.2 A jitter per oxygen, rigid O-H 0.957 A / H-O-H 104.5 deg water
  with a uniformly random orientation (random unit quaternion) -- the 34-water (4x3x3 grid) and
  2000-water (13x13x12 grid) clusters.
* ``organic``: a neutral closed-shell C/H/N/O/S molecule grown as a random valence-satisfying
  tree (C4 N3 O2 S2 H1, C=O carbonyls), standard bond lengths, roughly tetrahedral / trigonal
  bond angles, +-0.05 A coordinate jitter, rejected if two non-bonded atoms come closer than
  0.9 A.
* ``radical``: an organic molecule with one hydrogen removed (a doublet).

No public dataset is involved: these stand in for the workloads' shapes, sizes and element
distributions. Coordinates are returned in Angstrom.
"""
from __future__ import annotations

import math

import numpy as np

SYMBOLS = {1: "H", 6: "C", 7: "N", 8: "O", 16: "S"}
VALENCE = {1: 1, 6: 4, 7: 3, 8: 2, 16: 2}
# single-bond lengths (A); the carbonyl C=O uses 1.21
BOND = {
    (1, 6): 1.09, (1, 7): 1.01, (1, 8): 0.96, (1, 16): 1.34,
    (6, 6): 1.53, (6, 7): 1.47, (6, 8): 1.43, (6, 16): 1.82,
    (7, 7): 1.45, (7, 8): 1.40, (7, 16): 1.70, (8, 8): 1.48, (8, 16): 1.70, (16, 16): 2.05,
}
CARBONYL = 1.21
ELEMENT_WEIGHTS = ((6, 0.35), (1, 0.45), (7, 0.08), (8, 0.10), (16, 0.02))


def bond_length(za: int, zb: int) -> float:
    return BOND[(min(za, zb), max(za, zb))]


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    u1, u2, u3 = rng.random(3)
    x = math.sqrt(1 - u1) * math.sin(2 * math.pi * u2)
    y = math.sqrt(1 - u1) * math.cos(2 * math.pi * u2)
    z = math.sqrt(u1) * math.sin(2 * math.pi * u3)
    w = math.sqrt(u1) * math.cos(2 * math.pi * u3)
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def water_cluster(n_mol: int, grid=(4, 3, 3), spacing: float = 3.1, jitter: float = 0.2, seed: int = 20260826):
    """(z, xyz_angstrom) of ``n_mol`` waters on the first ``n_mol`` sites of ``grid``."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = grid
    if n_mol > nx * ny * nz:
        raise ValueError("grid too small")
    oh, ang = 0.957, math.radians(104.5)
    base = np.array([[0.0, 0.0, 0.0], [oh, 0.0, 0.0], [oh * math.cos(ang), oh * math.sin(ang), 0.0]])
    z, xyz = [], []
    k = 0
    for i in range(nx):
        for j in range(ny):
            for l in range(nz):
                if k == n_mol:
                    break
                site = np.array([i, j, l], dtype=float) * spacing + rng.uniform(-jitter, jitter, 3)
                rot = _random_rotation(rng)
                for a, p in enumerate(base):
                    z.append(8 if a == 0 else 1)
                    xyz.append(site + rot @ p)
                k += 1
    return np.array(z, dtype=np.int32), np.array(xyz)


def _unit(v):
    return v / np.linalg.norm(v)


def organic(n_atoms: int, seed: int, max_tries: int = 200):
    """(z, xyz_angstrom) of a random closed-shell organic with about ``n_atoms`` atoms."""
    rng = np.random.default_rng(seed)
    zs_w = np.array([w for _, w in ELEMENT_WEIGHTS])
    zs = [z for z, _ in ELEMENT_WEIGHTS]
    for _ in range(max_tries):
        mol = _grow(rng, n_atoms, zs, zs_w / zs_w.sum())
        if mol is not None:
            return mol
    raise RuntimeError("could not grow a molecule")


def _perp(b, rng):
    t = np.cross(b, rng.normal(size=3))
    return _unit(t)


def _tetra_slots(b, rng):
    """Three unit vectors at 109.47 deg from ``b`` (and from each other), random azimuth."""
    u = _perp(b, rng)
    v = np.cross(b, u)
    ct = math.cos(math.radians(109.471))
    st = math.sin(math.radians(109.471))
    phi = rng.uniform(0.0, 2.0 * math.pi)
    out = []
    for k in range(3):
        a = phi + 2.0 * math.pi * k / 3.0
        out.append(_unit(ct * b + st * (math.cos(a) * u + math.sin(a) * v)))
    return out


def _trig_slots(b, rng):
    """Two unit vectors at 120 deg from ``b`` in a random plane containing ``b``."""
    u = _perp(b, rng)
    c, s_ = math.cos(math.radians(120.0)), math.sin(math.radians(120.0))
    return [_unit(c * b + s_ * u), _unit(c * b - s_ * u)]


def _grow(rng, target, zs, w):
    """Tree growth with ideal hybridisation directions: sp3 atoms take tetrahedral slots, a
    carbonyl carbon is planar trigonal (C=O 1.21 A)."""
    z, pos, nbr, slots = [], [], [], []  # slots[i]: free bond directions of atom i

    def add_atom(el, p, parent, carbonyl=False):
        i = len(z)
        z.append(el)
        pos.append(p)
        nbr.append([] if parent is None else [parent])
        if parent is not None:
            nbr[parent].append(i)
        free = []
        if el != 1:
            if parent is None:
                b = _unit(rng.normal(size=3))
                free = [b] + _tetra_slots(b, rng)
            else:
                b = _unit(pos[parent] - p)
                free = _trig_slots(b, rng) if carbonyl else _tetra_slots(b, rng)
        slots.append(free[: VALENCE[el] - (0 if parent is None else 1) - (2 if carbonyl else 0)])
        return i

    def margin(q, parent, el, loose=False):
        """Smallest clearance surplus against all non-bonded atoms. Strict: 2.2 A heavy-heavy,
        1.7 A heavy-H, 1.5 A H-H; loose (hydrogen caps): 1.3 A and 1.1 A."""
        if not pos:
            return 1.0
        d = np.sqrt(((np.array(pos) - q) ** 2).sum(-1))
        d[parent] = 9.0
        zz = np.array(z)
        if loose:
            need = np.where(zz == 1, 1.1, 1.3)
        else:
            need = np.where(zz == 1, 1.5 if el == 1 else 1.7, 1.7 if el == 1 else 2.2)
        return float((d - need).min())

    def rotations(parent, d):
        """d, then d rotated about the parent's own bond axis in 30 degree steps."""
        yield d
        if not nbr[parent]:
            return
        axis = _unit(pos[nbr[parent][0]] - pos[parent])
        for k in range(1, 12):
            a = math.radians(30.0 * k)
            yield _unit(d * math.cos(a) + np.cross(axis, d) * math.sin(a) + axis * np.dot(axis, d) * (1 - math.cos(a)))

    def attach(parent, d0, el, loose=False):
        """Attach a new atom of element el near slot direction d0 of parent (None if blocked)."""
        carbonyl = el == 6 and not loose and rng.random() < 0.15
        best, best_m = None, -1e9
        for d in rotations(parent, d0):
            q = pos[parent] + bond_length(z[parent], el) * d
            m = margin(q, parent, el, loose)
            if m < 0.0:
                if loose and m > best_m:
                    best, best_m = q, m
                continue
            if carbonyl:  # the =O sits in the trigonal plane of the new carbon
                b = _unit(pos[parent] - q)
                dirs = _trig_slots(b, rng)
                qo = q + CARBONYL * dirs[0]
                if margin(qo, parent, 8) < 0.0 or np.linalg.norm(qo - pos[parent]) < 2.2:
                    continue
                i = add_atom(el, q, parent, carbonyl)
                slots[i] = [dirs[1]]
                add_atom(8, qo, i)
                slots[-1] = []
                return i
            return add_atom(el, q, parent, carbonyl)
        return None

    def cap(parent, d):
        """A hydrogen on this valence: strict clearance if possible, else the least crowded
        rotation that still keeps 1.3 A / 1.1 A."""
        i = attach(parent, d, 1)
        if i is None:
            i = attach(parent, d, 1, loose=True)
        return i

    root_carbonyl = rng.random() < 0.15
    add_atom(6, np.zeros(3), None)
    if root_carbonyl:
        b = slots[0][0]
        tr = _trig_slots(b, rng)
        slots[0] = tr
        add_atom(8, CARBONYL * b, 0)
        slots[-1] = []
    while True:
        open_sites = [(i, k) for i in range(len(z)) for k in range(len(slots[i]))]
        if not open_sites:
            break
        if len(z) + len(open_sites) >= target:
            break
        # grow mostly from the newest atoms: chain-like trees, less crowding
        recent = sorted({a for a, _ in open_sites})[-4:]
        cand = [(a, kk) for a, kk in open_sites if a in recent]
        i, k = cand[int(rng.integers(len(cand)))]
        el = int(rng.choice(zs, p=w))
        if el == 1 and len(open_sites) <= 2 and len(z) + len(open_sites) < target - 1:
            el = 6  # keep the tree growing while it is small
        d = slots[i].pop(k)
        if attach(i, d, el) is None:
            if cap(i, d) is None:
                return None
    for i in range(len(z)):  # cap every open valence with hydrogen
        while slots[i]:
            d = slots[i].pop(0)
            if cap(i, d) is None:
                return None
    if len(z) < 5 or sum(VALENCE[x] for x in z) % 2:
        return None
    xyz = np.array(pos) + rng.uniform(-0.05, 0.05, (len(z), 3))
    diff = xyz[:, None, :] - xyz[None, :, :]
    dist = np.sqrt((diff ** 2).sum(-1))
    bonded = np.zeros_like(dist, dtype=bool)
    for i, nb in enumerate(nbr):
        bonded[i, nb] = True
    np.fill_diagonal(bonded, True)
    if (dist[~bonded] < 0.9).any():  # reject non-bonded contacts below 0.9 A
        return None
    return np.array(z, dtype=np.int32), xyz


def radical(n_atoms: int, seed: int):
    """An organic molecule with one hydrogen removed (multiplicity 2)."""
    rng = np.random.default_rng(seed + 7919)
    for k in range(100):
        z, xyz = organic(n_atoms, seed + 104729 * k)
        hs = np.flatnonzero(z == 1)
        if len(hs):
            drop = int(rng.choice(hs))
            keep = np.ones(len(z), dtype=bool)
            keep[drop] = False
            return z[keep], xyz[keep]
    raise RuntimeError("no hydrogen to remove")


def organic_batch(n_mol: int, lo: int = 5, hi: int = 60, seed: int = 1234, only=None):
    """List of (z, xyz_angstrom) for ``n_mol`` organics with sizes uniform in [lo, hi]. With
    ``only`` (molecule indices), just those molecules of the same batch, in that order."""
    sizes = organic_batch_sizes(n_mol, lo, hi, seed)
    idx = range(n_mol) if only is None else only
    return [organic(int(sizes[i]), seed * 1000003 + int(i)) for i in idx]


def organic_batch_sizes(n_mol: int, lo: int = 5, hi: int = 60, seed: int = 1234):
    """Atom counts of the molecules of ``organic_batch`` (cheap: no molecule is built)."""
    return np.random.default_rng(seed).integers(lo, hi + 1, n_mol)


def radical_batch(n_mol: int, lo: int = 10, hi: int = 80, seed: int = 4321, only=None):
    sizes = np.random.default_rng(seed).integers(lo, hi + 1, n_mol)
    idx = range(n_mol) if only is None else only
    return [radical(int(sizes[i]), seed * 1000003 + int(i)) for i in idx]


def pack(mols):
    """Concatenate [(z, xyz_angstrom)] into (offsets, z, xyz_angstrom) batch arrays."""
    offs = np.zeros(len(mols) + 1, dtype=np.int32)
    for i, (z, _) in enumerate(mols):
        offs[i + 1] = offs[i] + len(z)
    z = np.concatenate([m[0] for m in mols]).astype(np.int32) if mols else np.zeros(0, np.int32)
    xyz = np.concatenate([m[1] for m in mols]) if mols else np.zeros((0, 3))
    return offs, z, xyz
