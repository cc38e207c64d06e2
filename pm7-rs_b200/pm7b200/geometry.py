"""Seeded synthetic molecules of the benchmark workloads (positions returned in Bohr).

* `decane(seed)` - n-decane C10H22 in the all-staggered zig-zag (C-C 1.54 A, C-H
  1.09 A, tetrahedral angles), every coordinate jittered by U(-0.02, 0.02) A.
* `alkane(n, seed, jitter)` - the same builder for C_nH_(2n+2).
* `water_cluster(k, seed)` - k H2O (O-H 0.96 A, H-O-H 104.5 deg) on the first k sites
  of a cubic grid of spacing 3.1 A, uniformly random orientation (normalised Gaussian
  quaternion), U(-0.1, 0.1) A centre jitter.
* `batch(count, seed)` - half alkanes C_nH_2n+2 with n ~ U{1..40}, half water clusters
  of 2..64 molecules, jitter 0.02 A.
* `substituted_chain(n, rng)` - a zig-zag chain of n heavy atoms where each interior CH2
  becomes S with probability 0.1 (C-S 1.82 A) and each H becomes Cl with probability 0.1
  (C-Cl 1.77 A); `stream(count, seed)` - molecules of log-uniform size in 3..500 atoms,
  half such chains and half water clusters.
* `flat_alkane(n)` - the flat zig-zag C_nH_(2n+2) chain (no jitter) of the divide-and-
  conquer workload.
All draws use numpy.random.default_rng(seed).
"""
import math

import numpy as np

A0 = 0.529177210903
ANG = 1.0 / A0


def _tetra_hydrogens(c, prev, nxt, r):
    """Two hydrogens on an sp3 carbon with backbone neighbours prev/nxt (Angstrom)."""
    b1 = prev - c
    b2 = nxt - c
    b1 /= np.linalg.norm(b1)
    b2 /= np.linalg.norm(b2)
    bis = -(b1 + b2)
    bis /= np.linalg.norm(bis)
    perp = np.cross(b1, b2)
    perp /= np.linalg.norm(perp)
    half = math.radians(109.471) / 2.0
    return [c + r * (math.cos(half) * bis + math.sin(half) * perp),
            c + r * (math.cos(half) * bis - math.sin(half) * perp)]


def alkane_angstrom(n):
    """Ideal all-staggered C_nH_(2n+2): list of (Z, xyz Angstrom)."""
    cc, ch = 1.54, 1.09
    theta = math.radians(109.471)
    dx = cc * math.sin(theta / 2.0)
    dz = cc * math.cos(theta / 2.0)
    carbons = [np.array([i * dx, 0.0, (i % 2) * dz]) for i in range(n)]
    atoms = [(6, c) for c in carbons]
    hyd = []
    for i, c in enumerate(carbons):
        if n == 1:
            # methane
            s = ch / math.sqrt(3.0)
            for v in ((1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1)):
                hyd.append(c + s * np.array(v, dtype=float))
            continue
        prev = carbons[i - 1] if i > 0 else None
        nxt = carbons[i + 1] if i + 1 < n else None
        if prev is None:
            prev = c + (c - nxt) * 1.0 + np.array([0.0, 0.0, 0.0])
            prev = c - (nxt - c)
            # mirror of the next bond through the carbon, rotated into the zig-zag
            ang = np.array([-dx, 0.0, dz if i % 2 == 0 else -dz])
            prev = c + ang
        if nxt is None:
            ang = np.array([dx, 0.0, -dz if i % 2 == 1 else dz])
            nxt = c + ang
        hyd.extend(_tetra_hydrogens(c, prev, nxt, ch))
        if i == 0:
            d = (prev - c)
            hyd.append(c + ch * d / np.linalg.norm(d))
        if i == n - 1:
            d = (nxt - c)
            hyd.append(c + ch * d / np.linalg.norm(d))
    atoms += [(1, h) for h in hyd]
    return atoms


def _finish(atoms, rng, jitter):
    z = np.array([a[0] for a in atoms], dtype=np.uint8)
    xyz = np.array([a[1] for a in atoms], dtype=np.float64)
    if jitter:
        xyz = xyz + rng.uniform(-jitter, jitter, size=xyz.shape)
    return z, xyz * ANG


def alkane(n, seed=0, jitter=0.02, rng=None):
    rng = rng if rng is not None else np.random.default_rng(seed)
    return _finish(alkane_angstrom(n), rng, jitter)


def decane(seed=0):
    return alkane(10, seed=seed, jitter=0.02)


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def water_cluster(k, seed=0, spacing=3.1, centre_jitter=0.1, rng=None):
    """k waters on the first k sites of the smallest cube grid holding them (Bohr out)."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    side = 1
    while side ** 3 < k:
        side += 1
    r, half = 0.96, math.radians(104.5) / 2.0
    mono = np.array([[0.0, 0.0, 0.0], [r * math.sin(half), 0.0, r * math.cos(half)],
                     [-r * math.sin(half), 0.0, r * math.cos(half)]])
    z, xyz = [], []
    count = 0
    for i in range(side):
        for j in range(side):
            for l in range(side):
                if count == k:
                    break
                centre = np.array([i, j, l], dtype=float) * spacing
                centre = centre + rng.uniform(-centre_jitter, centre_jitter, size=3)
                rot = _random_rotation(rng)
                for zz, p in zip((8, 1, 1), mono):
                    z.append(zz)
                    xyz.append(centre + rot @ p)
                count += 1
    return np.array(z, dtype=np.uint8), np.array(xyz) * ANG


def batch(count, seed=0):
    """The mixed-size batch: alternating alkanes C_nH_2n+2 (n ~ U{1..40}) and water
    clusters (k ~ U{2..64}) with 0.02 A jitter."""
    rng = np.random.default_rng(seed)
    mols = []
    for i in range(count):
        if i % 2 == 0:
            n = int(rng.integers(1, 41))
            mols.append(alkane(n, jitter=0.02, rng=rng))
        else:
            k = int(rng.integers(2, 65))
            mols.append(water_cluster(k, centre_jitter=0.02, rng=rng))
    return mols


def substituted_chain(n, rng, p_s=0.1, p_cl=0.1, jitter=0.02):
    """Zig-zag C/S chain of n heavy atoms with hydrogens, some H replaced by Cl (Bohr out)."""
    theta = math.radians(109.471)
    sx, sz = math.sin(theta / 2.0), math.cos(theta / 2.0)
    kinds = [6] * n
    for i in range(1, n - 1):
        if rng.random() < p_s and kinds[i - 1] != 16:
            kinds[i] = 16
    pos = [np.zeros(3)]
    for i in range(1, n):
        b = 1.82 if (kinds[i] == 16 or kinds[i - 1] == 16) else 1.54
        step = np.array([sx, 0.0, sz if i % 2 == 1 else -sz]) * b
        pos.append(pos[-1] + step)
    atoms = [(kinds[i], pos[i]) for i in range(n)]
    hyd = []
    for i in range(n):
        if kinds[i] != 6:
            continue
        c = pos[i]
        if n == 1:
            s = 1.09 / math.sqrt(3.0)
            hyd += [(c, c + s * np.array(v, dtype=float)) for v in ((1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1))]
            continue
        prev = pos[i - 1] if i > 0 else c + np.array([-sx, 0.0, -sz if i % 2 == 1 else sz])
        nxt = pos[i + 1] if i + 1 < n else c + np.array([sx, 0.0, sz if (i + 1) % 2 == 1 else -sz])
        hyd += [(c, h) for h in _tetra_hydrogens(c, prev, nxt, 1.09)]
        if i == 0:
            d = prev - c
            hyd.append((c, c + 1.09 * d / np.linalg.norm(d)))
        if i == n - 1:
            d = nxt - c
            hyd.append((c, c + 1.09 * d / np.linalg.norm(d)))
    for c, h in hyd:
        if rng.random() < p_cl:
            d = (h - c) / np.linalg.norm(h - c)
            atoms.append((17, c + 1.77 * d))
        else:
            atoms.append((1, h))
    return _finish(atoms, rng, jitter)


def stream(count, seed=0, lo=3, hi=500):
    """Molecules of the served stream: sizes log-uniform in lo..hi atoms, alternating
    substituted chains and water clusters."""
    rng = np.random.default_rng(seed)
    mols = []
    for i in range(count):
        target = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        if i % 2 == 0:
            n = max(1, int(round((target - 2.0) / 3.0)))
            mols.append(substituted_chain(n, rng))
        else:
            k = max(1, int(round(target / 3.0)))
            mols.append(water_cluster(k, centre_jitter=0.1, rng=rng))
    return mols


def flat_alkane(n):
    """C_nH_{2n+2} as a flat all-anti zig-zag (1.26 Angstrom along x, 0.44 across y, CH2
    hydrogens at z = +-0.89, caps 1.09 Angstrom out along x): the one-dimensional chain of
    pm7-rs tests/dandc.rs:95-127, on which the divide-and-conquer subsystem count grows with
    n while the subsystem size does not. Returns (z, xyz in Bohr)."""
    dx, dy = 1.26, 0.44
    z, x = [], []
    for i in range(n):
        xx, yy = i * dx, (0.0 if i % 2 == 0 else dy)
        s = -0.5 if i % 2 == 0 else 0.5
        z += [6, 1, 1]
        x += [(xx, yy, 0.0), (xx, yy + s, 0.89), (xx, yy + s, -0.89)]
    z += [1, 1]
    x += [(-1.09, 0.0, 0.0), ((n - 1) * dx + 1.09, 0.0 if (n - 1) % 2 == 0 else dy, 0.0)]
    return np.array(z, dtype=np.uint8), np.array(x) * ANG
