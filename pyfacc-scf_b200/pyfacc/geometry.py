"""Seeded synthetic geometries of the benchmark workloads (bohr).

* ``water()``            O at the origin, O-H 0.958 A, H-O-H 104.5 deg
* ``alkane(n, seed)``    all-anti C_nH_{2n+2}: C-C 1.54 A, C-H 1.09 A,
                         tetrahedral angles, Gaussian jitter sigma on every
                         coordinate from numpy.random.default_rng(seed)
* ``radical(n, seed)``   the alkane with its first terminal H removed
* ``water_clusters(count, seed)``  (H2O)_n, n ~ U{4..16}: rigid monomers,
                         Haar-random orientations, O uniform in a cube of
                         side 3.1 n^(1/3) A, O-O >= 2.7 A by rejection
"""
from __future__ import annotations

import math

import numpy as np

ANG = 1.8897259886
TET = math.radians(109.4712)


def water():
    a = math.radians(104.5) / 2
    r = 0.958
    xyz = np.array([[0.0, 0.0, 0.0], [0.0, r * math.sin(a), r * math.cos(a)], [0.0, -r * math.sin(a), r * math.cos(a)]])
    return ["O", "H", "H"], xyz * ANG


def _unit(v):
    return v / np.linalg.norm(v)


def alkane(n: int, seed: int | None = None, sigma: float = 0.02, jitter: bool = True):
    """All-anti zig-zag C_nH_{2n+2} (bohr); carbons first, then hydrogens."""
    cc, ch = 1.54, 1.09
    dx = cc * math.sin(TET / 2)
    dy = cc * math.cos(TET / 2)
    C = np.array([[i * dx, (dy / 2) * (1 if i % 2 else -1), 0.0] for i in range(n)])
    zhat = np.array([0.0, 0.0, 1.0])
    H = []
    half = TET / 2
    for i in range(n):
        nb = []
        if i > 0:
            nb.append(_unit(C[i - 1] - C[i]))
        if i < n - 1:
            nb.append(_unit(C[i + 1] - C[i]))
        if len(nb) == 2:
            b = _unit(-(nb[0] + nb[1]))
            for s in (+1, -1):
                H.append(C[i] + ch * (math.cos(half) * b + s * math.sin(half) * zhat))
        else:
            # methyl (or methane): one H in-plane trans to the backbone, two out of plane
            u = nb[0] if nb else np.array([1.0, 0.0, 0.0])
            perp = np.array([-u[1], u[0], 0.0])
            if np.linalg.norm(perp) < 1e-12:
                perp = np.array([0.0, 1.0, 0.0])
            perp = _unit(perp)
            # in-plane direction pointing away from the next-but-one carbon
            if i == 0 and n > 2:
                ref = C[2] - C[1]
            elif i == n - 1 and n > 2:
                ref = C[n - 3] - C[n - 2]
            else:
                ref = perp
            if np.dot(perp, ref) > 0:
                perp = -perp
            w = np.cross(u, perp)
            count = 3 if nb else 4
            if not nb:  # methane
                dirs = [np.array(d) / math.sqrt(3) for d in ((1, 1, 1), (1, -1, -1), (-1, 1, -1), (-1, -1, 1))]
            else:
                dirs = []
                for k in range(3):
                    phi = 2 * math.pi * k / 3
                    d = math.cos(TET) * u + math.sin(TET) * (math.cos(phi) * perp + math.sin(phi) * w)
                    dirs.append(d)
            for d in dirs[:count]:
                H.append(C[i] + ch * _unit(d))
    xyz = np.vstack([C, np.array(H)])
    if jitter and seed is not None and sigma > 0:
        rng = np.random.default_rng(seed)
        xyz = xyz + rng.normal(0.0, sigma, size=xyz.shape)
    species = ["C"] * n + ["H"] * (len(xyz) - n)
    return species, xyz * ANG


def radical(n: int, seed: int | None = None, sigma: float = 0.02):
    """C_nH_{2n+1}: the alkane with the first terminal (in-plane methyl) H removed."""
    sp, xyz = alkane(n, seed, sigma)
    drop = n  # first hydrogen = in-plane H of the first methyl
    keep = [i for i in range(len(sp)) if i != drop]
    return [sp[i] for i in keep], xyz[keep]


def _haar_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d],
    ])


def water_cluster(n: int, rng, min_oo: float = 2.7, max_tries: int = 100000):
    sp0, w = water()
    w = w / ANG
    side = 3.1 * n ** (1.0 / 3.0)
    Os = []
    tries = 0
    while len(Os) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("water cluster placement failed")
        p = rng.uniform(0.0, side, size=3)
        if all(np.linalg.norm(p - o) >= min_oo for o in Os):
            Os.append(p)
    sp, xyz = [], []
    for o in Os:
        R = _haar_rotation(rng)
        for s, r in zip(sp0, w):
            sp.append(s)
            xyz.append(o + R @ r)
    return sp, np.array(xyz) * ANG


def water_clusters(count: int = 256, seed: int = 3, nmin: int = 4, nmax: int = 16):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        out.append(water_cluster(n, rng))
    return out
