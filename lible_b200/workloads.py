"""Seeded synthetic inputs: water monomer, water clusters and random occupied densities.

Water geometry: O at the origin, H at (+-1.4305, 1.1093, 0) bohr.  A cluster of n waters puts the
molecules on the first n sites of a ceil(n^(1/3))^3 cubic lattice with 5.7 bohr spacing, rotates
each one uniformly at random about its oxygen and jitters it rigidly by U(-0.6, 0.6) bohr per axis,
all drawn from numpy's PCG64 generator with the given seed.  A density is D = C C^T with C (N x occ)
drawn N(0, 1) from the same generator and orthonormalised by a reduced QR.
"""
import math

import numpy as np

WATER_BOHR = np.array([[0.0, 0.0, 0.0], [1.4305, 1.1093, 0.0], [-1.4305, 1.1093, 0.0]])
WATER_Z = [8, 1, 1]
SPACING = 5.7
JITTER = 0.6


def water_cluster(n, seed):
    """Returns (atomic numbers, coordinates in bohr [3n, 3], rng after the geometry draws)."""
    from scipy.spatial.transform import Rotation

    rng = np.random.default_rng(seed)
    side = max(1, math.ceil(round(n ** (1.0 / 3.0), 12)))
    while side ** 3 < n:
        side += 1
    sites = [(i, j, k) for i in range(side) for j in range(side) for k in range(side)][:n]
    Z, xyz = [], []
    for site in sites:
        rot = Rotation.random(random_state=rng)
        shift = rng.uniform(-JITTER, JITTER, size=3)
        pos = rot.apply(WATER_BOHR) + np.array(site, dtype=float) * SPACING + shift
        Z.extend(WATER_Z)
        xyz.append(pos)
    return Z, np.vstack(xyz), rng


def random_density(nao, occ, rng):
    C = rng.standard_normal((nao, occ))
    Q, _ = np.linalg.qr(C, mode="reduced")
    return Q @ Q.T


def even_tempered_aux(Z, lmax=3, n_exp=12, base=0.1, ratio=2.5):
    """Per-atom auxiliary basis of uncontracted shells l = 0..lmax with exponents base*ratio^k."""
    shells = [(l, [base * ratio ** k], [1.0]) for l in range(lmax + 1) for k in range(n_exp)]
    return [list(shells) for _ in Z]


def batch_clusters(n_mol=64, seed=7, n_max=12):
    """The heterogeneous batch: n_mol water clusters with n drawn uniformly from 1..n_max, even
    index cc-pVDZ and odd index cc-pVTZ; each cluster and its density (occupation 5n) come from
    their own generator seeded with (seed, index).  Returns [(basis, Z, xyz, D_factory)], where
    D_factory(nao) draws the density."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, n_max + 1, size=n_mol)
    out = []
    for i, n in enumerate(sizes):
        Z, xyz, r = water_cluster(int(n), seed * 1000 + i)
        basis = "cc-pvdz" if i % 2 == 0 else "cc-pvtz"
        out.append((basis, Z, xyz, (lambda nao, r=r, n=int(n): random_density(nao, 5 * n, r))))
    return out
