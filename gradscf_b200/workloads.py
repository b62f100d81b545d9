"""Seeded synthetic water-cluster inputs for the J/K workloads.

Generator (all lengths in Angstrom):
  * monomer: O (0, 0, 0), H (0, +-0.7572, 0.5865) -- the single-water geometry;
  * lattice: the first N points, in C order, of a k x k x k cubic grid with
    k = ceil(N^(1/3)) and spacing 3.1, centred on the origin;
  * per monomer, in lattice order: a jitter U(-0.3, 0.3) per axis, then a
    uniform rotation about the monomer's nuclear-charge centre (a normalised
    4-D Gaussian quaternion); the rotation is redrawn while any atom lies
    closer than 1.3 to an atom of an already placed monomer.
  * random numbers: numpy.random.default_rng(seed), draws in the order above.
Workload seeds: (H2O)32 cc-pVDZ seed 1; (H2O)16 6-31G* seed 2; batch of 256
clusters with N ~ U{1..24} drawn from seed 3 and cluster m built with seed
1000+m; (H2O)64 cc-pVTZ seed 4.
"""
from __future__ import annotations

import math

import numpy as np

MONOMER = np.array([[0.0, 0.0, 0.0], [0.0, 0.7572, 0.5865], [0.0, -0.7572, 0.5865]])
CHARGES = np.array([8.0, 1.0, 1.0])
SPACING = 3.1
JITTER = 0.3
MIN_DIST = 1.3


def _rotation(q):
    a, b, c, d = q / np.linalg.norm(q)
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def water_cluster_coords(n: int, seed: int) -> np.ndarray:
    """(3n, 3) coordinates in Angstrom, atoms O, H, H per monomer."""
    rng = np.random.default_rng(seed)
    k = max(1, math.ceil(round(n ** (1.0 / 3.0), 12)))
    while k ** 3 < n:
        k += 1
    grid = np.array([(i, j, l) for i in range(k) for j in range(k) for l in range(k)], dtype=float)
    points = (grid[:n] - (k - 1) / 2.0) * SPACING
    centre = (CHARGES[:, None] * MONOMER).sum(0) / CHARGES.sum()
    local = MONOMER - centre
    placed = np.zeros((0, 3))
    for m in range(n):
        shift = points[m] + rng.uniform(-JITTER, JITTER, size=3)
        while True:
            atoms = local @ _rotation(rng.normal(size=4)).T + shift
            if placed.shape[0] == 0:
                break
            d = np.linalg.norm(atoms[:, None, :] - placed[None, :, :], axis=-1)
            if d.min() >= MIN_DIST:
                break
        placed = np.concatenate([placed, atoms])
    return placed


def water_cluster(n: int, seed: int) -> str:
    """'Sym x y z; ...' specification (Angstrom) of the seeded (H2O)_n cluster."""
    xyz = water_cluster_coords(n, seed)
    syms = ["O", "H", "H"] * n
    return "; ".join(f"{s} {x:.10f} {y:.10f} {z:.10f}" for s, (x, y, z) in zip(syms, xyz))


WATER = "O 0 0 0; H 0 0.7572 0.5865; H 0 -0.7572 0.5865"


def batch_sizes(count=256, seed=3, low=1, high=24):
    return np.random.default_rng(seed).integers(low, high + 1, size=count)


def psd_density(n: int, nocc: int, seed: int) -> np.ndarray:
    """D = C C^T with C ~ N(0, 1)/sqrt(n), nocc columns (seeded)."""
    c = np.random.default_rng(seed).normal(size=(n, nocc)) / np.sqrt(n)
    return c @ c.T
