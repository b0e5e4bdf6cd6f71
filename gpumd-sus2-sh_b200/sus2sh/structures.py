"""Seeded synthetic structures of the benchmark workloads (the reference's
million-atom Cu-Zr model.xyz is not shipped; these generators stand in for it).

All positions are returned SoA, shape (3, N), in Angstrom; boxes as
``potential.Box``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .potential import Box

AMU = {"Cu": 63.546, "Zr": 91.224, "Al": 26.9815385}
KB_EV = 8.617333262e-5          # eV/K
ACCEL = 9.648533212331002e-3    # (eV/A/amu) -> A/fs^2


def _species(n: int, fractions, rng) -> np.ndarray:
    """Exact species counts from fractions, randomly permuted."""
    counts = [int(round(f * n)) for f in fractions]
    counts[-1] = n - sum(counts[:-1])
    t = np.concatenate([np.full(c, s, dtype=np.int32) for s, c in enumerate(counts)])
    return rng.permutation(t).astype(np.int32)


def fcc(nx: int, ny: int, nz: int, a: float, fractions=(0.5, 0.5), jitter: float = 0.0, seed: int = 0):
    """FCC crystal of nx*ny*nz cubic cells (4 atoms each), random species with
    exact fractions, Gaussian jitter N(0, jitter) per coordinate."""
    rng = np.random.default_rng(seed)
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    cells = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1).astype(np.float64)
    pos = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    N = pos.shape[0]
    types = _species(N, fractions, rng)
    if jitter > 0:
        pos = pos + rng.normal(0.0, jitter, size=pos.shape)
    box = Box.orthorhombic(nx * a, ny * a, nz * a)
    pos = np.mod(pos, np.array([nx * a, ny * a, nz * a]))
    return box, types, np.ascontiguousarray(pos.T)


def random_insertion(N: int, density: float, dmin: float, edge_ratios=(1.0, 1.0, 1.0),
                     fractions=(0.5, 0.5), seed: int = 0):
    """Random sequential insertion at number density ``density`` (A^-3) with
    minimum distance ``dmin`` in an orthorhombic periodic box whose edges are
    proportional to ``edge_ratios``."""
    rng = np.random.default_rng(seed)
    r = np.asarray(edge_ratios, dtype=np.float64)
    scale = (N / density / np.prod(r)) ** (1.0 / 3.0)
    lx, ly, lz = (r * scale).tolist()
    pos = np.zeros(3 * N)
    lib = _lib.load_tools()
    rc = lib.sus2sh_random_insertion(N, lx, ly, lz, dmin, ctypes.c_ulonglong(int(seed) & (2**64 - 1)),
                                     pos.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise RuntimeError("random insertion budget exhausted")
    types = _species(N, fractions, rng)
    return Box.orthorhombic(lx, ly, lz), types, pos.reshape(3, N)


def maxwell_boltzmann(types: np.ndarray, masses, temperature: float, seed: int = 0) -> np.ndarray:
    """Velocities (3, N) in A/fs at ``temperature`` K, zero total momentum,
    rescaled so the kinetic temperature (3N-3 degrees of freedom) is exact."""
    rng = np.random.default_rng(seed)
    m = np.asarray(masses, dtype=np.float64)[types]
    sigma = np.sqrt(KB_EV * temperature / m * ACCEL)  # sqrt(kT/m) in A/fs
    v = rng.normal(size=(3, types.size)) * sigma
    p = (v * m).sum(axis=1) / m.sum()
    v -= p[:, None]
    ke = 0.5 * (m * v * v).sum() / ACCEL  # eV
    t_now = 2.0 * ke / ((3 * types.size - 3) * KB_EV)
    if t_now > 0:
        v *= np.sqrt(temperature / t_now)
    return np.ascontiguousarray(v)


def cell_batch(n_cells: int, n_min: int = 16, n_max: int = 512, density: float = 0.06, dmin: float = 2.1,
               ratio_range=(0.8, 1.25), fractions=(0.5, 0.5), seed: int = 0):
    """Batch of independent periodic random-insertion cells with atom counts
    uniform in [n_min, n_max] and orthorhombic edge ratios uniform in
    ratio_range.  Returns (offsets[n_cells+1], cell_h[n_cells, 9], boxes,
    types[N], positions[3, N]) with the cells concatenated."""
    rng = np.random.default_rng(seed)
    counts = rng.integers(n_min, n_max + 1, size=n_cells)
    offsets = np.zeros(n_cells + 1, dtype=np.int32)
    offsets[1:] = np.cumsum(counts)
    hs, boxes, ts, ps = [], [], [], []
    for c in range(n_cells):
        ratios = rng.uniform(ratio_range[0], ratio_range[1], size=3)
        box, types, pos = random_insertion(int(counts[c]), density, dmin, ratios, fractions,
                                           seed=int(rng.integers(1 << 31)))
        hs.append(box.cpu_h)
        boxes.append(box)
        ts.append(types)
        ps.append(pos)
    return (offsets, np.stack(hs), boxes, np.concatenate(ts).astype(np.int32),
            np.ascontiguousarray(np.concatenate(ps, axis=1)))
