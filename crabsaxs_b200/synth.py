"""Seeded synthetic workloads with the shapes of the five benchmark configurations.

No public dataset is named for the path, and the reference's validation PDB
files are downloaded at run time; these generated structures stand in for
them with the stated sizes, radii and element mix.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .api import Structure


def protein(seed: int, n_atoms: int, radius: float) -> Structure:
    """Cα-walk protein-like structure (crab_synth_protein), residue code 'SYN'
    (no united-atom groups, so element Cromer–Mann form factors apply)."""
    xyz = np.empty((n_atoms, 3))
    el = np.empty(n_atoms, dtype=np.int8)
    st = N.lib.crab_synth_protein(C.c_uint64(seed), n_atoms, radius, xyz.ctypes.data_as(N.D),
                                  el.ctypes.data_as(N.I8P))
    if st != N.OK:
        raise ValueError("invalid synthetic structure request")
    return Structure(xyz, el)


def q_grid(lo: float, hi: float, n: int) -> np.ndarray:
    return np.linspace(lo, hi, n)


@dataclass
class Workload:
    name: str
    n_atoms: int
    radius: float
    q: np.ndarray
    seed: int


# 1,000 atoms, R 20 Å, q 0.005..0.5 step 0.005.
DEBYE_1K = Workload("debye-1k", 1000, 20.0, np.arange(1, 101) * 0.005, 1)
# 20,000 atoms, R 45 Å, plus adaptive 3 Å hydration sites; 500 q on [0.001, 0.5].
DEBYE_20K_SOLVATED = Workload("debye-20k-solvated", 20000, 45.0, q_grid(0.001, 0.5, 500), 2)
# 100,000 atoms, R 80 Å, 1000 q on [0.001, 0.6], l_max 50.
ATOMS_100K = Workload("multipole-100k", 100000, 80.0, q_grid(0.001, 0.6, 1000), 3)
# 5,000 atoms, R 28 Å, q 0.005..0.5 step 0.005.
GRADIENT_5K = Workload("gradient-5k", 5000, 28.0, np.arange(1, 101) * 0.005, 4)
# Ensemble: 256 conformers, N log-uniform in [2000, 40000]; 300 q on [0.005, 0.45].
ENSEMBLE_Q = q_grid(0.005, 0.45, 300)


def ensemble_sizes(k: int = 256, seed: int = 5, lo: int = 2000, hi: int = 40000) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), size=k))).astype(np.int64)


def ensemble(k: int = 256, seed: int = 5, lo: int = 2000, hi: int = 40000) -> list[Structure]:
    """Conformers with per-conformer seeds; radius scaled as N^(1/3) around 45 Å at 20k atoms."""
    sizes = ensemble_sizes(k, seed, lo, hi)
    return [protein(1000 + seed * 100003 + i, int(n), 45.0 * (n / 20000.0) ** (1.0 / 3.0))
            for i, n in enumerate(sizes)]


def solvent_draw(seed: int = 2) -> tuple[float, float]:
    """c1 ~ U[0.95, 1.05], c2 ~ U[0, 2] from the seed (the 20,000-atom solvated workload)."""
    rng = np.random.default_rng(seed)
    return float(rng.uniform(0.95, 1.05)), float(rng.uniform(0.0, 2.0))
