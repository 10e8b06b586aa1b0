import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA engine through the C ABI")


@pytest.fixture(scope="session")
def engine():
    from crabsaxs_b200.api import Engine

    e = Engine.default(int(os.environ.get("CRAB_DEVICE", "0")))
    yield e


def rel_err(a, b, floor=0.0):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


# Reference test structures (restated from the reference's unit tests).
def helix96():
    """scattering.rs:312-339: 96 mixed atoms on a golden-angle helix (C/N/O/S/P)."""
    idx = np.arange(96)
    angle = idx * 2.399963229728653
    radial = 4.0 + (idx % 13)
    xyz = np.stack([radial * np.cos(angle), radial * np.sin(angle), (idx - 47.5) * 0.31], axis=1)
    el = np.array([[1, 2, 3, 4, 5][i % 5] for i in idx], dtype=np.int32)
    return xyz, el


def ring24():
    """spherical.rs:682-705: 24 atoms, C/N/O/S."""
    idx = np.arange(24)
    angle = idx * 0.71
    xyz = np.stack([7.0 * np.cos(angle), 7.0 * np.sin(angle), idx * 0.45 - 5.0], axis=1)
    el = np.array([[1, 2, 3, 4][i % 4] for i in idx], dtype=np.int32)
    return xyz, el


def chain8():
    """spherical.rs:731-753: 8 atoms for the adaptive-grid six-term test."""
    idx = np.arange(8)
    xyz = np.stack([idx * 1.4 - 4.9, np.sin(idx * 0.9) * 2.0, np.cos(idx * 0.7)], axis=1)
    el = np.array([[1, 2, 3, 4][i % 4] for i in idx], dtype=np.int32)
    return xyz, el


def two_atoms_co():
    """solvent.rs:623-648: C at (-1,0,0), O at (1,0,0)."""
    return np.array([[-1.0, 0, 0], [1.0, 0, 0]]), np.array([1, 3], dtype=np.int32)


def two_carbons():
    """examples/data/small.pdb: two carbons 2 Å apart (scattering.rs:219-244)."""
    return np.array([[0.0, 0, 0], [2.0, 0, 0]]), np.array([1, 1], dtype=np.int32)
