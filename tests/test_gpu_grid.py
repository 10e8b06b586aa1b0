"""Hydration-shell sites from the device are bit-exact against the oracle
(site set and z→y→x order), for the adaptive coarse shell
(solvent.rs:121-223) and the exterior flood-fill shell (solvent.rs:259-401)."""
import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O
from conftest import chain8, helix96, two_atoms_co

pytestmark = pytest.mark.gpu


def _cases():
    yield "co", *two_atoms_co()
    yield "chain8", *chain8()
    yield "helix96", *helix96()
    from crabsaxs_b200 import synth

    s = synth.protein(5, 2000, 18.0)
    yield "synth2000", s.xyz, s.element.astype(np.int32)


@pytest.mark.parametrize("spacing", [8.0, 4.0, 3.0, 2.5])
def test_adaptive_grid_bit_exact(engine, spacing):
    for name, xyz, el in _cases():
        s = cs.Structure(xyz, el)
        got, gv = cs.hydration_grid_adaptive(s, spacing, engine=engine)
        ref, rv = O.adaptive_grid(xyz, spacing)
        assert gv == rv
        assert got.shape == ref.shape, name
        assert np.array_equal(got, ref), name


def test_adaptive_grid_config2_bit_exact(engine):
    from crabsaxs_b200 import synth

    w = synth.CONFIG2
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    got, _ = cs.hydration_grid_adaptive(s, 3.0, engine=engine)
    ref, _ = O.adaptive_grid(s.xyz, 3.0)
    assert np.array_equal(got, ref)
    # shell is clearance..clearance+width(Rg) from the nearest atom
    assert 0.05 < len(got) / s.atom_count < 2.0


def test_adaptive_grid_translation_invariant(engine):  # solvent.rs:740-771
    xyz, el = two_atoms_co()
    shift = np.array([3.17, -8.4, 2.6])
    a, _ = cs.hydration_grid_adaptive(cs.Structure(xyz, el), engine=engine)
    b, _ = cs.hydration_grid_adaptive(cs.Structure(xyz + shift, el), engine=engine)
    assert a.shape == b.shape and np.all(np.linalg.norm(b - a - shift, axis=1) < 1e-12)


def test_adaptive_grid_rejects_bad_spacing(engine):
    xyz, el = two_atoms_co()
    with pytest.raises(cs.InvalidInput):
        cs.hydration_grid_adaptive(cs.Structure(xyz, el), 0.0, engine=engine)


@pytest.mark.parametrize("spacing", [1.0, 1.5])
def test_exterior_grid_bit_exact(engine, spacing):
    for name, xyz, el in _cases():
        s = cs.Structure(xyz, el)
        got, gv = cs.hydration_grid_exterior(s, spacing, engine=engine)
        ref, rv = O.exterior_grid(xyz, el, spacing)
        assert gv == rv
        assert got.shape == ref.shape, name
        assert np.array_equal(got, ref), name


def test_exterior_grid_single_atom_bounds(engine):  # solvent.rs:688-705
    xyz = np.array([[-1.0, 0.0, 0.0]])
    got, _ = cs.hydration_grid_exterior(cs.Structure(xyz, [1]), engine=engine)
    d = np.linalg.norm(got - xyz[0], axis=1)
    assert len(got) > 0 and np.all(d > 1.7 + 1.4) and np.all(d <= 1.7 + 1.4 + 3.0 + 1e-12)


def test_exterior_grid_limit(engine):
    xyz = np.array([[0.0, 0.0, 0.0], [700.0, 700.0, 700.0]])
    with pytest.raises(cs.InvalidInput):
        cs.hydration_grid_exterior(cs.Structure(xyz, [1, 1]), 0.1, engine=engine)
