"""The C ABI library loads, exports every function include/crab_cuda.h declares,
and its host-only entry points agree with the oracle (no GPU needed)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from crabsaxs_b200 import _native as N

HEADER = Path(__file__).resolve().parents[1] / "include" / "crab_cuda.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(crab_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_function_is_exported_and_bound():
    names = declared_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(N.lib, name), name
    assert set(names) == set(N.EXPORTED), set(names) ^ set(N.EXPORTED)


def test_context_creation_reports_a_status_code():
    h = C.c_void_p()
    st = N.lib.crab_ctx_create(0, C.byref(h))
    assert st in (N.OK, N.ENODEVICE)
    if st == N.OK:
        N.lib.crab_ctx_destroy(h)
    assert N.lib.crab_ctx_create(0, None) == N.EINVAL


RESIDUES = ["ALA", "ARG", "ASN", "ASP", "ASH", "CYS", "CYX", "GLN", "GLU", "GLH", "GLY", "HIS", "HID", "HIE", "HIP",
            "ILE", "LEU", "LYS", "MET", "MSE", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL", "PCA", "A", "DA", "RA",
            "ADE", "C", "DC", "G", "DG", "U", "T", "DT", "THY", "HOH", "SYN", "TST", " ala "]
NAMES = ["N", "CA", "C", "O", "CB", "CG", "CD", "CE", "NZ", "NE", "NH1", "NH2", "ND1", "ND2", "NE1", "NE2", "OD1",
         "OD2", "OE1", "OE2", "OG", "OG1", "OH", "SG", "SD", "CG1", "CG2", "CD1", "CD2", "CE1", "CE2", "CE3", "CZ",
         "CZ2", "CZ3", "CH2", "C1'", "C2'", "C3'", "C4'", "C5'", "O2'", "C2*", "OP1", "O1P", "C8", "C2", "N6", "N1",
         "N2", "N4", "C5", "C6", "N3", "C7", "C5M", "HB1", " cb "]


def test_united_atom_typing_matches_oracle():
    for r in RESIDUES:
        for a in NAMES:
            assert N.lib.crab_united_atom_group(r.encode(), a.encode()) == O.lib.orc_united_atom_group(
                r.encode(), a.encode()), (r, a)


def test_form_factor_and_volume_tables_match_oracle():
    for e in range(15):
        for g in range(-1, 14):
            for implicit in (0, 1):
                assert N.lib.crab_excluded_volume_for_atom(e, g, implicit) == O.lib.orc_excluded_volume_for_atom(
                    e, g, implicit)
                for q in (0.0, 0.013, 0.2, 0.5, 0.9):
                    a = N.lib.crab_form_factor(e, g, 0.75, implicit, q)
                    b = O.lib.orc_form_factor(e, g, 0.75, implicit, q)
                    assert a == b, (e, g, implicit, q)


def test_combine_solvent_basis_matches_oracle():
    rng = np.random.default_rng(0)
    q = np.linspace(0.0, 0.5, 37)
    basis = rng.normal(size=(6, 37)) * 100 + 200
    out = np.empty(37)
    assert N.lib.crab_combine_solvent_basis(q.ctypes.data_as(N.D), 37, basis.ctypes.data_as(N.D), 1.03, 0.7,
                                            out.ctypes.data_as(N.D)) == N.OK
    np.testing.assert_array_equal(out, O.combine_solvent_basis(basis, q, 1.03, 0.7))


def test_reweight_curves_matches_oracle():
    import crabsaxs_b200 as cs

    rng = np.random.default_rng(2)
    curves = rng.uniform(0.5, 2.0, size=(6, 40))
    y = 0.5 * curves[0] + 0.5 * curves[4] + 0.01 * rng.normal(size=40)
    sigma = np.full(40, 0.02)
    q = np.linspace(0.01, 0.4, 40)
    ex = cs.ExperimentalCurve(q, y, sigma)
    opt = cs.MaximumEntropyOptions(kl_strength=0.05)
    got = cs.reweight_curves([f"c{i}" for i in range(6)], curves, ex, opt)
    ref = O.reweight_curves(curves, y, sigma, kl_strength=0.05)
    np.testing.assert_allclose(got.weights, ref["weights"], rtol=0, atol=1e-12)
    assert got.iterations == ref["iterations"]
    assert got.reduced_chi2 == pytest.approx(ref["reduced_chi2"], rel=1e-12)


def test_reweight_rejects_invalid_options():
    import crabsaxs_b200 as cs

    ex = cs.ExperimentalCurve([0.01, 0.02], [0.2, 0.8], [0.01, 0.01])
    with pytest.raises(cs.InvalidInput):
        cs.reweight_curves(["a", "b"], [[1.0, 0.0], [0.0, 1.0]], ex, cs.MaximumEntropyOptions(min_weight=0.6))
    with pytest.raises(cs.InvalidInput):
        cs.reweight_curves(["a"], [[1.0, 0.0], [0.0, 1.0]], ex)


def test_synthetic_structures_are_deterministic_and_shaped():
    from crabsaxs_b200 import synth

    a = synth.protein(7, 5000, 28.0)
    b = synth.protein(7, 5000, 28.0)
    c = synth.protein(8, 5000, 28.0)
    np.testing.assert_array_equal(a.xyz, b.xyz)
    assert not np.array_equal(a.xyz, c.xyz)
    frac = np.bincount(a.element, minlength=5)[1:5] / 5000
    assert abs(frac[0] - 0.63) < 0.03 and abs(frac[1] - 0.17) < 0.03 and abs(frac[2] - 0.19) < 0.03
    r = np.linalg.norm(a.xyz - a.xyz.mean(axis=0), axis=1)
    assert r.max() < 28.0 + 8.0


def test_ensemble_sizes_are_log_uniform_in_range():
    from crabsaxs_b200 import synth

    s = synth.ensemble_sizes()
    assert len(s) == 256 and s.min() >= 2000 and s.max() <= 40000
    assert 9000 < np.mean(s) < 16000
