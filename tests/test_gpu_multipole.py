"""Multipole engine on the GPU against the oracle's direct f64 multipole
(spherical.rs:266-565) and against Debye, as the reference's own tests do.

Tolerances: the FP64 device path must equal the oracle to 1e-9 relative
(the radial interpolation is exact to ~1e-15; the rest is f64 round-off);
the FP32 path to 1e-5 relative per q (basis terms: relative to the largest
magnitude of that term, as cross terms pass through zero).  Multipole against
Debye keeps the reference's own gates (truncation error, not precision).
"""
import math

import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O
from crabsaxs_b200 import _native as N
from crabsaxs_b200 import synth

from conftest import chain8, helix96, ring24, two_carbons

pytestmark = pytest.mark.gpu

FP32_RTOL = 1e-5
FP64_RTOL = 1e-9


def _rel(got, ref):
    return np.max(np.abs(got - ref) / np.abs(ref))


def _oracle_atoms(s: cs.Structure):
    return O.Atoms(s.xyz, s.element, s.group, s.occupancy)


@pytest.mark.parametrize("fixture,l_max", [(helix96, 16), (helix96, 32), (ring24, 24)])
def test_multipole_intensity_matches_oracle(engine, fixture, l_max):
    xyz, el = fixture()
    s = cs.Structure(xyz, el)
    q = np.concatenate([[0.0], np.arange(1, 101) * 0.005])
    ref = O.multipole_intensity(_oracle_atoms(s), q, l_max)
    got64 = cs.multipole_intensity(s, q, l_max, precision=N.PREC_FP64, engine=engine)
    got32 = cs.multipole_intensity(s, q, l_max, precision=N.PREC_FP32, engine=engine)
    assert _rel(got64, ref) <= FP64_RTOL
    assert _rel(got32, ref) <= FP32_RTOL


def test_two_atom_multipole_matches_debye(engine):  # spherical.rs:595-634
    xyz, el = two_carbons()
    s = cs.Structure(xyz, el)
    q = np.array([0.1, 0.2, 0.5])
    m = cs.multipole_intensity(s, q, 32, engine=engine)
    d = O.debye_intensity(_oracle_atoms(s), q)
    assert np.all(np.abs(m - d) / d < 1e-6)


def test_large_separation_multipole_matches_debye(engine):  # spherical.rs:636-678
    s = cs.Structure(np.array([[-20.0, 0, 0], [20.0, 0, 0]]), np.array([1, 3]))
    q = np.array([0.2, 0.35, 0.5])
    m = cs.multipole_intensity(s, q, 32, engine=engine)
    d = O.debye_intensity(_oracle_atoms(s), q)
    assert np.all(np.abs(m - d) / d < 1e-6)


def test_adaptive_public_multipole_matches_debye(engine):  # scattering.rs:311-365
    xyz, el = helix96()
    s = cs.Structure(xyz, el)
    q = np.arange(1, 101) * 0.005
    opt = cs.ComputeOptions(method=cs.ScatteringMethod.Multipole)
    m = cs.compute_curve(s, q, opt, engine=engine).intensity
    d = O.debye_intensity(_oracle_atoms(s), q)
    assert math.sqrt(np.sum((m - d) ** 2) / np.sum(d**2)) <= 1e-3


@pytest.mark.parametrize("model,spacing", [(0, 4.0), (2, 8.0), (2, 3.0), (1, 4.0)])
def test_solvent_basis_matches_oracle(engine, model, spacing):
    xyz, el = chain8() if model == 2 and spacing == 8.0 else helix96()
    s = cs.Structure(xyz, el)
    q = np.arange(1, 51) * 0.01
    p = cs.SolventParams(c1=1.02, c2=0.7, hydration_model=cs.HydrationModel(model), hydration_grid_spacing_angstrom=spacing)
    ref = O.multipole_solvent_basis(_oracle_atoms(s), q, 24, c1=p.c1, c2=p.c2, model=model, spacing=spacing)
    for prec, tol in [(N.PREC_FP64, FP64_RTOL), (N.PREC_FP32, FP32_RTOL)]:
        got = cs.multipole_solvent_basis(s, q, 24, p, precision=prec, engine=engine)
        for k in range(6):
            scale = max(np.max(np.abs(ref[k])), 1e-300)
            assert np.max(np.abs(got[k] - ref[k])) / scale <= tol, (prec, k)


def test_six_term_grid_basis_matches_debye(engine):  # spherical.rs:729-787
    xyz, el = chain8()
    s = cs.Structure(xyz, el)
    q = np.arange(1, 51) * 0.01
    p = cs.SolventParams(hydration_model=cs.HydrationModel.AdaptiveGrid, hydration_grid_spacing_angstrom=8.0)
    m = cs.multipole_solvent_basis(s, q, 32, p, engine=engine)
    d = O.debye_solvent_basis(_oracle_atoms(s), q, model=2, spacing=8.0)
    for k in range(6):
        err = math.sqrt(np.sum((m[k] - d[k]) ** 2) / max(np.sum(d[k] ** 2), 1e-30))
        assert err <= 1e-3, (k, err)


@pytest.mark.parametrize("model", [0, 2])
def test_solvent_curve_matches_oracle(engine, model):
    s = synth.protein(31, 800, 14.0)
    q = np.linspace(0.0, 0.5, 60)
    p = cs.SolventParams(c1=0.98, c2=1.3, hydration_model=cs.HydrationModel(model), hydration_grid_spacing_angstrom=3.0)
    opt = cs.ComputeOptions(method=cs.ScatteringMethod.Multipole, solvent=p, multipole_l_max=24)
    got = cs.compute_curve(s, q, opt, engine=engine)
    assert got.method == "Multipole"
    ref = O.multipole_solvent_intensity(_oracle_atoms(s), q, 24, c1=p.c1, c2=p.c2, model=model, spacing=3.0)
    assert _rel(got.intensity, ref) <= FP32_RTOL


def test_synthetic_protein_fp32_matches_oracle(engine):
    s = synth.protein(32, 3000, 20.0)
    q = np.linspace(0.001, 0.5, 150)
    ref = O.multipole_intensity(_oracle_atoms(s), q, 30)
    got = cs.multipole_intensity(s, q, 30, engine=engine)
    assert _rel(got, ref) <= FP32_RTOL


def test_wide_q_range_uses_several_radial_segments(engine):
    """q·r_max ≈ 120 needs more than 64 nodes on [0, r_max]: the radial range
    is cut into segments, each with its own nodes."""
    s = synth.protein(33, 600, 12.0)
    q = np.linspace(0.01, 2.5, 40)
    ref = O.multipole_intensity(_oracle_atoms(s), q, 64)
    got64 = cs.multipole_intensity(s, q, 64, precision=N.PREC_FP64, engine=engine)
    got32 = cs.multipole_intensity(s, q, 64, engine=engine)
    assert _rel(got64, ref) <= FP64_RTOL
    assert _rel(got32, ref) <= FP32_RTOL


def test_100k_subset_matches_oracle_and_fp64(engine):
    """100,000 atoms (R 80 Å), 1000 q on [0.001, 0.6], L = 50: FP32 against the
    FP64 device path on every q, and against the oracle on every 50th q."""
    w = synth.ATOMS_100K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    got32 = cs.multipole_intensity(s, w.q, 50, engine=engine)
    got64 = cs.multipole_intensity(s, w.q, 50, precision=N.PREC_FP64, engine=engine)
    assert _rel(got32, got64) <= FP32_RTOL
    sub = np.arange(0, len(w.q), 50)
    ref = O.multipole_intensity(_oracle_atoms(s), w.q[sub], 50)
    assert _rel(got64[sub], ref) <= FP64_RTOL
    assert _rel(got32[sub], ref) <= FP32_RTOL


def test_auto_method_switches_to_multipole_at_500_atoms(engine):  # scattering.rs:145-156
    q = np.linspace(0.01, 0.3, 20)
    small = synth.protein(34, 499, 10.0)
    large = synth.protein(34, 500, 10.0)
    assert cs.compute_curve(small, q, cs.ComputeOptions(), engine=engine).method == "Debye"
    assert cs.compute_curve(large, q, cs.ComputeOptions(), engine=engine).method == "Multipole"


def test_empty_structure_and_invalid_arguments(engine):
    q = np.linspace(0.01, 0.3, 5)
    empty = cs.Structure(np.zeros((0, 3)), np.zeros(0, dtype=np.int8))
    assert np.all(cs.multipole_intensity(empty, q, 16, engine=engine) == 0.0)
    s = synth.protein(35, 50, 8.0)
    with pytest.raises(cs.InvalidInput):
        cs.multipole_intensity(s, q, 65, engine=engine)
    with pytest.raises(cs.InvalidInput):
        cs.multipole_intensity(s, q, 16, precision=99, engine=engine)
    with pytest.raises(cs.InvalidInput):
        cs.multipole_intensity(s, np.array([0.1, -0.2]), 16, engine=engine)


# Tensor-core moment GEMM (tcgen05): TF32 or BF16 operands as one term or
# split in two (hi + lo).  Tolerances per q against f64: TF32 hi+lo is within
# the FP32 contract; the others are set by their operand rounding (measured
# at 100,000 atoms, L = 50: TF32 8e-4, BF16 hi+lo 1.3e-5, BF16 5.9e-3; BF16
# hi+lo reaches 5.5e-5 on 700 atoms at L = 0 and q up to 0.9, where the
# monopole sum cancels).
BF16_SPLIT_RTOL = 1e-4
BF16_RTOL = 2e-2
TC_MODES = [(N.PREC_TF32_SPLIT, FP32_RTOL), (N.PREC_TF32, 5e-3), (N.PREC_TF32_SPLIT_FUSED, FP32_RTOL),
            (N.PREC_TF32_FUSED, 5e-3), (N.PREC_BF16_SPLIT, BF16_SPLIT_RTOL), (N.PREC_BF16, BF16_RTOL)]


@pytest.mark.parametrize("prec,tol", TC_MODES)
def test_tensor_core_moments_match_oracle(engine, prec, tol):
    xyz, el = helix96()
    s = cs.Structure(xyz, el)
    q = np.concatenate([[0.0], np.arange(1, 101) * 0.005])
    ref = O.multipole_intensity(_oracle_atoms(s), q, 32)
    got = cs.multipole_intensity(s, q, 32, precision=prec, engine=engine)
    assert _rel(got, ref) <= tol
    big = synth.protein(32, 3000, 20.0)
    q2 = np.linspace(0.001, 0.5, 150)
    ref2 = O.multipole_intensity(_oracle_atoms(big), q2, 30)
    got2 = cs.multipole_intensity(big, q2, 30, precision=prec, engine=engine)
    assert _rel(got2, ref2) <= tol


def test_tensor_core_split_matches_fp64_on_100k_atoms(engine):
    """100,000 atoms, 1000 q, L = 50: the two-term TF32 GEMM against the FP64
    device path (2e-6), and the solvent basis on a grid (1e-6 of each term's
    largest magnitude; the combined curve within the FP32 contract)."""
    w = synth.ATOMS_100K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    got = cs.multipole_intensity(s, w.q, 50, precision=N.PREC_TF32_SPLIT, engine=engine)
    ref = cs.multipole_intensity(s, w.q, 50, precision=N.PREC_FP64, engine=engine)
    assert _rel(got, ref) <= 2e-6
    s2 = synth.protein(36, 2000, 16.0)
    q = np.linspace(0.01, 0.5, 80)
    p = cs.SolventParams(c1=1.01, c2=0.9, hydration_model=cs.HydrationModel.AdaptiveGrid,
                         hydration_grid_spacing_angstrom=3.0)
    b64 = cs.multipole_solvent_basis(s2, q, 28, p, precision=N.PREC_FP64, engine=engine)
    btc = cs.multipole_solvent_basis(s2, q, 28, p, precision=N.PREC_TF32_SPLIT, engine=engine)
    for k in range(6):
        assert np.max(np.abs(btc[k] - b64[k])) / np.max(np.abs(b64[k])) <= 1e-6, k
    i64 = cs.combine_solvent_basis(b64, q, p.c1, p.c2)
    itc = cs.combine_solvent_basis(btc, q, p.c1, p.c2)
    assert _rel(itc, i64) <= FP32_RTOL


@pytest.mark.parametrize("prec", [N.PREC_TF32_SPLIT, N.PREC_TF32])
def test_fused_tf32_equals_staged_tf32(engine, prec):
    """The fused kernel generates Y_lm with k_mp_prep's f64 operations in the
    same order and rounds them the same way, and its 32-point stages hold the
    same points: the curves agree to f64 round-off of the stage sums."""
    s = synth.protein(37, 3000, 20.0)
    q = np.linspace(0.001, 0.5, 150)
    fused = {N.PREC_TF32_SPLIT: N.PREC_TF32_SPLIT_FUSED, N.PREC_TF32: N.PREC_TF32_FUSED}[prec]
    a = cs.multipole_intensity(s, q, 30, precision=prec, engine=engine)
    b = cs.multipole_intensity(s, q, 30, precision=fused, engine=engine)
    assert _rel(b, a) <= 1e-12


@pytest.mark.parametrize("l_max", [0, 1, 7, 8, 20, 64])
def test_fused_modes_at_tile_boundaries(engine, l_max):
    """L = 0..64: tiles that start inside a run of m, on the sin row of an
    (l, m), or in the padding past the last harmonic (a wrong walk gives
    errors of order one; q on the workloads' range)."""
    s = synth.protein(38, 700, 12.0)
    q = np.linspace(0.01, 0.6, 50)
    ref = O.multipole_intensity(_oracle_atoms(s), q, l_max)
    for prec, tol in [(N.PREC_TF32_SPLIT_FUSED, FP32_RTOL), (N.PREC_BF16_SPLIT, BF16_SPLIT_RTOL),
                      (N.PREC_BF16, BF16_RTOL)]:
        got = cs.multipole_intensity(s, q, l_max, precision=prec, engine=engine)
        assert _rel(got, ref) <= tol, (prec, l_max)


def test_bf16_modes_match_fp64_on_100k_atoms(engine):
    """100,000 atoms (R 80 Å), 1000 q on [0.001, 0.6], L = 50: max and RMS
    relative error per q of the BF16 hi+lo and BF16 GEMMs against the FP64
    device multipole, and the solvent basis of a grid-hydrated structure."""
    w = synth.ATOMS_100K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    ref = cs.multipole_intensity(s, w.q, 50, precision=N.PREC_FP64, engine=engine)
    for prec, tol, rms_tol in [(N.PREC_BF16_SPLIT, BF16_SPLIT_RTOL, 1e-5), (N.PREC_BF16, BF16_RTOL, 5e-3)]:
        got = cs.multipole_intensity(s, w.q, 50, precision=prec, engine=engine)
        rel = np.abs(got - ref) / ref
        assert rel.max() <= tol and np.sqrt(np.mean(rel**2)) <= rms_tol, (prec, rel.max())
    s2 = synth.protein(36, 2000, 16.0)
    q = np.linspace(0.01, 0.5, 80)
    p = cs.SolventParams(c1=1.01, c2=0.9, hydration_model=cs.HydrationModel.AdaptiveGrid,
                         hydration_grid_spacing_angstrom=3.0)
    b64 = cs.multipole_solvent_basis(s2, q, 28, p, precision=N.PREC_FP64, engine=engine)
    bbf = cs.multipole_solvent_basis(s2, q, 28, p, precision=N.PREC_BF16_SPLIT, engine=engine)
    for k in range(6):
        assert np.max(np.abs(bbf[k] - b64[k])) / np.max(np.abs(b64[k])) <= BF16_SPLIT_RTOL, k
