"""Parity of the CUDA Debye engine (through the C ABI) with the oracle.

Tolerances: intensities and six-term recombinations within 1e-5 relative per
q point (the FP32 path's contract against FP64); per-type-pair partials within
2e-6 of their q = 0 magnitude Σ|w_i w_j| (they cross zero, so a relative
bound is undefined there); the FP64 device kernel within 1e-11.
"""
import math

import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O
from conftest import helix96, two_atoms_co, two_carbons

pytestmark = pytest.mark.gpu

INTENSITY_RTOL = 1e-5
PARTIAL_ATOL = 2e-6


def _random_typed(n, T, seed, radius=15.0, occ=True):
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(-radius, radius, size=(n, 3)) + np.array([40.0, -12.0, 7.0])
    w = rng.uniform(0.3, 1.0, size=n) if occ else np.ones(n)
    t = rng.integers(0, T, size=n)
    return xyz, w, t


def _partials_scale(w, t, T):
    s = np.array([w[t == a].sum() for a in range(T)])
    scale = np.outer(s, s)
    idx = [(a, b) for a in range(T) for b in range(a, T)]
    return np.array([max(scale[a, b], 1e-12) for a, b in idx])


@pytest.mark.parametrize("n,T,seed", [(1, 1, 0), (2, 1, 1), (3, 2, 2), (130, 3, 3), (300, 5, 4), (517, 4, 5)])
@pytest.mark.parametrize("qkind", ["uniform", "with_zero", "nonuniform", "single"])
def test_partials_match_oracle(engine, n, T, seed, qkind):
    xyz, w, t = _random_typed(n, T, seed)
    if qkind == "uniform":
        q = np.arange(1, 101) * 0.005
    elif qkind == "with_zero":
        q = np.linspace(0.0, 0.6, 77)
    elif qkind == "nonuniform":
        q = np.sort(np.random.default_rng(seed).uniform(0.0, 0.5, size=45))
    else:
        q = np.array([0.37])
    got, self_g = cs.debye_partials(xyz, w, t, T, q, engine=engine)
    ref, self_r = O.debye_partials(xyz, w, t, T, q)
    np.testing.assert_allclose(self_g, self_r, rtol=1e-14)
    scale = _partials_scale(w, t, T)[:, None]
    err = np.abs(got - ref) / scale
    assert err.max() <= PARTIAL_ATOL, err.max()


def test_fp64_partials_match_oracle(engine):
    xyz, w, t = _random_typed(400, 3, 9)
    q = np.concatenate([[0.0], np.linspace(0.01, 0.5, 40)])
    got, _ = cs.debye_partials(xyz, w, t, 3, q, fp64=True, engine=engine)
    ref, _ = O.debye_partials(xyz, w, t, 3, q)
    scale = _partials_scale(w, t, 3)[:, None]
    assert (np.abs(got - ref) / scale).max() <= 1e-11


def test_two_atoms_match_closed_form(engine):  # scattering.rs:249-257
    xyz, el = two_carbons()
    s = cs.Structure(xyz, el)
    q = 0.2
    got = cs.debye_intensity(s, [q], engine=engine)[0]
    f = O.lib.orc_form_factor(1, -1, 1.0, 1, q)
    expected = 2.0 * f * f * (1.0 + math.sin(q * 2.0) / (q * 2.0))
    assert abs(got - expected) / expected < 1e-6


def _oracle_atoms(s: cs.Structure):
    return O.Atoms(s.xyz, s.element, s.group, s.occupancy)


@pytest.mark.parametrize("implicit", [True, False])
def test_vacuum_intensity_matches_oracle_helix(engine, implicit):  # scattering.rs:86-110
    xyz, el = helix96()
    s = cs.Structure(xyz, el)
    q = np.arange(1, 101) * 0.005
    got = cs.debye_intensity(s, q, implicit, engine=engine)
    ref = O.debye_intensity(_oracle_atoms(s), q, implicit)
    assert np.max(np.abs(got - ref) / ref) <= INTENSITY_RTOL


def test_vacuum_intensity_1k(engine):
    from crabsaxs_b200 import synth

    w = synth.DEBYE_1K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    got = cs.debye_intensity(s, w.q, engine=engine)
    ref = O.debye_intensity(_oracle_atoms(s), w.q)
    assert np.max(np.abs(got - ref) / ref) <= INTENSITY_RTOL


def test_hydrogens_groups_and_occupancy(engine):
    """Mixed elements incl. H and united-atom residues, fractional occupancy, both hydrogen modes."""
    rng = np.random.default_rng(11)
    atoms = []
    names = [("ALA", "CB", cs.Element.C), ("GLY", "CA", cs.Element.C), ("LYS", "NZ", cs.Element.N),
             ("ASP", "OD1", cs.Element.O), ("CYS", "SG", cs.Element.S), ("ALA", "HB1", cs.Element.H),
             ("HOH", "O", cs.Element.O), ("ZN", "ZN", cs.Element.Zn), ("DA", "C2'", cs.Element.C)]
    for i in range(260):
        r, a, e = names[i % len(names)]
        atoms.append(cs.Atom(tuple(rng.uniform(-12, 12, 3)), e, float(rng.uniform(0.5, 1.0)), False, a, r))
    s = cs.Structure.from_atoms(atoms)
    q = np.linspace(0.0, 0.5, 51)
    for implicit in (True, False):
        got = cs.debye_intensity(s, q, implicit, engine=engine)
        ref = O.debye_intensity(_oracle_atoms(s), q, implicit)
        assert np.max(np.abs(got - ref) / ref) <= INTENSITY_RTOL
        sp = cs.SolventParams(c1=1.03, c2=0.6)
        gb = cs.debye_solvent_basis(s, q, sp, implicit, engine=engine)
        rb = O.debye_solvent_basis(_oracle_atoms(s), q, 1.03, 0.6, implicit=implicit)
        gi = cs.combine_solvent_basis(gb, q, 1.03, 0.6)
        ri = O.combine_solvent_basis(rb, q, 1.03, 0.6)
        assert np.max(np.abs(gi - ri) / ri) <= INTENSITY_RTOL


def test_solvent_basis_two_atoms_nonuniform_q(engine):  # solvent.rs:650-665
    xyz, el = two_atoms_co()
    s = cs.Structure(xyz, el)
    q = [0.0, 0.1, 0.3, 0.5]
    sp = cs.SolventParams(c1=1.04, c2=0.35)
    gb = cs.debye_solvent_basis(s, q, sp, engine=engine)
    rb = O.debye_solvent_basis(_oracle_atoms(s), q, 1.04, 0.35)
    assert np.max(np.abs(gb - rb) / np.maximum(np.abs(rb), 1.0)) < 1e-6
    gi = cs.solvent_corrected_intensity(s, q, sp, engine=engine)
    ri = O.combine_solvent_basis(rb, q, 1.04, 0.35)
    assert np.max(np.abs(gi - ri) / ri) <= INTENSITY_RTOL


@pytest.mark.parametrize("c1,c2", [(1.0, 0.0), (0.97, 1.3), (1.05, 2.0)])
def test_solvent_1k_matches_oracle(engine, c1, c2):
    from crabsaxs_b200 import synth

    w = synth.DEBYE_1K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    sp = cs.SolventParams(c1=c1, c2=c2)
    got = cs.solvent_corrected_intensity(s, w.q, sp, engine=engine)
    ref = O.combine_solvent_basis(O.debye_solvent_basis(_oracle_atoms(s), w.q, c1, c2), w.q, c1, c2)
    assert np.max(np.abs(got - ref) / ref) <= INTENSITY_RTOL


@pytest.mark.parametrize("spacing", [8.0, 4.0, 3.0])
def test_adaptive_grid_solvent_basis_matches_oracle(engine, spacing):
    from crabsaxs_b200 import synth

    s = synth.protein(21, 600, 14.0)
    q = np.linspace(0.005, 0.5, 60)
    sp = cs.SolventParams(c1=1.02, c2=0.8, hydration_model=cs.HydrationModel.AdaptiveGrid,
                          hydration_grid_spacing_angstrom=spacing)
    gb = cs.debye_solvent_basis(s, q, sp, engine=engine)
    rb = O.debye_solvent_basis(_oracle_atoms(s), q, 1.02, 0.8, model=2, spacing=spacing)
    gi = cs.combine_solvent_basis(gb, q, 1.02, 0.8)
    ri = O.combine_solvent_basis(rb, q, 1.02, 0.8)
    assert np.max(np.abs(gi - ri) / ri) <= INTENSITY_RTOL
    for k in (0, 1, 2):  # the self terms are positive definite
        assert np.max(np.abs(gb[k] - rb[k]) / rb[k]) <= INTENSITY_RTOL


def test_20k_solvated_fp32_matches_fp64_and_oracle(engine):
    """The full solvated workload (20k atoms + 3 Å adaptive sites, 500 q): FP32 vs the FP64 device kernel
    at every q, and vs the CPU oracle at four q values."""
    from crabsaxs_b200 import synth

    w = synth.DEBYE_20K_SOLVATED
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    c1, c2 = synth.solvent_draw(w.seed)
    sp = cs.SolventParams(c1=c1, c2=c2, hydration_model=cs.HydrationModel.AdaptiveGrid,
                          hydration_grid_spacing_angstrom=3.0)
    sites, vol = cs.hydration_grid_adaptive(s, 3.0, engine=engine)
    gb = cs.debye_solvent_basis(s, w.q, sp, engine=engine)
    gi = cs.combine_solvent_basis(gb, w.q, c1, c2)
    # FP64 device reference of the same decomposition
    xyz = np.concatenate([s.xyz, sites])
    el = np.concatenate([s.element.astype(np.int32), np.full(len(sites), -1)])
    classes = sorted(set(el.tolist()) - {-1}) + [-1]
    t = np.array([classes.index(e) for e in el])
    wts = np.ones(len(xyz))
    P64, D64 = cs.debye_partials(xyz, wts, t, len(classes), w.q, fp64=True, engine=engine)
    P32, D32 = cs.debye_partials(xyz, wts, t, len(classes), w.q, engine=engine)
    T = len(classes)
    scale = _partials_scale(wts, t, T)[:, None]
    assert (np.abs(P32 - P64) / scale).max() <= PARTIAL_ATOL
    sub = np.array([0, 123, 321, 499])
    rb = O.debye_solvent_basis(_oracle_atoms(s), w.q[sub], c1, c2, model=2, spacing=3.0)
    ri = O.combine_solvent_basis(rb, w.q[sub], c1, c2)
    assert np.max(np.abs(gi[sub] - ri) / ri) <= INTENSITY_RTOL


def test_size_independent_properties(engine):
    """Linearity in the weights, translation and permutation invariance at 20k atoms."""
    from crabsaxs_b200 import synth

    s = synth.protein(33, 20000, 45.0)
    t = s.element.astype(np.int32) - 1
    q = np.linspace(0.001, 0.5, 500)
    w = np.ones(s.atom_count)
    P, D = cs.debye_partials(s.xyz, w, t, 4, q, engine=engine)
    scale = _partials_scale(w, t, 4)[:, None]
    P2, _ = cs.debye_partials(s.xyz, 2.0 * w, t, 4, q, engine=engine)
    assert (np.abs(P2 - 4.0 * P) / scale).max() <= 1e-6
    Pt, _ = cs.debye_partials(s.xyz + np.array([123.4, -56.7, 8.9]), w, t, 4, q, engine=engine)
    assert (np.abs(Pt - P) / scale).max() <= PARTIAL_ATOL
    perm = np.random.default_rng(0).permutation(s.atom_count)
    Pp, _ = cs.debye_partials(s.xyz[perm], w, t[perm], 4, q, engine=engine)
    assert (np.abs(Pp - P) / scale).max() <= PARTIAL_ATOL


def test_rejects_bad_q(engine):  # scattering.rs:258-262
    xyz, el = two_carbons()
    s = cs.Structure(xyz, el)
    with pytest.raises(cs.InvalidInput):
        cs.compute_curve(s, [float("nan")], cs.ComputeOptions(), engine=engine)
    with pytest.raises(cs.InvalidInput):
        cs.compute_curve(s, [0.2, 0.1], cs.ComputeOptions(), engine=engine)
    with pytest.raises(cs.InvalidInput):
        cs.compute_curve(s, [0.1], cs.ComputeOptions(multipole_l_max=4), engine=engine)
    with pytest.raises(cs.InvalidInput):
        cs.compute_curve(s, [0.1], cs.ComputeOptions(solvent=cs.SolventParams(c1=0.0)), engine=engine)


def test_debye_supports_adaptive_grid_solution_curve(engine):  # scattering.rs:287-309
    xyz, el = two_carbons()
    s = cs.Structure(xyz, el)
    opt = cs.ComputeOptions(method=cs.ScatteringMethod.Debye,
                            solvent=cs.SolventParams(c2=0.02, hydration_model=cs.HydrationModel.AdaptiveGrid,
                                                     hydration_grid_spacing_angstrom=8.0))
    curve = cs.compute_curve(s, [0.05, 0.1], opt, engine=engine)
    assert curve.method == "Debye"
    assert np.all(np.isfinite(curve.intensity)) and np.all(curve.intensity >= 0)
    ref = O.combine_solvent_basis(O.debye_solvent_basis(_oracle_atoms(s), [0.05, 0.1], 1.0, 0.02, model=2,
                                                        spacing=8.0), [0.05, 0.1], 1.0, 0.02)
    assert np.max(np.abs(curve.intensity - ref) / ref) <= INTENSITY_RTOL


def test_profile_calculator_debye(engine):  # analysis.rs:90-105
    xyz, el = helix96()
    s = cs.Structure(xyz, el)
    q = np.arange(1, 101) * 0.005
    calc = cs.ProfileCalculator(q, cs.ComputeOptions(), engine=engine)
    curve = calc.calculate(s)
    assert curve.method == "Debye"  # Auto with fewer than 500 atoms
    ref = O.debye_intensity(_oracle_atoms(s), q)
    assert np.max(np.abs(curve.intensity - ref) / ref) <= INTENSITY_RTOL
    with pytest.raises(cs.InvalidInput):
        cs.ProfileCalculator([0.2, 0.1])


def test_empty_structure_gives_zero_curve(engine):
    s = cs.Structure(np.zeros((0, 3)), np.zeros(0, dtype=np.int8))
    out = cs.debye_intensity(s, [0.0, 0.1], engine=engine)
    assert np.all(out == 0.0)


def test_partials_are_bit_reproducible(engine):
    """Each flushed FP32 sum is rounded onto a power-of-two fixed-point grid
    sized by a bound on the structure's sums, so the f64 atomic adds are exact
    in whatever order they land: repeated calls return identical bits, for one
    structure and for a batch of structures (the ensemble's segmented plan)."""
    from crabsaxs_b200 import synth

    xyz, w, t = _random_typed(6000, 3, 29, radius=30.0)
    t = t.astype(np.int32)
    q = np.linspace(0.001, 0.5, 500)
    first, _ = cs.debye_partials(xyz, w, t, 3, q, engine=engine)
    for _ in range(3):
        again, _ = cs.debye_partials(xyz, w, t, 3, q, engine=engine)
        assert np.array_equal(again, first)
    P64, _ = cs.debye_partials(xyz, w, t, 3, q, fp64=True, engine=engine)
    assert np.max(np.abs(first - P64) / _partials_scale(w, t, 3)[:, None]) <= PARTIAL_ATOL
    confs = [synth.protein(900 + i, n, 12.0 + 0.004 * n) for i, n in enumerate([700, 2500, 1200, 4000])]
    qe = np.linspace(0.005, 0.45, 300)
    cand = cs.solvent_candidates(cs.FitOptions())[[0, 12]]
    c0 = cs.ensemble_curves(confs, qe, cs.SolventParams(), cand, engine=engine)
    for _ in range(2):
        assert np.array_equal(cs.ensemble_curves(confs, qe, cs.SolventParams(), cand, engine=engine), c0)


def test_pair_kernel_launches_are_counted(engine):
    engine.reset_stats()
    xyz, w, t = _random_typed(300, 2, 1)
    cs.debye_partials(xyz, w, t, 2, np.linspace(0.01, 0.3, 40), engine=engine)
    launches, ms, pq = engine.stats()
    assert launches >= 1 and ms > 0 and pq == pytest.approx(300 * 299 / 2 * 40)


def test_lattice_plan_matches_fp64_20k(engine):
    """The site–site block from the lattice histogram equals the FP64 pair sum
    over the same sites; every other block stays within the FP32 bound."""
    import ctypes as C

    from crabsaxs_b200 import _native as N
    from crabsaxs_b200 import synth

    w = synth.DEBYE_20K_SOLVATED
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    sites, _ = cs.hydration_grid_adaptive(s, 3.0, engine=engine)
    el = s.element.astype(np.int64)
    classes = sorted(set(el.tolist()))
    t = np.concatenate([np.searchsorted(classes, el), np.full(len(sites), len(classes))]).astype(np.int32)
    xyz = np.ascontiguousarray(np.concatenate([s.xyz, sites]))
    wts = np.ones(len(xyz))
    T = len(classes) + 1
    q = np.ascontiguousarray(w.q)
    cells = np.ascontiguousarray(np.rint((sites - sites.min(axis=0)) / 3.0).astype(np.int32))
    plan = C.c_void_p()
    engine.check(N.lib.crab_pair_plan_create_lattice(engine.handle, xyz.ctypes.data_as(N.D), wts.ctypes.data_as(N.D),
                                                     t.ctypes.data_as(N.I32P), len(wts), T, q.ctypes.data_as(N.D),
                                                     len(q), cells.ctypes.data_as(N.I32P), len(sites), 3.0,
                                                     C.byref(plan)))
    try:
        engine.check(N.lib.crab_pair_plan_run(engine.handle, plan, 2, 0, None))
        P = np.empty((T * (T + 1) // 2, len(q)))
        engine.check(N.lib.crab_pair_plan_read(engine.handle, plan, P.ctypes.data_as(N.D), None))
    finally:
        N.lib.crab_pair_plan_destroy(plan)
    P64, _ = cs.debye_partials(xyz, wts, t, T, q, fp64=True, engine=engine)
    scale = _partials_scale(wts, t, T)[:, None]
    err = np.abs(P - P64) / scale
    assert err[-1].max() <= 1e-12  # site–site row: exact lattice sums
    assert err.max() <= PARTIAL_ATOL


# Every kernel variant the plan can dispatch (Q*16 + jb; jb >= 8: q-packed, jb >= 12: 3 CTAs/SM;
# jb 5, 6, 7, 3: q-packed with the weight folded into the recurrence, 1 or 2 chains, 2 to 4 CTAs/SM;
# jb 11: folded with two chains per pair, q points 4n, 4n+1 and 4n+2, 4n+3, the one-chain build on wide plans).
ALL_VARIANTS = [8 * 16 + 2, 16 * 16 + 2, 32 * 16 + 2, 48 * 16 + 2, 64 * 16 + 2, 96 * 16 + 2, 128 * 16 + 2,
                64 * 16 + 4, 96 * 16 + 4, 64 * 16 + 10, 96 * 16 + 10, 128 * 16 + 9, 128 * 16 + 10, 128 * 16 + 13,
                100 * 16 + 13, 126 * 16 + 13, 150 * 16 + 9, 168 * 16 + 9,
                168 * 16 + 5, 150 * 16 + 5, 168 * 16 + 6, 150 * 16 + 6, 128 * 16 + 6, 126 * 16 + 7, 100 * 16 + 7,
                84 * 16 + 3, 126 * 16 + 14, 126 * 16 + 15, 100 * 16 + 14, 100 * 16 + 15,
                84 * 16 + 12, 100 * 16 + 12, 168 * 16 + 11]


@pytest.mark.parametrize("qkind", ["uniform", "nonuniform", "coarse", "wide"])
def test_every_kernel_variant_matches_fp64(engine, qkind):
    import ctypes as C

    from crabsaxs_b200 import _native as N

    T = 3
    xyz, w, t = _random_typed(700, T, 11, radius=20.0)
    t = t.astype(np.int32)
    if qkind == "uniform":
        q = np.linspace(0.001, 0.5, 333)
    elif qkind == "nonuniform":
        q = np.concatenate([np.linspace(0.0, 0.1, 57), np.linspace(0.102, 0.6, 141), [0.65, 0.7, 0.8]])
    elif qkind == "coarse":  # half step angle about 0.19 rad over the 63 Å extent: near the largest
        q = np.linspace(0.01, 1.202, 201)  # that the two-chain build takes (its chains step 1.5 rad)
    else:  # steps of about 0.05 Å⁻¹ over a 70 Å extent: the seed path for the step angle
        q = np.linspace(0.01, 3.0, 61)
    q = np.ascontiguousarray(q)
    xyz = np.ascontiguousarray(xyz)
    P64, _ = cs.debye_partials(xyz, w, t, T, q, fp64=True, engine=engine)
    scale = _partials_scale(w, t, T)[:, None]
    plan = C.c_void_p()
    engine.check(N.lib.crab_pair_plan_create(engine.handle, xyz.ctypes.data_as(N.D), w.ctypes.data_as(N.D),
                                             t.ctypes.data_as(N.I32P), len(w), T, q.ctypes.data_as(N.D), len(q),
                                             C.byref(plan)))
    try:
        for v in ALL_VARIANTS:
            engine.check(N.lib.crab_pair_plan_select(engine.handle, plan, v))
            engine.check(N.lib.crab_pair_plan_run(engine.handle, plan, 1, 0, None))
            P = np.empty((T * (T + 1) // 2, len(q)))
            engine.check(N.lib.crab_pair_plan_read(engine.handle, plan, P.ctypes.data_as(N.D), None))
            err = np.abs(P - P64) / scale
            assert err.max() <= PARTIAL_ATOL, (v, err.max())
        assert N.lib.crab_pair_plan_select(engine.handle, plan, 100 * 16 + 2) == N.EINVAL
    finally:
        N.lib.crab_pair_plan_destroy(plan)


def test_every_kernel_variant_keeps_solvent_curve_parity(engine):
    """Curve-level check of every variant through the public solvent-basis call:
    with the adaptive grid the solvent curve cancels to a few percent of its
    vacuum term at high q, which magnifies any per-pair error of the kernel."""
    from crabsaxs_b200 import _native as N
    from crabsaxs_b200 import synth

    s = synth.protein(61, 4000, 22.0)
    q = np.linspace(0.001, 0.5, 240)
    c1, c2 = 0.976, 0.6
    sp = cs.SolventParams(c1=c1, c2=c2, hydration_model=cs.HydrationModel.AdaptiveGrid,
                          hydration_grid_spacing_angstrom=3.0)
    i64 = cs.combine_solvent_basis(cs.debye_solvent_basis(s, q, sp, engine=engine, fp64=True), q, c1, c2)
    try:
        for v in ALL_VARIANTS:
            engine.check(N.lib.crab_ctx_set_pair_variant(engine.handle, v))
            i32 = cs.combine_solvent_basis(cs.debye_solvent_basis(s, q, sp, engine=engine), q, c1, c2)
            err = float(np.max(np.abs(i32 - i64) / np.abs(i64)))
            assert err <= INTENSITY_RTOL, (v, err)
        assert N.lib.crab_ctx_set_pair_variant(engine.handle, 100 * 16 + 2) == N.EINVAL
    finally:
        engine.check(N.lib.crab_ctx_set_pair_variant(engine.handle, 0))
