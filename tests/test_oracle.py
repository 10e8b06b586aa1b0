"""Pins the oracle (oracle/oracle.cpp) against the reference's own tests.

Each test restates a known-answer, closed-form or cross-method test of the
crabSAXS crate (file:line cited) and runs it against the C++ f64 restatement.
These are the parity anchor: the reference itself (Rust) cannot be built here.
"""
import math

import numpy as np
import pytest

import oracle as O
from conftest import chain8, helix96, ring24, two_atoms_co, two_carbons

C, N_, O_, S, P = 1, 2, 3, 4, 5


def test_sinc_at_zero_is_one():  # scattering.rs:245-248
    assert O.lib.orc_sinc(0.0) == 1.0
    assert O.lib.orc_sinc(5e-9) == 1.0
    assert abs(O.lib.orc_sinc(0.3) - math.sin(0.3) / 0.3) < 1e-16


def test_two_atoms_match_closed_form():  # scattering.rs:249-257
    xyz, el = two_carbons()
    a = O.Atoms(xyz, el)
    q = 0.2
    got = O.debye_intensity(a, [q])[0]
    f = O.lib.orc_form_factor(C, -1, 1.0, 1, q)
    expected = 2.0 * f * f * (1.0 + math.sin(q * 2.0) / (q * 2.0))
    assert abs(got - expected) < 1e-10


def test_bessel_zero_limit():  # spherical.rs:591-594
    assert list(O.spherical_bessel(4, 0.0)) == [1.0, 0.0, 0.0, 0.0, 0.0]


def test_bessel_matches_closed_forms():
    # Miller's recurrence starts at l_max + 24 (spherical.rs:111); it is
    # accurate when that start order is well above x.
    for x in [0.3, 1.7, 5.0, 23.0]:
        j = O.spherical_bessel(40, x)
        assert abs(j[0] - math.sin(x) / x) < 1e-14
        assert abs(j[1] - (math.sin(x) / x**2 - math.cos(x) / x)) < 1e-13
        j2 = (3 / x**2 - 1) * math.sin(x) / x - 3 * math.cos(x) / x**2
        assert abs(j[2] - j2) < 1e-12


def test_multipole_matches_debye_for_two_atoms():  # spherical.rs:595-634
    xyz, el = two_carbons()
    a = O.Atoms(xyz, el)
    q = [0.1, 0.2, 0.5]
    m = O.multipole_intensity(a, q, 32)
    d = O.debye_intensity(a, q)
    assert np.all(np.abs(m - d) / d < 1e-6)


def test_multipole_matches_debye_at_large_qr():  # spherical.rs:636-678
    a = O.Atoms([[-20.0, 0, 0], [20.0, 0, 0]], [C, O_])
    q = [0.2, 0.35, 0.5]
    m = O.multipole_intensity(a, q, 32)
    d = O.debye_intensity(a, q)
    assert np.all(np.abs(m - d) / d < 1e-6)


def test_multipole_curve_matches_debye_below_one_tenth_percent():  # spherical.rs:680-727
    xyz, el = ring24()
    a = O.Atoms(xyz, el)
    q = np.arange(1, 101) * 0.005
    m = O.multipole_intensity(a, q, 24)
    d = O.debye_intensity(a, q)
    nrmse = math.sqrt(np.sum((m - d) ** 2) / np.sum(d**2))
    assert nrmse <= 1e-3


def test_adaptive_public_multipole_matches_debye():  # scattering.rs:311-365
    xyz, el = helix96()
    a = O.Atoms(xyz, el)
    q = np.arange(1, 101) * 0.005
    c = xyz.mean(axis=0)
    rmax = np.max(np.linalg.norm(xyz - c, axis=1))
    l_max = int(min(64, max(8, math.ceil(q.max() * rmax) + 8)))
    m = O.multipole_intensity(a, q, l_max)
    d = O.debye_intensity(a, q)
    rel_l2 = math.sqrt(np.sum((m - d) ** 2) / np.sum(d**2))
    assert rel_l2 <= 1e-3


def test_adaptive_grid_solvent_basis_matches_debye_oracle():  # spherical.rs:729-787
    xyz, el = chain8()
    a = O.Atoms(xyz, el)
    q = np.arange(1, 51) * 0.01
    m = O.multipole_solvent_basis(a, q, 32, model=2, spacing=8.0)
    d = O.debye_solvent_basis(a, q, model=2, spacing=8.0)
    for k in range(6):
        err = math.sqrt(np.sum((m[k] - d[k]) ** 2) / max(np.sum(d[k] ** 2), 1e-30))
        assert err <= 1e-3, (k, err)


def _direct_solvent_intensity(xyz, el, q, c1, c2, thickness=3.0, density=0.334):
    """Independent per-atom Debye of A_i = v_i - G e_i + c2 h_i (solvent.rs:454-500)."""
    out = []
    for qq in q:
        G = O.lib.orc_excluded_volume_scale(qq, c1)
        amps = []
        for e in el:
            v = O.lib.orc_form_factor(int(e), -1, 1.0, 1, qq)
            vol = O.lib.orc_excluded_volume_for_atom(int(e), -1, 1)
            rad = (3.0 * vol / (4.0 * math.pi)) ** (1.0 / 3.0)
            ex = density * vol * math.exp(-(vol ** (2.0 / 3.0)) * qq * qq / (4.0 * math.pi))
            sv = 4.0 * math.pi * (rad + thickness / 2.0) ** 2 * thickness
            h = density * 0.1 * sv * math.exp(-(sv ** (2.0 / 3.0)) * qq * qq / (4.0 * math.pi))
            amps.append(v - G * ex + c2 * h)
        s = 0.0
        for i in range(len(el)):
            for j in range(len(el)):
                r = np.linalg.norm(xyz[i] - xyz[j])
                x = qq * r
                s += amps[i] * amps[j] * (1.0 if abs(x) < 1e-8 else math.sin(x) / x)
        out.append(max(s, 0.0))
    return np.array(out)


def test_solvent_basis_recombines_to_direct_debye_curve():  # solvent.rs:650-665
    xyz, el = two_atoms_co()
    a = O.Atoms(xyz, el)
    q = [0.0, 0.1, 0.3, 0.5]
    b = O.debye_solvent_basis(a, q, c1=1.04, c2=0.35)
    comb = O.combine_solvent_basis(b, q, 1.04, 0.35)
    direct = _direct_solvent_intensity(xyz, el, q, 1.04, 0.35)
    assert np.all(np.abs(comb - direct) <= np.maximum(np.abs(direct), 1.0) * 1e-12)


def test_hydration_grid_is_deterministic_and_exterior():  # solvent.rs:688-705
    xyz = np.array([[-1.0, 0, 0]])
    s1, _ = O.exterior_grid(xyz, [C])
    s2, _ = O.exterior_grid(xyz, [C])
    assert len(s1) > 0 and np.array_equal(s1, s2)
    excl = O.lib.orc_vdw_radius(C) + 1.4
    outer = excl + 3.0
    d = np.linalg.norm(s1 - xyz[0], axis=1)
    assert np.all(d > excl) and np.all(d <= outer + 1e-12)


def test_adaptive_shell_width_matches_published_piecewise_rule():  # solvent.rs:707-714
    w = O.lib.orc_adaptive_shell_width
    assert w(10.0) == 3.0 and w(15.0) == 3.0 and w(20.0) == 5.0 and w(30.0) == 5.0
    assert abs(w(17.5) - 4.0) < np.finfo(float).eps


def test_adaptive_hydration_grid_is_deterministic():  # solvent.rs:716-725
    xyz, _ = two_atoms_co()
    s1, v1 = O.adaptive_grid(xyz)
    s2, _ = O.adaptive_grid(xyz)
    assert len(s1) > 0 and np.array_equal(s1, s2) and v1 == 4.0**3


def test_adaptive_fast_grid_halves_linear_point_density_weight():  # solvent.rs:727-738
    xyz, _ = two_atoms_co()
    _, v = O.adaptive_grid(xyz, spacing=8.0)
    assert v == 2.0 * 4.0**3


def test_hydration_grids_are_translation_invariant():  # solvent.rs:740-771
    xyz, el = two_atoms_co()
    shift = np.array([3.17, -8.4, 2.6])
    a1, _ = O.adaptive_grid(xyz)
    a2, _ = O.adaptive_grid(xyz + shift)
    assert a1.shape == a2.shape and np.all(np.linalg.norm(a2 - a1 - shift, axis=1) < 1e-12)
    e1, _ = O.exterior_grid(xyz, el)
    e2, _ = O.exterior_grid(xyz + shift, el)
    assert e1.shape == e2.shape and np.all(np.linalg.norm(e2 - e1 - shift, axis=1) < 1e-12)


def test_water_form_factor_has_ten_electrons_at_zero():  # solvent.rs:773-777
    assert abs(O.lib.orc_water_form_factor(0.0) - 10.0) < 1e-3


def test_displaced_volume_table_matches_cited_values():  # solvent.rs:779-799
    table = {0: 5.15, 1: 16.44, 2: 2.49, 3: 9.13, 5: 3.37, 4: 26.09, 6: 4.45, 7: 1.56, 8: 24.84, 12: 11.01, 9: 4.19,
             10: 7.99, 11: 9.85, 13: 44.60}
    for e, v in table.items():
        assert O.lib.orc_excluded_volume_for(e) == v


def test_carbon_form_factor_at_q_zero_is_atomic_number():  # formfactor.rs:444-453
    assert abs(O.lib.orc_form_factor(C, -1, 1.0, 0, 0.0) - 6.0) < 0.01
    assert O.lib.orc_form_factor(C, -1, 1.0, 0, 0.5) < O.lib.orc_form_factor(C, -1, 1.0, 0, 0.0)


def test_ion_and_metal_factors_match_atomic_numbers():  # formfactor.rs:455-471
    for e, z in [(6, 11.0), (7, 12.0), (8, 17.0), (12, 19.0), (9, 20.0), (10, 26.0), (11, 30.0), (13, 53.0)]:
        f0 = O.lib.orc_form_factor(e, -1, 1.0, 0, 0.0)
        assert abs(f0 - z) < 0.02
        assert O.lib.orc_form_factor(e, -1, 1.0, 0, 0.5) < f0


def _ff(res, name, el, implicit=1, q=0.0):
    g = O.lib.orc_united_atom_group(res.encode(), name.encode())
    return O.lib.orc_form_factor(el, g, 1.0, implicit, q)


def test_united_atom_electron_counts_match_chemistry():  # formfactor.rs:486-500
    assert abs(_ff("ALA", "CB", C) - 9.0) < 0.01
    assert abs(_ff("GLY", "CA", C) - 8.0) < 0.01
    assert abs(_ff("LYS", "NZ", N_) - 9.0) < 0.01
    assert abs(_ff("ASP", "OD1", O_) - 8.5) < 0.01


def test_nucleotide_united_atoms_include_covalent_hydrogens():  # formfactor.rs:502-517
    for res, name, el, e in [("DA", "C2'", C, 8.0), ("A", "C2'", C, 7.0), ("A", "N6", N_, 9.0), ("DG", "N1", N_, 8.0),
                             ("DT", "C7", C, 9.0)]:
        assert abs(_ff(res, name, el) - e) < 0.02, (res, name)


def test_explicit_hydrogens_are_not_double_counted():  # formfactor.rs:519-524
    assert _ff("ALA", "HB1", 0, implicit=1, q=0.1) == 0.0
    assert _ff("ALA", "HB1", 0, implicit=0, q=0.1) > 0.0


def _two_atom_fit_structure():  # fit.rs:462-487 (C at origin, O at 2 Å)
    return O.Atoms([[0.0, 0, 0], [2.0, 0, 0]], [C, O_])


def test_recovers_scale_and_background_on_synthetic_curve():  # fit.rs:489-518
    a = _two_atom_fit_structure()
    q = np.arange(1, 9) * 0.03
    raw = O.multipole_solvent_intensity(a, q, 8, c1=1.05, c2=0.4, implicit=False)
    y = 1.7 * raw + 0.02
    s, b, chi = O.solve_linear(raw, y, np.full(len(q), 0.01))
    assert abs(s - 1.7) < 1e-8 and abs(b - 0.02) < 1e-8 and chi < 1e-16


def test_fixed_zero_background_uses_weighted_scale_only():  # fit.rs:520-533
    s, b, chi = O.solve_linear([1.0, 2.0, 3.0], [2.0, 4.0, 6.0], [1.0, 2.0, 1.0], bg_mode=1)
    assert abs(s - 2.0) < 1e-12 and b == 0.0 and chi < 1e-24


def test_curve_fit_respects_fixed_scale_and_background():  # reweight.rs:402-410
    r = O.reweight_curves([[0.2, 0.8]], [0.2, 0.8], [0.01, 0.01], kl_strength=1.0, scale_mode=1, scale_value=1.0,
                          bg_mode=1)
    assert r["scale"] == 1.0 and abs(r["reduced_chi2"]) < 1e-12


def test_maximum_entropy_moves_toward_the_experimental_curve():  # reweight.rs:412-433
    r = O.reweight_curves([[1.0, 0.0], [0.0, 1.0]], [0.2, 0.8], [0.01, 0.01], kl_strength=0.01, scale_mode=1,
                          scale_value=1.0, bg_mode=1)
    w = r["weights"]
    assert abs(w.sum() - 1.0) < 1e-12 and w[1] > w[0]


def test_project_simplex_properties():  # ensemble.rs:449-465
    rng = np.random.default_rng(0)
    for _ in range(20):
        v = rng.normal(size=7)
        p = O.project_simplex(v)
        assert abs(p.sum() - 1.0) < 1e-12 and np.all(p >= 0)
    u = np.array([0.2, 0.3, 0.5])
    assert np.allclose(O.project_simplex(u), u)


def test_optimize_weights_recovers_a_mixture():  # ensemble.rs:317-381
    rng = np.random.default_rng(1)
    curves = rng.uniform(1.0, 2.0, size=(4, 30))
    y = 0.7 * curves[1] + 0.3 * curves[3]
    w, s, b, chi, fitted = O.optimize_weights(curves, y, np.full(30, 0.01), bg_mode=1)
    assert w.sum() == pytest.approx(1.0) and w[1] > w[0] and w[3] > w[2]
    chi_uniform = O.optimize_weights(curves, y, np.full(30, 0.01), bg_mode=1, uniform=True)[3]
    assert chi < 0.1 * chi_uniform


def test_solvent_candidates_grid():  # ensemble.rs:302-315
    c = O.solvent_candidates(0.95, 1.05, -2.0, 4.0)
    assert c.shape == (25, 2) and c[0, 0] == 0.95 and c[-1, 0] == 1.05 and c[0, 1] == -2.0 and c[-1, 1] == 4.0


def test_cubic_hermite_reproduces_cubic_interpolant_at_knots():  # fit.rs:93-123
    x = np.linspace(0.01, 0.5, 11)
    y = np.sin(10 * x)
    assert np.allclose(O.cubic_hermite(x, y, x), y, atol=1e-15)


def test_chi2_gradient_matches_central_differences():
    """New capability (no reference counterpart): analytic ∂χ²/∂x of the oracle vs FP64 central differences."""
    rng = np.random.default_rng(3)
    xyz = rng.normal(scale=4.0, size=(12, 3))
    el = rng.choice([C, N_, O_, S], size=12)
    a = O.Atoms(xyz, el)
    q = np.arange(1, 41) * 0.0125
    clean = O.debye_solvent_basis(a, q, c1=1.01, c2=0.3)
    y = 1.3 * O.combine_solvent_basis(clean, q, 1.01, 0.3) * (1 + 0.01 * rng.normal(size=len(q)))
    sigma = 0.01 * np.abs(y) + 1e-3
    chi, gx, gp = O.chi2_grad(a, q, y, sigma, 1.0, 0.5, 1.2, 0.01)
    h = 1e-5
    for i in [0, 5, 11]:
        for d in range(3):
            xp = xyz.copy()
            xp[i, d] += h
            xm = xyz.copy()
            xm[i, d] -= h
            cp = O.chi2_grad(O.Atoms(xp, el), q, y, sigma, 1.0, 0.5, 1.2, 0.01, want_xyz=False)[0]
            cm = O.chi2_grad(O.Atoms(xm, el), q, y, sigma, 1.0, 0.5, 1.2, 0.01, want_xyz=False)[0]
            fd = (cp - cm) / (2 * h)
            assert abs(gx[i, d] - fd) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(gx).max()), (i, d, gx[i, d], fd)
    for k, (c1, c2, s, b) in enumerate([(1.0 + h, 0.5, 1.2, 0.01), (1.0, 0.5 + h, 1.2, 0.01),
                                        (1.0, 0.5, 1.2 + h, 0.01), (1.0, 0.5, 1.2, 0.01 + h)]):
        cp = O.chi2_grad(a, q, y, sigma, c1, c2, s, b, want_xyz=False)[0]
        c1m, c2m, sm, bm = (2 * np.array([1.0, 0.5, 1.2, 0.01]) - np.array([c1, c2, s, b]))
        cm = O.chi2_grad(a, q, y, sigma, c1m, c2m, sm, bm, want_xyz=False)[0]
        fd = (cp - cm) / (2 * h)
        assert abs(gp[k] - fd) <= 1e-5 * max(abs(fd), 1e-6), (k, gp[k], fd)


def _two_carbons_4a():  # metrics.rs:651-677: C at the origin and at 4 Å
    return O.Atoms(np.array([[0.0, 0.0, 0.0], [4.0, 0.0, 0.0]]), np.array([C, C]))


def test_coordinate_features_report_pair_distance():  # metrics.rs:678-684
    f = O.coordinate_features(_two_carbons_4a())
    assert abs(f["dmax"] - 4.0) < 1e-12
    assert f["rg"] > 1.0
    assert len(f["p"]) > 0


def test_two_atom_distribution_closed_form():
    """One pair at exactly dmax lands in the last bin (the bins-1 cap); the
    trapezoid area is step/2 * p_last, so p_last = 2/step, the distribution's
    Rg is r_last/sqrt(2) and its Dmax is r_last (metrics.rs:550-583)."""
    f = O.coordinate_features(_two_carbons_4a(), bins=160)
    step = 4.0 / 160
    r_last = 159.5 * step
    assert f["rg"] == 2.0 and f["dmax"] == 4.0
    assert np.count_nonzero(f["p"]) == 1 and f["p"][-1] == pytest.approx(2.0 / step, rel=1e-15)
    assert f["pr_rg"] == pytest.approx(r_last / math.sqrt(2.0), rel=1e-15)
    assert f["pr_dmax"] == r_last


def test_coordinate_pr_single_point_results():  # metrics.rs:489-498
    same = O.Atoms(np.tile([1.0, 2.0, 3.0], (5, 1)), np.full(5, C))
    f = O.coordinate_features(same)
    assert f["dmax"] == 0.0 and list(f["r"]) == [0.0] and list(f["p"]) == [1.0]
    assert f["pr_rg"] == 0.0 and f["pr_dmax"] == 0.0
    with pytest.raises(ValueError):
        O.coordinate_features(O.Atoms(np.zeros((0, 3)), np.zeros(0, dtype=int)))


def test_coordinate_pr_bins_on_exact_edges():
    """17 atoms on a line at integer positions with 16 bins: step = 1, so every
    distance k falls exactly on the lower edge of bin k; distance 16 is capped
    into bin 15 (metrics.rs:515-516)."""
    xyz = np.zeros((17, 3))
    xyz[:, 0] = np.arange(17)
    dmax, hist = O.pair_distance_histogram(xyz, np.ones(17), 16)
    expected = np.array([0.0] + [17.0 - k for k in range(1, 16)])
    expected[15] += 1.0
    assert dmax == 16.0 and np.array_equal(hist, expected)


def test_coordinate_pr_bins_floor_at_sixteen():  # metrics.rs:268: options.bins.max(16)
    f = O.coordinate_features(_two_carbons_4a(), bins=3)
    assert len(f["p"]) == 16


def test_oracle_synthetic_generator_equals_the_library_one():
    """The reference arm of bench.py builds its input with the oracle's copy of
    the generator: it must be the same structure bit for bit."""
    from crabsaxs_b200 import synth

    for seed, n, radius in [(2, 20000, 45.0), (7, 1000, 20.0), (11, 3, 5.0)]:
        xyz, el = O.synth_protein(seed, n, radius)
        s = synth.protein(seed, n, radius)
        assert np.array_equal(xyz, s.xyz) and np.array_equal(el, s.element)
