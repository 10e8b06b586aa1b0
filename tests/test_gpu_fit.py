"""Fitting on the GPU (crab_fit: fit.rs:288-454) with the reference's own
recovery tests (fit.rs:489-660), the L-BFGS option against Nelder-Mead, and
SaxsScorer (analysis.rs:137-178).

Tolerances are the reference's (they are recovery gates, not precision
gates): c1 within 0.02, c2 within 0.08, scale within 0.4e-4, background within
0.01, reduced chi^2 below 0.01; the stride-20 and full-q fits within 1e-3
relative RMSE of each other.
"""
import math

import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O
from crabsaxs_b200 import synth

pytestmark = pytest.mark.gpu

C_, O_ = 1, 3


def _two_atoms():  # fit.rs:462-487: C at the origin, O at 2 Å, residue "TST"
    return cs.Structure(np.array([[0.0, 0.0, 0.0], [2.0, 0.0, 0.0]]), np.array([C_, O_]))


def _lcg_gaussian(n, seed=0x5EED):
    """The deterministic Box-Muller noise of fit.rs:555-566 (64-bit LCG)."""
    state = seed
    mask = (1 << 64) - 1

    def uniform():
        nonlocal state
        state = (state * 6364136223846793005 + 1) & mask
        return max((state >> 11) / float(1 << 53), np.finfo(float).tiny)

    out = np.empty(n)
    for i in range(n):
        u1, u2 = uniform(), uniform()
        out[i] = math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)
    return out


def _noisy_two_atom_fit(engine, optimizer):
    s = _two_atoms()
    q = np.arange(1, 81) * 0.006
    raw = O.multipole_solvent_intensity(O.Atoms(s.xyz, s.element), q, 8, c1=1.02, c2=0.55, implicit=False)
    y = 1.4e-4 * raw + 0.03 + 0.0001 * _lcg_gaussian(len(q))
    ex = cs.ExperimentalCurve(q, y, np.full(len(q), 0.002))
    opt = cs.FitOptions(method=cs.ScatteringMethod.Multipole, hydrogen_mode=cs.HydrogenMode.Explicit,
                        max_iterations=100, q_sampling_stride=1, optimizer=optimizer)
    return cs.fit_to_experimental_with_options(s, ex, cs.FitParams(1.4e-4, 0.03, 1.02, 0.55), opt, engine=engine)


def test_recovers_solvent_parameters_with_deterministic_noise(engine):  # fit.rs:536-600
    r = _noisy_two_atom_fit(engine, "nelder-mead")
    assert abs(r.params.c1 - 1.02) < 0.02, r
    assert abs(r.params.c2 - 0.55) < 0.08, r
    assert abs(r.params.scale - 1.4e-4) < 0.4e-4, r
    assert abs(r.params.background - 0.03) < 0.01, r
    assert r.chi2 < 0.01, r


def test_lbfgs_reaches_at_least_the_nelder_mead_optimum(engine):
    """The same noisy two-atom data: its chi^2 surface over (c1, c2) is nearly
    flat (0.00283 at the truth, 0.00281 at the grid minimum c1 = 1.03,
    c2 = 0.15), so the parameters are not identifiable; the reference's
    recovery gates hold for Nelder-Mead started at the truth, and the
    gradient-based L-BFGS must reach a chi^2 no worse than it."""
    nm = _noisy_two_atom_fit(engine, "nelder-mead")
    lb = _noisy_two_atom_fit(engine, "lbfgs")
    assert lb.chi2 <= nm.chi2 * (1.0 + 1e-6) and lb.chi2 < 0.01
    assert lb.converged


def test_sampled_basis_matches_full_basis_fit(engine):  # fit.rs:602-660
    s = _two_atoms()
    q = np.arange(1, 102) * 0.005
    raw = O.multipole_solvent_intensity(O.Atoms(s.xyz, s.element), q, 8, c1=1.03, c2=0.3, implicit=False)
    ex = cs.ExperimentalCurve(q, 0.8 * raw + 0.01, np.full(len(q), 0.01))
    common = dict(method=cs.ScatteringMethod.Multipole, hydrogen_mode=cs.HydrogenMode.Explicit, max_iterations=64)
    full = cs.fit_to_experimental_with_options(s, ex, cs.FitParams(), cs.FitOptions(q_sampling_stride=1, **common),
                                               engine=engine)
    sampled = cs.fit_to_experimental_with_options(s, ex, cs.FitParams(), cs.FitOptions(**common), engine=engine)
    rel = math.sqrt(np.sum((full.fitted_curve - sampled.fitted_curve) ** 2) / np.sum(full.fitted_curve**2))
    assert rel < 1e-3, rel


def _debye_experiment(s, q, c1, c2, scale, bg, seed):
    sp = cs.SolventParams(c1=c1, c2=c2)
    clean = scale * cs.compute_curve(s, q, cs.ComputeOptions(method=cs.ScatteringMethod.Debye, solvent=sp)).intensity + bg
    sigma = 0.01 * clean
    return clean + sigma * np.random.default_rng(seed).normal(size=len(q)), sigma


def test_lbfgs_and_nelder_mead_agree_on_5k_atoms(engine):
    """5,000 atoms (R 28 Å), 100 q, Debye method: the analytic-gradient L-BFGS fit
    and the derivative-free Nelder-Mead fit land on the same optimum."""
    w = synth.GRADIENT_5K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    y, sigma = _debye_experiment(s, w.q, 1.015, 0.9, 3.7, 50.0, 11)
    ex = cs.ExperimentalCurve(w.q, y, sigma)
    res = {}
    for optimizer in ("nelder-mead", "lbfgs"):
        opt = cs.FitOptions(method=cs.ScatteringMethod.Debye, q_sampling_stride=1, max_iterations=200,
                            optimizer=optimizer)
        res[optimizer] = cs.fit_to_experimental_with_options(s, ex, cs.FitParams(), opt, engine=engine)
    nm, lb = res["nelder-mead"], res["lbfgs"]
    assert lb.chi2 <= nm.chi2 * (1.0 + 1e-3) + 1e-9
    assert abs(lb.params.c1 - nm.params.c1) < 5e-3 and abs(lb.params.c2 - nm.params.c2) < 5e-2
    assert abs(lb.params.c1 - 1.015) < 0.01 and abs(lb.params.c2 - 0.9) < 0.2
    assert lb.chi2 < 2.0


def test_saxs_scorer_reports_the_fit(engine):  # analysis.rs:137-178
    """Quality::Fast (the scorer's default) fits on every 20th q with cubic
    Hermite interpolation of the basis: 600 q give 30 sampled points, as the
    reference's own 612-point fits do."""
    s = synth.protein(77, 1200, 16.0)
    q = np.linspace(0.01, 0.45, 600)
    y, sigma = _debye_experiment(s, q, 1.0, 0.5, 2.0, 10.0, 3)
    ex = cs.ExperimentalCurve(q, y, sigma)
    fo = cs.FitOptions(method=cs.ScatteringMethod.Debye)
    r = cs.SaxsScorer(ex, cs.ScoreOptions(fit=fo), engine=engine).score(s)
    assert r.points == len(q) and r.q_min == q[0] and r.q_max == q[-1] and r.has_errors
    assert r.reduced_chi2 == pytest.approx(r.fit.chi2)
    cmp = cs.compare_curves(ex, r.fit.fitted_curve)
    assert cmp.reduced_chi2 == pytest.approx(r.reduced_chi2, rel=1e-9)
    assert r.reduced_chi2 < 3.0 and cmp.pearson_correlation > 0.999
    with pytest.raises(cs.InvalidInput):
        cs.SaxsScorer(cs.ExperimentalCurve(np.zeros(0), np.zeros(0), np.zeros(0)))
