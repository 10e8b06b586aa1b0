"""Batched ensemble scoring on the GPU against the oracle.

The batched curves must equal the per-conformer plain curves and the oracle
curves (1e-5 relative); the device weight fit, KL reweighting and gradients
follow ensemble.rs / reweight.rs on the same curves (f64 on both sides, so
they agree to round-off: 1e-8).
"""
import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O
from crabsaxs_b200 import synth

pytestmark = pytest.mark.gpu

CURVE_RTOL = 1e-5


def _small_ensemble(k=12, seed=3):
    sizes = np.random.default_rng(seed).integers(150, 700, size=k)
    return [synth.protein(500 + i, int(n), 6.0 + 0.02 * n) for i, n in enumerate(sizes)]


def _experiment(curves, hidden, seed):
    rng = np.random.default_rng(seed)
    w = rng.dirichlet(np.ones(len(hidden)))
    clean = (w[:, None] * curves[hidden]).sum(axis=0)
    sigma = 0.01 * clean
    return clean + sigma * rng.normal(size=clean.shape), sigma


def test_batched_curves_match_plain_and_oracle(engine):
    confs = _small_ensemble()
    q = np.linspace(0.005, 0.45, 120)
    cand = cs.solvent_candidates(cs.FitOptions())[[0, 7, 24]]
    got = cs.ensemble_curves(confs, q, cs.SolventParams(), cand, engine=engine)
    for ci, (c1, c2) in enumerate(cand):
        for k in (0, 5, 11):
            plain = cs.compute_curve(confs[k], q, cs.ComputeOptions(method=cs.ScatteringMethod.Debye,
                                                                    solvent=cs.SolventParams(c1=c1, c2=c2)),
                                     engine=engine).intensity
            ref = O.combine_solvent_basis(O.debye_solvent_basis(O.Atoms(confs[k].xyz, confs[k].element), q, c1, c2),
                                          q, c1, c2)
            assert np.max(np.abs(got[ci, k] - plain) / ref) <= 1e-6
            assert np.max(np.abs(got[ci, k] - ref) / ref) <= CURVE_RTOL


def test_plan_score_matches_oracle_weights_and_reweighting(engine):
    confs = _small_ensemble(16, 9)
    q = np.linspace(0.005, 0.45, 90)
    cand = cs.solvent_candidates(cs.FitOptions())
    curves = cs.ensemble_curves(confs, q, cs.SolventParams(), cand, engine=engine)
    y, sigma = _experiment(curves[12], [1, 4, 7, 9], 5)
    plan = cs.EnsemblePlan(confs, q, cs.SolventParams(), cand, engine=engine)
    try:
        rw = cs.MaximumEntropyOptions(kl_strength=0.05)
        out = plan.score(y, sigma, cs.FitOptions(), rw)
        out2 = plan.score(y, sigma, cs.FitOptions(), rw)  # graph replay
    finally:
        plan.close()
    # oracle: optimize_weights per candidate on the same curves, best by χ²
    best, best_chi, best_w = None, None, None
    for c in range(len(cand)):
        w, s, b, chi, _ = O.optimize_weights(curves[c], y, sigma)
        if best_chi is None or chi < best_chi:
            best, best_chi, best_w = c, chi, w
    assert out["candidate"] == best
    assert out["reduced_chi2"] == pytest.approx(best_chi, rel=1e-8)
    np.testing.assert_allclose(out["weights"], best_w, atol=1e-8)
    assert out2["candidate"] == best and np.allclose(out2["weights"], out["weights"], atol=1e-14)
    ref = O.reweight_curves(curves[best], y, sigma, kl_strength=0.05)
    np.testing.assert_allclose(out["kl_weights"], ref["weights"], atol=1e-8)
    assert out["kl_iterations"] == ref["iterations"]
    # ∂χ²/∂w at the final weights (scale, background held) by central differences
    s, b = out["scale"], out["background"]
    dof = len(q) - 1

    def chi_w(w):
        return np.sum(((s * (w @ curves[best]) + b - y) / sigma) ** 2) / dof

    h = 1e-7
    for k in (0, 3, 15):
        e = np.zeros(len(confs))
        e[k] = h
        fd = (chi_w(out["weights"] + e) - chi_w(out["weights"] - e)) / (2 * h)
        assert abs(out["dchi2_dw"][k] - fd) <= 1e-5 * max(abs(fd), 1.0)
    # ∂χ²/∂(c1, c2) at the best candidate by central differences of the curves
    c1, c2 = cand[best]
    for m, dc in enumerate([(1e-5, 0.0), (0.0, 1e-4)]):
        cp = cs.ensemble_curves(confs, q, cs.SolventParams(), [[c1 + dc[0], c2 + dc[1]]], engine=engine)[0]
        cm = cs.ensemble_curves(confs, q, cs.SolventParams(), [[c1 - dc[0], c2 - dc[1]]], engine=engine)[0]
        hstep = dc[0] or dc[1]
        fd = (chi_w_curves(cp, out, y, sigma) - chi_w_curves(cm, out, y, sigma)) / (2 * hstep)
        got = out["dchi2_dc1" if m == 0 else "dchi2_dc2"]
        assert abs(got - fd) <= 1e-3 * max(abs(fd), 1e-6), (m, got, fd)


def chi_w_curves(curves, out, y, sigma):
    s, b, w = out["scale"], out["background"], out["weights"]
    return np.sum(((s * (w @ curves) + b - y) / sigma) ** 2) / (len(y) - 1)


def test_ensemble_fitter_matches_oracle_fit_core(engine):  # ensemble.rs:127-299
    confs = _small_ensemble(10, 21)
    q = np.linspace(0.005, 0.45, 80)
    fo = cs.FitOptions(method=cs.ScatteringMethod.Debye)
    cand = cs.solvent_candidates(fo)
    curves = cs.ensemble_curves(confs, q, cs.SolventParams(), cand, engine=engine)
    y, sigma = _experiment(curves[6], [2, 5], 2)
    ex = cs.ExperimentalCurve(q, y, sigma)
    res = cs.EnsembleFitter(confs, [f"c{i}" for i in range(10)], ex, cs.EnsembleOptions(fit=fo), engine=engine).fit()
    oc = [O.optimize_weights(curves[c], y, sigma) for c in range(25)]
    best = min(range(25), key=lambda c: (oc[c][3], c))
    assert res.reduced_chi2 == pytest.approx(oc[best][3], rel=1e-8)
    assert (res.params.c1, res.params.c2) == pytest.approx(tuple(cand[best]))
    np.testing.assert_allclose(res.weights, oc[best][0], atol=1e-8)
    np.testing.assert_allclose(res.fitted_curve, oc[best][4], rtol=1e-9)


def test_ensemble_pruning_and_bootstrap(engine):
    confs = _small_ensemble(8, 4)
    q = np.linspace(0.005, 0.45, 60)
    fo = cs.FitOptions(method=cs.ScatteringMethod.Debye)
    curves = cs.ensemble_curves(confs, q, cs.SolventParams(), cs.solvent_candidates(fo), engine=engine)
    y, sigma = _experiment(curves[12], [0, 3], 8)
    ex = cs.ExperimentalCurve(q, y, sigma)
    opt = cs.EnsembleOptions(fit=fo, min_weight=0.05, max_conformers=3, bootstrap=4)
    res = cs.EnsembleFitter(confs, [f"c{i}" for i in range(8)], ex, opt, engine=engine).fit()
    assert 1 <= len(res.conformers) <= 3
    assert res.weights.sum() == pytest.approx(1.0)
    assert len(res.weight_intervals) == len(res.conformers) and len(res.bootstrap_reduced_chi2) == 4
    for iv in res.weight_intervals:
        assert iv.lower <= iv.median <= iv.upper


def test_ensemble_rejects_bad_input(engine):
    confs = _small_ensemble(3, 1)
    ex = cs.ExperimentalCurve(np.linspace(0.01, 0.3, 10), np.ones(10), np.ones(10))
    with pytest.raises(cs.InvalidInput):
        cs.EnsembleFitter(confs, ["a"], ex)
    with pytest.raises(cs.InvalidInput):
        cs.EnsembleFitter(confs, ["a", "b", "c"], ex, cs.EnsembleOptions(min_weight=1.5))
