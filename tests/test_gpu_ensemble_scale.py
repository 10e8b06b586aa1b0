"""The batched ensemble at full size: 256 conformers with log-uniform atom
counts in 2,000-40,000, 300 q on [0.005, 0.45], the 25 (c1, c2) candidates of
ensemble.rs:302-315, analytic hydration (the FitOptions default).

The reference scores such an ensemble with 25 x 256 compute_curve calls
(ensemble.rs:244-261), then fits simplex weights per candidate
(ensemble.rs:317-381) and reweights by KL mirror descent (reweight.rs:84-154).
Checks, with the tolerances of the other ensemble tests:
  * batched curves against the f64 oracle at 8 q points (the whole grid is
    out of reach of the CPU for 40,000 atoms) for the smallest, the largest
    and two middle conformers, all 25 candidates: 1e-5 relative;
  * all 25 x 256 batched curves against the FP64 device kernel at every q:
    1e-5 relative;
  * the graph's simplex weights and KL weights against the oracle's
    optimize_weights and reweight_curves on the same curves: 1e-8.
"""
import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O
from crabsaxs_b200 import synth

pytestmark = pytest.mark.gpu

CURVE_RTOL = 1e-5
WEIGHT_ATOL = 1e-8


@pytest.fixture(scope="module")
def ensemble256(engine):
    confs = synth.ensemble(256)
    q = synth.ENSEMBLE_Q
    fo = cs.FitOptions(method=cs.ScatteringMethod.Debye)
    cand = cs.solvent_candidates(fo)
    curves = cs.ensemble_curves(confs, q, cs.SolventParams(), cand, engine=engine)
    return confs, q, fo, cand, curves


def test_ensemble_spans_the_workload_sizes(ensemble256):
    confs, q, _, cand, curves = ensemble256
    sizes = np.array([c.atom_count for c in confs])
    assert len(confs) == 256 and len(q) == 300 and cand.shape == (25, 2)
    assert sizes.min() < 2200 and sizes.max() > 36000
    assert curves.shape == (25, 256, 300) and np.all(np.isfinite(curves)) and np.all(curves > 0)


def test_batched_curves_match_oracle_on_a_q_subset(ensemble256):
    confs, q, _, cand, curves = ensemble256
    order = np.argsort([c.atom_count for c in confs])
    pick = [order[0], order[85], order[170], order[-1]]
    qi = np.array([0, 37, 80, 121, 166, 210, 255, 299])
    for k in pick:
        c = confs[k]
        basis = O.debye_solvent_basis(O.Atoms(c.xyz, c.element, c.group, c.occupancy), q[qi])
        for ci, (c1, c2) in enumerate(cand):
            ref = O.combine_solvent_basis(basis, q[qi], c1, c2)
            err = np.max(np.abs(curves[ci, k, qi] - ref) / ref)
            assert err <= CURVE_RTOL, (c.atom_count, ci, err)


def test_all_batched_curves_match_fp64_device_kernel(engine, ensemble256):
    confs, q, _, cand, curves = ensemble256
    worst = 0.0
    for k, c in enumerate(confs):
        b64 = cs.debye_solvent_basis(c, q, cs.SolventParams(), engine=engine, fp64=True)
        for ci, (c1, c2) in enumerate(cand):
            ref = cs.combine_solvent_basis(b64, q, c1, c2)
            worst = max(worst, float(np.max(np.abs(curves[ci, k] - ref) / ref)))
    assert worst <= CURVE_RTOL, worst


def test_graph_weights_and_kl_reweighting_match_oracle(engine, ensemble256):
    confs, q, fo, cand, curves = ensemble256
    rng = np.random.default_rng(55)
    hidden = rng.choice(len(confs), 8, replace=False)
    clean = rng.dirichlet(np.ones(8)) @ curves[12, hidden]
    sigma = 0.01 * clean
    y = clean + sigma * rng.normal(size=len(q))
    plan = cs.EnsemblePlan(confs, q, cs.SolventParams(), cand, engine=engine)
    try:
        out = plan.score(y, sigma, fo, cs.MaximumEntropyOptions())
    finally:
        plan.close()
    fits = [O.optimize_weights(curves[c], y, sigma) for c in range(len(cand))]
    best = min(range(len(cand)), key=lambda c: (fits[c][3], c))
    assert out["candidate"] == best
    assert out["reduced_chi2"] == pytest.approx(fits[best][3], rel=1e-8)
    np.testing.assert_allclose(out["weights"], fits[best][0], atol=WEIGHT_ATOL)
    ref = O.reweight_curves(curves[best], y, sigma)
    np.testing.assert_allclose(out["kl_weights"], ref["weights"], atol=WEIGHT_ATOL)
    assert out["kl_iterations"] == ref["iterations"]
