"""χ² and its adjoint gradient on the GPU (crab_chi2_grad) against the
oracle's f64 analytic gradient and FP64 central finite differences.

Tolerance: gradients within 1e-5 of their largest component (max-norm
relative error; individual components pass through zero), χ² within 1e-5
relative.
"""
import math

import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-5


def _amplitudes(s: cs.Structure, q, c1, c2, thickness=3.0, density=0.334):
    """Per-atom A_i(q) = v_i - G e_i + c2 h_i in f64 (solvent.rs:454-488, 448-452)."""
    A = np.empty((s.atom_count, len(q)))
    G = np.array([O.lib.orc_excluded_volume_scale(x, c1) for x in q])
    for i in range(s.atom_count):
        e, g = int(s.element[i]), int(s.group[i])
        v = np.array([O.lib.orc_form_factor(e, g, s.occupancy[i], 1, x) for x in q])
        vol = O.lib.orc_excluded_volume_for_atom(e, g, 1)
        rad = (3.0 * vol / (4.0 * math.pi)) ** (1.0 / 3.0)
        ex = s.occupancy[i] * density * vol * np.exp(-(vol ** (2.0 / 3.0)) * q * q / (4.0 * math.pi))
        sv = 4.0 * math.pi * (rad + thickness / 2.0) ** 2 * thickness
        h = s.occupancy[i] * density * 0.1 * sv * np.exp(-(sv ** (2.0 / 3.0)) * q * q / (4.0 * math.pi))
        A[i] = v - G * ex + c2 * h
    return A


def _sinc(x):
    out = np.ones_like(x)
    m = np.abs(x) >= 1e-8
    out[m] = np.sin(x[m]) / x[m]
    return out


def _experiment(s, q, seed):
    """5,000 atoms: Debye of a copy perturbed by N(0, 0.5 Å), scale 3.7, background 1e-3·I(0),
    σ(q) = 0.01·I(q) + 1e-4·I(0), Gaussian noise of that σ."""
    rng = np.random.default_rng(seed)
    pert = cs.Structure(s.xyz + rng.normal(scale=0.5, size=s.xyz.shape), s.element)
    a = O.Atoms(pert.xyz, pert.element)
    I = O.combine_solvent_basis(O.debye_solvent_basis(a, q, 1.0, 0.0), q, 1.0, 0.0)
    I0 = I[0]
    clean = 3.7 * I + 1e-3 * I0
    sigma = 0.01 * I + 1e-4 * I0
    return clean + sigma * rng.normal(size=len(q)), sigma


def test_gradient_matches_oracle_analytic(engine):
    from crabsaxs_b200 import synth

    s = synth.protein(44, 400, 12.0)
    q = np.arange(1, 101) * 0.005
    y, sigma = _experiment(s, q, 1)
    a = O.Atoms(s.xyz, s.element)
    for c1, c2, sc, bg in [(1.0, 0.0, 3.7, 0.0), (1.03, 0.8, 3.5, 1e3)]:
        chi, gx, gp = cs.chi2_grad(s, q, y, sigma, cs.SolventParams(c1=c1, c2=c2), sc, bg, engine=engine)
        rchi, rgx, rgp = O.chi2_grad(a, q, y, sigma, c1, c2, sc, bg)
        assert abs(chi - rchi) / rchi <= 1e-5
        assert np.max(np.abs(gx - rgx)) / np.max(np.abs(rgx)) <= GRAD_TOL
        assert np.max(np.abs(gp - rgp) / np.maximum(np.abs(rgp), 1e-12 * np.abs(rgp).max())) <= 1e-4


def test_gradient_5k_central_differences(engine):
    """5,000 atoms (R 28 Å), 100 q: 64 seeded coordinates against FP64 central differences
    (h = 1e-4 Å) computed with incremental O(N·Nq) pair deltas, and the four scalars against
    FP64 central differences of the oracle's χ²."""
    from crabsaxs_b200 import synth

    w = synth.GRADIENT_5K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    q = w.q
    y, sigma = _experiment(s, q, 4)
    c1, c2, sc, bg = 1.0, 0.0, 3.7, 1e-3 * 0.0
    sp = cs.SolventParams(c1=c1, c2=c2)
    chi, gx, gp = cs.chi2_grad(s, q, y, sigma, sp, sc, bg, engine=engine)
    a = O.Atoms(s.xyz, s.element)
    basis = O.debye_solvent_basis(a, q, c1, c2)
    I = O.combine_solvent_basis(basis, q, c1, c2)
    dof = len(q) - 1

    def chi_of(Iq):
        return float(np.sum(((sc * Iq + bg - y) / sigma) ** 2) / dof)

    assert abs(chi - chi_of(I)) / chi_of(I) <= 1e-5
    A = _amplitudes(s, q, c1, c2)
    rng = np.random.default_rng(7)
    picks = [(int(i), int(d)) for i, d in zip(rng.choice(s.atom_count, 64, replace=False), rng.integers(0, 3, 64))]
    h = 1e-4
    fd = np.empty(len(picks))
    for n, (i, d) in enumerate(picks):
        others = np.delete(np.arange(s.atom_count), i)
        xo = s.xyz[others]
        r0 = np.linalg.norm(xo - s.xyz[i], axis=1)
        base = (2.0 * A[i][None, :] * A[others]) * _sinc(q[None, :] * r0[:, None])
        vals = []
        for sgn in (1.0, -1.0):
            xi = s.xyz[i].copy()
            xi[d] += sgn * h
            r1 = np.linalg.norm(xo - xi, axis=1)
            dI = np.sum((2.0 * A[i][None, :] * A[others]) * _sinc(q[None, :] * r1[:, None]) - base, axis=0)
            vals.append(chi_of(I + dI))
        fd[n] = (vals[0] - vals[1]) / (2 * h)
    got = np.array([gx[i, d] for i, d in picks])
    scale = np.max(np.abs(gx))
    assert np.max(np.abs(got - fd)) / scale <= GRAD_TOL, np.max(np.abs(got - fd)) / scale
    # scalars: central differences of the oracle χ² (f64)
    for k, delta in enumerate([(1e-5, 0, 0, 0), (0, 1e-5, 0, 0), (0, 0, 1e-5, 0), (0, 0, 0, 1e-2)]):
        p = np.array([c1, c2, sc, bg])
        hp = np.array(delta)
        cp = O.chi2_grad(a, q, y, sigma, *(p + hp), want_xyz=False)[0]
        cm = O.chi2_grad(a, q, y, sigma, *(p - hp), want_xyz=False)[0]
        fdk = (cp - cm) / (2 * hp[k])
        assert abs(gp[k] - fdk) <= 1e-4 * max(abs(fdk), 1e-9), (k, gp[k], fdk)


def test_gradient_rejects_grid_hydration(engine):
    from crabsaxs_b200 import synth

    s = synth.protein(1, 50, 8.0)
    q = np.linspace(0.01, 0.3, 20)
    with pytest.raises(cs.InvalidInput):
        cs.chi2_grad(s, q, np.ones(20), np.ones(20),
                     cs.SolventParams(hydration_model=cs.HydrationModel.AdaptiveGrid), 1.0, 0.0, engine=engine)
