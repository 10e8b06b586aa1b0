"""Coordinate P(r) on the GPU (metrics.rs:236-270, 475-583) against the oracle.

Bins are index work and must be the reference's bit for bit: with unit
weights every bin holds an integer count, which f64 sums exactly in any
order, so those histograms must equal the oracle's exactly.  Weighted sums
differ only by summation order: 1e-12 of the largest bin.  Rg and dmax are
computed in the reference's own order and must be equal.
"""
import math

import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O
from crabsaxs_b200 import synth

pytestmark = pytest.mark.gpu

C_, H_, N_, O_, S_ = 1, 0, 2, 3, 4
SUM_RTOL = 1e-12


def _oracle_atoms(s: cs.Structure):
    return O.Atoms(s.xyz, s.element, s.group, s.occupancy)


def _check_features(s: cs.Structure, bins, engine):
    got = cs.coordinate_features(s, cs.PrOptions(bins=bins), engine=engine)
    ref = O.coordinate_features(_oracle_atoms(s), bins)
    assert got.rg == ref["rg"] and got.dmax == ref["dmax"]
    assert np.array_equal(got.p_r.r, ref["r"])
    scale = np.max(np.abs(ref["p"]))
    assert np.max(np.abs(got.p_r.p - ref["p"])) <= SUM_RTOL * scale
    assert got.p_r.rg == pytest.approx(ref["pr_rg"], rel=SUM_RTOL)
    assert got.p_r.dmax == ref["pr_dmax"]
    return got


def test_coordinate_features_report_pair_distance(engine):  # metrics.rs:678-684
    s = cs.Structure(np.array([[0.0, 0.0, 0.0], [4.0, 0.0, 0.0]]), np.array([C_, C_]))
    f = _check_features(s, 160, engine)
    assert abs(f.dmax - 4.0) < 1e-12 and f.rg > 1.0 and len(f.p_r.p) > 0


@pytest.mark.parametrize("n,bins", [(300, 160), (1000, 16), (2500, 160), (2500, 1000), (777, 7)])
def test_protein_features_match_oracle(engine, n, bins):
    s = synth.protein(40 + n, n, 6.0 + n ** (1.0 / 3.0))
    _check_features(s, bins, engine)


def test_groups_occupancy_and_hydrogen_floor(engine):
    """United-atom groups change the weights, occupancies scale them, and
    hydrogens (form factor 0 with implicit hydrogens) take the 1e-6 floor."""
    base = synth.protein(91, 1500, 14.0)
    rng = np.random.default_rng(5)
    n = len(base.xyz)
    el = base.element.copy()
    el[rng.random(n) < 0.1] = H_
    group = np.where(el == C_, rng.integers(-1, 4, n), -1).astype(np.int8)
    group[(el == N_) & (rng.random(n) < 0.5)] = 7
    occ = np.where(rng.random(n) < 0.2, 0.5, 1.0)
    s = cs.Structure(base.xyz, el, occ, group)
    _check_features(s, 200, engine)


def _mode(engine):
    return cs.pr_last_timing(engine)[3]


def test_unit_weight_bins_are_exact(engine):
    """Unit weights: one weight class, integer pair counts (mode 0)."""
    s = synth.protein(17, 3000, 20.0)
    for bins in (16, 160, 4096):
        dmax, hist = cs.pair_distance_histogram(s.xyz, np.ones(len(s.xyz)), bins, engine=engine)
        assert _mode(engine) == 0
        rd, rh = O.pair_distance_histogram(s.xyz, np.ones(len(s.xyz)), bins)
        assert dmax == rd and np.array_equal(hist, rh), bins


def test_integer_weight_bins_are_exact_in_the_f64_mode(engine):
    """100 distinct integer weights exceed the 64 weight classes, so the
    products go through the per-warp f64 histograms (mode 1); integer sums
    below 2^53 are exact in any order, so the bins must equal the oracle's."""
    s = synth.protein(18, 2800, 19.0)
    w = 1.0 + (np.arange(len(s.xyz)) % 100)
    for bins in (16, 160, 3000):
        dmax, hist = cs.pair_distance_histogram(s.xyz, w, bins, engine=engine)
        assert _mode(engine) == 1
        rd, rh = O.pair_distance_histogram(s.xyz, w, bins)
        assert dmax == rd and np.array_equal(hist, rh), bins


def test_several_weight_classes_count_exactly(engine):
    """A few distinct weights: per-class-pair counts (mode 0) combined as
    count * w_a * w_b against the oracle's pair-by-pair sums."""
    s = synth.protein(19, 2000, 16.0)
    w = np.array([1.0, 6.5, 7.25, 8.0, 16.125])[np.arange(len(s.xyz)) % 5]
    dmax, hist = cs.pair_distance_histogram(s.xyz, w, 160, engine=engine)
    assert _mode(engine) == 0
    rd, rh = O.pair_distance_histogram(s.xyz, w, 160)
    assert dmax == rd and np.array_equal(hist, rh)


def test_pairs_on_exact_bin_edges(engine):
    """Integer distances with step 1 sit exactly on bin edges; distance 16 is
    capped into the last bin (metrics.rs:515-516)."""
    xyz = np.zeros((17, 3))
    xyz[:, 0] = np.arange(17)
    dmax, hist = cs.pair_distance_histogram(xyz, np.ones(17), 16, engine=engine)
    expected = np.array([0.0] + [17.0 - k for k in range(1, 16)])
    expected[15] += 1.0
    assert dmax == 16.0 and np.array_equal(hist, expected)
    # a cubic lattice away from the origin: many equal distances at every radius
    g = np.stack(np.meshgrid(*[np.arange(9) * 1.25] * 3, indexing="ij"), -1).reshape(-1, 3) + 500.0
    for bins in (20, 160, 333):
        d, h = cs.pair_distance_histogram(g, np.ones(len(g)), bins, engine=engine)
        rd, rh = O.pair_distance_histogram(g, np.ones(len(g)), bins)
        assert d == rd and np.array_equal(h, rh), bins


def test_many_bins_use_the_global_histogram(engine):
    """Above ~6,000 bins (f64) or ~8,000 (counts) the histograms no longer fit
    in shared memory and each block accumulates into its own row in device
    memory (mode 2).  20,000 bins still take the FP32 fast path with a wide
    edge margin; above 75,000 bins the margin reaches a quarter bin and every
    pair takes the exact f64 path; above 2^20 bins as well."""
    s = synth.protein(23, 1200, 13.0)
    w = np.random.default_rng(2).uniform(1.0, 16.0, len(s.xyz))
    dmax, hist = cs.pair_distance_histogram(s.xyz, w, 20000, engine=engine)
    assert _mode(engine) == 2
    rd, rh = O.pair_distance_histogram(s.xyz, w, 20000)
    assert dmax == rd
    assert np.max(np.abs(hist - rh)) <= SUM_RTOL * np.max(rh)
    small = synth.protein(24, 300, 8.0)
    for atoms, bins in ((s, 20000), (s, 100000), (small, 1_200_000)):
        n = len(atoms.xyz)
        d1, h1 = cs.pair_distance_histogram(atoms.xyz, np.ones(n), bins, engine=engine)
        assert _mode(engine) == 2
        r1 = O.pair_distance_histogram(atoms.xyz, np.ones(n), bins)[1]
        assert np.array_equal(h1, r1), bins


def test_single_point_and_invalid_inputs(engine):  # metrics.rs:241-244, 489-498
    same = cs.Structure(np.tile([1.0, -2.0, 3.0], (300, 1)), np.full(300, C_))
    for s in (same, cs.Structure(np.array([[5.0, 5.0, 5.0]]), np.array([O_]))):
        f = cs.coordinate_features(s, engine=engine)
        assert f.dmax == 0.0 and list(f.p_r.r) == [0.0] and list(f.p_r.p) == [1.0]
        assert f.p_r.rg == 0.0 and f.p_r.dmax == 0.0
    d, h = cs.pair_distance_histogram(np.zeros((0, 3)), np.zeros(0), 16, engine=engine)
    assert d == 0.0 and not h.any()
    with pytest.raises(cs.InvalidInput):
        cs.coordinate_features(cs.Structure(np.zeros((0, 3)), np.zeros(0, dtype=np.int8)), engine=engine)
    with pytest.raises(cs.InvalidInput):
        cs.pair_distance_histogram(np.zeros((3, 3)), np.ones(3), 0, engine=engine)
    with pytest.raises(cs.InvalidInput):
        cs.pair_distance_histogram(np.array([[0.0, 0, 0], [1e101, 0, 0]]), np.ones(2), 16, engine=engine)


def test_large_structure_matches_oracle(engine):
    """30,000 atoms (4.5e8 pairs): P(r) against the oracle, with the element
    weights (class counts) and with random per-atom weights (f64 mode)."""
    s = synth.protein(29, 30000, 40.0)
    _check_features(s, 160, engine)
    assert _mode(engine) == 0
    w = np.random.default_rng(4).uniform(0.5, 9.0, len(s.xyz))
    dmax, hist = cs.pair_distance_histogram(s.xyz, w, 160, engine=engine)
    assert _mode(engine) == 1
    rd, rh = O.pair_distance_histogram(s.xyz, w, 160)
    assert dmax == rd and np.max(np.abs(hist - rh)) <= SUM_RTOL * np.max(rh)


def test_100k_atoms_size_properties(engine):
    """100,000 atoms (R 80 Å): unit weights count every pair exactly once
    (sum n(n-1)/2, exact in f64), weighted sums total ((Σw)² - Σw²)/2, and
    dmax is at least the largest distance between extreme atoms."""
    w_ = synth.ATOMS_100K
    s = synth.protein(w_.seed, w_.n_atoms, w_.radius)
    n = len(s.xyz)
    _, h1 = cs.pair_distance_histogram(s.xyz, np.ones(n), 160, engine=engine)
    assert h1.sum() == n * (n - 1) / 2 and np.all(h1 == np.round(h1))
    w = np.random.default_rng(8).uniform(0.5, 9.0, n)
    dmax, h = cs.pair_distance_histogram(s.xyz, w, 160, engine=engine)
    total = (math.fsum(w) ** 2 - math.fsum(w * w)) / 2.0
    assert abs(h.sum() - total) <= 1e-11 * total
    ext = s.xyz[np.concatenate([np.argmin(s.xyz, 0), np.argmax(s.xyz, 0)])]
    dd = ext[:, None, :] - ext[None, :, :]
    assert dmax >= math.sqrt(np.max(np.sum(dd * dd, -1))) - 1e-9
    total_ms, hist_ms, pairs, mode = cs.pr_last_timing(engine)
    assert pairs == n * (n - 1) / 2 and 0.0 < hist_ms <= total_ms and mode == 1
