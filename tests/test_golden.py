"""Golden fixture tests/golden/small_protein.json (made by
tests/golden/make_golden.py from the oracle): a 300-atom structure and the
oracle's Debye solvent basis, hydration sites, pair-distance histogram and
FP64 multipole curve for it.  On the CPU the oracle must still reproduce the
fixture; on the GPU the CUDA path must match it with the tolerances of the
parity tests (bit-exact for sites and unit-weight bins)."""
import json
from pathlib import Path

import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O
from crabsaxs_b200 import _native as N

G = json.loads((Path(__file__).parent / "golden" / "small_protein.json").read_text())
ST = G["structure"]
XYZ = np.array(ST["xyz"])
EL = np.array(ST["element"], dtype=np.int8)
GROUP = np.array(ST["group"], dtype=np.int8)
OCC = np.array(ST["occupancy"])
Q = np.array(G["q"])


def _structure():
    return cs.Structure(XYZ, EL, OCC, GROUP)


def test_oracle_reproduces_the_fixture():
    a = O.Atoms(XYZ, EL, GROUP, OCC)
    np.testing.assert_allclose(O.debye_solvent_basis(a, Q, 1.0, 0.0), np.array(G["debye_solvent_basis"]),
                               rtol=1e-13, atol=0.0)
    ad, av = O.adaptive_grid(XYZ, 3.0)
    assert np.array_equal(ad, np.array(G["adaptive_grid_3A"]["sites"])) and av == G["adaptive_grid_3A"]["voxel_volume"]
    ex, ev = O.exterior_grid(XYZ, EL.astype(np.int32), 1.5)
    assert np.array_equal(ex, np.array(G["exterior_grid_1p5A"]["sites"]))
    assert ev == G["exterior_grid_1p5A"]["voxel_volume"]
    dmax, hist = O.pair_distance_histogram(XYZ, np.ones(len(XYZ)), 64)
    ref = G["pair_distance_histogram_64"]
    assert dmax == ref["dmax"] and np.array_equal(hist, np.array(ref["counts"]))
    assert hist.sum() == len(XYZ) * (len(XYZ) - 1) / 2
    np.testing.assert_allclose(O.multipole_intensity(a, Q, 14), np.array(G["multipole_intensity_L14"]), rtol=1e-12)


@pytest.mark.gpu
def test_device_matches_the_fixture(engine):
    s = _structure()
    basis = cs.debye_solvent_basis(s, Q, cs.SolventParams(), engine=engine)
    ref = np.array(G["debye_solvent_basis"])
    for c1, c2 in ((1.0, 0.0), (1.03, 0.8), (0.96, -0.4)):
        got_i = cs.combine_solvent_basis(basis, Q, c1, c2)
        ref_i = cs.combine_solvent_basis(ref, Q, c1, c2)
        assert np.max(np.abs(got_i - ref_i) / np.abs(ref_i)) <= 1e-5, (c1, c2)
    ad, av = cs.hydration_grid_adaptive(s, 3.0, engine=engine)
    assert np.array_equal(ad, np.array(G["adaptive_grid_3A"]["sites"])) and av == G["adaptive_grid_3A"]["voxel_volume"]
    ex, ev = cs.hydration_grid_exterior(s, 1.5, engine=engine)
    assert np.array_equal(ex, np.array(G["exterior_grid_1p5A"]["sites"]))
    dmax, hist = cs.pair_distance_histogram(XYZ, np.ones(len(XYZ)), 64, engine=engine)
    ref_h = G["pair_distance_histogram_64"]
    assert dmax == ref_h["dmax"] and np.array_equal(hist, np.array(ref_h["counts"]))
    mp_ref = np.array(G["multipole_intensity_L14"])
    mp64 = cs.multipole_intensity(s, Q, 14, precision=N.PREC_FP64, engine=engine)
    np.testing.assert_allclose(mp64, mp_ref, rtol=1e-9)
    mp = cs.multipole_intensity(s, Q, 14, engine=engine)  # tensor-core TF32 hi+lo
    assert np.max(np.abs(mp - mp_ref) / np.abs(mp_ref)) <= 1e-5
