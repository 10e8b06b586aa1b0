"""Error paths of the C ABI, with the failure made on the host.

The reference validates its inputs and reports SaxsError values
(scattering.rs:71-80, 117-143; error.rs:4-25).  Here the same validation
returns CRAB_EINVAL (InvalidInput), and the device-side failure modes are
reached without a GPU fault: a context option shortens the kernels' bounded
waits to zero iterations, so their first wait gives up and the call returns
CRAB_ETIMEOUT after the kernel has drained its own copies and tensor-core work
in flight; another option fails the context's allocations.  After each
failure the same context must compute the same curve as an untouched one.
"""
import numpy as np
import pytest

import crabsaxs_b200 as cs
from crabsaxs_b200 import _native as N
from crabsaxs_b200 import synth
from crabsaxs_b200.api import Engine, InvalidInput, Other

pytestmark = pytest.mark.gpu

Q = np.arange(1, 101) * 0.005  # uniform: the FP32 recurrence kernel


@pytest.fixture()
def fresh():
    e = Engine(0)
    yield e
    e.close()


def test_pair_kernel_wait_runs_out_then_context_recovers(engine, fresh):
    s = synth.protein(301, 1500, 18.0)
    ref = cs.debye_intensity(s, Q, engine=engine)
    fresh.set_wait_budget(0)
    for _ in range(2):  # every launch gives up at its first tile, drains and reports
        with pytest.raises(Other, match="ETIMEOUT"):
            cs.debye_intensity(s, Q, engine=fresh)
    fresh.set_wait_budget(None)
    got = cs.debye_intensity(s, Q, engine=fresh)
    assert np.array_equal(got, ref) or np.max(np.abs(got - ref) / ref) <= 1e-12


@pytest.mark.parametrize("variant", [168 * 16 + 5, 168 * 16 + 11, 126 * 16 + 13, 126 * 16 + 14, 126 * 16 + 15, 100 * 16 + 15,
                                     84 * 16 + 12])
def test_every_pair_kernel_family_wait_runs_out_then_recovers(engine, fresh, variant):
    """The folded q-packed kernel, the three-CTA build and the set-up /
    recurrence split: each gives up at its first wait, reports, and leaves the
    context usable."""
    s = synth.protein(307, 2500, 20.0)
    ref = cs.debye_intensity(s, Q, engine=engine)
    fresh.check(N.lib.crab_ctx_set_pair_variant(fresh.handle, variant))
    fresh.set_wait_budget(0)
    for _ in range(2):
        with pytest.raises(Other, match="ETIMEOUT"):
            cs.debye_intensity(s, Q, engine=fresh)
    fresh.set_wait_budget(None)
    got = cs.debye_intensity(s, Q, engine=fresh)
    np.testing.assert_allclose(got, ref, rtol=2e-6)


def test_solvent_basis_wait_runs_out_then_recovers(engine, fresh):
    s = synth.protein(302, 900, 15.0)
    p = cs.SolventParams(c1=1.02, c2=1.3, hydration_model=cs.HydrationModel.AdaptiveGrid)
    ref = cs.debye_solvent_basis(s, Q, p, engine=engine)
    fresh.set_wait_budget(0)
    with pytest.raises(Other, match="ETIMEOUT"):
        cs.debye_solvent_basis(s, Q, p, engine=fresh)
    fresh.set_wait_budget(None)
    got = cs.debye_solvent_basis(s, Q, p, engine=fresh)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("precision", [N.PREC_TF32_SPLIT, N.PREC_TF32, N.PREC_TF32_SPLIT_FUSED, N.PREC_BF16_SPLIT,
                                       N.PREC_BF16])
def test_tensor_core_gemm_wait_runs_out_then_recovers(engine, fresh, precision):
    s = synth.protein(303, 3000, 22.0)
    q = np.linspace(0.001, 0.5, 120)
    ref = cs.multipole_intensity(s, q, 30, precision=precision, engine=engine)
    fresh.set_wait_budget(0)
    with pytest.raises(Other, match="ETIMEOUT"):
        cs.multipole_intensity(s, q, 30, precision=precision, engine=fresh)
    fresh.set_wait_budget(None)
    got = cs.multipole_intensity(s, q, 30, precision=precision, engine=fresh)
    np.testing.assert_allclose(got, ref, rtol=1e-12)


@pytest.mark.parametrize("after", [0, 1, 3])
def test_allocation_failure_is_enomem_then_recovers(engine, fresh, after):
    s = synth.protein(304, 800, 14.0)
    p = cs.SolventParams(c1=0.98, c2=0.7)
    ref = cs.debye_solvent_basis(s, Q, p, engine=engine)
    fresh.fail_allocations(after)
    with pytest.raises(Other, match="ENOMEM"):
        cs.debye_solvent_basis(s, Q, p, engine=fresh)
    fresh.fail_allocations(None)
    got = cs.debye_solvent_basis(s, Q, p, engine=fresh)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_non_finite_coordinates_and_occupancies_are_invalid_input(engine, bad):
    s = synth.protein(305, 50, 8.0)
    xyz = s.xyz.copy()
    xyz[17, 1] = bad
    with pytest.raises(InvalidInput, match="finite"):
        cs.debye_intensity(cs.Structure(xyz, s.element), Q, engine=engine)
    occ = np.ones(len(s))
    occ[3] = bad
    with pytest.raises(InvalidInput, match="finite"):
        cs.debye_intensity(cs.Structure(s.xyz, s.element, occ), Q, engine=engine)


@pytest.mark.parametrize("q", [[0.1, np.nan], [0.1, np.inf], [-0.01, 0.1], [0.2, 0.1]])
def test_bad_q_grids_are_invalid_input(engine, q):
    s = synth.protein(306, 40, 8.0)
    with pytest.raises(InvalidInput):
        cs.debye_intensity(s, np.array(q), engine=engine)
    with pytest.raises(InvalidInput):
        cs.multipole_intensity(s, np.array(q), 20, engine=engine)
