"""The Debye sums of one structure split into shards (one per GPU in a
multi-GPU run) add up to the unsplit sums.  Here every shard runs on the one
GPU in turn, as independent launches.  Every work item is computed exactly
as in the unsplit run; only the order of the f64 additions across items
differs, hence 1e-12 of the largest entry."""
import numpy as np
import pytest

import crabsaxs_b200 as cs
from crabsaxs_b200 import _native as N
from crabsaxs_b200 import synth

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _close(a, b):
    return np.max(np.abs(a - b)) <= RTOL * np.max(np.abs(b))


@pytest.mark.parametrize("model", [cs.HydrationModel.Analytic, cs.HydrationModel.AdaptiveGrid])
@pytest.mark.parametrize("fp64", [False, True])
def test_basis_shards_sum_to_the_basis(engine, model, fp64):
    s = synth.protein(31, 2500 if fp64 else 6000, 16.0 if fp64 else 22.0)
    q = np.linspace(0.0, 0.5, 101)  # q = 0 included: its exact sums come from shard 0 only
    sp = cs.SolventParams(c1=1.02, c2=0.7, hydration_model=model, hydration_grid_spacing_angstrom=3.0)
    whole = cs.debye_solvent_basis(s, q, sp, engine=engine, fp64=fp64)
    for n in (2, 3, 5):
        parts = [cs.debye_solvent_basis(s, q, sp, engine=engine, fp64=fp64, shard=(k, n)) for k in range(n)]
        assert _close(sum(parts), whole), n
        assert all(np.any(p != 0.0) for p in parts)


def test_partials_shards_and_self_sums(engine):
    s = synth.protein(32, 3000, 18.0)
    w = np.random.default_rng(3).uniform(1.0, 9.0, len(s.xyz))
    t = s.element.astype(np.int32) % 4
    q = np.linspace(0.01, 0.45, 300)
    pair, self_ = cs.debye_partials(s.xyz, w, t, 4, q, engine=engine)
    for n in (2, 4):
        got = [cs.debye_partials(s.xyz, w, t, 4, q, engine=engine, shard=(k, n)) for k in range(n)]
        assert _close(sum(g[0] for g in got), pair)
        assert np.array_equal(got[0][1], self_) and all(not g[1].any() for g in got[1:])


def test_lattice_plan_shards_sum_to_the_plan(engine):
    """The sharded pair plan of the bench's multi-GPU split: the shards'
    partials (read back after one run each) add up to the unsplit plan's."""
    import ctypes as C

    s = synth.protein(39, 3000, 18.0)
    sites, _ = cs.hydration_grid_adaptive(s, 3.0, engine=engine)
    el = np.unique(s.element)
    xyz = np.ascontiguousarray(np.concatenate([s.xyz, sites]))
    w = np.ascontiguousarray(np.concatenate([s.occupancy, np.ones(len(sites))]))
    t = np.ascontiguousarray(np.concatenate([np.searchsorted(el, s.element), np.full(len(sites), len(el))]).astype(np.int32))
    T = len(el) + 1
    cells = np.ascontiguousarray(np.rint((sites - sites.min(axis=0)) / 3.0).astype(np.int32))
    q = np.ascontiguousarray(np.linspace(0.0, 0.5, 120))

    def run(shard, n):
        plan = C.c_void_p()
        engine.check(N.lib.crab_pair_plan_create_lattice_shard(
            engine.handle, xyz.ctypes.data_as(N.D), w.ctypes.data_as(N.D), t.ctypes.data_as(N.I32P), len(w), T,
            q.ctypes.data_as(N.D), len(q), cells.ctypes.data_as(N.I32P), len(sites), 3.0, shard, n, C.byref(plan)))
        try:
            engine.check(N.lib.crab_pair_plan_run(engine.handle, plan, 1, 0, None))
            out = np.empty((T * (T + 1) // 2, len(q)))
            self_ = np.empty(T)
            engine.check(N.lib.crab_pair_plan_read(engine.handle, plan, out.ctypes.data_as(N.D),
                                                   self_.ctypes.data_as(N.D)))
            return out, self_
        finally:
            N.lib.crab_pair_plan_destroy(plan)

    whole, whole_self = run(0, 1)
    for n in (2, 3, 8):
        parts = [run(k, n) for k in range(n)]
        assert _close(sum(p[0] for p in parts), whole), n
        assert np.array_equal(parts[0][1], whole_self) and all(not p[1].any() for p in parts[1:])
    bad = C.c_void_p()
    assert N.lib.crab_pair_plan_create_lattice_shard(engine.handle, xyz.ctypes.data_as(N.D), w.ctypes.data_as(N.D),
                                                     t.ctypes.data_as(N.I32P), len(w), T, q.ctypes.data_as(N.D),
                                                     len(q), cells.ctypes.data_as(N.I32P), len(sites), 3.0, 2, 2,
                                                     C.byref(bad)) == N.EINVAL


def test_more_shards_than_work_items(engine):
    """90 atoms: one tile per atom type (at most 4) and one q block, so at
    most 10 tile-pair work items; the other shards return zeros and the sum is
    still the whole."""
    s = synth.protein(33, 90, 8.0)
    q = np.linspace(0.001, 0.3, 40)
    sp = cs.SolventParams()
    whole = cs.debye_solvent_basis(s, q, sp, engine=engine)
    parts = [cs.debye_solvent_basis(s, q, sp, engine=engine, shard=(k, 16)) for k in range(16)]
    assert _close(sum(parts), whole)
    assert sum(1 for p in parts if not p.any()) >= 6


def test_invalid_shard_arguments(engine):
    s = synth.protein(34, 200, 9.0)
    q = np.linspace(0.01, 0.3, 10)
    for shard in ((0, 0), (2, 2), (-1, 3)):
        with pytest.raises(cs.InvalidInput):
            cs.debye_solvent_basis(s, q, cs.SolventParams(), engine=engine, shard=shard)
        with pytest.raises(cs.InvalidInput):
            cs.debye_partials(s.xyz, np.ones(len(s.xyz)), np.zeros(len(s.xyz), np.int32), 1, q, engine=engine,
                              shard=shard)


def test_sharded_basis_without_a_process_group_is_the_basis(engine):
    from crabsaxs_b200 import shard as S

    s = synth.protein(35, 1500, 14.0)
    q = np.linspace(0.001, 0.5, 64)
    sp = cs.SolventParams(c2=0.3)
    whole = cs.debye_solvent_basis(s, q, sp, engine=engine)
    assert _close(S.sharded_debye_solvent_basis(s, q, sp, engine=engine), whole)


def _ensemble(k, seed):
    sizes = np.random.default_rng(seed).integers(150, 1500, size=k)
    return [synth.protein(700 + i, int(n), 6.0 + 0.02 * n) for i, n in enumerate(sizes)]


def _fitter(engine, confs, q, curve_index, hidden, **opts):
    fo = cs.FitOptions(method=cs.ScatteringMethod.Debye)
    curves = cs.ensemble_curves(confs, q, cs.SolventParams(), cs.solvent_candidates(fo), engine=engine)
    rng = np.random.default_rng(len(confs))
    w = rng.dirichlet(np.ones(len(hidden)))
    clean = (w[:, None] * curves[curve_index][hidden]).sum(axis=0)
    sigma = 0.01 * clean
    ex = cs.ExperimentalCurve(q, clean + sigma * rng.normal(size=clean.shape), sigma)
    names = [f"c{i}" for i in range(len(confs))]
    return cs.EnsembleFitter(confs, names, ex, cs.EnsembleOptions(fit=fo, **opts), engine=engine)


def test_ensemble_partials_shards_gather_every_conformer(engine):
    """Each conformer's pair sums come from exactly one shard (split by N²,
    longest first), and the shards' buffers sum to the unsplit buffer."""
    confs = _ensemble(14, 5)
    fitter = _fitter(engine, confs, np.linspace(0.005, 0.45, 90), 3, [1, 4])
    T, whole = fitter.partials()
    whole = whole.reshape(len(confs), -1)
    n2 = np.array([c.atom_count ** 2 for c in confs], dtype=float)
    for n in (2, 3, 5):
        parts = [fitter.partials(shard=(k, n)) for k in range(n)]
        assert all(p[0] == T for p in parts)
        blocks = np.stack([p[1].reshape(len(confs), -1) for p in parts])
        owned = np.abs(blocks).sum(-1) > 0
        assert np.all(owned.sum(0) == 1)
        assert _close(blocks.sum(0), whole)
        loads = (owned * n2[None, :]).sum(1)
        assert loads.max() <= n2.sum() / n + n2.max()


def test_ensemble_fit_from_gathered_partials_matches_fit(engine):
    """The fit from the summed shard buffers (what every rank runs after the
    all-reduce) is EnsembleFitter.fit's: pruning, weights, best candidate and
    the bootstrap."""
    confs = _ensemble(10, 21)
    fitter = _fitter(engine, confs, np.linspace(0.005, 0.45, 80), 6, [2, 5], min_weight=0.02, bootstrap=3)
    ref = fitter.fit()
    for n in (1, 3):
        parts = [fitter.partials(shard=(k, n)) for k in range(n)]
        got = fitter.fit_from_partials(parts[0][0], sum(p[1] for p in parts))
        assert got.conformers == ref.conformers
        assert (got.params.c1, got.params.c2) == (ref.params.c1, ref.params.c2)
        np.testing.assert_allclose(got.weights, ref.weights, atol=1e-9)
        assert got.reduced_chi2 == pytest.approx(ref.reduced_chi2, rel=1e-9)
        np.testing.assert_allclose(got.fitted_curve, ref.fitted_curve, rtol=1e-9)
        np.testing.assert_allclose(got.bootstrap_reduced_chi2, ref.bootstrap_reduced_chi2, rtol=1e-7)


def test_ensemble_fit_from_partials_rejects_a_mismatched_buffer(engine):
    confs = _ensemble(4, 8)
    fitter = _fitter(engine, confs, np.linspace(0.01, 0.4, 30), 0, [0, 1])
    T, buf = fitter.partials()
    with pytest.raises(cs.InvalidInput):
        fitter.fit_from_partials(T, buf[:-1])
    with pytest.raises(cs.InvalidInput):
        fitter.fit_from_partials(T + 1, np.zeros(len(confs) * ((T + 1) * (T + 2) // 2 * 30 + 2 * (T + 1))))


class _Stop(Exception):
    pass


def _moments_of_every_shard(call, n):
    """Each shard's moments, taken in its sum callback, which then raises:
    the library call ends with an error and the exception comes back."""
    got = []
    for k in range(n):
        def grab(a):
            got.append(a.copy())
            raise _Stop()

        with pytest.raises(_Stop):
            call(shard=(k, n), moment_sum=grab)
    return got


def _sharded_results(call, n, total):
    def put(a):
        a[:] = total

    return [call(shard=(k, n), moment_sum=put) for k in range(n)]


@pytest.mark.parametrize("precision,rtol", [(N.PREC_FP64, 1e-12), (N.PREC_TF32_SPLIT, 2e-6)])
def test_multipole_moments_of_the_shards_sum_to_the_whole(engine, precision, rtol):
    """Moments are linear in the atoms: the shards' moments summed (the
    all-reduce) give the unsplit curve on every rank.  FP64 differs only in
    the order of additions; the TF32 split groups its FP32 accumulations
    differently, within its own 5e-7 error."""
    s = synth.protein(36, 5000, 24.0)
    q = np.linspace(0.001, 0.5, 120)

    def call(**kw):
        return cs.multipole_intensity(s, q, 30, precision=precision, engine=engine, **kw)

    whole = call()
    for n in (2, 3):
        parts = _moments_of_every_shard(call, n)
        assert len({p.size for p in parts}) == 1 and all(np.any(p != 0.0) for p in parts)
        for got in _sharded_results(call, n, sum(parts)):
            assert np.max(np.abs(got - whole)) <= rtol * np.max(whole)


@pytest.mark.parametrize("precision", [N.PREC_FP64, N.PREC_BF16_SPLIT])
def test_multipole_moments_summed_in_device_memory(engine, precision):
    """crab_ctx_set_device_sums: the callback gets the moments in device
    memory (wrapped for torch without a copy by shard.device_array), sums
    them in place, and the curves are those of the host-memory path."""
    import torch

    from crabsaxs_b200 import shard as S

    s = synth.protein(38, 4000, 22.0)
    q = np.linspace(0.001, 0.5, 100)

    def call(**kw):
        return cs.multipole_intensity(s, q, 30, precision=precision, engine=engine, **kw)

    host_parts = _moments_of_every_shard(call, 2)
    dev_parts = []
    for k in range(2):
        def grab(ptr, count):
            dev_parts.append(S.device_array(ptr, count, engine.device).cpu().numpy())
            raise _Stop()

        with pytest.raises(_Stop):
            call(shard=(k, 2), moment_sum=grab, device_sums=True)
    for h, d in zip(host_parts, dev_parts):
        assert np.array_equal(h, d)
    total = torch.from_numpy(sum(host_parts)).to(f"cuda:{engine.device}")

    def put(ptr, count):
        S.device_array(ptr, count, engine.device).copy_(total)
        torch.cuda.synchronize(engine.device)

    host = _sharded_results(call, 2, sum(host_parts))
    for k in range(2):
        got = call(shard=(k, 2), moment_sum=put, device_sums=True)
        assert np.array_equal(got, host[k])
    # the option is per call: the next sharded call without it gets host memory again
    again = _sharded_results(call, 2, sum(host_parts))
    assert np.array_equal(again[0], host[0])


def test_multipole_solvent_basis_shards_with_grid_sites(engine):
    """The hydration sites are part of the typed list the shards divide."""
    s = synth.protein(37, 3000, 20.0)
    q = np.linspace(0.001, 0.4, 80)
    sp = cs.SolventParams(c1=1.01, c2=0.8, hydration_model=cs.HydrationModel.AdaptiveGrid,
                          hydration_grid_spacing_angstrom=3.0)

    def call(**kw):
        return cs.multipole_solvent_basis(s, q, 25, sp, precision=N.PREC_FP64, engine=engine, **kw)

    whole = call()
    parts = _moments_of_every_shard(call, 4)
    for got in _sharded_results(call, 4, sum(parts)):
        assert np.max(np.abs(got - whole)) <= 1e-12 * np.max(np.abs(whole))


def test_multipole_more_shards_than_atoms(engine):
    s = cs.Structure(np.array([[0.0, 0.0, 0.0], [3.0, 0.5, -1.0], [-2.0, 2.5, 1.0]]), np.array([1, 2, 3]))
    q = np.linspace(0.01, 0.5, 30)

    def call(**kw):
        return cs.multipole_intensity(s, q, 12, precision=N.PREC_FP64, engine=engine, **kw)

    whole = call()
    parts = _moments_of_every_shard(call, 5)
    assert sum(1 for p in parts if not p.any()) == 2
    for got in _sharded_results(call, 5, sum(parts)):
        assert np.max(np.abs(got - whole)) <= 1e-12 * np.max(whole)


def test_multipole_shard_needs_a_sum(engine):
    """A NULL sum callback (N.SUM_FN()) is refused for two or more shards."""
    s = synth.protein(38, 300, 9.0)
    q = np.linspace(0.01, 0.3, 10)
    out = np.empty(10)
    rc = N.lib.crab_multipole_intensity_shard(engine.handle, s.handle(engine), q.ctypes.data_as(N.D), 10, 10, 1,
                                              N.PREC_FP64, 0, 2, N.SUM_FN(), None, out.ctypes.data_as(N.D))
    assert rc == N.EINVAL
    # one shard needs no sum: the unsplit call
    rc = N.lib.crab_multipole_intensity_shard(engine.handle, s.handle(engine), q.ctypes.data_as(N.D), 10, 10, 1,
                                              N.PREC_FP64, 0, 1, N.SUM_FN(), None, out.ctypes.data_as(N.D))
    assert rc == N.OK and np.allclose(out, cs.multipole_intensity(s, q, 10, precision=N.PREC_FP64, engine=engine),
                                      rtol=1e-12)
