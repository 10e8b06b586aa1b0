"""Hydration-shell sites from the device are bit-exact against the oracle
(site set and z→y→x order), for the adaptive coarse shell
(solvent.rs:121-223) and the exterior flood-fill shell (solvent.rs:259-401)."""
import numpy as np
import pytest

import crabsaxs_b200 as cs
import oracle as O
from conftest import chain8, helix96, two_atoms_co

pytestmark = pytest.mark.gpu


def _cases():
    yield "co", *two_atoms_co()
    yield "chain8", *chain8()
    yield "helix96", *helix96()
    from crabsaxs_b200 import synth

    s = synth.protein(5, 2000, 18.0)
    yield "synth2000", s.xyz, s.element.astype(np.int32)


@pytest.mark.parametrize("spacing", [8.0, 4.0, 3.0, 2.5])
def test_adaptive_grid_bit_exact(engine, spacing):
    for name, xyz, el in _cases():
        s = cs.Structure(xyz, el)
        got, gv = cs.hydration_grid_adaptive(s, spacing, engine=engine)
        ref, rv = O.adaptive_grid(xyz, spacing)
        assert gv == rv
        assert got.shape == ref.shape, name
        assert np.array_equal(got, ref), name


def test_adaptive_grid_20k_bit_exact(engine):
    from crabsaxs_b200 import synth

    w = synth.DEBYE_20K_SOLVATED
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    got, _ = cs.hydration_grid_adaptive(s, 3.0, engine=engine)
    ref, _ = O.adaptive_grid(s.xyz, 3.0)
    assert np.array_equal(got, ref)
    # shell is clearance..clearance+width(Rg) from the nearest atom
    assert 0.05 < len(got) / s.atom_count < 2.0


def test_adaptive_grid_translation_invariant(engine):  # solvent.rs:740-771
    xyz, el = two_atoms_co()
    shift = np.array([3.17, -8.4, 2.6])
    a, _ = cs.hydration_grid_adaptive(cs.Structure(xyz, el), engine=engine)
    b, _ = cs.hydration_grid_adaptive(cs.Structure(xyz + shift, el), engine=engine)
    assert a.shape == b.shape and np.all(np.linalg.norm(b - a - shift, axis=1) < 1e-12)


def test_adaptive_grid_rejects_bad_spacing(engine):
    xyz, el = two_atoms_co()
    with pytest.raises(cs.InvalidInput):
        cs.hydration_grid_adaptive(cs.Structure(xyz, el), 0.0, engine=engine)


@pytest.mark.parametrize("spacing", [1.0, 1.5])
def test_exterior_grid_bit_exact(engine, spacing):
    for name, xyz, el in _cases():
        s = cs.Structure(xyz, el)
        got, gv = cs.hydration_grid_exterior(s, spacing, engine=engine)
        ref, rv = O.exterior_grid(xyz, el, spacing)
        assert gv == rv
        assert got.shape == ref.shape, name
        assert np.array_equal(got, ref), name


def test_exterior_grid_single_atom_bounds(engine):  # solvent.rs:688-705
    xyz = np.array([[-1.0, 0.0, 0.0]])
    got, _ = cs.hydration_grid_exterior(cs.Structure(xyz, [1]), engine=engine)
    d = np.linalg.norm(got - xyz[0], axis=1)
    assert len(got) > 0 and np.all(d > 1.7 + 1.4) and np.all(d <= 1.7 + 1.4 + 3.0 + 1e-12)


def test_exterior_grid_limit(engine):
    xyz = np.array([[0.0, 0.0, 0.0], [700.0, 700.0, 700.0]])
    with pytest.raises(cs.InvalidInput):
        cs.hydration_grid_exterior(cs.Structure(xyz, [1, 1]), 0.1, engine=engine)


def _serpentine(plates=20, side=40.0, pitch=10.0, step=1.5, gap=8.0):
    """A closed column, open at the top, divided by plates that leave a gap on
    alternating sides: the exterior reaches the lower levels only through a
    zig-zag corridor (one more sweep round per level), and the lowest plate
    has no gap, so the chamber under it is a sealed cavity (not exterior)."""
    g = np.arange(0.0, side + 1e-9, step)
    h = np.arange(0.0, plates * pitch + 1e-9, step)
    a, z = np.meshgrid(g, h, indexing="ij")
    a, z = a.ravel(), z.ravel()
    zero, full = np.zeros_like(a), np.full_like(a, side)
    walls = [np.stack(c, 1) for c in ((a, zero, z), (a, full, z), (zero, a, z), (full, a, z))]
    u, v = np.meshgrid(g, g, indexing="ij")
    u, v = u.ravel(), v.ravel()
    layers = [np.stack([u, v, np.zeros_like(u)], 1)]
    for k in range(1, plates):
        keep = np.ones_like(u, bool)
        if k > 1:
            keep = u >= gap if k % 2 == 0 else u <= side - gap
        layers.append(np.stack([u[keep], v[keep], np.full(keep.sum(), k * pitch)], 1))
    return np.unique(np.round(np.concatenate(walls + layers), 6), axis=0)


def test_exterior_grid_many_sweep_rounds(engine):
    """About 20 sweep rounds (several batches between host reads of the change
    flag) and a sealed cavity: sites bit-exact against the oracle's BFS."""
    xyz = _serpentine()
    el = np.full(len(xyz), 1, np.int32)
    got, gv = cs.hydration_grid_exterior(cs.Structure(xyz, el), 1.0, engine=engine)
    ref, rv = O.exterior_grid(xyz, el, 1.0)
    assert gv == rv and got.shape == ref.shape and np.array_equal(got, ref)
    # no site lies in the sealed chamber under the lowest plate; the chamber
    # above it, reached through the corridor, has sites
    def chamber(z0):
        return (got[:, 2] > z0 + 3.2) & (got[:, 2] < z0 + 6.8) & np.all((got[:, :2] > 3.2) & (got[:, :2] < 36.8), 1)

    assert not chamber(0.0).any() and chamber(10.0).any()


def test_exterior_grid_20k_bit_exact(engine):
    """20,000 atoms at 1 Å: a 1.3-million-voxel box filled in about 11 rounds."""
    from crabsaxs_b200 import synth

    w = synth.DEBYE_20K_SOLVATED
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    got, gv = cs.hydration_grid_exterior(s, engine=engine)
    ref, rv = O.exterior_grid(s.xyz, s.element.astype(np.int32))
    assert gv == rv and np.array_equal(got, ref)


def _grid_call(engine, kind, s, options, capacity):
    import ctypes as C

    from crabsaxs_b200 import _native as N

    fn = N.lib.crab_hydration_grid_adaptive if kind == "adaptive" else N.lib.crab_hydration_grid_exterior
    m, vol = C.c_int64(), C.c_double()
    out = np.full((max(capacity, 1), 3), np.nan)
    rc = fn(engine.handle, s.handle(engine), *options, out.ctypes.data_as(C.POINTER(C.c_double)) if capacity else None,
            capacity, C.byref(m), C.byref(vol))
    return rc, m.value, out[: m.value] if capacity else None


def test_grid_size_query_then_fill_with_other_arguments(engine):
    """The size query keeps its result for the fill call that follows with
    the same structure and options; any other fill builds its own grid."""
    from crabsaxs_b200 import _native as N

    xyz, el = helix96()
    s1, s2 = cs.Structure(xyz, el), cs.Structure(xyz + np.array([0.3, 0.0, 0.0]), el)
    ref = {
        ("exterior", 1): O.exterior_grid(xyz, np.asarray(el, np.int32), 1.0)[0],
        ("exterior", 2): O.exterior_grid(xyz + np.array([0.3, 0.0, 0.0]), np.asarray(el, np.int32), 1.0)[0],
        ("exterior15", 1): O.exterior_grid(xyz, np.asarray(el, np.int32), 1.5)[0],
        ("adaptive", 1): O.adaptive_grid(xyz, 1.0, 1.4, 3.0)[0],
    }
    ext1, ext15 = (1.0, 1.4, 3.0), (1.5, 1.4, 3.0)
    big = 10 * max(len(r) for r in ref.values())
    # query one structure, fill another
    assert _grid_call(engine, "exterior", s1, ext1, 0)[0] == N.OK
    rc, m, got = _grid_call(engine, "exterior", s2, ext1, big)
    assert rc == N.OK and np.array_equal(got, ref[("exterior", 2)])
    # query with one spacing, fill with another
    assert _grid_call(engine, "exterior", s1, ext1, 0)[0] == N.OK
    rc, m, got = _grid_call(engine, "exterior", s1, ext15, big)
    assert rc == N.OK and np.array_equal(got, ref[("exterior15", 1)])
    # the same numbers for the other grid kind
    assert _grid_call(engine, "exterior", s1, ext1, 0)[0] == N.OK
    rc, m, got = _grid_call(engine, "adaptive", s1, (1.0, 1.4, 3.0), big)
    assert rc == N.OK and np.array_equal(got, ref[("adaptive", 1)])
    # too small a buffer leaves the query's result for the retry
    rc, m, _ = _grid_call(engine, "exterior", s1, ext1, 0)
    assert rc == N.OK and m == len(ref[("exterior", 1)])
    rc, m2, _ = _grid_call(engine, "exterior", s1, ext1, m - 1)
    assert rc == N.ECAPACITY and m2 == m
    rc, m3, got = _grid_call(engine, "exterior", s1, ext1, m)
    assert rc == N.OK and m3 == m and np.array_equal(got, ref[("exterior", 1)])
    # another grid built between the query and the fill (a calculation with
    # adaptive hydration reuses the context's device grid slots)
    assert _grid_call(engine, "exterior", s1, ext1, 0)[0] == N.OK
    sol = cs.SolventParams(c2=0.5, hydration_model=cs.HydrationModel.AdaptiveGrid)
    cs.compute_curve(s2, np.linspace(0.01, 0.3, 8), cs.ComputeOptions(method=cs.ScatteringMethod.Debye, solvent=sol),
                     engine=engine)
    rc, _, got = _grid_call(engine, "exterior", s1, ext1, big)
    assert rc == N.OK and np.array_equal(got, ref[("exterior", 1)])
    # a fill without a query, twice
    for _ in range(2):
        rc, _, got = _grid_call(engine, "exterior", s1, ext1, big)
        assert rc == N.OK and np.array_equal(got, ref[("exterior", 1)])


def _corners(half):
    return np.array([[x, y, z] for x in (-half, half) for y in (-half, half) for z in (-half, half)], float)


def _workspace(engine):
    import ctypes as C

    from crabsaxs_b200 import _native as N

    b = C.c_int64()
    assert N.lib.crab_ctx_workspace_bytes(engine.handle, C.byref(b)) == N.OK
    return b.value


def test_exterior_grid_large_box(engine):
    """Eight atoms at the corners of a 400 Å cube: a 71-million-voxel box at
    1 Å (the limit is 250 million), bit-exact against the oracle's BFS."""
    xyz = _corners(200.0) + np.array([0.31, -0.17, 0.05])
    el = np.full(8, 1, np.int32)
    got, gv = cs.hydration_grid_exterior(cs.Structure(xyz, el), 1.0, engine=engine)
    ref, rv = O.exterior_grid(xyz, el, 1.0)
    assert gv == rv and got.shape == ref.shape and np.array_equal(got, ref)


def test_adaptive_grid_large_box_releases_its_masks(engine):
    """A 321-million-voxel adaptive box (corners of a 660 Å cube, 1 Å):
    bit-exact, and its two 321 MB voxel masks leave the context's buffer
    pool when the call returns (grid slots above 256 MB are not kept)."""
    xyz = _corners(330.0)
    before = _workspace(engine)
    got, gv = cs.hydration_grid_adaptive(cs.Structure(xyz, np.full(8, 1)), 1.0, engine=engine)
    after = _workspace(engine)
    ref, rv = O.adaptive_grid(xyz, 1.0)
    assert gv == rv and got.shape == ref.shape and np.array_equal(got, ref)
    assert after - before < (64 << 20)
