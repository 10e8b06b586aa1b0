"""The no-allocation hydration-grid entry point (crab_hydration_grid_adaptive_noalloc).

It exists for callers that cannot allocate device memory through the CUDA
runtime: the caller owns the input and output device buffers (here torch
allocates them for the test; the entry point itself allocates nothing) and
the entry point keeps its temporaries in a fixed file-scope device array.
Its sites must equal, bit for bit, those of crab_hydration_grid_adaptive
(the tolerance every hydration-grid test uses), on consecutive calls that
reuse the shared array.
"""
import ctypes as C

import numpy as np
import pytest

import crabsaxs_b200 as cs
from crabsaxs_b200 import _native as N
from crabsaxs_b200 import synth

pytestmark = pytest.mark.gpu


def _noalloc(xyz, spacing, capacity):
    import torch

    dx = torch.from_numpy(np.ascontiguousarray(xyz)).to("cuda:0")
    ds = torch.zeros((max(capacity, 1), 3), dtype=torch.float64, device="cuda:0")
    m = C.c_int64()
    vol = C.c_double()
    stream = C.c_void_p(torch.cuda.current_stream(0).cuda_stream)
    st = N.lib.crab_hydration_grid_adaptive_noalloc(C.cast(dx.data_ptr(), N.D), xyz.shape[0], spacing, 3.0, 12.0,
                                                    C.cast(ds.data_ptr(), N.D) if capacity > 0 else None, capacity,
                                                    C.byref(m), C.byref(vol), stream)
    return st, m.value, vol.value, ds[: m.value].cpu().numpy() if capacity >= m.value else None


def test_noalloc_grid_matches_allocating_entry_point_on_consecutive_calls(engine):
    # a larger structure first, then a smaller one: the second call must not
    # see the first call's voxels left in the shared scratch
    cases = [(synth.protein(71, 6000, 26.0), 3.0), (synth.protein(72, 900, 14.0), 4.0)]
    for s, spacing in cases:
        ref, ref_vol = cs.hydration_grid_adaptive(s, spacing, engine=engine)
        st, m, vol, sites = _noalloc(s.xyz, spacing, 0)  # size query
        assert st == N.OK and m == len(ref) and vol == ref_vol
        st, m, vol, sites = _noalloc(s.xyz, spacing, m)
        assert st == N.OK and m == len(ref)
        assert np.array_equal(sites, ref)


def test_noalloc_grid_reports_capacity_and_limits(engine):
    s = synth.protein(73, 500, 12.0)
    ref, _ = cs.hydration_grid_adaptive(s, 4.0, engine=engine)
    st, m, _, _ = _noalloc(s.xyz, 4.0, max(len(ref) - 1, 1))
    assert st == N.ECAPACITY and m == len(ref)
    far = np.array([[0.0, 0.0, 0.0], [2000.0, 2000.0, 2000.0]])
    st, _, _, _ = _noalloc(far, 3.0, 0)
    assert st == N.EINVAL
    bad = s.xyz.copy()
    bad[123, 2] = np.nan
    st, m, _, _ = _noalloc(bad, 4.0, 0)
    assert st == N.EINVAL and m == 0
