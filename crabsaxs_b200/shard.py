"""Debye sums split over several GPUs: one structure's pair work, or an
ensemble's conformers.

One process per GPU, each with its own :class:`~crabsaxs_b200.api.Engine`
and a ``torch.distributed`` process group (NCCL between GPUs, gloo on the
host).  Every rank derives the same split from the same inputs
(:func:`shard_assign`: longest first, each item to the least-loaded shard),
so the split needs no exchange; the only collective is one all-reduce (sum)
of the result, whose parts are zero where a rank did no work:

- one structure: the six basis rows (6 x nq f64, 24 kB at 500 q) or the
  type-pair partials (T(T+1)/2 x nq f64, 60 kB for 5 types at 500 q);
- an ensemble: every conformer's raw pair sums (k blocks of T(T+1)/2 x nq +
  2T f64, about 9 MB for 256 conformers at 300 q), after which every rank
  runs the same weight fit;
- the multipole expansion: each rank's moments over its share of the atoms
  (about 11 MB at 100k atoms and L = 50), summed in place in device memory
  on an NCCL group, after which every rank runs the q pass.

The reference runs on one host and has no counterpart; its loops over q and
over conformers are split over threads (solvent.rs:528, ensemble.rs:244).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _native as N
from .api import (Engine, EnsembleFitter, EnsembleResult, InvalidInput, SolventParams, Structure, debye_partials,
                  debye_solvent_basis, multipole_intensity, multipole_solvent_basis)


def shard_assign(cost, n_shards: int) -> np.ndarray:
    """Owner shard of every work item (crab_shard_assign): items in order,
    each to the shard with the least total cost so far (lowest index among
    equals).  Host-only."""
    c = np.ascontiguousarray(np.asarray(cost, dtype=np.int64))
    owner = np.empty(len(c), dtype=np.int32)
    rc = N.lib.crab_shard_assign(c.ctypes.data_as(C.POINTER(C.c_int64)), len(c), int(n_shards),
                                 owner.ctypes.data_as(N.I32P))
    if rc != N.OK:
        raise InvalidInput(f"shard_assign: {N.STATUS_NAMES.get(rc, rc)}")
    return owner


def _rank_world(group) -> tuple[int, int]:
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def reduce_shards(part: np.ndarray, group=None) -> np.ndarray:
    """Element-wise f64 sum of every rank's ``part`` (same shape on every
    rank), returned on every rank.  On an NCCL group the sum runs on this
    rank's current CUDA device; on gloo on the host."""
    import torch
    import torch.distributed as dist

    a = np.ascontiguousarray(part, dtype=np.float64)
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return a.copy()
    t = torch.from_numpy(a.copy())
    if dist.get_backend(group) == "nccl":
        t = t.to(torch.device("cuda", torch.cuda.current_device()))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def sharded_debye_solvent_basis(structure: Structure, q, params: SolventParams, implicit_hydrogen: bool = True,
                                group=None, engine: Optional[Engine] = None, fp64: bool = False) -> np.ndarray:
    """debye_solvent_basis over the ranks of ``group``: this rank's part on
    its engine's GPU, then the all-reduce.  Every rank returns the whole
    basis."""
    rank, world = _rank_world(group)
    part = debye_solvent_basis(structure, q, params, implicit_hydrogen, engine, fp64, shard=(rank, world))
    return reduce_shards(part, group)


def sharded_debye_partials(xyz, w, types, n_types: int, q, group=None, engine: Optional[Engine] = None,
                           fp64: bool = False):
    """debye_partials over the ranks of ``group``: (pair partials, self sums),
    both whole on every rank."""
    rank, world = _rank_world(group)
    pair, self_ = debye_partials(xyz, w, types, n_types, q, fp64, engine, shard=(rank, world))
    both = reduce_shards(np.concatenate([pair.ravel(), self_]), group)
    return both[: pair.size].reshape(pair.shape), both[pair.size:]


def sharded_ensemble_fit(fitter: EnsembleFitter, group=None) -> EnsembleResult:
    """EnsembleFitter.fit over the ranks of ``group``: each rank's engine sums
    the pairs of the conformers it owns, the all-reduce gathers them, and
    every rank runs the same fit (ensemble.rs:127-232) and returns the same
    result."""
    rank, world = _rank_world(group)
    n_types, part = fitter.partials(shard=(rank, world))
    return fitter.fit_from_partials(n_types, reduce_shards(part, group))


def _in_place_sum(group):
    def fn(a: np.ndarray) -> None:
        a[:] = reduce_shards(a, group)

    return fn


# DLPack description of a device buffer, so that torch can wrap the
# library's moment buffer without a copy (torch.utils.dlpack.from_dlpack).
class _DLDevice(C.Structure):
    _fields_ = [("device_type", C.c_int), ("device_id", C.c_int)]


class _DLDataType(C.Structure):
    _fields_ = [("code", C.c_uint8), ("bits", C.c_uint8), ("lanes", C.c_uint16)]


class _DLTensor(C.Structure):
    _fields_ = [("data", C.c_void_p), ("device", _DLDevice), ("ndim", C.c_int), ("dtype", _DLDataType),
                ("shape", C.POINTER(C.c_int64)), ("strides", C.POINTER(C.c_int64)), ("byte_offset", C.c_uint64)]


class _DLManagedTensor(C.Structure):
    pass


_DL_DELETER = C.CFUNCTYPE(None, C.POINTER(_DLManagedTensor))
_DLManagedTensor._fields_ = [("dl_tensor", _DLTensor), ("manager_ctx", C.c_void_p), ("deleter", _DL_DELETER)]
_DL_KEEP: dict[int, tuple] = {}


@_DL_DELETER
def _dl_delete(ptr):
    _DL_KEEP.pop(C.addressof(ptr.contents), None)


def device_array(ptr: int, count: int, device: int):
    """A torch float64 tensor over `count` doubles of CUDA device memory at
    `ptr` (no copy).  It views memory the library owns: use it only inside the
    callback that received the pointer."""
    import torch
    from torch.utils.dlpack import from_dlpack

    shape = (C.c_int64 * 1)(int(count))
    m = _DLManagedTensor()
    m.dl_tensor = _DLTensor(C.c_void_p(ptr), _DLDevice(2, int(device)), 1, _DLDataType(2, 64, 1), shape, None, 0)
    m.manager_ctx = None
    m.deleter = _dl_delete
    _DL_KEEP[C.addressof(m)] = (m, shape)
    pycapsule_new = C.pythonapi.PyCapsule_New
    pycapsule_new.restype = C.py_object
    pycapsule_new.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
    t = from_dlpack(pycapsule_new(C.addressof(m), b"dltensor", None))
    assert t.device.type == "cuda" and t.dtype == torch.float64
    return t


def _device_sum(group, device: int):
    """In-place all-reduce of the moments in device memory (NCCL)."""
    def fn(ptr: int, count: int) -> None:
        import torch
        import torch.distributed as dist

        t = device_array(ptr, count, device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        torch.cuda.current_stream(device).synchronize()  # the sum is complete before the library goes on

    return fn


def _moment_sum(group, engine: Optional[Engine]):
    """(callback, device mode): device memory and an NCCL all-reduce in place
    on an NCCL group, a host copy otherwise."""
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized() and dist.get_backend(group) == "nccl":
        eng = engine or Engine.default()
        return _device_sum(group, eng.device), True
    return _in_place_sum(group), False


def sharded_multipole_intensity(structure: Structure, q, l_max: int, implicit_hydrogen: bool = True,
                                precision: int = N.PREC_TF32_SPLIT, group=None,
                                engine: Optional[Engine] = None) -> np.ndarray:
    """multipole_intensity over the ranks of ``group``: each rank's moments
    cover its share of the atoms, one all-reduce of the moments (about 11 MB
    at 100k atoms and L = 50), then every rank runs the q pass."""
    rank, world = _rank_world(group)
    if world == 1:
        return multipole_intensity(structure, q, l_max, implicit_hydrogen, precision, engine)
    fn, on_device = _moment_sum(group, engine)
    return multipole_intensity(structure, q, l_max, implicit_hydrogen, precision, engine, shard=(rank, world),
                               moment_sum=fn, device_sums=on_device)


def sharded_multipole_solvent_basis(structure: Structure, q, l_max: int, params: SolventParams,
                                    implicit_hydrogen: bool = True, precision: int = N.PREC_TF32_SPLIT, group=None,
                                    engine: Optional[Engine] = None) -> np.ndarray:
    """multipole_solvent_basis over the ranks of ``group`` (as
    sharded_multipole_intensity)."""
    rank, world = _rank_world(group)
    if world == 1:
        return multipole_solvent_basis(structure, q, l_max, params, implicit_hydrogen, precision, engine)
    fn, on_device = _moment_sum(group, engine)
    return multipole_solvent_basis(structure, q, l_max, params, implicit_hydrogen, precision, engine,
                                   shard=(rank, world), moment_sum=fn, device_sums=on_device)
