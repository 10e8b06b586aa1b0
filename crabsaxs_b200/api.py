"""Python mirror of crabSAXS's public calculation API over the C ABI.

Names, fields, defaults and error behaviour follow the reference crate:
``ProfileCalculator`` / ``SaxsFitter`` / ``SaxsScorer`` / ``compare_curves``
(src/analysis.rs), ``EnsembleFitter`` (src/ensemble.rs), ``reweight_curves``
(src/reweight.rs), ``ComputeOptions`` (src/scattering.rs:28-47),
``SolventParams`` (src/solvent.rs:27-50), ``FitOptions`` (src/fit.rs:49-82),
``Atom`` / ``Structure`` / ``Element`` (src/structure.rs:88-165) and
``SaxsError`` (src/error.rs).  Every computation runs in libcrabsaxs_b200 on
the GPU; this module only marshals arrays.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import enum
import math
import threading
from pathlib import Path
from dataclasses import dataclass, field, replace
from typing import Optional, Sequence

import numpy as np

from . import _native as N


# ---------------------------------------------------------------- errors (error.rs)
class SaxsError(Exception):
    """Base of every error raised by the engine."""


class InvalidInput(SaxsError):
    pass


class FitDidNotConverge(SaxsError):
    pass


class StructureParse(SaxsError):
    """error.rs: failed to parse structure file."""


class UnsupportedElement(SaxsError):
    """error.rs: unsupported element."""


class Other(SaxsError):
    pass


def _raise(status: int, ctx: Optional[C.c_void_p] = None) -> None:
    if status == N.OK:
        return
    msg = N.lib.crab_ctx_last_error(ctx).decode() if ctx else ""
    name = N.STATUS_NAMES.get(status, str(status))
    if status == N.EINVAL:
        raise InvalidInput(msg or name)
    if status == N.ENOTCONV:
        raise FitDidNotConverge(msg or name)
    if status == N.EPARSE:
        raise StructureParse(msg or name)
    if status == N.EELEMENT:
        raise UnsupportedElement(msg or name)
    if status == N.EIO:
        raise OSError(msg or name)
    raise Other(f"{name}: {msg}")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(N.D)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


# ---------------------------------------------------------------- engine context
class Engine:
    """One device context (stream, workspace, statistics) on one GPU."""

    _default: dict[int, "Engine"] = {}
    _lock = threading.Lock()

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = N.lib.crab_ctx_create(device, C.byref(h))
        if st != N.OK:
            raise Other(f"cannot create a CUDA context on device {device}: {N.STATUS_NAMES.get(st, st)}")
        self.handle = h
        self.device = device

    @classmethod
    def default(cls, device: int = 0) -> "Engine":
        with cls._lock:
            if device not in cls._default:
                cls._default[device] = Engine(device)
            return cls._default[device]

    def check(self, status: int) -> None:
        _raise(status, self.handle)

    def stats(self) -> tuple[int, float, float]:
        launches = C.c_int64()
        ms = C.c_double()
        pq = C.c_double()
        N.lib.crab_ctx_stats(self.handle, C.byref(launches), C.byref(ms), C.byref(pq))
        return launches.value, ms.value, pq.value

    def reset_stats(self) -> None:
        N.lib.crab_ctx_reset_stats(self.handle)

    def set_wait_budget(self, iterations: int | None) -> None:
        """Iteration budget of the kernels' bounded device-side waits (None:
        the defaults; 0: the first wait gives up and the call raises Other
        with status CRAB_ETIMEOUT).  For tests of the error paths."""
        self.check(N.lib.crab_ctx_set_wait_budget(self.handle, -1 if iterations is None else int(iterations)))

    def fail_allocations(self, after: int | None) -> None:
        """Let `after` more device or pinned host allocations of this context
        succeed and fail the rest with CRAB_ENOMEM (None: off).  For tests."""
        self.check(N.lib.crab_ctx_fail_allocations(self.handle, -1 if after is None else int(after)))

    def close(self) -> None:
        if self.handle:
            N.lib.crab_ctx_destroy(self.handle)
            self.handle = None


# ---------------------------------------------------------------- structure (structure.rs)
class Element(enum.IntEnum):
    H = 0
    C = 1
    N = 2
    O = 3
    S = 4
    P = 5
    Na = 6
    Mg = 7
    Cl = 8
    Ca = 9
    Fe = 10
    Zn = 11
    K = 12
    I = 13
    Other = 14

    @classmethod
    def from_symbol(cls, symbol: str) -> "Element":
        s = symbol.strip().upper()
        table = {"H": cls.H, "D": cls.H, "C": cls.C, "N": cls.N, "O": cls.O, "S": cls.S, "P": cls.P, "NA": cls.Na,
                 "MG": cls.Mg, "CL": cls.Cl, "CA": cls.Ca, "FE": cls.Fe, "ZN": cls.Zn, "K": cls.K, "I": cls.I}
        return table.get(s, cls.Other)


@dataclass
class Atom:
    pos: tuple
    element: Element
    occupancy: float = 1.0
    is_hetatm: bool = False
    atom_name: str = ""
    residue_name: str = ""
    chain_id: str = "A"
    residue_id: int = 0


def united_atom_group(residue_name: str, atom_name: str) -> int:
    """formfactor.rs:357-417 typing, -1 when not a standard united atom."""
    return int(N.lib.crab_united_atom_group(residue_name.encode(), atom_name.encode()))


def _text_field(which: int, name: str):
    """Per-atom strings of a parsed structure (atom names, residue names,
    chain ids): kept as the library's newline-joined bytes and split into a
    list on first use."""

    def get(self):
        v = self.__dict__.get(name)
        if v is None:
            raw = self.__dict__.get("_text_raw")
            if raw is None:
                raise AttributeError(name)
            v = raw[which].decode().split("\n")[: self.atom_count]
            self.__dict__[name] = v
        return v

    def put(self, value):
        self.__dict__[name] = value

    return property(get, put)


class Structure:
    """Atoms as arrays (xyz f64 [n,3], element, occupancy, united-atom group).

    The device copy is created lazily per engine and cached.
    """

    atom_name = _text_field(0, "atom_name")
    residue_name = _text_field(1, "residue_name")
    chain_id = _text_field(2, "chain_id")

    def __init__(self, xyz, element, occupancy=None, group=None):
        self.xyz = _f64(xyz).reshape(-1, 3)
        n = self.xyz.shape[0]
        self.element = np.ascontiguousarray(np.asarray(element, dtype=np.int8).reshape(n))
        self.occupancy = _f64(np.ones(n) if occupancy is None else occupancy).reshape(n)
        self.group = np.ascontiguousarray(
            np.full(n, -1, dtype=np.int8) if group is None else np.asarray(group, dtype=np.int8).reshape(n))
        self._handles: dict[int, C.c_void_p] = {}

    @classmethod
    def from_atoms(cls, atoms: Sequence[Atom]) -> "Structure":
        xyz = np.array([a.pos for a in atoms], dtype=np.float64).reshape(-1, 3)
        el = np.array([int(a.element) for a in atoms], dtype=np.int8)
        occ = np.array([a.occupancy for a in atoms], dtype=np.float64)
        grp = np.array([united_atom_group(a.residue_name, a.atom_name) for a in atoms], dtype=np.int8)
        return cls(xyz, el, occ, grp)

    @classmethod
    def from_pdb_file(cls, path, options: Optional["ParseOptions"] = None) -> "Structure":
        """structure.rs:205-207 / 209-327: PDB or mmCIF by extension."""
        p = C.c_void_p()
        o = (options or ParseOptions()).to_c()
        _parse_check(N.lib.crab_read_structure_file(str(path).encode(), C.byref(o), C.byref(p)))
        return cls._from_parsed(p)

    from_pdb_file_with_options = from_pdb_file

    @classmethod
    def from_text(cls, text, options: Optional["ParseOptions"] = None, fmt: int = N.FORMAT_AUTO) -> "Structure":
        """The same on PDB or mmCIF text (format detected unless given)."""
        data = text.encode() if isinstance(text, str) else bytes(text)
        p = C.c_void_p()
        o = (options or ParseOptions()).to_c()
        _parse_check(N.lib.crab_parse_structure(data, len(data), fmt, C.byref(o), C.byref(p)))
        return cls._from_parsed(p)

    @classmethod
    def from_pdb_file_models_with_options(cls, path, options: Optional["ParseOptions"] = None) -> list["Structure"]:
        """structure.rs:330-345: every model of the file, in order."""
        data = Path(path).read_bytes()
        fmt = N.FORMAT_MMCIF if str(path).lower().endswith((".cif", ".mmcif")) else N.FORMAT_PDB
        n = C.c_int32()
        _parse_check(N.lib.crab_parse_model_count(data, len(data), fmt, C.byref(n)))
        base = options or ParseOptions()
        out = []
        for k in range(max(n.value, 1)):
            o = dataclasses.replace(base, model_index=k)
            out.append(cls.from_text(data, o, fmt))
        return out

    @classmethod
    def _from_parsed(cls, p: C.c_void_p) -> "Structure":
        try:
            n = int(N.lib.crab_parsed_atom_count(p))
            xyz = np.empty((n, 3))
            occ = np.empty(n)
            el = np.empty(n, dtype=np.int8)
            grp = np.empty(n, dtype=np.int8)
            het = np.empty(n, dtype=np.int8)
            rid = np.empty(n, dtype=np.int64)
            N.lib.crab_parsed_arrays(p, _dp(xyz), _dp(occ), el.ctypes.data_as(N.I8P), grp.ctypes.data_as(N.I8P),
                                     het.ctypes.data_as(N.I8P), rid.ctypes.data_as(C.POINTER(C.c_int64)))
            s = cls(xyz, el, occ, grp)
            s.is_hetatm = het.astype(bool)
            s.residue_id = rid
            s._text_raw = [_parsed_bytes(p, k) for k in range(3)]
            return s
        finally:
            N.lib.crab_parsed_destroy(p)

    @property
    def atoms(self) -> list[Atom]:
        """Per-atom records (structure.rs:151-160); names only for parsed structures."""
        n = self.atom_count
        names = getattr(self, "atom_name", [""] * n)
        res = getattr(self, "residue_name", [""] * n)
        chains = getattr(self, "chain_id", [""] * n)
        het = getattr(self, "is_hetatm", np.zeros(n, dtype=bool))
        rid = getattr(self, "residue_id", np.zeros(n, dtype=np.int64))
        return [Atom(tuple(self.xyz[i]), Element(int(self.element[i])), float(self.occupancy[i]), bool(het[i]),
                     names[i], res[i], chains[i], int(rid[i])) for i in range(n)]

    @property
    def atom_count(self) -> int:
        return int(self.xyz.shape[0])

    def __len__(self) -> int:
        return self.atom_count

    def handle(self, engine: Engine) -> C.c_void_p:
        key = id(engine)
        h = self._handles.get(key)
        if h is None:
            h = C.c_void_p()
            engine.check(N.lib.crab_structure_create(engine.handle, _dp(self.xyz), _dp(self.occupancy),
                                                     self.element.ctypes.data_as(N.I8P),
                                                     self.group.ctypes.data_as(N.I8P), self.atom_count, C.byref(h)))
            self._handles[key] = h
        return h

    def release(self) -> None:
        for h in self._handles.values():
            N.lib.crab_structure_destroy(h)
        self._handles.clear()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class AltlocPolicy(enum.IntEnum):
    """structure.rs:14-21."""
    Highest = N.ALTLOC_HIGHEST
    First = N.ALTLOC_FIRST
    All = N.ALTLOC_ALL


class OccupancyPolicy(enum.IntEnum):
    """structure.rs:167-175."""
    Reported = N.OCC_REPORTED
    SelectedConformerFull = N.OCC_SELECTED_FULL


@dataclass
class ParseOptions:
    """structure.rs:177-201 with its defaults."""
    include_hetatm: bool = False
    include_waters: bool = False
    include_glycans: bool = True
    model_index: int = 0
    allow_unknown_elements: bool = False
    occupancy_policy: OccupancyPolicy = OccupancyPolicy.Reported
    altloc_policy: AltlocPolicy = AltlocPolicy.Highest
    chains: Optional[list] = None

    def to_c(self) -> N.ParseOpts:
        o = N.ParseOpts()
        N.lib.crab_parse_options_default(C.byref(o))
        o.include_hetatm = int(self.include_hetatm)
        o.include_waters = int(self.include_waters)
        o.include_glycans = int(self.include_glycans)
        o.model_index = int(self.model_index)
        o.allow_unknown_elements = int(self.allow_unknown_elements)
        o.occupancy_policy = int(self.occupancy_policy)
        o.altloc_policy = int(self.altloc_policy)
        if self.chains:
            arr = (C.c_char_p * len(self.chains))(*[c.encode() for c in self.chains])
            o._chains_keep = arr
            o.n_chains = len(self.chains)
            o.chains = C.cast(arr, C.POINTER(C.c_char_p))
        return o


def _parsed_bytes(p: C.c_void_p, which: int) -> bytes:
    size = C.c_int64()
    N.lib.crab_parsed_strings(p, which, None, 0, C.byref(size))
    buf = C.create_string_buffer(max(size.value, 1))
    N.lib.crab_parsed_strings(p, which, buf, size.value, C.byref(size))
    return buf.raw[:size.value]


def _parse_check(status: int) -> None:
    if status != N.OK:
        msg = (N.lib.crab_parse_last_error() or b"").decode()
        _raise_parse(status, msg)


def _raise_parse(status: int, msg: str) -> None:
    name = N.STATUS_NAMES.get(status, str(status))
    if status == N.EPARSE:
        raise StructureParse(msg or name)
    if status == N.EELEMENT:
        raise UnsupportedElement(msg or name)
    if status == N.EIO:
        raise OSError(msg or name)
    if status == N.EINVAL:
        raise InvalidInput(msg or name)
    raise Other(f"{name}: {msg}")


# ---------------------------------------------------------------- options
class HydrogenMode(enum.Enum):
    Implicit = 1
    Explicit = 0


class ScatteringMethod(enum.Enum):
    Auto = N.METHOD_AUTO
    Debye = N.METHOD_DEBYE
    Multipole = N.METHOD_MULTIPOLE


class HydrationModel(enum.Enum):
    Analytic = N.HYD_ANALYTIC
    Grid = N.HYD_GRID
    AdaptiveGrid = N.HYD_ADAPTIVE


@dataclass
class SolventParams:
    c1: float = 1.0
    c2: float = 0.0
    shell_thickness_angstrom: float = 3.0
    bulk_density_e_per_a3: float = 0.334
    hydration_model: HydrationModel = HydrationModel.Analytic
    hydration_grid_spacing_angstrom: float = 4.0

    def to_c(self) -> N.Solvent:
        return N.Solvent(self.c1, self.c2, self.shell_thickness_angstrom, self.bulk_density_e_per_a3,
                         self.hydration_model.value, 0, self.hydration_grid_spacing_angstrom)


@dataclass
class ComputeOptions:
    method: ScatteringMethod = ScatteringMethod.Auto
    hydrogen_mode: HydrogenMode = HydrogenMode.Implicit
    include_hetatm: bool = False
    multipole_l_max: Optional[int] = None
    solvent: Optional[SolventParams] = None

    def to_c(self) -> N.ComputeOpts:
        s = self.solvent.to_c() if self.solvent else SolventParams().to_c()
        return N.ComputeOpts(self.method.value, self.hydrogen_mode.value, self.multipole_l_max or 0,
                             1 if self.solvent else 0, s)


@dataclass
class ScatteringCurve:
    q: np.ndarray
    intensity: np.ndarray
    method: str
    atom_count: int


class ScaleMode:
    """fit.rs:30-34: ``ScaleMode.Fit`` or ``ScaleMode.Fixed(value)``."""

    def __init__(self, fixed: Optional[float] = None):
        self.fixed = fixed

    @classmethod
    def Fixed(cls, value: float) -> "ScaleMode":
        return cls(value)


ScaleMode.Fit = ScaleMode()


class BackgroundMode:
    """fit.rs:41-47: ``Fit``, ``FixedZero`` or ``Fixed(value)``."""

    def __init__(self, kind: int, value: float = 0.0):
        self.kind = kind
        self.value = value

    @classmethod
    def Fixed(cls, value: float) -> "BackgroundMode":
        return cls(N.BG_FIXED, value)


BackgroundMode.Fit = BackgroundMode(N.BG_FIT)
BackgroundMode.FixedZero = BackgroundMode(N.BG_FIXED_ZERO)


@dataclass
class FitOptions:
    method: ScatteringMethod = ScatteringMethod.Auto
    hydrogen_mode: HydrogenMode = HydrogenMode.Implicit
    c1_bounds: tuple = (0.95, 1.05)
    c2_bounds: tuple = (-2.0, 4.0)
    max_iterations: int = 64
    q_sampling_stride: int = 20
    solvent: SolventParams = field(default_factory=SolventParams)
    background_mode: BackgroundMode = field(default_factory=lambda: BackgroundMode.Fit)
    scale_mode: ScaleMode = field(default_factory=lambda: ScaleMode.Fit)
    optimizer: str = "nelder-mead"  # or "lbfgs"

    def to_c(self) -> N.FitOpts:
        return N.FitOpts(self.method.value, self.hydrogen_mode.value, self.c1_bounds[0], self.c1_bounds[1],
                         self.c2_bounds[0], self.c2_bounds[1], self.max_iterations, self.q_sampling_stride,
                         self.solvent.to_c(),
                         N.SCALE_FIT if self.scale_mode.fixed is None else N.SCALE_FIXED,
                         self.background_mode.kind, self.scale_mode.fixed or 0.0, self.background_mode.value,
                         1 if self.optimizer == "lbfgs" else 0, 0)


@dataclass
class FitParams:
    scale: float = 1.0
    background: float = 0.0
    c1: float = 1.0
    c2: float = 0.0


@dataclass
class FitResult:
    params: FitParams
    chi2: float
    fitted_curve: np.ndarray
    iterations: int
    converged: bool


@dataclass
class ExperimentalCurve:
    q: np.ndarray
    intensity: np.ndarray
    sigma: np.ndarray
    has_errors: bool = True

    def __post_init__(self):
        self.q = _f64(self.q)
        self.intensity = _f64(self.intensity)
        self.sigma = _f64(self.sigma)

    def __len__(self) -> int:
        return len(self.q)

    def is_empty(self) -> bool:
        return len(self.q) == 0


# ---------------------------------------------------------------- engines
def debye_intensity(structure: Structure, q, implicit_hydrogen: bool = True, engine: Optional[Engine] = None):
    """scattering.rs:82-110 on the GPU."""
    eng = engine or Engine.default()
    qa = _f64(q)
    out = np.empty(len(qa))
    eng.check(N.lib.crab_debye_intensity(eng.handle, structure.handle(eng), _dp(qa), len(qa),
                                         1 if implicit_hydrogen else 0, _dp(out)))
    return out


def debye_solvent_basis(structure: Structure, q, params: SolventParams, implicit_hydrogen: bool = True,
                        engine: Optional[Engine] = None, fp64: bool = False,
                        shard: Optional[tuple[int, int]] = None) -> np.ndarray:
    """solvent.rs:504-584: rows vv, ee, hh, ve, vh, eh.  fp64=True runs the pair
    sums with the FP64 device reference kernel instead of the FP32 recurrence.
    shard=(k, n): only part k of n (see crab_debye_solvent_basis_shard); the
    n parts sum to the whole basis."""
    eng = engine or Engine.default()
    qa = _f64(q)
    out = np.empty((6, len(qa)))
    s = params.to_c()
    prec = N.PREC_FP64 if fp64 else N.PREC_FP32
    if shard is None:
        eng.check(N.lib.crab_debye_solvent_basis_ex(eng.handle, structure.handle(eng), _dp(qa), len(qa), C.byref(s),
                                                    1 if implicit_hydrogen else 0, prec, _dp(out)))
    else:
        k, n = shard
        eng.check(N.lib.crab_debye_solvent_basis_shard(eng.handle, structure.handle(eng), _dp(qa), len(qa),
                                                       C.byref(s), 1 if implicit_hydrogen else 0, prec, int(k),
                                                       int(n), _dp(out)))
    return out


def combine_solvent_basis(basis: np.ndarray, q, c1: float, c2: float) -> np.ndarray:
    """spherical.rs:567-584."""
    qa = _f64(q)
    b = _f64(basis)
    out = np.empty(len(qa))
    _raise(N.lib.crab_combine_solvent_basis(_dp(qa), len(qa), _dp(b), c1, c2, _dp(out)))
    return out


def solvent_corrected_intensity(structure, q, params: SolventParams, implicit_hydrogen=True, engine=None):
    """solvent.rs:490-500."""
    b = debye_solvent_basis(structure, q, params, implicit_hydrogen, engine)
    return combine_solvent_basis(b, q, params.c1, params.c2)


class _MomentSum:
    """crab_sum_fn around a Python function that sums a float64 array over
    the ranks in place; an exception inside it ends the library call and is
    raised again after it returns.  With device=True the function receives
    (device pointer as an int, count) instead of a host array."""

    def __init__(self, fn, device: bool = False):
        self.error = None

        def call(values, count, user):
            try:
                if device:
                    fn(C.cast(values, C.c_void_p).value, int(count))
                else:
                    fn(np.ctypeslib.as_array(values, shape=(count,)))
                return N.OK
            except BaseException as e:  # noqa: BLE001 - re-raised by check()
                self.error = e
                return N.EINVAL

        self.c = N.SUM_FN(call)

    def check(self, eng: "Engine", rc: int):
        if self.error is not None:
            raise self.error
        eng.check(rc)


class _DeviceSums:
    """crab_ctx_set_device_sums on for the duration of one call."""

    def __init__(self, eng: "Engine", on: bool):
        self.eng, self.on = eng, on

    def __enter__(self):
        if self.on:
            self.eng.check(N.lib.crab_ctx_set_device_sums(self.eng.handle, 1))

    def __exit__(self, *exc):
        if self.on:
            N.lib.crab_ctx_set_device_sums(self.eng.handle, 0)


def multipole_intensity(structure: Structure, q, l_max: int, implicit_hydrogen: bool = True,
                        precision: int = N.PREC_TF32_SPLIT, engine: Optional[Engine] = None,
                        shard: Optional[tuple[int, int]] = None, moment_sum=None,
                        device_sums: bool = False) -> np.ndarray:
    """spherical.rs:266-403.  shard=(k, n) with moment_sum(array) (an in-place
    sum over the ranks): this rank's share of the atoms in the moments, the
    whole curve returned (crab_multipole_intensity_shard).  device_sums=True:
    moment_sum(device pointer, count) sums the moments in device memory
    (crab_ctx_set_device_sums)."""
    eng = engine or Engine.default()
    qa = _f64(q)
    out = np.empty(len(qa))
    if shard is None:
        eng.check(N.lib.crab_multipole_intensity(eng.handle, structure.handle(eng), _dp(qa), len(qa), l_max,
                                                 1 if implicit_hydrogen else 0, precision, _dp(out)))
    else:
        cb = _MomentSum(moment_sum or (lambda *a: None), device=device_sums)
        with _DeviceSums(eng, device_sums):
            rc = N.lib.crab_multipole_intensity_shard(eng.handle, structure.handle(eng), _dp(qa), len(qa), l_max,
                                                      1 if implicit_hydrogen else 0, precision, int(shard[0]),
                                                      int(shard[1]), cb.c, None, _dp(out))
        cb.check(eng, rc)
    return out


def multipole_solvent_basis(structure: Structure, q, l_max: int, params: SolventParams,
                            implicit_hydrogen: bool = True, precision: int = N.PREC_TF32_SPLIT,
                            engine: Optional[Engine] = None, shard: Optional[tuple[int, int]] = None,
                            moment_sum=None, device_sums: bool = False) -> np.ndarray:
    """spherical.rs:474-565.  shard / moment_sum / device_sums as in
    multipole_intensity (crab_multipole_solvent_basis_shard)."""
    eng = engine or Engine.default()
    qa = _f64(q)
    out = np.empty((6, len(qa)))
    s = params.to_c()
    if shard is None:
        eng.check(N.lib.crab_multipole_solvent_basis(eng.handle, structure.handle(eng), _dp(qa), len(qa), l_max,
                                                     C.byref(s), 1 if implicit_hydrogen else 0, precision,
                                                     _dp(out)))
    else:
        cb = _MomentSum(moment_sum or (lambda *a: None), device=device_sums)
        with _DeviceSums(eng, device_sums):
            rc = N.lib.crab_multipole_solvent_basis_shard(eng.handle, structure.handle(eng), _dp(qa), len(qa),
                                                          l_max, C.byref(s), 1 if implicit_hydrogen else 0,
                                                          precision, int(shard[0]), int(shard[1]), cb.c, None,
                                                          _dp(out))
        cb.check(eng, rc)
    return out


def compute_curve(structure: Structure, q, options: ComputeOptions, engine: Optional[Engine] = None):
    """scattering.rs:112-212."""
    eng = engine or Engine.default()
    qa = _f64(q)
    out = np.empty(len(qa))
    used = C.c_int32()
    o = options.to_c()
    eng.check(N.lib.crab_compute_curve(eng.handle, structure.handle(eng), _dp(qa), len(qa), C.byref(o), _dp(out),
                                       C.byref(used)))
    name = {N.METHOD_DEBYE: "Debye", N.METHOD_MULTIPOLE: "Multipole"}.get(used.value, "?")
    return ScatteringCurve(qa.copy(), out, name, structure.atom_count)


def hydration_grid_adaptive(structure: Structure, spacing=4.0, clearance=3.0, padding=12.0, engine=None):
    """solvent.rs:121-223: (sites [m,3], voxel volume)."""
    eng = engine or Engine.default()
    m = C.c_int64()
    vol = C.c_double()
    h = structure.handle(eng)
    eng.check(N.lib.crab_hydration_grid_adaptive(eng.handle, h, spacing, clearance, padding, None, 0, C.byref(m),
                                                 C.byref(vol)))
    sites = np.empty((m.value, 3))
    eng.check(N.lib.crab_hydration_grid_adaptive(eng.handle, h, spacing, clearance, padding, _dp(sites), m.value,
                                                 C.byref(m), C.byref(vol)))
    return sites, vol.value


def hydration_grid_exterior(structure: Structure, spacing=1.0, probe=1.4, thickness=3.0, engine=None):
    """solvent.rs:259-401: (sites [m,3], voxel volume)."""
    eng = engine or Engine.default()
    m = C.c_int64()
    vol = C.c_double()
    h = structure.handle(eng)
    eng.check(N.lib.crab_hydration_grid_exterior(eng.handle, h, spacing, probe, thickness, None, 0, C.byref(m),
                                                 C.byref(vol)))
    sites = np.empty((m.value, 3))
    eng.check(N.lib.crab_hydration_grid_exterior(eng.handle, h, spacing, probe, thickness, _dp(sites), m.value,
                                                 C.byref(m), C.byref(vol)))
    return sites, vol.value


def debye_partials(xyz, w, types, n_types: int, q, fp64: bool = False, engine: Optional[Engine] = None,
                   shard: Optional[tuple[int, int]] = None):
    """Per type-pair pair sums P[ab, k] and self sums D[a] (see crab_debye_partials).
    shard=(k, n): only part k of n (crab_debye_partials_shard)."""
    eng = engine or Engine.default()
    x = _f64(xyz).reshape(-1, 3)
    ww = _f64(w)
    t = np.ascontiguousarray(np.asarray(types, dtype=np.int32))
    qa = _f64(q)
    P = n_types * (n_types + 1) // 2
    out = np.empty((P, len(qa)))
    self_ = np.empty(n_types)
    if shard is None:
        fn = N.lib.crab_debye_partials_fp64 if fp64 else N.lib.crab_debye_partials
        eng.check(fn(eng.handle, _dp(x), _dp(ww), t.ctypes.data_as(N.I32P), x.shape[0], n_types, _dp(qa), len(qa),
                     _dp(out), _dp(self_)))
    else:
        k, n = shard
        eng.check(N.lib.crab_debye_partials_shard(eng.handle, _dp(x), _dp(ww), t.ctypes.data_as(N.I32P), x.shape[0],
                                                  n_types, _dp(qa), len(qa), N.PREC_FP64 if fp64 else N.PREC_FP32,
                                                  int(k), int(n), _dp(out), _dp(self_)))
    return out, self_


def chi2_grad(structure: Structure, q, y, sigma, solvent: SolventParams, scale: float, background: float,
              implicit_hydrogen: bool = True, engine: Optional[Engine] = None):
    """Reduced chi² of scale·I(q)+background and its gradient (coordinates, and c1, c2, scale, background)."""
    eng = engine or Engine.default()
    qa, ya, sa = _f64(q), _f64(y), _f64(sigma)
    chi = C.c_double()
    gx = np.empty((structure.atom_count, 3))
    gp = np.empty(4)
    s = solvent.to_c()
    eng.check(N.lib.crab_chi2_grad(eng.handle, structure.handle(eng), _dp(qa), _dp(ya), _dp(sa), len(qa),
                                   C.byref(s), 1 if implicit_hydrogen else 0, scale, background, C.byref(chi),
                                   _dp(gx), _dp(gp)))
    return chi.value, gx, gp


# ---------------------------------------------------------------- analysis.rs
class Quality(enum.Enum):
    Fast = "fast"
    Balanced = "balanced"
    Accurate = "accurate"

    def fit_options(self, options: FitOptions) -> FitOptions:
        """analysis.rs:23-42."""
        o = replace(options, solvent=replace(options.solvent))
        if self is Quality.Fast:
            o.q_sampling_stride = max(o.q_sampling_stride, 20)
            o.max_iterations = min(o.max_iterations, 32)
            o.solvent.hydration_grid_spacing_angstrom = 8.0
        elif self is Quality.Balanced:
            o.q_sampling_stride = 20
            o.max_iterations = max(o.max_iterations, 64)
            o.solvent.hydration_grid_spacing_angstrom = 4.0
        else:
            o.q_sampling_stride = 1
            o.max_iterations = max(o.max_iterations, 128)
            o.solvent.hydration_grid_spacing_angstrom = 3.0
        return o

    def compute_options(self, options: ComputeOptions) -> ComputeOptions:
        """analysis.rs:44-55."""
        o = replace(options)
        if o.solvent is not None:
            o.solvent = replace(o.solvent)
            if self is Quality.Fast:
                o.solvent.hydration_grid_spacing_angstrom = 8.0
            elif self is Quality.Accurate:
                o.solvent.hydration_grid_spacing_angstrom = 3.0
        return o


def _validate_q(q) -> np.ndarray:
    qa = _f64(q)
    if not np.all(np.isfinite(qa)) or np.any(qa < 0) or np.any(np.diff(qa) < 0):
        raise InvalidInput("q grid must be finite, non-negative, and non-decreasing")
    return qa


class ProfileCalculator:
    """analysis.rs:59-105."""

    def __init__(self, q, options: Optional[ComputeOptions] = None, engine: Optional[Engine] = None):
        self.q = _validate_q(q)
        self.options = options or ComputeOptions()
        self.engine = engine or Engine.default()

    def calculate(self, structure: Structure) -> ScatteringCurve:
        return compute_curve(structure, self.q, self.options, self.engine)


def _fit(structure: Structure, experimental: ExperimentalCurve, initial: FitParams, options: FitOptions,
         engine: Engine) -> FitResult:
    o = options.to_c()
    res = N.FitResult()
    fitted = np.empty(len(experimental))
    engine.check(N.lib.crab_fit(engine.handle, structure.handle(engine), _dp(experimental.q),
                                _dp(experimental.intensity), _dp(experimental.sigma), len(experimental), C.byref(o),
                                initial.c1, initial.c2, C.byref(res), _dp(fitted)))
    return FitResult(FitParams(res.scale, res.background, res.c1, res.c2), res.chi2, fitted, res.iterations,
                     bool(res.converged))


def fit_to_experimental_with_options(structure, experimental, initial: FitParams, options: FitOptions,
                                     engine: Optional[Engine] = None) -> FitResult:
    """fit.rs:288-454."""
    return _fit(structure, experimental, initial, options, engine or Engine.default())


class SaxsFitter:
    """analysis.rs:67-88."""

    def __init__(self, options: Optional[FitOptions] = None, engine: Optional[Engine] = None):
        self.options = options or FitOptions()
        self.engine = engine or Engine.default()

    def fit(self, structure: Structure, experimental: ExperimentalCurve) -> FitResult:
        return _fit(structure, experimental, FitParams(), self.options, self.engine)


@dataclass
class ScoreOptions:
    fit: FitOptions = field(default_factory=FitOptions)
    quality: Quality = Quality.Fast


@dataclass
class ScoreResult:
    chi2: float
    reduced_chi2: float
    scale: float
    background: float
    q_min: float
    q_max: float
    points: int
    has_errors: bool
    fit: FitResult


class SaxsScorer:
    """analysis.rs:137-178."""

    def __init__(self, experimental: ExperimentalCurve, options: Optional[ScoreOptions] = None,
                 engine: Optional[Engine] = None):
        if experimental.is_empty():
            raise InvalidInput("experimental curve is empty")
        self.experimental = experimental
        self.options = options or ScoreOptions()
        self.engine = engine or Engine.default()

    def score(self, structure: Structure) -> ScoreResult:
        fo = self.options.quality.fit_options(self.options.fit)
        fit = _fit(structure, self.experimental, FitParams(), fo, self.engine)
        dof = max(len(self.experimental) - 1, 1)
        return ScoreResult(fit.chi2 * dof, fit.chi2, fit.params.scale, fit.params.background,
                           float(self.experimental.q[0]), float(self.experimental.q[-1]), len(self.experimental),
                           self.experimental.has_errors, fit)


@dataclass
class ComparisonResult:
    chi2: float
    reduced_chi2: float
    pearson_correlation: float
    r_factor: float
    weighted_rmse: float
    residuals: np.ndarray


def compare_curves(experimental: ExperimentalCurve, calculated) -> ComparisonResult:
    """analysis.rs:190-251 (host post-processing of two curves)."""
    calc = _f64(calculated)
    if len(experimental) != len(calc) or experimental.is_empty():
        raise InvalidInput("experimental and calculated curves must have equal non-zero lengths")
    res = calc - experimental.intensity
    dof = max(len(experimental) - 1, 1)
    chi = float(np.sum((res / experimental.sigma) ** 2))
    mo, mm = experimental.intensity.mean(), calc.mean()
    cov = float(np.sum((experimental.intensity - mo) * (calc - mm)))
    vo, vm = float(np.sum((experimental.intensity - mo) ** 2)), float(np.sum((calc - mm) ** 2))
    pearson = cov / math.sqrt(vo * vm) if vo > 0 and vm > 0 else 0.0
    den = float(np.sum(np.abs(experimental.intensity)))
    r = float(np.sum(np.abs(res))) / den if den > 0 else 0.0
    return ComparisonResult(chi, chi / dof, pearson, r, math.sqrt(chi / len(experimental)), res)


# ---------------------------------------------------------------- ensembles
@dataclass
class EnsembleOptions:
    fit_weights: bool = True
    uniform: bool = False
    regularization: float = 0.0
    max_conformers: Optional[int] = None
    min_weight: float = 0.0
    bootstrap: int = 0
    seed: int = 0xC0FFEE
    fit: FitOptions = field(default_factory=FitOptions)


@dataclass
class WeightInterval:
    median: float
    lower: float
    upper: float


@dataclass
class EnsembleResult:
    conformers: list
    weights: np.ndarray
    params: FitParams
    chi2: float
    reduced_chi2: float
    fitted_curve: np.ndarray
    iterations: int
    converged: bool
    weight_intervals: list = field(default_factory=list)
    bootstrap_reduced_chi2: list = field(default_factory=list)


class EnsembleFitter:
    """ensemble.rs:61-299."""

    def __init__(self, conformers: Sequence[Structure], names: Sequence[str], experimental: ExperimentalCurve,
                 options: Optional[EnsembleOptions] = None, engine: Optional[Engine] = None):
        if not conformers or any(c.atom_count == 0 for c in conformers):
            raise InvalidInput("ensemble must contain non-empty conformers")
        if len(names) != len(conformers):
            raise InvalidInput("ensemble names and conformers differ in length")
        if experimental.is_empty():
            raise InvalidInput("ensemble requires a validated experimental curve")
        o = options or EnsembleOptions()
        if (not math.isfinite(o.regularization) or o.regularization < 0 or not math.isfinite(o.min_weight)
                or not 0.0 <= o.min_weight <= 1.0 or o.max_conformers == 0):
            raise InvalidInput("ensemble regularization and pruning options are invalid")
        self.conformers = list(conformers)
        self.names = list(names)
        self.experimental = experimental
        self.options = o
        self.engine = engine or Engine.default()

    def fit(self) -> EnsembleResult:
        return self._fit(None)

    def _handles(self):
        k = len(self.conformers)
        return (C.c_void_p * k)(*[c.handle(self.engine) for c in self.conformers])

    def partials(self, shard: tuple[int, int] = (0, 1)) -> tuple[int, np.ndarray]:
        """This shard's pair sums of the ensemble (crab_ensemble_partials):
        (type count T, buffer of k blocks, zero for conformers it does not
        own).  Summing the buffers of all shards gathers every conformer."""
        e = self.engine
        k = len(self.conformers)
        ex = self.experimental
        implicit = self.options.fit.to_c().implicit_hydrogen
        handles = self._handles()
        t = C.c_int32()
        e.check(N.lib.crab_ensemble_partials(e.handle, handles, k, _dp(ex.q), len(ex), implicit, int(shard[0]),
                                             int(shard[1]), C.byref(t), None, 0))
        T = t.value
        buf = np.empty(k * (T * (T + 1) // 2 * len(ex) + 2 * T))
        e.check(N.lib.crab_ensemble_partials(e.handle, handles, k, _dp(ex.q), len(ex), implicit, int(shard[0]),
                                             int(shard[1]), C.byref(t), _dp(buf), buf.size))
        return T, buf

    def fit_from_partials(self, n_types: int, partials: np.ndarray) -> EnsembleResult:
        """fit() with the pair sums of every conformer given (the sum over
        shards of partials()): crab_ensemble_fit_partials."""
        return self._fit((int(n_types), np.ascontiguousarray(partials, dtype=np.float64)))

    def _fit(self, given) -> EnsembleResult:
        e = self.engine
        k = len(self.conformers)
        handles = self._handles()
        o = self.options
        eo = N.EnsembleOpts(1 if o.fit_weights else 0, 1 if o.uniform else 0, o.regularization,
                            o.max_conformers or 0, o.bootstrap, o.min_weight, o.seed)
        fo = o.fit.to_c()
        res = N.EnsembleResult()
        sel = np.empty(k, dtype=np.int32)
        w = np.empty(k)
        fitted = np.empty(len(self.experimental))
        ex = self.experimental
        intervals = np.empty((k, 3))
        boot = np.empty(max(o.bootstrap, 1))
        if given is None:
            e.check(N.lib.crab_ensemble_fit(e.handle, handles, k, _dp(ex.q), _dp(ex.intensity), _dp(ex.sigma),
                                            len(ex), C.byref(eo), C.byref(fo), C.byref(res),
                                            sel.ctypes.data_as(N.I32P), _dp(w), _dp(fitted), _dp(intervals),
                                            _dp(boot)))
        else:
            T, buf = given
            if buf.size != k * (T * (T + 1) // 2 * len(ex) + 2 * T):
                raise InvalidInput("partials buffer does not match the ensemble")
            e.check(N.lib.crab_ensemble_fit_partials(e.handle, handles, k, _dp(ex.q), _dp(ex.intensity),
                                                     _dp(ex.sigma), len(ex), C.byref(eo), C.byref(fo), _dp(buf), T,
                                                     C.byref(res), sel.ctypes.data_as(N.I32P), _dp(w), _dp(fitted),
                                                     _dp(intervals), _dp(boot)))
        n = res.n_selected
        return EnsembleResult([self.names[i] for i in sel[:n]], w[:n].copy(),
                              FitParams(res.scale, res.background, res.c1, res.c2), res.chi2, res.reduced_chi2,
                              fitted, res.iterations, True,
                              [WeightInterval(*row) for row in intervals[:n]], list(boot[:o.bootstrap]))


def ensemble_curves(conformers: Sequence[Structure], q, solvent: SolventParams, candidates,
                    implicit_hydrogen: bool = True, engine: Optional[Engine] = None) -> np.ndarray:
    """Debye curves of every conformer at every (c1, c2) candidate: [n_cand, k, nq]."""
    e = engine or Engine.default()
    k = len(conformers)
    handles = (C.c_void_p * k)(*[c.handle(e) for c in conformers])
    qa = _f64(q)
    cand = _f64(candidates).reshape(-1, 2)
    out = np.empty((cand.shape[0], k, len(qa)))
    s = solvent.to_c()
    e.check(N.lib.crab_ensemble_curves(e.handle, handles, k, _dp(qa), len(qa), C.byref(s),
                                       1 if implicit_hydrogen else 0, _dp(cand), cand.shape[0], _dp(out)))
    return out


def solvent_candidates(fit: FitOptions) -> np.ndarray:
    """ensemble.rs:302-315: the 5x5 (c1, c2) grid over the fit bounds."""
    c1 = fit.c1_bounds[0] + (fit.c1_bounds[1] - fit.c1_bounds[0]) * np.arange(5) / 4.0
    c2 = fit.c2_bounds[0] + (fit.c2_bounds[1] - fit.c2_bounds[0]) * np.arange(5) / 4.0
    return np.array([(a, b) for a in c1 for b in c2])


class EnsemblePlan:
    """Device-resident ensemble scoring (crab_ensemble_plan_*): one CUDA graph
    per score() call covering pair sums of every conformer, curves at every
    (c1, c2) candidate, simplex weight fits, gradients and KL reweighting."""

    def __init__(self, conformers: Sequence[Structure], q, solvent: Optional[SolventParams] = None,
                 candidates=None, implicit_hydrogen: bool = True, engine: Optional[Engine] = None):
        self.engine = engine or Engine.default()
        e = self.engine
        self.k = len(conformers)
        self.q = _f64(q)
        self.cand = _f64(solvent_candidates(FitOptions()) if candidates is None else candidates).reshape(-1, 2)
        self._keep = list(conformers)
        handles = (C.c_void_p * self.k)(*[c.handle(e) for c in conformers])
        s = (solvent or SolventParams()).to_c()
        self.handle = C.c_void_p()
        e.check(N.lib.crab_ensemble_plan_create(e.handle, handles, self.k, _dp(self.q), len(self.q), C.byref(s),
                                                1 if implicit_hydrogen else 0, _dp(self.cand), self.cand.shape[0],
                                                C.byref(self.handle)))

    def autotune(self) -> int:
        c = C.c_int32()
        self.engine.check(N.lib.crab_ensemble_plan_autotune(self.engine.handle, self.handle, C.byref(c)))
        return c.value

    def score(self, y, sigma, fit: Optional[FitOptions] = None, reweight: Optional["MaximumEntropyOptions"] = None):
        e = self.engine
        yy, ss = _f64(y), _f64(sigma)
        fo = (fit or FitOptions()).to_c()
        ro = None
        if reweight is not None:
            f = reweight.fit
            ro = N.ReweightOpts(reweight.kl_strength, reweight.step_size, reweight.tolerance, reweight.min_weight,
                                reweight.max_iterations, N.SCALE_FIT if f.scale_mode.fixed is None else N.SCALE_FIXED,
                                f.background_mode.kind, 0, f.scale_mode.fixed or 0.0, f.background_mode.value)
        ms = C.c_double()
        best = np.empty(8)
        w, gw, kw = np.empty(self.k), np.empty(self.k), np.empty(self.k)
        rw = np.empty(6)
        e.check(N.lib.crab_ensemble_plan_score(e.handle, self.handle, _dp(yy), _dp(ss), C.byref(fo),
                                               None if ro is None else C.byref(ro), C.byref(ms), _dp(best), _dp(w),
                                               _dp(gw), _dp(kw), _dp(rw)))
        return dict(elapsed_ms=ms.value, candidate=int(best[0]), c1=best[1], c2=best[2], scale=best[3],
                    background=best[4], reduced_chi2=best[5], dchi2_dc1=best[6], dchi2_dc2=best[7], weights=w,
                    dchi2_dw=gw, kl_weights=kw, kl_scale=rw[0], kl_background=rw[1], kl_reduced_chi2=rw[2],
                    kl_divergence=rw[3], kl_iterations=int(rw[4]), kl_converged=bool(rw[5]))

    def close(self):
        if self.handle:
            N.lib.crab_ensemble_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class MaximumEntropyOptions:
    kl_strength: float = 1.0
    max_iterations: int = 500
    step_size: float = 0.5
    tolerance: float = 1e-8
    min_weight: float = 1e-10
    prior_weights: Optional[Sequence[float]] = None
    fit: FitOptions = field(default_factory=FitOptions)


@dataclass
class MaximumEntropyResult:
    names: list
    weights: np.ndarray
    prior_weights: np.ndarray
    params: FitParams
    chi2: float
    reduced_chi2: float
    kl_divergence: float
    effective_sample_size: float
    iterations: int
    converged: bool


def reweight_curves(names: Sequence[str], curves, experimental: ExperimentalCurve,
                    options: Optional[MaximumEntropyOptions] = None) -> MaximumEntropyResult:
    """reweight.rs:84-154."""
    o = options or MaximumEntropyOptions()
    cv = _f64(curves)
    if cv.ndim != 2 or cv.shape[0] == 0 or len(names) != cv.shape[0]:
        raise InvalidInput("reweighting names and curves must have equal non-zero lengths")
    if cv.shape[1] != len(experimental):
        raise InvalidInput("all reweighting curves must match the experimental q grid")
    k = cv.shape[0]
    prior = None if o.prior_weights is None else _f64(o.prior_weights)
    if prior is not None and len(prior) != k:
        raise InvalidInput("maximum-entropy prior weights must be positive and match the ensemble")
    fo = o.fit
    ro = N.ReweightOpts(o.kl_strength, o.step_size, o.tolerance, o.min_weight, o.max_iterations,
                        N.SCALE_FIT if fo.scale_mode.fixed is None else N.SCALE_FIXED, fo.background_mode.kind, 0,
                        fo.scale_mode.fixed or 0.0, fo.background_mode.value)
    w = np.empty(k)
    res = N.ReweightResult()
    ex = experimental
    st = N.lib.crab_reweight_curves(_dp(cv), k, _dp(ex.q), _dp(ex.intensity), _dp(ex.sigma), len(ex),
                                    None if prior is None else _dp(prior), C.byref(ro), _dp(w), C.byref(res))
    if st != N.OK:
        raise InvalidInput("maximum-entropy options are invalid")
    pr = np.ones(k) / k if prior is None else prior / prior.sum()
    return MaximumEntropyResult(list(names), w, pr, FitParams(res.scale, res.background, fo.solvent.c1,
                                                              fo.solvent.c2),
                                res.chi2, res.reduced_chi2, res.kl_divergence, res.effective_sample_size,
                                res.iterations, bool(res.converged))


# ---------------------------------------------------------------- coordinate P(r)
@dataclass
class PrOptions:
    """metrics.rs:15-29: bins of the coordinate P(r) (raised to at least 16);
    max_r only bounds the experimental transform, which is not on this path."""
    bins: int = 160
    max_r: Optional[float] = None


@dataclass
class PairDistribution:
    """metrics.rs:31-37; rg / dmax are None where the reference has None."""
    r: np.ndarray
    p: np.ndarray
    rg: Optional[float]
    dmax: Optional[float]


@dataclass
class CoordinateFeatures:
    """metrics.rs:60-65."""
    rg: float
    dmax: float
    p_r: PairDistribution


def coordinate_features(structure: Structure, options: Optional[PrOptions] = None,
                        engine: Optional[Engine] = None) -> CoordinateFeatures:
    """metrics.rs:236-270: scattering-weighted Rg, Dmax and normalised P(r)."""
    eng = engine or Engine.default()
    o = options or PrOptions()
    m = max(int(o.bins), 16)
    r, p = np.empty(m), np.empty(m)
    rg, dmax, prg, pdm = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    used = C.c_int64()
    eng.check(N.lib.crab_coordinate_features(eng.handle, structure.handle(eng), int(o.bins), C.byref(rg),
                                             C.byref(dmax), _dp(r), _dp(p), C.byref(used), C.byref(prg),
                                             C.byref(pdm)))
    k = used.value

    def opt(x):
        return None if math.isnan(x) else x

    return CoordinateFeatures(rg.value, dmax.value,
                              PairDistribution(r[:k].copy(), p[:k].copy(), opt(prg.value), opt(pdm.value)))


def pair_distance_histogram(xyz, w, bins: int, engine: Optional[Engine] = None):
    """metrics.rs:475-522 before normalisation: (dmax, weighted histogram [bins])."""
    eng = engine or Engine.default()
    x = _f64(xyz).reshape(-1, 3)
    ww = _f64(w)
    if len(ww) != x.shape[0]:
        raise InvalidInput("one weight per atom")
    hist = np.empty(max(int(bins), 0))
    dmax = C.c_double()
    eng.check(N.lib.crab_pair_distance_histogram(eng.handle, _dp(x), _dp(ww), x.shape[0], int(bins),
                                                 C.byref(dmax), _dp(hist)))
    return dmax.value, hist


def pr_last_timing(engine: Optional[Engine] = None):
    """Device ms of the last P(r) call (all kernels, histogram kernel), its pair
    count and accumulation mode (0 class counts, 1 shared f64, 2 device-memory f64)."""
    eng = engine or Engine.default()
    t, h, n, m = C.c_double(), C.c_double(), C.c_double(), C.c_int32()
    eng.check(N.lib.crab_pr_last_timing(eng.handle, C.byref(t), C.byref(h), C.byref(n), C.byref(m)))
    return t.value, h.value, n.value, m.value
