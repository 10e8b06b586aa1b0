"""ORACLE — test infrastructure only (see oracle.cpp).

ctypes binding of ``oracle/liboracle.so``, the C++ f64 restatement of the
crabSAXS reference algorithms.  Only tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py use it, as the checker and as the timed CPU
baseline; the crabsaxs_b200 package never imports it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle.so"
if not _LIB_PATH.exists():
    from .build import build as _build

    _build()
lib = C.CDLL(str(_LIB_PATH))

D = C.POINTER(C.c_double)
I32 = C.POINTER(C.c_int32)
I64 = C.c_int64

_SIGS = {
    "orc_form_factor": (C.c_double, [C.c_int, C.c_int, C.c_double, C.c_int, C.c_double]),
    "orc_excluded_volume_for_atom": (C.c_double, [C.c_int, C.c_int, C.c_int]),
    "orc_excluded_volume_for": (C.c_double, [C.c_int]),
    "orc_vdw_radius": (C.c_double, [C.c_int]),
    "orc_water_form_factor": (C.c_double, [C.c_double]),
    "orc_excluded_volume_scale": (C.c_double, [C.c_double, C.c_double]),
    "orc_adaptive_shell_width": (C.c_double, [C.c_double]),
    "orc_sinc": (C.c_double, [C.c_double]),
    "orc_united_atom_group": (C.c_int, [C.c_char_p, C.c_char_p]),
    "orc_debye_intensity": (C.c_int, [I64, D, I32, I32, D, C.c_int, I64, D, D]),
    "orc_debye_partials": (C.c_int, [I64, D, D, I32, C.c_int, I64, D, D, D]),
    "orc_adaptive_grid": (C.c_int, [I64, D, C.c_double, C.c_double, C.c_double, D, I64, C.POINTER(I64), D]),
    "orc_exterior_grid": (C.c_int, [I64, D, I32, C.c_double, C.c_double, C.c_double, D, I64, C.POINTER(I64), D]),
    "orc_debye_solvent_basis": (C.c_int, [I64, D, I32, I32, D, C.c_int, I64, D, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_int, C.c_double, D]),
    "orc_combine_solvent_basis": (None, [I64, D, D, C.c_double, C.c_double, D]),
    "orc_spherical_bessel": (None, [C.c_int, C.c_double, D]),
    "orc_real_harmonics": (None, [C.c_int, C.c_double, C.c_double, D]),
    "orc_multipole_intensity": (C.c_int, [I64, D, I32, I32, D, C.c_int, I64, D, C.c_int, D]),
    "orc_multipole_solvent_basis": (C.c_int, [I64, D, I32, I32, D, C.c_int, I64, D, C.c_int, C.c_double, C.c_double,
                                              C.c_double, C.c_double, C.c_int, C.c_double, D]),
    "orc_multipole_solvent_intensity": (C.c_int, [I64, D, I32, I32, D, C.c_int, I64, D, C.c_int, C.c_double,
                                                  C.c_double, C.c_double, C.c_double, C.c_int, C.c_double, D]),
    "orc_solve_linear": (None, [I64, D, D, D, C.c_int, C.c_double, D, D, D]),
    "orc_solve_scale_background": (None, [I64, D, D, D, C.c_int, C.c_double, C.c_int, C.c_double, D, D, D]),
    "orc_cubic_hermite": (None, [I64, D, D, I64, D, D]),
    "orc_project_simplex": (None, [I64, D, D]),
    "orc_optimize_weights": (None, [I64, I64, D, D, D, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int,
                                    C.c_double, D, D, D, D, D]),
    "orc_solvent_candidates": (None, [C.c_double, C.c_double, C.c_double, C.c_double, D]),
    "orc_reweight_curves": (C.c_int, [I64, I64, D, D, D, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
                                      D, C.c_int, C.c_double, C.c_int, C.c_double, D, D, D, D, D,
                                      C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "orc_chi2_grad": (C.c_int, [I64, D, I32, I32, D, C.c_int, I64, D, D, D, C.c_double, C.c_double, C.c_double,
                                C.c_double, C.c_double, C.c_double, D, D, D]),
    "orc_pair_distance_histogram": (C.c_double, [I64, D, D, I64, D]),
    "orc_normalize_distribution": (C.c_int, [I64, D, D, D, D]),
    "orc_coordinate_features": (C.c_int, [I64, D, I32, I32, D, I64, D, D, D, D, C.POINTER(I64), D, D]),
    "orc_synth_protein": (C.c_int, [C.c_uint64, I64, C.c_double, D, C.POINTER(C.c_int8)]),
}
for _n, (_r, _a) in _SIGS.items():
    _f = getattr(lib, _n)
    _f.restype = _r
    _f.argtypes = _a


def _d(a):
    return a.ctypes.data_as(D)


def _i(a):
    return a.ctypes.data_as(I32)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


class Atoms:
    """Structure arrays for the oracle: xyz [n,3], element, group, occupancy."""

    def __init__(self, xyz, element, group=None, occupancy=None):
        self.xyz = _f64(xyz).reshape(-1, 3)
        n = self.xyz.shape[0]
        self.element = _i32(element).reshape(n)
        self.group = _i32(np.full(n, -1) if group is None else group).reshape(n)
        self.occ = _f64(np.ones(n) if occupancy is None else occupancy).reshape(n)

    @property
    def n(self):
        return self.xyz.shape[0]


def debye_intensity(a: Atoms, q, implicit=True):
    qa = _f64(q)
    out = np.empty(len(qa))
    lib.orc_debye_intensity(a.n, _d(a.xyz), _i(a.element), _i(a.group), _d(a.occ), int(implicit), len(qa), _d(qa),
                            _d(out))
    return out


def debye_partials(xyz, w, types, T, q):
    x, ww, t, qa = _f64(xyz).reshape(-1, 3), _f64(w), _i32(types), _f64(q)
    out = np.empty((T * (T + 1) // 2, len(qa)))
    self_ = np.empty(T)
    lib.orc_debye_partials(x.shape[0], _d(x), _d(ww), _i(t), T, len(qa), _d(qa), _d(out), _d(self_))
    return out, self_


def adaptive_grid(xyz, spacing=4.0, clearance=3.0, padding=12.0):
    x = _f64(xyz).reshape(-1, 3)
    m = C.c_int64()
    vol = C.c_double()
    rc = lib.orc_adaptive_grid(x.shape[0], _d(x), spacing, clearance, padding, None, 0, C.byref(m), C.byref(vol))
    if rc:
        raise ValueError("invalid adaptive grid input")
    sites = np.empty((m.value, 3))
    lib.orc_adaptive_grid(x.shape[0], _d(x), spacing, clearance, padding, _d(sites), m.value, C.byref(m),
                          C.byref(vol))
    return sites, vol.value


def exterior_grid(xyz, element, spacing=1.0, probe=1.4, thickness=3.0):
    x = _f64(xyz).reshape(-1, 3)
    e = _i32(element)
    m = C.c_int64()
    vol = C.c_double()
    rc = lib.orc_exterior_grid(x.shape[0], _d(x), _i(e), spacing, probe, thickness, None, 0, C.byref(m),
                               C.byref(vol))
    if rc:
        raise ValueError("invalid exterior grid input")
    sites = np.empty((m.value, 3))
    lib.orc_exterior_grid(x.shape[0], _d(x), _i(e), spacing, probe, thickness, _d(sites), m.value, C.byref(m),
                          C.byref(vol))
    return sites, vol.value


def debye_solvent_basis(a: Atoms, q, c1=1.0, c2=0.0, thickness=3.0, density=0.334, model=0, spacing=4.0,
                        implicit=True):
    qa = _f64(q)
    out = np.empty((6, len(qa)))
    rc = lib.orc_debye_solvent_basis(a.n, _d(a.xyz), _i(a.element), _i(a.group), _d(a.occ), int(implicit), len(qa),
                                     _d(qa), c1, c2, thickness, density, model, spacing, _d(out))
    if rc:
        raise ValueError("invalid solvent input")
    return out


def combine_solvent_basis(basis, q, c1, c2):
    qa, b = _f64(q), _f64(basis)
    out = np.empty(len(qa))
    lib.orc_combine_solvent_basis(len(qa), _d(qa), _d(b), c1, c2, _d(out))
    return out


def spherical_bessel(l_max, x):
    out = np.empty(l_max + 1)
    lib.orc_spherical_bessel(l_max, x, _d(out))
    return out


def real_harmonics(l_max, cos_theta, phi):
    out = np.empty((l_max + 1) ** 2)
    lib.orc_real_harmonics(l_max, cos_theta, phi, _d(out))
    return out


def multipole_intensity(a: Atoms, q, l_max, implicit=True):
    qa = _f64(q)
    out = np.empty(len(qa))
    lib.orc_multipole_intensity(a.n, _d(a.xyz), _i(a.element), _i(a.group), _d(a.occ), int(implicit), len(qa),
                                _d(qa), l_max, _d(out))
    return out


def multipole_solvent_basis(a: Atoms, q, l_max, c1=1.0, c2=0.0, thickness=3.0, density=0.334, model=0,
                            spacing=4.0, implicit=True):
    qa = _f64(q)
    out = np.empty((6, len(qa)))
    lib.orc_multipole_solvent_basis(a.n, _d(a.xyz), _i(a.element), _i(a.group), _d(a.occ), int(implicit), len(qa),
                                    _d(qa), l_max, c1, c2, thickness, density, model, spacing, _d(out))
    return out


def multipole_solvent_intensity(a: Atoms, q, l_max, c1=1.0, c2=0.0, thickness=3.0, density=0.334, model=0,
                                spacing=4.0, implicit=True):
    qa = _f64(q)
    out = np.empty(len(qa))
    lib.orc_multipole_solvent_intensity(a.n, _d(a.xyz), _i(a.element), _i(a.group), _d(a.occ), int(implicit),
                                        len(qa), _d(qa), l_max, c1, c2, thickness, density, model, spacing, _d(out))
    return out


def solve_linear(theory, y, sigma, bg_mode=0, bg_value=0.0):
    th, yy, ss = _f64(theory), _f64(y), _f64(sigma)
    s, b, c = C.c_double(), C.c_double(), C.c_double()
    lib.orc_solve_linear(len(th), _d(th), _d(yy), _d(ss), bg_mode, bg_value, C.byref(s), C.byref(b), C.byref(c))
    return s.value, b.value, c.value


def cubic_hermite(x, y, t):
    xx, yy, tt = _f64(x), _f64(y), _f64(t)
    out = np.empty(len(tt))
    lib.orc_cubic_hermite(len(xx), _d(xx), _d(yy), len(tt), _d(tt), _d(out))
    return out


def project_simplex(v):
    vv = _f64(v)
    out = np.empty(len(vv))
    lib.orc_project_simplex(len(vv), _d(vv), _d(out))
    return out


def optimize_weights(curves, y, sigma, scale_mode=0, scale_value=0.0, bg_mode=0, bg_value=0.0, uniform=False,
                     regularization=0.0):
    cv, yy, ss = _f64(curves), _f64(y), _f64(sigma)
    K, nq = cv.shape
    w = np.empty(K)
    fitted = np.empty(nq)
    s, b, c = C.c_double(), C.c_double(), C.c_double()
    lib.orc_optimize_weights(K, nq, _d(cv), _d(yy), _d(ss), scale_mode, scale_value, bg_mode, bg_value, int(uniform),
                             regularization, _d(w), C.byref(s), C.byref(b), C.byref(c), _d(fitted))
    return w, s.value, b.value, c.value, fitted


def solvent_candidates(c1_lo, c1_hi, c2_lo, c2_hi):
    out = np.empty(50)
    lib.orc_solvent_candidates(c1_lo, c1_hi, c2_lo, c2_hi, _d(out))
    return out.reshape(25, 2)


def reweight_curves(curves, y, sigma, kl_strength=1.0, max_iterations=500, step_size=0.5, tolerance=1e-8,
                    min_weight=1e-10, prior=None, scale_mode=0, scale_value=0.0, bg_mode=0, bg_value=0.0):
    cv, yy, ss = _f64(curves), _f64(y), _f64(sigma)
    K, nq = cv.shape
    w = np.empty(K)
    s, b, chi, kl = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    it, conv = C.c_int(), C.c_int()
    pr = None if prior is None else _f64(prior)
    rc = lib.orc_reweight_curves(K, nq, _d(cv), _d(yy), _d(ss), kl_strength, max_iterations, step_size, tolerance,
                                 min_weight, None if pr is None else _d(pr), scale_mode, scale_value, bg_mode,
                                 bg_value, _d(w), C.byref(s), C.byref(b), C.byref(chi), C.byref(kl), C.byref(it),
                                 C.byref(conv))
    if rc:
        raise ValueError("invalid reweighting options")
    return dict(weights=w, scale=s.value, background=b.value, reduced_chi2=chi.value, kl=kl.value,
                iterations=it.value, converged=bool(conv.value))


def chi2_grad(a: Atoms, q, y, sigma, c1, c2, scale, background, thickness=3.0, density=0.334, implicit=True,
              want_xyz=True):
    qa, yy, ss = _f64(q), _f64(y), _f64(sigma)
    chi = C.c_double()
    gx = np.empty((a.n, 3)) if want_xyz else None
    gp = np.empty(4)
    lib.orc_chi2_grad(a.n, _d(a.xyz), _i(a.element), _i(a.group), _d(a.occ), int(implicit), len(qa), _d(qa),
                      _d(yy), _d(ss), c1, c2, thickness, density, scale, background, C.byref(chi),
                      None if gx is None else _d(gx), _d(gp))
    return chi.value, gx, gp


def pair_distance_histogram(xyz, w, bins):
    """metrics.rs:475-522: (dmax, raw weighted histogram of `bins` bins)."""
    x, ww = _f64(xyz).reshape(-1, 3), _f64(w)
    hist = np.empty(bins)
    dmax = lib.orc_pair_distance_histogram(x.shape[0], _d(x), _d(ww), bins, _d(hist))
    return dmax, hist


def coordinate_features(a: Atoms, bins=160):
    """metrics.rs:236-270: dict(rg, dmax, r, p, pr_rg, pr_dmax); None fields as NaN."""
    m = max(int(bins), 16)
    r, p = np.empty(m), np.empty(m)
    rg, dmax, prg, pdm = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    used = C.c_int64()
    rc = lib.orc_coordinate_features(a.n, _d(a.xyz), _i(a.element), _i(a.group), _d(a.occ), int(bins),
                                     C.byref(rg), C.byref(dmax), _d(r), _d(p), C.byref(used), C.byref(prg),
                                     C.byref(pdm))
    if rc:
        raise ValueError("coordinate features require a non-empty structure")
    k = used.value
    return dict(rg=rg.value, dmax=dmax.value, r=r[:k].copy(), p=p[:k].copy(), pr_rg=prg.value, pr_dmax=pdm.value)


def synth_protein(seed, n_atoms, radius):
    """The seeded synthetic structure of crabsaxs_b200.synth.protein (same
    generator source, compiled into this library): (xyz [n,3], element int8)."""
    xyz = np.empty((int(n_atoms), 3))
    el = np.empty(int(n_atoms), dtype=np.int8)
    if lib.orc_synth_protein(C.c_uint64(seed), int(n_atoms), float(radius), _d(xyz),
                             el.ctypes.data_as(C.POINTER(C.c_int8))) != 0:
        raise ValueError("invalid synthetic structure request")
    return xyz, el
