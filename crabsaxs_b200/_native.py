"""ctypes binding of libcrabsaxs_b200.so (the C ABI in include/crab_cuda.h).

Importing this module loads the in-tree shared library.  There is no
fallback: if the library is missing or cannot be loaded the import fails with
an error that says how to build it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcrabsaxs_b200.so"

if not LIB_PATH.exists():
    raise ImportError(f"{LIB_PATH} is missing: build it with `python crabsaxs_b200/build.py`")
lib = C.CDLL(str(LIB_PATH))

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, ENOTCONV, ECAPACITY, ENODEVICE, EPARSE, EELEMENT, EIO = range(11)
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "ECUDA", 4: "ETIMEOUT", 5: "ENOTCONV", 6: "ECAPACITY",
                7: "ENODEVICE", 8: "EPARSE", 9: "EELEMENT", 10: "EIO"}
FORMAT_AUTO, FORMAT_PDB, FORMAT_MMCIF = 0, 1, 2
ALTLOC_HIGHEST, ALTLOC_FIRST, ALTLOC_ALL = 0, 1, 2
OCC_REPORTED, OCC_SELECTED_FULL = 0, 1

HYD_ANALYTIC, HYD_GRID, HYD_ADAPTIVE = 0, 1, 2
METHOD_AUTO, METHOD_DEBYE, METHOD_MULTIPOLE = 0, 1, 2
PREC_FP64, PREC_TF32, PREC_BF16, PREC_BF16_SPLIT, PREC_TF32_SPLIT, PREC_FP32 = 0, 1, 2, 3, 4, 5
PREC_TF32_FUSED, PREC_TF32_SPLIT_FUSED = 6, 7
SCALE_FIT, SCALE_FIXED = 0, 1
BG_FIT, BG_FIXED_ZERO, BG_FIXED = 0, 1, 2


class ParseOpts(C.Structure):
    _fields_ = [("include_hetatm", C.c_int32), ("include_waters", C.c_int32), ("include_glycans", C.c_int32),
                ("model_index", C.c_int32), ("allow_unknown_elements", C.c_int32),
                ("occupancy_policy", C.c_int32), ("altloc_policy", C.c_int32), ("n_chains", C.c_int32),
                ("chains", C.POINTER(C.c_char_p))]


class Solvent(C.Structure):
    _fields_ = [("c1", C.c_double), ("c2", C.c_double), ("shell_thickness", C.c_double),
                ("bulk_density", C.c_double), ("hydration_model", C.c_int32), ("_pad", C.c_int32),
                ("grid_spacing", C.c_double)]


class ComputeOpts(C.Structure):
    _fields_ = [("method", C.c_int32), ("implicit_hydrogen", C.c_int32), ("l_max", C.c_int32),
                ("has_solvent", C.c_int32), ("solvent", Solvent)]


class FitOpts(C.Structure):
    _fields_ = [("method", C.c_int32), ("implicit_hydrogen", C.c_int32), ("c1_lo", C.c_double),
                ("c1_hi", C.c_double), ("c2_lo", C.c_double), ("c2_hi", C.c_double),
                ("max_iterations", C.c_int32), ("q_sampling_stride", C.c_int32), ("solvent", Solvent),
                ("scale_mode", C.c_int32), ("bg_mode", C.c_int32), ("scale_value", C.c_double),
                ("bg_value", C.c_double), ("optimizer", C.c_int32), ("_pad", C.c_int32)]


class FitResult(C.Structure):
    _fields_ = [("scale", C.c_double), ("background", C.c_double), ("c1", C.c_double), ("c2", C.c_double),
                ("chi2", C.c_double), ("iterations", C.c_int32), ("converged", C.c_int32)]


class EnsembleOpts(C.Structure):
    _fields_ = [("fit_weights", C.c_int32), ("uniform", C.c_int32), ("regularization", C.c_double),
                ("max_conformers", C.c_int32), ("bootstrap", C.c_int32), ("min_weight", C.c_double),
                ("seed", C.c_uint64)]


class EnsembleResult(C.Structure):
    _fields_ = [("scale", C.c_double), ("background", C.c_double), ("c1", C.c_double), ("c2", C.c_double),
                ("chi2", C.c_double), ("reduced_chi2", C.c_double), ("iterations", C.c_int32),
                ("n_selected", C.c_int32)]


class ReweightOpts(C.Structure):
    _fields_ = [("kl_strength", C.c_double), ("step_size", C.c_double), ("tolerance", C.c_double),
                ("min_weight", C.c_double), ("max_iterations", C.c_int32), ("scale_mode", C.c_int32),
                ("bg_mode", C.c_int32), ("_pad", C.c_int32), ("scale_value", C.c_double), ("bg_value", C.c_double)]


class ReweightResult(C.Structure):
    _fields_ = [("scale", C.c_double), ("background", C.c_double), ("chi2", C.c_double),
                ("reduced_chi2", C.c_double), ("kl_divergence", C.c_double), ("effective_sample_size", C.c_double),
                ("iterations", C.c_int32), ("converged", C.c_int32)]


P = C.c_void_p
D = C.POINTER(C.c_double)
I64 = C.c_int64
I32P = C.POINTER(C.c_int32)
I8P = C.POINTER(C.c_int8)

# crab_sum_fn: in-place sum over GPUs of a host buffer of doubles
SUM_FN = C.CFUNCTYPE(C.c_int, D, I64, P)

_SIGS = {
    "crab_ctx_create": (C.c_int, [C.c_int, C.POINTER(P)]),
    "crab_ctx_destroy": (C.c_int, [P]),
    "crab_ctx_last_error": (C.c_char_p, [P]),
    "crab_ctx_stats": (C.c_int, [P, C.POINTER(I64), D, D]),
    "crab_ctx_reset_stats": (C.c_int, [P]),
    "crab_ctx_workspace_bytes": (C.c_int, [P, C.POINTER(I64)]),
    "crab_ctx_set_wait_budget": (C.c_int, [P, I64]),
    "crab_ctx_fail_allocations": (C.c_int, [P, I64]),
    "crab_ctx_set_device_sums": (C.c_int, [P, C.c_int32]),
    "crab_united_atom_group": (C.c_int, [C.c_char_p, C.c_char_p]),
    "crab_form_factor": (C.c_double, [C.c_int, C.c_int, C.c_double, C.c_int, C.c_double]),
    "crab_excluded_volume_for_atom": (C.c_double, [C.c_int, C.c_int, C.c_int]),
    "crab_structure_create": (C.c_int, [P, D, D, I8P, I8P, I64, C.POINTER(P)]),
    "crab_structure_destroy": (C.c_int, [P]),
    "crab_structure_atom_count": (I64, [P]),
    "crab_debye_intensity": (C.c_int, [P, P, D, I64, C.c_int, D]),
    "crab_debye_solvent_basis": (C.c_int, [P, P, D, I64, C.POINTER(Solvent), C.c_int, D]),
    "crab_debye_solvent_basis_ex": (C.c_int, [P, P, D, I64, C.POINTER(Solvent), C.c_int, C.c_int, D]),
    "crab_combine_solvent_basis": (C.c_int, [D, I64, D, C.c_double, C.c_double, D]),
    "crab_debye_partials": (C.c_int, [P, D, D, I32P, I64, C.c_int32, D, I64, D, D]),
    "crab_debye_partials_fp64": (C.c_int, [P, D, D, I32P, I64, C.c_int32, D, I64, D, D]),
    "crab_debye_partials_shard": (C.c_int, [P, D, D, I32P, I64, C.c_int32, D, I64, C.c_int, C.c_int, C.c_int,
                                            D, D]),
    "crab_debye_solvent_basis_shard": (C.c_int, [P, P, D, I64, C.POINTER(Solvent), C.c_int, C.c_int, C.c_int,
                                                 C.c_int, D]),
    "crab_shard_assign": (C.c_int, [C.POINTER(I64), I64, C.c_int32, I32P]),
    "crab_compute_curve": (C.c_int, [P, P, D, I64, C.POINTER(ComputeOpts), D, I32P]),
    "crab_hydration_grid_adaptive": (C.c_int, [P, P, C.c_double, C.c_double, C.c_double, D, I64,
                                               C.POINTER(I64), D]),
    "crab_hydration_grid_exterior": (C.c_int, [P, P, C.c_double, C.c_double, C.c_double, D, I64,
                                               C.POINTER(I64), D]),
    "crab_hydration_grid_adaptive_noalloc": (C.c_int, [D, I64, C.c_double, C.c_double, C.c_double, D, I64,
                                                       C.POINTER(I64), D, P]),
    "crab_multipole_intensity": (C.c_int, [P, P, D, I64, C.c_int, C.c_int, C.c_int, D]),
    "crab_multipole_solvent_basis": (C.c_int, [P, P, D, I64, C.c_int, C.POINTER(Solvent), C.c_int, C.c_int, D]),
    "crab_multipole_last_timing": (C.c_int, [P, D, D, D]),
    "crab_multipole_intensity_shard": (C.c_int, [P, P, D, I64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, SUM_FN,
                                                 P, D]),
    "crab_multipole_solvent_basis_shard": (C.c_int, [P, P, D, I64, C.c_int, C.POINTER(Solvent), C.c_int, C.c_int,
                                                     C.c_int, C.c_int, SUM_FN, P, D]),
    "crab_fit": (C.c_int, [P, P, D, D, D, I64, C.POINTER(FitOpts), C.c_double, C.c_double,
                           C.POINTER(FitResult), D]),
    "crab_chi2_grad": (C.c_int, [P, P, D, D, D, I64, C.POINTER(Solvent), C.c_int, C.c_double, C.c_double, D, D, D]),
    "crab_ensemble_fit": (C.c_int, [P, C.POINTER(P), C.c_int32, D, D, D, I64, C.POINTER(EnsembleOpts),
                                    C.POINTER(FitOpts), C.POINTER(EnsembleResult), I32P, D, D, D, D]),
    "crab_ensemble_partials": (C.c_int, [P, C.POINTER(P), C.c_int32, D, I64, C.c_int, C.c_int, C.c_int, I32P, D,
                                         I64]),
    "crab_ensemble_fit_partials": (C.c_int, [P, C.POINTER(P), C.c_int32, D, D, D, I64, C.POINTER(EnsembleOpts),
                                             C.POINTER(FitOpts), D, C.c_int32, C.POINTER(EnsembleResult), I32P, D,
                                             D, D, D]),
    "crab_ensemble_plan_create": (C.c_int, [P, C.POINTER(P), C.c_int32, D, I64, C.POINTER(Solvent), C.c_int, D,
                                            C.c_int32, C.POINTER(P)]),
    "crab_ensemble_plan_autotune": (C.c_int, [P, P, I32P]),
    "crab_ensemble_plan_score": (C.c_int, [P, P, D, D, C.POINTER(FitOpts), C.POINTER(ReweightOpts), D, D, D, D,
                                           D, D]),
    "crab_ensemble_plan_destroy": (C.c_int, [P]),
    "crab_ensemble_curves": (C.c_int, [P, C.POINTER(P), C.c_int32, D, I64, C.POINTER(Solvent), C.c_int, D,
                                       C.c_int32, D]),
    "crab_reweight_curves": (C.c_int, [D, C.c_int32, D, D, D, I64, D, C.POINTER(ReweightOpts), D,
                                       C.POINTER(ReweightResult)]),
    "crab_synth_protein": (C.c_int, [C.c_uint64, I64, C.c_double, D, I8P]),
    "crab_pair_distance_histogram": (C.c_int, [P, D, D, I64, I64, D, D]),
    "crab_parse_options_default": (None, [C.POINTER(ParseOpts)]),
    "crab_parse_last_error": (C.c_char_p, []),
    "crab_parse_structure": (C.c_int, [C.c_char_p, I64, C.c_int32, C.POINTER(ParseOpts), C.POINTER(P)]),
    "crab_parse_model_count": (C.c_int, [C.c_char_p, I64, C.c_int32, C.POINTER(C.c_int32)]),
    "crab_read_structure_file": (C.c_int, [C.c_char_p, C.POINTER(ParseOpts), C.POINTER(P)]),
    "crab_parsed_atom_count": (I64, [P]),
    "crab_parsed_arrays": (C.c_int, [P, D, D, I8P, I8P, I8P, C.POINTER(I64)]),
    "crab_parsed_atom_name": (C.c_char_p, [P, I64]),
    "crab_parsed_residue_name": (C.c_char_p, [P, I64]),
    "crab_parsed_chain_id": (C.c_char_p, [P, I64]),
    "crab_parsed_strings": (C.c_int, [P, C.c_int32, C.c_char_p, I64, C.POINTER(I64)]),
    "crab_parsed_destroy": (C.c_int, [P]),
    "crab_structure_from_parsed": (C.c_int, [P, P, C.POINTER(P)]),
    "crab_coordinate_features": (C.c_int, [P, P, I64, D, D, D, D, C.POINTER(I64), D, D]),
    "crab_pr_last_timing": (C.c_int, [P, D, D, D, C.POINTER(C.c_int32)]),
    "crab_pair_plan_create": (C.c_int, [P, D, D, I32P, I64, C.c_int32, D, I64, C.POINTER(P)]),
    "crab_pair_plan_create_lattice": (C.c_int, [P, D, D, I32P, I64, C.c_int32, D, I64, I32P, I64, C.c_double,
                                                C.POINTER(P)]),
    "crab_pair_plan_create_lattice_shard": (C.c_int, [P, D, D, I32P, I64, C.c_int32, D, I64, I32P, I64, C.c_double,
                                                      C.c_int32, C.c_int32, C.POINTER(P)]),
    "crab_pair_plan_run": (C.c_int, [P, P, C.c_int32, I64, D]),
    "crab_pair_plan_autotune": (C.c_int, [P, P, I32P, I32P, D, C.c_int32, I32P]),
    "crab_pair_plan_select": (C.c_int, [P, P, C.c_int32]),
    "crab_ctx_set_pair_variant": (C.c_int, [P, C.c_int32]),
    "crab_pair_plan_read": (C.c_int, [P, P, D, D]),
    "crab_pair_plan_pairq": (C.c_double, [P]),
    "crab_pair_plan_destroy": (C.c_int, [P]),
    "crab_measure_fp32_peak": (C.c_int, [P, C.c_double, D]),
    "crab_ctx_transfer_stats": (C.c_int, [P, C.POINTER(I64), C.POINTER(I64)]),
}

for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args

EXPORTED = tuple(_SIGS)
