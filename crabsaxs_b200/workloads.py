"""Named benchmark workloads, run a fixed number of times (for profilers).

    python -m crabsaxs_b200.workloads debye-20k [--variant V] [--repeats N]
    python -m crabsaxs_b200.workloads multipole-100k [--precision fp32|fp64|tf32|tf32x2|tf32x2-fused|bf16|bf16x2]
                                      [--repeats N]
    python -m crabsaxs_b200.workloads gradient-5k [--repeats N]
    python -m crabsaxs_b200.workloads pr-100k [--bins B] [--repeats N]
    python -m crabsaxs_b200.workloads grid-20k [--repeats N]

debye-20k: the 20,000-atom synthetic protein plus its adaptive 3 Å
hydration sites, 500 q on [0.001, 0.5], one lattice pair plan (atoms by the
FP32 recurrence kernel, site-site pairs by the exact lattice histogram),
`repeats` launches of the chosen kernel variant (Q*16 + jb; default: the
plan's untuned choice).
multipole-100k: 100,000 atoms (R 80 Å), 1000 q on [0.001, 0.6], L = 50.
gradient-5k: 5,000 atoms (R 28 Å), 100 q, chi^2 and its full gradient.
pr-100k: coordinate features (Rg, Dmax, P(r) with 160 bins) of the
100,000-atom structure of multipole-100k.
grid-20k: the exterior 1 Å hydration grid (1.28 million voxels) and the
adaptive 3 Å grid of the debye-20k structure, one public call each.
Each prints one line with its device or wall times.
"""
from __future__ import annotations

import argparse
import ctypes as C
import time

import numpy as np

from . import _native as N
from . import api as cs
from . import synth


def debye_20k(engine: cs.Engine, variant: int | None, repeats: int) -> str:
    w = synth.DEBYE_20K_SOLVATED
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    sites, _ = cs.hydration_grid_adaptive(s, 3.0, engine=engine)
    el = s.element.astype(np.int64)
    classes = sorted(set(el.tolist()))
    t = np.concatenate([np.searchsorted(classes, el), np.full(len(sites), len(classes))]).astype(np.int32)
    xyz = np.ascontiguousarray(np.concatenate([s.xyz, sites]))
    wts = np.ones(len(xyz))
    T = len(classes) + 1
    cells = np.ascontiguousarray(np.rint((sites - sites.min(axis=0)) / 3.0).astype(np.int32))
    q = np.ascontiguousarray(w.q)
    plan = C.c_void_p()
    engine.check(N.lib.crab_pair_plan_create_lattice(engine.handle, xyz.ctypes.data_as(N.D), wts.ctypes.data_as(N.D),
                                                     t.ctypes.data_as(N.I32P), len(wts), T, q.ctypes.data_as(N.D),
                                                     len(q), cells.ctypes.data_as(N.I32P), len(sites), 3.0,
                                                     C.byref(plan)))
    try:
        if variant is not None:
            engine.check(N.lib.crab_pair_plan_select(engine.handle, plan, variant))
        ms = np.zeros(repeats)
        engine.check(N.lib.crab_pair_plan_run(engine.handle, plan, repeats, 0, ms.ctypes.data_as(N.D)))
    finally:
        N.lib.crab_pair_plan_destroy(plan)
    return f"debye-20k variant={variant} step_ms={np.round(ms, 3).tolist()}"


def multipole_100k(engine: cs.Engine, precision: str, repeats: int) -> str:
    w = synth.ATOMS_100K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    prec = {"fp64": N.PREC_FP64, "fp32": N.PREC_FP32, "tf32": N.PREC_TF32, "tf32x2": N.PREC_TF32_SPLIT,
            "tf32x2-fused": N.PREC_TF32_SPLIT_FUSED, "bf16": N.PREC_BF16, "bf16x2": N.PREC_BF16_SPLIT}[precision]
    wall = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        cs.multipole_intensity(s, w.q, 50, precision=prec, engine=engine)
        wall.append((time.perf_counter() - t0) * 1e3)
    return f"multipole-100k precision={precision} wall_ms={np.round(wall, 3).tolist()}"


def gradient_5k(engine: cs.Engine, repeats: int) -> str:
    w = synth.GRADIENT_5K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    y = np.ones(len(w.q))
    sigma = np.full(len(w.q), 0.01)
    wall = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        cs.chi2_grad(s, w.q, y, sigma, cs.SolventParams(), 1.0, 0.0, engine=engine)
        wall.append((time.perf_counter() - t0) * 1e3)
    return f"gradient-5k wall_ms={np.round(wall, 3).tolist()}"


def pr_100k(engine: cs.Engine, bins: int, repeats: int) -> str:
    w = synth.ATOMS_100K
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    wall, dev, hist = [], [], []
    for _ in range(repeats):
        t0 = time.perf_counter()
        cs.coordinate_features(s, cs.PrOptions(bins=bins), engine=engine)
        wall.append((time.perf_counter() - t0) * 1e3)
        total_ms, hist_ms, pairs, mode = cs.pr_last_timing(engine)
        dev.append(total_ms)
        hist.append(hist_ms)
    return (f"pr-100k bins={bins} mode={mode} pairs={pairs:.6g} wall_ms={np.round(wall, 3).tolist()} "
            f"device_ms={np.round(dev, 3).tolist()} histogram_ms={np.round(hist, 3).tolist()}")


def grid_20k(engine: cs.Engine, repeats: int) -> str:
    w = synth.DEBYE_20K_SOLVATED
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    ext, ada = [], []
    for _ in range(repeats):
        t0 = time.perf_counter()
        sites_e, _ = cs.hydration_grid_exterior(s, engine=engine)
        t1 = time.perf_counter()
        sites_a, _ = cs.hydration_grid_adaptive(s, 3.0, engine=engine)
        t2 = time.perf_counter()
        ext.append((t1 - t0) * 1e3)
        ada.append((t2 - t1) * 1e3)
    return (f"grid-20k exterior_sites={len(sites_e)} adaptive_sites={len(sites_a)} "
            f"exterior_wall_ms={np.round(ext, 3).tolist()} adaptive_wall_ms={np.round(ada, 3).tolist()}")


def parser() -> argparse.ArgumentParser:
    ap = argparse.ArgumentParser(prog="python -m crabsaxs_b200.workloads", description=__doc__.splitlines()[0])
    ap.add_argument("workload",
                    choices=["debye-20k", "multipole-100k", "gradient-5k", "pr-100k", "grid-20k"])
    ap.add_argument("--bins", type=int, default=160)
    ap.add_argument("--variant", type=int, default=None)
    ap.add_argument("--precision", choices=["fp32", "fp64", "tf32", "tf32x2", "tf32x2-fused", "bf16", "bf16x2"],
                    default="tf32x2")
    ap.add_argument("--repeats", type=int, default=2)
    return ap


def main(argv=None) -> None:
    a = parser().parse_args(argv)
    engine = cs.Engine.default(0)
    if a.workload == "debye-20k":
        print(debye_20k(engine, a.variant, a.repeats))
    elif a.workload == "multipole-100k":
        print(multipole_100k(engine, a.precision, a.repeats))
    elif a.workload == "pr-100k":
        print(pr_100k(engine, a.bins, a.repeats))
    elif a.workload == "grid-20k":
        print(grid_20k(engine, a.repeats))
    else:
        print(gradient_5k(engine, a.repeats))


if __name__ == "__main__":
    main()
