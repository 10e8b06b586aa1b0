"""Named benchmark workloads, run a fixed number of times (for profilers).

    python -m crabsaxs_b200.workloads debye-config2 [--variant V] [--repeats N]
    python -m crabsaxs_b200.workloads multipole-config3 [--precision fp32|fp64|tf32|tf32x2] [--repeats N]
    python -m crabsaxs_b200.workloads gradient-config4 [--repeats N]
    python -m crabsaxs_b200.workloads pr-config3 [--bins B] [--repeats N]
    python -m crabsaxs_b200.workloads grid-config2 [--repeats N]

debye-config2: the 20,000-atom synthetic protein plus its adaptive 3 Å
hydration sites, 500 q on [0.001, 0.5], one lattice pair plan (atoms by the
FP32 recurrence kernel, site-site pairs by the exact lattice histogram),
`repeats` launches of the chosen kernel variant (Q*16 + jb; default: the
plan's untuned choice).
multipole-config3: 100,000 atoms (R 80 Å), 1000 q on [0.001, 0.6], L = 50.
gradient-config4: 5,000 atoms (R 28 Å), 100 q, chi^2 and its full gradient.
pr-config3: coordinate features (Rg, Dmax, P(r) with 160 bins) of the
100,000-atom structure of multipole-config3.
grid-config2: the exterior 1 Å hydration grid (1.28 million voxels) and the
adaptive 3 Å grid of the debye-config2 structure, one public call each.
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


def debye_config2(engine: cs.Engine, variant: int | None, repeats: int) -> str:
    w = synth.CONFIG2
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
    return f"debye-config2 variant={variant} step_ms={np.round(ms, 3).tolist()}"


def multipole_config3(engine: cs.Engine, precision: str, repeats: int) -> str:
    w = synth.CONFIG3
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    prec = {"fp64": N.PREC_FP64, "fp32": N.PREC_FP32, "tf32": N.PREC_TF32, "tf32x2": N.PREC_TF32_SPLIT}[precision]
    wall = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        cs.multipole_intensity(s, w.q, 50, precision=prec, engine=engine)
        wall.append((time.perf_counter() - t0) * 1e3)
    return f"multipole-config3 precision={precision} wall_ms={np.round(wall, 3).tolist()}"


def gradient_config4(engine: cs.Engine, repeats: int) -> str:
    w = synth.CONFIG4
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    y = np.ones(len(w.q))
    sigma = np.full(len(w.q), 0.01)
    wall = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        cs.chi2_grad(s, w.q, y, sigma, cs.SolventParams(), 1.0, 0.0, engine=engine)
        wall.append((time.perf_counter() - t0) * 1e3)
    return f"gradient-config4 wall_ms={np.round(wall, 3).tolist()}"


def pr_config3(engine: cs.Engine, bins: int, repeats: int) -> str:
    w = synth.CONFIG3
    s = synth.protein(w.seed, w.n_atoms, w.radius)
    wall, dev, hist = [], [], []
    for _ in range(repeats):
        t0 = time.perf_counter()
        cs.coordinate_features(s, cs.PrOptions(bins=bins), engine=engine)
        wall.append((time.perf_counter() - t0) * 1e3)
        total_ms, hist_ms, pairs, mode = cs.pr_last_timing(engine)
        dev.append(total_ms)
        hist.append(hist_ms)
    return (f"pr-config3 bins={bins} mode={mode} pairs={pairs:.6g} wall_ms={np.round(wall, 3).tolist()} "
            f"device_ms={np.round(dev, 3).tolist()} histogram_ms={np.round(hist, 3).tolist()}")


def grid_config2(engine: cs.Engine, repeats: int) -> str:
    w = synth.CONFIG2
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
    return (f"grid-config2 exterior_sites={len(sites_e)} adaptive_sites={len(sites_a)} "
            f"exterior_wall_ms={np.round(ext, 3).tolist()} adaptive_wall_ms={np.round(ada, 3).tolist()}")


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(prog="python -m crabsaxs_b200.workloads", description=__doc__.splitlines()[0])
    ap.add_argument("workload",
                    choices=["debye-config2", "multipole-config3", "gradient-config4", "pr-config3", "grid-config2"])
    ap.add_argument("--bins", type=int, default=160)
    ap.add_argument("--variant", type=int, default=None)
    ap.add_argument("--precision", choices=["fp32", "fp64", "tf32", "tf32x2"], default="tf32x2")
    ap.add_argument("--repeats", type=int, default=2)
    a = ap.parse_args(argv)
    engine = cs.Engine.default(0)
    if a.workload == "debye-config2":
        print(debye_config2(engine, a.variant, a.repeats))
    elif a.workload == "multipole-config3":
        print(multipole_config3(engine, a.precision, a.repeats))
    elif a.workload == "pr-config3":
        print(pr_config3(engine, a.bins, a.repeats))
    elif a.workload == "grid-config2":
        print(grid_config2(engine, a.repeats))
    else:
        print(gradient_config4(engine, a.repeats))


if __name__ == "__main__":
    main()
