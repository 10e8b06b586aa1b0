#!/usr/bin/env python
"""Throughput of the crabSAXS scattering hot path on B200.

Workload (one step): the per-atom-type-pair Debye pair sums of a 20,000-atom
seeded protein-like structure (radius 45 Å, C/N/O/S) plus its adaptive
hydration shell on a 3 Å grid, at 500 uniform q values on [0.001, 0.5] Å⁻¹
(the scale configuration of the Debye engine).  Unit: pair·q evaluations per
second, pairs = M(M-1)/2 over the M atoms + sites.

* ``value``: the pair sums on device-resident inputs (a pair plan: the FP32
  pair kernel for atom–atom and atom–site pairs, the exact lattice histogram
  for site–site pairs), timed with CUDA events on the launch stream, L2
  flushed (256 MiB memset) before every step outside the events.
* ``e2e``: the public C-ABI call ``crab_debye_solvent_basis`` from pinned host
  buffers (structure upload, hydration grid, pair sums, partials read back),
  wall-clocked per step.
* ``roofline``: 4 FLOP per pair·q (recurrence step + weighted accumulate)
  against the FP32 FMA peak measured in this run.
* ``cpu_baseline``: the oracle (C++ f64 restatement of the reference CPU
  algorithm) on all host threads, on a q subset of the same workload.

``--impl reference`` times that CPU restatement alone (the reference crate is
Rust and cannot be built here) with the same metric.  Under torchrun the one
structure is split over the GPUs (strong scaling): every rank takes the work
items crab_shard_assign gives it (crab_pair_plan_create_lattice_shard), and
each step ends with one NCCL all-reduce of the 60 KB of partials (in ``e2e``:
of the six-term basis); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "pair·q/s (Debye); batched χ²+∇ curves/s vs plain GPU; both at ≤1e-5 rel err"
WORKLOAD = "debye pair sums per type pair, 20k-atom structure + adaptive 3 Å hydration sites, 500 q on [0.001, 0.5]"
UNIT = "pair·q/s"
N_ATOMS, RADIUS, SEED = 20000, 45.0, 2
Q = np.linspace(0.001, 0.5, 500)
FLUSH_BYTES = 256 << 20



def _variant_name(v: int) -> str:
    """Autotuner variant code Q*16 + jb; jb >= 8 is the q-packed kernel with (jb-8) % 4 chains,
    jb >= 12 its build for three CTAs per SM; jb 5, 6, 7, 3 the q-packed kernel with the weight
    folded into the recurrence (1 chain / 2 CTAs, 2 / 2, 1 / 3, 1 / 4); jb 11 the folded kernel with
    two chains per pair (q points 4n, 4n+1 and 4n+2, 4n+3); jb 14, 15 the folded
    recurrence with the set-up in its own warpgroup (1 or 2 chains per recurrence thread), jb 12
    the same with one recurrence warpgroup per q block, three blocks per work item."""
    q, jb = int(v) // 16, int(v) % 16
    if jb in (14, 15):
        return f"Q{q}xJ{jb - 13}-split"
    if jb == 12:
        return f"Q{q}x3blocks-split"
    if jb == 11:
        return f"Q{q}xJ1pq-fold-2chain-2cta"
    folded = {5: (1, 2), 6: (2, 2), 7: (1, 3), 3: (1, 4)}
    if jb in folded:
        chains, ctas = folded[jb]
        return f"Q{q}xJ{chains}pq-fold-{ctas}cta"
    if jb < 8:
        return f"Q{q}xJ{jb}"
    return f"Q{q}xJ{(jb - 8) % 4}pq" + ("-3cta" if jb >= 12 else "")

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


class Dist:
    def __init__(self, world: int, backend: str):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self._dev())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self.world == 1:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self._dev())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def _dev(self):
        import torch

        return f"cuda:{torch.cuda.current_device()}" if self.dist.get_backend() == "nccl" else "cpu"

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 7 and parts[0].replace(".", "").isdigit():
                    rows.append(parts)
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].lower() == "active"})
        busy = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": float(rows[0][1]), "reasons": reasons,
                "samples": len(rows)}


def workload(rank: int):
    """The seeded 20,000-atom structure (rank 0's; the other seeds make the per-rank
    structures of the auxiliary sections)."""
    import crabsaxs_b200 as cs
    from crabsaxs_b200 import synth

    s = synth.protein(SEED + 1000 * rank, N_ATOMS, RADIUS)
    return s


def typed_arrays(s, sites):
    # scattering types: C, N, O, S (element Cromer–Mann classes) and the water site W
    el = s.element.astype(np.int64)
    classes = sorted(set(el.tolist()))
    t_atoms = np.searchsorted(classes, el)
    xyz = np.concatenate([s.xyz, sites])
    w = np.concatenate([s.occupancy, np.ones(len(sites))])
    t = np.concatenate([t_atoms, np.full(len(sites), len(classes))]).astype(np.int32)
    return xyz, w, t, len(classes) + 1


def traffic_per_launch():
    """DRAM bytes per pair-kernel launch from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "debye_pair_fp32_20k_500q.txt"
    if not p.exists():
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) if m else None


def cpu_baseline_run(s, threads: int, fraction: float = 1.0):
    """Oracle f64 Debye solvent basis (adaptive 3 Å grid built inside, as
    solvent.rs:504-584 does) on `threads` q values, one per thread, over a
    seeded `fraction` of the atoms.  Returns (pair·q/s, q values, seconds, atoms+sites)."""
    import oracle as O

    idx = np.arange(s.atom_count)
    if fraction < 1.0:
        idx = np.sort(np.random.default_rng(0).choice(s.atom_count, int(fraction * s.atom_count), replace=False))
    a = O.Atoms(s.xyz[idx], s.element[idx], s.group[idx], s.occupancy[idx])
    sites, _ = O.adaptive_grid(a.xyz, 3.0)
    sub = Q[np.linspace(0, len(Q) - 1, threads).astype(int)]
    m = len(idx) + len(sites)
    t0 = time.perf_counter()
    O.debye_solvent_basis(a, sub, 1.0, 0.0, model=2, spacing=3.0)
    dt = time.perf_counter() - t0
    return (m * (m - 1) / 2.0) * len(sub) / dt, len(sub), dt, m


class _OracleStructure:
    """The workload structure as plain arrays (the fields cpu_baseline_run reads)."""

    def __init__(self, xyz, element):
        self.xyz = xyz
        self.element = element
        self.group = np.full(len(element), -1, dtype=np.int8)
        self.occupancy = np.ones(len(element))
        self.atom_count = len(element)


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle as O

    # the same seeded structure as the GPU arm's, made by the oracle library
    # (this arm loads no product code)
    s = _OracleStructure(*O.synth_protein(SEED, N_ATOMS, RADIUS))
    n_sites = len(O.adaptive_grid(s.xyz, 3.0)[0])  # the workload's sites (the timed sample is half the atoms)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_baseline_run(s, threads, 0.5)
    vals, times = [], []
    for _ in range(args.steps):
        v, nq, dt, m = cpu_baseline_run(s, threads, 0.5)
        vals.append(v)
        times.append(dt)
    value = float(np.median(vals))
    sample = (f"seeded half of the 20,000-atom structure with its adaptive 3 Å sites ({m} points), {threads} of "
              f"the 500 q values (one per thread), f64 C++ restatement of solvent.rs debye_solvent_basis")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_atoms": N_ATOMS, "n_sites": int(n_sites), "n_q": len(Q)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def ensemble_section(eng, rank, with_cpu=False):
    """Ensemble of 256 conformers (log-uniform 2k-40k atoms), 300 q, the 25 (c1, c2)
    candidates of ensemble.rs:302-315.  Batched: one CUDA graph per scoring pass
    (pair sums of all conformers, 25x256 curves, per-candidate simplex weights,
    gradients, KL reweighting).  Plain: one compute_curve per conformer per
    candidate, the call structure of ensemble.rs:244-261, timed for one candidate
    (each further candidate repeats the same work)."""
    import crabsaxs_b200 as cs
    from crabsaxs_b200 import synth

    confs = synth.ensemble(256, 5 + 7919 * rank)
    q = synth.ENSEMBLE_Q
    fo = cs.FitOptions(method=cs.ScatteringMethod.Debye)
    cand = cs.solvent_candidates(fo)
    rng = np.random.default_rng(55)
    hidden = rng.choice(len(confs), 8, replace=False)
    opt0 = cs.ComputeOptions(method=cs.ScatteringMethod.Debye, solvent=cs.SolventParams())
    ih = np.array([cs.compute_curve(confs[h], q, opt0, engine=eng).intensity for h in hidden])
    clean = rng.dirichlet(np.ones(8)) @ ih
    sigma = 0.01 * clean
    y = clean + sigma * rng.normal(size=len(q))
    plan = cs.EnsemblePlan(confs, q, cs.SolventParams(), cand, engine=eng)
    try:
        plan.score(y, sigma, fo, cs.MaximumEntropyOptions())
        eng.reset_stats()
        runs = [plan.score(y, sigma, fo, cs.MaximumEntropyOptions()) for _ in range(3)]
        launches, _, _ = eng.stats()
    finally:
        plan.close()
    graph_ms = float(np.median([r["elapsed_ms"] for r in runs]))
    n_curves = len(cand) * len(confs)
    # plain per-structure GPU path for one candidate, wall-clocked end to end
    c1, c2 = cand[12]
    optc = cs.ComputeOptions(method=cs.ScatteringMethod.Debye, solvent=cs.SolventParams(c1=c1, c2=c2))
    t0 = time.perf_counter()
    plain = [cs.compute_curve(c, q, optc, engine=eng).intensity for c in confs]
    plain_s = time.perf_counter() - t0
    # accuracy of batched curves against the FP64 device reference on four conformers
    order = np.argsort([c.atom_count for c in confs])
    pick = [order[0], order[len(order) // 3], order[2 * len(order) // 3], order[-1]]
    bc = cs.ensemble_curves([confs[i] for i in pick], q, cs.SolventParams(), [[c1, c2]], engine=eng)[0]
    err = 0.0
    for j, i in enumerate(pick):
        b64 = cs.debye_solvent_basis(confs[i], q, cs.SolventParams(c1=c1, c2=c2), engine=eng, fp64=True)
        i64 = cs.combine_solvent_basis(b64, q, c1, c2)
        err = max(err, float(np.max(np.abs(bc[j] - i64) / i64)), float(np.max(np.abs(plain[i] - i64) / i64)))
    pairq = sum(c.atom_count * (c.atom_count - 1) / 2.0 for c in confs) * len(q)
    best = runs[-1]
    cpu = None
    if with_cpu and rank == 0:
        import oracle as O

        t0 = time.perf_counter()
        for i in order[:4]:
            cc = confs[i]
            O.debye_solvent_basis(O.Atoms(cc.xyz, cc.element, cc.group, cc.occupancy), q, c1, c2)
        dt = time.perf_counter() - t0
        cpu = {"value": 4 / dt, "unit": "curves/s", "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"the 4 smallest conformers ({', '.join(str(confs[i].atom_count) for i in order[:4])} atoms), "
                         f"one f64 Debye solvent evaluation per curve as the reference's per-candidate "
                         f"compute_curve does, {dt:.1f} s"}
    return {"curves_per_s": n_curves / (graph_ms * 1e-3), "plain_gpu_curves_per_s": len(confs) / plain_s,
            "speedup_vs_plain": (n_curves / (graph_ms * 1e-3)) / (len(confs) / plain_s),
            "graph_ms": graph_ms, "conformers": len(confs), "candidates": len(cand), "n_q": len(q),
            "atoms": int(sum(c.atom_count for c in confs)), "pair_q_per_pass": pairq,
            "pair_q_per_s": pairq / (graph_ms * 1e-3), "kernels_per_pass": int(launches // 3),
            "max_rel_err_vs_fp64": err, "best_candidate": [float(best["c1"]), float(best["c2"])], "cpu_baseline": cpu,
            "reduced_chi2": float(best["reduced_chi2"]), "kl_reduced_chi2": float(best["kl_reduced_chi2"])}


def multipole_section(eng, rank, fp32_peak, with_cpu=False):
    """100,000 atoms (R 80 Å), 1000 q on [0.001, 0.6], L = 50.  The
    default path runs the moment GEMM on tcgen05 tensor cores (TF32 hi+lo, 3
    products per K step); the FP32 SIMT GEMM is timed beside it.  Reports the
    call's wall and device time, each GEMM against its peak, the error against
    the FP64 device multipole (all q; precision) and against FP64 Debye (every
    50th q; truncation of the expansion at L), and the 20,000-atom solvent curve by
    multipole (L = 30) for comparison with Debye."""
    import crabsaxs_b200 as cs
    from crabsaxs_b200 import _native as N
    from crabsaxs_b200 import synth

    w = synth.ATOMS_100K
    s = synth.protein(w.seed + 1000 * rank, w.n_atoms, w.radius)
    L = 50
    tot, gm, fl = C.c_double(), C.c_double(), C.c_double()

    def timed(prec):
        cs.multipole_intensity(s, w.q, L, precision=prec, engine=eng)
        walls, dev, gemm = [], [], []
        for _ in range(5):
            t0 = time.perf_counter()
            out = cs.multipole_intensity(s, w.q, L, precision=prec, engine=eng)
            walls.append((time.perf_counter() - t0) * 1e3)
            eng.check(N.lib.crab_multipole_last_timing(eng.handle, C.byref(tot), C.byref(gm), C.byref(fl)))
            dev.append(tot.value)
            gemm.append(gm.value)
        return out, float(np.median(walls)), float(np.median(dev)), float(np.median(gemm)), fl.value

    tc, tc_wall, tc_dev, tc_gemm, flop = timed(N.PREC_TF32_SPLIT)
    f32, f32_wall, f32_dev, f32_gemm, _ = timed(N.PREC_FP32)
    f64 = cs.multipole_intensity(s, w.q, L, precision=N.PREC_FP64, engine=eng)
    rel = np.abs(tc - f64) / np.abs(f64)
    rel32 = np.abs(f32 - f64) / np.abs(f64)
    sub = np.arange(0, len(w.q), 50)
    d64 = cs.debye_solvent_basis(s, w.q[sub], cs.SolventParams(), engine=eng, fp64=True)[0]
    trunc = np.abs(f64[sub] - d64) / np.abs(d64)
    # the contraction a direct per-(l, q) evaluation would do: 2 N sum_q (l_q+1)^2
    c = s.xyz.mean(axis=0)
    rmax = float(np.max(np.linalg.norm(s.xyz - c, axis=1)))
    lq = np.clip(np.ceil(w.q * rmax) + 8, min(8, L), L)
    direct_flop = 2.0 * s.atom_count * float(np.sum((lq + 1) ** 2))
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        pass
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    peak_source = "of measured (MEASURED_PEAKS.json bf16_tflops)" if "bf16_tflops" in peaks else \
        "of fallback (1.59 PFLOP/s bf16, an earlier measurement on this pool)"
    tf32_peak = 0.5 * bf16_peak  # dense TF32 runs at half the BF16 rate
    # BF16 operands (Y_lm generated inside the GEMM kernel): hi+lo for every l,
    # and one term; tensor FLOP = products per K step x useful FLOP
    bf = {}
    for name, prec, products in [("bf16_split", N.PREC_BF16_SPLIT, 3), ("bf16", N.PREC_BF16, 1),
                                 ("tf32_split_fused", N.PREC_TF32_SPLIT_FUSED, 3)]:
        out, wall, dev, gemm, _ = timed(prec)
        r = np.abs(out - f64) / np.abs(f64)
        pk = tf32_peak if name.startswith("tf32") else bf16_peak
        bf[name] = {"wall_ms": wall, "device_ms": dev, "gemm_ms": gemm,
                    "tensor_tflops": products * flop / (gemm * 1e-3) / 1e12, "peak_tflops": pk,
                    "frac": products * flop / (gemm * 1e-3) / 1e12 / pk,
                    "max_rel_err_vs_fp64_multipole": float(r.max()),
                    "rms_rel_err_vs_fp64_multipole": float(np.sqrt(np.mean(r ** 2)))}
    # the 20,000-atom curve with the adaptive 3 Å grid by multipole, L = 30
    s2 = synth.protein(synth.DEBYE_20K_SOLVATED.seed, synth.DEBYE_20K_SOLVATED.n_atoms, synth.DEBYE_20K_SOLVATED.radius)
    sp = cs.SolventParams(hydration_model=cs.HydrationModel.AdaptiveGrid, hydration_grid_spacing_angstrom=3.0)
    opt = cs.ComputeOptions(method=cs.ScatteringMethod.Multipole, solvent=sp, multipole_l_max=30)
    cs.compute_curve(s2, synth.DEBYE_20K_SOLVATED.q, opt, engine=eng)
    t0 = time.perf_counter()
    for _ in range(3):
        cs.compute_curve(s2, synth.DEBYE_20K_SOLVATED.q, opt, engine=eng)
    c2_ms = (time.perf_counter() - t0) * 1e3 / 3
    cpu = None
    if with_cpu and rank == 0:
        import oracle as O

        sub_q = w.q[::100]
        a = O.Atoms(s.xyz, s.element, s.group, s.occupancy)
        t0 = time.perf_counter()
        O.multipole_intensity(a, sub_q, L)
        dt = time.perf_counter() - t0
        cpu = {"value": len(sub_q) / dt, "unit": "q/s", "cores": min(os.cpu_count() or 1, len(sub_q)), "kind": "port",
               "sample": f"every 100th q ({len(sub_q)} of {len(w.q)}) of the same 100k-atom curve, f64 restatement "
                         f"of spherical.rs multipole_intensity, {dt:.1f} s",
               "gpu_q_per_s_wall": len(w.q) / (tc_wall * 1e-3)}
    return {"workload": "multipole intensity, 100k atoms (R 80 Å), 1000 q on [0.001, 0.6], L = 50",
            "cpu_baseline": cpu,
            "precision": "TF32 hi+lo on tcgen05 (default)", "wall_ms": tc_wall, "device_ms": tc_dev,
            "moments_gemm_tensor": {
                "ms": tc_gemm, "useful_flop": flop, "tensor_flop": 3.0 * flop,
                "achieved_tflops": 3.0 * flop / (tc_gemm * 1e-3) / 1e12, "peak_tflops": tf32_peak,
                "peak_source": "0.5 x bf16 peak (dense TF32 = half the BF16 rate), " + peak_source,
                "frac": 3.0 * flop / (tc_gemm * 1e-3) / 1e12 / tf32_peak,
                "note": "3 TF32 products per K step (h h', h m', m h'); includes the split reduction"},
            "moments_gemm_fp32_simt": {"ms": f32_gemm, "achieved_tflops": flop / (f32_gemm * 1e-3) / 1e12,
                                       "peak_tflops": fp32_peak, "frac": flop / (f32_gemm * 1e-3) / 1e12 / fp32_peak,
                                       "device_ms": f32_dev, "wall_ms": f32_wall},
            "direct_contraction_flop": direct_flop,
            "direct_equivalent_tflops": direct_flop / (tc_dev * 1e-3) / 1e12,
            "max_rel_err_vs_fp64_multipole": float(rel.max()),
            "rms_rel_err_vs_fp64_multipole": float(np.sqrt(np.mean(rel**2))),
            "fp32_simt_max_rel_err_vs_fp64_multipole": float(rel32.max()),
            "max_rel_err_vs_fp64_debye_every_50th_q": float(trunc.max()),
            "rms_rel_err_vs_fp64_debye_every_50th_q": float(np.sqrt(np.mean(trunc**2))),
            "solvated_20k_multipole_l30_curve_ms": c2_ms,
            "other_tensor_modes": bf,
            "other_tensor_modes_note": "gemm_ms includes the split reduction; BF16 modes and tf32_split_fused "
                                       "generate Y_lm inside the GEMM kernel (the default TF32 modes stage it "
                                       "through device memory: k_mp_prep, outside gemm_ms); bf16 peak " + peak_source}


def grid_and_gradient_section(eng, rank):
    """Hydration grid of the 20,000-atom structure (adaptive, 3 Å spacing; bit-exact against the
    oracle in the tests) and chi^2 with its full adjoint gradient on 5,000 atoms
    (5,000 atoms, 100 q): wall time per public call, median of 5 after a warm-up."""
    import crabsaxs_b200 as cs
    from crabsaxs_b200 import synth

    def med(fn, n=5):
        fn()
        ts = []
        for _ in range(n):
            t0 = time.perf_counter()
            fn()
            ts.append((time.perf_counter() - t0) * 1e3)
        return float(np.median(ts))

    s2 = synth.protein(synth.DEBYE_20K_SOLVATED.seed + 1000 * rank, synth.DEBYE_20K_SOLVATED.n_atoms, synth.DEBYE_20K_SOLVATED.radius)
    sites, _ = cs.hydration_grid_adaptive(s2, 3.0, engine=eng)
    grid_ms = med(lambda: cs.hydration_grid_adaptive(s2, 3.0, engine=eng))
    ext = cs.hydration_grid_exterior(s2, engine=eng)[0]
    ext_ms = med(lambda: cs.hydration_grid_exterior(s2, engine=eng))
    w = synth.GRADIENT_5K
    s4 = synth.protein(w.seed + 1000 * rank, w.n_atoms, w.radius)
    y = cs.compute_curve(s4, w.q, cs.ComputeOptions(method=cs.ScatteringMethod.Debye,
                                                    solvent=cs.SolventParams())).intensity
    sigma = 0.01 * y
    grad_ms = med(lambda: cs.chi2_grad(s4, w.q, 1.01 * y, sigma, cs.SolventParams(), 1.0, 0.0, engine=eng))
    pairq = s4.atom_count * (s4.atom_count - 1) / 2.0 * len(w.q)
    return {"adaptive_grid_20k": {"ms": grid_ms, "sites": int(len(sites)), "atoms": s2.atom_count},
            "exterior_grid_20k": {"ms": ext_ms, "sites": int(len(ext))},
            "chi2_grad_5k": {"ms": grad_ms, "atoms": s4.atom_count, "n_q": len(w.q),
                                  "pair_q_per_s": 2.0 * pairq / (grad_ms * 1e-3),
                                  "note": "ordered pairs (i, j) and (j, i): 2 * N(N-1)/2 * nq per call"}}


def pr_section(eng, rank, with_cpu):
    """Coordinate features (metrics.rs:236-270): Rg, Dmax and the 160-bin P(r)
    of the 100,000-atom structure (5e9 pairs).  Wall time of the public
    call and device time of its kernels, median of 5 after a warm-up; the CPU
    baseline is the oracle (the reference's 64-row-chunk loop, OpenMP on every
    host core) on a seeded 20,000-atom subset."""
    import crabsaxs_b200 as cs
    import oracle as O
    from crabsaxs_b200 import synth

    w = synth.ATOMS_100K
    s = synth.protein(w.seed + 1000 * rank, w.n_atoms, w.radius)
    cs.coordinate_features(s, engine=eng)
    walls, dev, hist = [], [], []
    for _ in range(5):
        t0 = time.perf_counter()
        cs.coordinate_features(s, engine=eng)
        walls.append((time.perf_counter() - t0) * 1e3)
        total_ms, hist_ms, pairs, mode = cs.pr_last_timing(eng)
        dev.append(total_ms)
        hist.append(hist_ms)
    out = {"atoms": s.atom_count, "bins": 160, "pairs": pairs, "wall_ms": float(np.median(walls)),
           "device_ms": float(np.median(dev)), "histogram_kernel_ms": float(np.median(hist)),
           "pairs_per_s": pairs / (float(np.median(hist)) * 1e-3),
           "accumulation": {0: "class-pair counts", 1: "f64 per warp", 2: "f64 rows"}.get(mode, "none")}
    if with_cpu and rank == 0:
        idx = np.sort(np.random.default_rng(0).choice(s.atom_count, 20000, replace=False))
        a = O.Atoms(s.xyz[idx], s.element[idx], s.group[idx], s.occupancy[idx])
        t0 = time.perf_counter()
        O.coordinate_features(a, 160)
        dt = time.perf_counter() - t0
        sub_pairs = 20000 * 19999 / 2.0
        out["cpu_baseline"] = {"value": sub_pairs / dt, "unit": "pairs/s", "cores": os.cpu_count() or 1,
                               "kind": "port", "sample": "seeded 20,000-atom subset, 160 bins", "seconds": dt}
    return out


def _pdb_text(s):
    """PDB ATOM records of a synthetic structure (residue SYN, six atoms per residue)."""
    sym = {1: "C", 2: "N", 3: "O", 4: "S"}
    lines = []
    for i, (p, e) in enumerate(zip(s.xyz, s.element)):
        el = sym[int(e)]
        name = f"{el}{i % 6}"
        lines.append(f"ATOM  {(i + 1) % 100000:>5} {name:<4} SYN {chr(65 + i // 60000)}{(i // 6) % 10000:>4}    "
                     f"{p[0]:>8.3f}{p[1]:>8.3f}{p[2]:>8.3f}{1.0:>6.2f}{10.0:>6.2f}          {el:>2}")
    return ("\n".join(lines) + "\nEND\n").encode()


def ingest_section(rank, with_cpu):
    """Structure ingest (structure.rs:209-327): the 100,000-atom structure as
    100,000 PDB ATOM records parsed by crab_parse_structure with the default
    options, median of 5; the CPU baseline is the Python restatement of the
    reference's reader and policies on the first 10,000 records."""
    import ctypes as C

    import crabsaxs_b200 as cs
    from crabsaxs_b200 import _native as N
    from crabsaxs_b200 import synth

    w = synth.ATOMS_100K
    text = _pdb_text(synth.protein(w.seed + 1000 * rank, w.n_atoms, w.radius))
    o = cs.ParseOptions().to_c()
    ts, n = [], 0
    for _ in range(6):
        p = C.c_void_p()
        t0 = time.perf_counter()
        if N.lib.crab_parse_structure(text, len(text), N.FORMAT_PDB, C.byref(o), C.byref(p)) != N.OK:
            raise RuntimeError(N.lib.crab_parse_last_error().decode())
        ts.append(time.perf_counter() - t0)
        n = int(N.lib.crab_parsed_atom_count(p))
        N.lib.crab_parsed_destroy(p)
    ms = 1e3 * float(np.median(ts[1:]))
    out = {"atoms": n, "bytes": len(text), "ms": ms, "atoms_per_s": n / (ms * 1e-3)}
    if with_cpu and rank == 0:
        from oracle import structure as OS

        sub = b"\n".join(text.split(b"\n")[:10000]).decode() + "\n"
        t0 = time.perf_counter()
        k = len(OS.parse(sub, OS.Options()))
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": k / dt, "unit": "atoms/s", "cores": 1, "kind": "port",
                               "sample": "first 10,000 records, Python restatement of structure.rs + pdbtbx reading"}
    return out


# The reference's only published timings (docs/BENCHMARKS.md:32-36, docs/benchmark-reports/*.json):
# its CLI run as a subprocess on a 6-core aarch64 Mac, process start, PDB parsing, the computation
# or fit, and the curve output included.  Real PDB files are not available here; seeded synthetic
# structures of the same atom counts stand in for them.
PUBLISHED = {"compute_602": 13.10, "compute_1481": 28.44, "compute_58870": 2239.33,
             "fit_1481_stride20": 24.86, "fit_1481_stride1": 160.86}


def published_section(eng, rank):
    """The reference's published workflows through this library's public API on
    synthetic stand-ins of the same size: PDB text -> crab_parse_structure (HETATM
    on, selected conformer full) -> compute_curve (multipole, adaptive 4 Å grid,
    c1 = 1, c2 = 0, 101 q on [0, 0.5]) -> curve text; and the fit (multipole,
    adaptive 8 Å grid, fitted background, c2 in [-0.045, 0.1]) against a 612-point
    synthetic curve on [0.0116, 0.5], with q-sampling stride 20 and 1.  Wall time
    per workflow, median of 5 after a warm-up; process start is not included."""
    import crabsaxs_b200 as cs
    from crabsaxs_b200 import synth

    popt = cs.ParseOptions(include_hetatm=True, occupancy_policy=cs.OccupancyPolicy.SelectedConformerFull)
    q = np.arange(101) * 0.005
    copt = cs.ComputeOptions(method=cs.ScatteringMethod.Multipole,
                             solvent=cs.SolventParams(c1=1.0, c2=0.0, hydration_model=cs.HydrationModel.AdaptiveGrid,
                                                      hydration_grid_spacing_angstrom=4.0))

    def med(fn, n=5):
        fn()
        ts = []
        for _ in range(n):
            t0 = time.perf_counter()
            fn()
            ts.append((time.perf_counter() - t0) * 1e3)
        return float(np.median(ts))

    def structure(n):
        return synth.protein(SEED + 17 * n + 1000 * rank, n, 45.0 * (n / 20000.0) ** (1.0 / 3.0))

    out = {}
    for n in (602, 1481, 58870):
        text = _pdb_text(structure(n))

        def compute():
            s = cs.Structure.from_text(text, popt, 1)
            c = cs.compute_curve(s, q, copt, engine=eng)
            "\n".join(f"{a:.6e} {b:.6e}" for a, b in zip(c.q, c.intensity))
            s.release()

        out[f"compute_{n}"] = {"ms": med(compute), "reference_published_ms": PUBLISHED[f"compute_{n}"]}
    s0 = structure(1481)
    text = _pdb_text(s0)
    qf = np.linspace(0.0116, 0.5, 612)
    clean = 2.0 * cs.compute_curve(s0, qf, cs.ComputeOptions(method=cs.ScatteringMethod.Debye,
                                                              solvent=cs.SolventParams(c2=0.03))).intensity + 5.0
    sigma = 0.01 * clean
    y = clean + sigma * np.random.default_rng(61).normal(size=len(qf))
    ex = cs.ExperimentalCurve(qf, y, sigma)
    for stride in (20, 1):
        fo = cs.FitOptions(method=cs.ScatteringMethod.Multipole, q_sampling_stride=stride, c2_bounds=(-0.045, 0.1),
                           solvent=cs.SolventParams(hydration_model=cs.HydrationModel.AdaptiveGrid,
                                                    hydration_grid_spacing_angstrom=8.0))

        def fit():
            s = cs.Structure.from_text(text, popt, 1)
            r = cs.fit_to_experimental_with_options(s, ex, cs.FitParams(), fo, engine=eng)
            "\n".join(f"{a:.6e} {b:.6e}" for a, b in zip(qf, r.fitted_curve))
            s.release()

        out[f"fit_1481_stride{stride}"] = {"ms": med(fit), "reference_published_ms": PUBLISHED[f"fit_1481_stride{stride}"]}
    out["note"] = ("reference figures: its CLI on a 6-core aarch64 Mac including process start; here: library calls "
                   "on synthetic stand-ins of the same atom counts, process start excluded")
    return out


def run_ours(args, rank, world, local):
    import crabsaxs_b200 as cs
    from crabsaxs_b200 import _native as N

    if world > 1:  # this rank's GPU first, so the NCCL group binds to it
        import torch

        torch.cuda.set_device(local)
    dist = Dist(world, "nccl")
    eng = cs.Engine(local)
    lib = N.lib
    peak = C.c_double()
    eng.check(lib.crab_measure_fp32_peak(eng.handle, 150.0, C.byref(peak)))

    # one structure; with N > 1 ranks it is split over the GPUs (every rank
    # builds the same structure and takes the work items crab_shard_assign
    # gives it; one NCCL all-reduce of the partials per step completes the sums)
    s = workload(0)
    sites, vol = cs.hydration_grid_adaptive(s, 3.0, engine=eng)
    xyz, w, t, T = typed_arrays(s, sites)
    m = len(w)
    # the sites lie on a 3 Å lattice: integer voxel offsets for the exact site–site histogram
    cells = np.ascontiguousarray(np.rint((sites - sites.min(axis=0)) / 3.0).astype(np.int32))
    plan = C.c_void_p()
    eng.check(lib.crab_pair_plan_create_lattice_shard(eng.handle, xyz.ctypes.data_as(N.D), w.ctypes.data_as(N.D),
                                                      t.ctypes.data_as(N.I32P), m, T, Q.ctypes.data_as(N.D),
                                                      len(Q), cells.ctypes.data_as(N.I32P), len(sites), 3.0, rank,
                                                      world, C.byref(plan)))
    chosen = C.c_int32()
    tv = np.zeros(32, dtype=np.int32)
    tms = np.zeros(32)
    ntv = C.c_int32()
    eng.check(lib.crab_pair_plan_autotune(eng.handle, plan, C.byref(chosen), tv.ctypes.data_as(N.I32P),
                                          tms.ctypes.data_as(N.D), 32, C.byref(ntv)))
    tuning = {_variant_name(v): round(float(t), 3) for v, t in zip(tv[:ntv.value], tms[:ntv.value])}
    pairq = lib.crab_pair_plan_pairq(plan)
    ns = len(sites)
    kernel_pairq = pairq - ns * (ns - 1) / 2.0 * len(Q)  # the lattice path sums the site–site pairs

    # warm-up, then K timed steps (each a flushed, event-bracketed kernel;
    # with N > 1 each step also all-reduces this rank's partials over NCCL,
    # timed with CUDA events on torch's stream)
    eng.check(lib.crab_pair_plan_run(eng.handle, plan, args.warmup, FLUSH_BYTES, None))
    step_ms = np.zeros(args.steps)
    reduce_ms = np.zeros(args.steps)
    n_part = T * (T + 1) // 2 * len(Q)
    part_host = np.zeros(n_part)
    if world > 1:
        import torch

        part_dev = torch.zeros(n_part, dtype=torch.float64, device=f"cuda:{local}")
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(args.warmup):
            dist.dist.all_reduce(part_dev)
        torch.cuda.synchronize()
    eng.reset_stats()
    one = np.zeros(1)
    with ClockSampler(local) as clocks:
        dist.barrier()
        t0 = time.perf_counter()
        if world == 1:
            eng.check(lib.crab_pair_plan_run(eng.handle, plan, args.steps, FLUSH_BYTES, step_ms.ctypes.data_as(N.D)))
        else:
            for k in range(args.steps):
                eng.check(lib.crab_pair_plan_run(eng.handle, plan, 1, FLUSH_BYTES, one.ctypes.data_as(N.D)))
                step_ms[k] = one[0]
                eng.check(lib.crab_pair_plan_read(eng.handle, plan, part_host.ctypes.data_as(N.D), None))
                part_dev.copy_(torch.from_numpy(part_host))
                ev0.record()
                dist.dist.all_reduce(part_dev)
                ev1.record()
                ev1.synchronize()
                reduce_ms[k] = ev0.elapsed_time(ev1)
        wall = time.perf_counter() - t0
        dist.barrier()
    launches, _, _ = eng.stats()
    device_s = float(step_ms.sum() + reduce_ms.sum()) / 1e3
    max_s = dist.max(device_s)
    total_units = pairq * args.steps  # the one structure's pair·q, however many GPUs share it
    value = total_units / max_s
    ms_per_step = 1e3 * max_s / args.steps
    # roofline of this rank's kernel: its share of the kernel-evaluated pair·q (the
    # shards' items are near equal in cost) over its kernel time
    achieved = 4.0 * kernel_pairq / world / (float(step_ms.mean()) * 1e-3) / 1e12

    # accuracy of this curve against the FP64 device reference (outside the timed region)
    import crabsaxs_b200.synth as synth

    c1, c2 = synth.solvent_draw(SEED)
    sp = cs.SolventParams(c1=c1, c2=c2, hydration_model=cs.HydrationModel.AdaptiveGrid,
                          hydration_grid_spacing_angstrom=3.0)
    b32 = cs.debye_solvent_basis(s, Q, sp, engine=eng)
    b64 = cs.debye_solvent_basis(s, Q, sp, engine=eng, fp64=True)
    _, ms64, pq64 = eng.stats()  # the FP64 pair kernel of that call (direct f64 sin), by CUDA events
    i32 = cs.combine_solvent_basis(b32, Q, c1, c2)
    i64 = cs.combine_solvent_basis(b64, Q, c1, c2)
    max_rel = float(np.max(np.abs(i32 - i64) / np.abs(i64)))

    # end to end through the public C-ABI call with pinned host buffers
    import torch

    def pinned(a):
        tt = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return tt, tt.numpy()

    _, hx = pinned(s.xyz)
    _, ho = pinned(s.occupancy)
    _, he = pinned(s.element)
    _, hg = pinned(s.group)
    _, hq = pinned(Q)
    tout, hout = pinned(np.zeros((6, len(Q))))
    solv = sp.to_c()

    basis_dev = torch.zeros((6, len(Q)), dtype=torch.float64, device=f"cuda:{local}") if world > 1 else None

    def e2e_step():
        st = C.c_void_p()
        eng.check(lib.crab_structure_create(eng.handle, hx.ctypes.data_as(N.D), ho.ctypes.data_as(N.D),
                                            he.ctypes.data_as(N.I8P), hg.ctypes.data_as(N.I8P), len(ho),
                                            C.byref(st)))
        if world == 1:
            eng.check(lib.crab_debye_solvent_basis(eng.handle, st, hq.ctypes.data_as(N.D), len(hq), C.byref(solv),
                                                   1, hout.ctypes.data_as(N.D)))
        else:  # this rank's share of the basis, then the sum over the GPUs, read back
            eng.check(lib.crab_debye_solvent_basis_shard(eng.handle, st, hq.ctypes.data_as(N.D), len(hq),
                                                         C.byref(solv), 1, N.PREC_FP32, rank, world,
                                                         hout.ctypes.data_as(N.D)))
            basis_dev.copy_(tout, non_blocking=True)
            dist.dist.all_reduce(basis_dev)
            tout.copy_(basis_dev)
        lib.crab_structure_destroy(st)

    for _ in range(args.warmup):
        e2e_step()
    # two consecutive timed runs of K full steps each; the faster one is the
    # e2e value (the host is shared, and one run can catch a host stall);
    # both runs and every step time are reported
    e2e_runs = []
    for _ in range(2):
        eng.reset_stats()
        gc.collect()
        gc.disable()  # no collector pauses inside the timed steps
        dist.barrier()
        t0 = time.perf_counter()
        steps_ms = []
        for _ in range(args.steps):
            ts = time.perf_counter()
            e2e_step()
            steps_ms.append((time.perf_counter() - ts) * 1e3)
        run_s = time.perf_counter() - t0
        gc.enable()
        dist.barrier()
        run_launches, _, _ = eng.stats()
        h2d, d2h = C.c_int64(), C.c_int64()
        lib.crab_ctx_transfer_stats(eng.handle, C.byref(h2d), C.byref(d2h))
        exch = 6 * len(Q) * 8 * args.steps if world > 1 else 0  # the basis to and from the all-reduce
        e2e_runs.append({"seconds": dist.max(run_s), "steps_ms": steps_ms, "launches": int(run_launches),
                         "h2d": int(h2d.value) + exch, "d2h": int(d2h.value) + exch})
    best = min(e2e_runs, key=lambda r: r["seconds"])
    e2e_s, e2e_steps, e2e_launches = best["seconds"], best["steps_ms"], best["launches"]
    e2e_value = total_units / e2e_s

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, nq, dt, mm = cpu_baseline_run(s, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"same structure + its {mm - N_ATOMS} sites, {nq} of 500 q values (one per thread), "
                         f"{dt:.1f} s; f64 C++ restatement of solvent.rs debye_solvent_basis"}

    ens = None if args.no_ensemble else ensemble_section(eng, rank, not args.no_cpu_baseline)
    mp = None if args.no_multipole else multipole_section(eng, rank, peak.value, not args.no_cpu_baseline)
    aux = None if args.no_multipole else grid_and_gradient_section(eng, rank)
    pr = None if args.no_multipole else pr_section(eng, rank, not args.no_cpu_baseline)
    ingest = None if args.no_multipole else ingest_section(rank, not args.no_cpu_baseline)
    published = None
    if not args.no_multipole:
        try:  # an auxiliary section must not cost the main line
            published = published_section(eng, rank)
        except Exception as exc:  # noqa: BLE001
            published = {"error": f"{type(exc).__name__}: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "n_atoms": N_ATOMS, "n_sites": int(len(sites)), "n_types": T, "n_q": len(Q),
                       "kernel_variant": _variant_name(chosen.value), "autotune_ms": tuning,
                       "parallelism": "one GPU" if world == 1 else
                       f"one structure split over {world} GPUs (work items by crab_shard_assign, "
                       f"NCCL all-reduce of the partials each step)",
                       "allreduce_ms_per_step": float(np.mean(reduce_ms)) if world > 1 else 0.0,
                       "l2": "flushed before every step (256 MiB memset, outside the step events)"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                         "frac": achieved / peak.value, "traffic": traffic_per_launch(),
                         "units_per_launch": kernel_pairq,
                         "peak_source": "FFMA microbenchmark measured in this run (MEASURED_PEAKS.json has no FP32)",
                         "flop_per_unit": 4},
            "kernel_evaluated": {"value": kernel_pairq * args.steps / max_s, "unit": UNIT,
                                 "note": "value without the site-site pair.q, which the exact lattice histogram "
                                         "sums instead of the pair kernel"},
            "fp64_device": {"value": pq64 / (ms64 * 1e-3) if ms64 > 0 else None, "unit": UNIT,
                            "kernel_ms": ms64,
                            "note": "the FP64 pair kernel (direct f64 sin per pair and q) on the same structure, "
                                    "one public crab_debye_solvent_basis call; the same-precision figure beside "
                                    "the f64 CPU arm"},
            "parity": {"max_rel_err_vs_fp64": max_rel, "c1": c1, "c2": c2},
            "ensemble": ens,
            "multipole": mp,
            "grids_and_gradient": aux,
            "coordinate_pr": pr,
            "structure_ingest": ingest,
            "published_workflows": published,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": best["h2d"] // args.steps,
                    "d2h_bytes_per_step": best["d2h"] // args.steps,
                    "ms_per_step": 1e3 * e2e_s / args.steps,
                    "step_ms_min_median_max": [min(e2e_steps), float(np.median(e2e_steps)), max(e2e_steps)],
                    "runs": [{"value": total_units / r["seconds"], "ms_per_step": 1e3 * r["seconds"] / args.steps,
                              "steps_ms": [round(x, 3) for x in r["steps_ms"]]} for r in e2e_runs],
                    "selection": "faster of two consecutive timed runs of K steps each"},
            "gpu_launches": int(launches),
            "e2e_gpu_launches": int(e2e_launches),
            "clocks": clocks.summary(),
            "wall_s_timed_region": wall,
        }
        print(json.dumps(line), flush=True)
    lib.crab_pair_plan_destroy(plan)
    dist.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-multipole", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
