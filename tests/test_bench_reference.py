"""bench.py --impl reference (the reference's CPU algorithm, the oracle's f64
restatement, on the host cores) prints one JSON line with the keys the bench
contract asks for, on the same workload as the GPU arm, without loading the
product library."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


RUN_AND_LIST_LIBRARIES = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    if e.code:
        raise
maps = open("/proc/self/maps").read()
print("PRODUCT_LIBRARY_LOADED=" + str("libcrabsaxs_b200" in maps or "crabsaxs_b200" in sys.modules))
"""


def test_reference_arm_prints_its_line():
    out = subprocess.run([sys.executable, "-c", RUN_AND_LIST_LIBRARIES], cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "PRODUCT_LIBRARY_LOADED=False" in out.stdout  # the reference arm runs no product code
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, str(ROOT))
    import bench

    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["config"]["workload"] == bench.WORKLOAD and d["config"]["n_sites"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] >= 3
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_variant_names_cover_every_kernel_family():
    """The bench line names the autotuned Debye kernel by its family: plain
    j-packed, q-packed (3 CTAs/SM from jb 12), folded with 1 or 2 chains, the
    two-chains-per-pair build, and the set-up / recurrence splits."""
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench._variant_name(96 * 16 + 2) == "Q96xJ2"
    assert bench._variant_name(128 * 16 + 13) == "Q128xJ1pq-3cta"
    assert bench._variant_name(168 * 16 + 5) == "Q168xJ1pq-fold-2cta"
    assert bench._variant_name(150 * 16 + 6) == "Q150xJ2pq-fold-2cta"
    assert bench._variant_name(126 * 16 + 7) == "Q126xJ1pq-fold-3cta"
    assert bench._variant_name(168 * 16 + 11) == "Q168xJ1pq-fold-2chain-2cta"
    assert bench._variant_name(126 * 16 + 14) == "Q126xJ1-split"
    assert bench._variant_name(84 * 16 + 12) == "Q84x3blocks-split"
