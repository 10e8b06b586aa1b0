"""Writes tests/golden/small_protein.json: a seeded 300-atom synthetic protein
(coordinates, elements, groups, occupancies stored, so the fixture does not
depend on the generator) and the oracle's outputs for it:

- the Debye solvent basis (analytic hydration) at 40 q (solvent.rs:504-584);
- the adaptive 3 Å hydration sites (solvent.rs:121-223);
- the exterior 1.5 Å hydration sites (solvent.rs:259-401);
- the unit-weight pair-distance histogram with 64 bins (metrics.rs:475-522);
- the FP64 multipole intensity at L = 14 (spherical.rs:266-403).

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle as O  # noqa: E402
from crabsaxs_b200 import synth  # noqa: E402

Q = np.linspace(0.01, 0.5, 40)


def main() -> None:
    s = synth.protein(101, 300, 10.0)
    rng = np.random.default_rng(7)
    occ = np.where(rng.random(len(s.xyz)) < 0.1, 0.5, 1.0)
    a = O.Atoms(s.xyz, s.element, s.group, occ)
    basis = O.debye_solvent_basis(a, Q, 1.0, 0.0)
    adaptive, adaptive_volume = O.adaptive_grid(s.xyz, 3.0)
    exterior, exterior_volume = O.exterior_grid(s.xyz, s.element.astype(np.int32), 1.5)
    dmax, hist = O.pair_distance_histogram(s.xyz, np.ones(len(s.xyz)), 64)
    mp = O.multipole_intensity(a, Q, 14)
    out = {
        "structure": {"xyz": s.xyz.tolist(), "element": s.element.astype(int).tolist(),
                      "group": s.group.astype(int).tolist(), "occupancy": occ.tolist()},
        "q": Q.tolist(),
        "debye_solvent_basis": basis.tolist(),
        "adaptive_grid_3A": {"sites": adaptive.tolist(), "voxel_volume": adaptive_volume},
        "exterior_grid_1p5A": {"sites": exterior.tolist(), "voxel_volume": exterior_volume},
        "pair_distance_histogram_64": {"dmax": dmax, "counts": hist.tolist()},
        "multipole_intensity_L14": mp.tolist(),
    }
    (Path(__file__).parent / "small_protein.json").write_text(json.dumps(out, separators=(",", ":")))


if __name__ == "__main__":
    main()
