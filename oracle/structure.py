"""ORACLE — test infrastructure only.

A pure-Python restatement of crabSAXS structure ingest (src/structure.rs:37-345):
the PDB fixed-column and mmCIF _atom_site records read the way pdbtbx 0.12
reads them in loose mode, then the reference's own selection policies.  Only
tests/ use it, as the checker for the C++ parser behind crab_parse_structure.

pdbtbx is a third-party crate (pinned 0.12.0 in the reference's Cargo.lock)
and is not present here.  Its blank-altloc expansion is restated from the
reference's comment at structure.rs:309-313: a blank-altloc atom of a residue
that also has named altlocs is placed in every named conformer with its
occupancy divided by the number of conformers including the blank one.
"""
from __future__ import annotations

import math
import shlex
from dataclasses import dataclass, field

ELEMENTS = {"H": 0, "D": 0, "C": 1, "N": 2, "O": 3, "S": 4, "P": 5, "NA": 6, "MG": 7, "CL": 8, "CA": 9,
            "FE": 10, "ZN": 11, "K": 12, "I": 13}
OTHER = 14
GLYCANS = {"NAG", "NDG", "BMA", "MAN", "GLC", "GAL", "FUC", "SIA", "NAN", "NEU", "XYS", "XYP", "ARA", "ARB",
           "RIB", "FRU", "G6D", "G1P", "BGC", "AFD", "AGS", "AMU", "API", "DGA", "DGL", "DGU", "GCU", "GTR",
           "IDR", "LBT", "MMA", "RM4", "SUC", "TRE", "MAL", "LMT", "KDO", "KDN", "DAN", "XUL"}
WATERS = {"HOH", "WAT", "DOD"}


class ParseError(Exception):
    pass


class ElementError(Exception):
    pass


@dataclass
class Rec:
    hetatm: bool
    name: str
    alt: str
    resname: str
    chain: str
    resseq: int
    icode: str
    x: float
    y: float
    z: float
    occ: float
    element: str


@dataclass
class Options:  # structure.rs:177-201
    include_hetatm: bool = False
    include_waters: bool = False
    include_glycans: bool = True
    model_index: int = 0
    allow_unknown_elements: bool = False
    occupancy_full: bool = False
    altloc: str = "highest"  # highest | first | all
    chains: list = field(default_factory=list)


def element_from_symbol(s: str) -> int:  # structure.rs:109-127
    return ELEMENTS.get(s.strip().upper(), OTHER)


def _num(s: str) -> float:
    try:
        v = float(s)
    except ValueError as e:
        raise ParseError(s) from e
    if not math.isfinite(v):
        raise ParseError(s)
    return v


def read_pdb(text: str) -> list[list[Rec]]:
    models: list[list[Rec]] = []
    for line in text.splitlines():
        rec = line[:6]
        if rec.startswith("MODEL"):
            models.append([])
            continue
        if rec.startswith("ENDMDL"):
            continue
        if rec not in ("ATOM  ", "ATOM", "HETATM"):
            continue
        if not models:
            models.append([])
        col = lambda a, b: line[a - 1:b].strip()  # noqa: E731
        occ = col(55, 60)
        models[-1].append(Rec(rec == "HETATM", col(13, 16), col(17, 17), col(18, 20), col(22, 22),
                              int(col(23, 26)), col(27, 27), _num(col(31, 38)), _num(col(39, 46)),
                              _num(col(47, 54)), _num(occ) if occ else 1.0, col(77, 78)))
    return models


def read_cif(text: str) -> list[list[Rec]]:
    cols: list[str] = []
    values: list[str] = []
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        t = lines[i].strip()
        if t == "loop_" and i + 1 < len(lines) and lines[i + 1].strip().startswith("_atom_site."):
            i += 1
            while i < len(lines) and lines[i].strip().startswith("_atom_site."):
                cols.append(lines[i].strip()[len("_atom_site."):])
                i += 1
            while i < len(lines):
                t = lines[i].strip()
                if not t or t.startswith("#") or t.startswith("_") or t.startswith("loop_"):
                    break
                values += shlex.split(t, posix=True)
                i += 1
            break
        i += 1
    if not cols:
        raise ParseError("no _atom_site loop")
    if len(values) % len(cols):
        raise ParseError("truncated row")
    models: dict[str, list[Rec]] = {}
    for r in range(len(values) // len(cols)):
        row = dict(zip(cols, values[r * len(cols):(r + 1) * len(cols)]))

        def get(a, b=None):
            v = row.get(a)
            if (v is None or v in "?.") and b is not None:
                v = row.get(b)
            return "" if v is None or v in ("?", ".") else v

        seq = get("auth_seq_id", "label_seq_id")
        occ = get("occupancy")
        rec = Rec(get("group_PDB") == "HETATM", get("auth_atom_id", "label_atom_id"), get("label_alt_id"),
                  get("auth_comp_id", "label_comp_id"), get("auth_asym_id", "label_asym_id"),
                  int(seq) if seq else 0, get("pdbx_PDB_ins_code"), _num(get("Cartn_x")), _num(get("Cartn_y")),
                  _num(get("Cartn_z")), _num(occ) if occ else 1.0, get("type_symbol"))
        models.setdefault(get("pdbx_PDB_model_num"), []).append(rec)
    return list(models.values())


def expand_conformers(recs: list[Rec]) -> list[Rec]:
    residues: dict[tuple, list[int]] = {}
    alts: dict[tuple, list[str]] = {}
    for k, r in enumerate(recs):
        key = (r.chain, r.resseq, r.icode)
        residues.setdefault(key, []).append(k)
        if r.alt and r.alt not in alts.setdefault(key, []):
            alts[key].append(r.alt)
    out = []
    for key, idx in residues.items():
        named = alts.get(key, [])
        for k in idx:
            r = recs[k]
            if r.alt or not named:
                out.append(r)
                continue
            for a in named:
                out.append(Rec(r.hetatm, r.name, a, r.resname, r.chain, r.resseq, r.icode, r.x, r.y, r.z,
                               r.occ / (len(named) + 1), r.element))
    return out


def select(model: list[Rec], o: Options) -> list[dict]:  # structure.rs:238-327
    groups: dict[tuple, list] = {}
    for r in expand_conformers(model):
        resname = r.resname or "UNK"
        code = resname.strip().upper()
        if o.chains and r.chain not in o.chains:
            continue
        if r.hetatm:
            if code in WATERS and not o.include_waters:
                continue
            if not o.include_hetatm and not (o.include_glycans and code in GLYCANS):
                continue
        el = element_from_symbol(r.element if r.element else r.name)
        if el == OTHER and not o.allow_unknown_elements:
            raise ElementError(r.name)
        atom = dict(pos=(r.x, r.y, r.z), element=el, occupancy=max(r.occ, 0.0), hetatm=r.hetatm, name=r.name,
                    resname=resname, chain=r.chain, resid=r.resseq)
        groups.setdefault((r.chain, r.resseq, r.icode, r.name), []).append(atom)
    atoms = []
    for alts in groups.values():
        if o.altloc == "all":
            atoms += alts
            continue
        n = len(alts)
        same = n > 1 and all(a["pos"] == alts[0]["pos"] for a in alts[1:])
        if o.altloc == "highest":
            best = 0
            for k in range(1, n):  # Iterator::max_by keeps the last of equal maxima
                if alts[k]["occupancy"] >= alts[best]["occupancy"]:
                    best = k
            sel = dict(alts[best])
        else:
            sel = dict(alts[0])
        if o.occupancy_full and n > 1:
            sel["occupancy"] = 1.0
        elif not o.occupancy_full and same:
            sel["occupancy"] = min(sel["occupancy"] * (n + 1), 1.0)
        atoms.append(sel)
    atoms.sort(key=lambda a: (a["chain"].encode(), a["resid"], a["name"].encode()))
    return atoms


def parse(text: str, o: Options, cif: bool = False) -> list[dict]:
    models = read_cif(text) if cif else read_pdb(text)
    if o.model_index >= len(models):
        raise ParseError(f"model {o.model_index} is not present")
    return select(models[o.model_index], o)
