"""Structure ingest (crab_parse_structure; structure.rs:205-345) on the CPU.

The first five tests are the reference's own parser tests
(structure.rs:357-441) on its fixtures, restated inline
(examples/data/test_structure.pdb, test_structure.cif, malformed.pdb).  The
rest compare the C++ parser with the Python restatement in oracle/structure.py
on seeded random PDB and mmCIF files: alternate locations (named and blank),
insertion codes, HETATM ligands, waters and glycans, several chains and
models, blank element columns, negative occupancies.
"""
import numpy as np
import pytest

import crabsaxs_b200 as cs
from oracle import structure as OS

FIXTURE_PDB = """HEADER    crabSAXS deterministic parser fixture
MODEL        1
ATOM      1  CA  ALA A   1       0.000   0.000   0.000  0.50 10.00           C
ATOM      2  CA AALA A   1       0.100   0.000   0.000  0.80 10.00           C
ATOM      3  N   ALA A   1       1.330   0.000   0.000  1.00 10.00           N
HETATM    4  O   HOH A   2       2.000   0.000   0.000  1.00 10.00           O
ENDMDL
MODEL        2
ATOM      5  C   GLY A   1       9.000   0.000   0.000  1.00 10.00           C
ENDMDL
END
"""

FIXTURE_CIF = """data_crabsaxs_test
_entry.id crabsaxs_test

loop_
_atom_site.group_PDB
_atom_site.id
_atom_site.type_symbol
_atom_site.label_atom_id
_atom_site.label_alt_id
_atom_site.label_comp_id
_atom_site.label_asym_id
_atom_site.label_entity_id
_atom_site.label_seq_id
_atom_site.pdbx_PDB_ins_code
_atom_site.Cartn_x
_atom_site.Cartn_y
_atom_site.Cartn_z
_atom_site.occupancy
_atom_site.B_iso_or_equiv
_atom_site.pdbx_formal_charge
_atom_site.auth_seq_id
_atom_site.auth_comp_id
_atom_site.auth_asym_id
_atom_site.auth_atom_id
_atom_site.pdbx_PDB_model_num
ATOM 1 C CA . GLY A 1 1 ? 0.000 0.000 0.000 1.00 10.0 ? 1 GLY A CA 1
ATOM 2 O O  . GLY A 1 1 ? 1.200 0.000 0.000 1.00 10.0 ? 1 GLY A O  1
ATOM 3 N N  . GLY A 1 1 ? -1.200 0.000 0.000 1.00 10.0 ? 1 GLY A N  2
"""

FIXTURE_MALFORMED = "ATOM      1  CA  GLY A   1      NOT_A_NUMBER  0.000   0.000  1.00 10.00           C\n"


@pytest.fixture
def fixture_files(tmp_path):
    pdb = tmp_path / "test_structure.pdb"
    pdb.write_text(FIXTURE_PDB)
    cif = tmp_path / "test_structure.cif"
    cif.write_text(FIXTURE_CIF)
    bad = tmp_path / "malformed.pdb"
    bad.write_text(FIXTURE_MALFORMED)
    return pdb, cif, bad


def _ca(s):
    return next(a for a in s.atoms if a.atom_name == "CA")


def test_parses_known_atom_count_and_altloc(fixture_files):  # structure.rs:357-372
    s = cs.Structure.from_pdb_file(fixture_files[0])
    assert s.atom_count == 2
    assert abs(_ca(s).occupancy - 0.8) < 1e-12


def test_selected_conformer_can_be_treated_as_full_occupancy(fixture_files):  # structure.rs:374-393
    o = cs.ParseOptions(occupancy_policy=cs.OccupancyPolicy.SelectedConformerFull)
    assert _ca(cs.Structure.from_pdb_file(fixture_files[0], o)).occupancy == 1.0


def test_applies_hetatm_water_and_model_policies(fixture_files):  # structure.rs:395-429
    path = fixture_files[0]
    assert cs.Structure.from_pdb_file(path, cs.ParseOptions(include_hetatm=True)).atom_count == 2
    assert cs.Structure.from_pdb_file(path, cs.ParseOptions(include_hetatm=True, include_waters=True)).atom_count == 3
    second = cs.Structure.from_pdb_file(path, cs.ParseOptions(model_index=1))
    assert second.atom_count == 1 and second.atoms[0].pos[0] == 9.0


def test_parses_first_model_from_mmcif(fixture_files):  # structure.rs:431-436
    s = cs.Structure.from_pdb_file(fixture_files[1])
    assert s.atom_count == 2 and s.atoms[0].chain_id == "A"


def test_malformed_structure_returns_an_error(fixture_files):  # structure.rs:438-441
    with pytest.raises(cs.StructureParse):
        cs.Structure.from_pdb_file(fixture_files[2])


def test_models_unknown_elements_and_io_errors(fixture_files, tmp_path):
    models = cs.Structure.from_pdb_file_models_with_options(fixture_files[0])
    assert [m.atom_count for m in models] == [2, 1]
    assert [m.atom_count for m in cs.Structure.from_pdb_file_models_with_options(fixture_files[1])] == [2, 1]
    with pytest.raises(cs.StructureParse):
        cs.Structure.from_pdb_file(fixture_files[0], cs.ParseOptions(model_index=2))
    odd = tmp_path / "odd.pdb"
    odd.write_text("ATOM      1  XX  LIG A   1       0.000   0.000   0.000  1.00 10.00           XX\n")
    with pytest.raises(cs.UnsupportedElement):
        cs.Structure.from_pdb_file(odd)
    s = cs.Structure.from_pdb_file(odd, cs.ParseOptions(allow_unknown_elements=True))
    assert s.atom_count == 1 and s.element[0] == cs.Element.Other
    with pytest.raises(OSError):
        cs.Structure.from_pdb_file(tmp_path / "missing.pdb")


# ---------------------------------------------------------------- random files
POLY = ["ALA", "GLY", "SER", "LYS", "ASP", "PHE", "MET", "CYS"]
NAMES = {"ALA": ["N", "CA", "C", "O", "CB"], "GLY": ["N", "CA", "C", "O"], "SER": ["N", "CA", "C", "O", "CB", "OG"],
         "LYS": ["N", "CA", "C", "O", "CB", "NZ"], "ASP": ["N", "CA", "C", "O", "OD1", "OD2"],
         "PHE": ["N", "CA", "C", "O", "CZ"], "MET": ["N", "CA", "SD", "CE"], "CYS": ["N", "CA", "SG"],
         "NAG": ["C1", "O5", "N2"], "HOH": ["O"], "HEM": ["FE", "NA", "C1A"], "ZN": ["ZN"]}
ELEM = {"N": "N", "CA": "C", "C": "C", "O": "O", "CB": "C", "OG": "O", "NZ": "N", "OD1": "O", "OD2": "O",
        "CZ": "C", "SD": "S", "CE": "C", "SG": "S", "C1": "C", "O5": "O", "N2": "N", "FE": "FE", "NA": "N",
        "C1A": "C", "ZN": "ZN"}


def _records(rng, n_models):
    models = []
    for m in range(n_models):
        recs = []
        for chain in ["A", "B", ""][: 1 + int(rng.integers(0, 3))]:
            seq = int(rng.integers(-3, 5))
            for _ in range(int(rng.integers(3, 9))):
                seq += int(rng.integers(1, 3))
                kind = rng.random()
                if kind < 0.7:
                    res, het = POLY[int(rng.integers(len(POLY)))], False
                else:
                    res, het = ["NAG", "HOH", "HEM", "ZN"][int(rng.integers(4))], True
                icode = "A" if rng.random() < 0.1 else ""
                alts = [] if rng.random() < 0.6 else ["A", "B"][: 1 + int(rng.integers(0, 2))]
                for name in NAMES[res]:
                    base = rng.normal(size=3) * 10 + m
                    blank_el = rng.random() < 0.15
                    el = "" if blank_el and name not in ("CA", "NA", "FE", "ZN") else ELEM[name]
                    occ = float(rng.choice([0.25, 0.5, 0.7, 1.0, -0.1]))
                    named = alts and rng.random() < 0.6
                    for a in (alts if named else [""]):
                        pos = base + (rng.normal(size=3) if a and rng.random() < 0.7 else 0.0)
                        recs.append(dict(het=het, name=name, alt=a, res=res, chain=chain, seq=seq, icode=icode,
                                         pos=np.round(pos, 3), occ=occ if rng.random() < 0.8 else round(rng.random(), 2),
                                         el=el))
        models.append(recs)
    return models


def _pdb_text(models):
    out = []
    serial = 1
    for k, recs in enumerate(models):
        if len(models) > 1:
            out.append(f"MODEL     {k + 1:>4}")
        for r in recs:
            rec = "HETATM" if r["het"] else "ATOM  "
            nm = r["name"] if len(r["name"]) == 4 else " " + r["name"]
            x, y, z = r["pos"]
            out.append(f"{rec}{serial:>5} {nm:<4}{r['alt']:1}{r['res']:>3} {r['chain']:1}{r['seq']:>4}{r['icode']:1}"
                       f"   {x:>8.3f}{y:>8.3f}{z:>8.3f}{r['occ']:>6.2f}{10.0:>6.2f}          {r['el']:>2}")
            serial += 1
        if len(models) > 1:
            out.append("ENDMDL")
    out.append("END")
    return "\n".join(out) + "\n"


def _cif_text(models):
    cols = ["group_PDB", "id", "type_symbol", "label_atom_id", "label_alt_id", "label_comp_id", "label_asym_id",
            "label_seq_id", "pdbx_PDB_ins_code", "Cartn_x", "Cartn_y", "Cartn_z", "occupancy", "auth_seq_id",
            "auth_comp_id", "auth_asym_id", "auth_atom_id", "pdbx_PDB_model_num"]
    out = ["data_random", "loop_"] + [f"_atom_site.{c}" for c in cols]
    serial = 1
    for k, recs in enumerate(models):
        for r in recs:
            x, y, z = r["pos"]
            v = ["HETATM" if r["het"] else "ATOM", str(serial), r["el"] or "?", r["name"], r["alt"] or ".", r["res"],
                 r["chain"] or "?", str(r["seq"]), r["icode"] or "?", f"{x:.3f}", f"{y:.3f}", f"{z:.3f}",
                 f"{r['occ']:.2f}", str(r["seq"]), r["res"], r["chain"] or "?", f'"{r["name"]}"', str(k + 1)]
            out.append(" ".join(v))
            serial += 1
    out.append("#")
    return "\n".join(out) + "\n"


def _as_tuples(s: cs.Structure):
    return [(tuple(np.round(s.xyz[i], 6)), int(s.element[i]), round(float(s.occupancy[i]), 12), s.atom_name[i],
             s.residue_name[i], s.chain_id[i], int(s.residue_id[i]), bool(s.is_hetatm[i])) for i in range(s.atom_count)]


def _oracle_tuples(atoms):
    return [(tuple(np.round(a["pos"], 6)), a["element"], round(a["occupancy"], 12), a["name"], a["resname"],
             a["chain"], a["resid"], a["hetatm"]) for a in atoms]


OPTION_SETS = [
    (cs.ParseOptions(), OS.Options()),
    (cs.ParseOptions(include_hetatm=True, include_waters=True, allow_unknown_elements=True),
     OS.Options(include_hetatm=True, include_waters=True, allow_unknown_elements=True)),
    (cs.ParseOptions(include_hetatm=True, include_glycans=False, altloc_policy=cs.AltlocPolicy.First,
                     allow_unknown_elements=True),
     OS.Options(include_hetatm=True, include_glycans=False, altloc="first", allow_unknown_elements=True)),
    (cs.ParseOptions(altloc_policy=cs.AltlocPolicy.All, chains=["B", "A"], allow_unknown_elements=True),
     OS.Options(altloc="all", chains=["B", "A"], allow_unknown_elements=True)),
    (cs.ParseOptions(occupancy_policy=cs.OccupancyPolicy.SelectedConformerFull, model_index=1,
                     allow_unknown_elements=True, include_hetatm=True),
     OS.Options(occupancy_full=True, model_index=1, allow_unknown_elements=True, include_hetatm=True)),
]


@pytest.mark.parametrize("seed", range(12))
def test_random_pdb_and_mmcif_match_the_restatement(seed):
    rng = np.random.default_rng(seed)
    models = _records(rng, 2)
    pdb, cif = _pdb_text(models), _cif_text(models)
    for opt, oopt in OPTION_SETS:
        try:
            ref = _oracle_tuples(OS.parse(pdb, oopt))
        except OS.ElementError:
            with pytest.raises(cs.UnsupportedElement):
                cs.Structure.from_text(pdb, opt)
            continue
        got = _as_tuples(cs.Structure.from_text(pdb, opt))
        assert got == ref, (seed, opt)
        got_cif = _as_tuples(cs.Structure.from_text(cif, opt))
        assert got_cif == _oracle_tuples(OS.parse(cif, oopt, cif=True)), (seed, opt)
        assert got_cif == got, (seed, opt)


def test_united_atom_groups_follow_residue_and_atom_names():
    rng = np.random.default_rng(3)
    models = _records(rng, 1)
    s = cs.Structure.from_text(_pdb_text(models), cs.ParseOptions(include_hetatm=True, allow_unknown_elements=True))
    for i in range(s.atom_count):
        assert s.group[i] == cs.united_atom_group(s.residue_name[i], s.atom_name[i])


@pytest.mark.gpu
def test_parsed_structure_scatters_like_its_arrays(engine):
    """crab_structure_from_parsed hands the parsed arrays to the engine: the
    Debye curve equals the one from the same arrays through Structure."""
    import ctypes as C

    from crabsaxs_b200 import _native as N

    rng = np.random.default_rng(21)
    text = _pdb_text(_records(rng, 1)).encode()
    opt = cs.ParseOptions(include_hetatm=True, allow_unknown_elements=True)
    s = cs.Structure.from_text(text, opt)
    q = np.linspace(0.01, 0.5, 40)
    ref = cs.debye_intensity(s, q, engine=engine)
    parsed, st = C.c_void_p(), C.c_void_p()
    o = opt.to_c()
    assert N.lib.crab_parse_structure(text, len(text), N.FORMAT_PDB, C.byref(o), C.byref(parsed)) == N.OK
    try:
        engine.check(N.lib.crab_structure_from_parsed(engine.handle, parsed, C.byref(st)))
        out = np.empty(len(q))
        engine.check(N.lib.crab_debye_intensity(engine.handle, st, q.ctypes.data_as(N.D), len(q), 1,
                                                out.ctypes.data_as(N.D)))
        N.lib.crab_structure_destroy(st)
    finally:
        N.lib.crab_parsed_destroy(parsed)
    assert np.array_equal(out, ref)


SMALL_PDB = """HEADER    crabSAXS two atom scattering fixture
ATOM      1  C1  TST A   1       0.000   0.000   0.000  1.00 10.00           C
ATOM      2  C2  TST A   1       2.000   0.000   0.000  1.00 10.00           C
END
"""  # examples/data/small.pdb


@pytest.mark.gpu
def test_compute_curve_for_example_structure_is_well_formed(engine):  # tests/end_to_end.rs:3-10
    """The two-atom fixture read by the PDB reader, then the vacuum Debye
    curve on 100 q: finite, non-negative, and the oracle's within 1e-5."""
    import oracle as O

    s = cs.Structure.from_text(SMALL_PDB)
    q = np.arange(100) * 0.005
    got = cs.debye_intensity(s, q, engine=engine)
    assert len(got) == len(q) and np.all(np.isfinite(got)) and np.all(got >= 0.0)
    ref = O.debye_intensity(O.Atoms(s.xyz, s.element, s.group, s.occupancy), q)
    assert np.max(np.abs(got - ref) / ref) <= 1e-5


@pytest.mark.gpu
def test_calc_of_the_example_structure_with_adaptive_hydration(engine):  # tests/end_to_end.rs:12-49
    """What `calc small.pdb --qmin 0.01 --qmax 0.05 --qstep 0.01 --method auto
    --hydration adaptive-grid --c1 1.0 --c2 0.02` computes (4 Å grid, the
    CLI's spacing): a grid hydration model sends Auto to the multipole
    (scattering.rs:145-151) with l_max = clamp(ceil(q_max R) + 8, 8, 64)
    (scattering.rs:168-175); five finite values, the oracle's within 1e-5."""
    import math

    import oracle as O

    s = cs.Structure.from_text(SMALL_PDB)
    q = np.array([0.01, 0.02, 0.03, 0.04, 0.05])
    sp = cs.SolventParams(c1=1.0, c2=0.02, hydration_model=cs.HydrationModel.AdaptiveGrid,
                          hydration_grid_spacing_angstrom=4.0)
    got = cs.compute_curve(s, q, cs.ComputeOptions(solvent=sp), engine=engine)
    assert got.method == "Multipole" and len(got.intensity) == 5 and np.all(np.isfinite(got.intensity))
    r = float(np.max(np.linalg.norm(s.xyz - s.xyz.mean(axis=0), axis=1)))
    l_max = min(max(math.ceil(q.max() * r) + 8, 8), 64)
    a = O.Atoms(s.xyz, s.element, s.group, s.occupancy)
    ref = O.multipole_solvent_intensity(a, q, l_max, c1=1.0, c2=0.02, model=2, spacing=4.0)
    assert np.max(np.abs(got.intensity - ref) / np.abs(ref)) <= 1e-5


# ---------------------------------------------------------------- large files
# Texts above 1 MB are read by several threads, one chunk of whole lines each,
# and stitched in order; these cases cross many chunk boundaries.
def _big_models(seed, n_models):
    rng = np.random.default_rng(seed)
    return _records(rng, n_models)


def _big_text(models, head=None, crlf=False):
    text = _pdb_text(models)
    if head is not None:  # records before the first MODEL line
        text = _pdb_text([head]).replace("END\n", "") + text
    return text.replace("\n", "\r\n") if crlf else text


@pytest.mark.parametrize("crlf", [False, True])
def test_large_multi_model_pdb_matches_the_restatement(crlf):
    models = _big_models(41, 330)
    text = _big_text(models, crlf=crlf)
    assert len(text) > (1 << 20)
    n = ctypes_model_count(text)
    assert n == 330
    for k in (0, 1, 164, 329):
        opt = cs.ParseOptions(model_index=k, include_hetatm=True, allow_unknown_elements=True)
        oopt = OS.Options(model_index=k, include_hetatm=True, allow_unknown_elements=True)
        ref = _oracle_tuples(OS.parse(text.replace("\r\n", "\n"), oopt))
        assert _as_tuples(cs.Structure.from_text(text, opt)) == ref, k


def test_large_pdb_with_records_before_the_first_model():
    models = _big_models(42, 300)
    head = _big_models(43, 1)[0]
    text = _big_text(models, head=head)
    assert len(text) > (1 << 20) and ctypes_model_count(text) == 301
    for k in (0, 1, 300):
        opt = cs.ParseOptions(model_index=k, include_hetatm=True, allow_unknown_elements=True)
        oopt = OS.Options(model_index=k, include_hetatm=True, allow_unknown_elements=True)
        assert _as_tuples(cs.Structure.from_text(text, opt)) == _oracle_tuples(OS.parse(text, oopt)), k


def test_large_single_model_pdb():
    """One model of about 28,000 records (no MODEL lines) over every chunk."""
    rng = np.random.default_rng(44)
    recs = [r for m in _records(rng, 560) for r in m]
    text = _pdb_text([recs])
    assert len(text) > (2 << 20) and ctypes_model_count(text) == 1
    opt = cs.ParseOptions(include_hetatm=True, allow_unknown_elements=True, altloc_policy=cs.AltlocPolicy.All)
    oopt = OS.Options(include_hetatm=True, allow_unknown_elements=True, altloc="all")
    assert _as_tuples(cs.Structure.from_text(text, opt)) == _oracle_tuples(OS.parse(text, oopt))


@pytest.mark.parametrize("where", [0.02, 0.5, 0.97])
def test_large_pdb_reports_the_first_malformed_line(where):
    lines = _big_text(_big_models(45, 330)).split("\n")
    atom_lines = [i for i, l in enumerate(lines) if l.startswith(("ATOM", "HETATM"))]
    bad = atom_lines[int(where * len(atom_lines))]
    later = atom_lines[-3]
    for i in (bad, later):  # two malformed records: the first one is reported
        lines[i] = lines[i][:30] + "  12x.45" + lines[i][38:]
    text = "\n".join(lines)
    with pytest.raises(cs.StructureParse, match=rf"^line {bad + 1}: invalid x coordinate"):
        cs.Structure.from_text(text, cs.ParseOptions(include_hetatm=True, allow_unknown_elements=True))


def ctypes_model_count(text):
    import ctypes as C

    from crabsaxs_b200 import _native as N

    data = text.encode()
    m = C.c_int32()
    assert N.lib.crab_parse_model_count(data, len(data), N.FORMAT_PDB, C.byref(m)) == N.OK
    return m.value
