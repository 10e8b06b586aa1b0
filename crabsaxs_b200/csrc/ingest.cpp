// Structure ingest: PDB and mmCIF atom records to the arrays the scattering
// engines take (crabSAXS src/structure.rs:205-345).
//
// The reference reads files through pdbtbx 0.12 in loose mode and then
// applies its own policies, which are restated here:
//   - a model is chosen by index (MODEL records, or pdbx_PDB_model_num);
//   - chains can be filtered; HETATM records are dropped unless requested,
//     except glycans (kept by default) and waters (dropped unless requested);
//   - the element comes from the element column, else from the atom name,
//     through Element::from_symbol (structure.rs:109-127); an unknown element
//     is an error unless allowed;
//   - atoms are grouped by (chain, residue number, insertion code, atom name)
//     and one alternate location is kept per group (highest occupancy, the
//     last of equal maxima as Iterator::max_by does; or the first; or all);
//   - occupancy is clamped at 0 and, by policy, either kept or set to 1 for a
//     selected conformer; atoms are sorted by (chain, residue number, name).
// pdbtbx places blank-altloc atoms of a residue that also has named altlocs
// into each named conformer with their occupancy divided by the number of
// conformers including the blank one (the reference undoes the division at
// structure.rs:305-313); that expansion is reproduced before grouping.

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.hpp"

// Atom names, residue names and chain ids have few distinct values: each
// atom holds an index into the field's table of distinct strings.
struct crab_parsed {
  std::vector<double> xyz, occ;
  std::vector<int8_t> element, group, hetatm;
  std::vector<int64_t> residue_id;
  std::vector<uint32_t> text_id[3];           // per atom: atom name, residue name, chain id
  std::vector<std::string> text_table[3];     // distinct strings of each field
  const std::string& text(int which, size_t i) const { return text_table[which][text_id[which][i]]; }
};

namespace crab {
namespace {

thread_local std::string g_parse_error;

struct ParseFail {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const std::string& msg) { throw ParseFail{code, msg}; }

struct Record {
  bool hetatm = false;
  int8_t el = -1;  // element code of the element column or the atom name (-1: not yet looked up)
  std::string name, alt, resname, chain, icode, element;
  int64_t resseq = 0;
  double x = 0, y = 0, z = 0, occ = 1.0;
};

int element_from_symbol(const std::string& s);

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

std::string upper(std::string s) {
  for (auto& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

// Columns from..to (1-based, inclusive) of a line, trimmed.
std::string field(const char* line, size_t n, size_t from, size_t to) {
  if (n < from) return std::string();
  size_t a = from - 1, b = std::min(n, to);
  while (a < b && std::isspace((unsigned char)line[a])) ++a;
  while (b > a && std::isspace((unsigned char)line[b - 1])) --b;
  return std::string(line + a, b - a);
}

double number(const std::string& s, const char* what, int64_t line_no) {
  if (s.empty()) fail(CRAB_EPARSE, std::string("line ") + std::to_string(line_no) + ": missing " + what);
  // fixed-point decimals with at most 15 digits: the integer mantissa and the
  // power of ten are exact doubles, so one IEEE division gives the correctly
  // rounded value, the same as strtod
  {
    static const double kPow10[] = {1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9, 1e10, 1e11, 1e12, 1e13, 1e14, 1e15};
    size_t i = 0;
    bool neg = false;
    if (s[i] == '-' || s[i] == '+') neg = s[i++] == '-';
    uint64_t m = 0;
    int digits = 0, frac = -1;
    bool ok = i < s.size();
    for (; i < s.size() && ok; ++i) {
      const char c = s[i];
      if (c >= '0' && c <= '9') {
        m = m * 10 + (uint64_t)(c - '0');
        ++digits;
        if (frac >= 0) ++frac;
      } else if (c == '.' && frac < 0) {
        frac = 0;
      } else {
        ok = false;
      }
    }
    if (ok && digits > 0 && digits <= 15) {
      const double v = (double)m / kPow10[frac > 0 ? frac : 0];
      return neg ? -v : v;
    }
  }
  char* end = nullptr;
  errno = 0;
  const double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str() || *end != '\0' || errno == ERANGE || !std::isfinite(v))
    fail(CRAB_EPARSE, std::string("line ") + std::to_string(line_no) + ": invalid " + what + " '" + s + "'");
  return v;
}

int64_t integer(const std::string& s, const char* what, int64_t line_no) {
  char* end = nullptr;
  errno = 0;
  const long long v = std::strtoll(s.c_str(), &end, 10);
  if (s.empty() || end == s.c_str() || *end != '\0' || errno == ERANGE)
    fail(CRAB_EPARSE, std::string("line ") + std::to_string(line_no) + ": invalid " + what + " '" + s + "'");
  return (int64_t)v;
}

// Columns from..to of a line as a fixed-point decimal, without building a
// string (the same exact fast path as number()); anything else goes through
// number() and its strtod fallback.
double column_number(const char* line, size_t n, size_t from, size_t to, const char* what, int64_t line_no) {
  static const double kPow10[] = {1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9, 1e10, 1e11, 1e12, 1e13, 1e14, 1e15};
  size_t a = from - 1, b = n < to ? n : to;
  if (n < from) b = a;
  while (a < b && line[a] == ' ') ++a;
  while (b > a && line[b - 1] == ' ') --b;
  size_t i = a;
  bool neg = false;
  if (i < b && (line[i] == '-' || line[i] == '+')) neg = line[i++] == '-';
  uint64_t m = 0;
  int digits = 0, frac = -1;
  bool ok = i < b;
  for (; i < b && ok; ++i) {
    const char c = line[i];
    if (c >= '0' && c <= '9') {
      m = m * 10 + (uint64_t)(c - '0');
      ++digits;
      if (frac >= 0) ++frac;
    } else if (c == '.' && frac < 0) {
      frac = 0;
    } else {
      ok = false;
    }
  }
  if (ok && digits > 0 && digits <= 15) {
    const double v = (double)m / kPow10[frac > 0 ? frac : 0];
    return neg ? -v : v;
  }
  return number(field(line, n, from, to), what, line_no);
}

// The records of a file and its models: the records stay where the reader
// stored them (one vector per reader chunk), and each model lists its
// records in file order by address, so no record is moved or copied.
struct Models {
  std::vector<std::vector<Record>> store;
  std::vector<std::vector<const Record*>> list;
};

// PDB fixed columns (wwPDB format 3.3): ATOM/HETATM 1-6, name 13-16, altLoc 17,
// resName 18-20, chainID 22, resSeq 23-26, iCode 27, x 31-38, y 39-46,
// z 47-54, occupancy 55-60, element 77-78.  Models are MODEL ... ENDMDL.
//
// The lines of one chunk of the text: its records in order, where MODEL
// records fall among them, and its line count.
struct PdbChunk {
  std::vector<Record> recs;
  std::vector<size_t> model_starts;  // index in recs of the first record after each MODEL line
  int64_t lines = 0;
  bool failed = false;
};

// Parses the whole lines of [p, end) (line numbers from first_line); a
// malformed record throws ParseFail naming its line.
void parse_pdb_lines(const char* p, const char* end, int64_t first_line, PdbChunk& c) {
  int64_t line_no = first_line - 1;
  c.recs.reserve((size_t)(end - p) / 81 + 16);  // about 81 bytes a record
  while (p < end) {
    const char* nl = (const char*)memchr(p, '\n', (size_t)(end - p));
    const char* line = p;
    size_t n = (size_t)((nl ? nl : end) - p);
    if (n && line[n - 1] == '\r') --n;
    p = nl ? nl + 1 : end;
    ++line_no;
    ++c.lines;
    auto starts = [&](const char* tag) {
      const size_t k = std::strlen(tag);
      return n >= k && std::memcmp(line, tag, k) == 0;
    };
    if (starts("MODEL")) {
      c.model_starts.push_back(c.recs.size());
      continue;
    }
    const bool het = starts("HETATM");
    const bool atom = !het && starts("ATOM") && (n == 4 || line[4] == ' ');
    if (!atom && !het) continue;
    Record r;
    r.hetatm = het;
    r.name = field(line, n, 13, 16);
    r.alt = field(line, n, 17, 17);
    r.resname = field(line, n, 18, 20);
    r.chain = field(line, n, 22, 22);
    r.resseq = integer(field(line, n, 23, 26), "residue number", line_no);
    r.icode = field(line, n, 27, 27);
    r.x = column_number(line, n, 31, 38, "x coordinate", line_no);
    r.y = column_number(line, n, 39, 46, "y coordinate", line_no);
    r.z = column_number(line, n, 47, 54, "z coordinate", line_no);
    bool blank_occ = true;
    for (size_t k = 54; k < 60 && k < n; ++k) blank_occ = blank_occ && line[k] == ' ';
    r.occ = blank_occ ? 1.0 : column_number(line, n, 55, 60, "occupancy", line_no);
    r.element = field(line, n, 77, 78);
    if (r.name.empty()) fail(CRAB_EPARSE, "line " + std::to_string(line_no) + ": missing atom name");
    r.el = (int8_t)element_from_symbol(r.element.empty() ? r.name : r.element);
    c.recs.push_back(std::move(r));
  }
}

// Texts above this size are parsed by several threads, one chunk of whole
// lines each (at least this many bytes a chunk); selections above
// kParallelFillAtoms atoms fill their output arrays on several threads.
constexpr int64_t kParallelParseBytes = 1 << 20;
constexpr int64_t kParseChunkBytes = 1 << 19;
constexpr size_t kParallelFillAtoms = 1 << 14;

// Every MODEL record starts a model; records outside MODEL/ENDMDL join the
// current model (a first one if there is none).  Chunks are stitched in
// order, so the models are those of one pass over the text.  A chunk that
// failed is parsed again alone from its first line number, which raises the
// error of its first malformed line: the first in the text, since the
// chunks before it parsed cleanly.
Models read_pdb(const char* text, int64_t len) {
  const int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
  const int n_chunks =
      len < kParallelParseBytes ? 1 : (int)std::min<int64_t>({hw, (int64_t)16, len / kParseChunkBytes});
  std::vector<const char*> cut(n_chunks + 1);
  cut[0] = text;
  cut[n_chunks] = text + len;
  for (int k = 1; k < n_chunks; ++k) {
    const char* at = std::max(cut[k - 1], text + len * k / n_chunks);
    const char* nl = (const char*)memchr(at, '\n', (size_t)(text + len - at));
    cut[k] = nl ? nl + 1 : text + len;
  }
  std::vector<PdbChunk> chunks(n_chunks);
  auto run = [&](int k) {
    try {
      parse_pdb_lines(cut[k], cut[k + 1], 1, chunks[k]);
    } catch (...) {
      chunks[k].failed = true;
    }
  };
  if (n_chunks == 1) {
    parse_pdb_lines(text, text + len, 1, chunks[0]);
  } else {
    std::vector<std::thread> pool;
    for (int k = 1; k < n_chunks; ++k) pool.emplace_back(run, k);
    run(0);
    for (auto& t : pool) t.join();
  }
  Models models;
  int64_t first_line = 1;
  for (int k = 0; k < n_chunks; ++k) {
    PdbChunk& c = chunks[k];
    if (c.failed) {
      PdbChunk again;
      parse_pdb_lines(cut[k], cut[k + 1], first_line, again);  // throws the error
      c = std::move(again);
    }
    first_line += c.lines;
    const size_t n_seg = c.model_starts.size();
    auto append = [&](size_t from, size_t to) {
      std::vector<const Record*>& m = models.list.back();
      for (size_t i = from; i < to; ++i) m.push_back(&c.recs[i]);
    };
    const size_t head_end = n_seg ? c.model_starts[0] : c.recs.size();
    if (head_end > 0) {
      if (models.list.empty()) models.list.emplace_back();
      append(0, head_end);
    }
    for (size_t s = 0; s < n_seg; ++s) {
      models.list.emplace_back();
      append(c.model_starts[s], s + 1 < n_seg ? c.model_starts[s + 1] : c.recs.size());
    }
    models.store.push_back(std::move(c.recs));  // moving the vector keeps the records' addresses
  }
  return models;
}

// mmCIF: the _atom_site loop; chain, residue number, residue and atom names
// come from the auth_* items when present, else the label_* items.
std::vector<std::string> cif_tokens(const std::string& line) {
  std::vector<std::string> t;
  size_t i = 0;
  while (i < line.size()) {
    while (i < line.size() && std::isspace((unsigned char)line[i])) ++i;
    if (i >= line.size()) break;
    if (line[i] == '\'' || line[i] == '"') {
      const char q = line[i];
      size_t j = i + 1;
      while (j < line.size() && !(line[j] == q && (j + 1 == line.size() || std::isspace((unsigned char)line[j + 1]))))
        ++j;
      t.push_back(line.substr(i + 1, j - i - 1));
      i = j + 1;
    } else {
      size_t j = i;
      while (j < line.size() && !std::isspace((unsigned char)line[j])) ++j;
      t.push_back(line.substr(i, j - i));
      i = j;
    }
  }
  return t;
}

std::vector<std::vector<Record>> read_cif_records(const char* text, int64_t len) {
  std::istringstream in(std::string(text, (size_t)len));
  std::string line;
  std::vector<std::string> cols;
  std::vector<std::string> pending;
  std::vector<std::vector<Record>> models;
  std::map<std::string, size_t> model_of;
  bool in_header = false, in_rows = false, seen = false;
  int64_t line_no = 0;
  auto col = [&](const char* name) -> int {
    for (size_t k = 0; k < cols.size(); ++k)
      if (cols[k] == name) return (int)k;
    return -1;
  };
  auto flush_row = [&](const std::vector<std::string>& v) {
    auto get = [&](const char* a, const char* b) -> std::string {
      int k = col(a);
      if (k < 0 || (k < (int)v.size() && (v[k] == "?" || v[k] == "."))) k = b ? col(b) : -1;
      if (k < 0 || k >= (int)v.size()) return std::string();
      return (v[k] == "?" || v[k] == ".") ? std::string() : v[k];
    };
    Record r;
    const std::string grp = get("group_PDB", nullptr);
    r.hetatm = grp == "HETATM";
    r.name = get("auth_atom_id", "label_atom_id");
    r.alt = get("label_alt_id", nullptr);
    r.resname = get("auth_comp_id", "label_comp_id");
    r.chain = get("auth_asym_id", "label_asym_id");
    const std::string seq = get("auth_seq_id", "label_seq_id");
    r.resseq = seq.empty() ? 0 : integer(seq, "residue number", line_no);
    r.icode = get("pdbx_PDB_ins_code", nullptr);
    r.x = number(get("Cartn_x", nullptr), "x coordinate", line_no);
    r.y = number(get("Cartn_y", nullptr), "y coordinate", line_no);
    r.z = number(get("Cartn_z", nullptr), "z coordinate", line_no);
    const std::string o = get("occupancy", nullptr);
    r.occ = o.empty() ? 1.0 : number(o, "occupancy", line_no);
    r.element = get("type_symbol", nullptr);
    if (r.name.empty()) fail(CRAB_EPARSE, "line " + std::to_string(line_no) + ": missing atom name");
    const std::string m = get("pdbx_PDB_model_num", nullptr);
    auto it = model_of.find(m);
    if (it == model_of.end()) {
      it = model_of.emplace(m, models.size()).first;
      models.emplace_back();
    }
    models[it->second].push_back(std::move(r));
  };
  while (std::getline(in, line)) {
    ++line_no;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    const std::string t = trim(line);
    if (t.empty() || t[0] == '#') {
      if (in_rows) in_rows = in_header = false;
      continue;
    }
    if (t == "loop_") {
      in_header = in_rows = false;
      cols.clear();
      in_header = true;
      continue;
    }
    if (in_header && t.rfind("_atom_site.", 0) == 0) {
      cols.push_back(t.substr(11));
      continue;
    }
    if (in_header && !cols.empty() && t[0] != '_') {
      in_header = false;
      in_rows = true;
      seen = true;
    } else if (in_header && t[0] == '_') {
      in_header = false;  // another category's loop
      cols.clear();
      continue;
    }
    if (in_rows) {
      if (t[0] == '_' || t.rfind("loop_", 0) == 0 || t.rfind("data_", 0) == 0) {
        in_rows = false;
        continue;
      }
      auto tok = cif_tokens(t);
      pending.insert(pending.end(), tok.begin(), tok.end());
      while (pending.size() >= cols.size()) {
        std::vector<std::string> row(pending.begin(), pending.begin() + (long)cols.size());
        pending.erase(pending.begin(), pending.begin() + (long)cols.size());
        flush_row(row);
      }
    }
  }
  if (!seen) fail(CRAB_EPARSE, "no _atom_site loop in the mmCIF data");
  if (!pending.empty()) fail(CRAB_EPARSE, "truncated _atom_site row");
  return models;
}

// structure.rs:37-86
enum Kind { kPolymer, kGlycan, kWater, kOther };
Kind residue_kind(const std::string& name) {
  const std::string c = upper(trim(name));
  if (c == "HOH" || c == "WAT" || c == "DOD") return kWater;
  static const char* kGlycans[] = {"NAG", "NDG", "BMA", "MAN", "GLC", "GAL", "FUC", "SIA", "NAN", "NEU",
                                   "XYS", "XYP", "ARA", "ARB", "RIB", "FRU", "G6D", "G1P", "BGC", "AFD",
                                   "AGS", "AMU", "API", "DGA", "DGL", "DGU", "GCU", "GTR", "IDR", "LBT",
                                   "MMA", "RM4", "SUC", "TRE", "MAL", "LMT", "KDO", "KDN", "DAN", "XUL"};
  for (const char* g : kGlycans)
    if (c == g) return kGlycan;
  static const char* kPolymers[] = {"ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE", "LEU",
                                    "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL", "A",   "C",
                                    "G",   "U",   "T",   "DA",  "DC",  "DG",  "DT"};
  for (const char* g : kPolymers)
    if (c == g) return kPolymer;
  return kOther;
}

// structure.rs:109-127 Element::from_symbol
int element_from_symbol(const std::string& s) {
  const std::string u = upper(trim(s));
  static const std::pair<const char*, int> kMap[] = {
      {"H", CRAB_EL_H},   {"D", CRAB_EL_H},   {"C", CRAB_EL_C},   {"N", CRAB_EL_N},   {"O", CRAB_EL_O},
      {"S", CRAB_EL_S},   {"P", CRAB_EL_P},   {"NA", CRAB_EL_NA}, {"MG", CRAB_EL_MG}, {"CL", CRAB_EL_CL},
      {"CA", CRAB_EL_CA}, {"FE", CRAB_EL_FE}, {"ZN", CRAB_EL_ZN}, {"K", CRAB_EL_K},   {"I", CRAB_EL_I}};
  for (const auto& m : kMap)
    if (u == m.first) return m.second;
  return CRAB_EL_OTHER;
}

// Composite keys: fields joined by a unit separator.
std::string residue_key(const Record& r) {
  std::string k = r.chain;
  k += '\x1f';
  k += std::to_string(r.resseq);
  k += '\x1f';
  k += r.icode;
  return k;
}

// Blank-altloc atoms of a residue that also has named altlocs go into every
// named conformer with occupancy / (named + 1), in the named conformers' order.
std::vector<Record> expand_conformers(const std::vector<const Record*>& in) {
  struct Res {
    std::vector<size_t> atoms;
    std::vector<std::string> alts;
  };
  std::vector<Res> res;
  std::unordered_map<std::string, size_t> index;
  for (size_t i = 0; i < in.size(); ++i) {
    const std::string key = residue_key(*in[i]);
    auto it = index.find(key);
    if (it == index.end()) {
      it = index.emplace(key, res.size()).first;
      res.emplace_back();
    }
    Res& r = res[it->second];
    r.atoms.push_back(i);
    if (!in[i]->alt.empty() && std::find(r.alts.begin(), r.alts.end(), in[i]->alt) == r.alts.end())
      r.alts.push_back(in[i]->alt);
  }
  std::vector<Record> out;
  out.reserve(in.size());
  for (const Res& r : res) {
    for (size_t i : r.atoms) {
      const Record& a = *in[i];
      if (!a.alt.empty() || r.alts.empty()) {
        out.push_back(a);
        continue;
      }
      for (const auto& alt : r.alts) {
        Record c = a;
        c.alt = alt;
        c.occ = a.occ / (double)(r.alts.size() + 1);
        out.push_back(c);
      }
    }
  }
  return out;
}

// Dense ids of distinct strings, then their ranks in byte order, so that
// comparing ranks compares the strings.
struct Ranks {
  std::unordered_map<std::string, uint32_t> id;
  std::vector<const std::string*> str;
  std::vector<uint32_t> rank;
  const std::string* last = nullptr;
  uint32_t last_id = 0;
  uint32_t add(const std::string& s) {
    if (last && *last == s) return last_id;
    auto it = id.find(s);
    if (it == id.end()) {
      it = id.emplace(s, (uint32_t)str.size()).first;
      str.push_back(&it->first);
    }
    last = &it->first;
    last_id = it->second;
    return it->second;
  }
  void finish() {
    std::vector<uint32_t> order(str.size());
    for (uint32_t k = 0; k < order.size(); ++k) order[k] = k;
    std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return *str[a] < *str[b]; });
    rank.assign(str.size(), 0);
    for (uint32_t k = 0; k < order.size(); ++k) rank[order[k]] = k;
  }
};

crab_parsed* select_atoms(const std::vector<const Record*>& model_in, const crab_parse_options& o) {
  std::vector<Record> expanded;
  std::vector<const Record*> expanded_list;
  bool any_alt = false;
  for (const Record* r : model_in) any_alt = any_alt || !r->alt.empty();
  if (any_alt) {
    expanded = expand_conformers(model_in);
    expanded_list.reserve(expanded.size());
    for (const Record& r : expanded) expanded_list.push_back(&r);
  }
  const std::vector<const Record*>& model = any_alt ? expanded_list : model_in;
  std::vector<std::string> chains;
  for (int32_t k = 0; k < o.n_chains; ++k) chains.emplace_back(o.chains[k] ? o.chains[k] : "");
  static const std::string kUnk("UNK");

  // filters and elements (structure.rs:243-272), in file order
  struct Kept {
    uint32_t rec, chain, icode, name, resname;
    int element;
  };
  std::vector<Kept> kept;
  kept.reserve(model.size());
  Ranks chain_r, icode_r, name_r, res_r;
  for (uint32_t i = 0; i < (uint32_t)model.size(); ++i) {
    const Record& r = *model[i];
    const std::string& resname = r.resname.empty() ? kUnk : r.resname;
    if (o.n_chains > 0 && std::find(chains.begin(), chains.end(), r.chain) == chains.end()) continue;
    if (r.hetatm) {
      const Kind kind = residue_kind(resname);
      if (kind == kWater && !o.include_waters) continue;
      if (!o.include_hetatm && !(o.include_glycans && kind == kGlycan)) continue;
    }
    const int el = r.el >= 0 ? r.el : element_from_symbol(r.element.empty() ? r.name : r.element);
    if (el == CRAB_EL_OTHER && !o.allow_unknown_elements) fail(CRAB_EELEMENT, "unsupported element: " + r.name);
    kept.push_back({i, chain_r.add(r.chain), icode_r.add(r.icode), name_r.add(r.name), res_r.add(resname), el});
  }
  chain_r.finish();
  icode_r.finish();
  name_r.finish();
  res_r.finish();

  // groups of alternates: records sorted by (chain, residue number, name,
  // insertion code, file order); a group is a run of equal keys
  struct Key {
    uint64_t a, b;
    uint32_t k;  // index into kept
  };
  std::vector<Key> keys(kept.size());
  for (uint32_t k = 0; k < (uint32_t)kept.size(); ++k) {
    const Kept& e = kept[k];
    const uint64_t seq = (uint64_t)((int64_t)model[e.rec]->resseq + ((int64_t)1 << 40));
    keys[k] = {((uint64_t)chain_r.rank[e.chain] << 42) | (seq & (((uint64_t)1 << 42) - 1)),
               ((uint64_t)name_r.rank[e.name] << 32) | icode_r.rank[e.icode], k};
  }
  std::sort(keys.begin(), keys.end(), [](const Key& x, const Key& y) {
    if (x.a != y.a) return x.a < y.a;
    if (x.b != y.b) return x.b < y.b;
    return x.k < y.k;
  });
  // groups that share (chain, residue number, name) but differ in insertion
  // code keep the order in which they first appear (the reference's stable sort)
  struct Group {
    size_t begin, end;
  };
  std::vector<Group> groups;
  for (size_t s0 = 0; s0 < keys.size();) {
    size_t run_end = s0;
    while (run_end < keys.size() && keys[run_end].a == keys[s0].a && (keys[run_end].b >> 32) == (keys[s0].b >> 32))
      ++run_end;
    const size_t first_group = groups.size();
    for (size_t g = s0; g < run_end;) {
      size_t e = g;
      while (e < run_end && keys[e].b == keys[g].b) ++e;
      groups.push_back({g, e});
      g = e;
    }
    if (groups.size() - first_group > 1)
      std::sort(groups.begin() + (long)first_group, groups.end(),
                [&](const Group& x, const Group& y) { return keys[x.begin].k < keys[y.begin].k; });
    s0 = run_end;
  }

  struct Out {
    uint32_t k;
    double occ;
  };
  std::vector<Out> atoms;
  atoms.reserve(groups.size());
  auto occ_of = [&](size_t s) { return std::max(model[kept[keys[s].k].rec]->occ, 0.0); };
  for (const Group& g : groups) {
    if (o.altloc_policy == CRAB_ALTLOC_ALL) {
      for (size_t s = g.begin; s < g.end; ++s) atoms.push_back({keys[s].k, occ_of(s)});
      continue;
    }
    const size_t count = g.end - g.begin;
    const bool has_alt = count > 1;
    const Record& r0 = *model[kept[keys[g.begin].k].rec];
    bool same_pos = has_alt;
    for (size_t s = g.begin + 1; s < g.end && same_pos; ++s) {
      const Record& r = *model[kept[keys[s].k].rec];
      same_pos = r.x == r0.x && r.y == r0.y && r.z == r0.z;
    }
    size_t pick = g.begin;
    if (o.altloc_policy == CRAB_ALTLOC_HIGHEST)
      for (size_t s = g.begin + 1; s < g.end; ++s)  // the last of equal maxima
        if (occ_of(s) >= occ_of(pick)) pick = s;
    double occ = occ_of(pick);
    if (o.occupancy_policy == CRAB_OCC_SELECTED_FULL && has_alt) occ = 1.0;
    else if (o.occupancy_policy == CRAB_OCC_REPORTED && same_pos) occ = std::min(occ * (double)(count + 1), 1.0);
    atoms.push_back({keys[pick].k, occ});
  }

  auto* p = new crab_parsed();
  const size_t n = atoms.size();
  p->xyz.resize(3 * n);
  p->occ.resize(n);
  p->element.resize(n);
  p->group.resize(n);
  p->hetatm.resize(n);
  p->residue_id.resize(n);
  const Ranks* fields[3] = {&name_r, &res_r, &chain_r};
  for (int f = 0; f < 3; ++f) {
    p->text_id[f].resize(n);
    for (const std::string* str : fields[f]->str) p->text_table[f].push_back(*str);
  }
  // every atom's fields are independent: large structures fill them in
  // ranges on several threads, each with its own group cache
  auto fill = [&](size_t a, size_t b) {
    std::unordered_map<uint64_t, int8_t> group_cache;  // (residue name, atom name) -> united-atom group
    for (size_t i = a; i < b; ++i) {
      const Kept& e = kept[atoms[i].k];
      const Record& r = *model[e.rec];
      p->xyz[3 * i] = r.x;
      p->xyz[3 * i + 1] = r.y;
      p->xyz[3 * i + 2] = r.z;
      p->occ[i] = atoms[i].occ;
      p->element[i] = (int8_t)e.element;
      p->text_id[0][i] = e.name;
      p->text_id[1][i] = e.resname;
      p->text_id[2][i] = e.chain;
      const uint64_t gk = ((uint64_t)e.resname << 32) | e.name;
      auto it = group_cache.find(gk);
      if (it == group_cache.end())
        it = group_cache.emplace(gk, (int8_t)united_atom_group(res_r.str[e.resname]->c_str(), r.name.c_str())).first;
      p->group[i] = it->second;
      p->hetatm[i] = r.hetatm ? 1 : 0;
      p->residue_id[i] = r.resseq;
    }
  };
  const size_t n_fill = n < kParallelFillAtoms ? 1
                                               : std::min<size_t>({(size_t)std::max(1u, std::thread::hardware_concurrency()),
                                                                   16, n / (kParallelFillAtoms / 2)});
  if (n_fill <= 1) {
    fill(0, n);
  } else {
    std::vector<std::thread> pool;
    for (size_t k = 1; k < n_fill; ++k) pool.emplace_back(fill, n * k / n_fill, n * (k + 1) / n_fill);
    fill(0, n / n_fill);
    for (auto& t : pool) t.join();
  }
  return p;
}

bool looks_like_cif(const char* text, int64_t len) {
  int64_t i = 0;
  while (i < len && std::isspace((unsigned char)text[i])) ++i;
  if (len - i >= 5 && std::strncmp(text + i, "data_", 5) == 0) return true;
  const std::string head(text, (size_t)std::min<int64_t>(len, 1 << 16));
  return head.find("_atom_site.") != std::string::npos;
}

Models read_models(const char* text, int64_t len, int format) {
  const bool cif = format == CRAB_FORMAT_MMCIF || (format == CRAB_FORMAT_AUTO && looks_like_cif(text, len));
  if (!cif) return read_pdb(text, len);
  Models m;
  m.store = read_cif_records(text, len);
  for (const auto& v : m.store) {
    m.list.emplace_back();
    for (const Record& r : v) m.list.back().push_back(&r);
  }
  return m;
}

template <class F>
int parse_guard(F&& f) {
  try {
    f();
    g_parse_error.clear();
    return CRAB_OK;
  } catch (const ParseFail& e) {
    g_parse_error = e.msg;
    return e.code;
  } catch (const Error& e) {
    g_parse_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_parse_error = "out of host memory";
    return CRAB_ENOMEM;
  } catch (const std::exception& e) {
    g_parse_error = e.what();
    return CRAB_EINVAL;
  }
}

void validate(const crab_parse_options* o) {
  if (!o) fail(CRAB_EINVAL, "null parse options");
  if (o->model_index < 0) fail(CRAB_EINVAL, "negative model index");
  if (o->altloc_policy < 0 || o->altloc_policy > CRAB_ALTLOC_ALL) fail(CRAB_EINVAL, "unknown altloc policy");
  if (o->occupancy_policy < 0 || o->occupancy_policy > CRAB_OCC_SELECTED_FULL)
    fail(CRAB_EINVAL, "unknown occupancy policy");
  if (o->n_chains < 0 || (o->n_chains > 0 && !o->chains)) fail(CRAB_EINVAL, "invalid chain list");
}

}  // namespace
}  // namespace crab

using namespace crab;

extern "C" {

void crab_parse_options_default(crab_parse_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->include_glycans = 1;
  o->altloc_policy = CRAB_ALTLOC_HIGHEST;
  o->occupancy_policy = CRAB_OCC_REPORTED;
}

const char* crab_parse_last_error(void) { return g_parse_error.c_str(); }

int crab_parse_structure(const char* text, int64_t len, int32_t format, const crab_parse_options* options,
                         crab_parsed** out) {
  if (!out) return CRAB_EINVAL;
  *out = nullptr;
  return parse_guard([&]() {
    if (!text && len > 0) fail(CRAB_EINVAL, "null text");
    if (len < 0) fail(CRAB_EINVAL, "negative text length");
    if (format < CRAB_FORMAT_AUTO || format > CRAB_FORMAT_MMCIF) fail(CRAB_EINVAL, "unknown format");
    validate(options);
    const Models models = read_models(text, len, format);
    if ((size_t)options->model_index >= models.list.size())
      fail(CRAB_EPARSE, "model " + std::to_string(options->model_index) + " is not present");
    *out = select_atoms(models.list[(size_t)options->model_index], *options);
  });
}

int crab_parse_model_count(const char* text, int64_t len, int32_t format, int32_t* n_models) {
  if (!n_models) return CRAB_EINVAL;
  return parse_guard([&]() {
    if ((!text && len > 0) || len < 0) fail(CRAB_EINVAL, "invalid text");
    *n_models = (int32_t)read_models(text, len, format).list.size();
  });
}

int crab_read_structure_file(const char* path, const crab_parse_options* options, crab_parsed** out) {
  if (!out || !path) return CRAB_EINVAL;
  *out = nullptr;
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    g_parse_error = std::string("cannot open ") + path;
    return CRAB_EIO;
  }
  std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  std::string ext(path);
  const size_t dot = ext.find_last_of('.');
  ext = dot == std::string::npos ? std::string() : upper(ext.substr(dot + 1));
  const int32_t format = (ext == "CIF" || ext == "MMCIF") ? CRAB_FORMAT_MMCIF : CRAB_FORMAT_PDB;
  return crab_parse_structure(text.data(), (int64_t)text.size(), format, options, out);
}

int64_t crab_parsed_atom_count(const crab_parsed* p) { return p ? (int64_t)p->occ.size() : -1; }

int crab_parsed_arrays(const crab_parsed* p, double* xyz, double* occupancy, int8_t* element, int8_t* group,
                       int8_t* hetatm, int64_t* residue_id) {
  if (!p) return CRAB_EINVAL;
  const size_t n = p->occ.size();
  if (xyz) std::copy(p->xyz.begin(), p->xyz.end(), xyz);
  if (occupancy) std::copy(p->occ.begin(), p->occ.end(), occupancy);
  if (element) std::copy(p->element.begin(), p->element.end(), element);
  if (group) std::copy(p->group.begin(), p->group.end(), group);
  if (hetatm) std::copy(p->hetatm.begin(), p->hetatm.end(), hetatm);
  if (residue_id) std::copy(p->residue_id.begin(), p->residue_id.begin() + (long)n, residue_id);
  return CRAB_OK;
}

const char* crab_parsed_atom_name(const crab_parsed* p, int64_t i) {
  return (p && i >= 0 && (size_t)i < p->occ.size()) ? p->text(0, (size_t)i).c_str() : nullptr;
}
const char* crab_parsed_residue_name(const crab_parsed* p, int64_t i) {
  return (p && i >= 0 && (size_t)i < p->occ.size()) ? p->text(1, (size_t)i).c_str() : nullptr;
}
const char* crab_parsed_chain_id(const crab_parsed* p, int64_t i) {
  return (p && i >= 0 && (size_t)i < p->occ.size()) ? p->text(2, (size_t)i).c_str() : nullptr;
}

int crab_parsed_strings(const crab_parsed* p, int32_t which, char* buf, int64_t cap, int64_t* len) {
  if (!p || !len || which < 0 || which > 2 || cap < 0 || (cap > 0 && !buf)) return CRAB_EINVAL;
  const std::vector<uint32_t>& ids = p->text_id[which];
  const std::vector<std::string>& table = p->text_table[which];
  int64_t need = 0;
  for (uint32_t id : ids) need += (int64_t)table[id].size() + 1;
  *len = need;
  if (!buf) return CRAB_OK;
  if (cap < need) return CRAB_ECAPACITY;
  char* o = buf;
  for (uint32_t id : ids) {
    const std::string& x = table[id];
    std::memcpy(o, x.data(), x.size());
    o += x.size();
    *o++ = '\n';
  }
  return CRAB_OK;
}

int crab_parsed_destroy(crab_parsed* p) {
  delete p;
  return CRAB_OK;
}

int crab_structure_from_parsed(crab_ctx* ctx, const crab_parsed* p, crab_struct** out) {
  if (!ctx || !p || !out) return CRAB_EINVAL;
  const int64_t n = (int64_t)p->occ.size();
  return crab_structure_create(ctx, p->xyz.data(), p->occ.data(), p->element.data(), p->group.data(), n, out);
}

}  // extern "C"
