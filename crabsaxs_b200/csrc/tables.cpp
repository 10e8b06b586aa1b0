// Host-side physics tables of the engine: X-ray form factors, displaced
// volumes, van der Waals radii and the united-atom typing of standard
// residues.  The coefficient values are physical data that must equal the
// reference's tables for parity: Cromer–Mann 4-Gaussian fits (International
// Tables for Crystallography Vol. C, Table 6.1.1.4) as listed in crabSAXS
// src/formfactor.rs:52-121, the united-atom 5-Gaussian fits of Grudinin et al.
// (2017) Table 2 as listed in src/formfactor.rs:204-277, displaced volumes
// src/solvent.rs:406-424 and radii src/solvent.rs:235-253.

#include <cctype>
#include <cmath>
#include <cstring>
#include <string>

#include "engine.hpp"

namespace crab {
namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;

struct Gauss {
  int terms;       // 4 (Cromer–Mann) or 5 (united atom)
  double a[5];
  double b[5];
  double c;
};

// Element order H C N O S P Na Mg Cl Ca Fe Zn K I Other (structure.rs:90-106).
const Gauss kElement[15] = {
    {4, {0.493002, 0.322912, 0.140191, 0.04081}, {10.5109, 26.1257, 3.14236, 57.7997}, 0.003038},
    {4, {2.31, 1.02, 1.5886, 0.865}, {20.8439, 10.2075, 0.5687, 51.6512}, 0.2156},
    {4, {12.2126, 3.1322, 2.0125, 1.1663}, {0.0057, 9.8933, 28.9975, 0.5826}, -11.529},
    {4, {3.0485, 2.2868, 1.5463, 0.867}, {13.2771, 5.7011, 0.3239, 32.9089}, 0.2508},
    {4, {6.9053, 5.2034, 1.4379, 1.5863}, {1.4679, 22.2151, 0.2536, 56.172}, 0.8669},
    {4, {6.4345, 4.1791, 1.7800, 1.4908}, {1.9067, 27.1570, 0.5260, 68.1645}, 1.1149},
    {4, {4.7626, 3.1736, 1.2674, 1.1128}, {3.285, 8.8422, 0.3136, 129.424}, 0.676},
    {4, {5.4204, 2.1735, 1.2269, 2.3073}, {2.8275, 79.2611, 0.3808, 7.1937}, 0.8584},
    {4, {11.4604, 7.1964, 6.2556, 1.6455}, {0.0104, 1.1662, 18.5194, 47.7784}, -9.5574},
    {4, {8.6266, 7.3873, 1.5899, 1.0211}, {10.4421, 0.6599, 85.7484, 178.437}, 1.3751},
    {4, {11.7695, 7.3573, 3.5222, 2.3045}, {4.7611, 0.3072, 15.3535, 76.8805}, 1.0369},
    {4, {14.0743, 7.0318, 5.1652, 2.41}, {3.2655, 0.2333, 10.3163, 58.7097}, 1.3041},
    {4, {8.2186, 7.4398, 1.0519, 0.8659}, {12.7949, 0.7748, 213.187, 41.6841}, 1.4228},
    {4, {20.1472, 18.9949, 7.5138, 2.2735}, {4.347, 0.3814, 27.766, 66.8776}, 4.0712},
    {4, {0, 0, 0, 0}, {0, 0, 0, 0}, 0.0},
};

// United-atom groups in formfactor.rs:168-183 order.
const Gauss kGroup[14] = {
    {5, {2.909530, 0.485267, 1.516151, 0.206905, 1.541626}, {13.933084, 23.221524, 41.990403, 4.974183, 0.679266}, 0.337670},
    {5, {3.275723, 0.870037, 1.534606, 0.395078, 1.544562}, {13.408502, 23.785175, 41.922444, 5.019072, 0.724439}, 0.377096},
    {5, {3.681341, 1.228691, 1.549320, 0.574033, 1.554377}, {13.026207, 24.131974, 41.869426, 4.984373, 0.765769}, 0.409294},
    {5, {2.168070, 1.275811, 1.561096, 0.742395, -6.151144}, {12.642907, 18.420069, 41.768517, 1.535360, -0.045937}, 7.400917},
    {5, {0.456221, 3.219608, 0.812773, 2.666928, 1.380927}, {21.503498, 13.397134, 34.547137, 5.826620, 0.412902}, 0.463202},
    {5, {3.213280, 0.463019, 0.815724, 2.664450, 1.384266}, {13.383078, 21.362223, 34.531415, 5.823549, 0.410805}, 0.458919},
    {5, {0.688944, 2.929687, 0.416472, 2.606983, 1.319232}, {29.319200, 6.572228, 64.951658, 16.267799, 0.455640}, 0.537548},
    {5, {1.650531, 0.429639, 2.144736, 1.851894, 1.408921}, {10.603730, 6.987283, 29.939901, 10.573859, 0.611678}, 0.510589},
    {5, {1.904157, 1.942536, 2.435585, 0.730512, 1.379728}, {10.803702, 10.792421, 29.610479, 6.847755, 0.709687}, 0.603738},
    {5, {1.426540, 0.426903, 1.878894, 1.608251, 1.200216}, {10.652268, 7.017651, 29.878525, 10.619493, 0.631765}, 0.456024},
    {5, {1.882162, 1.933200, 2.465843, 0.927311, 1.190889}, {10.975157, 10.956008, 29.208572, 6.663555, 0.843650}, 0.597322},
    {5, {3.630164, 0.228310, 1.869734, 0.170550, 1.440894}, {10.267139, 25.118086, 30.241288, 3.412776, 0.486644}, 0.323504},
    {5, {1.792216, 0.724464, 2.347044, 1.903020, 1.313042}, {10.830060, 6.846763, 29.579607, 10.800018, 0.720448}, 0.583312},
    {5, {0.570042, 6.337416, 1.641643, 5.398549, 1.527982}, {11.447986, 1.197657, 55.401032, 22.420955, 2.356552}, 1.523944},
};

// Covalently attached hydrogens per group (formfactor.rs:186-200).
const double kGroupH[14] = {1, 2, 3, 1, 1, 1, 0, 1, 2, 1, 3, 1, 2, 1};
const double kVolume[15] = {5.15, 16.44, 2.49, 9.13, 26.09, 3.37, 4.45, 1.56, 24.84, 4.19, 7.99, 9.85, 11.01, 44.60, 0.0};
const double kRadius[15] = {1.20, 1.70, 1.55, 1.52, 1.80, 1.80, 2.27, 1.73, 1.75, 2.31, 1.72, 1.39, 2.75, 1.98, 1.70};

double gauss_eval(const Gauss& g, double q) {
  const double s = q / (4.0 * kPi);
  const double s2 = s * s;
  double sum = 0.0;
  for (int k = 0; k < g.terms; ++k) sum += g.a[k] * std::exp(-g.b[k] * s2);
  return sum + g.c;
}

std::string upper_trim(const char* s) {
  std::string t(s ? s : "");
  size_t a = t.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return std::string();
  size_t b = t.find_last_not_of(" \t\r\n");
  t = t.substr(a, b - a + 1);
  for (char& ch : t) ch = (char)std::toupper((unsigned char)ch);
  return t;
}

bool one_of(const std::string& s, std::initializer_list<const char*> xs) {
  for (const char* x : xs)
    if (s == x) return true;
  return false;
}

}  // namespace

double sinc(double x) { return std::fabs(x) < 1e-8 ? 1.0 : std::sin(x) / x; }

double form_factor_value(int element, int group, double q) {
  if (group >= 0) return gauss_eval(kGroup[group], q);
  return gauss_eval(kElement[element], q);
}

double form_factor(int element, int group, double occ, bool implicit_h, double q) {
  if (implicit_h && element == CRAB_EL_H) return 0.0;
  return occ * form_factor_value(element, implicit_h ? group : -1, q);
}

double excluded_volume_for_atom(int element, int group, bool implicit_h) {
  if (implicit_h && element == CRAB_EL_H) return 0.0;
  const double nh = (implicit_h && group >= 0) ? kGroupH[group] : 0.0;
  return kVolume[element] + (implicit_h ? nh * kVolume[CRAB_EL_H] : 0.0);
}

double vdw_radius(int element) { return kRadius[element]; }

double water_form_factor(double q) {
  return gauss_eval(kElement[CRAB_EL_O], q) + 2.0 * gauss_eval(kElement[CRAB_EL_H], q) * sinc(q * 0.9572);
}

double excluded_volume_scale(double q, double c1) {
  const double r = 1.62;
  return (c1 * c1) * c1 * std::exp(-(c1 * c1 - 1.0) * (r * r) * q * q / 4.0);
}

double fraser_gaussian(double q, double volume) {
  return volume * std::exp(-std::pow(volume, 2.0 / 3.0) * q * q / (4.0 * kPi));
}

double adaptive_shell_width(double rg) {
  if (rg <= 15.0) return 3.0;
  if (rg >= 20.0) return 5.0;
  return 3.0 + 0.4 * (rg - 15.0);
}

double adaptive_site_volume(double spacing) {
  if (spacing > 4.0) {
    const double h = spacing / 2.0;
    return 2.0 * ((h * h) * h);
  }
  return (spacing * spacing) * spacing;
}

void debye_class_amplitudes(const AtomClass& c, bool implicit_h, double q, double density, double thickness, double* v,
                            double* e, double* h) {
  *v = form_factor(c.element, c.group, 1.0, implicit_h, q);
  const double volume = excluded_volume_for_atom(c.element, c.group, implicit_h);
  const double radius = std::cbrt(3.0 * volume / (4.0 * kPi));
  *e = density * fraser_gaussian(q, volume);
  const double rs = radius + thickness / 2.0;
  const double shell_volume = 4.0 * kPi * (rs * rs) * thickness;
  *h = density * 0.1 * fraser_gaussian(q, shell_volume);
}

void debye_class_amplitude_rows(const AtomClass& c, bool implicit_h, const double* q, int64_t nq, double density,
                                double thickness, double* v, double* e, double* h) {
  // debye_class_amplitudes at every q, with the class's volumes and their
  // 2/3 powers formed once: the same operations in the same order per q
  // (h may be null: the shell term is not needed with a hydration grid)
  const double volume = excluded_volume_for_atom(c.element, c.group, implicit_h);
  const double radius = std::cbrt(3.0 * volume / (4.0 * kPi));
  const double rs = radius + thickness / 2.0;
  const double shell_volume = 4.0 * kPi * (rs * rs) * thickness;
  const double pv = std::pow(volume, 2.0 / 3.0), ps = std::pow(shell_volume, 2.0 / 3.0);
  for (int64_t k = 0; k < nq; ++k) {
    const double qk = q[k];
    v[k] = form_factor(c.element, c.group, 1.0, implicit_h, qk);
    e[k] = density * (volume * std::exp(-pv * qk * qk / (4.0 * kPi)));
    if (h) h[k] = density * 0.1 * (shell_volume * std::exp(-ps * qk * qk / (4.0 * kPi)));
  }
}

void multipole_class_amplitudes(const AtomClass& c, bool implicit_h, double q, double density, double thickness,
                                double* v, double* e, double* h) {
  const double volume = excluded_volume_for_atom(c.element, c.group, implicit_h);
  const double radius = std::cbrt(3.0 * volume / (4.0 * kPi));
  *e = density * volume * std::exp(-std::pow(volume, 2.0 / 3.0) * q * q / (4.0 * kPi));
  const double sr = radius + thickness / 2.0;
  const double shell_volume = 4.0 * kPi * (sr * sr) * thickness;
  *h = density * 0.1 * shell_volume * std::exp(-q * q * sr * sr / 4.0);
  *v = form_factor(c.element, c.group, 1.0, implicit_h, q);
}

void multipole_class_amplitude_rows(const AtomClass& c, bool implicit_h, const double* q, int64_t nq, double density,
                                    double thickness, double* v, double* e, double* h) {
  // multipole_class_amplitudes at every q, with the class's constants formed
  // once: the same operations in the same order per q (h may be null)
  const double volume = excluded_volume_for_atom(c.element, c.group, implicit_h);
  const double radius = std::cbrt(3.0 * volume / (4.0 * kPi));
  const double pv = std::pow(volume, 2.0 / 3.0);
  const double sr = radius + thickness / 2.0;
  const double shell_volume = 4.0 * kPi * (sr * sr) * thickness;
  for (int64_t k = 0; k < nq; ++k) {
    const double qk = q[k];
    e[k] = density * volume * std::exp(-pv * qk * qk / (4.0 * kPi));
    if (h) h[k] = density * 0.1 * shell_volume * std::exp(-qk * qk * sr * sr / 4.0);
    v[k] = form_factor(c.element, c.group, 1.0, implicit_h, qk);
  }
}

// Residue/atom-name typing of formfactor.rs:280-417.
int united_atom_group(const char* residue_in, const char* name_in) {
  const std::string res = upper_trim(residue_in);
  std::string name = upper_trim(name_in);
  char base = 0;
  if (one_of(res, {"A", "DA", "RA", "ADE"})) base = 'A';
  else if (one_of(res, {"C", "DC", "RC", "CYT"})) base = 'C';
  else if (one_of(res, {"G", "DG", "RG", "GUA"})) base = 'G';
  else if (one_of(res, {"U", "DU", "RU", "URA"})) base = 'U';
  else if (one_of(res, {"T", "DT", "RT", "THY"})) base = 'T';
  if (base) {
    for (char& ch : name)
      if (ch == '*') ch = '\'';
    const bool deoxy = (!res.empty() && res[0] == 'D') || base == 'T';
    if (one_of(name, {"C1'", "C3'", "C4'"})) return 0;
    if (name == "C2'") return deoxy ? 1 : 0;
    if (name == "C5'") return 1;
    if (name == "O2'" && !deoxy) return 4;
    if (one_of(name, {"OP1", "OP2", "O1P", "O2P"})) return 6;
    if (name == "C8" && (base == 'A' || base == 'G')) return 3;
    if (base == 'A' && name == "C2") return 3;
    if (base == 'A' && name == "N6") return 8;
    if (base == 'G' && name == "N1") return 7;
    if (base == 'G' && name == "N2") return 8;
    if (base == 'C' && name == "N4") return 8;
    if ((base == 'C' || base == 'U') && (name == "C5" || name == "C6")) return 3;
    if (base == 'T' && name == "C6") return 3;
    if ((base == 'U' || base == 'T') && name == "N3") return 7;
    if (base == 'T' && (name == "C7" || name == "C5M")) return 2;
    return -1;
  }
  if (!one_of(res, {"ALA", "ARG", "ASN", "ASP", "ASH", "CYS", "CYX", "GLN", "GLU", "GLH", "GLY", "HIS", "HID", "HIE",
                    "HIP", "ILE", "LEU", "LYS", "MET", "MSE", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL", "PCA"}))
    return -1;
  const std::string& r = res;
  const std::string& a = name;
  if (a == "N") return one_of(r, {"PRO", "PCA"}) ? -1 : 7;
  if (a == "CA") return r == "GLY" ? 1 : 0;
  struct Rule {
    const char* residues[6];  // nullptr-terminated
    const char* atoms[6];     // nullptr-terminated
    int group;
  };
  auto listed = [](const std::string& s, const char* const* xs) {
    for (int i = 0; i < 6 && xs[i]; ++i)
      if (s == xs[i]) return true;
    return false;
  };
  static const Rule rules[] = {
      {{"ALA"}, {"CB"}, 2},
      {{"ARG"}, {"CB", "CG", "CD"}, 1},
      {{"ARG"}, {"NE"}, 11},
      {{"ARG"}, {"NH1", "NH2"}, 12},
      {{"ASN", "ASP", "ASH", "CYS", "CYX"}, {"CB"}, 1},
      {{"ASN"}, {"ND2"}, 8},
      {{"ASP", "GLU"}, {"OD1", "OD2", "OE1", "OE2"}, 6},
      {{"ASH"}, {"OD2"}, 5},
      {{"GLH"}, {"OE2"}, 5},
      {{"CYS"}, {"SG"}, 13},
      {{"GLN", "GLU", "GLH"}, {"CB", "CG"}, 1},
      {{"GLN"}, {"NE2"}, 8},
      {{"HIS", "HID", "HIE", "HIP"}, {"CB"}, 1},
      {{"HIS", "HID"}, {"ND1"}, 7},
      {{"HIE"}, {"NE2"}, 7},
      {{"HIP"}, {"ND1", "NE2"}, 9},
      {{"HIS", "HID", "HIE", "HIP"}, {"CD2", "CE1"}, 3},
      {{"ILE", "THR", "VAL"}, {"CB"}, 0},
      {{"LEU"}, {"CG"}, 0},
      {{"ILE"}, {"CG1"}, 1},
      {{"LEU"}, {"CB"}, 1},
      {{"ILE"}, {"CG2", "CD1"}, 2},
      {{"LEU"}, {"CD1", "CD2"}, 2},
      {{"LYS"}, {"CB", "CG", "CD", "CE"}, 1},
      {{"LYS"}, {"NZ"}, 10},
      {{"MET", "MSE"}, {"CB", "CG"}, 1},
      {{"MET", "MSE"}, {"CE"}, 2},
      {{"PHE", "TYR", "TRP"}, {"CB"}, 1},
      {{"PHE"}, {"CD1", "CD2", "CE1", "CE2", "CZ"}, 3},
      {{"TYR"}, {"CD1", "CD2", "CE1", "CE2"}, 3},
      {{"TRP"}, {"CD1", "CE3", "CZ2", "CZ3", "CH2"}, 3},
      {{"PRO"}, {"CB", "CG", "CD"}, 1},
      {{"SER"}, {"CB"}, 1},
      {{"SER"}, {"OG"}, 4},
      {{"THR"}, {"OG1"}, 4},
      {{"TYR"}, {"OH"}, 4},
      {{"THR"}, {"CG2"}, 2},
      {{"VAL"}, {"CG1", "CG2"}, 2},
      {{"TRP"}, {"NE1"}, 7},
      {{"PCA"}, {"CB", "CG"}, 1},
  };
  for (const Rule& rule : rules)
    if (listed(r, rule.residues) && listed(a, rule.atoms)) return rule.group;
  return -1;
}

}  // namespace crab
