// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A plain C++ f64 restatement of the crabSAXS reference algorithms on the
// scattering hot path.  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load this library, and only as the checker or as the
// timed CPU baseline.  Nothing in the crabsaxs_b200 package links or calls it.
//
// The reference is Rust (crate `crabsaxs`).  It cannot be compiled here (no
// cargo/rustc), so this file restates it function by function, keeping the
// reference's f64 arithmetic order (sequential i, then j>i; self term first)
// and its libm calls (sin, cos, exp, pow, cbrt, atan2, sqrt: the same glibc
// routines the Rust standard library calls on Linux).  Build with
// -ffp-contract=off so no multiply-add is fused where Rust would not fuse it.
//
// Parity pin: tests/test_oracle.py checks this file against every closed-form
// and cross-method test the reference holds for the path (scattering.rs,
// spherical.rs, solvent.rs, formfactor.rs, fit.rs, reweight.rs tests).
// Third-party arithmetic on the path: nalgebra 0.33.3 `Vector3::norm` is
// restated as sqrt(((0 + dx*dx) + dy*dy) + dz*dz) in f64.
//
// Element codes follow the reference enum order (structure.rs:90-106):
//   H=0 C=1 N=2 O=3 S=4 P=5 Na=6 Mg=7 Cl=8 Ca=9 Fe=10 Zn=11 K=12 I=13 Other=14
// United-atom group codes follow formfactor.rs:168-183 (-1 = none):
//   CSp3H=0 CSp3H2=1 CSp3H3=2 CAromaticH=3 OAlcoholH=4 OAcidH=5 OResonance=6
//   NH=7 NH2=8 NHPositive=9 NH3Positive=10 GuanidineNH=11 GuanidineNH2=12 SH=13

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#define ORC_API extern "C" __attribute__((visibility("default")))

namespace {

const double PI = 3.14159265358979323846264338327950288;

struct CM4 { double a[4]; double b[4]; double c; };
struct G5 { double a[5]; double b[5]; double c; };

// formfactor.rs:52-121 — International Tables Vol. C, Table 6.1.1.4 values as
// tabulated by the reference (the numbers must be identical for parity).
const CM4 kElementCM[15] = {
    {{0.493002, 0.322912, 0.140191, 0.04081}, {10.5109, 26.1257, 3.14236, 57.7997}, 0.003038},  // H
    {{2.31, 1.02, 1.5886, 0.865}, {20.8439, 10.2075, 0.5687, 51.6512}, 0.2156},                   // C
    {{12.2126, 3.1322, 2.0125, 1.1663}, {0.0057, 9.8933, 28.9975, 0.5826}, -11.529},              // N
    {{3.0485, 2.2868, 1.5463, 0.867}, {13.2771, 5.7011, 0.3239, 32.9089}, 0.2508},                // O
    {{6.9053, 5.2034, 1.4379, 1.5863}, {1.4679, 22.2151, 0.2536, 56.172}, 0.8669},                // S
    {{6.4345, 4.1791, 1.7800, 1.4908}, {1.9067, 27.1570, 0.5260, 68.1645}, 1.1149},               // P
    {{4.7626, 3.1736, 1.2674, 1.1128}, {3.285, 8.8422, 0.3136, 129.424}, 0.676},                  // Na
    {{5.4204, 2.1735, 1.2269, 2.3073}, {2.8275, 79.2611, 0.3808, 7.1937}, 0.8584},                // Mg
    {{11.4604, 7.1964, 6.2556, 1.6455}, {0.0104, 1.1662, 18.5194, 47.7784}, -9.5574},             // Cl
    {{8.6266, 7.3873, 1.5899, 1.0211}, {10.4421, 0.6599, 85.7484, 178.437}, 1.3751},              // Ca
    {{11.7695, 7.3573, 3.5222, 2.3045}, {4.7611, 0.3072, 15.3535, 76.8805}, 1.0369},              // Fe
    {{14.0743, 7.0318, 5.1652, 2.41}, {3.2655, 0.2333, 10.3163, 58.7097}, 1.3041},                // Zn
    {{8.2186, 7.4398, 1.0519, 0.8659}, {12.7949, 0.7748, 213.187, 41.6841}, 1.4228},              // K
    {{20.1472, 18.9949, 7.5138, 2.2735}, {4.347, 0.3814, 27.766, 66.8776}, 4.0712},               // I
    {{0, 0, 0, 0}, {0, 0, 0, 0}, 0.0},                                                            // Other
};

// formfactor.rs:204-277 — Grudinin et al. (2017) Table 2 five-Gaussian fits.
const G5 kGroupG5[14] = {
    {{2.909530, 0.485267, 1.516151, 0.206905, 1.541626}, {13.933084, 23.221524, 41.990403, 4.974183, 0.679266}, 0.337670},
    {{3.275723, 0.870037, 1.534606, 0.395078, 1.544562}, {13.408502, 23.785175, 41.922444, 5.019072, 0.724439}, 0.377096},
    {{3.681341, 1.228691, 1.549320, 0.574033, 1.554377}, {13.026207, 24.131974, 41.869426, 4.984373, 0.765769}, 0.409294},
    {{2.168070, 1.275811, 1.561096, 0.742395, -6.151144}, {12.642907, 18.420069, 41.768517, 1.535360, -0.045937}, 7.400917},
    {{0.456221, 3.219608, 0.812773, 2.666928, 1.380927}, {21.503498, 13.397134, 34.547137, 5.826620, 0.412902}, 0.463202},
    {{3.213280, 0.463019, 0.815724, 2.664450, 1.384266}, {13.383078, 21.362223, 34.531415, 5.823549, 0.410805}, 0.458919},
    {{0.688944, 2.929687, 0.416472, 2.606983, 1.319232}, {29.319200, 6.572228, 64.951658, 16.267799, 0.455640}, 0.537548},
    {{1.650531, 0.429639, 2.144736, 1.851894, 1.408921}, {10.603730, 6.987283, 29.939901, 10.573859, 0.611678}, 0.510589},
    {{1.904157, 1.942536, 2.435585, 0.730512, 1.379728}, {10.803702, 10.792421, 29.610479, 6.847755, 0.709687}, 0.603738},
    {{1.426540, 0.426903, 1.878894, 1.608251, 1.200216}, {10.652268, 7.017651, 29.878525, 10.619493, 0.631765}, 0.456024},
    {{1.882162, 1.933200, 2.465843, 0.927311, 1.190889}, {10.975157, 10.956008, 29.208572, 6.663555, 0.843650}, 0.597322},
    {{3.630164, 0.228310, 1.869734, 0.170550, 1.440894}, {10.267139, 25.118086, 30.241288, 3.412776, 0.486644}, 0.323504},
    {{1.792216, 0.724464, 2.347044, 1.903020, 1.313042}, {10.830060, 6.846763, 29.579607, 10.800018, 0.720448}, 0.583312},
    {{0.570042, 6.337416, 1.641643, 5.398549, 1.527982}, {11.447986, 1.197657, 55.401032, 22.420955, 2.356552}, 1.523944},
};

// formfactor.rs:186-200
const double kGroupHCount[14] = {1, 2, 3, 1, 1, 1, 0, 1, 2, 1, 3, 1, 2, 1};

// solvent.rs:406-424
const double kExcludedVolume[15] = {5.15, 16.44, 2.49, 9.13, 26.09, 3.37, 4.45, 1.56,
                                    24.84, 4.19, 7.99, 9.85, 11.01, 44.60, 0.0};
// solvent.rs:235-253
const double kVdwRadius[15] = {1.20, 1.70, 1.55, 1.52, 1.80, 1.80, 2.27, 1.73,
                               1.75, 2.31, 1.72, 1.39, 2.75, 1.98, 1.70};

// formfactor.rs:40-50 (and FiveGaussian::evaluate 26-38)
double cm_eval(const CM4& t, double q) {
  double s = q / (4.0 * PI);
  double s2 = s * s;
  double sum = 0.0;
  for (int k = 0; k < 4; ++k) sum += t.a[k] * std::exp(-t.b[k] * s2);
  return sum + t.c;
}
double g5_eval(const G5& t, double q) {
  double s = q / (4.0 * PI);
  double s2 = s * s;
  double sum = 0.0;
  for (int k = 0; k < 5; ++k) sum += t.a[k] * std::exp(-t.b[k] * s2);
  return sum + t.c;
}

// formfactor.rs:425-439
double form_factor(int elem, int group, double occ, bool implicit_h, double q) {
  if (implicit_h && elem == 0) return 0.0;
  double value;
  if (implicit_h && group >= 0) value = g5_eval(kGroupG5[group], q);
  else value = cm_eval(kElementCM[elem], q);
  return occ * value;
}

// solvent.rs:428-438
double excluded_volume_for_atom(int elem, int group, bool implicit_h) {
  if (implicit_h && elem == 0) return 0.0;
  double nh = (implicit_h && group >= 0) ? kGroupHCount[group] : 0.0;
  return kExcludedVolume[elem] + (implicit_h ? nh * kExcludedVolume[0] : 0.0);
}

// scattering.rs:62-69
inline double sinc(double x) { return std::fabs(x) < 1e-8 ? 1.0 : std::sin(x) / x; }

// nalgebra Vector3::norm_squared / norm in f64, left-to-right.
inline double norm2(double dx, double dy, double dz) { return ((0.0 + dx * dx) + dy * dy) + dz * dz; }
inline double dist(const double* a, const double* b) {
  return std::sqrt(norm2(a[0] - b[0], a[1] - b[1], a[2] - b[2]));
}

// solvent.rs:441-443
double fraser_gaussian(double q, double volume) {
  return volume * std::exp(-std::pow(volume, 2.0 / 3.0) * q * q / (4.0 * PI));
}

// solvent.rs:448-452
double excluded_volume_scale(double q, double c1) {
  const double r = 1.62;
  return (c1 * c1) * c1 * std::exp(-(c1 * c1 - 1.0) * (r * r) * q * q / 4.0);
}

// solvent.rs:227-231
double water_form_factor(double q) {
  return cm_eval(kElementCM[3], q) + 2.0 * cm_eval(kElementCM[0], q) * sinc(q * 0.9572);
}

// solvent.rs:96-104
double adaptive_shell_width(double rg) {
  if (rg <= 15.0) return 3.0;
  if (rg >= 20.0) return 5.0;
  return 3.0 + 0.4 * (rg - 15.0);
}
// solvent.rs:106-115
double adaptive_site_volume(double spacing) {
  if (spacing > 4.0) { double h = spacing / 2.0; return 2.0 * ((h * h) * h); }
  return (spacing * spacing) * spacing;
}

struct SolventP {
  double c1, c2, thickness, density;
  int model;  // 0 Analytic, 1 Grid, 2 AdaptiveGrid  (solvent.rs:18-25)
  double spacing;
};

// solvent.rs:121-223
int adaptive_grid(int64_t n, const double* xyz, double spacing, double clearance, double padding,
                  std::vector<double>& sites, double* volume) {
  sites.clear();
  if (n == 0) { *volume = adaptive_site_volume(spacing); return 0; }
  if (!std::isfinite(spacing) || spacing <= 0.0 || !std::isfinite(clearance) || clearance <= 0.0 ||
      !std::isfinite(padding) || padding < 0.0)
    return 1;
  double cx = 0, cy = 0, cz = 0;
  for (int64_t i = 0; i < n; ++i) { cx = cx + xyz[3 * i]; cy = cy + xyz[3 * i + 1]; cz = cz + xyz[3 * i + 2]; }
  cx = cx / (double)n; cy = cy / (double)n; cz = cz / (double)n;
  double acc = 0.0;
  for (int64_t i = 0; i < n; ++i) acc += norm2(xyz[3 * i] - cx, xyz[3 * i + 1] - cy, xyz[3 * i + 2] - cz);
  double rg = std::sqrt(acc / (double)n);
  double inner = clearance, outer = clearance + adaptive_shell_width(rg);
  double mn[3] = {xyz[0], xyz[1], xyz[2]}, mx[3] = {xyz[0], xyz[1], xyz[2]};
  for (int64_t i = 1; i < n; ++i)
    for (int d = 0; d < 3; ++d) { mn[d] = std::fmin(mn[d], xyz[3 * i + d]); mx[d] = std::fmax(mx[d], xyz[3 * i + d]); }
  for (int d = 0; d < 3; ++d) { mn[d] = mn[d] - padding; mx[d] = mx[d] + padding; }
  uint64_t dim[3];
  for (int d = 0; d < 3; ++d) dim[d] = (uint64_t)std::ceil(((mx[d] - mn[d]) / spacing) - 1e-10) + 1;
  uint64_t count = dim[0] * dim[1] * dim[2];
  uint64_t nx = dim[0], ny = dim[1], nz = dim[2];
  std::vector<uint8_t> shell(count, 0), mol(count, 0);
  auto rasterize = [&](double radius, std::vector<uint8_t>& mask) {
    double r2 = radius * radius;
    for (int64_t a = 0; a < n; ++a) {
      const double* p = xyz + 3 * a;
      double lo[3], hi[3];
      for (int d = 0; d < 3; ++d) { lo[d] = ((p[d] - radius) - mn[d]) / spacing; hi[d] = ((p[d] + radius) - mn[d]) / spacing; }
      uint64_t x0 = (uint64_t)std::fmax(std::floor(lo[0] - 1e-10), 0.0);
      uint64_t y0 = (uint64_t)std::fmax(std::floor(lo[1] - 1e-10), 0.0);
      uint64_t z0 = (uint64_t)std::fmax(std::floor(lo[2] - 1e-10), 0.0);
      uint64_t x1 = std::min((uint64_t)std::fmax(std::ceil(hi[0] + 1e-10), 0.0), nx - 1);
      uint64_t y1 = std::min((uint64_t)std::fmax(std::ceil(hi[1] + 1e-10), 0.0), ny - 1);
      uint64_t z1 = std::min((uint64_t)std::fmax(std::ceil(hi[2] + 1e-10), 0.0), nz - 1);
      for (uint64_t z = z0; z <= z1; ++z)
        for (uint64_t y = y0; y <= y1; ++y)
          for (uint64_t x = x0; x <= x1; ++x) {
            double px = mn[0] + (double)x * spacing, py = mn[1] + (double)y * spacing, pz = mn[2] + (double)z * spacing;
            if (norm2(px - p[0], py - p[1], pz - p[2]) <= r2 + 1e-10) mask[(z * ny + y) * nx + x] = 1;
          }
    }
  };
  rasterize(outer, shell);
  rasterize(inner, mol);
  for (uint64_t z = 0; z < nz; ++z)
    for (uint64_t y = 0; y < ny; ++y)
      for (uint64_t x = 0; x < nx; ++x) {
        uint64_t c = (z * ny + y) * nx + x;
        if (shell[c] && !mol[c]) {
          sites.push_back(mn[0] + (double)x * spacing);
          sites.push_back(mn[1] + (double)y * spacing);
          sites.push_back(mn[2] + (double)z * spacing);
        }
      }
  *volume = adaptive_site_volume(spacing);
  return 0;
}

// solvent.rs:259-401
int exterior_grid(int64_t n, const double* xyz, const int* elem, double spacing, double probe,
                  double thickness, std::vector<double>& sites, double* volume) {
  sites.clear();
  if (n == 0) { *volume = (spacing * spacing) * spacing; return 0; }
  if (!std::isfinite(spacing) || spacing <= 0.0 || !std::isfinite(probe) || probe < 0.0 ||
      !std::isfinite(thickness) || thickness <= 0.0)
    return 1;
  double vmax = 0.0;
  for (int64_t i = 0; i < n; ++i) vmax = std::fmax(vmax, kVdwRadius[elem[i]]);
  double margin = vmax + probe + thickness + spacing;
  double mn[3] = {xyz[0], xyz[1], xyz[2]}, mx[3] = {xyz[0], xyz[1], xyz[2]};
  for (int64_t i = 1; i < n; ++i)
    for (int d = 0; d < 3; ++d) { mn[d] = std::fmin(mn[d], xyz[3 * i + d]); mx[d] = std::fmax(mx[d], xyz[3 * i + d]); }
  for (int d = 0; d < 3; ++d) { mn[d] = mn[d] - margin; mx[d] = mx[d] + margin; }
  uint64_t dim[3];
  for (int d = 0; d < 3; ++d) dim[d] = (uint64_t)std::ceil(((mx[d] - mn[d]) / spacing) - 1e-10) + 1;
  uint64_t count = dim[0] * dim[1] * dim[2];
  if (count > 250000000ull) return 2;
  uint64_t nx = dim[0], ny = dim[1], nz = dim[2];
  std::vector<uint8_t> state(count, 0);
  auto rasterize = [&](double extra, uint8_t value, bool exterior_only) {
    for (int64_t a = 0; a < n; ++a) {
      const double* p = xyz + 3 * a;
      double radius = kVdwRadius[elem[a]] + extra;
      double lo[3], hi[3];
      for (int d = 0; d < 3; ++d) { lo[d] = ((p[d] - radius) - mn[d]) / spacing; hi[d] = ((p[d] + radius) - mn[d]) / spacing; }
      uint64_t x0 = (uint64_t)std::fmax(std::floor(lo[0] - 1e-10), 0.0);
      uint64_t y0 = (uint64_t)std::fmax(std::floor(lo[1] - 1e-10), 0.0);
      uint64_t z0 = (uint64_t)std::fmax(std::floor(lo[2] - 1e-10), 0.0);
      uint64_t x1 = std::min((uint64_t)std::fmax(std::ceil(hi[0] + 1e-10), 0.0), nx - 1);
      uint64_t y1 = std::min((uint64_t)std::fmax(std::ceil(hi[1] + 1e-10), 0.0), ny - 1);
      uint64_t z1 = std::min((uint64_t)std::fmax(std::ceil(hi[2] + 1e-10), 0.0), nz - 1);
      double r2 = radius * radius;
      for (uint64_t z = z0; z <= z1; ++z)
        for (uint64_t y = y0; y <= y1; ++y)
          for (uint64_t x = x0; x <= x1; ++x) {
            uint64_t c = (z * ny + y) * nx + x;
            double px = mn[0] + (double)x * spacing, py = mn[1] + (double)y * spacing, pz = mn[2] + (double)z * spacing;
            if ((!exterior_only || state[c] == 2) && norm2(px - p[0], py - p[1], pz - p[2]) <= r2 + 1e-10) state[c] = value;
          }
    }
  };
  rasterize(probe, 1, false);
  std::vector<uint64_t> queue;
  queue.reserve(count / 4 + 16);
  for (uint64_t z = 0; z < nz; ++z)
    for (uint64_t y = 0; y < ny; ++y)
      for (uint64_t x = 0; x < nx; ++x) {
        if (x != 0 && x + 1 != nx && y != 0 && y + 1 != ny && z != 0 && z + 1 != nz) continue;
        uint64_t c = (z * ny + y) * nx + x;
        if (state[c] == 0) { state[c] = 2; queue.push_back(c); }
      }
  for (size_t head = 0; head < queue.size(); ++head) {
    uint64_t c = queue[head];
    uint64_t x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
    uint64_t nb[6]; int k = 0;
    if (x > 0) nb[k++] = c - 1;
    if (x + 1 < nx) nb[k++] = c + 1;
    if (y > 0) nb[k++] = c - nx;
    if (y + 1 < ny) nb[k++] = c + nx;
    if (z > 0) nb[k++] = c - nx * ny;
    if (z + 1 < nz) nb[k++] = c + nx * ny;
    for (int t = 0; t < k; ++t)
      if (state[nb[t]] == 0) { state[nb[t]] = 2; queue.push_back(nb[t]); }
  }
  rasterize(probe + thickness, 3, true);
  for (uint64_t z = 0; z < nz; ++z)
    for (uint64_t y = 0; y < ny; ++y)
      for (uint64_t x = 0; x < nx; ++x)
        if (state[(z * ny + y) * nx + x] == 3) {
          sites.push_back(mn[0] + (double)x * spacing);
          sites.push_back(mn[1] + (double)y * spacing);
          sites.push_back(mn[2] + (double)z * spacing);
        }
  *volume = (spacing * spacing) * spacing;
  return 0;
}

int build_grid(int64_t n, const double* xyz, const int* elem, const SolventP& p, std::vector<double>& sites,
               double* volume) {
  if (p.model == 1) return exterior_grid(n, xyz, elem, 1.0, 1.4, p.thickness, sites, volume);  // SolventGridOptions default + thickness
  if (p.model == 2) return adaptive_grid(n, xyz, p.spacing, 3.0, 12.0, sites, volume);           // AdaptiveHydrationOptions default + spacing
  sites.clear();
  *volume = 0.0;
  return 0;
}

// solvent.rs:454-488 (one atom)
void component_amplitudes(int elem, int group, double occ, bool implicit_h, double q, const SolventP& p,
                          double* v, double* e, double* h) {
  *v = form_factor(elem, group, occ, implicit_h, q);
  double volume = excluded_volume_for_atom(elem, group, implicit_h);
  double radius = std::cbrt(3.0 * volume / (4.0 * PI));
  *e = occ * p.density * fraser_gaussian(q, volume);
  double rs = radius + p.thickness / 2.0;
  double shell_volume = 4.0 * PI * (rs * rs) * p.thickness;
  *h = occ * p.density * 0.1 * fraser_gaussian(q, shell_volume);
}

// spherical.rs:33-51
std::vector<double> harmonic_norms(int l_max) {
  std::vector<double> norms((l_max + 1) * (l_max + 1), 0.0);
  for (int l = 0; l <= l_max; ++l)
    for (int m = 0; m <= l; ++m) {
      double ratio = 1.0;
      for (int k = l - m + 1; k <= l + m; ++k) ratio /= (double)k;
      norms[l * l + l + m] = std::sqrt(((double)(2 * l + 1) / (4.0 * PI)) * ratio);
    }
  return norms;
}

// spherical.rs:54-93
void real_harmonics_all(int l_max, double x, double phi, const double* norms, double* out) {
  int count = (l_max + 1) * (l_max + 1);
  for (int k = 0; k < count; ++k) out[k] = 0.0;
  double sin_theta = std::sqrt(std::fmax(1.0 - x * x, 0.0));
  double sin_phi = std::sin(phi), cos_phi = std::cos(phi);
  double sin_m = 0.0, cos_m = 1.0, pmm = 1.0;
  const double sqrt2 = std::sqrt(2.0);
  for (int m = 0; m <= l_max; ++m) {
    if (m > 0) {
      pmm *= -((double)(2 * m - 1)) * sin_theta;
      double next_cos = cos_m * cos_phi - sin_m * sin_phi;
      sin_m = sin_m * cos_phi + cos_m * sin_phi;
      cos_m = next_cos;
    }
    auto emit = [&](int l, double p) {
      int pos = l * l + l + m;
      if (m == 0) out[pos] = norms[pos] * p;
      else {
        double value = sqrt2 * norms[pos] * p;
        out[pos] = value * cos_m;
        out[l * l + l - m] = value * sin_m;
      }
    };
    emit(m, pmm);
    if (m == l_max) continue;
    double pm1 = x * (double)(2 * m + 1) * pmm;
    emit(m + 1, pm1);
    double prev = pmm, cur = pm1;
    for (int l = m + 2; l <= l_max; ++l) {
      double next = ((double)(2 * l - 1) * x * cur - (double)(l + m - 1) * prev) / (double)(l - m);
      emit(l, next);
      prev = cur;
      cur = next;
    }
  }
}

// spherical.rs:95-133 (j has l_max+1 entries; work has >= l_max+26)
void spherical_bessel_all_into(int l_max, double x, double* j, double* work) {
  for (int l = 0; l <= l_max; ++l) j[l] = 0.0;
  if (std::fabs(x) < 1e-8) { j[0] = 1.0; return; }
  if (l_max == 0) { j[0] = std::sin(x) / x; return; }
  int start = l_max + 24;
  for (int l = 0; l < start + 2; ++l) work[l] = 0.0;
  work[start] = 1.0;
  for (int l = start; l >= 1; --l) {
    work[l - 1] = (double)(2 * l + 1) * work[l] / x - work[l + 1];
    if (std::fabs(work[l - 1]) > 1e100)
      for (int k = l - 1; k <= start + 1; ++k) work[k] *= 1e-100;
  }
  double j0 = std::sin(x) / x;
  double j1 = std::sin(x) / (x * x) - std::cos(x) / x;
  double scale = std::fabs(j0) >= std::fabs(j1) ? j0 / work[0] : j1 / work[1];
  for (int l = 0; l <= l_max; ++l) j[l] = work[l] * scale;
}

struct Geometry {
  std::vector<double> radii, harmonics;
  int coeff_count = 0;
  double max_radius = 0.0;
};

// spherical.rs:165-199
Geometry geometry_for_points(int64_t n, const double* pts, const double* centre, int l_max) {
  Geometry g;
  g.coeff_count = (l_max + 1) * (l_max + 1);
  g.radii.resize(n);
  g.harmonics.assign((size_t)n * g.coeff_count, 0.0);
  std::vector<double> norms = harmonic_norms(l_max);
  for (int64_t i = 0; i < n; ++i) {
    double px = pts[3 * i] - centre[0], py = pts[3 * i + 1] - centre[1], pz = pts[3 * i + 2] - centre[2];
    double r = std::sqrt(norm2(px, py, pz));
    g.radii[i] = r;
    double ct, phi;
    if (r < 1e-12) { ct = 1.0; phi = 0.0; }
    else { ct = std::fmin(std::fmax(pz / r, -1.0), 1.0); phi = std::atan2(py, px); }
    real_harmonics_all(l_max, ct, phi, norms.data(), g.harmonics.data() + (size_t)i * g.coeff_count);
  }
  for (int64_t i = 0; i < n; ++i) g.max_radius = std::fmax(g.max_radius, g.radii[i]);
  return g;
}

void centroid(int64_t n, const double* xyz, double* c) {
  double cx = 0, cy = 0, cz = 0;
  for (int64_t i = 0; i < n; ++i) { cx = cx + xyz[3 * i]; cy = cy + xyz[3 * i + 1]; cz = cz + xyz[3 * i + 2]; }
  double d = (double)std::max<int64_t>(n, 1);
  c[0] = cx / d; c[1] = cy / d; c[2] = cz / d;
}

// spherical.rs:201-203
int adaptive_l_max(double q, double max_radius, int maximum) {
  long v = (long)std::ceil(q * max_radius) + 8;
  long lo = std::min(maximum, 8);
  if (v < lo) v = lo;
  if (v > maximum) v = maximum;
  return (int)v;
}

// spherical.rs:205-231
void solvent_components_for_atom(int elem, int group, double occ, bool implicit_h, double q, const SolventP& s,
                                 double* out) {
  double volume = excluded_volume_for_atom(elem, group, implicit_h);
  double radius = std::cbrt(3.0 * volume / (4.0 * PI));
  double excluded = occ * s.density * volume * std::exp(-std::pow(volume, 2.0 / 3.0) * q * q / (4.0 * PI));
  double sr = radius + s.thickness / 2.0;
  double shell_volume = 4.0 * PI * (sr * sr) * s.thickness;
  double hydration = occ * s.density * 0.1 * shell_volume * std::exp(-q * q * sr * sr / 4.0);
  out[0] = form_factor(elem, group, occ, implicit_h, q);
  out[1] = excluded;
  out[2] = hydration;
}

}  // namespace

// ---------------------------------------------------------------- exports

ORC_API double orc_form_factor(int elem, int group, double occ, int implicit_h, double q) {
  return form_factor(elem, group, occ, implicit_h != 0, q);
}
ORC_API double orc_excluded_volume_for_atom(int elem, int group, int implicit_h) {
  return excluded_volume_for_atom(elem, group, implicit_h != 0);
}
ORC_API double orc_excluded_volume_for(int elem) { return kExcludedVolume[elem]; }
ORC_API double orc_vdw_radius(int elem) { return kVdwRadius[elem]; }
ORC_API double orc_water_form_factor(double q) { return water_form_factor(q); }
ORC_API double orc_excluded_volume_scale(double q, double c1) { return excluded_volume_scale(q, c1); }
ORC_API double orc_adaptive_shell_width(double rg) { return adaptive_shell_width(rg); }
ORC_API double orc_sinc(double x) { return sinc(x); }

// formfactor.rs:280-417 — residue/atom-name typing (returns -1 for none).
ORC_API int orc_united_atom_group(const char* residue_in, const char* name_in) {
  auto norm = [](const char* s) {
    std::string t(s ? s : "");
    size_t a = t.find_first_not_of(" \t\r\n"), b = t.find_last_not_of(" \t\r\n");
    t = (a == std::string::npos) ? std::string() : t.substr(a, b - a + 1);
    for (auto& ch : t) ch = (char)std::toupper((unsigned char)ch);
    return t;
  };
  std::string res = norm(residue_in), name = norm(name_in);
  auto in = [](const std::string& s, std::initializer_list<const char*> xs) {
    for (auto x : xs) if (s == x) return true;
    return false;
  };
  char base = 0;
  if (in(res, {"A", "DA", "RA", "ADE"})) base = 'A';
  else if (in(res, {"C", "DC", "RC", "CYT"})) base = 'C';
  else if (in(res, {"G", "DG", "RG", "GUA"})) base = 'G';
  else if (in(res, {"U", "DU", "RU", "URA"})) base = 'U';
  else if (in(res, {"T", "DT", "RT", "THY"})) base = 'T';
  if (base) {  // formfactor.rs:325-355
    for (auto& ch : name) if (ch == '*') ch = '\'';
    bool deoxy = (!res.empty() && res[0] == 'D') || base == 'T';
    if (in(name, {"C1'", "C3'", "C4'"})) return 0;
    if (name == "C2'") return deoxy ? 1 : 0;
    if (name == "C5'") return 1;
    if (name == "O2'" && !deoxy) return 4;
    if (in(name, {"OP1", "OP2", "O1P", "O2P"})) return 6;
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
  if (!in(res, {"ALA", "ARG", "ASN", "ASP", "ASH", "CYS", "CYX", "GLN", "GLU", "GLH", "GLY", "HIS", "HID",
                "HIE", "HIP", "ILE", "LEU", "LYS", "MET", "MSE", "PHE", "PRO", "SER", "THR", "TRP", "TYR",
                "VAL", "PCA"}))
    return -1;
  if (name == "N") return in(res, {"PRO", "PCA"}) ? -1 : 7;
  if (name == "CA") return res == "GLY" ? 1 : 0;
  const std::string& r = res;
  const std::string& a = name;
  if (r == "ALA" && a == "CB") return 2;
  if (r == "ARG" && in(a, {"CB", "CG", "CD"})) return 1;
  if (r == "ARG" && a == "NE") return 11;
  if (r == "ARG" && in(a, {"NH1", "NH2"})) return 12;
  if ((r == "ASN" && a == "CB") || (in(r, {"ASP", "ASH"}) && a == "CB") || (in(r, {"CYS", "CYX"}) && a == "CB")) return 1;
  if (r == "ASN" && a == "ND2") return 8;
  if (in(r, {"ASP", "GLU"}) && in(a, {"OD1", "OD2", "OE1", "OE2"})) return 6;
  if ((r == "ASH" && a == "OD2") || (r == "GLH" && a == "OE2")) return 5;
  if (r == "CYS" && a == "SG") return 13;
  if ((r == "GLN" && in(a, {"CB", "CG"})) || (in(r, {"GLU", "GLH"}) && in(a, {"CB", "CG"}))) return 1;
  if (r == "GLN" && a == "NE2") return 8;
  if (in(r, {"HIS", "HID", "HIE", "HIP"}) && a == "CB") return 1;
  if ((in(r, {"HIS", "HID"}) && a == "ND1") || (r == "HIE" && a == "NE2")) return 7;
  if (r == "HIP" && in(a, {"ND1", "NE2"})) return 9;
  if (in(r, {"HIS", "HID", "HIE", "HIP"}) && in(a, {"CD2", "CE1"})) return 3;
  if ((r == "ILE" && a == "CB") || (r == "LEU" && a == "CG") || (r == "THR" && a == "CB") || (r == "VAL" && a == "CB")) return 0;
  if ((r == "ILE" && a == "CG1") || (r == "LEU" && a == "CB")) return 1;
  if ((r == "ILE" && in(a, {"CG2", "CD1"})) || (r == "LEU" && in(a, {"CD1", "CD2"}))) return 2;
  if (r == "LYS" && in(a, {"CB", "CG", "CD", "CE"})) return 1;
  if (r == "LYS" && a == "NZ") return 10;
  if (in(r, {"MET", "MSE"}) && in(a, {"CB", "CG"})) return 1;
  if (in(r, {"MET", "MSE"}) && a == "CE") return 2;
  if ((in(r, {"PHE", "TYR"}) && a == "CB") || (r == "TRP" && a == "CB")) return 1;
  if ((r == "PHE" && in(a, {"CD1", "CD2", "CE1", "CE2", "CZ"})) || (r == "TYR" && in(a, {"CD1", "CD2", "CE1", "CE2"})) ||
      (r == "TRP" && in(a, {"CD1", "CE3", "CZ2", "CZ3", "CH2"})))
    return 3;
  if (r == "PRO" && in(a, {"CB", "CG", "CD"})) return 1;
  if (r == "SER" && a == "CB") return 1;
  if ((r == "SER" && a == "OG") || (r == "THR" && a == "OG1") || (r == "TYR" && a == "OH")) return 4;
  if ((r == "THR" && a == "CG2") || (r == "VAL" && in(a, {"CG1", "CG2"}))) return 2;
  if (r == "TRP" && a == "NE1") return 7;
  if (r == "PCA" && in(a, {"CB", "CG"})) return 1;
  return -1;
}

// scattering.rs:86-110 — vacuum Debye.  OpenMP over q mirrors the rayon
// par_iter over q; each q is summed sequentially as in the reference.
ORC_API int orc_debye_intensity(int64_t n, const double* xyz, const int* elem, const int* group, const double* occ,
                                int implicit_h, int64_t nq, const double* q, double* out) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t k = 0; k < nq; ++k) {
    std::vector<double> f(n);
    for (int64_t i = 0; i < n; ++i) f[i] = form_factor(elem[i], group[i], occ[i], implicit_h != 0, q[k]);
    double intensity = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      intensity += f[i] * f[i];
      for (int64_t j = i + 1; j < n; ++j) intensity += 2.0 * f[i] * f[j] * sinc(q[k] * dist(xyz + 3 * i, xyz + 3 * j));
    }
    out[k] = std::fmax(intensity, 0.0);
  }
  return 0;
}

// Per-atom-type pair partials, the decomposition the GPU kernel computes:
//   out[ab*nq + k] = sum_{i<j, {t_i,t_j}={a,b}} occ_i occ_j sinc(q_k r_ij), a<=b,
//   ab = a*T - a*(a-1)/2 + (b-a);  self[a] = sum_{t_i=a} occ_i^2.
// It is the pair loop of scattering.rs:99-106 / solvent.rs:533-558 grouped by
// type pair, in f64 with the reference sinc.
ORC_API int orc_debye_partials(int64_t n, const double* xyz, const double* occ, const int* type, int T, int64_t nq,
                               const double* q, double* out, double* self) {
  int P = T * (T + 1) / 2;
  for (int a = 0; a < T; ++a) self[a] = 0.0;
  for (int64_t i = 0; i < n; ++i) self[type[i]] += occ[i] * occ[i];
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t k = 0; k < nq; ++k) {
    std::vector<double> acc(P, 0.0);
    for (int64_t i = 0; i < n; ++i)
      for (int64_t j = i + 1; j < n; ++j) {
        int a = std::min(type[i], type[j]), b = std::max(type[i], type[j]);
        int ab = a * T - a * (a - 1) / 2 + (b - a);
        acc[ab] += occ[i] * occ[j] * sinc(q[k] * dist(xyz + 3 * i, xyz + 3 * j));
      }
    for (int p = 0; p < P; ++p) out[(size_t)p * nq + k] = acc[p];
  }
  return 0;
}

// Adaptive hydration grid (solvent.rs:121-223).  Two-call size query:
// pass sites=NULL to get *m; returns 1 on invalid input.
ORC_API int orc_adaptive_grid(int64_t n, const double* xyz, double spacing, double clearance, double padding,
                              double* sites, int64_t capacity, int64_t* m, double* volume) {
  std::vector<double> s;
  int rc = adaptive_grid(n, xyz, spacing, clearance, padding, s, volume);
  if (rc) return rc;
  *m = (int64_t)(s.size() / 3);
  if (sites) {
    if (capacity < *m) return 3;
    std::memcpy(sites, s.data(), s.size() * sizeof(double));
  }
  return 0;
}

// Exterior flood-fill hydration grid (solvent.rs:259-401).
ORC_API int orc_exterior_grid(int64_t n, const double* xyz, const int* elem, double spacing, double probe,
                              double thickness, double* sites, int64_t capacity, int64_t* m, double* volume) {
  std::vector<double> s;
  int rc = exterior_grid(n, xyz, elem, spacing, probe, thickness, s, volume);
  if (rc) return rc;
  *m = (int64_t)(s.size() / 3);
  if (sites) {
    if (capacity < *m) return 3;
    std::memcpy(sites, s.data(), s.size() * sizeof(double));
  }
  return 0;
}

// solvent.rs:504-584 — six Debye self/cross terms vv, ee, hh, ve, vh, eh
// (out6 is [6][nq]).  model: 0 Analytic, 1 Grid, 2 AdaptiveGrid.
ORC_API int orc_debye_solvent_basis(int64_t n, const double* xyz, const int* elem, const int* group, const double* occ,
                                    int implicit_h, int64_t nq, const double* q, double c1, double c2,
                                    double thickness, double density, int model, double spacing, double* out6) {
  SolventP p{c1, c2, thickness, density, model, spacing};
  std::vector<double> sites;
  double voxel_volume = 0.0;
  int rc = build_grid(n, xyz, elem, p, sites, &voxel_volume);
  if (rc) return rc;
  bool grid = model != 0;
  int64_t ns = (int64_t)sites.size() / 3;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t k = 0; k < nq; ++k) {
    double qq = q[k];
    std::vector<double> v(n), e(n), h(n);
    for (int64_t i = 0; i < n; ++i) component_amplitudes(elem[i], group[i], occ[i], implicit_h != 0, qq, p, &v[i], &e[i], &h[i]);
    double t[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t i = 0; i < n; ++i) {
      t[0] += v[i] * v[i];
      t[1] += e[i] * e[i];
      t[3] += v[i] * e[i];
      if (!grid) { t[2] += h[i] * h[i]; t[4] += v[i] * h[i]; t[5] += e[i] * h[i]; }
      for (int64_t j = i + 1; j < n; ++j) {
        double s = sinc(qq * dist(xyz + 3 * i, xyz + 3 * j));
        t[0] += 2.0 * v[i] * v[j] * s;
        t[1] += 2.0 * e[i] * e[j] * s;
        t[3] += (v[i] * e[j] + v[j] * e[i]) * s;
        if (!grid) {
          t[2] += 2.0 * h[i] * h[j] * s;
          t[4] += (v[i] * h[j] + v[j] * h[i]) * s;
          t[5] += (e[i] * h[j] + e[j] * h[i]) * s;
        }
      }
    }
    if (grid) {
      double amp = p.density / 10.0 * voxel_volume * water_form_factor(qq);
      for (int64_t i = 0; i < ns; ++i) {
        t[2] += amp * amp;
        for (int64_t o = i + 1; o < ns; ++o) t[2] += 2.0 * amp * amp * sinc(qq * dist(&sites[3 * i], &sites[3 * o]));
        for (int64_t a = 0; a < n; ++a) {
          double s = sinc(qq * dist(xyz + 3 * a, &sites[3 * i]));
          t[4] += v[a] * amp * s;
          t[5] += e[a] * amp * s;
        }
      }
    }
    for (int c = 0; c < 6; ++c) out6[(size_t)c * nq + k] = t[c];
  }
  return 0;
}

// spherical.rs:567-584
ORC_API void orc_combine_solvent_basis(int64_t nq, const double* q, const double* basis6, double c1, double c2,
                                       double* out) {
  for (int64_t i = 0; i < nq; ++i) {
    double es = excluded_volume_scale(q[i], c1);
    const double* b = basis6;
    double v = b[i] + es * es * b[nq + i] + c2 * c2 * b[2 * nq + i] - 2.0 * es * b[3 * nq + i] + 2.0 * c2 * b[4 * nq + i] -
               2.0 * es * c2 * b[5 * nq + i];
    out[i] = std::fmax(v, 0.0);
  }
}

// spherical.rs:95-133 and 54-93, exposed for unit tests.
ORC_API void orc_spherical_bessel(int l_max, double x, double* out) {
  std::vector<double> work(l_max + 26);
  spherical_bessel_all_into(l_max, x, out, work.data());
}
ORC_API void orc_real_harmonics(int l_max, double x, double phi, double* out) {
  std::vector<double> norms = harmonic_norms(l_max);
  real_harmonics_all(l_max, x, phi, norms.data(), out);
}

// spherical.rs:266-312 (the cached-harmonics path; the streaming variant at
// 314-403 computes the same sums in a rayon-dependent order).
ORC_API int orc_multipole_intensity(int64_t n, const double* xyz, const int* elem, const int* group, const double* occ,
                                    int implicit_h, int64_t nq, const double* q, int l_max, double* out) {
  if (n == 0) { for (int64_t k = 0; k < nq; ++k) out[k] = 0.0; return 0; }
  double c[3];
  centroid(n, xyz, c);
  Geometry g = geometry_for_points(n, xyz, c, l_max);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t k = 0; k < nq; ++k) {
    int ql = adaptive_l_max(q[k], g.max_radius, l_max);
    std::vector<double> coeff(g.coeff_count, 0.0), js(ql + 1), work(ql + 26);
    for (int64_t i = 0; i < n; ++i) {
      double f = form_factor(elem[i], group[i], occ[i], implicit_h != 0, q[k]);
      spherical_bessel_all_into(ql, q[k] * g.radii[i], js.data(), work.data());
      const double* Y = g.harmonics.data() + (size_t)i * g.coeff_count;
      for (int l = 0; l <= ql; ++l)
        for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) coeff[kk] += f * js[l] * Y[kk];
    }
    double s = 0.0;
    for (double v : coeff) s += v * v;
    out[k] = std::fmax(4.0 * PI * s, 0.0);
  }
  return 0;
}

// spherical.rs:474-565 — multipole six-term basis (out6 is [6][nq]).
ORC_API int orc_multipole_solvent_basis(int64_t n, const double* xyz, const int* elem, const int* group,
                                        const double* occ, int implicit_h, int64_t nq, const double* q, int l_max,
                                        double c1, double c2, double thickness, double density, int model,
                                        double spacing, double* out6) {
  if (n == 0) { for (int64_t k = 0; k < 6 * nq; ++k) out6[k] = 0.0; return 0; }
  SolventP p{c1, c2, thickness, density, model, spacing};
  double c[3];
  centroid(n, xyz, c);
  Geometry g = geometry_for_points(n, xyz, c, l_max);
  std::vector<double> sites;
  double voxel_volume = 0.0;
  int rc = build_grid(n, xyz, elem, p, sites, &voxel_volume);
  if (rc) return rc;
  bool grid = model != 0;
  Geometry gg;
  if (grid) gg = geometry_for_points((int64_t)sites.size() / 3, sites.data(), c, l_max);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t k = 0; k < nq; ++k) {
    double qq = q[k];
    int ql = adaptive_l_max(qq, g.max_radius, l_max);
    if (grid) ql = std::max(ql, adaptive_l_max(qq, gg.max_radius, l_max));
    std::vector<double> c0(g.coeff_count, 0.0), c1v(g.coeff_count, 0.0), c2v(g.coeff_count, 0.0), js(ql + 1), work(ql + 26);
    for (int64_t i = 0; i < n; ++i) {
      double amp[3];
      solvent_components_for_atom(elem[i], group[i], occ[i], implicit_h != 0, qq, p, amp);
      spherical_bessel_all_into(ql, qq * g.radii[i], js.data(), work.data());
      const double* Y = g.harmonics.data() + (size_t)i * g.coeff_count;
      for (int l = 0; l <= ql; ++l)
        for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) {
          double cc = js[l] * Y[kk];
          c0[kk] += amp[0] * cc;
          c1v[kk] += amp[1] * cc;
          if (!grid) c2v[kk] += amp[2] * cc;
        }
    }
    if (grid) {
      double amp = p.density / 10.0 * voxel_volume * water_form_factor(qq);
      for (size_t i = 0; i < gg.radii.size(); ++i) {
        spherical_bessel_all_into(ql, qq * gg.radii[i], js.data(), work.data());
        const double* Y = gg.harmonics.data() + i * gg.coeff_count;
        for (int l = 0; l <= ql; ++l)
          for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) c2v[kk] += amp * js[l] * Y[kk];
      }
    }
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int kk = 0; kk < g.coeff_count; ++kk) s[0] += c0[kk] * c0[kk];
    for (int kk = 0; kk < g.coeff_count; ++kk) s[1] += c1v[kk] * c1v[kk];
    for (int kk = 0; kk < g.coeff_count; ++kk) s[2] += c2v[kk] * c2v[kk];
    for (int kk = 0; kk < g.coeff_count; ++kk) s[3] += c0[kk] * c1v[kk];
    for (int kk = 0; kk < g.coeff_count; ++kk) s[4] += c0[kk] * c2v[kk];
    for (int kk = 0; kk < g.coeff_count; ++kk) s[5] += c1v[kk] * c2v[kk];
    for (int t = 0; t < 6; ++t) out6[(size_t)t * nq + k] = 4.0 * PI * s[t];
  }
  return 0;
}

// spherical.rs:408-470
ORC_API int orc_multipole_solvent_intensity(int64_t n, const double* xyz, const int* elem, const int* group,
                                            const double* occ, int implicit_h, int64_t nq, const double* q, int l_max,
                                            double c1, double c2, double thickness, double density, int model,
                                            double spacing, double* out) {
  if (n == 0) { for (int64_t k = 0; k < nq; ++k) out[k] = 0.0; return 0; }
  SolventP p{c1, c2, thickness, density, model, spacing};
  double c[3];
  centroid(n, xyz, c);
  Geometry g = geometry_for_points(n, xyz, c, l_max);
  std::vector<double> sites;
  double voxel_volume = 0.0;
  int rc = build_grid(n, xyz, elem, p, sites, &voxel_volume);
  if (rc) return rc;
  bool grid = model != 0;
  Geometry gg;
  if (grid) gg = geometry_for_points((int64_t)sites.size() / 3, sites.data(), c, l_max);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t k = 0; k < nq; ++k) {
    double qq = q[k];
    int ql = adaptive_l_max(qq, g.max_radius, l_max);
    if (grid) ql = std::max(ql, adaptive_l_max(qq, gg.max_radius, l_max));
    std::vector<double> coeff(g.coeff_count, 0.0), js(ql + 1), work(ql + 26);
    for (int64_t i = 0; i < n; ++i) {
      double amp[3];
      solvent_components_for_atom(elem[i], group[i], occ[i], implicit_h != 0, qq, p, amp);
      double f = amp[0] - excluded_volume_scale(qq, c1) * amp[1] + (model == 0 ? c2 * amp[2] : 0.0);
      spherical_bessel_all_into(ql, qq * g.radii[i], js.data(), work.data());
      const double* Y = g.harmonics.data() + (size_t)i * g.coeff_count;
      for (int l = 0; l <= ql; ++l)
        for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) coeff[kk] += f * js[l] * Y[kk];
    }
    if (grid) {
      double amp = p.density / 10.0 * voxel_volume * water_form_factor(qq);
      for (size_t i = 0; i < gg.radii.size(); ++i) {
        spherical_bessel_all_into(ql, qq * gg.radii[i], js.data(), work.data());
        const double* Y = gg.harmonics.data() + i * gg.coeff_count;
        for (int l = 0; l <= ql; ++l)
          for (int kk = l * l; kk < (l + 1) * (l + 1); ++kk) coeff[kk] += c2 * amp * js[l] * Y[kk];
      }
    }
    double s = 0.0;
    for (double v : coeff) s += v * v;
    out[k] = std::fmax(4.0 * PI * s, 0.0);
  }
  return 0;
}

// ---------------------------------------------------------------- fitting

// fit.rs:137-198 (bg_mode: 0 Fit, 1 FixedZero, 2 Fixed(bg_value)).
ORC_API void orc_solve_linear(int64_t nq, const double* theory, const double* y, const double* sigma, int bg_mode,
                              double bg_value, double* scale_out, double* bg_out, double* chi_out) {
  double sw = 0, sx = 0, sy = 0, sxx = 0, sxy = 0;
  for (int64_t i = 0; i < nq; ++i) {
    double x = theory[i], w = 1.0 / (sigma[i] * sigma[i]);
    sw += w; sx += w * x; sy += w * y[i]; sxx += w * x * x; sxy += w * x * y[i];
  }
  double scale, bg;
  if (bg_mode == 0) {
    double det = sxx * sw - sx * sx;
    scale = std::fmax(std::fabs(det) > 1e-20 ? (sxy * sw - sx * sy) / det : 0.0, 0.0);
    bg = sw > 0.0 ? (sy - scale * sx) / sw : 0.0;
  } else if (bg_mode == 1) {
    scale = std::fmax(sxx > 0.0 ? sxy / sxx : 0.0, 0.0);
    bg = 0.0;
  } else {
    scale = std::fmax(sxx > 0.0 ? (sxy - bg_value * sx) / sxx : 0.0, 0.0);
    bg = bg_value;
  }
  double dof = (double)std::max<int64_t>(nq - 1, 1);
  double chi = 0.0;
  for (int64_t i = 0; i < nq; ++i) { double r = (scale * theory[i] + bg - y[i]) / sigma[i]; chi += r * r; }
  *scale_out = scale; *bg_out = bg; *chi_out = chi / dof;
}

// fit.rs:200-244 (scale_mode: 0 Fit, 1 Fixed(scale_value)).
ORC_API void orc_solve_scale_background(int64_t nq, const double* theory, const double* y, const double* sigma,
                                        int scale_mode, double scale_value, int bg_mode, double bg_value,
                                        double* scale_out, double* bg_out, double* chi_out) {
  if (scale_mode == 0) { orc_solve_linear(nq, theory, y, sigma, bg_mode, bg_value, scale_out, bg_out, chi_out); return; }
  double scale = std::fmax(scale_value, 0.0), bg;
  if (bg_mode == 0) {
    double weighted = 0, weight = 0;
    for (int64_t i = 0; i < nq; ++i) { double w = 1.0 / (sigma[i] * sigma[i]); weighted += w * (y[i] - scale * theory[i]); weight += w; }
    bg = weight > 0.0 ? weighted / weight : 0.0;
  } else if (bg_mode == 1) bg = 0.0;
  else bg = bg_value;
  double dof = (double)std::max<int64_t>(nq - 1, 1);
  double chi = 0.0;
  for (int64_t i = 0; i < nq; ++i) { double r = (scale * theory[i] + bg - y[i]) / sigma[i]; chi += r * r; }
  *scale_out = scale; *bg_out = bg; *chi_out = chi / dof;
}

// fit.rs:93-123
ORC_API void orc_cubic_hermite(int64_t n, const double* x, const double* y, int64_t nt, const double* t, double* out) {
  if (n == 1) { for (int64_t i = 0; i < nt; ++i) out[i] = y[0]; return; }
  std::vector<double> sl(n);
  int64_t last = n - 1;
  sl[0] = (y[1] - y[0]) / (x[1] - x[0]);
  sl[last] = (y[last] - y[last - 1]) / (x[last] - x[last - 1]);
  for (int64_t i = 1; i < last; ++i) sl[i] = (y[i + 1] - y[i - 1]) / (x[i + 1] - x[i - 1]);
  int64_t seg = 0;
  for (int64_t k = 0; k < nt; ++k) {
    while (seg + 1 < last && t[k] > x[seg + 1]) ++seg;
    double h = x[seg + 1] - x[seg];
    double u = std::fmin(std::fmax((t[k] - x[seg]) / h, 0.0), 1.0);
    double u2 = u * u, u3 = u2 * u;
    out[k] = (2.0 * u3 - 3.0 * u2 + 1.0) * y[seg] + (u3 - 2.0 * u2 + u) * h * sl[seg] + (-2.0 * u3 + 3.0 * u2) * y[seg + 1] +
             (u3 - u2) * h * sl[seg + 1];
  }
}

// ---------------------------------------------------------------- ensemble

// ensemble.rs:449-465
ORC_API void orc_project_simplex(int64_t n, const double* values, double* out) {
  std::vector<double> sorted(values, values + n);
  std::sort(sorted.begin(), sorted.end(), [](double a, double b) { return a > b; });
  double cumulative = 0.0;
  int64_t rho = 0;
  for (int64_t i = 0; i < n; ++i) {
    cumulative += sorted[i];
    if (sorted[i] + (1.0 - cumulative) / (double)(i + 1) > 0.0) rho = i + 1;
  }
  double top = 0.0;
  for (int64_t i = 0; i < rho; ++i) top += sorted[i];
  double theta = (top - 1.0) / (double)std::max<int64_t>(rho, 1);
  for (int64_t i = 0; i < n; ++i) out[i] = std::fmax(values[i] - theta, 0.0);
}

namespace {
void mix_curves(int64_t K, int64_t nq, const double* curves, const double* w, double* out) {
  for (int64_t p = 0; p < nq; ++p) {
    double s = 0.0;
    for (int64_t k = 0; k < K; ++k) s += curves[k * nq + p] * w[k];
    out[p] = s;
  }
}
// ensemble.rs:383-434
void solve_linear_fixed(int64_t nq, const double* th, const double* y, const double* sg, int scale_mode,
                        double scale_value, int bg_mode, double bg_value, double* so, double* bo, double* co) {
  double scale;
  if (scale_mode == 0) {
    double num = 0, den = 0;
    for (int64_t i = 0; i < nq; ++i) { num += th[i] * y[i] / (sg[i] * sg[i]); den += th[i] * th[i] / (sg[i] * sg[i]); }
    scale = den > 0.0 ? num / den : 0.0;
  } else scale = scale_value;
  scale = std::fmax(scale, 0.0);
  double bg;
  if (bg_mode == 0) {
    double num = 0, den = 0;
    for (int64_t i = 0; i < nq; ++i) { num += (y[i] - scale * th[i]) / (sg[i] * sg[i]); den += 1.0 / (sg[i] * sg[i]); }
    bg = den > 0.0 ? num / den : 0.0;
  } else if (bg_mode == 1) bg = 0.0;
  else bg = bg_value;
  double chi = 0.0;
  for (int64_t i = 0; i < nq; ++i) { double r = (scale * th[i] + bg - y[i]) / sg[i]; chi += r * r; }
  *so = scale; *bo = bg; *co = chi / (double)std::max<int64_t>(nq - 1, 1);
}
}  // namespace

// ensemble.rs:317-381 — projected-gradient simplex weights for one (c1,c2)
// candidate.  curves is [K][nq].
ORC_API void orc_optimize_weights(int64_t K, int64_t nq, const double* curves, const double* y, const double* sigma,
                                  int scale_mode, double scale_value, int bg_mode, double bg_value, int uniform,
                                  double regularization, double* weights, double* scale_out, double* bg_out,
                                  double* chi2_out, double* fitted) {
  std::vector<double> w(K, 1.0 / (double)K), mix(nq), res(nq), grad(K), prop(K), step(K);
  if (!uniform) {
    for (int it = 0; it < 250; ++it) {
      mix_curves(K, nq, curves, w.data(), mix.data());
      double s, b, c;
      solve_linear_fixed(nq, mix.data(), y, sigma, scale_mode, scale_value, bg_mode, bg_value, &s, &b, &c);
      for (int64_t i = 0; i < nq; ++i) res[i] = (s * mix[i] + b - y[i]) / sigma[i];
      for (int64_t k = 0; k < K; ++k) {
        double acc = 0.0;
        for (int64_t i = 0; i < nq; ++i) acc += res[i] * s * curves[k * nq + i] / sigma[i];
        grad[k] = 2.0 * acc + 2.0 * regularization * (w[k] - 1.0 / (double)K);
      }
      double nrm = 0.0;
      for (int64_t k = 0; k < K; ++k) nrm += grad[k] * grad[k];
      nrm = std::fmax(std::sqrt(nrm), 1.0);
      for (int64_t k = 0; k < K; ++k) step[k] = w[k] - 0.05 * grad[k] / nrm;
      orc_project_simplex(K, step.data(), prop.data());
      double delta = 0.0;
      for (int64_t k = 0; k < K; ++k) delta += std::fabs(prop[k] - w[k]);
      w = prop;
      if (delta < 1e-8) break;
    }
  }
  mix_curves(K, nq, curves, w.data(), mix.data());
  double s, b, c;
  solve_linear_fixed(nq, mix.data(), y, sigma, scale_mode, scale_value, bg_mode, bg_value, &s, &b, &c);
  for (int64_t i = 0; i < nq; ++i) fitted[i] = s * mix[i] + b;
  for (int64_t k = 0; k < K; ++k) weights[k] = w[k];
  *scale_out = s; *bg_out = b; *chi2_out = c;
}

// ensemble.rs:302-315
ORC_API void orc_solvent_candidates(double c1_lo, double c1_hi, double c2_lo, double c2_hi, double* out50) {
  int idx = 0;
  for (int i = 0; i < 5; ++i) {
    double c1 = c1_lo + (c1_hi - c1_lo) * (double)i / 4.0;
    for (int j = 0; j < 5; ++j) {
      double c2 = c2_lo + (c2_hi - c2_lo) * (double)j / 4.0;
      out50[idx++] = c1;
      out50[idx++] = c2;
    }
  }
}

// ---------------------------------------------------------------- reweight

namespace {
// reweight.rs:236-301
void rw_solve(int64_t nq, const double* th, const double* y, const double* sg, int scale_mode, double scale_value,
              int bg_mode, double bg_value, double* so, double* bo, double* chi_red) {
  double sw = 0, sx = 0, sy = 0, sxx = 0, sxy = 0;
  for (int64_t i = 0; i < nq; ++i) {
    double w = 1.0 / (sg[i] * sg[i]);
    sw += w; sx += w * th[i]; sy += w * y[i]; sxx += w * th[i] * th[i]; sxy += w * th[i] * y[i];
  }
  auto fitted_scale = [&](double b) { return sxx > 0.0 ? std::fmax((sxy - b * sx) / sxx, 0.0) : 0.0; };
  auto fitted_bg = [&](double s) { return sw > 0.0 ? (sy - s * sx) / sw : 0.0; };
  double s, b;
  if (scale_mode == 1 && bg_mode == 2) { s = std::fmax(scale_value, 0.0); b = bg_value; }
  else if (scale_mode == 1 && bg_mode == 1) { s = std::fmax(scale_value, 0.0); b = 0.0; }
  else if (scale_mode == 1 && bg_mode == 0) { s = std::fmax(scale_value, 0.0); b = fitted_bg(s); }
  else if (scale_mode == 0 && bg_mode == 2) { s = fitted_scale(bg_value); b = bg_value; }
  else if (scale_mode == 0 && bg_mode == 1) { s = fitted_scale(0.0); b = 0.0; }
  else {
    double det = sxx * sw - sx * sx;
    s = std::fabs(det) > 1e-20 ? std::fmax((sxy * sw - sx * sy) / det, 0.0) : 0.0;
    b = fitted_bg(s);
  }
  double chi = 0.0;
  for (int64_t i = 0; i < nq; ++i) { double r = (s * th[i] + b - y[i]) / sg[i]; chi += r * r; }
  *so = s; *bo = b; *chi_red = chi / (double)std::max<int64_t>(nq - 1, 1);
}
double kl_div(const std::vector<double>& w, const std::vector<double>& p) {
  double s = 0.0;
  for (size_t i = 0; i < w.size(); ++i) s += w[i] * std::log(w[i] / p[i]);
  return s;
}
std::vector<double> apply_floor(std::vector<double> w, double floor) {
  double sum = 0.0;
  for (double v : w) sum += v;
  sum = std::fmax(sum, 1e-300);
  if (floor <= 0.0) { for (double& v : w) v /= sum; return w; }
  double residual = 1.0 - floor * (double)w.size();
  for (double& v : w) v = floor + residual * v / sum;
  return w;
}
}  // namespace

// reweight.rs:84-154 — maximum-entropy mirror descent.  prior may be NULL
// (uniform).  Returns 0 on success, 1 on invalid options.
ORC_API int orc_reweight_curves(int64_t K, int64_t nq, const double* curves, const double* y, const double* sigma,
                                double kl_strength, int max_iterations, double step_size, double tolerance,
                                double min_weight, const double* prior_in, int scale_mode, double scale_value,
                                int bg_mode, double bg_value, double* weights_out, double* scale_out, double* bg_out,
                                double* reduced_chi2_out, double* kl_out, int* iterations_out, int* converged_out) {
  if (K == 0 || !std::isfinite(kl_strength) || kl_strength < 0.0 || max_iterations == 0 || !std::isfinite(step_size) ||
      step_size <= 0.0 || !std::isfinite(tolerance) || tolerance <= 0.0 || !std::isfinite(min_weight) ||
      min_weight < 0.0 || min_weight * (double)K >= 1.0)
    return 1;
  std::vector<double> prior(K, 1.0);
  if (prior_in) for (int64_t k = 0; k < K; ++k) prior[k] = prior_in[k];
  double psum = 0.0;
  for (double v : prior) psum += v;
  for (double& v : prior) v /= psum;
  std::vector<double> w = apply_floor(prior, min_weight), mix(nq), grad(K);
  int iterations = 0, converged = 0;
  double dof = (double)std::max<int64_t>(nq - 1, 1);
  for (int it = 0; it < max_iterations; ++it) {
    iterations = it + 1;
    mix_curves(K, nq, curves, w.data(), mix.data());
    double s, b, chi;
    rw_solve(nq, mix.data(), y, sigma, scale_mode, scale_value, bg_mode, bg_value, &s, &b, &chi);
    for (int64_t k = 0; k < K; ++k) {
      double dg = 0.0;
      for (int64_t i = 0; i < nq; ++i) {
        double fitted = s * mix[i] + b;
        dg += 2.0 * (fitted - y[i]) * s * curves[k * nq + i] / (sigma[i] * sigma[i]) / dof;
      }
      grad[k] = dg + kl_strength * (std::log(w[k] / prior[k]) + 1.0);
    }
    double gmax = 0.0;
    for (double g : grad) gmax = std::fmax(gmax, std::fabs(g));
    gmax = std::fmax(gmax, 1e-12);
    double step = step_size / gmax;
    double objective = chi + kl_strength * kl_div(w, prior);
    bool accepted = false;
    std::vector<double> prop;
    for (int h = 0; h < 14; ++h) {
      std::vector<double> lw(K);
      double mx = -INFINITY;
      for (int64_t k = 0; k < K; ++k) { lw[k] = std::log(std::fmax(w[k], 1e-300)) - step * grad[k]; mx = std::fmax(mx, lw[k]); }
      std::vector<double> pr(K);
      double sum = 0.0;
      for (int64_t k = 0; k < K; ++k) { pr[k] = std::exp(lw[k] - mx); }
      for (int64_t k = 0; k < K; ++k) sum += pr[k];
      sum = std::fmax(sum, 1e-300);
      for (double& v : pr) v /= sum;
      pr = apply_floor(pr, min_weight);
      mix_curves(K, nq, curves, pr.data(), mix.data());
      double s2, b2, chi2;
      rw_solve(nq, mix.data(), y, sigma, scale_mode, scale_value, bg_mode, bg_value, &s2, &b2, &chi2);
      if (chi2 + kl_strength * kl_div(pr, prior) <= objective + 1e-12) { prop = pr; accepted = true; break; }
      step *= 0.5;
    }
    if (!accepted) break;
    double delta = 0.0;
    for (int64_t k = 0; k < K; ++k) delta += std::fabs(prop[k] - w[k]);
    w = prop;
    if (delta <= tolerance) { converged = 1; break; }
  }
  mix_curves(K, nq, curves, w.data(), mix.data());
  double s, b, chi;
  rw_solve(nq, mix.data(), y, sigma, scale_mode, scale_value, bg_mode, bg_value, &s, &b, &chi);
  for (int64_t k = 0; k < K; ++k) weights_out[k] = w[k];
  *scale_out = s; *bg_out = b; *reduced_chi2_out = chi; *kl_out = kl_div(w, prior);
  *iterations_out = iterations; *converged_out = converged;
  return 0;
}

// ---------------------------------------------------------------- chi2 + gradient (no reference counterpart)

// Reduced chi^2 of the solvent-corrected Debye model (analytic hydration):
//   model(q) = scale * I(q; x, c1, c2) + background,
//   I(q) = sum_ij A_i A_j sinc(q r_ij),  A_i = v_i - G(q,c1) e_i + c2 h_i
// with v, e, h from solvent.rs:454-488 and G from solvent.rs:448-452, and
//   chi2 = sum_k ((model_k - y_k)/sigma_k)^2 / max(nq-1, 1)   (fit.rs:185-196).
// grad_xyz (3n) and grad_p (c1, c2, scale, background) may be NULL.  The
// coordinate gradient is the analytic pair-sum adjoint in f64; the c1/c2
// derivatives are taken through the six-term basis.
ORC_API int orc_chi2_grad(int64_t n, const double* xyz, const int* elem, const int* group, const double* occ,
                          int implicit_h, int64_t nq, const double* q, const double* y, const double* sigma,
                          double c1, double c2, double thickness, double density, double scale, double background,
                          double* chi2_out, double* grad_xyz, double* grad_p) {
  SolventP p{c1, c2, thickness, density, 0, 4.0};
  std::vector<double> basis(6 * nq), inten(nq);
  orc_debye_solvent_basis(n, xyz, elem, group, occ, implicit_h, nq, q, c1, c2, thickness, density, 0, 4.0, basis.data());
  double dof = (double)std::max<int64_t>(nq - 1, 1);
  std::vector<double> wq(nq);
  double chi = 0.0, dc1 = 0.0, dc2 = 0.0, ds = 0.0, db = 0.0;
  for (int64_t k = 0; k < nq; ++k) {
    double G = excluded_volume_scale(q[k], c1);
    const double* b = basis.data();
    double I = b[k] + G * G * b[nq + k] + c2 * c2 * b[2 * nq + k] - 2.0 * G * b[3 * nq + k] + 2.0 * c2 * b[4 * nq + k] -
               2.0 * G * c2 * b[5 * nq + k];
    double r = (scale * I + background - y[k]) / sigma[k];
    chi += r * r;
    double dchi_dmodel = 2.0 * r / sigma[k] / dof;
    wq[k] = dchi_dmodel * scale;  // d chi2 / d I(q_k)
    // dG/dc1 = G * (3/c1 - 2 c1 * 1.62^2 q^2 / 4)
    double dG = G * (3.0 / c1 - 2.0 * c1 * (1.62 * 1.62) * q[k] * q[k] / 4.0);
    double dI_dG = 2.0 * G * b[nq + k] - 2.0 * b[3 * nq + k] - 2.0 * c2 * b[5 * nq + k];
    double dI_dc2 = 2.0 * c2 * b[2 * nq + k] + 2.0 * b[4 * nq + k] - 2.0 * G * b[5 * nq + k];
    dc1 += wq[k] * dI_dG * dG;
    dc2 += wq[k] * dI_dc2;
    ds += dchi_dmodel * I;
    db += dchi_dmodel;
  }
  *chi2_out = chi / dof;
  if (grad_p) { grad_p[0] = dc1; grad_p[1] = dc2; grad_p[2] = ds; grad_p[3] = db; }
  if (grad_xyz) {
    std::vector<double> A((size_t)n * nq);
    for (int64_t k = 0; k < nq; ++k) {
      double G = excluded_volume_scale(q[k], c1);
      for (int64_t i = 0; i < n; ++i) {
        double v, e, h;
        component_amplitudes(elem[i], group[i], occ[i], implicit_h != 0, q[k], p, &v, &e, &h);
        A[(size_t)i * nq + k] = v - G * e + c2 * h;
      }
    }
    for (int64_t i = 0; i < 3 * n; ++i) grad_xyz[i] = 0.0;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n; ++i) {
      double g[3] = {0, 0, 0};
      for (int64_t j = 0; j < n; ++j) {
        if (j == i) continue;
        double dx = xyz[3 * i] - xyz[3 * j], dy = xyz[3 * i + 1] - xyz[3 * j + 1], dz = xyz[3 * i + 2] - xyz[3 * j + 2];
        double r = std::sqrt(norm2(dx, dy, dz));
        if (r < 1e-12) continue;
        double dr = 0.0;  // sum_q w_q * 2 A_i A_j * d sinc(q r)/dr
        for (int64_t k = 0; k < nq; ++k) {
          double x = q[k] * r;
          if (std::fabs(x) < 1e-8) continue;
          double dsinc = (x * std::cos(x) - std::sin(x)) / (x * x) * q[k];
          dr += wq[k] * 2.0 * A[(size_t)i * nq + k] * A[(size_t)j * nq + k] * dsinc;
        }
        g[0] += dr * dx / r; g[1] += dr * dy / r; g[2] += dr * dz / r;
      }
      grad_xyz[3 * i] = g[0]; grad_xyz[3 * i + 1] = g[1]; grad_xyz[3 * i + 2] = g[2];
    }
  }
  return 0;
}

// ---------------------------------------------------------------- coordinate P(r)
namespace {

// metrics.rs:535-541 squared_distance: dx*dx + dy*dy + dz*dz, left to right.
inline double squared_distance(const double* a, const double* b) {
  const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return dx * dx + dy * dy + dz * dz;
}

// `(distance / step).floor() as usize` clamped to bins-1 (metrics.rs:515-516);
// Rust's float-to-usize cast saturates and maps NaN to 0.
inline int64_t pr_bin_index(double distance, double step, int64_t bins) {
  const double v = std::floor(distance / step);
  if (!(v >= 0.0)) return 0;
  if (v >= (double)bins) return bins - 1;
  return std::min<int64_t>((int64_t)v, bins - 1);
}

}  // namespace

// metrics.rs:475-522 coordinate_pr up to the raw histogram: the maximum
// squared pair distance (f64::max fold, which skips NaN), step = dmax/bins,
// and per 64-row chunk a histogram of w_left*w_right over right > left,
// the chunks added in order.  Returns dmax; hist (bins values) is zero when
// every pair distance is zero (the reference returns early there).
ORC_API double orc_pair_distance_histogram(int64_t n, const double* xyz, const double* w, int64_t bins, double* hist) {
  double dmax2 = 0.0;
#pragma omp parallel for reduction(max : dmax2) schedule(dynamic, 64)
  for (int64_t l = 0; l < n; ++l) {
    double m = 0.0;
    for (int64_t r = l + 1; r < n; ++r) m = std::fmax(m, squared_distance(xyz + 3 * l, xyz + 3 * r));
    dmax2 = std::fmax(dmax2, m);
  }
  for (int64_t k = 0; k < bins; ++k) hist[k] = 0.0;
  if (dmax2 <= 0.0) return 0.0;
  const double dmax = std::sqrt(dmax2);
  const double step = dmax / (double)bins;
  const int64_t kChunk = 64;
  const int64_t n_chunks = (n + kChunk - 1) / kChunk;
  std::vector<double> part((size_t)n_chunks * bins, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t c = 0; c < n_chunks; ++c) {
    double* h = part.data() + (size_t)c * bins;
    const int64_t end = std::min(n, (c + 1) * kChunk);
    for (int64_t l = c * kChunk; l < end; ++l)
      for (int64_t r = l + 1; r < n; ++r) {
        const double d = std::sqrt(squared_distance(xyz + 3 * l, xyz + 3 * r));
        h[pr_bin_index(d, step, bins)] += w[l] * w[r];
      }
  }
  for (int64_t c = 0; c < n_chunks; ++c)
    for (int64_t k = 0; k < bins; ++k) hist[k] += part[(size_t)c * bins + k];
  return dmax;
}

// metrics.rs:550-583 normalize_distribution on (r, p) in place: trapezoid
// area to 1, rg = sqrt(max(moment/2, 0)) from the trapezoid of r^2 p, dmax =
// r at the last p above 1% of the maximum.  Returns 0 when the area is not
// finite and positive (the reference's None); rg / dmax are NaN for None.
ORC_API int orc_normalize_distribution(int64_t m, const double* r, double* p, double* rg, double* dmax) {
  if (m <= 0) return 0;
  double area = 0.0;
  for (int64_t i = 0; i + 1 < m; ++i) area += 0.5 * (r[i + 1] - r[i]) * (p[i] + p[i + 1]);
  if (!std::isfinite(area) || area <= 0.0) return 0;
  for (int64_t i = 0; i < m; ++i) p[i] /= area;
  double moment = 0.0;
  for (int64_t i = 0; i + 1 < m; ++i)
    moment += 0.5 * (r[i + 1] - r[i]) * (r[i] * r[i] * p[i] + r[i + 1] * r[i + 1] * p[i + 1]);
  const double g = std::sqrt(std::fmax(moment / 2.0, 0.0));
  *rg = std::isfinite(g) ? g : NAN;
  double maximum = 0.0;
  for (int64_t i = 0; i < m; ++i) maximum = std::fmax(maximum, p[i]);
  *dmax = NAN;
  for (int64_t i = m - 1; i >= 0; --i)
    if (p[i] > maximum * 0.01) { *dmax = r[i]; break; }
  return 1;
}

// metrics.rs:236-270 coordinate_features with metrics.rs:523-533: weights
// |form_factor_for_atom(atom, implicit = true, q = 0)| floored at 1e-6, the
// weighted centre and Rg, then coordinate_pr with max(bins, 16) bins.
// r_out / p_out hold max(bins, 16) values; *m_out is the length used (1 for
// the reference's single-point fallbacks).  Returns -1 for an empty structure.
ORC_API int orc_coordinate_features(int64_t n, const double* xyz, const int* elem, const int* group,
                                    const double* occ, int64_t bins, double* rg, double* dmax, double* r_out,
                                    double* p_out, int64_t* m_out, double* pr_rg, double* pr_dmax) {
  if (n <= 0) return -1;
  bins = std::max<int64_t>(bins, 16);
  std::vector<double> w(n);
  for (int64_t i = 0; i < n; ++i) w[i] = std::fmax(std::fabs(form_factor(elem[i], group[i], occ[i], true, 0.0)), 1e-6);
  double total = 0.0;
  for (int64_t i = 0; i < n; ++i) total += w[i];
  double c[3] = {0.0, 0.0, 0.0};
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) c[d] = c[d] + xyz[3 * i + d] * w[i];
  for (int d = 0; d < 3; ++d) c[d] = c[d] / total;
  double acc = 0.0;
  for (int64_t i = 0; i < n; ++i)
    acc += w[i] * norm2(xyz[3 * i] - c[0], xyz[3 * i + 1] - c[1], xyz[3 * i + 2] - c[2]);
  *rg = std::sqrt(acc / total);
  std::vector<double> hist(bins);
  const double dm = orc_pair_distance_histogram(n, xyz, w.data(), bins, hist.data());
  *dmax = dm;
  if (dm <= 0.0) {  // metrics.rs:489-498
    r_out[0] = 0.0; p_out[0] = 1.0; *m_out = 1; *pr_rg = 0.0; *pr_dmax = 0.0;
    return 0;
  }
  const double step = dm / (double)bins;
  for (int64_t k = 0; k < bins; ++k) { r_out[k] = ((double)k + 0.5) * step; p_out[k] = hist[k]; }
  *m_out = bins;
  if (!orc_normalize_distribution(bins, r_out, p_out, pr_rg, pr_dmax)) {  // metrics.rs:527-532
    r_out[0] = step * 0.5; p_out[0] = 1.0; *m_out = 1; *pr_rg = 0.0; *pr_dmax = dm;
  }
  return 0;
}
