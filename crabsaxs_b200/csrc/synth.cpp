// Seeded synthetic protein-like structures for benchmarks and tests (no
// counterpart in the crabSAXS reference, whose benches build a helix,
// benches/debye_bench.rs:7-29, and whose published numbers use PDB files that
// are fetched at run time).
//
// A Cα-style self-avoiding random walk with 3.8 Å steps, rejecting steps that
// come within 3.0 Å of an earlier Cα or leave a sphere of the given radius;
// every residue carries 4-8 side atoms at the Cα plus N(0, 1.5 Å) per axis.
// Elements are drawn C 63 %, N 17 %, O 19 %, S 1 %.  The generator uses
// splitmix64-seeded xoshiro256** and Box–Muller normals so the same seed gives
// the same structure on every platform.
//
// This file depends on nothing but the C ABI header, so the oracle library
// compiles the same source under another symbol name: a measurement of the
// reference's CPU path can build its input without loading this library.

#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "crab_cuda.h"

namespace {

struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t z = seed;
    for (int i = 0; i < 4; ++i) {
      z += 0x9E3779B97F4A7C15ull;
      uint64_t x = z;
      x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
      x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
      s[i] = x ^ (x >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0, 1)
  double normal() {
    double u1 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    const double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
  int element() {
    const double u = uniform();
    if (u < 0.63) return CRAB_EL_C;
    if (u < 0.80) return CRAB_EL_N;
    if (u < 0.99) return CRAB_EL_O;
    return CRAB_EL_S;
  }
};

struct CellHash {
  double cell;
  std::unordered_map<int64_t, std::vector<int32_t>> map;
  static int64_t key(int64_t x, int64_t y, int64_t z) {
    return ((x + 1048576) << 42) | ((y + 1048576) << 21) | (z + 1048576);
  }
  int64_t c(double v) const { return (int64_t)std::floor(v / cell); }
  void add(const double* p, int32_t id) { map[key(c(p[0]), c(p[1]), c(p[2]))].push_back(id); }
  double min_dist2(const double* p, const std::vector<double>& pts) const {
    double best = 1e300;
    const int64_t cx = c(p[0]), cy = c(p[1]), cz = c(p[2]);
    for (int64_t dx = -1; dx <= 1; ++dx)
      for (int64_t dy = -1; dy <= 1; ++dy)
        for (int64_t dz = -1; dz <= 1; ++dz) {
          auto it = map.find(key(cx + dx, cy + dy, cz + dz));
          if (it == map.end()) continue;
          for (int32_t id : it->second) {
            const double a = p[0] - pts[3 * id], b = p[1] - pts[3 * id + 1], e = p[2] - pts[3 * id + 2];
            best = std::fmin(best, a * a + b * b + e * e);
          }
        }
    return best;
  }
};

}  // namespace

extern "C" int crab_synth_protein(uint64_t seed, int64_t n_atoms, double radius, double* xyz, int8_t* element) {
  if (n_atoms < 0 || !(radius > 0.0) || (n_atoms > 0 && (!xyz || !element))) return CRAB_EINVAL;
  Rng rng(seed);
  CellHash hash{3.0, {}};
  std::vector<double> ca;
  double prev[3];
  {  // first Cα uniformly inside half the radius
    double p[3];
    do {
      for (double& v : p) v = (2.0 * rng.uniform() - 1.0) * 0.5 * radius;
    } while (p[0] * p[0] + p[1] * p[1] + p[2] * p[2] > 0.25 * radius * radius);
    for (int d = 0; d < 3; ++d) prev[d] = p[d];
  }
  int64_t n = 0;
  bool first = true;
  while (n < n_atoms) {
    double p[3];
    if (first) {
      for (int d = 0; d < 3; ++d) p[d] = prev[d];
      first = false;
    } else {
      double best[3] = {0, 0, 0}, best_d2 = -1.0;
      bool found = false;
      for (int attempt = 0; attempt < 64 && !found; ++attempt) {
        double u[3];
        double nrm;
        do {
          for (double& v : u) v = rng.normal();
          nrm = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        } while (nrm < 1e-12);
        double c[3];
        for (int d = 0; d < 3; ++d) c[d] = prev[d] + 3.8 * u[d] / nrm;
        if (c[0] * c[0] + c[1] * c[1] + c[2] * c[2] > radius * radius) continue;
        const double d2 = hash.min_dist2(c, ca);
        if (d2 >= 9.0) {
          for (int d = 0; d < 3; ++d) p[d] = c[d];
          found = true;
        } else if (d2 > best_d2) {
          best_d2 = d2;
          for (int d = 0; d < 3; ++d) best[d] = c[d];
        }
      }
      if (!found) {
        if (best_d2 >= 0.0) {
          for (int d = 0; d < 3; ++d) p[d] = best[d];
        } else {  // every try left the sphere: step towards the centre
          const double r = std::sqrt(prev[0] * prev[0] + prev[1] * prev[1] + prev[2] * prev[2]);
          for (int d = 0; d < 3; ++d) p[d] = prev[d] - 3.8 * prev[d] / std::fmax(r, 1e-9);
        }
      }
    }
    const int32_t id = (int32_t)(ca.size() / 3);
    for (int d = 0; d < 3; ++d) ca.push_back(p[d]);
    hash.add(p, id);
    for (int d = 0; d < 3; ++d) prev[d] = p[d];
    for (int d = 0; d < 3; ++d) xyz[3 * n + d] = p[d];
    element[n] = (int8_t)rng.element();
    ++n;
    const int side = 4 + (int)(rng.next() % 5);
    for (int k = 0; k < side && n < n_atoms; ++k, ++n) {
      for (int d = 0; d < 3; ++d) xyz[3 * n + d] = p[d] + 1.5 * rng.normal();
      element[n] = (int8_t)rng.element();
    }
  }
  return CRAB_OK;
}
