// Host orchestration shared by the entry points: typing, amplitude tables,
// basis assembly and the multipole/fit/ensemble drivers.
#pragma once

#include <functional>
#include <vector>

#include "engine.hpp"

namespace crab {

int guarded_impl(crab_ctx* ctx, const std::function<void()>& fn);
void validate_q(const double* q, int64_t nq);
void validate_solvent(const crab_solvent& s);

// Which amplitude terms a pair sum feeds; decides which atoms may be dropped
// because all their amplitudes vanish.
enum class TermSet { Vacuum, SolventAnalytic, SolventGrid };

// Atoms (plus optional hydration sites as the last type, element -1) mapped
// to dense scattering types.
struct TypedAtoms {
  std::vector<AtomClass> cls;
  std::vector<double> xyz, w;
  std::vector<int32_t> type;
  std::vector<int64_t> src;  // input atom index of each entry, -1 for hydration sites
  int T = 0;
};
TypedAtoms type_atoms(const crab_struct* st, bool implicit, TermSet need, const std::vector<double>* sites);
// The same into t, reusing its arrays' capacity.
void type_atoms_into(const crab_struct* st, bool implicit, TermSet need, const std::vector<double>* sites,
                     TypedAtoms& t);
// The context's reusable TypedAtoms (one per context; one user per call).
TypedAtoms& typed_scratch(crab_ctx* ctx);

// Per-type Debye amplitude tables [T][nq] (no occupancy).  solvent == NULL
// means vacuum form factors only.
void amplitude_tables(const TypedAtoms& t, const double* q, int64_t nq, const crab_solvent* solvent, bool implicit,
                      double site_volume, std::vector<double>& V, std::vector<double>& E, std::vector<double>& H);
Partials partials_for(crab_ctx* ctx, const TypedAtoms& t, const double* q, int64_t nq, bool fp64,
                      const GridResult* lattice_sites, int shard = 0, int n_shards = 1);
GridResult hydration_sites(crab_ctx* ctx, const crab_struct* st, const crab_solvent& s);
// With n_shards > 1 only shard `shard`'s part of the six rows (self terms on
// shard 0 only): the element-wise sum over all shards is the whole basis.
void debye_basis(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, const crab_solvent& s,
                 bool implicit, double* out6, bool fp64, int shard = 0, int n_shards = 1);
void debye_vacuum(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, bool implicit, double* out,
                  bool fp64);
void combine_basis(const double* q, int64_t nq, const double* b, double c1, double c2, double* out);
void centre_and_rmax(const crab_struct* st, double* c, double* rmax);

// Multipole engine (multipole.cu).
// Multi-GPU: with n_shards > 1 this rank's moments cover its share of the
// atoms and `sum` (called once) replaces them by the sum over all ranks; the
// output is then the whole result on every rank.
struct MpShard {
  int shard = 0, n_shards = 1;
  crab_sum_fn sum = nullptr;
  void* user = nullptr;
};
void multipole_intensity_impl(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, int l_max,
                              bool implicit, int precision, double* out, const MpShard& shard = MpShard());
void multipole_solvent_basis_impl(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, int l_max,
                                  const crab_solvent& s, bool implicit, int precision, double* out6,
                                  const MpShard& shard = MpShard());
void multipole_solvent_intensity_impl(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, int l_max,
                                      const crab_solvent& s, bool implicit, int precision, double* out);

}  // namespace crab
