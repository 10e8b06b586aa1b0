// Entry points whose device engines are added in later commits; they fail
// loudly with CRAB_EINVAL instead of computing anything on the host.
#include "engine.hpp"
#include "ops.hpp"

namespace crab {
void multipole_intensity_impl(crab_ctx*, const crab_struct*, const double*, int64_t, int, bool, int, double*) {
  throw Error(CRAB_EINVAL, "multipole engine not built in this version");
}
void multipole_solvent_basis_impl(crab_ctx*, const crab_struct*, const double*, int64_t, int, const crab_solvent&,
                                  bool, int, double*) {
  throw Error(CRAB_EINVAL, "multipole engine not built in this version");
}
void multipole_solvent_intensity_impl(crab_ctx*, const crab_struct*, const double*, int64_t, int, const crab_solvent&,
                                      bool, int, double*) {
  throw Error(CRAB_EINVAL, "multipole engine not built in this version");
}
}  // namespace crab

using namespace crab;
extern "C" {
int crab_multipole_intensity(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max, int implicit_hydrogen,
                             int precision, double* out) {
  return guarded_impl(ctx, [&]() { multipole_intensity_impl(ctx, st, q, nq, l_max, implicit_hydrogen, precision, out); });
}
int crab_multipole_solvent_basis(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max,
                                 const crab_solvent* solvent, int implicit_hydrogen, int precision, double* out6) {
  return guarded_impl(ctx, [&]() { multipole_solvent_basis_impl(ctx, st, q, nq, l_max, *solvent, implicit_hydrogen, precision, out6); });
}
}
