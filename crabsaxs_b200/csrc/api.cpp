// extern "C" entry points of libcrabsaxs_b200 and the host orchestration of
// the Debye engine.  See include/crab_cuda.h for the reference interfaces
// each function replaces.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>

#include "engine.hpp"
#include "ops.hpp"

// ---------------------------------------------------------------- context

bool crab::trace_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("CRAB_TRACE");
    return v && std::atoi(v) > 0;
  }();
  return on;
}

namespace {
thread_local crab::TraceScope* g_trace_top = nullptr;
}

crab::TraceScope::TraceScope(const char* n) : name(n), on(trace_enabled()), parent(nullptr) {
  if (!on) return;
  t0 = std::chrono::steady_clock::now();
  parent = g_trace_top;
  g_trace_top = this;
}

crab::TraceScope::~TraceScope() {
  if (!on) return;
  std::fprintf(stderr, "[crab] %s %.3f ms\n", name,
               std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  g_trace_top = parent;
}

void crab::trace_mark(const char* name) {
  if (!trace_enabled() || !g_trace_top) return;
  std::fprintf(stderr, "[crab] %s: %s at %.3f ms\n", g_trace_top->name, name,
               std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - g_trace_top->t0).count());
}

void crab_ctx::alloc_check() {
  if (fail_alloc_after < 0) return;
  if (fail_alloc_after == 0) throw crab::Error(CRAB_ENOMEM, "allocation failed (injected by crab_ctx_fail_allocations)");
  --fail_alloc_after;
}

void* crab_ctx::dev(const std::string& name, size_t bytes) {
  crab::DevBuf& b = bufs[name];
  if (b.bytes < bytes || !b.ptr) {
    alloc_check();
    if (b.ptr) cudaFree(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    const size_t want = std::max<size_t>(bytes, 256);
    CRAB_CUDA_CHECK(cudaMalloc(&b.ptr, want));
    b.bytes = want;
  }
  return b.ptr;
}

void* crab_ctx::host(const std::string& name, size_t bytes) {
  crab::HostBuf& b = hbufs[name];
  if (b.bytes < bytes || !b.ptr) {
    alloc_check();
    if (b.ptr) cudaFreeHost(b.ptr);
    b.ptr = nullptr;
    b.bytes = 0;
    const size_t want = std::max<size_t>(bytes, 256);
    CRAB_CUDA_CHECK(cudaMallocHost(&b.ptr, want));
    b.bytes = want;
  }
  return b.ptr;
}

namespace crab {

int guarded_impl(crab_ctx* ctx, const std::function<void()>& fn) {
  std::unique_lock<std::mutex> lock;
  if (ctx) {
    lock = std::unique_lock<std::mutex>(ctx->mu);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
      ctx->last_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
      return CRAB_ECUDA;
    }
  }
  try {
    fn();
    if (ctx) ctx->last_error.clear();
    return CRAB_OK;
  } catch (const Error& e) {
    if (ctx) ctx->last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    if (ctx) ctx->last_error = "host allocation failed";
    return CRAB_ENOMEM;
  } catch (const std::exception& e) {
    if (ctx) ctx->last_error = e.what();
    return CRAB_ECUDA;
  }
}

// scattering.rs:71-80
void validate_q(const double* q, int64_t nq) {
  for (int64_t k = 0; k < nq; ++k) {
    if (!std::isfinite(q[k]) || q[k] < 0.0 || (k > 0 && q[k] < q[k - 1]))
      throw Error(CRAB_EINVAL, "q values must be finite, non-negative, and non-decreasing");
  }
}

// scattering.rs:118-134
void validate_solvent(const crab_solvent& s) {
  if (!std::isfinite(s.c1) || s.c1 <= 0.0 || !std::isfinite(s.c2) || !std::isfinite(s.shell_thickness) ||
      s.shell_thickness <= 0.0 || !std::isfinite(s.bulk_density) || s.bulk_density <= 0.0 ||
      !std::isfinite(s.grid_spacing) || s.grid_spacing <= 0.0)
    throw Error(CRAB_EINVAL, "solvent parameters must be finite with positive dimensions, density, and c1");
  if (s.hydration_model < 0 || s.hydration_model > 2) throw Error(CRAB_EINVAL, "unknown hydration model");
}

// Whether every amplitude of a class vanishes for the requested terms.
static bool vacuum_zero(const AtomClass& c, bool implicit) {
  if (implicit && c.element == CRAB_EL_H) return true;
  return c.element == CRAB_EL_OTHER && c.group < 0;
}
static bool excluded_zero(const AtomClass& c, bool implicit) {
  return excluded_volume_for_atom(c.element, c.group, implicit) == 0.0;
}

TypedAtoms type_atoms(const crab_struct* st, bool implicit, TermSet need, const std::vector<double>* sites) {
  TypedAtoms t;
  type_atoms_into(st, implicit, need, sites, t);
  return t;
}

TypedAtoms& typed_scratch(crab_ctx* ctx) {
  if (!ctx->typed_scratch) ctx->typed_scratch = std::make_shared<TypedAtoms>();
  return *ctx->typed_scratch;
}

void type_atoms_into(const crab_struct* st, bool implicit, TermSet need, const std::vector<double>* sites,
                     TypedAtoms& t) {
  // Classes are (element 0..14, united-atom group -1..13), numbered in
  // (element, group) order; a direct 15 x 15 table replaces a map lookup per
  // atom.  Pass 1 finds the classes present and the kept count; pass 2 fills.
  t.cls.clear();
  t.T = 0;
  constexpr int kE = CRAB_EL_OTHER + 1, kG = 15;
  bool drop[kE][kG];
  for (int e = 0; e < kE; ++e)
    for (int g = 0; g < kG; ++g) {
      const AtomClass c{e, implicit ? g - 1 : -1};
      bool d = false;
      if (need == TermSet::Vacuum) d = vacuum_zero(c, implicit);
      else if (need == TermSet::SolventGrid) d = vacuum_zero(c, implicit) && excluded_zero(c, implicit);
      drop[e][g] = d;
    }
  int64_t present[kE][kG] = {};
  const int8_t* el = st->elem.data();
  const int8_t* gr = st->group.data();
  for (int64_t i = 0; i < st->n; ++i) ++present[el[i]][(implicit ? (int)gr[i] : -1) + 1];
  int index[kE][kG];
  int next = 0;
  int64_t nk = 0;
  for (int e = 0; e < kE; ++e)
    for (int g = 0; g < kG; ++g) {
      const bool used = present[e][g] > 0 && !drop[e][g];
      index[e][g] = used ? next++ : -1;
      if (used) {
        t.cls.push_back(AtomClass{e, g - 1});
        nk += present[e][g];
      }
    }
  const int64_t ns = sites ? (int64_t)sites->size() / 3 : 0;
  if (sites) t.cls.push_back(AtomClass{-1, -1});
  t.xyz.resize(3 * (size_t)(nk + ns));
  t.w.resize((size_t)(nk + ns));
  t.type.resize((size_t)(nk + ns));
  t.src.resize((size_t)(nk + ns));
  const double* xyz = st->xyz.data();
  const double* occ = st->occ.data();
  int64_t k = 0;
  for (int64_t i = 0; i < st->n; ++i) {
    const int ty = index[el[i]][(implicit ? (int)gr[i] : -1) + 1];
    if (ty < 0) continue;
    t.xyz[3 * k] = xyz[3 * i];
    t.xyz[3 * k + 1] = xyz[3 * i + 1];
    t.xyz[3 * k + 2] = xyz[3 * i + 2];
    t.w[k] = occ[i];
    t.type[k] = ty;
    t.src[k] = i;
    ++k;
  }
  for (int64_t s = 0; s < ns; ++s, ++k) {
    for (int d = 0; d < 3; ++d) t.xyz[3 * k + d] = (*sites)[3 * s + d];
    t.w[k] = 1.0;
    t.type[k] = next;
    t.src[k] = -1;
  }
  t.T = (int)t.cls.size();
}

void amplitude_tables(const TypedAtoms& t, const double* q, int64_t nq, const crab_solvent* solvent, bool implicit,
                      double site_volume, std::vector<double>& V, std::vector<double>& E, std::vector<double>& H) {
  const int T = t.T;
  V.assign((size_t)T * nq, 0.0);
  E.assign((size_t)T * nq, 0.0);
  H.assign((size_t)T * nq, 0.0);
  const bool grid = solvent && solvent->hydration_model != CRAB_HYD_ANALYTIC;
  for (int a = 0; a < T; ++a) {
    const size_t o = (size_t)a * nq;
    if (t.cls[a].element < 0) {
      for (int64_t k = 0; k < nq; ++k)
        H[o + k] = solvent->bulk_density / 10.0 * site_volume * water_form_factor(q[k]);
    } else if (!solvent) {
      for (int64_t k = 0; k < nq; ++k) V[o + k] = form_factor(t.cls[a].element, t.cls[a].group, 1.0, implicit, q[k]);
    } else {
      debye_class_amplitude_rows(t.cls[a], implicit, q, nq, solvent->bulk_density, solvent->shell_thickness,
                                 V.data() + o, E.data() + o, grid ? nullptr : H.data() + o);
    }
  }
}

Partials partials_for(crab_ctx* ctx, const TypedAtoms& t, const double* q, int64_t nq, bool fp64,
                      const GridResult* lattice_sites, int shard, int n_shards) {
  Partials P;
  Layout L;
  {
    TraceScope tl("build_layout");
    L = build_layout(t.xyz.data(), t.w.data(), t.type.data(), (int64_t)t.w.size(), t.T, fp64);
  }
  LatticeSpec spec;
  if (lattice_sites) {
    spec.cells = lattice_sites->cells.data();
    spec.m = (int64_t)lattice_sites->cells.size() / 3;
    spec.spacing = lattice_sites->spacing;
  }
  compute_partials(ctx, std::move(L), q, nq, fp64, P, lattice_sites ? &spec : nullptr, shard, n_shards);
  return P;
}

GridResult hydration_sites(crab_ctx* ctx, const crab_struct* st, const crab_solvent& s) {
  if (s.hydration_model == CRAB_HYD_ADAPTIVE)
    return adaptive_grid_device(ctx, st->xyz.data(), st->n, s.grid_spacing, 3.0, 12.0);
  return exterior_grid_device(ctx, st->xyz.data(), st->elem.data(), st->n, 1.0, 1.4, s.shell_thickness);
}

void debye_basis(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, const crab_solvent& s,
                 bool implicit, double* out6, bool fp64, int shard, int n_shards) {
  TraceScope trace("debye_basis");
  GridResult g;
  const bool grid = s.hydration_model != CRAB_HYD_ANALYTIC;
  if (grid) {
    TraceScope tg("hydration_sites");
    g = hydration_sites(ctx, st, s);
  }
  TypedAtoms& t = typed_scratch(ctx);
  std::vector<double> V, E, H;
  {
    TraceScope tt("type_atoms+tables");
    type_atoms_into(st, implicit, grid ? TermSet::SolventGrid : TermSet::SolventAnalytic, grid ? &g.sites : nullptr,
                    t);
    amplitude_tables(t, q, nq, &s, implicit, g.voxel_volume, V, E, H);
  }
  Partials P = partials_for(ctx, t, q, nq, fp64, grid ? &g : nullptr, shard, n_shards);
  quadratic_terms(P, V.data(), V.data(), out6);
  quadratic_terms(P, E.data(), E.data(), out6 + nq);
  quadratic_terms(P, H.data(), H.data(), out6 + 2 * nq);
  quadratic_terms(P, V.data(), E.data(), out6 + 3 * nq);
  quadratic_terms(P, V.data(), H.data(), out6 + 4 * nq);
  quadratic_terms(P, E.data(), H.data(), out6 + 5 * nq);
}

void debye_vacuum(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, bool implicit, double* out,
                  bool fp64) {
  TypedAtoms t = type_atoms(st, implicit, TermSet::Vacuum, nullptr);
  std::vector<double> V, E, H;
  amplitude_tables(t, q, nq, nullptr, implicit, 0.0, V, E, H);
  Partials P = partials_for(ctx, t, q, nq, fp64, nullptr);
  quadratic_terms(P, V.data(), V.data(), out);
  for (int64_t k = 0; k < nq; ++k) out[k] = std::fmax(out[k], 0.0);
}

void combine_basis(const double* q, int64_t nq, const double* b, double c1, double c2, double* out) {
  for (int64_t i = 0; i < nq; ++i) {
    const double es = excluded_volume_scale(q[i], c1);
    const double v = b[i] + es * es * b[nq + i] + c2 * c2 * b[2 * nq + i] - 2.0 * es * b[3 * nq + i] +
                     2.0 * c2 * b[4 * nq + i] - 2.0 * es * c2 * b[5 * nq + i];
    out[i] = std::fmax(v, 0.0);
  }
}

void centre_and_rmax(const crab_struct* st, double* c, double* rmax) {
  c[0] = c[1] = c[2] = 0.0;
  for (int64_t i = 0; i < st->n; ++i)
    for (int d = 0; d < 3; ++d) c[d] = c[d] + st->xyz[3 * i + d];
  const double n = (double)std::max<int64_t>(st->n, 1);
  for (int d = 0; d < 3; ++d) c[d] = c[d] / n;
  *rmax = 0.0;
  for (int64_t i = 0; i < st->n; ++i) {
    const double dx = st->xyz[3 * i] - c[0], dy = st->xyz[3 * i + 1] - c[1], dz = st->xyz[3 * i + 2] - c[2];
    *rmax = max_num(*rmax, std::sqrt(((0.0 + dx * dx) + dy * dy) + dz * dz));
  }
}

}  // namespace crab

using namespace crab;

#define GUARD(ctx, ...) return guarded_impl(ctx, [&]() __VA_ARGS__)

extern "C" {

int crab_ctx_create(int device, crab_ctx** out) {
  if (!out) return CRAB_EINVAL;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return CRAB_ENODEVICE;
  if (device < 0 || device >= count) return CRAB_EINVAL;
  crab_ctx* ctx = new (std::nothrow) crab_ctx();
  if (!ctx) return CRAB_ENOMEM;
  ctx->device = device;
  int rc = guarded_impl(ctx, [&]() {
    CRAB_CUDA_CHECK(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
    CRAB_CUDA_CHECK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    CRAB_CUDA_CHECK(cudaEventCreate(&ctx->ev_start));
    CRAB_CUDA_CHECK(cudaEventCreate(&ctx->ev_stop));
  });
  if (rc != CRAB_OK) {
    crab_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return CRAB_OK;
}

int crab_ctx_destroy(crab_ctx* ctx) {
  if (!ctx) return CRAB_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->bufs)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  for (auto& kv : ctx->hbufs)
    if (kv.second.ptr) cudaFreeHost(kv.second.ptr);
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return CRAB_OK;
}

const char* crab_ctx_last_error(const crab_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int crab_ctx_stats(crab_ctx* ctx, int64_t* launches, double* ms, double* pairq) {
  if (!ctx) return CRAB_EINVAL;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (launches) *launches = ctx->launches;
  if (ms) *ms = ctx->last_pair_ms;
  if (pairq) *pairq = ctx->last_pair_q;
  return CRAB_OK;
}

int crab_ctx_reset_stats(crab_ctx* ctx) {
  if (!ctx) return CRAB_EINVAL;
  std::lock_guard<std::mutex> g(ctx->mu);
  ctx->launches = 0;
  ctx->h2d_bytes = 0;
  ctx->d2h_bytes = 0;
  ctx->last_pair_ms = 0.0;
  ctx->last_pair_q = 0.0;
  return CRAB_OK;
}

int crab_ctx_workspace_bytes(crab_ctx* ctx, int64_t* bytes) {
  if (!ctx || !bytes) return CRAB_EINVAL;
  std::lock_guard<std::mutex> g(ctx->mu);
  int64_t s = 0;
  for (auto& kv : ctx->bufs) s += (int64_t)kv.second.bytes;
  *bytes = s;
  return CRAB_OK;
}

int crab_united_atom_group(const char* residue_name, const char* atom_name) {
  return united_atom_group(residue_name, atom_name);
}

double crab_form_factor(int element, int group, double occupancy, int implicit_hydrogen, double q) {
  if (element < 0 || element > CRAB_EL_OTHER || group < -1 || group > 13) return NAN;
  return form_factor(element, group, occupancy, implicit_hydrogen != 0, q);
}

double crab_excluded_volume_for_atom(int element, int group, int implicit_hydrogen) {
  if (element < 0 || element > CRAB_EL_OTHER || group < -1 || group > 13) return NAN;
  return excluded_volume_for_atom(element, group, implicit_hydrogen != 0);
}

int crab_structure_create(crab_ctx* ctx, const double* xyz, const double* occupancy, const int8_t* element,
                          const int8_t* group, int64_t n, crab_struct** out) {
  if (!ctx || !out) return CRAB_EINVAL;
  *out = nullptr;
  GUARD(ctx, {
    require(n >= 0, "negative atom count");
    require(n == 0 || (xyz && occupancy && element && group), "null structure array");
    for (int64_t i = 0; i < n; ++i) {
      require(std::isfinite(xyz[3 * i]) && std::isfinite(xyz[3 * i + 1]) && std::isfinite(xyz[3 * i + 2]),
              "atom coordinates must be finite");
      require(std::isfinite(occupancy[i]), "occupancy must be finite");
      require(element[i] >= 0 && element[i] <= CRAB_EL_OTHER, "unknown element code");
      require(group[i] >= -1 && group[i] <= 13, "unknown united-atom group code");
    }
    static std::atomic<uint64_t> next_serial{1};
    crab_struct* st = new crab_struct();
    st->ctx = ctx;
    st->serial = next_serial.fetch_add(1);
    st->n = n;
    st->xyz.assign(xyz, xyz + 3 * n);
    st->occ.assign(occupancy, occupancy + n);
    st->elem.assign(element, element + n);
    st->group.assign(group, group + n);
    *out = st;
  });
}

int crab_structure_destroy(crab_struct* st) {
  delete st;
  return CRAB_OK;
}

int64_t crab_structure_atom_count(const crab_struct* st) { return st ? st->n : -1; }

int crab_debye_intensity(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int implicit_hydrogen,
                         double* out) {
  if (!ctx || !st || (nq > 0 && (!q || !out))) return CRAB_EINVAL;
  GUARD(ctx, {
    validate_q(q, nq);
    debye_vacuum(ctx, st, q, nq, implicit_hydrogen != 0, out, false);
  });
}

int crab_debye_solvent_basis(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, const crab_solvent* solvent,
                             int implicit_hydrogen, double* out6) {
  if (!ctx || !st || !solvent || (nq > 0 && (!q || !out6))) return CRAB_EINVAL;
  GUARD(ctx, {
    validate_q(q, nq);
    validate_solvent(*solvent);
    debye_basis(ctx, st, q, nq, *solvent, implicit_hydrogen != 0, out6, false);
  });
}

int crab_debye_solvent_basis_ex(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq,
                                const crab_solvent* solvent, int implicit_hydrogen, int precision, double* out6) {
  if (!ctx || !st || !solvent || (nq > 0 && (!q || !out6))) return CRAB_EINVAL;
  if (precision != CRAB_PREC_FP32 && precision != CRAB_PREC_FP64) return CRAB_EINVAL;
  GUARD(ctx, {
    validate_q(q, nq);
    validate_solvent(*solvent);
    debye_basis(ctx, st, q, nq, *solvent, implicit_hydrogen != 0, out6, precision == CRAB_PREC_FP64);
  });
}

int crab_debye_solvent_basis_shard(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq,
                                   const crab_solvent* solvent, int implicit_hydrogen, int precision, int shard,
                                   int n_shards, double* out6) {
  if (!ctx || !st || !solvent || (nq > 0 && (!q || !out6))) return CRAB_EINVAL;
  if (precision != CRAB_PREC_FP32 && precision != CRAB_PREC_FP64) return CRAB_EINVAL;
  if (n_shards < 1 || shard < 0 || shard >= n_shards) return CRAB_EINVAL;
  GUARD(ctx, {
    validate_q(q, nq);
    validate_solvent(*solvent);
    debye_basis(ctx, st, q, nq, *solvent, implicit_hydrogen != 0, out6, precision == CRAB_PREC_FP64, shard,
                n_shards);
  });
}

int crab_shard_assign(const int64_t* cost, int64_t n, int32_t n_shards, int32_t* owner) {
  if (n < 0 || n_shards < 1 || (n > 0 && (!cost || !owner))) return CRAB_EINVAL;
  for (int64_t i = 0; i < n; ++i)
    if (cost[i] < 0) return CRAB_EINVAL;
  const std::vector<int32_t> o = shard_owners(cost, n, n_shards);
  std::copy(o.begin(), o.end(), owner);
  return CRAB_OK;
}

int crab_combine_solvent_basis(const double* q, int64_t nq, const double* basis6, double c1, double c2, double* out) {
  if (nq < 0 || (nq > 0 && (!q || !basis6 || !out))) return CRAB_EINVAL;
  combine_basis(q, nq, basis6, c1, c2, out);
  return CRAB_OK;
}

static int partials_entry(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                          int32_t T, const double* q, int64_t nq, double* out, double* self_out, bool fp64,
                          int shard = 0, int n_shards = 1) {
  if (!ctx || T <= 0 || n < 0 || nq < 0 || (n > 0 && (!xyz || !w || !type)) || (nq > 0 && (!q || !out)))
    return CRAB_EINVAL;
  if (n_shards < 1 || shard < 0 || shard >= n_shards) return CRAB_EINVAL;
  GUARD(ctx, {
    validate_q(q, nq);
    for (int64_t i = 0; i < n; ++i) require(type[i] >= 0 && type[i] < T, "atom type out of range");
    Layout L = build_layout(xyz, w, type, n, T, fp64);
    Partials P;
    compute_partials(ctx, std::move(L), q, nq, fp64, P, nullptr, shard, n_shards);
    std::copy(P.pair.begin(), P.pair.end(), out);
    if (self_out) std::copy(P.self.begin(), P.self.end(), self_out);
  });
}

int crab_debye_partials(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                        int32_t n_types, const double* q, int64_t nq, double* out, double* self_out) {
  return partials_entry(ctx, xyz, w, type, n, n_types, q, nq, out, self_out, false);
}

int crab_debye_partials_fp64(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                             int32_t n_types, const double* q, int64_t nq, double* out, double* self_out) {
  return partials_entry(ctx, xyz, w, type, n, n_types, q, nq, out, self_out, true);
}

int crab_debye_partials_shard(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                              int32_t n_types, const double* q, int64_t nq, int precision, int shard, int n_shards,
                              double* out, double* self_out) {
  if (precision != CRAB_PREC_FP32 && precision != CRAB_PREC_FP64) return CRAB_EINVAL;
  return partials_entry(ctx, xyz, w, type, n, n_types, q, nq, out, self_out, precision == CRAB_PREC_FP64, shard,
                        n_shards);
}

struct crab_pair_plan {
  crab_ctx* ctx;
  std::unique_ptr<crab::PairPlan> plan;
};

int crab_pair_plan_create(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                          int32_t T, const double* q, int64_t nq, crab_pair_plan** out) {
  if (!ctx || !out || T <= 0 || n < 0 || nq < 0 || (n > 0 && (!xyz || !w || !type)) || (nq > 0 && !q))
    return CRAB_EINVAL;
  *out = nullptr;
  GUARD(ctx, {
    validate_q(q, nq);
    for (int64_t i = 0; i < n; ++i) require(type[i] >= 0 && type[i] < T, "atom type out of range");
    Layout L = build_layout(xyz, w, type, n, T, false);
    crab_pair_plan* p = new crab_pair_plan{ctx, make_pair_plan(ctx, std::move(L), q, nq, false)};
    *out = p;
  });
}

int crab_pair_plan_create_lattice(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                                  int32_t T, const double* q, int64_t nq, const int32_t* cells, int64_t m,
                                  double spacing, crab_pair_plan** out) {
  return crab_pair_plan_create_lattice_shard(ctx, xyz, w, type, n, T, q, nq, cells, m, spacing, 0, 1, out);
}

int crab_pair_plan_create_lattice_shard(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type,
                                        int64_t n, int32_t T, const double* q, int64_t nq, const int32_t* cells,
                                        int64_t m, double spacing, int32_t shard, int32_t n_shards,
                                        crab_pair_plan** out) {
  if (!ctx || !out || T <= 0 || n < 0 || nq < 0 || (n > 0 && (!xyz || !w || !type)) || (nq > 0 && !q) ||
      m < 0 || (m > 0 && !cells) || !(spacing > 0.0) || n_shards < 1 || shard < 0 || shard >= n_shards)
    return CRAB_EINVAL;
  *out = nullptr;
  GUARD(ctx, {
    validate_q(q, nq);
    int64_t last = 0;
    for (int64_t i = 0; i < n; ++i) {
      require(type[i] >= 0 && type[i] < T, "atom type out of range");
      if (type[i] == T - 1) {
        require(w[i] == 1.0, "lattice sites must have unit weight");
        ++last;
      }
    }
    require(last == m, "cells must list every atom of the last type");
    Layout L = build_layout(xyz, w, type, n, T, false);
    LatticeSpec spec{cells, m, spacing};
    crab_pair_plan* p =
        new crab_pair_plan{ctx, make_pair_plan(ctx, std::move(L), q, nq, false, &spec, false, shard, n_shards)};
    *out = p;
  });
}

int crab_pair_plan_run(crab_ctx* ctx, crab_pair_plan* plan, int32_t repeats, int64_t flush_bytes, double* step_ms) {
  if (!ctx || !plan || repeats < 0 || flush_bytes < 0) return CRAB_EINVAL;
  GUARD(ctx, { pair_plan_run_timed(ctx, *plan->plan, repeats, flush_bytes, step_ms); });
}

int crab_pair_plan_read(crab_ctx* ctx, crab_pair_plan* plan, double* out, double* self_out) {
  if (!ctx || !plan || !out) return CRAB_EINVAL;
  GUARD(ctx, {
    pair_plan_fetch(ctx, *plan->plan, out, false);
    if (self_out) {  // the self sums belong to shard 0 (the shards' results add up to the whole)
      std::copy(plan->plan->L.self_w2.begin(), plan->plan->L.self_w2.end(), self_out);
      if (plan->plan->shard != 0) std::fill(self_out, self_out + plan->plan->L.T, 0.0);
    }
  });
}

int crab_pair_plan_autotune(crab_ctx* ctx, crab_pair_plan* plan, int32_t* chosen, int32_t* variants, double* ms,
                            int32_t capacity, int32_t* n_variants) {
  if (!ctx || !plan || capacity < 0) return CRAB_EINVAL;
  GUARD(ctx, {
    std::vector<int> v(capacity);
    int n = 0;
    const int c = pair_plan_autotune(ctx, *plan->plan, v.data(), ms, capacity, &n);
    if (chosen) *chosen = c;
    if (variants)
      for (int i = 0; i < n; ++i) variants[i] = v[i];
    if (n_variants) *n_variants = n;
  });
}

int crab_ctx_set_pair_variant(crab_ctx* ctx, int32_t variant) {
  if (!ctx) return CRAB_EINVAL;
  GUARD(ctx, {
    require(variant == 0 || pair_variant_known(variant), "unknown kernel variant " + std::to_string(variant));
    ctx->pair_variant = variant;
  });
}

int crab_ctx_set_wait_budget(crab_ctx* ctx, int64_t iterations) {
  if (!ctx) return CRAB_EINVAL;
  GUARD(ctx, { ctx->wait_budget = iterations < 0 ? -1 : (int)std::min<int64_t>(iterations, 1 << 30); });
}

int crab_ctx_set_device_sums(crab_ctx* ctx, int32_t on) {
  if (!ctx) return CRAB_EINVAL;
  GUARD(ctx, { ctx->device_sums = on != 0; });
}

int crab_ctx_fail_allocations(crab_ctx* ctx, int64_t after) {
  if (!ctx) return CRAB_EINVAL;
  GUARD(ctx, { ctx->fail_alloc_after = after < 0 ? -1 : after; });
}

int crab_pair_plan_select(crab_ctx* ctx, crab_pair_plan* plan, int32_t variant) {
  if (!ctx || !plan) return CRAB_EINVAL;
  GUARD(ctx, { pair_plan_select(ctx, *plan->plan, variant); });
}

double crab_pair_plan_pairq(const crab_pair_plan* plan) {
  if (!plan) return 0.0;
  const double n = (double)plan->plan->L.n;
  return n * (n - 1.0) / 2.0 * (double)plan->plan->nq;
}

int crab_pair_plan_destroy(crab_pair_plan* plan) {
  if (!plan) return CRAB_OK;
  cudaSetDevice(plan->ctx->device);
  delete plan;
  return CRAB_OK;
}

int crab_measure_fp32_peak(crab_ctx* ctx, double ms, double* tflops) {
  if (!ctx || !tflops || !(ms > 0.0)) return CRAB_EINVAL;
  GUARD(ctx, { *tflops = measure_fp32_peak(ctx, ms); });
}

int crab_ctx_transfer_stats(crab_ctx* ctx, int64_t* h2d, int64_t* d2h) {
  if (!ctx) return CRAB_EINVAL;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (h2d) *h2d = ctx->h2d_bytes;
  if (d2h) *d2h = ctx->d2h_bytes;
  return CRAB_OK;
}

int crab_compute_curve(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, const crab_compute_options* opt,
                       double* out, int32_t* method_used) {
  if (!ctx || !st || !opt || (nq > 0 && (!q || !out))) return CRAB_EINVAL;
  GUARD(ctx, {
    TraceScope trace("compute_curve");
    validate_q(q, nq);
    if (opt->has_solvent) validate_solvent(opt->solvent);
    if (opt->l_max != 0 && (opt->l_max < 8 || opt->l_max > 64))
      throw Error(CRAB_EINVAL, "multipole l_max must be between 8 and 64");
    require(opt->method >= 0 && opt->method <= 2, "unknown scattering method");
    const bool implicit = opt->implicit_hydrogen != 0;
    int method = opt->method;
    if (method == CRAB_METHOD_AUTO) {
      if (opt->has_solvent && opt->solvent.hydration_model != CRAB_HYD_ANALYTIC) method = CRAB_METHOD_MULTIPOLE;
      else if (st->n < 500) method = CRAB_METHOD_DEBYE;
      else method = CRAB_METHOD_MULTIPOLE;
    }
    double qmax = 0.0;
    for (int64_t k = 0; k < nq; ++k) qmax = std::fmax(qmax, q[k]);
    double c[3], rmax;
    centre_and_rmax(st, c, &rmax);
    int l_max = opt->l_max;
    if (l_max == 0) {
      long v = (long)std::ceil(qmax * rmax) + 8;
      l_max = (int)std::min(64L, std::max(8L, v));
    }
    if (method == CRAB_METHOD_DEBYE) {
      if (!opt->has_solvent) debye_vacuum(ctx, st, q, nq, implicit, out, false);
      else {
        std::vector<double> b(6 * nq);
        debye_basis(ctx, st, q, nq, opt->solvent, implicit, b.data(), false);
        combine_basis(q, nq, b.data(), opt->solvent.c1, opt->solvent.c2, out);
      }
    } else {
      if (!opt->has_solvent) multipole_intensity_impl(ctx, st, q, nq, l_max, implicit, CRAB_PREC_TF32_SPLIT, out);
      else multipole_solvent_intensity_impl(ctx, st, q, nq, l_max, opt->solvent, implicit, CRAB_PREC_TF32_SPLIT, out);
    }
    if (method_used) *method_used = method;
  });
}

// Two-call protocol: a size query (sites == NULL) builds the grid, leaves
// the sites on the device and keeps the result in the context; the fill call
// with the same structure and options copies those sites straight into the
// caller's buffer instead of building the grid again.  Structures are
// immutable, so the serial and the options identify the result; the device
// sites stay valid until the context builds another grid.
static int grid_entry(crab_ctx* ctx, crab_struct* st, int kind, double o0, double o1, double o2, double* sites,
                      int64_t capacity, int64_t* m, double* volume, const std::function<GridResult()>& build) {
  if (!ctx || !st || !m) return CRAB_EINVAL;
  GUARD(ctx, {
    const double option[3] = {o0, o1, o2};
    GridMemo* memo = ctx->grid_memo.get();
    const bool hit = memo && memo->serial == st->serial && memo->kind == kind &&
                     std::memcmp(memo->option, option, sizeof(option)) == 0 &&
                     (memo->result.m == 0 || memo->result.build == ctx->grid_builds);
    if (!hit) {
      ctx->grid_memo.reset();
      auto fresh = std::make_shared<GridMemo>();
      fresh->result = build();
      fresh->serial = st->serial;
      fresh->kind = kind;
      std::memcpy(fresh->option, option, sizeof(option));
      ctx->grid_memo = fresh;
    }
    const GridResult& g = ctx->grid_memo->result;
    const int64_t count = g.m;
    *m = count;
    if (volume) *volume = g.voxel_volume;
    if (sites) {
      if (capacity < count) throw Error(CRAB_ECAPACITY, "site buffer too small");
      copy_d2h(ctx, sites, g.d_sites, (size_t)count * 3 * sizeof(double), ctx->stream);
      CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
      ctx->grid_memo.reset();
      trim_grid_pool(ctx);
    }
  });
}

int crab_hydration_grid_adaptive(crab_ctx* ctx, crab_struct* st, double spacing, double clearance, double padding,
                                 double* sites, int64_t capacity, int64_t* m, double* voxel_volume) {
  return grid_entry(ctx, st, 0, spacing, clearance, padding, sites, capacity, m, voxel_volume,
                    [&]() { return adaptive_grid_device(ctx, st->xyz.data(), st->n, spacing, clearance, padding, false); });
}

int crab_hydration_grid_exterior(crab_ctx* ctx, crab_struct* st, double spacing, double probe, double thickness,
                                 double* sites, int64_t capacity, int64_t* m, double* voxel_volume) {
  return grid_entry(ctx, st, 1, spacing, probe, thickness, sites, capacity, m, voxel_volume, [&]() {
    return exterior_grid_device(ctx, st->xyz.data(), st->elem.data(), st->n, spacing, probe, thickness, false);
  });
}

}  // extern "C"
