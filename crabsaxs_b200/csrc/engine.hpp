// Internal declarations of the crabsaxs_b200 engine (host side).
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/crab_cuda.h"

namespace crab {

// Error carrying a crab status code; every extern "C" entry point catches it
// and stores the message in the context.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CRAB_CUDA_CHECK(expr)                                                                              \
  do {                                                                                                     \
    cudaError_t _e = (expr);                                                                               \
    if (_e != cudaSuccess)                                                                                 \
      throw ::crab::Error(_e == cudaErrorMemoryAllocation ? CRAB_ENOMEM : CRAB_ECUDA,                      \
                          std::string(#expr) + ": " + cudaGetErrorString(_e));                             \
  } while (0)

inline void require(bool ok, const std::string& msg) {
  if (!ok) throw Error(CRAB_EINVAL, msg);
}
// Literal messages: no std::string is built unless the check fails (these
// checks run once per atom).
inline void require(bool ok, const char* msg) {
  if (!ok) throw Error(CRAB_EINVAL, msg);
}

// std::fmin / std::fmax of operands that are not NaN (the second operand when
// the two compare equal, as minsd / maxsd give it), written as comparisons
// the compiler keeps inline; for the O(N) passes over validated, finite
// coordinates, where the library calls cost five times as much.
inline double min_num(double a, double b) { return a < b ? a : b; }
inline double max_num(double a, double b) { return a > b ? a : b; }

// Host-phase tracing: with CRAB_TRACE=1 in the environment every TraceScope
// prints "[crab] <name> <ms>" to stderr when it closes (wall time of the
// phase, including the stream synchronisations inside it).
bool trace_enabled();
// Prints the wall time since the innermost open TraceScope started (a split
// inside a phase).
void trace_mark(const char* name);
struct TraceScope {
  const char* name;
  bool on;
  std::chrono::steady_clock::time_point t0;
  TraceScope* parent;
  explicit TraceScope(const char* n);
  ~TraceScope();
};

// Grow-only device buffer: one per named slot in the context, so repeated
// calls reuse memory instead of allocating.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

// Pinned host staging buffer, grow-only.
struct HostBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace crab

namespace crab {
struct GridMemo;
struct TypedAtoms;
}

struct crab_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  std::mutex mu;
  std::string last_error;
  std::map<std::string, crab::DevBuf> bufs;
  std::map<std::string, crab::HostBuf> hbufs;
  int64_t launches = 0;
  int64_t h2d_bytes = 0, d2h_bytes = 0;
  double last_pair_ms = 0.0;
  double last_pair_q = 0.0;
  // device times of the last multipole call: all its kernels, the moment
  // GEMM alone, and the GEMM's algorithmic FLOP count
  double last_mp_ms = 0.0, last_mp_gemm_ms = 0.0, last_mp_gemm_flop = 0.0;
  int pair_variant = 0;  // kernel variant of plans built by one-shot calls (0: automatic)
  // Failure injection on the host (crab_ctx_set_wait_budget,
  // crab_ctx_fail_allocations): the iteration budget of the kernels'
  // bounded waits (-1: their defaults), and the number of device or pinned
  // host allocations that still succeed before the next one fails with
  // CRAB_ENOMEM (-1: never).
  int wait_budget = -1;
  int64_t fail_alloc_after = -1;
  // crab_ctx_set_device_sums: sharded multipole calls hand the sum callback
  // the moments in device memory instead of a host copy
  bool device_sums = false;
  // Called before every allocation the context makes: throws CRAB_ENOMEM
  // once the injected failure is due.
  void alloc_check();
  // device times of the last pair-distance histogram: all its kernels, the
  // histogram kernel alone, and the pairs it binned
  double last_pr_ms = 0.0, last_pr_hist_ms = 0.0, last_pr_pairs = 0.0;
  int last_pr_mode = -1;  // 0 class counts, 1 per-warp f64 shared, 2 f64 rows in device memory

  // Site list of the last hydration-grid size query (sites == NULL), kept
  // for the fill call that follows it with the same structure and options.
  std::shared_ptr<crab::GridMemo> grid_memo;
  // Host scratch of the one-structure calls, kept across calls so that their
  // multi-megabyte arrays are not mapped and faulted in afresh each time
  // (calls on a context are serialised): the typed atoms of the Debye and
  // multipole paths and the multipole's per-point radius, segment and group.
  std::shared_ptr<crab::TypedAtoms> typed_scratch;
  std::vector<double> mp_r;
  std::vector<int32_t> mp_seg_of, mp_group_of;
  uint64_t grid_builds = 0;  // hydration-grid builds on this context (each reuses the "grid." device slots)

  void* dev(const std::string& name, size_t bytes);
  void* host(const std::string& name, size_t bytes);
};

namespace crab {

// Counted host<->device copies on the context stream.
inline void copy_h2d(crab_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (!bytes) return;
  CRAB_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
  ctx->h2d_bytes += (int64_t)bytes;
}
inline void copy_d2h(crab_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (!bytes) return;
  CRAB_CUDA_CHECK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
  ctx->d2h_bytes += (int64_t)bytes;
}

// ---------------------------------------------------------------- tables
// Scattering class of an atom: element plus the united-atom group that is in
// effect for the requested hydrogen mode (-1 in explicit mode).
struct AtomClass {
  int element;
  int group;
  bool operator<(const AtomClass& o) const { return element != o.element ? element < o.element : group < o.group; }
  bool operator==(const AtomClass& o) const { return element == o.element && group == o.group; }
};

double form_factor_value(int element, int group, double q);  // without occupancy
double form_factor(int element, int group, double occ, bool implicit_h, double q);
double excluded_volume_for_atom(int element, int group, bool implicit_h);
double vdw_radius(int element);
double water_form_factor(double q);
double excluded_volume_scale(double q, double c1);
double fraser_gaussian(double q, double volume);
double adaptive_shell_width(double rg);
double adaptive_site_volume(double spacing);
int united_atom_group(const char* residue, const char* name);
double sinc(double x);

// Per-class amplitudes without occupancy for the Debye solvent model
// (solvent.rs:454-488): vacuum, excluded (times density), analytic shell.
void debye_class_amplitudes(const AtomClass& c, bool implicit_h, double q, double density, double thickness,
                            double* v, double* e, double* h);
// The same at nq values of q into rows v, e, h (bit-identical per q; h may be null).
void debye_class_amplitude_rows(const AtomClass& c, bool implicit_h, const double* q, int64_t nq, double density,
                                double thickness, double* v, double* e, double* h);
// Same for the multipole solvent model (spherical.rs:205-231).
void multipole_class_amplitudes(const AtomClass& c, bool implicit_h, double q, double density, double thickness,
                                double* v, double* e, double* h);
// The same at nq values of q into rows v, e, h (bit-identical per q; h may be null).
void multipole_class_amplitude_rows(const AtomClass& c, bool implicit_h, const double* q, int64_t nq, double density,
                                    double thickness, double* v, double* e, double* h);

// ---------------------------------------------------------------- layout
// Atoms of one pair-sum problem, grouped by type, spatially ordered inside
// each type, and padded per type to whole tiles of kTile atoms.
constexpr int kTile = 128;

struct Layout {
  int T = 0;
  int64_t n = 0;         // real atoms
  int64_t n_pad = 0;     // padded length
  int n_tiles = 0;
  std::vector<float> atoms;      // 4 floats per slot: x, y, z, w (centred)
  std::vector<double> atoms64;   // 4 doubles per slot (for the FP64 reference)
  std::vector<int32_t> tile_type;
  std::vector<float> tile_sphere;  // per tile: centre xyz + radius (for near/far tests)
  std::vector<double> self_w2;     // per type Σ w²
  std::vector<double> sum_w;       // per type Σ w
  std::vector<int64_t> source;     // per slot: index of the input atom, -1 for padding
  double extent = 0.0;             // max pair distance bound
};

// spatial: order the atoms of each type along a Morton curve, so that tiles
// are spatially compact (the P(r) distance bounds need it); otherwise they
// keep their input order within each type (the Debye sums compute every pair
// of a tile pair, so the order only changes the order of additions).
Layout build_layout(const double* xyz, const double* w, const int32_t* type, int64_t n, int T, bool with_f64,
                    bool spatial = false);

// Self + pair partials of a layout at every q (P = T(T+1)/2 rows).
struct Partials {
  int T = 0;
  int64_t nq = 0;
  std::vector<double> pair;  // [P][nq]
  std::vector<double> self;  // [T]
};

// Site–site block of a lattice type summed exactly by distance histogram.
struct LatticePart {
  bool active = false;
  int64_t m = 0;       // sites
  double spacing = 0.0;
  int bins = 0;        // squared lattice distances 0..bins-1
  int4* d_cells = nullptr;
  unsigned long long* d_hist = nullptr;
  double* d_out = nullptr;  // [nq] Σ_{i<j} sinc(q r_ij) over sites
};

// Device-resident pair-sum problem: layout, work list and q-block
// parameters uploaded once; launched any number of times.
struct PairPlan {
  Layout L;
  bool fp64 = false;
  int64_t nq = 0;
  std::vector<double> q;
  int n_pairs = 0, Q = 0, jb = 2, n_qblocks = 0, n_work = 0, wide = 0;
  double hmax = 0.0;  // largest half step angle Δr/2 of the plan's q blocks (rad)
  std::vector<void*> owned;
  std::vector<void*> qcfg;  // q-block and work-list buffers (rebuilt when Q changes)
  bool pooled = false;      // buffers from the context pool (a plan that lives inside one call)
  float4* d_atoms = nullptr;
  double4* d_atoms64 = nullptr;
  int* d_tile_type = nullptr;
  int4* d_work = nullptr;
  float4* d_qpar = nullptr;
  int2* d_qrange = nullptr;
  double* d_q = nullptr;
  double* d_out = nullptr;  // [n_pairs][nq] raw sums
  int* d_status = nullptr;
  int* d_next = nullptr;  // work-queue counter (the int after d_status)
  int64_t* d_work_out = nullptr;  // per work item output offset (batches of structures), or null
  double* d_scale = nullptr;      // per work item fixed-point scale of its structure's partials (a power of two)
  int lattice_first_tile = 0;
  // multi-GPU: this plan sums only the work items of shard `shard` of
  // `n_shards` (shard_owners); shard 0 alone adds the exact q = 0 sums and
  // the lattice block, so the shards' outputs add up to the whole
  int shard = 0, n_shards = 1;
  std::vector<int> segments;  // batch: tile start of every structure plus the end, else empty
  LatticePart lattice;
  ~PairPlan();
};

// Device memory of a pair plan: its own cudaMalloc, freed with the plan, or
// for a pooled plan the context's grow-only buffer of that name (no
// allocation once the pool is large enough).
inline void* plan_alloc(crab_ctx* ctx, PairPlan& P, std::vector<void*>& list, const char* name, size_t bytes) {
  bytes = bytes ? bytes : 1;
  if (P.pooled) return ctx->dev(std::string("pair.") + name, bytes);
  ctx->alloc_check();
  void* p = nullptr;
  CRAB_CUDA_CHECK(cudaMalloc(&p, bytes));
  list.push_back(p);
  return p;
}
// Lattice description of the last type (hydration sites on a voxel grid):
// cells are the sites' integer voxel indices (3 per site, in any order).
struct LatticeSpec {
  const int32_t* cells = nullptr;
  int64_t m = 0;
  double spacing = 0.0;
};
void lattice_plan_init(crab_ctx* ctx, PairPlan& P, const int32_t* cells, int64_t m, double spacing);
void lattice_plan_launch(crab_ctx* ctx, PairPlan& P, cudaStream_t s);
bool q_grid_uniform(const double* q, int64_t nq);
std::unique_ptr<PairPlan> make_pair_plan(crab_ctx* ctx, Layout&& L, const double* q, int64_t nq, bool fp64,
                                         const LatticeSpec* lattice = nullptr, bool pooled = false, int shard = 0,
                                         int n_shards = 1);
// Owner shard of every work item for n_shards GPUs: items are taken in the
// given order (work lists are sorted longest first) and each goes to the
// shard with the least cost so far, the lowest index among equals, so every
// rank computes the same owners without communicating.
std::vector<int32_t> shard_owners(const int64_t* cost, int64_t n, int n_shards);
// Enqueue the pair kernel on stream s (device time recorded when timed).
void pair_plan_launch(crab_ctx* ctx, PairPlan& P, cudaStream_t s, bool timed);
// Copy back and convert raw sums to P_ab(q) (divide by q; exact q = 0).
void pair_plan_fetch(crab_ctx* ctx, PairPlan& P, double* out, bool timed);
// One-shot: FP32 recurrence on a uniform grid, FP64 direct otherwise.
// With n_shards > 1 only shard `shard`'s part (self sums zero except on
// shard 0): the element-wise sum over all shards is the whole.
void compute_partials(crab_ctx* ctx, Layout&& L, const double* q, int64_t nq, bool force_fp64, struct Partials& out,
                      const LatticeSpec* lattice = nullptr, int shard = 0, int n_shards = 1);

std::unique_ptr<PairPlan> make_batch_pair_plan(crab_ctx* ctx, std::vector<Layout>&& parts, const double* q,
                                               int64_t nq);
void pair_plan_run_timed(crab_ctx* ctx, PairPlan& P, int repeats, int64_t flush_bytes, double* step_ms);
// Time each compiled kernel variant (q-block length Q, j atoms per iteration)
// once on this plan and keep the fastest; returns Q*16 + JB.
int pair_plan_autotune(crab_ctx* ctx, PairPlan& P, int* variants, double* ms_out, int capacity, int* n_out);
// Fix the kernel variant (Q*16 + jb, as pair_plan_autotune reports it).
void pair_plan_select(crab_ctx* ctx, PairPlan& P, int variant);
// True when `variant` (Q*16 + jb) names a compiled FP32 pair kernel.
bool pair_variant_known(int variant);
double measure_fp32_peak(crab_ctx* ctx, double target_ms);

// Quadratic form Σ_ij X_i Y_j sinc(q r_ij) for per-type amplitude tables
// X[t*nq+k], Y[t*nq+k] from partials.
void quadratic_terms(const Partials& P, const double* X, const double* Y, double* out);
inline int pair_index(int a, int b, int T) {
  if (a > b) { int t = a; a = b; b = t; }
  return a * T - a * (a - 1) / 2 + (b - a);
}

// ---------------------------------------------------------------- hydration grids
struct GridResult {
  std::vector<double> sites;   // 3 per site, z→y→x order (built with to_host)
  std::vector<int32_t> cells;  // 3 voxel indices per site (built with to_host)
  double spacing = 0.0;
  double voxel_volume = 0.0;
  int64_t m = 0;                   // number of sites
  const double* d_sites = nullptr;  // the sites on the device, valid until the context's next grid build
  uint64_t build = 0;               // crab_ctx::grid_builds of the build that made this result
};
// Key of a grid build: structure serial, grid kind (0 adaptive, 1 exterior)
// and the three options bit for bit.  The result's device sites are valid
// while result.build equals the context's grid_builds.
struct GridMemo {
  uint64_t serial = 0;
  int kind = -1;
  double option[3] = {0.0, 0.0, 0.0};
  GridResult result;
};
// With to_host false only m and d_sites are filled: the host vectors stay
// empty (the caller copies the sites itself before the next grid build).
GridResult adaptive_grid_device(crab_ctx* ctx, const double* xyz, int64_t n, double spacing, double clearance,
                                double padding, bool to_host = true);
GridResult exterior_grid_device(crab_ctx* ctx, const double* xyz, const int8_t* elem, int64_t n, double spacing,
                                double probe, double thickness, bool to_host = true);
// Releases "grid." device slots above the keep size (after a caller copied
// out the sites of a build made without to_host).
void trim_grid_pool(crab_ctx* ctx);

}  // namespace crab

struct crab_struct {
  crab_ctx* ctx = nullptr;
  uint64_t serial = 0;  // unique per structure in the process; the arrays never change after creation
  int64_t n = 0;
  std::vector<double> xyz;
  std::vector<double> occ;
  std::vector<int8_t> elem;
  std::vector<int8_t> group;
};

namespace crab {
// ---------------------------------------------------------------- coordinate P(r)
// Weighted pair-distance histogram (metrics.rs:475-522): returns dmax and
// fills hist[bins] with Σ w_i w_j per bin; dmax 0 and hist zero when every
// pair distance is zero.
double pair_distance_histogram(crab_ctx* ctx, const double* xyz, const double* w, int64_t n, int64_t bins,
                               double* hist);
// metrics.rs:236-270 coordinate_features (see crab_coordinate_features).
void coordinate_features(crab_ctx* ctx, const crab_struct* st, int64_t bins, double* rg, double* dmax, double* r,
                         double* p, int64_t* m, double* pr_rg, double* pr_dmax);
}  // namespace crab
