/*
 * crab_cuda.h — C ABI of the B200 (sm_100a) scattering engine.
 *
 * This is the boundary a host program (the crabSAXS Rust crate through
 * `extern "C"` declarations, Python through ctypes, C/C++ directly) binds to
 * replace crabSAXS's CPU engines.  Every entry point takes plain pointers and
 * sizes, returns an int status, and never retains a caller pointer after it
 * returns.  Host arrays are f64 (the reference's `Vec<f64>`); device memory
 * belongs to the context.
 *
 * Reference interfaces replaced (file:line in the crabSAXS repository):
 *   crab_debye_intensity          src/scattering.rs:86-110  debye_intensity_with_hydrogens
 *   crab_compute_curve            src/scattering.rs:112-212 compute_curve (Auto/Debye/Multipole dispatch)
 *   crab_debye_solvent_basis      src/solvent.rs:504-584    debye_solvent_basis
 *   crab_combine_solvent_basis    src/spherical.rs:567-584  combine_solvent_basis
 *   crab_hydration_grid_adaptive  src/solvent.rs:121-223    build_adaptive_hydration_grid
 *   crab_hydration_grid_exterior  src/solvent.rs:259-401    build_hydration_grid
 *   crab_multipole_intensity      src/spherical.rs:266-403  multipole_intensity(_streaming)
 *   crab_multipole_solvent_basis  src/spherical.rs:474-565  multipole_solvent_basis
 *   crab_fit                      src/fit.rs:288-454        fit_to_experimental_with_options
 *                                 (behind SaxsFitter::fit analysis.rs:76-87 and SaxsScorer::score analysis.rs:156-177)
 *   crab_ensemble_fit             src/ensemble.rs:127-299   EnsembleFitter::fit / fit_core
 *   crab_reweight_curves          src/reweight.rs:84-154    reweight_curves
 *   crab_coordinate_features      src/metrics.rs:236-270    coordinate_features (P(r): metrics.rs:475-583)
 *   crab_parse_structure          src/structure.rs:205-345  Structure::from_pdb_file(_with_options / _models_with_options)
 *
 * Status codes map onto crabSAXS's SaxsError (src/error.rs:4-25):
 *   CRAB_EINVAL -> SaxsError::InvalidInput, CRAB_ENOTCONV -> FitDidNotConverge,
 *   CRAB_EPARSE -> StructureParse, CRAB_EELEMENT -> UnsupportedElement, CRAB_EIO -> Io,
 *   every other non-zero code -> SaxsError::Other (message from crab_ctx_last_error;
 *   crab_parse_last_error for the ingest calls).
 *
 * Threading: a context serialises its own calls with an internal mutex; use
 * one context per host thread for concurrency (rayon workers in the reference
 * call compute_curve concurrently, ensemble.rs:244).
 */
#ifndef CRAB_CUDA_H
#define CRAB_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CRAB_OK 0
#define CRAB_EINVAL 1       /* invalid input (SaxsError::InvalidInput) */
#define CRAB_ENOMEM 2       /* device or host allocation failed */
#define CRAB_ECUDA 3        /* CUDA runtime error */
#define CRAB_ETIMEOUT 4     /* a bounded device-side wait ran out */
#define CRAB_ENOTCONV 5     /* fit did not converge (SaxsError::FitDidNotConverge) */
#define CRAB_ECAPACITY 6    /* caller buffer too small (two-call size query) */
#define CRAB_ENODEVICE 7    /* no CUDA device / extension not usable */
#define CRAB_EPARSE 8       /* malformed structure text (SaxsError::StructureParse) */
#define CRAB_EELEMENT 9     /* element without coefficients (SaxsError::UnsupportedElement) */
#define CRAB_EIO 10         /* file could not be read (SaxsError::Io) */

/* Element codes, in crabSAXS's `Element` order (src/structure.rs:90-106). */
enum {
  CRAB_EL_H = 0, CRAB_EL_C, CRAB_EL_N, CRAB_EL_O, CRAB_EL_S, CRAB_EL_P, CRAB_EL_NA, CRAB_EL_MG,
  CRAB_EL_CL, CRAB_EL_CA, CRAB_EL_FE, CRAB_EL_ZN, CRAB_EL_K, CRAB_EL_I, CRAB_EL_OTHER
};

/* Hydration models (src/solvent.rs:18-25). */
enum { CRAB_HYD_ANALYTIC = 0, CRAB_HYD_GRID = 1, CRAB_HYD_ADAPTIVE = 2 };
/* Scattering methods (src/scattering.rs:16-21). */
enum { CRAB_METHOD_AUTO = 0, CRAB_METHOD_DEBYE = 1, CRAB_METHOD_MULTIPOLE = 2 };
/* Multipole GEMM precision. */
enum { CRAB_PREC_FP64 = 0, CRAB_PREC_TF32 = 1, CRAB_PREC_BF16 = 2, CRAB_PREC_BF16_SPLIT = 3, CRAB_PREC_TF32_SPLIT = 4,
       CRAB_PREC_FP32 = 5, CRAB_PREC_TF32_FUSED = 6, CRAB_PREC_TF32_SPLIT_FUSED = 7 };
/* fit.rs:30-47 modes. */
enum { CRAB_SCALE_FIT = 0, CRAB_SCALE_FIXED = 1 };
enum { CRAB_BG_FIT = 0, CRAB_BG_FIXED_ZERO = 1, CRAB_BG_FIXED = 2 };

/* SolventParams (src/solvent.rs:27-50). Defaults: c1=1, c2=0, t=3 Å, ρ=0.334, Analytic, 4 Å. */
typedef struct crab_solvent {
  double c1;
  double c2;
  double shell_thickness;   /* Å */
  double bulk_density;      /* e/Å^3 */
  int32_t hydration_model;  /* CRAB_HYD_* */
  int32_t _pad;
  double grid_spacing;      /* Å, adaptive grid */
} crab_solvent;

/* ComputeOptions (src/scattering.rs:28-47); has_solvent=0 means `solvent: None`. */
typedef struct crab_compute_options {
  int32_t method;           /* CRAB_METHOD_* */
  int32_t implicit_hydrogen;/* HydrogenMode::Implicit = 1, Explicit = 0 */
  int32_t l_max;            /* 0 = adaptive (None), else 8..64 */
  int32_t has_solvent;
  crab_solvent solvent;
} crab_compute_options;

/* FitOptions (src/fit.rs:49-82). */
typedef struct crab_fit_options {
  int32_t method;
  int32_t implicit_hydrogen;
  double c1_lo, c1_hi, c2_lo, c2_hi;
  int32_t max_iterations;
  int32_t q_sampling_stride;
  crab_solvent solvent;
  int32_t scale_mode;       /* CRAB_SCALE_* */
  int32_t bg_mode;          /* CRAB_BG_* */
  double scale_value;
  double bg_value;
  int32_t optimizer;        /* 0 Nelder-Mead (reference), 1 L-BFGS-B on the analytic gradient */
  int32_t _pad;
} crab_fit_options;

/* FitResult (src/fit.rs:19-27), fitted curve written to a caller buffer. */
typedef struct crab_fit_result {
  double scale, background, c1, c2;
  double chi2;              /* reduced chi^2, N-1 convention (fit.rs:185-196) */
  int32_t iterations;
  int32_t converged;
} crab_fit_result;

typedef struct crab_ctx crab_ctx;
typedef struct crab_struct crab_struct;

/* ---- context ------------------------------------------------------------ */
int crab_ctx_create(int device, crab_ctx** out);
int crab_ctx_destroy(crab_ctx* ctx);
const char* crab_ctx_last_error(const crab_ctx* ctx);
/* Launch counter and the device time (ms, CUDA events on the context stream)
 * of the most recent pair-sum kernel; for measurement harnesses. */
int crab_ctx_stats(crab_ctx* ctx, int64_t* kernel_launches, double* last_pair_kernel_ms, double* last_pair_kernel_pairq);
int crab_ctx_reset_stats(crab_ctx* ctx);
/* Device-resident workspace size in bytes (for sizing studies). */
int crab_ctx_workspace_bytes(crab_ctx* ctx, int64_t* bytes);
/* Failure injection for tests of the error paths (no counterpart in the
 * reference; its error cases are SaxsError values, src/error.rs:4-25).
 * crab_ctx_set_wait_budget: iteration budget of every bounded device-side
 * wait (mbarrier waits on bulk copies and tensor-core stages) in kernels
 * this context launches; 0 makes the first wait give up, a negative value
 * restores the defaults.  A kernel whose wait runs out drains its own copies
 * and tensor-core work in flight (with a budget this option does not
 * shorten), and the call returns CRAB_ETIMEOUT; the context stays usable.
 * crab_ctx_fail_allocations: the next `after` device or pinned host
 * allocations of this context succeed, the one after fails with CRAB_ENOMEM
 * (and every later one until the option is reset); negative: off. */
int crab_ctx_set_wait_budget(crab_ctx* ctx, int64_t iterations);
int crab_ctx_fail_allocations(crab_ctx* ctx, int64_t after);

/* ---- atom typing (host) ------------------------------------------------- */
/* formfactor.rs:357-417 united_atom_group: residue + atom name -> group code,
 * -1 when the atom is not a standard united atom. */
int crab_united_atom_group(const char* residue_name, const char* atom_name);
/* formfactor.rs:425-439 form_factor_for_atom, f64, host. */
double crab_form_factor(int element, int group, double occupancy, int implicit_hydrogen, double q);
/* solvent.rs:428-438 excluded_volume_for_atom. */
double crab_excluded_volume_for_atom(int element, int group, int implicit_hydrogen);

/* ---- structures --------------------------------------------------------- */
/* Upload a structure (src/structure.rs:151-165 Atom/Structure): xyz is n*3 f64,
 * occupancy n f64, element n codes (CRAB_EL_*), group n codes (-1 = none).
 * Coordinates are centred and cast to FP32 on upload; an f64 copy is kept for
 * the bit-exact hydration grids. */
int crab_structure_create(crab_ctx* ctx, const double* xyz, const double* occupancy, const int8_t* element,
                          const int8_t* group, int64_t n, crab_struct** out);
int crab_structure_destroy(crab_struct* st);
int64_t crab_structure_atom_count(const crab_struct* st);

/* ---- Debye engine ------------------------------------------------------- */
/* Vacuum Debye intensity, clamp >= 0 (scattering.rs:86-110). */
int crab_debye_intensity(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int implicit_hydrogen,
                         double* out);
/* Six Debye terms vv, ee, hh, ve, vh, eh, out6 is [6][nq] (solvent.rs:504-584).
 * The hydration grid (if any) is built on the device. */
int crab_debye_solvent_basis(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq,
                             const crab_solvent* solvent, int implicit_hydrogen, double* out6);
/* Same six terms with the pair sums in the chosen precision: CRAB_PREC_FP32
 * (the recurrence kernel, as crab_debye_solvent_basis) or CRAB_PREC_FP64
 * (direct f64 sinc on the device: the FP64 reference for error reports). */
int crab_debye_solvent_basis_ex(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq,
                                const crab_solvent* solvent, int implicit_hydrogen, int precision, double* out6);
/* Multi-GPU (one process and one context per GPU): shard `shard` of
 * `n_shards` of crab_debye_solvent_basis_ex.  Each shard sums its share of
 * the pair work list (the owners of crab_shard_assign over the plan's work
 * items, the same on every rank, so no exchange is needed to split the
 * work); the self terms, the exact q = 0 sums and the hydration-site
 * lattice block are added on shard 0 only.  The element-wise sum of out6
 * over all shards is crab_debye_solvent_basis_ex's result up to the order of
 * the f64 additions: the caller all-reduces (sums) out6 across the GPUs,
 * 6 × nq doubles.  No counterpart in the reference, which runs on one host
 * (its q loop is split over threads, solvent.rs:528).
 * n_shards < 1 or shard outside [0, n_shards): CRAB_EINVAL. */
int crab_debye_solvent_basis_shard(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq,
                                   const crab_solvent* solvent, int implicit_hydrogen, int precision, int shard,
                                   int n_shards, double* out6);
/* Owner shard of each of n work items with the given costs: items in order
 * (longest first), each to the shard with the least total cost so far, the
 * lowest index among equals.  Host-only; the sharded entry points apply it
 * to their work lists (cost = tile pairs of the item). */
int crab_shard_assign(const int64_t* cost, int64_t n, int32_t n_shards, int32_t* owner);
/* Recombination I = vv + G²ee + c2²hh − 2G·ve + 2c2·vh − 2G·c2·eh, clamp ≥0
 * (spherical.rs:567-584; G from solvent.rs:448-452). Host-only, f64. */
int crab_combine_solvent_basis(const double* q, int64_t nq, const double* basis6, double c1, double c2, double* out);
/* Low level: per atom-type-pair partial sums for caller-supplied types.
 *   out[ab*nq+k] = Σ_{i<j,{t_i,t_j}={a,b}} w_i w_j sinc(q_k r_ij), a<=b,
 *   ab = a*T - a*(a-1)/2 + (b-a);  self_out[a] = Σ_{t_i=a} w_i².
 * xyz n*3 f64, w n f64, type n in [0,T). The pair sum runs in FP32 on the
 * device with FP64 cross-block reduction; the f64 sums are exact on a
 * power-of-two fixed-point grid (step about 2^-52 of q_max (Σ|w|)²), so the
 * result is bit-identical from call to call on the same inputs and kernel
 * variant. */
int crab_debye_partials(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                        int32_t n_types, const double* q, int64_t nq, double* out, double* self_out);
/* Same partials computed in FP64 on the device with direct sin (no
 * recurrence): the on-device FP64 reference used to report errors. */
int crab_debye_partials_fp64(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                             int32_t n_types, const double* q, int64_t nq, double* out, double* self_out);
/* Shard `shard` of `n_shards` of crab_debye_partials (CRAB_PREC_FP32) or
 * crab_debye_partials_fp64 (CRAB_PREC_FP64), split as in
 * crab_debye_solvent_basis_shard: out and self_out summed over all shards are
 * the whole (self_out is zero on every shard but 0). */
int crab_debye_partials_shard(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                              int32_t n_types, const double* q, int64_t nq, int precision, int shard, int n_shards,
                              double* out, double* self_out);

/* Device-resident pair-sum plan: the layout (typed, tiled atoms), work list
 * and q-block parameters are uploaded once; each run launches only the pair
 * kernel on the context stream.  For throughput measurement and repeated
 * evaluation of one structure. */
typedef struct crab_pair_plan crab_pair_plan;
int crab_pair_plan_create(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                          int32_t n_types, const double* q, int64_t nq, crab_pair_plan** out);
/* Same, with the last type a lattice of hydration sites (unit weights) whose
 * integer voxel indices are `cells` (m*3): their site–site block is summed
 * exactly by a squared-distance histogram instead of the pair kernel. */
int crab_pair_plan_create_lattice(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type, int64_t n,
                                  int32_t n_types, const double* q, int64_t nq, const int32_t* cells, int64_t m,
                                  double spacing, crab_pair_plan** out);
/* The plan of shard `shard` of `n_shards` of the same problem (one per GPU):
 * the work items crab_shard_assign gives this shard, the self sums, q = 0
 * and the lattice block on shard 0 only, so the element-wise sum of the
 * shards' crab_pair_plan_read results (an all-reduce) is the whole. */
int crab_pair_plan_create_lattice_shard(crab_ctx* ctx, const double* xyz, const double* w, const int32_t* type,
                                        int64_t n, int32_t n_types, const double* q, int64_t nq,
                                        const int32_t* cells, int64_t m, double spacing, int32_t shard,
                                        int32_t n_shards, crab_pair_plan** out);
/* Launch the pair kernel `repeats` times.  Before each launch, when
 * flush_bytes > 0, a buffer of that size is overwritten on the same stream
 * (evicting L2); each launch is bracketed by CUDA events and its device time
 * in ms written to step_ms[i] (may be NULL). */
int crab_pair_plan_run(crab_ctx* ctx, crab_pair_plan* plan, int32_t repeats, int64_t flush_bytes, double* step_ms);
/* Autotune: time every compiled kernel variant on this plan (q-block length Q
 * = q values one thread advances per pair between exact re-seeds, and JB = j
 * atoms per thread iteration; JB >= 8 selects the q-packed kernel, whose f32x2
 * registers hold two consecutive q points, with (JB-8) % 4 independent chains,
 * built for three CTAs per SM when JB >= 12; JB = 5, 6, 7, 3: the q-packed
 * kernel with the pair weight folded into the recurrence state, with 1, 2,
 * 1, 1 chains at 2, 2, 3, 4 CTAs per SM; JB = 11: the folded kernel with two
 * chains per pair (q points 4n, 4n+1 and 4n+2, 4n+3, each stepping 4 q
 * steps), two CTAs per SM, run as JB = 5 on plans whose step angle exceeds
 * 0.25 rad; JB = 14, 15: the folded recurrence
 * with the per-pair set-up in a warpgroup of its own that feeds two
 * recurrence warpgroups through shared memory, 1 or 2 chains per thread, one
 * CTA per SM; JB = 12: the same split with one recurrence warpgroup for each
 * of three q blocks per work item) and keep the fastest.  *chosen = Q*16 + JB;
 * the first `capacity` variants and their times (ms) are written to
 * variants/ms (may be NULL), their count to *n_variants. */
int crab_pair_plan_autotune(crab_ctx* ctx, crab_pair_plan* plan, int32_t* chosen, int32_t* variants, double* ms,
                            int32_t capacity, int32_t* n_variants);
/* Kernel variant used by the plans that one-shot calls (Debye curves, bases,
 * partials, ensembles) build on this context: a code as
 * crab_pair_plan_autotune reports it, or 0 for the automatic choice. */
int crab_ctx_set_pair_variant(crab_ctx* ctx, int32_t variant);
/* Fix the kernel variant of an FP32 plan (a code as crab_pair_plan_autotune
 * reports it); CRAB_EINVAL for a variant that is not compiled. */
int crab_pair_plan_select(crab_ctx* ctx, crab_pair_plan* plan, int32_t variant);
/* Copy the partials of the last run to the host (layout of crab_debye_partials). */
int crab_pair_plan_read(crab_ctx* ctx, crab_pair_plan* plan, double* out, double* self_out);
/* Pair·q evaluations of one run: (n(n-1)/2) * nq. */
double crab_pair_plan_pairq(const crab_pair_plan* plan);
int crab_pair_plan_destroy(crab_pair_plan* plan);

/* Measured FP32 FMA throughput of the device (TFLOP/s, FMA = 2 FLOP): a
 * register-resident FFMA loop on every SM for about `ms` milliseconds. */
int crab_measure_fp32_peak(crab_ctx* ctx, double ms, double* tflops);
/* Bytes copied host->device and device->host by this context since the last
 * crab_ctx_reset_stats. */
int crab_ctx_transfer_stats(crab_ctx* ctx, int64_t* h2d_bytes, int64_t* d2h_bytes);

/* ---- public calculation boundary -------------------------------------- */
/* compute_curve (scattering.rs:112-212): validation, Auto rule, adaptive
 * l_max, dispatch to Debye or multipole, solvent recombination.
 * method_used (may be NULL) receives CRAB_METHOD_DEBYE or CRAB_METHOD_MULTIPOLE. */
int crab_compute_curve(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, const crab_compute_options* opt,
                       double* out, int32_t* method_used);

/* ---- hydration grids ---------------------------------------------------- */
/* Adaptive coarse shell (solvent.rs:121-223), bit-exact site list in z→y→x
 * order. Two-call size query: pass sites=NULL to read *m.  The query leaves
 * its sites on the device; a fill call that follows with the same structure
 * and options copies them out without building the grid again (any other
 * call builds its own).  A fill with capacity < *m returns CRAB_ECAPACITY
 * and keeps the query's sites for a retry. */
int crab_hydration_grid_adaptive(crab_ctx* ctx, crab_struct* st, double spacing, double clearance, double padding,
                                 double* sites, int64_t capacity, int64_t* m, double* voxel_volume);
/* Largest box (voxels) crab_hydration_grid_adaptive_noalloc accepts. */
#define CRAB_NOALLOC_MAX_VOXELS 4194304ull
/* No counterpart in the reference.  The adaptive shell of
 * crab_hydration_grid_adaptive for callers that cannot allocate device
 * memory (their host runtime owns the device allocator, their memory budget
 * is fixed, or they run where cudaMalloc is not allowed).  Inputs and outputs
 * are caller-owned DEVICE pointers: d_xyz (n*3 f64) and d_sites (capacity*3
 * f64); `stream` is a cudaStream_t (NULL = default stream) on the current
 * device.  Every temporary lives in one file-scope __device__ array sized for
 * CRAB_NOALLOC_MAX_VOXELS voxels (about 8 MiB, held by every GPU that loads
 * the library until the process exits); a larger box returns CRAB_EINVAL.
 * The function calls no cudaMalloc, cudaFree or allocating library routine.
 * Its first call on a device looks up the array's device address (once per
 * device); make that first call before any stream capture.  The address is
 * kept for the life of the process: after a cudaDeviceReset of a device, do
 * not call this function on that device again.  All calls share
 * the array, so calls whose work overlaps on the GPU race: serialise them.
 * *m receives the site count; capacity 0 is a size query (returns CRAB_OK);
 * with a smaller non-zero capacity the sites beyond it are not written and
 * the call returns CRAB_ECAPACITY.  A coordinate that is not finite returns
 * CRAB_EINVAL, as crab_structure_create does.  The call synchronises
 * `stream` before returning. */
int crab_hydration_grid_adaptive_noalloc(const double* d_xyz, int64_t n, double spacing, double clearance,
                                         double padding, double* d_sites, int64_t capacity, int64_t* m,
                                         double* voxel_volume, void* stream);
/* Exterior flood-fill shell (solvent.rs:259-401), bit-exact; the same
 * two-call protocol as crab_hydration_grid_adaptive. */
int crab_hydration_grid_exterior(crab_ctx* ctx, crab_struct* st, double spacing, double probe, double thickness,
                                 double* sites, int64_t capacity, int64_t* m, double* voxel_volume);

/* ---- multipole engine ------------------------------------------------- */
/* multipole_intensity (spherical.rs:266-403) with per-q adaptive order.
 * precision of the moment GEMM (j_l interpolated at Chebyshev nodes in r, so
 * the expansion is one GEMM [(L+1)^2 x N] x [N x nodes]):
 *   CRAB_PREC_FP64        f64 SIMT (device reference, 1e-9 of the oracle)
 *   CRAB_PREC_FP32        FP32 SIMT (about 4e-7)
 *   CRAB_PREC_TF32_SPLIT  tcgen05 tensor cores, TF32 hi+lo terms (about 5e-7;
 *                         the compute_curve default)
 *   CRAB_PREC_TF32        tcgen05, single TF32 term (about 1e-3)
 *   CRAB_PREC_BF16_SPLIT  tcgen05, BF16 hi+lo terms for every l (1e-5 to 6e-5)
 *   CRAB_PREC_BF16        tcgen05, single BF16 term (about 6e-3)
 *   CRAB_PREC_TF32_SPLIT_FUSED, CRAB_PREC_TF32_FUSED  the TF32 products with
 *                         Y_lm generated inside the GEMM kernel (the same
 *                         values bit for bit, no (L+1)^2 x N buffer in device
 *                         memory, slower at 100,000 atoms)
 * The TF32 modes write Y_lm to device memory and stream it into the GEMM;
 * the BF16 modes generate it inside the GEMM kernel. */
int crab_multipole_intensity(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max,
                             int implicit_hydrogen, int precision, double* out);
/* Device time of the last multipole call on this context: all its kernels
 * (total_ms), the moment GEMM alone (moments_ms) and that GEMM's algorithmic
 * FLOP count, 2 * (L+1)^2 * nodes * points (moments_flop).  Any pointer may
 * be NULL. */
int crab_multipole_last_timing(crab_ctx* ctx, double* total_ms, double* moments_ms, double* moments_flop);
/* multipole_solvent_basis (spherical.rs:474-565), out6 [6][nq]. */
int crab_multipole_solvent_basis(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max,
                                 const crab_solvent* solvent, int implicit_hydrogen, int precision, double* out6);
/* Sum over GPUs supplied by the caller: replace values[0..count) in place by
 * their element-wise sum over all ranks (an all-reduce: NCCL, MPI, ...) and
 * return CRAB_OK; any other return ends the call with that status. */
typedef int (*crab_sum_fn)(double* values, int64_t count, void* user);
/* No counterpart in the reference.  on != 0: the sharded multipole calls of
 * this context pass `sum` a pointer to the moments in DEVICE memory (the
 * context's own buffer on its device, the context's stream synchronised
 * before the call); the callback sums them in place over the ranks (an NCCL
 * all-reduce, say) and returns once the sum is complete, with no copy
 * through the host.  on == 0 (the default): a host copy. */
int crab_ctx_set_device_sums(crab_ctx* ctx, int32_t on);
/* Multi-GPU multipole (one process and context per GPU; no counterpart in
 * the reference, which splits its q loop over threads, spherical.rs:337-394).
 * Every rank passes the whole structure; rank `shard` of `n_shards` takes the
 * atoms (and hydration sites) [n*shard/n_shards, n*(shard+1)/n_shards) of
 * the typed list into its moments M^t_{lm,b} (the radial basis and centre
 * come from all atoms, so every rank has the same moment layout).  `sum` is
 * called once, with this rank's moments in host memory
 * (types x segments x 64 x (L+1)^2 rounded up to 128, about 11 MB for 100k
 * atoms at L = 50), or in device memory after crab_ctx_set_device_sums;
 * after it returns the rank runs the q pass, so every rank returns the whole
 * curve / basis.  n_shards == 1 needs no `sum` and is the unsharded call. */
int crab_multipole_intensity_shard(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max,
                                   int implicit_hydrogen, int precision, int shard, int n_shards, crab_sum_fn sum,
                                   void* user, double* out);
int crab_multipole_solvent_basis_shard(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max,
                                       const crab_solvent* solvent, int implicit_hydrogen, int precision, int shard,
                                       int n_shards, crab_sum_fn sum, void* user, double* out6);

/* ---- fitting and gradients --------------------------------------------- */
/* fit_to_experimental_with_options (fit.rs:288-454). fitted (nq) may be NULL. */
int crab_fit(crab_ctx* ctx, crab_struct* st, const double* q, const double* intensity, const double* sigma,
             int64_t nq, const crab_fit_options* opt, double init_c1, double init_c2, crab_fit_result* result,
             double* fitted);
/* Reduced chi^2 of model = scale*I(q;x,c1,c2)+background against (y, sigma)
 * for the analytic-hydration Debye model, and its gradient with respect to
 * every coordinate (grad_xyz, n*3, may be NULL) and (c1, c2, scale,
 * background) (grad_params, 4, may be NULL). New in this engine: the
 * reference has no gradient (its fit is derivative-free, fit.rs:401-418). */
int crab_chi2_grad(crab_ctx* ctx, crab_struct* st, const double* q, const double* y, const double* sigma, int64_t nq,
                   const crab_solvent* solvent, int implicit_hydrogen, double scale, double background, double* chi2,
                   double* grad_xyz, double* grad_params);

/* ---- ensembles ------------------------------------------------------------ */
/* EnsembleFitter::fit (ensemble.rs:127-232) over k structures sharing one q
 * grid. All conformers' per-type partials are produced by one persistent
 * launch; the 25 (c1,c2) candidates recombine them. weights (k), fitted (nq).
 * Options follow EnsembleOptions (ensemble.rs:14-38); fit_opt follows FitOptions. */
typedef struct crab_ensemble_options {
  int32_t fit_weights;
  int32_t uniform;
  double regularization;
  int32_t max_conformers;   /* 0 = None */
  int32_t bootstrap;
  double min_weight;
  uint64_t seed;
} crab_ensemble_options;
typedef struct crab_ensemble_result {
  double scale, background, c1, c2;
  double chi2, reduced_chi2;
  int32_t iterations;
  int32_t n_selected;
} crab_ensemble_result;
int crab_ensemble_fit(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q, const double* y,
                      const double* sigma, int64_t nq, const crab_ensemble_options* eopt,
                      const crab_fit_options* fopt, crab_ensemble_result* result, int32_t* selected,
                      double* weights, double* fitted, double* intervals, double* bootstrap_chi2);
/* (intervals: 3 per selected conformer, median/lower/upper of the bootstrap
 * weights (ensemble.rs:174-216); bootstrap_chi2: one per replicate; both may
 * be NULL.) */
/* Multi-GPU ensemble (one process and context per GPU), in two steps; no
 * counterpart in the reference, whose conformer loop is split over threads
 * (ensemble.rs:244).
 * crab_ensemble_partials: every rank passes all k structures (so all derive
 * the same atom types) and computes the pair sums of the conformers it owns:
 * conformers ordered by N² (longest first), owners as crab_shard_assign
 * gives them for costs N².  *n_types receives the ensemble's type count T;
 * out == NULL is that size query.  out holds k blocks of
 * T(T+1)/2 * nq + 2T doubles: the raw pair sums Σ w_i w_j sin(q r)/r per type
 * pair and q, then Σw² and Σw per type.  Blocks of conformers this rank does
 * not own are zero, so summing out over all ranks (an all-reduce) gathers
 * every conformer.  capacity (doubles) below k blocks: CRAB_ECAPACITY.
 * implicit_hydrogen must be the fit's fopt->implicit_hydrogen. */
int crab_ensemble_partials(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q, int64_t nq,
                           int implicit_hydrogen, int shard, int n_shards, int32_t* n_types, double* out,
                           int64_t capacity);
/* crab_ensemble_fit with the pair sums taken from the summed partials buffer
 * (every rank gets the same result); n_types as crab_ensemble_partials
 * reported it. */
int crab_ensemble_fit_partials(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q,
                               const double* y, const double* sigma, int64_t nq, const crab_ensemble_options* eopt,
                               const crab_fit_options* fopt, const double* partials, int32_t n_types,
                               crab_ensemble_result* result, int32_t* selected, double* weights, double* fitted,
                               double* intervals, double* bootstrap_chi2);
/* Batched curves for k conformers at every (c1,c2) candidate: curves is
 * [n_cand][k][nq]; cand is n_cand (c1,c2) pairs. One persistent launch for
 * all conformers' partials, one recombination launch. */
int crab_ensemble_curves(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q, int64_t nq,
                         const crab_solvent* solvent, int implicit_hydrogen, const double* cand, int32_t n_cand,
                         double* curves);

/* reweight_curves (reweight.rs:84-154), curves [k][nq]; prior may be NULL. */
typedef struct crab_reweight_options {
  double kl_strength, step_size, tolerance, min_weight;
  int32_t max_iterations;
  int32_t scale_mode, bg_mode;
  int32_t _pad;
  double scale_value, bg_value;
} crab_reweight_options;
typedef struct crab_reweight_result {
  double scale, background, chi2, reduced_chi2, kl_divergence, effective_sample_size;
  int32_t iterations, converged;
} crab_reweight_result;
int crab_reweight_curves(const double* curves, int32_t k, const double* q, const double* y, const double* sigma,
                         int64_t nq, const double* prior, const crab_reweight_options* opt, double* weights,
                         crab_reweight_result* result);

/* Ensemble scoring plan: the structures' layouts, the (c1,c2) candidate
 * amplitude tables and all device buffers, built once.  crab_ensemble_plan_score
 * replays one CUDA graph that computes every conformer's pair sums (one
 * persistent launch), every (candidate, conformer) curve, the simplex weight
 * fit per candidate (ensemble.rs:317-381), ∂χ²/∂w and ∂χ²/∂(c1,c2) at the best
 * candidate, and the KL-penalised reweighting (reweight.rs:84-154, uniform
 * prior) of the best candidate's curves.
 * best_fit (8): candidate index, c1, c2, scale, background, reduced χ²,
 * ∂χ²/∂c1, ∂χ²/∂c2.  weights, grad_w, kl_weights: k values each.
 * reweight_out (6): scale, background, reduced χ², KL, iterations, converged.
 * Any output may be NULL; elapsed_ms is the device time of the graph. */
typedef struct crab_ensemble_plan crab_ensemble_plan;
int crab_ensemble_plan_create(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q, int64_t nq,
                              const crab_solvent* solvent, int implicit_hydrogen, const double* cand, int32_t n_cand,
                              crab_ensemble_plan** out);
int crab_ensemble_plan_autotune(crab_ctx* ctx, crab_ensemble_plan* plan, int32_t* chosen);
int crab_ensemble_plan_score(crab_ctx* ctx, crab_ensemble_plan* plan, const double* y, const double* sigma,
                             const crab_fit_options* fit_options, const crab_reweight_options* reweight_options,
                             double* elapsed_ms, double* best_fit, double* weights, double* grad_w,
                             double* kl_weights, double* reweight_out);
int crab_ensemble_plan_destroy(crab_ensemble_plan* plan);

/* ---- coordinate pair-distance distribution -------------------------------- */
/* Weighted pair-distance histogram, coordinate_pr before normalisation
 * (metrics.rs:475-522).  dmax is the square root of the largest squared pair
 * distance dx*dx + dy*dy + dz*dz (f64, as the reference computes it); pair
 * i < j adds w_i*w_j to hist[min(floor(r_ij / step), bins - 1)], step =
 * dmax / bins.  The bin of every pair is the reference's, bit for bit; the
 * sums differ from the reference's only by f64 summation order.  xyz (n*3) and
 * w (n) are host arrays, bins in [1, 16777216], coordinates finite and below
 * 1e100 in magnitude.  When every pair distance is zero (n < 2 included)
 * *dmax = 0 and hist is all zero. */
int crab_pair_distance_histogram(crab_ctx* ctx, const double* xyz, const double* w, int64_t n, int64_t bins,
                                 double* dmax, double* hist);
/* coordinate_features (metrics.rs:236-270) with PrOptions::bins = bins:
 * weights |form_factor_for_atom(atom, implicit hydrogens, q = 0)| floored at
 * 1e-6, Rg about the weighted centre (rg), the largest pair distance (dmax),
 * and the normalised P(r) of max(bins, 16) bins (normalize_distribution,
 * metrics.rs:550-583): r and p receive *m values (*m = 1 for the reference's
 * single-point results: all atoms at one position, or a non-positive area);
 * pr_rg and pr_dmax are the distribution's Rg and Dmax, NaN for None.
 * r and p must hold max(bins, 16) values.  Empty structure: CRAB_EINVAL. */
int crab_coordinate_features(crab_ctx* ctx, crab_struct* st, int64_t bins, double* rg, double* dmax, double* r,
                             double* p, int64_t* m, double* pr_rg, double* pr_dmax);
/* Device time of the last pair-distance histogram on this context: all its
 * kernels (dmax pass, bin edges, histogram), the histogram kernel alone, the
 * number of pairs n(n-1)/2, and how the histogram was accumulated (mode):
 *   0  integer pair counts per class pair (at most 64 distinct weights),
 *      combined as count * w_a * w_b: deterministic
 *   1  f64 products w_i*w_j into per-warp shared-memory histograms
 *   2  as 1, into one row per block in device memory (many bins)
 *  -1  no histogram kernel ran (fewer than two atoms).
 * Any pointer may be NULL. */
int crab_pr_last_timing(crab_ctx* ctx, double* total_ms, double* histogram_ms, double* pairs, int32_t* mode);

/* ---- structure ingest (host only; no context or GPU needed) -------------- */
/* ParseOptions (structure.rs:168-201) and its defaults: HETATM records off,
 * waters off, glycans on, model 0, unknown elements rejected, reported
 * occupancy, highest-occupancy altloc, every chain. */
#define CRAB_FORMAT_AUTO 0   /* mmCIF when the text starts with data_ or has _atom_site., else PDB */
#define CRAB_FORMAT_PDB 1
#define CRAB_FORMAT_MMCIF 2
#define CRAB_ALTLOC_HIGHEST 0 /* AltlocPolicy::Highest (the last of equal maxima, as Iterator::max_by) */
#define CRAB_ALTLOC_FIRST 1
#define CRAB_ALTLOC_ALL 2
#define CRAB_OCC_REPORTED 0   /* OccupancyPolicy::Reported */
#define CRAB_OCC_SELECTED_FULL 1
typedef struct crab_parse_options {
  int32_t include_hetatm;
  int32_t include_waters;
  int32_t include_glycans;
  int32_t model_index;          /* 0-based */
  int32_t allow_unknown_elements;
  int32_t occupancy_policy;     /* CRAB_OCC_* */
  int32_t altloc_policy;        /* CRAB_ALTLOC_* */
  int32_t n_chains;             /* 0: every chain */
  const char* const* chains;    /* n_chains chain ids to keep */
} crab_parse_options;
typedef struct crab_parsed crab_parsed;
void crab_parse_options_default(crab_parse_options* options);
/* Message of the last failed parse call on this thread. */
const char* crab_parse_last_error(void);
/* Structure::from_pdb_file_with_options (structure.rs:209-327) on PDB or
 * mmCIF text: model selection, chain/HETATM/water/glycan filters, element
 * from the element column else the atom name (structure.rs:109-127),
 * alternate-location and occupancy policies, atoms sorted by (chain, residue
 * number, atom name).  Malformed numbers or a missing model: CRAB_EPARSE;
 * an unknown element without allow_unknown_elements: CRAB_EELEMENT. */
int crab_parse_structure(const char* text, int64_t len, int32_t format, const crab_parse_options* options,
                         crab_parsed** out);
/* Models in the text (Structure::from_pdb_file_models_with_options reads
 * model_index 0 .. n-1). */
int crab_parse_model_count(const char* text, int64_t len, int32_t format, int32_t* n_models);
/* The same from a file; the format follows the extension (.cif/.mmcif: mmCIF,
 * else PDB), as the reference's reader does. Unreadable file: CRAB_EIO. */
int crab_read_structure_file(const char* path, const crab_parse_options* options, crab_parsed** out);
int64_t crab_parsed_atom_count(const crab_parsed* parsed);
/* Atom fields (structure.rs:151-160): xyz n*3, occupancy, element (CRAB_EL_*),
 * united-atom group of (residue name, atom name) (formfactor.rs:357-417; -1
 * none), HETATM flag, residue number.  Any pointer may be NULL. */
int crab_parsed_arrays(const crab_parsed* parsed, double* xyz, double* occupancy, int8_t* element, int8_t* group,
                       int8_t* hetatm, int64_t* residue_id);
/* Names of atom i, valid until crab_parsed_destroy; NULL out of range. */
const char* crab_parsed_atom_name(const crab_parsed* parsed, int64_t i);
const char* crab_parsed_residue_name(const crab_parsed* parsed, int64_t i);
const char* crab_parsed_chain_id(const crab_parsed* parsed, int64_t i);
/* Every atom's name (which = 0), residue name (1) or chain id (2), each
 * followed by a newline; *len receives the byte count.  buf NULL: size query;
 * cap too small: CRAB_ECAPACITY. */
int crab_parsed_strings(const crab_parsed* parsed, int32_t which, char* buf, int64_t cap, int64_t* len);
int crab_parsed_destroy(crab_parsed* parsed);
/* crab_structure_create from a parsed structure. */
int crab_structure_from_parsed(crab_ctx* ctx, const crab_parsed* parsed, crab_struct** out);

/* ---- synthetic inputs (no counterpart in the reference) ----------------- */
/* Seeded protein-like structure: Cα-style self-avoiding walk (3.8 Å steps,
 * 3.0 Å exclusion) inside a sphere of `radius`, 4-8 side atoms per residue at
 * N(0, 1.5 Å), elements C/N/O/S at 63/17/19/1 %. xyz n*3, element n. */
int crab_synth_protein(uint64_t seed, int64_t n_atoms, double radius, double* xyz, int8_t* element);

#ifdef __cplusplus
}
#endif
#endif /* CRAB_CUDA_H */
