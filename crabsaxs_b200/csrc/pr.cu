// Coordinate pair-distance distribution P(r) (crabSAXS src/metrics.rs:475-541).
//
// The reference takes dmax as the square root of the largest squared pair
// distance d2 = dx*dx + dy*dy + dz*dz (f64, left to right), sets
// step = dmax / bins, and adds w_i*w_j for every pair i < j to bin
// min(floor(sqrt(d2) / step), bins - 1).  On the device:
//
//   k_pr_dmax    the exact f64 maximum of d2 over all pairs, skipping tile
//                pairs whose bounding spheres cannot reach a known lower bound
//                (a real pair's d2, found on the host in two O(n) passes)
//   k_pr_edges   per bin k the smallest f64 d2 that the reference's
//                floor(sqrt(d2) / step) maps to k or above: a binary search
//                over the bit patterns of non-negative doubles, with the same
//                IEEE-rounded sqrt and division.  The bin of a pair is then
//                the number of edges at or below its d2: bit-exact, with no
//                square root or division per pair
//   k_pr_hist    per pair: d2 in f64 with the reference's operation order (no
//                fused multiply-add), a bin estimate from centred FP32
//                coordinates, corrected against the exact edges, and the f64
//                product w_i*w_j added to a per-warp shared histogram
//   k_pr_reduce  the per-block rows summed in block order
//
// Atoms are the spatially ordered 128-atom tiles of build_layout (one type).
// A warp's 32 i atoms are every fourth slot of the tile, so the distances of
// one j atom to them spread over many bins and the shared atomics rarely
// collide.

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "engine.hpp"
#include "ops.hpp"

namespace crab {
namespace {

constexpr int kPrThreads = kTile;              // one i atom per thread
constexpr size_t kPrDynSmem = 96 * 1024;       // edges + per-warp histograms
constexpr int64_t kPrMaxBins = 1 << 24;

struct PrParams {
  double step;
  float inv_step;
  int degenerate;  // every pair distance is zero: no histogram
};

__device__ __forceinline__ double pr_sqdist(const double4& a, const double4& b) {
  const double dx = __dsub_rn(a.x, b.x), dy = __dsub_rn(a.y, b.y), dz = __dsub_rn(a.z, b.z);
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Work item w of the upper triangle of tile pairs, column-major: (a, b), a <= b.
__device__ __forceinline__ void pr_tri_decode(int64_t w, int& a, int& b) {
  int64_t bb = (int64_t)((sqrt(8.0 * (double)w + 1.0) - 1.0) * 0.5);
  while (bb > 0 && bb * (bb + 1) / 2 > w) --bb;
  while ((bb + 1) * (bb + 2) / 2 <= w) ++bb;
  b = (int)bb;
  a = (int)(w - bb * (bb + 1) / 2);
}

__global__ void __launch_bounds__(kPrThreads)
    k_pr_dmax(const double4* __restrict__ pos, int64_t n, int n_tiles, const double4* __restrict__ sphere,
              double lower, unsigned long long* __restrict__ out) {
  __shared__ double4 sj[kPrThreads];
  __shared__ double red[kPrThreads / 32];
  double best = 0.0;
  const int64_t n_work = (int64_t)n_tiles * (n_tiles + 1) / 2;
  for (int64_t w = blockIdx.x; w < n_work; w += gridDim.x) {
    int a, b;
    pr_tri_decode(w, a, b);
    const double4 sa = sphere[a], sb = sphere[b];
    const double cx = sa.x - sb.x, cy = sa.y - sb.y, cz = sa.z - sb.z;
    const double ub = (sqrt(cx * cx + cy * cy + cz * cz) + sa.w + sb.w) * (1.0 + 1e-9);
    if (ub * ub < lower) continue;  // uniform over the block: no pair here reaches the bound
    const int64_t j0 = (int64_t)b * kPrThreads;
    __syncthreads();
    if (j0 + threadIdx.x < n) sj[threadIdx.x] = pos[j0 + threadIdx.x];
    __syncthreads();
    const int64_t i = (int64_t)a * kPrThreads + threadIdx.x;
    if (i < n) {
      const double4 pi = pos[i];
      const int jn = (int)(n - j0 < (int64_t)kPrThreads ? n - j0 : (int64_t)kPrThreads);
      for (int j = 0; j < jn; ++j) best = fmax(best, pr_sqdist(pi, sj[j]));
    }
  }
  for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kPrThreads / 32; ++k) best = fmax(best, red[k]);
    // non-negative doubles order as their bit patterns
    atomicMax(out, (unsigned long long)__double_as_longlong(best));
  }
}

// metrics.rs:515-516: floor(sqrt(d2) / step) as usize, capped at bins - 1
// (the cast saturates and sends NaN to 0).
__device__ __forceinline__ int64_t pr_bin_of(double d2, double step, int64_t bins) {
  const double v = floor(sqrt(d2) / step);
  if (!(v >= 0.0)) return 0;
  if (v >= (double)bins) return bins - 1;
  return (int64_t)v < bins - 1 ? (int64_t)v : bins - 1;
}

__global__ void k_pr_edges(const unsigned long long* __restrict__ dmax2_bits, int64_t bins, double* __restrict__ edges,
                           PrParams* __restrict__ par) {
  const double dmax2 = __longlong_as_double((long long)*dmax2_bits);
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (!(dmax2 > 0.0)) {
    if (k == 0) par->degenerate = 1;
    return;
  }
  const double step = sqrt(dmax2) / (double)bins;
  if (k == 0) {
    par->step = step;
    par->inv_step = (float)fmin(1.0 / step, (double)FLT_MAX);
    par->degenerate = 0;
  }
  if (k > bins) return;
  if (k == 0) { edges[0] = 0.0; return; }
  if (k == bins) { edges[bins] = __longlong_as_double(0x7FF0000000000000ll); return; }
  // smallest d2 with bin >= k: bin(+0) = 0 < k and bin(+inf) = bins - 1 >= k
  unsigned long long lo = 0ull, hi = 0x7FF0000000000000ull;
  while (hi - lo > 1ull) {
    const unsigned long long mid = lo + (hi - lo) / 2;
    if (pr_bin_of(__longlong_as_double((long long)mid), step, bins) >= k) hi = mid;
    else lo = mid;
  }
  edges[k] = __longlong_as_double((long long)hi);
}

template <bool kShared>
__global__ void __launch_bounds__(kPrThreads)
    k_pr_hist(const double4* __restrict__ pos, const float4* __restrict__ pos32, int64_t n, int n_tiles,
              const double* __restrict__ edges, const PrParams* __restrict__ par, int bins, int copies,
              double* __restrict__ rows) {
  extern __shared__ double pr_dyn[];  // kShared: edges[bins + 1], then copies x hist[bins]
  __shared__ double4 sj[kPrThreads];
  __shared__ float4 sj32[kPrThreads];
  if (par->degenerate) return;
  const float inv_step = par->inv_step;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double* E;
  double* H;
  if constexpr (kShared) {
    E = pr_dyn;
    H = pr_dyn + (bins + 1) + (size_t)(warp % copies) * bins;
    for (int k = threadIdx.x; k <= bins; k += kPrThreads) pr_dyn[k] = edges[k];
    for (int k = threadIdx.x; k < copies * bins; k += kPrThreads) pr_dyn[bins + 1 + k] = 0.0;
  } else {
    E = edges;
    H = rows + (size_t)blockIdx.x * bins;  // zeroed by the host
  }
  const int si = lane * 4 + warp;  // this thread's slot in the i tile
  const int64_t n_work = (int64_t)n_tiles * (n_tiles + 1) / 2;
  for (int64_t w = blockIdx.x; w < n_work; w += gridDim.x) {
    int a, b;
    pr_tri_decode(w, a, b);
    const int64_t j0 = (int64_t)b * kPrThreads;
    __syncthreads();
    if (j0 + threadIdx.x < n) {
      sj[threadIdx.x] = pos[j0 + threadIdx.x];
      sj32[threadIdx.x] = pos32[j0 + threadIdx.x];
    }
    __syncthreads();
    const int64_t i = (int64_t)a * kPrThreads + si;
    if (i >= n) continue;
    const double4 pi = pos[i];
    const float4 fi = pos32[i];
    const int jn = (int)(n - j0 < (int64_t)kPrThreads ? n - j0 : (int64_t)kPrThreads);
    for (int j = (a == b) ? si + 1 : 0; j < jn; ++j) {
      const double4 pj = sj[j];
      const float4 fj = sj32[j];
      const double d2 = pr_sqdist(pi, pj);
      const float fx = fi.x - fj.x, fy = fi.y - fj.y, fz = fi.z - fj.z;
      const float d2f = fx * fx + fy * fy + fz * fz;
      const float r = d2f * rsqrtf(fmaxf(d2f, 1e-30f));
      int e = min((int)(r * inv_step), bins - 1);
      e = max(e, 0);
      while (e + 1 < bins && d2 >= E[e + 1]) ++e;
      while (e > 0 && d2 < E[e]) --e;
      atomicAdd(&H[e], pi.w * pj.w);
    }
  }
  if constexpr (kShared) {
    __syncthreads();
    for (int k = threadIdx.x; k < bins; k += kPrThreads) {
      double s = 0.0;
      for (int c = 0; c < copies; ++c) s += pr_dyn[bins + 1 + (size_t)c * bins + k];
      rows[(size_t)blockIdx.x * bins + k] = s;
    }
  }
}

__global__ void k_pr_reduce(const double* __restrict__ rows, int n_rows, int bins, const PrParams* __restrict__ par,
                            double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= bins) return;
  double s = 0.0;
  if (!par->degenerate)
    for (int g = 0; g < n_rows; ++g) s += rows[(size_t)g * bins + k];
  out[k] = s;
}

inline double host_sqdist(const double* a, const double* b) {
  const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return dx * dx + dy * dy + dz * dz;
}

}  // namespace

double pair_distance_histogram(crab_ctx* ctx, const double* xyz, const double* w, int64_t n, int64_t bins,
                               double* hist) {
  TraceScope trace("pr.histogram");
  require(bins >= 1 && bins <= kPrMaxBins, "bins must be in [1, 16777216]");
  require(n >= 0, "negative atom count");
  for (int64_t i = 0; i < 3 * n; ++i)
    require(std::isfinite(xyz[i]) && std::fabs(xyz[i]) < 1e100, "coordinates must be finite and below 1e100");
  for (int64_t i = 0; i < n; ++i) require(std::isfinite(w[i]), "weights must be finite");
  std::fill(hist, hist + bins, 0.0);
  ctx->last_pr_ms = ctx->last_pr_hist_ms = 0.0;
  ctx->last_pr_pairs = (double)n * (double)(n > 0 ? n - 1 : 0) * 0.5;
  if (n < 2) return 0.0;

  // lower bound of the largest d2: a real pair, found by two farthest-point passes
  int64_t p0 = 0, p1 = 0;
  double best = -1.0;
  for (int64_t i = 0; i < n; ++i) {
    const double d = host_sqdist(xyz, xyz + 3 * i);
    if (d > best) { best = d; p0 = i; }
  }
  best = -1.0;
  for (int64_t i = 0; i < n; ++i) {
    const double d = host_sqdist(xyz + 3 * p0, xyz + 3 * i);
    if (d > best) { best = d; p1 = i; }
  }
  const double lower = host_sqdist(xyz + 3 * p0, xyz + 3 * p1);

  std::vector<int32_t> type(n, 0);
  Layout L;
  {
    TraceScope t2("pr.layout");
    L = build_layout(xyz, w, type.data(), n, 1, false);
  }
  const int n_tiles = L.n_tiles;
  const int64_t n_pad = L.n_pad;
  cudaStream_t s = ctx->stream;
  auto* h_pos = (double4*)ctx->host("pr.pos", (size_t)n_pad * sizeof(double4));
  auto* h_sph = (double4*)ctx->host("pr.sphere", (size_t)n_tiles * sizeof(double4));
  for (int64_t k = 0; k < n_pad; ++k) {
    const int64_t src = L.source[k];
    h_pos[k] = src >= 0 ? make_double4(xyz[3 * src], xyz[3 * src + 1], xyz[3 * src + 2], w[src])
                        : make_double4(0.0, 0.0, 0.0, 0.0);
  }
  for (int t = 0; t < n_tiles; ++t) {
    double c[3] = {0.0, 0.0, 0.0}, mag = 0.0;
    int cnt = 0;
    for (int k = t * kTile; k < (t + 1) * kTile && L.source[k] >= 0; ++k, ++cnt) {
      c[0] += h_pos[k].x; c[1] += h_pos[k].y; c[2] += h_pos[k].z;
    }
    for (int d = 0; d < 3; ++d) c[d] /= std::max(cnt, 1);
    double r2 = 0.0;
    for (int k = t * kTile; k < t * kTile + cnt; ++k) {
      const double p[3] = {h_pos[k].x, h_pos[k].y, h_pos[k].z};
      r2 = std::max(r2, host_sqdist(p, c));
      mag = std::max({mag, std::fabs(p[0]), std::fabs(p[1]), std::fabs(p[2])});
    }
    // inflated past the rounding of the centre and of every distance above
    h_sph[t] = make_double4(c[0], c[1], c[2], std::sqrt(r2) * (1.0 + 1e-12) + mag * 1e-12);
  }

  auto* d_pos = (double4*)ctx->dev("pr.pos", (size_t)n_pad * sizeof(double4));
  auto* d_pos32 = (float4*)ctx->dev("pr.pos32", (size_t)n_pad * sizeof(float4));
  auto* d_sph = (double4*)ctx->dev("pr.sphere", (size_t)n_tiles * sizeof(double4));
  auto* d_edges = (double*)ctx->dev("pr.edges", (size_t)(bins + 1) * sizeof(double));
  auto* d_out = (double*)ctx->dev("pr.out", (size_t)bins * sizeof(double));
  // PrParams and the dmax bits share one small buffer
  auto* d_misc = (char*)ctx->dev("pr.misc", 64);
  auto* d_dmax2 = (unsigned long long*)d_misc;
  auto* d_par = (PrParams*)(d_misc + 16);
  copy_h2d(ctx, d_pos, h_pos, (size_t)n_pad * sizeof(double4), s);
  copy_h2d(ctx, d_pos32, L.atoms.data(), (size_t)n_pad * sizeof(float4), s);
  copy_h2d(ctx, d_sph, h_sph, (size_t)n_tiles * sizeof(double4), s);
  CRAB_CUDA_CHECK(cudaMemsetAsync(d_misc, 0, 64, s));

  const int ibins = (int)bins;
  const size_t per_copy = (size_t)bins * sizeof(double);
  const size_t edge_bytes = (size_t)(bins + 1) * sizeof(double);
  int copies = 0;
  if (edge_bytes + per_copy <= kPrDynSmem)
    copies = (int)std::min<size_t>(kPrThreads / 32, (kPrDynSmem - edge_bytes) / per_copy);
  const bool shared_hist = copies > 0;
  const size_t dyn = shared_hist ? edge_bytes + (size_t)copies * per_copy : 0;
  int per_sm = 0;
  if (shared_hist) {
    CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_pr_hist<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    CRAB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pr_hist<true>, kPrThreads, dyn));
  } else {
    CRAB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pr_hist<false>, kPrThreads, 0));
  }
  const int64_t n_work = (int64_t)n_tiles * (n_tiles + 1) / 2;
  // one histogram row per block, at most 256 MB of rows (huge bin counts run fewer blocks)
  const int64_t max_rows = std::max<int64_t>(1, (int64_t)(256u << 20) / (int64_t)per_copy);
  const int grid = (int)std::max<int64_t>(
      1, std::min({(int64_t)ctx->sm_count * std::max(per_sm, 1), n_work, max_rows}));
  auto* d_rows = (double*)ctx->dev("pr.rows", (size_t)grid * per_copy);
  if (!shared_hist) CRAB_CUDA_CHECK(cudaMemsetAsync(d_rows, 0, (size_t)grid * per_copy, s));

  cudaEvent_t ev[3];
  for (auto& e : ev) CRAB_CUDA_CHECK(cudaEventCreate(&e));
  CRAB_CUDA_CHECK(cudaEventRecord(ev[0], s));
  int dgrid = 0;
  CRAB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&dgrid, k_pr_dmax, kPrThreads, 0));
  dgrid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->sm_count * std::max(dgrid, 1), n_work));
  k_pr_dmax<<<dgrid, kPrThreads, 0, s>>>(d_pos, n, n_tiles, d_sph, lower, d_dmax2);
  CRAB_CUDA_CHECK(cudaGetLastError());
  k_pr_edges<<<(unsigned)((bins + 1 + 127) / 128), 128, 0, s>>>(d_dmax2, bins, d_edges, d_par);
  CRAB_CUDA_CHECK(cudaGetLastError());
  CRAB_CUDA_CHECK(cudaEventRecord(ev[1], s));
  if (shared_hist)
    k_pr_hist<true><<<grid, kPrThreads, dyn, s>>>(d_pos, d_pos32, n, n_tiles, d_edges, d_par, ibins, copies, d_rows);
  else
    k_pr_hist<false><<<grid, kPrThreads, 0, s>>>(d_pos, d_pos32, n, n_tiles, d_edges, d_par, ibins, 1, d_rows);
  CRAB_CUDA_CHECK(cudaGetLastError());
  CRAB_CUDA_CHECK(cudaEventRecord(ev[2], s));
  k_pr_reduce<<<(ibins + 127) / 128, 128, 0, s>>>(d_rows, grid, ibins, d_par, d_out);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 4;
  auto* h_misc = (char*)ctx->host("pr.misc", 64);
  copy_d2h(ctx, h_misc, d_misc, 64, s);
  copy_d2h(ctx, hist, d_out, (size_t)bins * sizeof(double), s);
  CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
  float t_all = 0.f, t_hist = 0.f;
  CRAB_CUDA_CHECK(cudaEventElapsedTime(&t_hist, ev[1], ev[2]));
  CRAB_CUDA_CHECK(cudaEventElapsedTime(&t_all, ev[0], ev[2]));
  for (auto& e : ev) cudaEventDestroy(e);
  ctx->last_pr_ms = t_all;
  ctx->last_pr_hist_ms = t_hist;
  unsigned long long bits;
  std::memcpy(&bits, h_misc, sizeof bits);
  double dmax2;
  std::memcpy(&dmax2, &bits, sizeof dmax2);
  if (!(dmax2 > 0.0)) {
    std::fill(hist, hist + bins, 0.0);
    return 0.0;
  }
  return std::sqrt(dmax2);
}

namespace {

// metrics.rs:550-583 normalize_distribution, in place on (r, p): trapezoid
// area to one, rg = sqrt(max(moment / 2, 0)) from the trapezoid of r^2 p,
// dmax = r at the last p above 1 % of the maximum (NaN stands for None).
// False when the area is not finite and positive.
bool normalize_distribution(int64_t m, const double* r, double* p, double* rg, double* dmax) {
  if (m <= 0) return false;
  double area = 0.0;
  for (int64_t i = 0; i + 1 < m; ++i) area += 0.5 * (r[i + 1] - r[i]) * (p[i] + p[i + 1]);
  if (!std::isfinite(area) || area <= 0.0) return false;
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
    if (p[i] > maximum * 0.01) {
      *dmax = r[i];
      break;
    }
  return true;
}

}  // namespace

void coordinate_features(crab_ctx* ctx, const crab_struct* st, int64_t bins, double* rg, double* dmax, double* r,
                         double* p, int64_t* m, double* pr_rg, double* pr_dmax) {
  TraceScope trace("pr.features");
  require(st->n > 0, "coordinate features require a non-empty structure");
  bins = std::max<int64_t>(bins, 16);
  const int64_t n = st->n;
  const double* xyz = st->xyz.data();
  // metrics.rs:245-266: |form factor at q = 0| with implicit hydrogens, floored at 1e-6
  std::vector<double> w(n);
  for (int64_t i = 0; i < n; ++i)
    w[i] = std::fmax(std::fabs(form_factor(st->elem[i], st->group[i], st->occ[i], true, 0.0)), 1e-6);
  double total = 0.0;
  for (int64_t i = 0; i < n; ++i) total += w[i];
  double c[3] = {0.0, 0.0, 0.0};
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) c[d] = c[d] + xyz[3 * i + d] * w[i];
  for (int d = 0; d < 3; ++d) c[d] = c[d] / total;
  double acc = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double dx = xyz[3 * i] - c[0], dy = xyz[3 * i + 1] - c[1], dz = xyz[3 * i + 2] - c[2];
    acc += w[i] * (((0.0 + dx * dx) + dy * dy) + dz * dz);
  }
  *rg = std::sqrt(acc / total);
  std::vector<double> hist(bins);
  const double dm = pair_distance_histogram(ctx, xyz, w.data(), n, bins, hist.data());
  *dmax = dm;
  if (dm <= 0.0) {  // metrics.rs:489-498
    r[0] = 0.0; p[0] = 1.0; *m = 1; *pr_rg = 0.0; *pr_dmax = 0.0;
    return;
  }
  const double step = dm / (double)bins;
  for (int64_t k = 0; k < bins; ++k) {
    r[k] = ((double)k + 0.5) * step;
    p[k] = hist[k];
  }
  *m = bins;
  if (!normalize_distribution(bins, r, p, pr_rg, pr_dmax)) {  // metrics.rs:527-532
    r[0] = step * 0.5; p[0] = 1.0; *m = 1; *pr_rg = 0.0; *pr_dmax = dm;
  }
}

}  // namespace crab

using namespace crab;

extern "C" {

int crab_pair_distance_histogram(crab_ctx* ctx, const double* xyz, const double* w, int64_t n, int64_t bins,
                                 double* dmax, double* hist) {
  if (!ctx || !dmax || !hist || (n > 0 && (!xyz || !w))) return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() { *dmax = pair_distance_histogram(ctx, xyz, w, n, bins, hist); });
}

int crab_coordinate_features(crab_ctx* ctx, crab_struct* st, int64_t bins, double* rg, double* dmax, double* r,
                             double* p, int64_t* m, double* pr_rg, double* pr_dmax) {
  if (!ctx || !st || !rg || !dmax || !r || !p || !m || !pr_rg || !pr_dmax) return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() { coordinate_features(ctx, st, bins, rg, dmax, r, p, m, pr_rg, pr_dmax); });
}

int crab_pr_last_timing(crab_ctx* ctx, double* total_ms, double* histogram_ms, double* pairs) {
  if (!ctx) return CRAB_EINVAL;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (total_ms) *total_ms = ctx->last_pr_ms;
  if (histogram_ms) *histogram_ms = ctx->last_pr_hist_ms;
  if (pairs) *pairs = ctx->last_pr_pairs;
  return CRAB_OK;
}

}  // extern "C"
