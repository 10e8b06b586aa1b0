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
//                IEEE-rounded sqrt and division.  A pair's bin is the number
//                of edges at or below its d2
//   k_pr_hist    per pair the bin coordinate x = r / step from centred FP32
//                coordinates scaled by 1/step.  When x is farther than a
//                proven error bound delta from every integer, floor(x) is the
//                reference's bin; otherwise (about 2*delta of the pairs) d2 is
//                computed in f64 with the reference's operation order (no
//                fused multiply-add) and placed against the exact edges.  In
//                full tiles the near-edge pairs are marked in a 32-bit mask
//                and placed after each 32-pair chunk, so the chunk itself has
//                no branches.
//                Accumulation: when the atoms carry few distinct weights the
//                tiles are grouped by weight class and each block counts pairs
//                per class pair in u32 shared counters (flushed to u64 global
//                counts); otherwise each warp adds the f64 product w_i*w_j to
//                its own shared histogram
//   k_pr_combine hist[k] = Σ over class pairs (in order) of count * w_a * w_b
//   k_pr_reduce  (weighted mode) the per-block rows summed in block order
//
// Atoms are the spatially ordered 128-atom tiles of build_layout.  Each block
// takes a contiguous run of the upper-triangle tile pairs (column-major), so
// its j tile stays staged across consecutive items and its class pair rarely
// changes.  A warp's 32 i atoms are every fourth slot of the tile, so the
// distances of one j atom to them spread over many bins and the shared
// atomics rarely collide.

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "engine.hpp"
#include "ops.hpp"

namespace crab {
namespace {

constexpr int kPrThreads = kTile;         // one i atom per thread
constexpr size_t kPrDynSmem = 96 * 1024;  // edges + histograms
constexpr int64_t kPrMaxBins = 1 << 24;
constexpr int kPrMaxClasses = 64;                 // weight classes for integer counting
constexpr size_t kPrMaxCountBytes = 256u << 20;   // u64 counts [class pairs][bins]
constexpr int kPrFlushItems = 1 << 19;            // u32 counters: at most 4096 pairs per warp per item

enum PrMode { kPrCounts = 0, kPrWeighted = 1, kPrWeightedGlobal = 2 };

struct PrParams {
  double step;
  float inv_step;
  float delta;     // bound on |x_fp32 - x_exact| in bins; FLT_MAX: always exact
  int degenerate;  // every pair distance is zero: no histogram
  int pad;
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

__device__ __forceinline__ int pr_pair_index(int a, int b, int T) {
  if (a > b) { const int t = a; a = b; b = t; }
  return a * T - a * (a - 1) / 2 + (b - a);
}

// tiles[t] = (weight class, real atoms in the tile); real atoms come first.
__global__ void __launch_bounds__(kPrThreads)
    k_pr_dmax(const double4* __restrict__ pos, const int2* __restrict__ tiles, int n_tiles,
              const double4* __restrict__ sphere, double lower, unsigned long long* __restrict__ out) {
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
    const int na = tiles[a].y, nb = tiles[b].y;
    __syncthreads();
    if ((int)threadIdx.x < nb) sj[threadIdx.x] = pos[(int64_t)b * kPrThreads + threadIdx.x];
    __syncthreads();
    if ((int)threadIdx.x < na) {
      const double4 pi = pos[(int64_t)a * kPrThreads + threadIdx.x];
      for (int j = 0; j < nb; ++j) best = fmax(best, pr_sqdist(pi, sj[j]));
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

// radius: the largest distance of an atom from the centre of the FP32
// coordinates.  The kernel scales the FP32 coordinates by inv_step = fl(1/step)
// when it stages them and takes x = sqrt.approx(d2f) in bins.  With
// R = radius / step and d = sqrt(d2) / step, x differs from d by at most
//   sqrt(3) * 2^-22 * R + 11.5 * 2^-24 * d
// (per coordinate the rounding to float and the scaling, 2 * 2^-24 * R each
// side of the difference; the difference, the sum of squares, a 4-ulp
// sqrt.approx and the rounded reciprocal step relative to d).  delta is four
// times that with d <= bins + 1; when delta would exceed a quarter bin, or
// above 2^20 bins, every pair takes the exact path.
__global__ void k_pr_edges(const unsigned long long* __restrict__ dmax2_bits, int64_t bins, double radius,
                           double* __restrict__ edges, PrParams* __restrict__ par) {
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
    const double bound = (1.7320508075688772 * 0x1p-22 * radius / step + 11.5 * 0x1p-24 * (double)(bins + 1));
    par->delta = bins > (1 << 20) ? FLT_MAX : (float)fmin(4.0 * bound, 0.25);
    if (4.0 * bound > 0.25) par->delta = FLT_MAX;
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

__device__ __forceinline__ float pr_sqrt_approx(float v) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

// Bin coordinate of a pair from FP32 coordinates already in bins.
__device__ __forceinline__ float pr_bin_coord(const float4& fi, const float4& fj) {
  const float fx = fi.x - fj.x, fy = fi.y - fj.y, fz = fi.z - fj.z;
  return pr_sqrt_approx(fx * fx + fy * fy + fz * fz);
}

// The reference's bin of a pair from its exact f64 d2, starting the search at
// the FP32 estimate x.
__device__ __forceinline__ int pr_exact_bin(const double4& pi, const double4& pj, float x, const double* E, int bins) {
  int e = (int)fminf(fmaxf(x, 0.0f), (float)(bins - 1));
  const double d2 = pr_sqdist(pi, pj);
  while (e + 1 < bins && d2 >= E[e + 1]) ++e;
  while (e > 0 && d2 < E[e]) --e;
  return e;
}

constexpr float kPrMagic = 12582912.0f;  // 1.5 * 2^23: x + kPrMagic holds floor(x) in its low bits
constexpr int kPrMagicBits = 0x4B400000;

// Packed f32x2 arithmetic (two pairs per instruction, each lane rounded as
// the scalar operation).
__device__ __forceinline__ unsigned long long pr_pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void pr_unpack(unsigned long long v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long pr_sub2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long pr_mul2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ unsigned long long pr_fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ unsigned long long pr_add2_rd(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("add.rm.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

// Two pairs (i, j) and (i, j+1) from the packed j tile: their bin coordinates
// x, x + kPrMagic rounded down (whose bits are kPrMagicBits + floor(x)), and
// whether each is within delta of a bin edge.
struct PrTwo {
  float xa, xb, ta, tb;
  bool edge_a, edge_b;
};
__device__ __forceinline__ PrTwo pr_two(unsigned long long fx2, unsigned long long fy2, unsigned long long fz2,
                                        const float4& xy, const float2& zz, unsigned long long magic2,
                                        unsigned long long half2, float near_edge) {
  const unsigned long long dx = pr_sub2(fx2, pr_pack(xy.x, xy.y));
  const unsigned long long dy = pr_sub2(fy2, pr_pack(xy.z, xy.w));
  const unsigned long long dz = pr_sub2(fz2, pr_pack(zz.x, zz.y));
  const unsigned long long d2 = pr_fma2(dx, dx, pr_fma2(dy, dy, pr_mul2(dz, dz)));
  float d2a, d2b;
  pr_unpack(d2, d2a, d2b);
  PrTwo r;
  r.xa = pr_sqrt_approx(d2a);
  r.xb = pr_sqrt_approx(d2b);
  const unsigned long long x2 = pr_pack(r.xa, r.xb);
  const unsigned long long t2 = pr_add2_rd(x2, magic2);
  const unsigned long long c2 = pr_sub2(pr_sub2(x2, pr_sub2(t2, magic2)), half2);  // frac - 0.5
  float ca, cb;
  pr_unpack(t2, r.ta, r.tb);
  pr_unpack(c2, ca, cb);
  r.edge_a = fabsf(ca) > near_edge;
  r.edge_b = fabsf(cb) > near_edge;
  return r;
}

template <int kMode>
struct PrAcc {
  unsigned* c;  // kPrCounts
  double* w;    // weighted modes
  __device__ __forceinline__ void add(int e, double wij) const {
    if constexpr (kMode == kPrCounts) atomicAdd(&c[e], 1u);
    else atomicAdd(&w[e], wij);
  }
};

// Shared layout: kPrCounts: edges[bins + 1] (f64), then copies x u32[bins];
// kPrWeighted: edges, then copies x f64[bins]; kPrWeightedGlobal: no dynamic
// shared memory (edges and the block's row in device memory).
template <int kMode>
__global__ void __launch_bounds__(kPrThreads, 8)
    k_pr_hist(const double4* __restrict__ pos, const float4* __restrict__ pos32, const int2* __restrict__ tiles,
              int n_tiles, int n_types, int64_t chunk, const double* __restrict__ edges,
              const PrParams* __restrict__ par, int bins, int copies, unsigned long long* __restrict__ counts,
              double* __restrict__ rows) {
  extern __shared__ double pr_dyn[];
  __shared__ double4 sj[kPrThreads];
  __shared__ float4 sj32[kPrThreads];
  // the j tile in bins as pairs of atoms: {x_j, x_j+1, y_j, y_j+1} and {z_j, z_j+1}
  __shared__ float4 sjp[kPrThreads / 2];
  __shared__ float2 sjz[kPrThreads / 2];
  if (par->degenerate) return;
  const float inv_step = par->inv_step;
  // a pair is near an edge when its fractional bin coordinate is within delta
  // of 0 or 1: |frac - 0.5| > 0.5 - delta (always, when delta is FLT_MAX)
  const float near_edge = 0.5f - par->delta;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int si = lane * 4 + warp;  // this thread's slot in the i tile
  const double* E = kMode == kPrWeightedGlobal ? edges : pr_dyn;
  unsigned* Hc = reinterpret_cast<unsigned*>(pr_dyn + bins + 1);
  double* Hw = kMode == kPrWeightedGlobal ? rows + (size_t)blockIdx.x * bins : pr_dyn + bins + 1;
  if constexpr (kMode != kPrWeightedGlobal) {
    for (int k = threadIdx.x; k <= bins; k += kPrThreads) pr_dyn[k] = edges[k];
    if constexpr (kMode == kPrCounts)
      for (int k = threadIdx.x; k < copies * bins; k += kPrThreads) Hc[k] = 0u;
    else
      for (int k = threadIdx.x; k < copies * bins; k += kPrThreads) Hw[k] = 0.0;
  }
  PrAcc<kMode> acc;
  acc.c = Hc + (size_t)(warp % copies) * bins;
  acc.w = kMode == kPrWeightedGlobal ? Hw : Hw + (size_t)(warp % copies) * bins;
  const int top = kPrMagicBits + bins - 1;  // floor(x) capped at bins - 1, in magic bits
  // shared address of this warp's counter 0 less 4 * kPrMagicBits (32-bit
  // wrap-around), so that adding 4 * (kPrMagicBits + k) gives counter k
  const unsigned cbase =
      kMode == kPrCounts ? (unsigned)__cvta_generic_to_shared(acc.c) - ((unsigned)kPrMagicBits << 2) : 0u;

  const int64_t n_work = (int64_t)n_tiles * (n_tiles + 1) / 2;
  int64_t w = (int64_t)blockIdx.x * chunk;
  const int64_t w_end = min(w + chunk, n_work);
  int a = 0, b = 0;
  if (w < w_end) pr_tri_decode(w, a, b);
  int cur_b = -1, cur_pair = -1, since = 0;

  auto flush_counts = [&]() {
    __syncthreads();
    for (int k = threadIdx.x; k < bins; k += kPrThreads) {
      unsigned long long sum = 0ull;
      for (int c = 0; c < copies; ++c) {
        unsigned* h = Hc + (size_t)c * bins;
        sum += h[k];
        h[k] = 0u;
      }
      if (sum) atomicAdd(&counts[(size_t)cur_pair * bins + k], sum);
    }
    __syncthreads();
  };

  for (; w < w_end; ++w) {
    const int2 ta = tiles[a], tb = tiles[b];
    if constexpr (kMode == kPrCounts) {
      const int pair = pr_pair_index(ta.x, tb.x, n_types);
      if (pair != cur_pair || since == kPrFlushItems) {
        if (cur_pair >= 0) flush_counts();
        cur_pair = pair;
        since = 0;
      }
      ++since;
    }
    if (b != cur_b) {
      __syncthreads();
      if ((int)threadIdx.x < tb.y) {
        const int64_t g = (int64_t)b * kPrThreads + threadIdx.x;
        const float4 f = pos32[g];
        sj[threadIdx.x] = pos[g];
        const float4 fs = make_float4(f.x * inv_step, f.y * inv_step, f.z * inv_step, 0.0f);
        sj32[threadIdx.x] = fs;
        float* xy = reinterpret_cast<float*>(&sjp[threadIdx.x >> 1]);
        float* z = reinterpret_cast<float*>(&sjz[threadIdx.x >> 1]);
        const int h = threadIdx.x & 1;
        xy[h] = fs.x;
        xy[2 + h] = fs.y;
        z[h] = fs.z;
      }
      __syncthreads();
      cur_b = b;
    }
    if (si < ta.y) {
      const int64_t gi = (int64_t)a * kPrThreads + si;
      float4 fi = pos32[gi];
      fi = make_float4(fi.x * inv_step, fi.y * inv_step, fi.z * inv_step, 0.0f);
      double wi = 0.0;
      if constexpr (kMode != kPrCounts) wi = pos[gi].w;
      if (a != b && tb.y == kPrThreads) {
        // full off-diagonal tile: 32 pairs per chunk without branches, two
        // pairs per packed instruction; pairs near an edge are marked and
        // placed exactly after the chunk
        const unsigned long long fx2 = pr_pack(fi.x, fi.x), fy2 = pr_pack(fi.y, fi.y), fz2 = pr_pack(fi.z, fi.z);
        const unsigned long long magic2 = pr_pack(kPrMagic, kPrMagic), half2 = pr_pack(0.5f, 0.5f);
#pragma unroll 1
        for (int jc = 0; jc < kPrThreads; jc += 32) {
          unsigned marked = 0u;
#pragma unroll
          for (int jj = 0; jj < 32; jj += 2) {
            const PrTwo r = pr_two(fx2, fy2, fz2, sjp[(jc + jj) >> 1], sjz[(jc + jj) >> 1], magic2, half2, near_edge);
            marked |= ((r.edge_a ? 1u : 0u) | (r.edge_b ? 2u : 0u)) << jj;
            if constexpr (kMode == kPrCounts) {
              // t's bits are kPrMagicBits + floor(x): the counter's shared address
              // comes from one shift and add on the offset base
              const unsigned addr_a = cbase + ((unsigned)min(__float_as_int(r.ta), top) << 2);
              const unsigned addr_b = cbase + ((unsigned)min(__float_as_int(r.tb), top) << 2);
              if (!r.edge_a) asm volatile("red.shared.add.u32 [%0], 1;" ::"r"(addr_a) : "memory");
              if (!r.edge_b) asm volatile("red.shared.add.u32 [%0], 1;" ::"r"(addr_b) : "memory");
            } else {
              if (!r.edge_a) acc.add(min(__float_as_int(r.ta), top) - kPrMagicBits, wi * sj[jc + jj].w);
              if (!r.edge_b) acc.add(min(__float_as_int(r.tb), top) - kPrMagicBits, wi * sj[jc + jj + 1].w);
            }
          }
          while (marked) {
            const int j = jc + __ffs(marked) - 1;
            marked &= marked - 1u;
            const double4 pj = sj[j];
            acc.add(pr_exact_bin(pos[gi], pj, pr_bin_coord(fi, sj32[j]), E, bins), wi * pj.w);
          }
        }
      } else {
        for (int j = (a == b) ? si + 1 : 0; j < tb.y; ++j) {
          const float x = pr_bin_coord(fi, sj32[j]);
          const float t = __fadd_rd(x, kPrMagic);
          const float frac = x - (t - kPrMagic);
          const double4 pj = sj[j];
          int e;
          if (fabsf(frac - 0.5f) > near_edge) e = pr_exact_bin(pos[gi], pj, x, E, bins);
          else e = min(__float_as_int(t), top) - kPrMagicBits;
          acc.add(e, wi * pj.w);
        }
      }
    }
    if (++a > b) {
      a = 0;
      ++b;
    }
  }
  if constexpr (kMode == kPrCounts) {
    if (cur_pair >= 0) flush_counts();
  } else if constexpr (kMode == kPrWeighted) {
    __syncthreads();
    for (int k = threadIdx.x; k < bins; k += kPrThreads) {
      double sum = 0.0;
      for (int c = 0; c < copies; ++c) sum += Hw[(size_t)c * bins + k];
      rows[(size_t)blockIdx.x * bins + k] = sum;
    }
  }
}

// hist[k] = Σ_pairs counts[pair][k] * wprod[pair], pairs in order.
__global__ void k_pr_combine(const unsigned long long* __restrict__ counts, const double* __restrict__ wprod,
                             int n_pairs, int bins, const PrParams* __restrict__ par, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= bins) return;
  double s = 0.0;
  if (!par->degenerate)
    for (int p = 0; p < n_pairs; ++p) s += (double)counts[(size_t)p * bins + k] * wprod[p];
  out[k] = s;
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

template <int kMode>
int pr_blocks_per_sm(size_t dyn) {
  if (dyn) CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_pr_hist<kMode>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
  int per_sm = 0;
  CRAB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pr_hist<kMode>, kPrThreads, dyn));
  return std::max(per_sm, 1);
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
  ctx->last_pr_mode = -1;
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
  trace_mark("pr.lower_bound");

  // weight classes: distinct weight values (bit patterns), when there are few
  std::vector<int32_t> type(n, 0);
  std::vector<double> class_w;
  {
    // open addressing over the weight bit patterns; the table holds at most
    // kPrMaxClasses + 1 keys, so it never fills
    constexpr int kSlots = 256;
    uint64_t keys[kSlots];
    int ids[kSlots];
    std::fill(ids, ids + kSlots, -1);
    for (int64_t i = 0; i < n && (int)class_w.size() <= kPrMaxClasses; ++i) {
      uint64_t key;
      std::memcpy(&key, &w[i], sizeof key);
      uint32_t h = (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 56);
      while (ids[h] >= 0 && keys[h] != key) h = (h + 1) & (kSlots - 1);
      if (ids[h] < 0) {
        keys[h] = key;
        ids[h] = (int)class_w.size();
        class_w.push_back(w[i]);
      }
      type[i] = ids[h];
    }
  }
  const int T = (int)class_w.size();
  trace_mark("pr.classes");
  const int n_pairs = T * (T + 1) / 2;
  const size_t edge_bytes = (size_t)(bins + 1) * sizeof(double);
  int mode = kPrWeightedGlobal, copies = 1;
  if (T <= kPrMaxClasses && (size_t)n_pairs * bins * 8 <= kPrMaxCountBytes &&
      edge_bytes + (size_t)bins * 4 <= kPrDynSmem) {
    mode = kPrCounts;
    copies = (int)std::min<size_t>(kPrThreads / 32, (kPrDynSmem - edge_bytes) / ((size_t)bins * 4));
  } else if (edge_bytes + (size_t)bins * 8 <= kPrDynSmem) {
    mode = kPrWeighted;
    copies = (int)std::min<size_t>(kPrThreads / 32, (kPrDynSmem - edge_bytes) / ((size_t)bins * 8));
  }
  if (mode != kPrCounts) std::fill(type.begin(), type.end(), 0);
  Layout L;
  {
    TraceScope t2("pr.layout");
    L = build_layout(xyz, w, type.data(), n, mode == kPrCounts ? T : 1, false, true);
  }
  const int n_tiles = L.n_tiles;
  const int64_t n_pad = L.n_pad;
  double radius = 0.0;  // of the centred FP32 coordinates
  cudaStream_t s = ctx->stream;
  auto* h_pos = (double4*)ctx->host("pr.pos", (size_t)n_pad * sizeof(double4));
  auto* h_sph = (double4*)ctx->host("pr.sphere", (size_t)n_tiles * sizeof(double4));
  auto* h_tiles = (int2*)ctx->host("pr.tiles", (size_t)n_tiles * sizeof(int2));
  for (int64_t k = 0; k < n_pad; ++k) {
    const int64_t src = L.source[k];
    h_pos[k] = src >= 0 ? make_double4(xyz[3 * src], xyz[3 * src + 1], xyz[3 * src + 2], w[src])
                        : make_double4(0.0, 0.0, 0.0, 0.0);
    if (src >= 0) {
      const float* f = &L.atoms[4 * k];
      radius = std::max(radius, std::sqrt((double)f[0] * f[0] + (double)f[1] * f[1] + (double)f[2] * f[2]));
    }
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
    h_tiles[t] = make_int2(L.tile_type[t], cnt);
  }
  radius = radius * (1.0 + 1e-6) + 1e-30;
  trace_mark("pr.pack");

  auto* d_pos = (double4*)ctx->dev("pr.pos", (size_t)n_pad * sizeof(double4));
  auto* d_pos32 = (float4*)ctx->dev("pr.pos32", (size_t)n_pad * sizeof(float4));
  auto* d_sph = (double4*)ctx->dev("pr.sphere", (size_t)n_tiles * sizeof(double4));
  auto* d_tiles = (int2*)ctx->dev("pr.tiles", (size_t)n_tiles * sizeof(int2));
  auto* d_edges = (double*)ctx->dev("pr.edges", edge_bytes);
  auto* d_out = (double*)ctx->dev("pr.out", (size_t)bins * sizeof(double));
  // the dmax bits, PrParams and the class-pair weight products share one buffer
  auto* d_misc = (char*)ctx->dev("pr.misc", 64 + (size_t)n_pairs * sizeof(double));
  auto* d_dmax2 = (unsigned long long*)d_misc;
  auto* d_par = (PrParams*)(d_misc + 16);
  auto* d_wprod = (double*)(d_misc + 64);
  copy_h2d(ctx, d_pos, h_pos, (size_t)n_pad * sizeof(double4), s);
  copy_h2d(ctx, d_pos32, L.atoms.data(), (size_t)n_pad * sizeof(float4), s);
  copy_h2d(ctx, d_sph, h_sph, (size_t)n_tiles * sizeof(double4), s);
  copy_h2d(ctx, d_tiles, h_tiles, (size_t)n_tiles * sizeof(int2), s);
  CRAB_CUDA_CHECK(cudaMemsetAsync(d_misc, 0, 64, s));
  if (mode == kPrCounts) {
    auto* h_wprod = (double*)ctx->host("pr.wprod", (size_t)n_pairs * sizeof(double));
    for (int a = 0; a < T; ++a)
      for (int b = a; b < T; ++b) h_wprod[pair_index(a, b, T)] = class_w[a] * class_w[b];
    copy_h2d(ctx, d_wprod, h_wprod, (size_t)n_pairs * sizeof(double), s);
  }

  trace_mark("pr.upload");
  const int ibins = (int)bins;
  size_t dyn = 0;
  int per_sm = 1;
  if (mode == kPrCounts) {
    dyn = edge_bytes + (size_t)copies * bins * 4;
    per_sm = pr_blocks_per_sm<kPrCounts>(dyn);
  } else if (mode == kPrWeighted) {
    dyn = edge_bytes + (size_t)copies * bins * 8;
    per_sm = pr_blocks_per_sm<kPrWeighted>(dyn);
  } else {
    per_sm = pr_blocks_per_sm<kPrWeightedGlobal>(0);
  }
  const int64_t n_work = (int64_t)n_tiles * (n_tiles + 1) / 2;
  // weighted modes keep one f64 row per block: at most 256 MB of rows
  const int64_t max_rows = mode == kPrCounts ? INT64_MAX : std::max<int64_t>(1, (int64_t)(256u << 20) / (bins * 8));
  const int64_t grid0 = std::max<int64_t>(1, std::min({(int64_t)ctx->sm_count * per_sm, n_work, max_rows}));
  const int64_t chunk = (n_work + grid0 - 1) / grid0;
  const int grid = (int)((n_work + chunk - 1) / chunk);
  unsigned long long* d_counts = nullptr;
  double* d_rows = nullptr;
  if (mode == kPrCounts) {
    d_counts = (unsigned long long*)ctx->dev("pr.counts", (size_t)n_pairs * bins * 8);
    CRAB_CUDA_CHECK(cudaMemsetAsync(d_counts, 0, (size_t)n_pairs * bins * 8, s));
  } else {
    d_rows = (double*)ctx->dev("pr.rows", (size_t)grid * bins * 8);
    if (mode == kPrWeightedGlobal) CRAB_CUDA_CHECK(cudaMemsetAsync(d_rows, 0, (size_t)grid * bins * 8, s));
  }

  cudaEvent_t ev[3];
  for (auto& e : ev) CRAB_CUDA_CHECK(cudaEventCreate(&e));
  CRAB_CUDA_CHECK(cudaEventRecord(ev[0], s));
  int dgrid = 0;
  CRAB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&dgrid, k_pr_dmax, kPrThreads, 0));
  dgrid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)ctx->sm_count * std::max(dgrid, 1), n_work));
  k_pr_dmax<<<dgrid, kPrThreads, 0, s>>>(d_pos, d_tiles, n_tiles, d_sph, lower, d_dmax2);
  CRAB_CUDA_CHECK(cudaGetLastError());
  k_pr_edges<<<(unsigned)((bins + 1 + 127) / 128), 128, 0, s>>>(d_dmax2, bins, radius, d_edges, d_par);
  CRAB_CUDA_CHECK(cudaGetLastError());
  CRAB_CUDA_CHECK(cudaEventRecord(ev[1], s));
  if (mode == kPrCounts)
    k_pr_hist<kPrCounts><<<grid, kPrThreads, dyn, s>>>(d_pos, d_pos32, d_tiles, n_tiles, T, chunk, d_edges, d_par,
                                                        ibins, copies, d_counts, nullptr);
  else if (mode == kPrWeighted)
    k_pr_hist<kPrWeighted><<<grid, kPrThreads, dyn, s>>>(d_pos, d_pos32, d_tiles, n_tiles, 1, chunk, d_edges, d_par,
                                                          ibins, copies, nullptr, d_rows);
  else
    k_pr_hist<kPrWeightedGlobal><<<grid, kPrThreads, 0, s>>>(d_pos, d_pos32, d_tiles, n_tiles, 1, chunk, d_edges,
                                                              d_par, ibins, 1, nullptr, d_rows);
  CRAB_CUDA_CHECK(cudaGetLastError());
  CRAB_CUDA_CHECK(cudaEventRecord(ev[2], s));
  if (mode == kPrCounts)
    k_pr_combine<<<(ibins + 127) / 128, 128, 0, s>>>(d_counts, d_wprod, n_pairs, ibins, d_par, d_out);
  else
    k_pr_reduce<<<(ibins + 127) / 128, 128, 0, s>>>(d_rows, grid, ibins, d_par, d_out);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 4;
  auto* h_misc = (char*)ctx->host("pr.misc", 64);
  copy_d2h(ctx, h_misc, d_misc, 64, s);
  copy_d2h(ctx, hist, d_out, (size_t)bins * sizeof(double), s);
  trace_mark("pr.launch");
  CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
  trace_mark("pr.device");
  float t_all = 0.f, t_hist = 0.f;
  CRAB_CUDA_CHECK(cudaEventElapsedTime(&t_hist, ev[1], ev[2]));
  CRAB_CUDA_CHECK(cudaEventElapsedTime(&t_all, ev[0], ev[2]));
  for (auto& e : ev) cudaEventDestroy(e);
  ctx->last_pr_ms = t_all;
  ctx->last_pr_hist_ms = t_hist;
  ctx->last_pr_mode = mode;
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
  // the form factor at q = 0 once per (element, group); occupancy scales it as
  // form_factor_for_atom does (formfactor.rs:425-439)
  std::vector<double> w(n);
  double ff0[CRAB_EL_OTHER + 1][15];
  bool have[CRAB_EL_OTHER + 1][15] = {};
  for (int64_t i = 0; i < n; ++i) {
    const int el = st->elem[i], g = st->group[i] + 1;
    if (!have[el][g]) {
      ff0[el][g] = form_factor(el, g - 1, 1.0, true, 0.0);
      have[el][g] = true;
    }
    const double f = (el == CRAB_EL_H) ? 0.0 : st->occ[i] * ff0[el][g];
    w[i] = std::fmax(std::fabs(f), 1e-6);
  }
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

int crab_pr_last_timing(crab_ctx* ctx, double* total_ms, double* histogram_ms, double* pairs, int32_t* mode) {
  if (!ctx) return CRAB_EINVAL;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (total_ms) *total_ms = ctx->last_pr_ms;
  if (histogram_ms) *histogram_ms = ctx->last_pr_hist_ms;
  if (pairs) *pairs = ctx->last_pr_pairs;
  if (mode) *mode = ctx->last_pr_mode;
  return CRAB_OK;
}

}  // extern "C"
