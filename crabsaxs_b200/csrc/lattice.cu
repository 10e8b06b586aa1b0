// Exact site–site Debye sums for hydration sites on a voxel lattice.
//
// Hydration sites (crabSAXS src/solvent.rs:208-218, 387-396) are voxel
// centres min + (ix, iy, iz)·spacing, so every site pair is at distance
// spacing·√n with n = Δix² + Δiy² + Δiz² an integer.  The reference sums
// sinc(q r) over all site pairs (solvent.rs:563-570).  Here the pairs are
// counted per n in integer arithmetic (a histogram over all M(M-1)/2 pairs,
// shared-memory atomics), and the sum becomes Σ_n count[n]·sinc(q·spacing·√n)
// evaluated in f64 for the few thousand distinct n.  The result is exact up
// to f64 rounding (the reference's own r differs from spacing·√n by ~1e-15
// relative), and it avoids the coherent FP32 errors a lattice would
// otherwise accumulate: thousands of pairs share each distance.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "engine.hpp"

namespace crab {
namespace {

constexpr int kLT = 128;           // sites per tile
constexpr int kSharedBins = 11264; // 44 KB of u32 counters (+2 KB tile: under the 48 KB static limit)

__global__ void __launch_bounds__(kLT)
    k_lattice_hist(const int4* __restrict__ cells, int64_t m, int n_tiles, int bins, unsigned long long* __restrict__ hist) {
  __shared__ int4 sj[kLT];
  __shared__ unsigned int sh[kSharedBins];
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (tj < ti) return;  // upper triangle of tile pairs only
  const bool shared_hist = bins <= kSharedBins;
  if (shared_hist)
    for (int b = threadIdx.x; b < bins; b += kLT) sh[b] = 0u;
  const int64_t j_global = (int64_t)tj * kLT + threadIdx.x;
  sj[threadIdx.x] = j_global < m ? cells[j_global] : make_int4(0, 0, 0, -1);
  __syncthreads();
  const int64_t i = (int64_t)ti * kLT + threadIdx.x;
  if (i < m) {
    const int4 ci = cells[i];
    for (int j = 0; j < kLT; ++j) {
      const int4 cj = sj[j];
      if (cj.w < 0) break;  // past the last site
      if (ti == tj && j <= (int)threadIdx.x) continue;
      const int dx = ci.x - cj.x, dy = ci.y - cj.y, dz = ci.z - cj.z;
      const int n = dx * dx + dy * dy + dz * dz;
      if (shared_hist) atomicAdd(&sh[n], 1u);
      else atomicAdd(&hist[n], 1ull);
    }
  }
  if (shared_hist) {
    __syncthreads();
    for (int b = threadIdx.x; b < bins; b += kLT)
      if (sh[b]) atomicAdd(&hist[b], (unsigned long long)sh[b]);
  }
}

// out[k] = Σ_n count[n] sinc(q_k spacing √n) with the reference sinc
// (|x| < 1e-8 -> 1), one CTA per q.
__global__ void k_lattice_transform(const unsigned long long* __restrict__ hist, int bins, double spacing,
                                    const double* __restrict__ q, double* __restrict__ out) {
  __shared__ double red[32];
  const double qq = q[blockIdx.x];
  double acc = 0.0;
  for (int n = threadIdx.x; n < bins; n += blockDim.x) {
    const unsigned long long c = hist[n];
    if (!c) continue;
    const double x = qq * (spacing * sqrt((double)n));
    acc += (double)c * (fabs(x) < 1e-8 ? 1.0 : sin(x) / x);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) out[blockIdx.x] = v;
  }
}

}  // namespace

void lattice_plan_init(crab_ctx* ctx, PairPlan& P, const int32_t* cells, int64_t m, double spacing) {
  LatticePart& Lp = P.lattice;
  Lp.m = m;
  Lp.spacing = spacing;
  if (m < 2) {
    Lp.bins = 1;
  } else {
    int lo[3] = {cells[0], cells[1], cells[2]}, hi[3] = {cells[0], cells[1], cells[2]};
    for (int64_t i = 1; i < m; ++i)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], cells[3 * i + d]);
        hi[d] = std::max(hi[d], cells[3 * i + d]);
      }
    int64_t nmax = 0;
    for (int d = 0; d < 3; ++d) nmax += (int64_t)(hi[d] - lo[d]) * (hi[d] - lo[d]);
    require(nmax < (int64_t)1 << 30, "hydration lattice too large for the site histogram");
    require((m + kLT - 1) / kLT <= 65535, "too many lattice sites for one histogram launch");
    Lp.bins = (int)nmax + 1;
  }
  std::vector<int4> c4(std::max<int64_t>(m, 1));
  for (int64_t i = 0; i < m; ++i) c4[i] = make_int4(cells[3 * i], cells[3 * i + 1], cells[3 * i + 2], 0);
  Lp.d_cells = (int4*)plan_alloc(ctx, P, P.owned, "lattice_cells", c4.size() * sizeof(int4));
  copy_h2d(ctx, Lp.d_cells, c4.data(), (size_t)m * sizeof(int4), ctx->stream);
  Lp.d_hist = (unsigned long long*)plan_alloc(ctx, P, P.owned, "lattice_hist",
                                               (size_t)Lp.bins * sizeof(unsigned long long));
  Lp.d_out = (double*)plan_alloc(ctx, P, P.owned, "lattice_out", (size_t)std::max<int64_t>(P.nq, 1) * sizeof(double));
  if (!P.d_q) {
    P.d_q = (double*)plan_alloc(ctx, P, P.owned, "lattice_q", (size_t)std::max<int64_t>(P.nq, 1) * sizeof(double));
    copy_h2d(ctx, P.d_q, P.q.data(), (size_t)P.nq * sizeof(double), ctx->stream);
  }
  Lp.active = true;
}

void lattice_plan_launch(crab_ctx* ctx, PairPlan& P, cudaStream_t s) {
  LatticePart& Lp = P.lattice;
  if (!Lp.active || P.nq == 0) return;
  CRAB_CUDA_CHECK(cudaMemsetAsync(Lp.d_hist, 0, (size_t)Lp.bins * sizeof(unsigned long long), s));
  if (Lp.m >= 2) {
    const int nt = (int)((Lp.m + kLT - 1) / kLT);
    k_lattice_hist<<<dim3(nt, nt), kLT, 0, s>>>(Lp.d_cells, Lp.m, nt, Lp.bins, Lp.d_hist);
    CRAB_CUDA_CHECK(cudaGetLastError());
    ctx->launches += 1;
  }
  k_lattice_transform<<<(unsigned)P.nq, 256, 0, s>>>(Lp.d_hist, Lp.bins, Lp.spacing, P.d_q, Lp.d_out);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 1;
}

}  // namespace crab
