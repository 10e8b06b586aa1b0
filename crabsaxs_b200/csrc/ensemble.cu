// Batched ensemble scoring (crabSAXS src/ensemble.rs:127-465 and
// src/reweight.rs:84-374 on the device).
//
// The reference's EnsembleFitter::fit_core computes, for each of the 25
// (c1, c2) candidates, a full compute_curve of every conformer (ensemble.rs:
// 244-261): 25·K O(N²·Nq) sums.  c1 and c2 only enter through the amplitude
// recombination, so here:
//   1. one persistent launch of the pair kernel over the work items of every
//      conformer (a batch plan, longest items first across conformers of
//      uneven size) produces each conformer's per-type-pair partials once;
//   2. k_ens_curves recombines them into the curve of every (candidate,
//      conformer) pair;
//   3. k_ens_weights runs, one CTA per candidate, the projected-gradient
//      simplex fit of ensemble.rs:317-381 (250 iterations, bitonic sort for
//      the simplex projection of ensemble.rs:449-465);
//   4. k_ens_reweight picks the best candidate, returns ∂χ²/∂(c1, c2) at its
//      weights, and runs the maximum-entropy mirror descent of
//      reweight.rs:84-154 from a uniform prior.
// Steps 1-4 are captured once in a CUDA graph and replayed.

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <random>

#include "engine.hpp"
#include "ops.hpp"

namespace crab {
namespace {

constexpr int kEW = 256;  // threads of the weight kernels
constexpr int kMaxK = 1024;

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return t;
}

__device__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = -INFINITY;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
  __syncthreads();
  return t;
}

// curves[cand][k][p] from raw partials [c][ab][p] (Σ w w sin(q r)/r) and the
// per-candidate amplitude tables amp[cand][t][p] (Â_t = V - G E + c2 H).
__global__ void k_ens_curves(const double* __restrict__ raw, const int* __restrict__ sel, const double* __restrict__ q,
                             int nq, int T, const double* __restrict__ amp, const double* __restrict__ self_w2,
                             const double* __restrict__ sum_w, int K, double* __restrict__ curves) {
  const int k = blockIdx.x, cand = blockIdx.y;
  const int c = sel[k];
  const int NP = T * (T + 1) / 2;
  const double* Pc = raw + (size_t)c * NP * nq;
  const double* A = amp + (size_t)cand * T * nq;
  for (int p = threadIdx.x; p < nq; p += blockDim.x) {
    const double qq = q[p];
    double I = 0.0;
    for (int a = 0; a < T; ++a) {
      const double Aa = A[(size_t)a * nq + p];
      I += Aa * Aa * self_w2[(size_t)c * T + a];
      for (int b = a; b < T; ++b) {
        const int ab = a * T - a * (a - 1) / 2 + (b - a);
        double Pv;
        if (qq == 0.0) {
          const double sa = sum_w[(size_t)c * T + a], sb = sum_w[(size_t)c * T + b];
          Pv = (a == b) ? 0.5 * (sa * sa - self_w2[(size_t)c * T + a]) : sa * sb;
        } else {
          Pv = Pc[(size_t)ab * nq + p] / qq;
        }
        I += 2.0 * Aa * A[(size_t)b * nq + p] * Pv;
      }
    }
    curves[((size_t)cand * K + k) * nq + p] = fmax(I, 0.0);
  }
}

struct EnsOpts {
  int scale_mode, bg_mode;
  double scale_value, bg_value;
  int uniform;
  double regularization;
};

// ensemble.rs:383-434 on the mixture in smem.
__device__ void solve_fixed(const double* mix, const double* y, const double* sg, int nq, const EnsOpts& o, double* red,
                            double* s_out, double* b_out, double* chi_out) {
  double num = 0.0, den = 0.0;
  for (int p = threadIdx.x; p < nq; p += blockDim.x) {
    const double w = 1.0 / (sg[p] * sg[p]);
    num += mix[p] * y[p] * w;
    den += mix[p] * mix[p] * w;
  }
  num = block_sum(num, red);
  den = block_sum(den, red);
  double scale = o.scale_mode == CRAB_SCALE_FIT ? (den > 0.0 ? num / den : 0.0) : o.scale_value;
  scale = fmax(scale, 0.0);
  double bg = 0.0;
  if (o.bg_mode == CRAB_BG_FIT) {
    double n2 = 0.0, d2 = 0.0;
    for (int p = threadIdx.x; p < nq; p += blockDim.x) {
      const double w = 1.0 / (sg[p] * sg[p]);
      n2 += (y[p] - scale * mix[p]) * w;
      d2 += w;
    }
    n2 = block_sum(n2, red);
    d2 = block_sum(d2, red);
    bg = d2 > 0.0 ? n2 / d2 : 0.0;
  } else if (o.bg_mode == CRAB_BG_FIXED) {
    bg = o.bg_value;
  }
  double chi = 0.0;
  for (int p = threadIdx.x; p < nq; p += blockDim.x) {
    const double r = (scale * mix[p] + bg - y[p]) / sg[p];
    chi += r * r;
  }
  chi = block_sum(chi, red);
  *s_out = scale;
  *b_out = bg;
  *chi_out = chi / (double)max(nq - 1, 1);
}

// Descending bitonic sort of n (power of two) values in smem.
__device__ void bitonic_desc(double* v, int n) {
  for (int size = 2; size <= n; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool desc = (i & size) == 0;
          const double a = v[i], b = v[j];
          if (desc ? (a < b) : (a > b)) {
            v[i] = b;
            v[j] = a;
          }
        }
      }
      __syncthreads();
    }
}

// ensemble.rs:449-465: out = max(v - θ, 0) with θ from the sorted prefix.
__device__ void project_simplex_dev(const double* v, double* out, int K, double* sorted, int n2) {
  for (int i = threadIdx.x; i < n2; i += blockDim.x) sorted[i] = i < K ? v[i] : -INFINITY;
  __syncthreads();
  bitonic_desc(sorted, n2);
  __shared__ double theta;
  if (threadIdx.x == 0) {
    double cumulative = 0.0;
    int rho = 0;
    for (int i = 0; i < K; ++i) {
      cumulative += sorted[i];
      if (sorted[i] + (1.0 - cumulative) / (double)(i + 1) > 0.0) rho = i + 1;
    }
    double top = 0.0;
    for (int i = 0; i < rho; ++i) top += sorted[i];
    theta = (top - 1.0) / (double)max(rho, 1);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < K; i += blockDim.x) out[i] = fmax(v[i] - theta, 0.0);
  __syncthreads();
}

// One CTA per candidate: ensemble.rs:317-381.
__global__ void __launch_bounds__(kEW)
    k_ens_weights(const double* __restrict__ curves, int K, int nq, const double* __restrict__ y,
                  const double* __restrict__ sg, EnsOpts o, double* __restrict__ weights, double* __restrict__ fit,
                  double* __restrict__ fitted, double* __restrict__ grad_w) {
  extern __shared__ double sm[];
  double* w = sm;               // K
  double* g = w + K;            // K
  double* prop = g + K;         // K
  double* mix = prop + K;       // nq
  double* res = mix + nq;       // nq
  int n2 = 1;
  while (n2 < K) n2 <<= 1;
  double* sorted = res + nq;    // n2
  __shared__ double red[32];
  const int cand = blockIdx.x;
  const double* cv = curves + (size_t)cand * K * nq;
  for (int k = threadIdx.x; k < K; k += blockDim.x) w[k] = 1.0 / (double)K;
  __syncthreads();
  double s, b, chi;
  const int iters = o.uniform ? 0 : 250;
  for (int it = 0; it < iters; ++it) {
    for (int p = threadIdx.x; p < nq; p += blockDim.x) {
      double m = 0.0;
      for (int k = 0; k < K; ++k) m += cv[(size_t)k * nq + p] * w[k];
      mix[p] = m;
    }
    __syncthreads();
    solve_fixed(mix, y, sg, nq, o, red, &s, &b, &chi);
    for (int p = threadIdx.x; p < nq; p += blockDim.x) res[p] = (s * mix[p] + b - y[p]) / sg[p];
    __syncthreads();
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
      double acc = 0.0;
      for (int p = 0; p < nq; ++p) acc += res[p] * s * cv[(size_t)k * nq + p] / sg[p];
      g[k] = 2.0 * acc + 2.0 * o.regularization * (w[k] - 1.0 / (double)K);
    }
    __syncthreads();
    double nrm = 0.0;
    for (int k = threadIdx.x; k < K; k += blockDim.x) nrm += g[k] * g[k];
    nrm = fmax(sqrt(block_sum(nrm, red)), 1.0);
    for (int k = threadIdx.x; k < K; k += blockDim.x) prop[k] = w[k] - 0.05 * g[k] / nrm;
    __syncthreads();
    project_simplex_dev(prop, prop, K, sorted, n2);
    double delta = 0.0;
    for (int k = threadIdx.x; k < K; k += blockDim.x) delta += fabs(prop[k] - w[k]);
    delta = block_sum(delta, red);
    for (int k = threadIdx.x; k < K; k += blockDim.x) w[k] = prop[k];
    __syncthreads();
    if (delta < 1e-8) break;
  }
  for (int p = threadIdx.x; p < nq; p += blockDim.x) {
    double m = 0.0;
    for (int k = 0; k < K; ++k) m += cv[(size_t)k * nq + p] * w[k];
    mix[p] = m;
  }
  __syncthreads();
  solve_fixed(mix, y, sg, nq, o, red, &s, &b, &chi);
  for (int p = threadIdx.x; p < nq; p += blockDim.x) {
    fitted[(size_t)cand * nq + p] = s * mix[p] + b;
    res[p] = (s * mix[p] + b - y[p]) / sg[p];
  }
  __syncthreads();
  // ∂χ²_red/∂w_k at the final weights (scale and background held)
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    double acc = 0.0;
    for (int p = 0; p < nq; ++p) acc += res[p] * s * cv[(size_t)k * nq + p] / sg[p];
    grad_w[(size_t)cand * K + k] = 2.0 * acc / (double)max(nq - 1, 1);
    weights[(size_t)cand * K + k] = w[k];
  }
  if (threadIdx.x == 0) {
    fit[4 * cand] = s;
    fit[4 * cand + 1] = b;
    fit[4 * cand + 2] = chi;
    fit[4 * cand + 3] = (double)iters;
  }
}

struct RwOpts {
  double kl, step, tol, floor;
  int max_iter, scale_mode, bg_mode;
  double scale_value, bg_value;
};

// reweight.rs:236-301 on the mixture mix[p] (scale, background, reduced χ²).
__device__ void rw_solve(const double* mix, int nq, const double* y, const double* sg, const RwOpts& o, double* red,
                         double* s_out, double* b_out, double* chi_out) {
  double sw = 0, sx = 0, sy = 0, sxx = 0, sxy = 0;
  for (int p = threadIdx.x; p < nq; p += blockDim.x) {
    const double ww = 1.0 / (sg[p] * sg[p]);
    sw += ww;
    sx += ww * mix[p];
    sy += ww * y[p];
    sxx += ww * mix[p] * mix[p];
    sxy += ww * mix[p] * y[p];
  }
  sw = block_sum(sw, red);
  sx = block_sum(sx, red);
  sy = block_sum(sy, red);
  sxx = block_sum(sxx, red);
  sxy = block_sum(sxy, red);
  double s, b;
  auto fscale = [&](double bb) { return sxx > 0.0 ? fmax((sxy - bb * sx) / sxx, 0.0) : 0.0; };
  auto fbg = [&](double ss) { return sw > 0.0 ? (sy - ss * sx) / sw : 0.0; };
  if (o.scale_mode == CRAB_SCALE_FIXED) {
    s = fmax(o.scale_value, 0.0);
    b = o.bg_mode == CRAB_BG_FIXED ? o.bg_value : (o.bg_mode == CRAB_BG_FIXED_ZERO ? 0.0 : fbg(s));
  } else if (o.bg_mode == CRAB_BG_FIXED) {
    s = fscale(o.bg_value);
    b = o.bg_value;
  } else if (o.bg_mode == CRAB_BG_FIXED_ZERO) {
    s = fscale(0.0);
    b = 0.0;
  } else {
    const double det = sxx * sw - sx * sx;
    s = fabs(det) > 1e-20 ? fmax((sxy * sw - sx * sy) / det, 0.0) : 0.0;
    b = fbg(s);
  }
  double chi = 0.0;
  for (int p = threadIdx.x; p < nq; p += blockDim.x) {
    const double r = (s * mix[p] + b - y[p]) / sg[p];
    chi += r * r;
  }
  chi = block_sum(chi, red);
  *s_out = s;
  *b_out = b;
  *chi_out = chi / (double)max(nq - 1, 1);
}

// ---- KL reweighting over a cluster of kRwCluster CTAs ----------------------
// reweight.rs:84-154 on the best candidate's K curves.  CTA r of the cluster
// keeps rows [r kr, (r+1) kr) of those curves (kr = ceil(K / kRwCluster)) in
// its shared memory, with their weights, gradients and proposals; the
// mixture and every sum or maximum over K are exchanged through distributed
// shared memory: each CTA publishes its partial, one cluster barrier, and
// every CTA adds the partials of all ranks in rank order, so every CTA holds
// the same values and takes the same branches.  Exchange buffers alternate
// between two halves, so the barrier of one exchange also releases the
// buffer of the exchange before it.
constexpr int kRwCluster = 8;
namespace cg = cooperative_groups;

struct RwCluster {
  cg::cluster_group cl;
  double* xs;  // [2] scalar partial
  double* pm;  // [2][3 nq] array partials
  double* red;
  int nq, par;
  __device__ double sum(double v) {
    v = block_sum(v, red);
    if (threadIdx.x == 0) xs[par] = v;
    cl.sync();
    double t = 0.0;
    for (int r = 0; r < kRwCluster; ++r) t += *cl.map_shared_rank(&xs[par], r);
    par ^= 1;
    return t;
  }
  __device__ double max(double v) {
    v = block_max(v, red);
    if (threadIdx.x == 0) xs[par] = v;
    cl.sync();
    double t = -INFINITY;
    for (int r = 0; r < kRwCluster; ++r) t = fmax(t, *cl.map_shared_rank(&xs[par], r));
    par ^= 1;
    return t;
  }
  // out[i] = sum over ranks of the published part[i], i < n (n <= 3 nq); part
  // is written by this CTA into pm[par] by the caller's loop before the call
  __device__ double* slot() { return pm + (size_t)par * 3 * nq; }
  __device__ void sum_array(double* out, int n) {
    __syncthreads();
    cl.sync();
    double* mine = slot();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double t = 0.0;
      for (int r = 0; r < kRwCluster; ++r) t += cl.map_shared_rank(mine, r)[i];
      out[i] = t;
    }
    par ^= 1;
    __syncthreads();
  }
};

// The mixture Σ_k w_k I_k(q) over the cluster's rows, then reweight.rs:236-301.
__device__ void rw_fit_cl(RwCluster& X, const double* cvr, const double* w, int nk, int nq, const double* y,
                          const double* sg, const RwOpts& o, double* mix, double* s_out, double* b_out,
                          double* chi_out) {
  double* part = X.slot();
  for (int p = threadIdx.x; p < nq; p += blockDim.x) {
    double m = 0.0;
    for (int k = 0; k < nk; ++k) m += cvr[(size_t)k * nq + p] * w[k];
    part[p] = m;
  }
  X.sum_array(mix, nq);
  rw_solve(mix, nq, y, sg, o, X.red, s_out, b_out, chi_out);
}
__device__ double kl_div_cl(RwCluster& X, const double* w, int nk, double prior) {
  double s = 0.0;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) s += w[k] * log(w[k] / prior);
  return X.sum(s);
}
__device__ void apply_floor_cl(RwCluster& X, double* w, int nk, int K, double floor) {
  double sum = 0.0;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) sum += w[k];
  sum = fmax(X.sum(sum), 1e-300);
  const double residual = 1.0 - floor * (double)K;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) w[k] = floor <= 0.0 ? w[k] / sum : floor + residual * w[k] / sum;
  __syncthreads();
}

// Shared memory of one cluster CTA for K curves of nq points: weights,
// gradients and proposals of its rows, the mixture, the exchange buffers and,
// when they fit, its rows of the curves.
__host__ __device__ inline int rw_rows(int K) { return (K + kRwCluster - 1) / kRwCluster; }
__host__ __device__ inline bool rw_rows_on_chip(int K, int nq) {
  return (size_t)rw_rows(K) * (size_t)nq * sizeof(double) <= 128 * 1024;
}
__host__ __device__ inline size_t rw_smem(int K, int nq) {
  const size_t kr = (size_t)rw_rows(K);
  return (3 * kr + (size_t)nq + 6 * (size_t)nq + 2 + (rw_rows_on_chip(K, nq) ? kr * (size_t)nq : 0)) * sizeof(double);
}

// Best candidate, ∂χ²/∂(c1, c2) there, then reweight.rs:84-154.
// out: [0] best candidate, [1] scale, [2] bg, [3] reduced chi2, [4] KL,
// [5] iterations, [6] converged, [7] dchi/dc1, [8] dchi/dc2.
__global__ void __cluster_dims__(kRwCluster, 1, 1) __launch_bounds__(kEW)
    k_ens_reweight(const double* __restrict__ curves, const double* __restrict__ fitc, int n_cand, int K, int nq,
                   const double* __restrict__ y, const double* __restrict__ sg, const double* __restrict__ weights,
                   const double* __restrict__ dcurves, RwOpts o, double* __restrict__ w_out,
                   double* __restrict__ out) {
  extern __shared__ double sm[];
  __shared__ double red[32];
  __shared__ int best;
  RwCluster X{cg::this_cluster(), nullptr, nullptr, red, nq, 0};
  const int rank = (int)X.cl.block_rank();
  const int kr = rw_rows(K), k0 = min(K, rank * kr), nk = min(K, k0 + kr) - k0;
  double* w = sm;              // kr
  double* g = w + kr;          // kr
  double* pr = g + kr;         // kr
  double* mix = pr + kr;       // nq
  X.pm = mix + nq;             // 2 x 3 nq
  X.xs = X.pm + 6 * (size_t)nq;  // 2
  double* cvs = X.xs + 2;      // kr x nq, when the rows fit
  if (threadIdx.x == 0) {
    best = 0;
    for (int c = 1; c < n_cand; ++c)
      if (fitc[4 * c + 2] < fitc[4 * best + 2]) best = c;
  }
  __syncthreads();
  const double* cvg = curves + ((size_t)best * K + k0) * nq;  // this CTA's rows
  const double* cvr = cvg;
  if (rw_rows_on_chip(K, nq)) {
    for (size_t i = threadIdx.x; i < (size_t)nk * nq; i += blockDim.x) cvs[i] = cvg[i];
    cvr = cvs;
  }
  __syncthreads();
  // ∂χ²/∂c1 and ∂χ²/∂c2 at the best candidate's weights, scale and background
  {
    const double s = fitc[4 * best], b = fitc[4 * best + 1];
    const double* wb = weights + (size_t)best * K + k0;
    const double* d1c = dcurves + ((size_t)(2 * best) * K + k0) * nq;
    const double* d2c = dcurves + ((size_t)(2 * best + 1) * K + k0) * nq;
    double* part = X.slot();
    for (int p = threadIdx.x; p < nq; p += blockDim.x) {
      double m = 0.0, d1 = 0.0, d2 = 0.0;
      for (int k = 0; k < nk; ++k) {
        m += cvr[(size_t)k * nq + p] * wb[k];
        d1 += d1c[(size_t)k * nq + p] * wb[k];
        d2 += d2c[(size_t)k * nq + p] * wb[k];
      }
      part[p] = m;
      part[nq + p] = d1;
      part[2 * nq + p] = d2;
    }
    // the sums land in this CTA's other exchange half: no peer reads it
    // before the next array exchange, which comes after their last use here
    double* sums = X.pm + (size_t)(X.par ^ 1) * 3 * nq;
    X.sum_array(sums, 3 * nq);
    double g1 = 0.0, g2 = 0.0;
    for (int p = threadIdx.x; p < nq; p += blockDim.x) {
      const double wgt = 2.0 * (s * sums[p] + b - y[p]) / (sg[p] * sg[p]) / (double)max(nq - 1, 1) * s;
      g1 += wgt * sums[nq + p];
      g2 += wgt * sums[2 * nq + p];
    }
    g1 = block_sum(g1, red);
    g2 = block_sum(g2, red);
    if (rank == 0 && threadIdx.x == 0) {
      out[7] = g1;
      out[8] = g2;
    }
    __syncthreads();
  }
  const double prior = 1.0 / (double)K;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) w[k] = prior;
  __syncthreads();
  apply_floor_cl(X, w, nk, K, o.floor);
  int iterations = 0, converged = 0;
  const double dof = (double)max(nq - 1, 1);
  double s, b, chi;
  for (int it = 0; it < o.max_iter; ++it) {
    iterations = it + 1;
    rw_fit_cl(X, cvr, w, nk, nq, y, sg, o, mix, &s, &b, &chi);
    for (int k = threadIdx.x; k < nk; k += blockDim.x) {
      double dg = 0.0;
      for (int p = 0; p < nq; ++p)
        dg += 2.0 * ((s * mix[p] + b) - y[p]) * s * cvr[(size_t)k * nq + p] / (sg[p] * sg[p]) / dof;
      g[k] = dg + o.kl * (log(w[k] / prior) + 1.0);
    }
    __syncthreads();
    double gmax = 0.0;
    for (int k = threadIdx.x; k < nk; k += blockDim.x) gmax = fmax(gmax, fabs(g[k]));
    gmax = fmax(X.max(gmax), 1e-12);
    double step = o.step / gmax;
    const double objective = chi + o.kl * kl_div_cl(X, w, nk, prior);
    bool accepted = false;
    for (int h = 0; h < 14 && !accepted; ++h) {
      double mx = -INFINITY;
      for (int k = threadIdx.x; k < nk; k += blockDim.x) {
        pr[k] = log(fmax(w[k], 1e-300)) - step * g[k];
        mx = fmax(mx, pr[k]);
      }
      mx = X.max(mx);
      for (int k = threadIdx.x; k < nk; k += blockDim.x) pr[k] = exp(pr[k] - mx);
      __syncthreads();
      double sum = 0.0;
      for (int k = threadIdx.x; k < nk; k += blockDim.x) sum += pr[k];
      sum = fmax(X.sum(sum), 1e-300);
      for (int k = threadIdx.x; k < nk; k += blockDim.x) pr[k] /= sum;
      __syncthreads();
      apply_floor_cl(X, pr, nk, K, o.floor);
      double s2, b2, chi2;
      rw_fit_cl(X, cvr, pr, nk, nq, y, sg, o, mix, &s2, &b2, &chi2);
      if (chi2 + o.kl * kl_div_cl(X, pr, nk, prior) <= objective + 1e-12) accepted = true;
      else step *= 0.5;
    }
    if (!accepted) break;
    double delta = 0.0;
    for (int k = threadIdx.x; k < nk; k += blockDim.x) delta += fabs(pr[k] - w[k]);
    delta = X.sum(delta);
    for (int k = threadIdx.x; k < nk; k += blockDim.x) w[k] = pr[k];
    __syncthreads();
    if (delta <= o.tol) {
      converged = 1;
      break;
    }
  }
  rw_fit_cl(X, cvr, w, nk, nq, y, sg, o, mix, &s, &b, &chi);
  const double kl = kl_div_cl(X, w, nk, prior);
  for (int k = threadIdx.x; k < nk; k += blockDim.x) w_out[k0 + k] = w[k];
  if (rank == 0 && threadIdx.x == 0) {
    out[0] = best;
    out[1] = s;
    out[2] = b;
    out[3] = chi;
    out[4] = kl;
    out[5] = iterations;
    out[6] = converged;
  }
  X.cl.sync();  // no CTA leaves while a peer may still read its shared memory
}

// Derivative curves dI/dc1 and dI/dc2 of every conformer at every candidate:
// dcurves[2*cand + m][k][p] (m = 0: c1, 1: c2) from dÂ tables damp.
__global__ void k_ens_dcurves(const double* __restrict__ raw, const int* __restrict__ sel,
                              const double* __restrict__ q, int nq, int T, const double* __restrict__ amp,
                              const double* __restrict__ damp, const double* __restrict__ self_w2,
                              const double* __restrict__ sum_w, int K, const double* __restrict__ curves,
                              double* __restrict__ dcurves) {
  const int k = blockIdx.x, cm = blockIdx.y, cand = cm >> 1;
  const int c = sel[k];
  const int NP = T * (T + 1) / 2;
  const double* Pc = raw + (size_t)c * NP * nq;
  const double* A = amp + (size_t)cand * T * nq;
  const double* dA = damp + (size_t)cm * T * nq;
  for (int p = threadIdx.x; p < nq; p += blockDim.x) {
    const double qq = q[p];
    double d = 0.0;
    for (int a = 0; a < T; ++a) {
      const double Aa = A[(size_t)a * nq + p], dAa = dA[(size_t)a * nq + p];
      d += 2.0 * Aa * dAa * self_w2[(size_t)c * T + a];
      for (int b = a; b < T; ++b) {
        const int ab = a * T - a * (a - 1) / 2 + (b - a);
        double Pv;
        if (qq == 0.0) {
          const double sa = sum_w[(size_t)c * T + a], sb = sum_w[(size_t)c * T + b];
          Pv = (a == b) ? 0.5 * (sa * sa - self_w2[(size_t)c * T + a]) : sa * sb;
        } else {
          Pv = Pc[(size_t)ab * nq + p] / qq;
        }
        d += 2.0 * (dAa * A[(size_t)b * nq + p] + Aa * dA[(size_t)b * nq + p]) * Pv;
      }
    }
    // the clamp at zero has no derivative
    dcurves[((size_t)cm * K + k) * nq + p] = curves[((size_t)cand * K + k) * nq + p] > 0.0 ? d : 0.0;
  }
}

}  // namespace

// ------------------------------------------------------------------ host side

struct EnsemblePlan {
  crab_ctx* ctx = nullptr;
  int K = 0, T = 0, n_cand = 0;
  int64_t nq = 0;
  std::vector<double> q, cand;
  std::vector<AtomClass> classes;
  bool implicit = true;
  crab_solvent solvent{};
  std::unique_ptr<PairPlan> pair;
  std::vector<double> self_w2, sum_w;  // [K][T]
  std::vector<double> amp, damp;       // [n_cand][T][nq], [2 n_cand][T][nq]
  std::vector<void*> owned;
  double* d_partials = nullptr;  // raw pair sums [K][T(T+1)/2][nq]: the pair plan's output, or uploaded
  double *d_q = nullptr, *d_amp = nullptr, *d_damp = nullptr, *d_self = nullptr, *d_sumw = nullptr;
  double *d_curves = nullptr, *d_dcurves = nullptr;
  int* d_sel = nullptr;
  // fit state
  double *d_y = nullptr, *d_sg = nullptr, *d_weights = nullptr, *d_fit = nullptr, *d_fitted = nullptr,
         *d_gradw = nullptr, *d_wkl = nullptr, *d_out = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_k = -1;
  int64_t graph_kernels = 0;
  ~EnsemblePlan() {
    if (graph) cudaGraphExecDestroy(graph);
    for (void* p : owned) cudaFree(p);
  }
  template <class T_>
  T_* alloc(size_t n) {
    void* p = nullptr;
    CRAB_CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T_)));
    owned.push_back(p);
    return (T_*)p;
  }
};

// Scattering classes of the whole ensemble (sorted) and their type indices:
// every conformer uses the same types.
static std::map<AtomClass, int> ensemble_class_index(crab_struct* const* sts, int K, bool implicit) {
  std::map<AtomClass, int> index;
  for (int c = 0; c < K; ++c) {
    require(sts[c] && sts[c]->n > 0, "ensemble must contain non-empty conformers");
    for (int64_t i = 0; i < sts[c]->n; ++i)
      index[AtomClass{sts[c]->elem[i], implicit ? (int)sts[c]->group[i] : -1}] = 0;
  }
  int T = 0;
  for (auto& kv : index) kv.second = T++;
  return index;
}

static std::vector<int32_t> conformer_types(const crab_struct* st, const std::map<AtomClass, int>& index,
                                            bool implicit) {
  std::vector<int32_t> type(st->n);
  for (int64_t i = 0; i < st->n; ++i) type[i] = index.at(AtomClass{st->elem[i], implicit ? (int)st->group[i] : -1});
  return type;
}

// Doubles per conformer in a gathered partials buffer: the raw pair sums
// [T(T+1)/2][nq], then Σw² and Σw per type.
static size_t partials_block(int T, int64_t nq) { return (size_t)(T * (T + 1) / 2) * nq + 2 * (size_t)T; }

// With `given` (a gathered buffer of K partials blocks) the pair sums are
// uploaded instead of computed, and no pair plan is built.
static std::unique_ptr<EnsemblePlan> make_ensemble_plan(crab_ctx* ctx, crab_struct* const* sts, int K, const double* q,
                                                        int64_t nq, const crab_solvent& s, bool implicit,
                                                        const double* cand, int n_cand,
                                                        const double* given = nullptr) {
  require(K > 0 && K <= kMaxK, "ensemble size must be between 1 and 1024");
  require(n_cand > 0, "at least one (c1, c2) candidate");
  require(s.hydration_model == CRAB_HYD_ANALYTIC, "the batched ensemble covers the analytic hydration model");
  for (int c = 0; c < n_cand; ++c)
    require(std::isfinite(cand[2 * c]) && cand[2 * c] > 0.0 && std::isfinite(cand[2 * c + 1]),
            "candidate c1 must be finite and positive, c2 finite");
  std::unique_ptr<EnsemblePlan> E(new EnsemblePlan());
  E->ctx = ctx;
  E->K = K;
  E->nq = nq;
  E->n_cand = n_cand;
  E->q.assign(q, q + nq);
  E->cand.assign(cand, cand + 2 * n_cand);
  E->implicit = implicit;
  E->solvent = s;
  // shared scattering types over the whole ensemble
  const std::map<AtomClass, int> index = ensemble_class_index(sts, K, implicit);
  for (const auto& kv : index) E->classes.push_back(kv.first);
  const int T = (int)index.size();
  E->T = T;
  E->self_w2.assign((size_t)K * T, 0.0);
  E->sum_w.assign((size_t)K * T, 0.0);
  if (!given) {
    std::vector<Layout> parts;
    for (int c = 0; c < K; ++c) {
      const crab_struct* st = sts[c];
      const std::vector<int32_t> type = conformer_types(st, index, implicit);
      parts.push_back(build_layout(st->xyz.data(), st->occ.data(), type.data(), st->n, T, false));
      for (int a = 0; a < T; ++a) {
        E->self_w2[(size_t)c * T + a] = parts.back().self_w2[a];
        E->sum_w[(size_t)c * T + a] = parts.back().sum_w[a];
      }
    }
    E->pair = make_batch_pair_plan(ctx, std::move(parts), q, nq);
    E->d_partials = E->pair->d_out;
  } else {
    const size_t P = (size_t)(T * (T + 1) / 2), block = partials_block(T, nq);
    std::vector<double> raw((size_t)K * P * nq);
    for (int c = 0; c < K; ++c) {
      const double* b = given + (size_t)c * block;
      std::copy(b, b + P * nq, raw.begin() + (size_t)c * P * nq);
      for (int a = 0; a < T; ++a) {
        E->self_w2[(size_t)c * T + a] = b[P * nq + a];
        E->sum_w[(size_t)c * T + a] = b[P * nq + T + a];
      }
    }
    E->d_partials = E->alloc<double>(raw.size());
    copy_h2d(ctx, E->d_partials, raw.data(), raw.size() * sizeof(double), ctx->stream);
  }
  // amplitude tables per candidate and their c1/c2 derivatives
  E->amp.assign((size_t)n_cand * T * nq, 0.0);
  E->damp.assign((size_t)2 * n_cand * T * nq, 0.0);
  for (int a = 0; a < T; ++a)
    for (int64_t p = 0; p < nq; ++p) {
      double v, e, h;
      debye_class_amplitudes(E->classes[a], implicit, q[p], s.bulk_density, s.shell_thickness, &v, &e, &h);
      for (int c = 0; c < n_cand; ++c) {
        const double c1 = cand[2 * c], c2 = cand[2 * c + 1];
        const double G = excluded_volume_scale(q[p], c1);
        const double dG = G * (3.0 / c1 - 2.0 * c1 * (1.62 * 1.62) * q[p] * q[p] / 4.0);
        E->amp[((size_t)c * T + a) * nq + p] = v - G * e + c2 * h;
        E->damp[((size_t)(2 * c) * T + a) * nq + p] = -dG * e;
        E->damp[((size_t)(2 * c + 1) * T + a) * nq + p] = h;
      }
    }
  cudaStream_t sm = ctx->stream;
  E->d_q = E->alloc<double>(nq);
  E->d_amp = E->alloc<double>(E->amp.size());
  E->d_damp = E->alloc<double>(E->damp.size());
  E->d_self = E->alloc<double>(E->self_w2.size());
  E->d_sumw = E->alloc<double>(E->sum_w.size());
  E->d_sel = E->alloc<int>(K);
  E->d_curves = E->alloc<double>((size_t)n_cand * K * nq);
  E->d_dcurves = E->alloc<double>((size_t)2 * n_cand * K * nq);
  copy_h2d(ctx, E->d_q, q, nq * sizeof(double), sm);
  copy_h2d(ctx, E->d_amp, E->amp.data(), E->amp.size() * sizeof(double), sm);
  copy_h2d(ctx, E->d_damp, E->damp.data(), E->damp.size() * sizeof(double), sm);
  copy_h2d(ctx, E->d_self, E->self_w2.data(), E->self_w2.size() * sizeof(double), sm);
  copy_h2d(ctx, E->d_sumw, E->sum_w.data(), E->sum_w.size() * sizeof(double), sm);
  std::vector<int> all(K);
  std::iota(all.begin(), all.end(), 0);
  copy_h2d(ctx, E->d_sel, all.data(), K * sizeof(int), sm);
  CRAB_CUDA_CHECK(cudaStreamSynchronize(sm));
  return E;
}

static void ensemble_launch_curves(EnsemblePlan& E, int Ksel) {
  crab_ctx* ctx = E.ctx;
  k_ens_curves<<<dim3(Ksel, E.n_cand), 128, 0, ctx->stream>>>(E.d_partials, E.d_sel, E.d_q, (int)E.nq, E.T, E.d_amp,
                                                             E.d_self, E.d_sumw, Ksel, E.d_curves);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 1;
}

static size_t weights_smem(int K, int64_t nq) {
  int n2 = 1;
  while (n2 < K) n2 <<= 1;
  return (size_t)(3 * K + 2 * nq + n2) * sizeof(double);
}

static void ensemble_fit_buffers(EnsemblePlan& E, const double* y, const double* sg) {
  crab_ctx* ctx = E.ctx;
  // shared-memory opt-in for the largest subset, done before any graph capture
  const size_t shm = weights_smem(E.K, E.nq), shr = rw_smem(E.K, (int)E.nq);
  require(shm <= 200 * 1024 && shr <= 200 * 1024, "ensemble too large for the on-chip weight fit");
  CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_ens_weights, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(shm, 48 * 1024)));
  CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_ens_reweight, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(shr, 48 * 1024)));
  if (!E.d_y) {
    E.d_y = E.alloc<double>(E.nq);
    E.d_sg = E.alloc<double>(E.nq);
    E.d_weights = E.alloc<double>((size_t)E.n_cand * E.K);
    E.d_gradw = E.alloc<double>((size_t)E.n_cand * E.K);
    E.d_fit = E.alloc<double>((size_t)4 * E.n_cand);
    E.d_fitted = E.alloc<double>((size_t)E.n_cand * E.nq);
    E.d_wkl = E.alloc<double>(E.K);
    E.d_out = E.alloc<double>(16);
  }
  copy_h2d(ctx, E.d_y, y, E.nq * sizeof(double), ctx->stream);
  copy_h2d(ctx, E.d_sg, sg, E.nq * sizeof(double), ctx->stream);
}

// fit_core (ensemble.rs:234-299) on the selected conformers, all on the device.
static void ensemble_launch_fit(EnsemblePlan& E, int Ksel, const EnsOpts& eo, const RwOpts* ro) {
  crab_ctx* ctx = E.ctx;
  cudaStream_t sm = ctx->stream;
  ensemble_launch_curves(E, Ksel);
  const size_t shm = weights_smem(Ksel, E.nq);
  k_ens_weights<<<E.n_cand, kEW, shm, sm>>>(E.d_curves, Ksel, (int)E.nq, E.d_y, E.d_sg, eo, E.d_weights, E.d_fit,
                                            E.d_fitted, E.d_gradw);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 1;
  if (ro) {
    k_ens_dcurves<<<dim3(Ksel, 2 * E.n_cand), 128, 0, sm>>>(E.d_partials, E.d_sel, E.d_q, (int)E.nq, E.T, E.d_amp,
                                                           E.d_damp, E.d_self, E.d_sumw, Ksel, E.d_curves,
                                                           E.d_dcurves);
    CRAB_CUDA_CHECK(cudaGetLastError());
    const size_t shr = rw_smem(Ksel, (int)E.nq);
    k_ens_reweight<<<kRwCluster, kEW, shr, sm>>>(E.d_curves, E.d_fit, E.n_cand, Ksel, (int)E.nq, E.d_y, E.d_sg,
                                                 E.d_weights, E.d_dcurves, *ro, E.d_wkl, E.d_out);
    CRAB_CUDA_CHECK(cudaGetLastError());
    ctx->launches += 2;
  }
}

// The full scoring pass of a plan as one CUDA graph: pair sums of every
// conformer, curves at every candidate, weight fits, ∂χ²/∂(c1,c2), KL
// reweighting.  Captured on first use and replayed.
static void ensemble_graph_launch(EnsemblePlan& E, const EnsOpts& eo, const RwOpts& ro) {
  crab_ctx* ctx = E.ctx;
  if (!E.graph || E.graph_k != E.K) {
    if (E.graph) {
      cudaGraphExecDestroy(E.graph);
      E.graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    const int64_t before = ctx->launches;
    CRAB_CUDA_CHECK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    try {
      if (E.pair) pair_plan_launch(ctx, *E.pair, ctx->stream, false);
      ensemble_launch_fit(E, E.K, eo, &ro);
    } catch (...) {
      cudaStreamEndCapture(ctx->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CRAB_CUDA_CHECK(cudaStreamEndCapture(ctx->stream, &g));
    CRAB_CUDA_CHECK(cudaGraphInstantiate(&E.graph, g, 0));
    cudaGraphDestroy(g);
    E.graph_k = E.K;
    E.graph_kernels = ctx->launches - before;  // kernels recorded into the graph
    ctx->launches = before;
  }
  CRAB_CUDA_CHECK(cudaGraphLaunch(E.graph, ctx->stream));
  ctx->launches += E.graph_kernels;
}

static EnsOpts ens_opts(const crab_fit_options* fo, bool uniform, double reg) {
  EnsOpts o;
  o.scale_mode = fo ? fo->scale_mode : CRAB_SCALE_FIT;
  o.bg_mode = fo ? fo->bg_mode : CRAB_BG_FIT;
  o.scale_value = fo ? fo->scale_value : 0.0;
  o.bg_value = fo ? fo->bg_value : 0.0;
  o.uniform = uniform ? 1 : 0;
  o.regularization = reg;
  return o;
}

}  // namespace crab

using namespace crab;

struct crab_ensemble_plan {
  std::unique_ptr<crab::EnsemblePlan> plan;
};

extern "C" {

int crab_ensemble_curves(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q, int64_t nq,
                         const crab_solvent* solvent, int implicit_hydrogen, const double* cand, int32_t n_cand,
                         double* curves) {
  if (!ctx || !structures || k <= 0 || !q || nq <= 0 || !solvent || !cand || n_cand <= 0 || !curves)
    return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    validate_q(q, nq);
    validate_solvent(*solvent);
    auto E = make_ensemble_plan(ctx, structures, k, q, nq, *solvent, implicit_hydrogen != 0, cand, n_cand);
    pair_plan_launch(ctx, *E->pair, ctx->stream, false);
    ensemble_launch_curves(*E, k);
    copy_d2h(ctx, curves, E->d_curves, (size_t)n_cand * k * nq * sizeof(double), ctx->stream);
    CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  });
}

int crab_ensemble_plan_create(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q, int64_t nq,
                              const crab_solvent* solvent, int implicit_hydrogen, const double* cand, int32_t n_cand,
                              crab_ensemble_plan** out) {
  if (!ctx || !structures || k <= 0 || !q || nq <= 0 || !solvent || !cand || n_cand <= 0 || !out) return CRAB_EINVAL;
  *out = nullptr;
  return guarded_impl(ctx, [&]() {
    validate_q(q, nq);
    validate_solvent(*solvent);
    crab_ensemble_plan* p = new crab_ensemble_plan();
    p->plan = make_ensemble_plan(ctx, structures, k, q, nq, *solvent, implicit_hydrogen != 0, cand, n_cand);
    *out = p;
  });
}

int crab_ensemble_plan_autotune(crab_ctx* ctx, crab_ensemble_plan* plan, int32_t* chosen) {
  if (!ctx || !plan) return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    const int c = pair_plan_autotune(ctx, *plan->plan->pair, nullptr, nullptr, 0, nullptr);
    if (plan->plan->graph) {
      cudaGraphExecDestroy(plan->plan->graph);
      plan->plan->graph = nullptr;
    }
    if (chosen) *chosen = c;
  });
}

int crab_ensemble_plan_score(crab_ctx* ctx, crab_ensemble_plan* plan, const double* y, const double* sigma,
                             const crab_fit_options* fopt, const crab_reweight_options* ropt, double* elapsed_ms,
                             double* best_fit, double* weights, double* grad_w, double* kl_weights,
                             double* reweight_out) {
  if (!ctx || !plan || !y || !sigma) return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    EnsemblePlan& E = *plan->plan;
    for (int64_t p = 0; p < E.nq; ++p)
      require(std::isfinite(y[p]) && std::isfinite(sigma[p]) && sigma[p] > 0.0, "invalid experimental curve");
    ensemble_fit_buffers(E, y, sigma);
    const EnsOpts eo = ens_opts(fopt, false, 0.0);
    RwOpts ro{1.0, 0.5, 1e-8, 1e-10, 500, CRAB_SCALE_FIT, CRAB_BG_FIT, 0.0, 0.0};
    if (ropt) {
      ro = RwOpts{ropt->kl_strength, ropt->step_size, ropt->tolerance, ropt->min_weight, ropt->max_iterations,
                  ropt->scale_mode, ropt->bg_mode, ropt->scale_value, ropt->bg_value};
      require(ro.max_iter > 0 && ro.step > 0.0 && ro.tol > 0.0 && ro.floor >= 0.0 && ro.floor * E.K < 1.0 &&
                  ro.kl >= 0.0,
              "maximum-entropy options are invalid");
    }
    CRAB_CUDA_CHECK(cudaEventRecord(ctx->ev_start, ctx->stream));
    ensemble_graph_launch(E, eo, ro);
    CRAB_CUDA_CHECK(cudaEventRecord(ctx->ev_stop, ctx->stream));
    std::vector<double> fit((size_t)4 * E.n_cand), out(16);
    copy_d2h(ctx, fit.data(), E.d_fit, fit.size() * sizeof(double), ctx->stream);
    copy_d2h(ctx, out.data(), E.d_out, 9 * sizeof(double), ctx->stream);
    CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.0f;
    CRAB_CUDA_CHECK(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
    if (elapsed_ms) *elapsed_ms = ms;
    const int best = (int)out[0];
    if (best_fit) {
      best_fit[0] = best;
      best_fit[1] = E.cand[2 * best];
      best_fit[2] = E.cand[2 * best + 1];
      best_fit[3] = fit[4 * best];
      best_fit[4] = fit[4 * best + 1];
      best_fit[5] = fit[4 * best + 2];
      best_fit[6] = out[7];
      best_fit[7] = out[8];
    }
    if (weights) copy_d2h(ctx, weights, E.d_weights + (size_t)best * E.K, E.K * sizeof(double), ctx->stream);
    if (grad_w) copy_d2h(ctx, grad_w, E.d_gradw + (size_t)best * E.K, E.K * sizeof(double), ctx->stream);
    if (kl_weights) copy_d2h(ctx, kl_weights, E.d_wkl, E.K * sizeof(double), ctx->stream);
    if (reweight_out)
      for (int i = 0; i < 6; ++i) reweight_out[i] = out[1 + i];
    CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  });
}

int crab_ensemble_plan_destroy(crab_ensemble_plan* plan) {
  if (!plan) return CRAB_OK;
  if (plan->plan && plan->plan->ctx) cudaSetDevice(plan->plan->ctx->device);
  delete plan;
  return CRAB_OK;
}

}  // extern "C"

// ensemble.rs:302-315: the 5 x 5 (c1, c2) candidate grid.
static std::vector<double> fit_candidates(const crab_fit_options* fopt) {
  std::vector<double> cand;
  for (int i = 0; i < 5; ++i)
    for (int j = 0; j < 5; ++j) {
      cand.push_back(fopt->c1_lo + (fopt->c1_hi - fopt->c1_lo) * (double)i / 4.0);
      cand.push_back(fopt->c2_lo + (fopt->c2_hi - fopt->c2_lo) * (double)j / 4.0);
    }
  return cand;
}

static void check_ensemble_inputs(const crab_ensemble_options& eo, const double* y, const double* sigma, int64_t nq) {
  require(std::isfinite(eo.regularization) && eo.regularization >= 0.0 && std::isfinite(eo.min_weight) &&
              eo.min_weight >= 0.0 && eo.min_weight <= 1.0 && eo.max_conformers >= 0 && eo.bootstrap >= 0,
          "ensemble regularization and pruning options are invalid");
  for (int64_t p = 0; p < nq; ++p)
    require(std::isfinite(y[p]) && std::isfinite(sigma[p]) && sigma[p] > 0.0, "invalid experimental curve");
}

// EnsembleFitter::fit (ensemble.rs:127-232) once the pair sums are on the
// device: fit_core for every pruning round, the optional residual
// bootstrap, and the outputs.
static void ensemble_fit_rounds(crab_ctx* ctx, std::unique_ptr<EnsemblePlan>& E, const std::vector<double>& cand,
                                const double* y, const double* sigma, int64_t nq, const crab_ensemble_options& eo,
                                const crab_fit_options* fopt, crab_ensemble_result* result, int32_t* selected_out,
                                double* weights_out, double* fitted_out, double* intervals_out,
                                double* bootstrap_chi2_out) {
  ensemble_fit_buffers(*E, y, sigma);
  const EnsOpts o = ens_opts(fopt, eo.uniform || !eo.fit_weights, eo.regularization);
  struct Core {
    std::vector<double> w, fitted;
    double scale, bg, chi2, c1, c2;
  };
  auto fit_core = [&](const std::vector<int>& sel, const double* yy) {
    copy_h2d(ctx, E->d_sel, sel.data(), sel.size() * sizeof(int), ctx->stream);
    copy_h2d(ctx, E->d_y, yy, nq * sizeof(double), ctx->stream);
    ensemble_launch_fit(*E, (int)sel.size(), o, nullptr);
    std::vector<double> fit(4 * 25);
    copy_d2h(ctx, fit.data(), E->d_fit, fit.size() * sizeof(double), ctx->stream);
    CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    int best = 0;
    for (int c = 1; c < 25; ++c)
      if (fit[4 * c + 2] < fit[4 * best + 2]) best = c;
    Core core;
    core.w.resize(sel.size());
    core.fitted.resize(nq);
    copy_d2h(ctx, core.w.data(), E->d_weights + (size_t)best * sel.size(), sel.size() * sizeof(double), ctx->stream);
    copy_d2h(ctx, core.fitted.data(), E->d_fitted + (size_t)best * nq, nq * sizeof(double), ctx->stream);
    CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    core.scale = fit[4 * best];
    core.bg = fit[4 * best + 1];
    core.chi2 = fit[4 * best + 2];
    core.c1 = cand[2 * best];
    core.c2 = cand[2 * best + 1];
    return core;
  };
  std::vector<int> selected(E->K);
  std::iota(selected.begin(), selected.end(), 0);
  Core core = fit_core(selected, y);
  for (bool changed = true; changed;) {
    changed = false;
    std::vector<int> keep;
    for (size_t i = 0; i < selected.size(); ++i)
      if (core.w[i] + 1e-12 >= eo.min_weight) keep.push_back(selected[i]);
    if (keep.empty())
      keep.push_back(selected[std::max_element(core.w.begin(), core.w.end()) - core.w.begin()]);
    if (eo.max_conformers > 0 && (int)keep.size() > eo.max_conformers) {
      std::vector<std::pair<double, int>> ranked;
      for (size_t i = 0; i < selected.size(); ++i) ranked.push_back({core.w[i], selected[i]});
      std::stable_sort(ranked.begin(), ranked.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
      keep.clear();
      for (int i = 0; i < eo.max_conformers; ++i) keep.push_back(ranked[i].second);
    }
    std::sort(keep.begin(), keep.end());
    if (keep != selected) {
      selected = keep;
      core = fit_core(selected, y);
      changed = true;
    }
  }
  // weight intervals from a residual bootstrap (ensemble.rs:174-216); the
  // resampling indices come from a seeded std::mt19937_64 stream (the
  // reference draws them from ChaCha8, so individual replicates differ)
  const size_t ns = selected.size();
  std::vector<std::vector<double>> samples(ns);
  if (eo.bootstrap > 0) {
    std::mt19937_64 rng(eo.seed);
    std::vector<double> resid(nq), synth(nq);
    for (int64_t p = 0; p < nq; ++p) resid[p] = (y[p] - core.fitted[p]) / sigma[p];
    for (int b = 0; b < eo.bootstrap; ++b) {
      for (int64_t p = 0; p < nq; ++p) synth[p] = core.fitted[p] + resid[rng() % (uint64_t)nq] * sigma[p];
      Core rep = fit_core(selected, synth.data());
      for (size_t i = 0; i < ns; ++i) samples[i].push_back(rep.w[i]);
      if (bootstrap_chi2_out) bootstrap_chi2_out[b] = rep.chi2;
    }
    copy_h2d(ctx, E->d_y, y, nq * sizeof(double), ctx->stream);
  }
  if (intervals_out) {
    auto quantile = [](const std::vector<double>& v, double prob) {
      const double pos = std::min(std::max(prob, 0.0), 1.0) * (double)(v.size() - 1);
      const size_t lo = (size_t)std::floor(pos), hi = (size_t)std::ceil(pos);
      return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
    };
    for (size_t i = 0; i < ns; ++i) {
      if (eo.bootstrap > 0) {
        std::sort(samples[i].begin(), samples[i].end());
        intervals_out[3 * i] = quantile(samples[i], 0.5);
        intervals_out[3 * i + 1] = quantile(samples[i], 0.025);
        intervals_out[3 * i + 2] = quantile(samples[i], 0.975);
      } else {
        intervals_out[3 * i] = intervals_out[3 * i + 1] = intervals_out[3 * i + 2] = core.w[i];
      }
    }
  }
  const double dof = (double)std::max<int64_t>(nq - 1, 1);
  result->scale = core.scale;
  result->background = core.bg;
  result->c1 = core.c1;
  result->c2 = core.c2;
  result->reduced_chi2 = core.chi2;
  result->chi2 = core.chi2 * dof;
  result->iterations = 250;
  result->n_selected = (int)selected.size();
  if (selected_out)
    for (size_t i = 0; i < selected.size(); ++i) selected_out[i] = selected[i];
  if (weights_out) std::copy(core.w.begin(), core.w.end(), weights_out);
  if (fitted_out) std::copy(core.fitted.begin(), core.fitted.end(), fitted_out);
}

extern "C" {

// EnsembleFitter::fit (ensemble.rs:127-232): partials once, fit_core on the
// device for every pruning round, optional residual bootstrap.
int crab_ensemble_fit(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q, const double* y,
                      const double* sigma, int64_t nq, const crab_ensemble_options* eopt, const crab_fit_options* fopt,
                      crab_ensemble_result* result, int32_t* selected_out, double* weights_out, double* fitted_out,
                      double* intervals_out, double* bootstrap_chi2_out) {
  if (!ctx || !structures || k <= 0 || !q || !y || !sigma || nq <= 0 || !eopt || !fopt || !result) return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    validate_q(q, nq);
    validate_solvent(fopt->solvent);
    check_ensemble_inputs(*eopt, y, sigma, nq);
    const std::vector<double> cand = fit_candidates(fopt);
    auto E = make_ensemble_plan(ctx, structures, k, q, nq, fopt->solvent, fopt->implicit_hydrogen != 0, cand.data(), 25);
    pair_plan_launch(ctx, *E->pair, ctx->stream, false);
    ensemble_fit_rounds(ctx, E, cand, y, sigma, nq, *eopt, fopt, result, selected_out, weights_out, fitted_out,
                        intervals_out, bootstrap_chi2_out);
  });
}

int crab_ensemble_partials(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q, int64_t nq,
                           int implicit_hydrogen, int shard, int n_shards, int32_t* n_types, double* out,
                           int64_t capacity) {
  if (!ctx || !structures || k <= 0 || !q || nq <= 0 || !n_types || n_shards < 1 || shard < 0 || shard >= n_shards)
    return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    validate_q(q, nq);
    require(k <= kMaxK, "ensemble size must be between 1 and 1024");
    const bool implicit = implicit_hydrogen != 0;
    const std::map<AtomClass, int> index = ensemble_class_index(structures, k, implicit);
    const int T = (int)index.size();
    *n_types = T;
    if (!out) return;
    const size_t P = (size_t)(T * (T + 1) / 2), block = partials_block(T, nq);
    if (capacity < 0 || (uint64_t)capacity < block * (size_t)k) throw Error(CRAB_ECAPACITY, "partials buffer too small");
    std::fill(out, out + block * (size_t)k, 0.0);
    // conformers longest first by N², then the greedy owners
    std::vector<int> order(k);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return structures[a]->n > structures[b]->n; });
    std::vector<int64_t> cost(k);
    for (int i = 0; i < k; ++i) cost[i] = structures[order[i]]->n * structures[order[i]]->n;
    const std::vector<int32_t> owner = shard_owners(cost.data(), k, n_shards);
    std::vector<int> mine;
    for (int i = 0; i < k; ++i)
      if (owner[i] == shard) mine.push_back(order[i]);
    std::sort(mine.begin(), mine.end());
    if (mine.empty()) return;
    std::vector<Layout> parts;
    for (int c : mine) {
      const crab_struct* st = structures[c];
      const std::vector<int32_t> type = conformer_types(st, index, implicit);
      parts.push_back(build_layout(st->xyz.data(), st->occ.data(), type.data(), st->n, T, false));
      double* b = out + (size_t)c * block;
      for (int a = 0; a < T; ++a) {
        b[P * nq + a] = parts.back().self_w2[a];
        b[P * nq + T + a] = parts.back().sum_w[a];
      }
    }
    auto plan = make_batch_pair_plan(ctx, std::move(parts), q, nq);
    pair_plan_launch(ctx, *plan, ctx->stream, false);
    std::vector<double> raw(mine.size() * P * (size_t)nq);
    int status = 0;
    copy_d2h(ctx, raw.data(), plan->d_out, raw.size() * sizeof(double), ctx->stream);
    copy_d2h(ctx, &status, plan->d_status, sizeof(int), ctx->stream);
    CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    if (status) throw Error(status, "pair kernel: a bounded wait on a j-tile copy ran out");
    for (size_t i = 0; i < mine.size(); ++i)
      std::copy(raw.begin() + i * P * nq, raw.begin() + (i + 1) * P * nq, out + (size_t)mine[i] * block);
  });
}

int crab_ensemble_fit_partials(crab_ctx* ctx, crab_struct* const* structures, int32_t k, const double* q,
                               const double* y, const double* sigma, int64_t nq, const crab_ensemble_options* eopt,
                               const crab_fit_options* fopt, const double* partials, int32_t n_types,
                               crab_ensemble_result* result, int32_t* selected_out, double* weights_out,
                               double* fitted_out, double* intervals_out, double* bootstrap_chi2_out) {
  if (!ctx || !structures || k <= 0 || !q || !y || !sigma || nq <= 0 || !eopt || !fopt || !partials || !result)
    return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    validate_q(q, nq);
    validate_solvent(fopt->solvent);
    check_ensemble_inputs(*eopt, y, sigma, nq);
    require((int)ensemble_class_index(structures, k, fopt->implicit_hydrogen != 0).size() == n_types,
            "partials were computed for another set of atom types");
    const std::vector<double> cand = fit_candidates(fopt);
    auto E = make_ensemble_plan(ctx, structures, k, q, nq, fopt->solvent, fopt->implicit_hydrogen != 0, cand.data(), 25,
                                partials);
    ensemble_fit_rounds(ctx, E, cand, y, sigma, nq, *eopt, fopt, result, selected_out, weights_out, fitted_out,
                        intervals_out, bootstrap_chi2_out);
  });
}

}  // extern "C"
