// Adjoint gradient of the reduced χ² with respect to every atomic coordinate
// (new capability: the reference fit is derivative-free, crabSAXS
// src/fit.rs:401-418), plus the closed-form derivatives with respect to c1,
// c2, scale and background.
//
// Model (the reference's analytic-hydration Debye curve, solvent.rs:454-500
// and spherical.rs:567-584): I(q) = Σ_ij A_i A_j sinc(q r_ij) with
// A_i = occ_i Â_t(q), Â_t = V_t - G(q,c1) E_t + c2 H_t, and
// χ² = Σ_k ((s I_k + b - y_k)/σ_k)² / (Nq - 1) (fit.rs:185-196).  With
// w_k = ∂χ²/∂I_k = 2 s (s I_k + b - y_k) / σ_k² / (Nq-1):
//   ∂χ²/∂x_i = Σ_{j≠i} occ_i occ_j g_ab(r_ij) (x_i - x_j)/r_ij,
//   g_ab(r) = (1/r) Σ_k α_ab,k cos(q_k r) - (1/r²) Σ_k β_ab,k sin(q_k r),
//   α_ab,k = 2 w_k Â_a Â_b,  β_ab,k = α_ab,k / q_k.
// Since A_i depends only on the atom's type, the pair term depends only on
// the type pair and the distance:
//   ∂χ²/∂x_i = Σ_j occ_i occ_j h_ab(r_ij) (x_i - x_j),
//   h_ab(r) = g_ab(r) / r = Σ_k α_ab,k q_k² F(q_k r),  F(x) = (cos x - sin x / x) / x²,
// and F is smooth and even (F(0) = -1/3), so h_ab is a band-limited function
// of r (bandwidth q_max).  k_grad_h evaluates it in f64 on a uniform grid
// r_n = n δr, δr = 0.02 / q_max, up to the structure's largest pair distance;
// the pair kernel interpolates it with the 4-point Lagrange cubic (error below
// 4e-9 of max |h|, from (q_max δr)^4 × 0.0234), from one float4 of the four
// taps per grid cell.  Nothing O(N²) is stored: the table is O(T² × q_max × D).
// k_grad_pairs: one thread per atom i, j tiles staged in shared memory, every
// ordered pair (no cross-lane reductions); per (i tile, chunk of j tiles) an
// FP32 sum per j tile added into f64, and k_grad_reduce adds the chunks in a
// fixed order (deterministic).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "device_math.cuh"
#include "engine.hpp"
#include "ops.hpp"

namespace crab {
namespace {

using namespace dev;

constexpr int kGT = 128;

// F(x) = (cos x - sin x / x) / x² in f64: its series sum_{n>=1} (-1)^n 2n x^{2n-2} / (2n+1)!
// below 0.5 (ten terms: the next is below 1e-17 of F), the closed form above.
__device__ __forceinline__ double grad_F(double x) {
  if (x < 0.5) {
    const double x2 = x * x;
    double term = -1.0 / 3.0, sum = 0.0;  // n = 1
    for (int n = 1; n <= 10; ++n) {
      sum += term;
      // term_{n+1} / term_n = -x² (2n+2) / (2n) / ((2n+2)(2n+3)) = -x² / (2n (2n+3))
      term *= -x2 / ((double)(2 * n) * (double)(2 * n + 3));
    }
    return sum;
  }
  double sx, cx;
  sincos(x, &sx, &cx);
  return (cx - sx / x) / (x * x);
}

// h_ab(r_n) for n = 0 .. n_r + 2 (r_n = n dr) of every type pair: out[ab][n].
// One warp per grid point, the lanes over q, then a warp reduction (fixed order).
__global__ void k_grad_h(const double* __restrict__ alpha, const double* __restrict__ q, int nq, int n_pairs,
                         int n_r, double dr, double* __restrict__ out) {
  const int64_t idx = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t per = (int64_t)n_r + 3;
  if (idx >= per * n_pairs) return;  // uniform over the warp
  const int ab = (int)(idx / per), n = (int)(idx % per);
  const double r = n * dr;
  const double* al = alpha + (size_t)ab * nq;
  double h = 0.0;
  for (int k = lane; k < nq; k += 32) h += al[k] * q[k] * q[k] * grad_F(q[k] * r);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
  if (lane == 0) out[idx] = h;
}

// The four taps of cell n, h(r_{n-1}) .. h(r_{n+2}) (h is even: h(r_{-1}) = h(r_1)).
__global__ void k_grad_taps(const double* __restrict__ h, int n_pairs, int n_r, float4* __restrict__ taps) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)(n_r + 1) * n_pairs) return;
  const int ab = (int)(idx / (n_r + 1)), n = (int)(idx % (n_r + 1));
  const double* row = h + (size_t)ab * (n_r + 3);
  taps[idx] = make_float4((float)row[n == 0 ? 1 : n - 1], (float)row[n], (float)row[n + 1], (float)row[n + 2]);
}

// Partial coordinate gradient of the atoms of tile it over the j tiles of
// chunk c: part[c][it*128 + tid][3].
__global__ void __launch_bounds__(kGT)
    k_grad_pairs(const float4* __restrict__ atoms, const int* __restrict__ tile_type, int T, int n_tiles,
                 int chunk, const float4* __restrict__ taps, int n_r, float inv_dr, double* __restrict__ part) {
  __shared__ float4 sj[kGT];
  const int it = blockIdx.x, c = blockIdx.y, tid = threadIdx.x;
  const float4 ai = atoms[(size_t)it * kGT + tid];
  const int ta = tile_type[it];
  const float rmax_cell = (float)n_r - 0.001f;  // last cell index the taps cover, minus a margin
  double gx = 0.0, gy = 0.0, gz = 0.0;
  const int jt0 = c * chunk, jt1 = min(n_tiles, jt0 + chunk);
  for (int jt = jt0; jt < jt1; ++jt) {
    __syncthreads();
    sj[tid] = atoms[(size_t)jt * kGT + tid];
    __syncthreads();
    const int tb = tile_type[jt];
    const int a = min(ta, tb), b = max(ta, tb);
    const float4* tp = taps + (size_t)(a * T - a * (a - 1) / 2 + (b - a)) * (n_r + 1);
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
#pragma unroll 4
    for (int j = 0; j < kGT; ++j) {
      const float4 aj = sj[j];
      const float dx = ai.x - aj.x, dy = ai.y - aj.y, dz = ai.z - aj.z;
      const float x = fmaxf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), 1e-12f);
      const float y0 = rsqrtf(x);
      const float sq = x * y0;
      const float r = fmaf(fmaf(-sq, sq, x), 0.5f * y0, sq);  // Newton-refined sqrt
      const float t = fminf(r * inv_dr, rmax_cell);
      const float fl = floorf(t);
      const float u = t - fl;
      const float4 v = __ldg(tp + (int)fl);
      // Lagrange cubic on nodes -1, 0, 1, 2 at u in [0, 1)
      const float um1 = u - 1.0f, um2 = u - 2.0f, up1 = u + 1.0f;
      const float w0 = -u * um1 * um2 * (1.0f / 6.0f), w1 = up1 * um1 * um2 * 0.5f;
      const float w2 = -up1 * u * um2 * 0.5f, w3 = up1 * u * um1 * (1.0f / 6.0f);
      const float hv = fmaf(w0, v.x, fmaf(w1, v.y, fmaf(w2, v.z, w3 * v.w)));
      const float coefj = hv * (ai.w * aj.w);  // a pair of one atom with itself has dx = 0
      fx = fmaf(coefj, dx, fx);
      fy = fmaf(coefj, dy, fy);
      fz = fmaf(coefj, dz, fz);
    }
    gx += (double)fx;
    gy += (double)fy;
    gz += (double)fz;
  }
  double* out = part + ((size_t)c * n_tiles * kGT + (size_t)it * kGT + tid) * 3;
  out[0] = gx;
  out[1] = gy;
  out[2] = gz;
}

// grad[slot] = the sum over the chunks, in chunk order.
__global__ void k_grad_reduce(const double* __restrict__ part, int64_t n_slots, int n_chunks,
                              double* __restrict__ grad) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_slots * 3) return;
  double s = 0.0;
  for (int c = 0; c < n_chunks; ++c) s += part[(size_t)c * n_slots * 3 + i];
  grad[i] = s;
}

}  // namespace

std::vector<int2> q_blocks(const std::vector<double>& q, int Qmax);

void chi2_grad_impl(crab_ctx* ctx, const crab_struct* st, const double* q, const double* y, const double* sigma,
                    int64_t nq, const crab_solvent& s, bool implicit, double scale, double background, double* chi2_out,
                    double* grad_xyz, double* grad_p) {
  require(nq > 0, "gradient needs at least one q value");
  for (int64_t k = 0; k < nq; ++k)
    require(std::isfinite(y[k]) && std::isfinite(sigma[k]) && sigma[k] > 0.0,
            "intensity must be finite and sigma positive");
  require(s.hydration_model == CRAB_HYD_ANALYTIC, "the coordinate gradient covers the analytic hydration model");
  require(std::isfinite(scale) && std::isfinite(background), "scale and background must be finite");
  TypedAtoms t = type_atoms(st, implicit, TermSet::SolventAnalytic, nullptr);
  const int T = t.T;
  std::vector<double> V, E, H;
  amplitude_tables(t, q, nq, &s, implicit, 0.0, V, E, H);
  Partials P = partials_for(ctx, t, q, nq, false, nullptr);
  std::vector<double> b6(6 * nq), I(nq);
  quadratic_terms(P, V.data(), V.data(), b6.data());
  quadratic_terms(P, E.data(), E.data(), b6.data() + nq);
  quadratic_terms(P, H.data(), H.data(), b6.data() + 2 * nq);
  quadratic_terms(P, V.data(), E.data(), b6.data() + 3 * nq);
  quadratic_terms(P, V.data(), H.data(), b6.data() + 4 * nq);
  quadratic_terms(P, E.data(), H.data(), b6.data() + 5 * nq);
  combine_basis(q, nq, b6.data(), s.c1, s.c2, I.data());
  const double dof = (double)std::max<int64_t>(nq - 1, 1);
  std::vector<double> w(nq);
  double chi = 0.0, dc1 = 0.0, dc2 = 0.0, dsc = 0.0, dbg = 0.0;
  const double* B = b6.data();
  for (int64_t k = 0; k < nq; ++k) {
    const double res = (scale * I[k] + background - y[k]) / sigma[k];
    chi += res * res;
    const double dm = 2.0 * res / sigma[k] / dof;  // ∂χ²/∂model_k
    w[k] = I[k] > 0.0 ? dm * scale : 0.0;            // the clamp at zero has no gradient
    const double G = excluded_volume_scale(q[k], s.c1);
    const double dG = G * (3.0 / s.c1 - 2.0 * s.c1 * (1.62 * 1.62) * q[k] * q[k] / 4.0);
    const double dIdG = 2.0 * G * B[nq + k] - 2.0 * B[3 * nq + k] - 2.0 * s.c2 * B[5 * nq + k];
    const double dIdc2 = 2.0 * s.c2 * B[2 * nq + k] + 2.0 * B[4 * nq + k] - 2.0 * G * B[5 * nq + k];
    dc1 += w[k] * dIdG * dG;
    dc2 += w[k] * dIdc2;
    dsc += dm * I[k];
    dbg += dm;
  }
  if (chi2_out) *chi2_out = chi / dof;
  if (grad_p) {
    grad_p[0] = dc1;
    grad_p[1] = dc2;
    grad_p[2] = dsc;
    grad_p[3] = dbg;
  }
  if (!grad_xyz) return;
  std::fill(grad_xyz, grad_xyz + 3 * st->n, 0.0);
  if (t.w.empty()) return;
  // per type pair and q: alpha = 2 w_k A_a A_b (zero at q = 0, where the term has no r dependence)
  const int NP = T * (T + 1) / 2;
  std::vector<double> alpha((size_t)NP * nq, 0.0);
  double qmax = 0.0;
  for (int64_t k = 0; k < nq; ++k) qmax = std::max(qmax, q[k]);
  for (int a = 0; a < T; ++a)
    for (int bb = a; bb < T; ++bb)
      for (int64_t k = 0; k < nq; ++k) {
        if (!(q[k] > 0.0)) continue;
        const double G = excluded_volume_scale(q[k], s.c1);
        const double Aa = V[(size_t)a * nq + k] - G * E[(size_t)a * nq + k] + s.c2 * H[(size_t)a * nq + k];
        const double Ab = V[(size_t)bb * nq + k] - G * E[(size_t)bb * nq + k] + s.c2 * H[(size_t)bb * nq + k];
        alpha[(size_t)pair_index(a, bb, T) * nq + k] = 2.0 * w[k] * Aa * Ab;
      }
  Layout L = build_layout(t.xyz.data(), t.w.data(), t.type.data(), (int64_t)t.w.size(), T, false);
  // radial grid: dr = 0.02 / q_max up to the largest pair distance (bounded by the layout's extent)
  const double dr = qmax > 0.0 ? 0.02 / qmax : 1.0;
  const double reach = L.extent * 1.001 + 4.0 * dr;
  require(reach / dr < 4.0e7, "radial table of the gradient too long");
  const int n_r = std::max(2, (int)std::ceil(reach / dr));
  cudaStream_t sm = ctx->stream;
  float4* d_atoms = (float4*)ctx->dev("grad.atoms", (size_t)L.n_pad * sizeof(float4));
  int* d_tt = (int*)ctx->dev("grad.tt", L.tile_type.size() * sizeof(int));
  double* d_alpha = (double*)ctx->dev("grad.alpha", alpha.size() * sizeof(double));
  double* d_q = (double*)ctx->dev("grad.q", (size_t)nq * sizeof(double));
  double* d_h = (double*)ctx->dev("grad.h", (size_t)NP * (n_r + 3) * sizeof(double));
  float4* d_taps = (float4*)ctx->dev("grad.taps", (size_t)NP * (n_r + 1) * sizeof(float4));
  copy_h2d(ctx, d_atoms, L.atoms.data(), (size_t)L.n_pad * sizeof(float4), sm);
  copy_h2d(ctx, d_tt, L.tile_type.data(), L.tile_type.size() * sizeof(int), sm);
  copy_h2d(ctx, d_alpha, alpha.data(), alpha.size() * sizeof(double), sm);
  copy_h2d(ctx, d_q, q, (size_t)nq * sizeof(double), sm);
  const int64_t nh = (int64_t)NP * (n_r + 3), ntp = (int64_t)NP * (n_r + 1);
  k_grad_h<<<(unsigned)((nh * 32 + 255) / 256), 256, 0, sm>>>(d_alpha, d_q, (int)nq, NP, n_r, dr, d_h);
  k_grad_taps<<<(unsigned)((ntp + 127) / 128), 128, 0, sm>>>(d_h, NP, n_r, d_taps);
  // (i tile, chunk of j tiles) blocks: about four per SM
  const int n_tiles = L.n_tiles;
  const int want = std::max(1, (4 * ctx->sm_count + n_tiles - 1) / std::max(n_tiles, 1));
  const int chunk = std::max(1, (n_tiles + want - 1) / want);
  const int n_chunks = (n_tiles + chunk - 1) / chunk;
  double* d_part = (double*)ctx->dev("grad.part", (size_t)n_chunks * L.n_pad * 3 * sizeof(double));
  double* d_grad = (double*)ctx->dev("grad.out", (size_t)L.n_pad * 3 * sizeof(double));
  k_grad_pairs<<<dim3((unsigned)n_tiles, (unsigned)n_chunks), kGT, 0, sm>>>(d_atoms, d_tt, T, n_tiles, chunk, d_taps,
                                                                             n_r, (float)(1.0 / dr), d_part);
  k_grad_reduce<<<(unsigned)((L.n_pad * 3 + 255) / 256), 256, 0, sm>>>(d_part, L.n_pad, n_chunks, d_grad);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 4;
  std::vector<double> g((size_t)L.n_pad * 3);
  copy_d2h(ctx, g.data(), d_grad, g.size() * sizeof(double), sm);
  CRAB_CUDA_CHECK(cudaStreamSynchronize(sm));
  for (int64_t slot = 0; slot < L.n_pad; ++slot) {
    const int64_t k = L.source[slot];
    if (k < 0) continue;
    const int64_t i = t.src[k];
    if (i < 0) continue;
    for (int d = 0; d < 3; ++d) grad_xyz[3 * i + d] += g[3 * slot + d];
  }
}

}  // namespace crab

using namespace crab;

extern "C" int crab_chi2_grad(crab_ctx* ctx, crab_struct* st, const double* q, const double* y, const double* sigma,
                              int64_t nq, const crab_solvent* solvent, int implicit_hydrogen, double scale,
                              double background, double* chi2, double* grad_xyz, double* grad_params) {
  if (!ctx || !st || !solvent || !q || !y || !sigma || nq <= 0) return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    validate_q(q, nq);
    validate_solvent(*solvent);
    chi2_grad_impl(ctx, st, q, y, sigma, nq, *solvent, implicit_hydrogen != 0, scale, background, chi2, grad_xyz,
                   grad_params);
  });
}
