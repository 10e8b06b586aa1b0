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
// The kernel recomputes every pair term per tile (nothing O(N²) is stored):
// one thread per atom i, j tiles in shared memory, sin and cos of q r
// advanced together along each uniform q block by the Reinsch recurrence in
// one packed f32x2 register pair, the q sums accumulated per block in FP32
// and per atom in FP64.  A pair's term for atom j is the negative of its
// term for atom i (g_ab = g_ba), so only tile pairs it <= jt run: a diagonal
// tile computes its ordered pairs for its own atoms, an off-diagonal one also
// sums each j's terms over the block (a warp shuffle, then shared memory).

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

// Tile pair (it, jt), it <= jt, of block w = jt (jt + 1) / 2 + it.
__device__ __forceinline__ void grad_tri_decode(int w, int& it, int& jt) {
  int b = (int)((sqrt(8.0 * (double)w + 1.0) - 1.0) * 0.5);
  while (b > 0 && b * (b + 1) / 2 > w) --b;
  while ((b + 1) * (b + 2) / 2 <= w) ++b;
  jt = b;
  it = w - b * (b + 1) / 2;
}

__global__ void __launch_bounds__(kGT, 4)
    k_chi2_grad(const float4* __restrict__ atoms, const int* __restrict__ tile_type, int T,
                const float2* __restrict__ coef, int nq, const float4* __restrict__ qpar,
                const int2* __restrict__ qrange, int n_qb, int wide, double* __restrict__ grad) {
  extern __shared__ float2 s_coef[];  // nq (alpha, beta) of this tile pair's type pair
  __shared__ float4 sj[kGT];
  __shared__ double s_gj[kGT][3];     // the j tile's terms (off-diagonal tile pairs)
  int it, jt;
  grad_tri_decode((int)blockIdx.x, it, jt);
  const int tid = threadIdx.x, lane = tid & 31;
  const bool diag = it == jt;
  const float4 ai = atoms[(size_t)it * kGT + tid];
  sj[tid] = atoms[(size_t)jt * kGT + tid];
  s_gj[tid][0] = s_gj[tid][1] = s_gj[tid][2] = 0.0;
  const int ta = tile_type[it], tb = tile_type[jt];
  const int a = min(ta, tb), b = max(ta, tb);
  const int ab = a * T - a * (a - 1) / 2 + (b - a);
  for (int k = tid; k < nq; k += kGT) s_coef[k] = coef[(size_t)ab * nq + k];
  __syncthreads();
  double gx = 0.0, gy = 0.0, gz = 0.0;
  for (int j = 0; j < kGT; ++j) {
    const float4 aj = sj[j];
    const float wij = (jt == it && j == tid) ? 0.0f : ai.w * aj.w;
    const float dx = ai.x - aj.x, dy = ai.y - aj.y, dz = ai.z - aj.z;
    const float x = fmaxf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), 1e-8f);
    const float y0 = rsqrtf(x);
    const float sq = x * y0;
    const float hy = 0.5f * y0;
    const float r = fmaf(fmaf(-sq, sq, x), hy, sq);
    const float rinv = fmaf(fmaf(-sq, y0, 1.0f), hy, y0);
    double Csum = 0.0, Ssum = 0.0;
    for (int blk = 0; blk < n_qb; ++blk) {
      const float4 qp = qpar[blk];
      const int2 qr = qrange[blk];
      const float phi = fmaf(qp.x, r, qp.y * r);
      const float h = fmaf(qp.z, r, qp.w * r);
      float s0, c0, sh, ch;
      sincos_seed(phi, &s0, &c0);
      if (wide) sincos_seed(h, &sh, &ch);
      else sincos_small(h, &sh, &ch);
      const float half_l = 2.0f * sh * sh;     // λ/2 = 1 - cos θ
      const float sin_t = 2.0f * sh * ch;      // sin θ
      const float ds = fmaf(s0, half_l, c0 * sin_t);   // sin φ - sin(φ-θ)
      const float dc = fmaf(c0, half_l, -s0 * sin_t);  // cos φ - cos(φ-θ)
      unsigned long long cs2 = pack2(c0, s0), d2 = pack2(dc, ds);
      const unsigned long long nl2 = pack2(-2.0f * half_l, -2.0f * half_l);
      unsigned long long acc2 = pack2(0.0f, 0.0f);
      const unsigned long long* cf = reinterpret_cast<const unsigned long long*>(s_coef) + qr.x;
#pragma unroll 4
      for (int k = 0; k < qr.y; ++k) {
        const unsigned long long ab2 = cf[k];
        asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc2) : "l"(ab2), "l"(cs2));
        asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d2) : "l"(nl2), "l"(cs2));
        asm("add.rn.f32x2 %0, %0, %1;" : "+l"(cs2) : "l"(d2));
      }
      float C, S;
      unpack2(acc2, C, S);
      Csum += (double)C;
      Ssum += (double)S;
    }
    const double g = (double)wij * ((double)rinv * (Csum - Ssum * (double)rinv));
    const double gr = g * (double)rinv;
    gx += gr * dx;
    gy += gr * dy;
    gz += gr * dz;
    if (!diag) {  // uniform over the block: every thread is at the same j
      double jx = -gr * dx, jy = -gr * dy, jz = -gr * dz;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        jx += __shfl_xor_sync(0xffffffffu, jx, o);
        jy += __shfl_xor_sync(0xffffffffu, jy, o);
        jz += __shfl_xor_sync(0xffffffffu, jz, o);
      }
      if (lane == 0) {
        atomicAdd(&s_gj[j][0], jx);
        atomicAdd(&s_gj[j][1], jy);
        atomicAdd(&s_gj[j][2], jz);
      }
    }
  }
  double* out = grad + 3 * ((size_t)it * kGT + tid);
  atomicAdd(out, gx);
  atomicAdd(out + 1, gy);
  atomicAdd(out + 2, gz);
  if (!diag) {
    __syncthreads();
    double* outj = grad + 3 * ((size_t)jt * kGT + tid);
    atomicAdd(outj, s_gj[tid][0]);
    atomicAdd(outj + 1, s_gj[tid][1]);
    atomicAdd(outj + 2, s_gj[tid][2]);
  }
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
  // per type pair and q: (alpha, beta)
  const int NP = T * (T + 1) / 2;
  std::vector<float2> coef((size_t)NP * nq);
  for (int a = 0; a < T; ++a)
    for (int bb = a; bb < T; ++bb)
      for (int64_t k = 0; k < nq; ++k) {
        const double G = excluded_volume_scale(q[k], s.c1);
        const double Aa = V[(size_t)a * nq + k] - G * E[(size_t)a * nq + k] + s.c2 * H[(size_t)a * nq + k];
        const double Ab = V[(size_t)bb * nq + k] - G * E[(size_t)bb * nq + k] + s.c2 * H[(size_t)bb * nq + k];
        const double alpha = 2.0 * w[k] * Aa * Ab;
        const double beta = q[k] > 0.0 ? alpha / q[k] : 0.0;
        coef[(size_t)pair_index(a, bb, T) * nq + k] = make_float2((float)(q[k] > 0.0 ? alpha : 0.0), (float)beta);
      }
  Layout L = build_layout(t.xyz.data(), t.w.data(), t.type.data(), (int64_t)t.w.size(), T, false);
  std::vector<double> qv(q, q + nq);
  const std::vector<int2> qr = q_blocks(qv, 128);
  std::vector<float4> qp(qr.size());
  double max_half = 0.0;
  for (size_t bk = 0; bk < qr.size(); ++bk) {
    const int64_t st0 = qr[bk].x, cnt = qr[bk].y;
    const double q0 = q[st0];
    const double half = cnt > 1 ? 0.5 * (q[st0 + cnt - 1] - q[st0]) / (double)(cnt - 1) : 0.0;
    const float q0h = (float)q0, hh = (float)half;
    qp[bk] = make_float4(q0h, (float)(q0 - (double)q0h), hh, (float)(half - (double)hh));
    max_half = std::max(max_half, std::fabs(half));
  }
  const int wide = (max_half * (L.extent + 1.0) > 0.8) ? 1 : 0;
  cudaStream_t sm = ctx->stream;
  float4* d_atoms = (float4*)ctx->dev("grad.atoms", (size_t)L.n_pad * sizeof(float4));
  int* d_tt = (int*)ctx->dev("grad.tt", L.tile_type.size() * sizeof(int));
  float2* d_coef = (float2*)ctx->dev("grad.coef", coef.size() * sizeof(float2));
  float4* d_qp = (float4*)ctx->dev("grad.qpar", qp.size() * sizeof(float4));
  int2* d_qr = (int2*)ctx->dev("grad.qrange", qr.size() * sizeof(int2));
  double* d_grad = (double*)ctx->dev("grad.out", (size_t)L.n_pad * 3 * sizeof(double));
  copy_h2d(ctx, d_atoms, L.atoms.data(), (size_t)L.n_pad * sizeof(float4), sm);
  copy_h2d(ctx, d_tt, L.tile_type.data(), L.tile_type.size() * sizeof(int), sm);
  copy_h2d(ctx, d_coef, coef.data(), coef.size() * sizeof(float2), sm);
  copy_h2d(ctx, d_qp, qp.data(), qp.size() * sizeof(float4), sm);
  copy_h2d(ctx, d_qr, qr.data(), qr.size() * sizeof(int2), sm);
  CRAB_CUDA_CHECK(cudaMemsetAsync(d_grad, 0, (size_t)L.n_pad * 3 * sizeof(double), sm));
  const size_t smem = (size_t)nq * sizeof(float2);
  require(smem <= 200 * 1024, "too many q values for the gradient kernel");
  if (smem > 48 * 1024)
    CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_chi2_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t n_blocks = (int64_t)L.n_tiles * (L.n_tiles + 1) / 2;  // tile pairs it <= jt
  require(n_blocks < ((int64_t)1 << 31), "too many atoms for the gradient kernel");
  k_chi2_grad<<<(unsigned)n_blocks, kGT, smem, sm>>>(d_atoms, d_tt, T, d_coef, (int)nq, d_qp, d_qr,
                                                            (int)qr.size(), wide, d_grad);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 1;
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
