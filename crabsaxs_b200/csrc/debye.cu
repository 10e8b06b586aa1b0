// Debye pair sums per atom-type pair on B200 (sm_100a).
//
// Replaces the O(N²·Nq) pair loops of crabSAXS src/scattering.rs:99-106 and
// src/solvent.rs:533-577.  Instead of summing amplitude products per q, the
// kernel produces, for every unordered type pair (a<=b),
//     P_ab(q) = Σ_{i<j, {t_i,t_j}={a,b}} w_i w_j sinc(q r_ij),
// from which every Debye term (vacuum, excluded volume, hydration, their
// cross terms, any c1/c2) is a small f64 recombination on the host.
//
// FP32 kernel (uniform q grid):
//  * atoms are grouped by type and padded per type to 128-atom tiles, so each
//    (i-tile, j-tile) block has one type pair and the per-thread accumulators
//    stay in registers with static indices;
//  * a CTA of 128 threads keeps one i atom per thread in registers and stages
//    j tiles (float4 x,y,z,w; 2 KB) in shared memory with a bulk async copy;
//  * for each pair the thread seeds sin(q0 r) and cos(q0 r) once per block of
//    Q consecutive q values and advances sin(q r) along the grid with the
//    three-term (Chebyshev) recurrence in Reinsch's difference form
//        d_{k+1} = d_k - λ s_k,  s_{k+1} = s_k + d_{k+1},  λ = 4 sin²(Δr/2),
//    which keeps the frequency exact in FP32 for small Δr (the plain form
//    s_{k+1} = 2cos(Δr) s_k - s_{k-1} loses it: 2cos(Δr) rounds to ~1e-7
//    absolute while 2-2cos(Δr) may be 1e-6);
//  * the accumulated quantity is Σ w_i w_j sin(q r)/r; the host divides by q
//    in f64 (q = 0 is the exact Σ w_i w_j);
//  * per thread FP32 sums cover at most one run of same-type j tiles, then a
//    warp-shuffle reduction and an FP64 atomic add per (type pair, q).
// FP64 kernel: the same tiling with direct f64 sinc per pair and q; it is the
// on-device reference for the error reports and large-size checks.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "device_math.cuh"
#include "engine.hpp"

namespace crab {
namespace {

using namespace dev;

constexpr int kThreads = 128;  // one i atom per thread; equals kTile
constexpr int kQBlocks[] = {8, 16, 32, 48, 64, 96, 100, 126, 128, 150, 168};  // q-block lengths of the untuned choice
// jb values at or above kPackedQ select the q-packed kernel with
// (jb - kPackedQ) % kDenser chains; + kDenser asks for 3 CTAs per SM.
constexpr int kPackedQ = 8;
constexpr int kDenser = 4;
// q-packed with the weight folded into the recurrence state (pair_setup_pq_folded):
// one chain at two CTAs per SM, two chains at two, one chain at three, one at four
constexpr int kFolded1 = 5, kFolded2 = 6, kFolded1x3 = 7, kFolded1x4 = 3;
// folded, two packed chains per pair (q points 4n, 4n+1 and 4n+2, 4n+3),
// two CTAs per SM; plans whose half step angle Δr/2 exceeds kMax2cHalfAngle
// run the one-chain build kFolded1 of the same length instead
constexpr int kFolded2c = 11;
constexpr double kMax2cHalfAngle = 0.2;
// set-up and recurrences in separate warpgroups (k_pair_split), one or two
// chains per recurrence thread
constexpr int kSplit1 = 14, kSplit2 = 15;
// the split with one recurrence warpgroup for each of three q blocks per item
// (k_pair_split3)
constexpr int kSplit3 = 12;
static_assert(kThreads == kTile, "tile size and CTA size must match");

// v on the plan's fixed-point grid of step 1/sc (sc a power of two chosen on
// the host so that every partial sum stays below 2^52 steps): f64 sums of such
// values are exact, so the order in which the atomic adds land does not change
// the partials (bit-reproducible results), and the step, about 2^-52 of a
// bound on the sums, lies far below the FP32 terms' own rounding
__device__ __forceinline__ double on_grid(double v, double sc) {
  // 1/sc exactly: sc = 2^e (|e| <= 1000), whose reciprocal's exponent field is
  // 2046 minus sc's
  const double inv = __longlong_as_double(0x7FE0000000000000ll - __double_as_longlong(sc));
  return rint(v * sc) * inv;
}

template <int Q>
__device__ __forceinline__ void flush_fp32(float (&acc)[Q], float (*red)[Q], int ab, int qstart, int qcount, int nq,
                                           double* __restrict__ partials, double sc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    float v = acc[k];
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    if (lane == 0) red[warp][k] = v;
    acc[k] = 0.0f;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < qcount; k += kThreads) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s += (double)red[w][k];
    atomicAdd(&partials[(size_t)ab * nq + qstart + k], on_grid(s, sc));
  }
  __syncthreads();
}

// Per-pair set-up of the recurrence: weight u = w_i w_j / r, λ = 4 sin²(h),
// seed s0 = sin(q0 r) and first difference d0 = sin(q0 r) - sin((q0-Δ) r)
// = 2 sin(h) cos(q0 r - h), with h = Δr/2.  r and 1/r come from one MUFU
// reciprocal square root y0 refined with FMA residuals (Markstein): with
// s = x·y0, e = x - s² and t = 1 - s·y0 formed exactly by FMA,
// r = s + e·y0/2 and 1/r = y0 + t·y0/2, both within about half an ulp and
// unbiased.  (A refinement y0·(1.5 - 0.5·x·y0²) does not work in FP32: the
// correction factor rounds to 1.0 when y0 is already close.)
__device__ __forceinline__ void pair_setup(const float4& ai, const float4& aj, float wj, const float4& qp, int wide,
                                           float& u, float& nl, float& s, float& d) {
  const float dx = aj.x - ai.x, dy = aj.y - ai.y, dz = aj.z - ai.z;
  const float x = fmaxf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), 1e-8f);
  const float y0 = rsqrtf(x);
  const float sq = x * y0;
  const float hy = 0.5f * y0;
  const float r = fmaf(fmaf(-sq, sq, x), hy, sq);
  const float rinv = fmaf(fmaf(-sq, y0, 1.0f), hy, y0);
  u = ai.w * wj * rinv;
  const float phi = fmaf(qp.x, r, qp.y * r);
  const float h = fmaf(qp.z, r, qp.w * r);
  float c0, sh, ch;
  sincos_seed(phi, &s, &c0);
  if (wide) sincos_seed(h, &sh, &ch);
  else sincos_small(h, &sh, &ch);
  nl = -4.0f * sh * sh;
  d = 2.0f * sh * fmaf(s, sh, c0 * ch);
}

// Set-up for the q-packed recurrence: the two halves of each f32x2 register
// follow the even and the odd q points of the block, so each half steps by
// 2Δ (angle Δr, λ' = 4 sin²(Δr)).  S, C = sin, cos(q0 r) come from the
// reduced polynomial seed (within an ulp or two; the hardware sine, about
// 5e-7 absolute, is not accurate enough: solvent curves cancel to a few
// percent of their vacuum terms at high q and would carry its error 30-fold);
// s1, c1 = sin, cos(Δr) from short polynomials when the plan's largest step
// angle is at most 0.25 rad (wide == 0), else from the reduced seed.  Then:
//   lane A: s = S,                   d = S - sin(q0 r - 2Δr) = 2 s1 cos(q0 r - Δr)
//   lane B: s = sin(q0 r + Δr),      d = sin(q0 r + Δr) - sin(q0 r - Δr) = 2 s1 C.
// The per-pair part: r and u = w_i w_j / r.
__device__ __forceinline__ void pair_geom(const float4& ai, const float4& aj, float wj, float& r, float& u) {
  const float dx = aj.x - ai.x, dy = aj.y - ai.y, dz = aj.z - ai.z;
  const float x = fmaxf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), 1e-8f);
  const float y0 = rsqrtf(x);
  const float sq = x * y0;
  const float hy = 0.5f * y0;
  r = fmaf(fmaf(-sq, sq, x), hy, sq);
  const float rinv = fmaf(fmaf(-sq, y0, 1.0f), hy, y0);
  u = ai.w * wj * rinv;
}
// The per-block part: seeds and step of the block qp at distance r.
__device__ __forceinline__ void pair_seed_pq(float r, const float4& qp, int wide, float& nl, float& S, float& sB,
                                             float& dA, float& dB) {
  const float phi = fmaf(qp.x, r, qp.y * r);
  const float g = 2.0f * fmaf(qp.z, r, qp.w * r);  // Δr
  float C, s1, c1;
  sincos_seed(phi, &S, &C);
  if (wide) {
    sincos_seed(g, &s1, &c1);
  } else {
    // |g| <= 0.25: Taylor to g^7 for sin and g^6 for cos (truncation < 4e-10)
    const float g2 = g * g;
    float ps = fmaf(g2, -1.0f / 5040.0f, 1.0f / 120.0f);
    ps = fmaf(g2, ps, -1.0f / 6.0f);
    s1 = fmaf(g * g2, ps, g);
    float pc = fmaf(g2, -1.0f / 720.0f, 1.0f / 24.0f);
    pc = fmaf(g2, pc, -0.5f);
    c1 = fmaf(g2, pc, 1.0f);
  }
  sB = fmaf(S, c1, C * s1);
  dA = 2.0f * s1 * fmaf(C, c1, S * s1);
  dB = 2.0f * s1 * C;
  nl = -4.0f * s1 * s1;
}
__device__ __forceinline__ void pair_setup_pq(const float4& ai, const float4& aj, float wj, const float4& qp, int wide,
                                              unsigned long long& u2, unsigned long long& nl2,
                                              unsigned long long& s2, unsigned long long& d2) {
  float r, u, nl, S, sB, dA, dB;
  pair_geom(ai, aj, wj, r, u);
  pair_seed_pq(r, qp, wide, nl, S, sB, dA, dB);
  u2 = pack2(u, u);
  nl2 = pack2(nl, nl);
  s2 = pack2(S, sB);
  d2 = pack2(dA, dB);
}

// The same with the weight folded into the recurrence state: s' = u s and
// d' = u d follow the same linear recurrence, so the accumulate step becomes
// acc += s' (a packed add with two register sources instead of a packed FMA
// with three, and u needs no register during the steps).
__device__ __forceinline__ void pair_setup_pq_folded(const float4& ai, const float4& aj, float wj, const float4& qp,
                                                     int wide, unsigned long long& nl2, unsigned long long& s2,
                                                     unsigned long long& d2) {
  unsigned long long u2;
  pair_setup_pq(ai, aj, wj, qp, wide, u2, nl2, s2, d2);
  asm("mul.rn.f32x2 %0, %0, %1;" : "+l"(s2) : "l"(u2));
  asm("mul.rn.f32x2 %0, %0, %1;" : "+l"(d2) : "l"(u2));
}

// Two packed chains per pair, each stepping 4Δ: chain X holds the q points
// (4n, 4n+1) of the block and chain Y (4n+2, 4n+3), so a thread has two
// independent recurrences in flight with the registers of one.  With
// φ = q0 r, g = Δr, s1, c1 = sin, cos g (as in pair_seed_pq) and
// s2 = sin 2g = 2 s1 c1, c2 = cos 2g = 1 - 2 s1²:
//   s = sin φ, sin(φ+g), sin(φ+2g), sin(φ+3g) by angle addition,
//   d = s - sin(· - 4g) = 2 s2 cos(· - 2g), i.e. 2 s2 times
//       cos(φ-2g), cos(φ-g), cos φ, cos(φ+g),
//   λ' = 4 sin²(2g).
// The host runs this build only while g = Δr <= 0.4 (half step angle at most
// kMax2cHalfAngle), so the chains' step angle 4g stays at most 1.6 rad, where
// the difference form of the recurrence loses nothing (cos 2g > 0.69); s1, c1
// come from their Taylor series, to g^7 and g^6 while g <= 0.25 (wide == 0,
// truncation below 4e-10), else to g^9 and g^8 (below 3e-11).
__device__ __forceinline__ void pair_setup_pq2c_folded(const float4& ai, const float4& aj, float wj, const float4& qp,
                                                       int wide, unsigned long long& nl2, unsigned long long& sx,
                                                       unsigned long long& dx, unsigned long long& sy,
                                                       unsigned long long& dy) {
  float r, u;
  pair_geom(ai, aj, wj, r, u);
  const float phi = fmaf(qp.x, r, qp.y * r);
  const float g = 2.0f * fmaf(qp.z, r, qp.w * r);  // Δr
  float S0, C0;
  sincos_seed(phi, &S0, &C0);
  // every seed and difference below is linear in (sin φ, cos φ): scaling
  // these two by u folds the weight into the whole state
  const float S = u * S0, C = u * C0;
  const float g2 = g * g;
  float ps, pc;
  if (wide) {  // g <= 0.4: two more terms
    ps = fmaf(g2, 1.0f / 362880.0f, -1.0f / 5040.0f);
    ps = fmaf(g2, ps, 1.0f / 120.0f);
    pc = fmaf(g2, 1.0f / 40320.0f, -1.0f / 720.0f);
    pc = fmaf(g2, pc, 1.0f / 24.0f);
  } else {
    ps = fmaf(g2, -1.0f / 5040.0f, 1.0f / 120.0f);
    pc = fmaf(g2, -1.0f / 720.0f, 1.0f / 24.0f);
  }
  ps = fmaf(g2, ps, -1.0f / 6.0f);
  const float s1 = fmaf(g * g2, ps, g);
  pc = fmaf(g2, pc, -0.5f);
  const float c1 = fmaf(g2, pc, 1.0f);
  const float s2 = 2.0f * s1 * c1, c2 = fmaf(-2.0f * s1, s1, 1.0f);
  const float sp1 = fmaf(S, c1, C * s1);   // sin(φ+g)
  const float cp1 = fmaf(C, c1, -S * s1);  // cos(φ+g)
  const float cm1 = fmaf(C, c1, S * s1);   // cos(φ-g)
  const float t = 2.0f * s2;
  const float nl = -t * t;
  nl2 = pack2(nl, nl);
  sx = pack2(S, sp1);
  sy = pack2(fmaf(S, c2, C * s2), fmaf(sp1, c2, cp1 * s2));
  dx = pack2(t * fmaf(C, c2, S * s2), t * cm1);
  dy = pack2(t * C, t * cp1);
}

// Work item: (i tile, first j tile, end j tile, q block); items are taken
// from a global counter (longest first) so CTAs finish together.
// qpar[b] = (q0_hi, q0_lo, halfstep_hi, halfstep_lo), qrange[b] = (start, count).
template <int Q, int JB>
__global__ void __launch_bounds__(kThreads, JB == 2 ? (Q <= 64 ? 4 : (Q <= 96 ? 3 : 2)) : (Q <= 64 ? 3 : 2))
    k_pair_fp32(const float4* __restrict__ atoms, const int* __restrict__ tile_type, const int4* __restrict__ work,
                int n_work, const float4* __restrict__ qpar, const int2* __restrict__ qrange, int nq, int T, int wide,
                double* __restrict__ partials, int* __restrict__ status, int* __restrict__ next_work,
                const int64_t* __restrict__ work_out,
                const double* __restrict__ item_scale, int budget) {
  __shared__ __align__(16) float4 sj[2][kTile];
  __shared__ float red[kThreads / 32][Q];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_item;
  __shared__ double s_scale;  // the item's fixed-point scale, read at its flushes
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  unsigned phase_bits = 0u;  // bit b: parity of the next completion of bar[b]
  bool ok = true;
  if (budget < 0) budget = kWaitBudget;  // the context's default

  for (;;) {
    if (tid == 0) s_item = atomicAdd(next_work, 1);
    __syncthreads();
    const int w = s_item;
    // written between the two barriers: every thread has finished the last
    // item's flushes (which read it) before the first one
    if (tid == 0 && w < n_work) s_scale = item_scale[w];
    __syncthreads();
    if (w >= n_work || !ok) break;
    const int4 wk = work[w];
    const int it = wk.x, jt0 = wk.y, jt1 = wk.z, qb = wk.w;
    double* __restrict__ out = partials + (work_out ? work_out[w] : 0);  // per-structure output in a batch
    const float4 ai = atoms[(size_t)it * kTile + tid];
    const float4 qp = qpar[qb];
    const int2 qr = qrange[qb];
    const int ti = tile_type[it];
    float acc[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) acc[k] = 0.0f;
    int cur = tile_type[jt0];

    // prefetch the first j tile
    if (tid == 0) {
      mbar_expect_tx(&bar[0], kTile * sizeof(float4));
      bulk_g2s(&sj[0][0], atoms + (size_t)jt0 * kTile, kTile * sizeof(float4), &bar[0]);
    }
    int buf = 0;
    for (int jt = jt0; jt < jt1; ++jt) {
      const int tj = tile_type[jt];
      if (tj != cur) {
        const int a = min(ti, cur), b = max(ti, cur);
        flush_fp32<Q>(acc, red, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, s_scale);
        cur = tj;
      }
      // issue the next tile into the other buffer (its previous readers
      // finished at the __syncthreads that closed the previous iteration)
      if (tid == 0 && jt + 1 < jt1) {
        mbar_expect_tx(&bar[buf ^ 1], kTile * sizeof(float4));
        bulk_g2s(&sj[buf ^ 1][0], atoms + (size_t)(jt + 1) * kTile, kTile * sizeof(float4), &bar[buf ^ 1]);
      }
      const unsigned ph = (phase_bits >> buf) & 1u;
      if (!mbar_wait(&bar[buf], ph, budget)) {
        if (tid == 0) atomicExch(status, CRAB_ETIMEOUT);
        ok = false;
      }
      phase_bits ^= 1u << buf;
      if (!__syncthreads_and(ok)) {
        // leave only after this CTA's copies in flight have landed: the
        // current tile's and the prefetched one's (their shared memory may
        // belong to the next CTA on this SM once this one exits)
        if (tid == 0) {
          mbar_wait(&bar[buf], ph, kDrainBudget);
          if (jt + 1 < jt1) mbar_wait(&bar[buf ^ 1], (phase_bits >> (buf ^ 1)) & 1u, kDrainBudget);
        }
        __syncthreads();
        ok = false;
        break;
      }
      const bool diag = (jt == it);
      // JB j atoms per iteration, their recurrences advanced in pairs in
      // packed f32x2 registers (JB/2 independent chains per instruction stream)
#pragma unroll 1
      for (int j = 0; j < kTile; j += JB) {
        float u[JB];
        unsigned long long s2[JB / 2], d2[JB / 2], nl2[JB / 2];
#pragma unroll
        for (int p = 0; p < JB / 2; ++p) {
          const float4 aA = sj[buf][j + 2 * p], aB = sj[buf][j + 2 * p + 1];
          const float wA = (diag && j + 2 * p <= tid) ? 0.0f : aA.w;
          const float wB = (diag && j + 2 * p + 1 <= tid) ? 0.0f : aB.w;
          float nlA, sA, dA, nlB, sB, dB;
          pair_setup(ai, aA, wA, qp, wide >= 2, u[2 * p], nlA, sA, dA);
          pair_setup(ai, aB, wB, qp, wide >= 2, u[2 * p + 1], nlB, sB, dB);
          s2[p] = pack2(sA, sB);
          d2[p] = pack2(dA, dB);
          nl2[p] = pack2(nlA, nlB);
        }
#pragma unroll
        for (int k = 0; k < Q; ++k) {
#pragma unroll
          for (int p = 0; p < JB / 2; ++p) {
            float xa, xb;
            unpack2(s2[p], xa, xb);
            acc[k] = fmaf(u[2 * p], xa, acc[k]);
            acc[k] = fmaf(u[2 * p + 1], xb, acc[k]);
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d2[p]) : "l"(nl2[p]), "l"(s2[p]));
            asm("add.rn.f32x2 %0, %0, %1;" : "+l"(s2[p]) : "l"(d2[p]));
          }
        }
      }
      __syncthreads();
      buf ^= 1;
    }
    if (ok) {
      const int a = min(ti, cur), b = max(ti, cur);
      flush_fp32<Q>(acc, red, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, s_scale);
    }
  }
}

// Per-warp flush of packed accumulators (defined with the split kernels below).
template <int Q>
__device__ __forceinline__ void flush_split(unsigned long long (&acc2)[Q / 2], int ab, int qstart, int qcount,
                                            int nq, double* __restrict__ partials, double sc);

// The same work items with the q-packed recurrence: accumulators are f32x2
// pairs (q points 2m, 2m+1), and JB j atoms run JB independent packed chains,
// 3 packed instructions per chain and step (6 FP32 lane operations for 2
// pair·q, as the j-packed form, but with JB chains in flight per warp).  Each
// warp flushes its own sums (flush_split): on the fixed-point grid the order
// of the adds does not matter.

template <int Q, int JB, int OCC = (Q <= 64 ? 4 : (Q <= 96 ? 3 : 2)), bool FOLD = false, int CH = 1>
__global__ void __launch_bounds__(kThreads, OCC)
    k_pair_fp32_pq(const float4* __restrict__ atoms, const int* __restrict__ tile_type, const int4* __restrict__ work,
                   int n_work, const float4* __restrict__ qpar, const int2* __restrict__ qrange, int nq, int T,
                   int wide, double* __restrict__ partials, int* __restrict__ status, int* __restrict__ next_work,
                   const int64_t* __restrict__ work_out,
                const double* __restrict__ item_scale, int budget) {
  static_assert(Q % 2 == 0, "q-packed blocks hold an even number of q points");
  static_assert(CH == 1 || (CH == 2 && JB == 1 && FOLD && Q % 4 == 0), "two chains per pair: folded, one pair");
  __shared__ __align__(16) float4 sj[2][kTile];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_item;
  __shared__ double s_scale;  // the item's fixed-point scale, read at its flushes
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  unsigned phase_bits = 0u;
  bool ok = true;
  if (budget < 0) budget = kWaitBudget;  // the context's default

  for (;;) {
    if (tid == 0) s_item = atomicAdd(next_work, 1);
    __syncthreads();
    const int w = s_item;
    // written between the two barriers: every thread has finished the last
    // item's flushes (which read it) before the first one
    if (tid == 0 && w < n_work) s_scale = item_scale[w];
    __syncthreads();
    if (w >= n_work || !ok) break;
    const int4 wk = work[w];
    const int it = wk.x, jt0 = wk.y, jt1 = wk.z, qb = wk.w;
    double* __restrict__ out = partials + (work_out ? work_out[w] : 0);
    const float4 ai = atoms[(size_t)it * kTile + tid];
    const float4 qp = qpar[qb];
    const int2 qr = qrange[qb];
    const int ti = tile_type[it];
    unsigned long long acc2[Q / 2];
#pragma unroll
    for (int m = 0; m < Q / 2; ++m) acc2[m] = 0ull;
    int cur = tile_type[jt0];
    if (tid == 0) {
      mbar_expect_tx(&bar[0], kTile * sizeof(float4));
      bulk_g2s(&sj[0][0], atoms + (size_t)jt0 * kTile, kTile * sizeof(float4), &bar[0]);
    }
    int buf = 0;
    for (int jt = jt0; jt < jt1; ++jt) {
      const int tj = tile_type[jt];
      if (tj != cur) {
        const int a = min(ti, cur), b = max(ti, cur);
        flush_split<Q>(acc2, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, s_scale);
        cur = tj;
      }
      if (tid == 0 && jt + 1 < jt1) {
        mbar_expect_tx(&bar[buf ^ 1], kTile * sizeof(float4));
        bulk_g2s(&sj[buf ^ 1][0], atoms + (size_t)(jt + 1) * kTile, kTile * sizeof(float4), &bar[buf ^ 1]);
      }
      const unsigned ph = (phase_bits >> buf) & 1u;
      if (!mbar_wait(&bar[buf], ph, budget)) {
        if (tid == 0) atomicExch(status, CRAB_ETIMEOUT);
        ok = false;
      }
      phase_bits ^= 1u << buf;
      if (!__syncthreads_and(ok)) {
        // leave only after this CTA's copies in flight have landed: the
        // current tile's and the prefetched one's (their shared memory may
        // belong to the next CTA on this SM once this one exits)
        if (tid == 0) {
          mbar_wait(&bar[buf], ph, kDrainBudget);
          if (jt + 1 < jt1) mbar_wait(&bar[buf ^ 1], (phase_bits >> (buf ^ 1)) & 1u, kDrainBudget);
        }
        __syncthreads();
        ok = false;
        break;
      }
      const bool diag = (jt == it);
      if constexpr (CH == 2) {
#pragma unroll 1
        for (int j = 0; j < kTile; ++j) {
          const float4 aj = sj[buf][j];
          const float wj = (diag && j <= tid) ? 0.0f : aj.w;
          unsigned long long nl2, sx, dx, sy, dy;
          pair_setup_pq2c_folded(ai, aj, wj, qp, wide >= 1, nl2, sx, dx, sy, dy);
#pragma unroll
          for (int n = 0; n < Q / 4; ++n) {
            asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc2[2 * n]) : "l"(sx));
            asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc2[2 * n + 1]) : "l"(sy));
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(dx) : "l"(nl2), "l"(sx));
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(dy) : "l"(nl2), "l"(sy));
            asm("add.rn.f32x2 %0, %0, %1;" : "+l"(sx) : "l"(dx));
            asm("add.rn.f32x2 %0, %0, %1;" : "+l"(sy) : "l"(dy));
          }
        }
      } else
#pragma unroll 1
      for (int j = 0; j < kTile; j += JB) {
        unsigned long long u2[JB], nl2[JB], s2[JB], d2[JB];
#pragma unroll
        for (int c = 0; c < JB; ++c) {
          const float4 aj = sj[buf][j + c];
          const float wj = (diag && j + c <= tid) ? 0.0f : aj.w;
          if (FOLD) pair_setup_pq_folded(ai, aj, wj, qp, wide >= 1, nl2[c], s2[c], d2[c]);
          else pair_setup_pq(ai, aj, wj, qp, wide >= 1, u2[c], nl2[c], s2[c], d2[c]);
        }
#pragma unroll
        for (int m = 0; m < Q / 2; ++m) {
#pragma unroll
          for (int c = 0; c < JB; ++c) {
            if (FOLD) asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc2[m]) : "l"(s2[c]));
            else asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc2[m]) : "l"(u2[c]), "l"(s2[c]));
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d2[c]) : "l"(nl2[c]), "l"(s2[c]));
            asm("add.rn.f32x2 %0, %0, %1;" : "+l"(s2[c]) : "l"(d2[c]));
          }
        }
      }
      __syncthreads();
      buf ^= 1;
    }
    if (ok) {
      const int a = min(ti, cur), b = max(ti, cur);
      flush_split<Q>(acc2, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, s_scale);
    }
  }
}

// ---- set-up / recurrence split ---------------------------------------------
// One warpgroup (threads 0-127, one i atom each) computes the folded
// recurrence state (s', d', λ') of every pair of a chunk of kSpJ j atoms into
// a ring of shared-memory stages; two warpgroups (threads 128-383) run only
// the recurrences, each thread one i atom and every other j of the chunk.  The
// set-up work is that of k_pair_fp32_pq, but it leaves the recurrence warps'
// instruction streams: with two recurrence warps and one set-up warp per
// scheduler the FP32 pipe stays fed while a set-up chain waits on its latency.
// Each chunk carries a header {item, j tile, chunk, sequence number}.  The
// recurrence warps take every decision (new item, type change, end) from it,
// per warp, so no barrier spans recurrence warps and a wait that runs out
// (status CRAB_ETIMEOUT) cannot leave another warp waiting: a thread whose wait
// gave up stops waiting, a recurrence warp leaves at the first header whose
// sequence number is not the one it expects, and the set-up warps finish the
// work list.  Nothing is copied asynchronously, so nothing is in flight when a
// CTA leaves.
constexpr int kSpJ = 16;               // j atoms per chunk
constexpr int kSpStages = 4;           // chunks in the ring
constexpr int kSpThreads = 3 * kTile;  // set-up warpgroup + two recurrence warpgroups
struct SpSmem {
  static constexpr int kSd = 0;                                    // ulonglong2 [stage][jj][i]: (s', d')
  static constexpr int kNl = kSd + kSpStages * kSpJ * kTile * 16;  // u64 [stage][jj][i]: λ'
  static constexpr int kSj = kNl + kSpStages * kSpJ * kTile * 8;   // float4 [2][kTile]: j tiles
  static constexpr int kHdr = kSj + 2 * kTile * 16;                // int4 [stage]
  static constexpr int kBar = kHdr + kSpStages * 16;               // u64 full[stage], empty[stage]
  static constexpr int kItem = kBar + 2 * kSpStages * 8;           // int: the set-up warps' next item
  static constexpr int kBytes = kItem + 16;
};
static_assert(kTile % kSpJ == 0 && kSpJ % 4 == 0, "chunks tile the j tile; two warpgroups take alternate j");

__device__ __forceinline__ void sp_arrive(uint64_t* bar) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
// Barrier 1 among the 128 set-up threads only.
__device__ __forceinline__ void sp_setup_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kTile) : "memory"); }

// A bounded wait that gives up once per thread: after the first wait that
// runs out the thread records CRAB_ETIMEOUT and waits no more.
__device__ __forceinline__ void sp_wait(uint64_t* bar, unsigned parity, int budget, bool& ok, int* status) {
  if (!ok) return;
  if (!mbar_wait(bar, parity, budget)) {
    ok = false;
    atomicExch(status, CRAB_ETIMEOUT);
  }
}

// Warp sum of N = Q/2 packed accumulators by recursive halving: at offset o a
// lane keeps the half of its values that its lane bit o selects and adds the
// partner's copy of that half, so after five steps lane L holds the sums of
// packed values [L·P/32, (L+1)·P/32) (P = N rounded up to a multiple of 32):
// 31·P/32 packed shuffles and adds instead of 5·N.  Every lane then adds its
// own q points into the f64 partials.  Resets the accumulators.
template <int Q>
__device__ __forceinline__ void flush_split(unsigned long long (&acc2)[Q / 2], int ab, int qstart, int qcount,
                                            int nq, double* __restrict__ partials, double sc) {
  constexpr int N = Q / 2;
  constexpr int P = (N + 31) / 32 * 32;
  const int lane = threadIdx.x & 31;
  unsigned long long v[P / 2];
  {
    const bool upper = (lane & 16) != 0;
#pragma unroll
    for (int m = 0; m < P / 2; ++m) {
      const unsigned long long lo = m < N ? acc2[m] : 0ull;
      const unsigned long long hi = m + P / 2 < N ? acc2[m + P / 2] : 0ull;
      const unsigned long long got = __shfl_xor_sync(0xffffffffu, upper ? lo : hi, 16);
      asm("add.rn.f32x2 %0, %1, %2;" : "=l"(v[m]) : "l"(upper ? hi : lo), "l"(got));
    }
  }
#pragma unroll
  for (int m = 0; m < N; ++m) acc2[m] = 0ull;
#pragma unroll
  for (int st = 1; st < 5; ++st) {
    const int o = 16 >> st;
    const int half = P >> (st + 1);
    const bool upper = (lane & o) != 0;
#pragma unroll
    for (int m = 0; m < half; ++m) {
      const unsigned long long got = __shfl_xor_sync(0xffffffffu, upper ? v[m] : v[m + half], o);
      asm("add.rn.f32x2 %0, %1, %2;" : "=l"(v[m]) : "l"(upper ? v[m + half] : v[m]), "l"(got));
    }
  }
  constexpr int per = P / 32;
#pragma unroll
  for (int m = 0; m < per; ++m) {
    const int k = 2 * (lane * per + m);
    float a, b;
    unpack2(v[m], a, b);
    if (k < qcount) atomicAdd(&partials[(size_t)ab * nq + qstart + k], on_grid((double)a, sc));
    if (k + 1 < qcount) atomicAdd(&partials[(size_t)ab * nq + qstart + k + 1], on_grid((double)b, sc));
  }
}

template <int Q, int JB>
__global__ void __launch_bounds__(kSpThreads, 1)
    k_pair_split(const float4* __restrict__ atoms, const int* __restrict__ tile_type, const int4* __restrict__ work,
                 int n_work, const float4* __restrict__ qpar, const int2* __restrict__ qrange, int nq, int T,
                 int wide, double* __restrict__ partials, int* __restrict__ status, int* __restrict__ next_work,
                 const int64_t* __restrict__ work_out,
                const double* __restrict__ item_scale, int budget) {
  static_assert(Q % 2 == 0, "q-packed blocks hold an even number of q points");
  static_assert(kSpJ % (2 * JB) == 0, "each warpgroup takes JB of its j atoms per step");
  extern __shared__ __align__(16) unsigned char sp_smem[];
  ulonglong2* sd = (ulonglong2*)(sp_smem + SpSmem::kSd);
  unsigned long long* nlb = (unsigned long long*)(sp_smem + SpSmem::kNl);
  float4* sj = (float4*)(sp_smem + SpSmem::kSj);
  int4* hdr = (int4*)(sp_smem + SpSmem::kHdr);
  uint64_t* full = (uint64_t*)(sp_smem + SpSmem::kBar);
  uint64_t* empty = full + kSpStages;
  int* s_item = (int*)(sp_smem + SpSmem::kItem);
  const int tid = threadIdx.x;
  if (tid < kSpStages) {
    mbar_init(&full[tid], kTile);
    mbar_init(&empty[tid], 2 * kTile);
    hdr[tid] = make_int4(-1, -1, -1, -1);
  }
  if (tid == 0) fence_mbar_init();
  __syncthreads();
  if (budget < 0) budget = kWaitBudget;  // the context's default
  bool ok = true;

  if (tid < kTile) {
    // ---- set-up warpgroup: thread i = tid ----
    int n = 0, buf = 0;
    for (;;) {
      if (tid == 0) *s_item = atomicAdd(next_work, 1);
      sp_setup_sync();
      const int w = *s_item;  // thread 0 writes it again only after the tile barrier below
      if (w >= n_work) {
        const int stage = n % kSpStages;
        sp_wait(&empty[stage], ((n / kSpStages) & 1) ^ 1, budget, ok, status);
        if (tid == 0) hdr[stage] = make_int4(-1, 0, 0, n);
        sp_arrive(&full[stage]);
        break;
      }
      const int4 wk = work[w];
      const int it = wk.x, jt0 = wk.y, jt1 = wk.z;
      const float4 ai = atoms[(size_t)it * kTile + tid];
      const float4 qp = qpar[wk.w];
      float4 v = atoms[(size_t)jt0 * kTile + tid];
      for (int jt = jt0; jt < jt1; ++jt) {
        sj[buf * kTile + tid] = v;
        sp_setup_sync();  // the tile is in place; every reader of this buffer's previous tile is past it
        if (jt + 1 < jt1) v = atoms[(size_t)(jt + 1) * kTile + tid];
        const bool diag = (jt == it);
        const float4* tj = sj + buf * kTile;
#pragma unroll 1
        for (int c = 0; c < kTile / kSpJ; ++c, ++n) {
          const int stage = n % kSpStages;
          sp_wait(&empty[stage], ((n / kSpStages) & 1) ^ 1, budget, ok, status);
          ulonglong2* sdo = sd + (size_t)stage * kSpJ * kTile + tid;
          unsigned long long* nlo = nlb + (size_t)stage * kSpJ * kTile + tid;
#pragma unroll 4
          for (int jj = 0; jj < kSpJ; ++jj) {
            const int j = c * kSpJ + jj;
            const float4 aj = tj[j];
            const float wj = (diag && j <= tid) ? 0.0f : aj.w;
            unsigned long long nl2, s2, d2;
            pair_setup_pq_folded(ai, aj, wj, qp, wide >= 1, nl2, s2, d2);
            sdo[jj * kTile] = make_ulonglong2(s2, d2);
            nlo[jj * kTile] = nl2;
          }
          if (tid == 0) hdr[stage] = make_int4(w, jt, c, n);
          sp_arrive(&full[stage]);
        }
        buf ^= 1;
      }
    }
    return;
  }

  // ---- recurrence warpgroups: thread i = (tid - 128) % 128, j parity g ----
  const int r = tid - kTile, g = r / kTile, i = r % kTile;
  unsigned long long acc2[Q / 2];
#pragma unroll
  for (int m = 0; m < Q / 2; ++m) acc2[m] = 0ull;
  int cur_w = -1, ti = 0, cur = 0, jlo = 0, jhi = 0;
  int2 qr = make_int2(0, 0);
  double* __restrict__ out = partials;
  double sc = 1.0;
  for (int n = 0;; ++n) {
    const int stage = n % kSpStages;
    sp_wait(&full[stage], (n / kSpStages) & 1, budget, ok, status);
    int4 h = hdr[stage];
    h.x = __shfl_sync(0xffffffffu, h.x, 0);
    h.y = __shfl_sync(0xffffffffu, h.y, 0);
    h.z = __shfl_sync(0xffffffffu, h.z, 0);
    h.w = __shfl_sync(0xffffffffu, h.w, 0);
    if (h.w != n || h.x < 0 || h.x >= n_work) break;  // the end, or a ring that a failed wait left behind
    if (h.x != cur_w) {
      if (cur_w >= 0) {
        const int a = min(ti, cur), b = max(ti, cur);
        flush_split<Q>(acc2, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, sc);
      }
      const int4 wk = work[h.x];
      cur_w = h.x;
      ti = tile_type[wk.x];
      cur = tile_type[wk.y];
      jlo = wk.y;
      jhi = wk.z;
      qr = qrange[wk.w];
      out = partials + (work_out ? work_out[h.x] : 0);
      sc = item_scale[h.x];
    }
    if (h.y < jlo || h.y >= jhi) break;
    if (h.z == 0) {
      const int tj = tile_type[h.y];
      if (tj != cur) {
        const int a = min(ti, cur), b = max(ti, cur);
        flush_split<Q>(acc2, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, sc);
        cur = tj;
      }
    }
    const ulonglong2* sdi = sd + (size_t)stage * kSpJ * kTile + i;
    const unsigned long long* nli = nlb + (size_t)stage * kSpJ * kTile + i;
#pragma unroll 1
    for (int jj = g; jj < kSpJ; jj += 2 * JB) {
      unsigned long long s2[JB], d2[JB], nl2[JB];
#pragma unroll
      for (int c = 0; c < JB; ++c) {
        const ulonglong2 x = sdi[(jj + 2 * c) * kTile];
        s2[c] = x.x;
        d2[c] = x.y;
        nl2[c] = nli[(jj + 2 * c) * kTile];
      }
#pragma unroll
      for (int m = 0; m < Q / 2; ++m) {
#pragma unroll
        for (int c = 0; c < JB; ++c) {
          asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc2[m]) : "l"(s2[c]));
          asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d2[c]) : "l"(nl2[c]), "l"(s2[c]));
          asm("add.rn.f32x2 %0, %0, %1;" : "+l"(s2[c]) : "l"(d2[c]));
        }
      }
    }
    sp_arrive(&empty[stage]);
  }
  if (cur_w >= 0) {
    const int a = min(ti, cur), b = max(ti, cur);
    flush_split<Q>(acc2, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, sc);
  }
}

// ---- set-up / recurrence split over three q blocks ------------------------
// The same ring as k_pair_split, with one recurrence warpgroup per q block:
// a work item covers kS3Blocks consecutive q blocks, the set-up warpgroup
// computes each pair's distance and weight once and its seed for every block,
// and recurrence warpgroup b runs block b of the item over every j of the
// chunk.  512 threads leave 128 registers per thread, so 12 recurrence warps
// per SM run blocks of up to about 100 q (three per scheduler where
// k_pair_split has two).  A warpgroup whose block lies past the end of the q
// grid consumes the chunks without computing.
constexpr int kS3Blocks = 3;
constexpr int kS3J = 8;        // j atoms per chunk
constexpr int kS3Stages = 3;
constexpr int kS3Threads = (1 + kS3Blocks) * kTile;
struct S3Smem {
  static constexpr int kSd = 0;  // ulonglong2 [stage][block][jj][i]: (s', d')
  static constexpr int kNl = kSd + kS3Stages * kS3Blocks * kS3J * kTile * 16;  // float [stage][block][jj][i]: λ'
  static constexpr int kSj = kNl + kS3Stages * kS3Blocks * kS3J * kTile * 4;  // float4 [2][kTile]
  static constexpr int kHdr = kSj + 2 * kTile * 16;                           // int4 [stage]
  static constexpr int kBar = kHdr + kS3Stages * 16;                          // u64 full[stage], empty[stage]
  static constexpr int kItem = kBar + 2 * kS3Stages * 8;
  static constexpr int kBytes = kItem + 16;
};
static_assert(kTile % kS3J == 0, "chunks tile the j tile");

template <int Q>
__global__ void __launch_bounds__(kS3Threads, 1)
    k_pair_split3(const float4* __restrict__ atoms, const int* __restrict__ tile_type, const int4* __restrict__ work,
                  int n_work, const float4* __restrict__ qpar, const int2* __restrict__ qrange, int n_qblocks,
                  int nq, int T, int wide, double* __restrict__ partials, int* __restrict__ status,
                  int* __restrict__ next_work, const int64_t* __restrict__ work_out,
                const double* __restrict__ item_scale, int budget) {
  static_assert(Q % 2 == 0, "q-packed blocks hold an even number of q points");
  extern __shared__ __align__(16) unsigned char s3_smem[];
  ulonglong2* sd = (ulonglong2*)(s3_smem + S3Smem::kSd);
  float* nlb = (float*)(s3_smem + S3Smem::kNl);
  float4* sj = (float4*)(s3_smem + S3Smem::kSj);
  int4* hdr = (int4*)(s3_smem + S3Smem::kHdr);
  uint64_t* full = (uint64_t*)(s3_smem + S3Smem::kBar);
  uint64_t* empty = full + kS3Stages;
  int* s_item = (int*)(s3_smem + S3Smem::kItem);
  constexpr int kStage = kS3Blocks * kS3J * kTile;  // states per stage
  const int tid = threadIdx.x;
  if (tid < kS3Stages) {
    mbar_init(&full[tid], kTile);
    mbar_init(&empty[tid], kS3Blocks * kTile);
    hdr[tid] = make_int4(-1, -1, -1, -1);
  }
  if (tid == 0) fence_mbar_init();
  __syncthreads();
  if (budget < 0) budget = kWaitBudget;
  bool ok = true;

  if (tid < kTile) {
    // ---- set-up warpgroup: thread i = tid ----
    int n = 0, buf = 0;
    for (;;) {
      if (tid == 0) *s_item = atomicAdd(next_work, 1);
      sp_setup_sync();
      const int w = *s_item;
      if (w >= n_work) {
        const int stage = n % kS3Stages;
        sp_wait(&empty[stage], ((n / kS3Stages) & 1) ^ 1, budget, ok, status);
        if (tid == 0) hdr[stage] = make_int4(-1, 0, 0, n);
        sp_arrive(&full[stage]);
        break;
      }
      const int4 wk = work[w];
      const int it = wk.x, jt0 = wk.y, jt1 = wk.z;
      const int b0 = wk.w * kS3Blocks;
      const int nb = min(kS3Blocks, n_qblocks - b0);
      const float4 ai = atoms[(size_t)it * kTile + tid];
      float4 qp[kS3Blocks];
#pragma unroll
      for (int b = 0; b < kS3Blocks; ++b) qp[b] = qpar[b0 + min(b, nb - 1)];
      float4 v = atoms[(size_t)jt0 * kTile + tid];
      for (int jt = jt0; jt < jt1; ++jt) {
        sj[buf * kTile + tid] = v;
        sp_setup_sync();
        if (jt + 1 < jt1) v = atoms[(size_t)(jt + 1) * kTile + tid];
        const bool diag = (jt == it);
        const float4* tj = sj + buf * kTile;
#pragma unroll 1
        for (int c = 0; c < kTile / kS3J; ++c, ++n) {
          const int stage = n % kS3Stages;
          sp_wait(&empty[stage], ((n / kS3Stages) & 1) ^ 1, budget, ok, status);
          ulonglong2* sdo = sd + (size_t)stage * kStage + tid;
          float* nlo = nlb + (size_t)stage * kStage + tid;
#pragma unroll 2
          for (int jj = 0; jj < kS3J; ++jj) {
            const int j = c * kS3J + jj;
            const float4 aj = tj[j];
            const float wj = (diag && j <= tid) ? 0.0f : aj.w;
            float r, u;
            pair_geom(ai, aj, wj, r, u);
            const unsigned long long u2 = pack2(u, u);
#pragma unroll
            for (int b = 0; b < kS3Blocks; ++b) {
              float nl, S, sB, dA, dB;
              pair_seed_pq(r, qp[b], wide, nl, S, sB, dA, dB);
              unsigned long long s2 = pack2(S, sB), d2 = pack2(dA, dB);
              asm("mul.rn.f32x2 %0, %0, %1;" : "+l"(s2) : "l"(u2));
              asm("mul.rn.f32x2 %0, %0, %1;" : "+l"(d2) : "l"(u2));
              sdo[(b * kS3J + jj) * kTile] = make_ulonglong2(s2, d2);
              nlo[(b * kS3J + jj) * kTile] = nl;
            }
          }
          if (tid == 0) hdr[stage] = make_int4(w, jt, c, n);
          sp_arrive(&full[stage]);
        }
        buf ^= 1;
      }
    }
    return;
  }

  // ---- recurrence warpgroups: thread i = (tid - 128) % 128, q block b of the item ----
  const int r = tid - kTile, blk = r / kTile, i = r % kTile;
  unsigned long long acc2[Q / 2];
#pragma unroll
  for (int m = 0; m < Q / 2; ++m) acc2[m] = 0ull;
  int cur_w = -1, ti = 0, cur = 0, jlo = 0, jhi = 0;
  bool live = false;  // this warpgroup's block of the current item exists
  int2 qr = make_int2(0, 0);
  double* __restrict__ out = partials;
  double sc = 1.0;
  for (int n = 0;; ++n) {
    const int stage = n % kS3Stages;
    sp_wait(&full[stage], (n / kS3Stages) & 1, budget, ok, status);
    int4 h = hdr[stage];
    h.x = __shfl_sync(0xffffffffu, h.x, 0);
    h.y = __shfl_sync(0xffffffffu, h.y, 0);
    h.z = __shfl_sync(0xffffffffu, h.z, 0);
    h.w = __shfl_sync(0xffffffffu, h.w, 0);
    if (h.w != n || h.x < 0 || h.x >= n_work) break;
    if (h.x != cur_w) {
      if (live) {
        const int a = min(ti, cur), b = max(ti, cur);
        flush_split<Q>(acc2, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, sc);
      }
      const int4 wk = work[h.x];
      cur_w = h.x;
      const int qb = wk.w * kS3Blocks + blk;
      live = qb < n_qblocks;
      ti = tile_type[wk.x];
      cur = tile_type[wk.y];
      jlo = wk.y;
      jhi = wk.z;
      qr = live ? qrange[qb] : make_int2(0, 0);
      out = partials + (work_out ? work_out[h.x] : 0);
      sc = item_scale[h.x];
    }
    if (h.y < jlo || h.y >= jhi) break;
    if (h.z == 0) {
      const int tj = tile_type[h.y];
      if (tj != cur) {
        if (live) {
          const int a = min(ti, cur), b = max(ti, cur);
          flush_split<Q>(acc2, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, sc);
        }
        cur = tj;
      }
    }
    if (live) {
      const ulonglong2* sdi = sd + (size_t)stage * kStage + (size_t)blk * kS3J * kTile + i;
      const float* nli = nlb + (size_t)stage * kStage + (size_t)blk * kS3J * kTile + i;
#pragma unroll 1
      for (int jj = 0; jj < kS3J; ++jj) {
        const ulonglong2 x = sdi[jj * kTile];
        unsigned long long s2 = x.x, d2 = x.y;
        const float nl = nli[jj * kTile];
        const unsigned long long nl2 = pack2(nl, nl);
#pragma unroll
        for (int m = 0; m < Q / 2; ++m) {
          asm("add.rn.f32x2 %0, %0, %1;" : "+l"(acc2[m]) : "l"(s2));
          asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d2) : "l"(nl2), "l"(s2));
          asm("add.rn.f32x2 %0, %0, %1;" : "+l"(s2) : "l"(d2));
        }
      }
    }
    sp_arrive(&empty[stage]);
  }
  if (live) {
    const int a = min(ti, cur), b = max(ti, cur);
    flush_split<Q>(acc2, a * T - a * (a - 1) / 2 + (b - a), qr.x, qr.y, nq, out, sc);
  }
}

// FP64 reference: direct sinc per pair and q, QD q values per work item.
constexpr int kQD = 8;
__global__ void __launch_bounds__(kThreads)
    k_pair_fp64(const double4* __restrict__ atoms, const int* __restrict__ tile_type, const int4* __restrict__ work,
                int n_work, const double* __restrict__ q, int nq, int T, double* __restrict__ partials) {
  __shared__ double4 sj[kTile];
  __shared__ double red[kThreads / 32][kQD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
    const int4 wk = work[w];
    const int it = wk.x, jt0 = wk.y, jt1 = wk.z, qb = wk.w;
    const double4 ai = atoms[(size_t)it * kTile + tid];
    const int qstart = qb * kQD, qcount = min(kQD, nq - qstart);
    double qv[kQD], acc[kQD];
#pragma unroll
    for (int k = 0; k < kQD; ++k) {
      qv[k] = (k < qcount) ? q[qstart + k] : 0.0;
      acc[k] = 0.0;
    }
    const int ti = tile_type[it];
    int cur = tile_type[jt0];
    auto flush = [&](int tj) {
      const int a = min(ti, tj), b = max(ti, tj);
      const int ab = a * T - a * (a - 1) / 2 + (b - a);
#pragma unroll
      for (int k = 0; k < kQD; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
        acc[k] = 0.0;
      }
      __syncthreads();
      if (tid < qcount) {
        double s = 0.0;
        for (int w2 = 0; w2 < kThreads / 32; ++w2) s += red[w2][tid];
        atomicAdd(&partials[(size_t)ab * nq + qstart + tid], s);
      }
      __syncthreads();
    };
    for (int jt = jt0; jt < jt1; ++jt) {
      const int tj = tile_type[jt];
      if (tj != cur) {
        flush(cur);
        cur = tj;
      }
      sj[tid] = atoms[(size_t)jt * kTile + tid];
      __syncthreads();
      const bool diag = (jt == it);
      for (int j = 0; j < kTile; ++j) {
        const double4 aj = sj[j];
        const double wij = (diag && j <= tid) ? 0.0 : ai.w * aj.w;
        const double dx = ai.x - aj.x, dy = ai.y - aj.y, dz = ai.z - aj.z;
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
#pragma unroll
        for (int k = 0; k < kQD; ++k) {
          const double x = qv[k] * r;
          const double s = fabs(x) < 1e-8 ? 1.0 : sin(x) / x;
          acc[k] = fma(wij, s, acc[k]);
        }
      }
      __syncthreads();
    }
    flush(cur);
  }
}

uint32_t morton10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Work list: i tile x runs of up to `run` j tiles (j >= i) x q blocks.
// Tile pairs with both tiles at or beyond `skip_from` are left out (that
// block is summed elsewhere).  Items are ordered longest first; equal-cost
// items keep the q block fastest so concurrently running CTAs add into
// different q ranges.
std::vector<int4> make_work(const Layout& L, int n_qblocks, int run, int skip_from) {
  static thread_local std::vector<std::pair<int, int4>> items;  // keeps its capacity (and pages) across calls
  items.clear();
  for (int it = 0; it < L.n_tiles; ++it) {
    if (it >= skip_from) break;
    for (int j0 = it; j0 < L.n_tiles; j0 += run) {
      const int j1 = std::min(j0 + run, L.n_tiles);
      const int cost = 2 * (j1 - j0) - (j0 == it ? 1 : 0);
      for (int b = 0; b < n_qblocks; ++b) items.push_back({cost, make_int4(it, j0, j1, b)});
    }
  }
  // stable sort by cost, longest first: costs are 1 .. 2 * run, so one
  // counting pass places every item
  std::vector<size_t> start((size_t)2 * run + 2, 0);
  for (const auto& it : items) ++start[(size_t)(2 * run - it.first) + 1];
  for (size_t c = 1; c < start.size(); ++c) start[c] += start[c - 1];
  std::vector<int4> work(items.size());
  for (const auto& it : items) work[start[(size_t)(2 * run - it.first)]++] = it.second;
  return work;
}

template <int Q, int JB>
void launch_fp32(cudaStream_t stream, int sm_count, const float4* atoms, const int* tt, const int4* work, int n_work,
                 const float4* qpar, const int2* qrange, int nq, int T, int wide, double* partials, int* status,
                 int* next_work, const int64_t* work_out, const double* item_scale,
                    int budget) {
  int per_sm = 0;
  CRAB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_fp32<Q, JB>, kThreads, 0));
  int grid = std::max(1, std::min(n_work, sm_count * std::max(per_sm, 1)));
  k_pair_fp32<Q, JB><<<grid, kThreads, 0, stream>>>(atoms, tt, work, n_work, qpar, qrange, nq, T, wide, partials,
                                                     status, next_work, work_out, item_scale, budget);
  CRAB_CUDA_CHECK(cudaGetLastError());
}

template <int Q, int JB, int OCC, bool FOLD = false, int CH = 1>
void launch_fp32_pq(cudaStream_t stream, int sm_count, const float4* atoms, const int* tt, const int4* work,
                    int n_work, const float4* qpar, const int2* qrange, int nq, int T, int wide, double* partials,
                    int* status, int* next_work, const int64_t* work_out, const double* item_scale,
                    int budget) {
  int per_sm = 0;
  CRAB_CUDA_CHECK(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_fp32_pq<Q, JB, OCC, FOLD, CH>, kThreads, 0));
  int grid = std::max(1, std::min(n_work, sm_count * std::max(per_sm, 1)));
  k_pair_fp32_pq<Q, JB, OCC, FOLD, CH><<<grid, kThreads, 0, stream>>>(atoms, tt, work, n_work, qpar, qrange, nq, T, wide, partials,
                                                        status, next_work, work_out, item_scale, budget);
  CRAB_CUDA_CHECK(cudaGetLastError());
}

template <int Q, int JB>
void launch_split(cudaStream_t stream, int sm_count, const float4* atoms, const int* tt, const int4* work, int n_work,
                  const float4* qpar, const int2* qrange, int nq, int T, int wide, double* partials, int* status,
                  int* next_work, const int64_t* work_out, const double* item_scale,
                    int budget) {
  static bool attr = false;  // one CTA per SM: the ring takes most of the shared memory
  if (!attr) {
    CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_pair_split<Q, JB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         SpSmem::kBytes));
    attr = true;
  }
  const int grid = std::max(1, std::min(n_work, sm_count));
  k_pair_split<Q, JB><<<grid, kSpThreads, SpSmem::kBytes, stream>>>(atoms, tt, work, n_work, qpar, qrange, nq, T,
                                                                    wide, partials, status, next_work, work_out,
                                                                    item_scale, budget);
  CRAB_CUDA_CHECK(cudaGetLastError());
}

template <int Q>
void launch_split3(cudaStream_t stream, int sm_count, const float4* atoms, const int* tt, const int4* work,
                   int n_work, const float4* qpar, const int2* qrange, int n_qblocks, int nq, int T, int wide,
                   double* partials, int* status, int* next_work, const int64_t* work_out, const double* item_scale,
                    int budget) {
  static bool attr = false;
  if (!attr) {
    CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_pair_split3<Q>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         S3Smem::kBytes));
    attr = true;
  }
  const int grid = std::max(1, std::min(n_work, sm_count));
  k_pair_split3<Q><<<grid, kS3Threads, S3Smem::kBytes, stream>>>(atoms, tt, work, n_work, qpar, qrange, n_qblocks,
                                                                 nq, T, wide, partials, status, next_work, work_out,
                                                                 item_scale, budget);
  CRAB_CUDA_CHECK(cudaGetLastError());
}

template <class T>
T* upload(crab_ctx* ctx, PairPlan& P, std::vector<void*>& list, const char* name, const T* src, size_t count,
          cudaStream_t s) {
  void* p = plan_alloc(ctx, P, list, name, std::max<size_t>(count, 1) * sizeof(T));
  if (count && src) copy_h2d(ctx, p, src, count * sizeof(T), s);
  return (T*)p;
}

}  // namespace

Layout build_layout(const double* xyz, const double* w, const int32_t* type, int64_t n, int T, bool with_f64,
                    bool spatial) {
  Layout L;
  L.T = T;
  L.n = n;
  L.self_w2.assign(T, 0.0);
  L.sum_w.assign(T, 0.0);
  double c[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) c[d] += xyz[3 * i + d];
  for (int d = 0; d < 3; ++d) c[d] = n ? c[d] / (double)n : 0.0;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, rmax = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double r2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      double v = xyz[3 * i + d] - c[d];
      lo[d] = std::min(lo[d], v);
      hi[d] = std::max(hi[d], v);
      r2 += v * v;
    }
    rmax = std::max(rmax, std::sqrt(r2));
  }
  L.extent = 2.0 * rmax;
  // order: type, then (spatial) the 30-bit Morton code of the centred
  // position, ties by input index (a counting sort by type, then a stable LSD
  // radix sort of the packed (Morton code, index) words within each type,
  // three 10-bit digits); without `spatial`, type then input index
  require(n < ((int64_t)1 << 32), "at most 2^32 - 1 atoms per pair problem");
  static const std::vector<uint32_t> spread = [] {
    std::vector<uint32_t> t(1024);
    for (uint32_t v = 0; v < 1024; ++v) t[v] = morton10(v);
    return t;
  }();
  double scale[3];
  for (int d = 0; d < 3; ++d) scale[d] = 1024.0 / std::max(hi[d] - lo[d], 1e-9);
  std::vector<int64_t> count(T, 0);
  for (int64_t i = 0; i < n; ++i) count[type[i]]++;
  std::vector<int64_t> tstart(T + 1, 0);
  for (int t = 0; t < T; ++t) tstart[t + 1] = tstart[t] + count[t];
  // sort scratch kept per host thread with its capacity, so repeated calls
  // reuse its pages instead of faulting in fresh ones
  static thread_local std::vector<uint64_t> word, tmp;
  static thread_local std::vector<int64_t> order;
  word.resize((size_t)n);
  tmp.resize((size_t)n);
  {
    std::vector<int64_t> pos(tstart.begin(), tstart.end() - 1);
    for (int64_t i = 0; i < n; ++i) {
      uint32_t m = 0;
      if (spatial)
        for (int d = 0; d < 3; ++d) {
          const double cell = (xyz[3 * i + d] - c[d] - lo[d]) * scale[d];
          const int ci = cell <= 0.0 ? 0 : (cell >= 1023.0 ? 1023 : (int)cell);
          m |= spread[ci] << d;
        }
      word[pos[type[i]]++] = ((uint64_t)m << 32) | (uint64_t)i;
    }
  }
  for (int t = 0; t < T && spatial; ++t) {
    const int64_t a = tstart[t], b = tstart[t + 1];
    for (int shift = 32; shift < 62; shift += 10) {
      int64_t digit[1025] = {0};
      for (int64_t k = a; k < b; ++k) digit[((word[k] >> shift) & 1023u) + 1]++;
      for (int d = 0; d < 1024; ++d) digit[d + 1] += digit[d];
      for (int64_t k = a; k < b; ++k) tmp[a + digit[(word[k] >> shift) & 1023u]++] = word[k];
      std::copy(tmp.begin() + a, tmp.begin() + b, word.begin() + a);
    }
  }
  order.resize((size_t)n);
  for (int64_t k = 0; k < n; ++k) order[k] = (int64_t)(word[k] & 0xffffffffu);
  int64_t n_pad = 0;
  for (int t = 0; t < T; ++t) n_pad += (count[t] + kTile - 1) / kTile * kTile;
  L.n_pad = n_pad;
  L.n_tiles = (int)(n_pad / kTile);
  L.atoms.assign((size_t)n_pad * 4, 0.0f);
  if (with_f64) L.atoms64.assign((size_t)n_pad * 4, 0.0);
  L.tile_type.resize(L.n_tiles);
  L.source.assign((size_t)n_pad, -1);
  int64_t slot = 0, k = 0;
  for (int t = 0; t < T; ++t) {
    const int64_t start = slot;
    for (int64_t m = 0; m < count[t]; ++m, ++k, ++slot) {
      const int64_t i = order[k];
      for (int d = 0; d < 3; ++d) {
        const double v = xyz[3 * i + d] - c[d];
        L.atoms[4 * slot + d] = (float)v;
        if (with_f64) L.atoms64[4 * slot + d] = v;
      }
      L.atoms[4 * slot + 3] = (float)w[i];
      L.source[slot] = i;
      if (with_f64) L.atoms64[4 * slot + 3] = w[i];
      L.self_w2[t] += w[i] * w[i];
      L.sum_w[t] += w[i];
    }
    slot = start + (count[t] + kTile - 1) / kTile * kTile;
    for (int64_t tt = start / kTile; tt < slot / kTile; ++tt) L.tile_type[tt] = t;
  }
  return L;
}

bool q_grid_uniform(const double* q, int64_t nq) {
  if (nq < 3) return true;
  const double dq = (q[nq - 1] - q[0]) / (double)(nq - 1);
  const double tol = 1e-9 * std::max(std::fabs(q[nq - 1]), 1e-12);
  for (int64_t k = 1; k < nq; ++k)
    if (std::fabs(q[k] - (q[0] + (double)k * dq)) > tol) return false;
  return true;
}

PairPlan::~PairPlan() {
  for (void* p : owned) cudaFree(p);
  for (void* p : qcfg) cudaFree(p);
}

// q blocks: greedy runs of at most Qmax uniformly spaced q values, each
// seeded exactly at its first point (any non-decreasing grid works).
std::vector<int2> q_blocks(const std::vector<double>& q, int Qmax) {
  std::vector<int2> out;
  const int64_t nq = (int64_t)q.size();
  if (nq == 0) return out;
  const double tol = 1e-9 * std::max(std::fabs(q[nq - 1]), 1e-12);
  int64_t s0 = 0;
  while (s0 < nq) {
    int64_t e = s0 + 1;
    if (e < nq) {
      const double dq = q[s0 + 1] - q[s0];
      e = s0 + 2;
      while (e < nq && e - s0 < Qmax && std::fabs(q[e] - (q[s0] + (double)(e - s0) * dq)) <= tol) ++e;
    }
    out.push_back(make_int2((int)s0, (int)(e - s0)));
    s0 = e;
  }
  return out;
}

std::vector<int32_t> shard_owners(const int64_t* cost, int64_t n, int n_shards) {
  require(n_shards >= 1, "shard count must be positive");
  std::vector<int64_t> load((size_t)n_shards, 0);
  std::vector<int32_t> owner((size_t)std::max<int64_t>(n, 0));
  for (int64_t i = 0; i < n; ++i) {
    int best = 0;
    for (int s = 1; s < n_shards; ++s)
      if (load[s] < load[best]) best = s;
    owner[i] = best;
    load[best] += cost[i];
  }
  return owner;
}

// Tile pairs of one work item (i tile, j tiles j0..j1): the diagonal tile
// counts once.
inline int64_t work_cost(const int4& w) { return 2 * (int64_t)(w.z - w.y) - (w.y == w.x ? 1 : 0); }

// The items of `work` that shard `shard` owns, in their order.
std::vector<int4> shard_work(const std::vector<int4>& work, int shard, int n_shards) {
  if (n_shards <= 1) return work;
  std::vector<int64_t> cost(work.size());
  for (size_t i = 0; i < work.size(); ++i) cost[i] = work_cost(work[i]);
  const std::vector<int32_t> owner = shard_owners(cost.data(), (int64_t)cost.size(), n_shards);
  std::vector<int4> mine;
  for (size_t i = 0; i < work.size(); ++i)
    if (owner[i] == shard) mine.push_back(work[i]);
  return mine;
}

// Work list of a batch: every segment (one structure's tiles) is tiled on its
// own; items of all segments are ordered longest first and carry the output
// offset of their segment.
void make_work_segments(const PairPlan& P, int n_qblocks, int run, std::vector<int4>& work,
                        std::vector<int64_t>& out) {
  std::vector<std::pair<int, std::pair<int4, int64_t>>> items;
  const int K = (int)P.segments.size() - 1;
  for (int c = 0; c < K; ++c) {
    const int t0 = P.segments[c], t1 = P.segments[c + 1];
    const int64_t base = (int64_t)c * P.n_pairs * P.nq;
    for (int it = t0; it < t1; ++it)
      for (int j0 = it; j0 < t1; j0 += run) {
        const int j1 = std::min(j0 + run, t1);
        const int cost = 2 * (j1 - j0) - (j0 == it ? 1 : 0);
        for (int b = 0; b < n_qblocks; ++b) items.push_back({cost, {make_int4(it, j0, j1, b), base}});
      }
  }
  // stable sort by cost, longest first (costs 1 .. 2 * run): one counting pass
  std::vector<size_t> start((size_t)2 * run + 2, 0);
  for (const auto& it : items) ++start[(size_t)(2 * run - it.first) + 1];
  for (size_t c = 1; c < start.size(); ++c) start[c] += start[c - 1];
  work.resize(items.size());
  out.resize(items.size());
  for (const auto& it : items) {
    const size_t k = start[(size_t)(2 * run - it.first)]++;
    work[k] = it.second.first;
    out[k] = it.second.second;
  }
}

// Untuned choice of (Q, jb): the block length by a cost model (launched steps
// of 3 FP32 ops each plus a per-pair seed of about 60 ops per block), and the
// q-packed kernel where it is compiled for that length (one chain and three
// CTAs per SM at Q = 100, 126 and 128; one chain and two CTAs at Q = 150 and
// 168, whose fewer seeds per pair outweigh the lower occupancy: 3 x 168 for
// 500 q and 2 x 150 for 300 q are 1.3 % and 3 % faster than 4 x 126 and
// 3 x 100; two chains below Q = 100), with the weight folded in where that
// build exists, and two chains per pair at 168.
int2 default_variant(const std::vector<double>& q) {
  int bestQ = 64;
  long best_cost = -1;
  for (int Qc : kQBlocks) {
    const long cost = (long)q_blocks(q, Qc).size() * (3 * Qc + 60);
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      bestQ = Qc;
    }
  }
  // the folded builds (pair weight in the recurrence state), which the
  // autotuner measured 0.5-1.3 % faster than the unfolded ones
  if (bestQ == 126 || bestQ == 100) return make_int2(bestQ, kFolded1x3);
  if (bestQ == 128) return make_int2(bestQ, 1 + kPackedQ + kDenser);
  // 75 or 84 packed accumulators: two CTAs per SM; at Q = 150 two chains per
  // thread (1.4 % faster on the 300-q ensemble pass, 1.7 % at 500 q), at 168 one
  // 168: two chains per pair (4.8 % faster than one at 500 q)
  if (bestQ == 150) return make_int2(bestQ, kFolded2);
  if (bestQ == 168) return make_int2(bestQ, kFolded2c);
  const bool packed = bestQ == 64 || bestQ == 96;
  return make_int2(bestQ, packed ? 2 + kPackedQ : 2);
}

// (Re)build the q blocks and the work list of an FP32 plan for block length Q.
void configure_fp32(crab_ctx* ctx, PairPlan& P, int Q, int jb) {
  P.jb = jb;
  for (void* p : P.qcfg) cudaFree(p);
  P.qcfg.clear();
  P.d_work_out = nullptr;
  const std::vector<int2> qrange = q_blocks(P.q, Q);
  P.Q = Q;
  P.n_qblocks = (int)qrange.size();
  std::vector<float4> qpar(P.n_qblocks);
  double max_half = 0.0;
  for (int b = 0; b < P.n_qblocks; ++b) {
    const int64_t st = qrange[b].x, cnt = qrange[b].y;
    const double q0 = P.q[st];
    const double half = cnt > 1 ? 0.5 * (P.q[st + cnt - 1] - P.q[st]) / (double)(cnt - 1) : 0.0;
    const float q0h = (float)q0, hh = (float)half;
    qpar[b] = make_float4(q0h, (float)(q0 - (double)q0h), hh, (float)(half - (double)hh));
    max_half = std::max(max_half, std::fabs(half));
  }
  // largest half step angle h = Δr/2: above 0.8 rad both kernels seed the
  // step by range reduction (2), above 0.125 rad only the q-packed one,
  // whose step is 2h (1); otherwise both use short polynomials (0)
  const double hmax = max_half * (P.L.extent + 1.0);
  P.wide = hmax > 0.8 ? 2 : (hmax > 0.125 ? 1 : 0);
  P.hmax = hmax;
  // work items name a q block, or for k_pair_split3 a group of kS3Blocks
  const int item_blocks = jb == kSplit3 ? (P.n_qblocks + kS3Blocks - 1) / kS3Blocks : P.n_qblocks;
  // Fixed-point grid of each structure's partials: the largest power of two
  // 2^e with q_max (Σ|w|)² 2^e < 2^52.  Every pair term w_i w_j sin(q r)/r
  // is at most |w_i w_j| q in magnitude, so every sum of the structure's
  // terms stays below 2^52 steps of 2^-e, and f64 sums of values on that grid
  // are exact in any order.
  double qmax = 0.0;
  for (double v : P.q) qmax = std::max(qmax, std::fabs(v));
  auto scale_of = [&](int t0, int t1) {
    double s1 = 0.0;
    for (int64_t k = (int64_t)t0 * kTile; k < (int64_t)t1 * kTile; ++k) s1 += std::fabs((double)P.L.atoms[4 * k + 3]);
    const double bound = qmax * s1 * s1;
    if (!(bound > 0.0) || !std::isfinite(bound)) return 1.0;
    int ex = 0;
    std::frexp(bound, &ex);  // bound < 2^ex
    return std::ldexp(1.0, std::max(-1000, std::min(1000, 52 - ex)));
  };
  std::vector<int4> work;
  std::vector<double> scale;
  if (P.segments.empty()) {
    // runs of up to 8 j tiles per item, shorter when that leaves fewer items
    // than about four per resident CTA (small structures)
    const int64_t tile_pairs = (int64_t)P.L.n_tiles * (P.L.n_tiles + 1) / 2 * item_blocks;
    const int run = (int)std::max<int64_t>(1, std::min<int64_t>(8, tile_pairs / (4 * 3 * (int64_t)ctx->sm_count)));
    work = shard_work(make_work(P.L, item_blocks, run, P.lattice_first_tile), P.shard, P.n_shards);
    scale.assign(work.size(), scale_of(0, P.L.n_tiles));
  } else {
    std::vector<int64_t> out;
    make_work_segments(P, item_blocks, 8, work, out);
    P.d_work_out = upload(ctx, P, P.qcfg, "work_out", out.data(), out.size(), ctx->stream);
    const int K = (int)P.segments.size() - 1;
    std::vector<double> seg_scale(K);
    for (int c = 0; c < K; ++c) seg_scale[c] = scale_of(P.segments[c], P.segments[c + 1]);
    const int64_t per = (int64_t)P.n_pairs * P.nq;
    scale.resize(work.size());
    for (size_t k = 0; k < work.size(); ++k) scale[k] = seg_scale[(size_t)(out[k] / per)];
  }
  P.d_scale = upload(ctx, P, P.qcfg, "scale", scale.data(), scale.size(), ctx->stream);
  P.n_work = (int)work.size();
  P.d_work = upload(ctx, P, P.qcfg, "work", work.data(), work.size(), ctx->stream);
  P.d_qpar = upload(ctx, P, P.qcfg, "qpar", qpar.data(), qpar.size(), ctx->stream);
  P.d_qrange = upload(ctx, P, P.qcfg, "qrange", qrange.data(), qrange.size(), ctx->stream);
}

std::unique_ptr<PairPlan> make_pair_plan(crab_ctx* ctx, Layout&& L, const double* q, int64_t nq, bool fp64,
                                         const LatticeSpec* lattice, bool pooled, int shard, int n_shards) {
  require(n_shards >= 1 && shard >= 0 && shard < n_shards, "shard index out of range");
  std::unique_ptr<PairPlan> P(new PairPlan());
  P->pooled = pooled;
  P->shard = shard;
  P->n_shards = n_shards;
  P->L = std::move(L);
  P->fp64 = fp64;
  P->nq = nq;
  P->q.assign(q, q + nq);
  const int T = P->L.T;
  P->n_pairs = T * (T + 1) / 2;
  cudaStream_t s = ctx->stream;
  if (nq == 0 || P->L.n_tiles == 0) return P;
  if (lattice && fp64) lattice = nullptr;  // the FP64 reference sums every pair directly
  P->lattice_first_tile = P->L.n_tiles;
  if (lattice) {
    require(T >= 1, "lattice type needs a layout");
    int first = P->L.n_tiles;
    for (int t = 0; t < P->L.n_tiles; ++t)
      if (P->L.tile_type[t] == T - 1) { first = t; break; }
    P->lattice_first_tile = first;
  }
  if (!fp64) {
    P->d_atoms = upload(ctx, *P, P->owned, "atoms", (const float4*)P->L.atoms.data(), (size_t)P->L.n_pad, s);
    const int2 v = ctx->pair_variant ? make_int2(ctx->pair_variant / 16, ctx->pair_variant % 16)
                                      : default_variant(P->q);
    configure_fp32(ctx, *P, v.x, v.y);
  } else {
    P->n_qblocks = (int)((nq + kQD - 1) / kQD);
    const std::vector<int4> work = shard_work(make_work(P->L, P->n_qblocks, 8, P->L.n_tiles), shard, n_shards);
    P->n_work = (int)work.size();
    P->d_atoms64 = upload(ctx, *P, P->owned, "atoms64", (const double4*)P->L.atoms64.data(), (size_t)P->L.n_pad, s);
    P->d_work = upload(ctx, *P, P->owned, "work64", work.data(), work.size(), s);
    P->d_q = upload(ctx, *P, P->owned, "q", q, (size_t)nq, s);
  }
  P->d_tile_type = upload(ctx, *P, P->owned, "tile_type", P->L.tile_type.data(), P->L.tile_type.size(), s);
  P->d_out = upload<double>(ctx, *P, P->owned, "out", nullptr, (size_t)P->n_pairs * nq, s);
  P->d_status = upload<int>(ctx, *P, P->owned, "status", nullptr, 2, s);
  P->d_next = P->d_status + 1;
  if (lattice && shard == 0) lattice_plan_init(ctx, *P, lattice->cells, lattice->m, lattice->spacing);
  CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
  return P;
}

// One plan over a batch of structures that share types and q grid: their
// layouts are concatenated (each padded to whole tiles on its own), and the
// single launch covers every structure's tile pairs; the raw partials of
// structure c land at d_out + c*n_pairs*nq.
std::unique_ptr<PairPlan> make_batch_pair_plan(crab_ctx* ctx, std::vector<Layout>&& parts, const double* q,
                                               int64_t nq) {
  std::unique_ptr<PairPlan> P(new PairPlan());
  require(!parts.empty(), "empty batch");
  const int T = parts[0].T;
  Layout& L = P->L;
  L.T = T;
  L.self_w2.assign(T, 0.0);
  L.sum_w.assign(T, 0.0);
  P->segments.push_back(0);
  for (auto& part : parts) {
    require(part.T == T, "batch layouts must share the type count");
    L.n += part.n;
    L.n_pad += part.n_pad;
    L.n_tiles += part.n_tiles;
    L.atoms.insert(L.atoms.end(), part.atoms.begin(), part.atoms.end());
    L.tile_type.insert(L.tile_type.end(), part.tile_type.begin(), part.tile_type.end());
    L.extent = std::max(L.extent, part.extent);
    P->segments.push_back(L.n_tiles);
  }
  P->fp64 = false;
  P->nq = nq;
  P->q.assign(q, q + nq);
  P->n_pairs = T * (T + 1) / 2;
  P->lattice_first_tile = L.n_tiles;
  cudaStream_t s = ctx->stream;
  if (nq == 0 || L.n_tiles == 0) return P;
  P->d_atoms = upload(ctx, *P, P->owned, "atoms", (const float4*)L.atoms.data(), (size_t)L.n_pad, s);
  const int2 v = ctx->pair_variant ? make_int2(ctx->pair_variant / 16, ctx->pair_variant % 16)
                                    : default_variant(P->q);
  configure_fp32(ctx, *P, v.x, v.y);
  P->d_tile_type = upload(ctx, *P, P->owned, "tile_type", L.tile_type.data(), L.tile_type.size(), s);
  P->d_out = upload<double>(ctx, *P, P->owned, "out", nullptr, (size_t)(P->segments.size() - 1) * P->n_pairs * nq, s);
  P->d_status = upload<int>(ctx, *P, P->owned, "status", nullptr, 2, s);
  P->d_next = P->d_status + 1;
  CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
  return P;
}

void pair_plan_launch(crab_ctx* ctx, PairPlan& P, cudaStream_t s, bool timed) {
  if (P.nq == 0 || P.L.n_tiles == 0) return;
  const size_t n_out = (size_t)P.n_pairs * P.nq * (P.segments.empty() ? 1 : P.segments.size() - 1);
  CRAB_CUDA_CHECK(cudaMemsetAsync(P.d_out, 0, n_out * sizeof(double), s));
  CRAB_CUDA_CHECK(cudaMemsetAsync(P.d_status, 0, 2 * sizeof(int), s));  // status and work counter
  if (timed) CRAB_CUDA_CHECK(cudaEventRecord(ctx->ev_start, s));
  const int T = P.L.T, nq = (int)P.nq;
  if (P.fp64) {
    int per_sm = 0;
    CRAB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pair_fp64, kThreads, 0));
    const int grid = std::max(1, std::min(P.n_work, ctx->sm_count * std::max(per_sm, 1)));
    k_pair_fp64<<<grid, kThreads, 0, s>>>(P.d_atoms64, P.d_tile_type, P.d_work, P.n_work, P.d_q, nq, T, P.d_out);
    CRAB_CUDA_CHECK(cudaGetLastError());
  } else {
#define CRAB_LAUNCH(QQ, JJ)                                                                                    \
  if (P.Q == QQ && P.jb == JJ) {                                                                                 \
    launch_fp32<QQ, JJ>(s, ctx->sm_count, P.d_atoms, P.d_tile_type, P.d_work, P.n_work, P.d_qpar, P.d_qrange, nq, \
                        T, P.wide, P.d_out, P.d_status, P.d_next, P.d_work_out, P.d_scale, ctx->wait_budget);               \
    launched = true;                                                                                             \
  }
    bool launched = false;
    CRAB_LAUNCH(8, 2)
    CRAB_LAUNCH(16, 2)
    CRAB_LAUNCH(32, 2)
    CRAB_LAUNCH(48, 2)
    CRAB_LAUNCH(64, 2)
    CRAB_LAUNCH(96, 2)
    CRAB_LAUNCH(128, 2)
    CRAB_LAUNCH(64, 4)
    CRAB_LAUNCH(96, 4)
#undef CRAB_LAUNCH
#define CRAB_LAUNCH_PQ(QQ, JJ, OO, CODE)                                                                        \
  if (P.Q == QQ && P.jb == CODE) {                                                                               \
    launch_fp32_pq<QQ, JJ, OO>(s, ctx->sm_count, P.d_atoms, P.d_tile_type, P.d_work, P.n_work, P.d_qpar,          \
                               P.d_qrange, nq, T, P.wide, P.d_out, P.d_status, P.d_next, P.d_work_out, P.d_scale,            \
                               ctx->wait_budget);                                                                 \
    launched = true;                                                                                             \
  }
    CRAB_LAUNCH_PQ(64, 2, 4, 2 + kPackedQ)
    CRAB_LAUNCH_PQ(96, 2, 3, 2 + kPackedQ)
    CRAB_LAUNCH_PQ(128, 1, 2, 1 + kPackedQ)
    CRAB_LAUNCH_PQ(128, 2, 2, 2 + kPackedQ)
    CRAB_LAUNCH_PQ(128, 1, 3, 1 + kPackedQ + kDenser)
    CRAB_LAUNCH_PQ(100, 1, 3, 1 + kPackedQ + kDenser)
    CRAB_LAUNCH_PQ(126, 1, 3, 1 + kPackedQ + kDenser)
    CRAB_LAUNCH_PQ(150, 1, 2, 1 + kPackedQ)
    CRAB_LAUNCH_PQ(168, 1, 2, 1 + kPackedQ)
#undef CRAB_LAUNCH_PQ
#define CRAB_LAUNCH_PQF(QQ, JJ, OO, CODE)                                                                       \
  if (P.Q == QQ && P.jb == CODE) {                                                                               \
    launch_fp32_pq<QQ, JJ, OO, true>(s, ctx->sm_count, P.d_atoms, P.d_tile_type, P.d_work, P.n_work, P.d_qpar,    \
                                     P.d_qrange, nq, T, P.wide, P.d_out, P.d_status, P.d_next, P.d_work_out, P.d_scale,      \
                                     ctx->wait_budget);                                                           \
    launched = true;                                                                                             \
  }
    CRAB_LAUNCH_PQF(168, 1, 2, kFolded1)
    CRAB_LAUNCH_PQF(150, 1, 2, kFolded1)
    CRAB_LAUNCH_PQF(168, 2, 2, kFolded2)
    CRAB_LAUNCH_PQF(150, 2, 2, kFolded2)
    CRAB_LAUNCH_PQF(128, 2, 2, kFolded2)
    CRAB_LAUNCH_PQF(126, 1, 3, kFolded1x3)
    CRAB_LAUNCH_PQF(100, 1, 3, kFolded1x3)
    CRAB_LAUNCH_PQF(84, 1, 4, kFolded1x4)
#undef CRAB_LAUNCH_PQF
    // two chains per pair; a plan with a larger step angle runs the one-chain
    // build of the same length
#define CRAB_LAUNCH_PQ2C(QQ)                                                                                    \
  if (P.Q == QQ && P.jb == kFolded2c) {                                                                          \
    if (P.hmax > kMax2cHalfAngle)                                                                                \
      launch_fp32_pq<QQ, 1, 2, true>(s, ctx->sm_count, P.d_atoms, P.d_tile_type, P.d_work, P.n_work, P.d_qpar,    \
                                     P.d_qrange, nq, T, P.wide, P.d_out, P.d_status, P.d_next, P.d_work_out, P.d_scale,      \
                                     ctx->wait_budget);                                                           \
    else                                                                                                         \
      launch_fp32_pq<QQ, 1, 2, true, 2>(s, ctx->sm_count, P.d_atoms, P.d_tile_type, P.d_work, P.n_work,          \
                                        P.d_qpar, P.d_qrange, nq, T, P.wide, P.d_out, P.d_status, P.d_next,       \
                                        P.d_work_out, P.d_scale, ctx->wait_budget);                                          \
    launched = true;                                                                                             \
  }
    CRAB_LAUNCH_PQ2C(168)
#undef CRAB_LAUNCH_PQ2C
#define CRAB_LAUNCH_SPLIT(QQ, JJ, CODE)                                                                          \
  if (P.Q == QQ && P.jb == CODE) {                                                                               \
    launch_split<QQ, JJ>(s, ctx->sm_count, P.d_atoms, P.d_tile_type, P.d_work, P.n_work, P.d_qpar, P.d_qrange, nq, \
                         T, P.wide, P.d_out, P.d_status, P.d_next, P.d_work_out, P.d_scale, ctx->wait_budget);              \
    launched = true;                                                                                             \
  }
    CRAB_LAUNCH_SPLIT(126, 1, kSplit1)
    CRAB_LAUNCH_SPLIT(126, 2, kSplit2)
    CRAB_LAUNCH_SPLIT(100, 1, kSplit1)
    CRAB_LAUNCH_SPLIT(100, 2, kSplit2)
#undef CRAB_LAUNCH_SPLIT
#define CRAB_LAUNCH_SPLIT3(QQ)                                                                                    \
  if (P.Q == QQ && P.jb == kSplit3) {                                                                            \
    launch_split3<QQ>(s, ctx->sm_count, P.d_atoms, P.d_tile_type, P.d_work, P.n_work, P.d_qpar, P.d_qrange,       \
                      P.n_qblocks, nq, T, P.wide, P.d_out, P.d_status, P.d_next, P.d_work_out, P.d_scale, ctx->wait_budget); \
    launched = true;                                                                                             \
  }
    CRAB_LAUNCH_SPLIT3(84)
    CRAB_LAUNCH_SPLIT3(100)
#undef CRAB_LAUNCH_SPLIT3
    if (!launched) throw Error(CRAB_EINVAL, "unsupported q block");
  }
  ctx->launches += 1;
  if (P.lattice.active) lattice_plan_launch(ctx, P, s);
  if (timed) CRAB_CUDA_CHECK(cudaEventRecord(ctx->ev_stop, s));
}

void pair_plan_fetch(crab_ctx* ctx, PairPlan& P, double* out, bool timed) {
  const int T = P.L.T;
  const int64_t nq = P.nq;
  std::fill(out, out + (size_t)P.n_pairs * nq, 0.0);
  if (nq > 0 && P.L.n_tiles > 0) {
    int status = 0;
    copy_d2h(ctx, out, P.d_out, (size_t)P.n_pairs * nq * sizeof(double), ctx->stream);
    copy_d2h(ctx, &status, P.d_status, sizeof(int), ctx->stream);
    CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    if (timed) {
      float ms = 0.0f;
      CRAB_CUDA_CHECK(cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
      ctx->last_pair_ms = ms;
      ctx->last_pair_q = ((double)P.L.n * (double)(P.L.n - 1) / 2.0) * (double)nq;
    }
    if (status) throw Error(status, "pair kernel: a bounded wait on a j-tile copy ran out");
  }
  if (P.fp64) {
    for (int64_t k = 0; k < nq; ++k)
      if (P.q[k] == 0.0) {
        for (int a = 0; a < T; ++a)
          for (int b = a; b < T; ++b)
            out[(size_t)pair_index(a, b, T) * nq + k] =
                P.shard != 0 ? 0.0
                : (a == b)   ? 0.5 * (P.L.sum_w[a] * P.L.sum_w[a] - P.L.self_w2[a])
                             : P.L.sum_w[a] * P.L.sum_w[b];
      }
    return;
  }
  // raw sums are Σ w_i w_j sin(q r)/r: divide by q; q = 0 takes the exact Σ w_i w_j
  for (int a = 0; a < T; ++a)
    for (int b = a; b < T; ++b) {
      const int ab = pair_index(a, b, T);
      const double w0 = (a == b) ? 0.5 * (P.L.sum_w[a] * P.L.sum_w[a] - P.L.self_w2[a]) : P.L.sum_w[a] * P.L.sum_w[b];
      for (int64_t k = 0; k < nq; ++k) {
        double& v = out[(size_t)ab * nq + k];
        v = (P.q[k] == 0.0) ? (P.shard == 0 ? w0 : 0.0) : v / P.q[k];
      }
    }
  if (P.lattice.active && nq > 0) {
    // site weights are one: the lattice sums are the site–site partial itself
    copy_d2h(ctx, out + (size_t)pair_index(T - 1, T - 1, T) * nq, P.lattice.d_out, (size_t)nq * sizeof(double),
             ctx->stream);
    CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  }
}

void compute_partials(crab_ctx* ctx, Layout&& L, const double* q, int64_t nq, bool force_fp64, Partials& out,
                      const LatticeSpec* lattice, int shard, int n_shards) {
  const bool fp64 = force_fp64;
  if (fp64 && L.atoms64.empty()) throw Error(CRAB_EINVAL, "layout lacks an f64 copy");
  out.T = L.T;
  out.nq = nq;
  out.self = L.self_w2;
  if (shard != 0) std::fill(out.self.begin(), out.self.end(), 0.0);
  std::unique_ptr<PairPlan> P;
  {
    TraceScope tp("make_pair_plan");
    P = make_pair_plan(ctx, std::move(L), q, nq, fp64, lattice, true, shard, n_shards);  // lives inside this call
  }
  out.pair.assign((size_t)P->n_pairs * nq, 0.0);
  {
    TraceScope tr("pair_launch+fetch");
    pair_plan_launch(ctx, *P, ctx->stream, true);
    pair_plan_fetch(ctx, *P, out.pair.data(), true);
  }
  TraceScope td("pair_plan_free");
  P.reset();
}

void quadratic_terms(const Partials& P, const double* X, const double* Y, double* out) {
  const int T = P.T;
  const int64_t nq = P.nq;
  for (int64_t k = 0; k < nq; ++k) {
    double s = 0.0;
    for (int a = 0; a < T; ++a) s += X[(size_t)a * nq + k] * Y[(size_t)a * nq + k] * P.self[a];
    for (int a = 0; a < T; ++a)
      for (int b = a; b < T; ++b) {
        const double coef = (a == b) ? 2.0 * X[(size_t)a * nq + k] * Y[(size_t)a * nq + k]
                                     : X[(size_t)a * nq + k] * Y[(size_t)b * nq + k] +
                                           X[(size_t)b * nq + k] * Y[(size_t)a * nq + k];
        s += coef * P.pair[(size_t)pair_index(a, b, T) * nq + k];
      }
    out[k] = s;
  }
}

}  // namespace crab

namespace crab {

void pair_plan_run_timed(crab_ctx* ctx, PairPlan& P, int repeats, int64_t flush_bytes, double* step_ms) {
  cudaStream_t s = ctx->stream;
  void* flush = flush_bytes > 0 ? ctx->dev("bench.flush", (size_t)flush_bytes) : nullptr;
  std::vector<cudaEvent_t> ev(2 * (size_t)std::max(repeats, 0), nullptr);
  struct Guard {
    std::vector<cudaEvent_t>& e;
    ~Guard() {
      for (cudaEvent_t x : e)
        if (x) cudaEventDestroy(x);
    }
  } guard{ev};
  for (auto& e : ev) CRAB_CUDA_CHECK(cudaEventCreate(&e));
  for (int r = 0; r < repeats; ++r) {
    if (flush) CRAB_CUDA_CHECK(cudaMemsetAsync(flush, r & 0xff, (size_t)flush_bytes, s));
    CRAB_CUDA_CHECK(cudaEventRecord(ev[2 * r], s));
    pair_plan_launch(ctx, P, s, false);
    CRAB_CUDA_CHECK(cudaEventRecord(ev[2 * r + 1], s));
  }
  CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
  for (int r = 0; r < repeats; ++r) {
    float ms = 0.0f;
    CRAB_CUDA_CHECK(cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]));
    if (step_ms) step_ms[r] = ms;
    ctx->last_pair_ms = ms;
  }
  ctx->last_pair_q = ((double)P.L.n * (double)(P.L.n - 1) / 2.0) * (double)P.nq;
  int status = 0;
  copy_d2h(ctx, &status, P.d_status, sizeof(int), s);
  CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
  if (status) throw Error(status, "pair kernel: a bounded wait on a j-tile copy ran out");
}

}  // namespace crab

namespace crab {

// Every (Q, jb) pair that pair_plan_launch can dispatch.
static const int kLaunchable[][2] = {{8, 2},   {16, 2}, {32, 2}, {48, 2}, {64, 2},
                                     {96, 2},  {128, 2}, {64, 4}, {96, 4}, {64, 2 + kPackedQ},
                                     {96, 2 + kPackedQ}, {128, 1 + kPackedQ}, {128, 2 + kPackedQ},
                                     {128, 1 + kPackedQ + kDenser}, {100, 1 + kPackedQ + kDenser},
                                     {126, 1 + kPackedQ + kDenser}, {150, 1 + kPackedQ}, {168, 1 + kPackedQ},
                                     {168, kFolded1}, {150, kFolded1}, {168, kFolded2}, {150, kFolded2},
                                     {128, kFolded2}, {126, kFolded1x3}, {100, kFolded1x3}, {84, kFolded1x4}, {168, kFolded2c},
                                     {126, kSplit1}, {126, kSplit2}, {100, kSplit1}, {100, kSplit2},
                                     {84, kSplit3}, {100, kSplit3}};

bool pair_variant_known(int variant) {
  const int Q = variant / 16, jb = variant % 16;
  bool known = false;
  for (const auto& v : kLaunchable) known = known || (v[0] == Q && v[1] == jb);
  return known;
}

void pair_plan_select(crab_ctx* ctx, PairPlan& P, int variant) {
  require(!P.fp64, "the FP64 plan has a single kernel");
  const int Q = variant / 16, jb = variant % 16;
  require(pair_variant_known(variant), "unknown kernel variant " + std::to_string(variant));
  if (P.nq == 0 || P.L.n_tiles == 0) return;
  configure_fp32(ctx, P, Q, jb);
  CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
}

int pair_plan_autotune(crab_ctx* ctx, PairPlan& P, int* variants, double* ms_out, int capacity, int* n_out) {
  if (n_out) *n_out = 0;
  if (P.fp64 || P.nq == 0 || P.L.n_tiles == 0) return P.Q;
  static const int kVariants[][2] = {{64, 2},  {96, 2},  {128, 2}, {64, 4}, {96, 4}, {64, 2 + kPackedQ},
                                     {96, 2 + kPackedQ}, {128, 1 + kPackedQ}, {128, 2 + kPackedQ},
                                     {128, 1 + kPackedQ + kDenser}, {100, 1 + kPackedQ + kDenser},
                                     {126, 1 + kPackedQ + kDenser}, {150, 1 + kPackedQ}, {168, 1 + kPackedQ},
                                     {168, kFolded1}, {150, kFolded1}, {168, kFolded2}, {150, kFolded2},
                                     {128, kFolded2}, {126, kFolded1x3}, {100, kFolded1x3}, {84, kFolded1x4}, {168, kFolded2c},
                                     {126, kSplit1}, {126, kSplit2}, {100, kSplit1}, {100, kSplit2},
                                     {84, kSplit3}, {100, kSplit3}};
  int bestQ = P.Q, bestJ = P.jb, n = 0;
  float best_ms = -1.0f;
  cudaEvent_t a, b;
  CRAB_CUDA_CHECK(cudaEventCreate(&a));
  CRAB_CUDA_CHECK(cudaEventCreate(&b));
  for (const auto& v : kVariants) {
    configure_fp32(ctx, P, v[0], v[1]);
    pair_plan_launch(ctx, P, ctx->stream, false);  // warm-up
    CRAB_CUDA_CHECK(cudaEventRecord(a, ctx->stream));
    pair_plan_launch(ctx, P, ctx->stream, false);
    CRAB_CUDA_CHECK(cudaEventRecord(b, ctx->stream));
    CRAB_CUDA_CHECK(cudaEventSynchronize(b));
    float ms = 0.0f;
    CRAB_CUDA_CHECK(cudaEventElapsedTime(&ms, a, b));
    if (n < capacity) {
      if (variants) variants[n] = v[0] * 16 + v[1];
      if (ms_out) ms_out[n] = ms;
    }
    ++n;
    if (best_ms < 0.0f || ms < best_ms) {
      best_ms = ms;
      bestQ = v[0];
      bestJ = v[1];
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  configure_fp32(ctx, P, bestQ, bestJ);
  CRAB_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
  if (n_out) *n_out = std::min(n, capacity);
  return bestQ * 16 + bestJ;
}

}  // namespace crab
