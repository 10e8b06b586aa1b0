// Multipole engine: the spherical-harmonic expansion of spherical.rs:266-565,
//   A_lm(q) = sum_i a_i(q) j_l(q r_i) Y_lm(i),   I(q) = 4 pi sum_{l <= l_q} sum_m A_lm(q)^2,
// evaluated as one dense GEMM instead of a contraction per (l, q).
//
// The only coupling between the angular and the radial factor is j_l(q r_i).
// As a function of r on [0, R] it is band-limited by q (it is an average of
// exp(i q r t) over |t| <= 1 weighted by P_l(t)), so interpolating it at nb
// Chebyshev nodes rho_b is exact to round-off once nb is a little above
// q_max R / 2 (the Chebyshev coefficients of exp(i w s) are the Bessel J_k(w),
// which fall off like (e w / 2k)^k beyond k = w):
//   j_l(q r_i) = sum_b j_l(q rho_b) L_b(r_i)          (L_b: Lagrange basis)
//   A_lm(q)    = sum_t a_t(q) sum_b j_l(q rho_b) M^t_{lm,b},
//   M^t_{lm,b} = sum_{i in type t} Y_lm(i) w_i L_b(r_i).
// M is a GEMM [(L+1)^2 x N] x [N x nb] per scattering type, independent of q;
// the q dependence is a small f64 pass over (q, lm).  For wide radial ranges
// [0, R] is cut into S segments with their own nodes (points of a segment use
// only its nodes).  The interpolation error bound, 1e-15 of max |j_l|, is far
// below the FP32 rounding of the GEMM operands.
//
// Kernels:
//   k_mp_prep        per point: r, cos(theta), phi, real Y_lm (the f64
//                    recurrence of spherical.rs:54-93) and w_i L_b(r_i)
//   k_mp_moments     the GEMM, register-tiled SIMT, FP32 or FP64 operands,
//                    split over points with f64 atomic accumulation
//   k_mp_node_bessel j_0..j_{l_q}(q rho_b), the Miller recurrence of
//                    spherical.rs:95-133 in f64
//   k_mp_gram        per q: A^c_lm for each requested amplitude combination c
//                    and 4 pi sum_{l <= l_q, m} A^c A^d
#include <cuda.h>  // CUtensorMap and the tensor-map encoder's types
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "device_math.cuh"
#include "engine.hpp"
#include "ops.hpp"

namespace crab {
namespace {

constexpr double kPiD = 3.14159265358979323846;
constexpr int kMaxL = 64;
constexpr int kMaxNodes = 64;       // Chebyshev nodes per radial segment (GEMM N tile)
constexpr int kMaxSegments = 16;
constexpr int kGemmM = 128;         // lm rows per GEMM tile
constexpr int kPointAlign = 32;     // group padding (GEMM K step for FP32)
constexpr int64_t kSplitK = 4096;   // points per GEMM work item
constexpr int kTileElems = kGemmM * kMaxNodes;  // one partial tile

// spherical.rs:201-203
int adaptive_l(double q, double max_radius, int maximum) {
  long v = (long)std::ceil(q * max_radius) + 8;
  const long lo = std::min(maximum, 8);
  if (v < lo) v = lo;
  if (v > maximum) v = maximum;
  return (int)v;
}

// spherical.rs:33-51
std::vector<double> harmonic_norms(int L) {
  std::vector<double> norms((size_t)(L + 1) * (L + 1), 0.0);
  for (int l = 0; l <= L; ++l)
    for (int m = 0; m <= l; ++m) {
      double ratio = 1.0;
      for (int k = l - m + 1; k <= l + m; ++k) ratio /= (double)k;
      norms[(size_t)l * l + l + m] = std::sqrt(((double)(2 * l + 1) / (4.0 * kPiD)) * ratio);
    }
  return norms;
}

// Smallest node count whose Chebyshev interpolation of exp(i w s) on [-1, 1]
// errs by less than 1e-15: the tail sum_{k >= n} 2 |J_k(w)| with
// |J_k(w)| <= (e w / 2k)^k / sqrt(2 pi k).
int nodes_needed(double w) {
  int n = std::max(8, (int)std::ceil(w) + 8);
  for (;; ++n) {
    const double lb = n * std::log(std::exp(1.0) * std::max(w, 1e-300) / (2.0 * n)) - 0.5 * std::log(2.0 * kPiD * n);
    if (w <= 0.0 || lb < std::log(1e-16)) return n;
  }
}

struct RadialBasis {
  int S = 1, nb = 8;
  double R = 0.0;
  std::vector<double> nodes;  // S * nb
  std::vector<double> bary;   // nb (first-kind Chebyshev barycentric weights)
};

RadialBasis radial_basis(double R, double qmax) {
  RadialBasis B;
  B.R = R;
  for (B.S = 1; B.S <= kMaxSegments; ++B.S) {
    B.nb = nodes_needed(qmax * R / (2.0 * B.S));
    if (B.nb <= kMaxNodes) break;
  }
  if (B.S > kMaxSegments)
    throw Error(CRAB_EINVAL, "multipole radial range too wide for the q grid (q_max * r_max too large)");
  B.nodes.resize((size_t)B.S * B.nb);
  B.bary.resize(B.nb);
  for (int b = 0; b < B.nb; ++b) {
    const double th = (2.0 * b + 1.0) * kPiD / (2.0 * B.nb);
    B.bary[b] = ((b & 1) ? -1.0 : 1.0) * std::sin(th);
    for (int s = 0; s < B.S; ++s) {
      const double a0 = R * s / B.S, a1 = R * (s + 1) / B.S;
      B.nodes[(size_t)s * B.nb + b] = 0.5 * (a0 + a1) + 0.5 * (a1 - a0) * std::cos(th);
    }
  }
  return B;
}

struct MpWork {
  int32_t group, lm0;
  int64_t k0, k1;
};

// ------------------------------------------------------------------ kernels

// Operand layout of the moment GEMM: rows (lm or node) by points, blocked by
// 32 points so that a 32-point stage of a row tile is one contiguous block:
// element (row, k) at ((k / 32) * rows + row) * 32 + k % 32.
__host__ __device__ __forceinline__ int64_t mp_blocked(int row, int64_t k, int rows) {
  return ((k >> 5) * rows + row) * 32 + (k & 31);
}

// Per point: real harmonics (spherical.rs:54-93, 165-199) and the weighted
// Lagrange basis of its radial segment.  pts: x, y, z (centred), w, r.
// The recurrence divides by (l - m) as the reference does, here as a product
// with the f64 reciprocal inv[l - m] (at most one ulp apart per step).
template <typename E>
__global__ void k_mp_prep(const double* __restrict__ pts, const int32_t* __restrict__ seg, int64_t n_pad, int L,
                          int lm_pad, int nb, const double* __restrict__ norms, const double* __restrict__ nodes,
                          const double* __restrict__ bary, const double* __restrict__ inv, E* __restrict__ YT,
                          E* __restrict__ WT) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pad) return;
  const double px = pts[5 * i], py = pts[5 * i + 1], pz = pts[5 * i + 2], w = pts[5 * i + 3], r = pts[5 * i + 4];
  double x, phi;
  if (r < 1e-12) {
    x = 1.0;
    phi = 0.0;
  } else {
    x = fmin(fmax(__ddiv_rn(pz, r), -1.0), 1.0);
    phi = atan2(py, px);
  }
  const double sin_theta = sqrt(fmax(__dadd_rn(1.0, -__dmul_rn(x, x)), 0.0));
  double sin_phi, cos_phi;
  sincos(phi, &sin_phi, &cos_phi);
  const double sqrt2 = sqrt(2.0);
  double sin_m = 0.0, cos_m = 1.0, pmm = 1.0;
  auto emit = [&](int l, int m, double p) {
    const int pos = l * l + l + m;
    if (m == 0) {
      YT[mp_blocked(pos, i, lm_pad)] = (E)__dmul_rn(norms[pos], p);
    } else {
      const double v = __dmul_rn(__dmul_rn(sqrt2, norms[pos]), p);
      YT[mp_blocked(pos, i, lm_pad)] = (E)__dmul_rn(v, cos_m);
      YT[mp_blocked(l * l + l - m, i, lm_pad)] = (E)__dmul_rn(v, sin_m);
    }
  };
  for (int m = 0; m <= L; ++m) {
    if (m > 0) {
      pmm = __dmul_rn(pmm, __dmul_rn(-(double)(2 * m - 1), sin_theta));
      const double next_cos = __dadd_rn(__dmul_rn(cos_m, cos_phi), -__dmul_rn(sin_m, sin_phi));
      sin_m = __dadd_rn(__dmul_rn(sin_m, cos_phi), __dmul_rn(cos_m, sin_phi));
      cos_m = next_cos;
    }
    emit(m, m, pmm);
    if (m == L) continue;
    const double pm1 = __dmul_rn(__dmul_rn(x, (double)(2 * m + 1)), pmm);
    emit(m + 1, m, pm1);
    double prev = pmm, cur = pm1;
    for (int l = m + 2; l <= L; ++l) {
      const double num = __dadd_rn(__dmul_rn(__dmul_rn((double)(2 * l - 1), x), cur), -__dmul_rn((double)(l + m - 1), prev));
      const double next = __dmul_rn(num, inv[l - m]);
      emit(l, m, next);
      prev = cur;
      cur = next;
    }
  }
  for (int pos = (L + 1) * (L + 1); pos < lm_pad; ++pos) YT[mp_blocked(pos, i, lm_pad)] = (E)0;
  // Barycentric Lagrange basis at the segment's first-kind Chebyshev nodes.
  const double* nd = nodes + (int64_t)seg[i] * nb;
  int hit = -1;
  double den = 0.0;
  for (int b = 0; b < nb; ++b) {
    const double d = r - nd[b];
    if (d == 0.0) hit = b;
    else den += bary[b] / d;
  }
  for (int b = 0; b < kMaxNodes; ++b) {
    double v = 0.0;
    if (b < nb) {
      if (hit >= 0) v = (b == hit) ? w : 0.0;
      else v = w * ((bary[b] / (r - nd[b])) / den);
    }
    WT[mp_blocked(b, i, kMaxNodes)] = (E)v;
  }
}

// Partial tile of work item w: part[w][b][r] = sum_{k in [k0, k1)} YT[lm0 + r][k] WT[b][k]
// (128 lm rows x 64 nodes, plain stores; k_mp_reduce sums the point splits).
// 256 threads, 8 x 4 outputs each; operands staged through shared memory in
// 128-byte rows (32 floats or 16 doubles of K per step).
template <typename E>
__global__ void __launch_bounds__(256) k_mp_moments(const E* __restrict__ YT, const E* __restrict__ WT, int64_t n_pad,
                                                    int lm_pad, const MpWork* __restrict__ work,
                                                    double* __restrict__ part) {
  constexpr int KS = 128 / sizeof(E);
  constexpr int V = 16 / sizeof(E);
  typedef typename std::conditional<sizeof(E) == 4, float4, double2>::type Vec;
  __shared__ __align__(16) E As[KS][kGemmM + V];
  __shared__ __align__(16) E Bs[KS][kMaxNodes + V];
  const MpWork wk = work[blockIdx.x];
  const int tid = threadIdx.x, tm = tid >> 4, tn = tid & 15;
  E acc[8][4];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = (E)0;
  for (int64_t k0 = wk.k0; k0 < wk.k1; k0 += KS) {
#pragma unroll
    for (int it = 0; it < 4; ++it) {  // A: 128 rows x 8 vectors
      const int idx = it * 256 + tid, row = idx >> 3, c = (idx & 7) * V;
      const Vec v = *reinterpret_cast<const Vec*>(YT + mp_blocked(wk.lm0 + row, k0 + c, lm_pad));
      const E* pv = reinterpret_cast<const E*>(&v);
#pragma unroll
      for (int j = 0; j < V; ++j) As[c + j][row] = pv[j];
    }
#pragma unroll
    for (int it = 0; it < 2; ++it) {  // B: 64 rows x 8 vectors
      const int idx = it * 256 + tid, row = idx >> 3, c = (idx & 7) * V;
      const Vec v = *reinterpret_cast<const Vec*>(WT + mp_blocked(row, k0 + c, kMaxNodes));
      const E* pv = reinterpret_cast<const E*>(&v);
#pragma unroll
      for (int j = 0; j < V; ++j) Bs[c + j][row] = pv[j];
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < KS; ++kk) {
      E a[8], b[4];
#pragma unroll
      for (int j = 0; j < 8; ++j) a[j] = As[kk][tm * 8 + j];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tn * 4 + j];
#pragma unroll
      for (int x = 0; x < 8; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
    }
    __syncthreads();
  }
  double* tile = part + (int64_t)blockIdx.x * kTileElems;
#pragma unroll
  for (int x = 0; x < 8; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) tile[(tn * 4 + y) * kGemmM + tm * 8 + x] = (double)acc[x][y];
}

// ---- tensor-core moment GEMM (tcgen05, TF32 operands split into terms) ----
//
// The same product part[w] = YT-tile . WT-tile^T (128 lm rows x 64 nodes over
// the item's points) on the 5th-generation tensor cores, with TF32 terms
// (h = x rounded to TF32, m = x - h rounded to TF32):
//   S = 1: h h'                  (relative error ~5e-4)
//   S = 2: h h' + h m' + m h'    (relative error ~5e-7)
// The S = 2 error is set by the tensor core's FP32 accumulation, which rounds
// toward zero (about 2^-24 of the accumulator per MMA), so a TMEM accumulator
// covers one 32-point stage only and is then drained into f64 registers.
//
// Warp-specialised pipeline (18 warps):
//  * TMA, warp 9 lane 0: waits until term slot d is empty, then loads the
//    stage's FP32 tiles (A: 128 rows x 32 points, B: 64 x 32; point-blocked,
//    so each tile is a 2D box of 128-byte rows) with two tensor copies into
//    the slot's first-term areas, 128-byte swizzled by the copy itself (row r
//    at (r/8)*1024 + (r%8)*128, 16-byte chunk c at position c ^ (r%8)), the
//    K-major layout the MMA reads; the copies complete on tfull[d];
//  * producers, warps 0-7: wait tfull[d]; each thread takes six 16-byte
//    chunks of the tiles, rounds them to TF32 in place (h) and, for S = 2,
//    writes their m terms at the same offsets of the second-term areas; then
//    fences the generic-proxy writes for the tensor core and arrives on
//    full[d];
//  * MMA issuer, warp 8 lane 0: waits full[d] and accfree[a], issues
//    tcgen05.mma (M = 128, N = 64, K = 8, descriptor start +32 B per K step)
//    into TMEM accumulator a and commits to empty[d] and accfull[a];
//  * drainers, warps 10-17: wait accfull[a], read their lane quarter (warp %
//    4) and 32 of the 64 columns with tcgen05.ld, add them into f64
//    registers and arrive on accfree[a]; at the end they store the f64 tile.
// Four term slots, four accumulators.  The copies read only this GPU's
// memory and use no cluster multicast.  Every wait is bounded: a role whose
// wait runs out stops, the others run out in turn, and the CTA flags
// CRAB_ETIMEOUT, waits (bounded) for its own copies and MMAs and frees its
// TMEM.
constexpr int kTcK = 32;                    // points per stage
constexpr int kTcProducers = 256;           // warps 0-7
constexpr int kTcMmaWarp = 8;
constexpr int kTcTmaWarp = 9;
constexpr int kTcDrainers = 256;            // warps 10-17
constexpr int kTcThreads = kTcProducers + 64 + kTcDrainers;
constexpr int kTcSlots = 4;                 // term buffers
constexpr int kTcAccs = 4;                  // 64-column TMEM accumulators
constexpr int kTcTmemCols = 256;
constexpr int kTcAChunks = 4;               // 16-byte chunks per producer per stage: 4 of A, 2 of B
constexpr int kTcChunks = 6;
static_assert(kTcAChunks * kTcProducers * 16 == kGemmM * kTcK * 4, "A tile chunks");
static_assert((kTcChunks - kTcAChunks) * kTcProducers * 16 == kMaxNodes * kTcK * 4, "B tile chunks");
static_assert(kTcThreads % 32 == 0 && kTcProducers == 32 * kTcMmaWarp, "warp roles");
constexpr int kTcABytes = kGemmM * kTcK * 4;     // 16 KB
constexpr int kTcBBytes = kMaxNodes * kTcK * 4;  // 8 KB
constexpr int kTcBars = 3 * kTcSlots + 2 * kTcAccs + 1;
// TF32, FP32 accumulate, K-major A and B, N = 64 (bits 17-22, N>>3), M = 128 (bits 24-28, M>>4)
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
// the same with N = 128: the hi and lo B terms of a slot as one operand (rows 0-63 and 64-127)
constexpr uint32_t kTcIdescN128 = (1u << 4) | (2u << 7) | (2u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);
// TMEM columns of the staged kernel: S = 2 keeps 128 columns per accumulator
// (hi*hi' in the first 64, the hi*lo' + lo*hi' corrections in the next 64)
template <int S>
__host__ __device__ constexpr int tc_tmem_cols() {
  return S == 2 ? 512 : 256;
}

__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;                         // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;  // stride (8-row group) byte offset
  d |= (uint64_t)1 << 46;                         // descriptor version for sm_100
  d |= (uint64_t)2 << 61;                         // 128-byte swizzle
  return d;
}
// x rounded to the nearest TF32 value (ties away from zero): add half of the
// last kept bit (bit 13) to the magnitude bits and clear the 13 dropped bits;
// a carry into the exponent is the correct rounding.  Integer ALU work
// instead of a conversion instruction on the narrower XU pipe.
__device__ __forceinline__ float tf32_rna(float x) {
  return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate,
                                       uint32_t idesc = kTcIdesc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
// 2D tensor copy of one box into shared memory, completing on an mbarrier
// (no multicast: the box lies in this GPU's memory and lands in this CTA).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst), b = (uint32_t)__cvta_generic_to_shared(bar);
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(d), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(b)
      : "memory");
}

// The producers' pass over one 16-byte chunk at byte offset off of a copied
// tile (part_bytes: one term's tile size): the four values rounded to TF32 in
// place (h), and for S = 2 their m terms into the second-term tile.  A
// truncated h (the copied values as the tensor core reads them) would save
// the in-place store but bias the dropped m m' product by about 2^-22 of the
// product, since m then has the sign of x.
template <int S>
__device__ __forceinline__ void tc_term_pass(unsigned char* __restrict__ base, int part_bytes, int off) {
  const float4 x = *reinterpret_cast<const float4*>(base + off);
  const float4 h = make_float4(tf32_rna(x.x), tf32_rna(x.y), tf32_rna(x.z), tf32_rna(x.w));
  *reinterpret_cast<float4*>(base + off) = h;
  if (S == 2)
    *reinterpret_cast<float4*>(base + part_bytes + off) =
        make_float4(tf32_rna(x.x - h.x), tf32_rna(x.y - h.y), tf32_rna(x.z - h.z), tf32_rna(x.w - h.w));
}

template <int S>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_mp_moments_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int lm_pad,
                    const MpWork* __restrict__ work, double* __restrict__ part, int* __restrict__ status,
                    int budget) {
  static_assert(S == 1 || S == 2, "one or two TF32 terms");
  if (budget < 0) budget = dev::kSpinBudget;  // the context's default
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  constexpr int slot_bytes = S * (kTcABytes + kTcBBytes);  // S A terms, then S B terms
  // 1024-byte alignment (the 128-byte swizzle's period) as an offset into the
  // shared array, so that pointers derived from it keep the shared state space
  unsigned char* smem = tc_smem + ((1024u - ((uint32_t)__cvta_generic_to_shared(tc_smem) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kTcSlots * slot_bytes);
  uint64_t* tfull = bars;                     // [kTcSlots], the copies' bytes
  uint64_t* full = bars + kTcSlots;           // [kTcSlots], one arrival per producer
  uint64_t* empty = bars + 2 * kTcSlots;      // [kTcSlots], MMA commit
  uint64_t* accfull = bars + 3 * kTcSlots;    // [kTcAccs], MMA commit
  uint64_t* accfree = accfull + kTcAccs;      // [kTcAccs], one arrival per drainer
  uint64_t* done = accfree + kTcAccs;         // error path: all MMAs complete
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + kTcBars);
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const MpWork wk = work[blockIdx.x];
  if (warp == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                 "r"(tc_tmem_cols<S>())
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int d = 0; d < kTcSlots; ++d) {
      dev::mbar_init(&tfull[d], 1);
      dev::mbar_init(&full[d], kTcProducers);
      dev::mbar_init(&empty[d], 1);
    }
    for (int a = 0; a < kTcAccs; ++a) {
      dev::mbar_init(&accfull[a], 1);
      dev::mbar_init(&accfree[a], kTcDrainers);
    }
    dev::mbar_init(done, 1);
    dev::fence_mbar_init();
    s_fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int nk = (int)((wk.k1 - wk.k0) / kTcK);
  const int kb0 = (int)(wk.k0 >> 5);  // first 32-point block of the item
  bool ok = true;
  // set when a role gave up; the others stop at their next wait
  auto failed = [&]() { return *((volatile int*)&s_fail) != 0; };

  if (warp < kTcMmaWarp) {
    // ---------------- producers
    const int t = tid;
    for (int s = 0; s < nk; ++s) {
      const int d = s % kTcSlots;
      if (failed() || !dev::mbar_spin(&tfull[d], (unsigned)((s / kTcSlots) & 1), budget)) {
        ok = false;
        break;
      }
      unsigned char* sa = smem + d * slot_bytes;
      unsigned char* sb = sa + S * kTcABytes;
#pragma unroll
      for (int c = 0; c < kTcAChunks; ++c) tc_term_pass<S>(sa, kTcABytes, (c * kTcProducers + t) * 16);
#pragma unroll
      for (int c = 0; c < kTcChunks - kTcAChunks; ++c) tc_term_pass<S>(sb, kTcBBytes, (c * kTcProducers + t) * 16);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&full[d]);
    }
  } else if (warp == kTcTmaWarp) {
    // ---------------- tensor copies
    if (lane == 0) {
      int issued = 0;
      for (int s = 0; s < nk; ++s) {
        const int d = s % kTcSlots;
        if (s >= kTcSlots &&
            (failed() || !dev::mbar_spin(&empty[d], (unsigned)((s / kTcSlots - 1) & 1), budget))) {
          ok = false;
          break;
        }
        unsigned char* sa = smem + d * slot_bytes;
        dev::mbar_expect_tx(&tfull[d], kTcABytes + kTcBBytes);
        tma_load_2d(sa, &tmA, 0, (kb0 + s) * lm_pad + wk.lm0, &tfull[d]);
        tma_load_2d(sa + S * kTcABytes, &tmB, 0, (kb0 + s) * kMaxNodes, &tfull[d]);
        issued = s + 1;
      }
      // no copy may land after the CTA exits: when any role gave up, wait
      // (bounded) for the last copy issued into each slot
      if (!ok || failed())
        for (int s = issued - 1; s >= 0 && s >= issued - kTcSlots; --s)
          dev::mbar_spin(&tfull[s % kTcSlots], (unsigned)((s / kTcSlots) & 1), dev::kDrainBudget);
    }
  } else if (warp == kTcMmaWarp) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t smem_base = (uint32_t)__cvta_generic_to_shared(smem);
      constexpr int acc_stride = S == 2 ? 128 : 64;
      for (int s = 0; s < nk; ++s) {
        const int d = s % kTcSlots, a = s % kTcAccs;
        if (failed() || !dev::mbar_spin(&full[d], (unsigned)((s / kTcSlots) & 1), budget) ||
            (s >= kTcAccs && !dev::mbar_spin(&accfree[a], (unsigned)((s / kTcAccs - 1) & 1), budget))) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_base + d * slot_bytes, b0 = a0 + S * kTcABytes;
        const uint32_t acc_cols = tmem + (uint32_t)(a * acc_stride);
#pragma unroll
        for (int kk = 0; kk < kTcK / 8; ++kk) {
          if (S == 1) {
            tc_mma(acc_cols, tc_smem_desc(a0 + kk * 32), tc_smem_desc(b0 + kk * 32), kk ? 1u : 0u);
          } else {
            // A_hi against [B_hi; B_lo] (N = 128): hh' in columns 0-63, hm' in 64-127;
            // then A_lo against B_hi adds mh' to the corrections
            tc_mma(acc_cols, tc_smem_desc(a0 + kk * 32), tc_smem_desc(b0 + kk * 32), kk ? 1u : 0u, kTcIdescN128);
            tc_mma(acc_cols + 64u, tc_smem_desc(a0 + kTcABytes + kk * 32), tc_smem_desc(b0 + kk * 32), 1u);
          }
        }
        tc_commit(&empty[d]);
        tc_commit(&accfull[a]);
      }
    }
  } else {
    // ---------------- drainers
    const int quarter = warp & 3, half = (warp - kTcTmaWarp - 1) >> 2;
    double acc[32];  // this thread's lm row and 32 of the 64 node columns
#pragma unroll
    for (int i = 0; i < 32; ++i) acc[i] = 0.0;
    for (int s = 0; s < nk; ++s) {
      const int a = s % kTcAccs;
      if (failed() || !dev::mbar_spin(&accfull[a], (unsigned)((s / kTcAccs) & 1), budget)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      constexpr int acc_stride = S == 2 ? 128 : 64;
      const uint32_t row = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(a * acc_stride + half * 32);
      if (S == 1) {
#pragma unroll
        for (int c16 = 0; c16 < 2; ++c16) {
          float v[16];
          tc_ld16(row + (uint32_t)(c16 * 16), v);
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[c16 * 16 + i] += (double)v[i];
        }
      } else {
        // hh' plus the corrections, 8 columns at a time (the f64 sums hold 64 registers)
#pragma unroll
        for (int c8 = 0; c8 < 4; ++c8) {
          float v[8], w[8];
          tc_ld8(row + (uint32_t)(c8 * 8), v);
          tc_ld8(row + (uint32_t)(64 + c8 * 8), w);
#pragma unroll
          for (int i = 0; i < 8; ++i) acc[c8 * 8 + i] += (double)(v[i] + w[i]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(&accfree[a]);
    }
    if (ok) {
      double* tile = part + (int64_t)blockIdx.x * kTileElems + quarter * 32 + lane;
#pragma unroll
      for (int i = 0; i < 32; ++i) tile[(half * 32 + i) * kGemmM] = acc[i];
    }
  }
  if (!ok) atomicExch(&s_fail, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (s_fail) {
    // bounded wait for every MMA this CTA issued before freeing TMEM
    if (tid == kTcMmaWarp * 32) {
      tc_commit(done);
      atomicExch(status, CRAB_ETIMEOUT);
    }
    dev::mbar_spin(done, 0);
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc_tmem_cols<S>())
                 : "memory");
}

template <int S>
constexpr size_t tc_smem_bytes() {
  return 1024 /* alignment slack */ + kTcSlots * (size_t)S * (kTcABytes + kTcBBytes) + sizeof(uint64_t) * kTcBars + 16;
}

// Tensor map of a point-blocked FP32 operand viewed as rows of 32 floats
// (128 bytes): rows x 32, copied in boxes of box_rows x 32 with the 128-byte
// swizzle of the tensor-core tiles.  The encoder comes from the driver
// through the runtime's entry-point query, so the library links no libcuda.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
CUtensorMap tf32_tile_map(const void* base, uint64_t rows, uint32_t box_rows) {
  static EncodeTiledFn encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    CRAB_CUDA_CHECK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    require(q == cudaDriverEntryPointSuccess && fn, "the driver has no cuTensorMapEncodeTiled");
    return reinterpret_cast<EncodeTiledFn>(fn);
  }();
  require(((uintptr_t)base & 15u) == 0, "tensor-map base must be 16-byte aligned");
  CUtensorMap map;
  const cuuint64_t dims[2] = {32, rows};
  const cuuint64_t strides[1] = {32 * sizeof(float)};
  const cuuint32_t box[2] = {32, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(CRAB_ECUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return map;
}

// ---- fused moment GEMM: Y_lm generated by the producer warps ----
//
// The staged path above writes Y_lm of every point to device memory
// (k_mp_prep: 1 GB at 100,000 atoms and L = 50) and the GEMM reads it back.
// Here the producer warps run the harmonic recurrence themselves and write
// the operand terms straight into the swizzled shared tiles, so Y_lm never
// reaches device memory.
//
// Rows are taken in m-major order, the order in which the recurrence of
// spherical.rs:54-93 produces them: m = 0 with l = 0..L, then for every
// m >= 1 and l = m..L the cos row and the sin row.  A point's walk through
// the rows is then one pass of the recurrence, and its state (P_m^m,
// P_{l-1}^m, P_l^m, cos m phi, sin m phi) carries from one 128-row lm tile
// to the next.  A CTA owns a chunk of stages of one group and runs every lm
// tile over it, tile-major; the walk state of its points waits in a device
// array between tiles (40 bytes per point, L2-resident).  In the TF32 modes the
// values are the ones k_mp_prep writes, bit for bit: the same f64 operations
// in the same order, then the same rounding to the operand type; the BF16
// hi+lo mode takes each recurrence step as one fused multiply-add
// (fu_next_l).  k_mp_reduce maps rows back to the l^2 + l + m order of the
// moments.
//
// Element types; both give 128-byte stage rows, so the swizzled layout, the
// descriptors and the four K steps of 32 bytes per stage are those of the
// staged kernel:
//   E = 0, TF32: 32-point stages, K = 8 per MMA (kind::tf32)
//   E = 1, BF16: 64-point stages, K = 16 per MMA (kind::f16, BF16 A and B)
// S = 2 splits both operands into hi + lo terms (3 products per K step).
// W = w L_b(r) is the same for every lm tile: k_mp_prep_fused writes it once,
// already split and swizzled, one 8 KB block per (stage, term), and the
// producer warp of a stage fetches its blocks with a 1D bulk copy.
//
// Roles: producer warps 0..PW-1 (slot p takes the stages c = p mod P of
// every tile; a TF32 slot has one producer warp, a BF16 slot two, warps p
// and p + P, each walking half of the stage's points with one point per
// lane, so a point's walk state is handled by one warp only), the MMA
// issuer (warp PW, lane 0) and 8 drain warps, which read each stage's FP32
// accumulator from TMEM into f64 registers (one stage per accumulator, as in
// the staged kernel) and store the f64 tile of the chunk at the end of each
// lm tile.  Every wait is bounded, and the role waits suspend the warp
// (try_wait) rather than spin, so waiting warps leave the issue slots to the
// producers; a CTA that gives up drains its bulk copies and MMAs before it
// frees TMEM and exits.
constexpr int kFuDrainers = 256;
constexpr int kFuBatch = 4;  // recurrence steps a producer lane runs ahead of its row stores
template <int E, int S>
struct FuCfg {
  // slots, and producer warps per slot: a BF16 hi+lo stage (64 points, two
  // terms) is walked by two warps, one point per lane each, so every
  // scheduler runs two independent walks; a single-term stage by one warp
  // (two points per lane for BF16), which is faster there
  static constexpr int P = S == 1 ? 6 : 4;
  static constexpr int Slots = P;
  static constexpr int WPS = (E == 1 && S == 2) ? 2 : 1;
  static constexpr int PW = P * WPS;  // producer warps
  static constexpr int SlotBytes = S * (kTcABytes + kTcBBytes);
  // drain threads: 256 (two per lm row, 32 node columns each), or for BF16
  // hi+lo 128 (one per row, all 64 columns), which leaves its producers more
  // registers; draining a 64-point stage takes a fraction of producing it
  static constexpr int Drainers = WPS == 2 ? 128 : kFuDrainers;
  static constexpr int DrainCols = 64 * 128 / Drainers;
  static constexpr int Threads = (PW + 1) * 32 + Drainers;
  static constexpr int Bars = 3 * Slots + 2 * kTcAccs + 1;
  // slots, then per producer warp the normalisations of one tile's rows
  // (kGemmM doubles), the 1/k table (kMaxL + 2 doubles), the barriers
  static constexpr size_t NormOff = (size_t)Slots * SlotBytes;
  static constexpr size_t InvOff = NormOff + (size_t)PW * kGemmM * sizeof(double);
  static constexpr size_t BarOff = InvOff + (kMaxL + 2) * sizeof(double);
  static constexpr size_t Smem = 1024 + BarOff + sizeof(uint64_t) * Bars + 16;
};
static_assert(FuCfg<0, 1>::Smem <= 232448 && FuCfg<0, 2>::Smem <= 232448 && FuCfg<1, 1>::Smem <= 232448 &&
                  FuCfg<1, 2>::Smem <= 232448,
              "shared memory of the fused GEMM");

template <int E>
__host__ __device__ constexpr int fu_stage_points() { return E == 0 ? 32 : 64; }

// BF16, FP32 accumulate, K-major A and B, N = 64, M = 128
constexpr uint32_t kBfIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
__device__ __forceinline__ void tc_mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kBfIdesc), "r"(accumulate)
      : "memory");
}
// Two FP32 values rounded to BF16 (nearest even) in one word: lo = a, hi = b.
__device__ __forceinline__ uint32_t bf16x2_rn(float a, float b) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
  return r;
}
__device__ __forceinline__ uint16_t bf16_rn(float a) {
  uint16_t r;
  asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(r) : "f"(a));
  return r;
}
__device__ __forceinline__ float bf16_lo_f32(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi_f32(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// Byte offset of element (row, k) in a K-major 128-byte-swizzled tile whose
// rows hold 128 bytes of K (32 TF32 or 64 BF16 values).
template <int E>
__host__ __device__ __forceinline__ uint32_t fu_swz(int row, int k) {
  const int chunk = E == 0 ? (k >> 2) : (k >> 3);
  const int within = E == 0 ? (k & 3) * 4 : (k & 7) * 2;
  return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4) + within);
}

// The recurrence of spherical.rs:54-93 in the order of k_mp_prep.  Per point
// the walk keeps P_m^m (pmm), P_{l-1}^m, P_l^m (prev, cur) and cos, sin (m phi);
// the walk position (m, l, and whether the next row is the sin row of (l, m))
// is the same for every point.  The f64 operations and their order are
// k_mp_prep's (in the BF16 hi+lo mode except the l step, fu_next_l), so the TF32
// values are its values bit for bit.
struct FuWalk {
  double pmm, prev, cur, cm, sm;
  float cmf, smf;  // cos, sin (m phi) rounded to FP32 (the BF16 modes' rows)
};
// P_{m+1}^m = (x (2m+1)) P_m^m
__device__ __forceinline__ void fu_first_l(int m, const double4& k4, FuWalk& w) {
  const double nxt = __dmul_rn(__dmul_rn(k4.x, (double)(2 * m + 1)), w.pmm);
  w.prev = w.cur;
  w.cur = nxt;
}
// P_l^m = ((2l-1) x P_{l-1}^m - (l+m-1) P_{l-2}^m) / (l-m), with a = 2l-1,
// b = l+m-1 and iv = 1/(l-m) given.  EXACT: k_mp_prep's operations in its
// order (the TF32 modes, whose fused and staged curves are equal, and BF16).
// Otherwise (BF16 hi+lo) the same recurrence as one fused multiply-add on the walk's
// dependency chain, P_l = fma((a iv) x, P_{l-1}, -(b iv) P_{l-2}): the other
// products do not wait on P_{l-1}, so a step costs one f64 latency instead of
// three; its rounding differs from k_mp_prep's by about an ulp.  The
// generator takes the second form, the batches of fu_generate and the
// single-rounding rows of fu_emit_vals in the BF16 hi+lo layout (one point
// per lane), where they were measured faster, and the first elsewhere.
template <bool EXACT = true>
__device__ __forceinline__ void fu_next_l(double a, double b, double iv, const double4& k4, FuWalk& w) {
  if (EXACT) {
    const double num = __dadd_rn(__dmul_rn(__dmul_rn(a, k4.x), w.cur), -__dmul_rn(b, w.prev));
    w.prev = w.cur;
    w.cur = __dmul_rn(num, iv);
  } else {
    const double ax = __dmul_rn(__dmul_rn(a, iv), k4.x), bp = __dmul_rn(__dmul_rn(b, iv), w.prev);
    const double nxt = __fma_rn(ax, w.cur, -bp);
    w.prev = w.cur;
    w.cur = nxt;
  }
}
// next m: P_m^m = P_{m-1}^{m-1} (-(2m-1) sin theta), (cos, sin)(m phi) rotated
template <bool F32ROWS = false>
__device__ __forceinline__ void fu_next_m(int m, const double4& k4, FuWalk& w) {
  w.pmm = __dmul_rn(w.pmm, __dmul_rn(-(double)(2 * m - 1), k4.y));
  const double next_cos = __dadd_rn(__dmul_rn(w.cm, k4.z), -__dmul_rn(w.sm, k4.w));
  w.sm = __dadd_rn(__dmul_rn(w.sm, k4.z), __dmul_rn(w.cm, k4.w));
  w.cm = next_cos;
  if (F32ROWS) {
    w.cmf = (float)w.cm;
    w.smf = (float)w.sm;
  }
  w.cur = w.pmm;
  w.prev = 0.0;
}

// One row of the A tile: the S operand terms of this lane's PPT values at
// row r of the slot, in columns col .. col + PPT - 1.
// The slot (sa) and the tables the generator reads (srow, inv) are passed as
// __restrict__ pointers: the compiler may then move the table loads of the
// next rows above this row's stores, and the rows' dependency chains overlap.
template <int E, int S, int PPT>
__device__ __forceinline__ void fu_emit(unsigned char* __restrict__ sa, int r, int col, const double (&v)[PPT]) {
  const uint32_t off = fu_swz<E>(r, col);
  if (E == 0) {  // the terms of k_mp_moments_tc
    const float f = (float)v[0];
    const float h = tf32_rna(f);
    *reinterpret_cast<float*>(sa + off) = h;
    if (S == 2) *reinterpret_cast<float*>(sa + kTcABytes + off) = tf32_rna(f - h);
  } else if (PPT == 1) {
    const float f = (float)v[0];
    const uint16_t h = bf16_rn(f);
    *reinterpret_cast<uint16_t*>(sa + off) = h;
    if (S == 2) *reinterpret_cast<uint16_t*>(sa + kTcABytes + off) = bf16_rn(f - __uint_as_float((uint32_t)h << 16));
  } else {
    const float fa = (float)v[0], fb = (float)v[PPT - 1];
    const uint32_t h = bf16x2_rn(fa, fb);
    *reinterpret_cast<uint32_t*>(sa + off) = h;
    if (S == 2) *reinterpret_cast<uint32_t*>(sa + kTcABytes + off) = bf16x2_rn(fa - bf16_lo_f32(h), fb - bf16_hi_f32(h));
  }
}

// The rows of (l, m): one row for m = 0 (norm P_l^0), else the cos and the
// sin row (sqrt(2) norm P_l^m times cos / sin (m phi)); sn is the row's
// normalisation and cur the points' P_l^m.
template <int E, int S, int PPT>
__device__ __forceinline__ void fu_emit_vals(unsigned char* __restrict__ sa, int r, int col, int m, double sn,
                                             const double (&cur)[PPT], const FuWalk (&w)[PPT]) {
  if (E == 1 && PPT == 1) {
    // BF16, one point per lane: the entry's value rounded to FP32 once, the
    // cos and sin rows as FP32 products, both rounded to BF16 (and their lo
    // terms) by one packed conversion each (a few 1e-8 of relative rounding
    // beyond the f64 products, far below the BF16 terms)
    const float cf = (float)__dmul_rn(sn, cur[0]);
    if (m == 0) {
      const uint16_t h = bf16_rn(cf);
      const uint32_t off = fu_swz<E>(r, col);
      *reinterpret_cast<uint16_t*>(sa + off) = h;
      if (S == 2) *reinterpret_cast<uint16_t*>(sa + kTcABytes + off) = bf16_rn(cf - __uint_as_float((uint32_t)h << 16));
    } else {
      const float c = cf * w[0].cmf, v = cf * w[0].smf;
      const uint32_t h2 = bf16x2_rn(c, v);  // low half c, high half v
      const uint32_t oc = fu_swz<E>(r, col), ov = fu_swz<E>(r + 1, col);
      *reinterpret_cast<uint16_t*>(sa + oc) = (uint16_t)h2;
      *reinterpret_cast<uint16_t*>(sa + ov) = (uint16_t)(h2 >> 16);
      if (S == 2) {
        const uint32_t l2 = bf16x2_rn(c - bf16_lo_f32(h2), v - bf16_hi_f32(h2));
        *reinterpret_cast<uint16_t*>(sa + kTcABytes + oc) = (uint16_t)l2;
        *reinterpret_cast<uint16_t*>(sa + kTcABytes + ov) = (uint16_t)(l2 >> 16);
      }
    }
    return;
  }
  double v[PPT];
  if (m == 0) {
#pragma unroll
    for (int jj = 0; jj < PPT; ++jj) v[jj] = __dmul_rn(sn, cur[jj]);
    fu_emit<E, S, PPT>(sa, r, col, v);
  } else {
    double c[PPT];
#pragma unroll
    for (int jj = 0; jj < PPT; ++jj) {
      const double vv = __dmul_rn(sn, cur[jj]);
      c[jj] = __dmul_rn(vv, w[jj].cm);
      v[jj] = __dmul_rn(vv, w[jj].sm);
    }
    fu_emit<E, S, PPT>(sa, r, col, c);
    fu_emit<E, S, PPT>(sa, r + 1, col, v);
  }
}
template <int E, int S, int PPT>
__device__ __forceinline__ void fu_emit_entry(unsigned char* __restrict__ sa, int r, int col, int m, double sn,
                                              const FuWalk (&w)[PPT]) {
  double cur[PPT];
#pragma unroll
  for (int jj = 0; jj < PPT; ++jj) cur[jj] = w[jj].cur;
  fu_emit_vals<E, S, PPT>(sa, r, col, m, sn, cur, w);
}

// The 128 rows of one lm tile for this lane's points, from the walk position
// ts = (m, l, sin row next) at the tile's first row (srow: the rows'
// normalisations, in shared memory; inv[k] = 1/k); the walk state w moves
// on to the first row of the next tile.  Rows are produced run by run (one
// run = the l = m..L of one m); inside a run the steps are the same, so the
// loop over them has no branches and consecutive rows overlap.
template <int E, int S, int PPT>
__device__ __forceinline__ void fu_generate(unsigned char* __restrict__ sa, int col, int4 ts, int L,
                                            const double4 (&k4)[PPT], FuWalk (&w)[PPT],
                                            const double* __restrict__ srow, const double* __restrict__ inv) {
  int m = ts.x, l = ts.y, half = ts.z, r = 0;
  constexpr bool kHiLoRows = E == 1 && PPT == 1;  // the BF16 hi+lo layout's rows (fu_emit_vals)
  if (kHiLoRows)
#pragma unroll
    for (int jj = 0; jj < PPT; ++jj) {
      w[jj].cmf = (float)w[jj].cm;
      w[jj].smf = (float)w[jj].sm;
    }
  auto next_m = [&]() {
    ++m;
    if (m <= L) {
#pragma unroll
      for (int jj = 0; jj < PPT; ++jj) fu_next_m<kHiLoRows>(m, k4[jj], w[jj]);
    }
    l = m;
  };
  auto step_from = [&]() {  // after the rows of (l, m): on to (l+1, m) or to the next m
    if (l == L) {
      next_m();
    } else {
#pragma unroll
      for (int jj = 0; jj < PPT; ++jj) {
        if (l == m) fu_first_l(m, k4[jj], w[jj]);
        else fu_next_l<!(E == 1 && PPT == 1)>((double)(2 * l + 1), (double)(l + m), inv[l + 1 - m], k4[jj], w[jj]);
      }
      ++l;
    }
  };
  while (r < kGemmM) {
    if (m > L) {  // padding rows past the last harmonic
      const double z[PPT] = {};
      for (; r < kGemmM; ++r) fu_emit<E, S, PPT>(sa, r, col, z);
      break;
    }
    const double sn = srow[r];
    if (half) {  // the sin row of (l, m) opens the tile
      double v[PPT];
#pragma unroll
      for (int jj = 0; jj < PPT; ++jj)
        v[jj] = kHiLoRows ? (double)((float)__dmul_rn(sn, w[jj].cur) * w[jj].smf)  // as fu_emit_vals
                       : __dmul_rn(__dmul_rn(sn, w[jj].cur), w[jj].sm);
      fu_emit<E, S, PPT>(sa, r++, col, v);
      half = 0;
      step_from();
      continue;
    }
    const int per = m > 0 ? 2 : 1;
    if (r + per > kGemmM) {  // one row left: the cos row of (l, m); its sin row opens the next tile
      double v[PPT];
#pragma unroll
      for (int jj = 0; jj < PPT; ++jj)
        v[jj] = kHiLoRows ? (double)((float)__dmul_rn(sn, w[jj].cur) * w[jj].cmf)
                       : __dmul_rn(__dmul_rn(sn, w[jj].cur), w[jj].cm);
      fu_emit<E, S, PPT>(sa, r++, col, v);
      break;
    }
    const int n = min(L - l + 1, (kGemmM - r) / per);  // entries of this run in this tile (>= 1)
    fu_emit_entry<E, S, PPT>(sa, r, col, m, sn, w);
    r += per;
    step_from();
    if (m > L || l == m) continue;  // the run ended with its first entry
    // entries 2..n: every one but a run-closing (L, m) steps with the same form
    const int rest = n - 1, steady = min(rest, L - l);
    double a = (double)(2 * l + 1), b = (double)(l + m);  // coefficients of the step from l to l+1
    // in batches of kFuBatch entries: the batch's recurrence steps first (the
    // one dependent chain; each entry's P_l^m is kept), then its entries' rows,
    // which depend on nothing but those values, so a warp's in-order issue
    // overlaps their latencies with one another and with the chain
    int k = 0;
    for (; E == 1 && PPT == 1 && k + kFuBatch <= steady; k += kFuBatch) {  // the BF16 hi+lo layout
      double cv[kFuBatch][PPT];
#pragma unroll
      for (int u = 0; u < kFuBatch; ++u) {
        const double iv = inv[l + 1 - m];
#pragma unroll
        for (int jj = 0; jj < PPT; ++jj) {
          cv[u][jj] = w[jj].cur;
          fu_next_l<!(E == 1 && PPT == 1)>(a, b, iv, k4[jj], w[jj]);
        }
        a += 2.0;
        b += 1.0;
        ++l;
      }
#pragma unroll
      for (int u = 0; u < kFuBatch; ++u) fu_emit_vals<E, S, PPT>(sa, r + u * per, col, m, srow[r + u * per], cv[u], w);
      r += kFuBatch * per;
    }
#pragma unroll 4
    for (; k < steady; ++k) {
      fu_emit_entry<E, S, PPT>(sa, r, col, m, srow[r], w);
      r += per;
      const double iv = inv[l + 1 - m];
#pragma unroll
      for (int jj = 0; jj < PPT; ++jj) fu_next_l<!(E == 1 && PPT == 1)>(a, b, iv, k4[jj], w[jj]);
      a += 2.0;
      b += 1.0;
      ++l;
    }
    if (rest > steady) {  // (L, m) closes the run inside this tile
      fu_emit_entry<E, S, PPT>(sa, r, col, m, srow[r], w);
      r += per;
      next_m();
    }
  }
}

// Walk state arrays (structure of arrays over the padded points).
struct FuState {
  double* pmm;
  double* prev;
  double* cur;
  double* cm;
  double* sm;
};
__device__ __forceinline__ void fu_load(const FuState& st, int64_t i, FuWalk& w) {
  w.pmm = st.pmm[i];
  w.prev = st.prev[i];
  w.cur = st.cur[i];
  w.cm = st.cm[i];
  w.sm = st.sm[i];
}
__device__ __forceinline__ void fu_store(const FuState& st, int64_t i, const FuWalk& w) {
  st.pmm[i] = w.pmm;
  st.prev[i] = w.prev;
  st.cur[i] = w.cur;
  st.cm[i] = w.cm;
  st.sm[i] = w.sm;
}

// Per point: the recurrence constants (cos theta, sin theta, cos phi, sin phi;
// spherical.rs:165-199, as k_mp_prep) and the weighted Lagrange basis
// w L_b(r), rounded to the operand type, split into S terms and written into
// the swizzled B blocks of its stage.
template <int E, int S>
__global__ void k_mp_prep_fused(const double* __restrict__ pts, const int32_t* __restrict__ seg, int64_t n_pad, int nb,
                                const double* __restrict__ nodes, const double* __restrict__ bary,
                                double4* __restrict__ cst, unsigned char* __restrict__ Bimg) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pad) return;
  const double px = pts[5 * i], py = pts[5 * i + 1], pz = pts[5 * i + 2], w = pts[5 * i + 3], r = pts[5 * i + 4];
  double x, phi;
  if (r < 1e-12) {
    x = 1.0;
    phi = 0.0;
  } else {
    x = fmin(fmax(__ddiv_rn(pz, r), -1.0), 1.0);
    phi = atan2(py, px);
  }
  const double sin_theta = sqrt(fmax(__dadd_rn(1.0, -__dmul_rn(x, x)), 0.0));
  double sin_phi, cos_phi;
  sincos(phi, &sin_phi, &cos_phi);
  cst[i] = make_double4(x, sin_theta, cos_phi, sin_phi);
  constexpr int KS = fu_stage_points<E>();
  const int64_t stage = i / KS;
  const int k = (int)(i % KS);
  unsigned char* blk = Bimg + (size_t)stage * S * kTcBBytes;
  const double* nd = nodes + (int64_t)seg[i] * nb;
  int hit = -1;
  double den = 0.0;
  for (int b = 0; b < nb; ++b) {
    const double d = r - nd[b];
    if (d == 0.0) hit = b;
    else den += bary[b] / d;
  }
  for (int b = 0; b < kMaxNodes; ++b) {
    double v = 0.0;
    if (b < nb) {
      if (hit >= 0) v = (b == hit) ? w : 0.0;
      else v = w * ((bary[b] / (r - nd[b])) / den);
    }
    const float f = (float)v;
    const uint32_t off = fu_swz<E>(b, k);
    if (E == 0) {  // the terms of k_mp_moments_tc
      const float h = tf32_rna(f);
      *reinterpret_cast<float*>(blk + off) = h;
      if (S == 2) *reinterpret_cast<float*>(blk + kTcBBytes + off) = tf32_rna(f - h);
    } else {
      const uint16_t h = bf16_rn(f);
      *reinterpret_cast<uint16_t*>(blk + off) = h;
      if (S == 2) *reinterpret_cast<uint16_t*>(blk + kTcBBytes + off) = bf16_rn(f - __uint_as_float((uint32_t)h << 16));
    }
  }
}

// Work item of the fused GEMM: (group, first stage, stage count, unused).
template <int E, int S>
__global__ void __launch_bounds__(FuCfg<E, S>::Threads, 1)
    k_mp_moments_fused(const double4* __restrict__ cst, const unsigned char* __restrict__ Bimg,
                       const int4* __restrict__ work, const int4* __restrict__ tstart, int n_lmt, int L,
                       const double* __restrict__ snorm_rows, const double* __restrict__ inv, FuState state,
                       double* __restrict__ part, int* __restrict__ status, int budget) {
  using Cfg = FuCfg<E, S>;
  constexpr int P = Cfg::P, Slots = Cfg::Slots, PW = Cfg::PW, WPS = Cfg::WPS, KS = fu_stage_points<E>();
  static_assert(Slots == P, "one slot per producer warp");
  // TF32 hi+lo: the B terms as one N = 128 operand, 128 TMEM columns per accumulator
  constexpr bool kMergeB = E == 0 && S == 2;
  extern __shared__ __align__(1024) unsigned char fu_smem[];
  if (budget < 0) budget = dev::kWaitBudget;  // the context's default
  // 1024-byte alignment as an offset into the shared array (pointers derived
  // from it keep the shared state space)
  unsigned char* smem = fu_smem + ((1024u - ((uint32_t)__cvta_generic_to_shared(fu_smem) & 1023u)) & 1023u);
  double* s_inv = reinterpret_cast<double*>(smem + Cfg::InvOff);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::BarOff);
  uint64_t* full = bars;                 // [Slots], the 32 lanes of the producing warp
  uint64_t* bfull = bars + Slots;        // [Slots], the W blocks' bulk copy (one arrival + bytes)
  uint64_t* empty = bars + 2 * Slots;    // [Slots], MMA commit
  uint64_t* accfull = bars + 3 * Slots;  // [kTcAccs], MMA commit
  uint64_t* accfree = accfull + kTcAccs; // [kTcAccs], one arrival per drainer
  uint64_t* done = accfree + kTcAccs;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + Cfg::Bars);
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int4 wk = work[blockIdx.x];
  const int nc = wk.z, n_units = n_lmt * nc;
  if (warp == 0) {
    const uint32_t slot = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                 "r"(tc_tmem_cols<(E == 0 ? S : 1)>())
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    for (int d = 0; d < Slots; ++d) {
      dev::mbar_init(&full[d], 32 * WPS);
      dev::mbar_init(&bfull[d], 1);
      dev::mbar_init(&empty[d], 1);
    }
    for (int a = 0; a < kTcAccs; ++a) {
      dev::mbar_init(&accfull[a], 1);
      dev::mbar_init(&accfree[a], Cfg::Drainers);
    }
    dev::mbar_init(done, 1);
    dev::fence_mbar_init();
    s_fail = 0;
  }
  for (int k = tid; k < L + 2; k += blockDim.x) s_inv[k] = inv[k];
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  bool ok = true;
  auto failed = [&]() { return *((volatile int*)&s_fail) != 0; };

  if (warp < PW) {
    // ---------------- producers
    // slot d = warp mod P, half h of its stage's points; this warp's stages:
    // c = d + k P of every tile, item j = t * n_mine + k, which is also the
    // use index of its slot
    constexpr int PPT = (E == 0 || WPS == 2) ? 1 : 2;  // points per lane
    const int d = warp % P, h = warp / P;
    const int col = WPS == 2 ? h * 32 + lane : PPT * lane;  // this lane's first point in the stage
    const int n_mine = nc > d ? (nc - d + P - 1) / P : 0, total = n_mine * n_lmt;
    unsigned char* sa = smem + (size_t)d * Cfg::SlotBytes;
    unsigned char* sb = sa + S * kTcABytes;
    double* srow = reinterpret_cast<double*>(smem + Cfg::NormOff) + (size_t)warp * kGemmM;
    double nrm[kGemmM / 32];  // this lane's share of the next tile's row normalisations
    if (total > 0)
#pragma unroll
      for (int i = 0; i < kGemmM / 32; ++i) nrm[i] = snorm_rows[lane + 32 * i];
    bool issued = false;  // lane 0: a W copy into this warp's slot was issued (parity of the last: issued_ph)
    unsigned issued_ph = 0u;
    // walk state and constants of the current item (the first item starts the walk)
    double4 k4[PPT];
    FuWalk wv[PPT];
    if (total > 0)
#pragma unroll
      for (int jj = 0; jj < PPT; ++jj) {
        k4[jj] = cst[(int64_t)(wk.y + d) * KS + col + jj];
        wv[jj] = FuWalk{1.0, 0.0, 1.0, 1.0, 0.0, 1.0f, 0.0f};
      }
    for (int j = 0; j < total; ++j) {
      const int t = j / n_mine, c = d + (j % n_mine) * P;
      if (j > 0 && (failed() || !dev::mbar_wait(&empty[d], (unsigned)((j - 1) & 1), budget))) {
        ok = false;
        break;
      }
      if (lane == 0 && h == 0) {
        dev::mbar_expect_tx(&bfull[d], S * kTcBBytes);
#pragma unroll
        for (int p = 0; p < S; ++p)
          dev::bulk_g2s(sb + p * kTcBBytes, Bimg + ((size_t)(wk.y + c) * S + p) * kTcBBytes, kTcBBytes,
                        &bfull[d]);
        issued = true;
        issued_ph = (unsigned)(j & 1);
      }
      if (j % n_mine == 0) {  // first stage of a tile: its row normalisations into shared memory
        __syncwarp();
#pragma unroll
        for (int i = 0; i < kGemmM / 32; ++i) srow[lane + 32 * i] = nrm[i];
        __syncwarp();
        if (t + 1 < n_lmt)  // and the next tile's into registers
#pragma unroll
          for (int i = 0; i < kGemmM / 32; ++i) nrm[i] = snorm_rows[(size_t)(t + 1) * kGemmM + lane + 32 * i];
      }
      const int64_t p0 = (int64_t)(wk.y + c) * KS + col;
      // prefetch the next item's constants and walk state (a stage of this
      // warp whose state was stored an item or more ago); with one stage per
      // tile the state simply stays in registers
      const bool has_next = j + 1 < total, same = n_mine == 1;
      double4 k4n[PPT];
      FuWalk wn[PPT];
      if (has_next && !same) {
        const int tn = (j + 1) / n_mine, cn = d + ((j + 1) % n_mine) * P;
        const int64_t pn = (int64_t)(wk.y + cn) * KS + col;
#pragma unroll
        for (int jj = 0; jj < PPT; ++jj) {
          k4n[jj] = cst[pn + jj];
          if (tn == 0) wn[jj] = FuWalk{1.0, 0.0, 1.0, 1.0, 0.0, 1.0f, 0.0f};
          else fu_load(state, pn + jj, wn[jj]);
        }
      }
      fu_generate<E, S, PPT>(sa, col, tstart[t], L, k4, wv, srow, s_inv);
      if (has_next && !same && t + 1 < n_lmt)
#pragma unroll
        for (int jj = 0; jj < PPT; ++jj) fu_store(state, p0 + jj, wv[jj]);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(&full[d]);
      if (has_next && !same)
#pragma unroll
        for (int jj = 0; jj < PPT; ++jj) {
          k4[jj] = k4n[jj];
          wv[jj] = wn[jj];
        }
    }
    if (lane == 0 && issued && !ok)  // no bulk copy may land after the CTA exits
      dev::mbar_wait(&bfull[d], issued_ph, dev::kDrainBudget);
  } else if (warp == PW) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t smem_base = (uint32_t)__cvta_generic_to_shared(smem);
      constexpr int np = S == 1 ? 1 : 3;  // (A term, B term): hh', hm', mh'
      const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};
      for (int u = 0; u < n_units; ++u) {
        const int t = u / nc, c = u % nc, d = c % P, a = u % kTcAccs;
        const unsigned ph = (unsigned)((t * ((nc - d + P - 1) / P) + c / P) & 1);
        if (failed() || !dev::mbar_wait(&full[d], ph, budget) || !dev::mbar_wait(&bfull[d], ph, budget) ||
            (u >= kTcAccs && !dev::mbar_wait(&accfree[a], (unsigned)((u / kTcAccs - 1) & 1), budget))) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t a0 = smem_base + (uint32_t)d * Cfg::SlotBytes, b0 = a0 + S * kTcABytes;
        const uint32_t acc_cols = tmem + (uint32_t)(a * (kMergeB ? 128 : 64));
        if (kMergeB) {
          // as k_mp_moments_tc<2>: A_hi against [B_hi; B_lo] (N = 128), then A_lo against B_hi
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            tc_mma(acc_cols, tc_smem_desc(a0 + kk * 32), tc_smem_desc(b0 + kk * 32), kk ? 1u : 0u, kTcIdescN128);
            tc_mma(acc_cols + 64u, tc_smem_desc(a0 + kTcABytes + kk * 32), tc_smem_desc(b0 + kk * 32), 1u);
          }
        } else {
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
#pragma unroll
            for (int p = 0; p < np; ++p) {
              const uint64_t da = tc_smem_desc(a0 + pa[p] * kTcABytes + kk * 32);
              const uint64_t db = tc_smem_desc(b0 + pb[p] * kTcBBytes + kk * 32);
              if (E == 0) tc_mma(acc_cols, da, db, (kk || p) ? 1u : 0u);
              else tc_mma_bf16(acc_cols, da, db, (kk || p) ? 1u : 0u);
            }
        }
        tc_commit(&empty[d]);
        tc_commit(&accfull[a]);
      }
    }
  } else {
    // ---------------- drainers
    const int quarter = warp & 3, hf = (warp - PW - 1) >> 2;
    constexpr int DC = Cfg::DrainCols;  // this thread's lm row and DC of the 64 node columns
    // the chunk's sum of its stages' FP32 accumulators: in f64, or for BF16
    // hi+lo in FP32, round to nearest over the chunk's stages (a few 1e-7
    // relative, far below the BF16 terms), which halves its registers
    using Acc = typename std::conditional<Cfg::WPS == 2, float, double>::type;
    Acc acc[DC];
#pragma unroll
    for (int i = 0; i < DC; ++i) acc[i] = Acc(0);
    for (int t = 0; t < n_lmt && ok; ++t)
      for (int c = 0; c < nc; ++c) {
        const int u = t * nc + c, a = u % kTcAccs;
        if (failed() || !dev::mbar_wait(&accfull[a], (unsigned)((u / kTcAccs) & 1), budget)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (kMergeB) {
          const uint32_t row = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(a * 128 + hf * DC);
#pragma unroll
          for (int c8 = 0; c8 < DC / 8; ++c8) {
            float v[8], w[8];
            tc_ld8(row + (uint32_t)(c8 * 8), v);
            tc_ld8(row + (uint32_t)(64 + c8 * 8), w);
#pragma unroll
            for (int i = 0; i < 8; ++i) acc[c8 * 8 + i] += (Acc)(v[i] + w[i]);
          }
        } else {
#pragma unroll
          for (int c16 = 0; c16 < DC / 16; ++c16) {
            float v[16];
            tc_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(a * 64 + hf * DC + c16 * 16), v);
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[c16 * 16 + i] += (Acc)v[i];
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        mbar_arrive(&accfree[a]);
        if (c == nc - 1) {
          double* tile = part + ((int64_t)blockIdx.x * n_lmt + t) * kTileElems + quarter * 32 + lane;
#pragma unroll
          for (int i = 0; i < DC; ++i) {
            tile[(hf * DC + i) * kGemmM] = (double)acc[i];
            acc[i] = Acc(0);
          }
        }
      }
  }
  if (!ok) atomicExch(&s_fail, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (s_fail) {
    // bounded wait for every MMA this CTA issued before freeing TMEM
    if (tid == PW * 32) {
      tc_commit(done);
      atomicExch(status, CRAB_ETIMEOUT);
    }
    dev::mbar_spin(done, 0);
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tc_tmem_cols<(E == 0 ? S : 1)>())
                 : "memory");
}

// M[g][b][perm(t*128 + r)] = sum over the point splits of group g of the
// partial tiles of lm tile t, in a fixed order (perm: the l^2 + l + m
// position of a GEMM row; NULL for rows already in that order).
// One CTA per (group, lm tile, 1/kReduceSplit of the tile's elements).
constexpr int kReduceSplit = 8;
static_assert(kTileElems % kReduceSplit == 0, "reduce split");
__global__ void __launch_bounds__(256) k_mp_reduce(const double* __restrict__ part, const int32_t* __restrict__ gfirst,
                                                   const int32_t* __restrict__ gsplits, int n_lmt, int lm_pad,
                                                   const int32_t* __restrict__ perm, double* __restrict__ M) {
  const int g = blockIdx.x / n_lmt, t = blockIdx.x % n_lmt;
  const int first = gfirst[g], n = gsplits[g];
  constexpr int kPer = kTileElems / kReduceSplit;
  const int e0 = blockIdx.y * kPer;
  for (int e = e0 + threadIdx.x; e < e0 + kPer; e += blockDim.x) {
    double v = 0.0;
#pragma unroll 4
    for (int k = 0; k < n; ++k) v += part[(int64_t)(first + k * n_lmt + t) * kTileElems + e];
    const int row = t * kGemmM + e % kGemmM;
    M[((int64_t)g * kMaxNodes + e / kGemmM) * lm_pad + (perm ? perm[row] : row)] = v;
  }
}

// j_0..j_{l_q}(q rho) at every node (spherical.rs:95-133, f64 as the
// reference), zero for l_q < l <= L.  Jn[l][s*nb + b][k].
__global__ void k_mp_node_bessel(const double* __restrict__ q, const int32_t* __restrict__ lq, int64_t nq,
                                 const double* __restrict__ nodes, int n_nodes, int L, double* __restrict__ Jn) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nq * n_nodes) return;
  const int64_t k = idx % nq;  // q fastest: the stores of one l are contiguous across threads
  const int node = (int)(idx / nq);
  const int ql = lq[k];
  const double x = q[k] * nodes[node];
  const int64_t stride = (int64_t)n_nodes * nq;  // Jn is [l][node][q]
  double* out = Jn + (int64_t)node * nq + k;
  for (int l = 0; l <= L; ++l) out[l * stride] = 0.0;
  if (fabs(x) < 1e-8) {
    out[0] = 1.0;
    return;
  }
  double s, c;
  sincos(x, &s, &c);
  if (ql == 0) {
    out[0] = s / x;
    return;
  }
  double work[kMaxL + 26];
  const int start = ql + 24;
  for (int l = 0; l < start + 2; ++l) work[l] = 0.0;
  work[start] = 1.0;
  for (int l = start; l >= 1; --l) {
    work[l - 1] = __dadd_rn(__ddiv_rn(__dmul_rn((double)(2 * l + 1), work[l]), x), -work[l + 1]);
    if (fabs(work[l - 1]) > 1e100)
      for (int kk = l - 1; kk <= start + 1; ++kk) work[kk] *= 1e-100;
  }
  const double j0 = s / x;
  const double j1 = __dadd_rn(s / (x * x), -(c / x));
  const double scale = fabs(j0) >= fabs(j1) ? j0 / work[0] : j1 / work[1];
  for (int l = 0; l <= ql; ++l) out[l * stride] = work[l] * scale;
}

// The q pass.  For every q and amplitude combination c
//   A^c_lm(q) = sum_t amp[c][t][q] sum_s sum_b M[t*S+s][b][lm] j_l(q rho_{s,b})
// and 4 pi sum_{l <= l_q, m} A^c A^d accumulates per q for c <= d (order
// (0,0), (1,1), (2,2), (0,1), (0,2), (1,2) for three combinations).
// k_mp_gram: one block per (l, chunk of 32 m, chunk of 128 q).  Each warp
// owns 4 m and each lane 4 q (lane + 32 j), so one thread keeps a 4 x 4 tile
// of the contraction over the radial nodes in registers; the block's moments
// (per group) and node values (per segment) are staged in shared memory,
// where a warp's moment loads are broadcasts and its node-value loads are
// contiguous.  Each block writes its partial sums per (combination, q);
// k_mp_gram_reduce adds the rows in (l, m) order (deterministic).
constexpr int kGramM = 32, kGramQ = 128, kGramThreads = 256;

template <int K>
__global__ void __launch_bounds__(kGramThreads)
    k_mp_gram(const double* __restrict__ M, const double* __restrict__ Jn, const int32_t* __restrict__ lq,
              const double* __restrict__ amp, const int2* __restrict__ rows, int T, int S, int nb, int n_nodes,
              int lm_pad, int64_t nq, double* __restrict__ part) {
  constexpr int P = K * (K + 1) / 2;
  extern __shared__ double gram_smem[];
  double* Js = gram_smem;                               // [nb][kGramQ] node values of one segment
  double* Ms = gram_smem + (size_t)kMaxNodes * kGramQ;  // [nb][kGramM] moments of one group
  const int2 row = rows[blockIdx.x];
  const int l = row.x, m0 = row.y;
  const int nm = min(kGramM, 2 * l + 1 - m0);
  const int64_t q0 = (int64_t)blockIdx.y * kGramQ;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t jrow = (int64_t)l * n_nodes;
  double A[K][4][4];
#pragma unroll
  for (int c = 0; c < K; ++c)
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) A[c][i][j] = 0.0;
  for (int sg = 0; sg < S; ++sg) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < nb * kGramQ; idx += kGramThreads) {
      const int b = idx / kGramQ, ql = idx % kGramQ;
      const int64_t q = q0 + ql;
      Js[idx] = q < nq ? Jn[(jrow + sg * nb + b) * nq + q] : 0.0;
    }
    for (int t = 0; t < T; ++t) {
      const int g = t * S + sg;
      __syncthreads();
      for (int idx = threadIdx.x; idx < nb * kGramM; idx += kGramThreads) {
        const int b = idx / kGramM, mi = idx % kGramM;
        Ms[idx] = mi < nm ? M[((int64_t)g * kMaxNodes + b) * lm_pad + l * l + m0 + mi] : 0.0;
      }
      __syncthreads();
      double C[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) C[i][j] = 0.0;
      const double* mrow = Ms + warp * 4;
      const double* jcol = Js + lane;
#pragma unroll 2
      for (int b = 0; b < nb; ++b) {
        double mv[4], jv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) mv[i] = mrow[b * kGramM + i];
#pragma unroll
        for (int j = 0; j < 4; ++j) jv[j] = jcol[b * kGramQ + 32 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) C[i][j] = fma(mv[i], jv[j], C[i][j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int64_t q = q0 + lane + 32 * j;
#pragma unroll
        for (int c = 0; c < K; ++c) {
          const double a = q < nq ? amp[((int64_t)c * T + t) * nq + q] : 0.0;
#pragma unroll
          for (int i = 0; i < 4; ++i) A[c][i][j] = fma(a, C[i][j], A[c][i][j]);
        }
      }
    }
  }
  double acc[P][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int64_t q = q0 + lane + 32 * j;
    const bool on = q < nq && l <= lq[q];
    int p = 0;
#pragma unroll
    for (int c = 0; c < K; ++c) {
      double v = 0.0;
#pragma unroll
      for (int i = 0; i < 4; ++i) v = fma(A[c][i][j], A[c][i][j], v);
      acc[p++][j] = on ? v : 0.0;
    }
#pragma unroll
    for (int c = 0; c < K; ++c)
#pragma unroll
      for (int d = c + 1; d < K; ++d) {
        double v = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) v = fma(A[c][i][j], A[d][i][j], v);
        acc[p++][j] = on ? v : 0.0;
      }
  }
  __syncthreads();
  double* red = gram_smem;  // [warp][P][kGramQ], over the node values (no longer needed)
#pragma unroll
  for (int p = 0; p < P; ++p)
#pragma unroll
    for (int j = 0; j < 4; ++j) red[(warp * P + p) * kGramQ + lane + 32 * j] = acc[p][j];
  __syncthreads();
  for (int idx = threadIdx.x; idx < P * kGramQ; idx += kGramThreads) {
    const int p = idx / kGramQ, ql = idx % kGramQ;
    double v = 0.0;
    for (int w = 0; w < kGramThreads / 32; ++w) v += red[(w * P + p) * kGramQ + ql];
    const int64_t q = q0 + ql;
    if (q < nq) part[((int64_t)blockIdx.x * P + p) * nq + q] = v;
  }
}

// 32 (combination, q) outputs per CTA; thread row y sums the rows r = y, y + 8,
// ... in order, then row 0 adds the eight partial sums in order.
__global__ void __launch_bounds__(256) k_mp_gram_reduce(const double* __restrict__ part, int n_rows, int P,
                                                        int64_t nq, double* __restrict__ out) {
  __shared__ double red[8][32];
  const int64_t idx = (int64_t)blockIdx.x * 32 + threadIdx.x;
  const bool on = idx < (int64_t)P * nq;
  const int p = on ? (int)(idx / nq) : 0;
  const int64_t q = on ? idx % nq : 0;
  double v = 0.0;
  if (on)
    for (int r = threadIdx.y; r < n_rows; r += 8) v += part[((int64_t)r * P + p) * nq + q];
  red[threadIdx.y][threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.y == 0 && on) {
    double sum = 0.0;
    for (int y = 0; y < 8; ++y) sum += red[y][threadIdx.x];
    out[(int64_t)p * nq + q] = 4.0 * kPiD * sum;
  }
}

// ------------------------------------------------------------------ host

struct MpInput {
  const TypedAtoms* t;
  double centre[3];
  double rmax_lq;                 // radius for the per-q order (atoms, or atoms and sites)
  std::vector<double> amp;        // K x T x nq amplitude combinations (no occupancy)
  int K = 1;
  // multi-GPU: this rank takes the atoms [n*shard/n_shards, n*(shard+1)/n_shards)
  // into its moments, and `sum` replaces them by the sum over all ranks
  // before the q pass (the radial basis comes from all atoms, so every rank
  // has the same moment layout)
  int shard = 0, n_shards = 1;
  crab_sum_fn sum = nullptr;
  void* sum_user = nullptr;
};

// Chunk size (stages) of the fused GEMM's work items: items of one group
// cover whole stages of it; one CTA per SM, so the time goes as the rounds
// of items times the stages per item, plus the partial tiles every item
// writes and k_mp_reduce reads (n_lmt x 64 KB f64, counted here as 0.073 of
// a TF32 hi+lo stage per tile).
int fused_chunk_stages(const std::vector<int64_t>& group_stages, int sm_count, double stage_cost) {
  int64_t most = 1;
  for (int64_t v : group_stages) most = std::max(most, v);
  int best = 1;
  double best_cost = 1e300;
  for (int cs = 1; cs <= most; ++cs) {
    int64_t items = 0;
    for (int64_t v : group_stages) items += (v + cs - 1) / cs;
    const double rounds = (double)((items + sm_count - 1) / std::max(sm_count, 1));
    const double cost = rounds * cs * stage_cost + 0.073 * (double)items;
    if (cost < best_cost * (1.0 - 1e-12)) {
      best_cost = cost;
      best = cs;
    }
  }
  return best;
}

// Rows of the fused GEMM in the m-major order of the recurrence: the walk
// position (m, l, sin row next) at the start of every 128-row tile, and
// perm[row] = the l^2 + l + m position of the row (rows past the last
// harmonic keep their own index).
void fused_row_walk(int L, int lm_pad, std::vector<int4>& tstart, std::vector<int32_t>& perm) {
  tstart.assign((size_t)lm_pad / kGemmM, make_int4(0, 0, 0, 0));
  perm.assign((size_t)lm_pad, 0);
  int m = 0, l = 0, half = 0;
  for (int row = 0; row < lm_pad; ++row) {
    if (row % kGemmM == 0) tstart[row / kGemmM] = make_int4(m, l, half, 0);
    if (m > L) {
      perm[row] = row;
      continue;
    }
    perm[row] = l * l + l + (half ? -m : m);
    if (m > 0 && half == 0) {
      half = 1;
      continue;
    }
    half = 0;
    if (l < L) {
      ++l;
    } else {
      ++m;
      l = m;
    }
  }
}

// GEMM kernel of a precision mode: gemm = 0 SIMT (FP32, or FP64 with fp64),
// 1 the staged tensor-core kernel (Y_lm through device memory), 2 the fused
// tensor-core kernel with TF32 operands, 3 the fused kernel with BF16
// operands; tc_terms = operand terms (1, or 2 for hi + lo).
enum { kGemmSimt = 0, kGemmStaged = 1, kGemmFusedTf32 = 2, kGemmFusedBf16 = 3 };

// Sums 4 pi sum A^c A^d for the requested combinations; out is [K(K+1)/2][nq].
void multipole_run(crab_ctx* ctx, const MpInput& in, const double* q, int64_t nq, int L, bool fp64, int tc_terms,
                   int gemm, double* out) {
  TraceScope trace("multipole_run");
  const TypedAtoms& t = *in.t;
  const int T = t.T, K = in.K, P = K * (K + 1) / 2;
  const int64_t n = (int64_t)t.w.size();
  std::fill(out, out + (size_t)P * nq, 0.0);
  if (n == 0 || nq == 0) return;
  require(in.n_shards >= 1 && in.shard >= 0 && in.shard < in.n_shards, "shard index out of range");
  require(in.n_shards == 1 || in.sum, "a sharded multipole call needs the moment sum callback");
  // atoms of this rank's moments (all of them unless sharded)
  const int64_t own0 = n * in.shard / in.n_shards, own1 = n * (in.shard + 1) / in.n_shards;
  // geometry relative to the structure centroid (spherical.rs:165-199)
  std::vector<double>& r = ctx->mp_r;  // the context's scratch: no fresh pages per call
  r.resize((size_t)n);
  double R = 0.0, qmax = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double dx = t.xyz[3 * i] - in.centre[0], dy = t.xyz[3 * i + 1] - in.centre[1],
                 dz = t.xyz[3 * i + 2] - in.centre[2];
    r[i] = std::sqrt(((0.0 + dx * dx) + dy * dy) + dz * dz);
    R = std::max(R, r[i]);
  }
  for (int64_t k = 0; k < nq; ++k) qmax = std::max(qmax, q[k]);
  R = R > 0.0 ? R * (1.0 + 1e-12) : 1.0;
  const RadialBasis B = radial_basis(R, qmax);
  const int S = B.S, nb = B.nb, G = T * S;
  // group = type * S + segment; points sorted by group, padded per group
  std::vector<int32_t>& seg_of = ctx->mp_seg_of;  // written for the owned points before any read
  std::vector<int32_t>& group_of = ctx->mp_group_of;
  seg_of.resize((size_t)n);
  group_of.resize((size_t)n);
  std::vector<int64_t> count(G, 0);
  for (int64_t i = own0; i < own1; ++i) {
    seg_of[i] = std::min(S - 1, (int)(r[i] / R * S));
    group_of[i] = t.type[i] * S + seg_of[i];
    ++count[group_of[i]];
  }
  std::vector<int64_t> begin(G + 1, 0);
  // groups padded to whole GEMM stages (64 points for BF16 operands)
  const int align = gemm == kGemmFusedBf16 ? 2 * kPointAlign : kPointAlign;
  for (int g = 0; g < G; ++g) begin[g + 1] = begin[g] + (count[g] + align - 1) / align * align;
  const int64_t n_pad = std::max<int64_t>(begin[G], align);
  // points are built in the context's pinned staging buffers (reused across
  // calls, uploaded asynchronously); padding slots are zeroed explicitly
  auto* pts = (double*)ctx->host("mp_pts", sizeof(double) * 5 * (size_t)n_pad);
  auto* seg = (int32_t*)ctx->host("mp_seg", sizeof(int32_t) * (size_t)n_pad);
  std::vector<int64_t> fill(begin.begin(), begin.end() - 1);
  for (int g = 0; g < G; ++g) {
    for (int64_t k = begin[g]; k < begin[g + 1]; ++k) seg[k] = g % S;
    std::fill(pts + 5 * (begin[g] + count[g]), pts + 5 * begin[g + 1], 0.0);
  }
  if (begin[G] < n_pad) {  // no points at all: one zero tile
    std::fill(pts + 5 * begin[G], pts + 5 * n_pad, 0.0);
    std::fill(seg + begin[G], seg + n_pad, 0);
  }
  for (int64_t i = own0; i < own1; ++i) {
    const int64_t k = fill[group_of[i]]++;
    pts[5 * k] = t.xyz[3 * i] - in.centre[0];
    pts[5 * k + 1] = t.xyz[3 * i + 1] - in.centre[1];
    pts[5 * k + 2] = t.xyz[3 * i + 2] - in.centre[2];
    pts[5 * k + 3] = t.w[i];
    pts[5 * k + 4] = r[i];
  }
  const int lm_count = (L + 1) * (L + 1);
  const int lm_pad = (lm_count + kGemmM - 1) / kGemmM * kGemmM;
  std::vector<int32_t> lq(nq);
  for (int64_t k = 0; k < nq; ++k) lq[k] = adaptive_l(q[k], in.rmax_lq, L);
  const int n_lmt = lm_pad / kGemmM;
  const bool fused = gemm == kGemmFusedTf32 || gemm == kGemmFusedBf16;
  std::vector<int32_t> gfirst(G), gsplits(G);
  // staged and SIMT GEMMs: items (group, point split, lm tile), lm tile fastest
  // (k_mp_reduce relies on this order)
  std::vector<MpWork> work;
  // fused GEMM: items (group, first stage, stage count), each over every lm
  // tile; partial tiles item-major, lm tile fastest (the same order for
  // k_mp_reduce with gfirst in units of items x tiles)
  std::vector<int4> fwork, tstart;
  std::vector<int32_t> perm;
  std::vector<double> snorm;
  const int KS = gemm == kGemmFusedBf16 ? 64 : 32;
  if (!fused) {
    for (int g = 0; g < G; ++g) {
      gfirst[g] = (int32_t)work.size();
      gsplits[g] = 0;
      for (int64_t k0 = begin[g]; k0 < begin[g + 1]; k0 += kSplitK, ++gsplits[g])
        for (int lm0 = 0; lm0 < lm_pad; lm0 += kGemmM)
          work.push_back(MpWork{g, lm0, k0, std::min(begin[g + 1], k0 + kSplitK)});
    }
  } else {
    std::vector<int64_t> gst(G);
    for (int g = 0; g < G; ++g) gst[g] = (begin[g + 1] - begin[g]) / KS;
    const double stage_cost = (tc_terms == 2 ? 1.0 : 0.5) * (KS / 32.0);
    const int cs = fused_chunk_stages(gst, ctx->sm_count, stage_cost);
    for (int g = 0; g < G; ++g) {
      gfirst[g] = (int32_t)(fwork.size() * n_lmt);
      gsplits[g] = 0;
      for (int64_t s0 = begin[g] / KS; s0 < begin[g + 1] / KS; s0 += cs, ++gsplits[g])
        fwork.push_back(make_int4(g, (int)s0, (int)std::min<int64_t>(cs, begin[g + 1] / KS - s0), 0));
    }
  }
  const std::vector<double> norms = harmonic_norms(L);
  std::vector<double> inv(L + 2, 0.0);
  for (int k = 1; k <= L + 1; ++k) inv[k] = 1.0 / (double)k;
  if (fused) {  // the walk's tile starts, and per row the norm as k_mp_prep applies it
    fused_row_walk(L, lm_pad, tstart, perm);
    snorm.assign((size_t)lm_pad, 0.0);  // row order; zero past the last harmonic
    const double sqrt2 = std::sqrt(2.0);
    for (int row = 0; row < lm_pad; ++row) {
      if (perm[row] >= lm_count) continue;
      const int l = (int)std::sqrt((double)perm[row]), m = std::abs(perm[row] - l * l - l);
      const int pos = l * l + l + m;
      snorm[row] = m == 0 ? norms[pos] : sqrt2 * norms[pos];
    }
  }
  const size_t n_items = fused ? fwork.size() * (size_t)n_lmt : work.size();

  trace_mark("mp_host_prep");
  TraceScope tdev("multipole_device");
  cudaStream_t s = ctx->stream;
  const size_t esz = fp64 ? sizeof(double) : sizeof(float);
  double* d_pts = (double*)ctx->dev("mp_pts", sizeof(double) * 5 * (size_t)n_pad);
  int32_t* d_seg = (int32_t*)ctx->dev("mp_seg", sizeof(int32_t) * n_pad);
  double* d_norms = (double*)ctx->dev("mp_norms", sizeof(double) * norms.size());
  double* d_inv = (double*)ctx->dev("mp_inv", sizeof(double) * inv.size());
  double* d_nodes = (double*)ctx->dev("mp_nodes", sizeof(double) * B.nodes.size());
  double* d_bary = (double*)ctx->dev("mp_bary", sizeof(double) * B.bary.size());
  void* d_YT = fused ? nullptr : ctx->dev("mp_Y", esz * (size_t)lm_pad * n_pad);
  void* d_WT = fused ? nullptr : ctx->dev("mp_W", esz * (size_t)kMaxNodes * n_pad);
  MpWork* d_work = fused ? nullptr : (MpWork*)ctx->dev("mp_work", sizeof(MpWork) * std::max<size_t>(work.size(), 1));
  double* d_M = (double*)ctx->dev("mp_M", sizeof(double) * (size_t)G * kMaxNodes * lm_pad);
  double* d_part = (double*)ctx->dev("mp_part", sizeof(double) * (size_t)kTileElems * std::max<size_t>(n_items, 1));
  int32_t* d_gfirst = (int32_t*)ctx->dev("mp_gfirst", sizeof(int32_t) * G);
  int32_t* d_gsplits = (int32_t*)ctx->dev("mp_gsplits", sizeof(int32_t) * G);
  double* d_q = (double*)ctx->dev("mp_q", sizeof(double) * nq);
  int32_t* d_lq = (int32_t*)ctx->dev("mp_lq", sizeof(int32_t) * nq);
  double* d_Jn = (double*)ctx->dev("mp_Jn", sizeof(double) * (size_t)nq * S * nb * (L + 1));
  double* d_amp = (double*)ctx->dev("mp_amp", sizeof(double) * in.amp.size());
  double* d_out = (double*)ctx->dev("mp_out", sizeof(double) * (size_t)P * nq);
  int* d_status = (int*)ctx->dev("mp_status", sizeof(int));
  // fused GEMM: recurrence constants, W blocks, walk state, row tables
  double4* d_cst = nullptr;
  unsigned char* d_Bimg = nullptr;
  FuState fst{};
  int4* d_fwork = nullptr;
  int32_t* d_perm = nullptr;
  int4* d_tstart = nullptr;
  double* d_snorm = nullptr;
  if (fused) {
    d_cst = (double4*)ctx->dev("mp_cst", sizeof(double4) * (size_t)n_pad);
    d_Bimg = (unsigned char*)ctx->dev("mp_Bimg", (size_t)(n_pad / KS) * tc_terms * kTcBBytes);
    double* st = (double*)ctx->dev("mp_walk", sizeof(double) * 5 * (size_t)n_pad);
    fst = FuState{st, st + n_pad, st + 2 * n_pad, st + 3 * n_pad, st + 4 * n_pad};
    d_fwork = (int4*)ctx->dev("mp_fwork", sizeof(int4) * std::max<size_t>(fwork.size(), 1));
    d_perm = (int32_t*)ctx->dev("mp_perm", sizeof(int32_t) * perm.size());
    d_tstart = (int4*)ctx->dev("mp_tstart", sizeof(int4) * tstart.size());
    d_snorm = (double*)ctx->dev("mp_snorm", sizeof(double) * snorm.size());
    copy_h2d(ctx, d_fwork, fwork.data(), sizeof(int4) * fwork.size(), s);
    copy_h2d(ctx, d_perm, perm.data(), sizeof(int32_t) * perm.size(), s);
    copy_h2d(ctx, d_tstart, tstart.data(), sizeof(int4) * tstart.size(), s);
    copy_h2d(ctx, d_snorm, snorm.data(), sizeof(double) * snorm.size(), s);
  }
  copy_h2d(ctx, d_pts, pts, sizeof(double) * 5 * (size_t)n_pad, s);
  copy_h2d(ctx, d_seg, seg, sizeof(int32_t) * n_pad, s);
  copy_h2d(ctx, d_norms, norms.data(), sizeof(double) * norms.size(), s);
  copy_h2d(ctx, d_inv, inv.data(), sizeof(double) * inv.size(), s);
  copy_h2d(ctx, d_nodes, B.nodes.data(), sizeof(double) * B.nodes.size(), s);
  copy_h2d(ctx, d_bary, B.bary.data(), sizeof(double) * B.bary.size(), s);
  if (!fused) copy_h2d(ctx, d_work, work.data(), sizeof(MpWork) * work.size(), s);
  copy_h2d(ctx, d_q, q, sizeof(double) * nq, s);
  copy_h2d(ctx, d_lq, lq.data(), sizeof(int32_t) * nq, s);
  copy_h2d(ctx, d_amp, in.amp.data(), sizeof(double) * in.amp.size(), s);
  CRAB_CUDA_CHECK(cudaMemsetAsync(d_status, 0, sizeof(int), s));
  copy_h2d(ctx, d_gfirst, gfirst.data(), sizeof(int32_t) * G, s);
  copy_h2d(ctx, d_gsplits, gsplits.data(), sizeof(int32_t) * G, s);

  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int i = 0; i < 4; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } ev_guard{ev};
  for (int i = 0; i < 4; ++i) CRAB_CUDA_CHECK(cudaEventCreate(&ev[i]));
  CRAB_CUDA_CHECK(cudaEventRecord(ev[0], s));
  const unsigned prep_blocks = (unsigned)((n_pad + 127) / 128);
  if (fused) {
#define CRAB_FUSED(EE, SS)                                                                                        \
  if (KS == fu_stage_points<EE>() && tc_terms == SS) {                                                            \
    k_mp_prep_fused<EE, SS><<<prep_blocks, 128, 0, s>>>(d_pts, d_seg, n_pad, nb, d_nodes, d_bary, d_cst, d_Bimg);   \
    CRAB_CUDA_CHECK(cudaEventRecord(ev[1], s));                                                                    \
    if (!fwork.empty()) {                                                                                          \
      CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_mp_moments_fused<EE, SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                           (int)FuCfg<EE, SS>::Smem));                                             \
      k_mp_moments_fused<EE, SS><<<(unsigned)fwork.size(), FuCfg<EE, SS>::Threads, FuCfg<EE, SS>::Smem, s>>>(      \
          d_cst, d_Bimg, d_fwork, d_tstart, n_lmt, L, d_snorm, d_inv, fst, d_part, d_status, ctx->wait_budget);   \
    }                                                                                                              \
  }
    CRAB_FUSED(0, 1)
    CRAB_FUSED(0, 2)
    CRAB_FUSED(1, 1)
    CRAB_FUSED(1, 2)
#undef CRAB_FUSED
  } else if (fp64) {
    k_mp_prep<double><<<prep_blocks, 128, 0, s>>>(d_pts, d_seg, n_pad, L, lm_pad, nb, d_norms, d_nodes, d_bary,
                                                   d_inv, (double*)d_YT, (double*)d_WT);
    CRAB_CUDA_CHECK(cudaEventRecord(ev[1], s));
    if (!work.empty())  // empty only for a rank of a sharded call that owns no atoms
      k_mp_moments<double><<<(unsigned)work.size(), 256, 0, s>>>((const double*)d_YT, (const double*)d_WT, n_pad,
                                                                  lm_pad, d_work, d_part);
  } else {
    k_mp_prep<float><<<prep_blocks, 128, 0, s>>>(d_pts, d_seg, n_pad, L, lm_pad, nb, d_norms, d_nodes, d_bary,
                                                  d_inv, (float*)d_YT, (float*)d_WT);
    CRAB_CUDA_CHECK(cudaEventRecord(ev[1], s));
    if (work.empty()) {
      // a rank of a sharded call that owns no atoms: k_mp_reduce writes zero moments
    } else if (tc_terms == 0) {
      k_mp_moments<float><<<(unsigned)work.size(), 256, 0, s>>>((const float*)d_YT, (const float*)d_WT, n_pad,
                                                                 lm_pad, d_work, d_part);
    } else {
      const CUtensorMap tmA = tf32_tile_map(d_YT, (uint64_t)(n_pad / kTcK) * (uint64_t)lm_pad, kGemmM);
      const CUtensorMap tmB = tf32_tile_map(d_WT, (uint64_t)(n_pad / kTcK) * kMaxNodes, kMaxNodes);
#define CRAB_TC(SS)                                                                                               \
  if (tc_terms == SS) {                                                                                           \
    CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_mp_moments_tc<SS>, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                         (int)tc_smem_bytes<SS>()));                                              \
    k_mp_moments_tc<SS><<<(unsigned)work.size(), kTcThreads, tc_smem_bytes<SS>(), s>>>(                           \
        tmA, tmB, lm_pad, d_work, d_part, d_status, ctx->wait_budget);                                              \
  }
      CRAB_TC(1)
      CRAB_TC(2)
#undef CRAB_TC
    }
  }
  k_mp_reduce<<<dim3((unsigned)(G * n_lmt), kReduceSplit), 256, 0, s>>>(d_part, d_gfirst, d_gsplits, n_lmt, lm_pad,
                                                                         fused ? d_perm : nullptr, d_M);
  CRAB_CUDA_CHECK(cudaEventRecord(ev[2], s));
  if (in.n_shards > 1) {
    // every rank's moments summed by the caller (an all-reduce over the GPUs),
    // in device memory (the context's buffer, stream synchronised first) or
    // in a host copy
    const size_t m_count = (size_t)G * kMaxNodes * lm_pad;
    int status = 0;
    if (gemm != kGemmSimt) copy_d2h(ctx, &status, d_status, sizeof(int), s);
    if (ctx->device_sums) {
      CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
      if (status != 0) throw Error(status, "multipole tensor-core GEMM: an mbarrier wait ran out");
      const int rc = in.sum(d_M, (int64_t)m_count, in.sum_user);
      if (rc != CRAB_OK) throw Error(rc, "the moment sum callback failed");
    } else {
      auto* h_M = (double*)ctx->host("mp_M", sizeof(double) * m_count);
      copy_d2h(ctx, h_M, d_M, sizeof(double) * m_count, s);
      CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
      if (status != 0) throw Error(status, "multipole tensor-core GEMM: an mbarrier wait ran out");
      const int rc = in.sum(h_M, (int64_t)m_count, in.sum_user);
      if (rc != CRAB_OK) throw Error(rc, "the moment sum callback failed");
      copy_h2d(ctx, d_M, h_M, sizeof(double) * m_count, s);
    }
  }
  const int n_nodes = S * nb;
  const int64_t nbess = nq * n_nodes;
  k_mp_node_bessel<<<(unsigned)((nbess + 127) / 128), 128, 0, s>>>(d_q, d_lq, nq, d_nodes, n_nodes, L, d_Jn);
  {
    std::vector<int2> rows;
    for (int l = 0; l <= L; ++l)
      for (int m0 = 0; m0 < 2 * l + 1; m0 += kGramM) rows.push_back(make_int2(l, m0));
    auto* d_rows = (int2*)ctx->dev("mp_gram_rows", sizeof(int2) * rows.size());
    copy_h2d(ctx, d_rows, rows.data(), sizeof(int2) * rows.size(), s);
    auto* d_gpart = (double*)ctx->dev("mp_gram_part", sizeof(double) * rows.size() * (size_t)P * nq);
    const size_t gram_smem = sizeof(double) * (size_t)kMaxNodes * (kGramQ + kGramM);
    const dim3 grid((unsigned)rows.size(), (unsigned)((nq + kGramQ - 1) / kGramQ));
    if (K == 1) {
      CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_mp_gram<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gram_smem));
      k_mp_gram<1><<<grid, kGramThreads, gram_smem, s>>>(d_M, d_Jn, d_lq, d_amp, d_rows, T, S, nb, n_nodes, lm_pad,
                                                          nq, d_gpart);
    } else {
      CRAB_CUDA_CHECK(cudaFuncSetAttribute(k_mp_gram<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gram_smem));
      k_mp_gram<3><<<grid, kGramThreads, gram_smem, s>>>(d_M, d_Jn, d_lq, d_amp, d_rows, T, S, nb, n_nodes, lm_pad,
                                                          nq, d_gpart);
    }
    CRAB_CUDA_CHECK(cudaGetLastError());
    k_mp_gram_reduce<<<(unsigned)(((int64_t)P * nq + 31) / 32), dim3(32, 8), 0, s>>>(d_gpart, (int)rows.size(), P,
                                                                                       nq, d_out);
    ctx->launches += 1;
  }
  CRAB_CUDA_CHECK(cudaGetLastError());
  CRAB_CUDA_CHECK(cudaEventRecord(ev[3], s));
  ctx->launches += 5;
  copy_d2h(ctx, out, d_out, sizeof(double) * (size_t)P * nq, s);
  int status = 0;
  if (gemm != kGemmSimt) copy_d2h(ctx, &status, d_status, sizeof(int), s);
  CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
  if (status != 0) throw Error(status, "multipole tensor-core GEMM: an mbarrier wait ran out");
  float total_ms = 0.0f, gemm_ms = 0.0f;
  CRAB_CUDA_CHECK(cudaEventElapsedTime(&total_ms, ev[0], ev[3]));
  CRAB_CUDA_CHECK(cudaEventElapsedTime(&gemm_ms, ev[1], ev[2]));
  ctx->last_mp_ms = total_ms;
  ctx->last_mp_gemm_ms = gemm_ms;
  ctx->last_mp_gemm_flop = 2.0 * (double)lm_count * nb * (double)(own1 - own0);  // useful rows, nodes and points
}

// (fp64 operands, tensor-core TF32 terms) of a precision mode.
struct MpPrecision {
  bool fp64;
  int tc_terms;
  int gemm;
};
MpPrecision multipole_precision(int precision) {
  switch (precision) {
    case CRAB_PREC_FP64: return {true, 0, kGemmSimt};
    case CRAB_PREC_FP32: return {false, 0, kGemmSimt};
    case CRAB_PREC_TF32: return {false, 1, kGemmStaged};
    case CRAB_PREC_TF32_SPLIT: return {false, 2, kGemmStaged};
    case CRAB_PREC_BF16: return {false, 1, kGemmFusedBf16};
    case CRAB_PREC_BF16_SPLIT: return {false, 2, kGemmFusedBf16};
    case CRAB_PREC_TF32_FUSED: return {false, 1, kGemmFusedTf32};
    case CRAB_PREC_TF32_SPLIT_FUSED: return {false, 2, kGemmFusedTf32};
    default:
      throw Error(CRAB_EINVAL, "unknown multipole precision");
  }
}

void validate_multipole(const crab_struct* st, const double* q, int64_t nq, int l_max) {
  require(st != nullptr, "structure is NULL");
  require(nq >= 0 && (nq == 0 || q != nullptr), "q grid is NULL");
  validate_q(q, nq);
  require(l_max >= 0 && l_max <= kMaxL, "multipole l_max must be between 0 and 64");
}

// Per-type multipole amplitudes without occupancy (spherical.rs:205-231):
// V, E, H [T][nq].  Hydration sites (element -1) carry the grid amplitude
// rho/10 * V_voxel * f_water(q) in H.
void multipole_tables(const TypedAtoms& t, const double* q, int64_t nq, const crab_solvent* s, bool implicit,
                      double site_volume, std::vector<double>& V, std::vector<double>& E, std::vector<double>& H) {
  const int T = t.T;
  V.assign((size_t)T * nq, 0.0);
  E.assign((size_t)T * nq, 0.0);
  H.assign((size_t)T * nq, 0.0);
  const bool grid = s && s->hydration_model != CRAB_HYD_ANALYTIC;
  for (int a = 0; a < T; ++a) {
    const size_t o = (size_t)a * nq;
    if (t.cls[a].element < 0) {
      for (int64_t k = 0; k < nq; ++k) H[o + k] = s->bulk_density / 10.0 * site_volume * water_form_factor(q[k]);
    } else if (!s) {
      for (int64_t k = 0; k < nq; ++k) V[o + k] = form_factor(t.cls[a].element, t.cls[a].group, 1.0, implicit, q[k]);
    } else {
      multipole_class_amplitude_rows(t.cls[a], implicit, q, nq, s->bulk_density, s->shell_thickness, V.data() + o,
                                     E.data() + o, grid ? nullptr : H.data() + o);
    }
  }
}

// Atoms (and grid sites) with their amplitude tables, the centroid and the
// radius that sets l_q.
struct MpSolventSetup {
  GridResult g;
  TypedAtoms t;
  std::vector<double> V, E, H;
  double centre[3], rmax_lq;
};

void solvent_setup(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, const crab_solvent& s,
                   bool implicit, MpSolventSetup& u) {
  TraceScope trace("mp_solvent_setup");
  const bool grid = s.hydration_model != CRAB_HYD_ANALYTIC;
  if (grid) u.g = hydration_sites(ctx, st, s);
  trace_mark("hydration sites");
  u.t = type_atoms(st, implicit, grid ? TermSet::SolventGrid : TermSet::SolventAnalytic, grid ? &u.g.sites : nullptr);
  trace_mark("type_atoms");
  multipole_tables(u.t, q, nq, &s, implicit, u.g.voxel_volume, u.V, u.E, u.H);
  trace_mark("tables");
  double rmax;
  centre_and_rmax(st, u.centre, &rmax);
  u.rmax_lq = rmax;
  if (grid) {  // spherical.rs:423-427, 489-493: the order also covers the sites
    double rs = 0.0;
    const size_t ns = u.g.sites.size() / 3;
    for (size_t i = 0; i < ns; ++i) {
      const double dx = u.g.sites[3 * i] - u.centre[0], dy = u.g.sites[3 * i + 1] - u.centre[1],
                   dz = u.g.sites[3 * i + 2] - u.centre[2];
      rs = std::max(rs, std::sqrt(((0.0 + dx * dx) + dy * dy) + dz * dz));
    }
    if (ns > 0) u.rmax_lq = std::max(rmax, rs);
  }
}

}  // namespace

void multipole_intensity_impl(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, int l_max,
                              bool implicit, int precision, double* out, const MpShard& shard) {
  validate_multipole(st, q, nq, l_max);
  const MpPrecision mp = multipole_precision(precision);
  if (st->n == 0) {
    std::fill(out, out + nq, 0.0);
    return;
  }
  TraceScope trace("multipole_intensity");
  TypedAtoms& t = typed_scratch(ctx);
  MpInput in;
  std::vector<double> V, E, H;
  {
    TraceScope tt("mp_type_atoms+tables");
    type_atoms_into(st, implicit, TermSet::Vacuum, nullptr, t);
    in.t = &t;
    double rmax;
    centre_and_rmax(st, in.centre, &rmax);
    in.rmax_lq = rmax;
    multipole_tables(t, q, nq, nullptr, implicit, 0.0, V, E, H);
  }
  in.amp = V;
  in.K = 1;
  in.shard = shard.shard;
  in.n_shards = shard.n_shards;
  in.sum = shard.sum;
  in.sum_user = shard.user;
  multipole_run(ctx, in, q, nq, l_max, mp.fp64, mp.tc_terms, mp.gemm, out);
  for (int64_t k = 0; k < nq; ++k) out[k] = std::fmax(out[k], 0.0);
}

void multipole_solvent_basis_impl(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, int l_max,
                                  const crab_solvent& s, bool implicit, int precision, double* out6,
                                  const MpShard& shard) {
  validate_multipole(st, q, nq, l_max);
  validate_solvent(s);
  const MpPrecision mp = multipole_precision(precision);
  if (st->n == 0) {
    std::fill(out6, out6 + 6 * nq, 0.0);
    return;
  }
  MpSolventSetup u;
  solvent_setup(ctx, st, q, nq, s, implicit, u);
  MpInput in;
  in.t = &u.t;
  std::copy(u.centre, u.centre + 3, in.centre);
  in.rmax_lq = u.rmax_lq;
  in.K = 3;
  in.amp.reserve(u.V.size() * 3);
  in.amp.insert(in.amp.end(), u.V.begin(), u.V.end());
  in.amp.insert(in.amp.end(), u.E.begin(), u.E.end());
  in.amp.insert(in.amp.end(), u.H.begin(), u.H.end());
  in.shard = shard.shard;
  in.n_shards = shard.n_shards;
  in.sum = shard.sum;
  in.sum_user = shard.user;
  multipole_run(ctx, in, q, nq, l_max, mp.fp64, mp.tc_terms, mp.gemm, out6);
}

void multipole_solvent_intensity_impl(crab_ctx* ctx, const crab_struct* st, const double* q, int64_t nq, int l_max,
                                      const crab_solvent& s, bool implicit, int precision, double* out) {
  validate_multipole(st, q, nq, l_max);
  validate_solvent(s);
  const MpPrecision mp = multipole_precision(precision);
  if (st->n == 0) {
    std::fill(out, out + nq, 0.0);
    return;
  }
  MpSolventSetup u;
  solvent_setup(ctx, st, q, nq, s, implicit, u);
  MpInput in;
  in.t = &u.t;
  std::copy(u.centre, u.centre + 3, in.centre);
  in.rmax_lq = u.rmax_lq;
  in.K = 1;
  // spherical.rs:438-444, 453-462: f = v - G(q) e + c2 h per atom, c2 * amplitude per site
  in.amp.resize(u.V.size());
  for (int a = 0; a < u.t.T; ++a)
    for (int64_t k = 0; k < nq; ++k) {
      const size_t o = (size_t)a * nq + k;
      in.amp[o] = u.V[o] - excluded_volume_scale(q[k], s.c1) * u.E[o] + s.c2 * u.H[o];
    }
  multipole_run(ctx, in, q, nq, l_max, mp.fp64, mp.tc_terms, mp.gemm, out);
  for (int64_t k = 0; k < nq; ++k) out[k] = std::fmax(out[k], 0.0);
}

}  // namespace crab

using namespace crab;
extern "C" {
int crab_multipole_intensity(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max, int implicit_hydrogen,
                             int precision, double* out) {
  if (!ctx || !st || (nq > 0 && !out)) return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() { multipole_intensity_impl(ctx, st, q, nq, l_max, implicit_hydrogen != 0, precision, out); });
}
int crab_multipole_last_timing(crab_ctx* ctx, double* total_ms, double* moments_ms, double* moments_flop) {
  if (!ctx) return CRAB_EINVAL;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (total_ms) *total_ms = ctx->last_mp_ms;
  if (moments_ms) *moments_ms = ctx->last_mp_gemm_ms;
  if (moments_flop) *moments_flop = ctx->last_mp_gemm_flop;
  return CRAB_OK;
}
int crab_multipole_solvent_basis(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max,
                                 const crab_solvent* solvent, int implicit_hydrogen, int precision, double* out6) {
  if (!ctx || !st || !solvent || (nq > 0 && !out6)) return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    multipole_solvent_basis_impl(ctx, st, q, nq, l_max, *solvent, implicit_hydrogen != 0, precision, out6);
  });
}

int crab_multipole_intensity_shard(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max,
                                   int implicit_hydrogen, int precision, int shard, int n_shards, crab_sum_fn sum,
                                   void* user, double* out) {
  if (!ctx || !st || (nq > 0 && !out) || n_shards < 1 || shard < 0 || shard >= n_shards || (n_shards > 1 && !sum))
    return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    multipole_intensity_impl(ctx, st, q, nq, l_max, implicit_hydrogen != 0, precision, out,
                             MpShard{shard, n_shards, sum, user});
  });
}

int crab_multipole_solvent_basis_shard(crab_ctx* ctx, crab_struct* st, const double* q, int64_t nq, int l_max,
                                       const crab_solvent* solvent, int implicit_hydrogen, int precision, int shard,
                                       int n_shards, crab_sum_fn sum, void* user, double* out6) {
  if (!ctx || !st || !solvent || (nq > 0 && !out6) || n_shards < 1 || shard < 0 || shard >= n_shards ||
      (n_shards > 1 && !sum))
    return CRAB_EINVAL;
  return guarded_impl(ctx, [&]() {
    multipole_solvent_basis_impl(ctx, st, q, nq, l_max, *solvent, implicit_hydrogen != 0, precision, out6,
                                 MpShard{shard, n_shards, sum, user});
  });
}
}
