// Device helpers shared by the pair-sum kernels: bulk async copies with
// bounded mbarrier waits, FP32 sin/cos for recurrence seeds, and packed
// f32x2 register pairs.
#pragma once

#include <cstdint>

namespace crab {
namespace dev {

// ---- bulk async copy of one j tile into shared memory (1D TMA) ------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
               "l"(src), "r"(bytes), "r"(b)
               : "memory");
}
// Iteration budgets of the bounded waits.  The kernels take the budget of
// their context (crab_ctx_set_wait_budget; these defaults otherwise); a CTA
// that gives up drains its own copies in flight with kDrainBudget, which no
// context option shortens.
constexpr int kWaitBudget = 1 << 22;   // suspending try_wait (pair kernels)
constexpr int kSpinBudget = 1 << 26;   // non-suspending test_wait (tensor-core pipeline)
constexpr int kDrainBudget = 1 << 24;

// Bounded wait on an mbarrier phase. Returns false when the iteration budget
// runs out (the caller records an error and stops using the buffer); a
// budget of 0 gives up at once.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase, int budget = kWaitBudget) {
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  for (int it = 0; it < budget; ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// sin(h), cos(h) for |h| <= 1 by their Taylor series (error < 2e-10 before
// rounding); used for the half-step angle h = Δr/2 and for small seeds.
__device__ __forceinline__ void sincos_small(float h, float* sh, float* ch) {
  const float h2 = h * h;
  float ps = fmaf(h2, -1.0f / 39916800.0f, 1.0f / 362880.0f);
  ps = fmaf(h2, ps, -1.0f / 5040.0f);
  ps = fmaf(h2, ps, 1.0f / 120.0f);
  ps = fmaf(h2, ps, -1.0f / 6.0f);
  *sh = fmaf(h * h2, ps, h);
  float pc = fmaf(h2, 1.0f / 479001600.0f, -1.0f / 3628800.0f);
  pc = fmaf(h2, pc, 1.0f / 40320.0f);
  pc = fmaf(h2, pc, -1.0f / 720.0f);
  pc = fmaf(h2, pc, 1.0f / 24.0f);
  pc = fmaf(h2, pc, -0.5f);
  *ch = fmaf(h2, pc, 1.0f);
}

// sin(x), cos(x) for 0 <= x < 4096·π/2: Cody–Waite reduction by π/2 split
// into C1 + C2 + C3 (C1 and C2 carry 12 significant bits, so k·C1 and k·C2
// are exact for k < 4096), then Taylor polynomials on |y| <= π/4 (truncation
// below 2e-9) and quadrant selection.  Used for the per-pair seed sin(q0 r).
// k = nearest integer to x·2/π comes from adding 1.5·2^23 in the same fused
// multiply-add (the sum's unit is 1, so its low bits are k's quadrant), which
// keeps the conversions off the pipe the recurrence does not use.
__device__ __forceinline__ void sincos_seed(float x, float* s, float* c) {
  const float kMagic = 12582912.0f;  // 1.5·2^23
  const float tk = fmaf(x, 0x1.45f306p-1f, kMagic);  // kMagic + x·2/π, rounded to an integer
  const float k = tk - kMagic;
  float y = fmaf(-k, 0x1.92p+0f, x);
  y = fmaf(-k, 0x1.fb4p-12f, y);
  y = fmaf(-k, 0x1.4442d2p-24f, y);
  const float y2 = y * y;
  float ps = fmaf(y2, 1.0f / 362880.0f, -1.0f / 5040.0f);
  ps = fmaf(y2, ps, 1.0f / 120.0f);
  ps = fmaf(y2, ps, -1.0f / 6.0f);
  const float sy = fmaf(y * y2, ps, y);
  float pc = fmaf(y2, -1.0f / 3628800.0f, 1.0f / 40320.0f);
  pc = fmaf(y2, pc, -1.0f / 720.0f);
  pc = fmaf(y2, pc, 1.0f / 24.0f);
  pc = fmaf(y2, pc, -0.5f);
  const float cy = fmaf(y2, pc, 1.0f);
  const int qd = __float_as_int(tk) & 3;
  const float ss = (qd & 1) ? cy : sy;
  const float cc = (qd & 1) ? sy : cy;
  *s = (qd & 2) ? -ss : ss;
  *c = ((qd + 1) & 2) ? -cc : cc;
}

// Packed pair of FP32 values in one 64-bit register pair (Blackwell f32x2 ops).
__device__ __forceinline__ unsigned long long pack2(float x, float y) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float& x, float& y) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(v));
}


// Bounded spin on an mbarrier phase with the non-suspending test_wait (for
// waits expected to be short, where a suspended try_wait would oversleep).
__device__ __forceinline__ bool mbar_spin(uint64_t* bar, unsigned phase, int budget = kSpinBudget) {
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  for (int it = 0; it < budget; ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace dev
}  // namespace crab
