// Hydration-shell site placement on a voxel grid, bit-exact against the
// reference.
//
// Adaptive coarse shell (crabSAXS src/solvent.rs:121-223): a voxel centre is a
// site when it lies within the outer radius (clearance + shell width) of some
// atom and not within the clearance of any atom; sites are listed in z→y→x
// voxel order.  Exterior shell (src/solvent.rs:259-401): voxels inside a vdW +
// probe sphere are molecular, the unknown voxels 6-connected to the box
// boundary are exterior, and exterior voxels within vdW + probe + thickness of
// an atom are sites.
//
// Exactness: every per-voxel decision in the reference is an OR over atoms of
// (voxel inside the atom's clipped bounding box) AND (squared distance <=
// r² + 1e-10), and the flood fill's result is the connected component of the
// boundary, independent of visiting order.  The device evaluates the same f64
// expressions in the same order with explicitly rounded intrinsics (no fused
// multiply-add), so the site set and its order equal the reference's.  The
// O(N) prologue (centroid, Rg, bounding box) runs on the host in the
// reference's sequential order.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "engine.hpp"

namespace crab {
namespace {

struct Box {
  double mn[3];
  double spacing;
  uint64_t n[3];
};

__device__ __forceinline__ double norm2_rn(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Clipped voxel range of one atom (solvent.rs:187-194 / 322-329).
__device__ __forceinline__ void atom_range(const Box& b, const double* p, double radius, uint64_t* lo, uint64_t* hi) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double lower = __ddiv_rn(__dsub_rn(__dsub_rn(p[d], radius), b.mn[d]), b.spacing);
    const double upper = __ddiv_rn(__dsub_rn(__dadd_rn(p[d], radius), b.mn[d]), b.spacing);
    const double f = fmax(floor(__dsub_rn(lower, 1e-10)), 0.0);
    const double c = ceil(__dadd_rn(upper, 1e-10));
    lo[d] = (uint64_t)f;
    const uint64_t cu = c > 0.0 ? (uint64_t)c : 0ull;
    hi[d] = cu < b.n[d] - 1 ? cu : b.n[d] - 1;
  }
}

// One warp per atom: mark voxels of the atom's box within the radius.
// mode 0: mask[c] = value.  mode 1: only where mask[c] == 2 (exterior).
__global__ void k_rasterize(const double* __restrict__ xyz, const double* __restrict__ radius_per_atom,
                            double radius_all, double extra, int64_t n, Box b, uint8_t* __restrict__ mask,
                            uint8_t value, int exterior_only) {
  const int lane = threadIdx.x & 31;
  const int64_t atom = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (atom >= n) return;
  const double p[3] = {xyz[3 * atom], xyz[3 * atom + 1], xyz[3 * atom + 2]};
  const double radius = radius_per_atom ? __dadd_rn(radius_per_atom[atom], extra) : radius_all;
  const double thr = __dadd_rn(__dmul_rn(radius, radius), 1e-10);
  uint64_t lo[3], hi[3];
  atom_range(b, p, radius, lo, hi);
  if (hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2]) return;
  const uint64_t ex = hi[0] - lo[0] + 1, ey = hi[1] - lo[1] + 1, ez = hi[2] - lo[2] + 1;
  const uint64_t total = ex * ey * ez;
  for (uint64_t v = lane; v < total; v += 32) {
    const uint64_t x = lo[0] + v % ex, y = lo[1] + (v / ex) % ey, z = lo[2] + v / (ex * ey);
    const double px = __dadd_rn(b.mn[0], __dmul_rn((double)x, b.spacing));
    const double py = __dadd_rn(b.mn[1], __dmul_rn((double)y, b.spacing));
    const double pz = __dadd_rn(b.mn[2], __dmul_rn((double)z, b.spacing));
    if (norm2_rn(__dsub_rn(px, p[0]), __dsub_rn(py, p[1]), __dsub_rn(pz, p[2])) <= thr) {
      const uint64_t c = (z * b.n[1] + y) * b.n[0] + x;
      if (!exterior_only) mask[c] = value;
      else if (mask[c] == 2) mask[c] = value;
    }
  }
}

// Site flag of a voxel for the two shells.
__device__ __forceinline__ bool site_flag(const uint8_t* a, const uint8_t* b, uint64_t c, int kind) {
  return kind == 0 ? (a[c] != 0 && b[c] == 0) : (a[c] == 3);
}

constexpr int kScanThreads = 256;
constexpr int kPerThread = 16;
constexpr int kChunk = kScanThreads * kPerThread;

__global__ void k_count(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, uint64_t count, int kind,
                        uint32_t* __restrict__ chunk_count) {
  __shared__ uint32_t s[kScanThreads / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kChunk + (uint64_t)threadIdx.x * kPerThread;
  uint32_t c = 0;
  for (int i = 0; i < kPerThread; ++i)
    if (base + i < count && site_flag(a, b, base + i, kind)) ++c;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += s[w];
    chunk_count[blockIdx.x] = t;
  }
}

// Exclusive scan of chunk counts in one block; total at offsets[n].
__global__ void k_scan_chunks(const uint32_t* __restrict__ cnt, uint64_t n, uint64_t* __restrict__ offsets) {
  __shared__ uint64_t part[1024];
  const uint64_t per = (n + blockDim.x - 1) / blockDim.x;
  const uint64_t b0 = threadIdx.x * per, b1 = min(n, b0 + per);
  uint64_t s = 0;
  for (uint64_t i = b0; i < b1; ++i) s += cnt[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t run = 0;
    for (unsigned t = 0; t < blockDim.x; ++t) {
      uint64_t v = part[t];
      part[t] = run;
      run += v;
    }
    offsets[n] = run;
  }
  __syncthreads();
  uint64_t run = part[threadIdx.x];
  for (uint64_t i = b0; i < b1; ++i) {
    offsets[i] = run;
    run += cnt[i];
  }
}

__global__ void k_emit(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, uint64_t count, int kind, Box bx,
                       const uint64_t* __restrict__ offsets, double* __restrict__ sites, int32_t* __restrict__ cells) {
  __shared__ uint32_t warp_tot[kScanThreads / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kChunk + (uint64_t)threadIdx.x * kPerThread;
  uint32_t c = 0;
  for (int i = 0; i < kPerThread; ++i)
    if (base + i < count && site_flag(a, b, base + i, kind)) ++c;
  // block exclusive scan of c in thread order (= voxel order)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; ++w) before += warp_tot[w];
  uint64_t pos = offsets[blockIdx.x] + before + incl - c;
  for (int i = 0; i < kPerThread; ++i) {
    const uint64_t v = base + i;
    if (v < count && site_flag(a, b, v, kind)) {
      const uint64_t x = v % bx.n[0], y = (v / bx.n[0]) % bx.n[1], z = v / (bx.n[0] * bx.n[1]);
      sites[3 * pos] = __dadd_rn(bx.mn[0], __dmul_rn((double)x, bx.spacing));
      sites[3 * pos + 1] = __dadd_rn(bx.mn[1], __dmul_rn((double)y, bx.spacing));
      sites[3 * pos + 2] = __dadd_rn(bx.mn[2], __dmul_rn((double)z, bx.spacing));
      cells[3 * pos] = (int32_t)x;
      cells[3 * pos + 1] = (int32_t)y;
      cells[3 * pos + 2] = (int32_t)z;
      ++pos;
    }
  }
}

// Exterior flood fill: boundary seeds, then line sweeps along x, y and z that
// carry the exterior label (2) through unknown voxels (0), repeated until no
// voxel changes.  The fixed point is the 6-connected component of the
// boundary's unknown voxels, i.e. the reference's BFS result.
__global__ void k_seed_boundary(uint8_t* __restrict__ s, Box b) {
  const uint64_t count = b.n[0] * b.n[1] * b.n[2];
  for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < count; c += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t x = c % b.n[0], y = (c / b.n[0]) % b.n[1], z = c / (b.n[0] * b.n[1]);
    const bool edge = x == 0 || x + 1 == b.n[0] || y == 0 || y + 1 == b.n[1] || z == 0 || z + 1 == b.n[2];
    if (edge && s[c] == 0) s[c] = 2;
  }
}

// Voxels of a line a thread loads before it carries the label through them:
// one memory latency per batch instead of one per voxel.
constexpr int kSweepBatch = 16;
// Sweep rounds enqueued between two reads of the change flag by the host.
constexpr int kRoundsPerSync = 6;

// One thread per line; axis 0: lines along x (one per (y,z)); 1: along y;
// 2: along z.  A forward and a backward pass each carry the exterior label
// through runs of unknown voxels.  Lines of one axis are disjoint, so threads
// never touch the same voxel.  The round returns at once when the previous
// round changed nothing (*prev_changed == 0): the fixed point is reached.
__global__ void k_sweep(uint8_t* __restrict__ s, Box b, int axis, const int* __restrict__ prev_changed,
                        int* __restrict__ changed) {
  if (prev_changed && *prev_changed == 0) return;
  const uint64_t nx = b.n[0], ny = b.n[1], nz = b.n[2];
  uint64_t lines, len, stride;
  if (axis == 0) { lines = ny * nz; len = nx; stride = 1; }
  else if (axis == 1) { lines = nx * nz; len = ny; stride = nx; }
  else { lines = nx * ny; len = nz; stride = nx * ny; }
  const uint64_t l = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= lines) return;
  uint64_t start;
  if (axis == 0) start = l * nx;                       // l = z*ny + y
  else if (axis == 1) start = (l / nx) * nx * ny + (l % nx);  // l = z*nx + x
  else start = l;                                       // l = y*nx + x
  uint8_t* line = s + start;
  int any = 0;
  bool carry = false;
  // voxels past either end read as molecular (1): never written, stop the carry
  for (uint64_t i0 = 0; i0 < len; i0 += kSweepBatch) {
    uint8_t v[kSweepBatch];
#pragma unroll
    for (int k = 0; k < kSweepBatch; ++k) v[k] = i0 + k < len ? line[(i0 + k) * stride] : (uint8_t)1;
#pragma unroll
    for (int k = 0; k < kSweepBatch; ++k) {
      if (v[k] == 2) carry = true;
      else if (v[k] == 0) {
        if (carry) {
          line[(i0 + k) * stride] = 2;
          any = 1;
        }
      } else carry = false;
    }
  }
  carry = false;
  for (uint64_t e = len; e > 0;) {
    const uint64_t i0 = e - 1;  // this batch covers i0, i0 - 1, ..., down to index 0 at most
    uint8_t v[kSweepBatch];
#pragma unroll
    for (int k = 0; k < kSweepBatch; ++k) v[k] = (uint64_t)k <= i0 ? line[(i0 - k) * stride] : (uint8_t)1;
#pragma unroll
    for (int k = 0; k < kSweepBatch; ++k) {
      if (v[k] == 2) carry = true;
      else if (v[k] == 0) {
        if (carry) {
          line[(i0 - k) * stride] = 2;
          any = 1;
        }
      } else carry = false;
    }
    e = e > (uint64_t)kSweepBatch ? e - kSweepBatch : 0;
  }
  if (any) atomicOr(changed, 1);
}

// Lines of at most kWarpLine voxels are swept by one warp each: lane l holds
// voxels 4l .. 4l+3 (past the end of the line: molecular, never written).
// The forward pass carries the label through a voxel by one of three maps of
// the carry (exterior: set, molecular: clear, unknown: unchanged), and maps of
// this kind compose as "the later constant wins"; an inclusive shuffle scan of
// the lanes' composed maps gives every lane its incoming carry, and the lane
// then steps through its four voxels as the sequential pass does.  The
// backward pass does the same from the right on the updated voxels, so the
// line ends as k_sweep's forward and backward passes leave it.
constexpr int kWarpLine = 128;

// Carry map of four voxels in the given order: (constant?, value).
__device__ __forceinline__ void carry_map(const uint8_t (&v)[4], bool forward, int& is_const, int& value) {
  is_const = 0;
  value = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const uint8_t x = v[forward ? e : 3 - e];
    if (x == 2) { is_const = 1; value = 1; }
    else if (x != 0) { is_const = 1; value = 0; }
  }
}

__global__ void k_sweep_warp(uint8_t* __restrict__ s, Box b, int axis, const int* __restrict__ prev_changed,
                             int* __restrict__ changed) {
  if (prev_changed && *prev_changed == 0) return;
  const uint64_t nx = b.n[0], ny = b.n[1], nz = b.n[2];
  uint64_t lines, len, stride;
  if (axis == 0) { lines = ny * nz; len = nx; stride = 1; }
  else if (axis == 1) { lines = nx * nz; len = ny; stride = nx; }
  else { lines = nx * ny; len = nz; stride = nx * ny; }
  const uint64_t l = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // one line per warp
  if (l >= lines) return;  // the whole warp
  const int lane = threadIdx.x & 31;
  uint64_t start;
  if (axis == 0) start = l * nx;
  else if (axis == 1) start = (l / nx) * nx * ny + (l % nx);
  else start = l;
  uint8_t* line = s + start;
  uint8_t v[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const uint64_t k = (uint64_t)(4 * lane + e);
    v[e] = k < len ? line[k * stride] : (uint8_t)1;
  }
  unsigned wrote = 0u;  // bit e: voxel e became exterior
  // forward: lanes in increasing order
  int c, val;
  carry_map(v, true, c, val);
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int pc = __shfl_up_sync(0xffffffffu, c, o), pv = __shfl_up_sync(0xffffffffu, val, o);
    if (lane >= o && !c) { c = pc; val = pv; }
  }
  int carry = __shfl_up_sync(0xffffffffu, val, 1);
  if (lane == 0) carry = 0;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    if (v[e] == 2) carry = 1;
    else if (v[e] == 0) {
      if (carry) { v[e] = 2; wrote |= 1u << e; }
    } else carry = 0;
  }
  // backward: lanes in decreasing order, on the updated voxels
  carry_map(v, false, c, val);
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int pc = __shfl_down_sync(0xffffffffu, c, o), pv = __shfl_down_sync(0xffffffffu, val, o);
    if (lane + o < 32 && !c) { c = pc; val = pv; }
  }
  carry = __shfl_down_sync(0xffffffffu, val, 1);
  if (lane == 31) carry = 0;
#pragma unroll
  for (int e = 3; e >= 0; --e) {
    if (v[e] == 2) carry = 1;
    else if (v[e] == 0) {
      if (carry) { v[e] = 2; wrote |= 1u << e; }
    } else carry = 0;
  }
#pragma unroll
  for (int e = 0; e < 4; ++e)
    if (wrote & (1u << e)) line[(uint64_t)(4 * lane + e) * stride] = 2;
  if (__any_sync(0xffffffffu, wrote != 0u) && lane == 0) atomicOr(changed, 1);
}

// Grid buffers live in the context's pool ("grid." slots), so repeated calls
// allocate nothing.  A slot above kGridKeepBytes (a box of more than 2^28
// voxels) is released when the build ends, so a one-off large box does not
// keep its memory; a build that leaves its sites on the device keeps the
// sites slot, which trim_grid_pool releases once they are copied out.
constexpr size_t kGridKeepBytes = 256ull << 20;

template <class T>
T* pool(crab_ctx* ctx, const char* name, size_t count) {
  return (T*)ctx->dev(name, std::max<size_t>(count, 1) * sizeof(T));
}

void trim_slots(crab_ctx* ctx, bool keep_sites) {
  for (auto it = ctx->bufs.begin(); it != ctx->bufs.end();) {
    if (it->first.compare(0, 5, "grid.") == 0 && it->second.bytes > kGridKeepBytes &&
        !(keep_sites && it->first == "grid.sites")) {
      cudaFree(it->second.ptr);
      it = ctx->bufs.erase(it);
    } else {
      ++it;
    }
  }
}

struct GridPoolTrim {
  crab_ctx* ctx;
  bool keep_sites;
  ~GridPoolTrim() { trim_slots(ctx, keep_sites); }
};

GridResult compact_sites(crab_ctx* ctx, const uint8_t* a, const uint8_t* b, uint64_t count, int kind,
                         const Box& bx, bool to_host) {
  cudaStream_t s = ctx->stream;
  const uint64_t chunks = (count + kChunk - 1) / kChunk;
  uint32_t* d_cnt = pool<uint32_t>(ctx, "grid.chunk_count", chunks);
  uint64_t* d_off = pool<uint64_t>(ctx, "grid.chunk_offset", chunks + 1);
  k_count<<<(unsigned)chunks, kScanThreads, 0, s>>>(a, b, count, kind, d_cnt);
  CRAB_CUDA_CHECK(cudaGetLastError());
  k_scan_chunks<<<1, 1024, 0, s>>>(d_cnt, chunks, d_off);
  CRAB_CUDA_CHECK(cudaGetLastError());
  uint64_t m = 0;
  copy_d2h(ctx, &m, d_off + chunks, sizeof(uint64_t), s);
  CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
  trace_mark("sites counted");
  GridResult r;
  r.spacing = bx.spacing;
  r.m = (int64_t)m;
  r.build = ctx->grid_builds;
  if (m) {
    require(bx.n[0] < (1ull << 31) && bx.n[1] < (1ull << 31) && bx.n[2] < (1ull << 31), "grid axis too long");
    double* d_sites = pool<double>(ctx, "grid.sites", 3 * m);
    int32_t* d_cells = pool<int32_t>(ctx, "grid.cells", 3 * m);
    k_emit<<<(unsigned)chunks, kScanThreads, 0, s>>>(a, b, count, kind, bx, d_off, d_sites, d_cells);
    CRAB_CUDA_CHECK(cudaGetLastError());
    r.d_sites = d_sites;
    if (to_host) {
      r.sites.resize(3 * m);
      r.cells.resize(3 * m);
      copy_d2h(ctx, r.sites.data(), d_sites, 3 * m * sizeof(double), s);
      copy_d2h(ctx, r.cells.data(), d_cells, 3 * m * sizeof(int32_t), s);
    }
    CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
  }
  ctx->launches += m ? 4 : 3;
  return r;
}

// Box set-up shared by both grids (solvent.rs:160-176 / 290-306).
bool make_box(const double* xyz, int64_t n, double pad, double spacing, Box* b, uint64_t* count) {
  double mn[3] = {xyz[0], xyz[1], xyz[2]}, mx[3] = {xyz[0], xyz[1], xyz[2]};
  for (int64_t i = 1; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      mn[d] = min_num(mn[d], xyz[3 * i + d]);
      mx[d] = max_num(mx[d], xyz[3 * i + d]);
    }
  for (int d = 0; d < 3; ++d) {
    b->mn[d] = mn[d] - pad;
    mx[d] = mx[d] + pad;
  }
  b->spacing = spacing;
  unsigned __int128 total = 1;
  for (int d = 0; d < 3; ++d) {
    const double span = std::ceil(((mx[d] - b->mn[d]) / spacing) - 1e-10);
    if (!(span < 9.0e18)) return false;
    b->n[d] = (uint64_t)std::max(span, 0.0) + 1;
    total *= b->n[d];
    if (total > (unsigned __int128)UINT64_MAX) return false;
  }
  *count = (uint64_t)total;
  return true;
}

}  // namespace

GridResult adaptive_grid_device(crab_ctx* ctx, const double* xyz, int64_t n, double spacing, double clearance,
                                double padding, bool to_host) {
  GridResult r;
  if (n == 0) {
    r.voxel_volume = adaptive_site_volume(spacing);
    return r;
  }
  require(std::isfinite(spacing) && spacing > 0.0 && std::isfinite(clearance) && clearance > 0.0 &&
              std::isfinite(padding) && padding >= 0.0,
          "adaptive hydration-grid dimensions must be finite and positive");
  // centroid and radius of gyration in the reference's order (solvent.rs:144-155)
  double c[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) c[d] = c[d] + xyz[3 * i + d];
  for (int d = 0; d < 3; ++d) c[d] = c[d] / (double)n;
  double acc = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double dx = xyz[3 * i] - c[0], dy = xyz[3 * i + 1] - c[1], dz = xyz[3 * i + 2] - c[2];
    acc += ((0.0 + dx * dx) + dy * dy) + dz * dz;
  }
  const double rg = std::sqrt(acc / (double)n);
  const double inner = clearance, outer = clearance + adaptive_shell_width(rg);
  Box b;
  uint64_t count = 0;
  require(make_box(xyz, n, padding, spacing, &b, &count), "adaptive hydration grid is too large");
  require(count <= (uint64_t)4000000000ull, "adaptive hydration grid exceeds 4e9 voxels");
  TraceScope trace("adaptive_grid");
  ++ctx->grid_builds;
  GridPoolTrim trim{ctx, !to_host};
  cudaStream_t s = ctx->stream;
  uint8_t* shell = pool<uint8_t>(ctx, "grid.mask_a", count);
  uint8_t* mol = pool<uint8_t>(ctx, "grid.mask_b", count);
  double* d_xyz = pool<double>(ctx, "grid.xyz", 3 * n);
  CRAB_CUDA_CHECK(cudaMemsetAsync(shell, 0, count, s));
  CRAB_CUDA_CHECK(cudaMemsetAsync(mol, 0, count, s));
  copy_h2d(ctx, d_xyz, xyz, 3 * n * sizeof(double), s);
  const unsigned blocks = (unsigned)((n * 32 + 255) / 256);
  k_rasterize<<<blocks, 256, 0, s>>>(d_xyz, nullptr, outer, 0.0, n, b, shell, 1, 0);
  CRAB_CUDA_CHECK(cudaGetLastError());
  k_rasterize<<<blocks, 256, 0, s>>>(d_xyz, nullptr, inner, 0.0, n, b, mol, 1, 0);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 2;
  r = compact_sites(ctx, shell, mol, count, 0, b, to_host);
  r.voxel_volume = adaptive_site_volume(spacing);
  return r;
}

GridResult exterior_grid_device(crab_ctx* ctx, const double* xyz, const int8_t* elem, int64_t n, double spacing,
                                double probe, double thickness, bool to_host) {
  GridResult r;
  if (n == 0) {
    r.voxel_volume = (spacing * spacing) * spacing;
    return r;
  }
  require(std::isfinite(spacing) && spacing > 0.0 && std::isfinite(probe) && probe >= 0.0 &&
              std::isfinite(thickness) && thickness > 0.0,
          "solvent-grid dimensions must be finite and positive");
  double vmax = 0.0;
  std::vector<double> radius(n);
  for (int64_t i = 0; i < n; ++i) {
    radius[i] = vdw_radius(elem[i]);
    vmax = max_num(vmax, radius[i]);
  }
  const double margin = vmax + probe + thickness + spacing;
  Box b;
  uint64_t count = 0;
  require(make_box(xyz, n, margin, spacing, &b, &count), "solvent grid is too large");
  if (count > 250000000ull)
    throw Error(CRAB_EINVAL, "solvent grid requires " + std::to_string(count) + " voxels; limit is 250000000");
  TraceScope trace("exterior_grid");
  ++ctx->grid_builds;
  GridPoolTrim trim{ctx, !to_host};
  cudaStream_t s = ctx->stream;
  uint8_t* state = pool<uint8_t>(ctx, "grid.mask_a", count);
  double* d_xyz = pool<double>(ctx, "grid.xyz", 3 * n);
  double* d_rad = pool<double>(ctx, "grid.radius", n);
  int* d_changed = pool<int>(ctx, "grid.changed", kRoundsPerSync);
  CRAB_CUDA_CHECK(cudaMemsetAsync(state, 0, count, s));
  copy_h2d(ctx, d_xyz, xyz, 3 * n * sizeof(double), s);
  copy_h2d(ctx, d_rad, radius.data(), n * sizeof(double), s);
  const unsigned blocks = (unsigned)((n * 32 + 255) / 256);
  k_rasterize<<<blocks, 256, 0, s>>>(d_xyz, d_rad, 0.0, probe, n, b, state, 1, 0);
  CRAB_CUDA_CHECK(cudaGetLastError());
  k_seed_boundary<<<std::max<unsigned>(1, (unsigned)std::min<uint64_t>((count + 255) / 256, 65535)), 256, 0, s>>>(state, b);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 2;
  // Sweep rounds until the fixed point, kRoundsPerSync rounds per read of the
  // flag: round k writes d_changed[k] and returns at once when round k - 1
  // changed nothing, so the last flag of a batch is 0 exactly when the fill
  // has converged.  Every productive round labels at least one voxel, so the
  // number of rounds cannot exceed the number of voxels.
  for (uint64_t round = 0; round <= count; round += kRoundsPerSync) {
    CRAB_CUDA_CHECK(cudaMemsetAsync(d_changed, 0, kRoundsPerSync * sizeof(int), s));
    for (int k = 0; k < kRoundsPerSync; ++k) {
      const int* prev = k ? d_changed + k - 1 : nullptr;
      for (int axis = 0; axis < 3; ++axis) {
        const uint64_t lines = axis == 0 ? b.n[1] * b.n[2] : axis == 1 ? b.n[0] * b.n[2] : b.n[0] * b.n[1];
        if (b.n[axis] <= (uint64_t)kWarpLine)  // one warp per line
          k_sweep_warp<<<(unsigned)((lines + 3) / 4), 128, 0, s>>>(state, b, axis, prev, d_changed + k);
        else  // one thread per line
          k_sweep<<<(unsigned)((lines + 127) / 128), 128, 0, s>>>(state, b, axis, prev, d_changed + k);
        CRAB_CUDA_CHECK(cudaGetLastError());
        ctx->launches += 1;
      }
    }
    int changed = 0;
    copy_d2h(ctx, &changed, d_changed + kRoundsPerSync - 1, sizeof(int), s);
    CRAB_CUDA_CHECK(cudaStreamSynchronize(s));
    if (!changed) break;
  }
  trace_mark("flood fill");
  k_rasterize<<<blocks, 256, 0, s>>>(d_xyz, d_rad, 0.0, probe + thickness, n, b, state, 3, 1);
  CRAB_CUDA_CHECK(cudaGetLastError());
  ctx->launches += 1;
  r = compact_sites(ctx, state, state, count, 1, b, to_host);
  r.voxel_volume = (spacing * spacing) * spacing;
  return r;
}

void trim_grid_pool(crab_ctx* ctx) { trim_slots(ctx, false); }

}  // namespace crab

// ------------------------------------------------------- no-allocation variant
//
// crab_hydration_grid_adaptive_noalloc is for callers that cannot allocate
// device memory through the CUDA runtime (a host runtime whose own allocator
// owns the device, a process that must keep its memory budget fixed, code
// running inside a callback where cudaMalloc is not allowed).  It takes
// device pointers for the atoms and the site output and keeps every
// temporary (voxel masks, chunk counts, offsets, the box header) in one
// file-scope __device__ array of fixed size, so it calls no cudaMalloc,
// cudaFree or allocating library routine.

#include <mutex>

namespace crab {
namespace {

constexpr uint64_t kNoAllocMaxVoxels = CRAB_NOALLOC_MAX_VOXELS;
static_assert(kNoAllocMaxVoxels % kChunk == 0, "voxel limit must be a whole number of scan chunks");
constexpr uint64_t kNoAllocChunks = kNoAllocMaxVoxels / kChunk;

struct NoAllocHeader {
  Box box;
  uint64_t count;
  double inner, outer;
  int status;  // 0 ok, 1 grid larger than the static scratch, 2 a coordinate not finite
};
static_assert(sizeof(NoAllocHeader) <= 256, "header must fit its 256-byte slot");

constexpr size_t kHdrBytes = 256;
constexpr size_t kShellOff = kHdrBytes;
constexpr size_t kMolOff = kShellOff + kNoAllocMaxVoxels;
constexpr size_t kCntOff = kMolOff + kNoAllocMaxVoxels;
constexpr size_t kOffOff = kCntOff + kNoAllocChunks * sizeof(uint32_t);
constexpr size_t kNoAllocBytes = kOffOff + (kNoAllocChunks + 1) * sizeof(uint64_t);

// The scratch shared by every call on a device; it keeps the last call's
// contents, and calls whose kernels overlap on the GPU race on it.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Single-thread prologue in the reference's sequential order
// (solvent.rs:144-176): centroid, radius of gyration, shell radii, padded box.
__global__ void k_noalloc_prologue(const double* __restrict__ xyz, int64_t n, double spacing, double clearance,
                                   double padding, NoAllocHeader* hdr) {
  double c[3] = {0.0, 0.0, 0.0};
  bool finite = true;  // the allocating entry point rejects the same input (crab_structure_create)
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      finite = finite && isfinite(xyz[3 * i + d]);
      c[d] = __dadd_rn(c[d], xyz[3 * i + d]);
    }
  if (!finite) {
    hdr->status = 2;
    hdr->count = 0ull;
    return;
  }
  for (int d = 0; d < 3; ++d) c[d] = __ddiv_rn(c[d], (double)n);
  double acc = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double dx = __dsub_rn(xyz[3 * i], c[0]), dy = __dsub_rn(xyz[3 * i + 1], c[1]),
                 dz = __dsub_rn(xyz[3 * i + 2], c[2]);
    acc = __dadd_rn(acc, norm2_rn(dx, dy, dz));
  }
  const double rg = sqrt(__ddiv_rn(acc, (double)n));
  const double width = rg <= 15.0 ? 3.0 : (rg >= 20.0 ? 5.0 : __dadd_rn(3.0, __dmul_rn(0.4, __dsub_rn(rg, 15.0))));
  hdr->inner = clearance;
  hdr->outer = __dadd_rn(clearance, width);
  double mn[3] = {xyz[0], xyz[1], xyz[2]}, mx[3] = {xyz[0], xyz[1], xyz[2]};
  for (int64_t i = 1; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      mn[d] = fmin(mn[d], xyz[3 * i + d]);
      mx[d] = fmax(mx[d], xyz[3 * i + d]);
    }
  double total = 1.0;
  for (int d = 0; d < 3; ++d) {
    hdr->box.mn[d] = __dsub_rn(mn[d], padding);
    const double hi = __dadd_rn(mx[d], padding);
    const double span = ceil(__dsub_rn(__ddiv_rn(__dsub_rn(hi, hdr->box.mn[d]), spacing), 1e-10));
    const double nd = fmax(span, 0.0) + 1.0;
    total *= nd;
    hdr->box.n[d] = nd < 9.0e15 ? (uint64_t)nd : 0ull;
  }
  hdr->box.spacing = spacing;
  hdr->status = total > (double)kNoAllocMaxVoxels ? 1 : 0;
  hdr->count = hdr->status ? 0ull : hdr->box.n[0] * hdr->box.n[1] * hdr->box.n[2];
}

// k_emit restricted to the caller's capacity; no voxel indices.
__global__ void k_noalloc_emit(const uint8_t* __restrict__ shell, const uint8_t* __restrict__ mol, uint64_t count,
                               Box bx, const uint64_t* __restrict__ offsets, double* __restrict__ sites,
                               uint64_t capacity) {
  __shared__ uint32_t warp_tot[kScanThreads / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kChunk + (uint64_t)threadIdx.x * kPerThread;
  uint32_t c = 0;
  for (int i = 0; i < kPerThread; ++i)
    if (base + i < count && site_flag(shell, mol, base + i, 0)) ++c;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; ++w) before += warp_tot[w];
  uint64_t pos = offsets[blockIdx.x] + before + incl - c;
  for (int i = 0; i < kPerThread; ++i) {
    const uint64_t v = base + i;
    if (v < count && site_flag(shell, mol, v, 0)) {
      if (pos < capacity) {
        const uint64_t x = v % bx.n[0], y = (v / bx.n[0]) % bx.n[1], z = v / (bx.n[0] * bx.n[1]);
        sites[3 * pos] = __dadd_rn(bx.mn[0], __dmul_rn((double)x, bx.spacing));
        sites[3 * pos + 1] = __dadd_rn(bx.mn[1], __dmul_rn((double)y, bx.spacing));
        sites[3 * pos + 2] = __dadd_rn(bx.mn[2], __dmul_rn((double)z, bx.spacing));
      }
      ++pos;
    }
  }
}

// Device address of the scratch array, looked up once per device (the name
// g_noalloc_scratch is only a host-side handle; kernels need this address).
// The cached address belongs to the device's current CUDA context: after a
// cudaDeviceReset of that device it is stale, so a process that resets a
// device must not call the entry point on it again.
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_dev[256] = {};

cudaError_t noalloc_scratch(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_dev[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_dev[dev] = (unsigned char*)p;
  }
  *out = g_noalloc_dev[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace crab

extern "C" int crab_hydration_grid_adaptive_noalloc(const double* d_xyz, int64_t n, double spacing, double clearance,
                                                    double padding, double* d_sites, int64_t capacity, int64_t* m,
                                                    double* voxel_volume, void* stream) {
  using namespace crab;
  if (n < 0 || capacity < 0 || !m || (n > 0 && !d_xyz) || (capacity > 0 && !d_sites)) return CRAB_EINVAL;
  if (!std::isfinite(spacing) || spacing <= 0.0 || !std::isfinite(clearance) || clearance <= 0.0 ||
      !std::isfinite(padding) || padding < 0.0)
    return CRAB_EINVAL;
  if (voxel_volume) *voxel_volume = adaptive_site_volume(spacing);
  *m = 0;
  if (n == 0) return CRAB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned char* base = nullptr;
  if (noalloc_scratch(&base) != cudaSuccess) return CRAB_ECUDA;
  NoAllocHeader* hdr = (NoAllocHeader*)base;
  k_noalloc_prologue<<<1, 1, 0, s>>>(d_xyz, n, spacing, clearance, padding, hdr);
  if (cudaGetLastError() != cudaSuccess) return CRAB_ECUDA;
  NoAllocHeader h;
  if (cudaMemcpyAsync(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CRAB_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return CRAB_ECUDA;
  if (h.status) return CRAB_EINVAL;  // a coordinate not finite, or a grid larger than CRAB_NOALLOC_MAX_VOXELS
  uint8_t* shell = base + kShellOff;
  uint8_t* mol = base + kMolOff;
  uint32_t* cnt = (uint32_t*)(base + kCntOff);
  uint64_t* off = (uint64_t*)(base + kOffOff);
  // the masks keep the previous call's voxels: clear the part this grid uses
  if (cudaMemsetAsync(shell, 0, h.count, s) != cudaSuccess || cudaMemsetAsync(mol, 0, h.count, s) != cudaSuccess)
    return CRAB_ECUDA;
  const unsigned blocks = (unsigned)((n * 32 + 255) / 256);
  k_rasterize<<<blocks, 256, 0, s>>>(d_xyz, nullptr, h.outer, 0.0, n, h.box, shell, 1, 0);
  k_rasterize<<<blocks, 256, 0, s>>>(d_xyz, nullptr, h.inner, 0.0, n, h.box, mol, 1, 0);
  const uint64_t chunks = (h.count + kChunk - 1) / kChunk;
  k_count<<<(unsigned)chunks, kScanThreads, 0, s>>>(shell, mol, h.count, 0, cnt);
  k_scan_chunks<<<1, 1024, 0, s>>>(cnt, chunks, off);
  if (cudaGetLastError() != cudaSuccess) return CRAB_ECUDA;
  uint64_t total = 0;
  if (cudaMemcpyAsync(&total, off + chunks, sizeof(total), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CRAB_ECUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return CRAB_ECUDA;
  *m = (int64_t)total;
  if (total > 0 && capacity > 0) {
    k_noalloc_emit<<<(unsigned)chunks, kScanThreads, 0, s>>>(shell, mol, h.count, h.box, off, d_sites,
                                                            (uint64_t)capacity);
    if (cudaGetLastError() != cudaSuccess) return CRAB_ECUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CRAB_ECUDA;
  }
  return (capacity > 0 && (int64_t)total > capacity) ? CRAB_ECAPACITY : CRAB_OK;
}
