// Packed float32 fused convolution for Blackwell (sm_100a): the separable
// 13-tap turbulon filters of conv.cu's fused kernel, rebuilt around the
// hardware's paired float32 arithmetic and its tensor-copy engine.
//
// One CTA owns a 32 (y) x 32 (z) cross-section and marches along a chunk of
// x.  Per input x-plane:
//   * the (y, z) slab with its halo -- 44 rows x 48 columns, z from z0 - 8 so
//     that the copy starts on a 16-byte boundary -- arrives by ONE tensor copy
//     (cp.async.bulk.tensor, zero fill outside the array for the linear z
//     padding) that completes on an mbarrier; tiles whose rows wrap around y
//     take 22 two-row copies with the rows wrapped.  Four slab buffers keep
//     three planes in flight.
//   * z filters: one task = one staged row x 8 output columns, computed as
//     column pairs with f32x2 fused multiply-adds (fma.rn.f32x2) over the
//     even filters' folded tap pairs; results to shared memory.
//   * y filters and the (z, y) pair mixing: each thread owns rows (2g, 2g+1)
//     x columns (2p, 2p+1) and reads its columns as 8-byte pairs.
//   * x filters: a ring of 13 paired accumulators per row in registers; an
//     output plane is final 12 planes after its first contribution and goes
//     straight through the epilogue (store, or the flux update with its clip
//     count and window sum).
// One CTA barrier per plane.  Every paired operation rounds each lane as its
// scalar form does; the sums are the same as the scalar fused kernel's up to
// the order of the pair folding.
#include <cuda.h>

#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "conv.cuh"

namespace steam {

int chunk_override(int64_t nx, int64_t ny, int64_t nz);  // conv.cu

namespace {

constexpr int kPK = 13;              // taps per axis
constexpr int kPH = (kPK - 1) / 2;   // the filters' centre (half width)
constexpr int kPZ = 32;              // output columns per tile
constexpr int kPLead = 8;            // staged columns before the tile
constexpr int kPC = kPZ + 2 * kPLead;  // staged columns (z0 - 8 .. z0 + 39)
constexpr int kPStages = 4;          // slab buffers
constexpr int kPChunkMin = 16;
// polls of a slab's mbarrier before a block gives up (a tensor copy lands in
// microseconds; this is seconds)
constexpr long long kTmaWaitLimit = 1ll << 24;

// A tile of TY output rows (32 or 64) x kPZ columns: TY / 2 x 16 threads, each
// owning 2 rows x 2 columns; TY + 12 staged rows.  The arithmetic of an output
// voxel is the same for every tile height, so the height (chosen per shape by
// the autotuner) never changes a result.
template <int TY>
struct PTile {
  static constexpr int Y = TY;
  static constexpr int R = TY + kPK - 1;        // staged rows
  static constexpr int Threads = TY * 8;
  static constexpr int Slab = R * kPC;          // floats per slab buffer
  static constexpr int U = R * kPZ;             // floats per z-filter output plane
  static constexpr int Tasks = R * (kPZ / 8);   // z-filter tasks (8 columns each)
  static constexpr int MinBlocks = TY == 32 ? 2 : 1;
  static constexpr size_t Smem =
      sizeof(float) * ((size_t)kPStages * Slab + 4 * (size_t)U + kPC) +
      sizeof(uint64_t) * kPStages;
  static_assert(R % 2 == 0, "edge tiles copy the slab in row pairs");
  static_assert(Tasks <= Threads, "one z-filter task per thread");
  static_assert((Slab * 4) % 128 == 0, "slab buffers stay 128-byte aligned");
};

// Filters as {t, t} pairs (kernel-parameter constants): z and y filters by
// distance from the centre (tap kPH + d, d = 0..6), x filters by tap index,
// mix by (a, c * 2 + b).
struct PackedTaps {
  float2 z[2][kPH + 1];
  float2 y[2][kPH + 1];
  float2 x[2][kPK];
  float2 mix[2][4];
  int cx;
};

struct PackedGeom {
  int64_t nx, ny;
  int nz, nzt, nyt;
  int64_t chunk;
  long long wait_limit;  // polls of a slab's mbarrier before the block gives up
  int withhold;          // test hook: no slab copy is issued, so every wait runs out
};

// steam_set_copy_wait: the wait limit (default kTmaWaitLimit) and the test
// hook (default off), read when a launch is enqueued or a group prepared
std::atomic<long long> g_copy_wait_limit{kTmaWaitLimit};
std::atomic<int> g_copy_withhold{0};

__device__ unsigned g_tma_wait_errors;
std::atomic<long long> g_packed_launches{0};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// waits for the phase of `parity` to complete, at most `limit` polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit) {
  for (long long i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// a box of the 3D tensor map (x fastest: z, y, plane) into shared memory,
// completing `bar`'s transaction count; no multicast
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0,
                                            int c1, int c2, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// z filters of one staged row, output columns 8q .. 8q + 7 of the tile.
// Window element e is staged column 8q + 2 + e; output column 8q + o has its
// centre at e = o + 6.
template <bool PRE, int U>
__device__ __forceinline__ void z_task(const float* __restrict__ sl, float* __restrict__ su,
                                       const float* __restrict__ s_pre,
                                       const PackedTaps& tp, int task) {
  const int r = task >> 2, q = task & 3;
  const float* src = sl + r * kPC + 8 * q + 2;
  float w[20];
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    float2 v = *reinterpret_cast<const float2*>(src + 2 * i);
    if constexpr (PRE) {
      const float2 s = *reinterpret_cast<const float2*>(s_pre + 8 * q + 2 + 2 * i);
      v = __fmul2_rn(v, s);
    }
    w[2 * i] = v.x;
    w[2 * i + 1] = v.y;
  }
  float2 u0[4], u1[4];
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    const int m = 2 * o + kPH;  // centre of output column 2o
    const float2 c = f2(w[m], w[m + 1]);
    float2 a0 = __fmul2_rn(tp.z[0][0], c);
    float2 a1 = __fmul2_rn(tp.z[1][0], c);
#pragma unroll
    for (int d = 1; d <= kPH; ++d) {
      const float2 ps = __fadd2_rn(f2(w[m + d], w[m + d + 1]), f2(w[m - d], w[m - d + 1]));
      a0 = __ffma2_rn(tp.z[0][d], ps, a0);
      a1 = __ffma2_rn(tp.z[1][d], ps, a1);
    }
    u0[o] = a0;
    u1[o] = a1;
  }
  float* d0 = su + r * kPZ + 8 * q;
  float* d1 = d0 + U;
  *reinterpret_cast<float4*>(d0) = make_float4(u0[0].x, u0[0].y, u0[1].x, u0[1].y);
  *reinterpret_cast<float4*>(d0 + 4) = make_float4(u0[2].x, u0[2].y, u0[3].x, u0[3].y);
  *reinterpret_cast<float4*>(d1) = make_float4(u1[0].x, u1[0].y, u1[1].x, u1[1].y);
  *reinterpret_cast<float4*>(d1 + 4) = make_float4(u1[2].x, u1[2].y, u1[3].x, u1[3].y);
}

// One field's convolution on blocks vb = 0 .. nvb - 1 (the block index and
// count of a launch of its own, or a range of a grouped launch).
template <int TY, bool PRE, bool P3, bool FLUX>
__device__ __forceinline__ void packed_conv_body(
    const CUtensorMap* tm_box, const CUtensorMap* tm_pair, float* __restrict__ out,
    const float* __restrict__ pre, const PackedTaps& tp, const PackedGeom& g, const XEpi& epi,
    double* __restrict__ partials, int vb, int nvb) {
  using Tl = PTile<TY>;
  constexpr int kPY = Tl::Y, kPR = Tl::R, kPThreads = Tl::Threads, kPSlab = Tl::Slab,
                kPU = Tl::U, kPTasks = Tl::Tasks;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ double scratch[32];
  float* slab = reinterpret_cast<float*>(smem_raw);
  float* su0 = slab + kPStages * kPSlab;  // [2 parity][2 filters][kPR][kPZ]
  float* s_pre = su0 + 4 * kPU;           // [kPC]
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_pre + kPC);
  const int t = threadIdx.x, lane = t & 31;
  const int zt_i = vb % g.nzt;
  const int yt_i = (vb / g.nzt) % g.nyt;
  const int64_t xc = vb / ((int64_t)g.nzt * g.nyt);
  const int z0 = zt_i * kPZ;
  const int64_t y0 = (int64_t)yt_i * kPY;
  const int64_t xb = xc * g.chunk;
  const int64_t xe = (xb + g.chunk) < g.nx ? (xb + g.chunk) : g.nx;
  const int count = (int)(xe - xb) + kPK - 1;  // input planes
  const int64_t xin0 = xb - (kPK - 1 - tp.cx);
  const bool interior = y0 - kPH >= 0 && y0 - kPH + kPR <= g.ny;
  if (t == 0) {
    for (int b = 0; b < kPStages; ++b) mbar_init(smem_u32(bars + b), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  for (int c = t; c < kPC; c += kPThreads) {
    const int z = z0 - kPLead + c;
    s_pre[c] = (PRE && z >= 0 && z < g.nz) ? pre_scale(pre[z], pre[g.nz + z]) : 1.0f;
  }
  __syncthreads();
  // warp 0 stages input plane k into buffer k % kPStages
  auto issue = [&](int k) {
    if (g.withhold) return;  // test hook: nothing in flight, every wait runs out
    const int b = k % kPStages;
    const uint32_t bar = smem_u32(bars + b);
    const uint32_t dst = smem_u32(slab + b * kPSlab);
    int64_t xi = (xin0 + k) % g.nx;
    if (xi < 0) xi += g.nx;
    const int zc = z0 - kPLead;
    if (interior) {
      if (lane == 0) {
        mbar_expect_tx(bar, kPSlab * 4);
        tma_load_3d(dst, tm_box, zc, (int)(y0 - kPH), (int)xi, bar);
      }
    } else {
      if (lane == 0) mbar_expect_tx(bar, kPSlab * 4);
      __syncwarp();
      for (int pr = lane; pr < kPR / 2; pr += 32) {
        int64_t yy = (y0 - kPH + 2 * pr) % g.ny;
        if (yy < 0) yy += g.ny;
        tma_load_3d(dst + pr * 2 * kPC * 4, tm_pair, zc, (int)yy, (int)xi, bar);
      }
    }
  };
  if (t < 32)
    for (int k = 0; k < kPStages && k < count; ++k) issue(k);

  // this thread's outputs: rows oy, oy + 1 at columns oz, oz + 1
  const int p = t & 15, gq = t >> 4;
  const int64_t oy = y0 + 2 * gq;
  const int oz = z0 + 2 * p;
  const bool ok = oy < g.ny && oz < g.nz;
  const int64_t plane_elems = g.ny * (int64_t)g.nz;
  const int64_t o0 = oy * g.nz + oz;
  const bool iny0 = oy >= epi.wy0 && oy < epi.wy1;
  const bool iny1 = oy + 1 >= epi.wy0 && oy + 1 < epi.wy1;
  float2 acc[kPK][2];
#pragma unroll
  for (int s = 0; s < kPK; ++s) acc[s][0] = acc[s][1] = f2(0.f, 0.f);
  double s_f = 0.0, s_clip = 0.0;
  int rph = 0;  // ring phase: k mod kPK
  int k = 0;
  bool gave_up = false;
  for (; k < count; ++k) {
    const int b = k % kPStages;
    const bool landed =
        mbar_wait(smem_u32(bars + b), (uint32_t)((k / kPStages) & 1), g.wait_limit);
    const int j = k - (kPK - 1);  // the output plane this iteration completes
    const int64_t x = xb + j;
    float* outp = out + (j >= 0 ? x : 0) * plane_elems;
    float2 fprev0 = f2(0.f, 0.f), fprev1 = f2(0.f, 0.f);
    if (FLUX && j >= 0 && ok) {
      fprev0 = *reinterpret_cast<const float2*>(outp + o0);
      fprev1 = *reinterpret_cast<const float2*>(outp + o0 + g.nz);
    }
    float* su = su0 + (k & 1) * 2 * kPU;
    if (t < kPTasks) z_task<PRE, kPU>(slab + b * kPSlab, su, s_pre, tp, t);
    // one barrier per plane: the z filters of plane k are in su[k & 1] and
    // every read of slab buffer b is done; a block whose copy never landed
    // leaves together
    if (__syncthreads_or(landed ? 0 : 1)) {
      gave_up = true;
      break;
    }
    if (t < 32 && k + kPStages < count) issue(k + kPStages);
    // ---- y filters and the pair mixing for rows 2gq, 2gq + 1
    float2 w0a = f2(0.f, 0.f), w0b = w0a, w1a = w0a, w1b = w0a;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const float* col = su + c * kPU + (2 * gq) * kPZ + 2 * p;
      float2 cv[kPK + 1];
#pragma unroll
      for (int i = 0; i < kPK + 1; ++i) cv[i] = *reinterpret_cast<const float2*>(col + i * kPZ);
      const bool two = !(P3 && c == 1);
      float2 v00 = __fmul2_rn(tp.y[0][0], cv[kPH]);
      float2 v01 = __fmul2_rn(tp.y[0][0], cv[kPH + 1]);
      float2 v10 = f2(0.f, 0.f), v11 = v10;
      if (two) {
        v10 = __fmul2_rn(tp.y[1][0], cv[kPH]);
        v11 = __fmul2_rn(tp.y[1][0], cv[kPH + 1]);
      }
#pragma unroll
      for (int d = 1; d <= kPH; ++d) {
        const float2 ps0 = __fadd2_rn(cv[kPH + d], cv[kPH - d]);
        const float2 ps1 = __fadd2_rn(cv[kPH + 1 + d], cv[kPH + 1 - d]);
        v00 = __ffma2_rn(tp.y[0][d], ps0, v00);
        v01 = __ffma2_rn(tp.y[0][d], ps1, v01);
        if (two) {
          v10 = __ffma2_rn(tp.y[1][d], ps0, v10);
          v11 = __ffma2_rn(tp.y[1][d], ps1, v11);
        }
      }
      w0a = __ffma2_rn(tp.mix[0][c * 2], v00, w0a);
      w0b = __ffma2_rn(tp.mix[0][c * 2], v01, w0b);
      w1a = __ffma2_rn(tp.mix[1][c * 2], v00, w1a);
      w1b = __ffma2_rn(tp.mix[1][c * 2], v01, w1b);
      if (two) {
        w0a = __ffma2_rn(tp.mix[0][c * 2 + 1], v10, w0a);
        w0b = __ffma2_rn(tp.mix[0][c * 2 + 1], v11, w0b);
        w1a = __ffma2_rn(tp.mix[1][c * 2 + 1], v10, w1a);
        w1b = __ffma2_rn(tp.mix[1][c * 2 + 1], v11, w1b);
      }
    }
    // ---- the ring: plane k feeds output j + i in slot (k + i + 1) mod 13;
    //      output j is then complete and leaves
    const bool in_wx = x >= epi.wx0 && x < epi.wx1;
    auto ring_step = [&](auto rr_c) {
      constexpr int rr = decltype(rr_c)::value;
#pragma unroll
      for (int i = 0; i < kPK; ++i) {
        const int slot = (rr + i + 1) % kPK;
        acc[slot][0] = __ffma2_rn(tp.x[1][i], w1a, __ffma2_rn(tp.x[0][i], w0a, acc[slot][0]));
        acc[slot][1] = __ffma2_rn(tp.x[1][i], w1b, __ffma2_rn(tp.x[0][i], w0b, acc[slot][1]));
      }
      constexpr int es = (rr + 1) % kPK;
      if (j >= 0 && ok) {
        if constexpr (FLUX) {
          float2 f0 = __fadd2_rn(fprev0, acc[es][0]);
          float2 f1 = __fadd2_rn(fprev1, acc[es][1]);
          float e[4] = {f0.x, f0.y, f1.x, f1.y};
#pragma unroll
          for (int i = 0; i < 4; ++i)
            if (e[i] < 0.f) {
              s_clip += 1.0;
              e[i] = 0.f;
            }
          *reinterpret_cast<float2*>(outp + o0) = f2(e[0], e[1]);
          *reinterpret_cast<float2*>(outp + o0 + g.nz) = f2(e[2], e[3]);
          if (in_wx) {
            if (iny0) s_f += (double)e[0] + (double)e[1];
            if (iny1) s_f += (double)e[2] + (double)e[3];
          }
        } else {
          *reinterpret_cast<float2*>(outp + o0) = acc[es][0];
          *reinterpret_cast<float2*>(outp + o0 + g.nz) = acc[es][1];
        }
      }
      acc[es][0] = acc[es][1] = f2(0.f, 0.f);
    };
#define STEAM_PRING_CASE(n) \
  case n:                   \
    ring_step(std::integral_constant<int, n>{}); \
    break;
    switch (rph) {
      STEAM_PRING_CASE(0) STEAM_PRING_CASE(1) STEAM_PRING_CASE(2) STEAM_PRING_CASE(3)
      STEAM_PRING_CASE(4) STEAM_PRING_CASE(5) STEAM_PRING_CASE(6) STEAM_PRING_CASE(7)
      STEAM_PRING_CASE(8) STEAM_PRING_CASE(9) STEAM_PRING_CASE(10) STEAM_PRING_CASE(11)
      STEAM_PRING_CASE(12)
      default: break;
    }
#undef STEAM_PRING_CASE
    rph = rph + 1 == kPK ? 0 : rph + 1;
  }
  if (gave_up) {
    // the copies this block issued and has not consumed: planes k ..
    // min(count, k + kPStages) - 1 (plane k's included); wait for each (again
    // bounded) so that none lands after the block has left
    if (t == 0) {
      const int last = (k + kPStages) < count ? (k + kPStages) : count;
      for (int kk = k; kk < last; ++kk)
        (void)mbar_wait(smem_u32(bars + kk % kPStages), (uint32_t)((kk / kPStages) & 1),
                        g.wait_limit);
      atomicAdd(&g_tma_wait_errors, 1u);
    }
    __syncthreads();
    return;
  }
  if constexpr (FLUX) {
    const double t0 = block_sum(s_f, scratch);
    const double t1 = block_sum(s_clip, scratch);
    if (t == 0) {
      partials[vb] = t0;
      partials[nvb + vb] = t1;
    }
  }
}

template <int TY, bool PRE, bool P3, bool FLUX>
__global__ void __launch_bounds__(PTile<TY>::Threads, PTile<TY>::MinBlocks) packed_conv_kernel(
    const __grid_constant__ CUtensorMap tm_box, const __grid_constant__ CUtensorMap tm_pair,
    float* __restrict__ out, const float* __restrict__ pre,
    const __grid_constant__ PackedTaps tp, PackedGeom g, XEpi epi,
    double* __restrict__ partials) {
  packed_conv_body<TY, PRE, P3, FLUX>(&tm_box, &tm_pair, out, pre, tp, g, epi, partials,
                                      blockIdx.x, gridDim.x);
}

// ---- grouped form: many fields with the same filters, one launch ---------
// A member: its tensor maps (device memory, 64-byte aligned), geometry,
// epilogue window and partial sums, and its range of the launch's blocks.
// Its outputs are the same bits as a launch of its own (a voxel's arithmetic
// does not depend on the tiling); its flux sums too when it keeps its own
// chunk, and to rounding when the group gives it whole-x CTAs.
struct alignas(64) PackedMember {
  CUtensorMap box;
  CUtensorMap pair;
  float* out;
  const float* pre;
  double* partials;  // [2][nblocks] for the flux epilogue
  double* sums;      // the member's flux totals (device, 2 doubles) or null
  PackedGeom g;
  XEpi epi;
  int block0, nblocks;
};

template <int TY, bool PRE, bool P3, bool FLUX>
__global__ void __launch_bounds__(PTile<TY>::Threads, PTile<TY>::MinBlocks) packed_group_kernel(
    const PackedMember* __restrict__ mem, const int* __restrict__ start, int n,
    const __grid_constant__ PackedTaps tp) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(start + mid) <= (int)blockIdx.x)
      lo = mid;
    else
      hi = mid - 1;
  }
  const PackedMember& m = mem[lo];
  const PackedGeom g = m.g;
  const XEpi epi = m.epi;
  packed_conv_body<TY, PRE, P3, FLUX>(&m.box, &m.pair, m.out, m.pre, tp, g, epi, m.partials,
                                      (int)blockIdx.x - m.block0, m.nblocks);
}

// the members' flux totals {sum F over the window, clip count}, one block each
__global__ void packed_group_sums_kernel(const PackedMember* __restrict__ mem) {
  __shared__ double scratch[32];
  const PackedMember& m = mem[blockIdx.x];
  if (!m.sums) return;
  for (int q = 0; q < 2; ++q) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < m.nblocks; i += blockDim.x) acc += m.partials[q * m.nblocks + i];
    const double sum = block_sum(acc, scratch);
    if (threadIdx.x == 0) m.sums[q] = sum;
  }
}

// ---- host side ------------------------------------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// the field as a (nz, ny, nx) float32 tensor (z fastest), boxes of kPC
// columns x `rows` rows x 1 plane
bool encode_map(CUtensorMap* m, const float* base, int64_t nx, int64_t ny, int64_t nz,
                int rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
  const cuuint64_t strides[2] = {(cuuint64_t)nz * 4, (cuuint64_t)(ny * nz) * 4};
  const cuuint32_t box[3] = {(cuuint32_t)kPC, (cuuint32_t)rows, 1};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides,
            box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool even_about_centre(const double* t) {
  for (int d = 1; d <= kPH; ++d)
    if (t[kPH + d] != t[kPH - d]) return false;
  return true;
}

// x planes per CTA: the autotuner's choice for the shape, else the chunk
// that minimises the busiest SM's work.  Two 32-row CTAs fit an SM (registers
// and shared memory) and share its issue slots, so an SM's time is the planes
// of all CTAs it runs, halo included, plus about one CTA's worth for the
// uneven finish; a CTA alone on its SM runs at about 0.7 of the pair's
// throughput (its barrier stalls are not covered).
// output rows per tile for fields of a shape: the autotuner's choice
// (steam_conv_set_tile_rows), 32 otherwise
std::mutex g_rows_mu;
std::map<std::tuple<int64_t, int64_t, int64_t>, int> g_rows;

int packed_rows(int64_t nx, int64_t ny, int64_t nz) {
  std::lock_guard<std::mutex> lock(g_rows_mu);
  auto it = g_rows.find(std::make_tuple(nx, ny, nz));
  return it == g_rows.end() ? 32 : it->second;
}

int64_t packed_chunk(int64_t nx, int64_t ny, int64_t nz) {
  const int over = chunk_override(nx, ny, nz);
  if (over > 0) return over;
  const int rows = packed_rows(nx, ny, nz);
  const int64_t tiles = ((nz + kPZ - 1) / kPZ) * ((ny + rows - 1) / rows);
  const int64_t sms = sm_count();
  int64_t best = nx;
  double best_cost = -1.0;
  for (int64_t n = 1; n <= nx; ++n) {
    const int64_t chunk = (nx + n - 1) / n;
    if (chunk < kPChunkMin && n > 1) break;
    const int64_t ctas = tiles * ((nx + chunk - 1) / chunk);
    const int64_t per_sm = (ctas + sms - 1) / sms;
    // (one more CTA's planes for the spread of CTA times under the hardware's
    // dynamic dispatch; a 64-row CTA has the SM to itself: no pair to cover
    // its stalls)
    const double cost =
        (double)((per_sm + 1) * (chunk + kPK - 1)) / (per_sm == 1 && rows == 32 ? 0.7 : 1.0);
    if (best_cost < 0.0 || cost < best_cost) {
      best_cost = cost;
      best = chunk;
    }
  }
  return best < kPChunkMin && nx >= kPChunkMin ? kPChunkMin : best;
}

template <int TY, bool PRE, bool P3, bool FLUX>
cudaError_t launch_v(const CUtensorMap& box, const CUtensorMap& pair, float* out,
                     const float* pre, const PackedTaps& tp, const PackedGeom& g,
                     const XEpi& epi, double* partials, int64_t grid, cudaStream_t s) {
  using Tl = PTile<TY>;
  auto kern = packed_conv_kernel<TY, PRE, P3, FLUX>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Tl::Smem);
  if (e != cudaSuccess) return e;
  kern<<<(unsigned)grid, Tl::Threads, Tl::Smem, s>>>(box, pair, out, pre, tp, g, epi, partials);
  return cudaGetLastError();
}

template <int TY>
cudaError_t launch_rows(int v, const CUtensorMap& box, const CUtensorMap& pair, float* out,
                        const float* pre, const PackedTaps& tp, const PackedGeom& g,
                        const XEpi& epi, double* partials, int64_t grid, cudaStream_t s) {
  switch (v) {
    case 0: return launch_v<TY, false, false, false>(box, pair, out, pre, tp, g, epi, partials, grid, s);
    case 1: return launch_v<TY, false, false, true>(box, pair, out, pre, tp, g, epi, partials, grid, s);
    case 2: return launch_v<TY, false, true, false>(box, pair, out, pre, tp, g, epi, partials, grid, s);
    case 3: return launch_v<TY, false, true, true>(box, pair, out, pre, tp, g, epi, partials, grid, s);
    case 4: return launch_v<TY, true, false, false>(box, pair, out, pre, tp, g, epi, partials, grid, s);
    case 5: return launch_v<TY, true, false, true>(box, pair, out, pre, tp, g, epi, partials, grid, s);
    case 6: return launch_v<TY, true, true, false>(box, pair, out, pre, tp, g, epi, partials, grid, s);
    default: return launch_v<TY, true, true, true>(box, pair, out, pre, tp, g, epi, partials, grid, s);
  }
}

PackedTaps make_taps(const SepParams<float>& p, bool* p3_out) {
  PackedTaps tp;
  bool p3 = true;
  for (int d = 0; d <= kPH; ++d) {
    for (int f = 0; f < 2; ++f) {
      const float zv = f < p.nzf ? (float)p.ztap(f)[kPH + d] : 0.f;
      const float yv = f < p.nyf ? (float)p.ytap(f)[kPH + d] : 0.f;
      tp.z[f][d] = make_float2(zv, zv);
      tp.y[f][d] = make_float2(yv, yv);
    }
  }
  for (int i = 0; i < kPK; ++i)
    for (int f = 0; f < 2; ++f) {
      const float xv = f < p.nxf ? (float)p.xtap(f)[i] : 0.f;
      tp.x[f][i] = make_float2(xv, xv);
    }
  for (int a = 0; a < 2; ++a)
    for (int cb = 0; cb < 4; ++cb) {
      const int c = cb / 2, b = cb % 2;
      double v = 0.0;
      for (int q = 0; q < p.npairs; ++q)
        if (a < p.nxf && p.pair_z[q] == c && p.pair_y[q] == b) v += p.mix[a * p.npairs + q];
      tp.mix[a][cb] = make_float2((float)v, (float)v);
      if (cb == 3 && (float)v != 0.f) p3 = false;
    }
  tp.cx = p.cx;
  *p3_out = p3;
  return tp;
}

}  // namespace

bool packed_supported(const SepParams<float>& p, int64_t nx, int64_t ny, int64_t nz,
                      const void* in, const void* out, int epilogue) {
  if (epilogue != STEAM_EPI_STORE && epilogue != STEAM_EPI_FLUX) return false;
  if (p.kx != kPK || p.ky != kPK || p.kz != kPK || p.cz != kPH || p.cy != kPH) return false;
  if (p.nzf > 2 || p.nyf > 2 || p.nxf > 2 || p.npairs > 4) return false;
  for (int q = 0; q < p.npairs; ++q)
    if (p.pair_z[q] >= 2 || p.pair_y[q] >= 2) return false;
  for (int f = 0; f < p.nzf; ++f)
    if (!even_about_centre(p.ztap(f))) return false;
  for (int f = 0; f < p.nyf; ++f)
    if (!even_about_centre(p.ytap(f))) return false;
  // (a field thinner than the staged slab takes the same copies: the parts
  // past its extent arrive as zeros)
  if (nz % 4 != 0 || nz < 4 || ny % 2 != 0 || ny < 2 || nx < 1) return false;
  if (nx > INT32_MAX || ny > INT32_MAX || ny * nz > ((int64_t)1 << 31)) return false;
  if (((uintptr_t)in % 16) != 0 || ((uintptr_t)out % 16) != 0) return false;
  CUtensorMap probe;
  return encode_map(&probe, (const float*)in, nx, ny, nz, 2);
}

int64_t packed_grid(int64_t nx, int64_t ny, int64_t nz) {
  const int64_t chunk = packed_chunk(nx, ny, nz);
  const int rows = packed_rows(nx, ny, nz);
  return ((nz + kPZ - 1) / kPZ) * ((ny + rows - 1) / rows) * ((nx + chunk - 1) / chunk);
}

int packed_launch(const SepParams<float>& p, int64_t nx, int64_t ny, int64_t nz,
                  const float* in, float* out, const float* pre, int epilogue,
                  const XEpi& epi, double* partials, cudaStream_t s) {
  const int rows = packed_rows(nx, ny, nz);
  const int kPR = rows + kPK - 1;
  CUtensorMap box, pair;
  if (!encode_map(&pair, in, nx, ny, nz, 2))
    return fail(STEAM_ERR_CUDA, "steam_conv_separable: tensor map encoding failed");
  if (ny >= kPR) {
    if (!encode_map(&box, in, nx, ny, nz, kPR))
      return fail(STEAM_ERR_CUDA, "steam_conv_separable: tensor map encoding failed");
  } else {
    box = pair;  // every tile wraps in y: only the row-pair copies run
  }
  bool p3 = true;
  const PackedTaps tp = make_taps(p, &p3);
  PackedGeom g;
  g.nx = nx;
  g.ny = ny;
  g.nz = (int)nz;
  g.nzt = (int)((nz + kPZ - 1) / kPZ);
  g.nyt = (int)((ny + rows - 1) / rows);
  g.chunk = packed_chunk(nx, ny, nz);
  g.wait_limit = g_copy_wait_limit.load();
  g.withhold = g_copy_withhold.load();
  const int64_t grid = (int64_t)g.nzt * g.nyt * ((nx + g.chunk - 1) / g.chunk);
  STEAM_REQUIRE(grid < ((int64_t)1 << 31), "steam_conv_separable: grid too large");
  const int v = (pre != nullptr ? 4 : 0) | (p3 ? 2 : 0) | (epilogue == STEAM_EPI_FLUX ? 1 : 0);
  cudaError_t e = rows == 64
                      ? launch_rows<64>(v, box, pair, out, pre, tp, g, epi, partials, grid, s)
                      : launch_rows<32>(v, box, pair, out, pre, tp, g, epi, partials, grid, s);
  count_launch();
  if (e != cudaSuccess)
    return fail(STEAM_ERR_CUDA, std::string("conv packed launch: ") + cudaGetErrorString(e));
  g_packed_launches.fetch_add(1);
  return STEAM_OK;
}

// ---- grouped launches -------------------------------------------------------
struct PackedGroupPlan {
  int n = 0, total = 0, variant = 0;
  PackedTaps tp;
  PackedMember* mem = nullptr;
  int* start = nullptr;
};
static std::mutex g_pgroup_mu;
static std::map<void*, PackedGroupPlan> g_pgroups;

// A member's x chunk in a group: its whole x extent when the group's tiles
// alone give every SM at least kGroupTilesPerSm CTAs (the other members fill
// the GPU, so a member needs no short chunks of its own, and whole-x CTAs
// carry no repeated 12-plane halo), its own launch's chunk otherwise.
constexpr int kGroupTilesPerSm = 4;

static int64_t member_tiles(int64_t ny, int64_t nz) {
  return ((nz + kPZ - 1) / kPZ) * ((ny + 32 - 1) / 32);
}

static bool group_whole_x(int n, const steam_conv_problem_t* q) {
  int64_t tiles = 0;
  for (int i = 0; i < n; ++i) tiles += member_tiles(q[i].ny, q[i].nz);
  return tiles >= (int64_t)kGroupTilesPerSm * sm_count();
}

static int64_t group_member_chunk(const steam_conv_problem_t& m, bool whole_x) {
  return whole_x ? m.nx : packed_chunk(m.nx, m.ny, m.nz);
}

size_t packed_group_bytes(int n, const steam_conv_problem_t* q) {
  size_t b = carve_bytes((size_t)n, sizeof(PackedMember)) + carve_bytes((size_t)n, sizeof(int));
  const bool whole_x = group_whole_x(n, q);
  for (int i = 0; i < n; ++i) {
    const int64_t chunk = group_member_chunk(q[i], whole_x);
    b += carve_bytes((size_t)2 * member_tiles(q[i].ny, q[i].nz) *
                         ((q[i].nx + chunk - 1) / chunk),
                     sizeof(double));
  }
  return b + 4096;
}

int packed_group_prepare(const SepParams<float>& p, int n, const steam_conv_problem_t* q,
                         int epilogue, void* ws, size_t ws_bytes) {
  STEAM_REQUIRE(epilogue == STEAM_EPI_STORE || epilogue == STEAM_EPI_FLUX,
                "steam_conv_group_prepare: epilogue must be STORE or FLUX");
  STEAM_REQUIRE(p.cx == kPH, "steam_conv_group_prepare: the x filter's centre must be 6");
  const bool pre = q[0].pre != nullptr;
  for (int i = 0; i < n; ++i) {
    const steam_conv_problem_t& m = q[i];
    const std::string who = "steam_conv_group_prepare: field " + std::to_string(i);
    STEAM_REQUIRE((m.pre != nullptr) == pre, who + ": every field or none takes the scaling");
    STEAM_REQUIRE(m.nx >= kPK && m.ny >= kPK, who + ": narrower than the filters");
    STEAM_REQUIRE(packed_rows(m.nx, m.ny, m.nz) == 32, who + ": tuned to 64-row tiles");
    STEAM_REQUIRE(packed_supported(p, m.nx, m.ny, m.nz, m.in, m.out, epilogue),
                  who + ": not a packed-kernel layout (float32, nz % 4 == 0, ny even, "
                        "16-byte aligned)");
    if (m.has_window) {
      STEAM_REQUIRE(m.window.x0 >= 0 && m.window.x1 <= m.nx && m.window.x0 < m.window.x1 &&
                        m.window.y0 >= 0 && m.window.y1 <= m.ny && m.window.y0 < m.window.y1,
                    who + ": window outside the array");
    }
  }
  Carver c(ws, ws_bytes);
  PackedGroupPlan plan;
  plan.n = n;
  plan.mem = c.take<PackedMember>((size_t)n);
  plan.start = c.take<int>((size_t)n);
  if (!plan.mem || !plan.start)
    return fail(STEAM_ERR_WORKSPACE, "steam_conv_group_prepare: workspace too small");
  std::vector<PackedMember> mem((size_t)n);
  std::vector<int> start((size_t)n);
  const bool whole_x = group_whole_x(n, q);
  int64_t total = 0;
  for (int i = 0; i < n; ++i) {
    const steam_conv_problem_t& m = q[i];
    PackedMember& r = mem[(size_t)i];
    if (!encode_map(&r.pair, (const float*)m.in, m.nx, m.ny, m.nz, 2))
      return fail(STEAM_ERR_CUDA, "steam_conv_group_prepare: tensor map encoding failed");
    if (m.ny >= 32 + kPK - 1) {
      if (!encode_map(&r.box, (const float*)m.in, m.nx, m.ny, m.nz, 32 + kPK - 1))
        return fail(STEAM_ERR_CUDA, "steam_conv_group_prepare: tensor map encoding failed");
    } else {
      r.box = r.pair;
    }
    r.out = (float*)m.out;
    r.pre = (const float*)m.pre;
    r.g.nx = m.nx;
    r.g.ny = m.ny;
    r.g.nz = (int)m.nz;
    r.g.nzt = (int)((m.nz + kPZ - 1) / kPZ);
    r.g.nyt = (int)((m.ny + 31) / 32);
    r.g.chunk = group_member_chunk(m, whole_x);
    r.g.wait_limit = g_copy_wait_limit.load();
    r.g.withhold = g_copy_withhold.load();
    r.epi.mode = epilogue;
    r.epi.wx0 = m.has_window ? m.window.x0 : 0;
    r.epi.wx1 = m.has_window ? m.window.x1 : m.nx;
    r.epi.wy0 = m.has_window ? m.window.y0 : 0;
    r.epi.wy1 = m.has_window ? m.window.y1 : m.ny;
    const int64_t nb = (int64_t)r.g.nzt * r.g.nyt * ((m.nx + r.g.chunk - 1) / r.g.chunk);
    r.partials = c.take<double>((size_t)2 * nb);
    if (!r.partials)
      return fail(STEAM_ERR_WORKSPACE, "steam_conv_group_prepare: workspace too small");
    r.sums = epilogue == STEAM_EPI_FLUX ? m.sums : nullptr;
    r.block0 = (int)total;
    r.nblocks = (int)nb;
    start[(size_t)i] = (int)total;
    total += nb;
    STEAM_REQUIRE(total < ((int64_t)1 << 31), "steam_conv_group_prepare: grid too large");
  }
  bool p3 = true;
  plan.tp = make_taps(p, &p3);
  plan.total = (int)total;
  plan.variant = (pre ? 4 : 0) | (p3 ? 2 : 0) | (epilogue == STEAM_EPI_FLUX ? 1 : 0);
  STEAM_CUDA(cudaMemcpy(plan.mem, mem.data(), sizeof(PackedMember) * (size_t)n,
                        cudaMemcpyHostToDevice));
  STEAM_CUDA(cudaMemcpy(plan.start, start.data(), sizeof(int) * (size_t)n,
                        cudaMemcpyHostToDevice));
  std::lock_guard<std::mutex> lock(g_pgroup_mu);
  g_pgroups[ws] = plan;
  return STEAM_OK;
}

namespace {
template <bool PRE, bool P3, bool FLUX>
cudaError_t group_launch_v(const PackedGroupPlan& plan, cudaStream_t s) {
  using Tl = PTile<32>;
  auto kern = packed_group_kernel<32, PRE, P3, FLUX>;
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Tl::Smem);
  if (e != cudaSuccess) return e;
  kern<<<(unsigned)plan.total, Tl::Threads, Tl::Smem, s>>>(plan.mem, plan.start, plan.n,
                                                           plan.tp);
  return cudaGetLastError();
}
}  // namespace

int packed_group_enqueue(void* ws, cudaStream_t s) {
  PackedGroupPlan plan;
  {
    std::lock_guard<std::mutex> lock(g_pgroup_mu);
    auto it = g_pgroups.find(ws);
    STEAM_REQUIRE(it != g_pgroups.end(),
                  "steam_conv_group_async: workspace holds no prepared group");
    plan = it->second;
  }
  cudaError_t e;
  switch (plan.variant) {
    case 0: e = group_launch_v<false, false, false>(plan, s); break;
    case 1: e = group_launch_v<false, false, true>(plan, s); break;
    case 2: e = group_launch_v<false, true, false>(plan, s); break;
    case 3: e = group_launch_v<false, true, true>(plan, s); break;
    case 4: e = group_launch_v<true, false, false>(plan, s); break;
    case 5: e = group_launch_v<true, false, true>(plan, s); break;
    case 6: e = group_launch_v<true, true, false>(plan, s); break;
    default: e = group_launch_v<true, true, true>(plan, s); break;
  }
  count_launch();
  if (e != cudaSuccess)
    return fail(STEAM_ERR_CUDA, std::string("conv group launch: ") + cudaGetErrorString(e));
  g_packed_launches.fetch_add(1);
  if (plan.variant & 1) {
    packed_group_sums_kernel<<<plan.n, 256, 0, s>>>(plan.mem);
    STEAM_LAUNCH_CHECK("conv group sums");
  }
  return STEAM_OK;
}

int packed_group_release(void* ws) {
  std::lock_guard<std::mutex> lock(g_pgroup_mu);
  g_pgroups.erase(ws);
  return STEAM_OK;
}

}  // namespace steam

extern "C" int64_t steam_conv_packed_launches(void) { return steam::g_packed_launches.load(); }

extern "C" int steam_conv_set_tile_rows(int64_t nx, int64_t ny, int64_t nz, int32_t rows) {
  STEAM_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1, "steam_conv_set_tile_rows: empty shape");
  STEAM_REQUIRE(rows == 0 || rows == 32 || rows == 64,
                "steam_conv_set_tile_rows: rows must be 0 (default), 32 or 64");
  std::lock_guard<std::mutex> lock(steam::g_rows_mu);
  if (rows == 0)
    steam::g_rows.erase(std::make_tuple(nx, ny, nz));
  else
    steam::g_rows[std::make_tuple(nx, ny, nz)] = rows;
  return STEAM_OK;
}

extern "C" int steam_conv_get_tile_rows(int64_t nx, int64_t ny, int64_t nz) {
  return steam::packed_rows(nx, ny, nz);
}

extern "C" int steam_set_copy_wait(int64_t polls, int32_t withhold) {
  if (polls < 0 || (withhold != 0 && withhold != 1))
    return steam::fail(STEAM_ERR_ARG, "steam_set_copy_wait: polls >= 0, withhold 0 or 1");
  steam::g_copy_wait_limit.store(polls == 0 ? steam::kTmaWaitLimit : (long long)polls);
  steam::g_copy_withhold.store(withhold);
  return STEAM_OK;
}

extern "C" int steam_take_wait_errors(int32_t* count) {
  if (!count) return steam::fail(STEAM_ERR_ARG, "steam_take_wait_errors: count is null");
  unsigned h = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&h, steam::g_tma_wait_errors, sizeof(h)) != cudaSuccess)
    return steam::fail(STEAM_ERR_CUDA, "steam_take_wait_errors: read failed");
  if (h && cudaMemcpyToSymbol(steam::g_tma_wait_errors, &zero, sizeof(zero)) != cudaSuccess)
    return steam::fail(STEAM_ERR_CUDA, "steam_take_wait_errors: reset failed");
  *count = (int32_t)h;
  return STEAM_OK;
}
