// Circular-x/y, linear-z convolution on a separable network of 1D filters
// (the turbulon kernels are sums of a few separable terms).  Kernels without
// such a form go to fftconv.cu.
//
// Kernels the fused forms below do not take run as three passes, each a
// coalesced stencil over the z-fastest layout:
//   z-pass: u_c = f (*)_z Z_c
//   y-pass: w_a = sum_p mix_ap (u_c(p) (*)_y Y_b(p))
//   x-pass: out = sum_a w_a (*)_x X_a, with the epilogue,
// in float64 with scalar windows (tiles 32 columns wide: float64 fields, and
// float32 fields under the flux epilogue or the wide store) or, for a plain
// float32 convolution, paired (f32x2 windows on two adjacent columns: tiles
// 64 columns wide).
#include "common.cuh"
#include "conv.cuh"
#include <type_traits>

#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

#include <memory>
#include <vector>

namespace steam {

// ---- the three passes: shared structure ------------------------------------
// Each pass is a 1D correlation along one axis with every thread computing
// kSR consecutive outputs of that axis for one lane column: the taps, reversed
// and zero-padded to a multiple of kSU, sit in shared memory (one broadcast
// read per tap), the inputs in a register window of kSR + kSU - 1 values that
// slides by kSU taps per step, so a group of kSU taps costs kSU shared loads,
// kSU tap reads and kSR * kSU fused multiply-adds.  A is the arithmetic type:
// the field's own for a plain convolution, float64 for the flux epilogue and
// the wide store (the fused kernels make the same choice).
//
// With reversed taps r[m] = t[Kp - 1 - m] (zero for Kp - 1 - m >= K) and a
// staged line b[j] = f[j - (Kp - 1 - c)], output i of a filter with centre c
// is sum_m r[m] * b[i + m] = sum_l t[l] * f[i + c - l].
constexpr int kSR = 8;  // outputs per thread along the filter axis
constexpr int kSU = 8;  // taps per window step

__host__ __device__ inline int sep_padded(int k) { return (k + kSU - 1) / kSU * kSU; }

template <typename A>
__device__ __forceinline__ A fma_a(A a, A b, A c);
template <>
__device__ __forceinline__ float fma_a<float>(float a, float b, float c) {
  return __fmaf_rn(a, b, c);
}
template <>
__device__ __forceinline__ double fma_a<double>(double a, double b, double c) {
  return __fma_rn(a, b, c);
}

// kSU taps from shared memory by 16-byte loads (p 16-byte aligned).
__device__ __forceinline__ void load_taps(const float* p, float (&t)[kSU]) {
#pragma unroll
  for (int i = 0; i < kSU; i += 4) {
    const float4 v = *reinterpret_cast<const float4*>(p + i);
    t[i] = v.x;
    t[i + 1] = v.y;
    t[i + 2] = v.z;
    t[i + 3] = v.w;
  }
}
__device__ __forceinline__ void load_taps(const double* p, double (&t)[kSU]) {
#pragma unroll
  for (int i = 0; i < kSU; i += 2) {
    const double2 v = *reinterpret_cast<const double2*>(p + i);
    t[i] = v.x;
    t[i + 1] = v.y;
  }
}

// acc[r] += sum_m taps[m] * line[(r + m) * stride], m < kp (kp % kSU == 0,
// taps 16-byte aligned).  The step loop is unrolled twice so that the
// window's shift is a register renaming on every other step.
template <typename A>
__device__ __forceinline__ void sep_window(const A* __restrict__ line, int stride,
                                           const A* __restrict__ taps, int kp,
                                           A (&acc)[kSR]) {
  A w[kSR + kSU - 1];
#pragma unroll
  for (int i = 0; i < kSR - 1; ++i) w[i] = line[i * stride];
#pragma unroll 2
  for (int m0 = 0; m0 < kp; m0 += kSU) {
#pragma unroll
    for (int u = 0; u < kSU; ++u) w[kSR - 1 + u] = line[(m0 + kSR - 1 + u) * stride];
    A tv[kSU];
    load_taps(taps + m0, tv);
#pragma unroll
    for (int u = 0; u < kSU; ++u) {
      const A t = tv[u];
#pragma unroll
      for (int r = 0; r < kSR; ++r) acc[r] = fma_a<A>(t, w[r + u], acc[r]);
    }
#pragma unroll
    for (int i = 0; i < kSR - 1; ++i) w[i] = w[kSU + i];
  }
}

// v mod n in [0, n) for int extents; two compares on the common index
// within one period of the range.
__device__ __forceinline__ int wrap32(int v, int n) {
  if (v < 0) {
    v += n;
    if (v < 0) {
      v %= n;
      if (v < 0) v += n;
    }
  } else if (v >= n) {
    v -= n;
    if (v >= n) v %= n;
  }
  return v;
}

// taps_s[f * kp + m] = taps[f * k + (kp - 1 - m)], zero past the filter.
template <typename A>
__device__ __forceinline__ void stage_taps(A* taps_s, const double* taps, int nf, int k,
                                           int kp) {
  for (int i = threadIdx.x; i < nf * kp; i += blockDim.x) {
    const int f = i / kp, l = kp - 1 - (i - f * kp);
    taps_s[i] = l < k ? (A)taps[f * k + l] : (A)0;
  }
}

// One staged element: by cp.async when the field has the arithmetic type
// (zero-filled when not valid; the source is then not read), converted
// through registers otherwise.
template <typename T, typename A>
__device__ __forceinline__ void stage_elem(A* dst, const T* src, bool valid) {
  if constexpr (std::is_same<T, A>::value) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(A) == 4)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(src),
                   "r"(valid ? 4 : 0)
                   : "memory");
    else
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(src),
                   "r"(valid ? 8 : 0)
                   : "memory");
  } else {
    *dst = valid ? (A)*src : (A)0;
  }
}

// ---- z-pass -------------------------------------------------------------
// Tile = 32 consecutive columns (one per lane) x a chunk of z of 8 warps x
// SPW segments x kSR outputs; the columns are staged with their halo at an
// odd pitch (conflict-free column reads across the lanes) and each filter's
// outputs go back through a second buffer so that the stores run along z.
constexpr int kZCols = 32;
constexpr int kPassThreads = 256;

template <typename A>
constexpr int zpass_spw() { return sizeof(A) == 4 ? 4 : 2; }
template <typename A>
constexpr int zpass_chunk() { return (kPassThreads / 32) * kSR * zpass_spw<A>(); }

template <typename A>
static size_t zpass_smem(int nf, int kp) {
  const int zc = zpass_chunk<A>();
  const int ld = (zc + kp - 1) | 1;
  return sizeof(A) * ((size_t)nf * kp + (size_t)kZCols * ld + (size_t)kZCols * (zc + 1));
}

template <typename T, typename A, bool PRE>
__global__ void __launch_bounds__(kPassThreads) zpass_kernel(
    const T* __restrict__ in, int64_t ncol, int nz, int kp, const T* __restrict__ pre_div,
    const T* __restrict__ pre_mul, SepParams<T> p, T* __restrict__ out, int64_t plane) {
  constexpr int SPW = zpass_spw<A>();
  constexpr int ZC = zpass_chunk<A>();
  constexpr int NW = kPassThreads / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* taps_s = reinterpret_cast<A*>(smem_raw);
  const int ld = (ZC + kp - 1) | 1;
  constexpr int ldo = ZC + 1;
  A* buf = taps_s + p.nzf * kp;
  A* obuf = buf + kZCols * ld;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int off = kp - 1 - p.cz;
  stage_taps<A>(taps_s, p.ztap(0), p.nzf, p.kz, kp);
  const int64_t zchunks = (nz + ZC - 1) / ZC;
  const int64_t ntiles = ((ncol + kZCols - 1) / kZCols) * zchunks;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t col0 = (t / zchunks) * kZCols;
    const int z0 = (int)(t % zchunks) * ZC;
    const int zc = (nz - z0) < ZC ? (nz - z0) : ZC;
    const int nseg = (zc + kSR - 1) / kSR;
    const int len = nseg * kSR + kp - 1;
    const int ncb = (int)((ncol - col0) < kZCols ? (ncol - col0) : kZCols);
    __syncthreads();
    for (int c = warp; c < kZCols; c += NW) {
      const T* src = in + (col0 + (c < ncb ? c : 0)) * nz;
      for (int j = lane; j < len; j += 32) {
        const int s = z0 + j - off;
        const bool valid = c < ncb && s >= 0 && s < nz;
        stage_elem<T, A>(buf + c * ld + j, src + (valid ? s : 0), valid);
      }
    }
    cp_async_commit();
    cp_async_wait<0>();
    if (PRE) {
      // each thread scales the elements it staged itself (zeros stay zero)
      for (int c = warp; c < kZCols; c += NW) {
        for (int j = lane; j < len; j += 32) {
          const int s = z0 + j - off;
          if (c < ncb && s >= 0 && s < nz)
            buf[c * ld + j] = (A)mul_rn((T)buf[c * ld + j], pre_scale(pre_div[s], pre_mul[s]));
        }
      }
    }
    __syncthreads();
    for (int f = 0; f < p.nzf; ++f) {
      A acc[SPW][kSR];
#pragma unroll
      for (int q = 0; q < SPW; ++q) {
#pragma unroll
        for (int r = 0; r < kSR; ++r) acc[q][r] = (A)0;
        const int seg = warp + q * NW;
        if (seg < nseg)
          sep_window<A>(buf + lane * ld + seg * kSR, 1, taps_s + f * kp, kp, acc[q]);
      }
      __syncthreads();  // the previous filter's outputs have left obuf
#pragma unroll
      for (int q = 0; q < SPW; ++q) {
        const int seg = warp + q * NW;
        if (seg < nseg) {
#pragma unroll
          for (int r = 0; r < kSR; ++r) obuf[lane * ldo + seg * kSR + r] = acc[q][r];
        }
      }
      __syncthreads();
      T* o = out + f * plane + col0 * nz + z0;
      for (int c = warp; c < ncb; c += NW)
        for (int j = lane; j < zc; j += 32) o[(int64_t)c * nz + j] = (T)obuf[c * ldo + j];
    }
  }
}

// ---- y-pass -------------------------------------------------------------
// Tile = one x-plane's kYT rows x 32 z (one per lane), each warp owning kSR
// consecutive rows.  The tile's z-filtered fields are staged in turn with
// kp - 1 halo rows (wrapped: y is circular); every (z filter, y filter) pair
// on a field is one window run, folded at once into the x filters' mixes
// w_a = sum_q mix[a][q] v_q, so the pass writes nxf fields, not one per pair.
// A block's work is a sequence of stages (tile, input field); the rows of
// stage k + 1 are copied into the second of two buffers while stage k is
// computed (the x-pass runs the same way).
constexpr int kYT = (kPassThreads / 32) * kSR;  // 64 rows

template <typename A>
static size_t ypass_smem(int nyf, int kp) {
  return sizeof(A) * ((size_t)nyf * kp + (size_t)2 * (kYT + kp - 1) * 32);
}

template <typename T, typename A, int NX>
__global__ void __launch_bounds__(kPassThreads, 3) ypass_kernel(
    const T* __restrict__ u, int64_t nx, int64_t ny, int nz, int kp, SepParams<T> p,
    T* __restrict__ w, int64_t plane) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* taps_s = reinterpret_cast<A*>(smem_raw);
  const int rows = kYT + kp - 1;
  A* bufs = taps_s + p.nyf * kp;  // 2 x [kYT + kp - 1][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = kPassThreads / 32;
  const int off = kp - 1 - p.cy;
  const int nf = p.nzf;
  stage_taps<A>(taps_s, p.ytap(0), p.nyf, p.ky, kp);
  // tile t = (x, y tile, z tile), z fastest; the host keeps every count
  // below 2^31, so tile and row indices are 32-bit
  const int ny32 = (int)ny;
  const unsigned ytiles = (unsigned)((ny + kYT - 1) / kYT);
  const unsigned ztiles = (unsigned)((nz + 31) / 32);
  const unsigned ntiles = (unsigned)nx * ytiles * ztiles;
  const unsigned nfu = (unsigned)nf;
  // stage k: tile blockIdx.x + (k / nf) * gridDim.x, field k % nf
  auto issue = [&](unsigned k) {
    const unsigned t = blockIdx.x + (k / nfu) * gridDim.x;
    if (t < ntiles) {
      const int f = (int)(k % nfu);
      const unsigned rest = t / ztiles;
      const int z = (int)(t - rest * ztiles) * 32 + lane;
      const unsigned x = rest / ytiles;
      const int y0 = (int)(rest - x * ytiles) * kYT;
      const T* src = u + (int64_t)f * plane + ((int64_t)x * ny) * nz + (z < nz ? z : 0);
      A* dst = bufs + (k & 1) * rows * 32 + lane;
      for (int r = warp; r < rows; r += NW)
        stage_elem<T, A>(dst + r * 32, src + (int64_t)wrap32(y0 - off + r, ny32) * nz,
                         z < nz);
    }
    cp_async_commit();
  };
  A acc[NX][kSR];
  issue(0);
  for (unsigned k = 0;; ++k) {
    const unsigned t = blockIdx.x + (k / nfu) * gridDim.x;
    if (t >= ntiles) break;
    const int f = (int)(k % nfu);
    issue(k + 1);
    cp_async_wait<1>();
    __syncthreads();
    if (f == 0) {
#pragma unroll
      for (int a = 0; a < NX; ++a)
#pragma unroll
        for (int r = 0; r < kSR; ++r) acc[a][r] = (A)0;
    }
    const A* col = bufs + (k & 1) * rows * 32 + warp * kSR * 32 + lane;
    for (int q = 0; q < p.npairs; ++q) {
      if (p.pair_z[q] != f) continue;
      A c[kSR];
#pragma unroll
      for (int r = 0; r < kSR; ++r) c[r] = (A)0;
      sep_window<A>(col, 32, taps_s + p.pair_y[q] * kp, kp, c);
#pragma unroll
      for (int a = 0; a < NX; ++a) {
        if (a < p.nxf) {
          const A m = (A)p.mix[a * p.npairs + q];
#pragma unroll
          for (int r = 0; r < kSR; ++r) acc[a][r] = fma_a<A>(m, c[r], acc[a][r]);
        }
      }
    }
    if (f == nf - 1) {
      const unsigned rest = t / ztiles;
      const int z = (int)(t - rest * ztiles) * 32 + lane;
      const unsigned x = rest / ytiles;
      const int yw = (int)(rest - x * ytiles) * kYT + warp * kSR;
      if (z < nz) {
#pragma unroll
        for (int a = 0; a < NX; ++a) {
          if (a < p.nxf) {
            T* o = w + (int64_t)a * plane + ((int64_t)x * ny + yw) * nz + z;
#pragma unroll
            for (int r = 0; r < kSR; ++r)
              if (yw + r < ny) o[(int64_t)r * nz] = (T)acc[a][r];
          }
        }
      }
    }
    __syncthreads();  // stage k's buffer is free for stage k + 2
  }
  cp_async_wait<0>();
}

// ---- x-pass -------------------------------------------------------------
// Tile = kXT x-planes x 32 elements of the (y, z) plane (one per lane), each
// warp owning kSR consecutive x outputs; each x filter's mixed field is
// staged in turn with kp - 1 halo planes (wrapped: x is circular) and its
// window run adds into the same accumulators; the epilogue follows in
// registers.  Tiles run x-fastest, so neighbouring tiles' halo rows come
// from L2.
constexpr int kXT = (kPassThreads / 32) * kSR;  // 64 planes

template <typename A>
static size_t xpass_smem(int nxf, int kp) {
  return sizeof(A) * ((size_t)nxf * kp + (size_t)2 * (kXT + kp - 1) * 32);
}

static int64_t xpass_tiles(int64_t nx, int64_t ny, int64_t nz) {
  return ((nx + kXT - 1) / kXT) * ((ny * nz + 31) / 32);
}

template <typename T, typename A>
__global__ void __launch_bounds__(kPassThreads) xpass_kernel(
    const T* __restrict__ w, int64_t nx, int64_t ny, int nz, int kp, SepParams<T> p,
    T* __restrict__ out, int64_t plane, XEpi epi, double* __restrict__ partials) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double scratch[32];
  A* taps_s = reinterpret_cast<A*>(smem_raw);
  const int rows = kXT + kp - 1;
  A* bufs = taps_s + p.nxf * kp;  // 2 x [kXT + kp - 1][32]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = kPassThreads / 32;
  const int off = kp - 1 - p.cx;
  const int nf = p.nxf;
  stage_taps<A>(taps_s, p.xtap(0), p.nxf, p.kx, kp);
  // tile t = (32-element group of the (y, z) plane, x tile), x fastest; the
  // host keeps every count below 2^31, so tile and plane indices are 32-bit
  const int nx32 = (int)nx;
  const int pe = (int)(ny * nz);  // elements of one x-plane
  const unsigned xtiles = (unsigned)((nx + kXT - 1) / kXT);
  const unsigned ntiles = xtiles * (unsigned)((pe + 31) / 32);
  const unsigned nfu = (unsigned)nf;
  // stage k: tile blockIdx.x + (k / nf) * gridDim.x, x filter k % nf
  auto issue = [&](unsigned k) {
    const unsigned t = blockIdx.x + (k / nfu) * gridDim.x;
    if (t < ntiles) {
      const int a = (int)(k % nfu);
      const unsigned et = t / xtiles;
      const int x0 = (int)(t - et * xtiles) * kXT;
      const int e = (int)et * 32 + lane;
      const T* src = w + (int64_t)a * plane + (e < pe ? e : 0);
      A* dst = bufs + (k & 1) * rows * 32 + lane;
      for (int r = warp; r < rows; r += NW)
        stage_elem<T, A>(dst + r * 32, src + (int64_t)wrap32(x0 - off + r, nx32) * pe, e < pe);
    }
    cp_async_commit();
  };
  double s_f = 0.0, s_clip = 0.0;
  A acc[kSR];
  issue(0);
  for (unsigned k = 0;; ++k) {
    const unsigned t = blockIdx.x + (k / nfu) * gridDim.x;
    if (t >= ntiles) break;
    const int a = (int)(k % nfu);
    issue(k + 1);
    cp_async_wait<1>();
    __syncthreads();
    if (a == 0) {
#pragma unroll
      for (int r = 0; r < kSR; ++r) acc[r] = (A)0;
    }
    sep_window<A>(bufs + (k & 1) * rows * 32 + warp * kSR * 32 + lane, 32, taps_s + a * kp,
                  kp, acc);
    const unsigned et = t / xtiles;
    const int e = (int)et * 32 + lane;
    if (a == nf - 1 && e < pe) {
      const int xw = (int)(t - et * xtiles) * kXT + warp * kSR;
      bool in_win = false;
      if (epi.mode == STEAM_EPI_FLUX) {
        const int y = e / nz;
        in_win = y >= epi.wy0 && y < epi.wy1;
      }
#pragma unroll
      for (int r = 0; r < kSR; ++r) {
        const int x = xw + r;
        if (x < nx32) {
          const int64_t o = (int64_t)x * pe + e;
          if (epi.mode == STEAM_EPI_FLUX) {
            // F + conv rounded once to the storage dtype
            T f = (T)((double)out[o] + (double)acc[r]);
            if (f < (T)0) {
              s_clip += 1.0;
              f = (T)0;
            }
            out[o] = f;
            if (in_win && x >= epi.wx0 && x < epi.wx1) s_f += (double)f;
          } else {
            out[o] = (T)acc[r];
          }
        }
      }
    }
    __syncthreads();  // stage k's buffer is free for stage k + 2
  }
  cp_async_wait<0>();
  if (epi.mode == STEAM_EPI_FLUX) {
    double t0 = block_sum(s_f, scratch);
    double t1 = block_sum(s_clip, scratch);
    if (threadIdx.x == 0) {
      partials[blockIdx.x] = t0;
      partials[gridDim.x + blockIdx.x] = t1;
    }
  }
}

// ---- paired y and x passes (float32 fields, float32 arithmetic) -------------
// The same passes with each thread owning two adjacent columns of the
// stencil (z in the y pass, the (y, z) element in the x pass): a staged row is
// read as one 8-byte pair per lane, and every tap is one fma.rn.f32x2 on a
// {t, t} pair, each lane of which rounds as the scalar fma.  Tiles are
// 64 wide; a pair whose second column is past the end is staged as zero and
// not stored.

// acc[r] += sum_m taps2[m] * line[(r + m) * stride] on pairs.
__device__ __forceinline__ void sep_window2(const float2* __restrict__ line, int stride,
                                            const float2* __restrict__ taps2, int kp,
                                            float2 (&acc)[kSR]) {
  float2 w[kSR + kSU - 1];
#pragma unroll
  for (int i = 0; i < kSR - 1; ++i) w[i] = line[i * stride];
#pragma unroll 2
  for (int m0 = 0; m0 < kp; m0 += kSU) {
#pragma unroll
    for (int u = 0; u < kSU; ++u) w[kSR - 1 + u] = line[(m0 + kSR - 1 + u) * stride];
    float2 tv[kSU];
#pragma unroll
    for (int u = 0; u < kSU; u += 2) {
      const float4 v = *reinterpret_cast<const float4*>(taps2 + m0 + u);
      tv[u] = make_float2(v.x, v.y);
      tv[u + 1] = make_float2(v.z, v.w);
    }
#pragma unroll
    for (int u = 0; u < kSU; ++u) {
#pragma unroll
      for (int r = 0; r < kSR; ++r) acc[r] = __ffma2_rn(tv[u], w[r + u], acc[r]);
    }
#pragma unroll
    for (int i = 0; i < kSR - 1; ++i) w[i] = w[kSU + i];
  }
}

// taps2[f * kp + m] = {t, t}, t = taps[f * k + (kp - 1 - m)], zero past the filter.
__device__ __forceinline__ void stage_taps2(float2* taps2, const double* taps, int nf, int k,
                                            int kp) {
  for (int i = threadIdx.x; i < nf * kp; i += blockDim.x) {
    const int f = i / kp, l = kp - 1 - (i - f * kp);
    const float t = l < k ? (float)taps[f * k + l] : 0.0f;
    taps2[i] = make_float2(t, t);
  }
}

// Two adjacent elements src[0], src[1] into dst (8-byte aligned): one 8-byte
// copy when both are in range and the source is 8-byte aligned, else two
// 4-byte copies, each zero-filled when out of range.
__device__ __forceinline__ void stage_pair(float2* dst, const float* src, int n_valid,
                                           bool aligned) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  if (aligned) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(src),
                 "r"(n_valid >= 2 ? 8 : 0)
                 : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(src),
                 "r"(n_valid >= 1 ? 4 : 0)
                 : "memory");
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s + 4),
                 "l"(src + (n_valid >= 2 ? 1 : 0)), "r"(n_valid >= 2 ? 4 : 0)
                 : "memory");
  }
}

// Stores the pair's in-range elements.
__device__ __forceinline__ void store_pair(float* dst, float2 v, int n_valid, bool aligned) {
  if (aligned && n_valid >= 2) {
    *reinterpret_cast<float2*>(dst) = v;
  } else {
    if (n_valid >= 1) dst[0] = v.x;
    if (n_valid >= 2) dst[1] = v.y;
  }
}

constexpr int kPairW = 64;  // tile width in columns (32 lanes x 2)

static size_t ypass2_smem(int nyf, int kp) {
  return sizeof(float2) * ((size_t)nyf * kp + (size_t)2 * (kYT + kp - 1) * 32);
}

template <int NX>
__global__ void __launch_bounds__(kPassThreads) ypass2_kernel(
    const float* __restrict__ u, int64_t nx, int64_t ny, int nz, int kp, SepParams<float> p,
    float* __restrict__ w, int64_t plane) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* taps2 = reinterpret_cast<float2*>(smem_raw);
  const int rows = kYT + kp - 1;
  float2* bufs = taps2 + p.nyf * kp;  // 2 x [kYT + kp - 1][32 pairs]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = kPassThreads / 32;
  const int off = kp - 1 - p.cy;
  const int nf = p.nzf;
  stage_taps2(taps2, p.ytap(0), p.nyf, p.ky, kp);
  const int ny32 = (int)ny;
  const bool aligned = (nz & 1) == 0;
  const unsigned ytiles = (unsigned)((ny + kYT - 1) / kYT);
  const unsigned ztiles = (unsigned)((nz + kPairW - 1) / kPairW);
  const unsigned ntiles = (unsigned)nx * ytiles * ztiles;
  const unsigned nfu = (unsigned)nf;
  auto issue = [&](unsigned k) {
    const unsigned t = blockIdx.x + (k / nfu) * gridDim.x;
    if (t < ntiles) {
      const int f = (int)(k % nfu);
      const unsigned rest = t / ztiles;
      const int z = (int)(t - rest * ztiles) * kPairW + 2 * lane;
      const unsigned x = rest / ytiles;
      const int y0 = (int)(rest - x * ytiles) * kYT;
      const int nv = nz - z;
      const float* src = u + (int64_t)f * plane + ((int64_t)x * ny) * nz + (nv > 0 ? z : 0);
      float2* dst = bufs + (k & 1) * rows * 32 + lane;
      const int ys0 = y0 - off;
      if (ys0 >= 0 && ys0 + rows <= ny32) {
        const float* s = src + (int64_t)(ys0 + warp) * nz;
        const int64_t step = (int64_t)NW * nz;
        for (int r = warp; r < rows; r += NW, s += step) stage_pair(dst + r * 32, s, nv, aligned);
      } else {
        for (int r = warp; r < rows; r += NW)
          stage_pair(dst + r * 32, src + (int64_t)wrap32(ys0 + r, ny32) * nz, nv, aligned);
      }
    }
    cp_async_commit();
  };
  float2 acc[NX][kSR];
  issue(0);
  for (unsigned k = 0;; ++k) {
    const unsigned t = blockIdx.x + (k / nfu) * gridDim.x;
    if (t >= ntiles) break;
    const int f = (int)(k % nfu);
    issue(k + 1);
    cp_async_wait<1>();
    __syncthreads();
    if (f == 0) {
#pragma unroll
      for (int a = 0; a < NX; ++a)
#pragma unroll
        for (int r = 0; r < kSR; ++r) acc[a][r] = make_float2(0.0f, 0.0f);
    }
    const float2* col = bufs + (k & 1) * rows * 32 + warp * kSR * 32 + lane;
    for (int q = 0; q < p.npairs; ++q) {
      if (p.pair_z[q] != f) continue;
      float2 c[kSR];
#pragma unroll
      for (int r = 0; r < kSR; ++r) c[r] = make_float2(0.0f, 0.0f);
      sep_window2(col, 32, taps2 + p.pair_y[q] * kp, kp, c);
#pragma unroll
      for (int a = 0; a < NX; ++a) {
        if (a < p.nxf) {
          const float m = (float)p.mix[a * p.npairs + q];
          const float2 m2 = make_float2(m, m);
#pragma unroll
          for (int r = 0; r < kSR; ++r) acc[a][r] = __ffma2_rn(m2, c[r], acc[a][r]);
        }
      }
    }
    if (f == nf - 1) {
      const unsigned rest = t / ztiles;
      const int z = (int)(t - rest * ztiles) * kPairW + 2 * lane;
      const unsigned x = rest / ytiles;
      const int yw = (int)(rest - x * ytiles) * kYT + warp * kSR;
      const int nv = nz - z;
      if (nv > 0) {
#pragma unroll
        for (int a = 0; a < NX; ++a) {
          if (a < p.nxf) {
            float* o = w + (int64_t)a * plane + ((int64_t)x * ny + yw) * nz + z;
#pragma unroll
            for (int r = 0; r < kSR; ++r)
              if (yw + r < ny32) store_pair(o + (int64_t)r * nz, acc[a][r], nv, aligned);
          }
        }
      }
    }
    __syncthreads();  // stage k's buffer is free for stage k + 2
  }
  cp_async_wait<0>();
}

// Paired z-pass: tile = 64 consecutive columns x kZ2 z; the columns are staged
// transposed (row j = one z level of the 64 columns, pitch 66 floats: the
// pair reads are 8-byte aligned and conflict-free, the staging writes at most
// two-way conflicted), so each thread's window runs down z on its two columns
// as pairs; stages are double-buffered, one per tile, and the outputs go
// straight to global memory (16-byte stores when nz % 4 == 0).
constexpr int kZ2 = 128;      // z outputs per tile
constexpr int kZ2Pitch = 66;  // floats per staged row

static size_t zpass2_smem(int nzf, int kp) {
  return sizeof(float2) * (size_t)nzf * kp +
         sizeof(float) * (size_t)2 * (kZ2 + kp - 1) * kZ2Pitch;
}

template <bool PRE>
__global__ void __launch_bounds__(kPassThreads) zpass2_kernel(
    const float* __restrict__ in, int64_t ncol, int nz, int kp, const float* __restrict__ pre_div,
    const float* __restrict__ pre_mul, SepParams<float> p, float* __restrict__ out,
    int64_t plane) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* taps2 = reinterpret_cast<float2*>(smem_raw);
  float* bufs = reinterpret_cast<float*>(taps2 + p.nzf * kp);  // 2 x [kZ2 + kp - 1][66]
  const int rows = kZ2 + kp - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = kPassThreads / 32;
  const int off = kp - 1 - p.cz;
  stage_taps2(taps2, p.ztap(0), p.nzf, p.kz, kp);
  const unsigned zchunks = (unsigned)((nz + kZ2 - 1) / kZ2);
  const unsigned ntiles = (unsigned)((ncol + kPairW - 1) / kPairW) * zchunks;
  const bool vec = (nz & 3) == 0;
  // stage k = tile blockIdx.x + k * gridDim.x: (column block, z chunk), z fastest
  auto issue = [&](unsigned k) {
    const unsigned t = blockIdx.x + k * gridDim.x;
    if (t < ntiles) {
      const unsigned cb = t / zchunks;
      const int z0 = (int)(t - cb * zchunks) * kZ2;
      const int64_t col0 = (int64_t)cb * kPairW;
      const int ncb = (int)((ncol - col0) < kPairW ? (ncol - col0) : kPairW);
      float* buf = bufs + (k & 1) * rows * kZ2Pitch;
      for (int c = warp; c < kPairW; c += NW) {
        const float* src = in + (col0 + (c < ncb ? c : 0)) * nz;
        for (int j = lane; j < rows; j += 32) {
          const int s = z0 - off + j;
          const bool valid = c < ncb && s >= 0 && s < nz;
          stage_elem<float, float>(buf + j * kZ2Pitch + c, src + (valid ? s : 0), valid);
        }
      }
    }
    cp_async_commit();
  };
  issue(0);
  for (unsigned k = 0;; ++k) {
    const unsigned t = blockIdx.x + k * gridDim.x;
    if (t >= ntiles) break;
    issue(k + 1);
    cp_async_wait<1>();
    const unsigned cb = t / zchunks;
    const int z0 = (int)(t - cb * zchunks) * kZ2;
    const int64_t col0 = (int64_t)cb * kPairW;
    const int ncb = (int)((ncol - col0) < kPairW ? (ncol - col0) : kPairW);
    const int zc = (nz - z0) < kZ2 ? (nz - z0) : kZ2;
    float* buf = bufs + (k & 1) * rows * kZ2Pitch;
    if (PRE) {
      // each thread scales the elements it staged itself (zeros stay zero)
      for (int c = warp; c < ncb; c += NW) {
        for (int j = lane; j < rows; j += 32) {
          const int s = z0 - off + j;
          if (s >= 0 && s < nz)
            buf[j * kZ2Pitch + c] = mul_rn(buf[j * kZ2Pitch + c], pre_scale(pre_div[s], pre_mul[s]));
        }
      }
    }
    __syncthreads();
    const int c = 2 * lane;
    const int nv = ncb - c;  // columns of this thread's pair in range
    for (int seg = warp; seg * kSR < zc; seg += NW) {
      const float2* col = reinterpret_cast<const float2*>(buf + seg * kSR * kZ2Pitch) + lane;
      for (int f = 0; f < p.nzf; ++f) {
        float2 acc[kSR];
#pragma unroll
        for (int r = 0; r < kSR; ++r) acc[r] = make_float2(0.0f, 0.0f);
        sep_window2(col, kZ2Pitch / 2, taps2 + f * kp, kp, acc);
        if (nv > 0) {
          const int zs = z0 + seg * kSR;
          float* o0 = out + f * plane + (col0 + c) * nz + zs;
          if (vec && zs + kSR <= nz) {
            *reinterpret_cast<float4*>(o0) = make_float4(acc[0].x, acc[1].x, acc[2].x, acc[3].x);
            *reinterpret_cast<float4*>(o0 + 4) =
                make_float4(acc[4].x, acc[5].x, acc[6].x, acc[7].x);
            if (nv > 1) {
              *reinterpret_cast<float4*>(o0 + nz) =
                  make_float4(acc[0].y, acc[1].y, acc[2].y, acc[3].y);
              *reinterpret_cast<float4*>(o0 + nz + 4) =
                  make_float4(acc[4].y, acc[5].y, acc[6].y, acc[7].y);
            }
          } else {
#pragma unroll
            for (int r = 0; r < kSR; ++r) {
              if (zs + r < nz) {
                o0[r] = acc[r].x;
                if (nv > 1) o0[nz + r] = acc[r].y;
              }
            }
          }
        }
      }
    }
    __syncthreads();  // stage k's buffer is free for stage k + 2
  }
  cp_async_wait<0>();
}


static size_t xpass2_smem(int nxf, int kp) {
  return sizeof(float2) * ((size_t)nxf * kp + (size_t)2 * (kXT + kp - 1) * 32);
}

static int64_t xpass2_tiles(int64_t nx, int64_t ny, int64_t nz) {
  return ((nx + kXT - 1) / kXT) * ((ny * nz + kPairW - 1) / kPairW);
}

// The plain store only (the flux epilogue and the wide store take float64
// arithmetic); aligned_out: out is 8-byte aligned and ny * nz even.
__global__ void __launch_bounds__(kPassThreads) xpass2_kernel(
    const float* __restrict__ w, int64_t nx, int64_t ny, int nz, int kp, SepParams<float> p,
    float* __restrict__ out, int64_t plane, int aligned_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* taps2 = reinterpret_cast<float2*>(smem_raw);
  const int rows = kXT + kp - 1;
  float2* bufs = taps2 + p.nxf * kp;  // 2 x [kXT + kp - 1][32 pairs]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NW = kPassThreads / 32;
  const int off = kp - 1 - p.cx;
  const int nf = p.nxf;
  stage_taps2(taps2, p.xtap(0), p.nxf, p.kx, kp);
  const int nx32 = (int)nx;
  const int pe = (int)(ny * nz);  // elements of one x-plane
  const bool aligned = (pe & 1) == 0;
  const unsigned xtiles = (unsigned)((nx + kXT - 1) / kXT);
  const unsigned ntiles = xtiles * (unsigned)((pe + kPairW - 1) / kPairW);
  const unsigned nfu = (unsigned)nf;
  auto issue = [&](unsigned k) {
    const unsigned t = blockIdx.x + (k / nfu) * gridDim.x;
    if (t < ntiles) {
      const int a = (int)(k % nfu);
      const unsigned et = t / xtiles;
      const int x0 = (int)(t - et * xtiles) * kXT;
      const int e = (int)et * kPairW + 2 * lane;
      const int nv = pe - e;
      const float* src = w + (int64_t)a * plane + (nv > 0 ? e : 0);
      float2* dst = bufs + (k & 1) * rows * 32 + lane;
      const int xs0 = x0 - off;
      if (xs0 >= 0 && xs0 + rows <= nx32) {
        const float* s = src + (int64_t)(xs0 + warp) * pe;
        const int64_t step = (int64_t)NW * pe;
        for (int r = warp; r < rows; r += NW, s += step) stage_pair(dst + r * 32, s, nv, aligned);
      } else {
        for (int r = warp; r < rows; r += NW)
          stage_pair(dst + r * 32, src + (int64_t)wrap32(xs0 + r, nx32) * pe, nv, aligned);
      }
    }
    cp_async_commit();
  };
  float2 acc[kSR];
  issue(0);
  for (unsigned k = 0;; ++k) {
    const unsigned t = blockIdx.x + (k / nfu) * gridDim.x;
    if (t >= ntiles) break;
    const int a = (int)(k % nfu);
    issue(k + 1);
    cp_async_wait<1>();
    __syncthreads();
    if (a == 0) {
#pragma unroll
      for (int r = 0; r < kSR; ++r) acc[r] = make_float2(0.0f, 0.0f);
    }
    sep_window2(bufs + (k & 1) * rows * 32 + warp * kSR * 32 + lane, 32, taps2 + a * kp, kp,
                acc);
    const unsigned et = t / xtiles;
    const int e = (int)et * kPairW + 2 * lane;
    const int nv = pe - e;
    if (a == nf - 1 && nv > 0) {
      const int xw = (int)(t - et * xtiles) * kXT + warp * kSR;
#pragma unroll
      for (int r = 0; r < kSR; ++r)
        if (xw + r < nx32)
          store_pair(out + (int64_t)(xw + r) * pe + e, acc[r], nv, aligned_out != 0);
    }
    __syncthreads();  // stage k's buffer is free for stage k + 2
  }
  cp_async_wait<0>();
}

// ---- fused pencil convolution ----------------------------------------------
// One CTA owns a (kFY x kFZ) cross-section of y and z and marches along a
// chunk of x.  For every input x-plane it stages the plane's (y, z) slab with
// its halo in shared memory (in the arithmetic type A), runs the z filters (4 outputs per
// thread, sliding window) and the y filters (2 rows per thread) on chip, and
// folds the mixed result into a ring of K per-output-plane accumulators held
// in registers (indices static through a uniform switch on the ring phase).
// The next plane's slab is loaded into registers while the current plane is
// computed (two slab buffers).  An output plane is final K-1 planes after its
// first contribution and goes straight through the epilogue.  HBM sees the
// input once (halo re-reads hit L2) and the output once.
//
// A, the type of the taps, the staged slabs and every accumulator: the
// field's own type for a plain convolution (float32 fields are filtered in
// float32, the precision of the reference's float32 FFT, and land closer to
// the float64 result than it does), float64 for the flux epilogue whatever
// the field type: there F + conv cancels to near zero next to the clip, and
// float32 accumulation alone moved the log-flux past 1e-5 relative L2.
constexpr int kFY = 32;
constexpr int kFZ = 16;
constexpr int kFThreads = 256;
constexpr int kFChunk = 256;  // x planes per CTA
constexpr int kFMaxZ = 2, kFMaxPairs = 4, kFMaxX = 2;

template <typename T>
struct FusedGeom {
  int64_t nx, ny;
  int nz;
  int nzt, nyt;   // z and y tiles
  int64_t chunk;  // x planes per CTA
  int use_pre;
};

template <int K>
struct FusedShape {
  static constexpr int R = kFY + K - 1;          // staged rows
  static constexpr int C = kFZ + K - 1;          // staged columns
  static constexpr int NL = (R * C + kFThreads - 1) / kFThreads;  // loads/thread
  static constexpr int ZT = R * (kFZ / 4);       // z-filter tasks (4 outputs each)
};

// The fused kernel's filters as kernel-parameter constants: every tap index
// is a compile-time constant after unrolling, so the multiply-adds read their
// tap straight from the parameter bank (no shared-memory load per tap).
// mix is re-indexed by (a, c, b), the pairs enumerated c-major, b-minor.
__device__ __forceinline__ float fma_a(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_a(double a, double b, double c) { return fma(a, b, c); }

template <typename A, int K>
struct FusedTaps {
  A z[kFMaxZ][K], y[2][K], x[kFMaxX][K];
  A mix[kFMaxX * kFMaxPairs];
  int cx, cy, cz;
  int sym;     // every z and y filter is even about its centre (K - 1) / 2
  int skip11;  // no pair of z filter 1 with y filter 1: that y filter is skipped
};

template <typename T, typename A, int K>
static FusedTaps<A, K> fused_taps(const SepParams<T>& p) {
  FusedTaps<A, K> f;
  for (int i = 0; i < K; ++i) {
    f.z[0][i] = (A)p.taps[i];
    f.z[1][i] = p.nzf > 1 ? (A)p.taps[K + i] : (A)0;
    f.y[0][i] = (A)p.ytap(0)[i];
    f.y[1][i] = p.nyf > 1 ? (A)p.ytap(1)[i] : (A)0;
    f.x[0][i] = (A)p.xtap(0)[i];
    f.x[1][i] = p.nxf > 1 ? (A)p.xtap(1)[i] : (A)0;
  }
  for (int t = 0; t < kFMaxX * kFMaxPairs; ++t) {
    const int a = t / kFMaxPairs, cb = t % kFMaxPairs;
    const int c = cb / 2, b = cb % 2;
    double v = 0.0;
    for (int q = 0; q < p.npairs; ++q)
      if (a < p.nxf && p.pair_z[q] == c && p.pair_y[q] == b) v += p.mix[a * p.npairs + q];
    f.mix[t] = (A)v;
  }
  f.cx = p.cx;
  f.cy = p.cy;
  f.cz = p.cz;
  bool sym = p.cz == (K - 1) / 2 && p.cy == (K - 1) / 2;
  for (int i = 0; sym && i < K; ++i)
    sym = f.z[0][i] == f.z[0][K - 1 - i] && f.z[1][i] == f.z[1][K - 1 - i] &&
          f.y[0][i] == f.y[0][K - 1 - i] && f.y[1][i] == f.y[1][K - 1 - i];
  f.sym = sym ? 1 : 0;
  bool none11 = true;
  for (int a = 0; a < kFMaxX; ++a) none11 = none11 && f.mix[a * kFMaxPairs + 1 * 2 + 1] == (A)0;
  f.skip11 = none11 ? 1 : 0;
  return f;
}

template <typename T, typename A, int K, bool SYM, bool PRE, bool P3>
__global__ void __launch_bounds__(kFThreads, (sizeof(A) == 4 ? (K <= 13 ? 3 : 2) : (K <= 13 ? 2 : 1))) fused_conv_kernel(
    const T* __restrict__ in, T* __restrict__ out, const T* __restrict__ pre,
    const __grid_constant__ FusedTaps<A, K> tp, FusedGeom<T> g, XEpi epi,
    double* __restrict__ partials) {
  static_assert(K <= 25, "the ring dispatch covers K <= 25");
  static_assert((K + 3) % 4 == 0, "the z window moves in groups of 4");
  using S = FusedShape<K>;
  constexpr int R = S::R, C = S::C, NL = S::NL;
  extern __shared__ unsigned char smem_raw[];
  __shared__ double scratch[32];
  __shared__ __align__(16) T s_pre[C];  // read 4 at a time by the z pass
  A* s_in0 = reinterpret_cast<A*>(smem_raw);  // [2][R*C]
  // the z filters' output, double-buffered by plane parity so that one
  // barrier per plane suffices: [2 parity][kFMaxZ][R][kFZ]
  A* s_u0 = s_in0 + 2 * R * C;
  const int t = threadIdx.x;
  const int zt_i = blockIdx.x % g.nzt;
  const int yt_i = (blockIdx.x / g.nzt) % g.nyt;
  const int64_t xc = blockIdx.x / ((int64_t)g.nzt * g.nyt);
  const int64_t y0 = (int64_t)yt_i * kFY;
  const int z0 = zt_i * kFZ;
  const int64_t xb = xc * g.chunk;
  const int64_t xe = (xb + g.chunk) < g.nx ? (xb + g.chunk) : g.nx;
  const int64_t count = (xe - xb) + K - 1;  // planes to process
  const int64_t xin0 = xb - (K - 1 - tp.cx);
  const int padz = K - 1 - tp.cz, pady = K - 1 - tp.cy;
  for (int c = t; c < C; c += kFThreads) {
    const int z = z0 - padz + c;
    const bool in_z = z >= 0 && z < g.nz;
    s_pre[c] = (in_z && PRE) ? pre_scale(pre[z], pre[g.nz + z]) : (T)1;
  }
  // this thread's staged elements e = t + i*kFThreads: their offset within
  // an input plane (-1 for zero padding) and their staged column
  int goff[NL];
#pragma unroll
  for (int i = 0; i < NL; ++i) {
    const int e = t + i * kFThreads;
    const int r = e / C, c = e - r * C;
    const int z = z0 - padz + c;
    const bool v = e < R * C && z >= 0 && z < g.nz;
    goff[i] = v ? (int)(wrapi(y0 - pady + r, g.ny) * g.nz + z) : -1;
  }
  const int64_t plane_elems = g.ny * (int64_t)g.nz;
  // staged column of this thread's first element; element i sits at column
  // (c_base + i * kFThreads) mod C
  const int c_base = t % C;
  // Staging of the next plane: float32 in float32 arithmetic copies it
  // straight into shared memory with cp.async (no registers held across the
  // plane's filters); a conversion to float64 goes through registers.
  constexpr bool kAsync = std::is_same<T, A>::value && sizeof(T) == 4;
  T ld[NL];
  // input plane pointer, advanced one plane per iteration with the wrap in x
  int64_t xi = wrapi(xin0, g.nx);
  auto issue_loads = [&](A* dst) {
    const T* base = in + xi * plane_elems;
    if constexpr (kAsync) {
#pragma unroll
      for (int i = 0; i < NL; ++i) {
        const int e = t + i * kFThreads;
        if (e < R * C)
          cp_async4_zfill(dst + e, goff[i] >= 0 ? base + goff[i] : base, goff[i] >= 0 ? 4 : 0);
      }
      cp_async_commit();
    } else {
#pragma unroll
      for (int i = 0; i < NL; ++i) ld[i] = goff[i] >= 0 ? base[goff[i]] : (T)0;
    }
    xi = xi + 1 == g.nx ? 0 : xi + 1;
  };
  auto commit_loads = [&](A* dst) {
    if constexpr (kAsync) cp_async_wait<0>();
#pragma unroll
    for (int i = 0; i < NL; ++i) {
      const int e = t + i * kFThreads;
      if (e < R * C) {
        int c = c_base + (i * kFThreads) % C;  // compile-time offset
        c = c >= C ? c - C : c;
        if constexpr (kAsync) {
          // (the z pass applies the scaling as it reads the slab)
        } else {
          T v = ld[i];
          if (PRE) v = mul_rn(v, s_pre[c]);
          dst[e] = (A)v;
        }
      }
    }
  };
  // output points of this thread: rows 2*yp, 2*yp+1 at column zq; their
  // offsets within an output plane and whether they lie inside the array
  const int zq = t % kFZ, yp = t / kFZ;
  const int64_t oy0 = y0 + 2 * yp;
  const bool okz = z0 + zq < g.nz;
  const bool ok0 = okz && oy0 < g.ny, ok1 = okz && oy0 + 1 < g.ny;
  const int64_t o0 = oy0 * g.nz + z0 + zq, o1 = o0 + g.nz;
  const bool iny0 = oy0 >= epi.wy0 && oy0 < epi.wy1;
  const bool iny1 = oy0 + 1 >= epi.wy0 && oy0 + 1 < epi.wy1;
  A acc[K][2];
#pragma unroll
  for (int sl = 0; sl < K; ++sl) acc[sl][0] = acc[sl][1] = (A)0;
  double s_f = 0.0, s_clip = 0.0;
  __syncthreads();
  issue_loads(s_in0);
  commit_loads(s_in0);
  __syncthreads();
  if (count > 1) issue_loads(s_in0 + R * C);
  const bool flux_epi = epi.mode == STEAM_EPI_FLUX;
  const int count_i = (int)count;
  int rph = 0;  // ring phase: k mod K
  for (int k = 0; k < count_i; ++k) {
    // One barrier per plane.  Before it: the z pass of plane k (reads slab
    // k, writes s_u[k & 1]) and the arrival of slab k + 1.  After it: the
    // loads of slab k + 2 into slab k's buffer (every z read of it is done),
    // the y pass of plane k (reads s_u[k & 1], which is next written by the z
    // pass of plane k + 2, after the next barrier) and the ring step.
    A* s_in = s_in0 + (k & 1) * R * C;
    A* s_u = s_u0 + (k & 1) * kFMaxZ * R * kFZ;
    // the output plane this iteration completes (when j >= 0)
    const int j = k - (K - 1);
    const int64_t x = xb + j;
    T* outp = out + (j >= 0 ? x : 0) * plane_elems;
    // the flux under it, loaded now so that the load overlaps the filters
    T fprev0 = (T)0, fprev1 = (T)0;
    if (flux_epi && j >= 0) {
      if (ok0) fprev0 = outp[o0];
      if (ok1) fprev1 = outp[o1];
    }
    // ---- z filters, 4 outputs per task: u_c[r][z4 .. z4+3]
    for (int task = t; task < S::ZT; task += kFThreads) {
      const int r = task / (kFZ / 4), z4 = (task % (kFZ / 4)) * 4;
      const A* b = s_in + r * C + z4;  // 16-byte aligned: C and z4 are multiples of 4
      A win[K + 3];
#pragma unroll
      for (int i = 0; i < K + 3; i += 4) {
        const V4<A> q = ld4(b + i);
        win[i] = q.v[0];
        win[i + 1] = q.v[1];
        win[i + 2] = q.v[2];
        win[i + 3] = q.v[3];
        if constexpr (kAsync && PRE) {
          // the slab holds the raw input: scale by the factors of columns
          // z4 + i .. z4 + i + 3, the same multiply the staging would do
          const V4<T> f = ld4(s_pre + z4 + i);
          win[i] = mul_rn(win[i], f.v[0]);
          win[i + 1] = mul_rn(win[i + 1], f.v[1]);
          win[i + 2] = mul_rn(win[i + 2], f.v[2]);
          win[i + 3] = mul_rn(win[i + 3], f.v[3]);
        }
      }
      A a0[4] = {0, 0, 0, 0}, a1[4] = {0, 0, 0, 0};
      if constexpr (SYM) {
        // even filters: out = t[c] w[m] + sum_d t[c+d] (w[m+d] + w[m-d]), with
        // the pair sums shared by both z filters
        constexpr int c = (K - 1) / 2;
#pragma unroll
        for (int o = 0; o < 4; ++o) {
          const int m = o + c;
          a0[o] = tp.z[0][c] * win[m];
          a1[o] = tp.z[1][c] * win[m];
#pragma unroll
          for (int d = 1; d <= c; ++d) {
            const A ps = win[m + d] + win[m - d];
            a0[o] += tp.z[0][c + d] * ps;
            a1[o] += tp.z[1][c + d] * ps;
          }
        }
      } else {
#pragma unroll
        for (int l = 0; l < K; ++l) {
          const A t0 = tp.z[0][l], t1 = tp.z[1][l];
#pragma unroll
          for (int o = 0; o < 4; ++o) {
            // out[z] uses staged column z + K - 1 - l
            a0[o] += t0 * win[o + K - 1 - l];
            a1[o] += t1 * win[o + K - 1 - l];
          }
        }
      }
      st4(s_u + r * kFZ + z4, V4<A>{{a0[0], a0[1], a0[2], a0[3]}});
      st4(s_u + R * kFZ + r * kFZ + z4, V4<A>{{a1[0], a1[1], a1[2], a1[3]}});
    }
    if (k + 1 < count_i) commit_loads(s_in0 + ((k + 1) & 1) * R * C);
    __syncthreads();
    if (k + 2 < count_i) issue_loads(s_in);
    // ---- y filters for rows 2yp, 2yp+1 at column zq, then the mixing
    A w0[2] = {0, 0}, w1[2] = {0, 0};
#pragma unroll
    for (int c = 0; c < kFMaxZ; ++c) {
      A col[K + 1];
      const A* src = s_u + c * R * kFZ + (2 * yp) * kFZ + zq;
#pragma unroll
      for (int i = 0; i < K + 1; ++i) col[i] = src[i * kFZ];
      constexpr int cc = (K - 1) / 2;
      A ps0[cc + 1], ps1[cc + 1];  // pair sums about rows 2yp and 2yp + 1
      if constexpr (SYM) {
        ps0[0] = col[cc];
        ps1[0] = col[cc + 1];
#pragma unroll
        for (int d = 1; d <= cc; ++d) {
          ps0[d] = col[cc + d] + col[cc - d];
          ps1[d] = col[cc + 1 + d] + col[cc + 1 - d];
        }
      }
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        if (P3 && c == 1 && b == 1) continue;  // the zero pair
        A v0 = 0, v1 = 0;
        if constexpr (SYM) {
#pragma unroll
          for (int d = 0; d <= cc; ++d) {
            v0 += tp.y[b][cc + d] * ps0[d];
            v1 += tp.y[b][cc + d] * ps1[d];
          }
        } else {
#pragma unroll
          for (int jj = 0; jj < K; ++jj) {
            const A tj = tp.y[b][jj];
            v0 += tj * col[K - 1 - jj];
            v1 += tj * col[K - jj];
          }
        }
        const A m0 = tp.mix[0 * kFMaxPairs + c * 2 + b];
        const A m1 = tp.mix[1 * kFMaxPairs + c * 2 + b];
        w0[0] += m0 * v0;
        w0[1] += m0 * v1;
        w1[0] += m1 * v0;
        w1[1] += m1 * v1;
      }
    }
    // ---- fold into the ring: plane k feeds output j + i in slot (k + i + 1)
    //      mod K; output j is then complete and leaves the ring
    const bool in_wx = x >= epi.wx0 && x < epi.wx1;
    // the ring step for phase rr (a compile-time constant, so every slot
    // index is static); accumulated with two fused multiply-adds per slot
    auto ring_step = [&](auto rr_c) {
      constexpr int rr = decltype(rr_c)::value;
#pragma unroll
      for (int i = 0; i < K; ++i) {
        const int slot = (rr + i + 1) % K;
        const A c0 = tp.x[0][i], c1 = tp.x[1][i];
        acc[slot][0] = fma_a(c1, w1[0], fma_a(c0, w0[0], acc[slot][0]));
        acc[slot][1] = fma_a(c1, w1[1], fma_a(c0, w0[1], acc[slot][1]));
      }
      constexpr int es = (rr + 1) % K;
      if (j >= 0) {
        if (flux_epi) {
          T f0 = add_rn(fprev0, (T)acc[es][0]);
          T f1 = add_rn(fprev1, (T)acc[es][1]);
          if (ok0) {
            if (f0 < (T)0) {
              s_clip += 1.0;
              f0 = (T)0;
            }
            outp[o0] = f0;
            if (in_wx && iny0) s_f += (double)f0;
          }
          if (ok1) {
            if (f1 < (T)0) {
              s_clip += 1.0;
              f1 = (T)0;
            }
            outp[o1] = f1;
            if (in_wx && iny1) s_f += (double)f1;
          }
        } else {
          if (ok0) outp[o0] = (T)acc[es][0];
          if (ok1) outp[o1] = (T)acc[es][1];
        }
      }
      // a slot leaving the ring is cleared whether or not its output lies
      // in this chunk (planes before the chunk only feed the halo)
      acc[es][0] = (A)0;
      acc[es][1] = (A)0;
    };
#define STEAM_RING_CASE(n)                                  \
  case n:                                                   \
    if constexpr (n < K) ring_step(std::integral_constant<int, n>{}); \
    break;
    switch (rph) {
      STEAM_RING_CASE(0) STEAM_RING_CASE(1) STEAM_RING_CASE(2) STEAM_RING_CASE(3)
      STEAM_RING_CASE(4) STEAM_RING_CASE(5) STEAM_RING_CASE(6) STEAM_RING_CASE(7)
      STEAM_RING_CASE(8) STEAM_RING_CASE(9) STEAM_RING_CASE(10) STEAM_RING_CASE(11)
      STEAM_RING_CASE(12) STEAM_RING_CASE(13) STEAM_RING_CASE(14) STEAM_RING_CASE(15)
      STEAM_RING_CASE(16) STEAM_RING_CASE(17) STEAM_RING_CASE(18) STEAM_RING_CASE(19)
      STEAM_RING_CASE(20) STEAM_RING_CASE(21) STEAM_RING_CASE(22) STEAM_RING_CASE(23)
      STEAM_RING_CASE(24)
      default: break;
    }
#undef STEAM_RING_CASE
    rph = rph + 1 == K ? 0 : rph + 1;
  }
  if (epi.mode == STEAM_EPI_FLUX) {
    double t0 = block_sum(s_f, scratch);
    double t1 = block_sum(s_clip, scratch);
    if (threadIdx.x == 0) {
      partials[blockIdx.x] = t0;
      partials[gridDim.x + blockIdx.x] = t1;
    }
  }
}

template <typename T>
static bool fused_supported(const SepParams<T>& p) {
  const bool cube = p.kx == p.ky && p.ky == p.kz && (p.kx == 13 || p.kx == 25);
  if (!cube || p.nzf > kFMaxZ || p.nyf > 2 || p.nxf > kFMaxX || p.npairs > kFMaxPairs)
    return false;
  for (int q = 0; q < p.npairs; ++q)
    if (p.pair_z[q] >= 2 || p.pair_y[q] >= 2) return false;
  return true;
}

static size_t fused_smem(int k, size_t elem) {
  const int R = kFY + k - 1, C = kFZ + k - 1;
  return elem * ((size_t)2 * R * C + (size_t)2 * kFMaxZ * R * kFZ);
}

// x planes per CTA of the fused kernel, per field shape: set by the host's
// autotuner (steam_conv_set_xchunk), kFChunk otherwise.  The smallest
// allowed chunk bounds the workspace query.
constexpr int kFChunkMin = 16;
static std::mutex g_chunk_mu;
static std::map<std::tuple<int64_t, int64_t, int64_t>, int> g_chunk;

static int fused_chunk(int64_t nx, int64_t ny, int64_t nz) {
  std::lock_guard<std::mutex> lock(g_chunk_mu);
  auto it = g_chunk.find(std::make_tuple(nx, ny, nz));
  return it == g_chunk.end() ? kFChunk : it->second;
}

// the autotuner's chunk for the shape, 0 when it has set none
int chunk_override(int64_t nx, int64_t ny, int64_t nz) {
  std::lock_guard<std::mutex> lock(g_chunk_mu);
  auto it = g_chunk.find(std::make_tuple(nx, ny, nz));
  return it == g_chunk.end() ? 0 : it->second;
}

// float32 flux convolutions with float64 accumulation (the scalar fused
// kernel) instead of the packed float32 kernel: steam_conv_set_flux_wide
static std::atomic<int> g_flux_wide{0};

static int64_t fused_grid(int64_t nx, int64_t ny, int64_t nz, int chunk) {
  const int64_t nzt = (nz + kFZ - 1) / kFZ, nyt = (ny + kFY - 1) / kFY;
  const int64_t nxc = (nx + chunk - 1) / chunk;
  return nzt * nyt * nxc;
}

static int64_t fused_grid(int64_t nx, int64_t ny, int64_t nz) {
  return fused_grid(nx, ny, nz, fused_chunk(nx, ny, nz));
}

template <typename T>
static int fill_params(const steam_sepconv_t* s, const double* zt,
                       const double* yt, const double* xt, SepParams<T>& p) {
  STEAM_REQUIRE(s->kz >= 1 && s->ky >= 1 && s->kx >= 1,
                "steam_conv_separable: filter lengths must be >= 1");
  STEAM_REQUIRE(s->n_z >= 1 && s->n_z <= kMaxZ, "steam_conv_separable: n_z out of range");
  STEAM_REQUIRE(s->n_y >= 1, "steam_conv_separable: n_y must be >= 1");
  STEAM_REQUIRE(s->n_x >= 1 && s->n_x <= kMaxX, "steam_conv_separable: n_x out of range");
  STEAM_REQUIRE(s->n_pairs >= 1 && s->n_pairs <= kMaxPairs,
                "steam_conv_separable: n_pairs out of range");
  STEAM_REQUIRE(s->kz <= 256, "steam_conv_separable: kz above 256");
  const int total = s->n_z * s->kz + s->n_y * s->ky + s->n_x * s->kx;
  STEAM_REQUIRE(total <= kMaxTaps, "steam_conv_separable: too many taps");
  p.kz = s->kz;
  p.ky = s->ky;
  p.kx = s->kx;
  p.cz = s->cz;
  p.cy = s->cy;
  p.cx = s->cx;
  STEAM_REQUIRE(p.cz >= 0 && p.cz < p.kz && p.cy >= 0 && p.cy < p.ky &&
                    p.cx >= 0 && p.cx < p.kx,
                "steam_conv_separable: centre outside the filter");
  p.nzf = s->n_z;
  p.nyf = s->n_y;
  p.nxf = s->n_x;
  p.npairs = s->n_pairs;
  for (int q = 0; q < kMaxPairs; ++q) {
    p.pair_z[q] = q < s->n_pairs ? s->pair_z[q] : 0;
    p.pair_y[q] = q < s->n_pairs ? s->pair_y[q] : 0;
    if (q < s->n_pairs) {
      STEAM_REQUIRE(p.pair_z[q] >= 0 && p.pair_z[q] < s->n_z &&
                        p.pair_y[q] >= 0 && p.pair_y[q] < s->n_y,
                    "steam_conv_separable: pair index out of range");
    }
  }
  for (int i = 0; i < kMaxX * kMaxPairs; ++i)
    p.mix[i] = i < s->n_x * s->n_pairs ? s->mix[i] : 0.0;
  int o = 0;
  for (int i = 0; i < s->n_z * s->kz; ++i) p.taps[o++] = zt[i];
  for (int i = 0; i < s->n_y * s->ky; ++i) p.taps[o++] = yt[i];
  for (int i = 0; i < s->n_x * s->kx; ++i) p.taps[o++] = xt[i];
  for (; o < kMaxTaps; ++o) p.taps[o] = 0.0;
  return STEAM_OK;
}

static int64_t epi_cells(const steam_window_t* w, int64_t nx, int64_t ny) {
  if (!w) return nx * ny;
  return (w->x1 - w->x0) * (w->y1 - w->y0);
}

// The variant for the taps' structure: even filters folded in pairs (SYM),
// the input scaling prologue (PRE), no pair of z filter 1 with y filter 1 (P3).
template <typename T, typename A, int K, bool SYM, bool PRE, bool P3>
static cudaError_t launch_fused_v(const FusedTaps<A, K>& tp, int64_t grid, size_t sm,
                                  const T* in, T* out, const T* pre, const FusedGeom<T>& g,
                                  const XEpi& epi, double* partials, cudaStream_t s) {
  auto kern = fused_conv_kernel<T, A, K, SYM, PRE, P3>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sm);
  if (e != cudaSuccess) return e;
  kern<<<(unsigned)grid, kFThreads, sm, s>>>(in, out, pre, tp, g, epi, partials);
  return cudaSuccess;
}

template <typename T, typename A, int K>
static cudaError_t launch_fused_k(const FusedTaps<A, K>& tp, int64_t grid, size_t sm,
                                  const T* in, T* out, const T* pre, const FusedGeom<T>& g,
                                  const XEpi& epi, double* partials, cudaStream_t s) {
  // float64 accumulation keeps the full pair set: skipping the zero pair
  // there moved the register allocation into spills (13.7 -> 18.2 ms)
  if constexpr (sizeof(A) == 4) {
    const int v = (tp.sym ? 4 : 0) | (g.use_pre ? 2 : 0) | (tp.skip11 ? 1 : 0);
    switch (v) {
      case 0: return launch_fused_v<T, A, K, false, false, false>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      case 1: return launch_fused_v<T, A, K, false, false, true>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      case 2: return launch_fused_v<T, A, K, false, true, false>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      case 3: return launch_fused_v<T, A, K, false, true, true>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      case 4: return launch_fused_v<T, A, K, true, false, false>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      case 5: return launch_fused_v<T, A, K, true, false, true>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      case 6: return launch_fused_v<T, A, K, true, true, false>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      default: return launch_fused_v<T, A, K, true, true, true>(tp, grid, sm, in, out, pre, g, epi, partials, s);
    }
  } else {
    const int v = (tp.sym ? 2 : 0) | (g.use_pre ? 1 : 0);
    switch (v) {
      case 0: return launch_fused_v<T, A, K, false, false, false>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      case 1: return launch_fused_v<T, A, K, false, true, false>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      case 2: return launch_fused_v<T, A, K, true, false, false>(tp, grid, sm, in, out, pre, g, epi, partials, s);
      default: return launch_fused_v<T, A, K, true, true, false>(tp, grid, sm, in, out, pre, g, epi, partials, s);
    }
  }
}

template <typename T, typename A>
static int launch_fused(const SepParams<T>& p, int64_t grid, const T* in, T* out, const T* pre,
                        const FusedGeom<T>& g, const XEpi& epi, double* partials,
                        cudaStream_t s) {
  const size_t sm = fused_smem(p.kx, sizeof(A));
  STEAM_REQUIRE(sm <= 200 * 1024, "steam_conv_separable: filters too long for the fused path");
  if (p.kx == 13) {
    const FusedTaps<A, 13> tp = fused_taps<T, A, 13>(p);
    const cudaError_t e = launch_fused_k<T, A, 13>(tp, grid, sm, in, out, pre, g, epi, partials, s);
    STEAM_CUDA(e);
  } else {
    const FusedTaps<A, 25> tp = fused_taps<T, A, 25>(p);
    const cudaError_t e = launch_fused_k<T, A, 25>(tp, grid, sm, in, out, pre, g, epi, partials, s);
    STEAM_CUDA(e);
  }
  STEAM_LAUNCH_CHECK("conv fused");
  return STEAM_OK;
}

template <typename T>
static int run_fused(int64_t nx, int64_t ny, int64_t nz, const SepParams<T>& p,
                     const void* in_v, const double* pre_div,
                     const double* pre_mul, const T* pre_dev, void* out_v, int epilogue,
                     const steam_window_t* win, double* sums_out, double* totals_dev,
                     void* ws, size_t ws_bytes, cudaStream_t s) {
  int64_t grid = fused_grid(nx, ny, nz, fused_chunk(nx, ny, nz));
  Carver c(ws, ws_bytes);
  const bool use_pre = pre_div != nullptr || pre_mul != nullptr || pre_dev != nullptr;
  T* pre = c.take<T>((size_t)2 * nz);
  // room for either kernel's partial sums (the packed grid is at most this)
  double* partials = c.take<double>((size_t)fused_grid(nx, ny, nz, kFChunkMin) * 2);
  double* totals = c.take<double>(2);
  if (!pre || !partials || !totals)
    return fail(STEAM_ERR_WORKSPACE, "steam_conv_separable: workspace too small");
  if (totals_dev) totals = totals_dev;
  if (pre_dev) {
    pre = const_cast<T*>(pre_dev);
  } else if (use_pre) {
    std::vector<T> h(2 * nz);
    for (int64_t z = 0; z < nz; ++z) {
      h[z] = pre_div ? (T)pre_div[z] : (T)1;
      h[nz + z] = pre_mul ? (T)pre_mul[z] : (T)1;
    }
    STEAM_CUDA(cudaMemcpyAsync(pre, h.data(), sizeof(T) * 2 * nz,
                               cudaMemcpyHostToDevice, s));
  }
  FusedGeom<T> g;
  g.nx = nx;
  g.ny = ny;
  g.nz = (int)nz;
  g.nzt = (int)((nz + kFZ - 1) / kFZ);
  g.nyt = (int)((ny + kFY - 1) / kFY);
  g.chunk = fused_chunk(nx, ny, nz);
  g.use_pre = use_pre ? 1 : 0;
  XEpi epi;
  epi.mode = epilogue;
  epi.wx0 = win ? win->x0 : 0;
  epi.wx1 = win ? win->x1 : nx;
  epi.wy0 = win ? win->y0 : 0;
  epi.wy1 = win ? win->y1 : ny;
  int rc;
  bool packed = false;
  if constexpr (sizeof(T) == 4) {
    packed = (epilogue == STEAM_EPI_STORE || (epilogue == STEAM_EPI_FLUX && !g_flux_wide.load())) &&
             packed_supported(p, nx, ny, nz, in_v, out_v, epilogue);
  }
  if (packed) {
    grid = packed_grid(nx, ny, nz);
    rc = packed_launch(reinterpret_cast<const SepParams<float>&>(p), nx, ny, nz,
                       (const float*)in_v, (float*)out_v, use_pre ? (const float*)pre : nullptr,
                       epilogue, epi, partials, s);
  } else {
    rc = epilogue != STEAM_EPI_STORE
             ? launch_fused<T, double>(p, grid, (const T*)in_v, (T*)out_v, pre, g, epi,
                                       partials, s)
             : launch_fused<T, T>(p, grid, (const T*)in_v, (T*)out_v, pre, g, epi, partials, s);
  }
  if (rc) return rc;
  if (epilogue == STEAM_EPI_FLUX) {
    int rc = reduce_partials(partials, (int)grid, 2, totals, s);
    if (rc) return rc;
    if (totals_dev) return STEAM_OK;
    double h[2];
    STEAM_CUDA(cudaMemcpyAsync(h, totals, sizeof(h), cudaMemcpyDeviceToHost, s));
    STEAM_CUDA(cudaStreamSynchronize(s));
    sums_out[0] = h[0];
    sums_out[1] = (double)(epi_cells(win, nx, ny) * nz);
    sums_out[2] = h[1];
  }
  return STEAM_OK;
}

// Blocks of `kern` resident per SM with `sm` bytes of dynamic shared memory
// (at least 1, at most `cap`).
template <typename K>
static int pass_occupancy(K kern, size_t sm, int cap) {
  int occ = 0;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) !=
          cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kPassThreads, sm) !=
          cudaSuccess)
    occ = 1;
  return occ < 1 ? 1 : (occ > cap ? cap : occ);
}

// An upper bound of the x-pass grid (at most 8 blocks of 256 threads per SM):
// the flux partial pairs it can write.
static int xpass_grid_max(int64_t nx, int64_t ny, int64_t nz) {
  return stride_grid(xpass_tiles(nx, ny, nz), 1, 8);
}

// The z, y and x passes in arithmetic type A: u = z filters of the input
// (scaled by pre when given), w = the x filters' mixes of the y-filtered
// pairs of u, out = the x filters of w with the epilogue.
template <typename T, typename A>
static int launch_passes(const SepParams<T>& p, int64_t nx, int64_t ny, int64_t nz,
                         const T* in, const T* pre, T* u, T* w, T* out, const XEpi& epi,
                         double* partials, int* xgrid_out, cudaStream_t s) {
  const int64_t plane = nx * ny * nz;
  const int kpz = sep_padded(p.kz), kpy = sep_padded(p.ky), kpx = sep_padded(p.kx);
  const size_t smz = zpass_smem<A>(p.nzf, kpz), smy = ypass_smem<A>(p.nyf, kpy),
               smx = xpass_smem<A>(p.nxf, kpx);
  STEAM_REQUIRE(smz <= 200 * 1024, "steam_conv_separable: z filter too long");
  STEAM_REQUIRE(smy <= 200 * 1024, "steam_conv_separable: y filter too long");
  STEAM_REQUIRE(smx <= 200 * 1024, "steam_conv_separable: x filter too long");
  // the y and x passes index tiles, rows and plane elements in 32 bits
  const int64_t lim = (int64_t)1 << 31;
  STEAM_REQUIRE(nx < lim && ny * nz < lim && nx * ((ny + kYT - 1) / kYT) * ((nz + 31) / 32) < lim &&
                    xpass_tiles(nx, ny, nz) < lim,
                "steam_conv_separable: field too large for the three-pass form");
  if constexpr (std::is_same<T, float>::value && std::is_same<A, float>::value) {
    const int64_t ncol = nx * ny;
    const size_t smz2 = zpass2_smem(p.nzf, kpz);
    const int64_t tiles = ((ncol + kPairW - 1) / kPairW) * ((nz + kZ2 - 1) / kZ2);
    STEAM_REQUIRE(smz2 <= 200 * 1024, "steam_conv_separable: z filter too long");
    STEAM_REQUIRE(tiles < lim, "steam_conv_separable: field too large for the three-pass form");
    if (pre) {
      auto k = zpass2_kernel<true>;
      k<<<stride_grid(tiles, 1, pass_occupancy(k, smz2, 8)), kPassThreads, smz2, s>>>(
          in, ncol, (int)nz, kpz, pre, pre + nz, p, u, plane);
    } else {
      auto k = zpass2_kernel<false>;
      k<<<stride_grid(tiles, 1, pass_occupancy(k, smz2, 8)), kPassThreads, smz2, s>>>(
          in, ncol, (int)nz, kpz, nullptr, nullptr, p, u, plane);
    }
    STEAM_LAUNCH_CHECK("conv z-pass");
  } else {
    const int64_t ncol = nx * ny;
    const int64_t tiles = ((ncol + kZCols - 1) / kZCols) *
                          ((nz + zpass_chunk<A>() - 1) / zpass_chunk<A>());
    if (pre) {
      auto k = zpass_kernel<T, A, true>;
      k<<<stride_grid(tiles, 1, pass_occupancy(k, smz, 8)), kPassThreads, smz, s>>>(
          in, ncol, (int)nz, kpz, pre, pre + nz, p, u, plane);
    } else {
      auto k = zpass_kernel<T, A, false>;
      k<<<stride_grid(tiles, 1, pass_occupancy(k, smz, 8)), kPassThreads, smz, s>>>(
          in, ncol, (int)nz, kpz, nullptr, nullptr, p, u, plane);
    }
    STEAM_LAUNCH_CHECK("conv z-pass");
  }
  if constexpr (std::is_same<T, float>::value && std::is_same<A, float>::value) {
    // plain float32 convolution: the paired y and x passes
    const size_t smy2 = ypass2_smem(p.nyf, kpy), smx2 = xpass2_smem(p.nxf, kpx);
    STEAM_REQUIRE(smy2 <= 200 * 1024, "steam_conv_separable: y filter too long");
    STEAM_REQUIRE(smx2 <= 200 * 1024, "steam_conv_separable: x filter too long");
    const int64_t ytiles = nx * ((ny + kYT - 1) / kYT) * ((nz + kPairW - 1) / kPairW);
    if (p.nxf <= 2) {
      auto k = ypass2_kernel<2>;
      k<<<stride_grid(ytiles, 1, pass_occupancy(k, smy2, 8)), kPassThreads, smy2, s>>>(
          u, nx, ny, (int)nz, kpy, p, w, plane);
    } else {
      auto k = ypass2_kernel<kMaxX>;
      k<<<stride_grid(ytiles, 1, pass_occupancy(k, smy2, 8)), kPassThreads, smy2, s>>>(
          u, nx, ny, (int)nz, kpy, p, w, plane);
    }
    STEAM_LAUNCH_CHECK("conv y-pass");
    auto kx = xpass2_kernel;
    const int grid = stride_grid(xpass2_tiles(nx, ny, nz), 1, pass_occupancy(kx, smx2, 8));
    const int aligned_out = ((uintptr_t)out % 8 == 0 && (ny * nz) % 2 == 0) ? 1 : 0;
    kx<<<grid, kPassThreads, smx2, s>>>(w, nx, ny, (int)nz, kpx, p, out, plane, aligned_out);
    STEAM_LAUNCH_CHECK("conv x-pass");
    *xgrid_out = grid;
  } else {
    const int64_t tiles = nx * ((ny + kYT - 1) / kYT) * ((nz + 31) / 32);
    if (p.nxf <= 2) {
      auto k = ypass_kernel<T, A, 2>;
      k<<<stride_grid(tiles, 1, pass_occupancy(k, smy, 8)), kPassThreads, smy, s>>>(
          u, nx, ny, (int)nz, kpy, p, w, plane);
    } else {
      auto k = ypass_kernel<T, A, kMaxX>;
      k<<<stride_grid(tiles, 1, pass_occupancy(k, smy, 8)), kPassThreads, smy, s>>>(
          u, nx, ny, (int)nz, kpy, p, w, plane);
    }
    STEAM_LAUNCH_CHECK("conv y-pass");
    auto kx = xpass_kernel<T, A>;
    const int grid = stride_grid(xpass_tiles(nx, ny, nz), 1, pass_occupancy(kx, smx, 8));
    kx<<<grid, kPassThreads, smx, s>>>(w, nx, ny, (int)nz, kpx, p, out, plane, epi, partials);
    STEAM_LAUNCH_CHECK("conv x-pass");
    *xgrid_out = grid;
  }
  return STEAM_OK;
}

template <typename T>
static int run_separable(int64_t nx, int64_t ny, int64_t nz,
                         const steam_sepconv_t* spec, const double* zt,
                         const double* yt, const double* xt, const void* in_v,
                         const double* pre_div, const double* pre_mul, const T* pre_dev,
                         void* out_v, int epilogue, const steam_window_t* win,
                         double* sums_out, double* totals_dev, void* ws, size_t ws_bytes,
                         cudaStream_t s) {
  SepParams<T>* pp = new SepParams<T>();
  std::unique_ptr<SepParams<T>> guard(pp);
  int rc = fill_params<T>(spec, zt, yt, xt, *pp);
  if (rc) return rc;
  SepParams<T>& p = *pp;
  const int64_t plane = nx * ny * nz;
  if (fused_supported(p) && fused_grid(nx, ny, nz, kFChunkMin) < ((int64_t)1 << 31) &&
      ny * nz < ((int64_t)1 << 31))
    return run_fused<T>(nx, ny, nz, p, in_v, pre_div, pre_mul, pre_dev, out_v, epilogue,
                        win, sums_out, totals_dev, ws, ws_bytes, s);
  Carver c(ws, ws_bytes);
  T* u = c.take<T>((size_t)p.nzf * plane);
  T* w = c.take<T>((size_t)p.nxf * plane);
  T* pre = nullptr;
  const bool use_pre = pre_div != nullptr || pre_mul != nullptr || pre_dev != nullptr;
  if (use_pre) pre = c.take<T>((size_t)2 * nz);
  double* partials = c.take<double>((size_t)xpass_grid_max(nx, ny, nz) * 2);
  double* totals = c.take<double>(2);
  if (!u || !w || (use_pre && !pre) || !partials || !totals)
    return fail(STEAM_ERR_WORKSPACE,
                "steam_conv_separable: workspace too small");
  const T* in = (const T*)in_v;
  T* out = (T*)out_v;
  if (totals_dev) totals = totals_dev;
  if (pre_dev) {
    pre = const_cast<T*>(pre_dev);
  } else if (use_pre) {
    std::vector<T> h(2 * nz);
    for (int64_t z = 0; z < nz; ++z) {
      h[z] = pre_div ? (T)pre_div[z] : (T)1;
      h[nz + z] = pre_mul ? (T)pre_mul[z] : (T)1;
    }
    STEAM_CUDA(cudaMemcpyAsync(pre, h.data(), sizeof(T) * 2 * nz,
                               cudaMemcpyHostToDevice, s));
    STEAM_CUDA(cudaStreamSynchronize(s));
  }
  XEpi epi;
  epi.mode = epilogue;
  epi.wx0 = win ? win->x0 : 0;
  epi.wx1 = win ? win->x1 : nx;
  epi.wy0 = win ? win->y0 : 0;
  epi.wy1 = win ? win->y1 : ny;
  int xgrid = 0;
  // float64 arithmetic for float64 fields, the flux epilogue and the wide store
  rc = (sizeof(T) == 8 || epilogue != STEAM_EPI_STORE)
           ? launch_passes<T, double>(p, nx, ny, nz, in, use_pre ? pre : nullptr, u, w, out,
                                      epi, partials, &xgrid, s)
           : launch_passes<T, T>(p, nx, ny, nz, in, use_pre ? pre : nullptr, u, w, out, epi,
                                 partials, &xgrid, s);
  if (rc) return rc;
  if (epilogue == STEAM_EPI_FLUX) {
    rc = reduce_partials(partials, xgrid, 2, totals, s);
    if (rc) return rc;
    if (totals_dev) return STEAM_OK;
    double h[2];
    STEAM_CUDA(cudaMemcpyAsync(h, totals, sizeof(h), cudaMemcpyDeviceToHost, s));
    STEAM_CUDA(cudaStreamSynchronize(s));
    sums_out[0] = h[0];
    sums_out[1] = (double)((epi_cells(win, nx, ny)) * nz);
    sums_out[2] = h[1];
  }
  return STEAM_OK;
}

}  // namespace steam

using namespace steam;

extern "C" size_t steam_conv_workspace_bytes(int dtype, int64_t nx, int64_t ny,
                                             int64_t nz,
                                             const steam_sepconv_t* spec) {
  if (!spec) return 0;
  size_t elem = dtype == STEAM_F64 ? 8 : 4;
  size_t plane = (size_t)(nx * ny * nz);
  const int xgrid = xpass_grid_max(nx, ny, nz);
  const size_t multi = carve_bytes((size_t)spec->n_z * plane, elem) +
                      carve_bytes((size_t)spec->n_x * plane, elem) +
                      carve_bytes((size_t)2 * nz, elem) +
                      carve_bytes((size_t)xgrid * 2, sizeof(double)) +
                      carve_bytes(2, sizeof(double));
  bool fused = spec->kx == spec->ky && spec->ky == spec->kz &&
               (spec->kx == 13 || spec->kx == 25) && spec->n_z <= kFMaxZ &&
               spec->n_y <= 2 && spec->n_x <= kFMaxX && spec->n_pairs <= kFMaxPairs &&
               fused_grid(nx, ny, nz, kFChunkMin) < ((int64_t)1 << 31) &&
               ny * nz < ((int64_t)1 << 31);
  for (int q = 0; fused && q < spec->n_pairs; ++q)
    if (spec->pair_z[q] >= 2 || spec->pair_y[q] >= 2) fused = false;
  if (fused)
    return carve_bytes((size_t)2 * nz, elem) +
           carve_bytes((size_t)fused_grid(nx, ny, nz, kFChunkMin) * 2, sizeof(double)) +
           carve_bytes(2, sizeof(double));
  return multi;
}

extern "C" int steam_conv_separable(
    int dtype, int64_t nx, int64_t ny, int64_t nz, const steam_sepconv_t* spec,
    const double* z_taps, const double* y_taps, const double* x_taps,
    const void* in, const double* pre_div, const double* pre_mul, void* out,
    int32_t epilogue, const steam_window_t* window, double* sums_out,
    void* workspace, size_t workspace_bytes, steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0,
                "steam_conv_separable: negative extent");
  STEAM_REQUIRE(spec && z_taps && y_taps && x_taps,
                "steam_conv_separable: null spec or taps");
  STEAM_REQUIRE(epilogue == STEAM_EPI_STORE || epilogue == STEAM_EPI_FLUX ||
                    epilogue == STEAM_EPI_STORE_WIDE,
                "steam_conv_separable: unknown epilogue");
  STEAM_REQUIRE(epilogue != STEAM_EPI_FLUX || sums_out,
                "steam_conv_separable: flux epilogue needs sums_out");
  if (window) {
    STEAM_REQUIRE(window->x0 >= 0 && window->x1 <= nx &&
                      window->x0 <= window->x1 && window->y0 >= 0 &&
                      window->y1 <= ny && window->y0 <= window->y1,
                  "steam_conv_separable: window outside the array");
  }
  if (nx * ny * nz == 0) {
    if (epilogue == STEAM_EPI_FLUX) {
      sums_out[0] = 0.0;
      sums_out[1] = 0.0;
      sums_out[2] = 0.0;
    }
    return STEAM_OK;
  }
  STEAM_REQUIRE(in && out, "steam_conv_separable: null field pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    return run_separable<float>(nx, ny, nz, spec, z_taps, y_taps, x_taps, in,
                                pre_div, pre_mul, nullptr, out, epilogue, window,
                                sums_out, nullptr, workspace, workspace_bytes, s);
  if (dtype == STEAM_F64)
    return run_separable<double>(nx, ny, nz, spec, z_taps, y_taps, x_taps, in,
                                 pre_div, pre_mul, nullptr, out, epilogue, window,
                                 sums_out, nullptr, workspace, workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_conv_separable: bad dtype");
}

extern "C" int steam_conv_separable_async(
    int dtype, int64_t nx, int64_t ny, int64_t nz, const steam_sepconv_t* spec,
    const double* z_taps, const double* y_taps, const double* x_taps,
    const void* in, const void* pre_dev, void* out, int32_t epilogue,
    const steam_window_t* window, double* sums_dev, void* workspace,
    size_t workspace_bytes, steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0,
                "steam_conv_separable_async: negative extent");
  STEAM_REQUIRE(spec && z_taps && y_taps && x_taps,
                "steam_conv_separable_async: null spec or taps");
  STEAM_REQUIRE(epilogue == STEAM_EPI_STORE || epilogue == STEAM_EPI_FLUX ||
                    epilogue == STEAM_EPI_STORE_WIDE,
                "steam_conv_separable_async: unknown epilogue");
  STEAM_REQUIRE(epilogue != STEAM_EPI_FLUX || sums_dev,
                "steam_conv_separable_async: flux epilogue needs sums_dev");
  if (window) {
    STEAM_REQUIRE(window->x0 >= 0 && window->x1 <= nx &&
                      window->x0 <= window->x1 && window->y0 >= 0 &&
                      window->y1 <= ny && window->y0 <= window->y1,
                  "steam_conv_separable_async: window outside the array");
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (nx * ny * nz == 0) {
    if (epilogue == STEAM_EPI_FLUX) STEAM_CUDA(cudaMemsetAsync(sums_dev, 0, 2 * sizeof(double), s));
    return STEAM_OK;
  }
  STEAM_REQUIRE(in && out, "steam_conv_separable_async: null field pointer");
  if (dtype == STEAM_F32)
    return run_separable<float>(nx, ny, nz, spec, z_taps, y_taps, x_taps, in, nullptr,
                                nullptr, (const float*)pre_dev, out, epilogue, window, nullptr,
                                sums_dev, workspace, workspace_bytes, s);
  if (dtype == STEAM_F64)
    return run_separable<double>(nx, ny, nz, spec, z_taps, y_taps, x_taps, in, nullptr,
                                 nullptr, (const double*)pre_dev, out, epilogue, window,
                                 nullptr, sums_dev, workspace, workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_conv_separable_async: bad dtype");
}

extern "C" size_t steam_conv_group_workspace_bytes(int32_t n,
                                                 const steam_conv_problem_t* problems) {
  if (n < 1 || !problems) return 0;
  return packed_group_bytes(n, problems);
}

extern "C" int steam_conv_group_prepare(const steam_sepconv_t* spec, const double* z_taps,
                                        const double* y_taps, const double* x_taps, int32_t n,
                                        const steam_conv_problem_t* problems, int32_t epilogue,
                                        void* workspace, size_t workspace_bytes) {
  STEAM_REQUIRE(spec && z_taps && y_taps && x_taps, "steam_conv_group_prepare: null filters");
  STEAM_REQUIRE(n >= 1 && problems, "steam_conv_group_prepare: no fields");
  STEAM_REQUIRE(workspace, "steam_conv_group_prepare: null workspace");
  std::unique_ptr<SepParams<float>> p(new SepParams<float>());
  int rc = fill_params<float>(spec, z_taps, y_taps, x_taps, *p);
  if (rc) return rc;
  return packed_group_prepare(*p, n, problems, epilogue, workspace, workspace_bytes);
}

extern "C" int steam_conv_group_async(void* workspace, steam_stream_t stream) {
  return packed_group_enqueue(workspace, (cudaStream_t)stream);
}

extern "C" int steam_conv_group_release(void* workspace) {
  return packed_group_release(workspace);
}

extern "C" int steam_conv_set_flux_wide(int32_t wide) {
  STEAM_REQUIRE(wide == 0 || wide == 1, "steam_conv_set_flux_wide: wide must be 0 or 1");
  g_flux_wide.store(wide);
  return STEAM_OK;
}

extern "C" int steam_conv_set_xchunk(int64_t nx, int64_t ny, int64_t nz, int32_t chunk) {
  STEAM_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1, "steam_conv_set_xchunk: empty shape");
  STEAM_REQUIRE(chunk == 0 || (chunk >= kFChunkMin && chunk <= 4096),
                "steam_conv_set_xchunk: chunk must be 0 (default) or in [16, 4096]");
  std::lock_guard<std::mutex> lock(g_chunk_mu);
  if (chunk == 0)
    g_chunk.erase(std::make_tuple(nx, ny, nz));
  else
    g_chunk[std::make_tuple(nx, ny, nz)] = chunk;
  return STEAM_OK;
}

extern "C" int steam_conv_get_xchunk(int64_t nx, int64_t ny, int64_t nz) {
  return fused_chunk(nx, ny, nz);
}
