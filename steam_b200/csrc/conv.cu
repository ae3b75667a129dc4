// Circular-x/y, linear-z convolution on a separable network of 1D filters
// (the turbulon kernels are sums of a few separable terms), plus a dense
// direct-summation form for arbitrary kernels.
//
// Three passes, each a coalesced stencil over the z-fastest layout:
//   z-pass: u_c = f (*)_z Z_c       (columns staged in shared memory)
//   y-pass: v_p = u_c (*)_y Y_b     (TY x TZ tiles of one x-plane)
//   x-pass: out = sum_a (sum_p mix_ap v_p) (*)_x X_a, with the epilogue.
#include "common.cuh"

#include <memory>
#include <vector>

namespace steam {

constexpr int kMaxTaps = 1536;
constexpr int kMaxZ = 8;
constexpr int kMaxPairs = 16;
constexpr int kMaxX = 4;

// Taps, mixing weights and every accumulator are float64 for both storage
// dtypes: the turbulon kernel's terms cancel (it has zero sum), and float32
// taps with float32 sums put ~1e-5 relative error into the log of a flux
// advanced next to its clip.  Fields and intermediates stay in the storage
// dtype.
template <typename T>
struct SepParams {
  int kz, ky, kx, cz, cy, cx;
  int nzf, nyf, nxf, npairs;
  int pair_z[kMaxPairs];
  int pair_y[kMaxPairs];
  double mix[kMaxX * kMaxPairs];
  double taps[kMaxTaps];  // z taps, then y taps, then x taps
  __host__ __device__ const double* ztap(int f) const { return taps + f * kz; }
  __host__ __device__ const double* ytap(int f) const {
    return taps + nzf * kz + f * ky;
  }
  __host__ __device__ const double* xtap(int f) const {
    return taps + nzf * kz + nyf * ky + f * kx;
  }
};

__device__ __forceinline__ int64_t wrapi(int64_t v, int64_t n) {
  int64_t r = v % n;
  return r < 0 ? r + n : r;
}

// ---- z-pass -------------------------------------------------------------
// Block = CB consecutive columns (contiguous in memory), staged with zero
// padding: buf[j] = in[j - (kz-1-cz)].
template <typename T, bool PRE>
__global__ void __launch_bounds__(256) zpass_kernel(
    const T* __restrict__ in, int64_t ncol, int nz, int cb,
    const T* __restrict__ pre_div, const T* __restrict__ pre_mul,
    SepParams<T> p, T* __restrict__ out, int64_t plane) {
  extern __shared__ unsigned char smem_raw[];
  T* buf = reinterpret_cast<T*>(smem_raw);
  __shared__ double taps_s[kMaxZ * 256];
  const int kz = p.kz;
  const int len = nz + kz - 1;
  const int padlo = kz - 1 - p.cz;
  for (int i = threadIdx.x; i < p.nzf * kz; i += blockDim.x)
    taps_s[i] = p.taps[i];
  for (int64_t col0 = (int64_t)blockIdx.x * cb; col0 < ncol;
       col0 += (int64_t)gridDim.x * cb) {
    const int ncb = (int)((ncol - col0) < cb ? (ncol - col0) : cb);
    __syncthreads();
    for (int i = threadIdx.x; i < ncb * len; i += blockDim.x) {
      int c = i / len, j = i - c * len;
      int s = j - padlo;
      T v = (T)0;
      if (s >= 0 && s < nz) {
        v = in[(col0 + c) * nz + s];
        if (PRE) v = mul_rn(v / pre_div[s], pre_mul[s]);
      }
      buf[c * len + j] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ncb * nz; i += blockDim.x) {
      int c = i / nz, z = i - c * nz;
      const T* b = buf + c * len + z + kz - 1;
      double acc[kMaxZ];
#pragma unroll
      for (int f = 0; f < kMaxZ; ++f) acc[f] = 0.0;
      for (int l = 0; l < kz; ++l) {
        const double x = (double)b[-l];
#pragma unroll
        for (int f = 0; f < kMaxZ; ++f)
          if (f < p.nzf) acc[f] += taps_s[f * kz + l] * x;
      }
      const int64_t o = (col0 + c) * nz + z;
#pragma unroll
      for (int f = 0; f < kMaxZ; ++f)
        if (f < p.nzf) out[f * plane + o] = (T)acc[f];
    }
  }
}

// ---- y-pass -------------------------------------------------------------
constexpr int kTY = 16;
constexpr int kTZ = 64;

template <typename T>
__global__ void __launch_bounds__(256) ypass_kernel(
    const T* __restrict__ u, int64_t nx, int64_t ny, int nz, SepParams<T> p,
    T* __restrict__ v, int64_t plane) {
  extern __shared__ unsigned char smem_raw[];
  T* buf = reinterpret_cast<T*>(smem_raw);  // [nzf][TY+ky-1][TZ]
  const int ky = p.ky;
  const int rows = kTY + ky - 1;
  const int padlo = ky - 1 - p.cy;
  const int64_t ytiles = (ny + kTY - 1) / kTY;
  const int64_t ztiles = (nz + kTZ - 1) / kTZ;
  const int64_t ntiles = nx * ytiles * ztiles;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t zt = t % ztiles;
    const int64_t yt = (t / ztiles) % ytiles;
    const int64_t x = t / (ztiles * ytiles);
    const int64_t y0 = yt * kTY;
    const int z0 = (int)(zt * kTZ);
    const int tz = (nz - z0) < kTZ ? (nz - z0) : kTZ;
    __syncthreads();
    for (int i = threadIdx.x; i < p.nzf * rows * kTZ; i += blockDim.x) {
      int f = i / (rows * kTZ);
      int rem = i - f * rows * kTZ;
      int r = rem / kTZ, zz = rem - r * kTZ;
      T val = (T)0;
      if (zz < tz) {
        int64_t ys = wrapi(y0 - padlo + r, ny);
        val = u[(int64_t)f * plane + (x * ny + ys) * nz + z0 + zz];
      }
      buf[i] = val;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTY * kTZ; i += blockDim.x) {
      int r = i / kTZ, zz = i - r * kTZ;
      int64_t y = y0 + r;
      if (y >= ny || zz >= tz) continue;
      for (int q = 0; q < p.npairs; ++q) {
        const T* col = buf + (p.pair_z[q] * rows + r + ky - 1) * kTZ + zz;
        const double* tp = p.ytap(p.pair_y[q]);
        double acc = 0.0;
        for (int j = 0; j < ky; ++j) acc += tp[j] * (double)col[-j * kTZ];
        v[(int64_t)q * plane + (x * ny + y) * nz + z0 + zz] = (T)acc;
      }
    }
  }
}

// ---- x-pass -------------------------------------------------------------
constexpr int kTX = 16;
constexpr int kTE = 128;

struct XEpi {
  int mode;
  int64_t wx0, wx1, wy0, wy1;
};

template <typename T>
__global__ void __launch_bounds__(256) xpass_kernel(
    const T* __restrict__ v, int64_t nx, int64_t ny, int nz, SepParams<T> p,
    T* __restrict__ out, int64_t plane, XEpi epi,
    double* __restrict__ partials) {
  extern __shared__ unsigned char smem_raw[];
  double* buf = reinterpret_cast<double*>(smem_raw);  // [nxf][TX+kx-1][TE]
  __shared__ double scratch[32];
  const int kx = p.kx;
  const int rows = kTX + kx - 1;
  const int padlo = kx - 1 - p.cx;
  const int64_t pe = ny * nz;  // elements of one x-plane
  const int64_t etiles = (pe + kTE - 1) / kTE;
  const int64_t xtiles = (nx + kTX - 1) / kTX;
  const int64_t ntiles = xtiles * etiles;
  double s_f = 0.0, s_clip = 0.0;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t et = t % etiles;
    const int64_t xt = t / etiles;
    const int64_t x0 = xt * kTX;
    const int64_t e0 = et * kTE;
    const int te = (pe - e0) < kTE ? (int)(pe - e0) : kTE;
    __syncthreads();
    for (int i = threadIdx.x; i < rows * kTE; i += blockDim.x) {
      int r = i / kTE, ee = i - r * kTE;
      double w[kMaxX];
#pragma unroll
      for (int a = 0; a < kMaxX; ++a) w[a] = 0.0;
      if (ee < te) {
        int64_t xs = wrapi(x0 - padlo + r, nx);
        const int64_t off = xs * pe + e0 + ee;
        for (int q = 0; q < p.npairs; ++q) {
          const double vq = (double)v[(int64_t)q * plane + off];
#pragma unroll
          for (int a = 0; a < kMaxX; ++a)
            if (a < p.nxf) w[a] += p.mix[a * p.npairs + q] * vq;
        }
      }
#pragma unroll
      for (int a = 0; a < kMaxX; ++a)
        if (a < p.nxf) buf[(a * rows + r) * kTE + ee] = w[a];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTX * kTE; i += blockDim.x) {
      int r = i / kTE, ee = i - r * kTE;
      int64_t x = x0 + r;
      if (x >= nx || ee >= te) continue;
      double acc = 0.0;
      for (int a = 0; a < p.nxf; ++a) {
        const double* col = buf + (a * rows + r + kx - 1) * kTE + ee;
        const double* tp = p.xtap(a);
        for (int j = 0; j < kx; ++j) acc += tp[j] * col[-j * kTE];
      }
      const int64_t o = x * pe + e0 + ee;
      if (epi.mode == STEAM_EPI_FLUX) {
        // F + conv rounded once to the storage dtype
        T f = (T)((double)out[o] + acc);
        if (f < (T)0) {
          s_clip += 1.0;
          f = (T)0;
        }
        out[o] = f;
        int64_t y = (e0 + ee) / nz;
        if (x >= epi.wx0 && x < epi.wx1 && y >= epi.wy0 && y < epi.wy1)
          s_f += (double)f;
      } else {
        out[o] = (T)acc;
      }
    }
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

// ---- dense direct convolution ----------------------------------------------
template <typename T>
__global__ void dense_conv_kernel(const T* __restrict__ in, int64_t nx,
                                  int64_t ny, int64_t nz,
                                  const T* __restrict__ K, int kx, int ky,
                                  int kz, int cx, int cy, int cz,
                                  T* __restrict__ out) {
  const int64_t n = nx * ny * nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t z = i % nz;
    int64_t col = i / nz;
    int64_t y = col % ny;
    int64_t x = col / ny;
    double acc = 0.0;
    for (int a = 0; a < kx; ++a) {
      int64_t xs = wrapi(x - a + cx, nx);
      for (int b = 0; b < ky; ++b) {
        int64_t ys = wrapi(y - b + cy, ny);
        const T* src = in + (xs * ny + ys) * nz;
        const T* kk = K + ((int64_t)a * ky + b) * kz;
        for (int c = 0; c < kz; ++c) {
          int64_t zs = z - c + cz;
          if (zs >= 0 && zs < nz) acc += (double)kk[c] * (double)src[zs];
        }
      }
    }
    out[i] = (T)acc;
  }
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

static int zpass_cols(int nz, int kz, size_t elem) {
  int len = nz + kz - 1;
  int cb = (int)((40 * 1024) / ((size_t)len * elem));
  if (cb < 1) cb = 1;
  if (cb > 64) cb = 64;
  return cb;
}

static int64_t epi_cells(const steam_window_t* w, int64_t nx, int64_t ny) {
  if (!w) return nx * ny;
  return (w->x1 - w->x0) * (w->y1 - w->y0);
}

template <typename T>
static int run_separable(int64_t nx, int64_t ny, int64_t nz,
                         const steam_sepconv_t* spec, const double* zt,
                         const double* yt, const double* xt, const void* in_v,
                         const double* pre_div, const double* pre_mul,
                         void* out_v, int epilogue, const steam_window_t* win,
                         double* sums_out, void* ws, size_t ws_bytes,
                         cudaStream_t s) {
  SepParams<T>* pp = new SepParams<T>();
  std::unique_ptr<SepParams<T>> guard(pp);
  int rc = fill_params<T>(spec, zt, yt, xt, *pp);
  if (rc) return rc;
  SepParams<T>& p = *pp;
  const int64_t plane = nx * ny * nz;
  Carver c(ws, ws_bytes);
  T* u = c.take<T>((size_t)p.nzf * plane);
  T* v = c.take<T>((size_t)p.npairs * plane);
  T* pre = nullptr;
  const bool use_pre = pre_div != nullptr || pre_mul != nullptr;
  if (use_pre) pre = c.take<T>((size_t)2 * nz);
  int xgrid = stride_grid(((nx + kTX - 1) / kTX) * ((ny * nz + kTE - 1) / kTE), 1, 4);
  double* partials = c.take<double>((size_t)xgrid * 2);
  double* totals = c.take<double>(2);
  if (!u || !v || (use_pre && !pre) || !partials || !totals)
    return fail(STEAM_ERR_WORKSPACE,
                "steam_conv_separable: workspace too small");
  const T* in = (const T*)in_v;
  T* out = (T*)out_v;
  if (use_pre) {
    std::vector<T> h(2 * nz);
    for (int64_t z = 0; z < nz; ++z) {
      h[z] = pre_div ? (T)pre_div[z] : (T)1;
      h[nz + z] = pre_mul ? (T)pre_mul[z] : (T)1;
    }
    STEAM_CUDA(cudaMemcpyAsync(pre, h.data(), sizeof(T) * 2 * nz,
                               cudaMemcpyHostToDevice, s));
    STEAM_CUDA(cudaStreamSynchronize(s));
  }
  // z-pass
  {
    const int64_t ncol = nx * ny;
    int cb = zpass_cols((int)nz, p.kz, sizeof(T));
    size_t sm = (size_t)cb * (nz + p.kz - 1) * sizeof(T);
    int grid = stride_grid((ncol + cb - 1) / cb, 1, 4);
    if (use_pre) {
      STEAM_CUDA(cudaFuncSetAttribute(zpass_kernel<T, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sm));
      zpass_kernel<T, true><<<grid, 256, sm, s>>>(in, ncol, (int)nz, cb, pre,
                                                  pre + nz, p, u, plane);
    } else {
      STEAM_CUDA(cudaFuncSetAttribute(zpass_kernel<T, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)sm));
      zpass_kernel<T, false><<<grid, 256, sm, s>>>(in, ncol, (int)nz, cb,
                                                   nullptr, nullptr, p, u,
                                                   plane);
    }
    STEAM_LAUNCH_CHECK("conv z-pass");
  }
  // y-pass
  {
    size_t sm = (size_t)p.nzf * (kTY + p.ky - 1) * kTZ * sizeof(T);
    STEAM_REQUIRE(sm <= 200 * 1024, "steam_conv_separable: y filter too long");
    STEAM_CUDA(cudaFuncSetAttribute(ypass_kernel<T>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sm));
    int64_t tiles = nx * ((ny + kTY - 1) / kTY) * ((nz + kTZ - 1) / kTZ);
    int grid = stride_grid(tiles, 1, 4);
    ypass_kernel<T><<<grid, 256, sm, s>>>(u, nx, ny, (int)nz, p, v, plane);
    STEAM_LAUNCH_CHECK("conv y-pass");
  }
  // x-pass with epilogue
  {
    size_t sm = (size_t)p.nxf * (kTX + p.kx - 1) * kTE * sizeof(double);
    STEAM_REQUIRE(sm <= 200 * 1024, "steam_conv_separable: x filter too long");
    STEAM_CUDA(cudaFuncSetAttribute(xpass_kernel<T>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sm));
    XEpi epi;
    epi.mode = epilogue;
    epi.wx0 = win ? win->x0 : 0;
    epi.wx1 = win ? win->x1 : nx;
    epi.wy0 = win ? win->y0 : 0;
    epi.wy1 = win ? win->y1 : ny;
    xpass_kernel<T><<<xgrid, 256, sm, s>>>(v, nx, ny, (int)nz, p, out, plane,
                                           epi, partials);
    STEAM_LAUNCH_CHECK("conv x-pass");
  }
  if (epilogue == STEAM_EPI_FLUX) {
    rc = reduce_partials(partials, xgrid, 2, totals, s);
    if (rc) return rc;
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
  int xgrid = stride_grid(((nx + kTX - 1) / kTX) * ((ny * nz + kTE - 1) / kTE), 1, 4);
  return carve_bytes((size_t)spec->n_z * plane, elem) +
         carve_bytes((size_t)spec->n_pairs * plane, elem) +
         carve_bytes((size_t)2 * nz, elem) +
         carve_bytes((size_t)xgrid * 2, sizeof(double)) +
         carve_bytes(2, sizeof(double));
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
  STEAM_REQUIRE(epilogue == STEAM_EPI_STORE || epilogue == STEAM_EPI_FLUX,
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
                                pre_div, pre_mul, out, epilogue, window,
                                sums_out, workspace, workspace_bytes, s);
  if (dtype == STEAM_F64)
    return run_separable<double>(nx, ny, nz, spec, z_taps, y_taps, x_taps, in,
                                 pre_div, pre_mul, out, epilogue, window,
                                 sums_out, workspace, workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_conv_separable: bad dtype");
}

extern "C" int steam_conv_dense(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                const void* kernel, int32_t kx, int32_t ky,
                                int32_t kz, const void* in, void* out,
                                steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0,
                "steam_conv_dense: negative extent");
  STEAM_REQUIRE(kx >= 1 && ky >= 1 && kz >= 1,
                "steam_conv_dense: kernel extents must be >= 1");
  STEAM_REQUIRE(kx <= nx && ky <= ny,
                "steam_conv_dense: fold the kernel onto the field period first");
  const int64_t n = nx * ny * nz;
  if (n == 0) return STEAM_OK;
  STEAM_REQUIRE(kernel && in && out, "steam_conv_dense: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  int grid = stride_grid(n, 256, 8);
  const int cx = (kx - 1) / 2, cy = (ky - 1) / 2, cz = (kz - 1) / 2;
  if (dtype == STEAM_F32)
    dense_conv_kernel<float><<<grid, 256, 0, s>>>(
        (const float*)in, nx, ny, nz, (const float*)kernel, kx, ky, kz, cx, cy,
        cz, (float*)out);
  else if (dtype == STEAM_F64)
    dense_conv_kernel<double><<<grid, 256, 0, s>>>(
        (const double*)in, nx, ny, nz, (const double*)kernel, kx, ky, kz, cx,
        cy, cz, (double*)out);
  else
    return fail(STEAM_ERR_ARG, "steam_conv_dense: bad dtype");
  STEAM_LAUNCH_CHECK("steam_conv_dense");
  return STEAM_OK;
}
