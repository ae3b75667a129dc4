// Error state, device geometry, deterministic partial reduction and the
// elementwise helpers shared by the entry points.
#include "common.cuh"

#include <algorithm>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

namespace steam {

static thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int sm_count() {
  static std::mutex mu;
  static std::vector<int> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)cache.size() <= dev) cache.resize(dev + 1, 0);
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
            cudaSuccess ||
        n <= 0)
      n = 148;
    cache[dev] = n;
  }
  return cache[dev];
}

int stride_grid(int64_t n, int per_block, int blocks_per_sm) {
  int64_t need = (n + per_block - 1) / per_block;
  int64_t cap = (int64_t)sm_count() * blocks_per_sm;
  if (need < 1) need = 1;
  return (int)(need < cap ? need : cap);
}

__global__ void reduce_partials_kernel(const double* __restrict__ partials,
                                       int nblocks, double* __restrict__ out) {
  __shared__ double scratch[32];
  const double* src = partials + (size_t)blockIdx.x * nblocks;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) acc += src[i];
  double s = block_sum(acc, scratch);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

int reduce_partials(const double* partials, int nblocks, int nq, double* out,
                    cudaStream_t stream) {
  if (nq <= 0) return STEAM_OK;
  reduce_partials_kernel<<<nq, 256, 0, stream>>>(partials, nblocks, out);
  STEAM_LAUNCH_CHECK("reduce_partials");
  return STEAM_OK;
}

template <typename T>
__global__ void scale_kernel(int64_t n, T* __restrict__ f, T s, int fill) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    f[i] = fill ? s : f[i] * s;
  }
}

// One warp per output row (i, j): out[i][j][:] = box[x0 + i][y0 + j][z0 + :] * s
// (or s with fill), z the fastest axis on both sides.
template <typename T>
__global__ void tile_extract_kernel(int64_t ny, int64_t nz, const T* __restrict__ box,
                                    int64_t x0, int64_t y0, int64_t z0, int64_t ox,
                                    int64_t oy, int64_t oz, T s, int fill,
                                    T* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       row < ox * oy; row += warps) {
    const int64_t i = row / oy, j = row - i * oy;
    const T* src = box + ((x0 + i) * ny + (y0 + j)) * nz + z0;
    T* dst = out + row * oz;
    for (int64_t k = lane; k < oz; k += 32) dst[k] = fill ? s : src[k] * s;
  }
}

template <typename T>
__global__ void accumulate_levels_kernel(int64_t n, int64_t nz, T* __restrict__ acc,
                                         const T* __restrict__ a,
                                         const T* __restrict__ b,
                                         const T* __restrict__ coef) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const T d = b ? a[i] - b[i] : a[i];
    acc[i] = acc[i] + coef[i % nz] * d;
  }
}

template <typename T>
static int accumulate_impl(int64_t n, int64_t nz, void* acc, const void* a,
                           const void* b, const double* coef, cudaStream_t s) {
  T* dcoef = nullptr;
  STEAM_CUDA(cudaMallocAsync((void**)&dcoef, sizeof(T) * nz, s));
  std::vector<T> h(nz);
  for (int64_t z = 0; z < nz; ++z) h[z] = (T)coef[z];
  cudaError_t e = cudaMemcpyAsync(dcoef, h.data(), sizeof(T) * nz,
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    accumulate_levels_kernel<T><<<stride_grid(n, 1024), 256, 0, s>>>(
        n, nz, (T*)acc, (const T*)a, (const T*)b, dcoef);
    count_launch();
    e = cudaGetLastError();
  }
  cudaFreeAsync(dcoef, s);
  if (e != cudaSuccess)
    return fail(STEAM_ERR_CUDA, std::string("steam_accumulate_levels: ") +
                                    cudaGetErrorString(e));
  // The staging vector is pageable and copied before return; no sync needed.
  return STEAM_OK;
}

}  // namespace steam

using namespace steam;

extern "C" int steam_accumulate_levels(int dtype, int64_t nx, int64_t ny,
                                       int64_t nz, void* acc, const void* a,
                                       const void* b, const double* coef,
                                       steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0,
                "steam_accumulate_levels: negative extent");
  const int64_t n = nx * ny * nz;
  if (n == 0) return STEAM_OK;
  STEAM_REQUIRE(acc && a && coef, "steam_accumulate_levels: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32) return accumulate_impl<float>(n, nz, acc, a, b, coef, s);
  if (dtype == STEAM_F64) return accumulate_impl<double>(n, nz, acc, a, b, coef, s);
  return fail(STEAM_ERR_ARG, "steam_accumulate_levels: bad dtype");
}

// ---- output composition: add a level profile and clamp -------------------------
template <typename T>
__global__ void add_levels_clamp_kernel(int64_t n, int64_t nz, T* __restrict__ f,
                                        const T* __restrict__ add, T lo, T hi) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    T v = f[i] + add[i % nz];
    v = v < lo ? lo : v;
    f[i] = v > hi ? hi : v;
  }
}

template <typename T>
static int add_levels_clamp_impl(int64_t n, int64_t nz, void* f, const double* add, double lo,
                                 double hi, cudaStream_t s) {
  T* dadd = nullptr;
  STEAM_CUDA(cudaMallocAsync((void**)&dadd, sizeof(T) * nz, s));
  std::vector<T> h(nz);
  for (int64_t z = 0; z < nz; ++z) h[z] = (T)add[z];
  cudaError_t e = cudaMemcpyAsync(dadd, h.data(), sizeof(T) * nz, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // h dies with this frame
  if (e == cudaSuccess) {
    add_levels_clamp_kernel<T><<<stride_grid(n, 1024), 256, 0, s>>>(n, nz, (T*)f, dadd, (T)lo,
                                                                    (T)hi);
    count_launch();
    e = cudaGetLastError();
  }
  cudaFreeAsync(dadd, s);
  if (e != cudaSuccess)
    return fail(STEAM_ERR_CUDA, std::string("steam_add_levels_clamp: ") + cudaGetErrorString(e));
  return STEAM_OK;
}

// ---- z-major slab of a field (x, y, z) -> (z, x, y) ----------------------------
// The field as a matrix [nx*ny columns][nz levels]; a 32 x 32 tile goes
// through shared memory so both the reads (along z) and the writes (along
// the columns) are coalesced.
template <typename T>
__global__ void __launch_bounds__(256) slab_zmajor_kernel(const T* __restrict__ f, int64_t ncol,
                                                          int64_t nz, int64_t z0, int64_t dz,
                                                          T* __restrict__ out) {
  __shared__ T tile[32][33];
  const int64_t ctiles = (ncol + 31) / 32, ztiles = (dz + 31) / 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int64_t t = blockIdx.x; t < ctiles * ztiles; t += gridDim.x) {
    const int64_t c0 = (t / ztiles) * 32, zt0 = (t % ztiles) * 32;
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
      const int64_t c = c0 + r, z = zt0 + tx;
      if (c < ncol && z < dz) tile[r][tx] = f[c * nz + z0 + z];
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
      const int64_t z = zt0 + r, c = c0 + tx;
      if (c < ncol && z < dz) out[z * ncol + c] = tile[tx][r];
    }
  }
}

// ---- flux advance, device-side finish ---------------------------------------------
// The volume-mean restore of the flux advance (steam/simulate.py:2204-2218)
// with its scalars read from device memory: every thread derives the same
// factor from the entering and realized sums, so no host round trip is
// needed between the convolution and the restore.
template <typename T>
__device__ __forceinline__ void flux_factor(const double* ns, const double* cs, double cells,
                                            T& factor, int& fill) {
  const double c = cells > 1.0 ? cells : 1.0;
  const double entering = ns[0] / c, realized = cs[0] / c;
  fill = !(realized > 0.0);
  factor = fill ? (T)entering : (T)(entering / realized);
}

template <typename T>
__global__ void flux_finish_kernel(int64_t n, T* __restrict__ f, const double* __restrict__ ns,
                                   const double* __restrict__ cs, double cells,
                                   double* __restrict__ ledger) {
  T factor;
  int fill;
  flux_factor<T>(ns, cs, cells, factor, fill);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (sizeof(T) == 4 && ((uintptr_t)f % 16) == 0) {
    float4* f4 = reinterpret_cast<float4*>(f);
    const int64_t n4 = n / 4;
    for (int64_t i = i0; i < n4; i += stride) {
      float4 v = f4[i];
      if (fill) {
        v.x = v.y = v.z = v.w = (float)factor;
      } else {
        v.x = __fmul_rn(v.x, (float)factor);
        v.y = __fmul_rn(v.y, (float)factor);
        v.z = __fmul_rn(v.z, (float)factor);
        v.w = __fmul_rn(v.w, (float)factor);
      }
      f4[i] = v;
    }
    for (int64_t i = 4 * n4 + i0; i < n; i += stride) f[i] = fill ? factor : mul_rn(f[i], factor);
  } else {
    for (int64_t i = i0; i < n; i += stride) f[i] = fill ? factor : mul_rn(f[i], factor);
  }
  if (ledger && blockIdx.x == 0 && threadIdx.x == 0) {
    // entering (sum, cells), |noise| (sum, count), realized (sum, cells),
    // clipped count, S scale (rounded to T), restore factor (rounded to T)
    const double nnz = ns[2];
    const double mean_abs = ns[1] / (nnz > 1.0 ? nnz : 1.0);
    ledger[0] = ns[0];
    ledger[1] = cells;
    ledger[2] = ns[1];
    ledger[3] = nnz;
    ledger[4] = cs[0];
    ledger[5] = cells;
    ledger[6] = cs[1];
    ledger[7] = mean_abs > 0.0 ? (double)(T)(1.0 / mean_abs) : 1.0;
    ledger[8] = (double)factor;
    ledger[9] = fill;
  }
}

extern "C" int steam_flux_finish_async(int dtype, int64_t n, void* flux,
                                       const double* noise_sums_dev,
                                       const double* conv_sums_dev, double cells,
                                       double* ledger_dev, steam_stream_t stream) {
  STEAM_REQUIRE(n >= 0, "steam_flux_finish_async: negative size");
  STEAM_REQUIRE(noise_sums_dev && conv_sums_dev, "steam_flux_finish_async: null sums");
  STEAM_REQUIRE(n == 0 || flux, "steam_flux_finish_async: null flux");
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = stride_grid(n > 0 ? (n + 3) / 4 : 1, 256);
  if (dtype == STEAM_F32)
    flux_finish_kernel<float><<<grid, 256, 0, s>>>(n, (float*)flux, noise_sums_dev,
                                                   conv_sums_dev, cells, ledger_dev);
  else if (dtype == STEAM_F64)
    flux_finish_kernel<double><<<grid, 256, 0, s>>>(n, (double*)flux, noise_sums_dev,
                                                    conv_sums_dev, cells, ledger_dev);
  else
    return fail(STEAM_ERR_ARG, "steam_flux_finish_async: bad dtype");
  STEAM_LAUNCH_CHECK("steam_flux_finish_async");
  return STEAM_OK;
}

extern "C" const char* steam_last_error(void) { return g_last_error.c_str(); }

extern "C" int steam_version(void) { return 1; }

extern "C" unsigned long long steam_launch_count(void) {
  return g_launches.load(std::memory_order_relaxed);
}

extern "C" int steam_scale(int dtype, int64_t n, void* field, double scale,
                           int32_t fill, steam_stream_t stream) {
  STEAM_REQUIRE(n >= 0, "steam_scale: negative size");
  if (n == 0) return STEAM_OK;
  STEAM_REQUIRE(field != nullptr, "steam_scale: null field");
  cudaStream_t s = (cudaStream_t)stream;
  int grid = stride_grid(n, 256 * 4);
  if (dtype == STEAM_F32)
    scale_kernel<float><<<grid, 256, 0, s>>>(n, (float*)field, (float)scale, fill);
  else if (dtype == STEAM_F64)
    scale_kernel<double><<<grid, 256, 0, s>>>(n, (double*)field, scale, fill);
  else
    return fail(STEAM_ERR_ARG, "steam_scale: bad dtype");
  STEAM_LAUNCH_CHECK("steam_scale");
  return STEAM_OK;
}

extern "C" int steam_tile_extract(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                  const void* box, int64_t x0, int64_t y0, int64_t z0,
                                  int64_t ox, int64_t oy, int64_t oz, double scale,
                                  int32_t fill, void* out, steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0 && ox >= 0 && oy >= 0 && oz >= 0,
                "steam_tile_extract: negative size");
  STEAM_REQUIRE(x0 >= 0 && y0 >= 0 && z0 >= 0 && x0 + ox <= nx && y0 + oy <= ny &&
                    z0 + oz <= nz,
                "steam_tile_extract: window outside the box");
  if (ox == 0 || oy == 0 || oz == 0) return STEAM_OK;
  STEAM_REQUIRE(box != nullptr && out != nullptr, "steam_tile_extract: null array");
  cudaStream_t s = (cudaStream_t)stream;
  int grid = stride_grid(ox * oy, 8, 8);
  if (dtype == STEAM_F32)
    tile_extract_kernel<float><<<grid, 256, 0, s>>>(ny, nz, (const float*)box, x0, y0, z0,
                                                    ox, oy, oz, (float)scale, fill,
                                                    (float*)out);
  else if (dtype == STEAM_F64)
    tile_extract_kernel<double><<<grid, 256, 0, s>>>(ny, nz, (const double*)box, x0, y0,
                                                     z0, ox, oy, oz, scale, fill,
                                                     (double*)out);
  else
    return fail(STEAM_ERR_ARG, "steam_tile_extract: bad dtype");
  STEAM_LAUNCH_CHECK("steam_tile_extract");
  return STEAM_OK;
}

extern "C" int steam_add_levels_clamp(int dtype, int64_t nx, int64_t ny, int64_t nz, void* field,
                                      const double* add, double lo, double hi,
                                      steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "steam_add_levels_clamp: negative extent");
  STEAM_REQUIRE(lo <= hi, "steam_add_levels_clamp: lower bound above the upper");
  const int64_t n = nx * ny * nz;
  if (n == 0) return STEAM_OK;
  STEAM_REQUIRE(field && add, "steam_add_levels_clamp: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32) return add_levels_clamp_impl<float>(n, nz, field, add, lo, hi, s);
  if (dtype == STEAM_F64) return add_levels_clamp_impl<double>(n, nz, field, add, lo, hi, s);
  return fail(STEAM_ERR_ARG, "steam_add_levels_clamp: bad dtype");
}

extern "C" int steam_slab_zmajor(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                 const void* field, int64_t z0, int64_t dz, void* out,
                                 steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0 && dz >= 0,
                "steam_slab_zmajor: negative extent");
  STEAM_REQUIRE(z0 >= 0 && z0 + dz <= nz, "steam_slab_zmajor: levels outside the field");
  const int64_t ncol = nx * ny;
  if (ncol * dz == 0) return STEAM_OK;
  STEAM_REQUIRE(field && out, "steam_slab_zmajor: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t tiles = ((ncol + 31) / 32) * ((dz + 31) / 32);
  const int grid = stride_grid(tiles, 1, 8);
  if (dtype == STEAM_F32)
    slab_zmajor_kernel<float><<<grid, 256, 0, s>>>((const float*)field, ncol, nz, z0, dz,
                                                   (float*)out);
  else if (dtype == STEAM_F64)
    slab_zmajor_kernel<double><<<grid, 256, 0, s>>>((const double*)field, ncol, nz, z0, dz,
                                                    (double*)out);
  else
    return fail(STEAM_ERR_ARG, "steam_slab_zmajor: bad dtype");
  STEAM_LAUNCH_CHECK("steam_slab_zmajor");
  return STEAM_OK;
}

// ---- the flux epilogue on its own -------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) flux_clip_kernel(int64_t nx, int64_t ny, int64_t nz,
                                                        T* __restrict__ f,
                                                        const T* __restrict__ conv,
                                                        int64_t wx0, int64_t wx1, int64_t wy0,
                                                        int64_t wy1,
                                                        double* __restrict__ partials) {
  __shared__ double scratch[32];
  const int64_t n = nx * ny * nz;
  double s_f = 0.0, s_clip = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t col = i / nz;
    const int64_t y = col % ny, x = col / ny;
    const bool inw = x >= wx0 && x < wx1 && y >= wy0 && y < wy1;
    // F + conv rounded once to the storage dtype, as the fused epilogues do
    T v = (T)((double)f[i] + (double)conv[i]);
    if (v < (T)0) {
      if (inw) s_clip += 1.0;
      v = (T)0;
    }
    f[i] = v;
    if (inw) s_f += (double)v;
  }
  const double t0 = block_sum(s_f, scratch);
  const double t1 = block_sum(s_clip, scratch);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = t0;
    partials[gridDim.x + blockIdx.x] = t1;
  }
}

static int flux_clip_grid(int64_t n) { return stride_grid(n, 256, 4); }

// ---- wrapped boxes of columns between a host field and a device box --------------
// A box of bx x by columns starting at (x0, y0) of an (nx, ny, nz) field,
// wrapping in x and y, levels [z0, z0 + bz): up to four 3D copies (one per
// wrapped part), each a pitched copy of whole column runs.
static int box_copy(size_t elem, void* host, int64_t nx, int64_t ny, int64_t nz, int64_t x0,
                    int64_t y0, int64_t z0, int64_t bx, int64_t by, int64_t bz, void* dev,
                    int to_device, cudaStream_t s) {
  const char* who = to_device ? "steam_box_h2d" : "steam_box_d2h";
  STEAM_REQUIRE(nx > 0 && ny > 0 && nz > 0 && bx >= 0 && by >= 0 && bz >= 0,
                std::string(who) + ": bad extent");
  STEAM_REQUIRE(bx <= nx && by <= ny && z0 >= 0 && z0 + bz <= nz,
                std::string(who) + ": box larger than the field");
  STEAM_REQUIRE(x0 >= 0 && x0 < nx && y0 >= 0 && y0 < ny, std::string(who) + ": origin outside");
  if (bx * by * bz == 0) return STEAM_OK;
  STEAM_REQUIRE(host && dev, std::string(who) + ": null pointer");
  for (int64_t xa = 0; xa < bx;) {
    const int64_t hx = (x0 + xa) % nx;
    const int64_t nxp = std::min(bx - xa, nx - hx);
    for (int64_t ya = 0; ya < by;) {
      const int64_t hy = (y0 + ya) % ny;
      const int64_t nyp = std::min(by - ya, ny - hy);
      cudaMemcpy3DParms p = {};
      cudaPitchedPtr hp = make_cudaPitchedPtr(host, (size_t)nz * elem, (size_t)nz, (size_t)ny);
      cudaPitchedPtr dp = make_cudaPitchedPtr(dev, (size_t)bz * elem, (size_t)bz, (size_t)by);
      const cudaPos hpos = make_cudaPos((size_t)z0 * elem, (size_t)hy, (size_t)hx);
      const cudaPos dpos = make_cudaPos(0, (size_t)ya, (size_t)xa);
      p.extent = make_cudaExtent((size_t)bz * elem, (size_t)nyp, (size_t)nxp);
      if (to_device) {
        p.srcPtr = hp;
        p.srcPos = hpos;
        p.dstPtr = dp;
        p.dstPos = dpos;
        p.kind = cudaMemcpyHostToDevice;
      } else {
        p.srcPtr = dp;
        p.srcPos = dpos;
        p.dstPtr = hp;
        p.dstPos = hpos;
        p.kind = cudaMemcpyDeviceToHost;
      }
      STEAM_CUDA(cudaMemcpy3DAsync(&p, s));
      ya += nyp;
    }
    xa += nxp;
  }
  return STEAM_OK;
}

extern "C" int steam_box_h2d(int32_t elem_bytes, const void* host, int64_t nx, int64_t ny,
                             int64_t nz, int64_t x0, int64_t y0, int64_t z0, int64_t bx,
                             int64_t by, int64_t bz, void* dev, steam_stream_t stream) {
  STEAM_REQUIRE(elem_bytes == 4 || elem_bytes == 8, "steam_box_h2d: element size 4 or 8");
  return box_copy((size_t)elem_bytes, const_cast<void*>(host), nx, ny, nz, x0, y0, z0, bx, by,
                  bz, dev, 1, (cudaStream_t)stream);
}

extern "C" int steam_box_d2h(int32_t elem_bytes, const void* dev, int64_t bx_full,
                             int64_t by_full, int64_t bz_full, int64_t ox, int64_t oy,
                             int64_t oz, int64_t bx, int64_t by, int64_t bz, void* host,
                             int64_t nx, int64_t ny, int64_t nz, int64_t x0, int64_t y0,
                             int64_t z0, steam_stream_t stream) {
  STEAM_REQUIRE(elem_bytes == 4 || elem_bytes == 8, "steam_box_d2h: element size 4 or 8");
  STEAM_REQUIRE(ox >= 0 && oy >= 0 && oz >= 0 && ox + bx <= bx_full && oy + by <= by_full &&
                    oz + bz <= bz_full,
                "steam_box_d2h: window outside the device box");
  if (bx * by * bz == 0) return STEAM_OK;
  STEAM_REQUIRE(dev && host, "steam_box_d2h: null pointer");
  // the window of the device box as its own pitched array: start pointer at
  // (ox, oy, oz), pitches of the full box
  const size_t e = (size_t)elem_bytes;
  cudaStream_t s = (cudaStream_t)stream;
  STEAM_REQUIRE(bx <= nx && by <= ny && z0 >= 0 && z0 + bz <= nz,
                "steam_box_d2h: box larger than the field");
  STEAM_REQUIRE(x0 >= 0 && x0 < nx && y0 >= 0 && y0 < ny, "steam_box_d2h: origin outside");
  for (int64_t xa = 0; xa < bx;) {
    const int64_t hx = (x0 + xa) % nx;
    const int64_t nxp = std::min(bx - xa, nx - hx);
    for (int64_t ya = 0; ya < by;) {
      const int64_t hy = (y0 + ya) % ny;
      const int64_t nyp = std::min(by - ya, ny - hy);
      cudaMemcpy3DParms p = {};
      p.srcPtr = make_cudaPitchedPtr(const_cast<void*>(dev), (size_t)bz_full * e,
                                     (size_t)bz_full, (size_t)by_full);
      p.srcPos = make_cudaPos((size_t)oz * e, (size_t)(oy + ya), (size_t)(ox + xa));
      p.dstPtr = make_cudaPitchedPtr(host, (size_t)nz * e, (size_t)nz, (size_t)ny);
      p.dstPos = make_cudaPos((size_t)z0 * e, (size_t)hy, (size_t)hx);
      p.extent = make_cudaExtent((size_t)bz * e, (size_t)nyp, (size_t)nxp);
      p.kind = cudaMemcpyDeviceToHost;
      STEAM_CUDA(cudaMemcpy3DAsync(&p, s));
      ya += nyp;
    }
    xa += nxp;
  }
  return STEAM_OK;
}

extern "C" size_t steam_flux_clip_workspace_bytes(int64_t nx, int64_t ny, int64_t nz) {
  return carve_bytes((size_t)2 * flux_clip_grid(nx * ny * nz), sizeof(double));
}

extern "C" int steam_flux_clip_async(int dtype, int64_t nx, int64_t ny, int64_t nz, void* flux,
                                     const void* conv, const steam_window_t* window,
                                     double* sums_dev, void* workspace, size_t workspace_bytes,
                                     steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "steam_flux_clip_async: negative extent");
  STEAM_REQUIRE(sums_dev, "steam_flux_clip_async: null sums_dev");
  if (window)
    STEAM_REQUIRE(window->x0 >= 0 && window->x1 <= nx && window->x0 <= window->x1 &&
                      window->y0 >= 0 && window->y1 <= ny && window->y0 <= window->y1,
                  "steam_flux_clip_async: window outside the array");
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t n = nx * ny * nz;
  if (n == 0) {
    STEAM_CUDA(cudaMemsetAsync(sums_dev, 0, 2 * sizeof(double), s));
    return STEAM_OK;
  }
  STEAM_REQUIRE(flux && conv, "steam_flux_clip_async: null field");
  const int grid = flux_clip_grid(n);
  Carver c(workspace, workspace_bytes);
  double* partials = c.take<double>((size_t)2 * grid);
  if (!partials) return fail(STEAM_ERR_WORKSPACE, "steam_flux_clip_async: workspace too small");
  const int64_t wx0 = window ? window->x0 : 0, wx1 = window ? window->x1 : nx;
  const int64_t wy0 = window ? window->y0 : 0, wy1 = window ? window->y1 : ny;
  if (dtype == STEAM_F32)
    flux_clip_kernel<float><<<grid, 256, 0, s>>>(nx, ny, nz, (float*)flux, (const float*)conv,
                                                 wx0, wx1, wy0, wy1, partials);
  else if (dtype == STEAM_F64)
    flux_clip_kernel<double><<<grid, 256, 0, s>>>(nx, ny, nz, (double*)flux,
                                                  (const double*)conv, wx0, wx1, wy0, wy1,
                                                  partials);
  else
    return fail(STEAM_ERR_ARG, "steam_flux_clip_async: bad dtype");
  STEAM_LAUNCH_CHECK("steam_flux_clip_async");
  return reduce_partials(partials, grid, 2, sums_dev, s);
}
