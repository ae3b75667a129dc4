// World-keyed noise: Philox4x32-10 uniforms, the sparse extremal Levy field
// and the fused multiplier-noise / entering-measure pass of the flux advance.
#include "common.cuh"

namespace steam {

__device__ __forceinline__ int64_t wrap_mod(int64_t v, int64_t n) {
  if (v >= 0 && v < n) return v;  // the common case: no division
  int64_t r = v % n;
  return r < 0 ? r + n : r;
}

// Python-semantics divisibility test (sign of the remainder is irrelevant).
__device__ __forceinline__ bool divisible(int64_t v, int64_t f) {
  return f == 1 || (v % f) == 0;
}

struct RegionDev {
  int64_t nx, ny, nz;
  int64_t ox, oy, oz;
  int64_t wx, wy;
  int32_t sx, sy, sz;
  PhiloxKey key;
};

static RegionDev to_dev(const steam_region_t& r) {
  RegionDev d;
  d.nx = r.shape[0];
  d.ny = r.shape[1];
  d.nz = r.shape[2];
  d.ox = r.origin[0];
  d.oy = r.origin[1];
  d.oz = r.origin[2];
  d.wx = r.world[0];
  d.wy = r.world[1];
  d.sx = r.sparsity[0];
  d.sy = r.sparsity[1];
  d.sz = r.sparsity[2];
  d.key = philox_key(r.key[0], r.key[1], r.key[2]);
  return d;
}

static int check_region(const steam_region_t* r, const char* who) {
  STEAM_REQUIRE(r != nullptr, std::string(who) + ": null region");
  for (int a = 0; a < 3; ++a) {
    STEAM_REQUIRE(r->shape[a] >= 0, std::string(who) + ": negative shape");
    STEAM_REQUIRE(r->sparsity[a] >= 1,
                  std::string(who) + ": sparsity factors must be >= 1");
  }
  STEAM_REQUIRE(r->world[0] >= 1 && r->world[1] >= 1,
                std::string(who) + ": world x/y extents must be >= 1");
  STEAM_REQUIRE(r->world[1] <= 0xFFFFFFFFll,
                std::string(who) + ": world y extent beyond 2^32");
  return STEAM_OK;
}

// gamma at local cell (x, y, z) of the region; zero off the centre lattice.
template <typename T>
__device__ __forceinline__ T region_gamma(const RegionDev& r, int64_t x,
                                          int64_t y, int64_t z,
                                          const LevyParams<T>& lp) {
  int64_t gx = wrap_mod(x + r.ox, r.wx);
  int64_t gy = wrap_mod(y + r.oy, r.wy);
  int64_t gz = z + r.oz;
  if (!divisible(gx, r.sx) || !divisible(gy, r.sy) || !divisible(gz, r.sz))
    return (T)0;
  uint32_t r0, r1;
  philox_site(gx, (uint32_t)gy, gz, r.key, r0, r1);
  return levy_draw<T>((T)lattice_uniform(r0), (T)lattice_uniform(r1), lp);
}

// float32: the exactly reduced form (see levy_draw_f32).
template <>
__device__ __forceinline__ float region_gamma<float>(const RegionDev& r, int64_t x,
                                                     int64_t y, int64_t z,
                                                     const LevyParams<float>& lp) {
  int64_t gx = wrap_mod(x + r.ox, r.wx);
  int64_t gy = wrap_mod(y + r.oy, r.wy);
  int64_t gz = z + r.oz;
  if (!divisible(gx, r.sx) || !divisible(gy, r.sy) || !divisible(gz, r.sz))
    return 0.0f;
  uint32_t r0, r1;
  philox_site(gx, (uint32_t)gy, gz, r.key, r0, r1);
  return levy_draw_f32(lattice_uniform(r0), lattice_uniform(r1), lp);
}

__global__ void keyed_uniforms_kernel(const int64_t* __restrict__ ix,
                                      const int64_t* __restrict__ iy,
                                      const int64_t* __restrict__ iz,
                                      int64_t ny, int64_t nz, int64_t n,
                                      PhiloxKey key, float* __restrict__ lane0,
                                      float* __restrict__ lane1) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = i % nz;
    int64_t col = i / nz;
    int64_t b = col % ny;
    int64_t a = col / ny;
    uint32_t r0, r1;
    philox_site(ix[a], (uint32_t)iy[b], iz[c], key, r0, r1);
    lane0[i] = lattice_uniform(r0);
    lane1[i] = lattice_uniform(r1);
  }
}

template <typename T>
__global__ void levy_field_kernel(RegionDev r, LevyParams<T> lp,
                                  T* __restrict__ out) {
  const int64_t n = r.nx * r.ny * r.nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t z = i % r.nz;
    int64_t col = i / r.nz;
    int64_t y = col % r.ny;
    int64_t x = col / r.ny;
    out[i] = region_gamma<T>(r, x, y, z, lp);
  }
}

constexpr int kNoiseZLanes = 32;

struct NoiseArgs {
  double scale, shift;
  int32_t n_zero, zero_bottom, zero_top;
  int64_t wx0, wx1, wy0, wy1;
};

// eps = expm1(gamma*scale - shift) at centres (0 elsewhere), product =
// eps * flux; block partials of {sum flux, sum |eps|, nnz eps} over window.
// Threads walk the z levels of a column (coalesced), blocks walk columns, so
// the column's x and y come from one 32-bit division per column.
template <typename T>
__global__ void __launch_bounds__(256) flux_noise_kernel(
    RegionDev r, LevyParams<T> lp, NoiseArgs a, const T* __restrict__ flux,
    T* __restrict__ product, double* __restrict__ partials) {
  __shared__ double scratch[32];
  const T scale = (T)a.scale, shift = (T)a.shift;
  const uint32_t ncol = (uint32_t)(r.nx * r.ny);
  const uint32_t ny = (uint32_t)r.ny;
  const int nz = (int)r.nz;
  // up to kNoiseZLanes threads per column, each taking every kNoiseZLanes-th
  // level, so the per-column work (walk, wrap, window, the x and y words of
  // the Philox counter) is shared by several cells
  const int zlanes = nz < kNoiseZLanes ? nz : kNoiseZLanes;
  const int cols_per_iter = (int)blockDim.x / zlanes;
  const int cofs = threadIdx.x / zlanes;
  const int zt = threadIdx.x - cofs * zlanes;
  double s_flux = 0.0, s_abs = 0.0;
  unsigned s_nnz = 0u;  // nonzero count, exact as an integer
  if (cofs < cols_per_iter) {
    // columns visited with a fixed stride: x and y advance without a division
    const uint32_t c_step = gridDim.x * cols_per_iter;
    const uint32_t sx = c_step / ny, sy = c_step - sx * ny;
    uint32_t col = blockIdx.x * cols_per_iter + cofs;
    uint32_t x = col / ny, y = col - x * ny;
    for (; col < ncol; col += c_step, x += sx, y += sy) {
      if (y >= ny) {
        y -= ny;
        x += 1;
      }
      const bool in_win = x >= a.wx0 && x < a.wx1 && y >= a.wy0 && y < a.wy1;
      const int64_t base = (int64_t)col * nz;
      for (int z = zt; z < nz; z += zlanes) {
        T gamma = region_gamma<T>(r, x, y, z, lp);
        if (a.n_zero > 0) {
          if (a.zero_bottom && z < a.n_zero) gamma = (T)0;
          if (a.zero_top && z >= nz - a.n_zero) gamma = (T)0;
        }
        T g = mul_rn(gamma, scale);
        T e = (g == (T)0) ? (T)0 : d_expm1(sub_rn(g, shift));
        T f = flux[base + z];
        product[base + z] = mul_rn(e, f);
        if (in_win) {
          s_flux += (double)f;
          s_abs += (double)(e < (T)0 ? -e : e);
          s_nnz += (e != (T)0) ? 1u : 0u;
        }
      }
    }
  }
  double t0 = block_sum(s_flux, scratch);
  double t1 = block_sum(s_abs, scratch);
  double t2 = block_sum((double)s_nnz, scratch);
  if (threadIdx.x == 0) {
    partials[0 * gridDim.x + blockIdx.x] = t0;
    partials[1 * gridDim.x + blockIdx.x] = t1;
    partials[2 * gridDim.x + blockIdx.x] = t2;
  }
}

static constexpr int kNoiseBlocksPerSm = 8;

}  // namespace steam

using namespace steam;

extern "C" int steam_keyed_uniforms(const int64_t* world_ix, int64_t nx,
                                    const int64_t* world_iy, int64_t ny,
                                    const int64_t* world_iz, int64_t nz,
                                    uint32_t key0, uint32_t key1,
                                    uint32_t key2, float* lane0, float* lane1,
                                    steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0,
                "steam_keyed_uniforms: negative extent");
  const int64_t n = nx * ny * nz;
  if (n == 0) return STEAM_OK;
  STEAM_REQUIRE(world_ix && world_iy && world_iz && lane0 && lane1,
                "steam_keyed_uniforms: null pointer");
  int grid = stride_grid(n, 256, 16);
  keyed_uniforms_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(
      world_ix, world_iy, world_iz, ny, nz, n, philox_key(key0, key1, key2), lane0, lane1);
  STEAM_LAUNCH_CHECK("steam_keyed_uniforms");
  return STEAM_OK;
}

extern "C" int steam_levy_field(int dtype, const steam_region_t* region,
                                double alpha, void* out,
                                steam_stream_t stream) {
  int rc = check_region(region, "steam_levy_field");
  if (rc) return rc;
  STEAM_REQUIRE(alpha > 1.0 && alpha <= 2.0,
                "steam_levy_field: alpha must lie in (1, 2]");
  RegionDev r = to_dev(*region);
  const int64_t n = r.nx * r.ny * r.nz;
  if (n == 0) return STEAM_OK;
  STEAM_REQUIRE(out != nullptr, "steam_levy_field: null output");
  int grid = stride_grid(n, 256, 16);
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    levy_field_kernel<float><<<grid, 256, 0, s>>>(r, make_levy<float>(alpha),
                                                  (float*)out);
  else if (dtype == STEAM_F64)
    levy_field_kernel<double><<<grid, 256, 0, s>>>(
        r, make_levy<double>(alpha), (double*)out);
  else
    return fail(STEAM_ERR_ARG, "steam_levy_field: bad dtype");
  STEAM_LAUNCH_CHECK("steam_levy_field");
  return STEAM_OK;
}

extern "C" size_t steam_flux_noise_workspace_bytes(void) {
  int nb = sm_count() * kNoiseBlocksPerSm;
  return carve_bytes((size_t)nb * 3, sizeof(double)) +
         carve_bytes(4, sizeof(double));
}

// Launches the noise kernel and its reduction: totals (device) receives
// { sum F over the window, sum |eps| over the window, nonzero eps count }.
static int flux_noise_launch(int dtype, const steam_region_t* region, double alpha,
                             double per_class_scale, double shift, int32_t n_zero,
                             int32_t zero_bottom, int32_t zero_top, const void* flux,
                             void* product, const steam_window_t* window, double* totals,
                             double* cells_out, void* workspace, size_t workspace_bytes,
                             cudaStream_t s, const char* who) {
  int rc = check_region(region, who);
  if (rc) return rc;
  STEAM_REQUIRE(alpha > 1.0 && alpha <= 2.0, std::string(who) + ": alpha must lie in (1, 2]");
  RegionDev r = to_dev(*region);
  const int64_t n = r.nx * r.ny * r.nz;
  NoiseArgs a;
  a.scale = per_class_scale;
  a.shift = shift;
  a.n_zero = n_zero;
  a.zero_bottom = zero_bottom;
  a.zero_top = zero_top;
  if (window) {
    STEAM_REQUIRE(window->x0 >= 0 && window->x1 <= r.nx &&
                      window->x0 <= window->x1 && window->y0 >= 0 &&
                      window->y1 <= r.ny && window->y0 <= window->y1,
                  std::string(who) + ": window outside the array");
    a.wx0 = window->x0;
    a.wx1 = window->x1;
    a.wy0 = window->y0;
    a.wy1 = window->y1;
  } else {
    a.wx0 = 0;
    a.wx1 = r.nx;
    a.wy0 = 0;
    a.wy1 = r.ny;
  }
  *cells_out = (double)((a.wx1 - a.wx0) * (a.wy1 - a.wy0) * r.nz);
  if (n == 0) return STEAM_OK;
  STEAM_REQUIRE(flux && product, std::string(who) + ": null field pointer");
  STEAM_REQUIRE(r.nx * r.ny < ((int64_t)1 << 32), std::string(who) + ": more than 2^32 columns");
  const int64_t cols_per_block = 256 / (r.nz < kNoiseZLanes ? r.nz : kNoiseZLanes);
  int grid = stride_grid((r.nx * r.ny + cols_per_block - 1) / cols_per_block, 1,
                         kNoiseBlocksPerSm);
  Carver c(workspace, workspace_bytes);
  double* partials = c.take<double>((size_t)grid * 3);
  if (!partials) return fail(STEAM_ERR_WORKSPACE, std::string(who) + ": workspace too small");
  if (dtype == STEAM_F32)
    flux_noise_kernel<float><<<grid, 256, 0, s>>>(
        r, make_levy<float>(alpha), a, (const float*)flux, (float*)product,
        partials);
  else if (dtype == STEAM_F64)
    flux_noise_kernel<double><<<grid, 256, 0, s>>>(
        r, make_levy<double>(alpha), a, (const double*)flux,
        (double*)product, partials);
  else
    return fail(STEAM_ERR_ARG, std::string(who) + ": bad dtype");
  STEAM_LAUNCH_CHECK(who);
  return reduce_partials(partials, grid, 3, totals, s);
}

extern "C" int steam_flux_noise(int dtype, const steam_region_t* region,
                                double alpha, double per_class_scale,
                                double shift, int32_t n_zero,
                                int32_t zero_bottom, int32_t zero_top,
                                const void* flux, void* product,
                                const steam_window_t* window, double* sums_out,
                                void* workspace, size_t workspace_bytes,
                                steam_stream_t stream) {
  STEAM_REQUIRE(sums_out != nullptr, "steam_flux_noise: null sums_out");
  STEAM_REQUIRE(region != nullptr, "steam_flux_noise: null region");
  cudaStream_t s = (cudaStream_t)stream;
  // totals go after the partials in the workspace
  const size_t part = carve_bytes((size_t)sm_count() * kNoiseBlocksPerSm * 3, sizeof(double));
  STEAM_REQUIRE(workspace_bytes >= part + carve_bytes(4, sizeof(double)) || workspace == nullptr,
                "steam_flux_noise: workspace too small");
  double* totals = workspace ? reinterpret_cast<double*>(static_cast<char*>(workspace) + part)
                             : nullptr;
  double cells = 0.0;
  int rc = flux_noise_launch(dtype, region, alpha, per_class_scale, shift, n_zero, zero_bottom,
                             zero_top, flux, product, window, totals, &cells, workspace, part,
                             s, "steam_flux_noise");
  if (rc) return rc;
  double h[3] = {0.0, 0.0, 0.0};
  if (region->shape[0] * region->shape[1] * region->shape[2] > 0) {
    STEAM_CUDA(cudaMemcpyAsync(h, totals, sizeof(h), cudaMemcpyDeviceToHost, s));
    STEAM_CUDA(cudaStreamSynchronize(s));
  }
  sums_out[0] = h[0];
  sums_out[1] = cells;
  sums_out[2] = h[1];
  sums_out[3] = h[2];
  return STEAM_OK;
}

extern "C" int steam_flux_noise_async(int dtype, const steam_region_t* region, double alpha,
                                      double per_class_scale, double shift, int32_t n_zero,
                                      int32_t zero_bottom, int32_t zero_top, const void* flux,
                                      void* product, const steam_window_t* window,
                                      double* sums_dev, void* workspace,
                                      size_t workspace_bytes, steam_stream_t stream) {
  STEAM_REQUIRE(sums_dev != nullptr, "steam_flux_noise_async: null sums_dev");
  STEAM_REQUIRE(region != nullptr, "steam_flux_noise_async: null region");
  cudaStream_t s = (cudaStream_t)stream;
  double cells = 0.0;
  if (region->shape[0] * region->shape[1] * region->shape[2] == 0)
    STEAM_CUDA(cudaMemsetAsync(sums_dev, 0, 3 * sizeof(double), s));
  return flux_noise_launch(dtype, region, alpha, per_class_scale, shift, n_zero, zero_bottom,
                           zero_top, flux, product, window, sums_dev, &cells, workspace,
                           workspace_bytes, s, "steam_flux_noise_async");
}
