// Error state, device geometry, deterministic partial reduction and the
// elementwise helpers shared by the entry points.
#include "common.cuh"

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
