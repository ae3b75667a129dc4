// Shared device helpers for the STEAM B200 kernels: error plumbing, the
// Philox4x32-10 counter generator, the Chambers-Mallows-Stuck transform,
// deterministic block reductions and launch geometry.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <string>

#include "../../include/steam_b200.h"

namespace steam {

// ---------------------------------------------------------------------------
// Error plumbing: every C-ABI entry returns a status and records a message.
// ---------------------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

#define STEAM_CUDA(call)                                                       \
  do {                                                                         \
    cudaError_t err__ = (call);                                                \
    if (err__ != cudaSuccess)                                                  \
      return ::steam::fail(STEAM_ERR_CUDA,                                     \
                           std::string(#call) + ": " +                         \
                               cudaGetErrorString(err__));                     \
  } while (0)

// Counts every kernel this library enqueues (steam_launch_count()).
void count_launch();

#define STEAM_LAUNCH_CHECK(name)                                               \
  do {                                                                         \
    ::steam::count_launch();                                                   \
    cudaError_t err__ = cudaGetLastError();                                    \
    if (err__ != cudaSuccess)                                                  \
      return ::steam::fail(STEAM_ERR_CUDA, std::string(name) + " launch: " +   \
                                               cudaGetErrorString(err__));     \
  } while (0)

#define STEAM_REQUIRE(cond, msg)                                               \
  do {                                                                         \
    if (!(cond)) return ::steam::fail(STEAM_ERR_ARG, (msg));                   \
  } while (0)

// Number of SMs of the current device (cached per device).
int sm_count();
// Grid size for a grid-stride kernel over n items with `per_block` items per
// block-iteration: a multiple of the SM count, never more than needed.
int stride_grid(int64_t n, int per_block, int blocks_per_sm = 8);

// Workspace carving: bump allocator over the caller's workspace buffer.
struct Carver {
  char* base;
  size_t size;
  size_t used = 0;
  Carver(void* b, size_t s) : base(static_cast<char*>(b)), size(s) {}
  template <typename T>
  T* take(size_t count) {
    size_t off = (used + 255) & ~size_t(255);
    size_t bytes = count * sizeof(T);
    if (base == nullptr || off + bytes > size) return nullptr;
    used = off + bytes;
    return reinterpret_cast<T*>(base + off);
  }
};
inline size_t carve_bytes(size_t count, size_t elem) {
  return ((count * elem) + 255) & ~size_t(255);
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al. 2011), in the counter/key layout of the
// reference's world-keyed generator: counter (ix, iy, iz, key2), key
// (key0, key1).  Round 0 sees the raw 64-bit world indices of x and z, so an
// index outside [0, 2^32) (a negative z below a nest's ground) multiplies
// modulo 2^64 exactly as the reference's uint64 arithmetic does; every word
// is 32-bit from round 1 on.  The key schedule (key0 + r W0, key1 + r W1 for
// rounds r = 1..9) is the same at every site, so it is built once on the
// host and reaches the kernels as parameters.
// ---------------------------------------------------------------------------
struct PhiloxKey {
  uint32_t k0[10], k1[10];  // round keys; [0] is the raw key
  uint32_t k2;              // the counter's fourth word
};

__host__ __device__ inline PhiloxKey philox_key(uint32_t key0, uint32_t key1, uint32_t key2) {
  PhiloxKey k;
  uint32_t a = key0, b = key1;
  for (int r = 0; r < 10; ++r) {
    k.k0[r] = a;
    k.k1[r] = b;
    a += 0x9E3779B9u;
    b += 0xBB67AE85u;
  }
  k.k2 = key2;
  return k;
}

__device__ __forceinline__ void philox_site(int64_t ix, uint32_t iy, int64_t iz,
                                            const PhiloxKey& K, uint32_t& r0,
                                            uint32_t& r1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  uint32_t c0, c1, c2, c3;
  {
    unsigned long long p0 = (unsigned long long)M0 * (unsigned long long)ix;
    unsigned long long p1 = (unsigned long long)M1 * (unsigned long long)iz;
    c0 = (uint32_t)(p1 >> 32) ^ iy ^ K.k0[0];
    c1 = (uint32_t)p1;
    c2 = (uint32_t)(p0 >> 32) ^ K.k2 ^ K.k1[0];
    c3 = (uint32_t)p0;
  }
#pragma unroll
  for (int r = 1; r < 10; ++r) {
    // 32 x 32 -> 64-bit products: high and low words from one multiply
    const unsigned long long q0 = (unsigned long long)M0 * c0;
    const unsigned long long q1 = (unsigned long long)M1 * c2;
    const uint32_t n0 = (uint32_t)(q1 >> 32) ^ c1 ^ K.k0[r];
    const uint32_t n2 = (uint32_t)(q0 >> 32) ^ c3 ^ K.k1[r];
    c1 = (uint32_t)q1;
    c3 = (uint32_t)q0;
    c0 = n0;
    c2 = n2;
  }
  r0 = c0;
  r1 = c1;
}

// (r >> 8) * 2^-24: the float32 lattice of numpy's next_float.
__device__ __forceinline__ float lattice_uniform(uint32_t r) {
  return (float)(r >> 8) * (1.0f / 16777216.0f);
}

// ---------------------------------------------------------------------------
// Chambers-Mallows-Stuck extremal stable draw, in the operation order of the
// reference transform: phi=(u0-1/2)pi, R=-log(max(u1,eps)),
// fac=(max(cos phi,eps)|a-1|)^(-1/a), sh=a(phi-phi0),
// tail=(max(cos(phi-sh),eps)/R)^((1-a)/a), gamma=sin(sh)*sign*fac*tail.
// ---------------------------------------------------------------------------
template <typename T>
struct LevyParams {
  T alpha, phi0, sign, am1, fexp, texp, pi;
  double alpha_d, am1_d;  // alpha and alpha - 1 unrounded (float32 form)
};

template <typename T>
LevyParams<T> make_levy(double alpha) {
  LevyParams<T> p;
  const double PI = 3.14159265358979323846;
  p.alpha = (T)alpha;
  p.phi0 = (T)(-(PI / 2.0) * (1.0 - fabs(1.0 - alpha)) / alpha);
  p.sign = (T)(alpha > 1.0 ? 1.0 : -1.0);
  p.am1 = (T)fabs(alpha - 1.0);
  p.fexp = (T)(-1.0 / alpha);
  p.texp = (T)((1.0 - alpha) / alpha);
  p.pi = (T)PI;
  p.alpha_d = alpha;
  p.am1_d = fabs(alpha - 1.0);
  return p;
}

__device__ __forceinline__ float d_cos(float x) { return cosf(x); }
__device__ __forceinline__ double d_cos(double x) { return cos(x); }
__device__ __forceinline__ float d_sin(float x) { return sinf(x); }
__device__ __forceinline__ double d_sin(double x) { return sin(x); }
__device__ __forceinline__ float d_log(float x) { return logf(x); }
__device__ __forceinline__ double d_log(double x) { return log(x); }
__device__ __forceinline__ float d_pow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double d_pow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float d_exp(float x) { return expf(x); }
__device__ __forceinline__ double d_exp(double x) { return exp(x); }
__device__ __forceinline__ float d_expm1(float x) { return expm1f(x); }
__device__ __forceinline__ double d_expm1(double x) { return expm1(x); }
__device__ __forceinline__ float d_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double d_sqrt(double x) { return sqrt(x); }

// Four consecutive elements of a column, moved as 16-byte accesses (two for
// float64); the pointer is 16-byte aligned.
template <typename T>
struct V4 {
  T v[4];
};

template <typename T>
__device__ __forceinline__ V4<T> ld4(const T* p) {
  V4<T> r;
  if (sizeof(T) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    r.v[0] = (T)q.x; r.v[1] = (T)q.y; r.v[2] = (T)q.z; r.v[3] = (T)q.w;
  } else {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    r.v[0] = (T)a.x; r.v[1] = (T)a.y; r.v[2] = (T)b.x; r.v[3] = (T)b.y;
  }
  return r;
}

template <typename T>
__device__ __forceinline__ void st4(T* p, const V4<T>& r) {
  if (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4((float)r.v[0], (float)r.v[1],
                                                (float)r.v[2], (float)r.v[3]);
  } else {
    *reinterpret_cast<double2*>(p) = make_double2((double)r.v[0], (double)r.v[1]);
    *reinterpret_cast<double2*>(p + 2) = make_double2((double)r.v[2], (double)r.v[3]);
  }
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// one 4-byte element global -> shared through L1; src_bytes 0 writes a zero
// (the source is then not read)
__device__ __forceinline__ void cp_async4_zfill(void* sdst, const void* gsrc, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc),
               "r"(src_bytes)
               : "memory");
}

// Uncontracted arithmetic: the reference evaluates these products and sums as
// separate rounded operations, so they are kept out of FMA contraction.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ float d_sinpi(float x) { return sinpif(x); }
__device__ __forceinline__ double d_sinpi(double x) { return sinpi(x); }

// float32 form of the same draw with exact angle reduction.  With
// v = 1 - u0 (exact: u0 lies on the 2^-24 lattice) and alpha in (1, 2]:
//   cos(phi) = sin(pi v),  cos(phi - sh) = sin(pi (alpha-1) v),
//   sin(sh) = sin(pi alpha v),
// because phi = pi (1/2 - v) and sh = alpha (phi - phi0) = pi (1 - alpha v).
// The literal float32 evaluation loses most digits where the cosines near
// their zeros feed the negative powers (0.4-1.7 % relative L2 over the draws
// against float64); this form keeps every factor to a few float32 ulps.
// sin(pi r) for |r| <= 1/2 as r P(r^2), P the Taylor series of sin(pi r)/r
// through r^10 (the next term is below 2^-28 relative there): within 3
// float32 ulps, and relative accuracy is kept as r -> 0.
__device__ __forceinline__ float sinpi_half(float r) {
  const float s = r * r;
  float p = -7.370430945714348e-03f;     // -pi^11 / 11!
  p = fmaf(p, s, 8.214588661112823e-02f);  //  pi^9 / 9!
  p = fmaf(p, s, -5.992645293207921e-01f); // -pi^7 / 7!
  p = fmaf(p, s, 2.550164039877345e+00f);  //  pi^5 / 5!
  p = fmaf(p, s, -5.167712780049970e+00f); // -pi^3 / 3!
  p = fmaf(p, s, 3.141592653589793e+00f);  //  pi
  return r * p;
}

// sin(pi * a * v) with the product formed in float64 and reduced by its
// nearest integer n exactly, so the float32 sine sees an exact small argument:
// sin(pi a v) = (-1)^n sin(pi (a v - n)).
__device__ __forceinline__ float sinpi_scaled(double a, float v) {
  const double av = a * (double)v;
  const double n = rint(av);
  const float s = sinpi_half((float)(av - n));
  return ((long long)n & 1) ? -s : s;
}

// The two powers fac = x1^fexp and tail = x2^texp are taken together as one
// exp2 of fexp log2(x1) + texp log2(x2), with the hardware's approximate
// log2 (2^-22 absolute on [0.5, 2], 2 ulps elsewhere): the exponent carries
// those errors, so the product keeps a relative error of ~1e-7 |exponent|
// (measured: 1e-7 - 4e-7 relative L2 of the draws against float64), and one
// exp2 replaces two full pow evaluations.  R = -log(u1) keeps the accurate
// logarithm: near u1 = 1 it needs relative accuracy of a value near 0.
__device__ __forceinline__ float levy_draw_f32(float u0, float u1,
                                               const LevyParams<float>& p) {
  const float eps = 1e-6f;
  const float v = 1.0f - u0;
  const float R = -logf(u1 > eps ? u1 : eps);
  const float c = sinpi_half(v > 0.5f ? 1.0f - v : v);  // sin(pi v) = sin(pi (1 - v)), exact
  const float x1 = __fmul_rn(c > eps ? c : eps, p.am1);
  const float c2 = sinpi_scaled(p.am1_d, v);
  // the approximate quotient (2 ulps; R <= 14) only feeds the approximate log2
  const float x2 = __fdividef(c2 > eps ? c2 : eps, R);
  const float e = fmaf(p.fexp, __log2f(x1), p.texp * __log2f(x2));
  return __fmul_rn(__fmul_rn(sinpi_scaled(p.alpha_d, v), p.sign), exp2f(e));
}

template <typename T>
__device__ __forceinline__ T levy_draw(T u0, T u1, const LevyParams<T>& p) {
  const T eps = (T)1e-6;
  T phi = mul_rn(sub_rn(u0, (T)0.5), p.pi);
  T R = -d_log(u1 > eps ? u1 : eps);
  T c = d_cos(phi);
  T fac = d_pow(mul_rn(c > eps ? c : eps, p.am1), p.fexp);
  T sh = mul_rn(sub_rn(phi, p.phi0), p.alpha);
  T c2 = d_cos(sub_rn(phi, sh));
  T tail = d_pow((c2 > eps ? c2 : eps) / R, p.texp);
  return mul_rn(mul_rn(mul_rn(d_sin(sh), p.sign), fac), tail);
}

// ---------------------------------------------------------------------------
// Deterministic reductions: per-thread float64 accumulators, a fixed-shape
// block tree, per-block partials, and a final fixed-order pass.  The sum of
// the same data on the same device is therefore bit-identical run to run.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sums `v` over the block (blockDim.x a multiple of 32, <= 1024). Result valid
// in thread 0. `scratch` holds >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    r = lane < nw ? scratch[lane] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

// Sums partials[q * nblocks + b] over b for q < nq, in fixed order; writes
// out[q].  Launch with one block of 256 threads per q.
__global__ void reduce_partials_kernel(const double* __restrict__ partials,
                                       int nblocks, double* __restrict__ out);

int reduce_partials(const double* partials, int nblocks, int nq, double* out,
                    cudaStream_t stream);

}  // namespace steam
