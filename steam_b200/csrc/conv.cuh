// Shared definitions of the separable convolution (conv.cu) and its packed
// float32 fused kernel (conv_packed.cu).
#pragma once

#include "common.cuh"

namespace steam {

constexpr int kMaxTaps = 1536;
constexpr int kMaxZ = 8;
constexpr int kMaxPairs = 16;
constexpr int kMaxX = 4;

// The filters of a separable convolution as the host factored them, in
// float64 (each kernel rounds them to its arithmetic type).
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

// The input scaling of the second convolution, f' = f / mean(z) * C_k(z)
// (steam/simulate.py:1989-1992), as ONE multiply by C_k / mean formed in
// float64 and rounded to the field's type: within a unit in the last place
// of the two separately rounded operations, and a multiply instead of a
// division on every staged element.
template <typename T>
__device__ __forceinline__ T pre_scale(T div, T mul) {
  return (T)((double)mul / (double)div);
}

// The flux epilogue's window (sums of F over [wx0, wx1) x [wy0, wy1)).
struct XEpi {
  int mode;
  int64_t wx0, wx1, wy0, wy1;
};

// ---- the packed float32 fused kernel (conv_packed.cu) ----------------------
// Whether it runs this convolution: float32 fields, float32 arithmetic
// (STEAM_EPI_STORE or STEAM_EPI_FLUX), 13-tap filters even about their centre
// in z and y, at most 2 filters per axis and the pairs (0,0), (0,1), (1,0),
// (1,1); nz % 4 == 0, ny even; 16-byte aligned fields.
bool packed_supported(const SepParams<float>& p, int64_t nx, int64_t ny, int64_t nz,
                      const void* in, const void* out, int epilogue);
// CTAs of its launch for this shape (bounds the partial-sum workspace).
int64_t packed_grid(int64_t nx, int64_t ny, int64_t nz);
// Enqueues it; `partials` holds 2 * packed_grid doubles (the flux sums).
int packed_launch(const SepParams<float>& p, int64_t nx, int64_t ny, int64_t nz,
                  const float* in, float* out, const float* pre, int epilogue,
                  const XEpi& epi, double* partials, cudaStream_t s);

// Grouped launches of the packed kernel over many fields with the same
// filters (steam_conv_group_*).
size_t packed_group_bytes(int n, const steam_conv_problem_t* q);
int packed_group_prepare(const SepParams<float>& p, int n, const steam_conv_problem_t* q,
                         int epilogue, void* ws, size_t ws_bytes);
int packed_group_enqueue(void* ws, cudaStream_t s);
int packed_group_release(void* ws);

}  // namespace steam
