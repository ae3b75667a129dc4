// Convolution of a field with a kernel that has no low-rank separable form
// (the Morlet turbulon, cos(w0 r) e^(-r^2/2 sigma^2), is radial but not a
// sum of a few products), with the reference's boundary semantics: x and y
// circular over the field's period, z linear with zero padding
// (steam/utils.py:293-427).
//
// Float32 fields: overlap-save FFT on 32^3 cubes, one cube per CTA pass.
// The CTA reads the cube's input segment (the output block plus the kernel's
// support, x and y wrapped modulo the period, z zero outside the field),
// transforms it in shared memory -- real-to-complex along z (two real columns
// packed as one complex line), then complex along y and along x, every
// 32-point line transform held in one thread's registers -- multiplies by
// the kernel's spectrum, transforms back and writes the (33 - k)^3 outputs
// whose circular sums do not wrap.  The forward transforms are decimation in
// frequency (natural order in, bit-reversed out) and the inverse ones
// decimation in time (bit-reversed in, natural out), and the spectrum is
// stored in the bit-reversed order, so no permutation pass is ever made.
// The second convolution's per-level input scaling is applied as the
// segment is read, and the flux epilogue (F = max(F + conv, 0), the sum of
// F over the window, the clip count) as the outputs are written.
//
// Float64 fields: direct summation over the kernel's support (the same
// prologue and epilogues), the precise reference path.
//
// The kernel spectrum (steam/utils.py:367-375: the kernel zero-padded and
// transformed) is built on the device by steam_conv_fft_spectrum, in float64
// from the float64 kernel, scaled by the inverse transform's 1/32^3 and the
// real-pair separation's 1/2, and rounded to float32 once.
#include "common.cuh"

#include <vector>

namespace steam {
namespace {

constexpr int kN = 32;            // transform length per axis
constexpr int kNK = kN / 2 + 1;   // z frequencies kept by the real transform
constexpr int kPad = kN + 1;      // padded y stride of the shared spectrum
constexpr int kFftThreads = kNK * kN;  // 544: one line per thread in the y and x passes
constexpr int kMaxK = 25;         // longest kernel axis (>= 8 outputs per cube axis)
constexpr size_t kFftSmem = (size_t)kNK * kN * kPad * sizeof(float2);

__host__ __device__ constexpr int brev5(int i) {
  return ((i & 1) << 4) | ((i & 2) << 2) | (i & 4) | ((i & 8) >> 2) | ((i & 16) >> 4);
}

// cos and sin of 2 pi t / 32, t < 16 (the twiddles of a 32-point transform)
__device__ __forceinline__ constexpr float tw_cos(int t) {
  constexpr float c[16] = {
      1.0f, 0.98078528040323043f, 0.92387953251128674f, 0.83146961230254524f,
      0.70710678118654757f, 0.55557023301960229f, 0.38268343236508984f,
      0.19509032201612833f, 0.0f, -0.19509032201612819f, -0.38268343236508973f,
      -0.55557023301960196f, -0.70710678118654746f, -0.83146961230254535f,
      -0.92387953251128674f, -0.98078528040323043f};
  return c[t];
}
__device__ __forceinline__ constexpr float tw_sin(int t) {
  constexpr float s[16] = {
      0.0f, 0.19509032201612825f, 0.38268343236508978f, 0.55557023301960218f,
      0.70710678118654746f, 0.83146961230254524f, 0.92387953251128674f,
      0.98078528040323043f, 1.0f, 0.98078528040323043f, 0.92387953251128674f,
      0.83146961230254546f, 0.70710678118654757f, 0.55557023301960218f,
      0.38268343236508989f, 0.19509032201612861f};
  return s[t];
}

// d * exp(SIGN * 2 pi i t / 32)
template <int SIGN>
__device__ __forceinline__ float2 twiddle(float2 d, int t) {
  if (t == 0) return d;
  if (t == 8) return SIGN > 0 ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
  const float c = tw_cos(t), s = SIGN > 0 ? tw_sin(t) : -tw_sin(t);
  return make_float2(fmaf(c, d.x, -s * d.y), fmaf(c, d.y, s * d.x));
}

// Forward (SIGN = -1) or inverse (+1) 32-point transform, unnormalised,
// decimation in frequency: natural order in, v[j] = X[brev5(j)] out.
template <int SIGN>
__device__ __forceinline__ void fft_dif(float2 (&v)[kN]) {
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int half = 16 >> s;
#pragma unroll
    for (int g = 0; g < kN; g += 2 * half) {
#pragma unroll
      for (int j = 0; j < half; ++j) {
        const float2 a = v[g + j], b = v[g + j + half];
        v[g + j] = make_float2(a.x + b.x, a.y + b.y);
        v[g + j + half] = twiddle<SIGN>(make_float2(a.x - b.x, a.y - b.y), j << s);
      }
    }
  }
}

// Decimation in time: v[j] = X[brev5(j)] in, natural order out.
template <int SIGN>
__device__ __forceinline__ void fft_dit(float2 (&v)[kN]) {
#pragma unroll
  for (int s = 4; s >= 0; --s) {
    const int half = 16 >> s;
#pragma unroll
    for (int g = 0; g < kN; g += 2 * half) {
#pragma unroll
      for (int j = 0; j < half; ++j) {
        const float2 a = v[g + j];
        const float2 b = twiddle<SIGN>(v[g + j + half], j << s);
        v[g + j] = make_float2(a.x + b.x, a.y + b.y);
        v[g + j + half] = make_float2(a.x - b.x, a.y - b.y);
      }
    }
  }
}

__device__ __forceinline__ int sidx(int k, int x, int y) { return (k * kN + x) * kPad + y; }

__device__ __forceinline__ int64_t wrap64(int64_t v, int64_t n) {
  const int64_t r = v % n;
  return r < 0 ? r + n : r;
}

struct FftGeom {
  int64_t nx, ny;
  int nz;
  int kx, ky, kz;
  int ox, oy, oz;        // k - 1 - c per axis: the segment starts this far before the block
  int bx, by, bz;        // outputs per cube and axis (bz a multiple of 4 when vec4 stores)
  int64_t nbx, nby, nbz;  // cubes per axis
  int use_pre;
  int vec_load;          // float2 segment loads (segment start and nz even)
  int vec_store;         // float4 output stores (bz, nz multiples of 4)
  int mode;              // STEAM_EPI_STORE or STEAM_EPI_FLUX
  int64_t wx0, wx1, wy0, wy1;
};

// The second convolution's scaling f * (C_k / mean) formed in float64 and
// rounded once (the separable path's rule).
__device__ __forceinline__ float level_scale(const float* pre, int nz, int z) {
  return (float)((double)pre[nz + z] / (double)pre[z]);
}

__global__ void __launch_bounds__(kFftThreads, 1)
fft_conv_kernel(const float* __restrict__ in, float* __restrict__ out,
                const float* __restrict__ pre, const float2* __restrict__ spec, FftGeom g,
                double* __restrict__ partials) {
  extern __shared__ float2 S[];
  __shared__ double scratch[32];
  const int t = threadIdx.x;
  const int64_t ncubes = g.nbx * g.nby * g.nbz;
  double s_f = 0.0, s_clip = 0.0;
  for (int64_t cube = blockIdx.x; cube < ncubes; cube += gridDim.x) {
    const int64_t cz = cube % g.nbz;
    const int64_t cxy = cube / g.nbz;
    const int64_t cy = cxy % g.nby;
    const int64_t cx = cxy / g.nby;
    const int64_t X0 = cx * g.bx, Y0 = cy * g.by;
    const int Z0 = (int)(cz * g.bz);
    const int zs = Z0 - g.oz;  // first z of the input segment
    // ---- A: read the segment, z transform (two real columns per line) ----
    if (t < kN * kN / 2) {
      const int x = t >> 4, ya = t & 15, yb = ya + 16;
      const int64_t gx = wrap64(X0 - g.ox + x, g.nx);
      const float* ca = in + (gx * g.ny + wrap64(Y0 - g.oy + ya, g.ny)) * g.nz;
      const float* cb = in + (gx * g.ny + wrap64(Y0 - g.oy + yb, g.ny)) * g.nz;
      float2 v[kN];
      if (g.vec_load) {
#pragma unroll
        for (int m = 0; m < kN; m += 2) {
          const int z = zs + m;
          float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
          if (z >= 0 && z < g.nz) {
            a = *reinterpret_cast<const float2*>(ca + z);
            b = *reinterpret_cast<const float2*>(cb + z);
          }
          v[m] = make_float2(a.x, b.x);
          v[m + 1] = make_float2(a.y, b.y);
        }
      } else {
#pragma unroll
        for (int m = 0; m < kN; ++m) {
          const int z = zs + m;
          v[m] = (z >= 0 && z < g.nz) ? make_float2(ca[z], cb[z]) : make_float2(0.f, 0.f);
        }
      }
      if (g.use_pre) {
#pragma unroll
        for (int m = 0; m < kN; ++m) {
          const int z = zs + m;
          if (z >= 0 && z < g.nz) {
            const float sc = level_scale(pre, g.nz, z);
            v[m].x *= sc;
            v[m].y *= sc;
          }
        }
      }
      fft_dif<-1>(v);
      // C = A + iB with A, B the spectra of the two real columns:
      // 2A[k] = C[k] + conj(C[32-k]), 2B[k] = -i (C[k] - conj(C[32-k]))
      // (the 1/2 is in the kernel spectrum)
#pragma unroll
      for (int k = 0; k < kNK; ++k) {
        const float2 p = v[brev5(k)];
        const float2 r = v[brev5((kN - k) & (kN - 1))];
        S[sidx(k, x, ya)] = make_float2(p.x + r.x, p.y - r.y);
        S[sidx(k, x, yb)] = make_float2(p.y + r.y, r.x - p.x);
      }
    }
    __syncthreads();
    // ---- B: y transform, line (k, x) per thread ----
    {
      const int k = t >> 5, x = t & 31;
      float2 v[kN];
#pragma unroll
      for (int y = 0; y < kN; ++y) v[y] = S[sidx(k, x, y)];
      fft_dif<-1>(v);
#pragma unroll
      for (int y = 0; y < kN; ++y) S[sidx(k, x, y)] = v[y];
    }
    __syncthreads();
    // ---- C: x transform, spectrum product, inverse x transform ----
    {
      const int k = t >> 5, j = t & 31;  // j: y frequency brev5(j)
      float2 v[kN];
#pragma unroll
      for (int x = 0; x < kN; ++x) v[x] = S[sidx(k, x, j)];
      fft_dif<-1>(v);
      const float2* sp = spec + (size_t)k * kN * kN + j;
#pragma unroll
      for (int i = 0; i < kN; ++i) {
        const float2 h = __ldg(sp + i * kN);
        const float2 a = v[i];
        v[i] = make_float2(fmaf(a.x, h.x, -a.y * h.y), fmaf(a.x, h.y, a.y * h.x));
      }
      fft_dit<1>(v);
#pragma unroll
      for (int x = 0; x < kN; ++x)
        if (x >= g.kx - 1) S[sidx(k, x, j)] = v[x];
    }
    __syncthreads();
    // ---- D: inverse y transform of the lines whose x survives ----
    if (t < kNK * g.bx) {
      const int k = t / g.bx, x = g.kx - 1 + t % g.bx;
      float2 v[kN];
#pragma unroll
      for (int j = 0; j < kN; ++j) v[j] = S[sidx(k, x, j)];
      fft_dit<1>(v);
#pragma unroll
      for (int y = 0; y < kN; ++y)
        if (y >= g.ky - 1) S[sidx(k, x, y)] = v[y];
    }
    __syncthreads();
    // ---- E: inverse z transform of the surviving columns, in pairs ----
    {
      const int ncol = g.bx * g.by;
      const int half = (ncol + 1) >> 1;
      if (t < half) {
        const int c0 = t, c1 = t + half;
        const bool two = c1 < ncol;
        const int xa = g.kx - 1 + c0 / g.by, ya = g.ky - 1 + c0 % g.by;
        const int xb = two ? g.kx - 1 + c1 / g.by : xa, yb = two ? g.ky - 1 + c1 % g.by : ya;
        float2 v[kN];
#pragma unroll
        for (int k = 0; k < kNK; ++k) {
          const float2 A = S[sidx(k, xa, ya)];
          const float2 B = two ? S[sidx(k, xb, yb)] : make_float2(0.f, 0.f);
          // C[k] = A + iB and C[32 - k] = conj(A) + i conj(B); the terms
          // at k = 0 and 16 are real for real columns (a complex-to-real
          // transform takes their real parts)
          if (k == 0 || k == kN / 2) {
            v[brev5(k)] = make_float2(A.x, B.x);
          } else {
            v[brev5(k)] = make_float2(A.x - B.y, A.y + B.x);
            v[brev5(kN - k)] = make_float2(A.x + B.y, B.x - A.y);
          }
        }
        fft_dit<1>(v);
#pragma unroll
        for (int col = 0; col < 2; ++col) {
          if (col == 1 && !two) break;
          const int64_t ox = X0 + (col ? xb : xa) - (g.kx - 1);
          const int64_t oy = Y0 + (col ? yb : ya) - (g.ky - 1);
          if (ox >= g.nx || oy >= g.ny) continue;
          const bool inwin = ox >= g.wx0 && ox < g.wx1 && oy >= g.wy0 && oy < g.wy1;
          float* o = out + (ox * g.ny + oy) * g.nz;
          if (g.vec_store) {
#pragma unroll
            for (int m0 = 0; m0 < kN; m0 += 4) {
              // outputs m0..m0+3 map to z = Z0 + m - (kz - 1): Z0, kz - 1
              // and bz are multiples of 4, so a group is wholly kept or not,
              // and wholly inside nz (a multiple of 4) or not
              if (m0 < g.kz - 1 || m0 >= g.kz - 1 + g.bz) continue;
              const int z = Z0 + m0 - (g.kz - 1);
              if (z >= g.nz) continue;
              float4 c = make_float4(col ? v[m0].y : v[m0].x, col ? v[m0 + 1].y : v[m0 + 1].x,
                                     col ? v[m0 + 2].y : v[m0 + 2].x,
                                     col ? v[m0 + 3].y : v[m0 + 3].x);
              float4* dst = reinterpret_cast<float4*>(o + z);
              if (g.mode == STEAM_EPI_FLUX) {
                const float4 f = *dst;
                float r[4] = {(float)((double)f.x + (double)c.x), (float)((double)f.y + (double)c.y),
                              (float)((double)f.z + (double)c.z), (float)((double)f.w + (double)c.w)};
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                  if (r[q] < 0.f) {
                    s_clip += 1.0;
                    r[q] = 0.f;
                  }
                  if (inwin) s_f += (double)r[q];
                }
                c = make_float4(r[0], r[1], r[2], r[3]);
              }
              *dst = c;
            }
          } else {
#pragma unroll
            for (int m = 0; m < kN; ++m) {
              if (m < g.kz - 1) continue;
              const int z = Z0 + m - (g.kz - 1);
              if (z >= g.nz || m - (g.kz - 1) >= g.bz) continue;
              float c = col ? v[m].y : v[m].x;
              if (g.mode == STEAM_EPI_FLUX) {
                c = (float)((double)o[z] + (double)c);
                if (c < 0.f) {
                  s_clip += 1.0;
                  c = 0.f;
                }
                if (inwin) s_f += (double)c;
              }
              o[z] = c;
            }
          }
        }
      }
    }
    __syncthreads();
  }
  if (g.mode == STEAM_EPI_FLUX) {
    const double t0 = block_sum(s_f, scratch);
    const double t1 = block_sum(s_clip, scratch);
    if (t == 0) {
      partials[blockIdx.x] = t0;
      partials[gridDim.x + blockIdx.x] = t1;
    }
  }
}

// The kernel spectrum: one block per z frequency k.  kern (float64, C order
// (x, y, z)) zero-padded to 32^3; spec[k][i][j] = scale * K^(fx = brev5(i),
// fy = brev5(j), k) with every sum in float64.
__global__ void __launch_bounds__(256)
fft_spectrum_kernel(const double* __restrict__ kern, int kx, int ky, int kz, double scale,
                    float2* __restrict__ spec) {
  __shared__ double2 t1[kMaxK * kMaxK];  // sum over z, per (x, y)
  __shared__ double2 t2[kMaxK * kN];     // then over y, per (x, fy)
  const int k = blockIdx.x;
  for (int i = threadIdx.x; i < kx * ky; i += blockDim.x) {
    const double* col = kern + (size_t)i * kz;
    double re = 0.0, im = 0.0;
    for (int z = 0; z < kz; ++z) {
      double s, c;
      sincospi(2.0 * (double)((k * z) & (kN - 1)) / kN, &s, &c);
      re += col[z] * c;
      im -= col[z] * s;
    }
    t1[i] = make_double2(re, im);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kx * kN; i += blockDim.x) {
    const int x = i / kN, fy = i % kN;
    double re = 0.0, im = 0.0;
    for (int y = 0; y < ky; ++y) {
      double s, c;
      sincospi(2.0 * (double)((fy * y) & (kN - 1)) / kN, &s, &c);
      const double2 a = t1[x * ky + y];
      re += a.x * c + a.y * s;
      im += a.y * c - a.x * s;
    }
    t2[i] = make_double2(re, im);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kN * kN; i += blockDim.x) {
    const int fx = i / kN, fy = i % kN;
    double re = 0.0, im = 0.0;
    for (int x = 0; x < kx; ++x) {
      double s, c;
      sincospi(2.0 * (double)((fx * x) & (kN - 1)) / kN, &s, &c);
      const double2 a = t2[x * kN + fy];
      re += a.x * c + a.y * s;
      im += a.y * c - a.x * s;
    }
    spec[((size_t)k * kN + brev5(fx)) * kN + brev5(fy)] =
        make_float2((float)(re * scale), (float)(im * scale));
  }
}

// ---- direct summation (float64 fields, or a kernel longer than 25 taps) ----
template <typename T>
__global__ void __launch_bounds__(256)
direct_conv_kernel(const T* __restrict__ in, int64_t nx, int64_t ny, int nz,
                   const T* __restrict__ K, int kx, int ky, int kz, int cx, int cy, int cz,
                   const T* __restrict__ pre, int mode, int64_t wx0, int64_t wx1, int64_t wy0,
                   int64_t wy1, T* __restrict__ out, double* __restrict__ partials) {
  __shared__ double scratch[32];
  const int64_t n = nx * ny * (int64_t)nz;
  double s_f = 0.0, s_clip = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int z = (int)(i % nz);
    const int64_t col = i / nz;
    const int64_t y = col % ny;
    const int64_t x = col / ny;
    double acc = 0.0;
    for (int a = 0; a < kx; ++a) {
      const int64_t xs = wrap64(x - a + cx, nx);
      for (int b = 0; b < ky; ++b) {
        const int64_t ys = wrap64(y - b + cy, ny);
        const T* src = in + (xs * ny + ys) * nz;
        const T* kk = K + ((int64_t)a * ky + b) * kz;
        for (int c = 0; c < kz; ++c) {
          const int zs = z - c + cz;
          if (zs < 0 || zs >= nz) continue;
          T v = src[zs];
          if (pre) v = (T)(v * (T)((double)pre[nz + zs] / (double)pre[zs]));
          acc += (double)kk[c] * (double)v;
        }
      }
    }
    if (mode == STEAM_EPI_FLUX) {
      T f = (T)((double)out[i] + acc);
      if (f < (T)0) {
        s_clip += 1.0;
        f = (T)0;
      }
      out[i] = f;
      if (x >= wx0 && x < wx1 && y >= wy0 && y < wy1) s_f += (double)f;
    } else {
      out[i] = (T)acc;
    }
  }
  if (mode == STEAM_EPI_FLUX) {
    const double t0 = block_sum(s_f, scratch);
    const double t1 = block_sum(s_clip, scratch);
    if (threadIdx.x == 0) {
      partials[blockIdx.x] = t0;
      partials[gridDim.x + blockIdx.x] = t1;
    }
  }
}

int fft_grid(int64_t ncubes) {
  const int sms = sm_count();
  return (int)(ncubes < sms ? ncubes : sms);
}

FftGeom fft_geom(int64_t nx, int64_t ny, int64_t nz, int kx, int ky, int kz, int cx, int cy,
                 int epilogue, const steam_window_t* w, bool in_aligned8, bool out_aligned16) {
  FftGeom g;
  g.nx = nx;
  g.ny = ny;
  g.nz = (int)nz;
  g.kx = kx;
  g.ky = ky;
  g.kz = kz;
  const int czc = (kz - 1) / 2;
  g.ox = kx - 1 - cx;
  g.oy = ky - 1 - cy;
  g.oz = kz - 1 - czc;
  g.bx = kN - kx + 1;
  g.by = kN - ky + 1;
  g.bz = kN - kz + 1;
  // float4 stores need every block's first output z on a multiple of 4 (so
  // bz rounded down to one) and the first kept transform output (kz - 1)
  // on one as well
  g.vec_store = out_aligned16 && (nz % 4 == 0) && ((kz - 1) % 4 == 0) && (g.bz >= 4);
  if (g.vec_store) g.bz &= ~3;
  // float2 loads need every segment start Z0 - oz even: bz and oz even
  g.vec_load = in_aligned8 && (nz % 2 == 0) && (g.oz % 2 == 0) && (g.bz % 2 == 0);
  g.nbx = (nx + g.bx - 1) / g.bx;
  g.nby = (ny + g.by - 1) / g.by;
  g.nbz = (nz + g.bz - 1) / g.bz;
  g.use_pre = 0;
  g.mode = epilogue;
  g.wx0 = w ? w->x0 : 0;
  g.wx1 = w ? w->x1 : nx;
  g.wy0 = w ? w->y0 : 0;
  g.wy1 = w ? w->y1 : ny;
  return g;
}

int check_common(const char* fn, int64_t nx, int64_t ny, int64_t nz, int kx, int ky, int kz,
                 int cx, int cy, int epilogue, const steam_window_t* w) {
  const std::string f(fn);
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, f + ": negative extent");
  STEAM_REQUIRE(kx >= 1 && ky >= 1 && kz >= 1, f + ": kernel extents must be >= 1");
  STEAM_REQUIRE(cx >= 0 && cx < kx && cy >= 0 && cy < ky, f + ": centre outside the kernel");
  STEAM_REQUIRE(epilogue == STEAM_EPI_STORE || epilogue == STEAM_EPI_FLUX ||
                    epilogue == STEAM_EPI_STORE_WIDE,
                f + ": unknown epilogue");
  STEAM_REQUIRE(nz < ((int64_t)1 << 31), f + ": nz above 2^31");
  if (w)
    STEAM_REQUIRE(w->x0 >= 0 && w->x1 <= nx && w->x0 <= w->x1 && w->y0 >= 0 && w->y1 <= ny &&
                      w->y0 <= w->y1,
                  f + ": window outside the array");
  return STEAM_OK;
}

// Ordered reduction of the flux partials into totals (device), and the host
// copy for the synchronous forms.
int finish_sums(double* partials, int grid, double* totals, double* sums_out, int64_t cells,
                cudaStream_t s) {
  int rc = reduce_partials(partials, grid, 2, totals, s);
  if (rc || !sums_out) return rc;
  double h[2];
  STEAM_CUDA(cudaMemcpyAsync(h, totals, sizeof(h), cudaMemcpyDeviceToHost, s));
  STEAM_CUDA(cudaStreamSynchronize(s));
  sums_out[0] = h[0];
  sums_out[1] = (double)cells;
  sums_out[2] = h[1];
  return STEAM_OK;
}

int64_t win_cells(const steam_window_t* w, int64_t nx, int64_t ny) {
  return w ? (w->x1 - w->x0) * (w->y1 - w->y0) : nx * ny;
}

// pre (HOST div/mul per level, either may be NULL) -> a device [2][nz] vector
template <typename T>
int upload_pre(const double* pre_div, const double* pre_mul, int64_t nz, T* dst,
               cudaStream_t s) {
  std::vector<T> h(2 * nz);
  for (int64_t z = 0; z < nz; ++z) {
    h[z] = pre_div ? (T)pre_div[z] : (T)1;
    h[nz + z] = pre_mul ? (T)pre_mul[z] : (T)1;
  }
  STEAM_CUDA(cudaMemcpyAsync(dst, h.data(), sizeof(T) * 2 * nz, cudaMemcpyHostToDevice, s));
  // the host vector dies with this frame: the copy must have read it
  STEAM_CUDA(cudaStreamSynchronize(s));
  return STEAM_OK;
}

int run_fft(int64_t nx, int64_t ny, int64_t nz, int kx, int ky, int kz, int cx, int cy,
            const void* spectrum, const void* in, const float* pre_dev, const double* pre_div,
            const double* pre_mul, void* out, int epilogue, const steam_window_t* w,
            double* sums_dev, double* sums_out, void* ws, size_t ws_bytes, cudaStream_t s) {
  STEAM_REQUIRE(kx <= kMaxK && ky <= kMaxK && kz <= kMaxK,
                "steam_conv_fft: kernel longer than 25 taps on an axis");
  STEAM_REQUIRE(spectrum && in && out, "steam_conv_fft: null pointer");
  FftGeom g = fft_geom(nx, ny, nz, kx, ky, kz, cx, cy, epilogue, w, (uintptr_t)in % 8 == 0,
                       (uintptr_t)out % 16 == 0);
  const int64_t ncubes = g.nbx * g.nby * g.nbz;
  const int grid = fft_grid(ncubes);
  Carver c(ws, ws_bytes);
  float* pre = nullptr;
  const bool use_pre = pre_dev || pre_div || pre_mul;
  if (use_pre && !pre_dev) pre = c.take<float>((size_t)2 * nz);
  double* partials = c.take<double>((size_t)2 * grid);
  double* totals = c.take<double>(2);
  if ((use_pre && !pre_dev && !pre) || !partials || !totals)
    return fail(STEAM_ERR_WORKSPACE, "steam_conv_fft: workspace too small");
  if (pre_dev) pre = const_cast<float*>(pre_dev);
  else if (use_pre) {
    int rc = upload_pre<float>(pre_div, pre_mul, nz, pre, s);
    if (rc) return rc;
  }
  g.use_pre = use_pre ? 1 : 0;
  STEAM_CUDA(cudaFuncSetAttribute(fft_conv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kFftSmem));
  fft_conv_kernel<<<grid, kFftThreads, kFftSmem, s>>>(
      (const float*)in, (float*)out, pre, (const float2*)spectrum, g, partials);
  STEAM_LAUNCH_CHECK("steam_conv_fft");
  if (epilogue == STEAM_EPI_FLUX)
    return finish_sums(partials, grid, sums_dev ? sums_dev : totals, sums_out,
                       win_cells(w, nx, ny) * nz, s);
  return STEAM_OK;
}

int direct_grid(int64_t n) { return stride_grid(n, 256, 4); }

template <typename T>
int run_direct(int64_t nx, int64_t ny, int64_t nz, const void* kernel, int kx, int ky, int kz,
               int cx, int cy, const void* in, const T* pre_dev, const double* pre_div,
               const double* pre_mul, void* out, int epilogue, const steam_window_t* w,
               double* sums_dev, double* sums_out, void* ws, size_t ws_bytes, cudaStream_t s) {
  STEAM_REQUIRE(kernel && in && out, "steam_conv_direct: null pointer");
  const int64_t n = nx * ny * nz;
  const int grid = direct_grid(n);
  Carver c(ws, ws_bytes);
  T* pre = nullptr;
  const bool use_pre = pre_dev || pre_div || pre_mul;
  if (use_pre && !pre_dev) pre = c.take<T>((size_t)2 * nz);
  double* partials = c.take<double>((size_t)2 * grid);
  double* totals = c.take<double>(2);
  if ((use_pre && !pre_dev && !pre) || !partials || !totals)
    return fail(STEAM_ERR_WORKSPACE, "steam_conv_direct: workspace too small");
  if (pre_dev) pre = const_cast<T*>(pre_dev);
  else if (use_pre) {
    int rc = upload_pre<T>(pre_div, pre_mul, nz, pre, s);
    if (rc) return rc;
  }
  direct_conv_kernel<T><<<grid, 256, 0, s>>>(
      (const T*)in, nx, ny, (int)nz, (const T*)kernel, kx, ky, kz, cx, cy, (kz - 1) / 2,
      use_pre ? pre : nullptr, epilogue, w ? w->x0 : 0, w ? w->x1 : nx, w ? w->y0 : 0,
      w ? w->y1 : ny, (T*)out, partials);
  STEAM_LAUNCH_CHECK("steam_conv_direct");
  if (epilogue == STEAM_EPI_FLUX)
    return finish_sums(partials, grid, sums_dev ? sums_dev : totals, sums_out,
                       win_cells(w, nx, ny) * nz, s);
  return STEAM_OK;
}

size_t fft_ws_bytes(int64_t nz) {
  const int grid = sm_count();
  return carve_bytes((size_t)2 * nz, sizeof(double)) +
         carve_bytes((size_t)2 * grid, sizeof(double)) + carve_bytes(2, sizeof(double));
}

size_t direct_ws_bytes(int64_t nx, int64_t ny, int64_t nz) {
  const int grid = direct_grid(nx * ny * nz);
  return carve_bytes((size_t)2 * nz, sizeof(double)) +
         carve_bytes((size_t)2 * grid, sizeof(double)) + carve_bytes(2, sizeof(double));
}

}  // namespace
}  // namespace steam

using namespace steam;

extern "C" size_t steam_conv_fft_spectrum_bytes(void) {
  return (size_t)kNK * kN * kN * sizeof(float2);
}

extern "C" int steam_conv_fft_spectrum(const double* kernel_dev, int32_t kx, int32_t ky,
                                       int32_t kz, void* spectrum_dev, steam_stream_t stream) {
  STEAM_REQUIRE(kx >= 1 && ky >= 1 && kz >= 1 && kx <= kMaxK && ky <= kMaxK && kz <= kMaxK,
                "steam_conv_fft_spectrum: kernel extents must be in [1, 25]");
  STEAM_REQUIRE(kernel_dev && spectrum_dev, "steam_conv_fft_spectrum: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  const double scale = 0.5 / ((double)kN * kN * kN);
  fft_spectrum_kernel<<<kNK, 256, 0, s>>>(kernel_dev, kx, ky, kz, scale, (float2*)spectrum_dev);
  STEAM_LAUNCH_CHECK("steam_conv_fft_spectrum");
  return STEAM_OK;
}

extern "C" size_t steam_conv_fft_workspace_bytes(int64_t nx, int64_t ny, int64_t nz) {
  (void)nx;
  (void)ny;
  return fft_ws_bytes(nz);
}

extern "C" int steam_conv_fft(int64_t nx, int64_t ny, int64_t nz, int32_t kx, int32_t ky,
                              int32_t kz, int32_t cx, int32_t cy, const void* spectrum_dev,
                              const void* in, const double* pre_div, const double* pre_mul,
                              void* out, int32_t epilogue, const steam_window_t* window,
                              double* sums_out, void* workspace, size_t workspace_bytes,
                              steam_stream_t stream) {
  int rc = check_common("steam_conv_fft", nx, ny, nz, kx, ky, kz, cx, cy, epilogue, window);
  if (rc) return rc;
  STEAM_REQUIRE(epilogue != STEAM_EPI_FLUX || sums_out, "steam_conv_fft: flux epilogue needs sums_out");
  if (nx * ny * nz == 0) {
    if (epilogue == STEAM_EPI_FLUX) sums_out[0] = sums_out[1] = sums_out[2] = 0.0;
    return STEAM_OK;
  }
  return run_fft(nx, ny, nz, kx, ky, kz, cx, cy, spectrum_dev, in, nullptr, pre_div, pre_mul,
                 out, epilogue, window, nullptr, sums_out, workspace, workspace_bytes,
                 (cudaStream_t)stream);
}

extern "C" int steam_conv_fft_async(int64_t nx, int64_t ny, int64_t nz, int32_t kx, int32_t ky,
                                    int32_t kz, int32_t cx, int32_t cy,
                                    const void* spectrum_dev, const void* in,
                                    const void* pre_dev, void* out, int32_t epilogue,
                                    const steam_window_t* window, double* sums_dev,
                                    void* workspace, size_t workspace_bytes,
                                    steam_stream_t stream) {
  int rc = check_common("steam_conv_fft_async", nx, ny, nz, kx, ky, kz, cx, cy, epilogue, window);
  if (rc) return rc;
  STEAM_REQUIRE(epilogue != STEAM_EPI_FLUX || sums_dev,
                "steam_conv_fft_async: flux epilogue needs sums_dev");
  cudaStream_t s = (cudaStream_t)stream;
  if (nx * ny * nz == 0) {
    if (epilogue == STEAM_EPI_FLUX) STEAM_CUDA(cudaMemsetAsync(sums_dev, 0, 2 * sizeof(double), s));
    return STEAM_OK;
  }
  return run_fft(nx, ny, nz, kx, ky, kz, cx, cy, spectrum_dev, in, (const float*)pre_dev,
                 nullptr, nullptr, out, epilogue, window, sums_dev, nullptr, workspace,
                 workspace_bytes, s);
}

extern "C" size_t steam_conv_direct_workspace_bytes(int64_t nx, int64_t ny, int64_t nz) {
  return direct_ws_bytes(nx, ny, nz);
}

extern "C" int steam_conv_direct(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                 const void* kernel_dev, int32_t kx, int32_t ky, int32_t kz,
                                 int32_t cx, int32_t cy, const void* in, const double* pre_div,
                                 const double* pre_mul, void* out, int32_t epilogue,
                                 const steam_window_t* window, double* sums_out,
                                 void* workspace, size_t workspace_bytes,
                                 steam_stream_t stream) {
  int rc = check_common("steam_conv_direct", nx, ny, nz, kx, ky, kz, cx, cy, epilogue, window);
  if (rc) return rc;
  STEAM_REQUIRE(epilogue != STEAM_EPI_FLUX || sums_out,
                "steam_conv_direct: flux epilogue needs sums_out");
  if (nx * ny * nz == 0) {
    if (epilogue == STEAM_EPI_FLUX) sums_out[0] = sums_out[1] = sums_out[2] = 0.0;
    return STEAM_OK;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    return run_direct<float>(nx, ny, nz, kernel_dev, kx, ky, kz, cx, cy, in, nullptr, pre_div,
                             pre_mul, out, epilogue, window, nullptr, sums_out, workspace,
                             workspace_bytes, s);
  if (dtype == STEAM_F64)
    return run_direct<double>(nx, ny, nz, kernel_dev, kx, ky, kz, cx, cy, in, nullptr, pre_div,
                              pre_mul, out, epilogue, window, nullptr, sums_out, workspace,
                              workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_conv_direct: bad dtype");
}

extern "C" int steam_conv_direct_async(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                       const void* kernel_dev, int32_t kx, int32_t ky,
                                       int32_t kz, int32_t cx, int32_t cy, const void* in,
                                       const void* pre_dev, void* out, int32_t epilogue,
                                       const steam_window_t* window, double* sums_dev,
                                       void* workspace, size_t workspace_bytes,
                                       steam_stream_t stream) {
  int rc = check_common("steam_conv_direct_async", nx, ny, nz, kx, ky, kz, cx, cy, epilogue,
                        window);
  if (rc) return rc;
  STEAM_REQUIRE(epilogue != STEAM_EPI_FLUX || sums_dev,
                "steam_conv_direct_async: flux epilogue needs sums_dev");
  cudaStream_t s = (cudaStream_t)stream;
  if (nx * ny * nz == 0) {
    if (epilogue == STEAM_EPI_FLUX) STEAM_CUDA(cudaMemsetAsync(sums_dev, 0, 2 * sizeof(double), s));
    return STEAM_OK;
  }
  if (dtype == STEAM_F32)
    return run_direct<float>(nx, ny, nz, kernel_dev, kx, ky, kz, cx, cy, in,
                             (const float*)pre_dev, nullptr, nullptr, out, epilogue, window,
                             sums_dev, nullptr, workspace, workspace_bytes, s);
  if (dtype == STEAM_F64)
    return run_direct<double>(nx, ny, nz, kernel_dev, kx, ky, kz, cx, cy, in,
                              (const double*)pre_dev, nullptr, nullptr, out, epilogue, window,
                              sums_dev, nullptr, workspace, workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_conv_direct_async: bad dtype");
}
