// Per-level work on the z-fastest layout: level sums, the scalar pattern
// (advective weight x signed amplitude x bound taper), the bounded
// amplitude-preserving add and the mean-preserving projection.
//
// Every kernel here uses a level-fixed thread mapping: a thread keeps one (or,
// for nz > 256, up to four) z-levels for its whole life and walks columns, so
// loads are coalesced along z and per-level sums stay in registers.  Block
// partials are reduced in a fixed order, so sums are reproducible.
#include "common.cuh"

#include <atomic>

#include <cmath>
#include <limits>
#include <vector>
#include <algorithm>
#include <array>
#include <mutex>
#include <map>

namespace steam {

constexpr int kLvThreads = 256;
constexpr int kLvMaxJ = 4;  // nz <= 1024
constexpr int kLvBlocksPerSm = 8;
constexpr int kLvUnroll = 4;  // columns per thread per iteration (loads in flight)

struct LevelMap {
  int nz;
  int G;  // columns per block-iteration (packed mode)
  int J;  // levels per thread (unpacked mode)
  bool packed;
};

static LevelMap make_map(int64_t nz) {
  LevelMap m;
  m.nz = (int)nz;
  if (nz <= kLvThreads) {
    m.packed = true;
    m.G = kLvThreads / (int)nz;
    m.J = 1;
  } else {
    m.packed = false;
    m.G = 1;
    m.J = (int)((nz + kLvThreads - 1) / kLvThreads);
  }
  return m;
}

static int level_grid(int64_t ncol, const LevelMap& m) {
  int64_t per = m.packed ? m.G : 1;
  return stride_grid((ncol + per - 1) / per, 1, kLvBlocksPerSm);
}

struct Win {
  int64_t x0, x1, y0, y1;
  int full;  // the window is the whole array: no test needed
  __device__ __forceinline__ bool in(int64_t x, int64_t y) const {
    return full || (x >= x0 && x < x1 && y >= y0 && y < y1);
  }
};

static Win make_win(const steam_window_t* w, int64_t nx, int64_t ny) {
  Win r;
  r.x0 = w ? w->x0 : 0;
  r.x1 = w ? w->x1 : nx;
  r.y0 = w ? w->y0 : 0;
  r.y1 = w ? w->y1 : ny;
  r.full = r.x0 == 0 && r.x1 == nx && r.y0 == 0 && r.y1 == ny;
  return r;
}

static int check_win(const steam_window_t* w, int64_t nx, int64_t ny,
                     const char* who) {
  if (!w) return STEAM_OK;
  STEAM_REQUIRE(w->x0 >= 0 && w->x1 <= nx && w->x0 <= w->x1 && w->y0 >= 0 &&
                    w->y1 <= ny && w->y0 <= w->y1,
                std::string(who) + ": window outside the array");
  return STEAM_OK;
}

// Reduce acc[Q][J] of every thread to per-level block partials:
// partials[(q * nz + z) * nblocks + blockIdx.x].
template <int Q, int JM>
__device__ void store_level_partials(const LevelMap& m, double (&acc)[Q][JM],
                                     double* red, double* partials) {
  const int t = threadIdx.x;
  const int nb = gridDim.x;
  if (m.packed) {
    const int active = m.G * m.nz;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      __syncthreads();
      if (t < active) red[t] = acc[q][0];
      __syncthreads();
      if (t < m.nz) {
        double s = 0.0;
        for (int g = 0; g < m.G; ++g) s += red[g * m.nz + t];
        partials[((size_t)q * m.nz + t) * nb + blockIdx.x] = s;
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
      for (int j = 0; j < JM; ++j) {
        const int z = t + j * kLvThreads;
        if (j < m.J && z < m.nz)
          partials[((size_t)q * m.nz + z) * nb + blockIdx.x] = acc[q][j];
      }
  }
}

// Iterate (column, level) pairs of this thread: fn(col, x, y, z, j).  The
// column's x and y advance incrementally (no division per element).
struct ColWalk {
  int64_t col, x, y;
  int64_t sx, sy, ny;
  __device__ __forceinline__ void init(int64_t c, int64_t step, int64_t ny_) {
    ny = ny_;
    col = c;
    x = c / ny;
    y = c - x * ny;
    sx = step / ny;
    sy = step - sx * ny;
  }
  __device__ __forceinline__ void advance(int64_t step) {
    col += step;
    x += sx;
    y += sy;
    if (y >= ny) {
      y -= ny;
      x += 1;
    }
  }
};

template <int JM, typename F>
__device__ __forceinline__ void for_levels(const LevelMap& m, int64_t ncol, int64_t ny, F fn) {
  const int t = threadIdx.x;
  if (m.packed) {
    if (t >= m.G * m.nz) return;
    const int z = t % m.nz;
    const int64_t cofs = t / m.nz;
    const int64_t step = (int64_t)gridDim.x * m.G;
    ColWalk w;
    w.init((int64_t)blockIdx.x * m.G + cofs, step, ny);
    // kLvUnroll independent columns per iteration so their loads overlap
    while (w.col + (kLvUnroll - 1) * step < ncol) {
      ColWalk u = w;
#pragma unroll
      for (int k = 0; k < kLvUnroll; ++k) {
        fn(u.col, u.x, u.y, z, 0);
        u.advance(step);
      }
      w = u;
    }
    for (; w.col < ncol; w.advance(step)) fn(w.col, w.x, w.y, z, 0);
  } else {
    // j is a compile-time index after unrolling, so per-level accumulators
    // indexed by it stay in registers
    ColWalk w;
    w.init(blockIdx.x, gridDim.x, ny);
    for (; w.col < ncol; w.advance(gridDim.x)) {
#pragma unroll
      for (int j = 0; j < JM; ++j) {
        const int z = t + j * kLvThreads;
        if (j < m.J && z < m.nz) fn(w.col, w.x, w.y, z, j);
      }
    }
  }
}

// ---- level sums ---------------------------------------------------------------
template <typename T, int JM>
__global__ void __launch_bounds__(kLvThreads) level_sums_kernel(
    const T* __restrict__ f, int64_t nx, int64_t ny, LevelMap m, Win w,
    double* __restrict__ partials) {
  __shared__ double red[kLvThreads];
  double acc[3][JM];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int j = 0; j < JM; ++j) acc[q][j] = 0.0;
  const int64_t ncol = nx * ny;
  for_levels<JM>(m, ncol, ny, [&](int64_t col, int64_t x, int64_t y, int z, int j) {
    if (!w.in(x, y)) return;
    T v = f[col * m.nz + z];
    acc[0][j] += (double)v;
    acc[1][j] += (double)(v < (T)0 ? -v : v);
    acc[2][j] += v != (T)0 ? 1.0 : 0.0;
  });
  store_level_partials<3, JM>(m, acc, red, partials);
}

// ---- scalar pattern -------------------------------------------------------------
template <typename T>
struct PatternArgs {
  T two_dx, two_dy, two_dz, dz_first, dz_last, lo, span, s_scale;
  int uniform_z;
  int has_prod;   // 0: no signed amplitude (W alone)
  int has_taper;  // 0: no bound taper
  const double* s_scale_dev;  // non-NULL: s_scale is read here (device), rounded to T
  // reciprocals of the differencing denominators (the vectorised kernel
  // multiplies by them: at most one ulp from the quotient)
  T inv_two_dx, inv_two_dy, inv_two_dz, inv_dz_first, inv_dz_last;
};

// |grad_h phi| = sqrt(gx^2 + gy^2): float32 by the hardware's approximate
// square root (PTX sqrt.approx.f32, within 2 float32 ulps, exact at 0, no
// flush of subnormals), float64 correctly rounded.  The pattern's float32
// bar is 2e-5 relative.
__device__ __forceinline__ float grad_sqrt(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ double grad_sqrt(double x) { return sqrt(x); }

template <typename T, int JM>
__global__ void __launch_bounds__(kLvThreads) pattern_kernel(
    const T* __restrict__ pert, const T* __restrict__ mean,
    const T* __restrict__ prod, const T* __restrict__ za,
    const T* __restrict__ zb, const T* __restrict__ zc,
    const T* __restrict__ aspect, const T* __restrict__ bbuf, int64_t nx,
    int64_t ny, LevelMap m, Win w, PatternArgs<T> a, T* __restrict__ out,
    double* __restrict__ partials) {
  __shared__ double red[kLvThreads];
  if (a.s_scale_dev) a.s_scale = (T)a.s_scale_dev[0];
  double acc[2][JM];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int j = 0; j < JM; ++j) acc[q][j] = 0.0;
  const int nz = m.nz;
  const int64_t ncol = nx * ny;
  for_levels<JM>(m, ncol, ny, [&](int64_t col, int64_t x, int64_t y, int z, int j) {
    const int64_t xp = x + 1 < nx ? x + 1 : 0, xm = x > 0 ? x - 1 : nx - 1;
    const int64_t yp = y + 1 < ny ? y + 1 : 0, ym = y > 0 ? y - 1 : ny - 1;
    const T mz = mean[z];
    const int64_t i = col * nz + z;
    const T r = add_rn(pert[i], mz);
    const T rxp = add_rn(pert[(xp * ny + y) * nz + z], mz);
    const T rxm = add_rn(pert[(xm * ny + y) * nz + z], mz);
    const T ryp = add_rn(pert[(x * ny + yp) * nz + z], mz);
    const T rym = add_rn(pert[(x * ny + ym) * nz + z], mz);
    const T gx = sub_rn(rxp, rxm) / a.two_dx;
    const T gy = sub_rn(ryp, rym) / a.two_dy;
    const T gh = grad_sqrt(add_rn(mul_rn(gx, gx), mul_rn(gy, gy)));
    T gz;
    if (z == 0) {
      const T r1 = add_rn(pert[i + 1], mean[1]);
      gz = sub_rn(r1, r) / a.dz_first;
    } else if (z == nz - 1) {
      const T r0 = add_rn(pert[i - 1], mean[z - 1]);
      gz = sub_rn(r, r0) / a.dz_last;
    } else {
      const T rzm = add_rn(pert[i - 1], mean[z - 1]);
      const T rzp = add_rn(pert[i + 1], mean[z + 1]);
      if (a.uniform_z) {
        gz = sub_rn(rzp, rzm) / a.two_dz;
      } else {
        gz = add_rn(add_rn(mul_rn(za[z - 1], rzm), mul_rn(zb[z - 1], r)),
                    mul_rn(zc[z - 1], rzp));
      }
    }
    gz = gz < (T)0 ? -gz : gz;
    T W = add_rn(mul_rn(gz, aspect[z]), gh);
    if (a.has_prod) {
      const T S = mul_rn(prod[i], a.s_scale);
      W = mul_rn(W, S);
    }
    if (a.has_taper) {
      T g = sub_rn(r, a.lo);
      const T g2 = sub_rn(a.span, g);
      g = g2 < g ? g2 : g;
      const T bz = bbuf[z];
      g = g / (bz > (T)0 ? bz : (T)1e-30);
      g = g < (T)0 ? (T)0 : (g > (T)1 ? (T)1 : g);
      W = mul_rn(W, g);
    }
    out[i] = W;
    if (w.in(x, y)) {
      acc[0][j] += (double)(W < (T)0 ? -W : W);
      acc[1][j] += W != (T)0 ? 1.0 : 0.0;
    }
  });
  store_level_partials<2, JM>(m, acc, red, partials);
}

// ---- scalar pattern, one 4-level group per thread --------------------------------
// For nz % 4 == 0 (nz <= 1024): a column's nz/4 threads each own 4 consecutive
// levels for the whole grid-stride walk, so the per-level constants sit in
// registers; a block covers 256 / (nz/4) consecutive columns per step.  The
// x and y neighbours are 16-byte loads of adjacent columns.  The grid walks
// columns in memory order, so planes x-1, x and x+1 are all resident in L2
// while plane x is processed and DRAM sees every input once.
template <typename T>
__device__ __forceinline__ T pattern_cell(T r, T rxm, T rxp, T rym, T ryp, T rzm, T rzp,
                                          int z, int nz, T prod, T az, T bz, T cz,
                                          T asp, T bb, const PatternArgs<T>& a) {
  const T gx = sub_rn(rxp, rxm) / a.two_dx;
  const T gy = sub_rn(ryp, rym) / a.two_dy;
  const T gh = grad_sqrt(add_rn(mul_rn(gx, gx), mul_rn(gy, gy)));
  T gz;
  if (z == 0) {
    gz = sub_rn(rzp, r) / a.dz_first;
  } else if (z == nz - 1) {
    gz = sub_rn(r, rzm) / a.dz_last;
  } else if (a.uniform_z) {
    gz = sub_rn(rzp, rzm) / a.two_dz;
  } else {
    gz = add_rn(add_rn(mul_rn(az, rzm), mul_rn(bz, r)), mul_rn(cz, rzp));
  }
  gz = gz < (T)0 ? -gz : gz;
  T W = add_rn(mul_rn(gz, asp), gh);
  if (a.has_prod) W = mul_rn(W, mul_rn(prod, a.s_scale));
  if (a.has_taper) {
    T g = sub_rn(r, a.lo);
    const T g2 = sub_rn(a.span, g);
    g = g2 < g ? g2 : g;
    g = g / (bb > (T)0 ? bb : (T)1e-30);
    g = g < (T)0 ? (T)0 : (g > (T)1 ? (T)1 : g);
    W = mul_rn(W, g);
  }
  return W;
}

template <typename T, bool UNI>
__device__ __forceinline__ T pattern_cell_fast(T r, T rxm, T rxp, T rym, T ryp, T rzm, T rzp,
                                               int z, int nz, T prod, T az, T bz, T cz,
                                               T asp, T ibb, const PatternArgs<T>& a) {
  const T gx = mul_rn(sub_rn(rxp, rxm), a.inv_two_dx);
  const T gy = mul_rn(sub_rn(ryp, rym), a.inv_two_dy);
  const T gh = grad_sqrt(add_rn(mul_rn(gx, gx), mul_rn(gy, gy)));
  T gz;
  if (z == 0) {
    gz = mul_rn(sub_rn(rzp, r), a.inv_dz_first);
  } else if (z == nz - 1) {
    gz = mul_rn(sub_rn(r, rzm), a.inv_dz_last);
  } else if (UNI) {
    gz = mul_rn(sub_rn(rzp, rzm), a.inv_two_dz);
  } else {
    gz = add_rn(add_rn(mul_rn(az, rzm), mul_rn(bz, r)), mul_rn(cz, rzp));
  }
  gz = gz < (T)0 ? -gz : gz;
  T W = add_rn(mul_rn(gz, asp), gh);
  if (a.has_prod) W = mul_rn(W, mul_rn(prod, a.s_scale));
  if (a.has_taper) {
    T g = sub_rn(r, a.lo);
    const T g2 = sub_rn(a.span, g);
    g = g2 < g ? g2 : g;
    g = mul_rn(g, ibb);
    g = g < (T)0 ? (T)0 : (g > (T)1 ? (T)1 : g);
    W = mul_rn(W, g);
  }
  return W;
}

template <typename T, bool UNI>
__global__ void __launch_bounds__(kLvThreads, (sizeof(T) == 4 ? 3 : 2)) pattern_vec_kernel(
    const T* __restrict__ pert, const T* __restrict__ vecs, const T* __restrict__ prod,
    int64_t nx, int64_t ny, int nz, Win w, PatternArgs<T> a, T* __restrict__ out,
    double* __restrict__ partials) {
  __shared__ double red[4 * kLvThreads];
  if (a.s_scale_dev) a.s_scale = (T)a.s_scale_dev[0];
  const int nz4 = nz >> 2;
  const int cpb = kLvThreads / nz4;
  const int t = threadIdx.x;
  const int cs = t / nz4;
  const int z4 = (t - cs * nz4) * 4;
  const bool act = cs < cpb;
  // vecs: [0] mean, [1] a, [2] b, [3] c (np.gradient, indexed z-1), [4] aspect, [5] buffer
  T mz[4], asp[4], ibb[4], ca[4], cb[4], cc[4];
  T m_lo = (T)0, m_hi = (T)0;
  if (act) {
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const int z = z4 + l;
      mz[l] = vecs[z];
      asp[l] = vecs[4 * nz + z];
      const T bb = vecs[5 * nz + z];
      ibb[l] = (T)1 / (bb > (T)0 ? bb : (T)1e-30);
      if (!UNI) {
        ca[l] = z > 0 ? vecs[nz + z - 1] : (T)0;
        cb[l] = z > 0 ? vecs[2 * nz + z - 1] : (T)0;
        cc[l] = z > 0 ? vecs[3 * nz + z - 1] : (T)0;
      } else {
        ca[l] = cb[l] = cc[l] = (T)0;
      }
    }
    m_lo = z4 > 0 ? vecs[z4 - 1] : (T)0;
    m_hi = z4 + 4 < nz ? vecs[z4 + 4] : (T)0;
  }
  double acc0[4] = {0, 0, 0, 0};
  unsigned acc1[4] = {0u, 0u, 0u, 0u};  // nonzero counts, exact as integers
  const int64_t ncol = nx * ny;
  const int64_t step = (int64_t)gridDim.x * cpb;
  ColWalk cw;
  cw.init((int64_t)blockIdx.x * cpb + cs, step, ny);
  if (act) {
    for (; cw.col < ncol; cw.advance(step)) {
      const int64_t x = cw.x, y = cw.y;
      const int64_t xp = x + 1 < nx ? x + 1 : 0, xm = x > 0 ? x - 1 : nx - 1;
      const int64_t yp = y + 1 < ny ? y + 1 : 0, ym = y > 0 ? y - 1 : ny - 1;
      const int64_t base = cw.col * nz + z4;
      const V4<T> c = ld4(pert + base);
      const V4<T> vxp = ld4(pert + (xp * ny + y) * nz + z4);
      const V4<T> vxm = ld4(pert + (xm * ny + y) * nz + z4);
      const V4<T> vyp = ld4(pert + (x * ny + yp) * nz + z4);
      const V4<T> vym = ld4(pert + (x * ny + ym) * nz + z4);
      const T below = z4 > 0 ? pert[base - 1] : (T)0;
      const T above = z4 + 4 < nz ? pert[base + 4] : (T)0;
      V4<T> pr;
      if (a.has_prod) pr = ld4(prod + base);
      else pr.v[0] = pr.v[1] = pr.v[2] = pr.v[3] = (T)0;
      T r[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) r[l] = add_rn(c.v[l], mz[l]);
      const T r_lo = add_rn(below, m_lo), r_hi = add_rn(above, m_hi);
      V4<T> o;
      const bool in_w = w.in(x, y);
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const int z = z4 + l;
        const T rzm = l == 0 ? r_lo : r[l - 1];
        const T rzp = l == 3 ? r_hi : r[l + 1];
        const T Wv = pattern_cell_fast<T, UNI>(
            r[l], add_rn(vxm.v[l], mz[l]), add_rn(vxp.v[l], mz[l]), add_rn(vym.v[l], mz[l]),
            add_rn(vyp.v[l], mz[l]), rzm, rzp, z, nz, pr.v[l], ca[l], cb[l], cc[l], asp[l],
            ibb[l], a);
        o.v[l] = Wv;
        if (in_w) {
          acc0[l] += (double)(Wv < (T)0 ? -Wv : Wv);
          acc1[l] += Wv != (T)0 ? 1u : 0u;
        }
      }
      st4(out + base, o);
    }
  }
  // per-level partials: the block's column slots in order
  const int nb = gridDim.x;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    __syncthreads();
    if (act)
#pragma unroll
      for (int l = 0; l < 4; ++l) red[cs * nz + z4 + l] = q == 0 ? acc0[l] : (double)acc1[l];
    __syncthreads();
    for (int z = t; z < nz; z += blockDim.x) {
      double sacc = 0.0;
      for (int k = 0; k < cpb; ++k) sacc += red[k * nz + z];
      partials[((size_t)q * nz + z) * nb + blockIdx.x] = sacc;
    }
  }
}

// ---- bounded add sweeps --------------------------------------------------------
// Per-level chain (the replay form, ba_sweep_kernel, for any layout, applies
// it from the raw increment on every sweep; the write-back form below keeps
// its running state in the increment):
//   for s < nsteps[z]:  d = clip(d - demean[z,s], caps) * scale[z,s]
//   if has_final[z]:    d = clip(d - final_dm[z], caps)
//   if has_mu[z]:       d = clip(d - mu[z], caps)
// with caps = (lo - phi, hi - phi), phi = pert + mean.
constexpr int kMuCand = 4;
// BA_SUMS: the first sweep, sum d and sum |d| of the raw increment (no chain
// step is set yet, so the perturbation is not read)
enum { BA_STATS = 0, BA_MU = 1, BA_APPLY = 2, BA_SUMS = 3 };

template <typename T>
struct BAChain {
  const int* nsteps;
  const T* demean;  // [nz][R]
  const T* scale;   // [nz][R]
  const int* has_final;
  const T* final_dm;
  const int* has_mu;
  const T* mu;
  const T* cand;  // [nz][kMuCand]
  const T* mean;
  const int* run;  // device flag: the sweep returns at once when it is 0 (NULL: always run)
  // write-back form (ba_fold_kernel): the increment buffer holds the chain's
  // first applied[z] steps (and the final clip when fin_stored[z]) already
  // applied; still[z] marks a level whose last step's scale is not decided
  const int* applied;
  const int* fin_stored;
  const int* still;
  // write-back form: per group of 4 levels, whether this sweep stores the
  // group's pending steps (written by block 0 of a statistics or shift sweep)
  int* grp;
  int R;
  T lo, hi;
};

template <typename T>
__device__ __forceinline__ T clampv(T v, T a, T b) {
  v = v > a ? v : a;
  return v < b ? v : b;
}

template <typename T>
static size_t ba_smem_bytes(int64_t nz, int R) {
  return sizeof(T) * (size_t)nz * (2 * (size_t)R + 4 + kMuCand) + sizeof(int) * 3 * (size_t)nz;
}

template <typename T, int MODE, int JM>
__global__ void __launch_bounds__(kLvThreads) ba_sweep_kernel(
    const T* __restrict__ d0, T* __restrict__ pert, T* __restrict__ inc_out,
    int record, int64_t nx, int64_t ny, LevelMap m, Win w, BAChain<T> c,
    double* __restrict__ partials) {
  if (c.run && *c.run == 0) return;
  __shared__ double red[kLvThreads];
  extern __shared__ unsigned char ba_smem[];
  const int nz = m.nz, R = c.R;
  // the chain, level-fastest: s_dm[s * nz + z]
  T* s_dm = reinterpret_cast<T*>(ba_smem);
  T* s_sc = s_dm + (size_t)R * nz;
  T* s_fin = s_sc + (size_t)R * nz;
  T* s_mu = s_fin + nz;
  T* s_mean = s_mu + nz;
  T* s_cand = s_mean + nz;  // [kMuCand][nz]
  int* s_ns = reinterpret_cast<int*>(s_cand + (size_t)kMuCand * nz);
  int* s_hf = s_ns + nz;
  int* s_hm = s_hf + nz;
  for (int i = threadIdx.x; i < R * nz; i += blockDim.x) {
    const int z = i % nz, st = i / nz;
    s_dm[i] = c.demean[z * R + st];
    s_sc[i] = c.scale[z * R + st];
  }
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    s_fin[z] = c.final_dm[z];
    s_mu[z] = c.mu[z];
    s_mean[z] = c.mean[z];
    s_ns[z] = c.nsteps[z];
    s_hf[z] = c.has_final[z];
    s_hm[z] = c.has_mu[z];
#pragma unroll
    for (int k = 0; k < kMuCand; ++k) s_cand[k * nz + z] = c.cand[z * kMuCand + k];
  }
  __syncthreads();
  constexpr int Q = MODE == BA_MU ? 2 * kMuCand : 2;
  double acc[Q][JM];
#pragma unroll
  for (int q = 0; q < Q; ++q)
#pragma unroll
    for (int j = 0; j < JM; ++j) acc[q][j] = 0.0;
  const int64_t ncol = nx * ny;
  for_levels<JM>(m, ncol, ny, [&](int64_t col, int64_t x, int64_t y, int z, int j) {
    const int64_t i = col * nz + z;
    const T p0 = pert[i];
    T d = d0[i];
    const T phi = add_rn(p0, s_mean[z]);
    const T clo = sub_rn(c.lo, phi), chi = sub_rn(c.hi, phi);
    const int ns = s_ns[z];
    for (int st = 0; st < ns; ++st) {
      d = clampv(sub_rn(d, s_dm[st * nz + z]), clo, chi);
      d = mul_rn(d, s_sc[st * nz + z]);
    }
    if (s_hf[z]) d = clampv(sub_rn(d, s_fin[z]), clo, chi);
    if (MODE == BA_APPLY) {
      if (s_hm[z]) d = clampv(sub_rn(d, s_mu[z]), clo, chi);
      const T pn = add_rn(p0, d);
      pert[i] = pn;
      if (record) inc_out[i] = sub_rn(pn, p0);
      return;
    }
    if (!w.in(x, y)) return;
    if (MODE == BA_STATS) {
      acc[0][j] += (double)d;
      acc[1 % Q][j] += (double)(d < (T)0 ? -d : d);
    } else {
#pragma unroll
      for (int k = 0; k < kMuCand; ++k) {
        const T raw = sub_rn(d, s_cand[k * nz + z]);
        const bool in = raw > clo && raw < chi;
        // inside the caps the cell's value d - mu enters as d (the solver
        // subtracts mu times the inside count); outside, the cap
        acc[2 * k][j] += (double)(in ? d : clampv(raw, clo, chi));
        acc[(2 * k + 1) % Q][j] += in ? 1.0 : 0.0;
      }
    }
  });
  if (MODE != BA_APPLY) store_level_partials<Q, JM>(m, acc, red, partials);
}

// ---- bounded add sweeps, write-back form -------------------------------------------
// The increment buffer is the chain's running state: a sweep applies only the
// steps not yet stored -- at most one whose parameters are now final (the last
// rescale step of the previous sweep, or the final demean/clip of a level that
// left the loop) and at most one tentative step (the current rescale step,
// scale still 1) -- and writes the final part back.  Every sweep therefore
// costs the same few operations per cell instead of replaying the whole chain
// from the raw increment.  nz % 4 == 0; a thread owns 4 consecutive levels.
// Loads of values other blocks of the same grid wrote in this launch go
// through L2 (ld.cg), never a stale L1 line.
// Shared-memory ring of the statistics and shift sweeps: kBaStages columns
// per thread, 4 elements of the increment and 4 of the perturbation each.
constexpr int kBaStages = 4;

// per-level parameters at the front of the fold kernels' dynamic shared
// memory (rounded up to 16 bytes; the cp.async ring follows)
template <typename T>
__host__ __device__ constexpr size_t ba_fold_param_bytes(int64_t nz) {
  return (sizeof(T) * (size_t)nz * (13 + kMuCand) + 15) / 16 * 16;
}

// 4 elements (16 or 32 bytes) global -> shared, asynchronously (L2 only)
template <typename T>
__device__ __forceinline__ void cp_async_v4(T* sdst, const T* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
#pragma unroll
  for (int b = 0; b < (int)sizeof(T) / 4; ++b)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s + 16 * b),
                 "l"(reinterpret_cast<const char*>(gsrc) + 16 * b)
                 : "memory");
}

template <typename T>
__device__ __forceinline__ V4<T> lds4(const T* p) {
  return ld4(p);
}

template <bool COH, typename V>
__device__ __forceinline__ V ldc(const V* p) {
  if (COH) return __ldcg(p);
  return *p;
}

// vb / nvb: this block's index among the blocks that share the sweep of this
// field, and their count (blockIdx.x / gridDim.x for a launch of its own; a
// block's range within a grouped launch over several fields)
template <typename T, int MODE, bool COH>
__device__ __forceinline__ void ba_fold_body(T* __restrict__ d0, T* __restrict__ pert,
                                             int record, int64_t nx, int64_t ny, int nz,
                                             const Win& w, const BAChain<T>& c,
                                             double* __restrict__ partials,
                                             unsigned char* ba_smem, double* red, int vb,
                                             int nvb) {
  // per level: fold step (dm, sc), final clip (dm), tentative step (dm),
  // mean, mu, candidates; flags as 0/1 in T
  T* s_fdm = reinterpret_cast<T*>(ba_smem);
  T* s_fsc = s_fdm + nz;
  T* s_fon = s_fsc + nz;
  T* s_cdm = s_fon + nz;
  T* s_con = s_cdm + nz;
  T* s_tdm = s_con + nz;
  T* s_ton = s_tdm + nz;
  T* s_mean = s_ton + nz;
  T* s_mu = s_mean + nz;
  T* s_mon = s_mu + nz;
  T* s_cand = s_mon + nz;  // [kMuCand][nz]
  T* s_cmin = s_cand + kMuCand * nz;  // smallest and largest candidate
  T* s_cmax = s_cmin + nz;
  const int R = c.R;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    const int ns = ldc<COH>(c.nsteps + z), ap = ldc<COH>(c.applied + z);
    const int nfin = ldc<COH>(c.still + z) ? ns - 1 : ns;
    const bool fold_step = nfin > ap;  // == ap + 1 by construction
    s_fon[z] = fold_step ? (T)1 : (T)0;
    s_fdm[z] = fold_step ? ldc<COH>(c.demean + z * R + ap) : (T)0;
    s_fsc[z] = fold_step ? ldc<COH>(c.scale + z * R + ap) : (T)1;
    const bool fold_fin = ldc<COH>(c.has_final + z) && !ldc<COH>(c.fin_stored + z);
    s_con[z] = fold_fin ? (T)1 : (T)0;
    s_cdm[z] = ldc<COH>(c.final_dm + z);
    const bool tent = ns > nfin;  // the current rescale step, scale 1
    s_ton[z] = tent ? (T)1 : (T)0;
    s_tdm[z] = tent ? ldc<COH>(c.demean + z * R + nfin) : (T)0;
    s_mean[z] = ldc<COH>(c.mean + z);
    s_mon[z] = ldc<COH>(c.has_mu + z) ? (T)1 : (T)0;
    s_mu[z] = ldc<COH>(c.mu + z);
    T cmin = ldc<COH>(c.cand + z * kMuCand), cmax = cmin;
#pragma unroll
    for (int k = 0; k < kMuCand; ++k) {
      const T ck = ldc<COH>(c.cand + z * kMuCand + k);
      s_cand[k * nz + z] = ck;
      cmin = ck < cmin ? ck : cmin;
      cmax = ck > cmax ? ck : cmax;
    }
    s_cmin[z] = cmin;
    s_cmax[z] = cmax;
  }
  __syncthreads();
  constexpr int Q = MODE == BA_MU ? 2 * kMuCand : 2;
  const int nz4 = nz / 4;
  const int t = threadIdx.x;
  // A statistics sweep works only on the groups of 4 levels with a level
  // still in the rescale loop.  When some groups have left it, the block's
  // threads are dealt over the remaining groups alone (more columns per
  // block step) instead of idling on the groups that are done: s_act lists
  // the groups in the loop, s_gix maps a group to its place in that list
  // (-1: out of the loop).
  int ng = nz4;     // groups dealt over the threads
  int nact = nz4;   // groups with work
  const int* act = nullptr;
  const int* gix = nullptr;
  if constexpr (MODE == BA_STATS) {
    __shared__ int s_act[kLvThreads], s_gix[kLvThreads], s_nact;
    if (t == 0) {
      int n = 0;
      for (int g = 0; g < nz4; ++g) {
        const bool in = s_ton[4 * g] != (T)0 || s_ton[4 * g + 1] != (T)0 ||
                        s_ton[4 * g + 2] != (T)0 || s_ton[4 * g + 3] != (T)0;
        s_gix[g] = in ? n : -1;
        if (in) s_act[n++] = g;
      }
      s_nact = n;
    }
    __syncthreads();
    nact = s_nact;
    if (nact < nz4) {
      ng = nact > 0 ? nact : 1;
      act = s_act;
      gix = s_gix;
    }
  }
  const bool compact = act != nullptr;
  const int cpi = kLvThreads / ng;
  const bool active = t < cpi * ng && nact > 0;
  const int gi = t % ng;
  const int z4 = (compact ? (nact > 0 ? act[gi] : 0) : gi) * 4;
  const int cofs = t / ng;
  const V4<T> fdm = ld4(s_fdm + z4), fsc = ld4(s_fsc + z4);
  const V4<T> cdm = ld4(s_cdm + z4), tdm = ld4(s_tdm + z4);
  const V4<T> mean = ld4(s_mean + z4);
  // per-level switches as bits: fold step (l), fold final clip (4 + l),
  // tentative step (8 + l), shift (12 + l)
  unsigned on = 0;
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    on |= (s_fon[z4 + l] != (T)0 ? 1u : 0u) << l;
    on |= (s_con[z4 + l] != (T)0 ? 1u : 0u) << (4 + l);
    on |= (s_ton[z4 + l] != (T)0 ? 1u : 0u) << (8 + l);
    on |= (s_mon[z4 + l] != (T)0 ? 1u : 0u) << (12 + l);
  }
  const bool any_fold = (on & 0xffu) != 0;
  // a statistics sweep with no clip step on this thread's levels (the first
  // sweep, and levels that left the loop with their final clip stored) never
  // reads the perturbation
  const bool need_p = MODE == BA_SUMS ? false : (MODE != BA_STATS || (on & 0xfffu) != 0);
  // a statistics sweep has nothing to do for 4 levels none of which is still
  // in the rescale loop (their sums are not read, and steps they have pending
  // stay pending: no later step joins them, and the apply sweep applies
  // them): it reads and writes nothing for them
  const bool work = active && !(MODE == BA_STATS && (on & 0xf00u) == 0u);
  if ((MODE == BA_STATS || MODE == BA_MU) && vb == 0)
    for (int g = threadIdx.x; g < nz / 4; g += blockDim.x)
      c.grp[g] = MODE == BA_STATS && (s_ton[4 * g] != (T)0 || s_ton[4 * g + 1] != (T)0 ||
                                       s_ton[4 * g + 2] != (T)0 || s_ton[4 * g + 3] != (T)0);
  // sums in float64; the shift sweep's in-range counts as integers (exact)
  constexpr int QS = MODE == BA_MU ? kMuCand : 2;
  double acc[QS][4];
  unsigned cnt[MODE == BA_MU ? kMuCand : 1][4];
#pragma unroll
  for (int q = 0; q < QS; ++q)
#pragma unroll
    for (int l = 0; l < 4; ++l) acc[q][l] = 0.0;
#pragma unroll
  for (int q = 0; q < (MODE == BA_MU ? kMuCand : 1); ++q)
#pragma unroll
    for (int l = 0; l < 4; ++l) cnt[q][l] = 0u;
  // the shift sweep's terms common to every candidate (a cell inside the caps
  // for all of them, or beyond one cap for all), added to each candidate's
  // sums once, after the columns
  double acc_all[4] = {0.0, 0.0, 0.0, 0.0};
  unsigned cnt_all[4] = {0u, 0u, 0u, 0u};
  const int64_t ncol = nx * ny;
  auto process = [&](const ColWalk& cw, const V4<T>& dv, const V4<T>& pv) {
    const int64_t i = cw.col * nz + z4;
    const bool in_w = w.in(cw.x, cw.y);
    if constexpr (MODE == BA_SUMS) {
      if (in_w)
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          const double x = (double)dv.v[l];  // one conversion; |x| is exact
          acc[0][l] += x;
          acc[1][l] += fabs(x);
        }
    } else {
      V4<T> df, pn, dn;
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const T p0 = pv.v[l];
        const T phi = add_rn(p0, mean.v[l]);
        const T clo = sub_rn(c.lo, phi), chi = sub_rn(c.hi, phi);
        T d = dv.v[l];
        if (on & (1u << l)) d = mul_rn(clampv(sub_rn(d, fdm.v[l]), clo, chi), fsc.v[l]);
        if (on & (16u << l)) d = clampv(sub_rn(d, cdm.v[l]), clo, chi);
        df.v[l] = d;
        if (on & (256u << l)) d = clampv(sub_rn(d, tdm.v[l]), clo, chi);
        if (MODE == BA_APPLY) {
          if (on & (4096u << l)) d = clampv(sub_rn(d, s_mu[z4 + l]), clo, chi);
          pn.v[l] = add_rn(p0, d);
          dn.v[l] = sub_rn(pn.v[l], p0);
        } else if (in_w) {
          if (MODE == BA_STATS) {
            const double x = (double)d;
            acc[0][l] += x;
            acc[1 % QS][l] += fabs(x);
          } else {
            // d - mu over the candidates spans [d - cmax, d - cmin]: a cell
            // inside the caps (or beyond one cap) for all of them takes one
            // conversion; only a cell with a cap inside that span is
            // evaluated per candidate
            constexpr int KC = MODE == BA_MU ? kMuCand : 1;
            const T lo_all = sub_rn(d, s_cmax[z4 + l]), hi_all = sub_rn(d, s_cmin[z4 + l]);
            if (lo_all > clo && hi_all < chi) {
              acc_all[l] += (double)d;
              cnt_all[l] += 1u;
            } else if (lo_all >= chi || hi_all <= clo) {
              acc_all[l] += (double)(lo_all >= chi ? chi : clo);
            } else {
#pragma unroll
              for (int k = 0; k < kMuCand; ++k) {
                const T raw = sub_rn(d, s_cand[k * nz + z4 + l]);
                const bool in = raw > clo && raw < chi;
                acc[k][l] += (double)(in ? d : clampv(raw, clo, chi));
                cnt[k % KC][l] += in ? 1u : 0u;
              }
            }
          }
        }
      }
      if (MODE == BA_APPLY) {
        st4(pert + i, pn);
        if (record) st4(d0 + i, dn);
      } else if (MODE == BA_STATS && any_fold) {
        st4(d0 + i, df);
      }
    }
  };
  if (active && MODE == BA_APPLY) {
    const int64_t step = (int64_t)nvb * cpi;
    ColWalk cw;
    cw.init((int64_t)vb * cpi + cofs, step, ny);
    // two columns in flight per thread
    constexpr int U = 2;
    while (cw.col + (U - 1) * step < ncol) {
      ColWalk u[U];
      V4<T> dv[U], pv[U];
      u[0] = cw;
#pragma unroll
      for (int k = 1; k < U; ++k) {
        u[k] = u[k - 1];
        u[k].advance(step);
      }
#pragma unroll
      for (int k = 0; k < U; ++k) {
        dv[k] = ld4(d0 + u[k].col * nz + z4);
        pv[k] = ld4(pert + u[k].col * nz + z4);
      }
#pragma unroll
      for (int k = 0; k < U; ++k) process(u[k], dv[k], pv[k]);
      cw = u[U - 1];
      cw.advance(step);
    }
    for (; cw.col < ncol; cw.advance(step))
      process(cw, ld4(d0 + cw.col * nz + z4), ld4(pert + cw.col * nz + z4));
  } else if (work) {
    // statistics and shift sweeps: the thread's own 16-byte pieces of the
    // next kBaStages - 1 columns stream into its slots of a shared-memory
    // ring by cp.async while it works on the current column, so the loads in
    // flight do not depend on registers (a thread reads back only what it
    // copied itself: no block barrier)
    const int64_t step = (int64_t)nvb * cpi;
    ColWalk cw, front;
    cw.init((int64_t)vb * cpi + cofs, step, ny);
    front = cw;
    T* ring = reinterpret_cast<T*>(ba_smem + ba_fold_param_bytes<T>(nz));
    auto slot = [&](int s, int f) { return ring + ((size_t)(s * 2 + f) * kLvThreads + t) * 4; };
    auto issue = [&](int s) {
      if (front.col < ncol) {
        const size_t off = (size_t)front.col * nz + z4;
        cp_async_v4(slot(s, 0), d0 + off);
        if (need_p) cp_async_v4(slot(s, 1), pert + off);
      }
      cp_async_commit();  // one group per column, empty past the end
      front.advance(step);
    };
#pragma unroll
    for (int s = 0; s < kBaStages - 1; ++s) issue(s);
    int cur = 0;
    for (; cw.col < ncol; cw.advance(step)) {
      issue(cur == 0 ? kBaStages - 1 : cur - 1);
      cp_async_wait<kBaStages - 1>();
      const V4<T> dv = lds4(slot(cur, 0));
      const V4<T> pv = need_p ? lds4(slot(cur, 1)) : V4<T>{};
      process(cw, dv, pv);
      cur = cur + 1 == kBaStages ? 0 : cur + 1;
    }
    cp_async_wait<0>();
  }
  if (MODE == BA_APPLY) return;
  if constexpr (MODE == BA_MU) {
#pragma unroll
    for (int k = 0; k < kMuCand; ++k)
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        acc[k][l] += acc_all[l];
        cnt[k][l] += cnt_all[l];
      }
  }
  // deterministic reduction: per level, the cpi column slots in order
  const int nb = nvb;
  // partial rows: stats {sum d, sum |d|}; shift {mean_k, count_k} per candidate
  // (dealt over the groups in the loop: slot [cofs][gi][l], and 0 for the
  // levels of groups out of it, whose sums are not read)
  const int rw = compact ? 4 * ng : nz;  // red row width
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    __syncthreads();
    if (active)
#pragma unroll
      for (int l = 0; l < 4; ++l)
        red[cofs * rw + (compact ? 4 * gi : z4) + l] =
            MODE == BA_MU ? ((q & 1) ? (double)cnt[(q >> 1) % (MODE == BA_MU ? kMuCand : 1)][l]
                                     : acc[(q >> 1) % QS][l])
                          : acc[q % QS][l];
    __syncthreads();
    for (int z = t; z < nz; z += kLvThreads) {
      double sacc = 0.0;
      const int col = compact ? (gix[z >> 2] >= 0 ? 4 * gix[z >> 2] + (z & 3) : -1) : z;
      if (col >= 0)
        for (int cc = 0; cc < cpi; ++cc) sacc += red[cc * rw + col];
      partials[((size_t)q * nz + z) * nb + vb] = sacc;
    }
  }
}

// The bounded add's first sweep (BA_SUMS) and apply sweep (BA_APPLY) as
// launches of their own; its statistics and shift sweeps run inside
// ba_phase_kernel.
template <typename T, int MODE>
__global__ void __launch_bounds__(kLvThreads, 4)
    ba_fold_kernel(T* __restrict__ d0, T* __restrict__ pert, int record, int64_t nx,
                   int64_t ny, int nz, Win w, BAChain<T> c, double* __restrict__ partials) {
  if (c.run && *c.run == 0) return;
  __shared__ double red[4 * kLvThreads];
  extern __shared__ unsigned char ba_smem[];
  ba_fold_body<T, MODE, false>(d0, pert, record, nx, ny, nz, w, c, partials, ba_smem, red,
                               blockIdx.x, gridDim.x);
}

template <typename T>
static size_t ba_fold_smem_bytes(int64_t nz) {
  return ba_fold_param_bytes<T>(nz) + (size_t)kBaStages * 2 * kLvThreads * 4 * sizeof(T);
}

// ---- projection sweeps (float64 level arithmetic) -----------------------------
enum { PJ_STATS = 0, PJ_MU = 1, PJ_APPLY = 2 };

template <typename T, int MODE, int JM>
__global__ void __launch_bounds__(kLvThreads) proj_sweep_kernel(
    T* __restrict__ pert, const double* __restrict__ mean, double lo,
    double hi, const int* __restrict__ active, const double* __restrict__ mu,
    const double* __restrict__ cand, int64_t nx, int64_t ny, LevelMap m,
    Win w, double* __restrict__ partials) {
  __shared__ double red[kLvThreads];
  constexpr int Q = MODE == PJ_MU ? 2 * kMuCand : 3;
  double acc[Q][JM];
#pragma unroll
  for (int q = 0; q < Q; ++q)
#pragma unroll
    for (int j = 0; j < JM; ++j)
      acc[q][j] = (MODE == PJ_STATS && q == 1) ? INFINITY
                  : (MODE == PJ_STATS && q == 2) ? -INFINITY
                                                  : 0.0;
  const int nz = m.nz;
  const int64_t ncol = nx * ny;
  for_levels<JM>(m, ncol, ny, [&](int64_t col, int64_t x, int64_t y, int z, int j) {
    const int64_t i = col * nz + z;
    const double f = (double)pert[i] + mean[z];
    if (MODE == PJ_STATS) {
      acc[1][j] = fmin(acc[1][j], f);
      acc[2 % Q][j] = fmax(acc[2 % Q][j], f);
      if (w.in(x, y)) acc[0][j] += f;
      return;
    }
    if (!active[z]) return;
    if (MODE == PJ_APPLY) {
      pert[i] = (T)(fmin(fmax(f - mu[z], lo), hi) - mean[z]);
      return;
    }
    if (!w.in(x, y)) return;
#pragma unroll
    for (int k = 0; k < kMuCand; ++k) {
      const double raw = f - cand[z * kMuCand + k];
      acc[2 * k][j] += fmin(fmax(raw, lo), hi);
      acc[(2 * k + 1) % Q][j] += (raw > lo && raw < hi) ? 1.0 : 0.0;
    }
  });
  if (MODE == PJ_APPLY) return;
  if (MODE == PJ_STATS) {
    // min/max are reduced like sums but combine with fmin/fmax: store raw.
    const int t = threadIdx.x;
    const int nb = gridDim.x;
    if (m.packed) {
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        __syncthreads();
        if (t < m.G * m.nz) red[t] = acc[q][0];
        __syncthreads();
        if (t < m.nz) {
          double s = q == 0 ? 0.0 : (q == 1 ? INFINITY : -INFINITY);
          for (int g = 0; g < m.G; ++g) {
            double v = red[g * m.nz + t];
            s = q == 0 ? s + v : (q == 1 ? fmin(s, v) : fmax(s, v));
          }
          partials[((size_t)q * m.nz + t) * nb + blockIdx.x] = s;
        }
      }
    } else {
#pragma unroll
      for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int jj = 0; jj < JM; ++jj) {
          const int z = t + jj * kLvThreads;
          if (jj < m.J && z < m.nz)
            partials[((size_t)q * m.nz + z) * nb + blockIdx.x] = acc[q][jj];
        }
    }
  } else {
    store_level_partials<Q, JM>(m, acc, red, partials);
  }
}

__global__ void reduce_minmax_kernel(const double* __restrict__ partials,
                                     int nblocks, int nz,
                                     double* __restrict__ out) {
  // out[z] = sum (q=0); out[nz+z] = min (q=1); out[2nz+z] = max (q=2)
  const int q = blockIdx.y;
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz;
       z += gridDim.x * blockDim.x) {
    const double* src = partials + ((size_t)q * nz + z) * nblocks;
    double s = q == 0 ? 0.0 : (q == 1 ? INFINITY : -INFINITY);
    for (int b = 0; b < nblocks; ++b)
      s = q == 0 ? s + src[b] : (q == 1 ? fmin(s, src[b]) : fmax(s, src[b]));
    out[(size_t)q * nz + z] = s;
  }
}

// ---- host helpers ----------------------------------------------------------------
template <typename T>
static int upload(T* dst, const std::vector<T>& src, cudaStream_t s) {
  if (src.empty()) return STEAM_OK;
  STEAM_CUDA(cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(),
                             cudaMemcpyHostToDevice, s));
  return STEAM_OK;
}

static int fetch(std::vector<double>& dst, const double* src, size_t n,
                 cudaStream_t s) {
  dst.resize(n);
  STEAM_CUDA(cudaMemcpyAsync(dst.data(), src, sizeof(double) * n,
                             cudaMemcpyDeviceToHost, s));
  STEAM_CUDA(cudaStreamSynchronize(s));
  return STEAM_OK;
}

static size_t level_partial_bytes(int64_t nz, int q) {
  return carve_bytes((size_t)sm_count() * kLvBlocksPerSm * q * nz, sizeof(double)) +
         carve_bytes((size_t)q * nz, sizeof(double));
}

// Per-level bracketed Newton on a non-increasing piecewise-linear function
// m(mu) (the level mean of a clipped, shifted field, minus a target),
// evaluated at mu rounded to the working dtype T -- which is how the
// reference's bisection evaluates it too.  The bracket [a, b] always holds the
// sign change in the bisection's sense, m(a) > 0 >= m(b), with a and b values
// of T.  Each sweep evaluates kMuCand candidates (the Newton point, two
// points straddling it, the bracket midpoint); the solve ends when no value
// of T lies strictly inside the bracket, and returns its midpoint, as the
// bisection does.  The solver state lives in device memory, one per level,
// and is advanced by the update kernels between sweeps.
template <typename T>
__host__ __device__ inline double next_up_t(double x) {
  if (sizeof(T) == 4) return (double)nextafterf((float)x, INFINITY);
  return nextafter(x, (double)INFINITY);
}

template <typename T>
struct MuSolver {
  double a, b;
  double best_mu, best_m, best_slope;
  double abs_tol;
  int have_best;
  int done;

  // abs_tol: a bracket this narrow is accepted as converged.  In float32 the
  // level mean is a staircase in mu at the scale of the field's own ulps, so
  // below that scale any mu of the bracket gives the same field up to
  // single-ulp flips in a vanishing fraction of cells.
  __host__ __device__ void init(double width, double tol) {
    a = (double)(T)(-width);
    b = (double)(T)width;
    abs_tol = tol;
    have_best = 0;
    done = 0;
  }

  __host__ __device__ void candidates(double* out) const {
    const double mid = 0.5 * (a + b);
    double c0 = mid;
    if (have_best && best_slope < 0.0) {
      const double nt = best_mu - best_m / best_slope;  // Newton
      if (nt > a && nt < b) c0 = nt;
    }
    const double span = b - a;
    double eps = fabs(c0) * (sizeof(T) == 4 ? 2.4e-7 : 4.5e-16) * 4.0;
    if (eps < 0.5 * abs_tol) eps = 0.5 * abs_tol;
    if (eps > 0.25 * span) eps = 0.25 * span;
    out[0] = c0;
    out[1] = c0 - eps > a ? c0 - eps : 0.5 * (a + c0);
    out[2] = c0 + eps < b ? c0 + eps : 0.5 * (c0 + b);
    out[3] = mid;
  }

  // cand: the T-rounded candidates actually evaluated.
  __host__ __device__ void update(const double* cand, const double* mval, const double* slope) {
    for (int k = 0; k < kMuCand; ++k) {
      if (cand[k] <= a || cand[k] >= b) continue;
      if (mval[k] > 0.0)
        a = cand[k];
      else
        b = cand[k];
    }
    int kb = -1;
    for (int k = 0; k < kMuCand; ++k)
      if (kb < 0 || fabs(mval[k]) < fabs(mval[kb])) kb = k;
    if (kb >= 0) {
      have_best = 1;
      best_mu = cand[kb];
      best_m = mval[kb];
      best_slope = slope[kb];
    }
    if (next_up_t<T>(a) >= b || b - a <= abs_tol) done = 1;
  }
  __host__ __device__ double result() const { return 0.5 * (a + b); }
};

// Most mu sweeps a solve may take (the bracket at least halves per sweep).
constexpr int kMuMaxSweeps = 48;
// column groups (one block's pass of the vectorised sweep) per persistent
// phase block and sweep, at least
constexpr int kPhaseMinGroups = 32;

// Writable view of the chain the sweeps replay, plus the solver's state.
template <typename T>
struct BAState {
  int* nsteps;
  T* demean;  // [nz][R]
  T* scale;   // [nz][R]
  int* has_final;
  T* final_dm;
  int* has_mu;
  T* mu;
  T* cand;  // [nz][kMuCand]
  T* mean;
  double* a0;
  double* cur_mean;
  double* final_d;
  int* active;
  int* still;
  int* n_loop;
  int* need;
  int* applied;     // write-back form: chain steps already stored in the increment
  int* fin_stored;  // write-back form: final clip already stored
  int* grp;         // write-back form: the last sweep stored group z / 4
  int wb;           // the sweeps write back (vectorised path)
  MuSolver<T>* solver;
  // run flags: [0] the first sweep, [1 + k] rescale sweep k (k < R),
  // [1 + R + it] mu sweep it (it < kMuMaxSweeps); [kFlagSweeps] sweeps run
  int* flags;
  unsigned* bar;  // grid barrier of the persistent phases: arrivals, generation, error
  long long spin_limit;  // polls a block waits at that barrier before it gives up
  int R, nz;
  double N, width, tol_rel;
  double* ledger;  // [nz][ba_ledger_width(R)], see ba_finish_kernel
};

// Per-level ledger record: a0, n_loop, final demean, mu (NaN if none), sweeps
// of the whole solve, then the chain the apply sweep replays -- its step
// count, whether the final clip is set, the steps' demeans [R] and scales [R]
// (each the working dtype's value, exact in float64).
__host__ __device__ inline int ba_ledger_width(int R) { return 7 + 2 * R; }

template <typename T>
__host__ __device__ inline int ba_flag_count(int R) {
  return 2 + R + kMuMaxSweeps;
}

// chain reset and the mean profile, in the working dtype
template <typename T>
__device__ __forceinline__ void ba_init_body(const BAState<T>& st, const double* __restrict__ mean_1d) {
  const int nz = st.nz, R = st.R;
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
    st.nsteps[z] = 0;
    st.has_final[z] = 0;
    st.has_mu[z] = 0;
    st.final_dm[z] = (T)0;
    st.mu[z] = (T)0;
    st.mean[z] = (T)mean_1d[z];
    for (int k = 0; k < R; ++k) {
      st.demean[z * R + k] = (T)0;
      st.scale[z * R + k] = (T)1;
    }
    for (int k = 0; k < kMuCand; ++k) st.cand[z * kMuCand + k] = (T)0;
    st.active[z] = 0;
    st.still[z] = 0;
    st.n_loop[z] = 0;
    st.need[z] = 0;
    st.applied[z] = 0;
    st.fin_stored[z] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int nf = ba_flag_count<T>(R);
    for (int i = 0; i < nf; ++i) st.flags[i] = 0;
    st.flags[0] = 1;  // the first stats sweep always runs
    st.bar[0] = 0;
    st.bar[1] = 0;
    st.bar[2] = 0;
  }
}

template <typename T>
__global__ void ba_init_kernel(BAState<T> st, const double* __restrict__ mean_1d) {
  ba_init_body(st, mean_1d);
}

// reduce_partials_kernel that does nothing when its sweep did not run
__global__ void reduce_partials_if_kernel(const double* __restrict__ partials, int nblocks,
                                          double* __restrict__ out, const int* __restrict__ run) {
  if (run && *run == 0) return;
  __shared__ double scratch[32];
  const double* src = partials + (size_t)blockIdx.x * nblocks;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) acc += src[i];
  double s = block_sum(acc, scratch);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// Leaves the demean/clip/rescale loop: the final demean is the level's
// current mean, and its shift solve starts from a bracket symmetric about 0.
template <typename T>
__device__ void ba_leave_loop(const BAState<T>& st, int z) {
  st.still[z] = 0;
  st.final_d[z] = st.cur_mean[z];
  st.has_final[z] = 1;
  st.final_dm[z] = (T)st.cur_mean[z];
}

// Prepares rescale step k for a level still in the loop.
template <typename T>
__device__ void ba_prepare_step(const BAState<T>& st, int z, int k, int* next_flag) {
  st.demean[z * st.R + k] = (T)st.cur_mean[z];
  st.scale[z * st.R + k] = (T)1;
  st.nsteps[z] = k + 1;
  st.n_loop[z] = k + 1;
  atomicOr(next_flag, 1);
}

// After a write-back sweep: every final part of the chain is now stored.
template <typename T>
__device__ void ba_note_stored(const BAState<T>& st, int z) {
  // only a statistics sweep that processed the level's group stores its
  // pending steps; a shift sweep stores nothing (the apply sweep applies
  // whatever is still pending)
  if (!st.wb || !__ldcg(st.grp + (z >> 2))) return;
  st.applied[z] = st.still[z] ? st.nsteps[z] - 1 : st.nsteps[z];
  st.fin_stored[z] = st.has_final[z];
}

template <typename T>
__device__ void ba_count_sweep(const BAState<T>& st) {
  if (blockIdx.x == 0 && threadIdx.x == 0) st.flags[ba_flag_count<T>(st.R) - 1] += 1;
}

// After the first stats sweep: a0 = mean|d| and the entering mean.
template <typename T>
__device__ __forceinline__ void ba_a0_body(const BAState<T>& st, const double* __restrict__ tot) {
  const int nz = st.nz;
  ba_count_sweep(st);
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
    const double a0 = tot[nz + z] / st.N;
    st.a0[z] = a0;
    st.cur_mean[z] = tot[z] / st.N;
    if (a0 <= 0.0) {
      st.has_final[z] = 1;  // clip only
      st.final_dm[z] = (T)0;
      st.final_d[z] = 0.0;
      continue;
    }
    st.active[z] = 1;
    st.still[z] = 1;
    if (st.R > 0)
      ba_prepare_step(st, z, 0, &st.flags[1]);
    else
      ba_leave_loop(st, z);
  }
}

template <typename T>
__global__ void ba_a0_kernel(BAState<T> st, const double* __restrict__ tot) {
  ba_a0_body(st, tot);
}

// After rescale sweep k.
template <typename T, bool COH = false>
__device__ void ba_loop_level(const BAState<T>& st, const double* tot, int k, int z) {
  const int nz = st.nz;
  ba_note_stored(st, z);
  if (!st.still[z]) return;
  const double sum_d = ldc<COH>(tot + z), m_abs = ldc<COH>(tot + nz + z) / st.N;
  st.cur_mean[z] = sum_d / st.N;
  bool go = true;
  if (m_abs <= 0.0) {
    go = false;
  } else {
    double sc = st.a0[z] / m_abs;
    if (sc > 2.0) sc = 2.0;
    if (fabs(sc - 1.0) < 1e-4) {
      go = false;
    } else {
      st.scale[z * st.R + k] = (T)sc;
      st.cur_mean[z] = (double)(T)sc * sum_d / st.N;
    }
  }
  if (go && k + 1 < st.R)
    ba_prepare_step(st, z, k + 1, &st.flags[2 + k]);
  else
    ba_leave_loop(st, z);
}

template <typename T>
__global__ void ba_loop_kernel(BAState<T> st, const double* __restrict__ tot, int k) {
  if (st.flags[1 + k] == 0) return;
  ba_count_sweep(st);
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < st.nz; z += gridDim.x * blockDim.x)
    ba_loop_level(st, tot, k, z);
}

// After the loop: every active level starts its shift solve.  Its first
// candidate is mu = 0, whose mean is the post-clip level mean.
template <typename T>
__device__ __forceinline__ void ba_mu_init_body(const BAState<T>& st) {
  const int nz = st.nz;
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
    if (!st.active[z]) continue;
    st.need[z] = 1;
    MuSolver<T> sv;
    sv.init(st.width, st.a0[z] * st.tol_rel);
    double c[kMuCand];
    sv.candidates(c);
    for (int q = 0; q < kMuCand; ++q) st.cand[z * kMuCand + q] = (T)c[q];
    st.solver[z] = sv;
    atomicOr(&st.flags[1 + st.R], 1);
  }
}

template <typename T>
__global__ void ba_mu_init_kernel(BAState<T> st) {
  ba_mu_init_body(st);
}

// After mu sweep it.
template <typename T, bool COH = false>
__device__ void ba_mu_level(const BAState<T>& st, const double* tot, int it, int z) {
  const int nz = st.nz;
  ba_note_stored(st, z);
  if (!st.need[z]) return;
  MuSolver<T> sv = st.solver[z];
  if (sv.done) return;
  double mv[kMuCand], sl[kMuCand], cv[kMuCand];
  for (int q = 0; q < kMuCand; ++q) {
    // the candidate actually evaluated is the dtype-rounded one
    cv[q] = (double)st.cand[z * kMuCand + q];
    // the sweeps sum d over the cells inside the caps and the cap elsewhere:
    // the level mean at this candidate is (sum - mu * inside count) / N
    const double inside = ldc<COH>(tot + (size_t)(2 * q + 1) * nz + z);
    mv[q] = (ldc<COH>(tot + (size_t)(2 * q) * nz + z) - cv[q] * inside) / st.N;
    sl[q] = -inside / st.N;
  }
  if (it == 0 && fabs(mv[0]) <= 1e-9 * st.a0[z]) {
    st.need[z] = 0;  // the final clip left the level mean-free
    return;
  }
  sv.update(cv, mv, sl);
  if (!sv.done && it + 1 < kMuMaxSweeps) {
    double c[kMuCand];
    sv.candidates(c);
    for (int q = 0; q < kMuCand; ++q) st.cand[z * kMuCand + q] = (T)c[q];
    atomicOr(&st.flags[2 + st.R + it], 1);
  }
  st.solver[z] = sv;
}

template <typename T>
__global__ void ba_mu_kernel(BAState<T> st, const double* __restrict__ tot, int it) {
  if (st.flags[1 + st.R + it] == 0) return;
  ba_count_sweep(st);
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < st.nz; z += gridDim.x * blockDim.x)
    ba_mu_level(st, tot, it, z);
}

// ---- persistent phases --------------------------------------------------------------
// The rescale loop and the shift solve each run as ONE cooperative launch
// (all blocks co-resident) that iterates sweep -> grid barrier -> reduction ->
// grid barrier -> per-level update -> grid barrier until no level needs
// another sweep (a fixed launch sequence would spend an empty launch on each
// iteration a phase does not need).  The barrier spins with a
// bound: a block that waits past kBarSpinLimit polls records an error, and
// every block leaves at its next barrier.
constexpr long long kBarSpinLimit = 1ll << 26;  // ~ seconds with the back-off below
std::atomic<long long> g_bar_spin_limit{kBarSpinLimit};

// `nblocks` blocks meet at `bar` (the blocks of one field's phase)
__device__ bool grid_barrier(unsigned* bar, long long spin_limit, unsigned nblocks) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok_s = 1;
    volatile unsigned* vgen = bar + 1;
    volatile unsigned* verr = bar + 2;
    const unsigned g = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u) + 1u;
    if (arrived == nblocks) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long spins = 0;
      while (*vgen == g) {
        if (*verr || ++spins > spin_limit) {
          atomicExch(bar + 2, 1u);
          ok_s = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok_s != 0;
}

// One field's persistent phase on blocks vb = 0 .. nvb - 1 of the launch.
template <typename T, int MODE>
__device__ __forceinline__ void ba_phase_body(T* __restrict__ d0, T* __restrict__ pert,
                                              int64_t nx, int64_t ny, int nz, const Win& w,
                                              BAChain<T> c, const BAState<T>& st,
                                              double* __restrict__ partials,
                                              double* __restrict__ totals, int flag_base,
                                              int it0, int n_iter, unsigned char* ba_smem,
                                              double* red, int vb, int nvb) {
  constexpr int Q = MODE == BA_MU ? 2 * kMuCand : 2;
  const int nb = nvb;
  c.run = nullptr;
  for (int it = it0; it < n_iter; ++it) {
    // read after a barrier: every block sees the same flag
    if (__ldcg(st.flags + flag_base + it) == 0) break;
    ba_fold_body<T, MODE, true>(d0, pert, 0, nx, ny, nz, w, c, partials, ba_smem, red, vb,
                                nvb);
    if (!grid_barrier(st.bar, st.spin_limit, nvb)) return;
    // totals[r] = the r-th row of block partials, summed in a fixed order
    for (int r = vb; r < Q * nz; r += nb) {
      double acc = 0.0;
      for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += __ldcg(partials + (size_t)r * nb + i);
      const double sum = block_sum(acc, red);
      if (threadIdx.x == 0) totals[r] = sum;
    }
    if (!grid_barrier(st.bar, st.spin_limit, nvb)) return;
    if (vb == 0 && threadIdx.x == 0) st.flags[ba_flag_count<T>(st.R) - 1] += 1;
    for (int z = vb * blockDim.x + threadIdx.x; z < nz; z += nb * blockDim.x) {
      if (MODE == BA_MU)
        ba_mu_level<T, true>(st, totals, it, z);
      else
        ba_loop_level<T, true>(st, totals, it, z);
    }
    if (!grid_barrier(st.bar, st.spin_limit, nvb)) return;
  }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(kLvThreads, (MODE == BA_MU ? 2 : 3)) ba_phase_kernel(
    T* __restrict__ d0, T* __restrict__ pert, int64_t nx, int64_t ny, int nz, Win w,
    BAChain<T> c, BAState<T> st, double* __restrict__ partials, double* __restrict__ totals,
    int flag_base, int n_iter) {
  __shared__ double red[4 * kLvThreads];
  extern __shared__ unsigned char ba_smem[];
  ba_phase_body<T, MODE>(d0, pert, nx, ny, nz, w, c, st, partials, totals, flag_base, 0, n_iter,
                         ba_smem, red, blockIdx.x, gridDim.x);
}

// Fixes mu for the levels that needed a shift and writes the ledger.
template <typename T>
__device__ __forceinline__ void ba_finish_body(const BAState<T>& st) {
  const int nz = st.nz;
  // + the apply sweep; -1 when a persistent phase's grid barrier gave up
  const int sweeps = st.bar[2] ? -1 : st.flags[ba_flag_count<T>(st.R) - 1] + 1;
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
    double mu = __longlong_as_double(0x7ff8000000000000LL);  // NaN: no shift
    if (st.need[z]) {
      mu = st.solver[z].result();
      st.has_mu[z] = 1;
      st.mu[z] = (T)mu;
    }
    if (st.ledger) {
      const int R = st.R;
      double* l = st.ledger + (size_t)ba_ledger_width(R) * z;
      l[0] = st.a0[z];
      l[1] = st.n_loop[z];
      l[2] = st.active[z] ? st.final_d[z] : 0.0;
      l[3] = mu;
      l[4] = sweeps;
      l[5] = st.nsteps[z];
      l[6] = st.has_final[z];
      for (int k = 0; k < R; ++k) {
        l[7 + k] = (double)st.demean[(size_t)z * R + k];
        l[7 + R + k] = (double)st.scale[(size_t)z * R + k];
      }
    }
  }
}

template <typename T>
__global__ void ba_finish_kernel(BAState<T> st) {
  ba_finish_body(st);
}

static size_t ba_state_bytes(int64_t nz, int R, size_t elem) {
  return carve_bytes((size_t)3 * nz, sizeof(int)) +                       // nsteps, has_final, has_mu
         carve_bytes((size_t)nz * (2 * (size_t)R + 4 + kMuCand), elem) +   // chain values
         carve_bytes((size_t)3 * nz, sizeof(double)) +                      // a0, cur_mean, final_d
         carve_bytes((size_t)6 * nz, sizeof(int)) +  // active, still, n_loop, need, applied, fin_stored
         carve_bytes((size_t)nz * sizeof(MuSolver<double>), 1) +
         carve_bytes((size_t)(2 + R + kMuMaxSweeps), sizeof(int)) +
         carve_bytes(4, sizeof(unsigned)) +
         carve_bytes((size_t)ba_ledger_width(R) * nz, sizeof(double)) +     // ledger
         carve_bytes((size_t)nz, sizeof(double)) +                          // mean upload
         carve_bytes((size_t)nz / 4 + 1, sizeof(int)) +                     // grp
         (size_t)32 * 256;  // the 256-byte alignment of every separate carve
}

// The solve's per-level state, carved from a workspace (the ledger too when
// `own_ledger`); false when it does not fit.
template <typename T>
static bool carve_ba_state(Carver& c, int64_t nz, int R, bool own_ledger, BAState<T>& st) {
  st.nsteps = c.take<int>(nz);
  st.has_final = c.take<int>(nz);
  st.has_mu = c.take<int>(nz);
  st.demean = c.take<T>((size_t)nz * (R > 0 ? R : 1));
  st.scale = c.take<T>((size_t)nz * (R > 0 ? R : 1));
  st.final_dm = c.take<T>(nz);
  st.mu = c.take<T>(nz);
  st.mean = c.take<T>(nz);
  st.cand = c.take<T>((size_t)nz * kMuCand);
  st.a0 = c.take<double>(nz);
  st.cur_mean = c.take<double>(nz);
  st.final_d = c.take<double>(nz);
  st.active = c.take<int>(nz);
  st.still = c.take<int>(nz);
  st.n_loop = c.take<int>(nz);
  st.need = c.take<int>(nz);
  st.applied = c.take<int>(nz);
  st.fin_stored = c.take<int>(nz);
  st.grp = c.take<int>(nz / 4 + 1);
  st.solver = c.take<MuSolver<T>>(nz);
  st.flags = c.take<int>((size_t)ba_flag_count<T>(R));
  st.bar = c.take<unsigned>(4);
  st.ledger = own_ledger ? c.take<double>((size_t)ba_ledger_width(R) * nz) : nullptr;
  return st.nsteps && st.has_final && st.has_mu && st.demean && st.scale && st.final_dm &&
         st.mu && st.mean && st.cand && st.a0 && st.cur_mean && st.final_d && st.active &&
         st.still && st.n_loop && st.need && st.applied && st.fin_stored && st.grp &&
         st.solver && st.flags && st.bar && (st.ledger || !own_ledger);
}

template <typename T>
static void set_ba_scalars(BAState<T>& st, int64_t nz, int R, const Win& w, double phi_min,
                           double phi_max) {
  st.R = R;
  st.nz = (int)nz;
  st.spin_limit = g_bar_spin_limit.load();
  st.N = (double)((w.x1 - w.x0) * (w.y1 - w.y0));
  st.width = phi_max - phi_min;
  st.tol_rel = sizeof(T) == 4 ? ldexp(1.0, -20) : ldexp(1.0, -49);
}

template <typename T>
static BAChain<T> ba_chain(const BAState<T>& st, int R, double phi_min, double phi_max) {
  BAChain<T> ch;
  ch.nsteps = st.nsteps;
  ch.demean = st.demean;
  ch.scale = st.scale;
  ch.has_final = st.has_final;
  ch.final_dm = st.final_dm;
  ch.has_mu = st.has_mu;
  ch.mu = st.mu;
  ch.cand = st.cand;
  ch.mean = st.mean;
  ch.run = nullptr;
  ch.applied = st.applied;
  ch.fin_stored = st.fin_stored;
  ch.still = st.still;
  ch.grp = st.grp;
  ch.R = R;
  ch.lo = (T)phi_min;
  ch.hi = (T)phi_max;
  return ch;
}

// Enqueues the whole bounded add on stream s: no host synchronisation and no
// host decision between sweeps.  Vectorised layouts (nz % 4 == 0, 16-byte
// aligned fields): the first sweep, one persistent cooperative launch for the
// rescale loop and one for the shift solve, the apply sweep.  Other layouts:
// a fixed sequence (one stats sweep, R rescale sweeps, kMuMaxSweeps shift
// sweeps, one apply sweep) in which sweeps whose phase has ended return at
// once (their run flag is 0).  mean_dev
// (device, nz doubles) is the level mean profile; the ledger ends in
// st.ledger (device, [nz][5]).
template <typename T>
static int bounded_add_enqueue(int64_t nx, int64_t ny, int64_t nz, T* pert,
                               const double* mean_dev, T* inc, double phi_min,
                               double phi_max, const steam_window_t* window, int R,
                               int record, Carver& c, double** ledger_dev,
                               cudaStream_t s) {
  const LevelMap m = make_map(nz);
  const int64_t ncol = nx * ny;
  const int grid = level_grid(ncol, m);
  const Win w = make_win(window, nx, ny);
  const int Qmax = 2 * kMuCand;
  double* partials = c.take<double>((size_t)grid * Qmax * nz);
  double* totals = c.take<double>((size_t)Qmax * nz);
  BAState<T> st;
  if (!partials || !totals || !carve_ba_state<T>(c, nz, R, true, st))
    return fail(STEAM_ERR_WORKSPACE, "steam_bounded_add: workspace too small");
  set_ba_scalars(st, nz, R, w, phi_min, phi_max);
  *ledger_dev = st.ledger;

  const bool vec4 = nz % 4 == 0 && nz <= 4 * kLvThreads &&
                    ((uintptr_t)pert % 16 == 0) && ((uintptr_t)inc % 16 == 0) &&
                    ba_fold_smem_bytes<T>(nz) <= 200 * 1024;
  st.wb = vec4 ? 1 : 0;
  const size_t ba_sm = vec4 ? ba_fold_smem_bytes<T>(nz) : ba_smem_bytes<T>(nz, R);
  STEAM_REQUIRE(ba_sm <= 200 * 1024, "steam_bounded_add: n_rescale * nz too large");
  const int grid4 = vec4 ? stride_grid((ncol + (kLvThreads / (nz / 4)) - 1) /
                                           (kLvThreads / (nz / 4)), 1, kLvBlocksPerSm)
                         : 0;
  const int sweep_grid = vec4 ? grid4 : grid;
  if (vec4) {
    STEAM_CUDA(cudaFuncSetAttribute(ba_fold_kernel<T, BA_SUMS>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ba_sm));
    STEAM_CUDA(cudaFuncSetAttribute(ba_fold_kernel<T, BA_APPLY>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)ba_fold_param_bytes<T>(nz)));
  } else if (m.packed) {
    STEAM_CUDA(cudaFuncSetAttribute(ba_sweep_kernel<T, BA_STATS, 1>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ba_sm));
    STEAM_CUDA(cudaFuncSetAttribute(ba_sweep_kernel<T, BA_MU, 1>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ba_sm));
    STEAM_CUDA(cudaFuncSetAttribute(ba_sweep_kernel<T, BA_APPLY, 1>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ba_sm));
  } else {
    STEAM_CUDA(cudaFuncSetAttribute(ba_sweep_kernel<T, BA_STATS, kLvMaxJ>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ba_sm));
    STEAM_CUDA(cudaFuncSetAttribute(ba_sweep_kernel<T, BA_MU, kLvMaxJ>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ba_sm));
    STEAM_CUDA(cudaFuncSetAttribute(ba_sweep_kernel<T, BA_APPLY, kLvMaxJ>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ba_sm));
  }
  BAChain<T> ch = ba_chain(st, R, phi_min, phi_max);
  const int lv_blocks = (int)((nz + 255) / 256);

  auto sweep = [&](int mode, const int* run, T* out, int rec) -> int {
    ch.run = run;
    if (mode == BA_SUMS) {
      if (vec4)
        ba_fold_kernel<T, BA_SUMS><<<grid4, kLvThreads, ba_sm, s>>>(
            inc, pert, rec, nx, ny, (int)nz, w, ch, partials);
      else if (m.packed)
        ba_sweep_kernel<T, BA_STATS, 1><<<grid, kLvThreads, ba_sm, s>>>(
            inc, pert, out, rec, nx, ny, m, w, ch, partials);
      else
        ba_sweep_kernel<T, BA_STATS, kLvMaxJ><<<grid, kLvThreads, ba_sm, s>>>(
            inc, pert, out, rec, nx, ny, m, w, ch, partials);
    } else if (mode == BA_STATS) {
      // (the vectorised path runs its statistics and shift sweeps inside
      // ba_phase_kernel)
      if (m.packed)
        ba_sweep_kernel<T, BA_STATS, 1><<<grid, kLvThreads, ba_sm, s>>>(
            inc, pert, out, rec, nx, ny, m, w, ch, partials);
      else
        ba_sweep_kernel<T, BA_STATS, kLvMaxJ><<<grid, kLvThreads, ba_sm, s>>>(
            inc, pert, out, rec, nx, ny, m, w, ch, partials);
    } else if (mode == BA_MU) {
      if (m.packed)
        ba_sweep_kernel<T, BA_MU, 1><<<grid, kLvThreads, ba_sm, s>>>(
            inc, pert, out, rec, nx, ny, m, w, ch, partials);
      else
        ba_sweep_kernel<T, BA_MU, kLvMaxJ><<<grid, kLvThreads, ba_sm, s>>>(
            inc, pert, out, rec, nx, ny, m, w, ch, partials);
    } else {
      if (vec4)
        ba_fold_kernel<T, BA_APPLY><<<grid4, kLvThreads, ba_fold_param_bytes<T>(nz), s>>>(
            inc, pert, rec, nx, ny, (int)nz, w, ch, partials);
      else if (m.packed)
        ba_sweep_kernel<T, BA_APPLY, 1><<<grid, kLvThreads, ba_sm, s>>>(
            inc, pert, out, rec, nx, ny, m, w, ch, partials);
      else
        ba_sweep_kernel<T, BA_APPLY, kLvMaxJ><<<grid, kLvThreads, ba_sm, s>>>(
            inc, pert, out, rec, nx, ny, m, w, ch, partials);
    }
    STEAM_LAUNCH_CHECK("bounded_add sweep");
    return STEAM_OK;
  };
  auto reduce = [&](int nq, const int* run) -> int {
    reduce_partials_if_kernel<<<nq, 256, 0, s>>>(partials, sweep_grid, totals, run);
    STEAM_LAUNCH_CHECK("bounded_add reduce");
    return STEAM_OK;
  };
  int rc;
  ba_init_kernel<T><<<lv_blocks, 256, 0, s>>>(st, mean_dev);
  STEAM_LAUNCH_CHECK("bounded_add init");
  // sweep 0: a0 = mean|d|, mean d
  if ((rc = sweep(BA_SUMS, &st.flags[0], nullptr, 0))) return rc;
  if ((rc = reduce(2 * (int)nz, &st.flags[0]))) return rc;
  ba_a0_kernel<T><<<lv_blocks, 256, 0, s>>>(st, totals);
  STEAM_LAUNCH_CHECK("bounded_add a0");
  // One persistent cooperative launch per phase on the vectorised path (it
  // iterates only as long as a level needs another sweep); the fixed launch
  // sequence otherwise.
  auto phase = [&](int mode, int flag_base, int n_iter) -> int {
    auto kern = mode == BA_MU ? ba_phase_kernel<T, BA_MU> : ba_phase_kernel<T, BA_STATS>;
    STEAM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)ba_sm));
    int per_sm = 0;
    STEAM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLvThreads, ba_sm));
    STEAM_REQUIRE(per_sm >= 1, "steam_bounded_add: a persistent phase does not fit an SM");
    int pgrid = per_sm * sm_count();
    if (pgrid > grid4) pgrid = grid4;
    // A phase is persistent and spends much of its time at grid barriers, so
    // its blocks hold their SMs' slots for the whole loop.  Size it by the
    // work, at least kPhaseMinGroups column groups per block and sweep: a
    // large field still takes every slot, while a small one (an ensemble
    // member) leaves the other SMs to concurrent streams and pays for fewer
    // arrivals at each barrier.
    const int64_t cpb = kLvThreads / (nz / 4);
    const int64_t groups = (ncol + cpb - 1) / cpb;
    const int64_t want = (groups + kPhaseMinGroups - 1) / kPhaseMinGroups;
    if (want < pgrid) pgrid = want > 1 ? (int)want : 1;
    T* d0p = inc;
    T* pp = pert;
    int nzi = (int)nz;
    double* part = partials;
    double* tot = totals;
    void* args[] = {&d0p, &pp, &nx, &ny, &nzi, (void*)&w, (void*)&ch, (void*)&st, &part, &tot,
                    &flag_base, &n_iter};
    STEAM_CUDA(cudaLaunchCooperativeKernel((const void*)kern, dim3(pgrid), dim3(kLvThreads),
                                           args, ba_sm, s));
    count_launch();
    return STEAM_OK;
  };
  // demean / clip / rescale-to-A0 loop
  if (vec4) {
    if (R > 0 && (rc = phase(BA_STATS, 1, R))) return rc;
  } else {
    for (int k = 0; k < R; ++k) {
      if ((rc = sweep(BA_STATS, &st.flags[1 + k], nullptr, 0))) return rc;
      if ((rc = reduce(2 * (int)nz, &st.flags[1 + k]))) return rc;
      ba_loop_kernel<T><<<lv_blocks, 256, 0, s>>>(st, totals, k);
      STEAM_LAUNCH_CHECK("bounded_add loop");
    }
  }
  // zero-mean shift
  ba_mu_init_kernel<T><<<lv_blocks, 256, 0, s>>>(st);
  STEAM_LAUNCH_CHECK("bounded_add mu init");
  if (vec4) {
    if ((rc = phase(BA_MU, 1 + R, kMuMaxSweeps))) return rc;
  } else {
    for (int it = 0; it < kMuMaxSweeps; ++it) {
      const int* run = &st.flags[1 + R + it];
      if ((rc = sweep(BA_MU, run, nullptr, 0))) return rc;
      if ((rc = reduce(Qmax * (int)nz, run))) return rc;
      ba_mu_kernel<T><<<lv_blocks, 256, 0, s>>>(st, totals, it);
      STEAM_LAUNCH_CHECK("bounded_add mu");
    }
  }
  ba_finish_kernel<T><<<lv_blocks, 256, 0, s>>>(st);
  STEAM_LAUNCH_CHECK("bounded_add finish");
  // apply (always runs)
  if ((rc = sweep(BA_APPLY, nullptr, inc, record))) return rc;
  return STEAM_OK;
}

// ---- grouped bounded adds: many fields, one launch per stage ------------------
// An ensemble's members each run a bounded add on fields of their own shape.
// Launched one by one, each solve pays its launch and grid-barrier latency on
// its own; here all of them share one launch per stage: the first sweep and
// the apply sweep over a flat grid in which every field owns a contiguous
// range of blocks, the small per-level kernels over a (levels, fields) grid,
// and each persistent phase as ONE cooperative launch whose blocks split into
// per-field teams, each with its own grid barrier (a team waits only for its
// own field's blocks).  A team's size is its field's share of the co-resident
// capacity (in proportion to its column groups), so every team sweeps about
// the same bytes per block and the phase ends when they all do; a field's
// sums therefore depend on the group it is solved in (the same group gives
// the same bits every time).  Only the vectorised layout (nz % 4 == 0,
// 16-byte aligned fields) is grouped.
constexpr int kGroupFoldGroups = 64;     // column groups per block, every flat sweep

template <typename T>
struct BAGroupRec {
  BAState<T> st;
  BAChain<T> ch;
  T* pert;
  T* inc;
  double* partials;
  double* totals;
  const double* mean;
  Win w;
  int64_t nx, ny;
  int nz;
  int fold_nb;  // blocks of the first and apply sweeps
  int ph_nb;    // blocks of the rescale-loop phase
  int mu_nb;    // blocks of the shift-solve phase
};

// the field that owns block b of a grouped launch: start[p] <= b < start[p + 1]
__device__ __forceinline__ int group_owner(const int* __restrict__ start, int n, int b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(start + mid) <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <typename T>
__global__ void bag_init_kernel(const BAGroupRec<T>* __restrict__ recs) {
  const BAGroupRec<T>& r = recs[blockIdx.y];
  ba_init_body(r.st, r.mean);
}

template <typename T>
__global__ void bag_a0_kernel(const BAGroupRec<T>* __restrict__ recs) {
  const BAGroupRec<T>& r = recs[blockIdx.y];
  ba_a0_body(r.st, r.totals);
}

template <typename T>
__global__ void bag_mu_init_kernel(const BAGroupRec<T>* __restrict__ recs) {
  ba_mu_init_body(recs[blockIdx.y].st);
}

template <typename T>
__global__ void bag_finish_kernel(const BAGroupRec<T>* __restrict__ recs) {
  ba_finish_body(recs[blockIdx.y].st);
}

// totals[row] of the first sweep, rows 2 nz of each field (y: the field)
template <typename T>
__global__ void bag_reduce_kernel(const BAGroupRec<T>* __restrict__ recs) {
  __shared__ double scratch[32];
  const BAGroupRec<T>& r = recs[blockIdx.y];
  const int nb = r.fold_nb;
  for (int row = blockIdx.x; row < 2 * r.nz; row += gridDim.x) {
    const double* src = r.partials + (size_t)row * nb;
    double acc = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += src[i];
    const double sum = block_sum(acc, scratch);
    if (threadIdx.x == 0) r.totals[row] = sum;
  }
}

template <typename T, int MODE>
__global__ void __launch_bounds__(kLvThreads, 4)
    bag_fold_kernel(const BAGroupRec<T>* __restrict__ recs, const int* __restrict__ start,
                    int n) {
  __shared__ double red[4 * kLvThreads];
  extern __shared__ unsigned char ba_smem[];
  const int p = group_owner(start, n, blockIdx.x);
  const BAGroupRec<T>& r = recs[p];
  ba_fold_body<T, MODE, false>(r.inc, r.pert, 0, r.nx, r.ny, r.nz, r.w, r.ch, r.partials,
                               ba_smem, red, blockIdx.x - __ldg(start + p), r.fold_nb);
}

// one cooperative launch of a phase over fields p0 .. p0 + n - 1, iterations
// it0 .. n_iter - 1; start[i]: the first block of field p0 + i
template <typename T, int MODE>
__global__ void __launch_bounds__(kLvThreads, (MODE == BA_MU ? 2 : 3))
    bag_phase_kernel(const BAGroupRec<T>* __restrict__ recs, const int* __restrict__ start,
                     int p0, int n, int flag_base, int it0, int n_iter) {
  __shared__ double red[4 * kLvThreads];
  extern __shared__ unsigned char ba_smem[];
  const int i = group_owner(start, n, blockIdx.x);
  const BAGroupRec<T>& r = recs[p0 + i];
  ba_phase_body<T, MODE>(r.inc, r.pert, r.nx, r.ny, r.nz, r.w, r.ch, r.st, r.partials,
                         r.totals, flag_base, it0, n_iter, ba_smem, red,
                         blockIdx.x - __ldg(start + i), MODE == BA_MU ? r.mu_nb : r.ph_nb);
}

// The persistent phases as flat launches, one iteration at a time: a sweep
// over every field still in the loop (a field whose flag for this iteration
// is 0 has left it: its blocks return at once), the fixed-order sums of each
// field's block partials, and the per-level decision that sets the flag of
// the next iteration.  Every field sweeps at the flat grid's full width, so
// the fields that need more iterations do not hold the others' blocks idle.
template <typename T, int MODE>
__global__ void __launch_bounds__(kLvThreads, 4)
    bag_iter_sweep_kernel(const BAGroupRec<T>* __restrict__ recs, const int* __restrict__ start,
                          int n, int flag_base, int it) {
  __shared__ double red[4 * kLvThreads];
  extern __shared__ unsigned char ba_smem[];
  const int p = group_owner(start, n, blockIdx.x);
  const BAGroupRec<T>& r = recs[p];
  if (r.st.flags[flag_base + it] == 0) return;
  BAChain<T> c = r.ch;
  c.run = nullptr;
  ba_fold_body<T, MODE, false>(r.inc, r.pert, 0, r.nx, r.ny, r.nz, r.w, c, r.partials, ba_smem,
                               red, blockIdx.x - __ldg(start + p), r.fold_nb);
}

template <typename T, int MODE>
__global__ void bag_iter_rows_kernel(const BAGroupRec<T>* __restrict__ recs, int flag_base,
                                     int it) {
  __shared__ double scratch[32];
  constexpr int Q = MODE == BA_MU ? 2 * kMuCand : 2;
  const BAGroupRec<T>& r = recs[blockIdx.y];
  if (r.st.flags[flag_base + it] == 0) return;
  const int nb = r.fold_nb;
  for (int row = blockIdx.x; row < Q * r.nz; row += gridDim.x) {
    const double* src = r.partials + (size_t)row * nb;
    double acc = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) acc += src[i];
    const double sum = block_sum(acc, scratch);
    if (threadIdx.x == 0) r.totals[row] = sum;
  }
}

template <typename T, int MODE>
__global__ void bag_iter_decide_kernel(const BAGroupRec<T>* __restrict__ recs, int flag_base,
                                       int it) {
  const BAGroupRec<T>& r = recs[blockIdx.y];
  const BAState<T>& st = r.st;
  if (st.flags[flag_base + it] == 0) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) st.flags[ba_flag_count<T>(st.R) - 1] += 1;
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < st.nz; z += gridDim.x * blockDim.x) {
    if (MODE == BA_MU)
      ba_mu_level<T, false>(st, r.totals, it, z);
    else
      ba_loop_level<T, false>(st, r.totals, it, z);
  }
}

// iterations of each persistent phase that a grouped solve runs as flat
// launches before its cooperative launches take over (in the 256-member
// ensemble every rescale loop ends within 5 iterations and every shift solve
// within 2; a field that needs more finishes in its cooperative team)
constexpr int kGroupFlatRescaleIters = 6;
constexpr int kGroupFlatMuIters = 3;

struct BAGroupPlan {
  int dtype = 0, n = 0, R = 0;
  int nz_max = 0;
  int fold_blocks = 0;            // total blocks of the flat sweeps
  size_t sm_sums = 0, sm_apply = 0;
  void* recs = nullptr;           // device BAGroupRec<T>[n]
  int* fold_start = nullptr;      // device [n]
  int* ph_start = nullptr;        // device [n]: first block within the field's rescale batch
  int* mu_start = nullptr;        // device [n]: the same for the shift batches
  std::vector<std::array<int, 3>> batches;     // rescale phase: {first field, fields, blocks}
  std::vector<std::array<int, 3>> mu_batches;  // shift phase
};
static std::mutex g_group_mu;
static std::map<void*, BAGroupPlan> g_groups;

// blocks whose partial sums a field's buffers hold: its first sweep's, and
// the most a phase team can get (a share of the co-resident capacity, at most
// one block per kPhaseMinGroups column groups)
static int64_t group_partial_blocks(int64_t groups) {
  const int64_t fold = std::max<int64_t>((groups + kGroupFoldGroups - 1) / kGroupFoldGroups, 1);
  const int64_t team = std::min<int64_t>(
      std::max<int64_t>((groups + kPhaseMinGroups - 1) / kPhaseMinGroups, 1),
      (int64_t)4 * sm_count());
  return std::max(fold, team);
}

static size_t group_state_bytes(const steam_ba_problem_t& q, int R, size_t elem) {
  // state, partials of either sweep kind, totals
  const int64_t nz = q.nz;
  const int64_t ncol = q.nx * q.ny;
  const int64_t cpb = nz > 0 ? kLvThreads / (nz / 4) : 1;
  const int64_t groups = (ncol + cpb - 1) / cpb;
  const int64_t nb = group_partial_blocks(groups);
  return ba_state_bytes(nz, R, elem) +
         carve_bytes((size_t)nb * 2 * kMuCand * nz, sizeof(double)) +
         carve_bytes((size_t)2 * kMuCand * nz, sizeof(double)) + 512;
}

template <typename T>
static size_t group_bytes(int n, const steam_ba_problem_t* q, int R) {
  size_t b = carve_bytes((size_t)n, sizeof(BAGroupRec<T>)) + 3 * carve_bytes((size_t)n, sizeof(int));
  for (int i = 0; i < n; ++i) b += group_state_bytes(q[i], R, sizeof(T));
  return b + 4096;
}

template <typename T>
static int group_prepare(int n, const steam_ba_problem_t* q, int R, void* ws, size_t ws_bytes,
                         int dtype) {
  Carver c(ws, ws_bytes);
  BAGroupPlan plan;
  plan.dtype = dtype;
  plan.n = n;
  plan.R = R;
  plan.recs = c.take<BAGroupRec<T>>((size_t)n);
  plan.fold_start = c.take<int>((size_t)n);
  plan.ph_start = c.take<int>((size_t)n);
  plan.mu_start = c.take<int>((size_t)n);
  if (!plan.recs || !plan.fold_start || !plan.ph_start || !plan.mu_start)
    return fail(STEAM_ERR_WORKSPACE, "steam_bounded_add_group_prepare: workspace too small");
  std::vector<int64_t> groups((size_t)n);
  for (int i = 0; i < n; ++i) {
    const int64_t cpb = kLvThreads / (q[i].nz / 4);
    groups[(size_t)i] = (q[i].nx * q[i].ny + cpb - 1) / cpb;
    plan.nz_max = std::max(plan.nz_max, (int)q[i].nz);
  }
  plan.sm_sums = ba_fold_smem_bytes<T>(plan.nz_max);
  plan.sm_apply = ba_fold_param_bytes<T>(plan.nz_max);
  // co-resident capacity of each cooperative phase
  int caps[2] = {0, 0};
  for (int mode = 0; mode < 2; ++mode) {
    auto kern = mode ? bag_phase_kernel<T, BA_MU> : bag_phase_kernel<T, BA_STATS>;
    STEAM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)plan.sm_sums));
    int per_sm = 0;
    STEAM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kLvThreads,
                                                             plan.sm_sums));
    STEAM_REQUIRE(per_sm >= 1, "steam_bounded_add_group_prepare: a phase does not fit an SM");
    caps[mode] = per_sm * sm_count();
  }
  // Batches of fields, per phase: as few as leave at least 40 % of each
  // batch's slots to deal out beyond one block per field (a batch lasts as
  // long as its slowest field's iterations, so fewer batches win); the
  // fields dealt largest first to the batch with the least work so far.
  // Within a batch a field's team is one block plus its share of the spare
  // slots in proportion to its column groups (at most one block per
  // kPhaseMinGroups groups), so every team sweeps about the same bytes per
  // block.  The fields' records are laid out in the rescale phase's batch
  // order; the shift phase's batches are lists of fields, each contiguous
  // in that order when both phases take the same number of batches.
  auto layout = [&](int cap, std::vector<int>& order, std::vector<int>& team,
                    std::vector<std::vector<int>>& members) -> int {
    const int per_batch = std::max(1, (cap * 3) / 5);
    const int B = std::max(1, (n + per_batch - 1) / per_batch);
    std::vector<int> idx((size_t)n);
    for (int i = 0; i < n; ++i) idx[(size_t)i] = i;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int a, int b) { return groups[(size_t)a] > groups[(size_t)b]; });
    members.assign((size_t)B, {});
    std::vector<int64_t> load((size_t)B, 0);
    for (int i : idx) {
      int best = -1;
      for (int b = 0; b < B; ++b)
        if ((int)members[(size_t)b].size() < cap &&
            (best < 0 || load[(size_t)b] < load[(size_t)best]))
          best = b;
      STEAM_REQUIRE(best >= 0, "steam_bounded_add_group_prepare: too many fields");
      members[(size_t)best].push_back(i);
      load[(size_t)best] += groups[(size_t)i];
    }
    team.assign((size_t)n, 1);
    order.clear();
    for (int b = 0; b < B; ++b) {
      auto& m = members[(size_t)b];
      std::sort(m.begin(), m.end());
      const int64_t spare = cap - (int64_t)m.size();
      for (int i : m) {
        const int64_t g = groups[(size_t)i];
        const int64_t share = 1 + (int64_t)((double)spare * (double)g /
                                            (double)std::max<int64_t>(load[(size_t)b], 1));
        const int64_t useful =
            std::max<int64_t>((g + kPhaseMinGroups - 1) / kPhaseMinGroups, 1);
        team[(size_t)i] = (int)std::min(std::min(share, useful), group_partial_blocks(g));
        order.push_back(i);
      }
    }
    return STEAM_OK;
  };
  std::vector<int> order, team, mu_order, mu_team;
  std::vector<std::vector<int>> members, mu_members;
  int rcl = layout(caps[0], order, team, members);
  if (rcl) return rcl;
  rcl = layout(caps[1], mu_order, mu_team, mu_members);
  if (rcl) return rcl;
  // the fields' records in the rescale phase's batch order
  std::vector<int> pos((size_t)n);
  for (int k = 0; k < n; ++k) pos[(size_t)order[(size_t)k]] = k;
  std::vector<BAGroupRec<T>> recs((size_t)n);
  std::vector<int> fold_start((size_t)n), ph_start((size_t)n), mu_start((size_t)n);
  int fold_total = 0;
  for (int k = 0; k < n; ++k) {
    const int i = order[(size_t)k];
    const steam_ba_problem_t& p = q[i];
    const int64_t nz = p.nz;
    const steam_window_t* win = p.has_window ? &p.window : nullptr;
    BAGroupRec<T>& r = recs[(size_t)k];
    r.w = make_win(win, p.nx, p.ny);
    if (!carve_ba_state<T>(c, nz, R, p.ledger == nullptr, r.st))
      return fail(STEAM_ERR_WORKSPACE, "steam_bounded_add_group_prepare: workspace too small");
    if (p.ledger) r.st.ledger = p.ledger;
    set_ba_scalars(r.st, nz, R, r.w, p.phi_min, p.phi_max);
    r.ch = ba_chain(r.st, R, p.phi_min, p.phi_max);
    const int64_t g = groups[(size_t)i];
    r.fold_nb = (int)std::max<int64_t>((g + kGroupFoldGroups - 1) / kGroupFoldGroups, 1);
    r.ph_nb = team[(size_t)i];
    r.mu_nb = mu_team[(size_t)i];
    r.partials = c.take<double>((size_t)group_partial_blocks(g) * 2 * kMuCand * nz);
    r.totals = c.take<double>((size_t)2 * kMuCand * nz);
    if (!r.partials || !r.totals)
      return fail(STEAM_ERR_WORKSPACE, "steam_bounded_add_group_prepare: workspace too small");
    r.st.wb = 1;
    r.pert = (T*)p.pert;
    r.inc = (T*)p.increment;
    r.mean = p.mean;
    r.nx = p.nx;
    r.ny = p.ny;
    r.nz = (int)nz;
    fold_start[(size_t)k] = fold_total;
    fold_total += r.fold_nb;
  }
  plan.fold_blocks = fold_total;
  int k0 = 0;
  for (size_t b = 0; b < members.size(); ++b) {
    const int nb = (int)members[b].size();
    int blocks = 0;
    for (int k = k0; k < k0 + nb; ++k) {
      ph_start[(size_t)k] = blocks;
      blocks += recs[(size_t)k].ph_nb;
    }
    if (nb > 0) plan.batches.push_back({k0, nb, blocks});
    k0 += nb;
  }
  // the shift phase's batches must be contiguous runs of records: when its
  // layout differs in batch count, its fields take the rescale order and are
  // cut into runs that fit its capacity
  k0 = 0;
  while (k0 < n) {
    int blocks = 0, k = k0;
    while (k < n && blocks + recs[(size_t)k].mu_nb <= caps[1]) {
      mu_start[(size_t)k] = blocks;
      blocks += recs[(size_t)k].mu_nb;
      ++k;
    }
    STEAM_REQUIRE(k > k0, "steam_bounded_add_group_prepare: a team exceeds the capacity");
    plan.mu_batches.push_back({k0, k - k0, blocks});
    k0 = k;
  }
  (void)mu_order;
  (void)mu_members;
  (void)pos;
  STEAM_CUDA(cudaMemcpy(plan.recs, recs.data(), sizeof(BAGroupRec<T>) * (size_t)n,
                        cudaMemcpyHostToDevice));
  STEAM_CUDA(cudaMemcpy(plan.fold_start, fold_start.data(), sizeof(int) * (size_t)n,
                        cudaMemcpyHostToDevice));
  STEAM_CUDA(cudaMemcpy(plan.ph_start, ph_start.data(), sizeof(int) * (size_t)n,
                        cudaMemcpyHostToDevice));
  STEAM_CUDA(cudaMemcpy(plan.mu_start, mu_start.data(), sizeof(int) * (size_t)n,
                        cudaMemcpyHostToDevice));
  STEAM_CUDA(cudaFuncSetAttribute(bag_fold_kernel<T, BA_SUMS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)plan.sm_sums));
  STEAM_CUDA(cudaFuncSetAttribute(bag_fold_kernel<T, BA_APPLY>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)plan.sm_apply));
  STEAM_CUDA(cudaFuncSetAttribute(bag_iter_sweep_kernel<T, BA_STATS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)plan.sm_sums));
  STEAM_CUDA(cudaFuncSetAttribute(bag_iter_sweep_kernel<T, BA_MU>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)plan.sm_sums));
  std::lock_guard<std::mutex> lock(g_group_mu);
  g_groups[ws] = plan;
  return STEAM_OK;
}

template <typename T>
static int group_enqueue(const BAGroupPlan& plan, cudaStream_t s) {
  const auto* recs = (const BAGroupRec<T>*)plan.recs;
  const int n = plan.n, R = plan.R;
  const dim3 lv((unsigned)((plan.nz_max + 255) / 256), (unsigned)n);
  bag_init_kernel<T><<<lv, 256, 0, s>>>(recs);
  STEAM_LAUNCH_CHECK("bounded_add group init");
  bag_fold_kernel<T, BA_SUMS><<<plan.fold_blocks, kLvThreads, plan.sm_sums, s>>>(
      recs, plan.fold_start, n);
  STEAM_LAUNCH_CHECK("bounded_add group sweep");
  bag_reduce_kernel<T><<<dim3((unsigned)std::min(2 * plan.nz_max, 512), (unsigned)n), 256, 0,
                         s>>>(recs);
  STEAM_LAUNCH_CHECK("bounded_add group reduce");
  bag_a0_kernel<T><<<lv, 256, 0, s>>>(recs);
  STEAM_LAUNCH_CHECK("bounded_add group a0");
  auto phase = [&](int mode, int flag_base, int n_iter) -> int {
    // the first iterations as flat launches over the fields still in the loop
    // (most fields leave it within them), the rest, if any field is still in
    // it, as cooperative launches of per-field teams that start there
    const int n_flat = std::min(n_iter, mode == BA_MU ? kGroupFlatMuIters : kGroupFlatRescaleIters);
    const unsigned rows = (unsigned)std::min((mode == BA_MU ? 2 * kMuCand : 2) * plan.nz_max, 16);
    for (int it = 0; it < n_flat; ++it) {
      if (mode == BA_MU) {
        bag_iter_sweep_kernel<T, BA_MU><<<plan.fold_blocks, kLvThreads, plan.sm_sums, s>>>(
            recs, plan.fold_start, n, flag_base, it);
        STEAM_LAUNCH_CHECK("bounded_add group shift sweep");
        bag_iter_rows_kernel<T, BA_MU><<<dim3(rows, (unsigned)n), 256, 0, s>>>(recs, flag_base, it);
        STEAM_LAUNCH_CHECK("bounded_add group shift sums");
        bag_iter_decide_kernel<T, BA_MU><<<lv, 256, 0, s>>>(recs, flag_base, it);
        STEAM_LAUNCH_CHECK("bounded_add group shift step");
      } else {
        bag_iter_sweep_kernel<T, BA_STATS><<<plan.fold_blocks, kLvThreads, plan.sm_sums, s>>>(
            recs, plan.fold_start, n, flag_base, it);
        STEAM_LAUNCH_CHECK("bounded_add group rescale sweep");
        bag_iter_rows_kernel<T, BA_STATS><<<dim3(rows, (unsigned)n), 256, 0, s>>>(recs, flag_base,
                                                                                 it);
        STEAM_LAUNCH_CHECK("bounded_add group rescale sums");
        bag_iter_decide_kernel<T, BA_STATS><<<lv, 256, 0, s>>>(recs, flag_base, it);
        STEAM_LAUNCH_CHECK("bounded_add group rescale step");
      }
    }
    if (n_flat >= n_iter) return STEAM_OK;
    auto kern = mode == BA_MU ? bag_phase_kernel<T, BA_MU> : bag_phase_kernel<T, BA_STATS>;
    const auto& batches = mode == BA_MU ? plan.mu_batches : plan.batches;
    const int* starts = mode == BA_MU ? plan.mu_start : plan.ph_start;
    for (const auto& b : batches) {
      int p0 = b[0], nb = b[1], it0 = n_flat;
      const int* start = starts + p0;
      void* args[] = {(void*)&recs, (void*)&start, &p0, &nb, &flag_base, &it0, &n_iter};
      STEAM_CUDA(cudaLaunchCooperativeKernel((const void*)kern, dim3((unsigned)b[2]),
                                             dim3(kLvThreads), args, plan.sm_sums, s));
      count_launch();
    }
    return STEAM_OK;
  };
  int rc;
  if (R > 0 && (rc = phase(BA_STATS, 1, R))) return rc;
  bag_mu_init_kernel<T><<<lv, 256, 0, s>>>(recs);
  STEAM_LAUNCH_CHECK("bounded_add group mu init");
  if ((rc = phase(BA_MU, 1 + R, kMuMaxSweeps))) return rc;
  bag_finish_kernel<T><<<lv, 256, 0, s>>>(recs);
  STEAM_LAUNCH_CHECK("bounded_add group finish");
  bag_fold_kernel<T, BA_APPLY><<<plan.fold_blocks, kLvThreads, plan.sm_apply, s>>>(
      recs, plan.fold_start, n);
  STEAM_LAUNCH_CHECK("bounded_add group apply");
  return STEAM_OK;
}

// ---- apply-only replay of a recorded bounded add -------------------------------
// steam/simulate.py:3196-3213 (the APPLY-ONLY branch): given the per-level
// chain a solve recorded, the increment is taken through the same demeans,
// clips, scales, final demean and shift with no reduction at all, so any
// subset of the columns (a tile of the world that recorded it) replays to
// the same bits as the solve produced there.
template <typename T>
__global__ void ba_chain_from_ledger_kernel(BAState<T> st, const double* __restrict__ led,
                                            const double* __restrict__ mean_dev) {
  const int nz = st.nz, R = st.R, W = ba_ledger_width(R);
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
    const double* l = led + (size_t)W * z;
    st.nsteps[z] = (int)l[5];
    st.has_final[z] = (int)l[6];
    st.final_dm[z] = (T)l[2];
    const bool hm = !isnan(l[3]);
    st.has_mu[z] = hm ? 1 : 0;
    st.mu[z] = hm ? (T)l[3] : (T)0;
    st.mean[z] = (T)mean_dev[z];
    for (int k = 0; k < kMuCand; ++k) st.cand[(size_t)z * kMuCand + k] = (T)0;
    for (int k = 0; k < R; ++k) {
      st.demean[(size_t)z * R + k] = (T)l[7 + k];
      st.scale[(size_t)z * R + k] = (T)l[7 + R + k];
    }
  }
}

static size_t ba_replay_bytes(int64_t nz, int R, size_t elem) {
  return carve_bytes((size_t)3 * nz, sizeof(int)) +
         carve_bytes((size_t)nz * (2 * (size_t)R + 3 + kMuCand), elem) +
         carve_bytes((size_t)nz, sizeof(double)) +                       // mean upload
         carve_bytes((size_t)ba_ledger_width(R) * nz, sizeof(double)) +  // ledger upload
         (size_t)16 * 256;
}

template <typename T>
static int bounded_add_replay_impl(int64_t nx, int64_t ny, int64_t nz, T* pert,
                                   const double* mean, int mean_on_device, T* inc,
                                   double phi_min, double phi_max, int R, int record,
                                   const double* led, int led_on_device, void* ws,
                                   size_t ws_bytes, cudaStream_t s) {
  Carver c(ws, ws_bytes);
  BAState<T> st{};
  st.nsteps = c.take<int>(nz);
  st.has_final = c.take<int>(nz);
  st.has_mu = c.take<int>(nz);
  st.demean = c.take<T>((size_t)nz * (R > 0 ? R : 1));
  st.scale = c.take<T>((size_t)nz * (R > 0 ? R : 1));
  st.final_dm = c.take<T>(nz);
  st.mu = c.take<T>(nz);
  st.mean = c.take<T>(nz);
  st.cand = c.take<T>((size_t)nz * kMuCand);
  const double* mean_dev = mean;
  const double* led_dev = led;
  if (!mean_on_device) {
    double* up = c.take<double>(nz);
    if (!up) return fail(STEAM_ERR_WORKSPACE, "steam_bounded_add_replay: workspace too small");
    STEAM_CUDA(cudaMemcpyAsync(up, mean, sizeof(double) * nz, cudaMemcpyHostToDevice, s));
    mean_dev = up;
  }
  if (!led_on_device) {
    double* up = c.take<double>((size_t)ba_ledger_width(R) * nz);
    if (!up) return fail(STEAM_ERR_WORKSPACE, "steam_bounded_add_replay: workspace too small");
    STEAM_CUDA(cudaMemcpyAsync(up, led, sizeof(double) * ba_ledger_width(R) * nz,
                               cudaMemcpyHostToDevice, s));
    led_dev = up;
  }
  if (!st.nsteps || !st.has_final || !st.has_mu || !st.demean || !st.scale || !st.final_dm ||
      !st.mu || !st.mean || !st.cand)
    return fail(STEAM_ERR_WORKSPACE, "steam_bounded_add_replay: workspace too small");
  st.R = R;
  st.nz = (int)nz;
  const int lv_blocks = (int)((nz + 255) / 256);
  ba_chain_from_ledger_kernel<T><<<lv_blocks, 256, 0, s>>>(st, led_dev, mean_dev);
  STEAM_LAUNCH_CHECK("bounded_add replay chain");
  BAChain<T> ch{};
  ch.nsteps = st.nsteps;
  ch.demean = st.demean;
  ch.scale = st.scale;
  ch.has_final = st.has_final;
  ch.final_dm = st.final_dm;
  ch.has_mu = st.has_mu;
  ch.mu = st.mu;
  ch.cand = st.cand;
  ch.mean = st.mean;
  ch.run = nullptr;
  ch.R = R;
  ch.lo = (T)phi_min;
  ch.hi = (T)phi_max;
  const LevelMap m = make_map(nz);
  const int grid = level_grid(nx * ny, m);
  const Win w = make_win(nullptr, nx, ny);
  const size_t ba_sm = ba_smem_bytes<T>(nz, R);
  STEAM_REQUIRE(ba_sm <= 200 * 1024, "steam_bounded_add_replay: n_rescale * nz too large");
  if (m.packed) {
    STEAM_CUDA(cudaFuncSetAttribute(ba_sweep_kernel<T, BA_APPLY, 1>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ba_sm));
    ba_sweep_kernel<T, BA_APPLY, 1><<<grid, kLvThreads, ba_sm, s>>>(
        inc, pert, inc, record, nx, ny, m, w, ch, nullptr);
  } else {
    STEAM_CUDA(cudaFuncSetAttribute(ba_sweep_kernel<T, BA_APPLY, kLvMaxJ>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ba_sm));
    ba_sweep_kernel<T, BA_APPLY, kLvMaxJ><<<grid, kLvThreads, ba_sm, s>>>(
        inc, pert, inc, record, nx, ny, m, w, ch, nullptr);
  }
  STEAM_LAUNCH_CHECK("bounded_add replay");
  return STEAM_OK;
}

// Apply-only replay of a recorded projection (steam/simulate.py:3462-3488):
// the levels with a recorded shift become clip(field - mu, lo, hi), the rest
// stay bit-identical.
template <typename T>
static int project_replay_impl(int64_t nx, int64_t ny, int64_t nz, T* pert,
                               const double* mean_1d, double lo, double hi,
                               const double* mu_in, void* ws, size_t ws_bytes,
                               cudaStream_t s) {
  const LevelMap m = make_map(nz);
  const int grid = level_grid(nx * ny, m);
  const Win w = make_win(nullptr, nx, ny);
  Carver c(ws, ws_bytes);
  double* d_mean = c.take<double>(nz);
  int* d_active = c.take<int>(nz);
  double* d_mu = c.take<double>(nz);
  if (!d_mean || !d_active || !d_mu)
    return fail(STEAM_ERR_WORKSPACE, "steam_project_bounds_replay: workspace too small");
  std::vector<double> h_mean(mean_1d, mean_1d + nz), h_mu(nz, 0.0);
  std::vector<int> active(nz, 0);
  bool any = false;
  for (int64_t z = 0; z < nz; ++z) {
    if (std::isnan(mu_in[z])) continue;
    active[z] = 1;
    h_mu[z] = mu_in[z];
    any = true;
  }
  if (!any) return STEAM_OK;
  int rc;
  if ((rc = upload(d_mean, h_mean, s))) return rc;
  if ((rc = upload(d_active, active, s))) return rc;
  if ((rc = upload(d_mu, h_mu, s))) return rc;
  if (m.packed)
    proj_sweep_kernel<T, PJ_APPLY, 1><<<grid, kLvThreads, 0, s>>>(
        pert, d_mean, lo, hi, d_active, d_mu, nullptr, nx, ny, m, w, nullptr);
  else
    proj_sweep_kernel<T, PJ_APPLY, kLvMaxJ><<<grid, kLvThreads, 0, s>>>(
        pert, d_mean, lo, hi, d_active, d_mu, nullptr, nx, ny, m, w, nullptr);
  STEAM_LAUNCH_CHECK("project replay sweep");
  STEAM_CUDA(cudaStreamSynchronize(s));
  return STEAM_OK;
}

template <typename T>
static int project_impl(int64_t nx, int64_t ny, int64_t nz, T* pert,
                        const double* mean_1d, double lo, double hi,
                        const steam_window_t* window, double* mu_out, void* ws,
                        size_t ws_bytes, cudaStream_t s) {
  const LevelMap m = make_map(nz);
  const int64_t ncol = nx * ny;
  const int grid = level_grid(ncol, m);
  const Win w = make_win(window, nx, ny);
  const double N = (double)((w.x1 - w.x0) * (w.y1 - w.y0));
  const int Qmax = 2 * kMuCand;
  Carver c(ws, ws_bytes);
  double* partials = c.take<double>((size_t)grid * Qmax * nz);
  double* totals = c.take<double>((size_t)Qmax * nz);
  double* d_mean = c.take<double>(nz);
  int* d_active = c.take<int>(nz);
  double* d_mu = c.take<double>(nz);
  double* d_cand = c.take<double>((size_t)nz * kMuCand);
  if (!partials || !totals || !d_mean || !d_active || !d_mu || !d_cand)
    return fail(STEAM_ERR_WORKSPACE, "steam_project_bounds: workspace too small");
  std::vector<double> h_mean(mean_1d, mean_1d + nz);
  int rc;
  if ((rc = upload(d_mean, h_mean, s))) return rc;
    if (m.packed)
    proj_sweep_kernel<T, PJ_STATS, 1><<<grid, kLvThreads, 0, s>>>(
      pert, d_mean, lo, hi, nullptr, nullptr, nullptr, nx, ny, m, w, partials);
  else
    proj_sweep_kernel<T, PJ_STATS, kLvMaxJ><<<grid, kLvThreads, 0, s>>>(
      pert, d_mean, lo, hi, nullptr, nullptr, nullptr, nx, ny, m, w, partials);
  STEAM_LAUNCH_CHECK("project stats sweep");
  {
    dim3 g2((unsigned)((nz + 127) / 128), 3);
    reduce_minmax_kernel<<<g2, 128, 0, s>>>(partials, grid, (int)nz, totals);
    STEAM_LAUNCH_CHECK("project minmax reduce");
  }
  std::vector<double> tot;
  if ((rc = fetch(tot, totals, 3 * nz, s))) return rc;
  std::vector<int> active(nz, 0);
  std::vector<double> target(nz, 0.0), mu(nz, std::numeric_limits<double>::quiet_NaN());
  bool any = false;
  for (int64_t z = 0; z < nz; ++z) {
    if (tot[nz + z] < lo || tot[2 * nz + z] > hi) {
      active[z] = 1;
      any = true;
      target[z] = tot[z] / N;
    }
  }
  if (mu_out)
    for (int64_t z = 0; z < nz; ++z) mu_out[z] = mu[z];
  if (!any) return STEAM_OK;
  if ((rc = upload(d_active, active, s))) return rc;
  const double width = hi - lo;
  std::vector<MuSolver<double>> solver(nz);
  for (int64_t z = 0; z < nz; ++z)
    if (active[z]) solver[z].init(width, 1e-12 * width);
  std::vector<double> cands((size_t)nz * kMuCand, 0.0);
  for (int it = 0; it < 80; ++it) {
    bool pending = false;
    for (int64_t z = 0; z < nz; ++z) {
      if (!active[z] || solver[z].done) continue;
      pending = true;
      solver[z].candidates(&cands[z * kMuCand]);
    }
    if (!pending) break;
    if ((rc = upload(d_cand, cands, s))) return rc;
        if (m.packed)
      proj_sweep_kernel<T, PJ_MU, 1><<<grid, kLvThreads, 0, s>>>(
        pert, d_mean, lo, hi, d_active, nullptr, d_cand, nx, ny, m, w, partials);
    else
      proj_sweep_kernel<T, PJ_MU, kLvMaxJ><<<grid, kLvThreads, 0, s>>>(
        pert, d_mean, lo, hi, d_active, nullptr, d_cand, nx, ny, m, w, partials);
    STEAM_LAUNCH_CHECK("project mu sweep");
    if ((rc = reduce_partials(partials, grid, Qmax * (int)nz, totals, s))) return rc;
    if ((rc = fetch(tot, totals, (size_t)Qmax * nz, s))) return rc;
    for (int64_t z = 0; z < nz; ++z) {
      if (!active[z] || solver[z].done) continue;
      double mv[kMuCand], sl[kMuCand];
      for (int k = 0; k < kMuCand; ++k) {
        mv[k] = tot[(size_t)(2 * k) * nz + z] / N - target[z];
        sl[k] = -tot[(size_t)(2 * k + 1) * nz + z] / N;
      }
      solver[z].update(&cands[z * kMuCand], mv, sl);
    }
  }
  for (int64_t z = 0; z < nz; ++z)
    if (active[z]) mu[z] = solver[z].result();
  std::vector<double> h_mu(nz, 0.0);
  for (int64_t z = 0; z < nz; ++z) h_mu[z] = active[z] ? mu[z] : 0.0;
  if ((rc = upload(d_mu, h_mu, s))) return rc;
    if (m.packed)
    proj_sweep_kernel<T, PJ_APPLY, 1><<<grid, kLvThreads, 0, s>>>(
      pert, d_mean, lo, hi, d_active, d_mu, nullptr, nx, ny, m, w, partials);
  else
    proj_sweep_kernel<T, PJ_APPLY, kLvMaxJ><<<grid, kLvThreads, 0, s>>>(
      pert, d_mean, lo, hi, d_active, d_mu, nullptr, nx, ny, m, w, partials);
  STEAM_LAUNCH_CHECK("project apply sweep");
  STEAM_CUDA(cudaStreamSynchronize(s));
  if (mu_out)
    for (int64_t z = 0; z < nz; ++z) mu_out[z] = mu[z];
  return STEAM_OK;
}

}  // namespace steam

using namespace steam;

extern "C" size_t steam_level_sums_workspace_bytes(int64_t nz) {
  return level_partial_bytes(nz, 3);
}

extern "C" int steam_level_sums(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                const void* field,
                                const steam_window_t* window, double* sums_out,
                                void* workspace, size_t workspace_bytes,
                                steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "steam_level_sums: negative extent");
  STEAM_REQUIRE(nz <= kLvThreads * kLvMaxJ, "steam_level_sums: nz above 1024");
  STEAM_REQUIRE(sums_out != nullptr, "steam_level_sums: null sums_out");
  int rc = check_win(window, nx, ny, "steam_level_sums");
  if (rc) return rc;
  if (nz == 0) return STEAM_OK;
  const Win w = make_win(window, nx, ny);
  const double cells = (double)((w.x1 - w.x0) * (w.y1 - w.y0));
  if (nx * ny == 0) {
    for (int64_t z = 0; z < nz; ++z) {
      sums_out[4 * z] = sums_out[4 * z + 1] = sums_out[4 * z + 2] = 0.0;
      sums_out[4 * z + 3] = cells;
    }
    return STEAM_OK;
  }
  STEAM_REQUIRE(field != nullptr, "steam_level_sums: null field");
  const LevelMap m = make_map(nz);
  const int grid = level_grid(nx * ny, m);
  Carver c(workspace, workspace_bytes);
  double* partials = c.take<double>((size_t)grid * 3 * nz);
  double* totals = c.take<double>((size_t)3 * nz);
  if (!partials || !totals)
    return fail(STEAM_ERR_WORKSPACE, "steam_level_sums: workspace too small");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
        if (m.packed)
      level_sums_kernel<float, 1><<<grid, kLvThreads, 0, s>>>((const float*)field, nx,
                                                         ny, m, w, partials);
    else
      level_sums_kernel<float, kLvMaxJ><<<grid, kLvThreads, 0, s>>>((const float*)field, nx,
                                                         ny, m, w, partials);
  else if (dtype == STEAM_F64)
        if (m.packed)
      level_sums_kernel<double, 1><<<grid, kLvThreads, 0, s>>>(
        (const double*)field, nx, ny, m, w, partials);
    else
      level_sums_kernel<double, kLvMaxJ><<<grid, kLvThreads, 0, s>>>(
        (const double*)field, nx, ny, m, w, partials);
  else
    return fail(STEAM_ERR_ARG, "steam_level_sums: bad dtype");
  STEAM_LAUNCH_CHECK("steam_level_sums");
  rc = reduce_partials(partials, grid, 3 * (int)nz, totals, s);
  if (rc) return rc;
  std::vector<double> h;
  rc = fetch(h, totals, 3 * nz, s);
  if (rc) return rc;
  for (int64_t z = 0; z < nz; ++z) {
    sums_out[4 * z + 0] = h[z];
    sums_out[4 * z + 1] = h[nz + z];
    sums_out[4 * z + 2] = h[2 * nz + z];
    sums_out[4 * z + 3] = cells;
  }
  return STEAM_OK;
}

static bool pattern_vec_ok(int64_t nz) { return nz % 4 == 0 && nz >= 4 && nz <= 4 * kLvThreads; }

static int pattern_vec_grid(int64_t nx, int64_t ny, int64_t nz) {
  const int64_t cpb = kLvThreads / (nz / 4);
  return stride_grid((nx * ny + cpb - 1) / cpb, 1, kLvBlocksPerSm);
}

extern "C" size_t steam_scalar_pattern_workspace_bytes(int64_t nx, int64_t ny, int64_t nz) {
  size_t b = level_partial_bytes(nz, 2) + 8 * carve_bytes(nz, sizeof(double));
  if (pattern_vec_ok(nz)) {
    const size_t m = carve_bytes((size_t)pattern_vec_grid(nx, ny, nz) * 2 * nz, sizeof(double)) +
                     carve_bytes((size_t)2 * nz, sizeof(double)) + 8 * carve_bytes(nz, sizeof(double));
    b = m > b ? m : b;
  }
  return b;
}

// Per-level vectors of the pattern kernels, [6][nz] in T: mean, the three
// np.gradient coefficients (indexed z - 1), aspect, taper buffer; and the
// z scalars of PatternArgs.
template <typename T>
static void pattern_vectors(int64_t nz, const double* mean_1d, const double* z_coords,
                            const double* aspect, const double* bbuf, std::vector<T>& h,
                            PatternArgs<T>& a) {
  std::vector<T> zc(nz), dz(nz > 1 ? nz - 1 : 0);
  for (int64_t z = 0; z < nz; ++z) zc[z] = (T)z_coords[z];
  for (int64_t z = 0; z + 1 < nz; ++z) dz[z] = zc[z + 1] - zc[z];
  bool uniform = true;
  for (int64_t z = 1; z + 1 < nz; ++z)
    if (dz[z] != dz[0]) uniform = false;
  h.assign((size_t)6 * nz, (T)0);
  for (int64_t z = 0; z < nz; ++z) {
    h[z] = mean_1d ? (T)mean_1d[z] : (T)0;
    h[4 * nz + z] = aspect ? (T)aspect[z] : (T)0;
    h[5 * nz + z] = bbuf ? (T)bbuf[z] : (T)1;
  }
  if (!uniform) {
    for (int64_t z = 0; z + 2 < nz; ++z) {
      T d1 = dz[z], d2 = dz[z + 1];
      h[nz + z] = -(d2) / (d1 * (d1 + d2));
      h[2 * nz + z] = (d2 - d1) / (d1 * d2);
      h[3 * nz + z] = d1 / (d2 * (d1 + d2));
    }
  }
  a.two_dz = uniform ? (T)2 * dz[0] : (T)0;
  a.dz_first = dz[0];
  a.dz_last = dz[nz - 2];
  a.uniform_z = uniform ? 1 : 0;
}

// Launches the pattern kernel and the per-level reduction into totals
// (device, [2][nz]: sum |W|, count W != 0).
template <typename T>
static int pattern_launch(int64_t nx, int64_t ny, int64_t nz, const T* pert, const T* d_vec,
                          const T* prod, const PatternArgs<T>& a, T* out,
                          const steam_window_t* window, double* partials, double* totals,
                          int grid, bool vec, cudaStream_t s) {
  const LevelMap m = make_map(nz);
  const Win w = make_win(window, nx, ny);
  if (vec) {
    if (a.uniform_z)
      pattern_vec_kernel<T, true><<<grid, kLvThreads, 0, s>>>(pert, d_vec, prod, nx, ny, (int)nz,
                                                              w, a, out, partials);
    else
      pattern_vec_kernel<T, false><<<grid, kLvThreads, 0, s>>>(pert, d_vec, prod, nx, ny,
                                                               (int)nz, w, a, out, partials);
  } else if (m.packed)
    pattern_kernel<T, 1><<<grid, kLvThreads, 0, s>>>(
      pert, d_vec, prod, d_vec + nz, d_vec + 2 * nz, d_vec + 3 * nz,
      d_vec + 4 * nz, d_vec + 5 * nz, nx, ny, m, w, a, out, partials);
  else
    pattern_kernel<T, kLvMaxJ><<<grid, kLvThreads, 0, s>>>(
      pert, d_vec, prod, d_vec + nz, d_vec + 2 * nz, d_vec + 3 * nz,
      d_vec + 4 * nz, d_vec + 5 * nz, nx, ny, m, w, a, out, partials);
  STEAM_LAUNCH_CHECK("steam_scalar_pattern");
  return reduce_partials(partials, grid, 2 * (int)nz, totals, s);
}

template <typename T>
static bool pattern_use_vec(int64_t nz, const T* pert, const T* out, const T* prod) {
  return pattern_vec_ok(nz) && ((uintptr_t)pert % 16 == 0) && ((uintptr_t)out % 16 == 0) &&
         (!prod || (uintptr_t)prod % 16 == 0);
}

template <typename T>
static int pattern_impl(int64_t nx, int64_t ny, int64_t nz, const T* pert,
                        const double* mean_1d, const T* prod, double s_scale,
                        double dx, double dy, const double* z_coords,
                        const double* aspect, const double* bbuf,
                        double phi_min, double phi_max, T* out,
                        const steam_window_t* window, double* sums_out,
                        const double* s_scale_dev, const T* vecs_dev, double* sums_dev,
                        void* ws, size_t ws_bytes, cudaStream_t s) {
  const LevelMap m = make_map(nz);
  const bool vec = pattern_use_vec<T>(nz, pert, out, prod);
  const int grid = vec ? pattern_vec_grid(nx, ny, nz) : level_grid(nx * ny, m);
  Carver c(ws, ws_bytes);
  double* partials = c.take<double>((size_t)grid * 2 * nz);
  double* totals = c.take<double>((size_t)2 * nz);
  T* d_vec = c.take<T>((size_t)6 * nz);
  if (!partials || !totals || !d_vec)
    return fail(STEAM_ERR_WORKSPACE, "steam_scalar_pattern: workspace too small");
  std::vector<T> h;
  PatternArgs<T> a;
  pattern_vectors<T>(nz, mean_1d, z_coords, aspect, bbuf, h, a);
  a.two_dx = (T)(2 * dx);
  a.two_dy = (T)(2 * dy);
  a.lo = (T)phi_min;
  a.span = (T)(phi_max - phi_min);
  a.s_scale = (T)s_scale;
  a.s_scale_dev = s_scale_dev;
  a.inv_two_dx = (T)1 / a.two_dx;
  a.inv_two_dy = (T)1 / a.two_dy;
  a.inv_two_dz = a.uniform_z ? (T)1 / a.two_dz : (T)0;
  a.inv_dz_first = (T)1 / a.dz_first;
  a.inv_dz_last = (T)1 / a.dz_last;
  a.has_prod = prod != nullptr;
  a.has_taper = bbuf != nullptr;
  int rc;
  if (vecs_dev) {
    d_vec = const_cast<T*>(vecs_dev);
  } else if ((rc = upload(d_vec, h, s))) {
    return rc;
  }
  if (sums_dev) totals = sums_dev;
  rc = pattern_launch<T>(nx, ny, nz, pert, d_vec, prod, a, out, window, partials, totals, grid,
                         vec, s);
  if (rc || sums_dev) return rc;
  std::vector<double> t;
  rc = fetch(t, totals, 2 * nz, s);
  if (rc) return rc;
  for (int64_t z = 0; z < nz; ++z) {
    sums_out[2 * z] = t[z];
    sums_out[2 * z + 1] = t[nz + z];
  }
  return STEAM_OK;
}

extern "C" int steam_scalar_pattern(
    int dtype, int64_t nx, int64_t ny, int64_t nz, const void* pert,
    const double* mean_1d, const void* product, double s_scale, double dx,
    double dy, const double* z_coords, const double* aspect,
    const double* buffer_b, double phi_min, double phi_max, void* w_out,
    const steam_window_t* window, double* level_sums_out, void* workspace,
    size_t workspace_bytes, steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 1 && ny >= 1, "steam_scalar_pattern: empty horizontal extent");
  STEAM_REQUIRE(nz >= 2, "steam_scalar_pattern: the z gradient needs nz >= 2");
  STEAM_REQUIRE(nz <= kLvThreads * kLvMaxJ, "steam_scalar_pattern: nz above 1024");
  STEAM_REQUIRE(pert && w_out && mean_1d && z_coords && aspect && level_sums_out,
                "steam_scalar_pattern: null pointer");
  int rc = check_win(window, nx, ny, "steam_scalar_pattern");
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    return pattern_impl<float>(nx, ny, nz, (const float*)pert, mean_1d,
                               (const float*)product, s_scale, dx, dy, z_coords,
                               aspect, buffer_b, phi_min, phi_max,
                               (float*)w_out, window, level_sums_out, nullptr, nullptr,
                               nullptr, workspace, workspace_bytes, s);
  if (dtype == STEAM_F64)
    return pattern_impl<double>(nx, ny, nz, (const double*)pert, mean_1d,
                                (const double*)product, s_scale, dx, dy,
                                z_coords, aspect, buffer_b, phi_min, phi_max,
                                (double*)w_out, window, level_sums_out, nullptr, nullptr,
                                nullptr, workspace, workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_scalar_pattern: bad dtype");
}

extern "C" int steam_scalar_pattern_vectors(int dtype, int64_t nz, const double* mean_1d,
                                            const double* z_coords, const double* aspect,
                                            const double* buffer_b, void* vecs_dev,
                                            steam_stream_t stream) {
  STEAM_REQUIRE(nz >= 2 && nz <= kLvThreads * kLvMaxJ,
                "steam_scalar_pattern_vectors: nz outside [2, 1024]");
  STEAM_REQUIRE(mean_1d && z_coords && aspect && vecs_dev,
                "steam_scalar_pattern_vectors: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32) {
    std::vector<float> h;
    PatternArgs<float> a;
    pattern_vectors<float>(nz, mean_1d, z_coords, aspect, buffer_b, h, a);
    STEAM_CUDA(cudaMemcpyAsync(vecs_dev, h.data(), sizeof(float) * h.size(),
                               cudaMemcpyHostToDevice, s));
  } else if (dtype == STEAM_F64) {
    std::vector<double> h;
    PatternArgs<double> a;
    pattern_vectors<double>(nz, mean_1d, z_coords, aspect, buffer_b, h, a);
    STEAM_CUDA(cudaMemcpyAsync(vecs_dev, h.data(), sizeof(double) * h.size(),
                               cudaMemcpyHostToDevice, s));
  } else {
    return fail(STEAM_ERR_ARG, "steam_scalar_pattern_vectors: bad dtype");
  }
  STEAM_CUDA(cudaStreamSynchronize(s));
  return STEAM_OK;
}

extern "C" int steam_scalar_pattern_async(
    int dtype, int64_t nx, int64_t ny, int64_t nz, const void* pert, const void* vecs_dev,
    const void* product, const double* s_scale_dev, double dx, double dy,
    const double* z_coords, int32_t has_taper, double phi_min, double phi_max, void* w_out,
    const steam_window_t* window, double* level_sums_dev, void* workspace,
    size_t workspace_bytes, steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 1 && ny >= 1, "steam_scalar_pattern_async: empty horizontal extent");
  STEAM_REQUIRE(nz >= 2, "steam_scalar_pattern_async: the z gradient needs nz >= 2");
  STEAM_REQUIRE(nz <= kLvThreads * kLvMaxJ, "steam_scalar_pattern_async: nz above 1024");
  STEAM_REQUIRE(pert && vecs_dev && w_out && z_coords && level_sums_dev,
                "steam_scalar_pattern_async: null pointer");
  STEAM_REQUIRE(!product || s_scale_dev,
                "steam_scalar_pattern_async: a product needs s_scale_dev");
  int rc = check_win(window, nx, ny, "steam_scalar_pattern_async");
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  // the vectors are given; only the z scalars are taken from z_coords
  std::vector<double> zeros(nz, 0.0), ones(nz, 1.0);
  const double* bb = has_taper ? ones.data() : nullptr;
  if (dtype == STEAM_F32)
    return pattern_impl<float>(nx, ny, nz, (const float*)pert, zeros.data(),
                               (const float*)product, 1.0, dx, dy, z_coords, zeros.data(), bb,
                               phi_min, phi_max, (float*)w_out, window, nullptr, s_scale_dev,
                               (const float*)vecs_dev, level_sums_dev, workspace,
                               workspace_bytes, s);
  if (dtype == STEAM_F64)
    return pattern_impl<double>(nx, ny, nz, (const double*)pert, zeros.data(),
                                (const double*)product, 1.0, dx, dy, z_coords, zeros.data(),
                                bb, phi_min, phi_max, (double*)w_out, window, nullptr,
                                s_scale_dev, (const double*)vecs_dev, level_sums_dev,
                                workspace, workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_scalar_pattern_async: bad dtype");
}

// pre (device, [2][nz] in T) for the second convolution's input scaling:
// pre[0][z] = the level mean |W| rounded to T (1 where it is not positive),
// pre[1][z] = mul_dev[z] rounded to T (steam/simulate.py:1989-1992).
template <typename T>
__global__ void pattern_norm_kernel(int nz, const double* __restrict__ sums,
                                    const double* __restrict__ mul, T* __restrict__ pre) {
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
    const double cnt = sums[nz + z];
    const T mean = (T)(sums[z] / (cnt > 1.0 ? cnt : 1.0));
    pre[z] = mean > (T)0 ? mean : (T)1;
    pre[nz + z] = (T)mul[z];
  }
}

extern "C" int steam_pattern_norm_async(int dtype, int64_t nz, const double* level_sums_dev,
                                        const double* mul_dev, void* pre_dev,
                                        steam_stream_t stream) {
  STEAM_REQUIRE(nz >= 1 && level_sums_dev && mul_dev && pre_dev,
                "steam_pattern_norm_async: bad argument");
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = (int)((nz + 255) / 256);
  if (dtype == STEAM_F32)
    pattern_norm_kernel<float><<<grid, 256, 0, s>>>((int)nz, level_sums_dev, mul_dev,
                                                    (float*)pre_dev);
  else if (dtype == STEAM_F64)
    pattern_norm_kernel<double><<<grid, 256, 0, s>>>((int)nz, level_sums_dev, mul_dev,
                                                     (double*)pre_dev);
  else
    return fail(STEAM_ERR_ARG, "steam_pattern_norm_async: bad dtype");
  STEAM_LAUNCH_CHECK("steam_pattern_norm_async");
  return STEAM_OK;
}

extern "C" size_t steam_bounded_add_workspace_bytes(int64_t nz, int32_t n_rescale) {
  const int R = n_rescale > 0 ? n_rescale : 1;
  return level_partial_bytes(nz, 2 * kMuCand) + ba_state_bytes(nz, R, sizeof(double));
}

static int bounded_add_check(int64_t nx, int64_t ny, int64_t nz, int32_t n_rescale,
                             double phi_min, double phi_max, const steam_window_t* window,
                             const char* who) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, std::string(who) + ": negative extent");
  STEAM_REQUIRE(nz <= kLvThreads * kLvMaxJ, std::string(who) + ": nz above 1024");
  STEAM_REQUIRE(n_rescale >= 0 && n_rescale <= 64, std::string(who) + ": n_rescale out of range");
  STEAM_REQUIRE(phi_max > phi_min, std::string(who) + ": phi_max must exceed phi_min");
  int rc = check_win(window, nx, ny, who);
  if (rc) return rc;
  if (window) {
    STEAM_REQUIRE(window->x1 > window->x0 && window->y1 > window->y0,
                  std::string(who) + ": empty window");
  }
  return STEAM_OK;
}

template <typename T>
static int bounded_add_entry(int64_t nx, int64_t ny, int64_t nz, T* pert,
                             const double* mean_1d, int mean_on_device, T* inc,
                             double phi_min, double phi_max, const steam_window_t* window,
                             int R, int record, double* ledger_host, double* ledger_dev,
                             void* ws, size_t ws_bytes, cudaStream_t s) {
  Carver c(ws, ws_bytes);
  const double* mean_dev = mean_1d;
  if (!mean_on_device) {
    double* up = c.take<double>(nz);
    if (!up) return fail(STEAM_ERR_WORKSPACE, "steam_bounded_add: workspace too small");
    STEAM_CUDA(cudaMemcpyAsync(up, mean_1d, sizeof(double) * nz, cudaMemcpyHostToDevice, s));
    mean_dev = up;
  }
  double* led = nullptr;
  int rc = bounded_add_enqueue<T>(nx, ny, nz, pert, mean_dev, inc, phi_min, phi_max, window, R,
                                  record, c, &led, s);
  if (rc) return rc;
  const size_t led_bytes = sizeof(double) * ba_ledger_width(R) * nz;
  if (ledger_dev)
    STEAM_CUDA(cudaMemcpyAsync(ledger_dev, led, led_bytes, cudaMemcpyDeviceToDevice, s));
  if (ledger_host) {
    STEAM_CUDA(cudaMemcpyAsync(ledger_host, led, led_bytes, cudaMemcpyDeviceToHost, s));
    STEAM_CUDA(cudaStreamSynchronize(s));
    if (nz > 0 && ledger_host[4] < 0)
      return fail(STEAM_ERR_CUDA, "steam_bounded_add: a persistent phase gave up at a grid "
                                  "barrier (its blocks waited past the spin limit); the "
                                  "perturbation is partly updated");
  }
  return STEAM_OK;
}

extern "C" int steam_bounded_add(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                 void* pert, const double* mean_1d,
                                 void* increment, double phi_min,
                                 double phi_max, const steam_window_t* window,
                                 int32_t n_rescale, int32_t record_applied,
                                 double* ledger_out, void* workspace,
                                 size_t workspace_bytes,
                                 steam_stream_t stream) {
  int rc = bounded_add_check(nx, ny, nz, n_rescale, phi_min, phi_max, window,
                             "steam_bounded_add");
  if (rc) return rc;
  if (nx * ny * nz == 0) return STEAM_OK;
  STEAM_REQUIRE(pert && increment && mean_1d, "steam_bounded_add: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    rc = bounded_add_entry<float>(nx, ny, nz, (float*)pert, mean_1d, 0, (float*)increment,
                                  phi_min, phi_max, window, n_rescale, record_applied,
                                  ledger_out, nullptr, workspace, workspace_bytes, s);
  else if (dtype == STEAM_F64)
    rc = bounded_add_entry<double>(nx, ny, nz, (double*)pert, mean_1d, 0, (double*)increment,
                                   phi_min, phi_max, window, n_rescale, record_applied,
                                   ledger_out, nullptr, workspace, workspace_bytes, s);
  else
    return fail(STEAM_ERR_ARG, "steam_bounded_add: bad dtype");
  if (rc) return rc;
  if (!ledger_out) STEAM_CUDA(cudaStreamSynchronize(s));
  return STEAM_OK;
}

extern "C" int steam_set_barrier_spin_limit(int64_t polls) {
  STEAM_REQUIRE(polls >= 0, "steam_set_barrier_spin_limit: negative poll count");
  g_bar_spin_limit.store(polls == 0 ? kBarSpinLimit : (long long)polls);
  return STEAM_OK;
}

extern "C" int steam_bounded_add_async(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                       void* pert, const double* mean_dev, void* increment,
                                       double phi_min, double phi_max,
                                       const steam_window_t* window, int32_t n_rescale,
                                       int32_t record_applied, double* ledger_dev,
                                       void* workspace, size_t workspace_bytes,
                                       steam_stream_t stream) {
  int rc = bounded_add_check(nx, ny, nz, n_rescale, phi_min, phi_max, window,
                             "steam_bounded_add_async");
  if (rc) return rc;
  if (nx * ny * nz == 0) return STEAM_OK;
  STEAM_REQUIRE(pert && increment && mean_dev, "steam_bounded_add_async: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    return bounded_add_entry<float>(nx, ny, nz, (float*)pert, mean_dev, 1, (float*)increment,
                                    phi_min, phi_max, window, n_rescale, record_applied,
                                    nullptr, ledger_dev, workspace, workspace_bytes, s);
  if (dtype == STEAM_F64)
    return bounded_add_entry<double>(nx, ny, nz, (double*)pert, mean_dev, 1,
                                     (double*)increment, phi_min, phi_max, window, n_rescale,
                                     record_applied, nullptr, ledger_dev, workspace,
                                     workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_bounded_add_async: bad dtype");
}

static int group_check(int dtype, int32_t n, const steam_ba_problem_t* q, int32_t R) {
  STEAM_REQUIRE(dtype == STEAM_F32 || dtype == STEAM_F64,
                "steam_bounded_add_group: bad dtype");
  STEAM_REQUIRE(n >= 1 && q != nullptr, "steam_bounded_add_group: no fields");
  // the per-field launches index fields by blockIdx.y
  STEAM_REQUIRE(n <= 65535, "steam_bounded_add_group: more than 65535 fields");
  STEAM_REQUIRE(R >= 0 && R <= 64, "steam_bounded_add_group: n_rescale out of range");
  const size_t elem = dtype == STEAM_F64 ? 8 : 4;
  for (int i = 0; i < n; ++i) {
    const steam_ba_problem_t& p = q[i];
    const std::string who = "steam_bounded_add_group: field " + std::to_string(i);
    STEAM_REQUIRE(p.nx >= 1 && p.ny >= 1 && p.nz >= 4, who + ": empty or thinner than 4 levels");
    STEAM_REQUIRE(p.nz % 4 == 0 && p.nz <= 4 * kLvThreads,
                  who + ": nz must be a multiple of 4, at most 1024");
    STEAM_REQUIRE(p.pert && p.increment && p.mean, who + ": null pointer");
    STEAM_REQUIRE((uintptr_t)p.pert % 16 == 0 && (uintptr_t)p.increment % 16 == 0,
                  who + ": fields must be 16-byte aligned");
    STEAM_REQUIRE(p.phi_max > p.phi_min, who + ": phi_max must exceed phi_min");
    STEAM_REQUIRE((elem == 4 ? ba_fold_smem_bytes<float>(p.nz) : ba_fold_smem_bytes<double>(p.nz)) <=
                      200 * 1024,
                  who + ": nz too large");
    if (p.has_window) {
      int rc = check_win(&p.window, p.nx, p.ny, who.c_str());
      if (rc) return rc;
      STEAM_REQUIRE(p.window.x1 > p.window.x0 && p.window.y1 > p.window.y0,
                    who + ": empty window");
    }
  }
  return STEAM_OK;
}

extern "C" size_t steam_bounded_add_group_workspace_bytes(int dtype, int32_t n,
                                                          const steam_ba_problem_t* problems,
                                                          int32_t n_rescale) {
  if (n < 1 || !problems) return 0;
  return dtype == STEAM_F64 ? group_bytes<double>(n, problems, n_rescale)
                            : group_bytes<float>(n, problems, n_rescale);
}

extern "C" int steam_bounded_add_group_prepare(int dtype, int32_t n,
                                               const steam_ba_problem_t* problems,
                                               int32_t n_rescale, void* workspace,
                                               size_t workspace_bytes) {
  int rc = group_check(dtype, n, problems, n_rescale);
  if (rc) return rc;
  STEAM_REQUIRE(workspace != nullptr, "steam_bounded_add_group_prepare: null workspace");
  if (dtype == STEAM_F32)
    return group_prepare<float>(n, problems, n_rescale, workspace, workspace_bytes, dtype);
  return group_prepare<double>(n, problems, n_rescale, workspace, workspace_bytes, dtype);
}

extern "C" int steam_bounded_add_group_async(void* workspace, steam_stream_t stream) {
  BAGroupPlan plan;
  {
    std::lock_guard<std::mutex> lock(g_group_mu);
    auto it = g_groups.find(workspace);
    STEAM_REQUIRE(it != g_groups.end(),
                  "steam_bounded_add_group_async: workspace holds no prepared group");
    plan = it->second;
  }
  cudaStream_t s = (cudaStream_t)stream;
  return plan.dtype == STEAM_F32 ? group_enqueue<float>(plan, s) : group_enqueue<double>(plan, s);
}

extern "C" int steam_bounded_add_group_release(void* workspace) {
  std::lock_guard<std::mutex> lock(g_group_mu);
  g_groups.erase(workspace);
  return STEAM_OK;
}

extern "C" int steam_project_bounds(int dtype, int64_t nx, int64_t ny,
                                    int64_t nz, void* pert,
                                    const double* mean_1d, double phi_min,
                                    double phi_max,
                                    const steam_window_t* window,
                                    double* mu_out, void* workspace,
                                    size_t workspace_bytes,
                                    steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "steam_project_bounds: negative extent");
  STEAM_REQUIRE(nz <= kLvThreads * kLvMaxJ, "steam_project_bounds: nz above 1024");
  STEAM_REQUIRE(phi_max > phi_min, "steam_project_bounds: phi_max must exceed phi_min");
  int rc = check_win(window, nx, ny, "steam_project_bounds");
  if (rc) return rc;
  if (nx * ny * nz == 0) return STEAM_OK;
  STEAM_REQUIRE(pert && mean_1d, "steam_project_bounds: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    return project_impl<float>(nx, ny, nz, (float*)pert, mean_1d, phi_min,
                               phi_max, window, mu_out, workspace,
                               workspace_bytes, s);
  if (dtype == STEAM_F64)
    return project_impl<double>(nx, ny, nz, (double*)pert, mean_1d, phi_min,
                                phi_max, window, mu_out, workspace,
                                workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_project_bounds: bad dtype");
}

// ---- per-level sums without a caller workspace ---------------------------------
// steam_level_sums takes its scratch (block partials and totals) from a
// workspace the caller allocates.  Some callers cannot allocate device memory
// at all: a host application whose own allocator owns the whole device budget
// and forbids other libraries from calling cudaMalloc, a binding through a
// plain C FFI that has no device allocator to hand, or a latency-critical loop
// that must not risk an allocation's synchronisation.  This variant keeps its
// scratch in one file-scope device array instead.  The array is part of the
// loaded library image, so every GPU that loads the library holds it
// (kNoAllocScratchBytes) until the process exits.
namespace steam {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;  // 4 MiB per device
constexpr size_t kNoAllocScratchDoubles = kNoAllocScratchBytes / sizeof(double);
// In host code this name is only a handle for the runtime; the device address
// comes from cudaGetSymbolAddress below.
__device__ __align__(256) double g_level_sums_scratch[kNoAllocScratchDoubles];

// Device address of the scratch array in the calling thread's current
// context.  The address belongs to the context that loaded this module: a
// host application may switch between its own contexts, and after
// cudaDeviceReset the module is loaded again at another address, so the
// address is looked up on every call (a table lookup once the module is
// loaded) rather than remembered per device.
int noalloc_scratch(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_level_sums_scratch);
  if (e != cudaSuccess || p == nullptr)
    return fail(STEAM_ERR_CUDA, std::string("steam_level_sums_noalloc: cudaGetSymbolAddress: ") +
                                    cudaGetErrorString(e));
  *out = static_cast<double*>(p);
  return STEAM_OK;
}

// totals [3][nz] -> out [nz][4] = {sum, sum|f|, nonzero count, cells}
__global__ void pack_level_sums_kernel(const double* __restrict__ totals, int nz,
                                       double cells, double* __restrict__ out) {
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
    out[4 * z + 0] = totals[z];
    out[4 * z + 1] = totals[nz + z];
    out[4 * z + 2] = totals[2 * nz + z];
    out[4 * z + 3] = cells;
  }
}

}  // namespace
}  // namespace steam

extern "C" size_t steam_level_sums_noalloc_scratch_bytes(void) {
  return steam::kNoAllocScratchBytes;
}

extern "C" int steam_level_sums_noalloc(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                        const void* field, const steam_window_t* window,
                                        double* sums_out, steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "steam_level_sums_noalloc: negative extent");
  if (nz > kLvThreads * kLvMaxJ)
    return fail(STEAM_ERR_UNSUPPORTED,
                "steam_level_sums_noalloc: nz = " + std::to_string(nz) +
                    " is above the maximum of 1024 levels this entry point supports");
  STEAM_REQUIRE(sums_out != nullptr, "steam_level_sums_noalloc: null sums_out");
  STEAM_REQUIRE(dtype == STEAM_F32 || dtype == STEAM_F64, "steam_level_sums_noalloc: bad dtype");
  int rc = check_win(window, nx, ny, "steam_level_sums_noalloc");
  if (rc) return rc;
  if (nz == 0) return STEAM_OK;
  const Win w = make_win(window, nx, ny);
  const double cells = (double)((w.x1 - w.x0) * (w.y1 - w.y0));
  if (nx * ny == 0) {
    for (int64_t z = 0; z < nz; ++z) {
      sums_out[4 * z] = sums_out[4 * z + 1] = sums_out[4 * z + 2] = 0.0;
      sums_out[4 * z + 3] = cells;
    }
    return STEAM_OK;
  }
  STEAM_REQUIRE(field != nullptr, "steam_level_sums_noalloc: null field");
  // Scratch layout (doubles): partials [3][nz][B] | totals [3][nz] | packed [nz][4].
  // B, the block count, is the regular entry's grid capped so that the three
  // regions fit the static array; every kernel below is grid-stride, so a
  // smaller B changes only the order of the per-level double sums.
  const LevelMap m = make_map(nz);
  const size_t fixed = (size_t)7 * nz;
  const size_t cap_blocks = (kNoAllocScratchDoubles - fixed) / ((size_t)3 * nz);
  int grid = level_grid(nx * ny, m);
  if ((size_t)grid > cap_blocks) grid = (int)cap_blocks;
  double* scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  double* partials = scratch;
  double* totals = partials + (size_t)grid * 3 * nz;
  double* packed = totals + (size_t)3 * nz;
  cudaStream_t s = (cudaStream_t)stream;
  // Every partial slot is written by its block before the reduction reads
  // it, and every total before the pack reads it, so nothing carries over
  // from the previous call's contents.
  if (dtype == STEAM_F32) {
    if (m.packed)
      level_sums_kernel<float, 1><<<grid, kLvThreads, 0, s>>>((const float*)field, nx, ny, m, w,
                                                              partials);
    else
      level_sums_kernel<float, kLvMaxJ><<<grid, kLvThreads, 0, s>>>((const float*)field, nx, ny,
                                                                    m, w, partials);
  } else {
    if (m.packed)
      level_sums_kernel<double, 1><<<grid, kLvThreads, 0, s>>>((const double*)field, nx, ny, m,
                                                               w, partials);
    else
      level_sums_kernel<double, kLvMaxJ><<<grid, kLvThreads, 0, s>>>((const double*)field, nx,
                                                                     ny, m, w, partials);
  }
  STEAM_LAUNCH_CHECK("steam_level_sums_noalloc");
  if ((rc = reduce_partials(partials, grid, 3 * (int)nz, totals, s))) return rc;
  pack_level_sums_kernel<<<(int)((nz + 255) / 256), 256, 0, s>>>(totals, (int)nz, cells, packed);
  STEAM_LAUNCH_CHECK("steam_level_sums_noalloc pack");
  STEAM_CUDA(cudaMemcpyAsync(sums_out, packed, (size_t)4 * nz * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
  STEAM_CUDA(cudaStreamSynchronize(s));
  return STEAM_OK;
}

extern "C" size_t steam_bounded_add_ledger_doubles(int32_t n_rescale) {
  return n_rescale < 0 ? 0 : (size_t)ba_ledger_width(n_rescale);
}

extern "C" size_t steam_bounded_add_replay_workspace_bytes(int64_t nz, int32_t n_rescale) {
  return ba_replay_bytes(nz, n_rescale, sizeof(double));
}

static int replay_entry(int dtype, int64_t nx, int64_t ny, int64_t nz, void* pert,
                        const double* mean, int mean_dev, void* increment, double phi_min,
                        double phi_max, int32_t n_rescale, int32_t record,
                        const double* ledger, int led_dev, void* ws, size_t ws_bytes,
                        steam_stream_t stream, const char* who) {
  int rc = bounded_add_check(nx, ny, nz, n_rescale, phi_min, phi_max, nullptr, who);
  if (rc) return rc;
  if (nx * ny * nz == 0) return STEAM_OK;
  STEAM_REQUIRE(pert && increment && mean && ledger, std::string(who) + ": null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    return bounded_add_replay_impl<float>(nx, ny, nz, (float*)pert, mean, mean_dev,
                                          (float*)increment, phi_min, phi_max, n_rescale,
                                          record, ledger, led_dev, ws, ws_bytes, s);
  if (dtype == STEAM_F64)
    return bounded_add_replay_impl<double>(nx, ny, nz, (double*)pert, mean, mean_dev,
                                           (double*)increment, phi_min, phi_max, n_rescale,
                                           record, ledger, led_dev, ws, ws_bytes, s);
  return fail(STEAM_ERR_ARG, std::string(who) + ": bad dtype");
}

extern "C" int steam_bounded_add_replay(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                        void* pert, const double* mean_1d, void* increment,
                                        double phi_min, double phi_max, int32_t n_rescale,
                                        int32_t record_applied, const double* ledger,
                                        void* workspace, size_t workspace_bytes,
                                        steam_stream_t stream) {
  int rc = replay_entry(dtype, nx, ny, nz, pert, mean_1d, 0, increment, phi_min, phi_max,
                        n_rescale, record_applied, ledger, 0, workspace, workspace_bytes,
                        stream, "steam_bounded_add_replay");
  if (rc) return rc;
  STEAM_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  return STEAM_OK;
}

extern "C" int steam_bounded_add_replay_async(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                              void* pert, const double* mean_dev,
                                              void* increment, double phi_min,
                                              double phi_max, int32_t n_rescale,
                                              int32_t record_applied, const double* ledger_dev,
                                              void* workspace, size_t workspace_bytes,
                                              steam_stream_t stream) {
  return replay_entry(dtype, nx, ny, nz, pert, mean_dev, 1, increment, phi_min, phi_max,
                      n_rescale, record_applied, ledger_dev, 1, workspace, workspace_bytes,
                      stream, "steam_bounded_add_replay_async");
}

extern "C" int steam_project_bounds_replay(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                           void* pert, const double* mean_1d, double phi_min,
                                           double phi_max, const double* mu, void* workspace,
                                           size_t workspace_bytes, steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "steam_project_bounds_replay: negative extent");
  STEAM_REQUIRE(nz <= kLvThreads * kLvMaxJ, "steam_project_bounds_replay: nz above 1024");
  STEAM_REQUIRE(phi_max > phi_min, "steam_project_bounds_replay: phi_max must exceed phi_min");
  if (nx * ny * nz == 0) return STEAM_OK;
  STEAM_REQUIRE(pert && mean_1d && mu, "steam_project_bounds_replay: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    return project_replay_impl<float>(nx, ny, nz, (float*)pert, mean_1d, phi_min, phi_max, mu,
                                      workspace, workspace_bytes, s);
  if (dtype == STEAM_F64)
    return project_replay_impl<double>(nx, ny, nz, (double*)pert, mean_1d, phi_min, phi_max,
                                       mu, workspace, workspace_bytes, s);
  return fail(STEAM_ERR_ARG, "steam_project_bounds_replay: bad dtype");
}
