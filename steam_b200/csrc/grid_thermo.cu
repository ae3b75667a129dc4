// Class-to-class periodic trilinear regrid, the turbulon kernel build and the
// thermodynamic column solve.
#include "common.cuh"

#include <cmath>
#include <map>
#include <mutex>
#include <vector>

namespace steam {

// ---- a15: regrid ------------------------------------------------------------
// One axis of torch's align_corners=False linear resample over the wrapped-pad
// geometry of the reference (pad p source cells, crop c target cells per
// periodic side, p/c = n_in/n_out in lowest terms).  Source indices are mapped
// back onto the unpadded source periodically.
struct Axis {
  int64_t n_in, n_out, pad, crop, big_in;
  float scale;
  int periodic;
};

static int64_t gcd64(int64_t a, int64_t b) {
  while (b) {
    int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

static Axis make_axis(int64_t n_in, int64_t n_out, bool periodic) {
  Axis a;
  a.n_in = n_in;
  a.n_out = n_out;
  a.periodic = periodic ? 1 : 0;
  if (periodic) {
    int64_t g = gcd64(n_in, n_out);
    a.pad = n_in / g;
    a.crop = n_out / g;
  } else {
    a.pad = 0;
    a.crop = 0;
  }
  a.big_in = n_in + 2 * a.pad;
  const int64_t big_out = n_out + 2 * a.crop;
  a.scale = (float)a.big_in / (float)big_out;
  return a;
}

__device__ __forceinline__ void axis_weights(const Axis& a, int64_t t,
                                             int64_t& i0, int64_t& i1,
                                             float& l1) {
  float src = __fsub_rn(__fmul_rn(a.scale, (float)(t + a.crop) + 0.5f), 0.5f);
  if (src < 0.f) src = 0.f;
  int64_t f = (int64_t)floorf(src);
  if (f > a.big_in - 1) f = a.big_in - 1;
  float lam = src - (float)f;
  lam = lam < 0.f ? 0.f : (lam > 1.f ? 1.f : lam);
  int64_t g = f + (f < a.big_in - 1 ? 1 : 0);
  if (a.periodic) {
    i0 = ((f - a.pad) % a.n_in + a.n_in) % a.n_in;
    i1 = ((g - a.pad) % a.n_in + a.n_in) % a.n_in;
  } else {
    i0 = f;
    i1 = g;
  }
  l1 = lam;
}

template <typename T>
__global__ void regrid_kernel(const T* __restrict__ in, Axis ax, Axis ay,
                              Axis az, T* __restrict__ out) {
  const int64_t n = ax.n_out * ay.n_out * az.n_out;
  const int64_t ny = ay.n_in, nz = az.n_in;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = i % az.n_out;
    const int64_t col = i / az.n_out;
    const int64_t j = col % ay.n_out;
    const int64_t t = col / ay.n_out;
    int64_t x0, x1, y0, y1, z0, z1;
    float lx, ly, lz;
    axis_weights(ax, t, x0, x1, lx);
    axis_weights(ay, j, y0, y1, ly);
    axis_weights(az, k, z0, z1, lz);
    const T wx1 = (T)lx, wx0 = (T)1 - wx1;
    const T wy1 = (T)ly, wy0 = (T)1 - wy1;
    const T wz1 = (T)lz, wz0 = (T)1 - wz1;
    const T* p00 = in + (x0 * ny + y0) * nz;
    const T* p01 = in + (x0 * ny + y1) * nz;
    const T* p10 = in + (x1 * ny + y0) * nz;
    const T* p11 = in + (x1 * ny + y1) * nz;
    T v0 = wy0 * (wz0 * p00[z0] + wz1 * p00[z1]) +
           wy1 * (wz0 * p01[z0] + wz1 * p01[z1]);
    T v1 = wy0 * (wz0 * p10[z0] + wz1 * p10[z1]) +
           wy1 * (wz0 * p11[z0] + wz1 * p11[z1]);
    out[i] = wx0 * v0 + wx1 * v1;
  }
}

// ---- a8: kernel build ---------------------------------------------------------
template <typename T>
__global__ void kernel_build_kernel(int hx, int hy, int hz, T dx, T dy, T dz,
                                    T sigma2, T two_sigma2, T omega, int shape,
                                    T* __restrict__ out) {
  __shared__ double scratch[32];
  __shared__ double ratio_s;
  const int kx = 2 * hx + 1, ky = 2 * hy + 1, kz = 2 * hz + 1;
  const int64_t n = (int64_t)kx * ky * kz;
  double s_env = 0.0, s_g = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const int c = (int)(i % kz);
    const int b = (int)((i / kz) % ky);
    const int a = (int)(i / ((int64_t)kz * ky));
    const T x = mul_rn((T)(a - hx), dx), y = mul_rn((T)(b - hy), dy),
            z = mul_rn((T)(c - hz), dz);
    const T r2 = add_rn(add_rn(mul_rn(x, x), mul_rn(y, y)), mul_rn(z, z));
    const T rho = r2 / sigma2;
    T env;
    if (shape == 0)
      env = mul_rn(sub_rn((T)3, rho), d_exp(-rho / (T)2));
    else
      env = mul_rn(d_cos(mul_rn(omega, d_sqrt(r2))), d_exp(-rho / (T)2));
    const T g = d_exp(-r2 / two_sigma2);
    out[i] = env;
    s_env += (double)env;
    s_g += (double)g;
  }
  double te = block_sum(s_env, scratch);
  double tg = block_sum(s_g, scratch);
  if (threadIdx.x == 0) ratio_s = te / tg;
  __syncthreads();
  const T ratio = (T)ratio_s;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const int c = (int)(i % kz);
    const int b = (int)((i / kz) % ky);
    const int a = (int)(i / ((int64_t)kz * ky));
    const T x = mul_rn((T)(a - hx), dx), y = mul_rn((T)(b - hy), dy),
            z = mul_rn((T)(c - hz), dz);
    const T r2 = add_rn(add_rn(mul_rn(x, x), mul_rn(y, y)), mul_rn(z, z));
    const T g = d_exp(-r2 / two_sigma2);
    out[i] = sub_rn(out[i], mul_rn(g, ratio));
  }
}

// ---- a17: thermodynamics ------------------------------------------------------
// A warp owns 32 consecutive columns (contiguous in memory).  Levels go
// through shared memory kThZ at a time so that loads and stores are
// coalesced: each staging instruction moves 32 / kThZ columns x kThZ levels
// with every lane active (kThZ floats = one 64-byte run per column).  Each
// lane then marches its own column with a float64 pressure accumulator; the
// five outputs overwrite the two input slots and three more in place.
constexpr int kThZ = 16;
constexpr int kThWarps = 4;
constexpr int kThPitch = kThZ + 1;
constexpr int kThArrays = 5;  // h -> T, qt -> qv, qc, qi, p

template <typename T>
struct ThermoConst {
  T cp, lv, g, t0, t1, dt, c622, es0, ea, eb, ec, dq;
  // float32 path: ea log2(e), 1/cp, 1/dt, dq c622
  T ea2, inv_cp, inv_dt, dqc;
};

// The float32 form divides with the hardware's approximate division (two
// float32 ulps at most) and takes exp from the hardware exp2 outside the
// Newton loop too: the results stay within a few float32 ulps of the
// correctly rounded forms, far inside the float32 tolerances of T (1e-3 K),
// the mixing ratios and p.  The float64 form keeps the correctly rounded
// operations.
__device__ __forceinline__ float th_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double th_div(double a, double b) { return a / b; }
__device__ __forceinline__ float th_exp(float x) { return __expf(x); }
__device__ __forceinline__ double th_exp(double x) { return exp(x); }

template <typename T>
__device__ __forceinline__ T bolton(T Tk, const ThermoConst<T>& k) {
  return mul_rn(k.es0, th_exp(th_div(mul_rn(k.ea, sub_rn(Tk, k.eb)), sub_rn(Tk, k.ec))));
}

// the hardware's approximate reciprocal and base-2 exponential (PTX
// rcp.approx / ex2.approx: about 1 and 2 float32 ulps)
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Bolton's saturation vapour pressure in the float32 form:
// es0 2^(ea log2(e) (T - eb) / (T - ec))
__device__ __forceinline__ float bolton_f(float Tk, const ThermoConst<float>& k) {
  return k.es0 * ex2_approx(k.ea2 * (Tk - k.eb) * rcp_approx(Tk - k.ec));
}

// exp(a) for one hypsometric step: the exponent -g dz / (Rd Tv) is small
// (about -0.012 for 100 m levels), so the Taylor series of exp about 0 to
// degree 9 is exact to below 2^-61 relative for |a| <= 1/16 (the remainder
// is at most |a|^10 / 10! e^|a|); larger |a| take exp().
__device__ __forceinline__ double exp_hyps(double a) {
  if (!(fabs(a) <= 0.0625)) return exp(a);
  double s = 1.0 / 362880.0;  // 1/9!
  s = fma(s, a, 1.0 / 40320.0);
  s = fma(s, a, 1.0 / 5040.0);
  s = fma(s, a, 1.0 / 720.0);
  s = fma(s, a, 1.0 / 120.0);
  s = fma(s, a, 1.0 / 24.0);
  s = fma(s, a, 1.0 / 6.0);
  s = fma(s, a, 0.5);
  s = fma(s, a, 1.0);
  return fma(s, a, 1.0);
}

// Inside the Newton iterations the float64 form keeps the correctly rounded
// functions.
__device__ __forceinline__ double newton_exp(double x) { return exp(x); }
__device__ __forceinline__ double newton_rcp(double x) { return 1.0 / x; }

// Saturation adjustment of one cell: T and qv from h, qt at pressure p.
// Newton on f(T) = cp T + Lv qvs(T, p) + g z - h, 5 iterations from the dry
// temperature, when qt exceeds the saturation mixing ratio there.
// float32: fused multiply-adds and the approximate reciprocal and exp2; the
// reciprocal 1/(T - 29.65) is shared between the Bolton exponent and
// dqvs/dT = dq c622 p es / ((T - 29.65)^2 (p - es)^2), and the step needs
// one more reciprocal, of its denominator.
__device__ __forceinline__ void saturate(float hl, float ql, float pl, float gz,
                                         const ThermoConst<float>& k, float& Tl, float& qvl) {
  const float Td = __fmul_rn(__fsub_rn(__fsub_rn(hl, __fmul_rn(k.lv, ql)), gz), k.inv_cp);
  const float es = bolton_f(Td, k);
  const float qvs = k.c622 * es * rcp_approx(pl - es);
  Tl = Td;
  qvl = ql;
  if (ql > qvs) {
    // the Newton step f / f' with numerator and denominator both multiplied
    // by (p - es)^2, which takes the reciprocal of (p - es) out of the loop:
    //   f (p - es)^2  = ((cp T + g z - h)(p - es) + Lv c622 es)(p - es)
    //   f'(p - es)^2  = cp (p - es)^2 + Lv dq c622 p es / (T - 29.65)^2
    // Newton converges quadratically here: once a step is below 0.01 K the
    // remaining iterations of the 5 move T by less than 5e-6 K (float64
    // iterates of 590k saturated states over 190-320 K and 150-1060 hPa),
    // under a float32 ulp of T, so the loop stops there.  Cells still far
    // from the root take all 5 steps, as the reference does.  The exit
    // depends on the cell alone.
    const float gzh = gz - hl, lvc = k.lv * k.c622, lvdq = k.lv * k.dqc * pl;
    float Tn = Td;
#pragma unroll 1
    for (int it = 0; it < 5; ++it) {
      const float i1 = rcp_approx(Tn - k.ec);
      const float e = k.es0 * ex2_approx(k.ea2 * (Tn - k.eb) * i1);
      const float pe = pl - e;
      const float num = fmaf(fmaf(k.cp, Tn, gzh), pe, lvc * e) * pe;
      const float den = fmaf(k.cp * pe, pe, lvdq * e * i1 * i1);
      const float T1 = fmaf(-num, rcp_approx(den), Tn);
      const bool done = fabsf(T1 - Tn) < 1e-2f;
      Tn = T1;
      if (done) break;
    }
    Tl = Tn;
    const float e = bolton_f(Tn, k);
    qvl = k.c622 * e * rcp_approx(pl - e);
  }
}

// float64: the correctly rounded operations, in the reference's order.
__device__ __forceinline__ void saturate(double hl, double ql, double pl, double gz,
                                         const ThermoConst<double>& k, double& Tl,
                                         double& qvl) {
  const double Td = th_div(sub_rn(sub_rn(hl, mul_rn(k.lv, ql)), gz), k.cp);
  const double es = bolton(Td, k);
  const double qvs = th_div(mul_rn(k.c622, es), sub_rn(pl, es));
  Tl = Td;
  qvl = ql;
  if (ql > qvs) {
    double Tn = Td;
#pragma unroll 1
    for (int it = 0; it < 5; ++it) {
      const double i1 = newton_rcp(sub_rn(Tn, k.ec));
      const double e = mul_rn(k.es0, newton_exp(mul_rn(mul_rn(k.ea, sub_rn(Tn, k.eb)), i1)));
      const double i2 = newton_rcp(sub_rn(pl, e));
      const double q = mul_rn(mul_rn(k.c622, e), i2);
      const double f = sub_rn(add_rn(add_rn(mul_rn(k.cp, Tn), mul_rn(k.lv, q)), gz), hl);
      const double de = mul_rn(mul_rn(k.dq, e), mul_rn(i1, i1));
      const double dq = mul_rn(mul_rn(mul_rn(k.c622, pl), mul_rn(i2, i2)), de);
      Tn = sub_rn(Tn, mul_rn(f, newton_rcp(add_rn(k.cp, mul_rn(k.lv, dq)))));
    }
    Tl = Tn;
    const double e = bolton(Tn, k);
    qvl = th_div(mul_rn(k.c622, e), sub_rn(pl, e));
  }
}

// the ice fraction ramp (T - 235.15) / 38, unclamped
__device__ __forceinline__ float ice_ramp(float Tl, const ThermoConst<float>& k) {
  return (Tl - k.t0) * k.inv_dt;
}
__device__ __forceinline__ double ice_ramp(double Tl, const ThermoConst<double>& k) {
  return th_div(sub_rn(Tl, k.t0), k.dt);
}

// the hypsometric exponent -g dz / (Rd Tv) of the step to the next level:
// float32 from ghyp dz = -g dz / Rd and the approximate reciprocal (relative
// error ~1e-7 of a ~1e-2 exponent, ~1e-9 of p per level), float64 exact; p
// itself accumulates in float64 in both forms
__device__ __forceinline__ double hyps_exponent(float Tl, float qvl, float ghdz,
                                                const ThermoConst<float>&) {
  const float Tv = __fmul_rn(Tl, __fadd_rn(1.0f, __fmul_rn(0.608f, qvl)));
  return (double)(ghdz * rcp_approx(Tv));
}
__device__ __forceinline__ double hyps_exponent(double Tl, double qvl, double gdz,
                                                const ThermoConst<double>&) {
  const double Tv = Tl * (1.0 + 0.608 * qvl);
  return gdz / (287.04 * Tv);
}

// One block's work (block `vb` of the field's ceil(ncol / (32 kThWarps))):
// 32 columns per warp, marched along z in chunks of kThZ levels.
template <typename T>
__device__ __forceinline__ void thermo_body(
    int64_t vb, const T* __restrict__ h, const T* __restrict__ qt,
    const double* __restrict__ zv, const double* __restrict__ dzv,
    const double* __restrict__ hm, const double* __restrict__ qm, int compose,
    T hlo, T hhi, T qlo, T qhi, int64_t ncol,
    int nz, double ps, const double* __restrict__ ps_field, const ThermoConst<T>& k,
    T* __restrict__ To, T* __restrict__ qvo, T* __restrict__ qco,
    T* __restrict__ qio, T* __restrict__ po) {
  extern __shared__ unsigned char th_smem[];
  T* base = reinterpret_cast<T*>(th_smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // sh(a, c, z): slot a (0: h then T, 1: qt then qv, 2: qc, 3: qi, 4: p) of
  // column c, level z of the chunk
  auto sh = [&](int a, int c, int z) -> T& {
    return base[((warp * kThArrays + a) * 32 + c) * kThPitch + z];
  };
  // the chunk's per-level constants, per warp: g z, mean h, mean qt and the
  // hypsometric numerator (-g dz / Rd in float32, -g dz in float64)
  T* lv = base + (size_t)kThWarps * kThArrays * 32 * kThPitch + warp * 4 * kThZ;
  const int64_t col0 = (vb * kThWarps + warp) * 32;
  if (col0 >= ncol) return;
  const int ncols = (int)((ncol - col0) < 32 ? (ncol - col0) : 32);
  const int64_t mycol = col0 + lane;
  double p_cur = ps_field ? (lane < ncols ? ps_field[mycol] : 0.0) : ps;
  // staging geometry: lane -> (column group member, level) of a chunk
  constexpr int kCPI = 32 / kThZ;  // columns per staging instruction
  const int s_c = lane / kThZ, s_z = lane % kThZ;
  // the h and qt values this lane stages for a chunk, loaded one chunk ahead
  // so that the loads of chunk z0 + kThZ are in flight while chunk z0 is
  // computed
  constexpr int kPer = 32 / kCPI;  // staging instructions per chunk
  T nh[kPer], nq[kPer];
  auto fetch = [&](int z0f) {
    const int zcf = (nz - z0f) < kThZ ? (nz - z0f) : kThZ;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int c = i * kCPI + s_c;
      nh[i] = nq[i] = (T)0;
      if (c < ncols && s_z < zcf) {
        const int64_t o = (col0 + c) * nz + z0f + s_z;
        nh[i] = h[o];
        nq[i] = qt[o];
      }
    }
  };
  fetch(0);
  for (int z0 = 0; z0 < nz; z0 += kThZ) {
    const int zc = (nz - z0) < kThZ ? (nz - z0) : kThZ;
    if (lane < zc) {
      const int z = z0 + lane;
      lv[lane] = mul_rn(k.g, (T)zv[z]);
      lv[kThZ + lane] = (T)hm[z];
      lv[2 * kThZ + lane] = (T)qm[z];
      lv[3 * kThZ + lane] =
          sizeof(T) == 4 ? (T)(-9.81 * dzv[z] / 287.04) : (T)(-9.81 * dzv[z]);
    }
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int c = i * kCPI + s_c;
      if (c < ncols && s_z < zc) {
        sh(0, c, s_z) = nh[i];
        sh(1, c, s_z) = nq[i];
      }
    }
    if (z0 + kThZ < nz) fetch(z0 + kThZ);
    __syncwarp();
    if (lane < ncols) {
      for (int zz = 0; zz < zc; ++zz) {
        const int z = z0 + zz;
        T hl = sh(0, lane, zz), ql = sh(1, lane, zz);
        if (compose) {
          // _compose_output without a deficit: state + mean, clamped to bounds
          hl = add_rn(hl, lv[kThZ + zz]);
          ql = add_rn(ql, lv[2 * kThZ + zz]);
          hl = hl < hlo ? hlo : (hl > hhi ? hhi : hl);
          ql = ql < qlo ? qlo : (ql > qhi ? qhi : ql);
        }
        const T pl = (T)p_cur;
        T Tl, qvl;
        saturate(hl, ql, pl, lv[zz], k, Tl, qvl);
        T cond = sub_rn(ql, qvl);
        cond = cond > (T)0 ? cond : (T)0;
        T lam = ice_ramp(Tl, k);
        lam = lam < (T)0 ? (T)0 : (lam > (T)1 ? (T)1 : lam);
        sh(0, lane, zz) = Tl;
        sh(1, lane, zz) = qvl;
        sh(2, lane, zz) = mul_rn(lam, cond);
        sh(3, lane, zz) = mul_rn(sub_rn((T)1, lam), cond);
        sh(4, lane, zz) = pl;
        if (z < nz - 1) p_cur *= exp_hyps(hyps_exponent(Tl, qvl, lv[3 * kThZ + zz], k));
      }
    }
    __syncwarp();
    for (int c0 = 0; c0 < ncols; c0 += kCPI) {
      const int c = c0 + s_c;
      if (c < ncols && s_z < zc) {
        const int64_t o = (col0 + c) * nz + z0 + s_z;
        To[o] = sh(0, c, s_z);
        qvo[o] = sh(1, c, s_z);
        qco[o] = sh(2, c, s_z);
        qio[o] = sh(3, c, s_z);
        po[o] = sh(4, c, s_z);
      }
    }
    __syncwarp();
  }
}

template <typename T>
__global__ void __launch_bounds__(32 * kThWarps) thermo_kernel(
    const T* __restrict__ h, const T* __restrict__ qt,
    const double* __restrict__ zv, const double* __restrict__ dzv,
    const double* __restrict__ hm, const double* __restrict__ qm, int compose,
    T hlo, T hhi, T qlo, T qhi, int64_t ncol,
    int nz, double ps, const double* __restrict__ ps_field, ThermoConst<T> k,
    T* __restrict__ To, T* __restrict__ qvo, T* __restrict__ qco,
    T* __restrict__ qio, T* __restrict__ po) {
  thermo_body<T>(blockIdx.x, h, qt, zv, dzv, hm, qm, compose, hlo, hhi, qlo, qhi, ncol, nz, ps,
                 ps_field, k, To, qvo, qco, qio, po);
}

// One field of a grouped thermodynamics launch (device memory): its arrays,
// profiles (z, dz, mean h, mean qt: 4 nz), bounds and its first block.
struct ThermoMember {
  const void* h;
  const void* qt;
  const double* prof;
  const double* ps_field;
  void* T;
  void* qv;
  void* qc;
  void* qi;
  void* p;
  int64_t ncol;
  int64_t block0;
  int32_t nz;
  int32_t compose;
  double bounds[4];
  double ps;
};

// n fields in one launch: owner[b] is the field of block b.
template <typename T>
__global__ void __launch_bounds__(32 * kThWarps) thermo_group_kernel(
    const ThermoMember* __restrict__ mem, const int32_t* __restrict__ owner, ThermoConst<T> k) {
  const int64_t b = blockIdx.x;
  const ThermoMember& m = mem[owner[b]];
  const int nz = m.nz;
  thermo_body<T>(b - m.block0, (const T*)m.h, (const T*)m.qt, m.prof, m.prof + nz,
                 m.prof + 2 * nz, m.prof + 3 * nz, m.compose, (T)m.bounds[0], (T)m.bounds[1],
                 (T)m.bounds[2], (T)m.bounds[3], m.ncol, nz, m.ps, m.ps_field, k, (T*)m.T,
                 (T*)m.qv, (T*)m.qc, (T*)m.qi, (T*)m.p);
}

template <typename T>
static ThermoConst<T> thermo_const() {
  ThermoConst<T> k;
  k.cp = (T)1004.0;
  k.lv = (T)2.5e6;
  k.g = (T)9.81;
  k.t0 = (T)235.15;
  k.dt = (T)(273.15 - 235.15);
  k.c622 = (T)0.622;
  k.es0 = (T)611.2;
  k.ea = (T)17.67;
  k.eb = (T)273.15;
  k.ec = (T)29.65;
  k.dq = (T)4302.6;
  k.ea2 = (T)(17.67 * 1.4426950408889634);
  k.inv_cp = (T)(1.0 / 1004.0);
  k.inv_dt = (T)(1.0 / (273.15 - 235.15));
  k.dqc = (T)(4302.6 * 0.622);
  return k;
}

}  // namespace steam

using namespace steam;

extern "C" int steam_regrid(int dtype, const void* in, int64_t nx, int64_t ny,
                            int64_t nz, void* out, int64_t mx, int64_t my,
                            int64_t mz, int32_t periodic_x, int32_t periodic_y,
                            steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1 && mx >= 1 && my >= 1 && mz >= 1,
                "steam_regrid: extents must be >= 1");
  STEAM_REQUIRE(!periodic_x || mx >= nx,
                "steam_regrid: periodic resampling only goes finer (x)");
  STEAM_REQUIRE(!periodic_y || my >= ny,
                "steam_regrid: periodic resampling only goes finer (y)");
  STEAM_REQUIRE(in && out, "steam_regrid: null pointer");
  Axis ax = make_axis(nx, mx, periodic_x != 0);
  Axis ay = make_axis(ny, my, periodic_y != 0);
  Axis az = make_axis(nz, mz, false);
  const int64_t n = mx * my * mz;
  int grid = stride_grid(n, 256, 8);
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    regrid_kernel<float><<<grid, 256, 0, s>>>((const float*)in, ax, ay, az,
                                              (float*)out);
  else if (dtype == STEAM_F64)
    regrid_kernel<double><<<grid, 256, 0, s>>>((const double*)in, ax, ay, az,
                                               (double*)out);
  else
    return fail(STEAM_ERR_ARG, "steam_regrid: bad dtype");
  STEAM_LAUNCH_CHECK("steam_regrid");
  return STEAM_OK;
}

extern "C" int steam_kernel_build(int dtype, double k, double dx, double dy,
                                  double dz, double support_factor,
                                  int32_t shape, void* out, int64_t* dims_out,
                                  steam_stream_t stream) {
  STEAM_REQUIRE(k > 0 && dx > 0 && dy > 0 && dz > 0 && support_factor > 0,
                "steam_kernel_build: scales must be positive");
  STEAM_REQUIRE(shape == 0 || shape == 1, "steam_kernel_build: unknown shape");
  STEAM_REQUIRE(dims_out != nullptr, "steam_kernel_build: null dims_out");
  const double hxd = std::ceil(support_factor * k / dx);
  const double hyd = std::ceil(support_factor * k / dy);
  const double hzd = std::ceil(support_factor * k / dz);
  STEAM_REQUIRE(hxd < 4096 && hyd < 4096 && hzd < 4096,
                "steam_kernel_build: kernel support too large");
  const int hx = (int)hxd, hy = (int)hyd, hz = (int)hzd;
  dims_out[0] = 2 * hx + 1;
  dims_out[1] = 2 * hy + 1;
  dims_out[2] = 2 * hz + 1;
  if (out == nullptr) return STEAM_OK;
  const double PI = 3.14159265358979323846;
  const double sigma2 = (k / PI) * (k / PI);
  cudaStream_t s = (cudaStream_t)stream;
  if (dtype == STEAM_F32)
    kernel_build_kernel<float><<<1, 1024, 0, s>>>(
        hx, hy, hz, (float)dx, (float)dy, (float)dz, (float)sigma2,
        (float)(2.0 * sigma2), (float)(6.0 / k), shape, (float*)out);
  else if (dtype == STEAM_F64)
    kernel_build_kernel<double><<<1, 1024, 0, s>>>(
        hx, hy, hz, dx, dy, dz, sigma2, 2.0 * sigma2, 6.0 / k, shape,
        (double*)out);
  else
    return fail(STEAM_ERR_ARG, "steam_kernel_build: bad dtype");
  STEAM_LAUNCH_CHECK("steam_kernel_build");
  return STEAM_OK;
}

extern "C" int steam_thermo_async(int dtype, int64_t nx, int64_t ny, int64_t nz,
                                  const void* h, const void* qt, const double* prof_dev,
                                  int32_t compose, const double* bounds,
                                  double surface_pressure, const double* ps_field_dev,
                                  void* T, void* qv, void* qc, void* qi, void* p,
                                  steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "steam_thermo_async: negative extent");
  const int64_t ncol = nx * ny;
  if (ncol * nz == 0) return STEAM_OK;
  STEAM_REQUIRE(h && qt && prof_dev && T && qv && qc && qi && p,
                "steam_thermo_async: null pointer");
  STEAM_REQUIRE(!compose || bounds != nullptr,
                "steam_thermo_async: composing with mean profiles needs bounds");
  cudaStream_t s = (cudaStream_t)stream;
  const double b0 = compose ? bounds[0] : 0.0, b1 = compose ? bounds[1] : 0.0;
  const double b2 = compose ? bounds[2] : 0.0, b3 = compose ? bounds[3] : 0.0;
  const int64_t blocks = (ncol + 32 * kThWarps - 1) / (32 * kThWarps);
  const size_t sm_f = ((size_t)kThWarps * kThArrays * 32 * kThPitch + kThWarps * 4 * kThZ) *
                      sizeof(float);
  const size_t sm_d = ((size_t)kThWarps * kThArrays * 32 * kThPitch + kThWarps * 4 * kThZ) *
                      sizeof(double);
  const double* zv = prof_dev;
  if (dtype == STEAM_F32) {
    STEAM_CUDA(cudaFuncSetAttribute(thermo_kernel<float>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_f));
    thermo_kernel<float><<<(unsigned)blocks, 32 * kThWarps, sm_f, s>>>(
        (const float*)h, (const float*)qt, zv, zv + nz, zv + 2 * nz, zv + 3 * nz, compose,
        (float)b0, (float)b1, (float)b2, (float)b3, ncol, (int)nz, surface_pressure,
        ps_field_dev, thermo_const<float>(), (float*)T, (float*)qv, (float*)qc, (float*)qi,
        (float*)p);
  } else if (dtype == STEAM_F64) {
    STEAM_CUDA(cudaFuncSetAttribute(thermo_kernel<double>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_d));
    thermo_kernel<double><<<(unsigned)blocks, 32 * kThWarps, sm_d, s>>>(
        (const double*)h, (const double*)qt, zv, zv + nz, zv + 2 * nz, zv + 3 * nz, compose, b0,
        b1, b2, b3, ncol, (int)nz, surface_pressure, ps_field_dev, thermo_const<double>(),
        (double*)T, (double*)qv, (double*)qc, (double*)qi, (double*)p);
  } else {
    return fail(STEAM_ERR_ARG, "steam_thermo_async: bad dtype");
  }
  STEAM_LAUNCH_CHECK("steam_thermo_async");
  return STEAM_OK;
}

namespace {
struct ThermoGroupRec {
  int dtype;
  int n;
  int64_t blocks;
};
std::mutex g_thermo_groups_mu;
std::map<const void*, ThermoGroupRec> g_thermo_groups;

size_t thermo_smem(int dtype) {
  return ((size_t)kThWarps * kThArrays * 32 * kThPitch + kThWarps * 4 * kThZ) *
         (dtype == STEAM_F64 ? sizeof(double) : sizeof(float));
}
}  // namespace

// The group's workspace: the fields' descriptors, then the block -> field
// table (one int32 per block of 128 columns).
constexpr int64_t kThGroupMaxBlocks = (int64_t)1 << 30;

static int64_t thermo_blocks(int64_t nx, int64_t ny) {
  return (nx * ny + 32 * kThWarps - 1) / (32 * kThWarps);
}

extern "C" size_t steam_thermo_group_workspace_bytes(int32_t n,
                                                     const steam_thermo_problem_t* problems) {
  if (n <= 0 || !problems) return 0;
  int64_t blocks = 0;
  for (int i = 0; i < n; ++i)
    if (problems[i].nx > 0 && problems[i].ny > 0) blocks += thermo_blocks(problems[i].nx, problems[i].ny);
  return sizeof(ThermoMember) * (size_t)n + sizeof(int32_t) * (size_t)blocks;
}

extern "C" int steam_thermo_group_prepare(int dtype, int32_t n,
                                          const steam_thermo_problem_t* problems,
                                          void* workspace, size_t workspace_bytes) {
  STEAM_REQUIRE(dtype == STEAM_F32 || dtype == STEAM_F64, "steam_thermo_group_prepare: bad dtype");
  STEAM_REQUIRE(n > 0 && problems && workspace, "steam_thermo_group_prepare: empty group");
  STEAM_REQUIRE(workspace_bytes >= steam_thermo_group_workspace_bytes(n, problems),
                "steam_thermo_group_prepare: workspace too small");
  std::vector<ThermoMember> mem((size_t)n);
  int64_t blocks = 0;
  for (int i = 0; i < n; ++i) {
    const steam_thermo_problem_t& q = problems[i];
    STEAM_REQUIRE(q.nx > 0 && q.ny > 0 && q.nz > 0,
                  "steam_thermo_group_prepare: every field needs a positive extent");
    STEAM_REQUIRE(q.nz < ((int64_t)1 << 31), "steam_thermo_group_prepare: nz too large");
    STEAM_REQUIRE(q.h && q.qt && q.prof && q.T && q.qv && q.qc && q.qi && q.p,
                  "steam_thermo_group_prepare: null pointer");
    ThermoMember& m = mem[(size_t)i];
    m.h = q.h;
    m.qt = q.qt;
    m.prof = q.prof;
    m.ps_field = q.ps_field;
    m.T = q.T;
    m.qv = q.qv;
    m.qc = q.qc;
    m.qi = q.qi;
    m.p = q.p;
    m.ncol = q.nx * q.ny;
    m.block0 = blocks;
    m.nz = (int32_t)q.nz;
    m.compose = q.compose ? 1 : 0;
    for (int j = 0; j < 4; ++j) m.bounds[j] = q.compose ? q.bounds[j] : 0.0;
    m.ps = q.surface_pressure;
    blocks += thermo_blocks(q.nx, q.ny);
  }
  STEAM_REQUIRE(blocks <= kThGroupMaxBlocks,
                "steam_thermo_group_prepare: group too large (2^30 blocks of 128 columns)");
  std::vector<int32_t> owner((size_t)blocks);
  for (int i = 0; i < n; ++i) {
    const int64_t end = i + 1 < n ? mem[(size_t)i + 1].block0 : blocks;
    for (int64_t b = mem[(size_t)i].block0; b < end; ++b) owner[(size_t)b] = i;
  }
  STEAM_CUDA(cudaMemcpy(workspace, mem.data(), sizeof(ThermoMember) * mem.size(),
                        cudaMemcpyHostToDevice));
  STEAM_CUDA(cudaMemcpy((char*)workspace + sizeof(ThermoMember) * mem.size(), owner.data(),
                        sizeof(int32_t) * owner.size(), cudaMemcpyHostToDevice));
  std::lock_guard<std::mutex> lk(g_thermo_groups_mu);
  g_thermo_groups[workspace] = ThermoGroupRec{dtype, n, blocks};
  return STEAM_OK;
}

extern "C" int steam_thermo_group_async(void* workspace, steam_stream_t stream) {
  ThermoGroupRec r;
  {
    std::lock_guard<std::mutex> lk(g_thermo_groups_mu);
    auto it = g_thermo_groups.find(workspace);
    STEAM_REQUIRE(it != g_thermo_groups.end(), "steam_thermo_group_async: unknown group");
    r = it->second;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const ThermoMember* mem = (const ThermoMember*)workspace;
  const int32_t* owner = (const int32_t*)((const char*)workspace + sizeof(ThermoMember) * r.n);
  const size_t sm = thermo_smem(r.dtype);
  if (r.dtype == STEAM_F32) {
    STEAM_CUDA(cudaFuncSetAttribute(thermo_group_kernel<float>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    thermo_group_kernel<float><<<(unsigned)r.blocks, 32 * kThWarps, sm, s>>>(
        mem, owner, thermo_const<float>());
  } else {
    STEAM_CUDA(cudaFuncSetAttribute(thermo_group_kernel<double>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    thermo_group_kernel<double><<<(unsigned)r.blocks, 32 * kThWarps, sm, s>>>(
        mem, owner, thermo_const<double>());
  }
  STEAM_LAUNCH_CHECK("steam_thermo_group_async");
  return STEAM_OK;
}

extern "C" int steam_thermo_group_release(void* workspace) {
  std::lock_guard<std::mutex> lk(g_thermo_groups_mu);
  g_thermo_groups.erase(workspace);
  return STEAM_OK;
}

extern "C" int steam_thermo(int dtype, int64_t nx, int64_t ny, int64_t nz,
                            const void* h, const void* qt,
                            const double* z_values, const double* h_mean,
                            const double* qt_mean, const double* bounds,
                            double surface_pressure,
                            const double* ps_field_dev, void* T, void* qv,
                            void* qc, void* qi, void* p,
                            steam_stream_t stream) {
  STEAM_REQUIRE(nx >= 0 && ny >= 0 && nz >= 0, "steam_thermo: negative extent");
  const int64_t ncol = nx * ny;
  if (ncol * nz == 0) return STEAM_OK;
  STEAM_REQUIRE(h && qt && z_values && T && qv && qc && qi && p,
                "steam_thermo: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  // z and dz go to the device through a small staging buffer owned here.
  STEAM_REQUIRE((h_mean == nullptr) == (qt_mean == nullptr),
                "steam_thermo: give both mean profiles or neither");
  const int compose = h_mean != nullptr;
  STEAM_REQUIRE(!compose || bounds != nullptr,
                "steam_thermo: composing with mean profiles needs bounds");
  std::vector<double> hz(4 * nz, 0.0);
  for (int64_t z = 0; z < nz; ++z) {
    hz[z] = z_values[z];
    hz[nz + z] = z + 1 < nz ? (z_values[z + 1] - z_values[z]) : 0.0;
    hz[2 * nz + z] = compose ? h_mean[z] : 0.0;
    hz[3 * nz + z] = compose ? qt_mean[z] : 0.0;
  }
  const double b0 = compose ? bounds[0] : 0.0, b1 = compose ? bounds[1] : 0.0;
  const double b2 = compose ? bounds[2] : 0.0, b3 = compose ? bounds[3] : 0.0;
  double* dz_dev = nullptr;
  STEAM_CUDA(cudaMallocAsync((void**)&dz_dev, sizeof(double) * 4 * nz, s));
  cudaError_t e = cudaMemcpyAsync(dz_dev, hz.data(), sizeof(double) * 4 * nz,
                                  cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) {
    cudaFreeAsync(dz_dev, s);
    return fail(STEAM_ERR_CUDA, std::string("steam_thermo: ") + cudaGetErrorString(e));
  }
  const int64_t blocks = (ncol + 32 * kThWarps - 1) / (32 * kThWarps);
  const size_t sm_f = ((size_t)kThWarps * kThArrays * 32 * kThPitch + kThWarps * 4 * kThZ) *
                      sizeof(float);
  const size_t sm_d = ((size_t)kThWarps * kThArrays * 32 * kThPitch + kThWarps * 4 * kThZ) *
                      sizeof(double);
  if (dtype == STEAM_F32) {
    e = cudaFuncSetAttribute(thermo_kernel<float>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_f);
  } else if (dtype == STEAM_F64) {
    e = cudaFuncSetAttribute(thermo_kernel<double>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_d);
  }
  if (e != cudaSuccess) {
    cudaFreeAsync(dz_dev, s);
    return fail(STEAM_ERR_CUDA, std::string("steam_thermo: ") + cudaGetErrorString(e));
  }
  if (dtype == STEAM_F32)
    thermo_kernel<float><<<(unsigned)blocks, 32 * kThWarps, sm_f, s>>>(
        (const float*)h, (const float*)qt, dz_dev, dz_dev + nz, dz_dev + 2 * nz,
        dz_dev + 3 * nz, compose, (float)b0, (float)b1, (float)b2, (float)b3,
        ncol, (int)nz,
        surface_pressure, ps_field_dev, thermo_const<float>(), (float*)T,
        (float*)qv, (float*)qc, (float*)qi, (float*)p);
  else if (dtype == STEAM_F64)
    thermo_kernel<double><<<(unsigned)blocks, 32 * kThWarps, sm_d, s>>>(
        (const double*)h, (const double*)qt, dz_dev, dz_dev + nz, dz_dev + 2 * nz,
        dz_dev + 3 * nz, compose, b0, b1, b2, b3, ncol, (int)nz, surface_pressure, ps_field_dev, thermo_const<double>(),
        (double*)T, (double*)qv, (double*)qc, (double*)qi, (double*)p);
  else {
    cudaFreeAsync(dz_dev, s);
    return fail(STEAM_ERR_ARG, "steam_thermo: bad dtype");
  }
  count_launch();
  e = cudaGetLastError();
  cudaFreeAsync(dz_dev, s);
  if (e != cudaSuccess)
    return fail(STEAM_ERR_CUDA, std::string("steam_thermo launch: ") + cudaGetErrorString(e));
  STEAM_CUDA(cudaStreamSynchronize(s));
  return STEAM_OK;
}
