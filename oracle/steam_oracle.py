"""CPU oracle for the STEAM field-generation hot path -- TEST INFRASTRUCTURE.

This module is the checker, not the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product (``steam_b200``) never imports, links or calls anything here,
and it has no CPU fallback.

It restates, in plain numpy, the reference algorithm of every stage the CUDA
path implements.  Each function cites the file:line of thomasdewitt/STEAM that
it follows.  Two arithmetic modes:

* ``dtype=np.float32`` mirrors the reference's own float32 arithmetic (its
  operation order, its float32 casts, its float64 reductions), so it can be
  pinned against fixtures produced by the reference itself
  (``tests/golden/make_golden.py``).
* ``dtype=np.float64`` is the FP64 oracle: the same formulas evaluated in
  float64 throughout, against which the FP32 device path states its error.

Integer work (Philox4x32-10 and the uniform lattice) is exact in both modes
and is pinned against the Random123 known-answer vectors that the reference's
tests carry and against keyed-uniform fixtures generated by the reference.

Parity status: pinned.  The golden fixtures in ``tests/golden`` were produced
by running the reference implementation (see ``tests/golden/make_golden.py``)
and ``tests/test_oracle.py`` checks this module against them.
"""

from __future__ import annotations

import math
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

# ---------------------------------------------------------------------------
# Constants (steam/noise.py:48-64, steam/simulate.py:58,115-116,517,
# steam/constants.py:3-6)
# ---------------------------------------------------------------------------

PHILOX_M0 = 0xD2511F53
PHILOX_M1 = 0xCD9E8D57
PHILOX_W0 = 0x9E3779B9
PHILOX_W1 = 0xBB67AE85
PHILOX_ROUNDS = 10
MASK32 = 0xFFFFFFFF

SUPPORT_FACTOR = 3
LEVY_EPS = 1e-6

CP = 1004.0
LV = 2.5e6
GRAV = 9.81
RD = 287.04

N_THREADS = max(1, os.cpu_count() or 1)


def _pool_map(fn, items, threads=None):
    threads = N_THREADS if threads is None else threads
    if threads <= 1 or len(items) <= 1:
        return [fn(i) for i in items]
    with ThreadPoolExecutor(threads) as pool:
        return list(pool.map(fn, items))


# ---------------------------------------------------------------------------
# a1-a4: keyed counter RNG (steam/noise.py:67-146)
# ---------------------------------------------------------------------------

def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Ten Philox4x32 rounds, vectorised over numpy uint64 arrays.

    Follows steam/noise.py:67-85: round 0 uses the raw key, later rounds bump
    it by (W0, W1); each round multiplies words 0 and 2 by (M0, M1) and
    assembles (hi1^c1^k0, lo1, hi0^c3^k1, lo0).
    """
    u64 = np.uint64
    c0 = np.asarray(c0, dtype=u64)
    c1 = np.asarray(c1, dtype=u64)
    c2 = np.asarray(c2, dtype=u64)
    c3 = np.asarray(c3, dtype=u64)
    k0 = u64(int(k0) & MASK32)
    k1 = u64(int(k1) & MASK32)
    m0, m1 = u64(PHILOX_M0), u64(PHILOX_M1)
    w0, w1 = u64(PHILOX_W0), u64(PHILOX_W1)
    mask, s32 = u64(MASK32), u64(32)
    for r in range(PHILOX_ROUNDS):
        if r > 0:
            k0 = (k0 + w0) & mask
            k1 = (k1 + w1) & mask
        p0 = m0 * c0
        p1 = m1 * c2
        c0, c1, c2, c3 = ((p1 >> s32) ^ c1 ^ k0, p1 & mask,
                          (p0 >> s32) ^ c3 ^ k1, p0 & mask)
    return c0, c1, c2, c3


def uniform_pair(ix, iy, iz, key):
    """Lane 0 / lane 1 uniforms of world sites (steam/noise.py:88-100).

    Counter (ix, iy, iz, key2), key (key0, key1); words 0 and 1 become
    ``(r >> 8) * 2**-24`` in float32 (exact).
    """
    key0, key1, key2 = (int(k) for k in key)
    r0, r1, _, _ = philox4x32_10(ix, iy, iz, np.uint64(key2), key0, key1)
    scale = np.float32(1.0 / 16777216.0)
    return ((r0 >> np.uint64(8)).astype(np.float32) * scale,
            (r1 >> np.uint64(8)).astype(np.float32) * scale)


def keyed_uniforms(world_ix, world_iy, world_iz, key):
    """Both lanes over an index box, C order over (ix, iy, iz), flat.

    Restates keyed_uniforms (steam/noise.py:103-130).
    """
    ix = np.asarray(world_ix, dtype=np.int64).astype(np.uint64)
    iy = np.asarray(world_iy, dtype=np.int64).astype(np.uint64)
    iz = np.asarray(world_iz, dtype=np.int64).astype(np.uint64)
    n = ix.size * iy.size * iz.size
    lane0 = np.empty(n, dtype=np.float32)
    lane1 = np.empty(n, dtype=np.float32)
    plane = iy.size * iz.size
    if n == 0:
        return lane0, lane1
    IY = np.repeat(iy, iz.size)
    IZ = np.tile(iz, iy.size)

    def fill(a):
        u0, u1 = uniform_pair(np.full(plane, ix[a], dtype=np.uint64), IY, IZ, key)
        lane0[a * plane:(a + 1) * plane] = u0
        lane1[a * plane:(a + 1) * plane] = u1

    _pool_map(fill, list(range(ix.size)))
    return lane0, lane1


def class_key(seed_sequence):
    """96-bit class key from a SeedSequence child (steam/noise.py:133-146)."""
    if not isinstance(seed_sequence, np.random.SeedSequence):
        seed_sequence = np.random.SeedSequence(seed_sequence)
    state = seed_sequence.generate_state(3, dtype=np.uint32)
    return tuple(int(v) for v in state)


def center_indices(n, origin, world_n, factor, wrap):
    """Turbulon-centre cells of one axis (steam/noise.py:149-182)."""
    local = np.arange(int(n), dtype=np.int64)
    world = local + int(origin)
    if wrap:
        world = world % int(world_n)
    keep = (world % int(factor)) == 0
    return local[keep], world[keep]


# ---------------------------------------------------------------------------
# a6: Chambers-Mallows-Stuck extremal Levy transform (steam/simulate.py:413-479)
# ---------------------------------------------------------------------------

def levy_from_uniforms(alpha, u0, u1, dtype=np.float32):
    """CMS draws from two uniform lanes.

    float32 mode follows the operation order of _levy_chunk
    (steam/simulate.py:413-438) with phi0/sign from _levy_from_uniforms
    (:441-479); float64 mode evaluates the same expression in float64.
    """
    t = np.dtype(dtype).type
    alpha = float(alpha)
    phi0 = t(-(np.pi / 2.0) * (1.0 - abs(1.0 - alpha)) / alpha)
    sign = t(1.0 if alpha > 1.0 else -1.0)
    eps = t(LEVY_EPS)
    phi = np.asarray(u0).astype(dtype)
    R = np.asarray(u1).astype(dtype)
    phi = (phi - t(0.5)) * t(np.pi)
    R = -np.log(np.maximum(R, eps))
    factor = np.maximum(np.cos(phi), eps) * t(abs(alpha - 1.0))
    factor = factor ** t(-1.0 / alpha)
    shifted = (phi - phi0) * t(alpha)
    tail = np.maximum(np.cos(phi - shifted), eps) / R
    tail = tail ** t((1.0 - alpha) / alpha)
    return np.sin(shifted) * sign * factor * tail


def keyed_sparse_levy(shape, sparsity_factors, alpha, key, origin=(0, 0, 0),
                      world_shape=None, dtype=np.float32):
    """Sparse world-keyed Levy generator field (steam/simulate.py:554-598)."""
    nx, ny, nz = (int(n) for n in shape)
    if world_shape is None:
        world_shape = (nx, ny, nz)
    sx, sy, sz = sparsity_factors
    lx, wx = center_indices(nx, origin[0], world_shape[0], sx, True)
    ly, wy = center_indices(ny, origin[1], world_shape[1], sy, True)
    lz, wz = center_indices(nz, origin[2], world_shape[2], sz, False)
    field = np.zeros((nx, ny, nz), dtype=dtype)
    if lx.size * ly.size * lz.size == 0:
        return field
    u0, u1 = keyed_uniforms(wx, wy, wz, key)
    draws = levy_from_uniforms(alpha, u0, u1, dtype)
    field[np.ix_(lx, ly, lz)] = draws.reshape(lx.size, ly.size, lz.size)
    return field


# ---------------------------------------------------------------------------
# a8: turbulon kernel (steam/simulate.py:2503-2556, steam/turbulons.py:23-48)
# ---------------------------------------------------------------------------

def turbulon_envelope(k, dx, dy, dz, support_factor=SUPPORT_FACTOR,
                      shape='mexican_hat', dtype=np.float32):
    """Centred kernel with the Gaussian-weighted zero-sum correction."""
    t = np.dtype(dtype).type
    hx = int(np.ceil(support_factor * k / dx))
    hy = int(np.ceil(support_factor * k / dy))
    hz = int(np.ceil(support_factor * k / dz))
    x = np.arange(-hx, hx + 1, dtype=dtype) * t(dx)
    y = np.arange(-hy, hy + 1, dtype=dtype) * t(dy)
    z = np.arange(-hz, hz + 1, dtype=dtype) * t(dz)
    r2 = x[:, None, None] ** 2 + y[None, :, None] ** 2 + z[None, None, :] ** 2
    sigma2 = (k / np.pi) ** 2
    ratio = r2 / t(sigma2)
    if shape == 'mexican_hat':
        env = (t(3.0) - ratio) * np.exp(-ratio / t(2.0))
    elif shape == 'morlet_omega0_6':
        env = np.cos(t(6.0 / k) * np.sqrt(r2)) * np.exp(-ratio / t(2.0))
    else:
        raise ValueError(f"Unknown shape {shape!r}")
    env = env.astype(dtype)
    gauss = np.exp(-r2 / t(2.0 * sigma2)).astype(dtype)
    env -= gauss * (env.sum() / gauss.sum())
    return env


def fold_kernel_to_field(kernel, field_shape):
    """Periodise a kernel wider than the field (steam/utils.py:222-242)."""
    result = kernel
    for axis in (0, 1):
        n_field = field_shape[axis]
        n_kern = result.shape[axis]
        if n_kern <= n_field:
            continue
        folded_shape = list(result.shape)
        folded_shape[axis] = n_field
        folded = np.zeros(folded_shape, dtype=result.dtype)
        center = n_kern // 2
        for i in range(n_kern):
            target = (i - center) % n_field
            src = [slice(None)] * 3
            dst = [slice(None)] * 3
            src[axis] = i
            dst[axis] = target
            folded[tuple(dst)] += result[tuple(src)]
        result = np.roll(folded, n_field // 2, axis=axis)
    return result


# ---------------------------------------------------------------------------
# a9/a10: circular-x/y, linear-z convolution (steam/utils.py:293-427)
# ---------------------------------------------------------------------------

def convolve(field, kernel, workers=None):
    """out[x,y,z] = sum K[i,j,l] f[(x-i+cx)%nx, (y-j+cy)%ny, z-l+cz].

    cx, cy, cz = (k-1)//2 as in convolve_fft_xy_oa_z (steam/utils.py:315-318),
    after folding (:307).  Evaluated as one float64 FFT over the full x/y
    period and the linear z extent, then cast to the field's dtype.
    """
    import scipy.fft as sfft
    workers = N_THREADS if workers is None else workers
    kernel = fold_kernel_to_field(np.asarray(kernel), field.shape)
    nx, ny, nz = field.shape
    kx, ky, kz = kernel.shape
    cx, cy, cz = (kx - 1) // 2, (ky - 1) // 2, (kz - 1) // 2
    nzl = nz + kz - 1
    kp = np.zeros((nx, ny, kz), dtype=np.float64)
    kp[:kx, :ky, :] = kernel
    kp = np.roll(kp, (-cx, -cy), axis=(0, 1))
    shape = (nx, ny, nzl)
    ks = sfft.rfftn(kp, s=shape, workers=workers)
    fs = sfft.rfftn(np.asarray(field, dtype=np.float64), s=shape, workers=workers)
    fs *= ks
    out = sfft.irfftn(fs, s=shape, workers=workers)
    return np.ascontiguousarray(out[..., cz:cz + nz]).astype(field.dtype)


# ---------------------------------------------------------------------------
# a7/a11: multiplier noise and flux advance (steam/simulate.py:2066-2228)
# ---------------------------------------------------------------------------

def _inner(a, window):
    if window is None:
        return a
    x0, x1, y0, y1 = window
    return a[x0:x1, y0:y1]


def multiplier_noise(generator, per_class_scale, shift, n_zero=0,
                     zero_bottom=False, zero_top=False):
    """exp(gamma)-1 at centres, 0 elsewhere (steam/simulate.py:2144-2161)."""
    t = generator.dtype.type
    gen = generator.copy()
    if zero_bottom and n_zero > 0:
        gen[:, :, :n_zero] = 0
    if zero_top and n_zero > 0:
        gen[:, :, -n_zero:] = 0
    gen *= t(per_class_scale)
    off = gen == 0.0
    gen -= t(shift)
    np.expm1(gen, out=gen)
    gen[off] = 0
    return gen


def advance_flux(flux, key, kernel, flux_noise_scale, n_per_dyad,
                 sparsity_factors, n_zero=0, zero_bottom=False, zero_top=False,
                 alpha=1.8, origin=(0, 0, 0), world_shape=None, window=None,
                 dtype=None):
    """One flux advance.  Mutates ``flux``; returns (S, record).

    Follows _advance_flux (steam/simulate.py:2066-2228): entering volume sum,
    world-keyed sparse Levy, multiplier noise, mean |noise| over centres,
    P = noise*F, S = P / mean|noise|, F += T*P, clip at 0, realized sum,
    rescale to the entering mean.  Sums are float64 as in the reference.
    """
    dtype = flux.dtype if dtype is None else np.dtype(dtype)
    t = dtype.type
    ent = _inner(flux, window)
    entering = (float(ent.sum(dtype=np.float64)), ent.size)
    entering_mean = entering[0] / max(entering[1], 1)
    pcs = flux_noise_scale / n_per_dyad ** (1.0 / alpha)
    shift = (1.0 / (alpha - 1.0)) * pcs ** alpha
    gen = keyed_sparse_levy(flux.shape, sparsity_factors, alpha, key, origin,
                            world_shape, dtype)
    noise = multiplier_noise(gen, t(pcs), t(shift), n_zero, zero_bottom, zero_top)
    ni = _inner(noise, window)
    noise_abs = (float(np.abs(ni).sum(dtype=np.float64)), int(np.count_nonzero(ni)))
    mean_abs = noise_abs[0] / max(noise_abs[1], 1)
    noise *= flux
    if mean_abs > 0:
        S = noise * t(1.0 / mean_abs)
    else:
        S = noise.copy()
    inc = convolve(noise, kernel.astype(dtype))
    flux += inc
    n_clipped = int(np.count_nonzero(flux < 0))
    np.maximum(flux, t(0.0), out=flux)
    rv = _inner(flux, window)
    realized = (float(rv.sum(dtype=np.float64)), rv.size)
    realized_mean = realized[0] / max(realized[1], 1)
    if realized_mean > 0:
        flux *= t(entering_mean / realized_mean)
    else:
        flux[...] = t(entering_mean)
    record = {'entering': entering, 'noise_abs': noise_abs,
              'realized': realized, 'n_clipped': n_clipped,
              'per_class_scale': pcs, 'shift': shift}
    return S, record


# ---------------------------------------------------------------------------
# a12: scalar pattern (steam/simulate.py:1928-1992, 2787-2930)
# ---------------------------------------------------------------------------

def z_difference_coefficients(z_coords, dtype=np.float32):
    """np.gradient's z coefficients (steam/simulate.py:2729-2762), float32 in
    the reference; the FP64 oracle evaluates them in float64."""
    z = np.asarray(z_coords, dtype=dtype)
    dz = np.diff(z)
    uniform = bool((dz == dz[0]).all())
    if uniform:
        return True, z.dtype.type(2.0) * dz[0], None, None, None, dz[0], dz[-1]
    dz1, dz2 = dz[:-1], dz[1:]
    a = -(dz2) / (dz1 * (dz1 + dz2))
    b = (dz2 - dz1) / (dz1 * dz2)
    c = dz1 / (dz2 * (dz1 + dz2))
    return False, z.dtype.type(0.0), a, b, c, dz[0], dz[-1]


def advective_weight(field, dx, dy, z_coords, aspect, dtype=None):
    """W = |grad_h f| + aspect(z)|df/dz| (steam/simulate.py:2787-2868).

    Periodic central differences in x/y, np.gradient (edge_order=1) in z.
    """
    dtype = field.dtype if dtype is None else np.dtype(dtype)
    t = dtype.type
    f = field.astype(dtype)
    two_dx, two_dy = t(2 * dx), t(2 * dy)
    gx = (np.roll(f, -1, 0) - np.roll(f, 1, 0)) / two_dx
    gy = (np.roll(f, -1, 1) - np.roll(f, 1, 1)) / two_dy
    gh = np.sqrt(gx * gx + gy * gy)
    uni, two_dz, a, b, c, dzf, dzl = z_difference_coefficients(z_coords, dtype)
    gz = np.empty_like(f)
    if uni:
        gz[:, :, 1:-1] = np.abs((f[:, :, 2:] - f[:, :, :-2]) / t(two_dz))
    else:
        a, b, c = (np.asarray(v).astype(dtype) for v in (a, b, c))
        gz[:, :, 1:-1] = np.abs(a * f[:, :, :-2] + b * f[:, :, 1:-1] + c * f[:, :, 2:])
    gz[:, :, 0] = np.abs((f[:, :, 1] - f[:, :, 0]) / t(dzf))
    gz[:, :, -1] = np.abs((f[:, :, -1] - f[:, :, -2]) / t(dzl))
    return gz * np.asarray(aspect).astype(dtype) + gh


def bound_taper(running, b, phi_min, phi_max):
    """g = clip(min(phi-lo, span-(phi-lo))/b, 0, 1) (steam/simulate.py:2905-2930)."""
    t = running.dtype.type
    g = running - t(phi_min)
    span = t(phi_max - phi_min)
    g = np.minimum(g, span - g)
    b = np.asarray(b).astype(running.dtype)
    g = g / np.where(b > 0, b, t(1e-30))
    return np.clip(g, t(0.0), t(1.0))


def scalar_pattern(perturbation, mean_1d, S, dx, dy, z_coords, aspect, b,
                   phi_min, phi_max, C_k, window=None):
    """Normalised pattern W*S*g/level_mean*C_k and its level sums.

    Follows the per-scalar body of cascade_loop (steam/simulate.py:1928-1992).
    Returns (W, level_total, level_count).
    """
    t = perturbation.dtype.type
    running = perturbation + np.asarray(mean_1d).astype(perturbation.dtype)[None, None, :]
    W = advective_weight(running, dx, dy, z_coords, aspect)
    W = W * S
    W = W * bound_taper(running, b, phi_min, phi_max)
    inner = _inner(W, window)
    total = np.abs(inner).sum(axis=(0, 1), dtype=np.float64)
    count = np.count_nonzero(inner, axis=(0, 1))
    level_mean = (total / np.maximum(count, 1)).astype(perturbation.dtype)
    W = W / np.where(level_mean > 0, level_mean, t(1.0))[None, None, :]
    W = W * np.asarray(C_k).astype(perturbation.dtype)[None, None, :]
    return W, total, count


# ---------------------------------------------------------------------------
# a14: bounded amplitude-preserving add (steam/simulate.py:3114-3283, CPU path)
# ---------------------------------------------------------------------------

def bounded_amplitude_add(perturbation, mean_1d, increment, phi_min, phi_max,
                          window=None, n_rescale=10, record_applied=False):
    """Per-level solve; mutates ``perturbation`` (and ``increment`` when
    ``record_applied``).  Returns a dict of per-level scalars."""
    dtype = perturbation.dtype
    t = dtype.type
    nz = perturbation.shape[2]
    lo, hi = t(phi_min), t(phi_max)
    width = float(phi_max) - float(phi_min)
    out = {'a0': np.zeros(nz), 'n_loop': np.zeros(nz, np.int32),
           'mu': np.full(nz, np.nan)}

    def solve_level(lev):
        phi = perturbation[:, :, lev] + t(mean_1d[lev])
        cap_lo, cap_hi = lo - phi, hi - phi
        d = np.ascontiguousarray(increment[:, :, lev]).astype(dtype)
        dw = _inner(d, window)
        a0 = float(np.abs(dw).mean(dtype=np.float64))
        out['a0'][lev] = a0
        if a0 <= 0.0:
            np.clip(d, cap_lo, cap_hi, out=d)
        else:
            n_loop = 0
            for step in range(n_rescale):
                demean = dw.mean(dtype=np.float64)
                d -= t(demean)
                n_loop = step + 1
                np.clip(d, cap_lo, cap_hi, out=d)
                m_abs = float(np.abs(dw).mean(dtype=np.float64))
                if m_abs <= 0.0:
                    break
                scale = min(a0 / m_abs, 2.0)
                if abs(scale - 1.0) < 1e-4:
                    break
                d *= t(scale)
            out['n_loop'][lev] = n_loop
            final_demean = dw.mean(dtype=np.float64)
            d -= t(final_demean)
            np.clip(d, cap_lo, cap_hi, out=d)
            if abs(float(dw.mean(dtype=np.float64))) > 1e-9 * a0:
                mu_lo, mu_hi = -width, width
                trial = np.empty_like(d)
                tw = _inner(trial, window)
                for _ in range(60):
                    mu = 0.5 * (mu_lo + mu_hi)
                    np.subtract(d, t(mu), out=trial)
                    np.clip(trial, cap_lo, cap_hi, out=trial)
                    if float(tw.mean(dtype=np.float64)) > 0.0:
                        mu_lo = mu
                    else:
                        mu_hi = mu
                mu = 0.5 * (mu_lo + mu_hi)
                out['mu'][lev] = mu
                np.subtract(d, t(mu), out=d)
                np.clip(d, cap_lo, cap_hi, out=d)
        before = perturbation[:, :, lev].copy()
        perturbation[:, :, lev] += d
        if record_applied:
            increment[:, :, lev] = perturbation[:, :, lev] - before

    _pool_map(solve_level, list(range(nz)), threads=min(N_THREADS, max(1, nz)))
    return out


def project_onto_bounds(perturbation, mean_1d, phi_min, phi_max, window=None):
    """Mean-preserving projection per level (steam/simulate.py:3417-3489)."""
    lo, hi = float(phi_min), float(phi_max)
    width = hi - lo
    nz = perturbation.shape[2]
    mus = np.full(nz, np.nan)
    for lev in range(nz):
        f = perturbation[:, :, lev].astype(np.float64) + float(mean_1d[lev])
        if f.min() >= lo and f.max() <= hi:
            continue
        fi = _inner(f, window)
        target = fi.mean()
        mlo, mhi = -width, width
        for _ in range(60):
            mu = 0.5 * (mlo + mhi)
            if np.clip(fi - mu, lo, hi).mean() > target:
                mlo = mu
            else:
                mhi = mu
            if mhi - mlo < 1e-12 * width:
                break
        mu = 0.5 * (mlo + mhi)
        mus[lev] = mu
        f = np.clip(f - mu, lo, hi) - float(mean_1d[lev])
        perturbation[:, :, lev] = f
    return mus


def compose_output(state, deficit, mean_1d, phi_min, phi_max, window=None):
    """state + deficit + mean, projected and clamped (steam/simulate.py:3558-3599)."""
    t = state.dtype.type
    m = np.asarray(mean_1d).astype(state.dtype)[None, None, :]
    if deficit is None:
        out = state + m
    else:
        d = deficit + state
        project_onto_bounds(d, mean_1d, phi_min, phi_max, window)
        out = d + m
    return np.clip(out, t(phi_min), t(phi_max))


def compose_flux_output(state, deficit, window=None):
    """Flux state + deficit, clip, volume-mean restore (steam/simulate.py:3602-3649)."""
    if deficit is None:
        return state.copy()
    t = state.dtype.type
    e = _inner(state, window)
    em = float(e.sum(dtype=np.float64)) / e.size
    out = deficit + state
    np.maximum(out, t(0.0), out=out)
    r = _inner(out, window)
    rm = float(r.sum(dtype=np.float64)) / r.size
    if rm > 0:
        out *= t(em / rm)
    else:
        out[...] = t(em)
    return out


# ---------------------------------------------------------------------------
# a15: periodic trilinear regrid (steam/utils.py:435-534)
# ---------------------------------------------------------------------------

def _axis_weights(n_in, n_out, periodic):
    """Source indices and weights of align_corners=False linear resampling.

    Matches torch's area_pixel_compute_source_index in float32:
    src = max(scale*(dst+0.5)-0.5, 0) with scale = n_in/n_out, except that a
    periodic axis wraps instead of clamping (what the wrapped pad of
    steam/utils.py:_wrap_plan achieves).
    """
    scale = np.float32(np.float32(n_in) / np.float32(n_out))
    dst = np.arange(n_out, dtype=np.float32)
    src = scale * (dst + np.float32(0.5)) - np.float32(0.5)
    if periodic:
        i0 = np.floor(src).astype(np.int64)
        lam = (src - i0.astype(np.float32)).astype(np.float32)
        i1 = (i0 + 1) % n_in
        i0 = i0 % n_in
    else:
        src = np.maximum(src, np.float32(0.0))
        i0 = np.floor(src).astype(np.int64)
        lam = (src - i0.astype(np.float32)).astype(np.float32)
        i0 = np.minimum(i0, n_in - 1)
        i1 = np.minimum(i0 + 1, n_in - 1)
    return i0, i1, lam


def zoom_trilinear(field, target_shape, periodic=(True, True, False)):
    """Cell-consistent trilinear resample with periodic x/y (utils.py:507-534)."""
    f = np.asarray(field)
    t = f.dtype.type
    out = f
    for axis in range(3):
        n_in, n_out = out.shape[axis], int(target_shape[axis])
        if n_in == n_out:
            continue
        i0, i1, lam = _axis_weights(n_in, n_out, periodic[axis])
        a = np.take(out, i0, axis=axis)
        b = np.take(out, i1, axis=axis)
        shp = [1, 1, 1]
        shp[axis] = n_out
        lam = lam.astype(f.dtype).reshape(shp)
        out = (t(1.0) - lam) * a + lam * b
    return np.ascontiguousarray(out.astype(f.dtype))


# ---------------------------------------------------------------------------
# a17: thermodynamics (steam/thermodynamics.py:25-123, 447-477)
# ---------------------------------------------------------------------------

def _es(T):
    return 611.2 * np.exp(17.67 * (T - 273.15) / (T - 29.65))


def recover_diagnostics(h, qt, z_values, surface_pressure, dtype=None):
    """Column march upward; float64 pressure accumulator."""
    dtype = h.dtype if dtype is None else np.dtype(dtype)
    h = h.astype(dtype)
    qt = qt.astype(dtype)
    nx, ny, nz = h.shape
    T = np.empty_like(h)
    qv = np.empty_like(h)
    qc = np.empty_like(h)
    qi = np.empty_like(h)
    p = np.empty_like(h)
    p_cur = np.empty((nx, ny), dtype=np.float64)
    p_cur[:] = surface_pressure
    for iz in range(nz):
        z = z_values[iz]
        pl = p_cur.astype(dtype)
        p[:, :, iz] = pl
        hl, ql = h[:, :, iz], qt[:, :, iz]
        Td = (hl - LV * ql - GRAV * z) / CP
        es = _es(Td)
        qvs = 0.622 * es / (pl - es)
        sat = ql > qvs
        Tl = Td.copy()
        qvl = ql.copy()
        if np.any(sat):
            Tn = Td[sat].copy()
            ps = pl[sat]
            hs = hl[sat]
            for _ in range(5):
                e = _es(Tn)
                q = 0.622 * e / (ps - e)
                f = CP * Tn + LV * q + GRAV * z - hs
                de = 4302.6 * e / (Tn - 29.65) ** 2
                dq = 0.622 * ps / (ps - e) ** 2 * de
                Tn = Tn - f / (CP + LV * dq)
            Tl[sat] = Tn
            e = _es(Tn)
            qvl[sat] = 0.622 * e / (ps - e)
        cond = np.maximum(ql - qvl, 0.0)
        lam = np.clip((Tl - 235.15) / (273.15 - 235.15), 0.0, 1.0)
        T[:, :, iz] = Tl
        qv[:, :, iz] = qvl
        qc[:, :, iz] = lam * cond
        qi[:, :, iz] = (1.0 - lam) * cond
        if iz < nz - 1:
            dz = float(z_values[iz + 1] - z_values[iz])
            Tv = Tl.astype(np.float64) * (1.0 + 0.608 * qvl.astype(np.float64))
            p_cur *= np.exp(-GRAV * dz / (RD * Tv))
    return {"T": T, "qv": qv, "qc": qc, "qi": qi, "p": p}


# ---------------------------------------------------------------------------
# a18: one size class of cascade_loop (steam/simulate.py:1798-2029)
# ---------------------------------------------------------------------------

def class_step(h_pert, qt_pert, flux, key, kernel, *, h_mean, qt_mean,
               z_coords, dx, dy, aspect, C_h, C_qt, b_h, b_qt,
               h_min, h_max, qt_min, qt_max, flux_noise_scale, n_per_dyad,
               sparsity_factors, n_zero, zero_bottom=True, zero_top=True,
               alpha=1.8, origin=(0, 0, 0), world_shape=None, window=None):
    """One class of the cascade on one grid (no regrid).  Mutates the three
    state fields and returns the per-class record and the applied increments.
    """
    S, frec = advance_flux(flux, key, kernel, flux_noise_scale, n_per_dyad,
                           sparsity_factors, n_zero, zero_bottom, zero_top,
                           alpha, origin, world_shape, window)
    rec = {'flux': frec}
    incs = {}
    for name, pert, mean, C, b, lo, hi in (
            ('h', h_pert, h_mean, C_h, b_h, h_min, h_max),
            ('qt', qt_pert, qt_mean, C_qt, b_qt, qt_min, qt_max)):
        W, tot, cnt = scalar_pattern(pert, mean, S, dx, dy, z_coords, aspect,
                                     b, lo, hi, C, window)
        inc = convolve(W, kernel.astype(pert.dtype))
        rec[name] = bounded_amplitude_add(pert, mean, inc, lo, hi, window,
                                          record_applied=True)
        rec[name]['level_total'] = tot
        rec[name]['level_count'] = cnt
        incs[name] = inc
    return rec, incs
