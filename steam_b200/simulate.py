"""STEAM cascade on the B200: the reference's ``steam.simulate`` interface.

Host Python keeps the reference's signatures, argument checks, grid ladder and
1D amplitude tables; every field-sized operation runs in hand-written sm_100a
kernels through the C ABI (``_lib``), on fields that stay resident in HBM for
the whole cascade.  Public functions accept the reference's numpy arrays (and
return numpy arrays) or CUDA tensors (and stay on the device).

Citations are file:line into thomasdewitt/STEAM.
"""

from __future__ import annotations

import ctypes
from pathlib import Path
from typing import NamedTuple

import numpy as np

from . import _lib
from . import constants
from .constants import (
    hurst_horizontal as H_h,
    hurst_vertical_anisotropy as H_z,
    haar_to_mhat as HAAR_TO_MHAT,
)
from .ledger import (
    BoundedAddLedger,
    FluxAdvanceLedger,
    FluxOutputLedger,
    MeanReduction,
    PatternLedger,
    ProjectionLedger,
    RunLedger,
)
from .noise import center_indices, class_key
from .turbulons import SHAPES, SHAPE_CODES
from ._device import check_device, is_tensor, to_device, to_host, torch_dtype
from . import utils as _utils

# ---------------------------------------------------------------------------
# Model constants (steam/simulate.py:58, 115-116, 517)
# ---------------------------------------------------------------------------
SUPPORT_FACTOR = 3
FLUX_SCALE = 0.2085
FLUX_ALPHA = 1.8
BOUND_BUFFER_MULTIPLE = 3
LEVY_LOG_MEAN = 1.0 / (FLUX_ALPHA - 1.0)
VALID_ANISOTROPY = ('canonical', 'piecewise_isotropic_below_spheroscale')


def levy_log_mean(alpha):
    """ln <exp(gamma_0)> = 1/(alpha - 1) for the unit-scale generator
    (steam/simulate.py:505-517)."""
    return 1.0 / (float(alpha) - 1.0)


# ---------------------------------------------------------------------------
# Interpolation compensation tables (steam/simulate.py:226-351)
# ---------------------------------------------------------------------------
HOP_RETENTION = {
    'canonical': {2: 0.5664, 4: 0.7456, 8: 0.8926, 16: 0.9667,
                  32: 0.9730, 64: 0.9746, 128: 0.9871, 256: 0.9880},
    'isotropic': {2: 0.5401, 4: 0.8362, 8: 0.9587, 16: 0.9839,
                  32: 0.9956},
}


def _hop_retention(y, regime):
    table = HOP_RETENTION[regime]
    xs = np.array(sorted(table), dtype=np.float64)
    rs = np.array([table[x] for x in xs])
    if y >= 2.0 * xs[-1]:
        return 1.0
    if y <= xs[0]:
        return float(rs[0])
    return float(np.interp(np.log2(y), np.log2(xs), rs))


def _canonical_delivery_reference():
    d = 1.0
    for y in sorted(HOP_RETENTION['canonical']):
        d *= HOP_RETENTION['canonical'][y]
    return d


def _build_canonical_table():
    d_ref = _canonical_delivery_reference()
    table, d = {}, 1.0
    for y in sorted(HOP_RETENTION['canonical']):
        table[y] = d_ref / d
        d *= HOP_RETENTION['canonical'][y]
    table[2 * max(HOP_RETENTION['canonical'])] = 1.0
    return table


INTERPOLATION_COMPENSATION = _build_canonical_table()


def _interpolation_compensation(k_over_dx):
    if not INTERPOLATION_COMPENSATION:
        return 1.0
    xs = np.array(sorted(INTERPOLATION_COMPENSATION), dtype=np.float64)
    fs = np.array([INTERPOLATION_COMPENSATION[x] for x in xs])
    if k_over_dx >= xs[-1]:
        return float(fs[-1])
    if k_over_dx <= xs[0]:
        return float(fs[0])
    return float(np.interp(np.log2(k_over_dx), np.log2(xs), fs))


def _hop_retention_profile(y, k_dest, ls_z, anisotropy):
    r_can = _hop_retention(y, 'canonical')
    if anisotropy != 'piecewise_isotropic_below_spheroscale':
        return np.full(np.shape(ls_z), r_can)
    r_iso = _hop_retention(y, 'isotropic')
    return np.where(k_dest < np.asarray(ls_z), r_iso, r_can)


def _compensation_profiles(k_values, z_arrays, spheroscale_profile, z_profile,
                           anisotropy):
    """f_i(z) = D_REF / D_i(z) over each class's regrid chain
    (steam/simulate.py:320-351)."""
    if not INTERPOLATION_COMPENSATION:
        return [np.ones(len(z), dtype=np.float32) for z in z_arrays]
    d_ref = _canonical_delivery_reference()
    out = []
    for i, z_i in enumerate(z_arrays):
        ls_z = np.interp(z_i, z_profile, spheroscale_profile)
        D = np.ones(ls_z.shape, dtype=np.float64)
        for m in range(i + 1, len(k_values)):
            y = 2.0 * float(k_values[i]) / float(k_values[m - 1])
            D *= _hop_retention_profile(y, float(k_values[m]), ls_z, anisotropy)
        out.append((d_ref / D).astype(np.float32))
    return out


# ---------------------------------------------------------------------------
# World-keyed noise (steam/simulate.py:520-598)
# ---------------------------------------------------------------------------

class NoiseRegion(NamedTuple):
    """Where an array sits in the world: class key, world origin of cell
    (0,0,0), world grid shape (x/y wrap, z never) (steam/simulate.py:520-551)."""
    key: tuple
    origin: tuple
    world_shape: tuple

    @classmethod
    def root(cls, seed_sequence, shape):
        return cls(class_key(seed_sequence), (0, 0, 0), tuple(int(n) for n in shape))


def _region_struct(region, shape, sparsity_factors):
    r = _lib.Region()
    for a in range(3):
        r.shape[a] = int(shape[a])
        r.origin[a] = int(region.origin[a])
        r.world[a] = int(region.world_shape[a])
        r.sparsity[a] = int(sparsity_factors[a])
        r.key[a] = int(region.key[a]) & 0xFFFFFFFF
    for a, s in enumerate(sparsity_factors):
        if int(s) < 1:
            raise ValueError(f"sparsity factor {a} must be >= 1, got {s}")
    return r


def levy_field_device(shape, sparsity_factors, alpha, region, dtype=None):
    """Sparse keyed Levy generator as a CUDA tensor."""
    torch = _lib.require_cuda("_keyed_sparse_levy")
    dtype = torch.float32 if dtype is None else dtype
    out = torch.empty(tuple(int(n) for n in shape), dtype=dtype, device='cuda')
    lib = _lib.load()
    _lib.check(lib.steam_levy_field(_lib.dtype_code(out),
                                    ctypes.byref(_region_struct(region, shape, sparsity_factors)),
                                    float(alpha), _lib.ptr(out), _lib.stream()))
    return out


def _keyed_sparse_levy(shape, sparsity_factors, alpha, region, dtype=np.float32):
    """Sparse extremal-Levy generator field keyed to the world
    (steam/simulate.py:554-598).  Returns a float32 numpy array."""
    out = levy_field_device(shape, sparsity_factors, alpha, region, torch_dtype(dtype))
    return to_host(out)


# ---------------------------------------------------------------------------
# Grids (steam/simulate.py:604-626, 2356-2500)
# ---------------------------------------------------------------------------

def _k_z(anisotropy, k, spheroscale):
    """Vertical scale k_z(k, l_s) (steam/simulate.py:604-626)."""
    k = np.asarray(k, dtype=np.float64)
    spheroscale = np.asarray(spheroscale, dtype=np.float64)
    canonical = spheroscale * (k / spheroscale) ** H_z
    if anisotropy == 'canonical':
        return canonical
    if anisotropy == 'piecewise_isotropic_below_spheroscale':
        return np.where(k >= spheroscale, canonical, k)
    raise ValueError(f"Unknown anisotropy {anisotropy!r}. Valid options: {VALID_ANISOTROPY}")


def _compute_all_grids(k_values, inner_extent_x, inner_extent_y, inner_height,
                       sparsity_factors, spheroscale_profile, z_profile, z_min=0.0,
                       pad_x_per_class=None, pad_y_per_class=None,
                       pad_z_below_per_class=None, pad_z_above_per_class=None,
                       anisotropy='piecewise_isotropic_below_spheroscale'):
    """Per-class grid counts and variable-dz z ladders (steam/simulate.py:2356-2500)."""
    spheroscale_profile = np.asarray(spheroscale_profile, dtype=np.float64)
    z_profile = np.asarray(z_profile, dtype=np.float64)
    if spheroscale_profile.ndim == 0:
        spheroscale_profile = np.full_like(z_profile, float(spheroscale_profile))
    s_x, s_y, s_z = sparsity_factors
    n = len(k_values)
    zeros = np.zeros(n)

    def per_class(v):
        return zeros if v is None else np.asarray(v, dtype=np.float64)

    pad_x, pad_y = per_class(pad_x_per_class), per_class(pad_y_per_class)
    pad_zb, pad_za = per_class(pad_z_below_per_class), per_class(pad_z_above_per_class)
    out = {key: np.empty(n, dtype=np.int64) for key in ('nx', 'ny', 'nz')}
    for key in ('dx', 'dy', 'dz', 'padded_extent_x', 'padded_extent_y',
                'padded_height', 'z_min_per_class'):
        out[key] = np.empty(n, dtype=np.float64)
    z_arrays, dz_arrays = [], []
    for i, k in enumerate(k_values):
        ext_x = inner_extent_x + 2 * pad_x[i]
        ext_y = inner_extent_y + 2 * pad_y[i]
        height = inner_height + pad_zb[i] + pad_za[i]
        z_lo = z_min - pad_zb[i]
        out['nx'][i] = max(1, int(round(ext_x / (k / (2 * s_x)))))
        out['ny'][i] = max(1, int(round(ext_y / (k / (2 * s_y)))))
        out['dx'][i] = ext_x / out['nx'][i]
        out['dy'][i] = ext_y / out['ny'][i]
        edges = [z_lo]
        top = z_lo + height
        while edges[-1] < top:
            ls = np.interp(edges[-1], z_profile, spheroscale_profile)
            edges.append(edges[-1] + float(_k_z(anisotropy, k, ls)) / (2 * s_z))
        dz_raw = np.diff(edges)
        dz_k = dz_raw * (height / np.sum(dz_raw))
        z_k = z_lo + np.concatenate([[0.0], np.cumsum(dz_k[:-1])])
        out['nz'][i] = len(edges) - 1
        out['dz'][i] = float(np.mean(dz_k))
        out['padded_extent_x'][i] = ext_x
        out['padded_extent_y'][i] = ext_y
        out['padded_height'][i] = height
        out['z_min_per_class'][i] = z_lo
        z_arrays.append(z_k)
        dz_arrays.append(dz_k)
    out['k'] = k_values
    out['z_arrays'] = z_arrays
    out['dz_arrays'] = dz_arrays
    return out


# ---------------------------------------------------------------------------
# Turbulon kernel (steam/simulate.py:2503-2556)
# ---------------------------------------------------------------------------

def kernel_device(k, dx, dy, dz, support_factor=SUPPORT_FACTOR, shape='mexican_hat',
                  dtype=None):
    """Build the turbulon kernel on the device (float64 normalisation sums)."""
    torch = _lib.require_cuda("_turbulon_envelope")
    if shape not in SHAPES:
        raise ValueError(f"Unknown shape {shape!r}. Valid options: {sorted(SHAPES)}")
    dtype = torch.float32 if dtype is None else dtype
    lib = _lib.load()
    dims = (ctypes.c_int64 * 3)()
    code = _lib.STEAM_F64 if dtype == torch.float64 else _lib.STEAM_F32
    args = (float(k), float(dx), float(dy), float(dz), float(support_factor),
            SHAPE_CODES[shape])
    _lib.check(lib.steam_kernel_build(code, *args, None, dims, _lib.stream()))
    out = torch.empty(tuple(int(d) for d in dims), dtype=dtype, device='cuda')
    _lib.check(lib.steam_kernel_build(code, *args, _lib.ptr(out), dims, _lib.stream()))
    return out


def _turbulon_envelope(k, dx, dy, dz, support_factor=SUPPORT_FACTOR,
                       shape='mexican_hat', dtype=np.float32):
    """Compact centred turbulon kernel with the Gaussian-weighted zero-sum
    correction, as a host array (float32 like the reference by default)."""
    return to_host(kernel_device(k, dx, dy, dz, support_factor, shape, torch_dtype(dtype)))


# ---------------------------------------------------------------------------
# Normalisation ladder and buffers (steam/simulate.py:2559-2668, 2871-2902)
# ---------------------------------------------------------------------------

def _compute_normalization(profile, z_profile, k_z_L_on_profile, k_values, outer_scale,
                           z_arrays, n_scale_classes_per_dyad=1,
                           hurst_horizontal=None, haar_to_mhat=None, alpha=None):
    """C_k(z) = lambda |Haar_{k_z,L}(profile)|(z) (k/L)^H n^(-1/alpha)
    (steam/simulate.py:2559-2668): exact half-window means of the
    piecewise-linear profile."""
    H_used = H_h if hurst_horizontal is None else float(hurst_horizontal)
    lam = HAAR_TO_MHAT if haar_to_mhat is None else float(haar_to_mhat)
    alpha = FLUX_ALPHA if alpha is None else float(alpha)
    zp = np.asarray(z_profile, dtype=np.float64)
    pr = np.asarray(profile, dtype=np.float64)
    cum = np.concatenate([[0.0], np.cumsum(0.5 * (pr[1:] + pr[:-1]) * np.diff(zp))])

    def integral_to(x):
        j = np.clip(np.searchsorted(zp, x, side='right') - 1, 0, len(zp) - 2)
        inside = cum[j] + 0.5 * (pr[j] + np.interp(x, zp, pr)) * (x - zp[j])
        below = cum[0] - pr[0] * (zp[0] - x)
        above = cum[-1] + pr[-1] * (x - zp[-1])
        return np.where(x < zp[0], below, np.where(x > zp[-1], above, inside))

    half = 0.5 * np.asarray(k_z_L_on_profile, dtype=np.float64)
    centre = integral_to(zp)
    upper = (integral_to(zp + half) - centre) / half
    lower = (centre - integral_to(zp - half)) / half
    response = lam * np.abs(upper - lower)
    out = []
    for i, k in enumerate(k_values):
        scale = float((k / outer_scale) ** H_used) * n_scale_classes_per_dyad ** (-1.0 / alpha)
        out.append(np.interp(z_arrays['z_arrays'][i], zp, response).astype(np.float32) * scale)
    return out


def _bound_buffers(C_k, n_scale_classes_per_dyad, hurst_horizontal=None,
                   bound_buffer_multiple=None):
    """b_i(z) = n_b C_i(z) / (1 - 2^(-H/n)) (steam/simulate.py:2871-2902)."""
    H_used = H_h if hurst_horizontal is None else float(hurst_horizontal)
    n_b = BOUND_BUFFER_MULTIPLE if bound_buffer_multiple is None else float(bound_buffer_multiple)
    tail = 1.0 / (1.0 - 2.0 ** (-H_used / n_scale_classes_per_dyad))
    return [(n_b * tail * C_i).astype(np.float32) for C_i in C_k]


# ---------------------------------------------------------------------------
# Flux advance (steam/simulate.py:2066-2228)
# ---------------------------------------------------------------------------

class FluxStep(NamedTuple):
    """Device result of one flux advance: the product eps*F and the scale that
    turns it into the signed amplitude S = product * s_scale."""
    product: object
    s_scale: float
    ledger: FluxAdvanceLedger
    diagnostics: dict


def advance_flux_device(flux_t, noise_region, plan, flux_noise_scale,
                        n_scale_classes_per_dyad, sparsity_factors, n_zero=0,
                        zero_bottom=False, zero_top=False, window=None, ledger=None,
                        alpha=None, product_out=None):
    """Advance a resident flux tensor by one class (in place)."""
    torch = _lib.require_cuda("_advance_flux")
    lib = _lib.load()
    alpha = FLUX_ALPHA if alpha is None else float(alpha)
    shape = tuple(int(n) for n in flux_t.shape)
    code = _lib.dtype_code(flux_t)
    pcs = flux_noise_scale / n_scale_classes_per_dyad ** (1.0 / alpha)
    shift = levy_log_mean(alpha) * pcs ** alpha
    np_t = np.float64 if flux_t.dtype == torch.float64 else np.float32
    pcs_t, shift_t = float(np_t(pcs)), float(np_t(shift))
    product = torch.empty_like(flux_t) if product_out is None else product_out
    region = _region_struct(noise_region, shape, sparsity_factors)
    ws = _lib.WORKSPACE.get(lib.steam_flux_noise_workspace_bytes())
    sums = _lib.dout(4)
    _lib.check(lib.steam_flux_noise(
        code, ctypes.byref(region), alpha, pcs_t, shift_t, int(n_zero), int(bool(zero_bottom)),
        int(bool(zero_top)), _lib.ptr(flux_t), _lib.ptr(product), _lib.window_arg(window),
        sums, _lib.ptr(ws), ws.numel(), _lib.stream()))
    if ledger is None:
        entering = MeanReduction(sums[0], int(sums[1]))
        noise_abs = MeanReduction(sums[2], int(sums[3]))
    else:
        entering, noise_abs = ledger.entering, ledger.noise_abs
    mean_abs = noise_abs.mean
    s_scale = float(np_t(1.0 / mean_abs)) if mean_abs > 0 else 1.0
    plan_sums = _utils.run_plan(plan, product, flux_t, epilogue=_lib.STEAM_EPI_FLUX,
                                window=window)
    if ledger is None:
        realized = MeanReduction(plan_sums[0], int(plan_sums[1]))
        n_clipped = int(plan_sums[2])
    else:
        realized, n_clipped = ledger.realized, ledger.n_clipped
    n = flux_t.numel()
    if realized.mean > 0:
        _lib.check(lib.steam_scale(code, n, _lib.ptr(flux_t),
                                   float(np_t(entering.mean / realized.mean)), 0,
                                   _lib.stream()))
    else:
        _lib.check(lib.steam_scale(code, n, _lib.ptr(flux_t), float(np_t(entering.mean)), 1,
                                   _lib.stream()))
    diagnostics = {'n_clipped': n_clipped, 'n_points': int(n),
                   'clip_fraction': n_clipped / max(n, 1),
                   'entering_mean': entering.mean, 'realized_mean': realized.mean}
    return FluxStep(product, s_scale,
                    FluxAdvanceLedger(entering, noise_abs, realized, n_clipped), diagnostics)


def _kernel_plan(kernel, field_shape, dtype):
    return _utils.plan_convolution(np.asarray(kernel), field_shape, dtype)


def _advance_flux(flux, noise_region, kernel, flux_noise_scale, n_scale_classes_per_dyad,
                  sparsity_factors, n_zero=0, zero_bottom=False, zero_top=False,
                  device='cuda', window=None, ledger=None):
    """One flux advance (steam/simulate.py:2066-2228).  Mutates ``flux``;
    returns (scalar_amplitude, FluxAdvanceLedger, diagnostics)."""
    check_device(device, "_advance_flux")
    torch = _lib.require_cuda("_advance_flux")
    t, host = to_device(flux)
    np_t = np.float64 if t.dtype == torch.float64 else np.float32
    plan = _kernel_plan(kernel, t.shape, np_t)
    step = advance_flux_device(t, noise_region, plan, flux_noise_scale,
                               n_scale_classes_per_dyad, sparsity_factors, n_zero,
                               zero_bottom, zero_top, window, ledger)
    S = step.product
    lib = _lib.load()
    if step.ledger.noise_abs.mean > 0:
        _lib.check(lib.steam_scale(_lib.dtype_code(S), S.numel(), _lib.ptr(S),
                                   step.s_scale, 0, _lib.stream()))
    if host is not None:
        to_host(t, out=flux)
        return to_host(S), step.ledger, step.diagnostics
    return S, step.ledger, step.diagnostics


# ---------------------------------------------------------------------------
# Scalar pattern (steam/simulate.py:1928-1992, 2787-2930)
# ---------------------------------------------------------------------------

def pattern_device(pert_t, mean_1d, product_t, s_scale, dx, dy, z_coords, aspect, b,
                   phi_min, phi_max, window=None, out=None):
    """W = advective weight x S x taper on the device; returns (W, level_total,
    level_count)."""
    torch = _lib.require_cuda("scalar pattern")
    lib = _lib.load()
    nx, ny, nz = (int(n) for n in pert_t.shape)
    W = torch.empty_like(pert_t) if out is None else out
    ws = _lib.WORKSPACE.get(lib.steam_scalar_pattern_workspace_bytes(nx, ny, nz))
    sums = _lib.dout(2 * nz)
    _lib.check(lib.steam_scalar_pattern(
        _lib.dtype_code(pert_t), nx, ny, nz, _lib.ptr(pert_t), _lib.dvec(mean_1d),
        _lib.ptr(product_t) if product_t is not None else None, float(s_scale),
        float(dx), float(dy), _lib.dvec(z_coords), _lib.dvec(aspect),
        _lib.dvec(b) if b is not None else None, float(phi_min), float(phi_max),
        _lib.ptr(W), _lib.window_arg(window), sums, _lib.ptr(ws), ws.numel(),
        _lib.stream()))
    s = np.ctypeslib.as_array(sums)[:2 * nz].reshape(nz, 2)
    return W, s[:, 0].copy(), s[:, 1].astype(np.int64)


def _advective_weight(field_3d, dx, dy, z_coords, aspect_z):
    """W = |grad_h f| + aspect(z)|df/dz| (steam/simulate.py:2843-2868)."""
    _lib.require_cuda("_advective_weight")
    t, host = to_device(field_3d)
    nz = t.shape[2]
    aspect_z = np.asarray(aspect_z)
    if aspect_z.shape != (nz,):
        raise ValueError(f"aspect_z has shape {aspect_z.shape}, expected ({nz},) -- one value per level.")
    z = np.asarray(z_coords, dtype=np.float64)
    if z.ndim == 0:
        z = np.arange(nz, dtype=np.float64) * float(z)
    W, _, _ = pattern_device(t, np.zeros(nz), None, 1.0, dx, dy, z, aspect_z, None, 0.0, 1.0)
    return to_host(W) if host is not None else W


# ---------------------------------------------------------------------------
# Bounded add and projection (steam/simulate.py:3114-3489)
# ---------------------------------------------------------------------------

def bounded_add_device(pert_t, mean_1d, inc_t, phi_min, phi_max, window=None,
                       n_rescale=10, record_applied=False, ledger=None):
    """The bounded add on device tensors; with ``ledger`` (a recorded
    BoundedAddLedger) the apply-only replay, which reduces nothing and
    returns that ledger."""
    lib = _lib.load()
    nx, ny, nz = (int(n) for n in pert_t.shape)
    if ledger is not None:
        R = ledger.n_rescale
        if ledger.a0.shape[0] != nz:
            raise ValueError(f"bounded-add ledger has {ledger.a0.shape[0]} levels for {nz}")
        ws = _lib.WORKSPACE.get(lib.steam_bounded_add_replay_workspace_bytes(nz, R))
        _lib.check(lib.steam_bounded_add_replay(
            _lib.dtype_code(pert_t), nx, ny, nz, _lib.ptr(pert_t), _lib.dvec(mean_1d),
            _lib.ptr(inc_t), float(phi_min), float(phi_max), R, int(bool(record_applied)),
            _lib.dvec(ledger.to_device()), _lib.ptr(ws), ws.numel(), _lib.stream()))
        return ledger
    R = int(n_rescale)
    ws = _lib.WORKSPACE.get(lib.steam_bounded_add_workspace_bytes(nz, R))
    width = lib.steam_bounded_add_ledger_doubles(R)
    led = _lib.dout(width * nz)
    _lib.check(lib.steam_bounded_add(
        _lib.dtype_code(pert_t), nx, ny, nz, _lib.ptr(pert_t), _lib.dvec(mean_1d),
        _lib.ptr(inc_t), float(phi_min), float(phi_max), _lib.window_arg(window),
        R, int(bool(record_applied)), led, _lib.ptr(ws), ws.numel(), _lib.stream()))
    return BoundedAddLedger.from_device(np.ctypeslib.as_array(led)[:width * nz], R)


def _bounded_amplitude_add(perturbation_field, mean_1d, increment, phi_min, phi_max,
                           window=None, n_rescale=10, device='cuda', record_applied=False,
                           ledger=None):
    """Add a class increment under the three deposit conditions
    (steam/simulate.py:3114-3283).  Mutates ``perturbation_field`` (and
    ``increment`` with record_applied).  With ``ledger`` (a BoundedAddLedger a
    device solve recorded) the recorded per-level sequence is applied with no
    reduction (the apply-only replay, steam/simulate.py:3196-3213) and the
    same ledger is returned."""
    check_device(device, "_bounded_amplitude_add")
    p_t, p_host = to_device(perturbation_field)
    i_t, i_host = to_device(increment, dtype=p_t.dtype, copy=not record_applied)
    out = bounded_add_device(p_t, mean_1d, i_t, phi_min, phi_max, window, n_rescale,
                             record_applied, ledger=ledger)
    if p_host is not None:
        to_host(p_t, out=perturbation_field)
    if record_applied and i_host is not None:
        to_host(i_t, out=increment)
    return out


def project_device(pert_t, mean_1d, phi_min, phi_max, window=None, ledger=None):
    """The per-level mean-preserving projection on a device tensor; with
    ``ledger`` (a recorded ProjectionLedger) the apply-only replay."""
    lib = _lib.load()
    nx, ny, nz = (int(n) for n in pert_t.shape)
    ws = _lib.WORKSPACE.get(lib.steam_bounded_add_workspace_bytes(nz, 1))
    if ledger is not None:
        if np.asarray(ledger.mu).shape != (nz,):
            raise ValueError(f"projection ledger has {np.size(ledger.mu)} levels for {nz}")
        _lib.check(lib.steam_project_bounds_replay(
            _lib.dtype_code(pert_t), nx, ny, nz, _lib.ptr(pert_t), _lib.dvec(mean_1d),
            float(phi_min), float(phi_max), _lib.dvec(ledger.mu), _lib.ptr(ws), ws.numel(),
            _lib.stream()))
        return ledger
    mu = _lib.dout(nz)
    _lib.check(lib.steam_project_bounds(
        _lib.dtype_code(pert_t), nx, ny, nz, _lib.ptr(pert_t), _lib.dvec(mean_1d),
        float(phi_min), float(phi_max), _lib.window_arg(window), mu, _lib.ptr(ws),
        ws.numel(), _lib.stream()))
    return ProjectionLedger(np.ctypeslib.as_array(mu)[:nz].copy())


def _project_onto_bounds(perturbation_field, mean_1d, phi_min, phi_max, window=None,
                         device='cuda', ledger=None):
    """Mean-preserving projection onto [phi_min, phi_max] per level
    (steam/simulate.py:3417-3489); with ``ledger`` the recorded shifts are
    applied with no reduction (the replay branch)."""
    check_device(device, "_project_onto_bounds")
    t, host = to_device(perturbation_field)
    out = project_device(t, mean_1d, phi_min, phi_max, window, ledger=ledger)
    if host is not None:
        to_host(t, out=perturbation_field)
    return out


def _accumulate(acc_t, a_t, b_t, coef):
    lib = _lib.load()
    nx, ny, nz = (int(n) for n in acc_t.shape)
    _lib.check(lib.steam_accumulate_levels(
        _lib.dtype_code(acc_t), nx, ny, nz, _lib.ptr(acc_t), _lib.ptr(a_t),
        _lib.ptr(b_t) if b_t is not None else None, _lib.dvec(coef), _lib.stream()))


def _level_sums(t, window=None):
    lib = _lib.load()
    nx, ny, nz = (int(n) for n in t.shape)
    ws = _lib.WORKSPACE.get(lib.steam_level_sums_workspace_bytes(nz))
    out = _lib.dout(4 * nz)
    _lib.check(lib.steam_level_sums(_lib.dtype_code(t), nx, ny, nz, _lib.ptr(t),
                                    _lib.window_arg(window), out, _lib.ptr(ws), ws.numel(),
                                    _lib.stream()))
    return np.ctypeslib.as_array(out)[:4 * nz].reshape(nz, 4).copy()


def compose_output_device(state_t, deficit_t, mean_1d, phi_min, phi_max, window=None,
                          ledger=None):
    """state + deficit + mean, projected, clamped (steam/simulate.py:3558-3599).
    Consumes ``deficit_t`` (it becomes the output).  ``ledger``: a recorded
    ProjectionLedger to replay instead of solving the projection."""
    torch = _lib.require_cuda("_compose_output")
    np_t = np.float64 if state_t.dtype == torch.float64 else np.float32
    projection = None
    ones = np.ones(state_t.shape[2])
    if deficit_t is None:
        out = state_t.clone()
    else:
        _accumulate(deficit_t, state_t, None, ones)
        projection = project_device(deficit_t, mean_1d, phi_min, phi_max, window,
                                    ledger=ledger)
        out = deficit_t
    nx, ny, nz = (int(n) for n in out.shape)
    mean = np.asarray(mean_1d, dtype=np_t).astype(np.float64)
    _lib.check(_lib.load().steam_add_levels_clamp(
        _lib.dtype_code(out), nx, ny, nz, _lib.ptr(out), _lib.dvec(mean),
        float(np_t(phi_min)), float(np_t(phi_max)), _lib.stream()))
    return out, projection


def _compose_output(state, deficit, mean_1d, phi_min, phi_max, window=None,
                    device='cuda', ledger=None):
    check_device(device, "_compose_output")
    s_t, s_host = to_device(state)
    d_t = None if deficit is None else to_device(deficit, dtype=s_t.dtype, copy=True)[0]
    out, proj = compose_output_device(s_t, d_t, mean_1d, phi_min, phi_max, window,
                                      ledger=ledger)
    return (to_host(out) if s_host is not None else out), proj


def compose_flux_output_device(state_t, deficit_t, window=None, ledger=None):
    """Flux state + deficit, clip at 0, volume-mean restore
    (steam/simulate.py:3602-3649).  Consumes ``deficit_t``.  ``ledger``: a
    recorded FluxOutputLedger whose means are applied instead of measured."""
    torch = _lib.require_cuda("_compose_flux_output")
    if deficit_t is None:
        return state_t, None
    lib = _lib.load()
    np_t = np.float64 if state_t.dtype == torch.float64 else np.float32
    nx, ny, nz = (int(n) for n in state_t.shape)
    code = _lib.dtype_code(deficit_t)
    if ledger is None:
        ent = _level_sums(state_t, window)
        entering = MeanReduction(float(ent[:, 0].sum()), int(ent[:, 3].sum()))
    _accumulate(deficit_t, state_t, None, np.ones(nz))
    _lib.check(lib.steam_add_levels_clamp(code, nx, ny, nz, _lib.ptr(deficit_t),
                                          _lib.dvec(np.zeros(nz)), 0.0, float(np.inf),
                                          _lib.stream()))
    if ledger is None:
        rea = _level_sums(deficit_t, window)
        realized = MeanReduction(float(rea[:, 0].sum()), int(rea[:, 3].sum()))
    else:
        entering, realized = ledger.entering, ledger.realized
    if realized.mean > 0:
        _lib.check(lib.steam_scale(code, deficit_t.numel(), _lib.ptr(deficit_t),
                                   float(np_t(entering.mean / realized.mean)), 0, _lib.stream()))
    else:
        _lib.check(lib.steam_scale(code, deficit_t.numel(), _lib.ptr(deficit_t),
                                   float(np_t(entering.mean)), 1, _lib.stream()))
    return deficit_t, FluxOutputLedger(entering, realized)


def _compose_flux_output(state, deficit, window=None, ledger=None):
    s_t, s_host = to_device(state)
    d_t = None if deficit is None else to_device(deficit, dtype=s_t.dtype, copy=True)[0]
    out, led = compose_flux_output_device(s_t, d_t, window, ledger=ledger)
    if s_host is not None:
        return to_host(out), led
    return out, led


# ---------------------------------------------------------------------------
# Cascade drivers (steam/simulate.py:1566-2049, 2231-2353)
# ---------------------------------------------------------------------------

def _crop_between(carried, prev, cur):
    """Crop-before-zoom when the padded extent shrinks (steam/simulate.py:1839-1855)."""
    eps = 1e-9
    (px, py, ph, pdx, pdy, pdz, pzmin) = prev
    (cx, cy, ch, czmin) = cur
    lead = next(f for f in carried if f is not None)
    if cx < px - eps:
        keep = max(1, min(lead.shape[0], int(round(cx / pdx))))
        start = (lead.shape[0] - keep) // 2
        carried = [f if f is None else f[start:start + keep] for f in carried]
        lead = carried[0]
    if cy < py - eps:
        keep = max(1, min(lead.shape[1], int(round(cy / pdy))))
        start = (lead.shape[1] - keep) // 2
        carried = [f if f is None else f[:, start:start + keep] for f in carried]
        lead = carried[0]
    if ch < ph - eps:
        keep = max(1, min(lead.shape[2], int(round(ch / pdz))))
        start = int(round((czmin - pzmin) / pdz))
        start = max(0, min(lead.shape[2] - keep, start))
        carried = [f if f is None else f[:, :, start:start + keep] for f in carried]
    return [f if f is None else f.contiguous() for f in carried]


class ClassSetup(NamedTuple):
    """Everything one size class needs on its own grid (the per-class locals
    of cascade_loop, steam/simulate.py:1798-1935)."""
    shape: tuple
    z: np.ndarray
    dx: float
    dy: float
    h_mean: np.ndarray
    qt_mean: np.ndarray
    C_h: np.ndarray
    C_qt: np.ndarray
    b_h: np.ndarray
    b_qt: np.ndarray
    aspect: np.ndarray
    bounds: tuple
    region: NoiseRegion
    plan: object
    deficit: object
    window: object
    flux_noise_scale: float
    n_per_dyad: int
    sparsity: tuple
    n_zero: int
    zero_bottom: bool
    zero_top: bool
    alpha: float


def run_class(hp, qp, F, dh, dq, dF, cs, cl, increment_dir=None, index=0, resident=True):
    """One size class on resident fields (steam/simulate.py:1903-2029):
    flux advance, then for h and qt the pattern, the second convolution with
    the per-level normalisation fused into its input, and the bounded add.
    Mutates the state tensors and fills the class ledger ``cl``."""
    torch = _lib.require_cuda("cascade_loop")
    need_inc = cs.deficit is not None or increment_dir is not None
    if (resident and not need_inc and cl.flux is None and not cl.pattern
            and not cl.bounded_add):
        # measure mode: the resident step keeps every scalar on the device
        from .resident import resident_for
        resident_for(cs, F.dtype).step(hp, qp, F).class_ledger(cl)
        return
    F_before = F.clone() if need_inc else None
    step = advance_flux_device(F, cs.region, cs.plan, cs.flux_noise_scale, cs.n_per_dyad,
                               cs.sparsity, cs.n_zero, cs.zero_bottom, cs.zero_top,
                               cs.window, cl.flux, cs.alpha)
    cl.flux = step.ledger
    if need_inc:
        if cs.deficit is not None:
            _accumulate(dF, F, F_before, cs.deficit)
        if increment_dir is not None:
            np.save(Path(increment_dir) / f"c{index:02d}_flux.npy", to_host(F - F_before))
        del F_before
    h_min, h_max, qt_min, qt_max = cs.bounds
    for name, pert, dfield, mean_1d, C, b, lo, hi in (
            ('h', hp, dh, cs.h_mean, cs.C_h, cs.b_h, h_min, h_max),
            ('qt', qp, dq, cs.qt_mean, cs.C_qt, cs.b_qt, qt_min, qt_max)):
        W, tot, cnt = pattern_device(pert, mean_1d, step.product, step.s_scale, cs.dx, cs.dy,
                                     cs.z, cs.aspect, b, lo, hi, cs.window)
        if cl.pattern.get(name) is None:
            cl.pattern[name] = PatternLedger(tot, cnt)
        led = cl.pattern[name]
        # the reference divides by the level mean rounded to float32; the
        # float64 form keeps it in float64
        np_t = np.float64 if pert.dtype == torch.float64 else np.float32
        level_mean = (led.level_total / np.maximum(led.level_count, 1)).astype(np_t)
        div = np.where(level_mean > 0, level_mean, np_t(1.0))
        inc = torch.empty_like(W)
        _utils.run_plan(cs.plan, W, inc, pre_div=div, pre_mul=np.asarray(C, dtype=np.float32))
        del W
        # the applied increment is only needed for a deficit or a record
        record = (dfield is not None and cs.deficit is not None) or increment_dir is not None
        cl.bounded_add[name] = bounded_add_device(pert, mean_1d, inc, lo, hi, cs.window,
                                                  record_applied=record,
                                                  ledger=cl.bounded_add.get(name))
        if dfield is not None and cs.deficit is not None:
            _accumulate(dfield, inc, None, cs.deficit)
        if increment_dir is not None:
            np.save(Path(increment_dir) / f"c{index:02d}_{name}.npy", to_host(inc))
        del inc
    del step


def cascade_loop(h_profile, qt_profile, z_profile, grids, C_h_k, C_qt_k,
                 b_h_k, b_qt_k, aspect_k, h_min, h_max, qt_min, qt_max,
                 min_distance_to_ground, sparsity_factors, class_seeds,
                 n_scale_classes_per_dyad=1, h_perturbation=None, qt_perturbation=None,
                 flux=None, deficit_h=None, deficit_qt=None, deficit_flux=None,
                 inner_windows=None, world_origins=None, world_shapes=None, ledger=None,
                 flux_noise_scale=None, turbulon_shape='mexican_hat', zero_bottom=True,
                 zero_top=True, device='cuda', increment_dir=None, comp_k=None,
                 dtype=np.float32, resident=False, flux_alpha=None):
    """The multi-scale cascade (steam/simulate.py:1566-2049) with every field
    resident on the device.

    Returns (h', qt', flux, deficit_h, deficit_qt, deficit_flux, final_grid,
    ledger) as numpy arrays, or as CUDA tensors with ``resident=True``.
    ``dtype`` selects float32 (the reference's arithmetic) or float64.
    """
    check_device(device, "cascade_loop")
    torch = _lib.require_cuda("cascade_loop")
    tdt = torch_dtype(dtype)
    np_t = np.dtype(dtype).type
    s_x, s_y, s_z = sparsity_factors
    n_classes = len(grids['k'])
    n_zero = int(round(2 * s_z * min_distance_to_ground))
    alpha = FLUX_ALPHA if flux_alpha is None else float(flux_alpha)
    if not isinstance(n_scale_classes_per_dyad, int) or n_scale_classes_per_dyad < 1:
        raise ValueError("n_scale_classes_per_dyad must be a positive integer, "
                         f"got {n_scale_classes_per_dyad}")
    if n_classes > 1:
        ratio = 2.0 ** (1.0 / n_scale_classes_per_dyad)
        if not np.allclose(np.asarray(grids['k'][:-1]) / np.asarray(grids['k'][1:]), ratio):
            raise ValueError("grids['k'] spacing is inconsistent with "
                             f"n_scale_classes_per_dyad={n_scale_classes_per_dyad} "
                             f"(expected adjacent-class ratio {ratio})")
    if comp_k is None:
        k_fin = float(grids['k'][n_classes - 1])
        comp_k = [np.full(int(grids['nz'][i]), np.float32(
            _interpolation_compensation(2.0 * grids['k'][i] / k_fin)))
            for i in range(n_classes)]
    if not isinstance(class_seeds, (list, tuple, np.ndarray)):
        raise TypeError("class_seeds must be a sequence of SeedSequence, one per size class, "
                        f"got {type(class_seeds).__name__}")
    if len(class_seeds) != n_classes:
        raise ValueError(f"class_seeds has {len(class_seeds)} entries for {n_classes} size classes")
    if ledger is None:
        ledger = RunLedger(n_classes)
    elif len(ledger.classes) != n_classes:
        raise ValueError(f"ledger has {len(ledger.classes)} classes for {n_classes} size classes")
    if increment_dir is not None:
        increment_dir = Path(increment_dir)
        increment_dir.mkdir(parents=True, exist_ok=True)
    keys = [class_key(c) for c in class_seeds]
    # The kernel's normalisation and its separable factors are float64 for
    # both storage dtypes; float32 fields are convolved with float64 taps.
    kernel = _turbulon_envelope(1, 1 / (2 * s_x), 1 / (2 * s_y), 1 / (2 * s_z),
                                support_factor=SUPPORT_FACTOR, shape=turbulon_shape,
                                dtype=np.float64)
    c_noise = FLUX_SCALE if flux_noise_scale is None else flux_noise_scale

    def dev(a):
        return None if a is None else to_device(a, dtype=tdt, copy=True)[0]

    hp, qp, F = dev(h_perturbation), dev(qt_perturbation), dev(flux)
    dh, dq, dF = dev(deficit_h), dev(deficit_qt), dev(deficit_flux)
    prev = None
    for i in range(n_classes):
        shape = (int(grids['nx'][i]), int(grids['ny'][i]), int(grids['nz'][i]))
        z_k = grids['z_arrays'][i]
        window = None if inner_windows is None else tuple(inner_windows[i])
        cl = ledger.classes[i]
        if hp is None:
            hp = torch.zeros(shape, dtype=tdt, device='cuda')
            qp = torch.zeros(shape, dtype=tdt, device='cuda')
            F = torch.ones(shape, dtype=tdt, device='cuda')
        else:
            if F is None:
                F = torch.ones(hp.shape, dtype=tdt, device='cuda')
            carried = [hp, qp, F, dh, dq, dF]
            if prev is not None:
                carried = _crop_between(carried, prev, (
                    float(grids['padded_extent_x'][i]), float(grids['padded_extent_y'][i]),
                    float(grids['padded_height'][i]), float(grids['z_min_per_class'][i])))
            if tuple(carried[0].shape) != shape:
                carried = [f if f is None else _utils.zoom_device(f, shape) for f in carried]
            hp, qp, F, dh, dq, dF = carried
        h_mean = np.interp(z_k, z_profile, h_profile).astype(np.float32)
        qt_mean = np.interp(z_k, z_profile, qt_profile).astype(np.float32)
        region = NoiseRegion(
            keys[i],
            (0, 0, 0) if world_origins is None else tuple(int(v) for v in world_origins[i]),
            shape if world_shapes is None else tuple(int(v) for v in world_shapes[i]))
        deficit_i = np.asarray(comp_k[i], dtype=np.float32) - np.float32(1.0)
        has_deficit = bool(np.any(deficit_i))
        if has_deficit:
            if dh is None:
                dh = torch.zeros_like(hp)
                dq = torch.zeros_like(qp)
            if dF is None:
                dF = torch.zeros_like(F)
        cs = ClassSetup(shape=shape, z=z_k, dx=float(grids['dx'][i]),
                        dy=float(grids['dy'][i]), h_mean=h_mean, qt_mean=qt_mean,
                        C_h=C_h_k[i], C_qt=C_qt_k[i], b_h=b_h_k[i], b_qt=b_qt_k[i],
                        aspect=aspect_k[i], bounds=(h_min, h_max, qt_min, qt_max),
                        region=region, plan=_kernel_plan(kernel, shape, np_t),
                        deficit=deficit_i if has_deficit else None, window=window,
                        flux_noise_scale=c_noise, n_per_dyad=n_scale_classes_per_dyad,
                        sparsity=tuple(sparsity_factors), n_zero=n_zero,
                        zero_bottom=zero_bottom, zero_top=zero_top, alpha=alpha)
        run_class(hp, qp, F, dh, dq, dF, cs, cl, increment_dir=increment_dir, index=i)
        prev = (float(grids['padded_extent_x'][i]), float(grids['padded_extent_y'][i]),
                float(grids['padded_height'][i]), float(grids['dx'][i]),
                float(grids['dy'][i]), float(grids['dz'][i]),
                float(grids['z_min_per_class'][i]))
    last = n_classes - 1
    final_grid = {'nx': int(grids['nx'][last]), 'ny': int(grids['ny'][last]),
                  'nz': int(grids['nz'][last]), 'dx': float(grids['dx'][last]),
                  'dy': float(grids['dy'][last]), 'dz': grids['dz_arrays'][last],
                  'z': grids['z_arrays'][last]}
    fields = (hp, qp, F, dh, dq, dF)
    if not resident:
        fields = tuple(None if f is None else to_host(f) for f in fields)
    return (*fields, final_grid, ledger)


def simulate_flux_only(grids, sparsity_factors=(1, 1, 1), seed=None, flux_noise_scale=None,
                       n_scale_classes_per_dyad=1, min_distance_to_ground=0,
                       turbulon_shape='mexican_hat', zero_bottom=False, zero_top=False,
                       dtype=np.float32, resident=False, flux_alpha=None):
    """Flux cascade alone on root grids (steam/simulate.py:2231-2353)."""
    torch = _lib.require_cuda("simulate_flux_only")
    s_x, s_y, s_z = sparsity_factors
    for s, name in zip(sparsity_factors, ('s_x', 's_y', 's_z')):
        if not isinstance(s, int) or s < 1:
            raise ValueError(f"{name} must be a positive integer, got {s}")
    if not isinstance(min_distance_to_ground, int) or min_distance_to_ground < 0:
        raise ValueError("min_distance_to_ground must be a non-negative integer, "
                         f"got {min_distance_to_ground}")
    extents = (np.asarray(grids['padded_extent_x']), np.asarray(grids['padded_extent_y']),
               np.asarray(grids['padded_height']))
    if any(not np.allclose(v, v[0]) for v in extents):
        raise ValueError("simulate_flux_only requires a common physical extent across classes "
                         "(root-simulation grids without refinement padding)")
    c = FLUX_SCALE if flux_noise_scale is None else flux_noise_scale
    if not np.isfinite(c) or c < 0:
        raise ValueError(f"flux_noise_scale must be finite and non-negative, got {c}")
    if not isinstance(n_scale_classes_per_dyad, int) or n_scale_classes_per_dyad < 1:
        raise ValueError("n_scale_classes_per_dyad must be a positive integer, "
                         f"got {n_scale_classes_per_dyad}")
    n_classes = len(grids['k'])
    if n_classes > 1:
        ratio = 2.0 ** (1.0 / n_scale_classes_per_dyad)
        if not np.allclose(np.asarray(grids['k'][:-1]) / np.asarray(grids['k'][1:]), ratio):
            raise ValueError("simulate_flux_only: grids['k'] spacing is inconsistent with "
                             f"n_scale_classes_per_dyad={n_scale_classes_per_dyad} "
                             f"(expected adjacent-class ratio {ratio})")
    alpha = FLUX_ALPHA if flux_alpha is None else float(flux_alpha)
    np_t = np.dtype(dtype).type
    tdt = torch_dtype(dtype)
    seeds = np.random.SeedSequence(seed).spawn(n_classes)
    n_zero = int(round(2 * s_z * min_distance_to_ground))
    kernel = _turbulon_envelope(1, 1 / (2 * s_x), 1 / (2 * s_y), 1 / (2 * s_z),
                                support_factor=SUPPORT_FACTOR, shape=turbulon_shape,
                                dtype=np.float64)
    F = None
    steps = []
    total_clipped = total_points = 0
    for i, k in enumerate(grids['k']):
        shape = (int(grids['nx'][i]), int(grids['ny'][i]), int(grids['nz'][i]))
        if F is None:
            F = torch.ones(shape, dtype=tdt, device='cuda')
        elif tuple(F.shape) != shape:
            F = _utils.zoom_device(F, shape)
        region = NoiseRegion.root(seeds[i], shape)
        plan = _kernel_plan(kernel, shape, np_t)
        step = advance_flux_device(F, region, plan, c, n_scale_classes_per_dyad,
                                   sparsity_factors, n_zero, zero_bottom, zero_top,
                                   alpha=alpha)
        total_clipped += step.diagnostics['n_clipped']
        total_points += step.diagnostics['n_points']
        steps.append({'k': float(k), **step.diagnostics})
        del step
    diagnostics = {
        'flux_noise_scale': float(c), 'n_scale_classes_per_dyad': n_scale_classes_per_dyad,
        'steps': steps, 'n_clipped': total_clipped, 'n_points': total_points,
        'clip_fraction': total_clipped / max(total_points, 1),
        'final_zero_fraction': float((F == 0).sum().item() / F.numel()),
    }
    return (F if resident else to_host(F)), diagnostics


def _f32_ulp(value):
    return float(np.spacing(np.float32(abs(value))))


def simulate(h_profile, qt_profile, nx, ny, dx, dy, outer_scale, spheroscale,
             domain_height, profile_dz, output_path, sparsity_factors=(1, 1, 1),
             n_scale_classes_per_dyad=1, surface_pressure=101325.0, seed=None,
             h_min=315 * 1004, h_max=355 * 1004, qt_min=0.0, qt_max=30 / 1000,
             min_distance_to_ground=1, turbulon_shape='mexican_hat',
             anisotropy='piecewise_isotropic_below_spheroscale', compress=None,
             device='cuda', save_for_refinement=False, hurst_horizontal=None,
             haar_to_mhat=None, bound_buffer_multiple=None, ledger=None,
             stream_to_disk=False, scratch_dir=None, memory_budget=None,
             resumable=False, fresh=False, _force_tiling=None, _crash_hook=None,
             dtype=np.float32, resident=False):
    """Run the STEAM cascade and compose its output (steam/simulate.py:729-1563).

    The NetCDF writer is outside this package: when ``output_path`` is given
    the composed fields are written as a ``.npz`` beside it.  Returns a dict of
    the composed fields (h, qt, flux and, with save_for_refinement, the
    cascade states), the coordinates and the run ledger.
    """
    check_device(device, "simulate")
    torch = _lib.require_cuda("simulate")
    seed_was_none = seed is None
    if seed is None:
        seed = int(np.random.SeedSequence().generate_state(1)[0] >> 1)
    seed_sequence = np.random.SeedSequence(seed)
    for s, name in zip(sparsity_factors, ('s_x', 's_y', 's_z')):
        if not isinstance(s, int) or s < 1:
            raise ValueError(f"{name} must be a positive integer, got {s}")
    if not isinstance(n_scale_classes_per_dyad, int) or n_scale_classes_per_dyad < 1:
        raise ValueError("n_scale_classes_per_dyad must be a positive integer, "
                         f"got {n_scale_classes_per_dyad}")
    if not isinstance(min_distance_to_ground, int) or min_distance_to_ground < 0:
        raise ValueError("min_distance_to_ground must be a non-negative integer, "
                         f"got {min_distance_to_ground}")
    if anisotropy not in VALID_ANISOTROPY:
        raise ValueError(f"anisotropy must be one of {VALID_ANISOTROPY}, got {anisotropy!r}")
    domain_x, domain_y = nx * dx, ny * dy
    h_profile = np.asarray(h_profile, dtype=np.float32)
    qt_profile = np.asarray(qt_profile, dtype=np.float32)
    if np.any(np.isnan(h_profile)):
        raise ValueError('nans present in h_profile')
    if np.any(np.isnan(qt_profile)):
        raise ValueError('nans present in qt_profile')
    if h_profile.ndim != 1 or qt_profile.ndim != 1:
        raise ValueError("h_profile and qt_profile must be 1D arrays")
    if len(h_profile) == 0 or len(h_profile) != len(qt_profile):
        raise ValueError("h_profile and qt_profile must have equal nonzero length, "
                         f"got {len(h_profile)} and {len(qt_profile)}")
    for lo_v, hi_v, prof, name in ((h_min, h_max, h_profile, 'h'),
                                   (qt_min, qt_max, qt_profile, 'qt')):
        pmin, pmax = float(np.min(prof)), float(np.max(prof))
        if lo_v > pmin + _f32_ulp(pmin):
            raise ValueError(f"{name}_min ({lo_v}) must be <= min({name}_profile) ({pmin})")
        if hi_v < pmax - _f32_ulp(pmax):
            raise ValueError(f"{name}_max ({hi_v}) must be >= max({name}_profile) ({pmax})")
    if domain_height <= 0:
        raise ValueError(f"domain_height must be positive, got {domain_height}")
    if outer_scale / dx < 1:
        raise ValueError(f"outer_scale ({outer_scale}) must be >= dx ({dx})")
    if outer_scale <= 2 * dx:
        raise ValueError(f"outer_scale ({outer_scale}) must be greater than 2*dx ({2 * dx}); "
                         "at least two scale classes are required")
    for size, axis in ((domain_x, 'x'), (domain_y, 'y')):
        n_tiles = size / outer_scale
        if n_tiles >= 1 and abs(n_tiles - round(n_tiles)) > 1e-9:
            raise ValueError(f"domain_{axis} ({size}) must be an integer multiple of "
                             f"outer_scale ({outer_scale}) or smaller than it, got ratio={n_tiles}")
    sph = np.asarray(spheroscale, dtype=np.float64)
    if sph.ndim > 0:
        if len(sph) != len(h_profile):
            raise ValueError("spheroscale array must have the same length as profiles, "
                             f"got {len(sph)} vs {len(h_profile)}")
        sph_profile = sph
    else:
        sph_profile = np.full(len(h_profile), float(sph))
    z_profile = np.arange(len(h_profile), dtype=np.float64) * profile_dz
    if float(z_profile[-1]) < domain_height:
        raise ValueError(f"the h/qt profile spans 0 to {float(z_profile[-1]):.1f} m, which does "
                         f"not reach domain_height ({domain_height} m)")
    s_x, s_y, s_z = sparsity_factors
    gap = 2.0 ** (1.0 / n_scale_classes_per_dyad)
    n_classes = int(round(np.log(outer_scale / (2 * dx)) / np.log(gap))) + 1
    if n_classes < 2:
        raise ValueError("Fewer than 2 scale classes would be generated")
    k_values = outer_scale / gap ** np.arange(n_classes)
    sph_mean = float(np.mean(sph_profile))
    k_z_L_mean = float(_k_z(anisotropy, outer_scale, sph_mean))
    if profile_dz >= k_z_L_mean:
        raise ValueError(f"profile_dz ({profile_dz} m) must be less than the vertical outer "
                         f"scale k_z_L ({k_z_L_mean:.1f} m); use a finer profile resolution")
    k_z_L_max = float(np.max(_k_z(anisotropy, outer_scale, sph_profile)))
    if k_z_L_max >= domain_height:
        raise ValueError(f"domain_height ({domain_height} m) is shorter than the vertical scale "
                         f"of the outer-scale turbulons (max k_z,L = {k_z_L_max:.1f} m)")
    grids = _compute_all_grids(k_values, domain_x, domain_y, domain_height,
                               sparsity_factors, sph_profile, z_profile, anisotropy=anisotropy)
    k_z_L_on_profile = _k_z(anisotropy, outer_scale, sph_profile)
    C_h_k = _compute_normalization(h_profile, z_profile, k_z_L_on_profile, k_values,
                                   outer_scale, grids, n_scale_classes_per_dyad,
                                   hurst_horizontal, haar_to_mhat)
    C_qt_k = _compute_normalization(qt_profile, z_profile, k_z_L_on_profile, k_values,
                                    outer_scale, grids, n_scale_classes_per_dyad,
                                    hurst_horizontal, haar_to_mhat)
    aspect_k = [(_k_z(anisotropy, k, np.interp(grids['z_arrays'][i], z_profile, sph_profile))
                 / k).astype(np.float32) for i, k in enumerate(k_values)]
    b_h_k = _bound_buffers(C_h_k, n_scale_classes_per_dyad, hurst_horizontal,
                           bound_buffer_multiple)
    b_qt_k = _bound_buffers(C_qt_k, n_scale_classes_per_dyad, hurst_horizontal,
                            bound_buffer_multiple)
    comp_k = _compensation_profiles(k_values, grids['z_arrays'], sph_profile, z_profile,
                                    anisotropy)
    child_seeds = seed_sequence.spawn(n_classes)
    store = None
    if stream_to_disk or _force_tiling is not None:
        # the reference's out-of-core driver (steam/simulate.py:1240-1412): here
        # the cascade runs resident and its final fields leave through the store
        from .streaming import plan_tiling, streamed_cascade_loop
        if ledger is not None:
            raise ValueError("simulate: a ledger replay does not stream; drop ledger=")
        kshape = _turbulon_envelope(1, 1 / (2 * s_x), 1 / (2 * s_y), 1 / (2 * s_z),
                                    support_factor=SUPPORT_FACTOR, shape=turbulon_shape,
                                    dtype=np.float64).shape
        plan = plan_tiling(grids, kshape, budget_bytes=memory_budget, device=device,
                           force=_force_tiling, save_increments=save_for_refinement)
        if scratch_dir is None:
            scratch_dir = (Path(output_path).parent / f".steam_scratch_{Path(output_path).stem}"
                           if output_path is not None else Path.cwd() / ".steam_scratch")
        (h_m, qt_m, flux_m, dh_m, dq_m, dF_m, final_grid, run_ledger,
         store) = streamed_cascade_loop(
            h_profile, qt_profile, z_profile, grids, C_h_k, C_qt_k, b_h_k, b_qt_k, aspect_k,
            h_min, h_max, qt_min, qt_max, min_distance_to_ground, sparsity_factors,
            child_seeds, plan, scratch_dir, n_scale_classes_per_dyad=n_scale_classes_per_dyad,
            turbulon_shape=turbulon_shape, device=device, comp_k=comp_k, dtype=dtype)
        tdt = torch_dtype(dtype)

        def back(m):
            return None if m is None else to_device(np.ascontiguousarray(m), dtype=tdt)[0]

        h_pert, qt_pert, flux_field = back(h_m), back(qt_m), back(flux_m)
        deficit_h, deficit_qt, deficit_flux = back(dh_m), back(dq_m), back(dF_m)
        del h_m, qt_m, flux_m, dh_m, dq_m, dF_m
        store.destroy()
    else:
        (h_pert, qt_pert, flux_field, deficit_h, deficit_qt, deficit_flux, final_grid,
         run_ledger) = cascade_loop(
            h_profile, qt_profile, z_profile, grids, C_h_k, C_qt_k, b_h_k, b_qt_k, aspect_k,
            h_min, h_max, qt_min, qt_max, min_distance_to_ground, sparsity_factors,
            child_seeds, n_scale_classes_per_dyad=n_scale_classes_per_dyad,
            turbulon_shape=turbulon_shape, device=device, comp_k=comp_k, ledger=ledger,
            dtype=dtype, resident=True)
    z_final = final_grid['z'].astype(np.float32)
    h_mean_final = np.interp(z_final, z_profile, h_profile).astype(np.float32)
    qt_mean_final = np.interp(z_final, z_profile, qt_profile).astype(np.float32)
    h_3d, proj_h = compose_output_device(h_pert, deficit_h, h_mean_final, h_min, h_max,
                                         ledger=run_ledger.projection.get('h'))
    qt_3d, proj_qt = compose_output_device(qt_pert, deficit_qt, qt_mean_final, qt_min, qt_max,
                                           ledger=run_ledger.projection.get('qt'))
    flux_3d, run_ledger.flux_output = compose_flux_output_device(
        flux_field, deficit_flux, ledger=run_ledger.flux_output)
    if proj_h is not None:
        run_ledger.projection['h'] = proj_h
    if proj_qt is not None:
        run_ledger.projection['qt'] = proj_qt
    nxf, nyf = int(h_pert.shape[0]), int(h_pert.shape[1])
    result = {
        'h': h_3d, 'qt': qt_3d, 'flux': flux_3d,
        'x': np.arange(nxf, dtype=np.float32) * (domain_x / nxf),
        'y': np.arange(nyf, dtype=np.float32) * (domain_y / nyf),
        'z': z_final, 'k_values': k_values, 'seed': seed, 'ledger': run_ledger,
        'grids': grids,
    }
    if save_for_refinement:
        result.update({'h_perturbation': h_pert, 'qt_perturbation': qt_pert,
                       'flux_state': flux_field})
    if not resident:
        for key in ('h', 'qt', 'flux', 'h_perturbation', 'qt_perturbation', 'flux_state'):
            if key in result and is_tensor(result[key]):
                result[key] = to_host(result[key])
    if output_path is not None and not resident:
        path = Path(output_path)
        np.savez(path.with_suffix('.npz'), **{k: v for k, v in result.items()
                                             if isinstance(v, np.ndarray)})
    return result


# ---------------------------------------------------------------------------
# One class as a served unit: setup once, step many times
# ---------------------------------------------------------------------------

def make_class_setup(grids, i, *, h_profile, qt_profile, z_profile, C_h, C_qt, b_h, b_qt,
                     aspect, bounds, key, sparsity_factors=(1, 1, 1),
                     min_distance_to_ground=1, flux_noise_scale=None,
                     n_scale_classes_per_dyad=1, flux_alpha=None,
                     turbulon_shape='mexican_hat', comp=None, window=None, origin=None,
                     world_shape=None, zero_bottom=True, zero_top=True, dtype=np.float32):
    """The ClassSetup of class ``i`` of ``grids`` (the per-class locals of
    cascade_loop), for stepping one class outside the loop."""
    s_x, s_y, s_z = sparsity_factors
    shape = (int(grids['nx'][i]), int(grids['ny'][i]), int(grids['nz'][i]))
    z_k = grids['z_arrays'][i]
    np_t = np.dtype(dtype).type
    kernel = _turbulon_envelope(1, 1 / (2 * s_x), 1 / (2 * s_y), 1 / (2 * s_z),
                                support_factor=SUPPORT_FACTOR, shape=turbulon_shape,
                                dtype=np.float64)
    deficit = None
    if comp is not None:
        d = np.asarray(comp, dtype=np.float32) - np.float32(1.0)
        deficit = d if np.any(d) else None
    region = NoiseRegion(tuple(int(k) for k in key),
                         (0, 0, 0) if origin is None else tuple(int(v) for v in origin),
                         shape if world_shape is None else tuple(int(v) for v in world_shape))
    return ClassSetup(
        shape=shape, z=z_k, dx=float(grids['dx'][i]), dy=float(grids['dy'][i]),
        h_mean=np.interp(z_k, z_profile, h_profile).astype(np.float32),
        qt_mean=np.interp(z_k, z_profile, qt_profile).astype(np.float32),
        C_h=np.asarray(C_h, np.float32), C_qt=np.asarray(C_qt, np.float32),
        b_h=np.asarray(b_h, np.float32), b_qt=np.asarray(b_qt, np.float32),
        aspect=np.asarray(aspect, np.float32), bounds=tuple(float(b) for b in bounds),
        region=region, plan=_kernel_plan(kernel, shape, np_t), deficit=deficit,
        window=window,
        flux_noise_scale=FLUX_SCALE if flux_noise_scale is None else float(flux_noise_scale),
        n_per_dyad=int(n_scale_classes_per_dyad), sparsity=tuple(sparsity_factors),
        n_zero=int(round(2 * s_z * min_distance_to_ground)), zero_bottom=zero_bottom,
        zero_top=zero_top, alpha=FLUX_ALPHA if flux_alpha is None else float(flux_alpha))


def field_step(h_perturbation, qt_perturbation, flux, setup, surface_pressure=101325.0,
               diagnostics=('qc', 'qi'), ledger=None, out=None, wait=True):
    """One size class plus the thermodynamic map to condensate.

    Advances the flux, adds the h and qt increments (pattern, second
    convolution, bounded add), composes h = h' + <h>, qt = qt' + <qt> clamped
    to the bounds, and recovers the requested diagnostics
    (steam/thermodynamics.py:25-123).  numpy arrays are updated in place and
    host diagnostics returned; CUDA tensors stay on the device.  Returns
    (diagnostics dict, ClassLedger).  With numpy arrays, ``out`` (a dict of
    host arrays) receives the diagnostics; page-locked arrays let the
    pipelined transfers run at full PCIe bandwidth.

    ``wait=False`` (host arrays only) returns a ``PendingHostStep`` before the
    downloads finish; its ``result()`` gives (diagnostics, ClassLedger).  A
    following call on the same arrays is ordered after those downloads and
    its uploads overlap them, so a loop of steps keeps both directions of the
    link busy.  Read the arrays only after ``result()``.
    """
    from .ledger import ClassLedger
    from .thermodynamics import recover_diagnostics_device
    torch = _lib.require_cuda("field_step")
    if (not is_tensor(h_perturbation) and ledger is None and setup.deficit is None
            and np.ndim(surface_pressure) == 0):
        # host arrays: the resident step with pipelined transfers
        from .resident import resident_for
        np_t = np.asarray(h_perturbation).dtype
        rc = resident_for(setup, torch.float64 if np_t == np.float64 else torch.float32)
        pending = rc.host_step(h_perturbation, qt_perturbation, flux,
                               diagnostics=diagnostics, out=out,
                               surface_pressure=surface_pressure, wait=False)
        return pending.result() if wait else pending
    hp, h_host = to_device(h_perturbation)
    qp, q_host = to_device(qt_perturbation, dtype=hp.dtype)
    F, f_host = to_device(flux, dtype=hp.dtype)
    cl = ClassLedger() if ledger is None else ledger
    diag = {}
    resident = ledger is None and setup.deficit is None and np.ndim(surface_pressure) == 0
    if resident:
        from .resident import resident_for
        rc = resident_for(setup, hp.dtype)
        out = {k: torch.empty_like(hp) for k in ("T", "qv", "qc", "qi", "p")} \
            if diagnostics else None
        rc.step(hp, qp, F, diagnostics=out, surface_pressure=surface_pressure)
        if diagnostics:
            diag = {k: out[k] for k in diagnostics}
        del out
    else:
        run_class(hp, qp, F, None, None, None, setup, cl)
    if diagnostics and not resident:
        h_min, h_max, qt_min, qt_max = setup.bounds
        np_t = np.float64 if hp.dtype == torch.float64 else np.float32
        bounds = [float(np_t(h_min)), float(np_t(h_max)), float(np_t(qt_min)),
                  float(np_t(qt_max))]
        out = recover_diagnostics_device(hp, qp, setup.z, surface_pressure,
                                         h_mean=setup.h_mean, qt_mean=setup.qt_mean,
                                         bounds=bounds)
        diag = {k: out[k] for k in diagnostics}
        del out
    if h_host is not None:
        to_host(hp, out=h_perturbation)
        to_host(qp, out=qt_perturbation)
        to_host(F, out=flux)
        diag = {k: to_host(v) for k, v in diag.items()}
    if resident:
        rc.class_ledger(cl)
    return diag, cl
