"""Convolution and regrid entry points (steam/utils.py:222-534).

``convolve_fft_xy_oa_z`` keeps the reference's semantics -- x and y circular
over the full array period, z linear with zero padding, the kernel centred at
(k-1)//2 after being folded onto a narrower field -- but not its method.  A
turbulon kernel that is a sum of a few separable terms (the Mexican hat)
runs as three coalesced 1D stencil passes on the device (z, then y, then x)
over a Tucker factorisation of the kernel taken on the host in float64.  A
kernel without such a form (the Morlet turbulon) runs, for float32 fields,
as an overlap-save FFT convolution on 32^3 cubes with its spectrum built on
the device, and for float64 fields (or kernels longer than 25 taps) as a
direct sum over its taps.  Neither folds the kernel: a kernel longer than
the period is applied with the centre the fold implies (``effective_centre``).
"""

from __future__ import annotations

import ctypes
import hashlib
from dataclasses import dataclass
from math import gcd

import numpy as np

from . import _lib
from ._device import check_device, is_tensor, to_device, to_host

MAX_Z_FILTERS = 8
MAX_PAIRS = 16
MAX_X_FILTERS = 4
MAX_TAPS = 1536

# Relative Frobenius error allowed when a kernel is factored: well under the
# float32 rounding of the kernel itself for float32 fields, and at float64
# roundoff for float64 fields.
FACTOR_TOL = {np.float32: 1e-6, np.float64: 1e-12}


def effective_centre(k: int, n: int) -> int:
    """Centre tap of a kernel axis convolved circularly over period n.

    convolve_fft_xy_oa_z folds a kernel wider than the field (rolling the fold
    by n//2) and then centres it at (n-1)//2; as a circular convolution with
    the UNFOLDED taps that is a centre of k//2 - (1 if n is even else 0).  A
    kernel that fits keeps (k-1)//2.
    """
    if k <= n:
        return (k - 1) // 2
    return k // 2 - (1 if n % 2 == 0 else 0)


def _mode_basis(unfolded, tol_abs):
    U, s, _ = np.linalg.svd(unfolded, full_matrices=False)
    tail = np.sqrt(np.cumsum((s ** 2)[::-1]))[::-1]  # tail[r] = ||s[r:]||
    r = int(np.count_nonzero(tail > tol_abs))
    return U[:, :max(r, 1)]


FFT_MAX_TAPS = 25  # longest kernel axis of the 32^3-cube FFT convolution


@dataclass
class ConvPlan:
    """A kernel prepared for one field period (nx, ny) and dtype.

    ``kind``: 'separable' (Tucker factors), 'fft' (float32 fields, kernel
    spectrum on the device) or 'direct' (sum over the taps)."""
    kind: str
    shape: tuple
    spec: object = None
    z_taps: object = None
    y_taps: object = None
    x_taps: object = None
    kernel: object = None          # the unfolded kernel (host float64)
    centre: tuple = (0, 0)         # (cx, cy) for the unfolded kernel, fft / direct
    device_data: dict = None       # per (device, dtype): kernel / spectrum tensors
    error: float = 0.0             # relative Frobenius error of the factorisation


def factor_kernel(kernel, tol):
    """Tucker factorisation K ~ sum core[a,b,c] X_a(x) Y_b(y) Z_c(z).

    Returns (Px, Py, Pz, core, rel_err) with orthonormal factor columns.
    """
    K = np.asarray(kernel, dtype=np.float64)
    kx, ky, kz = K.shape
    norm = float(np.linalg.norm(K))
    if norm == 0.0:
        return (np.zeros((kx, 1)), np.zeros((ky, 1)), np.zeros((kz, 1)),
                np.zeros((1, 1, 1)), 0.0)
    tol_abs = tol * norm / np.sqrt(3.0)
    Px = _mode_basis(K.reshape(kx, -1), tol_abs)
    Py = _mode_basis(K.transpose(1, 0, 2).reshape(ky, -1), tol_abs)
    Pz = _mode_basis(K.transpose(2, 0, 1).reshape(kz, -1), tol_abs)
    core = np.einsum('ijk,ia,jb,kc->abc', K, Px, Py, Pz, optimize=True)
    approx = np.einsum('abc,ia,jb,kc->ijk', core, Px, Py, Pz, optimize=True)
    err = float(np.linalg.norm(K - approx)) / norm
    return Px, Py, Pz, core, err


def _sparse_core_rotation(core):
    """Rotations Ry, Rz of the y and z factor bases that make the core's
    (y 1, z 1) slice vanish, or None.

    With G_a[b, c] = core[a, b, c], the slice after rotating by unit vectors y
    (y column 1) and z (z column 1) is y^T G_a z.  A z for which G_0 z and
    G_1 z are parallel (a zero of the quadratic form det[G_0 z, G_1 z]) and a
    y orthogonal to both make it zero for every a.  The turbulon kernels,
    sums of separable terms g(x) g(y) g(z) (3 - x^2 - y^2 - z^2), have one:
    their y and z filter pairs then drop from 4 to 3.  Orthogonal rotations
    leave the factorisation's conditioning unchanged."""
    G = [core[a] for a in range(core.shape[0])]
    if len(G) == 1:
        z = np.array([0.0, 1.0])
    else:
        M = np.empty((2, 2))
        for i in range(2):
            for j in range(2):
                u, v = G[0][:, i], G[1][:, j]
                M[i, j] = u[0] * v[1] - u[1] * v[0]
        w, V = np.linalg.eigh(0.5 * (M + M.T))
        scale = max(float(np.max(np.abs(w))), 1e-300)
        if float(np.min(np.abs(w))) <= 1e-12 * scale:
            z = V[:, int(np.argmin(np.abs(w)))]
        elif w[0] * w[1] < 0:
            z = np.sqrt(abs(w[1])) * V[:, 0] + np.sqrt(abs(w[0])) * V[:, 1]
        else:
            return None
    z = z / np.linalg.norm(z)
    g = max((Ga @ z for Ga in G), key=np.linalg.norm)
    if np.linalg.norm(g) == 0.0:
        return None
    y = np.array([-g[1], g[0]]) / np.linalg.norm(g)
    Ry = np.column_stack([[y[1], -y[0]], y])
    Rz = np.column_stack([[z[1], -z[0]], z])
    rot = np.einsum('abc,bB,cC->aBC', core, Ry, Rz)
    if np.max(np.abs(rot[:, 1, 1])) > 1e-13 * max(float(np.max(np.abs(core))), 1e-300):
        return None
    return Ry, Rz


def plan_from_factors(Px, Py, Pz, core, kshape, field_shape, err=0.0):
    """Separable plan from explicit factors (x: Px[:, a], ...), or None when
    the factor counts exceed the kernels' limits."""
    kx, ky, kz = kshape
    nx, ny = int(field_shape[0]), int(field_shape[1])
    rx, ry, rz = Px.shape[1], Py.shape[1], Pz.shape[1]
    npairs = ry * rz
    taps = rz * kz + ry * ky + rx * kx
    if rz > MAX_Z_FILTERS or rx > MAX_X_FILTERS or npairs > MAX_PAIRS or taps > MAX_TAPS:
        return None
    # A filter that is even about its centre to within roundoff is made
    # exactly even (a change of ~1e-16 relative), so the kernels can fold
    # its symmetric taps in pairs.
    def even(P):
        P = np.array(P, dtype=np.float64, copy=True)
        for j in range(P.shape[1]):
            v = P[:, j]
            e = 0.5 * (v + v[::-1])
            if np.max(np.abs(v - e)) <= 1e-13 * max(np.max(np.abs(v)), 1e-300):
                P[:, j] = e
        return P

    pairs = [(c, b) for c in range(rz) for b in range(ry)]
    if ry == 2 and rz == 2:
        rot = _sparse_core_rotation(core)
        if rot is not None:
            Ry, Rz = rot
            Py, Pz = Py @ Ry, Pz @ Rz
            core = np.einsum('abc,bB,cC->aBC', core, Ry, Rz)
            core[:, 1, 1] = 0.0
            pairs = [(0, 0), (0, 1), (1, 0)]
    npairs = len(pairs)
    Px, Py, Pz = even(Px), even(Py), even(Pz)
    spec = _lib.SepConv()
    spec.kz, spec.ky, spec.kx = kz, ky, kx
    spec.cz = (kz - 1) // 2
    spec.cy = effective_centre(ky, ny)
    spec.cx = effective_centre(kx, nx)
    spec.n_z, spec.n_y, spec.n_x, spec.n_pairs = rz, ry, rx, npairs
    for q, (c, b) in enumerate(pairs):
        spec.pair_z[q] = c
        spec.pair_y[q] = b
        for a in range(rx):
            spec.mix[a * npairs + q] = float(core[a, b, c])
    return ConvPlan(
        kind='separable', shape=(kx, ky, kz), spec=spec,
        z_taps=_lib.dvec(Pz.T.ravel()), y_taps=_lib.dvec(Py.T.ravel()),
        x_taps=_lib.dvec(Px.T.ravel()), error=err)


def _fused_separable(plan):
    """Whether the library runs a separable plan as its fused single-pass
    kernel: a cubic 13 or 25-tap support, at most 2 z, 2 y and 2 x filters and
    4 (z, y) filter pairs drawn from the first two of each."""
    sp = plan.spec
    if not (sp.kx == sp.ky == sp.kz and sp.kx in (13, 25)):
        return False
    if sp.n_z > 2 or sp.n_y > 2 or sp.n_x > 2 or sp.n_pairs > 4:
        return False
    return all(sp.pair_z[q] < 2 and sp.pair_y[q] < 2 for q in range(sp.n_pairs))


_PLAN_CACHE: dict = {}


def plan_convolution(kernel, field_shape, dtype=np.float32, tol=None):
    """Prepare ``kernel`` for fields of ``field_shape`` (cached)."""
    kernel = np.asarray(kernel)
    if kernel.ndim != 3:
        raise ValueError(f"kernel must be 3D, got shape {kernel.shape}")
    dtype = np.dtype(dtype).type
    tol = FACTOR_TOL[dtype] if tol is None else float(tol)
    nx, ny = int(field_shape[0]), int(field_shape[1])
    key = (hashlib.sha1(np.ascontiguousarray(kernel, dtype=np.float64).tobytes()).hexdigest(),
           kernel.shape, nx, ny, dtype, tol)
    plan = _PLAN_CACHE.get(key)
    if plan is not None:
        return plan
    Px, Py, Pz, core, err = factor_kernel(kernel, tol)
    sep = None
    if err <= tol:
        sep = plan_from_factors(Px, Py, Pz, core, kernel.shape, (nx, ny), err)
    k64 = np.ascontiguousarray(kernel, dtype=np.float64)
    fft_ok = dtype == np.float32 and max(k64.shape) <= FFT_MAX_TAPS
    # the fused separable kernel is the fastest form; a separable plan beyond
    # it runs as three passes through HBM with one intermediate field per z
    # filter and per x filter, which the FFT convolution beats where it
    # applies (the rank-(3, 3, 3) Morlet at 512x512x256: 1.20 against 1.60 ms)
    if sep is not None and (_fused_separable(sep) or not fft_ok):
        plan = sep
        plan.kernel = k64
    else:
        plan = ConvPlan(kind='fft' if fft_ok else 'direct', shape=k64.shape, kernel=k64,
                        centre=(effective_centre(k64.shape[0], nx),
                                effective_centre(k64.shape[1], ny)),
                        device_data={}, error=0.0)
    if len(_PLAN_CACHE) > 256:
        _PLAN_CACHE.clear()
    _PLAN_CACHE[key] = plan
    return plan


def prepare_plan(plan, device, dtype):
    """The plan's kernel (direct) or spectrum (fft) on ``device``, built once
    per (device, dtype) on the current stream; call it before capturing a
    graph that runs the plan.  Returns the tensors the launches read."""
    import torch
    if plan.kind == 'separable':
        return None
    key = (torch.device(device), dtype)
    data = plan.device_data.get(key)
    if data is not None:
        return data
    lib = _lib.load()
    k64 = torch.as_tensor(plan.kernel, device=device).contiguous()
    if plan.kind == 'fft':
        spec = torch.empty(lib.steam_conv_fft_spectrum_bytes(), dtype=torch.uint8, device=device)
        kx, ky, kz = plan.shape
        _lib.check(lib.steam_conv_fft_spectrum(_lib.ptr(k64), kx, ky, kz, _lib.ptr(spec),
                                               _lib.stream()))
        data = (spec, k64)  # the float64 kernel stays alive while the build may run
    else:
        data = (k64.to(dtype).contiguous(),)
    plan.device_data[key] = data
    return data


def _device_data(plan, field_t):
    return prepare_plan(plan, field_t.device, field_t.dtype)


def plan_workspace_bytes(plan, code, shape):
    """Workspace of one launch of ``plan`` on a field of ``shape``."""
    lib = _lib.load()
    nx, ny, nz = (int(n) for n in shape)
    if plan.kind == 'separable':
        return lib.steam_conv_workspace_bytes(code, nx, ny, nz, ctypes.byref(plan.spec))
    if plan.kind == 'fft':
        return lib.steam_conv_fft_workspace_bytes(nx, ny, nz)
    return lib.steam_conv_direct_workspace_bytes(nx, ny, nz)


def run_plan_async(plan, field_t, out_t, pre_dev=None, epilogue=_lib.STEAM_EPI_STORE,
                   window=None, sums_dev=None, workspace=None, stream=None):
    """Enqueue a planned convolution with its scalars on the device:
    ``pre_dev`` a [2][nz] device tensor (or pointer) of the field's dtype,
    ``sums_dev`` a device pointer to 2 doubles for the flux epilogue."""
    lib = _lib.load()
    nx, ny, nz = (int(n) for n in field_t.shape)
    code = _lib.dtype_code(field_t)
    stream = _lib.stream() if stream is None else stream
    if workspace is None:
        workspace = _lib.WORKSPACE.get(plan_workspace_bytes(plan, code, field_t.shape))
    wsp, wsn = _lib.ptr(workspace), workspace.numel()
    pre = _lib.ptr(pre_dev) if hasattr(pre_dev, 'data_ptr') else pre_dev
    win = _lib.window_arg(window)
    if plan.kind == 'separable':
        _lib.check(lib.steam_conv_separable_async(
            code, nx, ny, nz, ctypes.byref(plan.spec), plan.z_taps, plan.y_taps, plan.x_taps,
            _lib.ptr(field_t), pre, _lib.ptr(out_t), epilogue, win, sums_dev, wsp, wsn, stream))
        return
    data = _device_data(plan, field_t)
    kx, ky, kz = plan.shape
    cx, cy = plan.centre
    if plan.kind == 'fft':
        _lib.check(lib.steam_conv_fft_async(
            nx, ny, nz, kx, ky, kz, cx, cy, _lib.ptr(data[0]), _lib.ptr(field_t), pre,
            _lib.ptr(out_t), epilogue, win, sums_dev, wsp, wsn, stream))
    else:
        _lib.check(lib.steam_conv_direct_async(
            code, nx, ny, nz, _lib.ptr(data[0]), kx, ky, kz, cx, cy, _lib.ptr(field_t), pre,
            _lib.ptr(out_t), epilogue, win, sums_dev, wsp, wsn, stream))


def run_plan(plan, field_t, out_t, pre_div=None, pre_mul=None,
             epilogue=_lib.STEAM_EPI_STORE, window=None):
    """Launch a planned convolution on device tensors; returns the epilogue
    sums (flux epilogue: sum F over the window, cells, clip count) or None."""
    lib = _lib.load()
    nx, ny, nz = (int(n) for n in field_t.shape)
    code = _lib.dtype_code(field_t)
    ws = _lib.WORKSPACE.get(plan_workspace_bytes(plan, code, field_t.shape))
    sums = _lib.dout(3)
    pd = _lib.dvec(pre_div) if pre_div is not None else None
    pm = _lib.dvec(pre_mul) if pre_mul is not None else None
    win = _lib.window_arg(window)
    if plan.kind == 'separable':
        _lib.check(lib.steam_conv_separable(
            code, nx, ny, nz, ctypes.byref(plan.spec), plan.z_taps, plan.y_taps, plan.x_taps,
            _lib.ptr(field_t), pd, pm, _lib.ptr(out_t), epilogue, win, sums, _lib.ptr(ws),
            ws.numel(), _lib.stream()))
    else:
        data = _device_data(plan, field_t)
        kx, ky, kz = plan.shape
        cx, cy = plan.centre
        if plan.kind == 'fft':
            _lib.check(lib.steam_conv_fft(
                nx, ny, nz, kx, ky, kz, cx, cy, _lib.ptr(data[0]), _lib.ptr(field_t), pd, pm,
                _lib.ptr(out_t), epilogue, win, sums, _lib.ptr(ws), ws.numel(), _lib.stream()))
        else:
            _lib.check(lib.steam_conv_direct(
                code, nx, ny, nz, _lib.ptr(data[0]), kx, ky, kz, cx, cy, _lib.ptr(field_t), pd,
                pm, _lib.ptr(out_t), epilogue, win, sums, _lib.ptr(ws), ws.numel(),
                _lib.stream()))
    if epilogue == _lib.STEAM_EPI_FLUX:
        return (sums[0], sums[1], sums[2])
    return None


def convolve_device(field_t, kernel, out=None, tol=None):
    """Convolve a CUDA tensor; returns a new (or the given) CUDA tensor."""
    import torch
    if field_t.ndim != 3:
        raise ValueError(f"field must be 3D, got shape {tuple(field_t.shape)}")
    np_dtype = np.float64 if field_t.dtype == torch.float64 else np.float32
    plan = plan_convolution(kernel, field_t.shape, np_dtype, tol)
    if out is None:
        out = torch.empty_like(field_t)
    if field_t.numel() == 0:
        return out
    run_plan(plan, field_t, out)
    return out


def convolve_fft_xy_oa_z(field, kernel, device='cuda'):
    """Convolution with circular x/y and linear zero-padded z
    (steam/utils.py:293-427).  Numpy in -> numpy out (transfers inside the
    call, as the reference's device='cuda' path does); a CUDA tensor in -> a
    CUDA tensor out."""
    check_device(device, "convolve_fft_xy_oa_z")
    t, host = to_device(field)
    out = convolve_device(t, np.asarray(kernel))
    if host is None:
        return out
    return to_host(out).astype(host.dtype, copy=False)


# ---------------------------------------------------------------------------
# Regrid (steam/utils.py:435-534)
# ---------------------------------------------------------------------------

def wrap_pad_factor(source_shape, target_shape, periodic=(True, True, False)):
    """Working-array growth the reference's wrapped pad would need
    (steam/utils.py:537-564).  The device regrid wraps natively, so this is
    informational only."""
    padded = 1
    target = 1
    for n_in, n_out, per in zip(source_shape, target_shape, periodic):
        target *= n_out
        if not per or n_out < n_in:
            padded *= n_out
            continue
        padded *= n_out + 2 * (n_out // gcd(n_in, n_out))
    return padded / target if target else 1.0


def zoom_device(field_t, target_shape, periodic=(True, True, False)):
    import torch
    nx, ny, nz = (int(n) for n in field_t.shape)
    mx, my, mz = (int(n) for n in target_shape)
    if periodic[2]:
        raise NotImplementedError("z never wraps in the cascade regrid")
    for axis, (n_in, n_out, per) in enumerate(zip((nx, ny), (mx, my), periodic[:2])):
        if per and n_out < n_in:
            raise NotImplementedError(
                f"Periodic resampling downsamples on axis {axis} ({n_in} -> {n_out}); "
                f"the cascade's hops only go finer.")
    out = torch.empty((mx, my, mz), dtype=field_t.dtype, device=field_t.device)
    lib = _lib.load()
    _lib.check(lib.steam_regrid(_lib.dtype_code(field_t), _lib.ptr(field_t), nx, ny, nz,
                                _lib.ptr(out), mx, my, mz, int(bool(periodic[0])),
                                int(bool(periodic[1])), _lib.stream()))
    return out


def zoom_trilinear(field, target_shape, periodic=(True, True, False)):
    """Cell-consistent trilinear resample, x/y periodic (steam/utils.py:507-534)."""
    _lib.require_cuda("zoom_trilinear")
    t, host = to_device(field)
    out = zoom_device(t, target_shape, periodic)
    if host is None:
        return out
    return to_host(out).astype(np.float32, copy=False)
