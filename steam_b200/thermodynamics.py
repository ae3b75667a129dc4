"""Thermodynamic recovery of T, qv, qc, qi, p from h and qt
(steam/thermodynamics.py:25-123).

One device kernel marches every column upward: dry temperature, Bolton (1980)
saturation, five Newton steps on cp T + Lv qvs(T, p) + g z = h for saturated
cells, the linear ice/liquid partition between 235.15 K and 273.15 K, and a
float64 hypsometric pressure accumulator.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from ._device import check_device, is_tensor, to_device, to_host


def recover_diagnostics_device(h_t, qt_t, z_values, surface_pressure, out=None,
                               h_mean=None, qt_mean=None, bounds=None):
    """Device form: returns a dict of CUDA tensors (or fills ``out``).  With
    mean profiles and bounds, h_t/qt_t are perturbations and the composition
    h = clamp(h' + mean) is fused in front of the column solve."""
    torch = _lib.require_cuda("recover_diagnostics")
    lib = _lib.load()
    nx, ny, nz = (int(n) for n in h_t.shape)
    if qt_t.shape != h_t.shape or qt_t.dtype != h_t.dtype:
        raise ValueError("recover_diagnostics: h and qt must share shape and dtype")
    z = np.asarray(z_values, dtype=np.float64)
    if z.shape != (nz,):
        raise ValueError(f"z_values has shape {z.shape}, expected ({nz},)")
    if out is None:
        out = {k: torch.empty_like(h_t) for k in ("T", "qv", "qc", "qi", "p")}
    ps = np.asarray(surface_pressure, dtype=np.float64)
    ps_dev = None
    scalar_ps = 0.0
    if ps.ndim == 0:
        scalar_ps = float(ps)
    else:
        if ps.shape != (nx, ny):
            raise ValueError(f"surface_pressure field has shape {ps.shape}, expected ({nx}, {ny})")
        ps_dev = torch.as_tensor(np.ascontiguousarray(ps), device='cuda')
    _lib.check(lib.steam_thermo(
        _lib.dtype_code(h_t), nx, ny, nz, _lib.ptr(h_t), _lib.ptr(qt_t), _lib.dvec(z),
        _lib.dvec(h_mean) if h_mean is not None else None,
        _lib.dvec(qt_mean) if qt_mean is not None else None,
        _lib.dvec(bounds) if bounds is not None else None,
        scalar_ps, _lib.ptr(ps_dev) if ps_dev is not None else None,
        _lib.ptr(out["T"]), _lib.ptr(out["qv"]), _lib.ptr(out["qc"]), _lib.ptr(out["qi"]),
        _lib.ptr(out["p"]), _lib.stream()))
    return out


def recover_diagnostics(h, qt, z_values, surface_pressure, device='cuda'):
    """Recover T, qv, qc, qi, p (steam/thermodynamics.py:25-123).  numpy in ->
    numpy out; CUDA tensors in -> CUDA tensors out."""
    check_device(device, "recover_diagnostics")
    h_t, h_host = to_device(h)
    qt_t, _ = to_device(qt, dtype=h_t.dtype)
    out = recover_diagnostics_device(h_t, qt_t, z_values, surface_pressure)
    if h_host is None:
        return out
    return {k: to_host(v).astype(h_host.dtype, copy=False) for k, v in out.items()}
