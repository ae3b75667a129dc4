"""steam_level_sums_noalloc against steam_level_sums, through the C ABI.

The allocation-free entry point keeps its scratch in one static device array
that every call reuses; two calls in a row on different fields must each match
the workspace entry point.  Collected last so that it also runs after every
other GPU test has used the library.
"""

import ctypes

import numpy as np
import pytest

from steam_b200 import _lib

pytestmark = pytest.mark.gpu

# per-level double sums: the two entry points may add the block partials in a
# different order (the static scratch caps the block count); counts are exact
RTOL = 1e-12


def _workspace_sums(lib, torch, f, window):
    nx, ny, nz = f.shape
    ws_bytes = lib.steam_level_sums_workspace_bytes(nz)
    ws = torch.empty(max(1, ws_bytes), dtype=torch.uint8, device="cuda")
    out = _lib.dout(4 * nz)
    _lib.check(lib.steam_level_sums(_lib.dtype_code(f), nx, ny, nz, _lib.ptr(f), window,
                                    out, _lib.ptr(ws), ws_bytes, _lib.stream()))
    return np.ctypeslib.as_array(out)[: 4 * nz].reshape(nz, 4).copy()


def _noalloc_sums(lib, f, window):
    nx, ny, nz = f.shape
    out = _lib.dout(4 * nz)
    _lib.check(lib.steam_level_sums_noalloc(_lib.dtype_code(f), nx, ny, nz, _lib.ptr(f),
                                            window, out, _lib.stream()))
    return np.ctypeslib.as_array(out)[: 4 * nz].reshape(nz, 4).copy()


def _field(torch, shape, dtype, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    f = torch.randn(shape, generator=g, device="cuda", dtype=dtype)
    f[f.abs() < 0.3] = 0.0  # exact zeros for the nonzero count
    return f


def _assert_same(got, want):
    np.testing.assert_allclose(got[:, 0], want[:, 0], rtol=RTOL,
                               atol=RTOL * np.abs(want[:, 1]).max())
    np.testing.assert_allclose(got[:, 1], want[:, 1], rtol=RTOL)
    np.testing.assert_array_equal(got[:, 2:], want[:, 2:])


@pytest.mark.parametrize("dtype_name", ["float32", "float64"])
@pytest.mark.parametrize("shape,win", [
    ((64, 48, 256), None),            # one level per thread, grid not capped
    ((40, 33, 96), (3, 31, 5, 30)),   # windowed means
    ((20, 16, 1000), None),           # several levels per thread, grid capped
    ((4, 4, 1024), None),             # the maximum nz: tightest grid cap, every slot used
])
def test_noalloc_matches_workspace_entry_twice(dtype_name, shape, win):
    torch = _lib.require_cuda("test")
    lib = _lib.load()
    dtype = getattr(torch, dtype_name)
    window = None
    if win is not None:
        window = ctypes.pointer(_lib.Window(*win))
    for call, seed in enumerate((11, 12)):
        f = _field(torch, shape, dtype, seed)
        want = _workspace_sums(lib, torch, f, window)
        got = _noalloc_sums(lib, f, window)
        assert np.all(got[:, 1] > 0), f"call {call}: empty level sums"
        _assert_same(got, want)


def test_noalloc_rejects_too_many_levels():
    torch = _lib.require_cuda("test")
    lib = _lib.load()
    f = torch.zeros((2, 2, 1025), dtype=torch.float32, device="cuda")
    out = _lib.dout(4 * 1025)
    rc = lib.steam_level_sums_noalloc(_lib.STEAM_F32, 2, 2, 1025, _lib.ptr(f), None, out,
                                      _lib.stream())
    assert rc == 4
    assert b"1024" in lib.steam_last_error()
    assert lib.steam_level_sums_noalloc_scratch_bytes() == 4 << 20


@pytest.mark.parametrize("shape", [(0, 5, 8), (5, 0, 8), (3, 3, 0)])
def test_noalloc_empty_extents_match_workspace_entry(shape):
    """An empty column set gives zero sums and the window's cell count per
    level; an empty z extent writes nothing.  Both entry points agree."""
    torch = _lib.require_cuda("test")
    lib = _lib.load()
    f = torch.zeros(shape, dtype=torch.float32, device="cuda")
    nz = shape[2]
    want = _workspace_sums(lib, torch, f, None)
    got = _noalloc_sums(lib, f, None)
    np.testing.assert_array_equal(got, want)
    if nz:
        np.testing.assert_array_equal(got[:, :3], 0.0)
