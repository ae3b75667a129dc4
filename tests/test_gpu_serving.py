"""World-coordinate tile serving: every tile equals the same cells of the
whole-world field, alone and when served in a mix of concurrent requests."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _world(dtype=np.float32):
    from steam_b200.serving import TileWorld
    return TileWorld((72, 64, 48), seed=7, dtype=dtype)


def _crop(Fw, origin, n):
    nx, ny, _ = Fw.shape
    x0, y0, z0 = origin
    xs = np.arange(x0, x0 + n) % nx
    ys = np.arange(y0, y0 + n) % ny
    return Fw[np.ix_(xs, ys, np.arange(z0, z0 + n))]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tile_alone_equals_world_cells(dtype):
    from steam_b200.serving import TileServer
    w = _world(dtype)
    Fw = w.world_field().cpu().numpy()
    assert np.all(Fw >= 0) and abs(Fw.mean() - 1.0) < 1e-3  # unit mean restored
    srv = TileServer(w, n_slots=2, max_n=24)
    for origin, n in (((0, 0, 0), 8), ((66, 60, 40), 8), ((10, 20, 5), 16),
                      ((50, 3, 24), 24), ((71, 63, 30), 16)):
        got = srv.tile(origin, n)
        np.testing.assert_array_equal(got, _crop(Fw, origin, n))


def test_tiles_in_a_mix_equal_alone():
    from steam_b200.serving import TileServer, poisson_trace, latency_summary
    w = _world()
    Fw = w.world_field().cpu().numpy()
    srv = TileServer(w, n_slots=4, max_n=32, budget_bytes=3 * 4 * 44 ** 3 * 3)
    reqs = poisson_trace(w, rate=20000.0, n_requests=40, sizes=(8, 16, 32),
                         weights=(0.4, 0.4, 0.2), adjacent=False)
    done = srv.serve(reqs, keep=True)
    assert len(done) == len(reqs)
    for r in done:
        np.testing.assert_array_equal(r['tile'], _crop(Fw, r['origin'], r['n']))
        assert r['latency'] >= 0 and r['done'] >= r['start'] >= r['arrival'] - 1e-9
    s = latency_summary(done)
    assert s['p99_ms'] >= s['p50_ms'] > 0
    # the budget admits at most three 32^3 boxes at once, yet all complete
    assert srv.in_flight_bytes == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("fill", [0, 1])
def test_tile_extract_window_times_scale(dtype, fill):
    """steam_tile_extract: an odd window of a box, rounded scale applied (or
    filled), written contiguously; the host refuses a window past the box."""
    import ctypes
    import torch
    from steam_b200 import _lib
    lib = _lib.load()
    code = _lib.STEAM_F32 if dtype == np.float32 else _lib.STEAM_F64
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    g = torch.Generator(device='cuda').manual_seed(3)
    box = torch.rand((37, 29, 45), generator=g, device='cuda', dtype=tdt) * 3
    x0, y0, z0, ox, oy, oz = 5, 2, 7, 31, 27, 33
    scale = 1.0 + 1.0 / 3.0
    out = torch.full((ox * oy * oz,), -1.0, device='cuda', dtype=tdt)
    _lib.check(lib.steam_tile_extract(code, 37, 29, 45, _lib.ptr(box), x0, y0, z0, ox, oy, oz,
                                      scale, fill, _lib.ptr(out), _lib.stream()))
    torch.cuda.synchronize()
    s = np.asarray(scale, dtype=dtype)
    want = (np.full((ox, oy, oz), s, dtype=dtype) if fill else
            box.cpu().numpy()[x0:x0 + ox, y0:y0 + oy, z0:z0 + oz] * s)
    np.testing.assert_array_equal(out.cpu().numpy().reshape(ox, oy, oz), want)
    with pytest.raises(Exception):
        _lib.check(lib.steam_tile_extract(code, 37, 29, 45, _lib.ptr(box), x0, y0, 13, ox, oy,
                                          oz, scale, fill, _lib.ptr(out), _lib.stream()))
