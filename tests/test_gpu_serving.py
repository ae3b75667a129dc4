"""World-coordinate tile serving of the full class step (needs a B200): every
field of every tile (h', qt', F, qc, qi) equals the same cells of the whole
world's step, bit for bit, alone and when served in a mix of concurrent
requests, through the apply-only replay of the world ledger."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ('h', 'qt', 'flux', 'qc', 'qi')


def _world(dtype=np.float32):
    from steam_b200.serving import TileWorld
    return TileWorld((72, 64, 48), seed=7, dtype=dtype, keep_fields=True)


def _world_host(w):
    return {k: w.world_field(k).cpu().numpy() for k in FIELDS}


def _crop(f, origin, n):
    nx, ny, _ = f.shape
    x0, y0, z0 = origin
    xs = np.arange(x0, x0 + n) % nx
    ys = np.arange(y0, y0 + n) % ny
    return f[np.ix_(xs, ys, np.arange(z0, z0 + n))]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tile_alone_equals_world_cells(dtype):
    from steam_b200.serving import TileServer
    w = _world(dtype)
    W = _world_host(w)
    assert np.all(W['flux'] >= 0) and abs(W['flux'].mean() - 1.0) < 1e-3  # unit mean
    assert np.abs(W['h']).max() > 0 and np.abs(W['qt']).max() > 0
    assert W['qc'].max() > 0  # the world condenses somewhere
    srv = TileServer(w, n_slots=2, max_n=24)
    for origin, n in (((0, 0, 0), 8), ((66, 60, 40), 8), ((10, 20, 5), 16),
                      ((50, 3, 24), 24), ((71, 63, 30), 16), ((30, 30, 20), 1)):
        got = srv.tile(origin, n)
        for k in FIELDS:
            np.testing.assert_array_equal(got[k], _crop(W[k], origin, n), err_msg=k)


def test_tiles_in_a_mix_equal_alone():
    from steam_b200.serving import TileServer, poisson_trace, latency_summary
    w = _world()
    W = _world_host(w)
    srv = TileServer(w, n_slots=4, max_n=32, budget_bytes=3 * w.box_bytes(32))
    reqs = poisson_trace(w, rate=20000.0, n_requests=40, sizes=(8, 16, 32),
                         weights=(0.4, 0.4, 0.2), adjacent=False)
    done = srv.serve(reqs, keep=True)
    assert len(done) == len(reqs)
    for r in done:
        for k in FIELDS:
            np.testing.assert_array_equal(r['tile'][k], _crop(W[k], r['origin'], r['n']),
                                          err_msg=k)
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
