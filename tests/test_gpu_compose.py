"""Output composition and the z-major slab on the device (needs a B200).

_compose_output (steam/simulate.py:3558-3599): state + deficit, projected per
level, plus the mean profile, clamped to the bounds -- against the oracle.
The z-major slab the streamed output writes (steam/streaming.py:1462-1692):
out[z][x][y] = field[x][y][z0 + z], bit for bit, on shapes that cut the 32 x 32
transpose tiles unevenly.
"""

import numpy as np
import pytest

from oracle import steam_oracle as O
from steam_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("with_deficit", [False, True])
def test_compose_output_against_oracle(dtype, with_deficit):
    from steam_b200 import simulate as sim
    rng = np.random.default_rng(12)
    shape = (30, 22, 14)
    mean = np.linspace(0.001, 0.02, shape[2]).astype(np.float32)
    state = (0.006 * rng.standard_normal(shape)).astype(dtype)
    deficit = (0.002 * rng.standard_normal(shape)).astype(dtype) if with_deficit else None
    want = O.compose_output(state.copy(), None if deficit is None else deficit.copy(), mean,
                            0.0, 0.03)
    got, _ = sim._compose_output(state.copy(), deficit, mean, 0.0, 0.03)
    assert got.dtype == dtype
    tol = 1e-12 if dtype == np.float64 else 2e-9
    np.testing.assert_allclose(got, want, rtol=0, atol=tol)
    assert got.min() >= 0.0 and got.max() <= 0.03


@pytest.mark.parametrize("shape,z0,dz", [((37, 29, 70), 3, 41), ((8, 8, 8), 0, 8),
                                         ((65, 1, 33), 32, 1), ((1, 100, 40), 5, 35)])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_slab_zmajor(shape, z0, dz, dtype):
    import torch
    lib = _lib.load()
    rng = np.random.default_rng(1)
    f = rng.standard_normal(shape).astype(dtype)
    ft = torch.as_tensor(f, device='cuda')
    out = torch.full((dz, shape[0], shape[1]), -7.0, dtype=ft.dtype, device='cuda')
    _lib.check(lib.steam_slab_zmajor(_lib.dtype_code(ft), *shape, _lib.ptr(ft), z0, dz,
                                     _lib.ptr(out), _lib.stream()))
    np.testing.assert_array_equal(out.cpu().numpy(), f[:, :, z0:z0 + dz].transpose(2, 0, 1))


def test_slab_zmajor_rejects_levels_outside():
    import torch
    lib = _lib.load()
    ft = torch.zeros((4, 4, 8), device='cuda')
    out = torch.zeros((8, 4, 4), device='cuda')
    rc = lib.steam_slab_zmajor(_lib.STEAM_F32, 4, 4, 8, _lib.ptr(ft), 4, 5, _lib.ptr(out),
                               _lib.stream())
    assert rc == 1
