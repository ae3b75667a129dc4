"""The packed convolution's slab waits give up instead of hanging (needs a
B200).

Every slab of the packed kernel arrives by a tensor copy that completes on an
mbarrier, and every wait on it is bounded.  The test hook of
``steam_set_copy_wait`` withholds every copy (a phase that nothing completes,
nothing in flight), with a short poll limit: every wait runs out, the blocks
count themselves in a device word and leave -- no fault, no hang.  The host reads the count (``steam_take_wait_errors``) and the
resident step's ledger read raises; with the defaults restored the same
convolution agrees with the oracle and counts nothing.
"""

import ctypes

import numpy as np
import pytest

from oracle import steam_oracle as O
from steam_b200 import _lib

pytestmark = pytest.mark.gpu

K64 = O.turbulon_envelope(1, 0.5, 0.5, 0.5, shape='mexican_hat', dtype=np.float64)


def _take(lib):
    n = ctypes.c_int32(-1)
    _lib.check(lib.steam_take_wait_errors(ctypes.byref(n)))
    return n.value


def test_slab_waits_give_up_and_are_counted():
    import torch
    from steam_b200 import utils as U
    lib = _lib.load()
    shape = (40, 70, 52)
    rng = np.random.default_rng(1)
    f = torch.as_tensor(rng.standard_normal(shape).astype(np.float32), device='cuda')
    plan = U.plan_convolution(K64, shape, np.float32)
    out = torch.zeros_like(f)
    assert _take(lib) == 0
    try:
        _lib.check(lib.steam_set_copy_wait(2000, 1))
        n0 = lib.steam_conv_packed_launches()
        U.run_plan_async(plan, f, out)
        torch.cuda.synchronize()
        assert lib.steam_conv_packed_launches() == n0 + 1
    finally:
        _lib.check(lib.steam_set_copy_wait(0, 0))
    gave_up = _take(lib)
    assert gave_up > 0  # every block waited out its first slab
    assert _take(lib) == 0  # read and reset
    # the context is intact: the same call with the defaults is correct
    U.run_plan_async(plan, f, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.float64)
    want = O.convolve(f.cpu().numpy().astype(np.float64), K64)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 5e-7
    assert _take(lib) == 0


def test_resident_step_reports_slab_waits_that_gave_up():
    import torch
    from steam_b200 import ensemble
    from steam_b200.resident import ResidentClass
    lib = _lib.load()
    shape = (64, 64, 32)
    setup = ensemble.member_setup(shape, seed=4)
    rc = ResidentClass(setup, torch.float32, autotune=False)
    g = torch.Generator(device='cuda')
    g.manual_seed(4)
    h = 600.0 * torch.randn(shape, generator=g, device='cuda')
    q = 0.0006 * torch.randn(shape, generator=g, device='cuda')
    F = 1.0 + 0.1 * torch.rand(shape, generator=g, device='cuda')
    try:
        _lib.check(lib.steam_set_copy_wait(2000, 1))
        rc.step(h.clone(), q.clone(), F.clone())
        with pytest.raises(RuntimeError, match="gave up"):
            rc.class_ledger()
    finally:
        _lib.check(lib.steam_set_copy_wait(0, 0))
        _take(lib)
    rc.step(h.clone(), q.clone(), F.clone())
    led = rc.class_ledger()
    assert led.flux.n_clipped >= 0 and led.bounded_add['h'].n_sweeps > 0
