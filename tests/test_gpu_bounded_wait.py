"""The bounded add's device-side waits give up instead of hanging (needs a B200).

The rescale loop and the shift solve of the bounded add run as persistent
cooperative launches whose blocks meet at a grid barrier; a block that waits
there longer than the spin limit records an error and every block leaves at
its next barrier.  Here the limit is set to one poll, so a block that arrives
before the last one gives up at once: no GPU is held, the kernel returns, and
the host turns the error into RuntimeError (synchronous entry) or into the
ledger's sweep count of -1 (resident step).  The context stays usable: with
the default limit restored the same call agrees with the oracle.
"""

import numpy as np
import pytest

from oracle import steam_oracle as O
from steam_b200 import _lib

pytestmark = pytest.mark.gpu


def _case(seed=3):
    rng = np.random.default_rng(seed)
    shape = (128, 128, 16)  # 8 blocks per persistent phase: blocks do wait
    mean = np.linspace(0.0025, 0.012, shape[2]).astype(np.float32)
    pert = (0.002 * rng.standard_normal(shape)).astype(np.float32)
    pert = np.clip(pert + mean, 0.0, 0.03).astype(np.float32) - mean
    inc = (0.004 * rng.standard_normal(shape)).astype(np.float32)
    return pert, mean, inc


def test_grid_barrier_gives_up_and_the_host_raises():
    from steam_b200 import simulate as sim
    lib = _lib.load()
    pert, mean, inc = _case()
    try:
        _lib.check(lib.steam_set_barrier_spin_limit(1))
        with pytest.raises(RuntimeError, match="grid barrier"):
            sim._bounded_amplitude_add(pert.copy(), mean, inc.copy(), 0.0, 0.03)
    finally:
        _lib.check(lib.steam_set_barrier_spin_limit(0))
    # the context is intact: the default limit gives the oracle's answer
    p_g = pert.copy()
    sim._bounded_amplitude_add(p_g, mean, inc.copy(), 0.0, 0.03)
    p_o = pert.copy()
    O.bounded_amplitude_add(p_o, mean, inc.copy(), 0.0, 0.03)
    np.testing.assert_allclose(p_g, p_o, rtol=0, atol=5e-8)


def test_resident_step_reports_a_barrier_that_gave_up():
    import torch
    from steam_b200 import ensemble
    from steam_b200.resident import ResidentClass
    lib = _lib.load()
    setup = ensemble.member_setup((128, 128, 16), seed=5)
    rc = ResidentClass(setup, torch.float32)
    g = torch.Generator(device='cuda')
    g.manual_seed(5)
    shape = setup.shape
    h = 600.0 * torch.randn(shape, generator=g, device='cuda')
    q = 0.004 * torch.randn(shape, generator=g, device="cuda")  # clips at qt = 0
    F = 1.0 + 0.1 * torch.rand(shape, generator=g, device='cuda')
    try:
        _lib.check(lib.steam_set_barrier_spin_limit(1))
        rc.step(h.clone(), q.clone(), F.clone())
        with pytest.raises(RuntimeError, match="grid barrier"):
            rc.class_ledger()
    finally:
        _lib.check(lib.steam_set_barrier_spin_limit(0))
    rc.step(h.clone(), q.clone(), F.clone())
    led = rc.class_ledger()
    assert led.bounded_add['h'].n_sweeps > 0 and led.bounded_add['qt'].n_sweeps > 0


def test_spin_limit_rejects_negative():
    lib = _lib.load()
    assert lib.steam_set_barrier_spin_limit(-1) == 1
