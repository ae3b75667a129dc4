"""Batched ensemble: members of uneven sizes and parameters, stepped eagerly
across streams and replayed from one captured CUDA graph, give the same
fields; the convolution autotuner never changes a result."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_graph_replay_equals_eager_steps():
    import torch
    from steam_b200.ensemble import Ensemble, Member
    members = [Member((32, 32, 32), 1000, alpha=1.6, c1=0.08, H=0.3, Hz=0.52),
               Member((48, 48, 32), 1001, alpha=1.9, c1=0.15, H=0.45, Hz=0.58),
               Member((64, 64, 48), 1002, alpha=1.8, c1=0.1, H=1 / 3, Hz=5 / 9)]
    ens = Ensemble(members, n_streams=2)
    ens.step_eager()
    torch.cuda.synchronize()
    eager = [(m.h.clone(), m.q.clone(), m.F.clone(), m.diag["qc"].clone()) for m in members]
    led_eager = [(cl.flux.realized.total, cl.flux.n_clipped) for cl in ens.check()]
    for m in members:  # scramble, so the replay must recompute everything
        for t in (m.h, m.q, m.F, m.diag["qc"]):
            t.fill_(-7.0)
        m.rc.ledger_host.zero_()
    ens.capture()
    for _ in range(2):
        ens.step_graph()
    torch.cuda.synchronize()
    for m, ref in zip(members, eager):
        for a, b in zip((m.h, m.q, m.F, m.diag["qc"]), ref):
            assert bool((a == b).all())
    # the replayed steps' ledgers (copied back inside the graph) are the eager ones
    assert [(cl.flux.realized.total, cl.flux.n_clipped) for cl in ens.check()] == led_eager
    # members differ from one another (their own seeds and parameters)
    assert not np.allclose(members[0].F.cpu().numpy().mean(), members[1].F.cpu().numpy().mean(),
                           rtol=0, atol=0)


def test_conv_chunk_never_changes_the_result():
    import torch
    from steam_b200 import _lib
    from steam_b200 import utils as U
    from steam_b200.ensemble import member_setup
    setup = member_setup((64, 64, 32), 5)
    f = torch.randn((64, 64, 32), device='cuda')
    outs = []
    lib = _lib.load()
    for chunk in (16, 48, 256):
        _lib.check(lib.steam_conv_set_xchunk(64, 64, 32, chunk))
        assert lib.steam_conv_get_xchunk(64, 64, 32) == chunk
        out = torch.empty_like(f)
        U.run_plan(setup.plan, f, out)
        outs.append(out.cpu().numpy())
    _lib.check(lib.steam_conv_set_xchunk(64, 64, 32, 0))
    assert lib.steam_conv_get_xchunk(64, 64, 32) == 256
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])
