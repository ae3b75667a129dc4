"""Grouped packed convolutions (needs a B200).

Fields of different shapes convolved with the same turbulon filters as one
launch (``steam_conv_group_*``): each field's output is the same bits as its
own launch of the packed kernel, and with the flux epilogue its window sum
and clip count are the same bits (a small group: each field keeps its own x
chunk); the ensemble step with its convolutions grouped (a large group: each
member's CTAs take its whole x extent) equals the one with per-member
convolutions to rounding.
"""

import numpy as np
import pytest

from oracle import steam_oracle as O
from steam_b200 import _lib

pytestmark = pytest.mark.gpu

K64 = O.turbulon_envelope(1, 0.5, 0.5, 0.5, shape='mexican_hat', dtype=np.float64)
SHAPES = [(64, 64, 64), (40, 70, 52), (96, 48, 32), (33, 30, 16)]
WINDOWS = [None, (3, 35, 4, 60), None, (0, 33, 2, 28)]


def _group(U, torch, epilogue, with_pre):
    lib = _lib.load()
    plan0 = U.plan_convolution(K64, SHAPES[0], np.float32)
    rng = np.random.default_rng(5)
    fields, probs = [], []
    for shape, win in zip(SHAPES, WINDOWS):
        src = torch.as_tensor((0.4 * rng.standard_normal(shape)).astype(np.float32), device='cuda')
        if epilogue == _lib.STEAM_EPI_FLUX:
            out = torch.as_tensor((1.0 + 0.1 * rng.random(shape)).astype(np.float32),
                                  device='cuda')
        else:
            out = torch.zeros(shape, dtype=torch.float32, device='cuda')
        pre = None
        if with_pre:
            pre = torch.as_tensor(np.concatenate([0.5 + rng.random(shape[2]),
                                                  0.5 + rng.random(shape[2])]).astype(np.float32),
                                  device='cuda')
        sums = torch.zeros(2, dtype=torch.float64, device='cuda')
        p = _lib.ConvProblem()
        p.nx, p.ny, p.nz = shape
        p.in_, p.out = src.data_ptr(), out.data_ptr()
        p.pre = None if pre is None else pre.data_ptr()
        p.has_window = 0 if win is None else 1
        if win is not None:
            p.window = _lib.Window(*win)
        p.sums = sums.data_ptr() if epilogue == _lib.STEAM_EPI_FLUX else None
        probs.append(p)
        fields.append((shape, win, src, out.clone(), out, pre, sums))
    arr = (_lib.ConvProblem * len(probs))(*probs)
    nbytes = lib.steam_conv_group_workspace_bytes(len(probs), arr)
    ws = torch.empty(int(nbytes), dtype=torch.uint8, device='cuda')
    import ctypes
    _lib.check(lib.steam_conv_group_prepare(ctypes.byref(plan0.spec), plan0.z_taps, plan0.y_taps,
                                            plan0.x_taps, len(probs), arr, epilogue,
                                            _lib.ptr(ws), int(nbytes)))
    return lib, ws, fields


@pytest.mark.parametrize("epilogue,with_pre", [(0, False), (0, True), (1, False)])
def test_group_equals_own_launches(epilogue, with_pre):
    import ctypes
    import torch
    from steam_b200 import utils as U
    lib, ws, fields = _group(U, torch, epilogue, with_pre)
    try:
        n0 = lib.steam_conv_packed_launches()
        _lib.check(lib.steam_conv_group_async(_lib.ptr(ws), _lib.stream()))
        torch.cuda.synchronize()
        assert lib.steam_conv_packed_launches() == n0 + 1
        for shape, win, src, out0, out, pre, sums in fields:
            plan = U.plan_convolution(K64, shape, np.float32)
            own = out0.clone()
            own_sums = torch.zeros(2, dtype=torch.float64, device='cuda')
            U.run_plan_async(plan, src, own, pre, epilogue, win,
                             ctypes.c_void_p(own_sums.data_ptr()) if epilogue else None)
            torch.cuda.synchronize()
            assert torch.equal(own, out), shape
            if epilogue == _lib.STEAM_EPI_FLUX:
                assert torch.equal(own_sums, sums), (shape, own_sums, sums)
                assert float(sums[1]) > 0 or float(out.min()) > 0
            else:
                s = pre.cpu().numpy().astype(np.float64) if pre is not None else None
                x = src.cpu().numpy().astype(np.float64)
                if s is not None:
                    nz = shape[2]
                    scale = (s[nz:] / s[:nz]).astype(np.float32).astype(np.float64)
                    x = x * scale[None, None, :]
                want = O.convolve(x, K64)
                got = out.cpu().numpy().astype(np.float64)
                assert np.linalg.norm(got - want) / np.linalg.norm(want) < 5e-7
    finally:
        lib.steam_conv_group_release(_lib.ptr(ws))


def test_group_rejects_other_layouts():
    import ctypes
    import torch
    from steam_b200 import utils as U
    lib = _lib.load()
    shape = (32, 33, 32)  # odd ny: not a packed-kernel layout
    plan = U.plan_convolution(K64, shape, np.float32)
    a = torch.zeros(shape, dtype=torch.float32, device='cuda')
    p = _lib.ConvProblem()
    p.nx, p.ny, p.nz = shape
    p.in_, p.out = a.data_ptr(), a.data_ptr()
    arr = (_lib.ConvProblem * 1)(p)
    ws = torch.empty(1 << 16, dtype=torch.uint8, device='cuda')
    rc = lib.steam_conv_group_prepare(ctypes.byref(plan.spec), plan.z_taps, plan.y_taps,
                                      plan.x_taps, 1, arr, _lib.STEAM_EPI_STORE, _lib.ptr(ws),
                                      1 << 16)
    assert rc != 0 and b"layout" in lib.steam_last_error()


def test_ensemble_with_grouped_convolutions_against_per_member_convolutions():
    import torch
    from steam_b200.ensemble import Ensemble, Member
    shapes = [(64, 64, 64), (80, 80, 64), (48, 48, 48), (96, 64, 32)]
    members = [Member(s, 1200 + j, alpha=1.6 + 0.1 * j) for j, s in enumerate(shapes)]
    ens = Ensemble(members, n_streams=2, tune=False, grouped=True)
    assert ens.grouped and set(ens.conv_groups) == {'flux', 'h', 'qt'}
    ens.step_eager()
    torch.cuda.synchronize()
    a = [(m.h.clone(), m.q.clone(), m.F.clone(), m.diag['qc'].clone()) for m in members]
    lib = _lib.load()
    for w, _ in ens.conv_groups.values():
        lib.steam_conv_group_release(_lib.ptr(w))
    ens.conv_groups = {}
    ens.step_eager()
    torch.cuda.synchronize()
    for m, ref in zip(members, a):
        for x, y in zip((m.h, m.q, m.F, m.diag['qc']), ref):
            rel = float(torch.linalg.vector_norm((x - y).double()) /
                        max(float(torch.linalg.vector_norm(y.double())), 1e-30))
            assert rel < 1e-6, rel
    ens.release()


def test_large_group_whole_x_chunks():
    """A group whose tiles fill every SM (each member's CTAs then take its
    whole x extent): outputs the same bits as own launches, flux sums equal
    to rounding, clip counts equal."""
    import ctypes
    import torch
    from steam_b200 import utils as U
    lib = _lib.load()
    shape = (24, 256, 256)  # 64 tiles each: 10 members fill 148 SMs x 4
    plan = U.plan_convolution(K64, shape, np.float32)
    rng = np.random.default_rng(8)
    fields, probs = [], []
    for i in range(10):
        src = torch.as_tensor((0.5 * rng.standard_normal(shape)).astype(np.float32), device='cuda')
        F = torch.as_tensor((1.0 + 0.1 * rng.random(shape)).astype(np.float32), device='cuda')
        sums = torch.zeros(2, dtype=torch.float64, device='cuda')
        p = _lib.ConvProblem()
        p.nx, p.ny, p.nz = shape
        p.in_, p.out, p.pre = src.data_ptr(), F.data_ptr(), None
        p.has_window = 0
        p.sums = sums.data_ptr()
        probs.append(p)
        fields.append((src, F.clone(), F, sums))
    arr = (_lib.ConvProblem * len(probs))(*probs)
    nbytes = lib.steam_conv_group_workspace_bytes(len(probs), arr)
    ws = torch.empty(int(nbytes), dtype=torch.uint8, device='cuda')
    _lib.check(lib.steam_conv_group_prepare(ctypes.byref(plan.spec), plan.z_taps, plan.y_taps,
                                            plan.x_taps, len(probs), arr, _lib.STEAM_EPI_FLUX,
                                            _lib.ptr(ws), int(nbytes)))
    try:
        _lib.check(lib.steam_conv_group_async(_lib.ptr(ws), _lib.stream()))
        torch.cuda.synchronize()
        for src, F0, F, sums in fields:
            own = F0.clone()
            own_sums = torch.zeros(2, dtype=torch.float64, device='cuda')
            U.run_plan_async(plan, src, own, None, _lib.STEAM_EPI_FLUX, None,
                             ctypes.c_void_p(own_sums.data_ptr()))
            torch.cuda.synchronize()
            assert torch.equal(own, F)
            assert float(sums[1]) == float(own_sums[1]) and float(sums[1]) > 0
            assert float(sums[0]) == pytest.approx(float(own_sums[0]), rel=1e-13)
    finally:
        lib.steam_conv_group_release(_lib.ptr(ws))
