"""Grouped thermodynamics (needs a B200).

n fields of different shapes mapped to condensate in ONE launch
(``steam_thermo_group_*``): every field's T, qv, qc, qi and p are the same
bits as its own ``steam_thermo_async`` call, with and without the
composition with mean profiles and with a surface-pressure field; the
ensemble step with its thermodynamics grouped equals the one with
per-member launches bit for bit.
"""

import numpy as np
import pytest

from steam_b200 import _lib

pytestmark = pytest.mark.gpu

SHAPES = [(40, 36, 30), (7, 9, 20), (64, 48, 5), (33, 17, 70), (128, 130, 16)]
BOUNDS = (315 * 1004.0, 355 * 1004.0, 0.0, 0.03)
OUT = ("T", "qv", "qc", "qi", "p")


def _field(torch, shape, rng, dtype, compose, with_ps):
    nx, ny, nz = shape
    tdt = torch.float32 if dtype == np.float32 else torch.float64
    z = np.arange(nz) * 100.0
    dz = np.append(np.diff(z), 0.0)
    hm = 330e3 - 15e3 * z / max(z[-1], 1.0)
    qm = 0.015 - 0.012 * z / max(z[-1], 1.0)
    prof = torch.as_tensor(np.concatenate([z, dz, hm, qm]), dtype=torch.float64, device='cuda')
    if compose:
        h = 800.0 * rng.standard_normal(shape)
        q = 0.002 * rng.standard_normal(shape)
    else:
        h = hm[None, None, :] + 800.0 * rng.standard_normal(shape)
        q = np.clip(qm[None, None, :] + 0.002 * rng.standard_normal(shape), 0.0, None)
    ps = (torch.as_tensor(101325.0 + 300.0 * rng.standard_normal((nx, ny)), dtype=torch.float64,
                          device='cuda') if with_ps else None)
    return dict(shape=shape, h=torch.as_tensor(h, dtype=tdt, device='cuda'),
                q=torch.as_tensor(q, dtype=tdt, device='cuda'), prof=prof, ps=ps,
                compose=compose,
                out={k: torch.full(shape, -1.0, dtype=tdt, device='cuda') for k in OUT})


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_group_equals_own_launches(dtype):
    import torch
    lib = _lib.load()
    code = _lib.STEAM_F32 if dtype == np.float32 else _lib.STEAM_F64
    rng = np.random.default_rng(21)
    fields = [_field(torch, s, rng, dtype, compose=i % 2 == 0, with_ps=i == 3)
              for i, s in enumerate(SHAPES)]
    probs = []
    for f in fields:
        p = _lib.ThermoProblem()
        p.nx, p.ny, p.nz = f['shape']
        p.h, p.qt, p.prof = _lib.ptr(f['h']), _lib.ptr(f['q']), _lib.ptr(f['prof'])
        p.compose = 1 if f['compose'] else 0
        for j, b in enumerate(BOUNDS):
            p.bounds[j] = b
        p.surface_pressure = 100500.0
        p.ps_field = None if f['ps'] is None else _lib.ptr(f['ps'])
        p.T, p.qv, p.qc, p.qi, p.p = (_lib.ptr(f['out'][k]) for k in OUT)
        probs.append(p)
    arr = (_lib.ThermoProblem * len(probs))(*probs)
    nbytes = lib.steam_thermo_group_workspace_bytes(len(probs), arr)
    ws = torch.empty(int(nbytes), dtype=torch.uint8, device='cuda')
    _lib.check(lib.steam_thermo_group_prepare(code, len(probs), arr, _lib.ptr(ws), int(nbytes)))
    try:
        n0 = lib.steam_launch_count()
        _lib.check(lib.steam_thermo_group_async(_lib.ptr(ws), _lib.stream()))
        torch.cuda.synchronize()
        assert lib.steam_launch_count() == n0 + 1
        for f in fields:
            own = {k: torch.full_like(f['out'][k], -2.0) for k in OUT}
            nx, ny, nz = f['shape']
            _lib.check(lib.steam_thermo_async(
                code, nx, ny, nz, _lib.ptr(f['h']), _lib.ptr(f['q']), _lib.ptr(f['prof']),
                1 if f['compose'] else 0, _lib.dvec(BOUNDS), 100500.0,
                None if f['ps'] is None else _lib.ptr(f['ps']),
                *(_lib.ptr(own[k]) for k in OUT), _lib.stream()))
            torch.cuda.synchronize()
            for k in OUT:
                assert torch.equal(own[k], f['out'][k]), (f['shape'], k)
            assert float(f['out']['T'].min()) > 150.0
    finally:
        lib.steam_thermo_group_release(_lib.ptr(ws))
    # a released group is unknown to the library
    assert lib.steam_thermo_group_async(_lib.ptr(ws), _lib.stream()) != 0


def test_ensemble_with_grouped_thermodynamics_against_per_member_launches():
    import torch
    from steam_b200.ensemble import Ensemble, Member
    shapes = [(64, 64, 64), (80, 80, 64), (48, 48, 48), (96, 64, 32)]
    members = [Member(s, 1300 + j, alpha=1.7 + 0.05 * j) for j, s in enumerate(shapes)]
    ens = Ensemble(members, n_streams=2, tune=False, grouped=True)
    assert ens.thermo_group is not None
    ens.step_eager()
    torch.cuda.synchronize()
    ref = [{k: m.diag[k].clone() for k in OUT} for m in members]
    lib = _lib.load()
    lib.steam_thermo_group_release(_lib.ptr(ens.thermo_group[0]))
    ens.thermo_group = None
    for m in members:
        for k in OUT:
            m.diag[k].fill_(-3.0)
    ens.step_eager()
    torch.cuda.synchronize()
    for m, r in zip(members, ref):
        for k in OUT:
            assert torch.equal(m.diag[k], r[k]), k
    ens.release()
