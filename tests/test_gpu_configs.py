"""Single class steps at the benchmark configurations (needs a B200).

Each case is the finest size class of a root run over the configuration's
domain (``tests/config_cases.py``: alpha 1.8, C1 0.1, H 1/3, Hz 5/9, seed 0)
on a seeded synthetic entering state, taken through this package's
``cascade_loop`` -- the call the reference makes -- and the condensate map.

* 128 x 128 x 64, Mexican hat and Morlet, FP64 and FP32: against the FP64
  oracle on every cell, and against the reference's own run of the same step
  (``tests/golden/c0_class_step.npz``) on its sampled cells, ledger scalars
  and per-level statistics.  The reference computes in float32, so the
  device is held to being as close to it as the FP64 oracle is, plus the
  device's own bar against that oracle (the triangle inequality).
* 128 x 128 x 64 at sparsity 5 (the 61^3 kernel): against the FP64 oracle.
* 512 x 512 x 256, FP64 and FP32: against the FP64 oracle on every cell.
* 2048 x 2048 x 256: FP32 against FP64 on the device, on the same inputs
  (the FP64 device step is the one pinned to the oracle above).

Bars.  FP64 device vs FP64 oracle: 1e-9 relative L2 (flux, condensate) and
1e-8 for the scalar increments (their bounded add solves a root per level).
FP32 device vs FP64: log-flux relative L2 <= 1e-5 over the cells clear of the
clip (F > 1e-3), clip states differing in at most 1 cell in 10,000, cells
within the clip band within 8 float32 ulps of the entering flux's magnitude
absolute (there F + T * (eps F) cancels to O(1e-4) from O(1) terms, so the
float32 rounding of those terms is all that is left); scalar increments, qc and qi
within 1e-4 relative L2 (the reference's own float32 step is 2e-5 - 4e-5
from FP64 on the full fields).
"""

import numpy as np
import pytest

import config_cases as cc
from oracle import steam_oracle as O

pytestmark = pytest.mark.gpu

GOLDEN_C0 = cc.__file__.replace("config_cases.py", "golden/c0_class_step.npz")

LOG_FLUX_BAR = 1e-5
F32_ULP = float(np.finfo(np.float32).eps)


def near_clip_bar(F0):
    """Absolute flux bar on the cells within the clip band: 8 float32 ulps
    of the largest entering flux."""
    return 8 * F32_ULP * float(np.max(np.abs(F0)))
F32_FIELD_BAR = 1e-4
F64_BAR = 1e-9
F64_INC_BAR = 1e-8


@pytest.fixture(scope="module")
def steam():
    import steam_b200.simulate
    import steam_b200.thermodynamics
    return steam_b200


@pytest.fixture(scope="module")
def c0_golden():
    with np.load(GOLDEN_C0) as g:
        return {k: g[k] for k in g.files}


_ORACLE_CACHE = {}


def _oracle64(steam, shape, s=1, tshape='mexican_hat'):
    key = (shape, s, tshape)
    if key not in _ORACLE_CACHE:
        case = cc.build(steam.simulate, shape, s=s)
        h, q, F = cc.inputs(shape)
        fields, rec = cc.oracle_step(O, case, h, q, F, tshape, np.float64)
        _ORACLE_CACHE.clear()  # one configuration's fields held at a time
        _ORACLE_CACHE[key] = (case, (h, q, F), fields, rec)
    return _ORACLE_CACHE[key]


def _check_against_oracle(dev, ora, inputs, dtype, report):
    h0, q0, _ = inputs
    errs = {}
    if dtype == np.float64:
        errs["flux"] = cc.rel_l2(dev["flux"], ora["flux"])
        assert errs["flux"] < F64_BAR, errs
    else:
        lf = cc.log_flux_error(dev["flux"], ora["flux"])
        errs.update(lf)
        assert lf["log_flux_rel_l2"] <= LOG_FLUX_BAR, lf
        assert lf["clip_mask_differs"] <= max(1, dev["flux"].size // 10000), lf
        assert lf["near_clip_max_abs"] < near_clip_bar(inputs[2]), lf
    inc_bar = F64_INC_BAR if dtype == np.float64 else F32_FIELD_BAR
    field_bar = F64_BAR if dtype == np.float64 else F32_FIELD_BAR
    errs["h_increment"] = cc.rel_l2(dev["h"] - h0, ora["h"] - h0)
    errs["qt_increment"] = cc.rel_l2(dev["qt"] - q0, ora["qt"] - q0)
    for name in ("qc", "qi", "T"):
        errs[name] = cc.rel_l2(dev[name], ora[name])
    report(errs)
    assert errs["h_increment"] < inc_bar, errs
    assert errs["qt_increment"] < inc_bar, errs
    for name in ("qc", "qi", "T"):
        assert errs[name] < field_bar, errs
    return errs


@pytest.mark.parametrize("tshape", ["mexican_hat", "morlet_omega0_6"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_c0_class_step_against_oracle_and_reference(steam, c0_golden, tshape, dtype):
    case, inputs, ora, rec = _oracle64(steam, cc.C0, tshape=tshape)
    h0, q0, F0 = inputs
    dev, led = cc.device_step(steam.simulate, steam.thermodynamics, case, h0, q0, F0, dtype,
                              turbulon_shape=tshape)
    errs = _check_against_oracle(dev, ora, inputs, dtype, print)
    # the reference's own step on the sampled cells
    tag = 'mh' if tshape == 'mexican_hat' else 'mo'
    g = c0_golden
    idx = g["idx"]
    bar = {"flux": F64_BAR if dtype == np.float64 else 2e-6,
           "h": F64_INC_BAR if dtype == np.float64 else F32_FIELD_BAR,
           "qt": F64_INC_BAR if dtype == np.float64 else F32_FIELD_BAR,
           "qc": F64_BAR if dtype == np.float64 else F32_FIELD_BAR,
           "qi": F64_BAR if dtype == np.float64 else F32_FIELD_BAR,
           "T": F64_BAR if dtype == np.float64 else F32_FIELD_BAR}
    for name in ("flux", "h", "qt", "qc", "qi", "T"):
        ref = g[f"{tag}_{name}_sample"]
        e_dev = cc.rel_l2(dev[name].reshape(-1)[idx], ref)
        e_ora = cc.rel_l2(ora[name].reshape(-1)[idx], ref)
        assert e_dev <= e_ora + bar[name], (name, e_dev, e_ora)
        lv_dev = cc.rel_l2(cc.level_stats(dev[name]), g[f"{tag}_{name}_levels"])
        lv_ora = cc.rel_l2(cc.level_stats(ora[name]), g[f"{tag}_{name}_levels"])
        assert lv_dev <= lv_ora + bar[name], (name, lv_dev, lv_ora)
    # integer ledger entries are exact; the clip count may move by the cells
    # whose clip state is within rounding of the bound
    fl = g[f"{tag}_flux_ledger"]
    assert led.flux.entering.count == fl[1]
    assert led.flux.noise_abs.count == fl[3]
    assert abs(led.flux.n_clipped - fl[6]) <= max(2, int(fl[6]) // 1000), \
        (led.flux.n_clipped, fl[6])
    assert led.flux.entering.total == pytest.approx(fl[0], rel=1e-12)
    for name in ("h", "qt"):
        pat = g[f"{tag}_{name}_pattern"]
        np.testing.assert_array_equal(np.asarray(led.pattern[name].level_count), pat[1])
        assert cc.rel_l2(led.pattern[name].level_total, pat[0]) < 1e-4
        assert cc.rel_l2(led.bounded_add[name].a0, g[f"{tag}_{name}_ba_a0"]) < 1e-4
    print(tshape, np.dtype(dtype).name, errs)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_c0_sparsity5_k61_class_step_against_oracle(steam, dtype):
    """The 61^3 kernel (sparsity 5) of the 512^3-class configuration's
    "64-voxel kernel support", on the 128 x 128 x 64 grid."""
    case, inputs, ora, _ = _oracle64(steam, cc.C0, s=5)
    dev, _ = cc.device_step(steam.simulate, steam.thermodynamics, case, *inputs, dtype)
    _check_against_oracle(dev, ora, inputs, dtype, print)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_c1_class_step_against_oracle(steam, dtype):
    """512 x 512 x 256 on every cell (the oracle's FP64 step is computed once
    for both dtypes)."""
    case, inputs, ora, _ = _oracle64(steam, cc.C1_SHAPE)
    dev, _ = cc.device_step(steam.simulate, steam.thermodynamics, case, *inputs, dtype)
    errs = _check_against_oracle(dev, ora, inputs, dtype, print)
    print("C1", np.dtype(dtype).name, errs)


def c2_float32_vs_float64(steam, torch):
    """FP32 and FP64 device steps at 2048 x 2048 x 256 on the same inputs;
    returns the error record (computed on the device)."""
    from steam_b200 import resident
    sim, thermo = steam.simulate, steam.thermodynamics
    case = cc.build(sim, cc.C2)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(2026)
    shape = cc.C2
    h0 = (600.0 * torch.randn(shape, generator=gen, device="cuda")).float()
    q0 = (0.0006 * torch.randn(shape, generator=gen, device="cuda")).float()
    F0 = (1.0 + 0.1 * torch.rand(shape, generator=gen, device="cuda")).float()
    f64, _ = cc.device_step(sim, thermo, case, h0.double(), q0.double(), F0.double(),
                            np.float64, resident=True)
    keep64 = {k: f64[k] for k in ("flux", "h", "qt", "qc", "qi")}
    del f64
    resident._CACHE.clear()
    torch.cuda.empty_cache()
    f32, _ = cc.device_step(sim, thermo, case, h0, q0, F0, np.float32, resident=True)
    keep32 = {k: f32[k] for k in ("flux", "h", "qt", "qc", "qi")}
    del f32
    resident._CACHE.clear()
    torch.cuda.empty_cache()
    errs = device_errors(torch, keep32, keep64, h0, q0)
    errs["near_clip_bar"] = near_clip_bar(float(F0.abs().max()))
    return errs


def device_errors(torch, d32, d64, h0, q0, clip_band=1e-3):
    """The same error record as ``config_cases.log_flux_error`` and the field
    relative L2s, evaluated on the device."""
    def rel(a, b):
        return float(torch.linalg.vector_norm((a - b).double())
                     / torch.linalg.vector_norm(b.double()))
    F, Fr = d32["flux"].double(), d64["flux"]
    clear = (Fr > clip_band) & (F > clip_band)
    both = (Fr == 0) & (F == 0)
    near = ~clear & ~both
    lf = torch.log(F[clear])
    lr = torch.log(Fr[clear])
    out = {"log_flux_rel_l2": float(torch.linalg.vector_norm(lf - lr)
                                    / torch.linalg.vector_norm(lr)),
           "clip_mask_differs": int(((F > 0) != (Fr > 0)).sum()),
           "near_clip_cells": int(near.sum()),
           "near_clip_max_abs": float((F[near] - Fr[near]).abs().max()) if bool(near.any())
           else 0.0}
    del F, clear, both, near, lf, lr
    out["h_increment"] = rel(d32["h"].double() - h0.double(), d64["h"] - h0.double())
    out["qt_increment"] = rel(d32["qt"].double() - q0.double(), d64["qt"] - q0.double())
    out["qc"] = rel(d32["qc"], d64["qc"])
    out["qi"] = rel(d32["qi"], d64["qi"])
    return out


def test_c2_float32_against_float64_device(steam):
    import torch
    errs = c2_float32_vs_float64(steam, torch)
    print("C2", errs)
    n = int(np.prod(cc.C2))
    assert errs["log_flux_rel_l2"] <= LOG_FLUX_BAR, errs
    assert errs["clip_mask_differs"] <= n // 10000, errs
    assert errs["near_clip_max_abs"] < errs["near_clip_bar"], errs
    for name in ("h_increment", "qt_increment", "qc", "qi"):
        assert errs[name] < F32_FIELD_BAR, errs
