"""The photometric-calibration oracle pinned on the CPU against the reference's
own composition (PhotometricCalibrationImpl::forward and
CameraResponseNetImpl::forward / ParamLoss, hyperacorn/csrc/modules/
ToneMapper.cpp:32-111,161-201) rebuilt from torch ops: index_select,
torch.nn.functional.grid_sample (the reference's dependency) and autograd,
in FP64. The oracle computes in FP32, so the comparison is within FP32
rounding; the clamp bounds and the leak threshold are hit exactly."""

import math

import numpy as np
import pytest
import torch
import torch.nn.functional as Fn

from oracle import tonemap_oracle as tmo

TOL = dict(rtol=2e-5, atol=2e-6)


def torch_reference(I, uv, iid, mode, exposure, sensor, response, value_range, leak):
    """ToneMapper.cpp:161-201 and :32-97 in torch ops (tensors in FP64)."""
    x = I
    if mode == tmo.FACTOR:
        x = x * torch.index_select(exposure, 0, iid)
    elif mode == tmo.BIAS:
        x = x + torch.index_select(exposure, 0, iid)
    if sensor is not None:
        g = (uv * 2 - 1).unsqueeze(0).unsqueeze(0)
        add = Fn.grid_sample(sensor, g, mode="bilinear", padding_mode="border", align_corners=False)
        x = x + add.squeeze(0).squeeze(1)
    if response is not None:
        img = x.unsqueeze(0).unsqueeze(2)
        leak_add = (img - value_range) * (img > value_range) if leak else None
        t = img * (1.0 / value_range)
        t = t * 2.0 - 1.0
        grid = torch.cat([t.unsqueeze(4), torch.zeros_like(t).unsqueeze(4)], 4)
        res = Fn.grid_sample(response, grid[:, 0], mode="bilinear", padding_mode="border", align_corners=True)
        if leak_add is not None:
            res = res + leak_add
        x = res.reshape(I.shape)
    return x


def case(seed, R=700, C=1, A=9, sw=32, sh=27, P=25, value_range=2.0):
    rng = np.random.default_rng(seed)
    uv = rng.uniform(0, 1, (R, 2)).astype(np.float32)
    uv[:8] = [[0, 0], [1, 1], [0, 1], [1, 0], [0.5, 0.5], [1 / sw, 0.25], [0.999, 0.0001], [0.25, 1 / sh]]
    I = rng.uniform(-0.3, 2.6, (C, R)).astype(np.float32)
    I[0, 8:14] = [0.0, 2.0, value_range, -1.0, 5.0, 1.0]
    iid = rng.integers(0, A, R)
    exposure = rng.uniform(0.8, 1.2, A).astype(np.float32)
    sensor = rng.uniform(0, 0.1, (sh, sw)).astype(np.float32)
    response = np.sort(rng.uniform(0, value_range, P)).astype(np.float32)
    response[0], response[-1] = 0.0, value_range
    g = rng.normal(size=(C, R)).astype(np.float32)
    return I, uv, iid, exposure, sensor, response, g


CONFIGS = [
    dict(mode=tmo.BIAS, sensor=True, response=True, leak=True),    # the reference's defaults, training
    dict(mode=tmo.BIAS, sensor=True, response=True, leak=False),   # evaluation
    dict(mode=tmo.FACTOR, sensor=False, response=True, leak=True),
    dict(mode=tmo.FACTOR, sensor=True, response=False, leak=False),
    dict(mode=0, sensor=False, response=True, leak=True),
    dict(mode=tmo.BIAS, sensor=False, response=False, leak=False),
]


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{int(v)}" for k, v in c.items()))
def test_oracle_matches_torch_composition(cfg):
    I, uv, iid, exposure, sensor, response, g = case(3)
    if cfg["mode"] == tmo.BIAS:
        exposure = (exposure - 1.0).astype(np.float32)
    sens = sensor if cfg["sensor"] else None
    resp = response if cfg["response"] else None
    kw = dict(mode=cfg["mode"], exposure=exposure, sensor=sens, response=resp, value_range=2.0, leak=cfg["leak"])
    out = tmo.forward(I, uv, iid, **kw)
    dI, gexp, gsens, gresp = tmo.backward(I, uv, iid, g, **kw)

    t = lambda a: torch.tensor(np.asarray(a, np.float64), requires_grad=True)
    It, et = t(I), t(exposure)
    st = t(sens.reshape(1, 1, *sens.shape)) if sens is not None else None
    rt = t(resp.reshape(1, 1, 1, -1)) if resp is not None else None
    ref = torch_reference(It, torch.tensor(uv, dtype=torch.float64), torch.from_numpy(iid), cfg["mode"], et, st, rt,
                          2.0, cfg["leak"])
    np.testing.assert_allclose(out, ref.detach().numpy(), **TOL)
    (ref * torch.tensor(g, dtype=torch.float64)).sum().backward()
    np.testing.assert_allclose(dI, It.grad.numpy(), **TOL)
    if cfg["mode"]:
        np.testing.assert_allclose(gexp, et.grad.numpy(), rtol=1e-5, atol=1e-5)
    else:
        assert gexp is None
    if sens is not None:
        np.testing.assert_allclose(gsens, st.grad.numpy()[0, 0], rtol=1e-5, atol=1e-5)
    if resp is not None:
        np.testing.assert_allclose(gresp, rt.grad.numpy().reshape(-1), rtol=1e-5, atol=1e-5)


def test_response_loss_matches_torch_composition():
    """CameraResponseNetImpl::ParamLoss (ToneMapper.cpp:98-111) with torch autograd."""
    rng = np.random.default_rng(8)
    P, value_range = 25, 2.0
    r = (np.linspace(0, value_range, P) + rng.normal(0, 0.05, P)).astype(np.float32)
    loss, grad = tmo.response_loss(r, value_range, scale=1.5)
    rt = torch.tensor(r.astype(np.float64).reshape(1, 1, 1, P), requires_grad=True)
    low, up = rt[..., 0:P - 2], rt[..., 2:P]
    target = rt.clone()
    target = torch.cat([torch.zeros_like(target[..., :1]), (up + low) * 0.5,
                        torch.full_like(target[..., :1], value_range)], 3)
    f = P * math.sqrt(1e-5)
    ref = Fn.mse_loss(rt * f, target * f, reduction="sum")
    (ref * 1.5).backward()
    np.testing.assert_allclose(loss, float(ref.detach()), rtol=1e-5)
    np.testing.assert_allclose(grad, rt.grad.numpy().reshape(-1), rtol=1e-4, atol=1e-7)


def test_initial_response_is_the_identity_ramp():
    """At gamma 1 the curve maps [0, range] to itself (and the leak continues it above)."""
    r = tmo.initial_response(25, 1.0, 2.0)
    np.testing.assert_allclose(r, np.linspace(0, 2, 25), rtol=1e-6, atol=1e-7)
    x = np.array([[0.0, 0.3, 1.0, 1.99, 2.0, 3.5]], np.float32)
    y = tmo.forward(x, None, None, mode=0, response=r, value_range=2.0, leak=True)
    np.testing.assert_allclose(y, x, rtol=1e-6, atol=1e-6)
    assert tmo.sensor_map_height(256, 256) == 32 and tmo.sensor_map_height(300, 200) == 22


def test_module_host_logic():
    """Parameter shapes, initial values and optimiser groups of
    PhotometricCalibration (ToneMapper.cpp:141-160, SceneBase.cpp:158-227),
    without launching a kernel."""
    from adaptivetensordf_b200 import tonemap

    m = tonemap.PhotometricCalibration(7, 1, 200, 300, device="cpu")
    assert m.exposure_factor.shape == (7,) and float(m.exposure_factor.sum()) == 7.0
    assert m.exposure_bias.shape == (7,) and float(m.exposure_bias.abs().sum()) == 0.0
    assert m.sensor_bias.shape == (1, 1, 22, 32)
    assert m.response.response.shape == (1, 1, 1, 25)
    np.testing.assert_allclose(m.response.response.detach().numpy().reshape(-1), np.linspace(0, 2, 25), rtol=1e-6)
    sgd, adam = m.make_optimizers()
    assert [g["lr"] for g in sgd.param_groups] == [0.01, 0.05]
    assert sgd.param_groups[0]["params"][0] is m.exposure_bias
    assert sgd.param_groups[1]["params"][0] is m.sensor_bias
    assert [g["lr"] for g in adam.param_groups] == [1e-4]
    p = tonemap.PhotometricCalibrationParams(exposure_mult=True, response_enable=False, sensor_bias_sgd=False)
    m2 = tonemap.PhotometricCalibration(3, 1, 16, 16, p, device="cpu")
    sgd, adam = m2.make_optimizers()
    assert [g["params"][0] is m2.exposure_factor for g in sgd.param_groups] == [False, True]
    assert adam.param_groups[0]["params"][0] is m2.sensor_bias and m2.response is None
    with torch.no_grad():
        m.exposure_bias.fill_(-1.0)
        m.sensor_bias.fill_(-0.5)
    m.ApplyConstraints()
    assert float(m.exposure_bias.min()) == 0.0 and float(m.sensor_bias.min()) == 0.0
