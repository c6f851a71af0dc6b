"""The photometric-calibration kernels (atdf_tone_map_forward / _backward,
atdf_tone_response_loss) against the numpy restatement of
PhotometricCalibrationImpl / CameraResponseNetImpl (ToneMapper.cpp). Every
per-element FP32 operation is rounded on its own in both, so the calibrated
integrals and their gradients are equal bit for bit; the parameter gradients
are sums over rays taken in a different order (atomics), within FP32_RTOL."""

import numpy as np
import pytest
import torch

from oracle import tonemap_oracle as tmo
from tests.test_tonemap_cpu import CONFIGS, case

pytestmark = pytest.mark.gpu

FP32_RTOL = 1e-5


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _module(cfg, A, h, w, exposure, sensor, response):
    from adaptivetensordf_b200 import tonemap

    p = tonemap.PhotometricCalibrationParams(exposure_enable=cfg["mode"] != 0, exposure_mult=cfg["mode"] == tmo.FACTOR,
                                             sensor_bias_enable=cfg["sensor"], response_enable=cfg["response"])
    m = tonemap.PhotometricCalibration(A, 1, h, w, p)
    with torch.no_grad():
        (m.exposure_factor if cfg["mode"] == tmo.FACTOR else m.exposure_bias).copy_(torch.from_numpy(exposure))
        if cfg["sensor"]:
            m.sensor_bias.copy_(torch.from_numpy(sensor).view(m.sensor_bias.shape))
        if cfg["response"]:
            m.response.response.copy_(torch.from_numpy(response).view(1, 1, 1, -1))
    m.train(cfg["leak"])
    return m


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: "-".join(f"{k}{int(v)}" for k, v in c.items()))
@pytest.mark.parametrize("R", [700, 50000])
def test_tone_map_matches_oracle(cfg, R):
    I, uv, iid, exposure, sensor, response, g = case(5 + R, R=R, A=61, sw=32, sh=32)
    if cfg["mode"] == tmo.BIAS:
        exposure = (exposure - 1.0).astype(np.float32)
    m = _module(cfg, 61, 256, 256, exposure, sensor, response)
    It = torch.from_numpy(I).cuda().requires_grad_(True)
    out = m(It, torch.from_numpy(uv).cuda(), torch.from_numpy(iid).cuda())
    out.backward(torch.from_numpy(g).cuda())
    kw = dict(mode=cfg["mode"], exposure=exposure, sensor=sensor if cfg["sensor"] else None,
              response=response if cfg["response"] else None, value_range=2.0, leak=cfg["leak"])
    ref = tmo.forward(I, uv, iid, **kw)
    dI, gexp, gsens, gresp = tmo.backward(I, uv, iid, g, **kw)
    np.testing.assert_array_equal(out.detach().cpu().numpy(), ref)
    np.testing.assert_array_equal(It.grad.cpu().numpy(), dI)
    if cfg["mode"]:
        got = (m.exposure_factor if cfg["mode"] == tmo.FACTOR else m.exposure_bias).grad.cpu().numpy()
        np.testing.assert_allclose(got, gexp, rtol=FP32_RTOL, atol=1e-6 * np.abs(gexp).max())
    if cfg["sensor"]:
        np.testing.assert_allclose(m.sensor_bias.grad.cpu().numpy()[0, 0], gsens, rtol=FP32_RTOL,
                                   atol=1e-6 * np.abs(gsens).max())
    else:
        assert m.sensor_bias.grad is None
    if cfg["response"]:
        np.testing.assert_allclose(m.response.response.grad.cpu().numpy().reshape(-1), gresp, rtol=FP32_RTOL,
                                   atol=1e-6 * np.abs(gresp).max())


def test_response_loss_matches_oracle():
    from adaptivetensordf_b200 import tonemap

    m = tonemap.PhotometricCalibration(4, 1, 64, 64)
    rng = np.random.default_rng(12)
    r = (np.linspace(0, 2, 25) + rng.normal(0, 0.05, 25)).astype(np.float32)
    with torch.no_grad():
        m.response.response.copy_(torch.from_numpy(r).view(1, 1, 1, 25))
    loss = m.ParameterLoss()
    (loss * 3.0).sum().backward()
    ref, grad = tmo.response_loss(r, 2.0, scale=3.0)
    np.testing.assert_allclose(float(loss.detach()), ref, rtol=FP32_RTOL)
    np.testing.assert_allclose(m.response.response.grad.cpu().numpy().reshape(-1), grad, rtol=1e-4,
                               atol=1e-6 * np.abs(grad).max())


def test_identity_at_initialisation():
    """The reference's initial calibration (zero biases, the identity ramp)
    returns non-negative integrals unchanged, with the leak above the range."""
    from adaptivetensordf_b200 import tonemap

    m = tonemap.PhotometricCalibration(3, 1, 32, 32)
    x = torch.tensor([[0.0, 0.25, 1.0, 1.9999, 2.0, 2.5, 7.0]], device="cuda")
    uv = torch.rand(7, 2, device="cuda")
    y = m(x, uv, torch.tensor([0, 1, 2, 0, 1, 2, 0], device="cuda"))
    torch.testing.assert_close(y, x, rtol=1e-6, atol=1e-6)


def test_errors():
    from adaptivetensordf_b200 import tonemap

    m = tonemap.PhotometricCalibration(3, 1, 32, 32)
    x = torch.rand(1, 10, device="cuda")
    uv = torch.rand(10, 2, device="cuda")
    bad = torch.zeros(10, dtype=torch.long, device="cuda")
    bad[7] = 3
    with pytest.raises(RuntimeError, match="out of range"):
        m(x, uv, bad)
    with pytest.raises(RuntimeError, match="not implement|unsupported|UNSUPPORTED"):
        m(torch.rand(2, 10, device="cuda"), uv, torch.zeros(10, dtype=torch.long, device="cuda"))
    # without the response curve any channel count is accepted
    p = tonemap.PhotometricCalibrationParams(response_enable=False)
    m2 = tonemap.PhotometricCalibration(3, 1, 32, 32, p)
    y = m2(torch.rand(2, 10, device="cuda"), uv, torch.zeros(10, dtype=torch.long, device="cuda"))
    assert y.shape == (2, 10)


def test_training_with_the_tone_mapper():
    """The trainer with the reference's default calibration (exposure bias,
    sensor bias, response curve, their SGD / Adam groups, constraints after
    each step; a larger exposure rate than the reference's 0.01 so that 40
    steps suffice) on a small tilt series whose tilts carry an additive
    offset: the loss falls and the learned biases follow the offsets."""
    import dataclasses

    from adaptivetensordf_b200 import recon, tonemap
    from adaptivetensordf_b200 import synthetic as syn

    cfg = dataclasses.replace(syn.CONFIGS["C1"], detector=32, angles=8, angle_step=15.0, noise=0.0, jitter=0.0)
    data = recon.make_tilt_series(cfg)
    offs = torch.linspace(0.0, 0.07, cfg.angles, device="cuda")
    data = dataclasses.replace(data, target=data.target + offs[data.image_id].float())
    opt = recon.TrainOptions(epochs=6, batch=1024, max_samples_per_node=cfg.max_samples_per_node, eval_every=0,
                             stop_at_target=False, init_scale=0.05, tone_mapper=True, tone_after_epochs=1,
                             tone_params=tonemap.PhotometricCalibrationParams(exposure_lr=0.5))
    recs, _ = recon.train(cfg, "fp32", data, opt)
    assert recs[-1]["loss"] < recs[0]["loss"]
    bias = recs[-1]["exposure_bias"]
    assert min(bias) >= 0.0
    assert np.corrcoef(bias, offs.cpu().numpy())[0, 1] > 0.5


def test_empty_batch():
    """No rays: nothing is launched, the outputs are empty and the parameter
    gradients stay zero."""
    from adaptivetensordf_b200 import tonemap

    m = tonemap.PhotometricCalibration(3, 1, 32, 32)
    x = torch.zeros(1, 0, device="cuda", requires_grad=True)
    y = m(x, torch.zeros(0, 2, device="cuda"), torch.zeros(0, dtype=torch.long, device="cuda"))
    assert y.shape == (1, 0)
    y.sum().backward()
    assert float(m.exposure_bias.grad.abs().sum()) == 0.0 and float(m.sensor_bias.grad.abs().sum()) == 0.0
