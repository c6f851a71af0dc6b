"""Photometric calibration of the projected ray integrals (the reference's tone
mapper, hyperacorn/csrc/modules/ToneMapper.h:7-106, ToneMapper.cpp).

``PhotometricCalibration`` keeps the reference's parameters and their
initial values:

  exposure_factor [num_images]        ones   (used when exposure_mult)
  exposure_bias   [num_images]        zeros  (used otherwise)
  sensor_bias     [1, 1, size_h, size_w]   zeros, size_h = ceil(size_w * h / w)
  response.response [1, 1, 1, 25]     the identity ramp on [0, response_range]

``forward(ray_integral [C, R], uv [R, 2], image_id [R])`` applies exposure,
sensor bias and the response curve (with the leak above the range in
training mode) in one CUDA kernel, and its autograd backward is one kernel
that writes the integral gradient and adds the parameter gradients
(atdf_tone_map_forward / atdf_tone_map_backward). ``ParameterLoss`` is the
curve's smoothness loss (atdf_tone_response_loss), ``ApplyConstraints`` keeps
the biases non-negative, and ``make_optimizers`` builds the SGD and Adam
groups of SceneBase (hyperacorn/csrc/data/SceneBase.cpp:158-227).
"""

from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import capi

RESPONSE_PARAMS = 25  # CameraResponseNet(25, 1, 1, range, 1), ToneMapper.cpp:155


@dataclass
class PhotometricCalibrationParams:
    """ToneMapper.h:7-53 (the defaults are the reference's)."""

    response_enable: bool = True
    response_sgd: bool = False
    response_range: float = 2.0
    response_lr: float = 1e-4
    exposure_sgd: bool = True
    exposure_enable: bool = True
    exposure_mult: bool = False
    exposure_lr: float = 0.01
    sensor_bias_sgd: bool = True
    sensor_bias_enable: bool = True
    sensor_bias_size_w: int = 32
    sensor_bias_lr: float = 0.05
    use_expose_constraint: bool = True


def initial_response(params: int, gamma: float, value_range: float) -> torch.Tensor:
    """The curve DiscreteResponseFunction::MakeGamma(gamma) + normalize(range)
    starts from: (i / (P - 1))^gamma scaled to end at range."""
    x = torch.arange(params, dtype=torch.float64) / (params - 1)
    y = x ** gamma
    return (y * (value_range / float(y[-1]))).float()


def _stream():
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(st, what):
    if st != 0:
        raise RuntimeError(f"{what}: {capi.lib().atdf_status_string(st).decode()}")


class _ToneMapFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, module, integral, uv, image_id, exposure, sensor, response):
        out = torch.empty_like(integral)
        err = torch.zeros(1, dtype=torch.int32, device=integral.device)
        tm = module._struct(exposure, sensor, response)
        C, R = integral.shape
        _check(capi.lib().atdf_tone_map_forward(ct.byref(tm), C, R, capi.ptr(integral), capi.ptr(uv),
                                                capi.ptr(image_id), capi.ptr(out), capi.ptr(err), _stream()),
               "atdf_tone_map_forward")
        if module.check_errors and int(err.item()) != 0:
            raise RuntimeError("atdf_tone_map_forward: image id out of range")
        ctx.module = module
        ctx.save_for_backward(integral, uv, image_id, exposure, sensor, response)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        integral, uv, image_id, exposure, sensor, response = ctx.saved_tensors
        m = ctx.module
        need = ctx.needs_input_grad
        gI = torch.empty_like(integral) if need[1] else None
        gexp = torch.zeros_like(exposure) if need[4] else None
        gsens = torch.zeros_like(sensor) if need[5] else None
        gresp = torch.zeros_like(response) if need[6] else None
        err = torch.zeros(1, dtype=torch.int32, device=integral.device)
        tm = m._struct(exposure, sensor, response)
        C, R = integral.shape
        _check(capi.lib().atdf_tone_map_backward(ct.byref(tm), C, R, capi.ptr(integral), capi.ptr(uv),
                                                 capi.ptr(image_id), capi.ptr(grad_out.contiguous()), capi.ptr(gI),
                                                 capi.ptr(gexp), capi.ptr(gsens), capi.ptr(gresp), capi.ptr(err),
                                                 _stream()),
               "atdf_tone_map_backward")
        return None, gI, None, None, gexp, gsens, gresp


class _ResponseLossFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, response, value_range):
        loss = torch.empty(1, dtype=torch.float32, device=response.device)
        _check(capi.lib().atdf_tone_response_loss(response.numel(), capi.ptr(response), value_range, capi.ptr(loss),
                                                  None, None, _stream()),
               "atdf_tone_response_loss")
        ctx.save_for_backward(response)
        ctx.value_range = value_range
        return loss

    @staticmethod
    def backward(ctx, grad_loss):
        (response,) = ctx.saved_tensors
        g = torch.zeros_like(response)
        # the kernel scales the loss gradient by the upstream gradient, read on the device
        scale = grad_loss.reshape(-1)[:1].float().contiguous()
        _check(capi.lib().atdf_tone_response_loss(response.numel(), capi.ptr(response), ctx.value_range, None,
                                                  capi.ptr(g), capi.ptr(scale), _stream()),
               "atdf_tone_response_loss")
        return g, None


class CameraResponseNet(torch.nn.Module):
    """The response curve (ToneMapper.cpp:7-31): one channel of ``params``
    samples spanning inputs [0, range]; leak_clamp_value > 0 adds the leak
    above the range in training mode."""

    def __init__(self, params: int = RESPONSE_PARAMS, initial_gamma: float = 1.0, value_range: float = 2.0,
                 leaky_clamp_value: float = 1.0, device="cuda"):
        super().__init__()
        self.range = float(value_range)
        self.leak = leaky_clamp_value > 0
        self.response = torch.nn.Parameter(
            initial_response(params, initial_gamma, value_range).view(1, 1, 1, params).to(device))

    def NumParameters(self):
        return self.response.shape[3]

    def ParamLoss(self):
        return _ResponseLossFn.apply(self.response.view(-1), self.range)


class PhotometricCalibration(torch.nn.Module):
    """PhotometricCalibrationImpl (ToneMapper.cpp:141-227) on the CUDA kernels."""

    def __init__(self, num_images: int, num_cameras: int, h: int, w: int,
                 params: PhotometricCalibrationParams = None, device="cuda"):
        super().__init__()
        if num_images <= 0 or num_cameras <= 0 or w <= 0 or h <= 0:
            raise ValueError("PhotometricCalibration: positive image count, camera count and size")
        self.params = params or PhotometricCalibrationParams()
        p = self.params
        self.exposure_factor = torch.nn.Parameter(torch.ones(num_images, device=device))
        self.exposure_bias = torch.nn.Parameter(torch.zeros(num_images, device=device))
        size_w = p.sensor_bias_size_w
        # iCeil(size_w * (float(h) / w)) in FP32
        size_h = math.ceil(float(np.float32(size_w) * (np.float32(h) / np.float32(w))))
        self.sensor_bias = torch.nn.Parameter(torch.zeros(1, 1, size_h, size_w, device=device))
        self.response = CameraResponseNet(RESPONSE_PARAMS, 1.0, p.response_range, 1.0, device) \
            if p.response_enable else None
        self.check_errors = True
        self.register_buffer("_unused", torch.zeros(0, device=device), persistent=False)

    def _struct(self, exposure, sensor, response):
        p = self.params
        t = capi.ToneMapper()
        t.num_images = self.exposure_factor.shape[0]
        t.exposure_mode = 0 if not p.exposure_enable else (2 if p.exposure_mult else 1)
        t.exposure = exposure.data_ptr() if t.exposure_mode else None
        if p.sensor_bias_enable:
            t.sensor_h, t.sensor_w = sensor.shape[-2], sensor.shape[-1]
            t.sensor_bias = sensor.data_ptr()
        if self.response is not None:
            t.response_params = response.numel()
            t.response = response.data_ptr()
            t.response_range = self.response.range
            t.leak = int(self.response.leak and self.training)
        return t

    def forward(self, ray_integral: torch.Tensor, uv: torch.Tensor, image_id: torch.Tensor) -> torch.Tensor:
        """ray_integral [C, R] float32, uv [R, 2] in [0, 1], image_id [R] -> [C, R]."""
        if ray_integral.dim() != 2 or uv.shape != (ray_integral.shape[1], 2):
            raise ValueError("PhotometricCalibration: ray_integral [C, R] and uv [R, 2]")
        p = self.params
        none = self._unused
        exposure = none if not p.exposure_enable else (self.exposure_factor if p.exposure_mult else self.exposure_bias)
        sensor = self.sensor_bias.view(self.sensor_bias.shape[-2:]) if p.sensor_bias_enable else none
        resp = self.response.response.view(-1) if self.response is not None else none
        return _ToneMapFn.apply(self, ray_integral.float().contiguous(), uv.float().contiguous(),
                                image_id.to(torch.int32).contiguous(), exposure, sensor, resp)

    def ParameterLoss(self, active_images=None) -> torch.Tensor:
        """The response curve's smoothness loss [1] (zero without a curve)."""
        if self.response is None:
            return torch.zeros(1, device=self.exposure_factor.device)
        return self.response.ParamLoss()

    @torch.no_grad()
    def ApplyConstraints(self):
        """Keeps the exposure bias (use_expose_constraint) and the sensor bias non-negative."""
        if self.params.use_expose_constraint:
            self.exposure_bias.clamp_min_(0)
        self.sensor_bias.clamp_min_(0)

    def make_optimizers(self):
        """(sgd, adam) over the calibration's parameters, grouped as SceneBase
        does (SceneBase.cpp:158-227); either may be None."""
        p = self.params
        sgd, adam = [], []
        if p.exposure_enable:
            sgd.append({"params": [self.exposure_bias], "lr": p.exposure_lr})
            if p.exposure_mult:
                (sgd if p.exposure_sgd else adam).append({"params": [self.exposure_factor], "lr": p.exposure_lr})
        if p.sensor_bias_enable:
            (sgd if p.sensor_bias_sgd else adam).append({"params": [self.sensor_bias], "lr": p.sensor_bias_lr})
        if self.response is not None:
            (sgd if p.response_sgd else adam).append({"params": [self.response.response], "lr": p.response_lr})
        return (torch.optim.SGD(sgd, lr=10) if sgd else None), (torch.optim.Adam(adam, lr=10) if adam else None)
