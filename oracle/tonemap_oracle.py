"""CPU restatement of the photometric calibration (the "tone mapper"), in numpy.

TEST INFRASTRUCTURE ONLY: tests/ compare the CUDA kernels of
adaptivetensordf_b200/csrc/tonemap.cu (atdf_tone_map_forward / _backward,
atdf_tone_response_loss) with these functions. Nothing in the product imports
this module.

Follows the reference:
  * PhotometricCalibrationImpl::forward   hyperacorn/csrc/modules/ToneMapper.cpp:161-201
  * CameraResponseNetImpl::forward        hyperacorn/csrc/modules/ToneMapper.cpp:32-97
  * CameraResponseNetImpl::ParamLoss      hyperacorn/csrc/modules/ToneMapper.cpp:98-111
  * PhotometricCalibrationImpl::ApplyConstraints   ToneMapper.cpp:215-227
and, for the two bilinear lookups, torch.nn.functional.grid_sample (PyTorch
1.9.1, the reference's pinned dependency; not vendored): source coordinate
((g + 1) size - 1) / 2 (align_corners = false) or ((g + 1) / 2)(size - 1)
(true), clamped to [0, size - 1] (border padding), corners outside the map
skipped, and in the adjoint a zero coordinate gradient on and beyond the
clamp bounds. Every FP32 operation is rounded on its own in the order the
reference's tensor ops apply them, so the per-element outputs are the
kernels' bit for bit; parameter gradients are summed in FP64.

Parity: the restatement is pinned against torch's own grid_sample and
autograd (the reference's composition rebuilt from torch ops) in
tests/test_tonemap_cpu.py. Saiga's DiscreteResponseFunction (MakeGamma,
normalize; Saiga @ a9c60bd, not vendored) is restated as a gamma curve
scaled to end at `range`; at the reference's gamma 1 it is the identity
ramp, whatever the normalisation details.
"""

from __future__ import annotations

import math

import numpy as np

F = np.float32
BIAS, FACTOR = 1, 2


def initial_response(params: int, gamma: float = 1.0, value_range: float = 2.0) -> np.ndarray:
    """CameraResponseNet's initial curve: (i / (P - 1))^gamma, scaled to end at range."""
    x = np.arange(params, dtype=np.float64) / (params - 1)
    y = x ** gamma
    return (y * (value_range / y[-1])).astype(F)


def sensor_map_height(w: int, h: int, size_w: int = 32) -> int:
    """iCeil(sensor_bias_size_w * (float(h) / w)) (ToneMapper.cpp:149-150)."""
    return int(math.ceil(F(size_w) * (F(h) / F(w))))


def _unnorm_edges(g, size):
    return ((g + F(1)) * F(size) - F(1)) / F(2)


def _unnorm_corners(g, size):
    return ((g + F(1)) / F(2)) * F(size - 1)


def _clamp(x, size):
    return np.minimum(F(size - 1), np.maximum(x, F(0)))


def sensor_tap(uv, sw, sh):
    """Corner indices [4, R] (-1 outside the map) and weights [4, R] (nw, ne, sw, se)."""
    uv = np.asarray(uv, F)
    gx = uv[:, 0] * F(2) - F(1)
    gy = uv[:, 1] * F(2) - F(1)
    ix = _clamp(_unnorm_edges(gx, sw), sw)
    iy = _clamp(_unnorm_edges(gy, sh), sh)
    x0, y0 = np.floor(ix), np.floor(iy)
    x1, y1 = x0 + F(1), y0 + F(1)
    w = np.stack([(x1 - ix) * (y1 - iy), (ix - x0) * (y1 - iy), (x1 - ix) * (iy - y0), (ix - x0) * (iy - y0)])
    i0, j0 = x0.astype(np.int64), y0.astype(np.int64)
    xin, yin = i0 + 1 < sw, j0 + 1 < sh
    idx = np.stack([j0 * sw + i0, np.where(xin, j0 * sw + i0 + 1, -1), np.where(yin, (j0 + 1) * sw + i0, -1),
                    np.where(xin & yin, (j0 + 1) * sw + i0 + 1, -1)])
    return idx, w.astype(F)


def response_tap(x, P, value_range):
    """Left tap, right-tap validity, weights and the clamp gradient of the coordinate."""
    inv = F(1) / F(value_range)
    t = (x * inv) * F(2) - F(1)
    raw = _unnorm_corners(t, P)
    ix = _clamp(raw, P)
    x0 = np.floor(ix)
    i0 = x0.astype(np.int64)
    right = i0 + 1 < P
    wl = (x0 + F(1)) - ix
    wr = ix - x0
    clip = np.where((raw <= F(0)) | (raw >= F(P - 1)), F(0), F(1))
    return i0, right, wl, wr, clip


def _pre_response(I, uv, image_id, mode, exposure, sensor):
    x = np.asarray(I, F).copy()
    if mode == FACTOR:
        x = x * exposure[image_id][None, :]
    elif mode == BIAS:
        x = x + exposure[image_id][None, :]
    tap = None
    if sensor is not None:
        idx, w = sensor_tap(uv, sensor.shape[1], sensor.shape[0])
        flat = sensor.reshape(-1)
        val = np.zeros(idx.shape[1], F)
        for k in range(4):
            ok = idx[k] >= 0
            val = np.where(ok, val + flat[np.maximum(idx[k], 0)] * w[k], val)
        x = x + val[None, :]
        tap = (idx, w)
    return x, tap


def forward(I, uv, image_id, mode=BIAS, exposure=None, sensor=None, response=None, value_range=2.0, leak=False):
    """out [C, R] of the integrals I [C, R] (float32)."""
    exposure = None if exposure is None else np.asarray(exposure, F)
    sensor = None if sensor is None else np.asarray(sensor, F)
    image_id = None if image_id is None else np.asarray(image_id, np.int64)
    x, _ = _pre_response(I, uv, image_id, mode, exposure, sensor)
    if response is None:
        return x
    r = np.asarray(response, F)
    P = r.shape[0]
    i0, right, wl, wr, _ = response_tap(x, P, value_range)
    y = r[i0] * wl
    y = np.where(right, y + r[np.minimum(i0 + 1, P - 1)] * wr, y)
    if leak:
        y = np.where(x > F(value_range), y + (x - F(value_range)), y)
    return y


def backward(I, uv, image_id, grad_out, mode=BIAS, exposure=None, sensor=None, response=None, value_range=2.0,
             leak=False):
    """(grad_I [C, R] f32, grad_exposure [A] f64, grad_sensor [sh, sw] f64, grad_response [P] f64);
    the parameter gradients of disabled parts are None."""
    exposure = None if exposure is None else np.asarray(exposure, F)
    sensor = None if sensor is None else np.asarray(sensor, F)
    image_id = None if image_id is None else np.asarray(image_id, np.int64)
    g = np.asarray(grad_out, F)
    I = np.asarray(I, F)
    x, tap = _pre_response(I, uv, image_id, mode, exposure, sensor)
    dx = g.copy()
    gresp = None
    if response is not None:
        r = np.asarray(response, F)
        P = r.shape[0]
        i0, right, wl, wr, clip = response_tap(x, P, value_range)
        gresp = np.zeros(P, np.float64)
        np.add.at(gresp, i0.reshape(-1), (wl * g).astype(np.float64).reshape(-1))
        rr = np.where(right, i0 + 1, 0)
        np.add.at(gresp, rr.reshape(-1), np.where(right, wr * g, F(0)).astype(np.float64).reshape(-1))
        gix = F(0) - r[i0] * g
        gix = np.where(right, gix + r[np.minimum(i0 + 1, P - 1)] * g, gix)
        mult = (F(P - 1) / F(2)) * clip
        dgrid = mult * gix
        inv = F(1) / F(value_range)
        dx = (dgrid * F(2)) * inv
        if leak:
            dx = np.where(x > F(value_range), dx + g, dx)
    gsens = None
    if sensor is not None:
        idx, w = tap
        gsens = np.zeros(sensor.size, np.float64)
        for k in range(4):
            ok = idx[k] >= 0
            contrib = (w[k][None, :] * dx).astype(np.float64)
            np.add.at(gsens, np.broadcast_to(np.maximum(idx[k], 0), dx.shape)[:, ok].reshape(-1),
                      contrib[:, ok].reshape(-1))
        gsens = gsens.reshape(sensor.shape)
    gexp = None
    dI = dx
    if mode in (BIAS, FACTOR):
        gexp = np.zeros(exposure.shape[0], np.float64)
        ids = np.broadcast_to(image_id[None, :], dx.shape).reshape(-1)
        if mode == FACTOR:
            np.add.at(gexp, ids, (dx * I).astype(np.float64).reshape(-1))
            dI = dx * exposure[image_id][None, :]
        else:
            np.add.at(gexp, ids, dx.astype(np.float64).reshape(-1))
    return dI, gexp, gsens, gresp


def response_loss(response, value_range=2.0, scale=1.0):
    """(loss, d loss / d r * scale) of CameraResponseNet::ParamLoss, FP64 sum."""
    r = np.asarray(response, F)
    P = r.shape[0]
    f = F(P * math.sqrt(1e-5))
    t = np.empty(P, F)
    t[0] = F(0)
    t[-1] = F(value_range)
    t[1:-1] = (r[2:] + r[:-2]) * F(0.5)
    d = r * f - t * f
    loss = float(np.sum(d.astype(np.float64) ** 2))
    da = (F(2) * d) * F(scale)
    g = (da * f).astype(np.float64)
    dt = (-da) * f
    for i in range(1, P - 1):
        g[i - 1] += float(dt[i] * F(0.5))
        g[i + 1] += float(dt[i] * F(0.5))
    return loss, g
