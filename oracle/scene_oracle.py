"""CPU restatement of the tilt-series ingestion path, in numpy.

TEST INFRASTRUCTURE ONLY: tests/ compare the CUDA ray generator
(atdf_camera_rays, adaptivetensordf_b200/csrc/camera.cu) and the projection
log conversion of adaptivetensordf_b200/scene.py with these functions.
Nothing in the product imports this module.

Follows the reference:
  * UVToPixel                 hyperacorn/csrc/modules/CameraPose.h:14-30
  * CameraModelModule::Unproject   hyperacorn/csrc/modules/CameraPose.cu:469-479
  * quaternion rotation of a point (Saiga/Eigen unit quaternion x, y, z, w)
  * SceneBase::GetRays        hyperacorn/csrc/data/SceneBase.cpp:369-450
  * SceneBase::LoadImagesCT   hyperacorn/csrc/data/SceneBase.cpp:904-975
  * SceneBase::PointInAnyImage hyperacorn/csrc/data/SceneBase.cu:13-97
Parity unpinned: the reference ships no test vectors for these; the
restatement is checked against the synthetic parallel-beam geometry and
against closed forms in the tests.
"""

from __future__ import annotations

import math

import numpy as np


def uv_to_pixel(uv, w, h, align_corners):
    """FP32 pixel coordinates [n, 2] (the reference computes them on float tensors)."""
    uv = np.asarray(uv, np.float32)
    u, v = uv[:, 0], uv[:, 1]
    if align_corners:
        return np.stack([u * np.float32(w - 1), v * np.float32(h - 1)], 1)
    return np.stack([u * np.float32(w) - np.float32(0.5), v * np.float32(h) - np.float32(0.5)], 1)


def cross(a, b):
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1], a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], 1)


def rotate(q, p):
    """Rotation of points p [n, 3] by unit quaternions q [n, 4] (x, y, z, w), FP64:
    p + w s + u x s with u = (x, y, z), s = 2 (u x p)."""
    q = np.asarray(q, np.float64)
    p = np.asarray(p, np.float64)
    u = q[:, :3]
    s = cross(u, p)
    s = s + s
    us = cross(u, s)
    return (p + q[:, 3:4] * s) + us


def camera_rays(uv, image_id, camera_id, rotation, translation, intrinsics, w, h, align_corners, model,
                volume_translation=(0.0, 0.0, 0.0)):
    """origin, direction [n, 3] float32 (model 0 pinhole, 1 orthographic)."""
    image_id = np.asarray(image_id, np.int64)
    camera_id = np.zeros_like(image_id) if camera_id is None else np.asarray(camera_id, np.int64)
    px = uv_to_pixel(uv, w, h, align_corners).astype(np.float64)
    K = np.asarray(intrinsics, np.float64)[camera_id]
    cx = (px[:, 0] - K[:, 2]) / K[:, 0]
    cy = (px[:, 1] - K[:, 3]) / K[:, 1]
    q = np.asarray(rotation, np.float64)[image_id]
    n = len(image_id)
    if model == 1:
        d = rotate(q, np.tile([0.0, 0.0, 1.0], (n, 1)))
        p = rotate(q, np.stack([cx, cy, np.zeros(n)], 1))
        tv = np.asarray(volume_translation, np.float32).astype(np.float64)
        o = (p + tv[None, :]) - d * math.sqrt(2.0)
    else:
        nrm = np.sqrt((cx * cx + cy * cy) + 1.0)
        d = rotate(q, np.stack([cx / nrm, cy / nrm, 1.0 / nrm], 1))
        o = np.asarray(translation, np.float64)[image_id]
    return o.astype(np.float32), d.astype(np.float32)


def log_convert(raw, xray_min, xray_max, projection_factor, log_space_input, use_log10):
    """Projection (absorption) from a raw image, FP64."""
    raw = np.asarray(raw, np.float64)
    if log_space_input:
        return raw / xray_max
    raw = np.maximum(raw, 1e-5)
    if use_log10:
        return -np.log10(raw / xray_max) * (projection_factor / -math.log10(xray_min / xray_max))
    return -np.log(raw / xray_max) * (projection_factor / -math.log(xray_min / xray_max))


def tilt_quaternion(angle_deg):
    """Unit quaternion (x, y, z, w) of a rotation by angle about the y axis."""
    a = math.radians(angle_deg) / 2
    return np.array([0.0, math.sin(a), 0.0, math.cos(a)])


def _round_half_away(x):
    """C's round(): to the nearest integer, halves away from zero (the
    fractional part x - trunc(x) is exact in FP64)."""
    r = np.trunc(x)
    return r + np.where(np.abs(x - r) >= 0.5, np.sign(x), 0.0)


def point_in_any_image(points, rotation, translation, intrinsics, w, h, model, roi_min, roi_max):
    """Visibility mask [n] float32 of SceneBase::PointInAnyImage: 1 where the
    point lies in the closed ROI box (FP32 comparison, BoxContainsPoint,
    HyperTree.h:382-392) and R^T (p - t) (FP64, the conjugate quaternion)
    projects, rounded half away from zero, into [0, w) x [0, h) for some pose
    (orthographic: fx v.x + cx, fy v.y + cy; pinhole: fx v.x / v.z + cx,
    fy v.y / v.z + cy; the skew ignored as the reference sets it to 0)."""
    pts = np.asarray(points, np.float32)
    lo = np.asarray(roi_min, np.float32)
    hi = np.asarray(roi_max, np.float32)
    inside = np.all((lo[None] <= pts) & (pts <= hi[None]), axis=1)
    p64 = pts.astype(np.float64)
    K = np.asarray(intrinsics, np.float64)
    rot = np.asarray(rotation, np.float64)
    mask = np.zeros(len(pts), bool)
    for a in range(len(rot)):
        qi = np.tile(rot[a] * np.array([-1.0, -1.0, -1.0, 1.0]), (len(pts), 1))
        p = p64 - np.asarray(translation, np.float64)[a][None] if translation is not None else p64
        v = rotate(qi, p)
        if model == 1:
            px, py = K[0] * v[:, 0] + K[2], K[1] * v[:, 1] + K[3]
        else:
            px, py = K[0] * (v[:, 0] / v[:, 2]) + K[2], K[1] * (v[:, 1] / v[:, 2]) + K[3]
        rx, ry = _round_half_away(px), _round_half_away(py)
        mask |= (rx >= 0) & (rx < w) & (ry >= 0) & (ry < h)
    return (mask & inside).astype(np.float32)
