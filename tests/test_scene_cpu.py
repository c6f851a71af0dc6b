"""Tilt-series ingestion on the CPU: the scene files of the reference's format,
the log conversion of projections (SceneBase::LoadImagesCT), and the
oracle's ray generation (SceneBase::GetRays) pinned against the synthetic
parallel-beam geometry that the trainer's series uses."""

import math
import os

import numpy as np
import torch

from oracle import scene_oracle as so

TOL_F32 = 1e-6


def write_scene(path, angles, n, model="orthographic", extra_ini="", images=True, scale=1.0, xray=(13046.0, 65535.0),
                raw=None):
    os.makedirs(os.path.join(path, "img"), exist_ok=True)
    with open(os.path.join(path, "dataset.ini"), "w") as f:
        f.write(f"[DatasetParams]\ncamera_model = {model}\nimage_dir = img\nscene_scale = {scale}\n"
                f"xray_min = {xray[0]}  # dark\nxray_max = {xray[1]}\nuse_log10_conversion = true\n"
                f"projection_factor = 1\n{extra_ini}")
    with open(os.path.join(path, "camera.ini"), "w") as f:
        f.write(f"w = {n}\nh = {n}\n; fx fy cx cy s\nK = {n / 2} {n / 2} {(n - 1) / 2} {(n - 1) / 2} 0\n")
    with open(os.path.join(path, "poses.txt"), "w") as f:
        for a in angles:
            q = so.tilt_quaternion(a)
            f.write(" ".join(f"{x:.17g}" for x in q) + " 0 0 1.5\n")
    if images:
        with open(os.path.join(path, "images.txt"), "w") as f:
            for i in range(len(angles)):
                f.write(f"p{i}.npy\n")
                img = raw[i] if raw is not None else np.full((n, n), 30000.0, np.float32)
                np.save(os.path.join(path, "img", f"p{i}.npy"), img.astype(np.float32))
    with open(os.path.join(path, "angles.txt"), "w") as f:
        f.write("\n".join(str(a) for a in angles) + "\n")


def test_scene_files_are_read(tmp_path):
    from adaptivetensordf_b200 import scene

    write_scene(str(tmp_path), [-10.0, 0.0, 25.0], 8, scale=2.0, extra_ini="roi_min = -1 -0.5 -1\n")
    s = scene.load_scene(str(tmp_path))
    assert s.params.camera_model == "orthographic" and s.params.image_dir == "img"
    assert s.params.xray_min == 13046.0 and s.params.use_log10_conversion
    assert s.params.roi_min == (-1.0, -0.5, -1.0)
    assert (s.width, s.height) == (8, 8)
    np.testing.assert_allclose(s.intrinsics[0], [4, 4, 3.5, 3.5, 0])
    assert s.num_images == 3 and s.images == ["p0.npy", "p1.npy", "p2.npy"]
    np.testing.assert_allclose(np.linalg.norm(s.rotation, axis=1), 1.0, rtol=1e-15)
    np.testing.assert_allclose(s.translation[:, 2], 3.0)  # scene_scale applied
    np.testing.assert_allclose(s.angles, [-10.0, 0.0, 25.0])


def test_log_conversion_matches_oracle():
    from adaptivetensordf_b200 import scene

    rng = np.random.default_rng(3)
    raw = rng.uniform(-5.0, 70000.0, (16, 16)).astype(np.float32)
    raw[0, 0] = 0.0
    for log10 in (True, False):
        for log_space in (False, True):
            for xmin in (13046.0, 0.0):
                p = scene.DatasetParams(xray_min=xmin, xray_max=65535.0, projection_factor=1.3,
                                        log_space_input=log_space, use_log10_conversion=log10)
                got = scene.log_convert(torch.from_numpy(raw), p).numpy()
                ref = so.log_convert(raw, xmin, 65535.0, 1.3, log_space, log10) if xmin > 0 or log_space else \
                    np.zeros_like(raw, np.float64)
                np.testing.assert_allclose(got, ref, rtol=2e-6, atol=1e-6)
                assert np.all(np.isfinite(got))


def test_oracle_rays_are_the_synthetic_parallel_beam():
    """Orthographic GetRays with a tilt quaternion about y, fx = n / 2 and
    cx = (n - 1) / 2 at pixel centres is the synthetic series' geometry."""
    from adaptivetensordf_b200 import synthetic as syn

    n, angles = 16, np.array([-60.0, -13.0, 0.0, 2.0, 47.0])
    img = np.repeat(np.arange(len(angles)), n * n)
    pix = np.tile(np.arange(n * n), len(angles))
    uv = np.stack([(pix % n + 0.5) / n, (pix // n + 0.5) / n], 1).astype(np.float32)
    rot = np.stack([so.tilt_quaternion(a) for a in angles])
    K = np.array([[n / 2, n / 2, (n - 1) / 2, (n - 1) / 2, 0.0]])
    o, d = so.camera_rays(uv, img, None, rot, None, K, n, n, False, 1)
    o2, d2 = syn.parallel_beam_rays(angles, n, img, pix)
    np.testing.assert_allclose(d, d2, atol=TOL_F32)
    np.testing.assert_allclose(o, o2, atol=4 * TOL_F32)


def test_oracle_pinhole_direction_is_unit_and_origin_is_the_pose():
    rng = np.random.default_rng(5)
    q = rng.normal(size=(4, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    t = rng.normal(size=(4, 3))
    K = np.array([[100.0, 90.0, 31.5, 20.0, 0.0]])
    uv = rng.uniform(0, 1, (50, 2)).astype(np.float32)
    img = rng.integers(0, 4, 50)
    o, d = so.camera_rays(uv, img, None, q, t, K, 64, 41, True, 0)
    np.testing.assert_allclose(np.linalg.norm(d.astype(np.float64), axis=1), 1.0, atol=1e-6)
    np.testing.assert_allclose(o, t[img].astype(np.float32))
    # the camera-frame ray (rotation undone) points through the pixel
    px = so.uv_to_pixel(uv, 64, 41, True).astype(np.float64)
    cam = np.stack([(px[:, 0] - 31.5) / 100.0, (px[:, 1] - 20.0) / 90.0, np.ones(50)], 1)
    cam /= np.linalg.norm(cam, axis=1, keepdims=True)
    qi = q[img] * np.array([-1, -1, -1, 1.0])  # inverse rotation
    np.testing.assert_allclose(so.rotate(qi, d.astype(np.float64)), cam, atol=2e-6)
    assert math.isclose(float(np.abs(so.tilt_quaternion(90.0)[1])), math.sin(math.pi / 4))


def test_tilt_quaternions_reproduce_the_parallel_beam():
    """recon.tilt_quaternions (with the off-axis rotation) rotate (0, 0, 1) to
    the synthetic rays' direction and (u, v, 0) to their detector point."""
    import math

    from adaptivetensordf_b200 import recon
    from adaptivetensordf_b200 import synthetic as syn
    from oracle import scene_oracle as so

    angles = np.array([-60.0, -13.5, 0.0, 42.0])
    for off in (0.0, -3.7):
        q = recon.tilt_quaternions(angles, off)
        n = 16
        img = np.repeat(np.arange(len(angles)), 3)
        pix = np.tile([0, 37, 255], len(angles))
        o, d = syn.parallel_beam_rays(angles, n, img, pix, off)
        dq = so.rotate(q[img], np.tile([0.0, 0.0, 1.0], (len(img), 1)))
        u = (pix % n + 0.5) / n * 2 - 1
        v = (pix // n + 0.5) / n * 2 - 1
        pq = so.rotate(q[img], np.stack([u, v, np.zeros_like(u)], 1)) - math.sqrt(2.0) * dq
        assert np.abs(dq - d).max() < 1e-6 and np.abs(pq - o).max() < 1e-6
