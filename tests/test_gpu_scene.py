"""Ray generation from camera poses on the GPU (atdf_camera_rays) against the
numpy restatement of SceneBase::GetRays, and a scene directory loaded end to
end into a tilt series the trainer runs on. Every FP64 operation of the
kernel is rounded on its own, so its FP32 rays equal the restatement's bit
for bit."""

import numpy as np
import pytest
import torch

from oracle import scene_oracle as so
from tests.test_scene_cpu import write_scene

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _scene(model, n_img, w, h, seed):
    from adaptivetensordf_b200 import scene

    rng = np.random.default_rng(seed)
    q = rng.normal(size=(n_img, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    K = np.array([[w * 0.61, h * 0.53, (w - 1) / 2 + 0.25, (h - 1) / 2 - 0.5, 0.0]])
    p = scene.DatasetParams(camera_model=model)
    return scene.Scene("", p, w, h, K, q, rng.normal(size=(n_img, 3)), [])


@pytest.mark.parametrize("model", ["orthographic", "pinhole"])
@pytest.mark.parametrize("align", [False, True])
def test_camera_rays_match_oracle(model, align):
    s = _scene(model, 7, 40, 23, 11 if align else 12)
    rng = np.random.default_rng(4)
    n = 5000
    uv = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    img = rng.integers(0, 7, n)
    tv = (0.125, -0.3, 0.05)
    o, d = s.get_rays(torch.from_numpy(uv).cuda(), torch.from_numpy(img).cuda(), align_corners=align,
                      volume_translation=tv)
    mid = 1 if model == "orthographic" else 0
    ro, rd = so.camera_rays(uv, img, None, s.rotation, s.translation - np.asarray(tv)[None, :], s.intrinsics,
                            s.width, s.height, align, mid, tv)
    np.testing.assert_array_equal(d.cpu().numpy(), rd)
    np.testing.assert_array_equal(o.cpu().numpy(), ro)


def test_camera_rays_reject_an_image_out_of_range():
    s = _scene("orthographic", 3, 8, 8, 1)
    uv = torch.rand(10, 2, device="cuda")
    img = torch.zeros(10, dtype=torch.long, device="cuda")
    img[4] = 3
    with pytest.raises(RuntimeError, match="out of range"):
        s.get_rays(uv, img)


def test_scene_directory_to_tilt_series(tmp_path):
    """A tilt series written in the reference's scene format (poses of a tilt
    about y, raw transmittance images of an ellipsoid phantom) loads into the
    same rays and absorption targets as the synthetic series, and the trainer
    runs on it."""
    import dataclasses

    from adaptivetensordf_b200 import recon, scene
    from adaptivetensordf_b200 import synthetic as syn

    n, angles = 16, np.array([-40.0, -20.0, 0.0, 20.0, 40.0])
    A = len(angles)
    img = np.repeat(np.arange(A), n * n)
    pix = np.tile(np.arange(n * n), A)
    o_ref, d_ref = syn.parallel_beam_rays(angles, n, img, pix)
    ph = syn.ellipsoid_phantom(12, 77)
    p = syn.analytic_projection(ph, o_ref, d_ref)
    xmin, xmax = 13046.0, 65535.0
    k = -np.log10(xmin / xmax)
    raw = (xmax * 10.0 ** (-p * k)).reshape(A, n, n)  # projection_factor 1
    write_scene(str(tmp_path), angles, n, raw=raw, xray=(xmin, xmax))
    s = scene.load_scene(str(tmp_path))
    data = s.tilt_series()
    np.testing.assert_allclose(data.direction.cpu().numpy(), d_ref, atol=1e-6)
    np.testing.assert_allclose(data.origin.cpu().numpy(), o_ref, atol=4e-6)
    np.testing.assert_allclose(data.target.cpu().numpy(), p, rtol=2e-4, atol=2e-5)
    assert data.volume is None and data.image_id.shape[0] == A * n * n

    cfg = dataclasses.replace(syn.CONFIGS["C1"], rays_per_batch=256)
    opt = recon.TrainOptions(epochs=3, batch=256, max_samples_per_node=cfg.max_samples_per_node, eval_every=0,
                             stop_at_target=False, init_scale=0.05)
    recs, reached = recon.train(cfg, "fp32", data, opt)
    assert reached is None and recs[-1]["psnr"] is None
    assert recs[-1]["loss"] < recs[0]["loss"]


@pytest.mark.parametrize("model", [0, 1])
def test_point_in_any_image_matches_oracle(model):
    """atdf_point_in_any_image (SceneBase::PointInAnyImage) bit for bit
    against the numpy restatement: points in and out of the ROI, some exactly
    on its bounds, on several orthographic tilts / pinhole poses."""
    import ctypes as ct

    from adaptivetensordf_b200 import capi
    from oracle import scene_oracle as so

    rng = np.random.default_rng(model + 3)
    P = 50000
    pts = rng.uniform(-1.3, 1.3, (P, 3)).astype(np.float32)
    pts[:100, 0] = 1.0  # on the ROI bound (closed)
    pts[100:200, 2] = -1.0
    angles = np.linspace(-60, 60, 9)
    rot = np.stack([so.tilt_quaternion(a) for a in angles])
    if model == 1:
        trans = None
        K = np.array([24.0, 24.0, 23.5, 23.5, 0.3])
        w = h = 48
    else:
        trans = np.stack([-3.0 * so.rotate(q[None], np.array([[0.0, 0.0, 1.0]]))[0] for q in rot])
        K = np.array([40.0, 40.0, 31.5, 31.5, 0.0])
        w, h = 64, 64
    roi_min, roi_max = (-1.0, -0.9, -1.0), (1.0, 0.9, 1.0)
    ref = so.point_in_any_image(pts, rot, trans, K, w, h, model, roi_min, roi_max)
    pt = torch.from_numpy(pts).cuda()
    rt = torch.from_numpy(rot).cuda()
    tt = None if trans is None else torch.from_numpy(trans).cuda()
    Kt = torch.from_numpy(K).cuda()
    mask = torch.full((P,), -1.0, device="cuda")
    L = capi.lib()
    st = L.atdf_point_in_any_image(P, capi.ptr(pt), capi.ptr(rt), capi.ptr(tt), len(rot), capi.ptr(Kt), w, h, model,
                                   (ct.c_float * 3)(*roi_min), (ct.c_float * 3)(*roi_max), capi.ptr(mask),
                                   ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0
    got = mask.cpu().numpy()
    assert np.array_equal(got, ref)
    assert 0.05 < ref.mean() < 0.95  # both outcomes occur
    assert ref[:100].max() == 1.0  # points on the closed ROI bound can count
