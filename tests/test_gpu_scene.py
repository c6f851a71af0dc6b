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
