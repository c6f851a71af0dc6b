"""Tilt-series ingestion: the reference's scene directory, its projections and
the rays of their pixels, as a ``recon.TiltSeries`` the trainer runs on.

A scene directory holds (hyperacorn/csrc/data/SceneBase.cpp:745-860):
  dataset.ini          key = value: camera_model ("orthographic" | "pinhole"),
                       image_dir, xray_min, xray_max, projection_factor,
                       log_space_input, use_log10_conversion, scene_scale,
                       volume_file, roi_min, roi_max (Settings.h:273-352)
  camera.ini           w, h, K = fx fy cx cy s
  poses.txt            one pose per image: qx qy qz qw tx ty tz
  images.txt           one projection file per image (.npy, or .npz with
                       the array "proj")
  camera_indices.txt   optional: the camera of each image
  angles.txt           optional: the tilt angle of each image (degrees)

Projections are converted as in SceneBase::LoadImagesCT (SceneBase.cpp:
904-975): raw transmittance clamped at 1e-5 and turned into absorption by
-log10 (or -ln) of raw / xray_max, scaled so that xray_min maps to
projection_factor; data already in log space is divided by xray_max. The
rays of the pixels come from ``atdf_camera_rays`` (SceneBase::GetRays,
SceneBase.cpp:369-450) on the GPU. Images in formats other than numpy
arrays, and masks, are not read here (no image library in this build).
"""

from __future__ import annotations

import ctypes as ct
import math
import os
from dataclasses import dataclass, field

import numpy as np
import torch

from . import capi

CAMERA_MODELS = {"pinhole": 0, "orthographic": 1}


def read_ini(path: str) -> dict:
    """``key = value`` pairs of an ini file (sections, '#' and ';' comments ignored)."""
    out = {}
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].split(";", 1)[0].strip()
            if not line or line.startswith("[") or "=" not in line:
                continue
            k, v = line.split("=", 1)
            out[k.strip()] = v.strip()
    return out


def _bool(v) -> bool:
    return str(v).strip().lower() in ("1", "true", "yes", "on")


@dataclass
class DatasetParams:
    """Settings.h:273-352 (the defaults are the reference's)."""

    camera_model: str = "pinhole"
    image_dir: str = ""
    projection_factor: float = 1.0
    scene_scale: float = 1.0
    xray_min: float = 0.0
    xray_max: float = 65535.0
    volume_file: str = ""
    log_space_input: bool = False
    use_log10_conversion: bool = True
    roi_min: tuple = (-1.0, -1.0, -1.0)
    roi_max: tuple = (1.0, 1.0, 1.0)

    @staticmethod
    def from_ini(d: dict) -> "DatasetParams":
        p = DatasetParams()
        for k in ("camera_model", "image_dir", "volume_file"):
            if k in d:
                setattr(p, k, d[k])
        for k in ("projection_factor", "scene_scale", "xray_min", "xray_max"):
            if k in d:
                setattr(p, k, float(d[k]))
        for k in ("log_space_input", "use_log10_conversion"):
            if k in d:
                setattr(p, k, _bool(d[k]))
        for k in ("roi_min", "roi_max"):
            if k in d:
                setattr(p, k, tuple(float(x) for x in d[k].split()))
        return p


def log_convert(raw: torch.Tensor, p: DatasetParams) -> torch.Tensor:
    """Absorption projection of a raw FP32 image (SceneBase.cpp:940-968)."""
    raw = raw.float()
    if p.log_space_input:
        return raw / p.xray_max
    raw = raw.clamp_min(1e-5)
    log = math.log10 if p.use_log10_conversion else math.log
    # -log(xray_min / xray_max) is +inf for xray_min = 0: the scale is then 0, as in the reference
    denom = -log(p.xray_min / p.xray_max) if p.xray_min > 0 else math.inf
    scale = p.projection_factor / denom
    lg = torch.log10 if p.use_log10_conversion else torch.log
    return -lg(raw / p.xray_max) * scale


@dataclass
class Scene:
    """A loaded scene: parameters, camera, poses, image files."""

    path: str
    params: DatasetParams
    width: int
    height: int
    intrinsics: np.ndarray      # [num_cameras, 5] fx fy cx cy s
    rotation: np.ndarray        # [num_images, 4] unit quaternions x, y, z, w
    translation: np.ndarray     # [num_images, 3] (scene_scale applied)
    images: list = field(default_factory=list)
    camera_index: np.ndarray = None
    angles: np.ndarray = None

    @property
    def num_images(self):
        return self.rotation.shape[0]

    def projection(self, i: int, device="cuda") -> torch.Tensor:
        """Image i as an absorption projection [h, w] float32."""
        f = os.path.join(self.path, self.params.image_dir, self.images[i])
        if f.endswith(".npz"):
            raw = np.load(f)["proj"]
        elif f.endswith(".npy"):
            raw = np.load(f)
        else:
            raise ValueError(f"unsupported projection file {f}: numpy .npy / .npz only")
        raw = np.asarray(raw, np.float32)
        if raw.shape != (self.height, self.width):
            raise ValueError(f"{f}: shape {raw.shape}, camera {self.height} x {self.width}")
        return log_convert(torch.from_numpy(raw).to(device), self.params)

    def get_rays(self, uv: torch.Tensor, image_id: torch.Tensor, camera_id: torch.Tensor = None,
                 align_corners: bool = False, volume_translation=(0.0, 0.0, 0.0)):
        """Rays of the pixels uv [n, 2] (CUDA float32) of images image_id [n]:
        (origin, direction) [n, 3] float32, through atdf_camera_rays."""
        dev = uv.device
        n = uv.shape[0]
        uv = uv.float().contiguous()
        iid = image_id.to(torch.int32).contiguous()
        cid = None if camera_id is None else camera_id.to(torch.int32).contiguous()
        rot = torch.from_numpy(np.ascontiguousarray(self.rotation, np.float64)).to(dev)
        # pinhole: camera centres relative to the volume (SceneBase::Finalize, SceneBase.cpp:99-113)
        tr_np = self.translation - np.asarray(volume_translation, np.float64)[None, :]
        tr = torch.from_numpy(np.ascontiguousarray(tr_np, np.float64)).to(dev)
        K = torch.from_numpy(np.ascontiguousarray(self.intrinsics, np.float64)).to(dev)
        o = torch.empty(n, 3, device=dev)
        d = torch.empty(n, 3, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        tv = (ct.c_float * 3)(*[float(x) for x in volume_translation])
        L = capi.lib()
        st = L.atdf_camera_rays(n, capi.ptr(uv), capi.ptr(iid), capi.ptr(cid), capi.ptr(rot), capi.ptr(tr),
                                self.num_images, capi.ptr(K), K.shape[0], self.width, self.height,
                                int(align_corners), CAMERA_MODELS[self.params.camera_model], ct.cast(tv, ct.c_void_p),
                                capi.ptr(o),
                                capi.ptr(d), capi.ptr(err), ct.c_void_p(torch.cuda.current_stream().cuda_stream))
        if st != 0:
            raise RuntimeError(f"atdf_camera_rays: {L.atdf_status_string(st).decode()}")
        if int(err.item()) != 0:
            raise RuntimeError("atdf_camera_rays: image or camera index out of range")
        return o, d

    def tilt_series(self, device="cuda", align_corners: bool = False, volume_translation=(0.0, 0.0, 0.0)):
        """Every pixel of every image as a ``recon.TiltSeries`` (targets are the
        converted projections; no phantom, so ``volume`` is the scene's
        ground-truth volume when it has one as .npy, else None)."""
        from .recon import TiltSeries

        w, h = self.width, self.height
        ys, xs = torch.meshgrid(torch.arange(h, device=device), torch.arange(w, device=device), indexing="ij")
        if align_corners:
            uv1 = torch.stack([xs.float() / max(w - 1, 1), ys.float() / max(h - 1, 1)], -1).reshape(-1, 2)
        else:
            uv1 = torch.stack([(xs.float() + 0.5) / w, (ys.float() + 0.5) / h], -1).reshape(-1, 2)
        A = self.num_images
        uv = uv1.repeat(A, 1)
        iid = torch.arange(A, device=device).repeat_interleave(w * h)
        cid = None
        if self.camera_index is not None:
            cid = torch.from_numpy(np.asarray(self.camera_index, np.int64)).to(device).repeat_interleave(w * h)
        o, d = self.get_rays(uv, iid, cid, align_corners, volume_translation)
        y = torch.cat([self.projection(i, device).reshape(-1) for i in range(A)])
        vol = None
        vf = self.params.volume_file
        if vf.endswith(".npy"):
            vol = torch.from_numpy(np.load(os.path.join(self.path, vf)).astype(np.float32)).to(device)
        angles = self.angles if self.angles is not None else np.zeros(A)
        # PointInAnyImage uses the first camera's intrinsics (SceneBase.cu:19-23)
        return TiltSeries(o, d, y, y.double(), vol, angles, iid, uv, h, w,
                          cam_rotation=np.asarray(self.rotation, np.float64),
                          cam_translation=np.asarray(self.translation, np.float64),
                          cam_intrinsics=tuple(np.asarray(self.intrinsics, np.float64)[0].tolist()),
                          cam_model=CAMERA_MODELS[self.params.camera_model],
                          roi_min=tuple(self.params.roi_min), roi_max=tuple(self.params.roi_max))


def load_scene(path: str) -> Scene:
    """Reads a scene directory (SceneBase.cpp:745-860)."""
    params = DatasetParams.from_ini(read_ini(os.path.join(path, "dataset.ini")))
    if params.camera_model not in CAMERA_MODELS:
        raise ValueError(f"camera_model {params.camera_model!r}: pinhole or orthographic")
    cam = read_ini(os.path.join(path, "camera.ini"))
    w, h = int(cam["w"]), int(cam["h"])
    K = np.array([float(x) for x in cam["K"].split()], np.float64)
    if K.size != 5 or w <= 0 or h <= 0:
        raise ValueError("camera.ini: w, h > 0 and K = fx fy cx cy s")
    poses = np.loadtxt(os.path.join(path, "poses.txt"), dtype=np.float64, ndmin=2)
    if poses.shape[1] != 7:
        raise ValueError("poses.txt: qx qy qz qw tx ty tz per line")
    rot = poses[:, :4] / np.linalg.norm(poses[:, :4], axis=1, keepdims=True)
    tr = poses[:, 4:] * params.scene_scale
    images = []
    f = os.path.join(path, "images.txt")
    if os.path.exists(f):
        images = [ln.strip() for ln in open(f) if ln.strip()]
        if len(images) != len(poses):
            raise ValueError("images.txt and poses.txt differ in length")
    ci = None
    f = os.path.join(path, "camera_indices.txt")
    if os.path.exists(f):
        ci = np.loadtxt(f, dtype=np.int64, ndmin=1)
        if ci.size != len(poses) or ci.min() < 0 or ci.max() > 0:
            raise ValueError("camera_indices.txt: one index per image, camera 0 (one camera.ini)")
    angles = None
    f = os.path.join(path, "angles.txt")
    if os.path.exists(f):
        angles = np.loadtxt(f, dtype=np.float64, ndmin=1)
    return Scene(path, params, w, h, K[None, :], rot, tr, images, ci, angles)
